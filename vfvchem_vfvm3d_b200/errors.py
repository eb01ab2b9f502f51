"""Error types mirroring the reference's ``VFVChemError`` variants for the linear solver
(src/base/error.rs:219-268). Non-zero status codes of the C ABI map onto them."""
from __future__ import annotations


class VFVChemError(RuntimeError):
    """Base class (the reference's ``#[non_exhaustive] enum VFVChemError``, error.rs:1-5)."""

    code = -1


class LinearGmresDidNotConverge(VFVChemError):
    """``LinearGmresDidNotConverge { message }`` (error.rs:265-268; raised at linear_gmres.rs:81)."""

    code = 1


class LinearGmresNonFinite(VFVChemError):
    code = 2


class LinearGmresBadInput(VFVChemError, ValueError):
    code = 3


class LinearGmresCudaError(VFVChemError):
    code = 4


class DeviceWaitTimeout(VFVChemError):
    """A bounded device wait gave up (status 5); the context stays usable. No reference
    counterpart: the reference's CPU solver has no device waits. Like any solve error it is
    recoverable by the caller (transient_adaptive.rs:190-205 retries a failed solve)."""

    code = 5


class OutputWriteError(VFVChemError, OSError):
    """``WriteVtu`` / ``WriteCsv { file_path, source }`` (error.rs:116-127): the file could not be
    written (status 6)."""

    code = 6


class OutputTypeError(VFVChemError, ValueError):
    """``ScalarUnknownOutputType`` / ``ScalarUnsupportedOutputType`` and their Vector twins
    (error.rs:78-100): an output path without an extension, or one other than csv or vtu."""


class LinearGmresNonPositiveThreads(LinearGmresBadInput):
    """``LinearGmresNonPositiveThreads { num_thread }`` (linear_gmres.rs:26-28)."""


class LinearGmresNonPositiveTolerance(LinearGmresBadInput):
    """``LinearGmresNonPositiveTolerance { tol }`` (linear_gmres.rs:29-31)."""


class LinearGmresNonPositiveRestart(LinearGmresBadInput):
    """``LinearGmresNonPositiveRestart { restart }`` (linear_gmres.rs:32-34)."""


class LinearGmresNonPositiveMaxOuter(LinearGmresBadInput):
    """``LinearGmresNonPositiveMaxOuter { max_outer }`` (linear_gmres.rs:35-37)."""


_BY_CODE = {1: LinearGmresDidNotConverge, 2: LinearGmresNonFinite, 3: LinearGmresBadInput, 4: LinearGmresCudaError,
            5: DeviceWaitTimeout, 6: OutputWriteError}


def raise_for(code: int, message: str) -> None:
    if code == 0:
        return
    raise _BY_CODE.get(code, VFVChemError)(message)
