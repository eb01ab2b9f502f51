"""B200-native assemble-and-solve path of vfvchem-vfvm3d.

Python face of libvfvgpu (C ABI in include/vfv_gpu.h). The names mirror the reference's Rust API:

* :class:`LinearGmres` — ``LinearBase`` / ``LinearGmres`` (src/linear/linear_base.rs:5-10,
  src/linear/linear_gmres.rs:8-85): ``update_sparse``, ``build_matrix``, ``solve_matrix``.
* :class:`SteadyHeatGpu` — the device assembly of ``SteadyHeat::assemble_matrix``
  (src/steady/core/steady_heat.rs:143-171) over a :class:`Mesh` (the Voronoi dual of
  ``Tetrahedron::update_tet``, src/base/geom_tet.rs:58-350).
* :class:`TransientTransportGpu` — batched transient advection-diffusion over many meshes.
* :class:`SteadyFlowGpu` — the coupled Navier-Stokes system of ``SteadyFlow``
  (src/steady/core/steady_flow.rs) and its damped Picard loop.
* :class:`Context`, :class:`Pattern` — the device context and a CSR pattern with its values.

Everything runs on the GPU through the compiled library; importing works without a GPU, but any
call that needs the device raises :class:`VFVChemError` when no CUDA device is usable.
"""
from .errors import (  # noqa: F401
    VFVChemError,
    LinearGmresDidNotConverge,
    LinearGmresNonFinite,
    LinearGmresBadInput,
    LinearGmresCudaError,
    DeviceWaitTimeout,
    OutputWriteError,
    OutputTypeError,
    LinearGmresNonPositiveTolerance,
    LinearGmresNonPositiveRestart,
    LinearGmresNonPositiveMaxOuter,
    LinearGmresNonPositiveThreads,
)
from .core import Context, Pattern, GmresOptions, SolveInfo, default_context  # noqa: F401
from .mesh import Mesh  # noqa: F401
from .heat import SteadyHeatGpu  # noqa: F401
from .linear import LinearGmres, Triplet, SparseMatrix  # noqa: F401
from .transport import TransientTransportGpu  # noqa: F401
from .flow import SteadyFlowGpu  # noqa: F401
from . import _lib  # noqa: F401
from . import output  # noqa: F401

__all__ = [
    "Context", "Pattern", "GmresOptions", "SolveInfo", "Mesh", "SteadyHeatGpu", "LinearGmres", "Triplet",
    "SparseMatrix", "VFVChemError", "LinearGmresDidNotConverge", "default_context", "TransientTransportGpu", "SteadyFlowGpu",
    "OutputWriteError", "OutputTypeError", "output",
]
