// Device assembly of the coupled Navier-Stokes system; see ns.cuh. Built with -fmad=false.
#include "ns.cuh"

namespace vfv {

namespace {

__device__ __forceinline__ double pow5(double x) {
    const double x2 = x * x;
    return x2 * x2 * x;
}

// skew-corrected arithmetic-mean face density (opscl_dom_div.rs:104-106, flow_helper.rs:51)
__device__ __forceinline__ double face_den(const NsDev& D, int64_t v, int32_t i) {
    const int64_t N = D.n, E = D.n_dir;
    const int32_t nb = D.ni[i];
    const double sx = D.skew[i], sy = D.skew[E + i], sz = D.skew[2 * E + i];
    return 0.5 * (D.den[v] + D.den[nb]) +
           0.5 * (sx * (D.gden[v] + D.gden[nb]) + sy * (D.gden[N + v] + D.gden[N + nb]) + sz * (D.gden[2 * N + v] + D.gden[2 * N + nb]));
}

// harmonic-mean, skew-corrected, guarded face viscosity (opvec_dom_diff.rs:76-79)
__device__ __forceinline__ double face_visc(const NsDev& D, int64_t v, int32_t i) {
    const int64_t N = D.n, E = D.n_dir;
    const int32_t nb = D.ni[i];
    const double mv = D.visc[v], mn = D.visc[nb];
    const double sx = D.skew[i], sy = D.skew[E + i], sz = D.skew[2 * E + i];
    const double vm = (mv + mn != 0.0) ? 2.0 * mv * mn / (mv + mn) : 0.0;
    const double vf = vm + 0.5 * (sx * (D.gvisc[v] + D.gvisc[nb]) + sy * (D.gvisc[N + v] + D.gvisc[N + nb]) +
                                  sz * (D.gvisc[2 * N + v] + D.gvisc[2 * N + nb]));
    return vf > 0.0 ? vf : vm;
}

// body force at the control-volume centroid (opvec_dom_src.rs:57-64)
__device__ __forceinline__ void force_centroid(const NsDev& D, int64_t v, double f[3]) {
    const int64_t N = D.n;
    const double cx = D.cskew[v], cy = D.cskew[N + v], cz = D.cskew[2 * N + v];
#pragma unroll
    for (int q = 0; q < 3; ++q)
        f[q] = D.fce[q * N + v] + D.gfce[(3 * q) * N + v] * cx + D.gfce[(3 * q + 1) * N + v] * cy + D.gfce[(3 * q + 2) * N + v] * cz;
}

// Rhie-Chow coefficient V / a_P with a_P = sum_f D_f A(|Pe_f|) + max(F_f, 0), F_f the central
// mass flux (flow_helper::update_flow, flow_helper.rs:19-66)
__global__ void __launch_bounds__(256) k_ns_rc(NsDev D) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= D.n) return;
    const int64_t N = D.n, E = D.n_dir;
    const double* u = D.x;
    double cp = 0.0;
    for (int32_t i = D.np[v]; i < D.np[v + 1]; ++i) {
        const int32_t nb = D.ni[i];
        const double face = D.area[i], dist = D.dist[i];
        const double nx = D.norm[i], ny = D.norm[E + i], nz = D.norm[2 * E + i];
        const double den_f = face_den(D, v, i);
        const double cond = face_visc(D, v, i) * face / dist;
        const double fl = den_f * 0.5 * ((u[v] + u[nb]) * nx + (u[N + v] + u[N + nb]) * ny + (u[2 * N + v] + u[2 * N + nb]) * nz) * face;
        const double pe = cond != 0.0 ? fl / cond : 0.0;
        const double a = fmax(1.0 - 0.1 * fabs(pe), 0.0);
        cp += cond * pow5(a) + fmax(fl, 0.0);
    }
    D.rc[v] = cp > 0.0 ? D.cvol[v] / cp : 0.0;
}

// d (grad p - fce) per vertex with grad p = sum_m c_m p_m / V (flow_helper.rs:86-113)
__global__ void __launch_bounds__(256) k_ns_mom(NsDev D) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= D.n) return;
    const int64_t N = D.n, G = D.n_gc;
    const double* p = D.x + 3 * N;
    const double vol = D.cvol[v];
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int32_t k = D.gcp[v]; k < D.gcp[v + 1]; ++k) {
        const double pm = p[D.gcv[k]];
        px += D.gcc[k] * pm / vol;
        py += D.gcc[G + k] * pm / vol;
        pz += D.gcc[2 * G + k] * pm / vol;
    }
    double f[3];
    force_centroid(D, v, f);
    const double r = D.rc[v];
    D.mom[v] = r * (px - f[0]);
    D.mom[N + v] = r * (py - f[1]);
    D.mom[2 * N + v] = r * (pz - f[2]);
}

// face mass flux with the Rhie-Chow correction (flow_helper.rs:116-173)
__global__ void __launch_bounds__(256) k_ns_flux(NsDev D) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= D.n) return;
    const int64_t N = D.n, E = D.n_dir;
    const double* u = D.x;
    const double* p = D.x + 3 * N;
    for (int32_t i = D.np[v]; i < D.np[v + 1]; ++i) {
        const int32_t nb = D.ni[i];
        const double face = D.area[i], dist = D.dist[i];
        const double nx = D.norm[i], ny = D.norm[E + i], nz = D.norm[2 * E + i];
        const double sx = D.skew[i], sy = D.skew[E + i], sz = D.skew[2 * E + i];
        const double den_f = face_den(D, v, i);
        double uf[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double* g = D.gvel + 3 * q * N;
            uf[q] = 0.5 * (u[q * N + v] + u[q * N + nb]) + 0.5 * (sx * (g[v] + g[nb]) + sy * (g[N + v] + g[N + nb]) + sz * (g[2 * N + v] + g[2 * N + nb]));
        }
        const double fce_e = 0.5 * (nx * (D.fce[v] + D.fce[nb]) + ny * (D.fce[N + v] + D.fce[N + nb]) + nz * (D.fce[2 * N + v] + D.fce[2 * N + nb]));
        const double mom_e = 0.5 * (nx * (D.mom[v] + D.mom[nb]) + ny * (D.mom[N + v] + D.mom[N + nb]) + nz * (D.mom[2 * N + v] + D.mom[2 * N + nb]));
        const double vel_rc = -0.5 * (D.rc[v] + D.rc[nb]) * ((p[nb] - p[v]) / dist - fce_e) + mom_e;
        D.flux[i] = den_f * (uf[0] * nx + uf[1] * ny + uf[2] * nz + vel_rc) * face;
    }
}

// Momentum rows: points push advection (opvec_dom_adv.rs:64-113), the pressure gradient
// (opvec_dom_grad.rs:53-67) and diffusion (opvec_dom_diff.rs:55-91); nodes the Dirichlet
// diagonal (opvec_bnd_dir.rs:56-80).
__global__ void __launch_bounds__(256) k_ns_trip_mom(NsDev D) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= D.n) return;
    const int64_t N = D.n, G = D.n_gc;
    if (v >= D.n_pts) {
#pragma unroll
        for (int q = 0; q < 3; ++q) D.tv[D.trip_ptr[q * N + v]] = 1.0;
        return;
    }
    const int32_t b = D.np[v], e = D.np[v + 1];
    const int32_t dg = e - b, gb = D.gcp[v], gn = D.gcp[v + 1] - gb;
    const int64_t t0 = D.trip_ptr[v], t1 = D.trip_ptr[N + v], t2 = D.trip_ptr[2 * N + v];
    for (int32_t i = b; i < e; ++i) {
        const int32_t k = i - b;
        const double cond = face_visc(D, v, i) * D.area[i] / D.dist[i];
        const double fl = D.flux[i];
        const double pe = cond != 0.0 ? fl / cond : 0.0;
        const double coeff = cond * (pow5(fmax(1.0 - 0.1 * fabs(pe), 0.0)) - 1.0) + fmax(-fl, 0.0);
        D.tv[t0 + 2 * k] = coeff;
        D.tv[t0 + 2 * k + 1] = -coeff;
        D.tv[t1 + 2 * k] = coeff;
        D.tv[t1 + 2 * k + 1] = -coeff;
        D.tv[t2 + 2 * k] = coeff;
        D.tv[t2 + 2 * k + 1] = -coeff;
        const int32_t o = 2 * dg + gn + 2 * k;
        D.tv[t0 + o] = cond;
        D.tv[t0 + o + 1] = -cond;
        D.tv[t1 + o] = cond;
        D.tv[t1 + o + 1] = -cond;
        D.tv[t2 + o] = cond;
        D.tv[t2 + o + 1] = -cond;
    }
    for (int32_t k = 0; k < gn; ++k) {
        D.tv[t0 + 2 * dg + k] = -D.gcc[gb + k];
        D.tv[t1 + 2 * dg + k] = -D.gcc[G + gb + k];
        D.tv[t2 + 2 * dg + k] = -D.gcc[2 * G + gb + k];
    }
}

// Pressure rows, one warp per vertex: divergence (opscl_dom_div.rs:84-148, and for nodes the
// boundary sub-faces of opscl_bnd_div.rs:163-181) then the pressure stabiliser
// (opscl_dom_pstab.rs:86-146). Lanes split the inner loops; every value has a fixed slot.
__global__ void __launch_bounds__(256) k_ns_trip_p(NsDev D) {
    const int lane = threadIdx.x & 31;
    const int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (v >= D.n) return;
    const int64_t N = D.n, E = D.n_dir, B = D.n_bsub, G = D.n_gc;
    const int64_t base = D.trip_ptr[3 * N + v];
    if (v == D.pref_vid) {
        if (lane == 0) D.tv[base] = 1.0;
        return;
    }
    const int32_t b = D.np[v], e = D.np[v + 1];
    const int32_t dv = e - b;
    for (int32_t i = b; i < e; ++i) {
        const int32_t nb = D.ni[i];
        const double face = D.area[i];
        const double nn[3] = {D.norm[i], D.norm[E + i], D.norm[2 * E + i]};
        const double sx = D.skew[i], sy = D.skew[E + i], sz = D.skew[2 * E + i];
        const double coeff = 0.5 * face_den(D, v, i) * face;
        double* blk = D.tv + base + D.div_off[i];
        if (lane < 3) {
            blk[2 * lane] = -coeff * nn[lane];
            blk[2 * lane + 1] = -coeff * nn[lane];
        }
        for (int32_t k = b + lane; k < e; k += 32) {
            const double ws = D.gw[k] * sx + D.gw[E + k] * sy + D.gw[2 * E + k] * sz;
            double* o = blk + 6 + 6 * (k - b);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double val = -coeff * ws * nn[c];
                o[2 * c] = val;
                o[2 * c + 1] = -val;
            }
        }
        const int32_t nb0 = D.np[nb], nb1 = D.np[nb + 1];
        for (int32_t k = nb0 + lane; k < nb1; k += 32) {
            const double ws = D.gw[k] * sx + D.gw[E + k] * sy + D.gw[2 * E + k] * sz;
            double* o = blk + 6 + 6 * dv + 6 * (k - nb0);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double val = -coeff * ws * nn[c];
                o[2 * c] = val;
                o[2 * c + 1] = -val;
            }
        }
    }
    if (v >= D.n_pts) {
        double* sb = D.tv + base + D.sub_off[v];
        const int32_t s0 = D.bp[v], s1 = D.bp[v + 1];
        for (int32_t s = s0 + lane; s < s1; s += 32) {
            const double area = D.barea[s];
            const double nn[3] = {D.bnorm[s], D.bnorm[B + s], D.bnorm[2 * B + s]};
            const double cs[3] = {D.bw[s] * D.den[v] * area, D.bw[B + s] * D.den[D.bj[s]] * area, D.bw[2 * B + s] * D.den[D.bk[s]] * area};
            double* o = sb + 9 * (s - s0);
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int c = 0; c < 3; ++c) o[3 * m + c] = -cs[m] * nn[c];
        }
    }
    const double rc_v = D.rc[v], vol_v = D.cvol[v];
    const int32_t gv0 = D.gcp[v], gv1 = D.gcp[v + 1];
    for (int32_t i = b; i < e; ++i) {
        const int32_t nb = D.ni[i];
        const double face = D.area[i], dist = D.dist[i];
        const double nx = D.norm[i], ny = D.norm[E + i], nz = D.norm[2 * E + i];
        const double rc_n = D.rc[nb], vol_n = D.cvol[nb];
        const double den_f = face_den(D, v, i);
        const double coeff = den_f * 0.5 * (rc_v + rc_n) * face;
        double* blk = D.tv + base + D.pst_off[i];
        if (lane == 0) {
            blk[0] = coeff / dist;
            blk[1] = -coeff / dist;
        }
        const double cv = den_f * 0.5 * rc_v / vol_v * face;
        for (int32_t k = gv0 + lane; k < gv1; k += 32)
            blk[2 + (k - gv0)] = -cv * (D.gcc[k] * nx + D.gcc[G + k] * ny + D.gcc[2 * G + k] * nz);
        const double cn = den_f * 0.5 * rc_n / vol_n * face;
        const int32_t gn0 = D.gcp[nb], gn1 = D.gcp[nb + 1];
        for (int32_t k = gn0 + lane; k < gn1; k += 32)
            blk[2 + (gv1 - gv0) + (k - gn0)] = -cn * (D.gcc[k] * nx + D.gcc[G + k] * ny + D.gcc[2 * G + k] * nz);
    }
}

// Right-hand side, one thread per vertex, each row in the reference's operator order:
// momentum rows of points: transpose term (opvec_dom_dtrn.rs:57-110), dilatational term
// (opvec_dom_ddil.rs:57-109), body force (opvec_dom_src.rs:52-69); momentum rows of nodes the
// boundary velocity; pressure rows the stabiliser's body-force part; the reference row p = pref.
__global__ void __launch_bounds__(256) k_ns_rhs(NsDev D) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= D.n) return;
    const int64_t N = D.n, E = D.n_dir;
    const int32_t b = D.np[v], e = D.np[v + 1];
    if (v < D.n_pts) {
        double s1[3] = {0.0, 0.0, 0.0}, s2[3] = {0.0, 0.0, 0.0};
        double gv[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) gv[q] = D.gvel[q * N + v];
        for (int32_t i = b; i < e; ++i) {
            const int32_t nb = D.ni[i];
            const double face = D.area[i];
            const double nx = D.norm[i], ny = D.norm[E + i], nz = D.norm[2 * E + i];
            const double vf = face_visc(D, v, i);
            double gf[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) gf[q] = 0.5 * (gv[q] + D.gvel[q * N + nb]);
            s1[0] += vf * (gf[0] * nx + gf[3] * ny + gf[6] * nz) * face;
            s1[1] += vf * (gf[1] * nx + gf[4] * ny + gf[7] * nz) * face;
            s1[2] += vf * (gf[2] * nx + gf[5] * ny + gf[8] * nz) * face;
        }
        const double div_v = gv[0] + gv[4] + gv[8];
        for (int32_t i = b; i < e; ++i) {
            const int32_t nb = D.ni[i];
            const double face = D.area[i];
            const double nx = D.norm[i], ny = D.norm[E + i], nz = D.norm[2 * E + i];
            const double lam_f = (-2.0 / 3.0) * face_visc(D, v, i);
            const double div_n = D.gvel[nb] + D.gvel[4 * N + nb] + D.gvel[8 * N + nb];
            const double c = lam_f * (0.5 * (div_v + div_n)) * face;
            s2[0] += c * nx;
            s2[1] += c * ny;
            s2[2] += c * nz;
        }
        double f[3];
        force_centroid(D, v, f);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            double bq = 0.0;
            bq += -s1[q];
            bq += -s2[q];
            bq += -f[q] * D.cvol[v];
            D.b[q * N + v] = bq;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) D.b[q * N + v] = 0.0 + D.bc_vel[q * N + v];
    }
    double bp = 0.0;
    double fv[3];
    force_centroid(D, v, fv);
    const double rc_v = D.rc[v];
    for (int32_t i = b; i < e; ++i) {
        const int32_t nb = D.ni[i];
        const double face = D.area[i];
        const double nx = D.norm[i], ny = D.norm[E + i], nz = D.norm[2 * E + i];
        double fn[3];
        force_centroid(D, nb, fn);
        const double rc_n = D.rc[nb];
        const double den_f = face_den(D, v, i);
        double frc[3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
            frc[q] = 0.5 * (rc_v + rc_n) * 0.5 * (D.fce[q * N + v] + D.fce[q * N + nb]) - 0.5 * (rc_v * fv[q] + rc_n * fn[q]);
        bp += den_f * (frc[0] * nx + frc[1] * ny + frc[2] * nz) * face;
    }
    D.b[3 * N + v] = v == D.pref_vid ? D.pref : bp;
}

// matrix values: one warp per row, each lane sums its slots' triplets in push order
__global__ void __launch_bounds__(256) k_ns_values(NsDev D) {
    const int lane = threadIdx.x & 31;
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= 4 * D.n) return;
    const double* t = D.tv + D.trip_ptr[r];
    for (int32_t s = D.rp[r] + lane; s < D.rp[r + 1]; s += 32) {
        double acc = 0.0;
        for (int64_t j = D.slot_ptr[s]; j < D.slot_ptr[s + 1]; ++j) acc += t[D.slot_loc[j]];
        D.val[s] = acc;
    }
}

// 4x4 block inverses for the block-Jacobi preconditioner
__global__ void __launch_bounds__(256) k_bj4_setup(int64_t nb, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                   const double* __restrict__ val, double* __restrict__ binv, int* bad) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nb) return;
    double a[4][8];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int64_t row = r * nb + v;
        const int32_t s0 = rp[row], s1 = rp[row + 1];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int32_t col = (int32_t)(c * nb + v);
            int32_t lo = s0, hi = s1;  // binary search of the column in the sorted row
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (ci[mid] < col) lo = mid + 1;
                else hi = mid;
            }
            a[r][c] = (lo < s1 && ci[lo] == col) ? val[lo] : 0.0;
            a[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    }
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int piv = k;
        double best = fabs(a[k][k]);
#pragma unroll
        for (int r = k + 1; r < 4; ++r)
            if (fabs(a[r][k]) > best) {
                best = fabs(a[r][k]);
                piv = r;
            }
        if (!(best > 0.0) || !isfinite(best)) ok = false;
#pragma unroll
        for (int c = 0; c < 8; ++c) {  // swap rows k and piv (branch-free over the unrolled rows)
#pragma unroll
            for (int r = k + 1; r < 4; ++r)
                if (r == piv) {
                    const double tmp = a[k][c];
                    a[k][c] = a[r][c];
                    a[r][c] = tmp;
                }
        }
        const double inv = ok ? 1.0 / a[k][k] : 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) a[k][c] *= inv;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r != k) {
                const double f = a[r][k];
#pragma unroll
                for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
            }
    }
    if (!ok) atomicExch(bad, 1);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) binv[(r * 4 + c) * nb + v] = a[r][4 + c];
}

inline int blocks_for(int64_t threads) { return (int)((threads + 255) / 256); }

}  // namespace

void launch_ns_assemble(cudaStream_t s, const NsDev& D) {
    k_ns_rc<<<blocks_for(D.n), 256, 0, s>>>(D);
    k_ns_mom<<<blocks_for(D.n), 256, 0, s>>>(D);
    k_ns_flux<<<blocks_for(D.n), 256, 0, s>>>(D);
    k_ns_trip_mom<<<blocks_for(D.n), 256, 0, s>>>(D);
    k_ns_trip_p<<<blocks_for(D.n * 32), 256, 0, s>>>(D);
    k_ns_rhs<<<blocks_for(D.n), 256, 0, s>>>(D);
    k_ns_values<<<blocks_for(4 * D.n * 32), 256, 0, s>>>(D);
}

void launch_bj4_setup(cudaStream_t s, int64_t nb, const int32_t* rp, const int32_t* ci, const double* val, double* binv, int* bad) {
    k_bj4_setup<<<blocks_for(nb), 256, 0, s>>>(nb, rp, ci, val, binv, bad);
}

}  // namespace vfv
