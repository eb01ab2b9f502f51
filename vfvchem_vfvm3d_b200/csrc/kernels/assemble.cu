// Device assembly of the steady heat operator into a fixed CSR pattern (sm_100a).
//
// Restates, per row and in the reference's push order:
//   ScalarDomain::update_grad          src/base/scl_dom.rs:146-164
//   OpSclDomDiffusion / OpSclBndDiffusion  src/operator/core/opscl_dom_diff.rs:40-91, opscl_bnd_diff.rs:40-96
//   OpSclDomProduction / OpSclBndProduction opscl_dom_prod.rs:39-76, opscl_bnd_prod.rs:39-81
//   OpSclDomSource / OpSclBndSource         opscl_dom_src.rs:37-68, opscl_bnd_src.rs:37-73
//   OpSclBndDirichlet                       opscl_bnd_dir.rs:56-78
//   OpSclBndNeumann                         opscl_bnd_neu.rs:36-88
// in the order of SteadyHeat::assemble_matrix (src/steady/core/steady_heat.rs:143-171).
// The triplets a row receives are summed in push order by LinearGmres::build_matrix
// (src/linear/linear_gmres.rs:66-74); here each row is owned by one group of lanes, the
// off-diagonal coefficients are written straight into their CSR slots and lane 0 of the group adds
// the diagonal contributions in the same order, so the result is deterministic and atomic-free.
// This file is compiled with -fmad=false: every product and sum rounds exactly like the
// reference's scalar code.
#include "assemble.cuh"

namespace vfv {


__device__ __forceinline__ unsigned group_mask(int G) {
    const int lane = threadIdx.x & 31;
    const unsigned base = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
    return base << (lane & ~(G - 1));
}

// grad_f[v] = sum_loc w[v][loc] * (f[n] - f[v]) for NF <= 4 fields at once; out layout [field][3][n].
// One thread per row: the 3 NF components are summed in registers in face order (the reference's
// summation order). Measured against 16 lanes per row with the terms staged in shared memory: half
// the time on the 10^6-vertex mesh (the faces of a row are contiguous, so a thread's loads stream
// through L1, and no lane waits on another).
template <int NF>
__global__ void __launch_bounds__(256) k_grad_lsq(int64_t n, const int32_t* __restrict__ np, const int32_t* __restrict__ ni,
                                                     const double* __restrict__ gw, int64_t n_dir, const double* __restrict__ f0,
                                                     const double* __restrict__ f1, const double* __restrict__ f2,
                                                     const double* __restrict__ f3, double* __restrict__ out) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const double* F[4] = {f0, f1, f2, f3};
    double fv[NF], acc[3 * NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) fv[f] = F[f][v];
#pragma unroll
    for (int c = 0; c < 3 * NF; ++c) acc[c] = 0.0;
    const int32_t b = np[v], e = np[v + 1];
    for (int32_t i = b; i < e; ++i) {
        const int32_t nb = ni[i];
        const double wx = gw[i], wy = gw[n_dir + i], wz = gw[2 * n_dir + i];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const double dlt = F[f][nb] - fv[f];
            acc[3 * f] += wx * dlt;
            acc[3 * f + 1] += wy * dlt;
            acc[3 * f + 2] += wz * dlt;
        }
    }
#pragma unroll
    for (int c = 0; c < 3 * NF; ++c) out[(int64_t)c * n + v] = acc[c];
}

// kHeatG lanes per row: a row's ~15 faces in 4 chunks. Measured on the 10^6-vertex mesh against 16
// lanes (one chunk): 40% less time, from more resident rows and a 4-step instead of a 16-step
// serial diagonal sum.
constexpr int kHeatG = 4;

__global__ void __launch_bounds__(256, 6) k_assemble_heat(HeatDev H) {
    const int lane = threadIdx.x & (kHeatG - 1);
    const int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kHeatG;
    if (v >= H.n) return;
    const unsigned mask = group_mask(kHeatG);
    const int32_t kind = H.kind[v];
    const int32_t rb = H.rp[v];
    if (kind == ROW_DIRICHLET) {
        if (lane == 0) {
            H.val[rb] = 1.0;
            H.b[v] = 0.0 + H.bcv[v];
        }
        return;
    }
    const int64_t N = H.n, D = H.n_dir;
    const double kv = H.k[v];
    const double gkx = H.gk[v], gky = H.gk[N + v], gkz = H.gk[2 * N + v];
    const int32_t b = H.np[v], e = H.np[v + 1];
    const int32_t dl = H.dloc[v];
    double diag = 0.0;
    for (int32_t c0 = b; c0 < e; c0 += kHeatG) {
        const int32_t i = c0 + lane;
        double cf = 0.0;
        if (i < e) {
            const int32_t nb = H.ni[i];
            const double kn = H.k[nb];
            const double sx = H.skew[i], sy = H.skew[D + i], sz = H.skew[2 * D + i];
            const double km = (kv + kn != 0.0) ? 2.0 * kv * kn / (kv + kn) : 0.0;
            double kf = km + 0.5 * (sx * (gkx + H.gk[nb]) + sy * (gky + H.gk[N + nb]) + sz * (gkz + H.gk[2 * N + nb]));
            kf = kf > 0.0 ? kf : km;
            cf = kf * H.area[i] / H.dist[i];
            const int32_t loc = i - b;
            H.val[rb + loc + (loc >= dl ? 1 : 0)] = cf;
        }
        const int cnt = min(kHeatG, (int)(e - c0));
        for (int q = 0; q < cnt; ++q) {
            const double t = __shfl_sync(mask, cf, q, kHeatG);
            diag += -t;
        }
    }
    if (lane != 0) return;
    // production (implicit diagonal + lagged skew term) then source, then Neumann on flux nodes
    const double sxc = H.cskew[v], syc = H.cskew[N + v], szc = H.cskew[2 * N + v];
    const double vol = H.cvol[v];
    const double sv = H.s[v];
    const double prd_c = sv + H.gs[v] * sxc + H.gs[N + v] * syc + H.gs[2 * N + v] * szc;
    const double unk_skew = H.gT[v] * sxc + H.gT[N + v] * syc + H.gT[2 * N + v] * szc;
    diag += prd_c * vol;
    H.val[rb + dl] = diag;
    double bb = 0.0;
    bb += -sv * unk_skew * vol;
    const double src_c = H.q[v] + H.gq[v] * sxc + H.gq[N + v] * syc + H.gq[2 * N + v] * szc;
    bb += -src_c * vol;
    if (kind == ROW_FLUX) {
        const int64_t B = H.n_bsub;
        const double fv = H.bcv[v];
        const int32_t my = H.node_bnd[v];
        for (int32_t s = H.bp[v]; s < H.bp[v + 1]; ++s) {
            const int32_t j = H.bj[s], k = H.bk[s];
            const double fj = H.node_bnd[j] == my ? H.bcv[j] : fv;
            const double fk = H.node_bnd[k] == my ? H.bcv[k] : fv;
            bb += H.barea[s] * (H.bw[s] * fv + H.bw[B + s] * fj + H.bw[2 * B + s] * fk);
        }
    }
    H.b[v] = bb;
}

// ---------------------------------------------------------------- transient transport (batched meshes)
// Face mass flux with zero pressure and body force (flow_helper.rs:72-179 with vel_rc = 0):
//   F = rho_f (u_f . n) A,  rho = 1,  u_f = skew-corrected arithmetic mean of the vertex velocities.
__global__ void __launch_bounds__(256) k_face_flux(TransportDev T) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= T.n) return;
    const int64_t N = T.n, D = T.n_dir;
    const double uv = T.vel[v], vv = T.vel[N + v], wv = T.vel[2 * N + v];
    double g[9];
    for (int c = 0; c < 9; ++c) g[c] = T.gvel[c * N + v];
    for (int32_t i = T.np[v]; i < T.np[v + 1]; ++i) {
        const int32_t nb = T.ni[i];
        const double sx = T.skew[i], sy = T.skew[D + i], sz = T.skew[2 * D + i];
        const double nx = T.norm[i], ny = T.norm[D + i], nz = T.norm[2 * D + i];
        const double den_f = 0.5 * (1.0 + 1.0) + 0.5 * (sx * (0.0 + 0.0) + sy * (0.0 + 0.0) + sz * (0.0 + 0.0));
        const double u_f = 0.5 * (uv + T.vel[nb]) + 0.5 * (sx * (g[0] + T.gvel[nb]) + sy * (g[1] + T.gvel[N + nb]) + sz * (g[2] + T.gvel[2 * N + nb]));
        const double v_f = 0.5 * (vv + T.vel[N + nb]) +
                           0.5 * (sx * (g[3] + T.gvel[3 * N + nb]) + sy * (g[4] + T.gvel[4 * N + nb]) + sz * (g[5] + T.gvel[5 * N + nb]));
        const double w_f = 0.5 * (wv + T.vel[2 * N + nb]) +
                           0.5 * (sx * (g[6] + T.gvel[6 * N + nb]) + sy * (g[7] + T.gvel[7 * N + nb]) + sz * (g[8] + T.gvel[8 * N + nb]));
        T.flux[i] = den_f * (u_f * nx + v_f * ny + w_f * nz + 0.0) * T.area[i];
    }
}

// power-law factor A(|Pe|) = max(0, 1 - 0.1 |Pe|)^5, the fifth power as x^2 x^2 x
__device__ __forceinline__ double power_law(double pe) {
    const double x = fmax(1.0 - 0.1 * fabs(pe), 0.0);
    const double x2 = x * x;
    return x2 * x2 * x;
}

// Row v, push order: time (v,v), diffusion (v,n)/(v,v) per face, advection (v,n)/(v,v) per face.
// Off-diagonal slot = c + coeff, diagonal = -vol/dt - sum c - sum coeff, each summed in that order.
__global__ void __launch_bounds__(256) k_assemble_transport(TransportDev T) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= T.n) return;
    const int64_t N = T.n, E = T.n_dir;
    const int32_t b = T.np[v], e = T.np[v + 1];
    const int32_t rb = T.rp[v], dl = T.dloc[v];
    const double Dv = T.D[v];
    const double gx = T.gD[v], gy = T.gD[N + v], gz = T.gD[2 * N + v];
    double diag = -T.cvol[v] / T.dt;
    for (int pass = 0; pass < 2; ++pass) {
        for (int32_t i = b; i < e; ++i) {
            const int32_t nb = T.ni[i];
            const double Dn = T.D[nb];
            const double sx = T.skew[i], sy = T.skew[E + i], sz = T.skew[2 * E + i];
            const double dm = (Dv + Dn != 0.0) ? 2.0 * Dv * Dn / (Dv + Dn) : 0.0;
            double df = dm + 0.5 * (sx * (gx + T.gD[nb]) + sy * (gy + T.gD[N + nb]) + sz * (gz + T.gD[2 * N + nb]));
            df = df > 0.0 ? df : dm;
            const double cond = df * T.area[i] / T.dist[i];
            const int32_t loc = i - b;
            const int32_t slot = rb + loc + (loc >= dl ? 1 : 0);
            if (pass == 0) {
                T.val[slot] = cond;
                diag += -cond;
            } else {
                const double wgt_f = 0.5 * (1.0 + 1.0) + 0.5 * (sx * (0.0 + 0.0) + sy * (0.0 + 0.0) + sz * (0.0 + 0.0));
                const double den_f = wgt_f;
                const double flux = den_f != 0.0 ? wgt_f / den_f * T.flux[i] : 0.0;
                const double pe = cond != 0.0 ? flux / cond : 0.0;
                const double coeff = cond * (power_law(pe) - 1.0) + fmax(-flux, 0.0);
                T.val[slot] += coeff;
                diag += -coeff;
            }
        }
    }
    T.val[rb + dl] = diag;
}

// b = -c_prev vol / dt  (OpSclDomTimeUnity::apply_time right-hand side; zero-flux walls add nothing)
__global__ void k_transport_rhs(int64_t n, const double* __restrict__ cvol, double dt, const double* __restrict__ c_prev, double* __restrict__ b) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) b[v] = 0.0 + -c_prev[v] * cvol[v] / dt;
}

// lam^T (dA/dD) c for a uniform D: per face cond = D A/d, coeff = cond (P(|Pe|) - 1) + max(-F, 0) with
// Pe = F / cond, so d(cond + coeff)/dD = (A/d) (P(|Pe|) - |Pe| P'(|Pe|)), P'(x) = -0.5 (1 - 0.1 x)^4.
// Deterministic: per-block partials, the last block sums them in block order into *out.
__global__ void __launch_bounds__(256) k_transport_dAdD_dot(TransportDev T, const double* __restrict__ lam, const double* __restrict__ c,
                                                           double* part, unsigned* counter, double* out) {
    __shared__ double red[8];
    __shared__ bool s_last;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (v < T.n) {
        const double Dv = T.D[v], cv = c[v];
        double sum = 0.0;
        for (int32_t i = T.np[v]; i < T.np[v + 1]; ++i) {
            const int32_t nb = T.ni[i];
            const double Dn = T.D[nb];
            const double dm = (Dv + Dn != 0.0) ? 2.0 * Dv * Dn / (Dv + Dn) : 0.0;
            const double g = T.area[i] / T.dist[i];
            const double cond = dm * g;
            const double pe = cond != 0.0 ? fabs(T.flux[i] / cond) : 0.0;
            const double x = fmax(1.0 - 0.1 * pe, 0.0);
            const double x2 = x * x;
            const double P = x2 * x2 * x;
            const double dP = -0.5 * x2 * x2;
            sum += g * (P - pe * dP) * (c[nb] - cv);
        }
        acc = lam[v] * sum;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += red[w];
        part[blockIdx.x] = b;
        __threadfence();
        s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double t = 0.0;
    for (unsigned bb = threadIdx.x; bb < gridDim.x; bb += blockDim.x) t += __ldcg(part + bb);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        *out = tot;
        *counter = 0u;
    }
}

void launch_transport_dAdD_dot(cudaStream_t s, const TransportDev& T, const double* lam, const double* c, double* part, unsigned* counter,
                               double* out) {
    k_transport_dAdD_dot<<<(unsigned)((T.n + 255) / 256), 256, 0, s>>>(T, lam, c, part, counter, out);
}

void launch_face_flux(cudaStream_t s, const TransportDev& T) { k_face_flux<<<(unsigned)((T.n + 255) / 256), 256, 0, s>>>(T); }
void launch_assemble_transport(cudaStream_t s, const TransportDev& T) {
    k_assemble_transport<<<(unsigned)((T.n + 255) / 256), 256, 0, s>>>(T);
}
void launch_transport_rhs(cudaStream_t s, int64_t n, const double* cvol, double dt, const double* c_prev, double* b) {
    k_transport_rhs<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, cvol, dt, c_prev, b);
}

// build_matrix from triplets: slot s receives the triplet values of its run, summed in push order.
__global__ void k_values_from_triplets(int64_t nnz, const int64_t* __restrict__ sp, const int64_t* __restrict__ st,
                                       const double* __restrict__ tv, double* __restrict__ val) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    double acc = 0.0;
    for (int64_t t = sp[s]; t < sp[s + 1]; ++t) acc += tv[st[t]];
    val[s] = acc;
}

void launch_grad(cudaStream_t s, int64_t n, const int32_t* np, const int32_t* ni, const double* gw, int64_t n_dir, int nf,
                 const double* const* f, double* out) {
    const int blocks = (int)((n + 255) / 256);
    const double* g1 = nf > 1 ? f[1] : nullptr;
    const double* g2 = nf > 2 ? f[2] : nullptr;
    const double* g3 = nf > 3 ? f[3] : nullptr;
    switch (nf) {
        case 1: k_grad_lsq<1><<<blocks, 256, 0, s>>>(n, np, ni, gw, n_dir, f[0], g1, g2, g3, out); break;
        case 2: k_grad_lsq<2><<<blocks, 256, 0, s>>>(n, np, ni, gw, n_dir, f[0], g1, g2, g3, out); break;
        case 3: k_grad_lsq<3><<<blocks, 256, 0, s>>>(n, np, ni, gw, n_dir, f[0], g1, g2, g3, out); break;
        default: k_grad_lsq<4><<<blocks, 256, 0, s>>>(n, np, ni, gw, n_dir, f[0], g1, g2, g3, out); break;
    }
}

void launch_assemble_heat(cudaStream_t s, const HeatDev& H) {
    const int blocks = (int)((H.n * kHeatG + 255) / 256);
    k_assemble_heat<<<blocks, 256, 0, s>>>(H);
}

void launch_values_from_triplets(cudaStream_t s, int64_t nnz, const int64_t* sp, const int64_t* st, const double* tv, double* val) {
    const int blocks = (int)((nnz + 255) / 256);
    if (blocks > 0) k_values_from_triplets<<<blocks, 256, 0, s>>>(nnz, sp, st, tv, val);
}

}  // namespace vfv
