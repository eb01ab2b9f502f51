// Adjoint of the steady heat assembly: dJ/d(log k) and dJ/dq for J(T(k, q)) (sm_100a).
//
// The residual is R(T; k, q) = A(k) T - b(q) with the operators of SteadyHeat::assemble_matrix
// (src/steady/core/steady_heat.rs:143-171) at zero production (s = 0, so b does not depend on T):
//   (A T)_v = sum_loc c_vn (T_n - T_v),  c_vn = k_f A_f / d_f          (opscl_dom_diff.rs:78-85)
//   k_f = k_m + 0.5 s_f . (grad k_v + grad k_n) if that is > 0, else k_m, k_m = 2 k_v k_n / (k_v + k_n)
//   grad k_v = sum_loc w_v,loc (k_n - k_v)                              (scl_dom.rs:146-164)
//   b_v = -(q_v + grad q_v . cskew_v) vol_v (+ terms independent of k and q) (opscl_dom_src.rs:48-65)
// With A^T lambda = dJ/dT: dJ/dp = -lambda^T dR/dp, i.e.
//   dJ/dk_m = sum_faces phi_vn dk_f,vn/dk_m,  phi_vn = -lambda_v (T_n - T_v) A_f / d_f
//   dJ/dq_m = lambda^T db/dq_m.
// The face derivative has a harmonic-mean part (k_v and k_n) and, where the guard did not fire, a
// skew part through the two gradients; the skew part is collected per vertex (Psi_u) and pushed
// through the gradient weights. Every sum is a gather in a fixed order (per row, using the
// reverse directed face for the opposite direction): deterministic, no atomics.
#include "adjoint.cuh"

namespace vfv {

// Phase 1, per directed face e = (v -> n) of non-Dirichlet rows:
//   pv[e] = phi dk_m/dk_v, pn[e] = phi dk_m/dk_n, sk[c][e] = 0.5 phi s_f (skew part, 0 if guarded)
__global__ void __launch_bounds__(256) k_adj_face(AdjDev D) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= D.n) return;
    const int64_t N = D.n, E = D.n_dir;
    const int32_t b = D.np[v], e = D.np[v + 1];
    if (D.kind[v] == ROW_DIRICHLET) {
        for (int32_t i = b; i < e; ++i) {
            D.pv[i] = 0.0;
            D.pn[i] = 0.0;
            D.sk[i] = D.sk[E + i] = D.sk[2 * E + i] = 0.0;
        }
        return;
    }
    const double kv = D.k[v], lam = D.lambda[v], Tv = D.T[v];
    const double gx = D.gk[v], gy = D.gk[N + v], gz = D.gk[2 * N + v];
    for (int32_t i = b; i < e; ++i) {
        const int32_t nb = D.ni[i];
        const double kn = D.k[nb];
        const double sx = D.skew[i], sy = D.skew[E + i], sz = D.skew[2 * E + i];
        const double ks = kv + kn;
        const double km = ks != 0.0 ? 2.0 * kv * kn / ks : 0.0;
        const double kraw = km + 0.5 * (sx * (gx + D.gk[nb]) + sy * (gy + D.gk[N + nb]) + sz * (gz + D.gk[2 * N + nb]));
        const double phi = -lam * (D.T[nb] - Tv) * D.area[i] / D.dist[i];
        const double inv = ks != 0.0 ? 1.0 / (ks * ks) : 0.0;
        D.pv[i] = phi * 2.0 * kn * kn * inv;
        D.pn[i] = phi * 2.0 * kv * kv * inv;
        const double h = kraw > 0.0 ? 0.5 * phi : 0.0;
        D.sk[i] = h * sx;
        D.sk[E + i] = h * sy;
        D.sk[2 * E + i] = h * sz;
    }
}

// Phase 2, per vertex m: gkm[m] = harmonic-mean part of dJ/dk_m, psi[c][m] = skew accumulators
__global__ void __launch_bounds__(256) k_adj_vertex(AdjDev D) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= D.n) return;
    const int64_t N = D.n, E = D.n_dir;
    double g = 0.0, px = 0.0, py = 0.0, pz = 0.0;
    for (int32_t i = D.np[m]; i < D.np[m + 1]; ++i) {
        const int32_t r = D.rev[i];
        g += D.pv[i] + D.pn[r];
        px += D.sk[i] + D.sk[r];
        py += D.sk[E + i] + D.sk[E + r];
        pz += D.sk[2 * E + i] + D.sk[2 * E + r];
    }
    D.gkm[m] = g;
    D.psi[m] = px;
    D.psi[N + m] = py;
    D.psi[2 * N + m] = pz;
}

// Phase 3, per vertex m: push psi through the gradient weights, chain rule to log k; source part
__global__ void __launch_bounds__(256) k_adj_final(AdjDev D) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= D.n) return;
    const int64_t N = D.n, E = D.n_dir;
    const double pmx = D.psi[m], pmy = D.psi[N + m], pmz = D.psi[2 * N + m];
    const bool own = D.kind[m] != ROW_DIRICHLET;
    const double csx = D.cskew[m], csy = D.cskew[N + m], csz = D.cskew[2 * N + m];
    double dk = D.gkm[m];
    double swx = 0.0, swy = 0.0, swz = 0.0, swc = 0.0, dq = 0.0;
    for (int32_t i = D.np[m]; i < D.np[m + 1]; ++i) {
        const int32_t u = D.ni[i], r = D.rev[i];
        const double wx = D.gw[i], wy = D.gw[E + i], wz = D.gw[2 * E + i];
        swx += wx;
        swy += wy;
        swz += wz;
        swc += wx * csx + wy * csy + wz * csz;
        const double rx = D.gw[r], ry = D.gw[E + r], rz = D.gw[2 * E + r];
        dk += D.psi[u] * rx + D.psi[N + u] * ry + D.psi[2 * N + u] * rz;
        if (D.kind[u] != ROW_DIRICHLET)
            dq += -D.lambda[u] * D.cvol[u] * (rx * D.cskew[u] + ry * D.cskew[N + u] + rz * D.cskew[2 * N + u]);
    }
    dk -= pmx * swx + pmy * swy + pmz * swz;
    if (own) dq += -D.lambda[m] * D.cvol[m] * (1.0 - swc);
    D.dlogk[m] = D.k[m] * dk;
    D.dq[m] = dq;
}

void launch_adjoint_partials(cudaStream_t s, const AdjDev& D) {
    const int blocks = (int)((D.n + 255) / 256);
    k_adj_face<<<blocks, 256, 0, s>>>(D);
    k_adj_vertex<<<blocks, 256, 0, s>>>(D);
    k_adj_final<<<blocks, 256, 0, s>>>(D);
}

}  // namespace vfv
