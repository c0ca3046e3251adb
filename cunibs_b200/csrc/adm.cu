// Auxiliary dipole method (reference adm/reciprocity.py, evaluate.py): a target functional of the
// E-field by reciprocity, so that any coil placement's target field is a dipole sum over a
// precomputed field instead of a FEM solve.
//
// For J_d = sum over target elements e of alpha_e (dir_d . E_e), E_e = -G_e v - dA/dt_e, the
// adjoint potential lambda_d solving K lambda_d = c_d, c_d[n] = sum_e alpha_e (dir_d . g_en), gives
//     J_d = sum_e w_e . dA/dt_e,   w_e = vol_e sigma_e G_e lambda_d - [e in target] alpha_e dir_d,
// and, dA/dt_e being the mean of its four nodal values, J_d = sum_n W_n . dA/dt_n with
// W_n = 1/4 sum_{e at n} w_e (reciprocity.py:1-8). The reciprocity field
//     Q_d(g) = mu0/4pi sum_n W_n x (g - r_n) / |g - r_n|^3
// then gives E_d = didt sum_j m_j . Q_d(s_j) for the placed coil dipoles (s_j, m_j).
#include <algorithm>
#include <climits>
#include <cmath>

#include "internal.hpp"

namespace cunibs {
namespace {

// c_red[r][d] = sum over the corners of node i of alpha_e (dir_d . g_corner), FP64, node-to-corner
// order; columns past n_dir repeat the last direction.
template <int K>
__global__ void __launch_bounds__(64 * K) adjoint_rhs_kernel(const double* __restrict__ alpha, const double* __restrict__ g,
                                                             const int* __restrict__ ptr, const int* __restrict__ idx,
                                                             int n_nodes, int ground, AdmDirections dirs,
                                                             double* __restrict__ c_red) {
    const int r = blockIdx.x * 64 + threadIdx.x / K;
    const int d = threadIdx.x % K;
    if (r >= n_nodes - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    const int src = d < dirs.n ? d : dirs.n - 1;
    const double ex = dirs.e[src][0], ey = dirs.e[src][1], ez = dirs.e[src][2];
    double acc = 0.0;
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
        const int corner = idx[q];
        const double a = alpha[corner >> 2];
        if (a == 0.0) continue;
        const double* gc = g + 3 * static_cast<long>(corner);
        acc += a * (ex * gc[0] + ey * gc[1] + ez * gc[2]);
    }
    c_red[static_cast<long>(r) * K + d] = acc;
}

// W[d][n] = 1/4 sum over the corners of node n of w_e, w_e = vol_e sigma_e G_e lambda_d -
// alpha_e dir_d, in node-to-corner order (the transpose of the corner reduction).
__global__ void node_weights_kernel(const double* __restrict__ lam, int K, const double* __restrict__ alpha,
                                    const double* __restrict__ g, const double* __restrict__ vols,
                                    const double* __restrict__ cond, const int* __restrict__ tets,
                                    const int* __restrict__ ptr, const int* __restrict__ idx, int n_nodes, int ground,
                                    AdmDirections dirs, double* __restrict__ W) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n_nodes) * dirs.n) return;
    const int d = static_cast<int>(q / n_nodes);
    const int n = static_cast<int>(q % n_nodes);
    double wx = 0.0, wy = 0.0, wz = 0.0;
    for (int p = ptr[n]; p < ptr[n + 1]; ++p) {
        const int e = idx[p] >> 2;
        const int4 tn = reinterpret_cast<const int4*>(tets)[e];
        const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
        const double* ge = g + 12 * static_cast<long>(e);
        double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int v = nd[c];
            const double l = v == ground ? 0.0 : lam[static_cast<long>(v - (v > ground ? 1 : 0)) * K + d];
            gx = fma(ge[3 * c], l, gx);
            gy = fma(ge[3 * c + 1], l, gy);
            gz = fma(ge[3 * c + 2], l, gz);
        }
        const double s = vols[e] * cond[e];
        const double a = alpha[e];
        wx += s * gx - a * dirs.e[d][0];
        wy += s * gy - a * dirs.e[d][1];
        wz += s * gz - a * dirs.e[d][2];
    }
    double* o = W + (static_cast<long>(d) * n_nodes + n) * 3;
    o[0] = 0.25 * wx;
    o[1] = 0.25 * wy;
    o[2] = 0.25 * wz;
}

// (nodes - centre) in metres: the sources of the reciprocity N-body, centred like its targets.
__global__ void centred_nodes_kernel(const double* __restrict__ nodes_mm, int n, double cx, double cy, double cz,
                                     double* __restrict__ out_m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out_m[3 * static_cast<long>(i)] = (nodes_mm[3 * static_cast<long>(i)] - cx) * 1e-3;
    out_m[3 * static_cast<long>(i) + 1] = (nodes_mm[3 * static_cast<long>(i) + 1] - cy) * 1e-3;
    out_m[3 * static_cast<long>(i) + 2] = (nodes_mm[3 * static_cast<long>(i) + 2] - cz) * 1e-3;
}

// Grid points in C order (x slowest), mm.
__global__ void grid_points_kernel(AdmGrid gr, double* __restrict__ out) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long total = static_cast<long>(gr.shape[0]) * gr.shape[1] * gr.shape[2];
    if (q >= total) return;
    const int iz = static_cast<int>(q % gr.shape[2]);
    const int iy = static_cast<int>((q / gr.shape[2]) % gr.shape[1]);
    const int ix = static_cast<int>(q / (static_cast<long>(gr.shape[1]) * gr.shape[2]));
    out[3 * q] = gr.origin_mm[0] + gr.spacing_mm[0] * ix;
    out[3 * q + 1] = gr.origin_mm[1] + gr.spacing_mm[1] * iy;
    out[3 * q + 2] = gr.origin_mm[2] + gr.spacing_mm[2] * iz;
}

constexpr int kEvalThreads = 256;
constexpr double kIndexTol = 1e-6;  // slack on the fractional grid index (3 nm at 3 mm)

__device__ __forceinline__ void place_dipole(const double* __restrict__ Tp, const double* __restrict__ pos,
                                             const double* __restrict__ mom, int j, double s_mm[3], double m[3]) {
    const double px = pos[3 * j] * 1e3, py = pos[3 * j + 1] * 1e3, pz = pos[3 * j + 2] * 1e3;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        s_mm[a] = Tp[4 * a] * px + Tp[4 * a + 1] * py + Tp[4 * a + 2] * pz + Tp[4 * a + 3];
        m[a] = Tp[4 * a] * mom[3 * j] + Tp[4 * a + 1] * mom[3 * j + 1] + Tp[4 * a + 2] * mom[3 * j + 2];
    }
}

// Fixed-order block sum of kAdmMaxDir accumulators into E[p][d] (thread 0 writes).
__device__ __forceinline__ void block_sum_write(double (&acc)[kAdmMaxDir], int n_dir, double didt, double* __restrict__ E,
                                                int p) {
    __shared__ double red[kAdmMaxDir][kEvalThreads];
#pragma unroll
    for (int d = 0; d < kAdmMaxDir; ++d) red[d][threadIdx.x] = acc[d];
    __syncthreads();
    for (int off = kEvalThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off)
#pragma unroll
            for (int d = 0; d < kAdmMaxDir; ++d) red[d][threadIdx.x] += red[d][threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < n_dir; ++d) E[static_cast<long>(p) * n_dir + d] = didt * red[d][0];
}

// One block per placement: E[p][d] = didt sum_j m_j . Q_d(s_j), Q trilinear on the grid (values
// clamped to the edge, as an interpolation in "nearest" mode; a dipole off the grid by more than
// the index slack is recorded per axis as its flat sample index p * n_dip + j and skipped).
__global__ void __launch_bounds__(kEvalThreads) evaluate_kernel(const float* __restrict__ Q, int n_dir, AdmGrid gr,
                                                                const double* __restrict__ pos,
                                                                const double* __restrict__ mom, int n_dip,
                                                                const double* __restrict__ T, double didt,
                                                                double* __restrict__ E,
                                                                unsigned long long* __restrict__ bad) {
    const int p = blockIdx.x;
    const double* Tp = T + 16 * static_cast<long>(p);
    const long nyz = static_cast<long>(gr.shape[1]) * gr.shape[2];
    const long n_grid = nyz * gr.shape[0];
    double acc[kAdmMaxDir] = {};
    for (int j = threadIdx.x; j < n_dip; j += kEvalThreads) {
        double s[3], m[3];
        place_dipole(Tp, pos, mom, j, s, m);
        int i0[3];
        double t[3];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double x = (s[a] - gr.origin_mm[a]) / gr.spacing_mm[a];
            const double hi = static_cast<double>(gr.shape[a] - 1);
            if (!(x >= -kIndexTol && x <= hi + kIndexTol)) {
                atomicMin(bad + a, static_cast<unsigned long long>(p) * n_dip + j);
                ok = false;
            }
            const double xc = fmin(fmax(x, 0.0), hi);
            int b = static_cast<int>(floor(xc));
            b = gr.shape[a] > 1 ? min(b, gr.shape[a] - 2) : 0;
            i0[a] = b;
            t[a] = gr.shape[a] > 1 ? xc - b : 0.0;
        }
        if (!ok) continue;
        const int dx = gr.shape[0] > 1 ? 1 : 0, dy = gr.shape[1] > 1 ? 1 : 0, dz = gr.shape[2] > 1 ? 1 : 0;
        const long base = (static_cast<long>(i0[0]) * gr.shape[1] + i0[1]) * gr.shape[2] + i0[2];
        const long off[8] = {0, dz, dy * gr.shape[2], dy * gr.shape[2] + dz, dx * nyz, dx * nyz + dz,
                             dx * nyz + dy * gr.shape[2], dx * nyz + dy * gr.shape[2] + dz};
        const double wx[2] = {1.0 - t[0], t[0]}, wy[2] = {1.0 - t[1], t[1]}, wz[2] = {1.0 - t[2], t[2]};
        for (int d = 0; d < n_dir; ++d) {
            const float* Qd = Q + static_cast<long>(d) * n_grid * 3;
            double qx = 0.0, qy = 0.0, qz = 0.0;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const double w = wx[c >> 2] * wy[(c >> 1) & 1] * wz[c & 1];
                const float* v = Qd + 3 * (base + off[c]);
                qx += w * v[0];
                qy += w * v[1];
                qz += w * v[2];
            }
            acc[d] += m[0] * qx + m[1] * qy + m[2] * qz;
        }
    }
    block_sum_write(acc, n_dir, didt, E, p);
}

// Placed dipole positions (mm) and moments of P placements, (P * n_dip, 3) each.
__global__ void placed_dipoles_kernel(const double* __restrict__ pos, const double* __restrict__ mom, int n_dip,
                                      const double* __restrict__ T, int P, double* __restrict__ s_mm,
                                      double* __restrict__ m_out) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(P) * n_dip) return;
    const int p = static_cast<int>(q / n_dip), j = static_cast<int>(q % n_dip);
    double s[3], m[3];
    place_dipole(T + 16 * static_cast<long>(p), pos, mom, j, s, m);
    for (int a = 0; a < 3; ++a) {
        s_mm[3 * q + a] = s[a];
        m_out[3 * q + a] = m[a];
    }
}

// E[p][d] = didt sum_j m_j . Qx[d][p * n_dip + j], Q evaluated at the dipoles themselves.
__global__ void __launch_bounds__(kEvalThreads) exact_reduce_kernel(const float* __restrict__ Qx, int n_dir, int P,
                                                                    int n_dip, const double* __restrict__ m_all,
                                                                    double didt, double* __restrict__ E) {
    const int p = blockIdx.x;
    const long n_pts = static_cast<long>(P) * n_dip;
    double acc[kAdmMaxDir] = {};
    for (int j = threadIdx.x; j < n_dip; j += kEvalThreads) {
        const long q = static_cast<long>(p) * n_dip + j;
        for (int d = 0; d < n_dir; ++d) {
            const float* v = Qx + (static_cast<long>(d) * n_pts + q) * 3;
            acc[d] += m_all[3 * q] * v[0] + m_all[3 * q + 1] * v[1] + m_all[3 * q + 2] * v[2];
        }
    }
    block_sum_write(acc, n_dir, didt, E, p);
}

}  // namespace

void adm_adjoint_rhs(const Mesh& m, const double* alpha, const AdmDirections& dirs, int K, double* c_red,
                     cudaStream_t s) {
    const unsigned grid = (m.n_nodes - 1 + 63) / 64;
    auto go = [&](auto kc) {
        constexpr int KK = decltype(kc)::value;
        adjoint_rhs_kernel<KK><<<grid, 64 * KK, 0, s>>>(alpha, m.g.get(), m.n2c_ptr.get(), m.n2c_idx.get(), m.n_nodes,
                                                        m.ground, dirs, c_red); count_launch();
    };
    switch (K) {
        case 1: go(std::integral_constant<int, 1>{}); break;
        case 2: go(std::integral_constant<int, 2>{}); break;
        case 4: go(std::integral_constant<int, 4>{}); break;
        default: fail(kEInval, "adjoint block width must be 1, 2 or 4");
    }
    CUNIBS_LAUNCH_CHECK("adjoint rhs");
}

void adm_node_weights(const Mesh& m, const double* lam, int K, const double* alpha, const AdmDirections& dirs,
                      double* W, cudaStream_t s) {
    const long total = static_cast<long>(m.n_nodes) * dirs.n;
    node_weights_kernel<<<grid_for(total), kBlock, 0, s>>>(lam, K, alpha, m.g.get(), m.vols.get(), m.cond.get(),
                                                          m.tets.get(), m.n2c_ptr.get(), m.n2c_idx.get(), m.n_nodes,
                                                          m.ground, dirs, W); count_launch();
    CUNIBS_LAUNCH_CHECK("adm node weights");
}

void adm_centred_nodes(const Mesh& m, const double* center_mm, double* out_m, cudaStream_t s) {
    centred_nodes_kernel<<<grid_for(m.n_nodes), kBlock, 0, s>>>(m.nodes.get(), m.n_nodes, center_mm[0], center_mm[1],
                                                               center_mm[2], out_m); count_launch();
    CUNIBS_LAUNCH_CHECK("adm centred nodes");
}

void adm_grid_points(const AdmGrid& gr, double* out, cudaStream_t s) {
    const long total = static_cast<long>(gr.shape[0]) * gr.shape[1] * gr.shape[2];
    grid_points_kernel<<<grid_for(total), kBlock, 0, s>>>(gr, out); count_launch();
    CUNIBS_LAUNCH_CHECK("adm grid points");
}

void adm_evaluate(const float* Q, int n_dir, const AdmGrid& gr, const double* pos, const double* mom, int n_dip,
                  const double* T, int P, double didt, double* E, unsigned long long* bad, cudaStream_t s) {
    if (n_dir < 1 || n_dir > kAdmMaxDir) fail(kEInval, "between 1 and 3 adjoint directions");
    evaluate_kernel<<<P, kEvalThreads, 0, s>>>(Q, n_dir, gr, pos, mom, n_dip, T, didt, E, bad); count_launch();
    CUNIBS_LAUNCH_CHECK("adm evaluate");
}

void adm_placed_dipoles(const double* pos, const double* mom, int n_dip, const double* T, int P, double* s_mm,
                        double* m_out, cudaStream_t s) {
    const long total = static_cast<long>(P) * n_dip;
    placed_dipoles_kernel<<<grid_for(total), kBlock, 0, s>>>(pos, mom, n_dip, T, P, s_mm, m_out); count_launch();
    CUNIBS_LAUNCH_CHECK("adm placed dipoles");
}

void adm_exact_reduce(const float* Qx, int n_dir, int P, int n_dip, const double* m_all, double didt, double* E,
                      cudaStream_t s) {
    if (n_dir < 1 || n_dir > kAdmMaxDir) fail(kEInval, "between 1 and 3 adjoint directions");
    exact_reduce_kernel<<<P, kEvalThreads, 0, s>>>(Qx, n_dir, P, n_dip, m_all, didt, E); count_launch();
    CUNIBS_LAUNCH_CHECK("adm exact reduce");
}

}  // namespace cunibs
