// Conductivity Monte Carlo on a fixed mesh and block of coil placements (reference
// uq/conductivity/assembly.py and run.py): the kernels that make each conductivity draw a value
// swap of the finest operator plus a sensitivity-subspace initial guess.
//
// Both the stiffness and the right-hand side are linear in the tissue conductivities, so the
// residual of the nominal solution x_nom under a draw is
//     r(sigma) = b(sigma) - A(sigma) x_nom = r_nom + sum_t (sigma_t - sigma_nom_t) c_t,
//     c_t[i]   = sum over the tissue-t elements e at node i of vol_e (g_ei . E_e),
// E_e = -grad v_nom - dA/dt_e the nominal field (r_nom is the nominal solve's residual, below
// its tolerance). The sensitivities s_t = A_nom^-1 c_t span the first-order change of the
// solution; a draw starts from x_nom plus the A_nom-Galerkin projection of its residual onto
// span{s_t} (run.py:105-200).
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "internal.hpp"

namespace cunibs {
namespace {

// out[p] = comp[0][p] + sum_t w_t comp[1 + t][p], in tag order (K(sigma) = K_base + sum sigma_t K_t).
__global__ void combine_values_kernel(const double* __restrict__ comp, int n_tags, long nnz, SigmaWeights w,
                                      double* __restrict__ out) {
    const long p = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    double v = comp[p];
#pragma unroll
    for (int t = 0; t < kSigmaMaxTags; ++t)
        if (t < n_tags) v = fma(w.w[t], comp[(t + 1) * nnz + p], v);
    out[p] = v;
}

// out[t][e] = -(vol_e * tables[t][tag_e]) in FP32, the right-hand side's element weights of table t
// (the same rounding as the mesh's own weights of a full conductivity table).
__global__ void element_weights_kernel(const float* __restrict__ vols32, const int* __restrict__ tags, int m,
                                       const double* __restrict__ tables, int n_tables, float* __restrict__ out) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(m) * n_tables) return;
    const int t = static_cast<int>(q / m), e = static_cast<int>(q % m);
    const int tag = tags[e];
    const double w = (tag >= 0 && tag <= 10) ? tables[11 * t + tag] : 0.0;
    out[q] = -(vols32[e] * static_cast<float>(w));
}

// c_out[r][a][j] = sum over the corners of node i whose element has tag tags_of_slot[a] of
// vol_e (g_corner . E_e), E_e from the grounded potential x_red (n_red, K) and the element dA/dt of
// placement j, accumulated in FP64 in node-to-corner order. Columns past k repeat column k-1.
template <int K>
__global__ void __launch_bounds__(64 * K) sens_rhs_kernel(const double* __restrict__ x_red, const float* __restrict__ dadt_elm,
                                                          const double* __restrict__ g, const double* __restrict__ vols,
                                                          const int* __restrict__ tets, const int* __restrict__ tags,
                                                          const int* __restrict__ ptr, const int* __restrict__ idx,
                                                          int n_nodes, int n_tets, int k, int ground, int P,
                                                          SigmaSlots slots, double* __restrict__ c_out) {
    const int r = blockIdx.x * 64 + threadIdx.x / K;
    const int j = threadIdx.x % K;
    if (r >= n_nodes - 1) return;
    const int i = r + (r >= ground ? 1 : 0);
    const int src = j < k ? j : k - 1;
    const float* el = dadt_elm + static_cast<long>(src) * n_tets * 3;
    double acc[kSigmaMaxTags];
#pragma unroll
    for (int a = 0; a < kSigmaMaxTags; ++a) acc[a] = 0.0;
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
        const int corner = idx[q];
        const int e = corner >> 2;
        const int a_of = slots.slot[tags[e]];
        if (a_of < 0) continue;
        const int4 tn = reinterpret_cast<const int4*>(tets)[e];
        const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
        const double* ge = g + 12 * static_cast<long>(e);
        double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int n = nd[c];
            const double xv = n == ground ? 0.0 : x_red[static_cast<long>(n - (n > ground ? 1 : 0)) * K + src];
            gx = fma(ge[3 * c], xv, gx);
            gy = fma(ge[3 * c + 1], xv, gy);
            gz = fma(ge[3 * c + 2], xv, gz);
        }
        const double ex = -gx - static_cast<double>(el[3 * static_cast<long>(e)]);
        const double ey = -gy - static_cast<double>(el[3 * static_cast<long>(e) + 1]);
        const double ez = -gz - static_cast<double>(el[3 * static_cast<long>(e) + 2]);
        const double* gc = ge + 3 * (corner & 3);
        const double val = vols[e] * (gc[0] * ex + gc[1] * ey + gc[2] * ez);
#pragma unroll
        for (int a = 0; a < kSigmaMaxTags; ++a)
            if (a == a_of) acc[a] += val;
    }
#pragma unroll
    for (int a = 0; a < kSigmaMaxTags; ++a)
        if (a < P) c_out[(static_cast<long>(r) * P + a) * K + j] = acc[a];
}

// Per-placement Gram blocks of two (n, P, K) arrays: out[j][a][b] = sum_r U[r][a][j] V[r][b][j].
// Row tiles of kGramRows are staged in shared memory; block b takes tiles b, b + grid, ... and
// each (j, a, b) sum runs over its tiles and rows in order, so the result depends on n only
// (not on K, P or the other placements). Tiles past n are zero-filled.
constexpr int kGramRows = 16;
constexpr int kGramThreads = 256;
constexpr int kGramPer = (16 * kSigmaMaxTags * kSigmaMaxTags + kGramThreads - 1) / kGramThreads;
constexpr int kGramBlocks = 296;

__global__ void __launch_bounds__(kGramThreads) gram_kernel(const double* __restrict__ U, const double* __restrict__ V,
                                                            long n, int P, int K, long n_tiles,
                                                            double* __restrict__ part) {
    extern __shared__ double sm[];
    const int W = P * K;
    double* su = sm;
    double* sv = sm + kGramRows * W;
    const int T = K * P * P;
    double acc[kGramPer];
#pragma unroll
    for (int m = 0; m < kGramPer; ++m) acc[m] = 0.0;
    for (long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const long r0 = tile * kGramRows;
        const long rows = n - r0 < kGramRows ? n - r0 : kGramRows;
        __syncthreads();
        for (int q = threadIdx.x; q < kGramRows * W; q += blockDim.x) {
            const bool in = q < rows * W;
            su[q] = in ? U[r0 * W + q] : 0.0;
            sv[q] = in ? V[r0 * W + q] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < kGramPer; ++m) {
            const int t = threadIdx.x + m * kGramThreads;
            if (t < T) {
                const int b = t % P, a = (t / P) % P, j = t / (P * P);
                double s = acc[m];
                for (int rr = 0; rr < kGramRows; ++rr) s = fma(su[rr * W + a * K + j], sv[rr * W + b * K + j], s);
                acc[m] = s;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < kGramPer; ++m) {
        const int t = threadIdx.x + m * kGramThreads;
        if (t < T) part[static_cast<long>(blockIdx.x) * T + t] = acc[m];
    }
}

__global__ void gram_final_kernel(const double* __restrict__ part, int blocks, int T, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    double s = 0.0;
    for (int b = 0; b < blocks; ++b) s += part[static_cast<long>(b) * T + t];
    out[t] = s;
}

// Y = A X for a row-major (n, W) block X (FP64 CSR, one thread per entry of Y).
__global__ void spmv_cols_kernel(const int* __restrict__ ptr, const int* __restrict__ col,
                                 const double* __restrict__ val, int n, int W, const double* __restrict__ X,
                                 double* __restrict__ Y) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n) * W) return;
    const int r = static_cast<int>(q / W), w = static_cast<int>(q % W);
    double acc = 0.0;
    for (int p = ptr[r]; p < ptr[r + 1]; ++p) acc = fma(val[p], X[static_cast<long>(col[p]) * W + w], acc);
    Y[q] = acc;
}

// A W-wide solve block (W <= 16) from chosen (a, j) columns of an (n, P, K) array; lanes past
// count repeat the last chosen column (the padding of a partial block).
__global__ void pack_columns_kernel(const double* __restrict__ C, int n, int P, int K, SigmaColumns cm, int W,
                                    double* __restrict__ Bw) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n) * W) return;
    const long r = q / W;
    const int l = static_cast<int>(q % W);
    const int u = l < cm.count ? l : cm.count - 1;
    Bw[q] = C[(r * P + cm.a[u]) * K + cm.j[u]];
}

__global__ void unpack_columns_kernel(const double* __restrict__ Xw, int n, int P, int K, SigmaColumns cm, int W,
                                      double* __restrict__ S) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n) * W) return;
    const long r = q / W;
    const int l = static_cast<int>(q % W);
    if (l >= cm.count) return;
    S[(r * P + cm.a[l]) * K + cm.j[l]] = Xw[q];
}

// X0[r][j] = x_nom[r][j] + sum_a S[r][a][j] y[a][j] (columns past k repeat column k-1).
__global__ void guess_kernel(const double* __restrict__ x_nom, const double* __restrict__ S, int n, int P, int K, int k,
                             SigmaDraw y, double* __restrict__ X0) {
    const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= static_cast<long>(n) * K) return;
    const long r = q / K;
    const int j = static_cast<int>(q % K);
    const int src = j < k ? j : k - 1;
    double v = x_nom[r * K + src];
    for (int a = 0; a < P; ++a) v = fma(S[(r * P + a) * K + src], y.y[a * 16 + src], v);
    X0[q] = v;
}

// Partial sums of (a - b)^2 and b^2 per block (fixed order), for the linearity check.
__global__ void diff_norms_kernel(const double* __restrict__ a, const double* __restrict__ b, long n,
                                  double* __restrict__ part) {
    __shared__ double sd[kBlock], sb[kBlock];
    double d2 = 0.0, b2 = 0.0;
    for (long p = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += static_cast<long>(gridDim.x) * blockDim.x) {
        const double d = a[p] - b[p];
        d2 = fma(d, d, d2);
        b2 = fma(b[p], b[p], b2);
    }
    sd[threadIdx.x] = d2;
    sb[threadIdx.x] = b2;
    __syncthreads();
    for (int off = kBlock / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            sd[threadIdx.x] += sd[threadIdx.x + off];
            sb[threadIdx.x] += sb[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sd[0];
        part[2 * blockIdx.x + 1] = sb[0];
    }
}

}  // namespace

void sigma_combine(const double* comp, int n_tags, long nnz, const SigmaWeights& w, double* out, cudaStream_t s) {
    combine_values_kernel<<<grid_for(nnz), kBlock, 0, s>>>(comp, n_tags, nnz, w, out); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma combine");
}

void sigma_element_weights(const Mesh& m, const double* tables_dev, int n_tables, float* out, cudaStream_t s) {
    const long total = static_cast<long>(m.n_tets) * n_tables;
    element_weights_kernel<<<grid_for(total), kBlock, 0, s>>>(m.vols32.get(), m.tags.get(), m.n_tets, tables_dev,
                                                             n_tables, out); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma element weights");
}

void sigma_sens_rhs(const Mesh& m, const double* x_red, const float* dadt_elm, int k, int K, const SigmaSlots& slots,
                    int P, double* c_out, cudaStream_t s) {
    if (P < 1 || P > kSigmaMaxTags) fail(kEInval, "between 1 and 10 perturbed tissues");
    const unsigned grid = (m.n_nodes - 1 + 63) / 64;
    auto go = [&](auto kc) {
        constexpr int KK = decltype(kc)::value;
        sens_rhs_kernel<KK><<<grid, 64 * KK, 0, s>>>(x_red, dadt_elm, m.g.get(), m.vols.get(), m.tets.get(), m.tags.get(),
                                                     m.n2c_ptr.get(), m.n2c_idx.get(), m.n_nodes, m.n_tets, k, m.ground,
                                                     P, slots, c_out); count_launch();
    };
    switch (K) {
        case 1: go(std::integral_constant<int, 1>{}); break;
        case 2: go(std::integral_constant<int, 2>{}); break;
        case 4: go(std::integral_constant<int, 4>{}); break;
        case 8: go(std::integral_constant<int, 8>{}); break;
        case 16: go(std::integral_constant<int, 16>{}); break;
        default: fail(kEInval, "block width must be one of {1, 2, 4, 8, 16}");
    }
    CUNIBS_LAUNCH_CHECK("sensitivity right-hand sides");
}

std::vector<double> sigma_gram(const double* U, const double* V, long n, int P, int K, cudaStream_t s) {
    if (P < 1 || P > kSigmaMaxTags || K < 1 || K > 16) fail(kEInval, "gram: P in [1, 10], K in [1, 16]");
    const long tiles = (n + kGramRows - 1) / kGramRows;
    const int blocks = static_cast<int>(tiles < kGramBlocks ? tiles : kGramBlocks);
    const int T = K * P * P;
    DevArray<double> part(static_cast<std::size_t>(blocks) * T), out(T);
    const std::size_t smem = sizeof(double) * 2 * kGramRows * P * K;
    gram_kernel<<<blocks, kGramThreads, smem, s>>>(U, V, n, P, K, tiles, part.get()); count_launch();
    gram_final_kernel<<<grid_for(T), kBlock, 0, s>>>(part.get(), blocks, T, out.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma gram");
    return out.to_host(s);
}

void sigma_spmv(const DevCsr<double>& A, const double* X, int W, double* Y, cudaStream_t s) {
    spmv_cols_kernel<<<grid_for(static_cast<std::int64_t>(A.n) * W), kBlock, 0, s>>>(A.ptr.get(), A.col.get(), A.val.get(),
                                                                                    A.n, W, X, Y); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma spmv");
}

void sigma_pack(const double* C, int n, int P, int K, const SigmaColumns& cm, int W, double* Bw, cudaStream_t s) {
    if (W < 1 || W > 16 || cm.count < 1 || cm.count > W) fail(kEInval, "sigma pack: 1 <= count <= W <= 16");
    pack_columns_kernel<<<grid_for(static_cast<std::int64_t>(n) * W), kBlock, 0, s>>>(C, n, P, K, cm, W, Bw); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma pack");
}

void sigma_unpack(const double* Xw, int n, int P, int K, const SigmaColumns& cm, int W, double* S, cudaStream_t s) {
    if (W < 1 || W > 16 || cm.count < 1 || cm.count > W) fail(kEInval, "sigma unpack: 1 <= count <= W <= 16");
    unpack_columns_kernel<<<grid_for(static_cast<std::int64_t>(n) * W), kBlock, 0, s>>>(Xw, n, P, K, cm, W, S); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma unpack");
}

void sigma_guess(const double* x_nom, const double* S, int n, int P, int K, int k, const SigmaDraw& y, double* X0,
                 cudaStream_t s) {
    guess_kernel<<<grid_for(static_cast<std::int64_t>(n) * K), kBlock, 0, s>>>(x_nom, S, n, P, K, k, y, X0); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma guess");
}

namespace {

// Eigen-decomposition of a symmetric m x m matrix (row-major, overwritten by its eigenvalues on the
// diagonal) by cyclic Jacobi rotations; V receives the eigenvectors as columns. The rotation angle
// is chosen as in Golub & Van Loan, Matrix Computations, sec. 8.5 (the smaller root of
// t^2 + 2 theta t - 1 = 0).
void symmetric_jacobi(int m, std::vector<double>& A, std::vector<double>& V) {
    V.assign(static_cast<std::size_t>(m) * m, 0.0);
    for (int i = 0; i < m; ++i) V[i * m + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int p = 0; p < m; ++p)
            for (int q = 0; q < m; ++q) (p == q ? diag : off) += A[p * m + q] * A[p * m + q];
        if (off <= 1e-32 * diag || off == 0.0) return;
        for (int p = 0; p < m - 1; ++p) {
            for (int q = p + 1; q < m; ++q) {
                const double apq = A[p * m + q];
                if (apq == 0.0) continue;
                const double theta = (A[q * m + q] - A[p * m + p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < m; ++r) {  // columns p, q
                    const double arp = A[r * m + p], arq = A[r * m + q];
                    A[r * m + p] = c * arp - s * arq;
                    A[r * m + q] = s * arp + c * arq;
                }
                for (int r = 0; r < m; ++r) {  // rows p, q
                    const double apr = A[p * m + r], aqr = A[q * m + r];
                    A[p * m + r] = c * apr - s * aqr;
                    A[q * m + r] = s * apr + c * aqr;
                }
                for (int r = 0; r < m; ++r) {
                    const double vrp = V[r * m + p], vrq = V[r * m + q];
                    V[r * m + p] = c * vrp - s * vrq;
                    V[r * m + q] = s * vrp + c * vrq;
                }
            }
        }
    }
}

}  // namespace

int sigma_coefficients(int P, const double* gram, const double* proj, const int* active, double rtol, double* Z) {
    for (int i = 0; i < P * P; ++i) Z[i] = 0.0;
    std::vector<int> act;
    for (int a = 0; a < P; ++a)
        if (active[a] && gram[a * P + a] > 0.0) act.push_back(a);
    const int m = static_cast<int>(act.size());
    if (m == 0) return 0;
    // Jacobi scaling first, so a tissue whose sensitivity is small but independent keeps its
    // direction; then the pseudo-inverse of the scaled Gram over the eigenvalues above rtol.
    std::vector<double> d(m), A(static_cast<std::size_t>(m) * m), V;
    for (int u = 0; u < m; ++u) d[u] = std::sqrt(gram[act[u] * P + act[u]]);
    for (int u = 0; u < m; ++u)
        for (int v = 0; v < m; ++v)
            A[u * m + v] = 0.5 * (gram[act[u] * P + act[v]] + gram[act[v] * P + act[u]]) / (d[u] * d[v]);
    symmetric_jacobi(m, A, V);
    double lmax = 0.0;
    for (int u = 0; u < m; ++u) lmax = std::max(lmax, A[u * m + u]);
    std::vector<double> pinv(static_cast<std::size_t>(m) * m, 0.0);
    int rank = 0;
    for (int e = 0; e < m; ++e) {
        const double lam = A[e * m + e];
        if (!(lam > rtol * lmax)) continue;
        ++rank;
        for (int u = 0; u < m; ++u)
            for (int v = 0; v < m; ++v) pinv[u * m + v] += V[u * m + e] * V[v * m + e] / lam;
    }
    // Z[a][t] = sum_b G+[a][b] proj[b][t], G+ = D^-1 pinv D^-1.
    for (int u = 0; u < m; ++u)
        for (int t = 0; t < P; ++t) {
            double z = 0.0;
            for (int v = 0; v < m; ++v) z += pinv[u * m + v] / (d[u] * d[v]) * proj[act[v] * P + t];
            Z[act[u] * P + t] = z;
        }
    return rank;
}

double sigma_relative_difference(const double* a, const double* b, long n, cudaStream_t s) {
    constexpr int blocks = 296;
    DevArray<double> part(2 * blocks);
    diff_norms_kernel<<<blocks, kBlock, 0, s>>>(a, b, n, part.get()); count_launch();
    CUNIBS_LAUNCH_CHECK("sigma difference");
    const std::vector<double> h = part.to_host(s);
    double d2 = 0.0, b2 = 0.0;
    for (int i = 0; i < blocks; ++i) {
        d2 += h[2 * i];
        b2 += h[2 * i + 1];
    }
    return b2 > 0.0 ? std::sqrt(d2 / b2) : std::sqrt(d2);
}

}  // namespace cunibs
