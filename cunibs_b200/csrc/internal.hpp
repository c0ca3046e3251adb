// Internal declarations shared by the cunibs_b200 translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace cunibs {

// Solver precision modes.
enum Precision : int {
    kPlainFp64 = 0,   // FP64 PCG over an FP64 V-cycle: the plain method
    kMixed = 1,       // FP32 PCG + FP32 V-cycle inside FP64 iterative refinement
    kFp64CgFp32Mg = 2 // FP64 PCG over an FP32 V-cycle (the reference's own split)
};

struct Params {
    int min_coarse_rows = 128;
    int max_levels = 50;
    int agg_rounds = 2;
    int cheby_degree = 2;
    double cheby_lower_ratio = 12.0;
    double tolerance = 1e-6;
    int max_iters = 2000;
    int precision = kFp64CgFp32Mg;
    double inner_reduction = 1e-4;  // deepest residual reduction asked of one inner FP32 solve
    int inner_max_iters = 60;
    int iters_per_sync = 4;         // PCG iterations launched between host convergence checks
    int dense_max_rows = 12288;     // the V-cycle ends in an exact dense solve at the first level
                                    // below the finest with at most this many rows (0: at the coarsest)
};

struct Cheby {
    int degree = 2;
    double alpha0 = 0.0;
    double c_cur[8] = {};
    double c_prev[8] = {};
    double alpha[8] = {};
};

Cheby make_cheby(int degree, double lower_ratio);

// One level of the smoothed-aggregation hierarchy. FP64 values are the built operator; the FP32
// copies (rounded once) are what the mixed-precision V-cycle streams.
struct Level {
    int n = 0;
    int n_coarse = 0;
    DevCsr<double> a;
    DevArray<float> a32;
    DevArray<double> dinv;
    DevArray<float> dinv32;
    DevArray<int> agg;
    DevCsr<double> p;
    DevArray<float> p32;
    DevCsr<double> r;
    DevArray<float> r32;
    // Threads per row of the V-cycle kernels on A, P and R, from each operator's shape.
    int tpr_a = 1, tpr_p = 1, tpr_r = 1;
};

// Sub-lanes per row for an SpMV-shaped kernel over n_rows rows and nnz entries: one while the rows
// alone fill the GPU, otherwise enough that each walks about sixteen entries (a power of two up to 32).
int choose_tpr(int n_rows, long nnz);

// Row length (entries) of a dense inverse of n rows: rows start on 32-byte boundaries in FP64 and
// 16-byte boundaries in FP32, padded with zeros past column n.
inline int dense_ld(int n) { return (n + 3) / 4 * 4; }

struct Hierarchy {
    std::vector<Level> levels;
    DevCsr<double> coarse;
    int nc = 0;
    DevArray<double> coarse_inv;   // dense (nc, dense_ld(nc)), FP64
    DevArray<float> coarse_inv32;
    // Where the V-cycle stops: it smooths levels [0, vcycle_levels) and solves the operator below
    // them exactly with the dense inverse bottom_inv (bottom_n rows): levels[vcycle_levels].a, or
    // the coarsest operator when vcycle_levels == levels.size() (then bottom_inv is coarse_inv).
    int vcycle_levels = 0;
    int bottom_n = 0;
    DevArray<double> level_inv;    // dense inverse of levels[vcycle_levels].a when the V-cycle stops early
                                   // (bottom_n, dense_ld(bottom_n))
    DevArray<float> level_inv32;
    std::vector<int> sizes;
    Cheby cheby;
};

// Per-subject device state, laid out along the Morton curve.
struct Mesh {
    int n_nodes = 0;
    int n_tets = 0;
    int n_skin = 0;
    DevArray<double> nodes;     // (N,3) mm
    DevArray<int> tets;         // (M,4)
    DevArray<int> tags;         // (M)
    DevArray<int> skin;         // (S,3)
    DevArray<int> node_perm;    // sorted position -> input node
    DevArray<int> tet_perm;     // sorted position -> input tet
    DevArray<double> g;         // (M,4,3) FP64, 1/m
    DevArray<float> g32;        // (M,4,3)
    DevArray<double> vols;      // (M) m^3
    DevArray<float> vols32;
    DevArray<double> cond;      // (M) S/m
    DevArray<int> cond_bad;     // (1) elements whose tag the last conductivity table left undefined
    DevArray<float> neg_vc32;   // -(vol*sigma) in FP32
    DevArray<double> bary;      // (M,3) mm
    DevArray<int> n2c_ptr;      // (N+1)
    DevArray<int> n2c_idx;      // (4M) corner ids
    DevArray<double> skin_normals;  // (S,3)
    // Stiffness pattern and the element-contribution map that assembles it.
    DevArray<int> k_ptr;        // (N+1)
    DevArray<int> k_col;        // (nnz)
    DevArray<int> contrib_ptr;  // (nnz+1) into contrib_idx
    DevArray<int> contrib_idx;  // (16M) e*16 + i*4 + j, ascending e within each entry
    DevArray<double> k_val;     // (nnz) FP64
    long k_nnz = 0;
    // Right-hand side weights per stiffness entry (i, j): w_ij = sum over the elements e holding both
    // of 1/4 neg_vc32[e] g32[e, i] (3 components, FP32 from an FP64 sum in contribution order), so the
    // block right-hand side is b_i = sum_j w_ij . dA/dt_j from the nodal field. Built on first use,
    // stale (rhs_w_ok false) once the element conductivities change.
    DevArray<float> rhs_w;
    bool rhs_w_ok = false;
    int ground = 0;
    // Gray-matter slice (tag 2): element index, FP32 volumes, barycentres.
    DevArray<int> gm_index;
    int n_gm = 0;
    // Placement scratch: per-segment nearest-triangle partials (grown on demand; a context is used
    // by one thread at a time).
    mutable DevArray<double> place_d;
    mutable DevArray<int> place_i;
};

// Setup stages (setup_mesh.cu).
void build_mesh(Mesh& m, const double* nodes_mm, int n_nodes, const int* tets, const int* tags, int n_tets,
                const int* skin, int n_skin, cudaStream_t s);
void assemble_stiffness(Mesh& m, const double* sigma_by_tag /* 11 entries or null */, cudaStream_t s);
// Per-element conductivity and right-hand side weights of a conductivity table (11 entries).
// validate: fail when the table leaves a tag of the mesh undefined (a host synchronisation); a
// caller whose table has passed that check once for the same tags may skip it.
void set_element_conductivity(Mesh& m, const double* sigma_by_tag, cudaStream_t s, bool validate = true);
// Grounded stiffness values of n_tables conductivity tables (11 entries each, zeros allowed) on the
// grounded pattern, out (n_tables, pattern.nnz), without touching the mesh's own values; the
// operator's linearity in sigma makes a table with one unit entry give that tissue's share of it.
void assemble_reduced_values(const Mesh& m, const double* tables, int n_tables, const DevCsr<double>& pattern,
                             double* out, cudaStream_t s);
void reduce_grounded(const Mesh& m, DevCsr<double>& out, cudaStream_t s);
// The grounded values of the mesh's stiffness on a grounded pattern already built (out: pattern.nnz).
void reduce_grounded_values(const Mesh& m, const DevCsr<double>& pattern, double* out, cudaStream_t s);

// Hierarchy (setup_amg.cu).
int select_size4(int n, long nnz, const int* rp, const int* ci, const float* va, int* agg, cudaStream_t s);
void build_hierarchy(Hierarchy& h, DevCsr<double>& a0, const Params& p, cudaStream_t s);
// The finest level's l1 smoother weights and FP32 copies, after its FP64 values were rewritten in
// place (queued on s, no synchronisation).
void refresh_finest_derived(Hierarchy& h, cudaStream_t s);
void spgemm(const DevCsr<double>& A, const DevCsr<double>& B, DevCsr<double>& C, cudaStream_t s);
void transpose(const DevCsr<double>& A, DevCsr<double>& T, cudaStream_t s);
void l1_dinv(const DevCsr<double>& a, DevArray<double>& dinv, cudaStream_t s);

// Solver (solve.cu).
struct SolveStats {
    std::vector<int> col_iters;
    std::vector<double> col_rel;
    std::vector<double> col_init_rel;  // with a warm start: the kept guess's relative residual, 1 if dropped
    int iterations = 0;
    int outer_steps = 0;
};
class Solver;
struct SolverDeleter {
    void operator()(Solver* s) const;
};
using SolverPtr = std::unique_ptr<Solver, SolverDeleter>;
SolverPtr make_solver(const Hierarchy& h, const Params& p);
void solver_solve(Solver& sv, const double* B, double* X, int k, int k_pad, const Params& p, cudaStream_t s,
                  SolveStats& stats, const double* X0 = nullptr);
void solver_vcycle(Solver& sv, const double* r, double* z, int k, bool fp32, cudaStream_t s);
// The widest block the solver's workspace holds now (solving wider grows it: every workspace
// array is reallocated and the captured loop graphs are dropped).
int solver_width_capacity(const Solver& sv);

// Coil and right-hand side (coil.cu).
void place_transforms(const Mesh& m, const double* centers, const double* handles, const double* dists, int k,
                      double* transforms_dev, int* degenerate_dev, cudaStream_t s);
std::size_t packed_dipole_bytes();
// Rotates the coil's dipoles into each placement's head frame: (k, n_dip) packed records.
void prep_dipoles(const double* pos, const double* mom, int n_dip, const double* transforms_dev, int k, void* out,
                  cudaStream_t s);
// max_blocks > 0 bounds the grid (blocks then walk the (node tile, placement) items), leaving SM
// room for kernels of other streams; the result does not depend on it.
void dadt_nodes(const Mesh& m, const float* dip_packed, int n_dip, const double* transforms_dev, int k, double didt,
                float* out /* (k, N, 3) */, cudaStream_t s, int max_blocks = 0);
// Coils whose moments all point along the coil's own z axis (every figure-8 and circular coil
// model) take a cheaper path evaluated in each placement's coil frame. general_flag_dev receives 0
// when the coil qualifies, 1 when some moment has an in-plane component; zpacked has room for
// packed_zdipole_bytes() * n_dip.
std::size_t packed_zdipole_bytes();
void prep_zdipoles(const double* pos, const double* mom, int n_dip, void* zpacked, int* general_flag_dev,
                   cudaStream_t s);
void dadt_nodes_zcoil(const Mesh& m, const void* zpacked, int n_dip, const double* transforms_dev, int k, double didt,
                      float* out /* (k, N, 3) */, cudaStream_t s, int max_blocks = 0);
void dadt_elements(const Mesh& m, const float* dadt_nodes, int k, float* dadt_elm /* (k, M, 3) */, cudaStream_t s);
// The general-moment dA/dt on raw device node coordinates (no Mesh), packed records from prep_dipoles.
void dadt_nodes_raw(const double* nodes_mm, int n_nodes, const float* dip_packed, int n_dip,
                    const double* transforms_dev, int k, double didt, float* out, cudaStream_t s);
// n_sets (1..3) source sets at common positions, records set * n_dip + j of prep_dipoles all made
// with the one transform transform_dev; out (n_sets, n_nodes, 3). Set d's field is bitwise
// dadt_nodes_raw's for that set alone; each pair's geometry is formed once for all sets.
// scratch holds the source chunks' partial fields when the targets alone do not fill the GPU (grown
// on demand and kept by the caller, so repeated calls allocate nothing).
void dadt_nodes_shared(const double* nodes_mm, int n_nodes, const float* dip_packed, int n_dip,
                       const double* transform_dev, int n_sets, double didt, float* out, cudaStream_t s,
                       DevArray<float>& scratch);
// The two direct sums on raw node coordinates with an explicit FP32 scale (1: the bare dipole sum).
void dadt_zcoil_raw(const double* nodes_mm, int n_nodes, const void* zpacked, int n_dip, const double* transforms_dev,
                    int k, float scale, float* out, cudaStream_t s, int max_blocks = 0);
void dadt_general_raw(const double* nodes_mm, int n_nodes, const float* dip_packed, int n_dip,
                      const double* transforms_dev, int k, float scale, float* out, cudaStream_t s);

// --- coil field table (coil_table.cu) ----------------------------------------------------------
// The coil's bare dipole sum sampled once per coil on a grid in its own frame, in layers below the
// deepest dipole whose depths grow geometrically, z_j = z0 (1 + step)^(j - 1), each layer a square
// grid of spacing step * z_j. A node deeper than z0 inside the grid takes the tricubic Lagrange
// interpolant of the table (four layers, four rows, four points); the others, the nodes near the coil,
// take the direct sum.
struct CoilTableLayer {
    float inv_h;       // grid lines at x = (i - half) / inv_h and y = (j - half) / inv_h, metres
    float z;           // depth below the deepest dipole, metres
    int half;          // index of the line through x = 0 (and y = 0)
    int n;             // points per row, rows per layer
    long long offset;  // first point of the layer in the table
};

constexpr int kCoilTableMaxLayers = 256;
// Tables above this many points (a mesh far larger than a head, or a tiny near depth) are not built.
constexpr long long kCoilTableMaxPoints = 16LL << 20;

struct CoilTable {
    bool built = false;   // built for the coil in pos/mom and the parameters below
    bool valid = false;   // and its check passed: the dA/dt path may read it
    int nc = 0;           // components per point: 2 (moments along the coil's z: A_z = 0) or 3
    int n_dip = 0;
    int n_layers = 0;
    long long points = 0;
    float z_top = 0.f;    // the deepest dipole's z in the coil frame (z points into the head), metres
    float z0 = 0.f, inv_z0 = 0.f, inv_log_step = 0.f;
    double near_m = 0.0, step = 0.0, lateral_m = 0.0;
    double check_rel = 0.0;  // relative L2 error of the interpolant at the check points
    int builds = 0;
    DevArray<CoilTableLayer> layers;
    DevArray<float> data;       // per point: 2 floats (nc 2) or 4 (nc 3, the fourth zero)
    DevArray<double> pos, mom;  // the coil it was built for
};

// Sets bit 1 of *flag when pos/mom differ from the table's coil (same n_dip).
void coil_compare(const double* pos, const double* mom, int n_dip, const CoilTable& tb, int* flag, cudaStream_t s);
// Builds (and checks) the table for the coil on the device in pos/mom; lateral_m is the half-width
// of the layers, depth_m the deepest depth sampled. Synchronises s. Leaves tb.valid false when the
// check fails or the table would exceed max_points.
void build_coil_table(CoilTable& tb, const double* pos, const double* mom, int n_dip, bool zcoil, const void* zpacked,
                      double near_m, double step, double lateral_m, double depth_m, long long max_points,
                      cudaStream_t s);
// dA/dt of every node the table covers, for k placements; the others are appended to their
// placement's list near_list[p * N + ...], counted in near_cnt[p] (zeroed here).
void dadt_table(const Mesh& m, const CoilTable& tb, const double* transforms_dev, int k, double didt, float* out,
                int* near_list, int* near_cnt, cudaStream_t s, int max_blocks = 0);
// The direct sum for the listed nodes: eight warps per block split the dipoles, their partial sums
// added in warp order (the result does not depend on the list's order or the grid).
void dadt_near_zcoil(const Mesh& m, const void* zpacked, int n_dip, const double* transforms_dev, int k, double didt,
                     float* out, const int* near_list, const int* near_cnt, cudaStream_t s, int max_blocks = 0);
void dadt_near_general(const Mesh& m, const float* dip_packed, int n_dip, const double* transforms_dev, int k,
                       double didt, float* out, const int* near_list, const int* near_cnt, cudaStream_t s,
                       int max_blocks = 0);

// Records the calling thread's message for cunibs_last_error.
void set_last_error(const std::string& message);
// neg_vc: the per-element weights -(vol * sigma) in FP32 (null: the mesh's own).
void rhs_block(const Mesh& m, const float* dadt_elm, int k, int k_pad, double* b_red /* (N-1, k_pad) */,
               cudaStream_t s, const float* neg_vc = nullptr);
// The same right-hand side from the nodal dA/dt (k, N, 3) through the mesh's rhs_w (built here when
// stale): equal to rhs_block of the element average up to rounding, with no element pass.
void rhs_block_nodes(Mesh& m, const float* dadt_nodes, int k, int k_pad, double* b_red, cudaStream_t s);

// Post-processing (post.cu).
void reconstruct_block(const Mesh& m, const double* x_red /* (N-1,k_pad) */, int k, int k_pad,
                       const float* dadt_elm, float* E /* (k,M,3) or null */, float* magnE /* (k,M) */,
                       cudaStream_t s);
void scatter_potential(const Mesh& m, const double* x_red, int k, int k_pad, double* v /* (k,N) */, cudaStream_t s);
constexpr int kSummaryLen = 16;
// Workspace of the gray-matter summary (post.cu): fixed-point volumes of the mesh's gray matter,
// the radix select's histograms, ranges and candidates, and the statistics' partial sums.
struct SummaryWork {
    int wfix_n = -1;
    DevArray<long long> wfix;
    DevArray<unsigned char> sel_mesh, sel_state, edges;
    DevArray<float> gv;
    DevArray<unsigned> hcnt;
    DevArray<unsigned long long> hw, cand;
    DevArray<int> cand_n, ticket;
    bool hist_clear = false;
    int hist_k = 0;
    DevArray<double> qval, part;
    DevArray<long long> foc;
    DevArray<int> part_i;
};
void gm_summary(const Mesh& m, const float* magnE, int k, double* summary_dev /* (k,16) */, SummaryWork& w,
                cudaStream_t s);

// BF16 tensor-core GEMM (gemm_tc.cu): C[M,N] = A[M,K] . B[N,K]^T, FP32 accumulation, fused tail:
//   z = acc (+ bias[col]) (* silu'(gate[row, col]));  out32 = z;  h = act ? silu(z) : z;
//   out16 = bf16(h) row-major;  out16t = bf16(h) transposed ([N, ld_t]).
struct GemmEpilogue {
    const float* bias = nullptr;
    const float* gate = nullptr;
    int ld_gate = 0;
    int act = 0;
    float* out32 = nullptr;
    __nv_bfloat16* out16 = nullptr;
    int ld_out = 0;
    __nv_bfloat16* out16t = nullptr;
    int ld_t = 0;
    int* error = nullptr;  // set to 1 when a bounded wait expired (NULL: the device's status word)
    // Filled by gemm_bf16 from the library's wait settings.
    long long wait_polls = 0;
    unsigned long long wait_ns = 0;
    int withhold_loads = 0;
};
struct GemmProblem {
    const __nv_bfloat16* a = nullptr;  // [M, lda], K-major
    int lda = 0;
    const __nv_bfloat16* b = nullptr;  // [N, ldb], K-major
    int ldb = 0;
    int M = 0, N = 0, K = 0;
    GemmEpilogue ep;
};
void gemm_bf16(const GemmProblem& p, cudaStream_t s);
// Whether a GEMM launched without an error flag of its own had a wait expire on the current device
// since the last call (synchronises `s`, then clears the word).
bool gemm_status(cudaStream_t s);
// Wait bounds of later GEMM launches (<= 0: the defaults); withhold_loads makes the producer issue
// no loads, for tests of the timeout path.
void gemm_set_waits(long long polls, unsigned long long limit_ns, int withhold_loads);

// Learned warm start (warmstart.cu): an MLP from coil pose to the coefficients of a reduced basis of
// the grounded potential, prolongated through the basis as the PCG initial guess.
struct WarmStart {
    int depth = 0;     // hidden layers
    int hidden = 0;
    int n_out = 0;     // basis size
    int n_out_pad = 0;
    int n_red = 0;     // rows of the basis (grounded system size)
    std::vector<DevArray<__nv_bfloat16>> w16;  // per layer [out_pad, in_pad]
    std::vector<DevArray<float>> bias;         // per layer [out_pad]
    DevArray<float> in_mean, in_std, out_mean, out_std;
    DevArray<__nv_bfloat16> basis;             // [n_red, n_out_pad]
    // Inference workspace.
    DevArray<__nv_bfloat16> x16, h16a, h16b, c16;
    DevArray<float> pred, x0f;
    DevArray<double> partials, norms;
    DevArray<int> error;
};
constexpr int kWarmInPad = 64;  // pose features (6) padded to one BF16 swizzle row
// Queues the network's guess for the k placements whose coil transforms are T_dev (k, 16) into X0
// (n_red, K); nothing waits on the host. The solver applies the per-column zero-guess fallback
// (SolveStats::col_init_rel). warm_start_check (after the solve) raises if a GEMM's bounded wait
// expired.
// Guess sources (cunibs_solve_opts.warm_start): the network's coefficients from the coil pose, or
// the Galerkin projection of the block's right-hand sides B (n_red, K) onto the same basis.
enum GuessMode : int { kGuessNone = 0, kGuessNetwork = 1, kGuessProjection = 2 };
void warm_start_guess(WarmStart& ws, const double* T_dev, const double* B, int k, int K, double* X0, int mode,
                      cudaStream_t s);
void warm_start_check(WarmStart& ws, cudaStream_t s);
void pose_features(const double* T_dev, int k, const float* mean, const float* std, __nv_bfloat16* x16, int ld,
                   cudaStream_t s);

// Field recovery (recovery.cu). Modes match CUNIBS_RECOVERY_*.
enum RecoveryMode : int { kRecRaw = 0, kRecSprGlobal = 1, kRecSprTissue = 2, kRecHarmonic = 3 };

struct RecoveryOp {
    int mode = kRecRaw;
    int n_slots = 0;
    std::int64_t nnz = 0;
    // SPR rows: corner ids per slot (spr_global uses the mesh's node-to-corner CSR instead).
    DevArray<int> ptr, idx;
    DevArray<float> w;          // SPR: one weight per corner entry
    // Harmonic rows (ptr is then the patch CSR): patch node per entry and {w_x, w_y, w_z, node}.
    DevArray<int> pidx;
    DevArray<float4> wq;
    DevArray<int> slot_of_corner;  // (4M); spr_global samples through the mesh's own tets
    DevArray<int> slot_node, slot_tag, status, is_boundary;
    int n_fallback = 0, n_undetermined = 0;
};
void build_recovery(const Mesh& m, RecoveryOp& op, int mode, cudaStream_t s);
const int* recovery_slot_of_corner(const Mesh& m, const RecoveryOp& op);
// Recovered E on slots (k, n_slots, 3) and at the barycentres: E (k,M,3) or null, magn (k,M).
// Harmonic reads the solver block x_red (N-1, K) and dadt_nodes (k,N,3); SPR reads e_elem (k,M,3).
void apply_recovery(const Mesh& m, const RecoveryOp& op, const double* x_red, int K, const float* dadt_nodes,
                    const float* e_elem, int k, float* e_slots, float* E, float* magn, cudaStream_t s);

// Conductivity Monte Carlo (sigma.cu): per-draw operator values and the sensitivity-subspace guess.
constexpr int kSigmaMaxTags = 10;
struct SigmaWeights {
    double w[kSigmaMaxTags];  // conductivity of each perturbed tissue, in study order
};
struct SigmaSlots {
    int slot[11];  // study position of each tissue tag, -1 for a tag that is not perturbed
};
struct SigmaColumns {
    int a[16], j[16];  // (tissue position, placement) of each lane of a solve block (at most 16 wide)
    int count;
};
struct SigmaDraw {
    double y[kSigmaMaxTags * 16];  // subspace coefficients, y[a * 16 + j]
};
// Values of the finest operator for one draw: comp[0] + sum_t w_t comp[1 + t] (comp (1 + n_tags, nnz)).
void sigma_combine(const double* comp, int n_tags, long nnz, const SigmaWeights& w, double* out, cudaStream_t s);
// -vol of the elements of each table entry's tissue, zero elsewhere: out (n_tables, n_tets) FP32,
// tables (n_tables, 11) of per-tag weights (the right-hand side's per-element weights of a
// conductivity table whose entries are those weights).
void sigma_element_weights(const Mesh& m, const double* tables_dev, int n_tables, float* out, cudaStream_t s);
// Sensitivity right-hand sides c_t of the nominal potential x_red (n_red, K): c_out (n_red, P, K).
void sigma_sens_rhs(const Mesh& m, const double* x_red, const float* dadt_elm, int k, int K, const SigmaSlots& slots,
                    int P, double* c_out, cudaStream_t s);
// Per-placement Gram blocks of two (n, P, K) arrays, (K, P, P) on the host; depends on n, not on K.
std::vector<double> sigma_gram(const double* U, const double* V, long n, int P, int K, cudaStream_t s);
// Y (n, W) = A X (n, W) in FP64.
void sigma_spmv(const DevCsr<double>& A, const double* X, int W, double* Y, cudaStream_t s);
// A W-wide solve block (n, W) from the chosen columns of an (n, P, K) array, and back.
void sigma_pack(const double* C, int n, int P, int K, const SigmaColumns& cm, int W, double* Bw, cudaStream_t s);
void sigma_unpack(const double* Xw, int n, int P, int K, const SigmaColumns& cm, int W, double* S, cudaStream_t s);
// X0 (n, K) = x_nom + S y per placement.
void sigma_guess(const double* x_nom, const double* S, int n, int P, int K, int k, const SigmaDraw& y, double* X0,
                 cudaStream_t s);
// ||a - b|| / ||b|| over n entries (synchronises s).
double sigma_relative_difference(const double* a, const double* b, long n, cudaStream_t s);
// Host: the draw-coefficient map of one placement. gram (P, P) = S^T A S and proj (P, P) with
// proj[a][t] = s_a . c_t over the active positions; Z (P, P) with y = Z (sigma - sigma_nom) the
// A-Galerkin coefficients of the linearised residual. Returns the rank kept (eigenvalues of the
// Jacobi-scaled Gram above rtol times the largest).
int sigma_coefficients(int P, const double* gram, const double* proj, const int* active, double rtol, double* Z);

// Auxiliary dipole method (adm.cu): adjoint right-hand sides, nodal reciprocity weights and the
// evaluation of placements against a reciprocity field sampled on a grid.
constexpr int kAdmMaxDir = 3;
struct AdmDirections {
    double e[kAdmMaxDir][3];
    int n;
};
struct AdmGrid {
    double origin_mm[3];
    double spacing_mm[3];
    int shape[3];
};
// Adjoint right-hand sides (n_red, K) of the target weights alpha (per element, zero off target).
void adm_adjoint_rhs(const Mesh& m, const double* alpha, const AdmDirections& dirs, int K, double* c_red,
                     cudaStream_t s);
// Nodal weights W (n_dir, n_nodes, 3) from the adjoint potentials lam (n_red, K).
void adm_node_weights(const Mesh& m, const double* lam, int K, const double* alpha, const AdmDirections& dirs,
                      double* W, cudaStream_t s);
void adm_centred_nodes(const Mesh& m, const double* center_mm, double* out_m, cudaStream_t s);
void adm_grid_points(const AdmGrid& gr, double* out /* (n_grid, 3) mm */, cudaStream_t s);
// E (P, n_dir) from the sampled field Q (n_dir, n_grid, 3); bad[3] receives, per axis, the smallest
// flat sample index p * n_dip + j of a dipole off the grid (left untouched when none is).
void adm_evaluate(const float* Q, int n_dir, const AdmGrid& gr, const double* pos, const double* mom, int n_dip,
                  const double* T, int P, double didt, double* E, unsigned long long* bad, cudaStream_t s);
void adm_placed_dipoles(const double* pos, const double* mom, int n_dip, const double* T, int P, double* s_mm,
                        double* m_out, cudaStream_t s);
void adm_exact_reduce(const float* Qx, int n_dir, int P, int n_dip, const double* m_all, double didt, double* E,
                      cudaStream_t s);

}  // namespace cunibs
