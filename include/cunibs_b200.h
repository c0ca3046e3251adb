/* cunibs_b200 -- C ABI of the B200-native per-placement TMS field solve.
 *
 * The reference (cuNIBS 0.4.0) exposes this path through a nanobind module,
 * cunibs.solver._solver_ext (src/cunibs/solver/bindings.cpp:30-676), driven from Python by
 * fem/solve.py:690-746 (build_context) and fem/solve.py:865-979 (solve_placements_block). This
 * library replaces that boundary with plain C: opaque handles, pointers and sizes, int status codes.
 * Every entry point returns CUNIBS_OK (0) or an error code; cunibs_last_error() returns the message
 * of the calling thread's last failure.
 *
 * Arrays are C-contiguous. Unless an entry point says "device", pointers are host memory and the
 * call copies in and out itself; it returns after results are in the caller's buffers.
 * A context is not thread-safe; callers serialise use of one handle.
 */
#ifndef CUNIBS_B200_H
#define CUNIBS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference raises ValueError (invalid_argument) and RuntimeError
 * (bindings.cpp:52-56) and, for a missed tolerance, SolverConvergenceError (fem/solve.py:368-392). */
#define CUNIBS_OK 0
#define CUNIBS_EINVAL 1
#define CUNIBS_ENOMEM 2
#define CUNIBS_ECUDA 3
#define CUNIBS_ENOCONV 4
#define CUNIBS_ETIMEOUT 5
#define CUNIBS_EINTERNAL 6

/* Solver precision. */
#define CUNIBS_PREC_DEFAULT 0    /* per-call option: use the context's precision */
#define CUNIBS_PREC_PLAIN_FP64 1 /* FP64 PCG over an FP64 V-cycle */
#define CUNIBS_PREC_MIXED 2      /* FP32 PCG + FP32 V-cycle inside FP64 iterative refinement */
#define CUNIBS_PREC_SPLIT 3      /* FP64 PCG over an FP32 V-cycle (the default) */

/* Field recovery: how the reported E is derived from the solve (fem/recovery.py:74-113).
 * RAW is the per-tetrahedron field; SPR_GLOBAL a linear patch fit per node; SPR_TISSUE the same per
 * (node, tissue) slot; HARMONIC the potential fitted per (node, tissue) slot in harmonic
 * polynomials and differentiated, plus the exact nodal dA/dt (the reference's default). */
#define CUNIBS_RECOVERY_RAW 0
#define CUNIBS_RECOVERY_SPR_GLOBAL 1
#define CUNIBS_RECOVERY_SPR_TISSUE 2
#define CUNIBS_RECOVERY_HARMONIC 3

/* Summary layout, one row of CUNIBS_SUMMARY_LEN doubles per placement (metrics.py:28-37,209-243). */
#define CUNIBS_SUMMARY_PEAK 0       /* peak |E| in gray matter, V/m */
#define CUNIBS_SUMMARY_PEAK_LOC 1   /* 3 values: barycentre of the peak element, mm */
#define CUNIBS_SUMMARY_COG 4        /* 3 values: volume*|E| weighted centre of gravity, mm */
#define CUNIBS_SUMMARY_VOLUME 7     /* gray-matter volume, m^3 */
#define CUNIBS_SUMMARY_MEAN 8
#define CUNIBS_SUMMARY_STD 9
#define CUNIBS_SUMMARY_P50 10
#define CUNIBS_SUMMARY_P95 11
#define CUNIBS_SUMMARY_P99 12
#define CUNIBS_SUMMARY_P999 13
#define CUNIBS_SUMMARY_FOCALITY_50 14 /* volume with |E| >= 0.5 * p99.9, m^3 */
#define CUNIBS_SUMMARY_FOCALITY_75 15
#define CUNIBS_SUMMARY_LEN 16

typedef struct cunibs_context cunibs_context;

typedef struct {
    int device;               /* CUDA device ordinal */
    int min_coarse_rows;      /* AggregationParams.min_coarse_rows (fem/solve.py:146) = 128 */
    int max_levels;           /* AggregationParams.max_levels = 50 */
    int agg_rounds;           /* AggregationParams.rounds = 2 */
    int cheby_degree;         /* SmootherParams.degree (fem/solve.py:167) = 2 */
    double cheby_lower_ratio; /* SmootherParams.lower_ratio = 12 */
    double tolerance;         /* ||r||/||b|| stopping criterion; DEFAULT_TOLERANCE = 1e-6 (fem/solve.py:56) */
    int max_iters;            /* DEFAULT_MAX_ITERS = 2000 */
    int precision;            /* CUNIBS_PREC_* */
    double inner_reduction;   /* mixed: deepest residual reduction asked of one inner FP32 solve */
    int inner_max_iters;      /* mixed: iteration cap of each inner FP32 solve */
    int iters_per_sync;       /* PCG iterations launched between host convergence checks */
    int dense_max_rows;       /* the V-cycle ends in an exact dense solve at the first level below the
                                 finest with at most this many rows (default 12288, at most 16384;
                                 its dense inverse takes 12 bytes per entry); 0: at the coarsest
                                 level, as the reference's V-cycle does (vcycle.cu:420-663) */
} cunibs_params;

typedef struct {
    int n_nodes;
    int n_tets;
    int n_skin;
    int n_gray_matter;
    long long stiffness_nnz;
    int ground_node; /* in the context's (Morton) node order */
    int n_levels;    /* AMG levels above the dense coarse solve */
    int coarse_rows;
    int vcycle_levels; /* levels the V-cycle smooths; the level below them (or the coarsest) is solved
                          exactly (cunibs_params.dense_max_rows) */
    int bottom_rows;   /* rows of that exactly solved operator */
    int hierarchy_builds; /* AMG hierarchy builds over the context's life: 1 at create, +1 for each
                             conductivity re-setup that rebuilds it and for each rebuild before the
                             FP64 retry of a block that missed tolerance */
} cunibs_info;

/* Per-call options of a block solve. Zero-initialise for the context defaults. */
typedef struct {
    int block_width;   /* padded width; 0 = smallest of {1,2,4,8,16} >= k */
    int precision;     /* CUNIBS_PREC_DEFAULT or a CUNIBS_PREC_* override */
    double tolerance;  /* <= 0: context default */
    int max_iters;     /* <= 0: context default */
    int recovery;      /* CUNIBS_RECOVERY_*; 0 = raw. magnE, E and the summary describe this field */
    int warm_start;    /* 1: start PCG from the installed network's guess (cunibs_context_set_warmstart);
                          2: from the Galerkin projection of the right-hand sides onto that network's
                          basis (no network: the A-norm-best guess the basis spans) */
} cunibs_solve_opts;

/* Outputs of a block solve of k placements. Required: transforms, summary. Optional (NULL to
 * skip): iterations, relres, magnE (k, n_tets), E (k, n_tets, 3), v (k, n_nodes). All in the
 * context's node and element order (cunibs_context_mesh returns it). */
typedef struct {
    double* transforms; /* (k, 4, 4) coil-to-head affines, mm */
    double* summary;    /* (k, CUNIBS_SUMMARY_LEN) gray-matter metrics */
    int* iterations;    /* (k) PCG iterations at which each column met tolerance */
    double* relres;     /* (k) final relative residual per column */
    float* magnE;       /* (k, n_tets) */
    float* E;           /* (k, n_tets, 3) */
    double* v;          /* (k, n_nodes) potential, grounded node = 0 */
    int total_iterations; /* filled: iterations the block ran */
    int outer_steps;      /* filled: FP64 refinement steps (mixed) */
    float* E_slots;     /* (k, n_slots, 3) recovered field on its slots (NULL to skip; recovery only) */
    int* warm_used;     /* (k) 1 where the warm-start guess was kept (its residual was below ||b||) */
    double* init_relres;/* (k) relative residual of the initial guess (1 for the zero guess) */
} cunibs_block_out;

typedef struct {
    int mode;
    int n_slots;        /* nodes (SPR_GLOBAL) or (node, tissue) pairs */
    long long nnz;      /* operator entries: corners (SPR) or patch nodes (HARMONIC) */
    int n_fallback;     /* SPR: slots on the volume average; HARMONIC: slots below the harmonic rungs */
    int n_undetermined; /* HARMONIC: slots with no gradient (E = -dA/dt there) */
} cunibs_recovery_info;

int cunibs_version(void);
const char* cunibs_last_error(void);
int cunibs_params_default(cunibs_params* out);

/* Builds a subject's solver state (replaces build_context, fem/solve.py:690-746): Morton layout,
 * P1 gradients and volumes (rejecting zero or non-finite volumes), conductivity lookup (rejecting
 * unknown tags), stiffness assembly, grounding of the lowest-z node, the SA-AMG hierarchy, skin
 * normals. tet_tags use the tissue table 1..10; skin_tris are the scalp triangles (tag 1005). */
int cunibs_context_create(const double* nodes_mm, int n_nodes, const int* tet_nodes, const int* tet_tags,
                          int n_tets, const int* skin_tris, int n_skin, const cunibs_params* params,
                          cunibs_context** out);
int cunibs_context_destroy(cunibs_context* ctx);
int cunibs_context_info(const cunibs_context* ctx, cunibs_info* out);

/* The context's Morton-ordered mesh; any pointer may be NULL. node_perm[i] / tet_perm[e] give the
 * input index of node i / tet e (fem/solve.py:645-662). */
int cunibs_context_mesh(const cunibs_context* ctx, double* nodes_mm, int* tet_nodes, int* tet_tags, int* skin_tris,
                        int* node_perm, int* tet_perm);

/* Hierarchy row counts, finest first then the dense coarse level (n_levels + 1 entries). */
int cunibs_context_levels(const cunibs_context* ctx, int* sizes, int cap);

/* Solves k placements as one block (replaces solve_placements_block, fem/solve.py:865-979, with
 * Subject._reduce_chunk's summary, simulation.py:330-376). dip_pos_m/dip_moment: (n_dip, 3) in the
 * coil frame. centers_mm/handles_mm: (k, 3); dists_mm: (k). A handle on the scalp normal is
 * CUNIBS_EINVAL; a column that misses tolerance after one FP64 retry is CUNIBS_ENOCONV with the
 * column in the message. */
int cunibs_solve_block(cunibs_context* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
                       const double* centers_mm, const double* handles_mm, const double* dists_mm, int k, double didt,
                       const cunibs_solve_opts* opts, cunibs_block_out* out);

/* Same, with every input and output pointer in device memory of the context's GPU (outputs are
 * written there; nothing is copied to the host). Returns after the work is complete. */
int cunibs_solve_block_device(cunibs_context* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
                              const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
                              double didt, const cunibs_solve_opts* opts, cunibs_block_out* out);

/* Two-stage form of the block solve, for a sequence of blocks (the block loop of
 * Subject.iter_simulate, simulation.py:473-546). A submit prepares a block (coil placement, dA/dt,
 * right-hand side) on the context's preparation stream and returns a ticket without waiting for
 * the work; the finish of that ticket solves the block and writes its outputs exactly as the
 * one-call entry does (same out fields, same host or device placement). At most two blocks are
 * submitted and not finished; a block submitted while another waits to be finished is prepared
 * beside that block's solve on the same GPU (its dA/dt kernel then takes a bounded grid,
 * cunibs_context_set_overlap). Host inputs are copied at submit; device inputs must stay valid
 * until their block is finished. Errors of a block (a degenerate placement, no convergence) are
 * returned by its finish call; the block is dropped either way. Results are bitwise those of the
 * one-call entries, which may be called while one block is submitted. */
int cunibs_submit_block(cunibs_context* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
                        const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
                        double didt, const cunibs_solve_opts* opts, long long* ticket);
int cunibs_finish_block(cunibs_context* ctx, long long ticket, cunibs_block_out* out);
int cunibs_submit_block_device(cunibs_context* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
                               const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
                               double didt, const cunibs_solve_opts* opts, long long* ticket);
int cunibs_finish_block_device(cunibs_context* ctx, long long ticket, cunibs_block_out* out);
/* Drops a submitted block without solving it (a consumer that stops early). */
int cunibs_cancel_block(cunibs_context* ctx, long long ticket);
/* Number of submitted blocks not yet finished (0, 1 or 2). */
int cunibs_context_pending(const cunibs_context* ctx, int* n);
/* Blocks per SM the dA/dt kernel takes while another block's solve may run beside it (default 2). */
int cunibs_context_set_overlap(cunibs_context* ctx, int blocks_per_sm);
/* How the block entries form the coil dA/dt at the nodes (fem/placement.py:279-317 sums every
 * dipole at every node, solver/coil/dadt.cu:27-113).
 *   mode 1 (default): a table of the coil's field, sampled once per coil in its own frame in layers
 *     below the coil whose spacing grows with depth (`step` times the depth, default 0.035), gives
 *     every node deeper than near_mm (default 15) below the coil by tricubic interpolation; nodes
 *     nearer the coil keep the dipole sum. The table is rebuilt when the coil changes, and checked
 *     when built against the dipole sum (relative L2 error at most 2e-6 at cell centres, else the
 *     dipole sum is used everywhere); its interpolation error is about 1e-7 relative at step 0.035.
 *   mode 0: the dipole sum at every node.
 * cunibs_dadt, cunibs_dadt_noalloc and the auxiliary dipole method always sum every dipole. */
int cunibs_context_set_coil_table(cunibs_context* ctx, int mode, double near_mm, double step);
/* out[8]: mode, table in use (0/1), table points, layers, check error (relative L2), builds, nodes
 * given the dipole sum in the last finished block (-1 when it did not read the table), nodes x
 * placements of that block. */
int cunibs_context_coil_table_info(const cunibs_context* ctx, double* out);
/* Diagnostics of the last cunibs_sigma_begin on this context (no counterpart in the reference):
 * out[8] = host wall-clock milliseconds from the call's start to the end of each phase: 0 nominal
 * assembly and kept hierarchy, 1 operator components, 2 the block's coil field, 3 its nominal solve,
 * 4 per-tissue right-hand sides, 5 sensitivity right-hand sides, 6 sensitivity solves, 7 the guess
 * coefficients. */
int cunibs_context_phase_times(const cunibs_context* ctx, double* out);

/* Re-assembles the stiffness with a new conductivity per tissue tag (sigma_by_tag[0..10], S/m;
 * index = tag) and rebuilds the AMG hierarchy: the per-sample step of a conductivity Monte Carlo
 * (uq/conductivity/run.py:324-361). */
int cunibs_context_set_conductivity(cunibs_context* ctx, const double* sigma_by_tag);

/* The cheap per-sample step: re-assembles the stiffness (and the right-hand side weights) for new
 * conductivities and refreshes the finest AMG level's values and smoother weights, but keeps the
 * coarser levels built for the earlier conductivities. PCG still solves the new operator to the
 * same tolerance; the preconditioner is only slightly off. This is the reference's Monte Carlo
 * scheme, which swaps the operator's values per draw and keeps the V-cycle built at the nominal
 * conductivities (uq/conductivity/assembly.py:1-7,53-70; run.py:203-387). A draw that then misses
 * the tolerance is the caller's cue for cunibs_context_set_conductivity. */
int cunibs_context_set_conductivity_keep_coarse(cunibs_context* ctx, const double* sigma_by_tag);

/* --- conductivity Monte Carlo of one block of placements (uq/conductivity/run.py:203-387) ---- */

/* Opens a study (replaces build_conductivity_uq_precompute, uq/conductivity/assembly.py:73-140, and
 * the per-placement set-up of run_conductivity_uq, run.py:236-314): sets the context to
 * sigma_nominal (11 entries, index = tag; coarse AMG levels kept), splits the grounded stiffness
 * into the unperturbed tissues plus one unit-conductivity component per tag in tags[0..n_tags)
 * (checked to give back the nominal operator to 1e-10), places the k coil placements and
 * evaluates their dA/dt once, solves the nominal block, and solves for the sensitivity of each
 * placement's potential to each perturbed conductivity to sensitivity_tol (the reference uses
 * 1e-3, run.py:44-49). basis_rank (k, may be NULL) receives the dimension of each placement's
 * sensitivity subspace. opts as for cunibs_solve_block (warm_start must be 0). Until
 * cunibs_sigma_end, block solves and cunibs_context_set_conductivity* are refused. */
int cunibs_sigma_begin(cunibs_context* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
                       const double* centers_mm, const double* handles_mm, const double* dists_mm, int k, double didt,
                       const cunibs_solve_opts* opts, const double* sigma_nominal, const int* tags, int n_tags,
                       double sensitivity_tol, int* basis_rank);

/* One draw (the loop body of run.py:324-380): sigma (n_tags, in the order of tags) replaces the
 * perturbed conductivities; the finest operator becomes the components' combination (its smoother
 * weights follow, the coarse levels stay nominal), the right-hand side is re-weighted from the held
 * dA/dt, and PCG starts from the nominal potential plus the A-Galerkin projection of the draw's
 * linearised residual onto the sensitivity subspace (run.py:157-200), then runs to the study's
 * tolerance. A draw the kept coarse levels cannot finish is solved again on a hierarchy built for
 * it, after which the nominal hierarchy is rebuilt; *resetup (may be NULL) is then 1. Outputs as
 * cunibs_solve_block (host buffers); out->init_relres is the guess's relative residual. */
int cunibs_sigma_draw(cunibs_context* ctx, const double* sigma, cunibs_block_out* out, int* resetup);

/* The initial guess of the following draws, for comparisons of guesses (the results are the same
 * to the tolerance): 0 the sensitivity-subspace guess above (the default, the reference's
 * _InitialGuess, run.py:105-200), 1 the nominal potential alone, 2 the zero guess. No counterpart
 * in the reference. */
int cunibs_sigma_set_guess(cunibs_context* ctx, int mode);

/* Closes the study and returns the context to the nominal conductivities (the same operator and
 * hierarchy values as before cunibs_sigma_begin). A no-op when no study is open. */
int cunibs_sigma_end(cunibs_context* ctx);

/* The host step behind a placement's draw guess, exposed for testing: gram (n_tags, n_tags) =
 * S^T A S of the sensitivities, proj (n_tags, n_tags) with proj[a][t] = s_a . c_t, active[a] = 0
 * for a tissue with no sensitivity. coef (n_tags, n_tags) receives Z with the subspace coefficients
 * y = Z (sigma - sigma_nominal): Z = G^+ proj, G^+ the pseudo-inverse of the Gram over its
 * Jacobi-scaled eigenvalues above rtol times the largest; *rank (may be NULL) the count kept. */
int cunibs_sigma_coefficients(int n_tags, const double* gram, const double* proj, const int* active, double rtol,
                              double* coef, int* rank);

/* --- auxiliary dipole method (adm/reciprocity.py, evaluate.py) ---------------------------- */

typedef struct cunibs_adm cunibs_adm;

/* The adjoint (reciprocity) solves of a target functional J_d = sum_i weights[i] (dir_d . E_e),
 * e = elem_idx[i] in the context's element order, for n_dir (1..3) directions (replaces
 * solve_adjoint, reciprocity.py:119-141): K lambda_d = c_d, all directions in one block solve to
 * tolerance (the reference's ADJOINT_TOLERANCE is 1e-9 with 3000 iterations), then the nodal
 * weights W_d (reciprocity.py:91-116) with J_d = sum_n W_d[n] . dA/dt[n] exactly. iterations and
 * relres (n_dir, may be NULL) receive the solve statistics. The context must outlive the handle
 * and have no conductivity study open. */
int cunibs_adm_create(cunibs_context* ctx, const int* elem_idx, const double* weights, int n_elem,
                      const double* directions, int n_dir, double tolerance, int max_iters, int* iterations,
                      double* relres, cunibs_adm** out);
int cunibs_adm_destroy(cunibs_adm* adm);

/* The nodal weights W (n_dir, n_nodes, 3), FP64, context node order. */
int cunibs_adm_node_weights(const cunibs_adm* adm, double* out);

/* Samples Q_d(g) = mu0/4pi sum_n W_d[n] x (g - r_n) / |g - r_n|^3 on a regular grid (origin and
 * spacing in mm, shape per axis; C order, x slowest) with the FP32 dipole N-body centred on the
 * grid's centre (replaces sample_qfield, reciprocity.py:183-213). The field stays on the device. */
int cunibs_adm_sample(cunibs_adm* adm, const double* origin_mm, const double* spacing_mm, const int* shape);

/* Copies the sampled field (n_dir, nx, ny, nz, 3) FP32 to host memory (cap: floats available). */
int cunibs_adm_qfield(const cunibs_adm* adm, float* out, long long cap);

/* E (P, n_dir) = didt sum_j m_j . Q_d(s_j) for the coil's dipoles placed by P coil-to-head affines
 * (transforms (P, 4, 4), translation in mm), Q interpolated trilinearly on the sampled grid
 * (replaces evaluate_frames, evaluate.py:82-152). One block per placement reduces in a fixed order,
 * so a placement's value does not depend on the others. A dipole off the grid is CUNIBS_EINVAL
 * naming the first offending sample. */
int cunibs_adm_evaluate(cunibs_adm* adm, const double* dip_pos_m, const double* dip_moment, int n_dip,
                        const double* transforms, int P, double didt, double* E);

/* The same functional with Q evaluated exactly at every placed dipole (no grid; evaluate.py:155-193),
 * the N-body centred on center_mm (NULL: the origin). */
int cunibs_adm_evaluate_exact(cunibs_adm* adm, const double* dip_pos_m, const double* dip_moment, int n_dip,
                              const double* transforms, int P, double didt, const double* center_mm, double* E);

/* --- stage-level entry points (the reference's kernel exports, bindings.cpp) --------------- */

/* Copies a named internal array to host memory. name / dtype:
 *   int32:   "node_perm" "tet_perm" "tet_nodes" "tet_tags" "skin_tris" "n2c_ptr" "n2c_idx"
 *            "stiff_ptr" "stiff_col" "gm_index" and per level "a_ptr" "a_col" "agg" "p_ptr" "p_col"
 *            "coarse_ptr" "coarse_col"
 *   float64: "nodes_mm" "g" "vols" "bary" "stiff_val" "skin_normals" "coarse_val" "coarse_inv"
 *            "bottom_inv" (the dense inverse the V-cycle ends in, bottom_rows square)
 *            and per level "a_val" "p_val" "dinv"
 * *len receives the element count; at most cap elements are written. */
int cunibs_context_array(const cunibs_context* ctx, const char* name, int level, void* out, long long cap,
                         long long* len);

/* Coil frames for k targets (place.cu:246-273 semantics); degenerate[i] = 1 where the handle left
 * the in-plane axis undefined. handles may be NULL. */
int cunibs_context_place(cunibs_context* ctx, const double* centers_mm, const double* handles_mm,
                         const double* dists_mm, int k, double* transforms, int* degenerate);

/* dA/dt at the context's nodes for k given transforms: out (k, n_nodes, 3) (dadt.cu semantics).
 * Coils whose moments all lie along the coil's z axis take the coil-frame path. */
int cunibs_context_dadt(cunibs_context* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
                        const double* transforms, int k, double didt, float* out);

/* Solves the grounded system for k right-hand sides B (n_nodes-1, width), width in {1,2,4,8,16};
 * X receives the solution in the same layout. x0 may be NULL. */
int cunibs_context_solve(cunibs_context* ctx, const double* B, double* X, int k, int width, int precision,
                         double tolerance, int max_iters, const double* x0, int* iterations, double* relres);

/* One V-cycle z = M r on the grounded system, k columns row-major (n_nodes-1, k); fp32 selects the
 * FP32 hierarchy. */
int cunibs_context_vcycle(cunibs_context* ctx, const double* r, double* z, int k, int fp32);

/* SIZE_4 pairwise aggregation of one FP32 CSR matrix (select_size4, aggregate.cu:368-472).
 * aggregates: (n) out; *n_coarse receives the aggregate count. */
int cunibs_select_size4(int n, const int* row_ptr, const int* col_idx, const float* values, int* aggregates,
                        int* n_coarse);

/* Builds (once per context and mode) and describes a recovery operator (build_recovery_operator,
 * fem/recovery.py:445-453): slot maps, patches, the boundary marks and the patch weights. */
int cunibs_context_recovery(cunibs_context* ctx, int mode, cunibs_recovery_info* out);

/* Copies an array of a recovery operator to host memory. int32: "ptr" (n_slots+1), "idx" (corner ids
 * for SPR, patch nodes for HARMONIC), "slot_of_corner" (4*n_tets), "slot_node", "slot_tag" (empty
 * for SPR_GLOBAL), "status" (HARMONIC: rung per slot, 0 cubic .. 3 none), "is_boundary" (SPR, per
 * node); float32: "w" (SPR: one per entry; HARMONIC: 3 per entry). */
int cunibs_context_recovery_array(cunibs_context* ctx, int mode, const char* name, void* out, long long cap,
                                  long long* len);

/* Applies a recovery operator to k columns of caller data (apply_recovery_into,
 * fem/recovery.py:482-525): HARMONIC reads v (k, n_nodes) float64 (the grounded node is taken as 0)
 * and dadt_nodes (k, n_nodes, 3); SPR reads E_elem (k, n_tets, 3). Writes E_slots (k, n_slots, 3),
 * E (k, n_tets, 3; may be NULL) and magnE (k, n_tets). */
int cunibs_context_recover(cunibs_context* ctx, int mode, int k, const double* v, const float* dadt_nodes,
                           const float* E_elem, float* E_slots, float* E, float* magnE);

/* Gray-matter summary of one |E| field on the context's elements (RegionSlice.summarize). */
int cunibs_context_summary(cunibs_context* ctx, const float* magnE, int k, double* summary);

/* --- learned warm start ------------------------------------------------------------------
 *
 * No counterpart in the reference's solver. A network maps a coil pose (the coil origin / 100 mm
 * and the handle axis: 6 numbers, standardised by feature_mean/std) through `depth` SiLU layers of
 * width `hidden` to n_out standardised coefficients (coef_mean/std) of a reduced basis of the
 * grounded potential; the guess is basis . coefficients. All products run on BF16 tensor cores with
 * FP32 accumulation. Per column, a guess whose relative residual is not below 1 is dropped for the
 * zero guess; PCG then runs to the same tolerance either way.
 *
 * cunibs_context_set_warmstart copies the network from device memory: weights[l] BF16 row-major
 * [out_l, in_l] with in_0 = 64 (features zero-padded), in_l = hidden, out_l = hidden and
 * out_depth = n_out rounded up to 64 (= r); biases[l] FP32 [out_l]; basis BF16 [n_nodes - 1, 2 r] in the
 * grounded (Morton) row order, holding [V_hi | V_lo]: the basis V rounded to BF16 and the BF16
 * rounding of its remainder (V_lo = bf16(V - V_hi)), so the guess keeps about 16 significant bits.
 * weights == NULL removes the warm start. */
int cunibs_context_set_warmstart(cunibs_context* ctx, int depth, int hidden, int n_out, const void* const* weights,
                                 const float* const* biases, const float* feature_mean, const float* feature_std,
                                 const float* coef_mean, const float* coef_std, const void* basis);

/* The tensor-core kernels the network is trained with, on device pointers, queued on `stream`
 * (a cudaStream_t). cunibs_gemm_bf16: C[M,N] = A[M,K] . B[N,K]^T (BF16, K-major, leading dimensions
 * in elements, K a multiple of 8, 16-byte aligned bases) with FP32 accumulation and the fused tail
 * z = acc + bias[col] (bias may be NULL), z *= silu'(gate[row, col]) (gate may be NULL),
 * out32 = z, out16 = bf16(act ? silu(z) : z), out16t = its transpose [N, ld_t]; any output may be
 * NULL. The others: column sums (bias gradients), mean-squared error and its gradient
 * (2 (pred - target) / (rows * cols); scratch holds 296 floats), one Adam step with bias correction
 * and decoupled weight decay that also refreshes BF16 copies [rows, cols] and [cols, rows], and the
 * standardised BF16 pose features of k coil transforms (k, 16). */
int cunibs_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K, const float* bias,
                     const float* gate, int ld_gate, int act, float* out32, void* out16, int ld_out, void* out16t,
                     int ld_t, void* stream);
int cunibs_mlp_colsum(const float* x, int rows, int cols, int ld, float* out, void* stream);
/* Every mbarrier wait of the GEMM is bounded (2^24 polls or 2 s). A GEMM queued through
 * cunibs_gemm_bf16 records an expired wait in a per-device status word; cunibs_gemm_status
 * synchronises `stream`, reads and clears that word, sets *expired (may be NULL) and returns
 * CUNIBS_ETIMEOUT if a wait expired since the last read (that GEMM's outputs are invalid), else OK.
 * No counterpart in the reference (its kernels do not wait on barriers). */
int cunibs_gemm_status(void* stream, int* expired);
/* For tests of the timeout path only: later GEMM launches give up their waits after max_polls polls
 * or max_ns nanoseconds (<= 0: the defaults), and with withhold_loads = 1 the producer issues no
 * loads, so the MMA warp's first wait can only run out. Process-wide; restore with (0, 0, 0). */
int cunibs_debug_gemm_waits(long long max_polls, long long max_ns, int withhold_loads);
int cunibs_mlp_mse(const float* pred, const float* target, int rows, int cols, int ld, float* loss, float* d32,
                   void* d16, void* d16t, int ld_t, float* scratch, void* stream);
int cunibs_mlp_adam(float* param, float* m, float* v, const float* grad, long long n, float lr, float beta1,
                    float beta2, float eps, int step, float weight_decay, int rows, int cols, void* w16, void* w16t,
                    void* stream);
int cunibs_mlp_features(const double* transforms, int k, const float* mean, const float* std, void* x16, int ld,
                        void* stream);

/* --- without device allocation ------------------------------------------------------------
 *
 * No counterpart in the reference. For callers that cannot have the library allocate GPU memory --
 * for example a process whose device memory is already reserved by another framework's caching
 * allocator, or code held to a fixed memory budget set up in advance.
 *
 * cunibs_dadt_noalloc computes the same dA/dt as cunibs_context_dadt's general-moment path, for k
 * placements: nodes_mm (n_nodes, 3), dip_pos_m and dip_moment (n_dip, 3) in the coil frame,
 * transforms (k, 4, 4) and out (k, n_nodes, 3) are all device pointers on the current device, and the
 * work is queued on `stream` (a cudaStream_t; NULL is the legacy default stream). The function
 * allocates nothing: its scratch -- k * n_dip rotated dipole records -- is a fixed array of
 * CUNIBS_DADT_NOALLOC_MAX_RECORDS records (768 KiB) compiled into the library. Larger k * n_dip is
 * rejected with CUNIBS_EINVAL.
 * When the array takes device memory: it belongs to the library's CUDA module. Under the runtime's
 * default lazy module loading (CUDA_MODULE_LOADING=LAZY) a device receives the module -- the array
 * and the kernel code -- at the first call on that device, and that first call can fail with
 * CUNIBS_ECUDA (out of memory) if another allocator has already reserved all of the device's memory.
 * So make one call on each device before the other allocator reserves its memory, or run with
 * CUDA_MODULE_LOADING=EAGER (the module is then loaded with the context). The device holds it until
 * the process exits.
 * The first call on a device also looks up the array's device address (cudaGetSymbolAddress, made
 * with the device current); make that first call before any stream capture. The address is kept per
 * device and looked up again when the device's context changes (after cudaDeviceReset, or with a
 * different driver-API context current).
 * A CUDA error already pending from the caller's earlier work is reported as such (CUNIBS_ECUDA) and
 * left pending; nothing is launched.
 * All calls share the one array, so calls that may overlap on the GPU (different streams, or
 * different host threads) race on it: order them on one stream. */
#define CUNIBS_DADT_NOALLOC_MAX_RECORDS 16384
int cunibs_dadt_noalloc(const double* nodes_mm, int n_nodes, const double* dip_pos_m, const double* dip_moment,
                        int n_dip, const double* transforms, int k, double didt, float* out, void* stream);

/* --- measurement ------------------------------------------------------------------------ */

/* With timing on, each block solve records CUDA events on the context's stream between its stages
 * and cunibs_context_stage_times returns the last call's milliseconds: [0] placement and dipole
 * rotation, [1] dA/dt, [2] element average + right-hand side, [3] linear solve, [4] E + summary. */
int cunibs_context_set_timing(cunibs_context* ctx, int on);
int cunibs_context_stage_times(const cunibs_context* ctx, double* ms, int cap);

/* The context's CUDA stream (a cudaStream_t), on which every block solve's work is ordered. */
int cunibs_context_stream(const cunibs_context* ctx, void** stream);

/* Kernels this process has enqueued through the library so far (graph replays count their nodes). */
long long cunibs_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif
