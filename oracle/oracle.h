/* CPU restatement of the cuNIBS per-placement field solve (FP64, OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity oracle and the timed CPU baseline. Only
 * the test suite, the smoke check and the CPU-baseline arm of the benchmark load it; the product
 * path (cunibs_b200) never links, loads or calls it, and has no CPU fallback.
 *
 * Every stage cites the reference file:line whose behaviour it restates. Integer outputs (Morton
 * order, CSR pattern, aggregation) are computed with the same IEEE operations, in the same order,
 * as the CUDA path, so they can be compared bit for bit; field outputs are FP64 ground truth.
 */
#ifndef CUNIBS_ORACLE_H
#define CUNIBS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int min_coarse_rows;      /* fem/solve.py:146 AggregationParams.min_coarse_rows = 128 */
    int max_levels;           /* fem/solve.py:147 = 50 */
    int agg_rounds;           /* fem/solve.py:150 = 2 */
    int cheby_degree;         /* fem/solve.py:167 SmootherParams.degree = 2 */
    double cheby_lower_ratio; /* fem/solve.py:168 = 12 */
    int n_threads;            /* OpenMP threads; <= 0 means all */
    int has_sigma;            /* nonzero: conductivity per tag from sigma_by_tag, not the table */
    double sigma_by_tag[11];  /* S/m indexed by tag (1..10); a conductivity draw */
} orc_params;

/* Summary layout shared with the CUDA C-ABI (cunibs_b200.h CUNIBS_SUMMARY_*). */
enum {
    ORC_S_PEAK = 0,
    ORC_S_PEAK_X = 1,
    ORC_S_COG_X = 4,
    ORC_S_VOLUME = 7,
    ORC_S_MEAN = 8,
    ORC_S_STD = 9,
    ORC_S_P50 = 10,
    ORC_S_P95 = 11,
    ORC_S_P99 = 12,
    ORC_S_P999 = 13,
    ORC_S_FOC50 = 14,
    ORC_S_FOC75 = 15,
    ORC_SUMMARY_LEN = 16
};

void orc_params_default(orc_params* p);

/* Builds the whole per-subject state: Morton order, P1 operator, stiffness, grounding, SA-AMG
 * hierarchy, skin normals. Returns NULL and fills err on failure. */
void* orc_ctx_create(const double* nodes_mm, int n_nodes, const int* tet_nodes, const int* tet_tags,
                     int n_tets, const int* skin_tris, int n_skin, const orc_params* params,
                     char* err, int err_len);
void orc_ctx_destroy(void* ctx);

/* Named views of internal arrays (for parity tests). level selects a hierarchy level where the
 * name is per level. Returns 0 and sets ptr and len, or -1 if the name is unknown. */
int orc_get_i32(void* ctx, const char* name, int level, const int** ptr, long* len);
int orc_get_f64(void* ctx, const char* name, int level, const double** ptr, long* len);
int orc_n_levels(void* ctx);

/* One V-cycle application z = M r on the reduced system, k right-hand sides, row-major (n, k). */
int orc_vcycle_apply(void* ctx, const double* r, double* z, int k);

/* Field recovery modes (fem/recovery.py:74-113). */
enum { ORC_REC_RAW = 0, ORC_REC_SPR_GLOBAL = 1, ORC_REC_SPR_TISSUE = 2, ORC_REC_HARMONIC = 3 };

/* Full per-placement pipeline for k placements. recovery selects the reported field (ORC_REC_*);
 * the recovered field is FP64 on slots (recovery weights are FP32, as the reference stores them). Outputs (any may be NULL):
 * transforms (k,16), v (k, n_nodes) potential per placement, magnE (k, n_tets), E (k, n_tets, 3),
 * summary (k, ORC_SUMMARY_LEN), iters (k), relres (k). Returns 0 or -1 (err filled). */
int orc_solve(void* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
              const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
              double didt, double tolerance, int max_iters, int recovery, double* transforms, double* v,
              float* magnE, float* E, double* summary, int* iters, double* relres, char* err,
              int err_len);

/* Stage-level entry points on caller data. */
int orc_select_size4(int n, const int* row_ptr, const int* col_idx, const float* values,
                     int* aggregates);
void orc_l1_dinv_f32(int n, const int* row_ptr, const int* col_idx, const float* values,
                     float* dinv);
void orc_dadt(const double* dip_pos_m, const double* dip_moment, int n_dip,
              const double* transform, double didt, const double* nodes_mm, int n_nodes,
              double* out);
int orc_place(void* ctx, const double* centers, const double* handles, const double* dists,
              int k, double* transforms, int* degenerate);
void orc_summary(const float* magnE, const float* vols, const double* barycenters_mm,
                 const int* tet_tags, int n_tets, int region_tag, double* out);
void orc_weighted_quantiles(const double* values, const double* weights, int n, const double* qs,
                            int nq, double* out);

/* Recovery operator of a mode, built once per context: the slot CSR (ptr, idx), slot maps,
 * weights (SPR: one per corner entry; harmonic: three per patch entry), the harmonic rung per
 * slot (status), the boundary marks of the SPR modes (is_boundary), and counts = (n_slots,
 * n_fallback, n_undetermined). */
int orc_recovery_build(void* ctx, int mode, char* err, int err_len);
int orc_recovery_i32(void* ctx, int mode, const char* name, const int** ptr, long* len);
int orc_recovery_w(void* ctx, int mode, const float** ptr, long* len);

/* Applies a built operator to k columns with the CUDA apply kernels' arithmetic: harmonic reads
 * v (k, n_nodes) f64 and dadt_nodes (k, n_nodes, 3) f32; SPR reads E_elem (k, n_tets, 3) f32.
 * Writes E_slots (k, n_slots, 3), E_out (k, n_tets, 3; may be NULL) and magn (k, n_tets). */
int orc_recovery_apply(void* ctx, int mode, int k, const double* v, const float* dadt_nodes, const float* E_elem,
                       float* E_slots, float* E_out, float* magn);

#ifdef __cplusplus
}
#endif
#endif
