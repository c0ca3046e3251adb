// The C ABI (include/cunibs_b200.h): context lifetime, the block solve, stage-level entry points.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <climits>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <type_traits>

#include "../../include/cunibs_b200.h"
#include "internal.hpp"

using namespace cunibs;

namespace {

thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return CUNIBS_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return CUNIBS_ENOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return CUNIBS_EINTERNAL;
    }
}

void require(bool ok, const char* msg) {
    if (!ok) fail(kEInval, msg);
}

int to_internal_precision(int p) {
    if (p == CUNIBS_PREC_PLAIN_FP64) return kPlainFp64;
    if (p == CUNIBS_PREC_MIXED) return kMixed;
    if (p == CUNIBS_PREC_SPLIT) return kFp64CgFp32Mg;
    fail(kEInval, "precision must be CUNIBS_PREC_PLAIN_FP64, CUNIBS_PREC_MIXED or CUNIBS_PREC_SPLIT");
}

int pad_width(int k) {
    for (int w : {1, 2, 4, 8, 16})
        if (w >= k) return w;
    fail(kEInval, "at most 16 placements per block");
}

}  // namespace

void cunibs::set_last_error(const std::string& message) { g_last_error = message; }

// What a block's preparation (placement, dA/dt, right-hand side) leaves for its solve. Two slots
// let the next block be prepared while the previous one is solved.
struct BlockSlot {
    DevArray<double> in_pos, in_mom, in_centers, in_handles, in_dists;  // host-entry inputs, uploaded
    DevArray<double> T, B, X0;  // X0: the learned initial guess
    DevArray<int> deg;
    DevArray<unsigned char> dip_packed;
    DevArray<float> dadt_nodes, dadt_elm;
    // Nodes the coil table does not cover, per placement (p * N + ...), and their counts.
    DevArray<int> near_list, near_cnt;
    cudaEvent_t prepared = nullptr;
    int* h_deg = nullptr;   // pinned: the degenerate-placement flags
    int* h_near = nullptr;  // pinned: near_cnt, copied when the block's dA/dt read the table
    bool near_valid = false;
};

// Pinned host staging of a finished block's per-column statistics (device outputs).
struct Staging {
    int iters[16];
    double rel[16];
    int used[16];
    double init[16];
};

struct PendingBlock {
    long long ticket = 0;
    int slot = 0, k = 0, K = 0;
    bool has_opts = false, has_handles = false;
    bool timed = false;  // stage events recorded (only for a block prepared with no other in flight)
    bool guess_due = false;  // a learned initial guess is wanted and not yet issued
    bool x0_given = false;   // the slot's X0 already holds this block's initial guess
    cunibs_solve_opts opts{};
};

// A conductivity Monte Carlo over one block of placements (uq/conductivity/run.py:203-387): the
// coil field of the block (held in one slot), the per-tissue operator components, the nominal
// solution and its sensitivities, from cunibs_sigma_begin to cunibs_sigma_end.
struct SigmaStudy {
    int k = 0, K = 0, P = 0, slot = 0;
    bool has_handles = false, has_opts = false;
    cunibs_solve_opts opts{};
    double nominal[11] = {};
    int tags[kSigmaMaxTags] = {};
    long nnz = 0;
    DevArray<double> comp;   // (1 + P, nnz): the other tissues at nominal, then each tissue at unit sigma
    DevArray<double> rhs;    // (1 + P, n_red, K): the block's right-hand sides split the same way
    DevArray<double> x_nom;  // (n_red, K) nominal potential
    DevArray<double> S;      // (n_red, P, K) sensitivities
    std::vector<double> Z;   // (K, P, P): y_j = Z_j (sigma - sigma_nom)
    std::vector<int> rank;   // (k)
    int guess_mode = 0;      // 0 subspace guess, 1 the nominal potential alone, 2 zero (cunibs_sigma_set_guess)
};

struct cunibs_context {
    int device = 0;
    Params prm;
    // The solve and everything after it run on `stream`; block preparation runs on `prep`, at a
    // lower priority, so that it fills what the latency-bound solve leaves of the SMs.
    cudaStream_t stream = nullptr;
    cudaStream_t prep = nullptr;
    Mesh mesh;
    Hierarchy hier;
    SolverPtr solver;
    SummaryWork sw;
    // Block workspace, grown on demand.
    DevArray<double> pos, mom, centers, handles, dists, T, X, summary, v;
    DevArray<int> deg, coil_flag;
    DevArray<unsigned char> dip_packed, zdip_packed;
    DevArray<float> dadt_nodes, magn, E;
    BlockSlot slots[2];
    std::deque<PendingBlock> pending;
    int next_slot = 0;
    long long next_ticket = 1;
    int* h_coil_flag = nullptr;  // pinned
    Staging* staging = nullptr;  // pinned
    cudaEvent_t ev_main = nullptr;
    // Blocks per SM given to the dA/dt kernel while another block's solve may run beside it.
    int overlap_blocks_per_sm = 2;
    // The coil field table (cunibs_context_set_coil_table): mode 1 reads it for nodes deeper than
    // table_near_m below the coil, mode 0 sums every dipole at every node.
    CoilTable coil_table;
    int table_mode = 1;
    double table_near_m = 0.015, table_step = 0.035;
    double mesh_rho_m = 0.0;  // largest distance of a node from the centre of the mesh's bounding box
    long long last_near = -1, last_near_of = 0;  // direct-sum nodes of the last finished block
    // Host wall-clock milliseconds from the start of the last cunibs_sigma_begin to the end of each of
    // its phases (cunibs_context_phase_times).
    double phase_ms[8] = {};
    int sm_count = 0;
    // Field-recovery operators, built on first use per mode, and their block workspace.
    std::unique_ptr<RecoveryOp> rec[4];
    DevArray<float> e_slots, e_raw;
    // Learned warm start (installed by cunibs_context_set_warmstart) and its per-block outputs.
    std::unique_ptr<WarmStart> warm;
    std::vector<int> warm_used;
    std::vector<double> init_rel;
    // The open conductivity study, if any (its block slot is reserved while it is open).
    std::unique_ptr<SigmaStudy> study;
    // Stage timing (CUDA events on the context stream), enabled by cunibs_context_set_timing.
    bool timing = false;
    cudaEvent_t ev[6] = {};
    double stage_ms[5] = {};

    void mark(int i, cudaStream_t on) {
        if (timing) CUNIBS_CHECK(cudaEventRecord(ev[i], on));
    }

    RecoveryOp& recovery(int mode) {
        if (mode < kRecSprGlobal || mode > kRecHarmonic) fail(kEInval, "unknown recovery mode " + std::to_string(mode));
        if (!rec[mode]) {
            auto op = std::make_unique<RecoveryOp>();
            build_recovery(mesh, *op, mode, stream);
            CUNIBS_CHECK(cudaStreamSynchronize(stream));
            rec[mode] = std::move(op);
        }
        return *rec[mode];
    }

    // The finest level takes the mesh's current stiffness values (same pattern), its smoother
    // weights and FP32 copies follow; coarser levels are kept. Without levels: a full rebuild.
    void keep_coarse_values() {
        if (hier.levels.empty()) {
            rebuild_hierarchy();
            return;
        }
        Level& L0 = hier.levels[0];
        reduce_grounded_values(mesh, L0.a, L0.a.val.get(), stream);
        refresh_finest_derived(hier, stream);
        CUNIBS_CHECK(cudaStreamSynchronize(stream));
    }

    // Hierarchy builds over the context's life (the first at create); cunibs_context_info reports it.
    int hierarchy_builds = 0;

    void rebuild_hierarchy() {
        ++hierarchy_builds;
        solver.reset();
        DevCsr<double> a0;
        reduce_grounded(mesh, a0, stream);
        build_hierarchy(hier, a0, prm, stream);
        solver = make_solver(hier, prm);
    }

    ~cunibs_context() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        for (BlockSlot& sl : slots) {
            if (sl.prepared) cudaEventDestroy(sl.prepared);
            if (sl.h_deg) cudaFreeHost(sl.h_deg);
            if (sl.h_near) cudaFreeHost(sl.h_near);
        }
        if (ev_main) cudaEventDestroy(ev_main);
        if (h_coil_flag) cudaFreeHost(h_coil_flag);
        if (staging) cudaFreeHost(staging);
        solver.reset();
        if (prep) cudaStreamDestroy(prep);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        CUNIBS_CHECK(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

Params resolve(const cunibs_context* c, const cunibs_solve_opts* o) {
    Params p = c->prm;
    if (o) {
        if (o->precision != CUNIBS_PREC_DEFAULT) p.precision = to_internal_precision(o->precision);
        if (o->tolerance > 0) p.tolerance = o->tolerance;
        if (o->max_iters > 0) p.max_iters = o->max_iters;
    }
    return p;
}

constexpr int kMaxBlock = 16;
// Eigenvalues of a placement's Jacobi-scaled sensitivity Gram kept for its draw guesses, relative
// to the largest (the reference keeps singular values above 1e-8 of the largest, run.py:108-123).
constexpr double kSigmaRtol = 1e-12;

void copy_out(void* dst, const void* src, std::size_t bytes, cudaMemcpyKind kind, cudaStream_t s);
std::size_t slot_bytes(const cunibs_context* c, const cunibs_solve_opts* opts, int k);

// Block preparation on the preparation stream: the coil placement, dA/dt at the nodes and
// elements, and the right-hand side, into a free slot. Device inputs are read asynchronously and
// must stay valid until the block is finished; host inputs are copied into the slot first.
// bounded_dadt gives the dA/dt kernel a bounded grid, for a preparation that runs beside another
// block's solve. The element average of dA/dt is formed when the block's recovery reads it (raw and
// SPR) or keep_elements asks for it (a conductivity study's block). Returns the block's ticket.
long long prepare_block(cunibs_context* c, const double* pos, const double* mom, int n_dip, const double* centers,
                        const double* handles, const double* dists, int k, double didt, const cunibs_solve_opts* opts,
                        bool host_inputs, bool bounded_dadt, bool keep_elements = false) {
    require(!c->study, "a conductivity study is open: end it (cunibs_sigma_end) before solving other blocks");
    require(k >= 1, "need at least one placement");
    require(n_dip >= 1, "the coil needs at least one dipole");
    require(pos && mom && centers && dists, "input arrays must not be NULL");
    const int K = (opts && opts->block_width > 0) ? opts->block_width : pad_width(k);
    require(K >= k, "block_width must be at least the number of placements");
    require(K <= kMaxBlock, "at most 16 placements per block");
    const int rec_mode = opts ? opts->recovery : kRecRaw;
    require(rec_mode >= kRecRaw && rec_mode <= kRecHarmonic, "unknown recovery mode");
    const bool warm = opts && opts->warm_start;
    if (warm) {
        require(opts->warm_start == kGuessNetwork || opts->warm_start == kGuessProjection,
                "warm_start must be 0, 1 (network) or 2 (projection onto its basis)");
        require(c->warm != nullptr, "warm_start requested but no warm-start network is installed");
        require(c->warm->n_red == c->mesh.n_nodes - 1, "the installed warm start was built for another mesh");
    }
    int si = -1;
    for (int t = 0; t < 2 && si < 0; ++t) {
        const int cand = (c->next_slot + t) & 1;
        bool used = false;
        for (const PendingBlock& q : c->pending) used = used || q.slot == cand;
        if (!used) si = cand;
    }
    require(si >= 0, "two blocks are already submitted: finish one before submitting another");
    const bool beside_solve = bounded_dadt && !c->pending.empty();
    BlockSlot& sl = c->slots[si];
    Mesh& m = c->mesh;
    cudaStream_t ps = c->prep;
    const bool timed = c->timing && c->pending.empty();
    auto mark = [&](int i) {
        if (timed) c->mark(i, ps);
    };
    const int n_red = m.n_nodes - 1;
    if (host_inputs) {
        sl.in_pos.upload(pos, 3 * static_cast<std::size_t>(n_dip), ps);
        sl.in_mom.upload(mom, 3 * static_cast<std::size_t>(n_dip), ps);
        sl.in_centers.upload(centers, 3 * static_cast<std::size_t>(k), ps);
        if (handles) sl.in_handles.upload(handles, 3 * static_cast<std::size_t>(k), ps);
        sl.in_dists.upload(dists, static_cast<std::size_t>(k), ps);
        pos = sl.in_pos.get();
        mom = sl.in_mom.get();
        centers = sl.in_centers.get();
        handles = handles ? sl.in_handles.get() : nullptr;
        dists = sl.in_dists.get();
    }
    // The coil's kind (all moments along its own z axis, or not) picks the dA/dt kernel.
    c->zdip_packed.reserve(packed_zdipole_bytes() * static_cast<std::size_t>(n_dip));
    c->coil_flag.reserve(1);
    prep_zdipoles(pos, mom, n_dip, c->zdip_packed.get(), c->coil_flag.get(), ps);
    CoilTable& tb = c->coil_table;
    const bool want_table = c->table_mode != 0;
    if (want_table && tb.built && tb.n_dip == n_dip) coil_compare(pos, mom, n_dip, tb, c->coil_flag.get(), ps);
    CUNIBS_CHECK(cudaMemcpyAsync(c->h_coil_flag, c->coil_flag.get(), sizeof(int), cudaMemcpyDeviceToHost, ps));
    CUNIBS_CHECK(cudaStreamSynchronize(ps));
    const bool zcoil = (*c->h_coil_flag & 1) == 0;
    // The table follows the coil: rebuilt (once) when the coil, its kind or the table's parameters
    // change.
    if (want_table && (!tb.built || tb.n_dip != n_dip || (*c->h_coil_flag & 2) || tb.nc != (zcoil ? 2 : 3) ||
                       tb.near_m != c->table_near_m || tb.step != c->table_step)) {
        const double rho = std::max(c->mesh_rho_m, c->table_near_m);
        build_coil_table(tb, pos, mom, n_dip, zcoil, c->zdip_packed.get(), c->table_near_m, c->table_step, 1.1 * rho,
                         2.5 * rho + 0.05, kCoilTableMaxPoints, ps);
    }
    const bool use_table = want_table && tb.valid;
    // The slot's previous block is finished on the context stream: start after what that stream
    // holds so far.
    CUNIBS_CHECK(cudaEventRecord(c->ev_main, c->stream));
    CUNIBS_CHECK(cudaStreamWaitEvent(ps, c->ev_main, 0));
    mark(0);
    sl.T.reserve(16 * static_cast<std::size_t>(k));
    sl.deg.reserve(k);
    place_transforms(m, centers, handles, dists, k, sl.T.get(), sl.deg.get(), ps);
    CUNIBS_CHECK(cudaMemcpyAsync(sl.h_deg, sl.deg.get(), sizeof(int) * k, cudaMemcpyDeviceToHost, ps));
    sl.dadt_nodes.reserve(static_cast<std::size_t>(m.n_nodes) * 3 * k);
    const int dadt_blocks = beside_solve ? c->overlap_blocks_per_sm * c->sm_count : 0;
    if (use_table) {
        sl.near_list.reserve(static_cast<std::size_t>(m.n_nodes) * k);
        sl.near_cnt.reserve(kMaxBlock);
    }
    sl.near_valid = use_table;
    if (zcoil) {
        mark(1);
        if (use_table) {
            dadt_table(m, tb, sl.T.get(), k, didt, sl.dadt_nodes.get(), sl.near_list.get(), sl.near_cnt.get(), ps,
                       dadt_blocks);
            dadt_near_zcoil(m, c->zdip_packed.get(), n_dip, sl.T.get(), k, didt, sl.dadt_nodes.get(),
                            sl.near_list.get(), sl.near_cnt.get(), ps, dadt_blocks);
        } else {
            dadt_nodes_zcoil(m, c->zdip_packed.get(), n_dip, sl.T.get(), k, didt, sl.dadt_nodes.get(), ps,
                             dadt_blocks);
        }
    } else {
        sl.dip_packed.reserve(packed_dipole_bytes() * static_cast<std::size_t>(n_dip) * k);
        prep_dipoles(pos, mom, n_dip, sl.T.get(), k, sl.dip_packed.get(), ps);
        mark(1);
        if (use_table) {
            dadt_table(m, tb, sl.T.get(), k, didt, sl.dadt_nodes.get(), sl.near_list.get(), sl.near_cnt.get(), ps,
                       dadt_blocks);
            dadt_near_general(m, reinterpret_cast<const float*>(sl.dip_packed.get()), n_dip, sl.T.get(), k, didt,
                              sl.dadt_nodes.get(), sl.near_list.get(), sl.near_cnt.get(), ps, dadt_blocks);
        } else {
            dadt_nodes(m, reinterpret_cast<const float*>(sl.dip_packed.get()), n_dip, sl.T.get(), k, didt,
                       sl.dadt_nodes.get(), ps, dadt_blocks);
        }
    }
    if (use_table)
        CUNIBS_CHECK(cudaMemcpyAsync(sl.h_near, sl.near_cnt.get(), sizeof(int) * k, cudaMemcpyDeviceToHost, ps));
    mark(2);
    if (keep_elements || rec_mode != kRecHarmonic) {
        sl.dadt_elm.reserve(static_cast<std::size_t>(m.n_tets) * 3 * k);
        dadt_elements(m, sl.dadt_nodes.get(), k, sl.dadt_elm.get(), ps);
    }
    sl.B.reserve(static_cast<std::size_t>(n_red) * K);
    // A conductivity study forms every draw's right-hand side from the element average, its nominal
    // one included; other blocks take it from the nodal field directly.
    if (keep_elements) rhs_block(m, sl.dadt_elm.get(), k, K, sl.B.get(), ps);
    else rhs_block_nodes(m, sl.dadt_nodes.get(), k, K, sl.B.get(), ps);
    mark(3);
    CUNIBS_CHECK(cudaEventRecord(sl.prepared, ps));
    PendingBlock pb;
    pb.slot = si;
    pb.k = k;
    pb.K = K;
    pb.has_handles = handles != nullptr;
    pb.has_opts = opts != nullptr;
    pb.timed = timed;
    pb.guess_due = warm;
    if (opts) pb.opts = *opts;
    pb.ticket = c->next_ticket++;
    c->pending.push_back(pb);
    c->next_slot = si ^ 1;
    return pb.ticket;
}

// The learned initial guess of a prepared block, on the context stream. It is issued once the
// block's preparation (its dA/dt included) is complete: the network's tensor-core tiles need SMs
// free of the long-lived dA/dt blocks, and a guess issued beside them waits for them to drain
// (measured: 6.6-9.2 ms per block, erratic, against 6.6 steady without a guess).
void issue_guess(cunibs_context* c, PendingBlock& q) {
    BlockSlot& ql = c->slots[q.slot];
    CUNIBS_CHECK(cudaStreamWaitEvent(c->stream, ql.prepared, 0));
    ql.X0.reserve(static_cast<std::size_t>(c->mesh.n_nodes - 1) * q.K);
    warm_start_guess(*c->warm, ql.T.get(), ql.B.get(), q.k, q.K, ql.X0.get(), q.opts.warm_start, c->stream);
    q.guess_due = false;
}

// Solve, field recovery and summary of a prepared block, on the context stream; outputs land in
// the context's workspace (and the slot's transforms). The block leaves the pending list whether
// or not this succeeds.
PendingBlock finish_block(cunibs_context* c, long long ticket, SolveStats& st, bool want_E) {
    auto it = c->pending.begin();
    while (it != c->pending.end() && it->ticket != ticket) ++it;
    if (it == c->pending.end()) fail(kEInval, "no submitted block with ticket " + std::to_string(ticket));
    PendingBlock pb = *it;
    c->pending.erase(it);
    BlockSlot& sl = c->slots[pb.slot];
    const int k = pb.k, K = pb.K;
    const cunibs_solve_opts* opts = pb.has_opts ? &pb.opts : nullptr;
    const Params prm = resolve(c, opts);
    const int rec_mode = opts ? opts->recovery : kRecRaw;
    RecoveryOp* op = rec_mode == kRecRaw ? nullptr : &c->recovery(rec_mode);
    Mesh& m = c->mesh;
    cudaStream_t s = c->stream;
    const int n_red = m.n_nodes - 1;
    CUNIBS_CHECK(cudaEventSynchronize(sl.prepared));
    c->last_near = -1;
    if (sl.near_valid) {
        c->last_near = 0;
        for (int i = 0; i < k; ++i) c->last_near += sl.h_near[i];
    }
    c->last_near_of = static_cast<long long>(m.n_nodes) * k;
    for (int i = 0; i < k; ++i)
        if (pb.has_handles && sl.h_deg[i])
            fail(kEInval, "degenerate coil placement at index " + std::to_string(i) + " of " + std::to_string(k) +
                              ": the handle lies on the outward scalp normal through the projected centre, so the "
                              "coil's rotation about the normal is undefined");
    CUNIBS_CHECK(cudaStreamWaitEvent(s, sl.prepared, 0));
    c->X.reserve(static_cast<std::size_t>(n_red) * K);
    const bool warm = opts && opts->warm_start;
    const bool guessed = warm || pb.x0_given;
    if (pb.guess_due) issue_guess(c, pb);
    c->warm_used.assign(k, 0);
    c->init_rel.assign(k, 1.0);
    solver_solve(*c->solver, sl.B.get(), c->X.get(), k, K, prm, s, st, guessed ? sl.X0.get() : nullptr);
    if (guessed) {
        if (warm) warm_start_check(*c->warm, s);
        for (int i = 0; i < k; ++i) {
            c->init_rel[i] = st.col_init_rel[i];
            c->warm_used[i] = st.col_init_rel[i] < 1.0 ? 1 : 0;
        }
    }
    // Columns that missed tolerance: the hierarchy is rebuilt at the operator's current values (a
    // V-cycle kept from other conductivities may be what failed), then one FP64 retry from their
    // current iterate, then an error (the rebuild-then-retry contract of fem/solve.py:528-551).
    // Inside a conductivity study the mesh's assembled values are the nominal ones, not the draw's,
    // so the draw's own failure path (cunibs_sigma_draw) does its rebuild instead.
    std::vector<int> missed;
    for (int i = 0; i < k; ++i)
        if (!(st.col_rel[i] <= prm.tolerance)) missed.push_back(i);
    if (!missed.empty()) {
        if (!c->study) c->rebuild_hierarchy();
        Params retry = prm;
        retry.precision = kPlainFp64;
        SolveStats st2;
        solver_solve(*c->solver, sl.B.get(), c->X.get(), k, K, retry, s, st2, c->X.get());
        for (int i : missed) {
            st.col_iters[i] += st2.col_iters[i];
            st.col_rel[i] = st2.col_rel[i];
            if (!(st2.col_rel[i] <= prm.tolerance)) {
                fail(kENoConv, "PCG did not converge (column " + std::to_string(i) + " of the block): " +
                                   std::to_string(st.col_iters[i]) + " iterations, relative residual " +
                                   std::to_string(st2.col_rel[i]) + " > tolerance " + std::to_string(prm.tolerance));
            }
        }
        st.iterations += st2.iterations;
    }
    if (pb.timed) c->mark(4, s);
    // The next block's guess goes here, between this solve and this block's recovery, when its
    // preparation is already complete (else its own finish issues it).
    for (PendingBlock& q : c->pending) {
        if (!q.guess_due || !c->warm) continue;
        const cudaError_t ready = cudaEventQuery(c->slots[q.slot].prepared);
        if (ready == cudaSuccess) {
            issue_guess(c, q);
        } else if (ready == cudaErrorNotReady) {
            if (cudaPeekAtLastError() == cudaErrorNotReady) (void)cudaGetLastError();  // not a failure
        } else {
            CUNIBS_CHECK(ready);
        }
    }
    c->magn.reserve(static_cast<std::size_t>(m.n_tets) * k);
    if (want_E) c->E.reserve(static_cast<std::size_t>(m.n_tets) * 3 * k);
    if (op == nullptr) {
        reconstruct_block(m, c->X.get(), k, K, sl.dadt_elm.get(), want_E ? c->E.get() : nullptr, c->magn.get(), s);
    } else {
        // The potential-consuming mode never forms the raw field (fem/solve.py:943-965).
        const float* e_elem = nullptr;
        if (rec_mode != kRecHarmonic) {
            c->e_raw.reserve(static_cast<std::size_t>(m.n_tets) * 3 * k);
            reconstruct_block(m, c->X.get(), k, K, sl.dadt_elm.get(), c->e_raw.get(), c->magn.get(), s);
            e_elem = c->e_raw.get();
        }
        c->e_slots.reserve(static_cast<std::size_t>(op->n_slots) * 3 * k);
        apply_recovery(m, *op, c->X.get(), K, sl.dadt_nodes.get(), e_elem, k, c->e_slots.get(),
                       want_E ? c->E.get() : nullptr, c->magn.get(), s);
    }
    c->summary.reserve(static_cast<std::size_t>(kSummaryLen) * k);
    gm_summary(m, c->magn.get(), k, c->summary.get(), c->sw, s);
    if (pb.timed) c->mark(5, s);
    if (pb.timed && c->timing) {
        CUNIBS_CHECK(cudaEventSynchronize(c->ev[5]));
        for (int i = 0; i < 5; ++i) {
            float ms = 0.0f;
            CUNIBS_CHECK(cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]));
            c->stage_ms[i] = ms;
        }
    }
    return pb;
}

// Host outputs of a finished block (cunibs_block_out host pointers).
void block_outputs_host(cunibs_context* c, const PendingBlock& pb, const SolveStats& st, cunibs_block_out* out) {
    const Mesh& m = c->mesh;
    cudaStream_t s = c->stream;
    const int k = pb.k;
    const cunibs_solve_opts* opts = pb.has_opts ? &pb.opts : nullptr;
    copy_out(out->transforms, c->slots[pb.slot].T.get(), sizeof(double) * 16 * k, cudaMemcpyDeviceToHost, s);
    copy_out(out->summary, c->summary.get(), sizeof(double) * kSummaryLen * k, cudaMemcpyDeviceToHost, s);
    copy_out(out->magnE, c->magn.get(), sizeof(float) * static_cast<std::size_t>(m.n_tets) * k, cudaMemcpyDeviceToHost, s);
    copy_out(out->E, c->E.get(), sizeof(float) * 3 * static_cast<std::size_t>(m.n_tets) * k, cudaMemcpyDeviceToHost, s);
    copy_out(out->E_slots, c->e_slots.get(), slot_bytes(c, opts, k), cudaMemcpyDeviceToHost, s);
    if (out->v) {
        c->v.reserve(static_cast<std::size_t>(m.n_nodes) * k);
        scatter_potential(m, c->X.get(), k, pb.K, c->v.get(), s);
        copy_out(out->v, c->v.get(), sizeof(double) * static_cast<std::size_t>(m.n_nodes) * k, cudaMemcpyDeviceToHost, s);
    }
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    for (int i = 0; i < k; ++i) {
        if (out->iterations) out->iterations[i] = st.col_iters[i];
        if (out->relres) out->relres[i] = st.col_rel[i];
        if (out->warm_used) out->warm_used[i] = c->warm_used[i];
        if (out->init_relres) out->init_relres[i] = c->init_rel[i];
    }
    out->total_iterations = st.iterations;
    out->outer_steps = st.outer_steps;
}

// Device outputs of a finished block (cunibs_block_out device pointers).
void block_outputs_device(cunibs_context* c, const PendingBlock& pb, const SolveStats& st, cunibs_block_out* out) {
    const Mesh& m = c->mesh;
    cudaStream_t s = c->stream;
    const int k = pb.k;
    const cunibs_solve_opts* opts = pb.has_opts ? &pb.opts : nullptr;
    copy_out(out->transforms, c->slots[pb.slot].T.get(), sizeof(double) * 16 * k, cudaMemcpyDeviceToDevice, s);
    copy_out(out->summary, c->summary.get(), sizeof(double) * kSummaryLen * k, cudaMemcpyDeviceToDevice, s);
    copy_out(out->magnE, c->magn.get(), sizeof(float) * static_cast<std::size_t>(m.n_tets) * k, cudaMemcpyDeviceToDevice, s);
    copy_out(out->E, c->E.get(), sizeof(float) * 3 * static_cast<std::size_t>(m.n_tets) * k, cudaMemcpyDeviceToDevice, s);
    copy_out(out->E_slots, c->e_slots.get(), slot_bytes(c, opts, k), cudaMemcpyDeviceToDevice, s);
    if (out->v) scatter_potential(m, c->X.get(), k, pb.K, out->v, s);
    // Per-column statistics go up from pinned staging (no pageable-memory copies).
    Staging& h = *c->staging;
    for (int i = 0; i < k; ++i) {
        h.iters[i] = st.col_iters[i];
        h.rel[i] = st.col_rel[i];
        h.used[i] = c->warm_used[i];
        h.init[i] = c->init_rel[i];
    }
    copy_out(out->iterations, h.iters, sizeof(int) * k, cudaMemcpyHostToDevice, s);
    copy_out(out->relres, h.rel, sizeof(double) * k, cudaMemcpyHostToDevice, s);
    copy_out(out->warm_used, h.used, sizeof(int) * k, cudaMemcpyHostToDevice, s);
    copy_out(out->init_relres, h.init, sizeof(double) * k, cudaMemcpyHostToDevice, s);
    // Returning only once the outputs are complete measured faster in a two-deep pipeline than
    // returning at once: the next submit then finds the previous block's work done.
    CUNIBS_CHECK(cudaStreamSynchronize(s));
    out->total_iterations = st.iterations;
    out->outer_steps = st.outer_steps;
}

void copy_out(void* dst, const void* src, std::size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
    if (dst && bytes) CUNIBS_CHECK(cudaMemcpyAsync(dst, src, bytes, kind, s));
}

// Bytes of the recovered slot field of a block solved with these options (0 for the raw field).
std::size_t slot_bytes(const cunibs_context* c, const cunibs_solve_opts* opts, int k) {
    const int mode = opts ? opts->recovery : kRecRaw;
    if (mode == kRecRaw || !c->rec[mode]) return 0;
    return sizeof(float) * 3 * static_cast<std::size_t>(c->rec[mode]->n_slots) * k;
}

}  // namespace

extern "C" {

int cunibs_version(void) { return 1; }

const char* cunibs_last_error(void) { return g_last_error.c_str(); }

int cunibs_params_default(cunibs_params* out) {
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        const Params p;
        out->device = 0;
        out->min_coarse_rows = p.min_coarse_rows;
        out->max_levels = p.max_levels;
        out->agg_rounds = p.agg_rounds;
        out->cheby_degree = p.cheby_degree;
        out->cheby_lower_ratio = p.cheby_lower_ratio;
        out->tolerance = p.tolerance;
        out->max_iters = p.max_iters;
        out->precision = CUNIBS_PREC_SPLIT;
        out->inner_reduction = p.inner_reduction;
        out->inner_max_iters = p.inner_max_iters;
        out->iters_per_sync = p.iters_per_sync;
        out->dense_max_rows = p.dense_max_rows;
    });
}

int cunibs_context_create(const double* nodes_mm, int n_nodes, const int* tet_nodes, const int* tet_tags, int n_tets,
                          const int* skin_tris, int n_skin, const cunibs_params* params, cunibs_context** out) {
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        *out = nullptr;
        require(nodes_mm && tet_nodes && tet_tags, "mesh arrays must not be NULL");
        require(n_skin == 0 || skin_tris != nullptr, "skin_tris is NULL");
        cunibs_params p;
        if (params) p = *params;
        else cunibs_params_default(&p);
        auto c = std::make_unique<cunibs_context>();
        c->device = p.device;
        DeviceGuard dg(c->device);
        c->prm.min_coarse_rows = p.min_coarse_rows;
        c->prm.max_levels = p.max_levels;
        c->prm.agg_rounds = p.agg_rounds;
        c->prm.cheby_degree = p.cheby_degree;
        c->prm.cheby_lower_ratio = p.cheby_lower_ratio;
        c->prm.tolerance = p.tolerance;
        c->prm.max_iters = p.max_iters;
        c->prm.precision = to_internal_precision(p.precision == CUNIBS_PREC_DEFAULT ? CUNIBS_PREC_SPLIT : p.precision);
        c->prm.inner_reduction = p.inner_reduction;
        c->prm.inner_max_iters = p.inner_max_iters;
        c->prm.iters_per_sync = p.iters_per_sync > 0 ? p.iters_per_sync : 4;
        require(p.dense_max_rows >= 0 && p.dense_max_rows <= 16384, "dense_max_rows must be in [0, 16384]");
        c->prm.dense_max_rows = p.dense_max_rows;
        require(c->prm.tolerance > 0 && c->prm.max_iters > 0, "tolerance and max_iters must be positive");
        int least = 0, greatest = 0;
        CUNIBS_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUNIBS_CHECK(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, greatest));
        CUNIBS_CHECK(cudaStreamCreateWithPriority(&c->prep, cudaStreamNonBlocking, least));
        CUNIBS_CHECK(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device));
        CUNIBS_CHECK(cudaEventCreateWithFlags(&c->ev_main, cudaEventDisableTiming));
        CUNIBS_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&c->h_coil_flag), sizeof(int), cudaHostAllocDefault));
        CUNIBS_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&c->staging), sizeof(Staging), cudaHostAllocDefault));
        for (BlockSlot& sl : c->slots) {
            CUNIBS_CHECK(cudaEventCreateWithFlags(&sl.prepared, cudaEventDisableTiming));
            CUNIBS_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&sl.h_deg), sizeof(int) * kMaxBlock,
                                       cudaHostAllocDefault));
            CUNIBS_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&sl.h_near), sizeof(int) * kMaxBlock,
                                       cudaHostAllocDefault));
        }
        {
            double lo[3] = {nodes_mm[0], nodes_mm[1], nodes_mm[2]}, hi[3] = {lo[0], lo[1], lo[2]};
            for (int i = 1; i < n_nodes; ++i)
                for (int a = 0; a < 3; ++a) {
                    lo[a] = std::min(lo[a], nodes_mm[3 * static_cast<long>(i) + a]);
                    hi[a] = std::max(hi[a], nodes_mm[3 * static_cast<long>(i) + a]);
                }
            double r2 = 0.0;
            for (int i = 0; i < n_nodes; ++i) {
                double d2 = 0.0;
                for (int a = 0; a < 3; ++a) {
                    const double d = nodes_mm[3 * static_cast<long>(i) + a] - 0.5 * (lo[a] + hi[a]);
                    d2 += d * d;
                }
                r2 = std::max(r2, d2);
            }
            c->mesh_rho_m = std::sqrt(r2) * 1e-3;
        }
        build_mesh(c->mesh, nodes_mm, n_nodes, tet_nodes, tet_tags, n_tets, skin_tris, n_skin, c->stream);
        c->rebuild_hierarchy();
        *out = c.release();
    });
}

int cunibs_context_destroy(cunibs_context* ctx) {
    return guarded([&] {
        if (!ctx) return;
        DeviceGuard dg(ctx->device);
        CUNIBS_CHECK(cudaStreamSynchronize(ctx->prep));
        CUNIBS_CHECK(cudaStreamSynchronize(ctx->stream));
        delete ctx;
    });
}

int cunibs_context_info(const cunibs_context* c, cunibs_info* out) {
    return guarded([&] {
        require(c && out, "NULL argument");
        out->n_nodes = c->mesh.n_nodes;
        out->n_tets = c->mesh.n_tets;
        out->n_skin = c->mesh.n_skin;
        out->n_gray_matter = c->mesh.n_gm;
        out->stiffness_nnz = c->mesh.k_nnz;
        out->ground_node = c->mesh.ground;
        out->n_levels = static_cast<int>(c->hier.levels.size());
        out->coarse_rows = c->hier.nc;
        out->vcycle_levels = c->hier.vcycle_levels;
        out->bottom_rows = c->hier.bottom_n;
        out->hierarchy_builds = c->hierarchy_builds;
    });
}

int cunibs_context_mesh(const cunibs_context* c, double* nodes_mm, int* tet_nodes, int* tet_tags, int* skin_tris,
                        int* node_perm, int* tet_perm) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        DeviceGuard dg(c->device);
        const Mesh& m = c->mesh;
        cudaStream_t s = c->stream;
        copy_out(nodes_mm, m.nodes.get(), sizeof(double) * 3 * m.n_nodes, cudaMemcpyDeviceToHost, s);
        copy_out(tet_nodes, m.tets.get(), sizeof(int) * 4 * static_cast<std::size_t>(m.n_tets), cudaMemcpyDeviceToHost, s);
        copy_out(tet_tags, m.tags.get(), sizeof(int) * m.n_tets, cudaMemcpyDeviceToHost, s);
        copy_out(skin_tris, m.skin.get(), sizeof(int) * 3 * m.n_skin, cudaMemcpyDeviceToHost, s);
        copy_out(node_perm, m.node_perm.get(), sizeof(int) * m.n_nodes, cudaMemcpyDeviceToHost, s);
        copy_out(tet_perm, m.tet_perm.get(), sizeof(int) * m.n_tets, cudaMemcpyDeviceToHost, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_levels(const cunibs_context* c, int* sizes, int cap) {
    return guarded([&] {
        require(c && sizes, "NULL argument");
        const std::size_t n = c->hier.sizes.size();
        require(cap >= static_cast<int>(n), "sizes buffer too small");
        for (std::size_t i = 0; i < n; ++i) sizes[i] = c->hier.sizes[i];
    });
}

int cunibs_solve_block(cunibs_context* c, const double* dip_pos_m, const double* dip_moment, int n_dip,
                       const double* centers_mm, const double* handles_mm, const double* dists_mm, int k, double didt,
                       const cunibs_solve_opts* opts, cunibs_block_out* out) {
    return guarded([&] {
        require(c && out, "NULL argument");
        require(dip_pos_m && dip_moment && centers_mm && handles_mm && dists_mm, "input arrays must not be NULL");
        require(out->transforms && out->summary, "out->transforms and out->summary are required");
        DeviceGuard dg(c->device);
        const long long t = prepare_block(c, dip_pos_m, dip_moment, n_dip, centers_mm, handles_mm, dists_mm, k, didt,
                                          opts, true, false);
        SolveStats st;
        const PendingBlock pb = finish_block(c, t, st, out->E != nullptr);
        block_outputs_host(c, pb, st, out);
    });
}

int cunibs_solve_block_device(cunibs_context* c, const double* dip_pos_m, const double* dip_moment, int n_dip,
                              const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
                              double didt, const cunibs_solve_opts* opts, cunibs_block_out* out) {
    return guarded([&] {
        require(c && out, "NULL argument");
        require(out->transforms && out->summary, "out->transforms and out->summary are required");
        DeviceGuard dg(c->device);
        const long long t = prepare_block(c, dip_pos_m, dip_moment, n_dip, centers_mm, handles_mm, dists_mm, k, didt,
                                          opts, false, false);
        SolveStats st;
        const PendingBlock pb = finish_block(c, t, st, out->E != nullptr);
        block_outputs_device(c, pb, st, out);
    });
}

int cunibs_submit_block(cunibs_context* c, const double* dip_pos_m, const double* dip_moment, int n_dip,
                        const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
                        double didt, const cunibs_solve_opts* opts, long long* ticket) {
    return guarded([&] {
        require(c && ticket, "NULL argument");
        require(dip_pos_m && dip_moment && centers_mm && handles_mm && dists_mm, "input arrays must not be NULL");
        DeviceGuard dg(c->device);
        *ticket = prepare_block(c, dip_pos_m, dip_moment, n_dip, centers_mm, handles_mm, dists_mm, k, didt, opts,
                                true, true);
    });
}

int cunibs_finish_block(cunibs_context* c, long long ticket, cunibs_block_out* out) {
    return guarded([&] {
        require(c && out, "NULL argument");
        require(out->transforms && out->summary, "out->transforms and out->summary are required");
        DeviceGuard dg(c->device);
        SolveStats st;
        const PendingBlock pb = finish_block(c, ticket, st, out->E != nullptr);
        block_outputs_host(c, pb, st, out);
    });
}

int cunibs_submit_block_device(cunibs_context* c, const double* dip_pos_m, const double* dip_moment, int n_dip,
                               const double* centers_mm, const double* handles_mm, const double* dists_mm, int k,
                               double didt, const cunibs_solve_opts* opts, long long* ticket) {
    return guarded([&] {
        require(c && ticket, "NULL argument");
        DeviceGuard dg(c->device);
        *ticket = prepare_block(c, dip_pos_m, dip_moment, n_dip, centers_mm, handles_mm, dists_mm, k, didt, opts,
                                false, true);
    });
}

int cunibs_finish_block_device(cunibs_context* c, long long ticket, cunibs_block_out* out) {
    return guarded([&] {
        require(c && out, "NULL argument");
        require(out->transforms && out->summary, "out->transforms and out->summary are required");
        DeviceGuard dg(c->device);
        SolveStats st;
        const PendingBlock pb = finish_block(c, ticket, st, out->E != nullptr);
        block_outputs_device(c, pb, st, out);
    });
}

int cunibs_cancel_block(cunibs_context* c, long long ticket) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        auto it = c->pending.begin();
        while (it != c->pending.end() && it->ticket != ticket) ++it;
        if (it == c->pending.end()) fail(kEInval, "no submitted block with ticket " + std::to_string(ticket));
        // The slot's buffers are next written on the preparation stream, behind this block's work.
        c->pending.erase(it);
    });
}

int cunibs_context_pending(const cunibs_context* c, int* n) {
    return guarded([&] {
        require(c && n, "NULL argument");
        *n = static_cast<int>(c->pending.size());
    });
}

int cunibs_context_phase_times(const cunibs_context* c, double* out) {
    return guarded([&] {
        require(c != nullptr && out != nullptr, "NULL argument");
        std::copy(c->phase_ms, c->phase_ms + 8, out);
    });
}

int cunibs_context_set_coil_table(cunibs_context* c, int mode, double near_mm, double step) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        require(mode == 0 || mode == 1, "mode must be 0 (direct sums) or 1 (coil table)");
        require(near_mm > 0.0 && near_mm <= 1000.0, "near_mm must be in (0, 1000]");
        require(step > 0.0 && step <= 0.5, "step must be in (0, 0.5]");
        c->table_mode = mode;
        c->table_near_m = near_mm * 1e-3;
        c->table_step = step;
    });
}

int cunibs_context_coil_table_info(const cunibs_context* c, double* out) {
    return guarded([&] {
        require(c != nullptr && out != nullptr, "NULL argument");
        const CoilTable& tb = c->coil_table;
        out[0] = c->table_mode;
        out[1] = tb.valid ? 1.0 : 0.0;
        out[2] = static_cast<double>(tb.built ? tb.points : 0);
        out[3] = tb.built ? tb.n_layers : 0;
        out[4] = tb.check_rel;
        out[5] = tb.builds;
        out[6] = static_cast<double>(c->last_near);
        out[7] = static_cast<double>(c->last_near_of);
    });
}

int cunibs_context_set_overlap(cunibs_context* c, int blocks_per_sm) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        require(blocks_per_sm >= 1 && blocks_per_sm <= 16, "blocks_per_sm must be in [1, 16]");
        c->overlap_blocks_per_sm = blocks_per_sm;
    });
}

int cunibs_context_set_conductivity(cunibs_context* c, const double* sigma_by_tag) {
    return guarded([&] {
        require(c && sigma_by_tag, "NULL argument");
        require(!c->study, "a conductivity study is open: its draws set the conductivities until cunibs_sigma_end");
        for (int t = 1; t <= 10; ++t) require(sigma_by_tag[t] > 0.0, "conductivities must be positive");
        require(c->pending.empty(), "finish the submitted blocks first");
        DeviceGuard dg(c->device);
        assemble_stiffness(c->mesh, sigma_by_tag, c->stream);
        c->rebuild_hierarchy();
    });
}

int cunibs_context_set_conductivity_keep_coarse(cunibs_context* c, const double* sigma_by_tag) {
    return guarded([&] {
        require(c && sigma_by_tag, "NULL argument");
        require(!c->study, "a conductivity study is open: its draws set the conductivities until cunibs_sigma_end");
        for (int t = 1; t <= 10; ++t) require(sigma_by_tag[t] > 0.0, "conductivities must be positive");
        require(c->pending.empty(), "finish the submitted blocks first");
        DeviceGuard dg(c->device);
        assemble_stiffness(c->mesh, sigma_by_tag, c->stream);
        c->keep_coarse_values();
    });
}

int cunibs_sigma_begin(cunibs_context* c, const double* dip_pos_m, const double* dip_moment, int n_dip,
                       const double* centers_mm, const double* handles_mm, const double* dists_mm, int k, double didt,
                       const cunibs_solve_opts* opts, const double* sigma_nominal, const int* tags, int n_tags,
                       double sensitivity_tol, int* basis_rank) {
    return guarded([&] {
        require(c && sigma_nominal && tags, "NULL argument");
        require(dip_pos_m && dip_moment && centers_mm && dists_mm, "input arrays must not be NULL");
        require(!c->study, "a conductivity study is already open");
        require(c->pending.empty(), "finish the submitted blocks first");
        require(n_tags >= 1 && n_tags <= kSigmaMaxTags, "between 1 and 10 perturbed tissues");
        require(sensitivity_tol > 0.0 && sensitivity_tol < 1.0, "sensitivity_tol must be in (0, 1)");
        require(!(opts && opts->warm_start), "a conductivity study starts its draws from its own guess: warm_start must be 0");
        for (int t = 1; t <= 10; ++t)
            require(sigma_nominal[t] > 0.0 && std::isfinite(sigma_nominal[t]), "nominal conductivities must be positive");
        auto st = std::make_unique<SigmaStudy>();
        SigmaSlots slots{};
        for (int& v : slots.slot) v = -1;
        for (int a = 0; a < n_tags; ++a) {
            require(tags[a] >= 1 && tags[a] <= 10, "perturbed tags must be in [1, 10]");
            require(slots.slot[tags[a]] < 0, "perturbed tags must be distinct");
            slots.slot[tags[a]] = a;
            st->tags[a] = tags[a];
        }
        const int P = st->P = n_tags;
        std::copy(sigma_nominal, sigma_nominal + 11, st->nominal);
        DeviceGuard dg(c->device);
        Mesh& m = c->mesh;
        cudaStream_t s = c->stream;
        const auto t_begin = std::chrono::steady_clock::now();
        auto phase = [&](int i) {
            c->phase_ms[i] =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
        };
        for (double& v : c->phase_ms) v = 0.0;
        // The context at the nominal conductivities, its coarse levels kept.
        assemble_stiffness(m, st->nominal, s);
        c->keep_coarse_values();
        phase(0);
        require(!c->hier.levels.empty(), "the operator is too small for a conductivity study (it has no AMG level)");
        const Level& L0 = c->hier.levels[0];
        st->nnz = L0.a.nnz;
        // Operator components on the grounded pattern (assembly.py:99-125): the unperturbed tissues at
        // nominal, then each perturbed tissue at unit conductivity.
        st->comp.resize(static_cast<std::size_t>(1 + P) * st->nnz);
        std::vector<double> tables(11 * static_cast<std::size_t>(1 + P), 0.0);
        for (int t = 1; t < 11; ++t) tables[t] = slots.slot[t] < 0 ? st->nominal[t] : 0.0;
        for (int a = 0; a < P; ++a) tables[11 * (1 + a) + st->tags[a]] = 1.0;
        assemble_reduced_values(m, tables.data(), 1 + P, L0.a, st->comp.get(), s);
        // The components must give back the nominal operator (the gate of assembly.py:126-131).
        {
            SigmaWeights w{};
            for (int a = 0; a < P; ++a) w.w[a] = st->nominal[st->tags[a]];
            DevArray<double> recon(st->nnz);
            sigma_combine(st->comp.get(), P, st->nnz, w, recon.get(), s);
            const double rel = sigma_relative_difference(recon.get(), L0.a.val.get(), st->nnz, s);
            if (!(rel <= 1e-10))
                fail(kEInternal, "conductivity decomposition mismatch (relative difference " + std::to_string(rel) + ")");
        }
        phase(1);
        // The block's coil field, kept in its slot for every draw, and the nominal solution.
        const long long ticket = prepare_block(c, dip_pos_m, dip_moment, n_dip, centers_mm, handles_mm, dists_mm, k,
                                               didt, opts, true, false, true);
        st->slot = c->pending.back().slot;
        CUNIBS_CHECK(cudaStreamSynchronize(c->prep));
        phase(2);
        SolveStats ss;
        const PendingBlock pb = finish_block(c, ticket, ss, false);
        phase(3);
        st->k = pb.k;
        st->K = pb.K;
        st->has_handles = pb.has_handles;
        st->has_opts = pb.has_opts;
        st->opts = pb.opts;
        const int K = st->K, n_red = m.n_nodes - 1;
        const std::size_t npk = static_cast<std::size_t>(n_red) * P * K;
        // The right-hand side is linear in sigma like the operator (run.py:59-84): one block of
        // right-hand sides per component table, so a draw's is one combination.
        {
            const BlockSlot& sl0 = c->slots[st->slot];
            DevArray<double> td;
            td.upload(tables.data(), tables.size(), s);
            DevArray<float> wts(static_cast<std::size_t>(1 + P) * m.n_tets);
            sigma_element_weights(m, td.get(), 1 + P, wts.get(), s);
            const std::size_t nk = static_cast<std::size_t>(n_red) * K;
            st->rhs.resize((1 + P) * nk);
            for (int t = 0; t <= P; ++t)
                rhs_block(m, sl0.dadt_elm.get(), st->k, K, st->rhs.get() + t * nk, s,
                          wts.get() + static_cast<std::size_t>(t) * m.n_tets);
            CUNIBS_CHECK(cudaStreamSynchronize(s));  // td and wts leave scope
        }
        phase(4);
        st->x_nom.resize(static_cast<std::size_t>(n_red) * K);
        CUNIBS_CHECK(cudaMemcpyAsync(st->x_nom.get(), c->X.get(), sizeof(double) * n_red * K, cudaMemcpyDeviceToDevice, s));
        // Sensitivity right-hand sides c_t = b_t - A_t x_nom, and which are nonzero (a tissue with no
        // element gives none).
        const BlockSlot& sl = c->slots[st->slot];
        DevArray<double> C(npk);
        sigma_sens_rhs(m, st->x_nom.get(), sl.dadt_elm.get(), st->k, K, slots, P, C.get(), s);
        const std::vector<double> cc = sigma_gram(C.get(), C.get(), n_red, P, K, s);
        std::vector<int> active(static_cast<std::size_t>(P) * K, 0);
        std::vector<std::pair<int, int>> cols;
        for (int j = 0; j < st->k; ++j)
            for (int a = 0; a < P; ++a)
                if (cc[(static_cast<std::size_t>(j) * P + a) * P + a] > 0.0) {
                    active[static_cast<std::size_t>(j) * P + a] = 1;
                    cols.emplace_back(a, j);
                }
        phase(5);
        // Sensitivities s_t = A_nom^-1 c_t to a loose tolerance (run.py:44-49: they only span the
        // guess's subspace; every draw is still solved to the full tolerance), in blocks as wide as
        // the solver's workspace already is (growing it would reallocate it and drop its graphs).
        st->S.resize(npk);
        st->S.zero(s);
        if (!cols.empty()) {
            Params sp = resolve(c, opts);
            sp.tolerance = sensitivity_tol;
            const int W = std::max(K, std::min(16, solver_width_capacity(*c->solver)));
            DevArray<double> Bw(static_cast<std::size_t>(n_red) * W), Xw(static_cast<std::size_t>(n_red) * W);
            for (std::size_t q0 = 0; q0 < cols.size(); q0 += W) {
                SigmaColumns cm{};
                cm.count = static_cast<int>(std::min<std::size_t>(W, cols.size() - q0));
                for (int l = 0; l < cm.count; ++l) {
                    cm.a[l] = cols[q0 + l].first;
                    cm.j[l] = cols[q0 + l].second;
                }
                sigma_pack(C.get(), n_red, P, K, cm, W, Bw.get(), s);
                SolveStats sw;
                solver_solve(*c->solver, Bw.get(), Xw.get(), cm.count, W, sp, s, sw);
                sigma_unpack(Xw.get(), n_red, P, K, cm, W, st->S.get(), s);
            }
        }
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        phase(6);
        // Per placement: the A_nom-Gram of its sensitivities and their products with the c_t give
        // the map from a draw's conductivity change to its subspace coefficients.
        DevArray<double> AS(npk);
        sigma_spmv(L0.a, st->S.get(), P * K, AS.get(), s);
        const std::vector<double> G = sigma_gram(st->S.get(), AS.get(), n_red, P, K, s);
        const std::vector<double> H = sigma_gram(st->S.get(), C.get(), n_red, P, K, s);
        st->Z.assign(static_cast<std::size_t>(K) * P * P, 0.0);
        st->rank.assign(st->k, 0);
        const std::size_t pp = static_cast<std::size_t>(P) * P;
        for (int j = 0; j < st->k; ++j)
            st->rank[j] = sigma_coefficients(P, &G[j * pp], &H[j * pp], &active[static_cast<std::size_t>(j) * P],
                                             kSigmaRtol, &st->Z[j * pp]);
        if (basis_rank)
            for (int j = 0; j < st->k; ++j) basis_rank[j] = st->rank[j];
        c->study = std::move(st);
        phase(7);
    });
}

int cunibs_sigma_draw(cunibs_context* c, const double* sigma, cunibs_block_out* out, int* resetup) {
    return guarded([&] {
        require(c && sigma && out, "NULL argument");
        require(out->transforms && out->summary, "out->transforms and out->summary are required");
        require(c->study != nullptr, "no conductivity study is open (cunibs_sigma_begin)");
        SigmaStudy& st = *c->study;
        const int P = st.P, k = st.k, K = st.K;
        double table[11];
        std::copy(st.nominal, st.nominal + 11, table);
        SigmaWeights w{};
        double dsig[kSigmaMaxTags] = {};
        for (int a = 0; a < P; ++a) {
            require(sigma[a] > 0.0 && std::isfinite(sigma[a]), "conductivities must be positive");
            table[st.tags[a]] = sigma[a];
            w.w[a] = sigma[a];
            dsig[a] = sigma[a] - st.nominal[st.tags[a]];
        }
        SigmaDraw y{};
        if (st.guess_mode == 0) {
            for (int j = 0; j < k; ++j)
                for (int a = 0; a < P; ++a) {
                    double v = 0.0;
                    for (int t = 0; t < P; ++t) v += st.Z[(static_cast<std::size_t>(j) * P + a) * P + t] * dsig[t];
                    y.y[a * 16 + j] = v;
                }
        }
        DeviceGuard dg(c->device);
        Mesh& m = c->mesh;
        cudaStream_t s = c->stream;
        const int n_red = m.n_nodes - 1;
        // The draw's finest operator (K(sigma) = K_base + sum sigma_t K_t), its smoother weights and
        // the right-hand side weights; the coarse levels stay the nominal ones (run.py:244-247).
        sigma_combine(st.comp.get(), P, st.nnz, w, c->hier.levels[0].a.val.get(), s);
        refresh_finest_derived(c->hier, s);
        set_element_conductivity(m, table, s, false);  // the nominal table passed the check at begin
        BlockSlot& sl = c->slots[st.slot];
        sigma_combine(st.rhs.get(), P, static_cast<long>(n_red) * K, w, sl.B.get(), s);
        sl.X0.reserve(static_cast<std::size_t>(n_red) * K);
        if (st.guess_mode != 2) sigma_guess(st.x_nom.get(), st.S.get(), n_red, P, K, k, y, sl.X0.get(), s);
        auto queue = [&] {
            PendingBlock pb;
            pb.slot = st.slot;
            pb.k = k;
            pb.K = K;
            pb.has_handles = st.has_handles;
            pb.has_opts = st.has_opts;
            pb.opts = st.opts;
            pb.x0_given = st.guess_mode != 2;
            pb.ticket = c->next_ticket++;
            c->pending.push_back(pb);
            return pb.ticket;
        };
        auto nominal_hierarchy = [&] {
            assemble_stiffness(m, st.nominal, s);
            c->rebuild_hierarchy();
        };
        SolveStats ss;
        PendingBlock done;
        int redone = 0;
        try {
            done = finish_block(c, queue(), ss, out->E != nullptr);
        } catch (const Error& e) {
            if (e.code != kENoConv) throw;
            // The nominal coarse levels were too far from this draw: solve it against a hierarchy
            // of its own (run.py:356-366), then rebuild the nominal one.
            assemble_stiffness(m, table, s);
            c->rebuild_hierarchy();
            ss = SolveStats{};
            try {
                done = finish_block(c, queue(), ss, out->E != nullptr);
            } catch (...) {
                nominal_hierarchy();
                throw;
            }
            nominal_hierarchy();
            redone = 1;
        }
        block_outputs_host(c, done, ss, out);
        if (resetup) *resetup = redone;
    });
}

int cunibs_sigma_set_guess(cunibs_context* c, int mode) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        require(c->study != nullptr, "no conductivity study is open (cunibs_sigma_begin)");
        require(mode >= 0 && mode <= 2, "guess mode must be 0 (subspace), 1 (nominal potential) or 2 (zero)");
        c->study->guess_mode = mode;
    });
}

int cunibs_sigma_end(cunibs_context* c) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        if (!c->study) return;
        DeviceGuard dg(c->device);
        const std::unique_ptr<SigmaStudy> st = std::move(c->study);
        assemble_stiffness(c->mesh, st->nominal, c->stream);
        c->keep_coarse_values();
    });
}

int cunibs_sigma_coefficients(int n_tags, const double* gram, const double* proj, const int* active, double rtol,
                              double* coef, int* rank) {
    return guarded([&] {
        require(gram && proj && active && coef, "NULL argument");
        require(n_tags >= 1 && n_tags <= kSigmaMaxTags, "between 1 and 10 perturbed tissues");
        require(rtol >= 0.0 && rtol < 1.0, "rtol must be in [0, 1)");
        const int r = sigma_coefficients(n_tags, gram, proj, active, rtol, coef);
        if (rank) *rank = r;
    });
}

}  // extern "C"

// A target functional's adjoint state on one context (adm/reciprocity.py:119-245): the nodal
// reciprocity weights and, once sampled, the reciprocity field on a grid.
struct cunibs_adm {
    cunibs_context* ctx = nullptr;
    AdmDirections dirs{};
    DevArray<double> alpha;          // (n_tets) target weight per element
    DevArray<double> W;              // (n_dir, n_nodes, 3)
    std::vector<int> iterations;
    std::vector<double> relres;
    bool sampled = false;
    AdmGrid grid{};
    DevArray<float> Q;               // (n_dir, n_grid, 3)
    DevArray<double> pos, mom, T, E; // evaluation workspace
    // Sampling workspace, grown on demand and kept, so that a repeated sampling allocates nothing:
    // the grid points, the sources' centred positions, their packed records and frames, and the
    // per-chunk partial fields.
    DevArray<double> q_pts, q_src, q_T;
    DevArray<unsigned char> q_packed;
    DevArray<float> q_part;
    DevArray<unsigned long long> bad;
};

namespace {

// Reciprocity N-body sources: the nodes centred on center_mm with the weights of each direction as
// moments, packed like rotated coil dipoles, and the matching (identity rotation, centre) frames.
void adm_sources(cunibs_adm* a, const double* center_mm, DevArray<unsigned char>& packed, DevArray<double>& Td,
                 cudaStream_t s) {
    const Mesh& m = a->ctx->mesh;
    const int nd = a->dirs.n;
    DevArray<double>& src = a->q_src;
    src.reserve(3 * static_cast<std::size_t>(m.n_nodes));
    adm_centred_nodes(m, center_mm, src.get(), s);
    std::vector<double> h(16 * static_cast<std::size_t>(nd), 0.0);
    for (int d = 0; d < nd; ++d) {
        double* t = &h[16 * d];
        t[0] = t[5] = t[10] = t[15] = 1.0;
        t[3] = center_mm[0];
        t[7] = center_mm[1];
        t[11] = center_mm[2];
    }
    Td.reserve(h.size());
    CUNIBS_CHECK(cudaMemcpyAsync(Td.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    const std::size_t rec = packed_dipole_bytes();
    packed.reserve(rec * m.n_nodes * nd);
    for (int d = 0; d < nd; ++d)
        prep_dipoles(src.get(), a->W.get() + 3 * static_cast<std::size_t>(m.n_nodes) * d, m.n_nodes, Td.get() + 16 * d,
                     1, packed.get() + rec * m.n_nodes * d, s);
    CUNIBS_CHECK(cudaStreamSynchronize(s));  // h leaves scope
}

void adm_inputs(cunibs_adm* a, const double* dip_pos_m, const double* dip_moment, int n_dip, const double* transforms,
                int P, cudaStream_t s) {
    require(dip_pos_m && dip_moment && transforms, "input arrays must not be NULL");
    require(n_dip >= 1 && P >= 1, "need at least one dipole and one placement");
    for (long i = 0; i < 16L * P; ++i) require(std::isfinite(transforms[i]), "transforms must be finite");
    a->pos.upload(dip_pos_m, 3 * static_cast<std::size_t>(n_dip), s);
    a->mom.upload(dip_moment, 3 * static_cast<std::size_t>(n_dip), s);
    a->T.upload(transforms, 16 * static_cast<std::size_t>(P), s);
    a->E.reserve(static_cast<std::size_t>(P) * a->dirs.n);
}

}  // namespace

extern "C" {

int cunibs_adm_create(cunibs_context* c, const int* elem_idx, const double* weights, int n_elem,
                      const double* directions, int n_dir, double tolerance, int max_iters, int* iterations,
                      double* relres, cunibs_adm** out) {
    return guarded([&] {
        require(c && elem_idx && weights && directions && out, "NULL argument");
        *out = nullptr;
        require(n_elem >= 1, "the target needs at least one element");
        require(n_dir >= 1 && n_dir <= kAdmMaxDir, "between 1 and 3 adjoint directions");
        require(tolerance > 0.0 && tolerance < 1.0 && max_iters >= 1, "tolerance in (0, 1) and max_iters >= 1");
        require(!c->study, "a conductivity study is open: end it first");
        require(c->pending.empty(), "finish the submitted blocks first");
        Mesh& m = c->mesh;
        std::vector<double> alpha(m.n_tets, 0.0);
        for (int i = 0; i < n_elem; ++i) {
            require(elem_idx[i] >= 0 && elem_idx[i] < m.n_tets, "target element index out of range");
            require(std::isfinite(weights[i]), "target weights must be finite");
            alpha[elem_idx[i]] += weights[i];
        }
        auto a = std::make_unique<cunibs_adm>();
        a->ctx = c;
        a->dirs.n = n_dir;
        for (int d = 0; d < n_dir; ++d) {
            double nrm = 0.0;
            for (int x = 0; x < 3; ++x) {
                a->dirs.e[d][x] = directions[3 * d + x];
                nrm += directions[3 * d + x] * directions[3 * d + x];
            }
            require(nrm > 0.0 && std::isfinite(nrm), "directions must be finite and non-zero");
        }
        DeviceGuard dg(c->device);
        cudaStream_t s = c->stream;
        a->alpha.upload(alpha.data(), alpha.size(), s);
        const int K = n_dir == 1 ? 1 : (n_dir == 2 ? 2 : 4);
        const int n_red = m.n_nodes - 1;
        DevArray<double> B(static_cast<std::size_t>(n_red) * K), X(static_cast<std::size_t>(n_red) * K);
        adm_adjoint_rhs(m, a->alpha.get(), a->dirs, K, B.get(), s);
        // All directions in one block solve (reciprocity.py:131-141 solves them one at a time).
        Params prm = c->prm;
        prm.tolerance = tolerance;
        prm.max_iters = max_iters;
        SolveStats st;
        solver_solve(*c->solver, B.get(), X.get(), n_dir, K, prm, s, st);
        bool missed = false;
        for (int d = 0; d < n_dir; ++d) missed = missed || !(st.col_rel[d] <= tolerance);
        if (missed) {
            Params retry = prm;
            retry.precision = kPlainFp64;
            SolveStats st2;
            solver_solve(*c->solver, B.get(), X.get(), n_dir, K, retry, s, st2, X.get());
            for (int d = 0; d < n_dir; ++d) {
                st.col_iters[d] += st2.col_iters[d];
                st.col_rel[d] = st2.col_rel[d];
                if (!(st2.col_rel[d] <= tolerance))
                    fail(kENoConv, "adjoint solve did not converge (direction " + std::to_string(d) + "): relative "
                                       "residual " + std::to_string(st2.col_rel[d]) + " > tolerance " +
                                       std::to_string(tolerance));
            }
        }
        a->W.resize(3 * static_cast<std::size_t>(m.n_nodes) * n_dir);
        adm_node_weights(m, X.get(), K, a->alpha.get(), a->dirs, a->W.get(), s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        a->iterations.assign(st.col_iters.begin(), st.col_iters.end());
        a->relres.assign(st.col_rel.begin(), st.col_rel.end());
        for (int d = 0; d < n_dir; ++d) {
            if (iterations) iterations[d] = a->iterations[d];
            if (relres) relres[d] = a->relres[d];
        }
        *out = a.release();
    });
}

int cunibs_adm_destroy(cunibs_adm* a) {
    return guarded([&] {
        if (!a) return;
        DeviceGuard dg(a->ctx->device);
        CUNIBS_CHECK(cudaStreamSynchronize(a->ctx->stream));
        delete a;
    });
}

int cunibs_adm_node_weights(const cunibs_adm* a, double* out) {
    return guarded([&] {
        require(a && out, "NULL argument");
        DeviceGuard dg(a->ctx->device);
        a->W.download(out, a->W.size(), a->ctx->stream);
        CUNIBS_CHECK(cudaStreamSynchronize(a->ctx->stream));
    });
}

int cunibs_adm_sample(cunibs_adm* a, const double* origin_mm, const double* spacing_mm, const int* shape) {
    return guarded([&] {
        require(a && origin_mm && spacing_mm && shape, "NULL argument");
        AdmGrid gr{};
        long long n_grid = 1;
        for (int x = 0; x < 3; ++x) {
            require(std::isfinite(origin_mm[x]), "grid origin must be finite");
            require(spacing_mm[x] > 0.0 && std::isfinite(spacing_mm[x]), "grid spacing must be positive");
            require(shape[x] >= 1 && shape[x] <= (1 << 16), "grid shape must be in [1, 65536] per axis");
            gr.origin_mm[x] = origin_mm[x];
            gr.spacing_mm[x] = spacing_mm[x];
            gr.shape[x] = shape[x];
            n_grid *= shape[x];
        }
        require(n_grid <= (1LL << 28), "at most 2^28 grid points");
        DeviceGuard dg(a->ctx->device);
        cudaStream_t s = a->ctx->stream;
        double center[3];
        for (int x = 0; x < 3; ++x) center[x] = gr.origin_mm[x] + 0.5 * gr.spacing_mm[x] * (gr.shape[x] - 1);
        DevArray<double>& pts = a->q_pts;
        DevArray<double>& Td = a->q_T;
        DevArray<unsigned char>& packed = a->q_packed;
        pts.reserve(3 * static_cast<std::size_t>(n_grid));
        adm_grid_points(gr, pts.get(), s);
        adm_sources(a, center, packed, Td, s);
        a->sampled = false;
        a->Q.resize(3 * static_cast<std::size_t>(n_grid) * a->dirs.n);
        // Q_d on the grid: the coil-field N-body with the mesh nodes as sources (reciprocity.py:183-213),
        // every direction in one pass over the sources.
        dadt_nodes_shared(pts.get(), static_cast<int>(n_grid), reinterpret_cast<const float*>(packed.get()),
                          a->ctx->mesh.n_nodes, Td.get(), a->dirs.n, 1.0, a->Q.get(), s, a->q_part);
        CUNIBS_LAUNCH_CHECK("reciprocity field");
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        a->grid = gr;
        a->sampled = true;
    });
}

int cunibs_adm_qfield(const cunibs_adm* a, float* out, long long cap) {
    return guarded([&] {
        require(a && out, "NULL argument");
        require(a->sampled, "the reciprocity field has not been sampled (cunibs_adm_sample)");
        require(cap >= static_cast<long long>(a->Q.size()), "output buffer too small");
        DeviceGuard dg(a->ctx->device);
        a->Q.download(out, a->Q.size(), a->ctx->stream);
        CUNIBS_CHECK(cudaStreamSynchronize(a->ctx->stream));
    });
}

int cunibs_adm_evaluate(cunibs_adm* a, const double* dip_pos_m, const double* dip_moment, int n_dip,
                        const double* transforms, int P, double didt, double* E) {
    return guarded([&] {
        require(a && E, "NULL argument");
        require(a->sampled, "the reciprocity field has not been sampled (cunibs_adm_sample)");
        DeviceGuard dg(a->ctx->device);
        cudaStream_t s = a->ctx->stream;
        adm_inputs(a, dip_pos_m, dip_moment, n_dip, transforms, P, s);
        a->bad.resize(3);
        CUNIBS_CHECK(cudaMemsetAsync(a->bad.get(), 0xFF, 3 * sizeof(unsigned long long), s));
        adm_evaluate(a->Q.get(), a->dirs.n, a->grid, a->pos.get(), a->mom.get(), n_dip, a->T.get(), P, didt,
                     a->E.get(), a->bad.get(), s);
        unsigned long long bad[3];
        a->bad.download(bad, 3, s);
        a->E.download(E, static_cast<std::size_t>(P) * a->dirs.n, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        for (int x = 0; x < 3; ++x) {
            if (bad[x] == ULLONG_MAX) continue;
            // The first axis with a dipole off the grid, and its first such sample (evaluate.py:49-79).
            const long long p = static_cast<long long>(bad[x] / n_dip), j = static_cast<long long>(bad[x] % n_dip);
            const double* Tp = transforms + 16 * p;
            const double pos = Tp[4 * x] * dip_pos_m[3 * j] * 1e3 + Tp[4 * x + 1] * dip_pos_m[3 * j + 1] * 1e3 +
                               Tp[4 * x + 2] * dip_pos_m[3 * j + 2] * 1e3 + Tp[4 * x + 3];
            const double lo = a->grid.origin_mm[x], hi = lo + a->grid.spacing_mm[x] * (a->grid.shape[x] - 1);
            char msg[512];
            std::snprintf(msg, sizeof(msg),
                          "A coil dipole falls outside the reciprocity grid: sample %lld of %d on axis %d (%c), dipole "
                          "at %.3f mm against a grid spanning [%.3f, %.3f] mm (%.3f mm outside). Sample the "
                          "reciprocity field on a grid that covers it: widen its coverage or margin, or evaluate at "
                          "the coil distance the grid was built for.",
                          p, P, x, "xyz"[x], pos, lo, hi, pos < lo ? lo - pos : pos - hi);
            fail(kEInval, msg);
        }
    });
}

int cunibs_adm_evaluate_exact(cunibs_adm* a, const double* dip_pos_m, const double* dip_moment, int n_dip,
                              const double* transforms, int P, double didt, const double* center_mm, double* E) {
    return guarded([&] {
        require(a && E, "NULL argument");
        require(static_cast<long long>(P) * n_dip <= (1LL << 26), "at most 2^26 placed dipoles per call");
        DeviceGuard dg(a->ctx->device);
        cudaStream_t s = a->ctx->stream;
        adm_inputs(a, dip_pos_m, dip_moment, n_dip, transforms, P, s);
        const double zero[3] = {0.0, 0.0, 0.0};
        const double* c0 = center_mm ? center_mm : zero;
        const std::size_t n_pts = static_cast<std::size_t>(P) * n_dip;
        DevArray<double> s_mm(3 * n_pts), m_all(3 * n_pts), Td;
        DevArray<float> Qx(3 * n_pts * a->dirs.n);
        adm_placed_dipoles(a->pos.get(), a->mom.get(), n_dip, a->T.get(), P, s_mm.get(), m_all.get(), s);
        DevArray<unsigned char> packed;
        adm_sources(a, c0, packed, Td, s);
        // Q evaluated at every placed dipole (no grid): evaluate.py:158-193.
        dadt_nodes_raw(s_mm.get(), static_cast<int>(n_pts), reinterpret_cast<const float*>(packed.get()),
                       a->ctx->mesh.n_nodes, Td.get(), a->dirs.n, 1.0, Qx.get(), s);
        CUNIBS_LAUNCH_CHECK("reciprocity field at dipoles");
        adm_exact_reduce(Qx.get(), a->dirs.n, P, n_dip, m_all.get(), didt, a->E.get(), s);
        a->E.download(E, static_cast<std::size_t>(P) * a->dirs.n, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_array(const cunibs_context* c, const char* name, int level, void* out, long long cap,
                         long long* len) {
    return guarded([&] {
        require(c && name && len, "NULL argument");
        DeviceGuard dg(c->device);
        const Mesh& m = c->mesh;
        const Hierarchy& h = c->hier;
        const std::string n(name);
        const void* src = nullptr;
        std::size_t count = 0, elem = 4;
        std::size_t pitch = 0, row_bytes = 0;  // a dense matrix stored with padded rows
        auto pick = [&](const void* p, std::size_t cnt, std::size_t es) {
            src = p;
            count = cnt;
            elem = es;
        };
        const bool lv_ok = level >= 0 && level < static_cast<int>(h.levels.size());
        if (n == "node_perm") pick(m.node_perm.get(), m.n_nodes, 4);
        else if (n == "tet_perm") pick(m.tet_perm.get(), m.n_tets, 4);
        else if (n == "tet_nodes") pick(m.tets.get(), 4 * static_cast<std::size_t>(m.n_tets), 4);
        else if (n == "tet_tags") pick(m.tags.get(), m.n_tets, 4);
        else if (n == "skin_tris") pick(m.skin.get(), 3 * static_cast<std::size_t>(m.n_skin), 4);
        else if (n == "n2c_ptr") pick(m.n2c_ptr.get(), m.n_nodes + 1, 4);
        else if (n == "n2c_idx") pick(m.n2c_idx.get(), 4 * static_cast<std::size_t>(m.n_tets), 4);
        else if (n == "stiff_ptr") pick(m.k_ptr.get(), m.n_nodes + 1, 4);
        else if (n == "stiff_col") pick(m.k_col.get(), m.k_nnz, 4);
        else if (n == "gm_index") pick(m.gm_index.get(), m.n_gm, 4);
        else if (n == "nodes_mm") pick(m.nodes.get(), 3 * static_cast<std::size_t>(m.n_nodes), 8);
        else if (n == "g") pick(m.g.get(), 12 * static_cast<std::size_t>(m.n_tets), 8);
        else if (n == "vols") pick(m.vols.get(), m.n_tets, 8);
        else if (n == "bary") pick(m.bary.get(), 3 * static_cast<std::size_t>(m.n_tets), 8);
        else if (n == "stiff_val") pick(m.k_val.get(), m.k_nnz, 8);
        else if (n == "skin_normals") pick(m.skin_normals.get(), 3 * static_cast<std::size_t>(m.n_skin), 8);
        else if (n == "coarse_ptr") pick(h.coarse.ptr.get(), h.nc + 1, 4);
        else if (n == "coarse_col") pick(h.coarse.col.get(), h.coarse.nnz, 4);
        else if (n == "coarse_val") pick(h.coarse.val.get(), h.coarse.nnz, 8);
        else if (n == "coarse_inv") {
            pick(h.coarse_inv.get(), static_cast<std::size_t>(h.nc) * h.nc, 8);
            pitch = static_cast<std::size_t>(dense_ld(h.nc)) * 8;
            row_bytes = static_cast<std::size_t>(h.nc) * 8;
        } else if (n == "bottom_inv") {  // the dense inverse the V-cycle ends in (bottom_rows square)
            const bool early = h.vcycle_levels < static_cast<int>(h.levels.size());
            pick(early ? h.level_inv.get() : h.coarse_inv.get(), static_cast<std::size_t>(h.bottom_n) * h.bottom_n, 8);
            pitch = static_cast<std::size_t>(dense_ld(h.bottom_n)) * 8;
            row_bytes = static_cast<std::size_t>(h.bottom_n) * 8;
        }
        else if (lv_ok && n == "a_ptr") pick(h.levels[level].a.ptr.get(), h.levels[level].n + 1, 4);
        else if (lv_ok && n == "a_col") pick(h.levels[level].a.col.get(), h.levels[level].a.nnz, 4);
        else if (lv_ok && n == "a_val") pick(h.levels[level].a.val.get(), h.levels[level].a.nnz, 8);
        else if (lv_ok && n == "agg") pick(h.levels[level].agg.get(), h.levels[level].n, 4);
        else if (lv_ok && n == "p_ptr") pick(h.levels[level].p.ptr.get(), h.levels[level].n + 1, 4);
        else if (lv_ok && n == "p_col") pick(h.levels[level].p.col.get(), h.levels[level].p.nnz, 4);
        else if (lv_ok && n == "p_val") pick(h.levels[level].p.val.get(), h.levels[level].p.nnz, 8);
        else if (lv_ok && n == "dinv") pick(h.levels[level].dinv.get(), h.levels[level].n, 8);
        else fail(kEInval, "unknown array name or level: " + n);
        *len = static_cast<long long>(count);
        if (out && count && pitch) {
            const std::size_t rows = std::min<std::size_t>(count, static_cast<std::size_t>(cap)) * elem / row_bytes;
            CUNIBS_CHECK(cudaMemcpy2D(out, row_bytes, src, pitch, row_bytes, rows, cudaMemcpyDeviceToHost));
        } else if (out && count) {
            const std::size_t nb = std::min<std::size_t>(count, static_cast<std::size_t>(cap)) * elem;
            CUNIBS_CHECK(cudaMemcpy(out, src, nb, cudaMemcpyDeviceToHost));
        }
    });
}

int cunibs_context_set_warmstart(cunibs_context* c, int depth, int hidden, int n_out, const void* const* weights,
                                 const float* const* biases, const float* feature_mean, const float* feature_std,
                                 const float* coef_mean, const float* coef_std, const void* basis) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        DeviceGuard dg(c->device);
        if (weights == nullptr) {
            c->warm.reset();
            return;
        }
        require(depth >= 1 && depth <= 16 && hidden >= 64 && hidden % 64 == 0 && n_out >= 1,
                "depth in [1, 16], hidden a positive multiple of 64, n_out >= 1");
        require(biases && feature_mean && feature_std && coef_mean && coef_std && basis, "NULL warm-start array");
        cudaStream_t s = c->stream;
        auto ws = std::make_unique<WarmStart>();
        ws->depth = depth;
        ws->hidden = hidden;
        ws->n_out = n_out;
        ws->n_out_pad = (n_out + 63) / 64 * 64;
        ws->n_red = c->mesh.n_nodes - 1;
        auto copy = [&](auto& dst, const void* src, std::size_t count) {
            using T = std::remove_reference_t<decltype(*dst.get())>;
            dst.resize(count);
            CUNIBS_CHECK(cudaMemcpyAsync(dst.get(), src, count * sizeof(T), cudaMemcpyDeviceToDevice, s));
        };
        for (int l = 0; l <= depth; ++l) {
            require(weights[l] && biases[l], "NULL layer weights or bias");
            const int in = l == 0 ? kWarmInPad : hidden;
            const int out = l == depth ? ws->n_out_pad : hidden;
            ws->w16.emplace_back();
            ws->bias.emplace_back();
            copy(ws->w16.back(), weights[l], static_cast<std::size_t>(out) * in);
            copy(ws->bias.back(), biases[l], static_cast<std::size_t>(out));
        }
        copy(ws->in_mean, feature_mean, 6);
        copy(ws->in_std, feature_std, 6);
        copy(ws->out_mean, coef_mean, n_out);
        copy(ws->out_std, coef_std, n_out);
        copy(ws->basis, basis, static_cast<std::size_t>(ws->n_red) * 2 * ws->n_out_pad);
        ws->error.resize(1);
        ws->error.zero(s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        c->warm = std::move(ws);
    });
}

int cunibs_context_recovery(cunibs_context* c, int mode, cunibs_recovery_info* out) {
    return guarded([&] {
        require(c && out, "NULL argument");
        DeviceGuard dg(c->device);
        const RecoveryOp& op = c->recovery(mode);
        out->mode = mode;
        out->n_slots = op.n_slots;
        out->nnz = op.mode == kRecSprGlobal ? 4LL * c->mesh.n_tets : static_cast<long long>(op.nnz);
        out->n_fallback = op.n_fallback;
        out->n_undetermined = op.n_undetermined;
    });
}

int cunibs_context_recovery_array(cunibs_context* c, int mode, const char* name, void* out, long long cap,
                                  long long* len) {
    return guarded([&] {
        require(c && name && len, "NULL argument");
        DeviceGuard dg(c->device);
        const RecoveryOp& op = c->recovery(mode);
        const Mesh& m = c->mesh;
        const bool nodes = mode == kRecSprGlobal, harmonic = mode == kRecHarmonic;
        const std::string n(name);
        const std::size_t nc = 4 * static_cast<std::size_t>(m.n_tets);
        std::vector<unsigned char> host;
        const void* src = nullptr;
        std::size_t count = 0, elem = 4;
        auto pick = [&](const void* p, std::size_t cnt) {
            src = p;
            count = cnt;
        };
        if (n == "ptr") pick(nodes ? m.n2c_ptr.get() : op.ptr.get(), op.n_slots + 1);
        else if (n == "idx") pick(nodes ? m.n2c_idx.get() : (harmonic ? op.pidx.get() : op.idx.get()),
                                  harmonic ? op.nnz : nc);
        else if (n == "slot_of_corner") pick(recovery_slot_of_corner(m, op), nc);
        else if (n == "slot_node") pick(op.slot_node.get(), op.n_slots);
        else if (n == "slot_tag") pick(op.slot_tag.get(), nodes ? 0 : op.n_slots);
        else if (n == "status") pick(op.status.get(), harmonic ? op.n_slots : 0);
        else if (n == "is_boundary") pick(op.is_boundary.get(), harmonic ? 0 : m.n_nodes);
        else if (n == "w" && !harmonic) pick(op.w.get(), nc);
        else if (n == "w") {
            // Unpacked from the {w_x, w_y, w_z, node} records: (nnz, 3).
            std::vector<float4> packed(op.nnz);
            CUNIBS_CHECK(cudaMemcpy(packed.data(), op.wq.get(), sizeof(float4) * op.nnz, cudaMemcpyDeviceToHost));
            host.resize(sizeof(float) * 3 * op.nnz);
            float* f = reinterpret_cast<float*>(host.data());
            for (std::int64_t i = 0; i < op.nnz; ++i) {
                f[3 * i] = packed[i].x;
                f[3 * i + 1] = packed[i].y;
                f[3 * i + 2] = packed[i].z;
            }
            count = 3 * static_cast<std::size_t>(op.nnz);
        } else fail(kEInval, "unknown recovery array name: " + n);
        *len = static_cast<long long>(count);
        if (out && count) {
            const std::size_t nb = std::min<std::size_t>(count, static_cast<std::size_t>(cap)) * elem;
            if (src) CUNIBS_CHECK(cudaMemcpy(out, src, nb, cudaMemcpyDeviceToHost));
            else std::memcpy(out, host.data(), nb);
        }
    });
}

int cunibs_context_recover(cunibs_context* c, int mode, int k, const double* v, const float* dadt_nodes,
                           const float* E_elem, float* E_slots, float* E, float* magnE) {
    return guarded([&] {
        require(c && E_slots && magnE, "NULL argument");
        require(k >= 1 && k <= 16, "k must be in [1, 16]");
        DeviceGuard dg(c->device);
        RecoveryOp& op = c->recovery(mode);
        const Mesh& m = c->mesh;
        cudaStream_t s = c->stream;
        DevArray<double> x;
        DevArray<float> da, ee, slots(static_cast<std::size_t>(op.n_slots) * 3 * k),
            mag(static_cast<std::size_t>(m.n_tets) * k), Ed;
        if (E) Ed.resize(static_cast<std::size_t>(m.n_tets) * 3 * k);
        if (mode == kRecHarmonic) {
            require(v && dadt_nodes, "harmonic recovery reads v and dadt_nodes");
            // (k, N) potentials into the solver's grounded row-major (N-1, k) layout.
            std::vector<double> red(static_cast<std::size_t>(m.n_nodes - 1) * k);
            for (int col = 0; col < k; ++col)
                for (int i = 0, r = 0; i < m.n_nodes; ++i) {
                    if (i == m.ground) continue;
                    red[static_cast<std::size_t>(r++) * k + col] = v[static_cast<std::size_t>(col) * m.n_nodes + i];
                }
            x.upload(red.data(), red.size(), s);
            da.upload(dadt_nodes, static_cast<std::size_t>(m.n_nodes) * 3 * k, s);
        } else {
            require(E_elem != nullptr, "SPR recovery reads E_elem");
            ee.upload(E_elem, static_cast<std::size_t>(m.n_tets) * 3 * k, s);
        }
        apply_recovery(m, op, x.get(), k, da.get(), ee.get(), k, slots.get(), E ? Ed.get() : nullptr, mag.get(), s);
        copy_out(E_slots, slots.get(), sizeof(float) * slots.size(), cudaMemcpyDeviceToHost, s);
        copy_out(magnE, mag.get(), sizeof(float) * mag.size(), cudaMemcpyDeviceToHost, s);
        if (E) copy_out(E, Ed.get(), sizeof(float) * Ed.size(), cudaMemcpyDeviceToHost, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_place(cunibs_context* c, const double* centers_mm, const double* handles_mm, const double* dists_mm,
                         int k, double* transforms, int* degenerate) {
    return guarded([&] {
        require(c && centers_mm && dists_mm && transforms, "NULL argument");
        require(k >= 1, "need at least one placement");
        DeviceGuard dg(c->device);
        cudaStream_t s = c->stream;
        c->centers.upload(centers_mm, 3 * static_cast<std::size_t>(k), s);
        if (handles_mm) c->handles.upload(handles_mm, 3 * static_cast<std::size_t>(k), s);
        c->dists.upload(dists_mm, k, s);
        c->T.reserve(16 * static_cast<std::size_t>(k));
        c->deg.reserve(k);
        place_transforms(c->mesh, c->centers.get(), handles_mm ? c->handles.get() : nullptr, c->dists.get(), k,
                         c->T.get(), c->deg.get(), s);
        copy_out(transforms, c->T.get(), sizeof(double) * 16 * k, cudaMemcpyDeviceToHost, s);
        copy_out(degenerate, c->deg.get(), sizeof(int) * k, cudaMemcpyDeviceToHost, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_dadt(cunibs_context* c, const double* dip_pos_m, const double* dip_moment, int n_dip,
                        const double* transforms, int k, double didt, float* out) {
    return guarded([&] {
        require(c && dip_pos_m && dip_moment && transforms && out, "NULL argument");
        require(k >= 1 && n_dip >= 1, "need at least one transform and one dipole");
        DeviceGuard dg(c->device);
        cudaStream_t s = c->stream;
        c->pos.upload(dip_pos_m, 3 * static_cast<std::size_t>(n_dip), s);
        c->mom.upload(dip_moment, 3 * static_cast<std::size_t>(n_dip), s);
        DevArray<double> T;
        T.upload(transforms, 16 * static_cast<std::size_t>(k), s);
        DevArray<int> flag(1);
        c->zdip_packed.reserve(packed_zdipole_bytes() * static_cast<std::size_t>(n_dip));
        prep_zdipoles(c->pos.get(), c->mom.get(), n_dip, c->zdip_packed.get(), flag.get(), s);
        int general = 0;
        CUNIBS_CHECK(cudaMemcpyAsync(&general, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        c->dadt_nodes.reserve(static_cast<std::size_t>(c->mesh.n_nodes) * 3 * k);
        if (general == 0) {
            dadt_nodes_zcoil(c->mesh, c->zdip_packed.get(), n_dip, T.get(), k, didt, c->dadt_nodes.get(), s);
        } else {
            c->dip_packed.reserve(packed_dipole_bytes() * static_cast<std::size_t>(n_dip) * k);
            prep_dipoles(c->pos.get(), c->mom.get(), n_dip, T.get(), k, c->dip_packed.get(), s);
            dadt_nodes(c->mesh, reinterpret_cast<const float*>(c->dip_packed.get()), n_dip, T.get(), k, didt,
                       c->dadt_nodes.get(), s);
        }
        copy_out(out, c->dadt_nodes.get(), sizeof(float) * 3 * static_cast<std::size_t>(c->mesh.n_nodes) * k,
                 cudaMemcpyDeviceToHost, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_solve(cunibs_context* c, const double* B, double* X, int k, int width, int precision,
                         double tolerance, int max_iters, const double* x0, int* iterations, double* relres) {
    return guarded([&] {
        require(c && B && X, "NULL argument");
        DeviceGuard dg(c->device);
        cudaStream_t s = c->stream;
        const std::size_t nk = static_cast<std::size_t>(c->mesh.n_nodes - 1) * width;
        DevArray<double> dB, dX, dX0;
        dB.upload(B, nk, s);
        dX.resize(nk);
        if (x0) dX0.upload(x0, nk, s);
        cunibs_solve_opts o{};
        o.precision = precision;
        o.tolerance = tolerance;
        o.max_iters = max_iters;
        const Params prm = resolve(c, &o);
        SolveStats st;
        solver_solve(*c->solver, dB.get(), dX.get(), k, width, prm, s, st, x0 ? dX0.get() : nullptr);
        dX.download(X, nk, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
        for (int i = 0; i < k; ++i) {
            if (iterations) iterations[i] = st.col_iters[i];
            if (relres) relres[i] = st.col_rel[i];
        }
    });
}

int cunibs_context_vcycle(cunibs_context* c, const double* r, double* z, int k, int fp32) {
    return guarded([&] {
        require(c && r && z, "NULL argument");
        DeviceGuard dg(c->device);
        cudaStream_t s = c->stream;
        const std::size_t nk = static_cast<std::size_t>(c->mesh.n_nodes - 1) * k;
        DevArray<double> dr, dz(nk);
        dr.upload(r, nk, s);
        solver_vcycle(*c->solver, dr.get(), dz.get(), k, fp32 != 0, s);
        dz.download(z, nk, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_select_size4(int n, const int* row_ptr, const int* col_idx, const float* values, int* aggregates,
                        int* n_coarse) {
    return guarded([&] {
        require(n >= 0 && row_ptr && aggregates && n_coarse, "NULL argument");
        cudaStream_t s = nullptr;
        CUNIBS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct StreamDel {
            cudaStream_t s;
            ~StreamDel() { cudaStreamDestroy(s); }
        } del{s};
        const int nnz = row_ptr[n];
        DevArray<int> rp, ci, agg(n > 0 ? n : 1);
        DevArray<float> va;
        rp.upload(row_ptr, n + 1, s);
        ci.upload(col_idx, nnz, s);
        va.upload(values, nnz, s);
        *n_coarse = select_size4(n, nnz, rp.get(), ci.get(), va.get(), agg.get(), s);
        agg.download(aggregates, n, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_summary(cunibs_context* c, const float* magnE, int k, double* summary) {
    return guarded([&] {
        require(c && magnE && summary && k >= 1, "NULL argument");
        DeviceGuard dg(c->device);
        cudaStream_t s = c->stream;
        DevArray<float> dm;
        dm.upload(magnE, static_cast<std::size_t>(c->mesh.n_tets) * k, s);
        DevArray<double> out(static_cast<std::size_t>(kSummaryLen) * k);
        gm_summary(c->mesh, dm.get(), k, out.get(), c->sw, s);
        out.download(summary, static_cast<std::size_t>(kSummaryLen) * k, s);
        CUNIBS_CHECK(cudaStreamSynchronize(s));
    });
}

int cunibs_context_set_timing(cunibs_context* c, int on) {
    return guarded([&] {
        require(c != nullptr, "NULL context");
        DeviceGuard dg(c->device);
        if (on && !c->ev[0])
            for (cudaEvent_t& e : c->ev) CUNIBS_CHECK(cudaEventCreate(&e));
        c->timing = on != 0;
    });
}

int cunibs_context_stage_times(const cunibs_context* c, double* ms, int cap) {
    return guarded([&] {
        require(c && ms && cap >= 5, "NULL argument or cap < 5");
        for (int i = 0; i < 5; ++i) ms[i] = c->stage_ms[i];
    });
}

int cunibs_context_stream(const cunibs_context* c, void** stream) {
    return guarded([&] {
        require(c && stream, "NULL argument");
        *stream = c->stream;
    });
}

long long cunibs_kernel_launches(void) { return launch_counter().load(); }

}  // extern "C"
