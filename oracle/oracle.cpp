// CPU restatement of the cuNIBS per-placement field solve. TEST INFRASTRUCTURE ONLY: the
// parity oracle and the timed CPU baseline. The product library never links or calls this.
//
// Built with -ffp-contract=off: every multiply-add below is a separate multiply and add unless
// written as std::fma, so the integer outputs that depend on floating-point comparisons (the
// Morton key, the aggregation's edge weights) come out bit-identical to the CUDA path, which is
// compiled the same way for its setup kernels.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using std::size_t;
using std::vector;

struct Csr {
    int n = 0;
    int ncol = 0;
    vector<int> ptr;
    vector<int> col;
    vector<double> val;
    long nnz() const { return static_cast<long>(col.size()); }
};

struct Level {
    Csr a;
    vector<double> dinv;
    vector<int> agg;
    int n_coarse = 0;
    Csr p;
    Csr r;
};

struct Cheby {
    double alpha0 = 0.0;
    double c_cur[8] = {};
    double c_prev[8] = {};
    double alpha[8] = {};
    int degree = 1;
};

struct Ctx {
    orc_params prm{};
    int n_nodes = 0;
    int n_tets = 0;
    int n_skin = 0;
    vector<double> nodes;  // (N,3) mm, Morton order
    vector<int> tets;      // (M,4)
    vector<int> tags;      // (M)
    vector<int> skin;      // (S,3)
    vector<int> node_perm;
    vector<int> tet_perm;
    vector<double> g;     // (M,4,3) 1/m
    vector<double> vols;  // (M) m^3
    vector<double> cond;  // (M) S/m
    vector<double> bary;  // (M,3) mm
    vector<float> vols_f32;
    vector<int> n2c_ptr;
    vector<int> n2c_idx;
    Csr stiff;
    int ground = 0;
    vector<int> red_idx;
    vector<Level> levels;
    Csr coarse;
    vector<double> coarse_inv;  // dense (nc, nc)
    Cheby cheby;
    vector<double> skin_normals;  // (S,3)
    vector<int> gm_index;
    // Flattened per-level views for the getters.
    vector<int> level_sizes;
    // Field-recovery operators, built on demand, indexed by mode (ORC_REC_*).
    struct Recovery {
        bool built = false;
        vector<int> ptr, idx;             // slot CSR over corners (SPR) or patch nodes (harmonic)
        vector<float> w;                  // SPR: one weight per entry; harmonic: three per entry
        vector<int> slot_of_corner;       // (4M) slot each corner samples back from
        vector<int> slot_node, slot_tag;  // (n_slots); slot_tag empty when slots are nodes
        vector<int> status;               // harmonic: rung per slot
        vector<int> is_boundary;          // SPR: per node
        vector<int> counts;               // n_slots, n_fallback, n_undetermined
    } rec[4];
};

// --- small helpers -----------------------------------------------------------------------

template <typename Key>
vector<int> stable_argsort(const vector<Key>& key) {
    vector<int> order(key.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return key[a] < key[b]; });
    return order;
}

// Tag -> S/m, fem/assembly.py:15-26.
double tissue_sigma(int tag) {
    switch (tag) {
        case 1: return 0.126;
        case 2: return 0.275;
        case 3: return 1.654;
        case 4: return 0.010;
        case 5: return 0.465;
        case 6: return 0.5;
        case 7: return 0.008;
        case 8: return 0.025;
        case 9: return 0.6;
        case 10: return 0.16;
        default: return std::nan("");
    }
}

// --- Morton order (fem/solve.py:302-348) -------------------------------------------------

uint64_t spread3(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

vector<int> morton_order(const vector<double>& pts, int n) {
    double lo[3], span[3];
    for (int a = 0; a < 3; ++a) {
        double mn = pts[a], mx = pts[a];
        for (int i = 1; i < n; ++i) {
            mn = std::min(mn, pts[3 * i + a]);
            mx = std::max(mx, pts[3 * i + a]);
        }
        lo[a] = mn;
        span[a] = std::max(mx - mn, 1e-12);
    }
    vector<uint64_t> key(n, 0);
    for (int i = 0; i < n; ++i) {
        uint64_t k = 0;
        for (int a = 0; a < 3; ++a) {
            const double t = (pts[3 * i + a] - lo[a]) / span[a] * 2097151.0;
            k |= spread3(static_cast<uint64_t>(t)) << a;
        }
        key[i] = k;
    }
    return stable_argsort(key);
}

// --- P1 operator (gradient.cu:29-66) --------------------------------------------------------

void p1_gradients(const vector<double>& nodes, const vector<int>& tets, int m, vector<double>& g,
                  vector<double>& vols) {
    g.assign(static_cast<size_t>(m) * 12, 0.0);
    vols.assign(m, 0.0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < m; ++e) {
        const int n0 = tets[4 * e];
        double t[3][3];
        for (int i = 0; i < 3; ++i) {
            const int ni = tets[4 * e + i + 1];
            for (int c = 0; c < 3; ++c) t[i][c] = nodes[3 * ni + c] - nodes[3 * n0 + c];
        }
        auto cross = [](const double* a, const double* b, double* o) {
            o[0] = a[1] * b[2] - a[2] * b[1];
            o[1] = a[2] * b[0] - a[0] * b[2];
            o[2] = a[0] * b[1] - a[1] * b[0];
        };
        double adj[3][3];
        cross(t[1], t[2], adj[0]);
        cross(t[2], t[0], adj[1]);
        cross(t[0], t[1], adj[2]);
        const double det = t[0][0] * adj[0][0] + t[0][1] * adj[0][1] + t[0][2] * adj[0][2];
        const double inv = 1e3 / det;
        for (int c = 0; c < 3; ++c) {
            const double g1 = adj[0][c] * inv;
            const double g2 = adj[1][c] * inv;
            const double g3 = adj[2][c] * inv;
            g[12 * e + 0 * 3 + c] = -(g1 + g2 + g3);
            g[12 * e + 1 * 3 + c] = g1;
            g[12 * e + 2 * 3 + c] = g2;
            g[12 * e + 3 * 3 + c] = g3;
        }
        vols[e] = std::fabs(det) * (1e-9 / 6.0);
    }
}

// node -> corner CSR by a stable sort of the corner keys (fem/assembly.py:142-162).
void node2corner(const vector<int>& elems, int per, int n_nodes, vector<int>& ptr, vector<int>& idx) {
    const int n_corner = static_cast<int>(elems.size());
    ptr.assign(n_nodes + 1, 0);
    for (int c = 0; c < n_corner; ++c) ptr[elems[c] + 1]++;
    for (int i = 0; i < n_nodes; ++i) ptr[i + 1] += ptr[i];
    idx.assign(n_corner, 0);
    vector<int> fill(ptr.begin(), ptr.end() - 1);
    // Counting sort visits corners in increasing id, i.e. a stable sort by node.
    for (int c = 0; c < n_corner; ++c) idx[fill[elems[c]]++] = c;
    (void)per;
}

// Stiffness CSR pattern (pattern.cu:145-299) and values (stiffness.cu:32-65): row i holds every
// node of every tetrahedron incident to i, sorted; A_ij sums vol*sigma*(g_i . g_j) over the shared
// elements in ascending element order, starting from zero.
Csr assemble_stiffness(const Ctx& c) {
    Csr a;
    a.n = a.ncol = c.n_nodes;
    vector<vector<int>> rows(c.n_nodes);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < c.n_nodes; ++i) {
        vector<int>& r = rows[i];
        for (int p = c.n2c_ptr[i]; p < c.n2c_ptr[i + 1]; ++p) {
            const int e = c.n2c_idx[p] >> 2;
            for (int j = 0; j < 4; ++j) r.push_back(c.tets[4 * e + j]);
        }
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
    }
    a.ptr.assign(c.n_nodes + 1, 0);
    for (int i = 0; i < c.n_nodes; ++i) a.ptr[i + 1] = a.ptr[i] + static_cast<int>(rows[i].size());
    a.col.resize(a.ptr[c.n_nodes]);
    a.val.assign(a.ptr[c.n_nodes], 0.0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < c.n_nodes; ++i) {
        const int b = a.ptr[i];
        std::copy(rows[i].begin(), rows[i].end(), a.col.begin() + b);
        for (int p = c.n2c_ptr[i]; p < c.n2c_ptr[i + 1]; ++p) {
            const int corner = c.n2c_idx[p];
            const int e = corner >> 2;
            const double s = c.vols[e] * c.cond[e];
            const double* gi = &c.g[3 * static_cast<size_t>(corner)];
            for (int j = 0; j < 4; ++j) {
                const double* gj = &c.g[12 * static_cast<size_t>(e) + 3 * j];
                const double dot = gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2];
                const int col = c.tets[4 * e + j];
                const int pos = static_cast<int>(
                    std::lower_bound(a.col.begin() + b, a.col.begin() + a.ptr[i + 1], col) -
                    a.col.begin());
                a.val[pos] = a.val[pos] + s * dot;
            }
        }
    }
    return a;
}

// Ground the lowest-z node (fem/solve.py:287-298,361-365).
Csr reduce_grounded(const Csr& a, int ground) {
    Csr r;
    r.n = r.ncol = a.n - 1;
    r.ptr.assign(r.n + 1, 0);
    for (int i = 0, ri = 0; i < a.n; ++i) {
        if (i == ground) continue;
        int cnt = 0;
        for (int p = a.ptr[i]; p < a.ptr[i + 1]; ++p) cnt += (a.col[p] != ground);
        r.ptr[ri + 1] = r.ptr[ri] + cnt;
        ++ri;
    }
    r.col.resize(r.ptr[r.n]);
    r.val.resize(r.ptr[r.n]);
    for (int i = 0, ri = 0; i < a.n; ++i) {
        if (i == ground) continue;
        int q = r.ptr[ri];
        for (int p = a.ptr[i]; p < a.ptr[i + 1]; ++p) {
            const int cc = a.col[p];
            if (cc == ground) continue;
            r.col[q] = cc - (cc > ground ? 1 : 0);
            r.val[q] = a.val[p];
            ++q;
        }
        ++ri;
    }
    return r;
}

// --- SIZE_4 pairwise aggregation (aggregate.cu:13-472; AMGx size4 selector semantics) --------

unsigned agg_hash(unsigned a, unsigned seed) {
    a ^= seed;
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) + (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a ^ 0xd3a2646cu) + (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) + (a >> 16);
    return a;
}

struct Best {
    float w;
    int col;
};

inline void best_take(Best& acc, float w, int col) {
    if (w > acc.w || (w == acc.w && col > acc.col)) {
        acc.w = w;
        acc.col = col;
    }
}

inline bool is_candidate(int col, int row, int n) {
    return col != row && static_cast<unsigned>(col) < static_cast<unsigned>(n);
}

int select_size4(int n, const int* rp, const int* ci, const float* va, int* agg) {
    if (n <= 0) return 0;
    const int nnz = rp[n];
    vector<float> diag(n, 0.0f), w(std::max(nnz, 1), -1.0f), wsn(n);
    vector<int> partner(n), strongest(n), aggregated(n), cand(n);
    for (int i = 0; i < n; ++i) {
        float d = 0.0f;
        for (int j = rp[i]; j < rp[i + 1]; ++j)
            if (ci[j] == i) {
                d = va[j];
                break;
            }
        diag[i] = d;
    }
    for (int i = 0; i < n; ++i) {
        const float di = std::fabs(diag[i]);
        for (int j = rp[i]; j < rp[i + 1]; ++j) {
            const int jc = ci[j];
            if (!is_candidate(jc, i, n)) {
                w[j] = -1.0f;
                continue;
            }
            const float den = std::fmax(di, std::fabs(diag[jc]));
            const float ed = std::fabs(va[j]) / den;
            const unsigned lo = static_cast<unsigned>(std::min(i, jc));
            const unsigned hi = static_cast<unsigned>(std::max(i, jc));
            const float frac = 1e-5f * static_cast<float>(agg_hash(lo, hi)) / 4294967295.0f;
            w[j] = std::fmaf(frac, ed, ed);
        }
    }
    for (int i = 0; i < n; ++i) {
        agg[i] = i;
        partner[i] = -1;
        strongest[i] = -1;
    }
    // Round 1: pairs.
    int unassigned = n;
    for (int iter = 0; iter <= 15; ++iter) {
        for (int t = 0; t < n; ++t) {
            if (partner[t] != -1) continue;
            Best b{0.0f, -1};
            for (int j = rp[t]; j < rp[t + 1]; ++j) {
                const int jc = ci[j];
                if (!is_candidate(jc, t, n) || partner[jc] != -1) continue;
                best_take(b, w[j], jc);
            }
            if (b.col != -1) strongest[t] = b.col;
        }
        int cnt = 0;
        // Every read below is of a slot no row writes in this pass except its own.
        vector<int> partner_in(partner);
        for (int t = 0; t < n; ++t) {
            if (partner_in[t] != -1) continue;
            const int pm = strongest[t];
            if (pm != -1 && strongest[pm] == t) {
                partner[t] = pm;
                agg[t] = std::min(pm, t);
            } else {
                ++cnt;
            }
        }
        const int prev = unassigned;
        unassigned = cnt;
        if (unassigned == 0 || unassigned == prev) break;
    }
    for (int t = 0; t < n; ++t)
        if (partner[t] == -1) partner[t] = t;
    for (int t = 0; t < n; ++t) {
        wsn[t] = -1.0f;
        aggregated[t] = -1;
    }
    // Round 2: pairs into quads.
    unassigned = n;
    for (int iter = 0; iter <= 15; ++iter) {
        for (int t = 0; t < n; ++t) {
            if (aggregated[t] != -1) continue;
            const int p = partner[t];
            Best b{0.0f, -1};
            for (int j = rp[t]; j < rp[t + 1]; ++j) {
                const int jc = ci[j];
                if (!is_candidate(jc, t, n)) continue;
                if (aggregated[jc] != -1 || jc == p) continue;
                best_take(b, w[j], jc);
            }
            if (b.col != -1) {
                wsn[t] = b.w;
                strongest[t] = agg[b.col];
            }
        }
        {
            const vector<int> strongest_in(strongest);
            for (int t = 0; t < n; ++t) {
                if (aggregated[t] != -1) continue;
                const int p = partner[t];
                const float mine = wsn[t];
                const float theirs = (p != -1) ? wsn[p] : -1.0f;
                if (mine < 0.0f && theirs < 0.0f) {
                    aggregated[t] = 1;
                    strongest[t] = -1;
                } else if (mine < theirs) {
                    strongest[t] = strongest_in[p];
                }
            }
        }
        int cnt = 0;
        const vector<int> aggregated_in(aggregated);
        for (int t = 0; t < n; ++t) {
            if (aggregated_in[t] != -1) continue;
            const int pm = strongest[t];
            const int mine = agg[t];
            if (pm != -1 && strongest[pm] == mine) {
                aggregated[t] = 1;
                agg[t] = std::min(pm, mine);
            } else {
                ++cnt;
            }
        }
        const int prev = unassigned;
        unassigned = cnt;
        if (unassigned == 0 || unassigned == prev ||
            static_cast<float>(unassigned) / static_cast<float>(n) < 0.05f)
            break;
    }
    if (unassigned != 0) {
        for (int t = 0; t < n; ++t) {
            if (aggregated[t] != -1) continue;
            Best b{0.0f, -1};
            for (int j = rp[t]; j < rp[t + 1]; ++j) {
                const int jc = ci[j];
                if (!is_candidate(jc, t, n) || aggregated[jc] == -1) continue;
                best_take(b, w[j], jc);
            }
            cand[t] = (b.col != -1) ? agg[b.col] : t;
        }
        for (int t = 0; t < n; ++t) {
            if (aggregated[t] == -1) {
                agg[t] = cand[t];
                aggregated[t] = 1;
            }
        }
    }
    vector<int> used(n + 1, 0), excl(n + 1, 0);
    for (int t = 0; t < n; ++t) used[agg[t]] = 1;
    for (int i = 0; i < n; ++i) excl[i + 1] = excl[i] + used[i];
    for (int t = 0; t < n; ++t) agg[t] = excl[agg[t]];
    return excl[n];
}

// --- hierarchy construction (fem/solve.py:69-256) ------------------------------------------

vector<double> l1_dinv(const Csr& a) {
    vector<double> d(a.n);
    for (int i = 0; i < a.n; ++i) {
        double acc = 0.0, diag = 0.0;
        for (int p = a.ptr[i]; p < a.ptr[i + 1]; ++p) {
            acc = acc + std::fabs(a.val[p]);
            if (a.col[p] == i) diag = a.val[p];
        }
        if (diag < 0.0) acc = -acc;
        if (acc == 0.0) acc = 1.0;
        d[i] = 1.0 / acc;
    }
    return d;
}

Csr tentative(const vector<int>& agg, int nc) {
    const int n = static_cast<int>(agg.size());
    vector<int> count(nc, 0);
    for (int a : agg) count[a]++;
    Csr p;
    p.n = n;
    p.ncol = nc;
    p.ptr.resize(n + 1);
    p.col.resize(n);
    p.val.resize(n);
    for (int i = 0; i <= n; ++i) p.ptr[i] = i;
    for (int i = 0; i < n; ++i) {
        p.col[i] = agg[i];
        p.val[i] = 1.0 / std::sqrt(static_cast<double>(count[agg[i]]));
    }
    return p;
}

// Row-wise product C = A B. Row i's partial products are listed in (A entry, B entry) order,
// stably sorted by column, and each column summed in that order from zero.
Csr spgemm(const Csr& A, const Csr& B) {
    Csr C;
    C.n = A.n;
    C.ncol = B.ncol;
    vector<vector<std::pair<int, double>>> rows(A.n);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < A.n; ++i) {
        vector<std::pair<int, double>> prod;
        for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
            const int j = A.col[p];
            const double a = A.val[p];
            for (int q = B.ptr[j]; q < B.ptr[j + 1]; ++q) prod.emplace_back(B.col[q], a * B.val[q]);
        }
        std::stable_sort(prod.begin(), prod.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        vector<std::pair<int, double>>& out = rows[i];
        size_t s = 0;
        while (s < prod.size()) {
            size_t e = s;
            double acc = 0.0;
            while (e < prod.size() && prod[e].first == prod[s].first) acc = acc + prod[e++].second;
            out.emplace_back(prod[s].first, acc);
            s = e;
        }
    }
    C.ptr.assign(A.n + 1, 0);
    for (int i = 0; i < A.n; ++i) C.ptr[i + 1] = C.ptr[i] + static_cast<int>(rows[i].size());
    C.col.resize(C.ptr[A.n]);
    C.val.resize(C.ptr[A.n]);
    for (int i = 0; i < A.n; ++i)
        for (size_t q = 0; q < rows[i].size(); ++q) {
            C.col[C.ptr[i] + q] = rows[i][q].first;
            C.val[C.ptr[i] + q] = rows[i][q].second;
        }
    return C;
}

// CSR transpose by a counting sort over columns: rows of the result list the source rows in
// increasing order, so its columns come out sorted.
Csr transpose(const Csr& A) {
    Csr T;
    T.n = A.ncol;
    T.ncol = A.n;
    T.ptr.assign(T.n + 1, 0);
    for (int c : A.col) T.ptr[c + 1]++;
    for (int i = 0; i < T.n; ++i) T.ptr[i + 1] += T.ptr[i];
    T.col.resize(A.col.size());
    T.val.resize(A.col.size());
    vector<int> fill(T.ptr.begin(), T.ptr.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
            const int q = fill[A.col[p]]++;
            T.col[q] = i;
            T.val[q] = A.val[p];
        }
    return T;
}

Csr galerkin(const Csr& A, const Csr& P) {
    const Csr ap = spgemm(A, P);
    return spgemm(transpose(P), ap);
}

// P = (I - 4/3 D^-1 A) P_tent (fem/solve.py:91,110-126).
Csr smooth_prolongator(const Csr& A, const vector<int>& agg, int nc, const vector<double>& dinv) {
    const Csr pt = tentative(agg, nc);
    Csr p = spgemm(A, pt);
    const double damping = 4.0 / 3.0;
    for (int i = 0; i < p.n; ++i) {
        for (int q = p.ptr[i]; q < p.ptr[i + 1]; ++q) {
            const double scaled = damping * (dinv[i] * p.val[q]);
            p.val[q] = (p.col[q] == agg[i]) ? (pt.val[i] - scaled) : -scaled;
        }
    }
    return p;
}

vector<float> to_f32(const vector<double>& v) {
    vector<float> f(v.size());
    for (size_t i = 0; i < v.size(); ++i) f[i] = static_cast<float>(v[i]);
    return f;
}

// Compose rounds of pairwise passes into one level (fem/solve.py:178-209).
int aggregate_level(const Csr& a, const orc_params& prm, vector<int>& agg_out) {
    Csr cur = a;
    bool have = false;
    int n_coarse = a.n;
    agg_out.clear();
    for (int round = 0; round < prm.agg_rounds; ++round) {
        if (cur.n <= prm.min_coarse_rows) break;
        vector<int> step(cur.n);
        const vector<float> vf = to_f32(cur.val);
        const int nc = select_size4(cur.n, cur.ptr.data(), cur.col.data(), vf.data(), step.data());
        if (nc == cur.n || nc < prm.min_coarse_rows) break;
        if (!have) {
            agg_out = step;
            have = true;
        } else {
            for (int& x : agg_out) x = step[x];
        }
        n_coarse = nc;
        if (round + 1 < prm.agg_rounds) cur = galerkin(cur, tentative(step, nc));
    }
    return have ? n_coarse : -1;
}

void cholesky_inverse(const Csr& a, vector<double>& inv) {
    const int n = a.n;
    vector<double> m(static_cast<size_t>(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int p = a.ptr[i]; p < a.ptr[i + 1]; ++p) m[static_cast<size_t>(i) * n + a.col[p]] = a.val[p];
    // L L^T in place (lower triangle).
    for (int j = 0; j < n; ++j) {
        double d = m[static_cast<size_t>(j) * n + j];
        for (int k = 0; k < j; ++k) d -= m[static_cast<size_t>(j) * n + k] * m[static_cast<size_t>(j) * n + k];
        if (!(d > 0.0)) throw std::runtime_error("coarse operator is not positive definite");
        d = std::sqrt(d);
        m[static_cast<size_t>(j) * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = m[static_cast<size_t>(i) * n + j];
            for (int k = 0; k < j; ++k) s -= m[static_cast<size_t>(i) * n + k] * m[static_cast<size_t>(j) * n + k];
            m[static_cast<size_t>(i) * n + j] = s / d;
        }
    }
    // inv = L^-T L^-1, column by column of the identity.
    inv.assign(static_cast<size_t>(n) * n, 0.0);
    vector<double> y(n);
    for (int c = 0; c < n; ++c) {
        for (int i = 0; i < n; ++i) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= m[static_cast<size_t>(i) * n + k] * y[k];
            y[i] = s / m[static_cast<size_t>(i) * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s -= m[static_cast<size_t>(k) * n + i] * inv[static_cast<size_t>(k) * n + c];
            inv[static_cast<size_t>(i) * n + c] = s / m[static_cast<size_t>(i) * n + i];
        }
    }
}

// Chebyshev over [1/lower_ratio, 1] in x-recurrence form (vcycle.cu:434-463).
Cheby make_cheby(int degree, double lower_ratio) {
    Cheby c;
    const double hi = 1.0, lo = hi / lower_ratio;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
    const double sigma = theta / delta;
    c.alpha0 = 1.0 / theta;
    double rho = 1.0 / sigma;
    for (int j = 0; j + 1 < degree; ++j) {
        const double rho_next = 1.0 / (2.0 * sigma - rho);
        const double beta = rho_next * rho;
        c.c_cur[j] = 1.0 + beta;
        c.c_prev[j] = -beta;
        c.alpha[j] = 2.0 * rho_next / delta;
        rho = rho_next;
    }
    c.degree = degree;
    return c;
}

void build_hierarchy(Ctx& c) {
    Csr a = reduce_grounded(c.stiff, c.ground);
    c.level_sizes.assign(1, a.n);
    for (int lev = 0; lev < c.prm.max_levels; ++lev) {
        if (a.n <= c.prm.min_coarse_rows) break;
        vector<int> agg;
        const int nc = aggregate_level(a, c.prm, agg);
        if (nc < 0 || nc == a.n || nc < c.prm.min_coarse_rows) break;
        Level L;
        L.dinv = l1_dinv(a);
        L.p = smooth_prolongator(a, agg, nc, L.dinv);
        L.r = transpose(L.p);
        L.agg = agg;
        L.n_coarse = nc;
        Csr next = galerkin(a, L.p);
        L.a = std::move(a);
        c.levels.push_back(std::move(L));
        a = std::move(next);
        c.level_sizes.push_back(a.n);
    }
    c.coarse = std::move(a);
    cholesky_inverse(c.coarse, c.coarse_inv);
    c.cheby = make_cheby(c.prm.cheby_degree, c.prm.cheby_lower_ratio);
}

// --- V-cycle (vcycle.cu:560-648), FP64 ------------------------------------------------------

void spmv(const Csr& a, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < a.n; ++i) {
        double s = 0.0;
        for (int p = a.ptr[i]; p < a.ptr[i + 1]; ++p) s = s + a.val[p] * x[a.col[p]];
        y[i] = s;
    }
}

// One smoothing sweep of `degree` Chebyshev steps. x holds the initial guess unless zero_guess.
void smooth(const Level& L, const Cheby& ch, const double* b, double* x, bool zero_guess,
            vector<double>& t0, vector<double>& t1) {
    const int n = L.a.n;
    vector<double>& ax = t0;
    vector<double>& prev = t1;
    ax.resize(n);
    prev.resize(n);
    if (zero_guess) {
        for (int i = 0; i < n; ++i) {
            x[i] = ch.alpha0 * L.dinv[i] * b[i];
            prev[i] = 0.0;
        }
    } else {
        spmv(L.a, x, ax.data());
        for (int i = 0; i < n; ++i) {
            prev[i] = x[i];
            x[i] = x[i] + ch.alpha0 * L.dinv[i] * (b[i] - ax[i]);
        }
    }
    for (int s = 1; s < ch.degree; ++s) {
        spmv(L.a, x, ax.data());
        const double cc = ch.c_cur[s - 1];
        const double cp = ch.c_prev[s - 1];
        const double al = ch.alpha[s - 1];
        for (int i = 0; i < n; ++i) {
            const double out = cc * x[i] + cp * prev[i] + al * L.dinv[i] * (b[i] - ax[i]);
            prev[i] = x[i];
            x[i] = out;
        }
    }
}

void vcycle(const Ctx& c, const double* b, double* x) {
    const int L = static_cast<int>(c.levels.size());
    vector<vector<double>> bs(L + 1), xs(L + 1);
    vector<double> t0, t1, r;
    if (L == 0) {
        const int n = c.coarse.n;
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = 0; j < n; ++j) s = s + c.coarse_inv[static_cast<size_t>(i) * n + j] * b[j];
            x[i] = s;
        }
        return;
    }
    bs[0].assign(b, b + c.levels[0].a.n);
    for (int l = 0; l < L; ++l) {
        const Level& lv = c.levels[l];
        xs[l].assign(lv.a.n, 0.0);
        smooth(lv, c.cheby, bs[l].data(), xs[l].data(), true, t0, t1);
        r.resize(lv.a.n);
        spmv(lv.a, xs[l].data(), r.data());
        for (int i = 0; i < lv.a.n; ++i) r[i] = bs[l][i] - r[i];
        bs[l + 1].resize(lv.n_coarse);
        spmv(lv.r, r.data(), bs[l + 1].data());
    }
    const int nc = c.coarse.n;
    xs[L].assign(nc, 0.0);
    for (int i = 0; i < nc; ++i) {
        double s = 0.0;
        for (int j = 0; j < nc; ++j) s = s + c.coarse_inv[static_cast<size_t>(i) * nc + j] * bs[L][j];
        xs[L][i] = s;
    }
    for (int l = L - 1; l >= 0; --l) {
        const Level& lv = c.levels[l];
        r.resize(lv.a.n);
        spmv(lv.p, xs[l + 1].data(), r.data());
        for (int i = 0; i < lv.a.n; ++i) xs[l][i] = xs[l][i] + r[i];
        smooth(lv, c.cheby, bs[l].data(), xs[l].data(), false, t0, t1);
    }
    std::copy(xs[0].begin(), xs[0].end(), x);
}

double dot(const vector<double>& a, const vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s = s + a[i] * b[i];
    return s;
}

// Single-column PCG, ||r||/||b|| <= tol (solver.cpp:84-198 column semantics).
int pcg(const Ctx& c, const vector<double>& b, vector<double>& x, double tol, int max_iters,
        double& rel_out) {
    const Csr& A = c.levels.empty() ? c.coarse : c.levels[0].a;
    const int n = A.n;
    const double ref = std::sqrt(dot(b, b));
    if (ref == 0.0) throw std::runtime_error("zero right-hand side");
    x.assign(n, 0.0);
    vector<double> r(b), z(n), p(n), ap(n);
    vcycle(c, r.data(), z.data());
    double rz = dot(r, z);
    p = z;
    int iters = max_iters;
    rel_out = 1.0;
    for (int it = 1; it <= max_iters; ++it) {
        spmv(A, p.data(), ap.data());
        const double alpha = rz / dot(p, ap);
        for (int i = 0; i < n; ++i) {
            x[i] = x[i] + alpha * p[i];
            r[i] = r[i] - alpha * ap[i];
        }
        rel_out = std::sqrt(dot(r, r)) / ref;
        if (rel_out <= tol) {
            iters = it;
            break;
        }
        vcycle(c, r.data(), z.data());
        const double rz_new = dot(r, z);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    return iters;
}

// --- skin normals (skin.cu:46-150) ----------------------------------------------------------

void skin_normals(Ctx& c) {
    const int s = c.n_skin;
    c.skin_normals.assign(static_cast<size_t>(s) * 3, 0.0);
    if (s == 0) return;
    vector<int> ptr, idx;
    node2corner(c.skin, 3, c.n_nodes, ptr, idx);
    vector<double> face(static_cast<size_t>(s) * 3), node(static_cast<size_t>(c.n_nodes) * 3, 0.0);
    for (int t = 0; t < s; ++t) {
        const double* a = &c.nodes[3 * c.skin[3 * t]];
        const double* b = &c.nodes[3 * c.skin[3 * t + 1]];
        const double* cc = &c.nodes[3 * c.skin[3 * t + 2]];
        double u[3], v[3];
        for (int i = 0; i < 3; ++i) {
            u[i] = b[i] - a[i];
            v[i] = cc[i] - a[i];
        }
        face[3 * t] = u[1] * v[2] - u[2] * v[1];
        face[3 * t + 1] = u[2] * v[0] - u[0] * v[2];
        face[3 * t + 2] = u[0] * v[1] - u[1] * v[0];
    }
    auto spread = [&]() {
        for (int nd = 0; nd < c.n_nodes; ++nd) {
            double acc[3] = {0.0, 0.0, 0.0};
            for (int p = ptr[nd]; p < ptr[nd + 1]; ++p) {
                const int t = idx[p] / 3;
                for (int i = 0; i < 3; ++i) acc[i] = acc[i] + face[3 * t + i];
            }
            for (int i = 0; i < 3; ++i) node[3 * nd + i] = acc[i];
        }
    };
    auto normalise = [](double* v) {
        const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (n > 0.0)
            for (int i = 0; i < 3; ++i) v[i] = v[i] / n;
    };
    auto gather = [&](double* out) {
        for (int t = 0; t < s; ++t) {
            double acc[3];
            for (int i = 0; i < 3; ++i)
                acc[i] = node[3 * c.skin[3 * t] + i] + node[3 * c.skin[3 * t + 1] + i] +
                         node[3 * c.skin[3 * t + 2] + i];
            normalise(acc);
            for (int i = 0; i < 3; ++i) out[3 * t + i] = acc[i];
        }
    };
    spread();
    gather(face.data());
    spread();
    for (int nd = 0; nd < c.n_nodes; ++nd) normalise(&node[3 * nd]);
    gather(c.skin_normals.data());
}

// --- placement (place.cu:64-230; Ericson's closest point on a triangle) --------------------

double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

double closest_on_tri(const double* p, const double* a, const double* b, const double* c, double* q) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int i = 0; i < 3; ++i) {
        ab[i] = b[i] - a[i];
        ac[i] = c[i] - a[i];
        ap[i] = p[i] - a[i];
        bp[i] = p[i] - b[i];
        cp[i] = p[i] - c[i];
    }
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    const double vc = d1 * d4 - d3 * d2;
    const double vb = d5 * d2 - d1 * d6;
    const double va = d3 * d6 - d5 * d4;
    if (d1 <= 0.0 && d2 <= 0.0) {
        for (int i = 0; i < 3; ++i) q[i] = a[i];
    } else if (d3 >= 0.0 && d4 <= d3) {
        for (int i = 0; i < 3; ++i) q[i] = b[i];
    } else if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double t = d1 / (d1 - d3);
        for (int i = 0; i < 3; ++i) q[i] = a[i] + t * ab[i];
    } else if (d6 >= 0.0 && d5 <= d6) {
        for (int i = 0; i < 3; ++i) q[i] = c[i];
    } else if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double t = d2 / (d2 - d6);
        for (int i = 0; i < 3; ++i) q[i] = a[i] + t * ac[i];
    } else if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int i = 0; i < 3; ++i) q[i] = b[i] + t * (c[i] - b[i]);
    } else {
        const double denom = 1.0 / (va + vb + vc);
        const double v = vb * denom, w = vc * denom;
        for (int i = 0; i < 3; ++i) q[i] = a[i] + v * ab[i] + w * ac[i];
    }
    const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
    return dx * dx + dy * dy + dz * dz;
}

void place_one(const Ctx& c, const double* center, const double* handle, double dist, double* T,
               int* degenerate) {
    double best = HUGE_VAL;
    int tri = -1;
    double q[3];
    for (int t = 0; t < c.n_skin; ++t) {
        const double d2 = closest_on_tri(center, &c.nodes[3 * c.skin[3 * t]], &c.nodes[3 * c.skin[3 * t + 1]],
                                         &c.nodes[3 * c.skin[3 * t + 2]], q);
        if (d2 < best) {
            best = d2;
            tri = t;
        }
    }
    if (tri < 0) throw std::runtime_error("no skin triangles to place the coil on");
    double proj[3];
    closest_on_tri(center, &c.nodes[3 * c.skin[3 * tri]], &c.nodes[3 * c.skin[3 * tri + 1]],
                   &c.nodes[3 * c.skin[3 * tri + 2]], proj);
    const double* nrm = &c.skin_normals[3 * tri];
    const double z[3] = {-nrm[0], -nrm[1], -nrm[2]};
    double y[3];
    bool from_handle = false;
    if (handle != nullptr) {
        for (int i = 0; i < 3; ++i) y[i] = handle[i] - proj[i];
        const double yy = dot3(y, y);
        if (yy > 0.0) {
            const double inv = 1.0 / std::sqrt(yy);
            for (int i = 0; i < 3; ++i) y[i] = y[i] * inv;
            const double cz = dot3(y, z);
            if ((1.0 - cz * cz) > 1e-12) {
                for (int i = 0; i < 3; ++i) y[i] = y[i] - z[i] * cz;
                const double inv2 = 1.0 / std::sqrt(dot3(y, y));
                for (int i = 0; i < 3; ++i) y[i] = y[i] * inv2;
                from_handle = true;
            }
        }
    }
    if (!from_handle) {
        int m = 0;
        if (std::fabs(z[1]) < std::fabs(z[m])) m = 1;
        if (std::fabs(z[2]) < std::fabs(z[m])) m = 2;
        double ref[3] = {0.0, 0.0, 0.0};
        ref[m] = 1.0;
        y[0] = z[1] * ref[2] - z[2] * ref[1];
        y[1] = z[2] * ref[0] - z[0] * ref[2];
        y[2] = z[0] * ref[1] - z[1] * ref[0];
        const double inv = 1.0 / std::sqrt(dot3(y, y));
        for (int i = 0; i < 3; ++i) y[i] = y[i] * inv;
    }
    if (degenerate) *degenerate = from_handle ? 0 : 1;
    const double x[3] = {y[1] * z[2] - y[2] * z[1], y[2] * z[0] - y[0] * z[2], y[0] * z[1] - y[1] * z[0]};
    for (int i = 0; i < 16; ++i) T[i] = 0.0;
    for (int r = 0; r < 3; ++r) {
        T[4 * r + 0] = x[r];
        T[4 * r + 1] = y[r];
        T[4 * r + 2] = z[r];
        T[4 * r + 3] = proj[r] + dist * nrm[r];
    }
    T[15] = 1.0;
}

// --- metrics (metrics.py:58-259) ------------------------------------------------------------

double interp(double x, const vector<double>& xp, const vector<double>& fp) {
    const size_t n = xp.size();
    if (x <= xp[0]) return fp[0];
    if (x >= xp[n - 1]) return fp[n - 1];
    const size_t j = static_cast<size_t>(std::upper_bound(xp.begin(), xp.end(), x) - xp.begin()) - 1;
    const double slope = (fp[j + 1] - fp[j]) / (xp[j + 1] - xp[j]);
    return slope * (x - xp[j]) + fp[j];
}

void weighted_quantiles_impl(const double* values, const double* weights, int n, const double* qs,
                             int nq, double* out) {
    vector<double> v(values, values + n);
    const vector<int> order = stable_argsort(v);
    vector<double> sv(n), sw(n), pos(n);
    for (int i = 0; i < n; ++i) {
        sv[i] = values[order[i]];
        sw[i] = weights[order[i]];
    }
    double cw = 0.0;
    vector<double> cws(n);
    for (int i = 0; i < n; ++i) {
        cw = cw + sw[i];
        cws[i] = cw;
    }
    for (int i = 0; i < n; ++i) pos[i] = (cws[i] - 0.5 * sw[i]) / cws[n - 1];
    for (int q = 0; q < nq; ++q) out[q] = interp(qs[q], pos, sv);
}

void summary_impl(const float* magnE, const float* vols, const double* bary, const int* tags,
                  int n_tets, int region_tag, double* out) {
    vector<double> m, w;
    vector<int> idx;
    for (int e = 0; e < n_tets; ++e)
        if (tags[e] == region_tag) {
            idx.push_back(e);
            m.push_back(magnE[e]);
            w.push_back(vols[e]);
        }
    for (int i = 0; i < ORC_SUMMARY_LEN; ++i) out[i] = std::nan("");
    const int n = static_cast<int>(m.size());
    if (n == 0) return;
    int arg = 0;
    for (int i = 1; i < n; ++i)
        if (m[i] > m[arg]) arg = i;
    out[ORC_S_PEAK] = m[arg];
    for (int a = 0; a < 3; ++a) out[ORC_S_PEAK_X + a] = bary[3 * idx[arg] + a];
    double wsum = 0.0, wm = 0.0, cog[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i) {
        wsum = wsum + w[i];
        const double ww = w[i] * m[i];
        wm = wm + ww;
        for (int a = 0; a < 3; ++a) cog[a] = cog[a] + ww * bary[3 * idx[i] + a];
    }
    for (int a = 0; a < 3; ++a) out[ORC_S_COG_X + a] = cog[a] / wm;
    out[ORC_S_VOLUME] = wsum;
    const double mean = wm / wsum;
    double var = 0.0;
    for (int i = 0; i < n; ++i) var = var + w[i] * (m[i] - mean) * (m[i] - mean);
    out[ORC_S_MEAN] = mean;
    out[ORC_S_STD] = std::sqrt(var / wsum);
    const double qs[4] = {static_cast<double>(0.5f), static_cast<double>(0.95f),
                          static_cast<double>(0.99f), static_cast<double>(0.999f)};
    double pv[4];
    weighted_quantiles_impl(m.data(), w.data(), n, qs, 4, pv);
    for (int q = 0; q < 4; ++q) out[ORC_S_P50 + q] = pv[q];
    const double fr[2] = {0.5, 0.75};
    for (int f = 0; f < 2; ++f) {
        const double thr = fr[f] * pv[3];
        double s = 0.0;
        for (int i = 0; i < n; ++i)
            if (m[i] >= thr) s = s + w[i];
        out[ORC_S_FOC50 + f] = s;
    }
}

// --- field recovery (fem/recovery.py:1-552; recovery.cu:1-774) ------------------------------
//
// Modes: 1 "spr_global" (a patch per node over every incident tetrahedron), 2 "spr_tissue" (a
// patch per (node, tissue) slot), 3 "harmonic" (potential fitted per (node, tissue) slot in the
// harmonic-polynomial space, then differentiated). Every accumulation below walks its CSR in
// order and names each fused multiply-add, so the weights are the same IEEE values the CUDA
// build kernels produce; the apply mirrors reproduce the CUDA apply kernels bit for bit.

using Recovery = Ctx::Recovery;

constexpr int kMinPatchNodes = 16;         // recovery.py:246-250 (_MIN_PATCH_NODES)
constexpr double kMaxLebesgue = 8.0;       // recovery.cu:32-35
constexpr double kMaxGradAmp = 50.0;       // recovery.cu:37-43

// Slots = (node, tissue) pairs: corners stably sorted by node * stride + tag (recovery.py:186-225).
void tissue_slots(const Ctx& c, Recovery& r) {
    const int M = c.n_tets;
    int max_tag = 0;
    for (int e = 0; e < M; ++e) max_tag = std::max(max_tag, c.tags[e]);
    const long stride = max_tag + 1;
    vector<long> key(4 * static_cast<size_t>(M));
    for (long q = 0; q < 4L * M; ++q) key[q] = c.tets[q] * stride + c.tags[q >> 2];
    const vector<int> order = stable_argsort(key);
    r.ptr.clear();
    r.idx.assign(order.begin(), order.end());
    r.slot_of_corner.assign(4 * static_cast<size_t>(M), 0);
    r.slot_node.clear();
    r.slot_tag.clear();
    for (long i = 0; i < 4L * M; ++i) {
        const long k = key[order[i]];
        if (i == 0 || k != key[order[i - 1]]) {
            r.ptr.push_back(static_cast<int>(i));
            r.slot_node.push_back(static_cast<int>(k / stride));
            r.slot_tag.push_back(static_cast<int>(k % stride));
        }
        r.slot_of_corner[order[i]] = static_cast<int>(r.slot_node.size()) - 1;
    }
    r.ptr.push_back(static_cast<int>(4L * M));
}

// Nodes on a face that exactly one tetrahedron owns (recovery.cu:46-110).
vector<int> outer_boundary(const Ctx& c) {
    const int M = c.n_tets;
    struct Face {
        int a, b, c;
        bool operator<(const Face& o) const {
            return a != o.a ? a < o.a : (b != o.b ? b < o.b : c < o.c);
        }
        bool operator==(const Face& o) const { return a == o.a && b == o.b && c == o.c; }
    };
    vector<Face> faces;
    faces.reserve(4 * static_cast<size_t>(M));
    for (int e = 0; e < M; ++e)
        for (int skip = 0; skip < 4; ++skip) {
            int v[3], m = 0;
            for (int i = 0; i < 4; ++i)
                if (i != skip) v[m++] = c.tets[4 * e + i];
            std::sort(v, v + 3);
            faces.push_back({v[0], v[1], v[2]});
        }
    std::sort(faces.begin(), faces.end());
    vector<int> mark(c.n_nodes, 0);
    for (size_t i = 0; i < faces.size();) {
        size_t j = i + 1;
        while (j < faces.size() && faces[j] == faces[i]) ++j;
        if (j - i == 1) mark[faces[i].a] = mark[faces[i].b] = mark[faces[i].c] = 1;
        i = j;
    }
    return mark;
}

// Cholesky of the lower triangle of an n x n SPD matrix (row-major, n <= 16); false on a pivot at
// or below 1e-12 * A[0][0] (recovery.cu:119-152 pivot rule).
bool chol_factor(const double* A, int n, double* L) {
    const double floor_pivot = 1e-12 * A[0];
    for (int j = 0; j < n; ++j) {
        double d = A[j * n + j];
        for (int k = 0; k < j; ++k) d = d - L[j * n + k] * L[j * n + k];
        if (!(d > floor_pivot)) return false;
        L[j * n + j] = std::sqrt(d);
        for (int i = j + 1; i < n; ++i) {
            double s = A[i * n + j];
            for (int k = 0; k < j; ++k) s = s - L[i * n + k] * L[j * n + k];
            L[i * n + j] = s / L[j * n + j];
        }
    }
    return true;
}

// Row `row` of A^-1 from the factor: forward then backward substitution against e_row.
void chol_unit_solve(const double* L, int n, int row, double* z) {
    double y[16];
    for (int i = 0; i < n; ++i) {
        double s = (i == row) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s = s - L[i * n + k] * y[k];
        y[i] = s / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < n; ++k) s = s - L[k * n + i] * z[k];
        z[i] = s / L[i * n + i];
    }
}

// SPR weights, one slot at a time (recovery.cu:166-283): linear fit over the barycentres of the
// slot's corners in the node-centred frame [1, (b - x_n)/h]; boundary slots, ill-posed fits and
// fits with sum|w| > 8 take the volume-weighted average.
void spr_weights(const Ctx& c, Recovery& r, bool node_slots) {
    const int S = static_cast<int>(r.ptr.size()) - 1;
    r.w.assign(r.idx.size(), 0.0f);
    int fallbacks = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : fallbacks)
    for (int s = 0; s < S; ++s) {
        const int node = node_slots ? s : r.slot_node[s];
        const int begin = r.ptr[s], end = r.ptr[s + 1], count = end - begin;
        if (count <= 0) continue;
        const double* xn = &c.nodes[3 * static_cast<size_t>(node)];
        bool fit = count >= 4 && !r.is_boundary[node];
        double h = 1.0;
        if (fit) {
            h = 0.0;
            for (int p = begin; p < end; ++p) {
                const double* b = &c.bary[3 * static_cast<size_t>(r.idx[p] >> 2)];
                for (int a = 0; a < 3; ++a) h = std::max(h, std::fabs(b[a] - xn[a]));
            }
            fit = h > 0.0;
        }
        double z[4] = {1.0, 0.0, 0.0, 0.0};
        auto basis = [&](int p, double* q) {
            const double* b = &c.bary[3 * static_cast<size_t>(r.idx[p] >> 2)];
            q[0] = 1.0;
            for (int a = 0; a < 3; ++a) q[1 + a] = (b[a] - xn[a]) / h;
        };
        auto weight = [&](const double* q) {
            double acc = 0.0;
            for (int i = 0; i < 4; ++i) acc = std::fma(z[i], q[i], acc);
            return acc;
        };
        if (fit) {
            double A[16] = {}, L[16] = {};
            for (int p = begin; p < end; ++p) {
                double q[4];
                basis(p, q);
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j <= i; ++j) A[i * 4 + j] = std::fma(q[i], q[j], A[i * 4 + j]);
            }
            fit = chol_factor(A, 4, L);
            if (fit) chol_unit_solve(L, 4, 0, z);
        }
        if (fit) {
            double leb = 0.0;
            for (int p = begin; p < end; ++p) {
                double q[4];
                basis(p, q);
                leb = leb + std::fabs(weight(q));
            }
            fit = leb <= kMaxLebesgue;
        }
        if (!fit) {
            ++fallbacks;
            double total = 0.0;
            for (int p = begin; p < end; ++p) total = total + static_cast<double>(c.vols_f32[r.idx[p] >> 2]);
            const bool by_volume = total > 0.0;
            const double inv = by_volume ? 1.0 / total : 1.0 / static_cast<double>(count);
            for (int p = begin; p < end; ++p) {
                const double num = by_volume ? static_cast<double>(c.vols_f32[r.idx[p] >> 2]) : 1.0;
                r.w[p] = static_cast<float>(num * inv);
            }
            continue;
        }
        for (int p = begin; p < end; ++p) {
            double q[4];
            basis(p, q);
            r.w[p] = static_cast<float>(weight(q));
        }
    }
    r.counts = {S, fallbacks, 0};
}

// Harmonic bases in the scaled frame (recovery.cu:285-362): 16 cubic, 9 quadratic, 4 linear terms.
int eval_basis(int rung, double u, double v, double t, double* p) {
    p[0] = 1.0;
    p[1] = u;
    p[2] = v;
    p[3] = t;
    if (rung == 2) return 4;
    p[4] = u * u - v * v;
    p[5] = v * v - t * t;
    p[6] = u * v;
    p[7] = u * t;
    p[8] = v * t;
    if (rung == 1) return 9;
    const double uu = u * u, vv = v * v, tt = t * t;
    p[9] = t * (2.0 * tt - 3.0 * uu - 3.0 * vv);
    p[10] = u * (4.0 * tt - uu - vv);
    p[11] = v * (4.0 * tt - uu - vv);
    p[12] = t * (uu - vv);
    p[13] = u * v * t;
    p[14] = u * (uu - 3.0 * vv);
    p[15] = v * (3.0 * uu - vv);
    return 16;
}

// Patches: the distinct nodes of a slot's own tetrahedra, grown to the union of its neighbours'
// rings where that holds fewer than 16 nodes (recovery.py:253-312; pattern.cu:86-138).
void harmonic_patches(const Ctx& c, Recovery& r) {
    const int S = static_cast<int>(r.slot_node.size());
    int max_tag = 0;
    for (int t : r.slot_tag) max_tag = std::max(max_tag, t);
    const long stride = max_tag + 1;
    vector<vector<int>> ring(S);
#pragma omp parallel for schedule(dynamic, 256)
    for (int s = 0; s < S; ++s) {
        vector<int>& out = ring[s];
        for (int p = r.ptr[s]; p < r.ptr[s + 1]; ++p) {
            const int e = r.idx[p] >> 2;
            for (int i = 0; i < 4; ++i) out.push_back(c.tets[4 * e + i]);
        }
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
    }
    vector<long> slot_key(S);
    for (int s = 0; s < S; ++s) slot_key[s] = r.slot_node[s] * stride + r.slot_tag[s];
    vector<vector<int>> patch(S);
#pragma omp parallel for schedule(dynamic, 256)
    for (int s = 0; s < S; ++s) {
        if (static_cast<int>(ring[s].size()) >= kMinPatchNodes) {
            patch[s] = ring[s];
            continue;
        }
        vector<int> out;
        for (int m : ring[s]) {
            const long key = m * stride + r.slot_tag[s];
            const int nb = static_cast<int>(std::lower_bound(slot_key.begin(), slot_key.end(), key) - slot_key.begin());
            out.insert(out.end(), ring[nb].begin(), ring[nb].end());
        }
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
        patch[s] = std::move(out);
    }
    r.ptr.assign(S + 1, 0);
    for (int s = 0; s < S; ++s) r.ptr[s + 1] = r.ptr[s] + static_cast<int>(patch[s].size());
    r.idx.resize(r.ptr[S]);
    for (int s = 0; s < S; ++s) std::copy(patch[s].begin(), patch[s].end(), r.idx.begin() + r.ptr[s]);
}

// One rung of the potential fit over slot s (recovery.cu:364-511): normal matrix accumulated over
// the patch in order, Cholesky, rows 1..3 of the inverse, gradient weights w = grad / h. Accepted
// when max_c sum_p |grad_c| <= 50, that sum taken as 32 strided partials (entry p to partial
// (p - begin) % 32) folded by halving.
bool harmonic_rung(const double* xm, const int* pidx, int begin, int end, const double* xn, double h, int rung,
                   float* w) {
    static const int kMin[3] = {20, 9, 4};
    const int n = rung == 0 ? 16 : (rung == 1 ? 9 : 4);
    if (end - begin < kMin[rung]) return false;
    double A[256] = {}, L[256] = {}, q[16];
    auto eval = [&](int p) {
        const double* x = &xm[3 * static_cast<size_t>(pidx[p])];
        eval_basis(rung, (x[0] - xn[0]) / h, (x[1] - xn[1]) / h, (x[2] - xn[2]) / h, q);
    };
    for (int p = begin; p < end; ++p) {
        eval(p);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j <= i; ++j) A[i * n + j] = std::fma(q[i], q[j], A[i * n + j]);
    }
    if (!chol_factor(A, n, L)) return false;
    double z[3][16];
    for (int cdir = 0; cdir < 3; ++cdir) chol_unit_solve(L, n, cdir + 1, z[cdir]);
    double part[3][32] = {};
    for (int p = begin; p < end; ++p) {
        eval(p);
        for (int cdir = 0; cdir < 3; ++cdir) {
            double g = 0.0;
            for (int i = 0; i < n; ++i) g = std::fma(z[cdir][i], q[i], g);
            part[cdir][(p - begin) % 32] = part[cdir][(p - begin) % 32] + std::fabs(g);
            w[3 * static_cast<size_t>(p) + cdir] = static_cast<float>(g / h);
        }
    }
    double worst = 0.0;
    for (int cdir = 0; cdir < 3; ++cdir) {
        for (int off = 16; off >= 1; off >>= 1)
            for (int l = 0; l < off; ++l) part[cdir][l] = part[cdir][l] + part[cdir][l + off];
        worst = std::max(worst, part[cdir][0]);
    }
    return worst <= kMaxGradAmp;
}

void harmonic_weights(const Ctx& c, Recovery& r) {
    const int S = static_cast<int>(r.slot_node.size());
    vector<double> xm(c.nodes.size());
    for (size_t i = 0; i < xm.size(); ++i) xm[i] = c.nodes[i] * 1e-3;
    r.w.assign(3 * r.idx.size(), 0.0f);
    r.status.assign(S, 3);
#pragma omp parallel for schedule(dynamic, 128)
    for (int s = 0; s < S; ++s) {
        const int begin = r.ptr[s], end = r.ptr[s + 1];
        const double* xn = &xm[3 * static_cast<size_t>(r.slot_node[s])];
        double h = 0.0;
        for (int p = begin; p < end; ++p)
            for (int a = 0; a < 3; ++a) h = std::max(h, std::fabs(xm[3 * static_cast<size_t>(r.idx[p]) + a] - xn[a]));
        int rung = 3;
        if (h > 0.0) {
            for (int t = 0; t < 3 && rung == 3; ++t)
                if (harmonic_rung(xm.data(), r.idx.data(), begin, end, xn, h, t, r.w.data())) rung = t;
        }
        if (rung == 3)
            for (int p = begin; p < end; ++p) r.w[3 * p] = r.w[3 * p + 1] = r.w[3 * p + 2] = 0.0f;
        r.status[s] = rung;
    }
    int fb = 0, und = 0;
    for (int st : r.status) {
        fb += st >= 2;
        und += st == 3;
    }
    r.counts = {S, fb, und};
}

void build_recovery(Ctx& c, int mode) {
    if (mode < 1 || mode > 3) throw std::invalid_argument("unknown recovery mode");
    Recovery& r = c.rec[mode];
    if (r.built) return;
    r = Recovery();
    if (mode == 1) {
        r.ptr = c.n2c_ptr;
        r.idx = c.n2c_idx;
        r.slot_of_corner = c.tets;
        r.slot_node.resize(c.n_nodes);
        std::iota(r.slot_node.begin(), r.slot_node.end(), 0);
        r.is_boundary = outer_boundary(c);
        spr_weights(c, r, true);
    } else if (mode == 2) {
        tissue_slots(c, r);
        r.is_boundary = outer_boundary(c);
        // A node touching more than one tissue is on each tissue's submesh boundary (recovery.py:127-158).
        for (size_t s = 1; s < r.slot_node.size(); ++s)
            if (r.slot_node[s] == r.slot_node[s - 1]) r.is_boundary[r.slot_node[s]] = 1;
        spr_weights(c, r, false);
    } else {
        tissue_slots(c, r);
        harmonic_patches(c, r);
        harmonic_weights(c, r);
    }
    r.built = true;
}

// Apply, FP64 ground truth on slots, then sampled at the barycentres (recovery.cu:513-687).
// Harmonic: E_s = -sum_p w_p v_m - dA/dt(x_node); SPR: E_s = sum_p w_p E_e.
void apply_recovery_f64(const Ctx& c, int mode, const double* v, const double* dadt_nodes, const double* E_elem,
                        vector<double>& slots, float* magn, double* E_out) {
    const Recovery& r = c.rec[mode];
    const int S = static_cast<int>(r.ptr.size()) - 1;
    slots.assign(3 * static_cast<size_t>(S), 0.0);
#pragma omp parallel for schedule(static)
    for (int s = 0; s < S; ++s) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int p = r.ptr[s]; p < r.ptr[s + 1]; ++p) {
            if (mode == 3) {
                const double vm = v[r.idx[p]];
                for (int a = 0; a < 3; ++a) acc[a] = std::fma(static_cast<double>(r.w[3 * static_cast<size_t>(p) + a]), vm, acc[a]);
            } else {
                const double* ee = &E_elem[3 * static_cast<size_t>(r.idx[p] >> 2)];
                for (int a = 0; a < 3; ++a) acc[a] = std::fma(static_cast<double>(r.w[p]), ee[a], acc[a]);
            }
        }
        for (int a = 0; a < 3; ++a)
            slots[3 * static_cast<size_t>(s) + a] =
                mode == 3 ? -acc[a] - dadt_nodes[3 * static_cast<size_t>(r.slot_node[s]) + a] : acc[a];
    }
#pragma omp parallel for schedule(static)
    for (int e = 0; e < c.n_tets; ++e) {
        double sx[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 4; ++i)
            for (int a = 0; a < 3; ++a) sx[a] = sx[a] + slots[3 * static_cast<size_t>(r.slot_of_corner[4 * e + i]) + a];
        for (int a = 0; a < 3; ++a) sx[a] = sx[a] * 0.25;
        if (E_out)
            for (int a = 0; a < 3; ++a) E_out[3 * static_cast<size_t>(e) + a] = sx[a];
        magn[e] = static_cast<float>(std::sqrt(sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]));
    }
}

void set_err(char* err, int len, const std::string& msg) {
    if (err && len > 0) std::snprintf(err, static_cast<size_t>(len), "%s", msg.c_str());
}

}  // namespace

extern "C" {

void orc_params_default(orc_params* p) {
    p->min_coarse_rows = 128;
    p->max_levels = 50;
    p->agg_rounds = 2;
    p->cheby_degree = 2;
    p->cheby_lower_ratio = 12.0;
    p->n_threads = 0;
    p->has_sigma = 0;
    for (double& v : p->sigma_by_tag) v = 0.0;
}

void* orc_ctx_create(const double* nodes_mm, int n_nodes, const int* tet_nodes, const int* tet_tags,
                     int n_tets, const int* skin_tris, int n_skin, const orc_params* params,
                     char* err, int err_len) {
    try {
        Ctx* c = new Ctx();
        if (params) c->prm = *params;
        else orc_params_default(&c->prm);
#ifdef _OPENMP
        if (c->prm.n_threads > 0) omp_set_num_threads(c->prm.n_threads);
#endif
        c->n_nodes = n_nodes;
        c->n_tets = n_tets;
        c->n_skin = n_skin;
        const vector<double> nodes0(nodes_mm, nodes_mm + 3 * static_cast<size_t>(n_nodes));
        const vector<int> tets0(tet_nodes, tet_nodes + 4 * static_cast<size_t>(n_tets));
        for (int i = 0; i < 4 * n_tets; ++i)
            if (tets0[i] < 0 || tets0[i] >= n_nodes) throw std::invalid_argument("tet_nodes out of range");
        // Morton layout (fem/solve.py:645-662).
        c->node_perm = morton_order(nodes0, n_nodes);
        vector<int> inverse(n_nodes);
        for (int i = 0; i < n_nodes; ++i) inverse[c->node_perm[i]] = i;
        vector<int> lowest(n_tets);
        for (int e = 0; e < n_tets; ++e) {
            int lo = inverse[tets0[4 * e]];
            for (int j = 1; j < 4; ++j) lo = std::min(lo, inverse[tets0[4 * e + j]]);
            lowest[e] = lo;
        }
        c->tet_perm = stable_argsort(lowest);
        c->nodes.resize(3 * static_cast<size_t>(n_nodes));
        for (int i = 0; i < n_nodes; ++i)
            for (int a = 0; a < 3; ++a) c->nodes[3 * i + a] = nodes0[3 * c->node_perm[i] + a];
        c->tets.resize(4 * static_cast<size_t>(n_tets));
        c->tags.resize(n_tets);
        for (int e = 0; e < n_tets; ++e) {
            const int src = c->tet_perm[e];
            for (int j = 0; j < 4; ++j) c->tets[4 * e + j] = inverse[tets0[4 * src + j]];
            c->tags[e] = tet_tags[src];
        }
        c->skin.resize(3 * static_cast<size_t>(n_skin));
        for (int i = 0; i < 3 * n_skin; ++i) c->skin[i] = inverse[skin_tris[i]];

        p1_gradients(c->nodes, c->tets, n_tets, c->g, c->vols);
        for (int e = 0; e < n_tets; ++e)
            if (!(c->vols[e] > 0.0) || !std::isfinite(c->vols[e]))
                throw std::invalid_argument("zero or non-finite tetrahedron volume");
        c->cond.resize(n_tets);
        for (int e = 0; e < n_tets; ++e) {
            c->cond[e] = tissue_sigma(c->tags[e]);
            if (std::isnan(c->cond[e])) throw std::invalid_argument("unknown tissue tag");
            if (c->prm.has_sigma) c->cond[e] = c->prm.sigma_by_tag[c->tags[e]];  // a conductivity draw
        }
        node2corner(c->tets, 4, n_nodes, c->n2c_ptr, c->n2c_idx);
        c->stiff = assemble_stiffness(*c);
        c->ground = 0;
        for (int i = 1; i < n_nodes; ++i)
            if (c->nodes[3 * i + 2] < c->nodes[3 * c->ground + 2]) c->ground = i;
        for (int i = 0; i < n_nodes; ++i)
            if (i != c->ground) c->red_idx.push_back(i);
        build_hierarchy(*c);
        c->bary.resize(3 * static_cast<size_t>(n_tets));
        c->vols_f32.resize(n_tets);
        for (int e = 0; e < n_tets; ++e) {
            for (int a = 0; a < 3; ++a)
                c->bary[3 * e + a] = (c->nodes[3 * c->tets[4 * e] + a] + c->nodes[3 * c->tets[4 * e + 1] + a] +
                                      c->nodes[3 * c->tets[4 * e + 2] + a] + c->nodes[3 * c->tets[4 * e + 3] + a]) /
                                     4.0;
            c->vols_f32[e] = static_cast<float>(c->vols[e]);
        }
        skin_normals(*c);
        return c;
    } catch (const std::exception& ex) {
        set_err(err, err_len, ex.what());
        return nullptr;
    }
}

void orc_ctx_destroy(void* ctx) { delete static_cast<Ctx*>(ctx); }

int orc_n_levels(void* ctx) { return static_cast<int>(static_cast<Ctx*>(ctx)->levels.size()); }

int orc_get_i32(void* ctx, const char* name, int level, const int** ptr, long* len) {
    Ctx* c = static_cast<Ctx*>(ctx);
    const std::string n(name);
    const vector<int>* v = nullptr;
    if (n == "node_perm") v = &c->node_perm;
    else if (n == "tet_perm") v = &c->tet_perm;
    else if (n == "tet_nodes") v = &c->tets;
    else if (n == "tet_tags") v = &c->tags;
    else if (n == "skin_tris") v = &c->skin;
    else if (n == "n2c_ptr") v = &c->n2c_ptr;
    else if (n == "n2c_idx") v = &c->n2c_idx;
    else if (n == "stiff_ptr") v = &c->stiff.ptr;
    else if (n == "stiff_col") v = &c->stiff.col;
    else if (n == "level_sizes") v = &c->level_sizes;
    else if (level >= 0 && level < static_cast<int>(c->levels.size())) {
        const Level& L = c->levels[level];
        if (n == "a_ptr") v = &L.a.ptr;
        else if (n == "a_col") v = &L.a.col;
        else if (n == "agg") v = &L.agg;
        else if (n == "p_ptr") v = &L.p.ptr;
        else if (n == "p_col") v = &L.p.col;
    }
    if (n == "coarse_ptr") v = &c->coarse.ptr;
    if (n == "coarse_col") v = &c->coarse.col;
    if (n == "ground") {
        *ptr = &c->ground;
        *len = 1;
        return 0;
    }
    if (!v) return -1;
    *ptr = v->data();
    *len = static_cast<long>(v->size());
    return 0;
}

int orc_get_f64(void* ctx, const char* name, int level, const double** ptr, long* len) {
    Ctx* c = static_cast<Ctx*>(ctx);
    const std::string n(name);
    const vector<double>* v = nullptr;
    if (n == "nodes_mm") v = &c->nodes;
    else if (n == "g") v = &c->g;
    else if (n == "vols") v = &c->vols;
    else if (n == "cond") v = &c->cond;
    else if (n == "bary") v = &c->bary;
    else if (n == "stiff_val") v = &c->stiff.val;
    else if (n == "skin_normals") v = &c->skin_normals;
    else if (n == "coarse_val") v = &c->coarse.val;
    else if (n == "coarse_inv") v = &c->coarse_inv;
    else if (level >= 0 && level < static_cast<int>(c->levels.size())) {
        const Level& L = c->levels[level];
        if (n == "a_val") v = &L.a.val;
        else if (n == "p_val") v = &L.p.val;
        else if (n == "dinv") v = &L.dinv;
    }
    if (!v) return -1;
    *ptr = v->data();
    *len = static_cast<long>(v->size());
    return 0;
}

int orc_vcycle_apply(void* ctx, const double* r, double* z, int k) {
    const Ctx* c = static_cast<Ctx*>(ctx);
    const int n = c->levels.empty() ? c->coarse.n : c->levels[0].a.n;
    vector<double> b(n), x(n);
    for (int col = 0; col < k; ++col) {
        for (int i = 0; i < n; ++i) b[i] = r[static_cast<size_t>(i) * k + col];
        vcycle(*c, b.data(), x.data());
        for (int i = 0; i < n; ++i) z[static_cast<size_t>(i) * k + col] = x[i];
    }
    return 0;
}

int orc_select_size4(int n, const int* row_ptr, const int* col_idx, const float* values, int* aggregates) {
    return select_size4(n, row_ptr, col_idx, values, aggregates);
}

void orc_l1_dinv_f32(int n, const int* rp, const int* ci, const float* va, float* dinv) {
    for (int i = 0; i < n; ++i) {
        float acc = 0.0f, diag = 0.0f;
        for (int p = rp[i]; p < rp[i + 1]; ++p) {
            acc = acc + std::fabs(va[p]);
            if (ci[p] == i) diag = va[p];
        }
        if (diag < 0.0f) acc = -acc;
        if (acc == 0.0f) acc = 1.0f;
        dinv[i] = 1.0f / acc;
    }
}

// dA/dt = didt * mu0/4pi * sum_j m_j x (r - s_j) / |r - s_j|^3 (fem/placement.py:279-317).
void orc_dadt(const double* dip_pos_m, const double* dip_moment, int n_dip, const double* T,
              double didt, const double* nodes_mm, int n_nodes, double* out) {
    vector<double> s(3 * static_cast<size_t>(n_dip)), m(3 * static_cast<size_t>(n_dip));
    for (int j = 0; j < n_dip; ++j) {
        for (int a = 0; a < 3; ++a) {
            double ps = 0.0, pm = 0.0;
            for (int b = 0; b < 3; ++b) {
                ps = ps + T[4 * a + b] * (dip_pos_m[3 * j + b] * 1e3);
                pm = pm + T[4 * a + b] * dip_moment[3 * j + b];
            }
            s[3 * j + a] = (ps + T[4 * a + 3]) * 1e-3;
            m[3 * j + a] = pm;
        }
    }
    const double scale = didt * 1e-7;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_nodes; ++i) {
        const double r[3] = {nodes_mm[3 * i] * 1e-3, nodes_mm[3 * i + 1] * 1e-3, nodes_mm[3 * i + 2] * 1e-3};
        double acc[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < n_dip; ++j) {
            const double d[3] = {r[0] - s[3 * j], r[1] - s[3 * j + 1], r[2] - s[3 * j + 2]};
            const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const double w = 1.0 / (d2 * std::sqrt(d2));
            const double* mj = &m[3 * j];
            acc[0] = acc[0] + w * (mj[1] * d[2] - mj[2] * d[1]);
            acc[1] = acc[1] + w * (mj[2] * d[0] - mj[0] * d[2]);
            acc[2] = acc[2] + w * (mj[0] * d[1] - mj[1] * d[0]);
        }
        for (int a = 0; a < 3; ++a) out[3 * i + a] = scale * acc[a];
    }
}

int orc_place(void* ctx, const double* centers, const double* handles, const double* dists, int k,
              double* transforms, int* degenerate) {
    const Ctx* c = static_cast<Ctx*>(ctx);
    try {
        for (int p = 0; p < k; ++p)
            place_one(*c, centers + 3 * p, handles ? handles + 3 * p : nullptr, dists[p], transforms + 16 * p,
                      degenerate ? degenerate + p : nullptr);
    } catch (const std::exception&) {
        return -1;
    }
    return 0;
}

void orc_summary(const float* magnE, const float* vols, const double* bary, const int* tags, int n_tets,
                 int region_tag, double* out) {
    summary_impl(magnE, vols, bary, tags, n_tets, region_tag, out);
}

void orc_weighted_quantiles(const double* values, const double* weights, int n, const double* qs, int nq,
                            double* out) {
    weighted_quantiles_impl(values, weights, n, qs, nq, out);
}

int orc_solve(void* ctx, const double* dip_pos_m, const double* dip_moment, int n_dip,
              const double* centers_mm, const double* handles_mm, const double* dists_mm, int k, double didt,
              double tolerance, int max_iters, int recovery, double* transforms, double* v_out, float* magnE_out,
              float* E_out, double* summary, int* iters, double* relres, char* err, int err_len) {
    Ctx* c = static_cast<Ctx*>(ctx);
    try {
        if (recovery != ORC_REC_RAW) build_recovery(*c, recovery);
        vector<double> rec_slots, rec_E;
        const int N = c->n_nodes, M = c->n_tets;
        vector<double> T(16), dadt(3 * static_cast<size_t>(N)), elm(3 * static_cast<size_t>(M)), b(N);
        vector<double> v(N), E(3 * static_cast<size_t>(M));
        vector<float> mag(M);
        for (int p = 0; p < k; ++p) {
            int deg = 0;
            place_one(*c, centers_mm + 3 * p, handles_mm + 3 * p, dists_mm[p], T.data(), &deg);
            if (deg) throw std::invalid_argument("degenerate coil placement: handle on the scalp normal");
            if (transforms) std::copy(T.begin(), T.end(), transforms + 16 * p);
            orc_dadt(dip_pos_m, dip_moment, n_dip, T.data(), didt, c->nodes.data(), N, dadt.data());
            // Element average, then b[n] = sum over corners of -vol*sigma*(dadt_e . g_c)
            // (dadt_element.cu:6-31, rhs.cu:4-6).
#pragma omp parallel for schedule(static)
            for (int e = 0; e < M; ++e)
                for (int a = 0; a < 3; ++a)
                    elm[3 * e + a] = 0.25 * (dadt[3 * c->tets[4 * e] + a] + dadt[3 * c->tets[4 * e + 1] + a] +
                                             dadt[3 * c->tets[4 * e + 2] + a] + dadt[3 * c->tets[4 * e + 3] + a]);
#pragma omp parallel for schedule(static)
            for (int nd = 0; nd < N; ++nd) {
                double acc = 0.0;
                for (int q = c->n2c_ptr[nd]; q < c->n2c_ptr[nd + 1]; ++q) {
                    const int corner = c->n2c_idx[q];
                    const int e = corner >> 2;
                    const double* gc = &c->g[3 * static_cast<size_t>(corner)];
                    const double d = elm[3 * e] * gc[0] + elm[3 * e + 1] * gc[1] + elm[3 * e + 2] * gc[2];
                    acc = acc + (-(c->vols[e] * c->cond[e])) * d;
                }
                b[nd] = acc;
            }
            vector<double> bred(N - 1), x;
            for (int i = 0; i < N - 1; ++i) bred[i] = b[c->red_idx[i]];
            double rel = 0.0;
            const int it = pcg(*c, bred, x, tolerance, max_iters, rel);
            if (iters) iters[p] = it;
            if (relres) relres[p] = rel;
            std::fill(v.begin(), v.end(), 0.0);
            for (int i = 0; i < N - 1; ++i) v[c->red_idx[i]] = x[i];
            if (v_out) std::copy(v.begin(), v.end(), v_out + static_cast<size_t>(p) * N);
            // E = -grad v - dadt_e (reconstruct.cu:12-33).
#pragma omp parallel for schedule(static)
            for (int e = 0; e < M; ++e) {
                double gr[3] = {0.0, 0.0, 0.0};
                for (int i = 0; i < 4; ++i) {
                    const double vi = v[c->tets[4 * e + i]];
                    for (int a = 0; a < 3; ++a) gr[a] = gr[a] + vi * c->g[12 * static_cast<size_t>(e) + 3 * i + a];
                }
                double ee[3];
                for (int a = 0; a < 3; ++a) ee[a] = -gr[a] - elm[3 * e + a];
                for (int a = 0; a < 3; ++a) E[3 * static_cast<size_t>(e) + a] = ee[a];
                mag[e] = static_cast<float>(std::sqrt(ee[0] * ee[0] + ee[1] * ee[1] + ee[2] * ee[2]));
            }
            if (recovery != ORC_REC_RAW) {
                rec_E.resize(3 * static_cast<size_t>(M));
                apply_recovery_f64(*c, recovery, v.data(), dadt.data(), E.data(), rec_slots, mag.data(), rec_E.data());
                E.swap(rec_E);
            }
            if (magnE_out) std::copy(mag.begin(), mag.end(), magnE_out + static_cast<size_t>(p) * M);
            if (E_out)
                for (size_t i = 0; i < 3 * static_cast<size_t>(M); ++i)
                    E_out[static_cast<size_t>(p) * 3 * M + i] = static_cast<float>(E[i]);
            if (summary)
                summary_impl(mag.data(), c->vols_f32.data(), c->bary.data(), c->tags.data(), M, 2,
                             summary + static_cast<size_t>(p) * ORC_SUMMARY_LEN);
        }
        return 0;
    } catch (const std::exception& ex) {
        set_err(err, err_len, ex.what());
        return -1;
    }
}

int orc_recovery_build(void* ctx, int mode, char* err, int err_len) {
    try {
        build_recovery(*static_cast<Ctx*>(ctx), mode);
        return 0;
    } catch (const std::exception& ex) {
        set_err(err, err_len, ex.what());
        return -1;
    }
}

int orc_recovery_i32(void* ctx, int mode, const char* name, const int** ptr, long* len) {
    Ctx* c = static_cast<Ctx*>(ctx);
    if (mode < 1 || mode > 3 || !c->rec[mode].built) return -1;
    const Recovery& r = c->rec[mode];
    const std::string n(name);
    const vector<int>* v = nullptr;
    if (n == "ptr") v = &r.ptr;
    else if (n == "idx") v = &r.idx;
    else if (n == "slot_of_corner") v = &r.slot_of_corner;
    else if (n == "slot_node") v = &r.slot_node;
    else if (n == "slot_tag") v = &r.slot_tag;
    else if (n == "status") v = &r.status;
    else if (n == "is_boundary") v = &r.is_boundary;
    else if (n == "counts") v = &r.counts;
    if (!v) return -1;
    *ptr = v->data();
    *len = static_cast<long>(v->size());
    return 0;
}

int orc_recovery_w(void* ctx, int mode, const float** ptr, long* len) {
    Ctx* c = static_cast<Ctx*>(ctx);
    if (mode < 1 || mode > 3 || !c->rec[mode].built) return -1;
    *ptr = c->rec[mode].w.data();
    *len = static_cast<long>(c->rec[mode].w.size());
    return 0;
}

int orc_recovery_apply(void* ctx, int mode, int k, const double* v, const float* dadt_nodes, const float* E_elem,
                       float* E_slots, float* E_out, float* magn) {
    Ctx* c = static_cast<Ctx*>(ctx);
    if (mode < 1 || mode > 3 || !c->rec[mode].built) return -1;
    const Recovery& r = c->rec[mode];
    const int S = static_cast<int>(r.ptr.size()) - 1, N = c->n_nodes, M = c->n_tets;
    for (int col = 0; col < k; ++col) {
        float* slots = E_slots + static_cast<size_t>(col) * S * 3;
#pragma omp parallel for schedule(static)
        for (int s = 0; s < S; ++s) {
            if (mode == 3) {
                const double* vc = v + static_cast<size_t>(col) * N;
                const float* da = dadt_nodes + (static_cast<size_t>(col) * N + r.slot_node[s]) * 3;
                double acc[3] = {0.0, 0.0, 0.0};
                for (int p = r.ptr[s]; p < r.ptr[s + 1]; ++p) {
                    const double vm = vc[r.idx[p]];
                    for (int a = 0; a < 3; ++a)
                        acc[a] = std::fma(static_cast<double>(r.w[3 * static_cast<size_t>(p) + a]), vm, acc[a]);
                }
                for (int a = 0; a < 3; ++a) slots[3 * static_cast<size_t>(s) + a] = static_cast<float>(-acc[a] - static_cast<double>(da[a]));
            } else {
                const float* ec = E_elem + static_cast<size_t>(col) * M * 3;
                float acc[3] = {0.0f, 0.0f, 0.0f};
                for (int p = r.ptr[s]; p < r.ptr[s + 1]; ++p) {
                    const float* ee = ec + 3 * static_cast<size_t>(r.idx[p] >> 2);
                    for (int a = 0; a < 3; ++a) acc[a] = std::fma(r.w[p], ee[a], acc[a]);
                }
                for (int a = 0; a < 3; ++a) slots[3 * static_cast<size_t>(s) + a] = acc[a];
            }
        }
#pragma omp parallel for schedule(static)
        for (int e = 0; e < M; ++e) {
            double sx[3] = {0.0, 0.0, 0.0};
            for (int i = 0; i < 4; ++i)
                for (int a = 0; a < 3; ++a)
                    sx[a] = sx[a] + static_cast<double>(slots[3 * static_cast<size_t>(r.slot_of_corner[4 * e + i]) + a]);
            for (int a = 0; a < 3; ++a) sx[a] = sx[a] * 0.25;
            if (E_out)
                for (int a = 0; a < 3; ++a) E_out[(static_cast<size_t>(col) * M + e) * 3 + a] = static_cast<float>(sx[a]);
            magn[static_cast<size_t>(col) * M + e] = static_cast<float>(std::sqrt(sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]));
        }
    }
    return 0;
}

}  // extern "C"
