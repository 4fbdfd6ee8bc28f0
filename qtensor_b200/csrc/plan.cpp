// Host plan compiler: circuit -> bucket network -> elimination order ->
// device plan (ops, dependency phases, arena offsets, gate-table entries).
//
// Follows, per step (paths within DaniloZZZ/QTensor):
//   simplify()       qtensor/simplify_circuit/simplify_circuit.py:30-138 and
//                    simplify_circuit_api.py:74-106 (pairs of equal kind on
//                    equal qubits, visited by distance; merge if every gate
//                    in between commutes with the first; cancel below 1e-5)
//   build_network()  qtree circ2buckets as used by TensorNet.py:60-68 (bra
//                    variables first, gates placed from the bra side, ket
//                    measurement tensors last; tensor -> bucket of its
//                    smallest variable)
//   greedy_order()   qtensor/utils.py:12-44,77-87 + Optimizer.py:65-87 (first
//                    node of least distinct-neighbour count, clique fill-in;
//                    peo = ket + bra + greedy)
//   eliminate()      qtree reorder_buckets / get_sliced_np_buckets /
//                    bucket_elimination as driven by Simulate.py:47-94, with
//                    the bucket arithmetic of ProcessingFrameworks.py:45-147
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <tuple>
#include <unordered_map>

#include <sched.h>

#include "plan.h"

namespace qtb {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

bool EntryKey::operator<(const EntryKey& o) const {
    return std::tie(kind, expr, rank_in, sliced_mask, sliced_value, perm) <
           std::tie(o.kind, o.expr, o.rank_in, o.sliced_mask, o.sliced_value, o.perm);
}

int rank_of_kind(int32_t kind) {
    switch (kind) {
        case QTB_GATE_Z: case QTB_GATE_T: case QTB_GATE_ZPHASE: return 1;
        case QTB_GATE_CX: return 3;
        default: return 2;
    }
}

static int qubits_of_kind(int32_t kind) {
    return (kind == QTB_GATE_CX || kind == QTB_GATE_CZ || kind == QTB_GATE_ZZ) ? 2 : 1;
}

static bool is_parametric(int32_t kind) {
    return kind == QTB_GATE_ZPHASE || kind == QTB_GATE_XPHASE || kind == QTB_GATE_YPHASE ||
           kind == QTB_GATE_ZZ;
}

// Position (in the gate's qubit list) of the qubit that gets a new variable,
// or -1 for gates diagonal on all their qubits.
static int changed_position(int32_t kind) {
    switch (kind) {
        case QTB_GATE_M: case QTB_GATE_H: case QTB_GATE_X: case QTB_GATE_Y:
        case QTB_GATE_XPHASE: case QTB_GATE_YPHASE: return 0;
        case QTB_GATE_CX: return 1;
        default: return -1;
    }
}

static Expr expr_add(const Expr& a, const Expr& b) {
    Expr out;
    size_t i = 0, j = 0;
    while (i < a.size() || j < b.size()) {
        if (j == b.size() || (i < a.size() && a[i].first < b[j].first)) {
            out.push_back(a[i++]);
        } else if (i == a.size() || b[j].first < a[i].first) {
            out.push_back(b[j++]);
        } else {
            double c = a[i].second + b[j].second;
            if (c != 0.0) out.emplace_back(a[i].first, c);
            ++i;
            ++j;
        }
    }
    return out;
}

// Runs of the operand bits below the summed bit (see DevIn).
uint64_t encode_runs(uint32_t mask, uint32_t w) {
    const uint32_t low = w >= 32 ? mask : (mask & ((1u << w) - 1u));
    uint64_t runs = 0;
    uint64_t n = 0;
    uint32_t first_start = 0, first_len = 0;
    // runs in ascending bit order: the lowest set bit starts one, and its
    // length is the number of ones from there
    for (uint64_t rest = low; rest;) {
        const uint32_t bit = (uint32_t)__builtin_ctzll(rest);
        const uint32_t len = (uint32_t)__builtin_ctzll(~(rest >> bit));
        if (n == (uint64_t)kMaxRuns) return kRunsFallback << 60;
        if (n == 0) {
            first_start = bit;
            first_len = len;
        }
        runs |= (uint64_t)(bit | (len << 5)) << (10 * n);
        ++n;
        rest &= ~(((1ull << len) - 1ull) << bit);
    }
    if (n <= 1) {   // pre-decoded single run
        const uint64_t lenmask = first_len >= 32 ? 0xffffffffull : ((1ull << first_len) - 1ull);
        return (n == 0 ? 0ull : (lenmask | ((uint64_t)first_start << 32))) | (n << 60);
    }
    return runs | (n << 60);
}

// ------------------------------------------------------------- simplifier
namespace {

enum SKind { SK_ZZ, SK_X, SK_Y, SK_ZP, SK_H, SK_CX, SK_Z, SK_ID };
enum SBasis { SB_Z = 1, SB_X, SB_Y, SB_XY, SB_CA, SB_CB };

// A gate as the simplifier sees it; its symbolic angle is expression
// `expr` of the pass's pool (-1: none), so gates move without copying it.
struct SGate {
    int kind = SK_ID;
    int nq = 0;
    int q[2] = {-1, -1};
    int basis[2] = {0, 0};
    double angle = 0.0;
    int32_t expr = -1;
};

SGate make_sgate(int kind, const int* qs, double angle, int32_t expr) {
    SGate g;
    g.kind = kind;
    g.angle = angle;
    g.expr = expr;
    switch (kind) {
        case SK_ZZ:
            g.nq = 2;
            g.q[0] = std::min(qs[0], qs[1]);
            g.q[1] = std::max(qs[0], qs[1]);
            g.basis[0] = g.basis[1] = SB_Z;
            break;
        case SK_CX:
            g.nq = 2;
            g.q[0] = qs[0];
            g.q[1] = qs[1];
            g.basis[0] = SB_CA;
            g.basis[1] = SB_CB;
            g.angle = 0.0;
            g.expr = -1;
            break;
        case SK_H:
            g.nq = 1;
            g.q[0] = qs[0];
            g.basis[0] = SB_XY;
            g.angle = M_PI / 2.0 / std::sqrt(2.0);   // fixed, gates.py hadamard
            g.expr = -1;
            break;
        case SK_Z:
            g.nq = 1;
            g.q[0] = qs[0];
            g.basis[0] = SB_Z;
            g.angle = 0.0;
            g.expr = -1;
            break;
        case SK_X: case SK_Y: case SK_ZP:
            g.nq = 1;
            g.q[0] = qs[0];
            g.basis[0] = kind == SK_X ? SB_X : (kind == SK_Y ? SB_Y : SB_Z);
            break;
        default:
            g.kind = SK_ID;
            g.nq = 0;
            g.angle = 0.0;
            g.expr = -1;
    }
    return g;
}

bool commute(const SGate& a, const SGate& b) {
    for (int i = 0; i < a.nq; ++i)
        for (int j = 0; j < b.nq; ++j)
            if (a.q[i] == b.q[j] && a.basis[i] != b.basis[j]) return false;
    return true;
}

bool same_site(const SGate& a, const SGate& b) {
    if (a.kind != b.kind || a.nq != b.nq) return false;
    for (int i = 0; i < a.nq; ++i)
        if (a.q[i] != b.q[i]) return false;
    return true;
}

struct Gate {
    int32_t kind;
    int32_t q[2];
    double angle;   // numeric alpha (parametric gates)
    Expr expr;      // symbolic alpha
};

int skind_of(int32_t kind) {
    switch (kind) {
        case QTB_GATE_ZZ: return SK_ZZ;
        case QTB_GATE_XPHASE: return SK_X;
        case QTB_GATE_YPHASE: return SK_Y;
        case QTB_GATE_ZPHASE: return SK_ZP;
        case QTB_GATE_H: return SK_H;
        case QTB_GATE_CX: return SK_CX;
        case QTB_GATE_Z: return SK_Z;
        default: return -1;
    }
}

int32_t kind_of_skind(int sk) {
    switch (sk) {
        case SK_ZZ: return QTB_GATE_ZZ;
        case SK_X: return QTB_GATE_XPHASE;
        case SK_Y: return QTB_GATE_YPHASE;
        case SK_ZP: return QTB_GATE_ZPHASE;
        case SK_H: return QTB_GATE_H;
        case SK_CX: return QTB_GATE_CX;
        default: return QTB_GATE_Z;
    }
}

// One pass of the commutation simplifier over a gate list.
int simplify(std::vector<Gate>* gates, std::vector<AngleCheck>* checks, bool* angle_specific,
             std::string* err) {
    const int n = (int)gates->size();
    if (n == 0) return QTB_OK;
    std::vector<SGate> cir(n);
    std::vector<Expr> pool(n);   // gate i's expression, then merged ones
    for (int i = 0; i < n; ++i) {
        const Gate& g = (*gates)[i];
        int sk = skind_of(g.kind);
        if (sk < 0) {
            *err = "simplifier: gate kind " + std::to_string(g.kind) + " has no commutation record";
            return QTB_ERR_UNSUPPORTED;
        }
        cir[i] = make_sgate(sk, g.q, g.angle, i);
    }
    for (int i = 0; i < n; ++i)
        if (cir[i].expr >= 0) pool[i] = std::move((*gates)[i].expr);
    static const Expr kNoExpr;
    auto expr_of = [&](const SGate& g) -> const Expr& { return g.expr >= 0 ? pool[g.expr] : kNoExpr; };
    // same-site pairs (i < j) visited by distance j - i, ties in order of i:
    // the reference's visiting order, with pairs formed within groups of
    // gates of the same kind on the same qubits instead of over all pairs.
    // Groups: gate indices sorted by (kind, qubits), ties by index.
    auto site_less = [&](int x, int y) {
        const SGate &gx = cir[x], &gy = cir[y];
        if (gx.kind != gy.kind) return gx.kind < gy.kind;
        if (gx.nq != gy.nq) return gx.nq < gy.nq;
        if (gx.q[0] != gy.q[0]) return gx.q[0] < gy.q[0];
        const int x1 = gx.nq > 1 ? gx.q[1] : -1, y1 = gy.nq > 1 ? gy.q[1] : -1;
        return x1 != y1 ? x1 < y1 : x < y;
    };
    std::vector<int> by_site(n), group_end(n), rank(n);
    std::iota(by_site.begin(), by_site.end(), 0);
    std::sort(by_site.begin(), by_site.end(), site_less);
    for (int s = n - 1; s >= 0; --s) {
        const bool last = s == n - 1 || !same_site(cir[by_site[s]], cir[by_site[s + 1]]);
        group_end[s] = last ? s + 1 : group_end[s + 1];
        rank[by_site[s]] = s;
    }
    // pairs generated in order of their first gate, then a stable counting
    // sort by distance: (distance, first) order without a comparison sort
    std::vector<std::pair<int, int>> by_first;
    std::vector<int> count_at(n + 1, 0);
    for (int a = 0; a < n; ++a)
        for (int s = rank[a] + 1; s < group_end[rank[a]]; ++s) {
            by_first.emplace_back(a, by_site[s]);
            ++count_at[by_site[s] - a];
        }
    if (by_first.empty()) return QTB_OK;
    for (int d = 0, acc = 0; d <= n; ++d) {
        const int c = count_at[d];
        count_at[d] = acc;
        acc += c;
    }
    std::vector<std::pair<int, int>> pairs(by_first.size());
    for (const auto& pr : by_first) pairs[count_at[pr.second - pr.first]++] = pr;
    // gates touching each qubit, in circuit order: a gate commutes with
    // every gate that shares none of its qubits, so the commutation scan
    // between a and b only visits the gates on a's qubits
    int n_q = 0;
    for (const SGate& g : cir)
        for (int k = 0; k < g.nq; ++k) n_q = std::max(n_q, g.q[k] + 1);
    std::vector<int> q_begin(n_q + 1, 0), on_qubit, slot(2 * (size_t)n, -1);
    for (const SGate& g : cir)
        for (int k = 0; k < g.nq; ++k) ++q_begin[g.q[k] + 1];
    for (int q = 0; q < n_q; ++q) q_begin[q + 1] += q_begin[q];
    on_qubit.resize(q_begin[n_q]);
    {
        std::vector<int> fill(q_begin.begin(), q_begin.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < cir[i].nq; ++k) {
                slot[2 * (size_t)i + k] = fill[cir[i].q[k]];
                on_qubit[fill[cir[i].q[k]]++] = i;
            }
    }
    for (const auto& pr : pairs) {
        const int a = pr.first, b = pr.second;
        if (cir[a].kind == SK_ID || cir[b].kind == SK_ID) continue;
        bool ok = true;
        for (int k = 0; k < cir[a].nq && ok; ++k) {
            const int end = q_begin[cir[a].q[k] + 1];
            for (int t = slot[2 * (size_t)a + k] + 1; t < end && on_qubit[t] < b && ok; ++t)
                ok = commute(cir[a], cir[on_qubit[t]]);
        }
        if (!ok) continue;
        const double total = cir[a].angle + cir[b].angle;
        Expr sym = expr_add(expr_of(cir[a]), expr_of(cir[b]));
        const bool param = cir[a].kind == SK_ZZ || cir[a].kind == SK_X || cir[a].kind == SK_Y ||
                           cir[a].kind == SK_ZP;
        if (std::fabs(total) < 1e-5) {
            if (param && !sym.empty()) {
                checks->push_back({sym, true});
                *angle_specific = true;
            }
            cir[a] = SGate();
            cir[b] = SGate();
        } else {
            if (param) checks->push_back({sym, false});
            pool.push_back(std::move(sym));
            SGate merged = make_sgate(cir[a].kind, cir[a].q, total, (int32_t)pool.size() - 1);
            cir[a] = SGate();
            cir[b] = merged;
        }
    }
    std::vector<Gate> out;
    for (const SGate& s : cir) {
        if (s.kind == SK_ID) continue;
        Gate g;
        g.kind = kind_of_skind(s.kind);
        g.q[0] = s.q[0];
        g.q[1] = s.nq > 1 ? s.q[1] : -1;
        g.angle = s.angle;
        if (s.expr >= 0) g.expr = std::move(pool[s.expr]);
        out.push_back(std::move(g));
    }
    gates->swap(out);
    return QTB_OK;
}

// ------------------------------------------------------ bucket network
struct TRec {
    int32_t kind;
    Expr expr;
    std::vector<int32_t> vars;   // native axis order
};

// A tensor of a bucket: a gate-table entry or an op's result, with its
// variables (sorted new ids, sliced ones included) at [off, off + len) of
// the circuit's variable pool; `next` links the tensors of one bucket.
struct Ref {
    bool table = false;
    int32_t id = -1;                // local entry id or op id
    int32_t off = 0, len = 0;
    int32_t next = -1;
};

// A bucket operation; its operands are [in_begin, in_begin + k) of the
// build's operand arrays.
struct OpRec {
    int32_t u = 0, sum = 0, w = 0;
    int32_t in_begin = 0, k = 0;
    int32_t level = 0;
    int32_t consumer_level = 0;
    uint32_t dst = 0;
};

}  // namespace

// Greedy minimum-degree elimination on the line graph (cliques = tensors,
// nodes in first-appearance order); returns the order and the degree of
// every eliminated node.  seed 0: the reference's rule, the first node
// (lowest index) of least distinct-neighbour count (qtensor/utils.py:30-32);
// other seeds: a uniformly random node among those of least count
// (xorshift64 on the seed; the zero-temperature limit of RGreedyOptimizer,
// qtensor/optimisation/RGreedy.py:36-62).  Nodes of each degree are
// kept in a bitset, so the lowest-index node of least degree is the lowest
// set bit of the least non-empty bucket and the k-th tie its k-th set bit.
// Returns sum over eliminations of 2^degree.
// The line graph as bit rows (one row of W words per node) with the
// distinct-neighbour count of every node; removed nodes have no edges.
struct LineGraph {
    int V = 0, W = 0;
    std::vector<uint64_t> adj;
    std::vector<int32_t> deg;
};

static void line_graph(int V, const std::vector<std::vector<int32_t>>& cliques,
                       const std::vector<char>& removed, LineGraph* g) {
    g->V = V;
    g->W = (V + 63) / 64;
    const int W = g->W;
    g->adj.assign((size_t)V * W, 0);
    g->deg.assign(V, 0);
    std::vector<uint64_t>& adj = g->adj;
    for (const auto& c : cliques)
        for (size_t i = 0; i < c.size(); ++i)
            for (size_t j = i + 1; j < c.size(); ++j) {
                const int a = c[i], b = c[j];
                if (a == b || removed[a] || removed[b] || ((adj[(size_t)a * W + (b >> 6)] >> (b & 63)) & 1))
                    continue;
                adj[(size_t)a * W + (b >> 6)] |= 1ull << (b & 63);
                adj[(size_t)b * W + (a >> 6)] |= 1ull << (a & 63);
                ++g->deg[a];
                ++g->deg[b];
            }
}

static double greedy_order(const LineGraph& g, const std::vector<char>& removed, uint64_t seed,
                           std::vector<int32_t>* order, std::vector<int32_t>* degrees) {
    const int V = g.V, W = g.W;
    static thread_local std::vector<uint64_t> adj;   // working copy, filled in per order
    adj.assign(g.adj.begin(), g.adj.end());
    std::vector<int32_t> deg(g.deg);
    auto gone = [&](int x) { return removed[x] != 0; };
    // degree buckets over the alive nodes: bucket d is W words at d * W
    // (a degree is below V)
    static thread_local std::vector<uint64_t> bucket;
    static thread_local std::vector<int32_t> bucket_count;
    bucket.assign((size_t)std::max(V, 1) * W, 0);
    bucket_count.assign(std::max(V, 1), 0);
    auto add = [&](int x, int d) {
        bucket[(size_t)d * W + (x >> 6)] |= 1ull << (x & 63);
        ++bucket_count[d];
    };
    auto del = [&](int x, int d) {
        bucket[(size_t)d * W + (x >> 6)] &= ~(1ull << (x & 63));
        --bucket_count[d];
    };
    int n_alive = 0;
    for (int x = 0; x < V; ++x)
        if (!gone(x)) {
            add(x, deg[x]);
            ++n_alive;
        }
    std::vector<int32_t> nbrs;
    uint64_t rng = seed;
    double cost = 0.0;
    order->clear();
    degrees->clear();
    // eliminating a node of least degree d leaves every degree at least
    // d - 1, so the search for the next least degree starts there
    int dmin = 0;
    for (; n_alive > 0; --n_alive) {
        dmin = std::max(0, dmin - 1);
        while (bucket_count[dmin] == 0) ++dmin;
        const uint64_t* bk = &bucket[(size_t)dmin * W];
        int x = -1;
        if (seed == 0) {
            for (int w = 0; w < W && x < 0; ++w)
                if (bk[w]) x = w * 64 + __builtin_ctzll(bk[w]);
        } else {
            rng ^= rng << 13;
            rng ^= rng >> 7;
            rng ^= rng << 17;
            int k = (int)(rng % (uint64_t)bucket_count[dmin]);
            for (int w = 0; w < W && x < 0; ++w) {
                const int c = __builtin_popcountll(bk[w]);
                if (k >= c) {
                    k -= c;
                    continue;
                }
                uint64_t bits = bk[w];
                for (; k > 0; --k) bits &= bits - 1;
                x = w * 64 + __builtin_ctzll(bits);
            }
        }
        del(x, dmin);
        nbrs.clear();
        for (int w = 0; w < W; ++w) {
            uint64_t bits = adj[(size_t)x * W + w];
            while (bits) {
                int b = __builtin_ctzll(bits);
                nbrs.push_back(w * 64 + b);
                bits &= bits - 1;
            }
        }
        order->push_back(x);
        degrees->push_back((int32_t)nbrs.size());
        cost += std::ldexp(1.0, (int)nbrs.size());
        // eliminate x: its neighbours become a clique.  Row by row, a
        // neighbour's row takes x's row, loses a and x, and its degree is
        // the row's population (the same graph as joining every pair).
        const uint64_t* rx = &adj[(size_t)x * W];
        for (int a : nbrs) {
            del(a, deg[a]);
            uint64_t* ra = &adj[(size_t)a * W];
            int d = 0;
            for (int w = 0; w < W; ++w) {
                ra[w] |= rx[w];
                if (w == (a >> 6)) ra[w] &= ~(1ull << (a & 63));
                if (w == (x >> 6)) ra[w] &= ~(1ull << (x & 63));
                d += __builtin_popcountll(ra[w]);
            }
            deg[a] = d;
            add(a, d);
        }
    }
    return cost;
}

// Minimum-fill elimination on the same line graph: the next node is the one
// whose elimination adds the fewest new edges among its neighbours (ties:
// least degree, then the lowest index for seed 0 or a random one).  It is
// the classic fill-in heuristic for treewidth (e.g. Bodlaender and Koster,
// "Treewidth computations I. Upper bounds", 2010), used here as extra
// candidates of the native order search; the reference's rule stays
// greedy_order with seed 0.  fill(x) = sum over neighbours a of x of the
// neighbours of x not adjacent to a, halved.  Eliminating x only changes the
// rows of its neighbours, so only they and their neighbours are rescored.
// Returns sum over eliminations of 2^degree.
static double minfill_order(const LineGraph& g, const std::vector<char>& removed, uint64_t seed,
                            std::vector<int32_t>* order, std::vector<int32_t>* degrees) {
    const int V = g.V, W = g.W;
    static thread_local std::vector<uint64_t> adj, touched;
    static thread_local std::vector<int64_t> fill;
    adj.assign(g.adj.begin(), g.adj.end());
    std::vector<int32_t> deg(g.deg);
    fill.assign(V, 0);
    touched.assign(W, 0);
    std::vector<char> alive(V, 0);
    auto row = [&](int x) { return &adj[(size_t)x * W]; };
    auto score = [&](int x) {
        const uint64_t* rx = row(x);
        int64_t f = 0;
        for (int w = 0; w < W; ++w)
            for (uint64_t bits = rx[w]; bits; bits &= bits - 1) {
                const int a = w * 64 + __builtin_ctzll(bits);
                const uint64_t* ra = row(a);
                int64_t miss = 0;
                for (int k = 0; k < W; ++k) miss += __builtin_popcountll(rx[k] & ~ra[k]);
                f += miss - 1;   // a itself is in rx and not in ra
            }
        return f / 2;
    };
    int n_alive = 0;
    for (int x = 0; x < V; ++x)
        if (!removed[x]) {
            alive[x] = 1;
            ++n_alive;
        }
    for (int x = 0; x < V; ++x)
        if (alive[x]) fill[x] = score(x);
    uint64_t rng = seed;
    double cost = 0.0;
    order->clear();
    degrees->clear();
    std::vector<int32_t> nbrs, ties;
    for (; n_alive > 0; --n_alive) {
        int64_t best_f = INT64_MAX;
        int best_d = INT_MAX;
        ties.clear();
        for (int x = 0; x < V; ++x) {
            if (!alive[x]) continue;
            if (fill[x] < best_f || (fill[x] == best_f && deg[x] < best_d)) {
                best_f = fill[x];
                best_d = deg[x];
                ties.clear();
            }
            if (fill[x] == best_f && deg[x] == best_d) ties.push_back(x);
        }
        int x = ties[0];
        if (seed != 0) {
            rng ^= rng << 13;
            rng ^= rng >> 7;
            rng ^= rng << 17;
            x = ties[rng % ties.size()];
        }
        alive[x] = 0;
        nbrs.clear();
        uint64_t* rx = row(x);
        for (int w = 0; w < W; ++w)
            for (uint64_t bits = rx[w]; bits; bits &= bits - 1) nbrs.push_back(w * 64 + __builtin_ctzll(bits));
        order->push_back(x);
        degrees->push_back((int32_t)nbrs.size());
        cost += std::ldexp(1.0, (int)nbrs.size());
        // neighbours become a clique; x leaves the graph
        std::fill(touched.begin(), touched.end(), 0);
        for (int a : nbrs) {
            uint64_t* ra = row(a);
            int d = 0;
            for (int w = 0; w < W; ++w) {
                ra[w] |= rx[w];
                if (w == (a >> 6)) ra[w] &= ~(1ull << (a & 63));
                if (w == (x >> 6)) ra[w] &= ~(1ull << (x & 63));
                d += __builtin_popcountll(ra[w]);
                touched[w] |= ra[w];
            }
            deg[a] = d;
            touched[a >> 6] |= 1ull << (a & 63);
        }
        for (int w = 0; w < W; ++w) rx[w] = 0;
        touched[x >> 6] &= ~(1ull << (x & 63));
        for (int w = 0; w < W; ++w)
            for (uint64_t bits = touched[w]; bits; bits &= bits - 1) {
                const int y = w * 64 + __builtin_ctzll(bits);
                if (alive[y]) fill[y] = score(y);
            }
    }
    return cost;
}

// ------------------------------------------------------ slicing choices
// The reference's line graph as a multigraph (QtreeTensorNet.get_line_graph,
// qtensor/optimisation/TensorNet.py:53-58, through qtree buckets2graph): one
// edge per pair of variables of every tensor and a self-loop for a tensor
// of one variable, multiplicities kept; eliminating a node adds one more
// edge between every pair of its neighbours (qtensor/utils.py:77-87).
// GreedyParvars ranks nodes by the multigraph degree (parallel edges
// counted, a self-loop twice: Greedy.py:78-91); the greedy order only sees
// distinct neighbours, kept as bit rows beside the multiplicities.
struct MultiGraph {
    int V = 0, W = 0;
    std::vector<uint32_t> cnt;    // V x V multiplicities, self-loops on the diagonal
    std::vector<uint64_t> bits;   // V x W distinct neighbours (no self)
    std::vector<int64_t> mdeg;    // multigraph degree
    std::vector<char> alive;

    void init(int v, const std::vector<std::vector<int32_t>>& tensors) {
        V = v;
        W = (V + 63) / 64;
        cnt.assign((size_t)V * V, 0);
        bits.assign((size_t)V * W, 0);
        mdeg.assign(V, 0);
        alive.assign(V, 1);
        for (const auto& t : tensors) {
            if (t.size() == 1) {
                ++cnt[(size_t)t[0] * V + t[0]];
                mdeg[t[0]] += 2;
            }
            for (size_t i = 0; i < t.size(); ++i)
                for (size_t j = i + 1; j < t.size(); ++j) add_edge(t[i], t[j]);
        }
    }
    void add_edge(int a, int b) {
        ++cnt[(size_t)a * V + b];
        ++cnt[(size_t)b * V + a];
        ++mdeg[a];
        ++mdeg[b];
        bits[(size_t)a * W + (b >> 6)] |= 1ull << (b & 63);
        bits[(size_t)b * W + (a >> 6)] |= 1ull << (a & 63);
    }
    void neighbours(int x, std::vector<int32_t>* out) const {
        out->clear();
        for (int w = 0; w < W; ++w)
            for (uint64_t m = bits[(size_t)x * W + w]; m; m &= m - 1) out->push_back(w * 64 + __builtin_ctzll(m));
    }
    // len(graph[x]): distinct neighbours, x itself included when it has a self-loop
    int n_neighbors(int x) const {
        int n = cnt[(size_t)x * V + x] ? 1 : 0;
        for (int w = 0; w < W; ++w) n += __builtin_popcountll(bits[(size_t)x * W + w]);
        return n;
    }
    void drop(int x, std::vector<int32_t>* nb) {
        neighbours(x, nb);
        for (int a : *nb) {
            mdeg[a] -= cnt[(size_t)a * V + x];
            cnt[(size_t)a * V + x] = cnt[(size_t)x * V + a] = 0;
            bits[(size_t)a * W + (x >> 6)] &= ~(1ull << (x & 63));
        }
        for (int w = 0; w < W; ++w) bits[(size_t)x * W + w] = 0;
        cnt[(size_t)x * V + x] = 0;
        mdeg[x] = 0;
        alive[x] = 0;
    }
    // graph.remove_node (slicing a variable)
    void remove(int x) {
        std::vector<int32_t> nb;
        drop(x, &nb);
    }
    // eliminate_node_no_structure
    void eliminate(int x) {
        std::vector<int32_t> nb;
        drop(x, &nb);
        for (size_t i = 0; i < nb.size(); ++i)
            for (size_t j = i + 1; j < nb.size(); ++j) add_edge(nb[i], nb[j]);
    }
    // GreedyParvars.step: the first node (node order) of largest degree
    int max_degree_node() const {
        int best = -1;
        for (int x = 0; x < V; ++x)
            if (alive[x] && (best < 0 || mdeg[x] > mdeg[best])) best = x;
        return best;
    }
    // the simple graph of the live nodes, optionally without node `skip`
    void simple(LineGraph* g, std::vector<char>* removed, int skip = -1) const {
        g->V = V;
        g->W = W;
        g->adj = bits;
        g->deg.assign(V, 0);
        removed->assign(V, 0);
        for (int x = 0; x < V; ++x) (*removed)[x] = alive[x] ? 0 : 1;
        if (skip >= 0) {
            (*removed)[skip] = 1;
            for (int w = 0; w < W; ++w) g->adj[(size_t)skip * W + w] = 0;
            for (int x = 0; x < V; ++x) g->adj[(size_t)x * W + (skip >> 6)] &= ~(1ull << (skip & 63));
        }
        for (int x = 0; x < V; ++x)
            for (int w = 0; w < W; ++w) g->deg[x] += __builtin_popcountll(g->adj[(size_t)x * W + w]);
    }
};

// Widths (neighbour counts at elimination) of `order` on the simple graph g.
static int order_width(const LineGraph& g, const std::vector<char>& removed, const std::vector<int32_t>& order,
                       std::vector<int32_t>* degrees) {
    const int W = g.W;
    std::vector<uint64_t> adj(g.adj);
    std::vector<char> gone(removed);
    degrees->clear();
    int width = 0;
    for (int x : order) {
        if (gone[x]) continue;
        uint64_t* rx = &adj[(size_t)x * W];
        std::vector<int32_t> nb;
        for (int w = 0; w < W; ++w)
            for (uint64_t m = rx[w]; m; m &= m - 1) nb.push_back(w * 64 + __builtin_ctzll(m));
        degrees->push_back((int32_t)nb.size());
        width = std::max(width, (int)nb.size());
        for (int a : nb) {
            uint64_t* ra = &adj[(size_t)a * W];
            for (int w = 0; w < W; ++w) ra[w] |= rx[w];
            ra[a >> 6] &= ~(1ull << (a & 63));
            ra[x >> 6] &= ~(1ull << (x & 63));
        }
        gone[x] = 1;
    }
    return width;
}

// LateParOptimizer (qtensor/optimisation/late_parallelisation.py:30-202)
// with one variable per bunch, until the width is at most `target`: from
// the reference's greedy order, for every step s of the order the graph is
// contracted up to s, its node of largest multigraph degree sliced
// (slice_greedy, GreedyParvars) and the rest ordered greedily; the step of
// least width max(widths of the contracted prefix, widths of the new order)
// wins (the first one on ties, numpy argmin), its prefix is kept and the
// search repeats on the sliced graph.  The neighbour count of a prefix step
// is taken with the +1 of find_slice_at_step (:101).  Steps whose prefix
// width alone already reaches the best width found are not evaluated (they
// cannot be chosen).  Returns false when the order runs out first.
static bool late_slicing(const MultiGraph& g0, int target, int max_vars, std::vector<int32_t>* peo,
                         std::vector<int32_t>* par, int* final_width) {
    MultiGraph g = g0;
    LineGraph lg;
    std::vector<char> removed;
    std::vector<int32_t> ordering, path, cand_order, cand_path;
    g.simple(&lg, &removed);
    greedy_order(lg, removed, 0, &ordering, &path);
    peo->clear();
    par->clear();
    *final_width = path.empty() ? 0 : *std::max_element(path.begin(), path.end());
    if (*final_width <= target) {
        *peo = ordering;
        return true;
    }
    while ((int)par->size() < max_vars) {
        // find_slice_at_step(ordering, g, 1)
        MultiGraph work = g;
        int best_tw = INT_MAX, best_step = -1, best_var = -1, largest = 0;
        std::vector<int32_t> best_order;
        for (size_t s = 0; s + 1 < ordering.size(); ++s) {
            const int node = ordering[s];
            const int step_tw = work.n_neighbors(node) + 1;
            if (std::max(largest, step_tw) >= best_tw) break;   // no later step can win
            const int x = work.max_degree_node();
            work.simple(&lg, &removed, x);
            greedy_order(lg, removed, 0, &cand_order, &cand_path);
            largest = std::max(largest, step_tw);
            const int tw = std::max(largest, cand_path.empty() ? 0 : *std::max_element(cand_path.begin(), cand_path.end()));
            if (tw < best_tw) {
                best_tw = tw;
                best_step = (int)s;
                best_var = x;
                best_order = cand_order;
            }
            work.eliminate(node);
        }
        if (best_step < 0) return false;
        for (int s = 0; s < best_step; ++s) {
            peo->push_back(ordering[s]);
            g.eliminate(ordering[s]);
        }
        g.remove(best_var);
        par->push_back(best_var);
        ordering = best_order;
        *final_width = best_tw;
        if (best_tw <= target) {
            peo->insert(peo->end(), ordering.begin(), ordering.end());
            return true;
        }
    }
    return false;
}

// Tree trimming (TreeTrimSplitter, qtensor/optimisation/Optimizer.py:178-224):
// while the greedy width exceeds `target`, remove int(0.2 * excess) + 1
// variables at once, then reorder.  The variables come from
// split_graph_by_tree_trimming of the qtree package (github.com/DaniloZZZ/
// qtree, PyPI qtensor-qtree, version unpinned), which is absent from the
// reference; this restates the published heuristic (Schutski, Khakhulin,
// Oseledets, Kolmakov, "Simple heuristics for efficient parallel tensor
// contraction and quantum circuit simulation", Phys. Rev. A 102, 062614,
// 2020): one variable at a time, the one lying in the most cliques of the
// largest size among the elimination cliques (a node with its neighbours
// when it is eliminated) of the current greedy order, ties to the earliest
// in that order (the reference relabels nodes by order position first),
// reordering after each removal.
static bool tree_trim_slicing(const LineGraph& g0, std::vector<char> removed, int target, int max_vars,
                              std::vector<int32_t>* order, std::vector<int32_t>* degrees,
                              std::vector<int32_t>* par) {
    const int V = g0.V, W = g0.W;
    LineGraph g = g0;
    par->clear();
    greedy_order(g, removed, 0, order, degrees);
    auto width = [&]() { return degrees->empty() ? 0 : *std::max_element(degrees->begin(), degrees->end()); };
    std::vector<int64_t> hits(V);
    std::vector<int32_t> nb;
    while (width() > target) {
        const int n_target = (int)((width() - target) * 0.2) + 1;
        for (int k = 0; k < n_target; ++k) {
            if ((int)par->size() >= max_vars) return false;
            // elimination cliques of the current order
            std::vector<uint64_t> adj(g.adj);
            std::fill(hits.begin(), hits.end(), 0);
            std::vector<int32_t> pos(V, INT_MAX);
            for (size_t i = 0; i < order->size(); ++i) pos[(*order)[i]] = (int32_t)i;
            const int w = width();
            std::vector<char> gone(removed);
            for (int x : *order) {
                uint64_t* rx = &adj[(size_t)x * W];
                nb.clear();
                for (int q = 0; q < W; ++q)
                    for (uint64_t m = rx[q]; m; m &= m - 1) nb.push_back(q * 64 + __builtin_ctzll(m));
                if ((int)nb.size() == w) {
                    ++hits[x];
                    for (int a : nb) ++hits[a];
                }
                for (int a : nb) {
                    uint64_t* ra = &adj[(size_t)a * W];
                    for (int q = 0; q < W; ++q) ra[q] |= rx[q];
                    ra[a >> 6] &= ~(1ull << (a & 63));
                    ra[x >> 6] &= ~(1ull << (x & 63));
                }
                gone[x] = 1;
            }
            int best = -1;
            for (int x = 0; x < V; ++x)
                if (!removed[x] && hits[x] > 0 &&
                    (best < 0 || hits[x] > hits[best] || (hits[x] == hits[best] && pos[x] < pos[best])))
                    best = x;
            if (best < 0) return false;
            // remove it from the graph (no fill-in)
            for (int q = 0; q < W; ++q)
                for (uint64_t m = g.adj[(size_t)best * W + q]; m; m &= m - 1) {
                    const int a = q * 64 + __builtin_ctzll(m);
                    g.adj[(size_t)a * W + (best >> 6)] &= ~(1ull << (best & 63));
                    --g.deg[a];
                }
            for (int q = 0; q < W; ++q) g.adj[(size_t)best * W + q] = 0;
            g.deg[best] = 0;
            removed[best] = 1;
            par->push_back(best);
            greedy_order(g, removed, 0, order, degrees);
        }
    }
    return true;
}

int compile_circuit(int32_t n_qubits, const qtb_gate* in_gates, int32_t n_gates,
                    int32_t simplify_passes, const double* params, int32_t n_params,
                    int32_t order_trials, int32_t max_width, int32_t max_slices, int32_t slicing,
                    int32_t batch_vars, std::vector<Network>* outs, std::string* err,
                    const std::atomic<bool>* abort) {
    outs->clear();
    if (batch_vars < 0 || batch_vars > n_qubits || batch_vars > kMaxBatchVars) {
        *err = "compile: batch_vars must be in 0.." + std::to_string(std::min(n_qubits, kMaxBatchVars));
        return QTB_ERR_ARG;
    }
    std::vector<AngleCheck> checks;
    if (n_qubits <= 0 || n_gates < 0 || (n_gates > 0 && in_gates == nullptr)) {
        *err = "compile: invalid circuit arguments";
        return QTB_ERR_ARG;
    }
    // ---- gates with numeric and symbolic angles
    std::vector<Gate> gates(n_gates);
    for (int i = 0; i < n_gates; ++i) {
        const qtb_gate& g = in_gates[i];
        if (g.kind < QTB_GATE_M || g.kind > QTB_GATE_T) {
            *err = "compile: unknown gate kind " + std::to_string(g.kind);
            return QTB_ERR_ARG;
        }
        const int nq = qubits_of_kind(g.kind);
        if (g.q0 < 0 || g.q0 >= n_qubits || (nq == 2 && (g.q1 < 0 || g.q1 >= n_qubits || g.q1 == g.q0))) {
            *err = "compile: gate " + std::to_string(i) + " has qubits out of range";
            return QTB_ERR_ARG;
        }
        Gate& o = gates[i];
        o.kind = g.kind;
        o.q[0] = g.q0;
        o.q[1] = nq == 2 ? g.q1 : -1;
        o.angle = 0.0;
        if (is_parametric(g.kind)) {
            if (g.param < 0 || g.param >= n_params || params == nullptr) {
                *err = "compile: parametric gate " + std::to_string(i) + " has no parameter";
                return QTB_ERR_ARG;
            }
            o.angle = g.coef * params[g.param];
            if (g.coef != 0.0) o.expr.emplace_back(g.param, g.coef);
        }
    }
    bool angle_specific = false;
    for (int pass = 0; pass < simplify_passes; ++pass) {
        int rc = simplify(&gates, &checks, &angle_specific, err);
        if (rc) return rc;
    }

    // ---- qtree layout: bra vars 0..nq-1, gates from the bra side
    const int nq = n_qubits;
    std::vector<TRec> tensors;
    std::vector<std::vector<int32_t>> buckets(nq);
    std::vector<int32_t> frame(nq);
    std::iota(frame.begin(), frame.end(), 0);
    int32_t next_id = nq;
    auto place = [&](int32_t kind, const Expr& expr, const int* qs, int nqub) {
        TRec t;
        t.kind = kind;
        t.expr = expr;
        const int cp = changed_position(kind);
        int32_t new_id = next_id;
        for (int i = 0; i < nqub; ++i) {
            t.vars.push_back(frame[qs[i]]);
            if (i == cp) t.vars.push_back(new_id++);
        }
        const int32_t smallest = *std::min_element(t.vars.begin(), t.vars.end());
        buckets[smallest].push_back((int32_t)tensors.size());
        tensors.push_back(std::move(t));
        if (cp >= 0) {
            frame[qs[cp]] = next_id++;
            buckets.emplace_back();
        }
    };
    const Expr none;
    for (int q = 0; q < nq; ++q) place(QTB_GATE_M, none, &q, 1);
    for (int i = (int)gates.size() - 1; i >= 0; --i)
        place(gates[i].kind, gates[i].expr, gates[i].q, qubits_of_kind(gates[i].kind));
    const int32_t ket_start = next_id;
    for (int q = 0; q < nq; ++q) {
        TRec t;
        t.kind = QTB_GATE_M;
        t.vars = {frame[q], next_id};
        buckets[frame[q]].push_back((int32_t)tensors.size());
        tensors.push_back(std::move(t));
        buckets.emplace_back();
        frame[q] = next_id++;
    }
    const int32_t n_vars = next_id;
    auto ignored = [&](int32_t v) { return v < nq || v >= ket_start; };

    // ---- line graph (first-appearance node order) and greedy order
    std::vector<int32_t> node_of(n_vars, -1), var_of;
    std::vector<std::vector<int32_t>> cliques, tnodes;   // tnodes: every tensor's nodes (late slicing)
    for (const auto& b : buckets)
        for (int32_t ti : b) {
            std::vector<int32_t> c;
            for (int32_t v : tensors[ti].vars) {
                if (ignored(v)) continue;
                if (node_of[v] < 0) {
                    node_of[v] = (int32_t)var_of.size();
                    var_of.push_back(v);
                }
                c.push_back(node_of[v]);
            }
            if (slicing == QTB_SLICE_LATE && !c.empty()) tnodes.push_back(c);
            if (c.size() > 1) cliques.push_back(std::move(c));
        }
    // trial 0: the reference's greedy rule; trials 1..order_trials: seeded
    // random tie-breaking; the cheapest order (sum of 2^degree) wins.  With
    // max_width > 0, variables of highest degree are sliced (removed from
    // the line graph, reference GreedyParvars, qtensor/optimisation/
    // Greedy.py:78-91 driven by Optimizer.py:109-129) until the order's
    // width drops below max_width.
    const int V = (int)var_of.size();
    std::vector<char> removed(V, 0);
    std::vector<int32_t> par;   // sliced line-graph nodes, in slicing order
    std::vector<int32_t> gorder, gdeg, torder, tdeg;
    LineGraph lg;
    // variables that may be sliced within max_slices
    int slice_budget = 0;
    while (slice_budget < kMaxSlicedVars && (2ll << slice_budget) <= (long long)max_slices) ++slice_budget;
    // With trials, the minimum-fill heuristic competes too: its
    // deterministic order plus one randomized order per four greedy trials.
    // It runs only while the greedy width is below max_width + 3, where it
    // can decide whether (and how much) the circuit is sliced; further
    // above, min-fill (which lowers widths by a few units) cannot change
    // the outcome of the slicing step at hand.
    auto best_order = [&]() {
        line_graph(V, cliques, removed, &lg);
        double best_cost = greedy_order(lg, removed, 0, &gorder, &gdeg);
        auto keep = [&](double c) {
            if (c < best_cost) {
                best_cost = c;
                gorder.swap(torder);
                gdeg.swap(tdeg);
            }
        };
        for (int32_t t = 1; t <= order_trials; ++t) {
            const uint64_t seed = 0x9E3779B97F4A7C15ull * (uint64_t)t + (uint64_t)V;
            keep(greedy_order(lg, removed, seed, &torder, &tdeg));
        }
        const int greedy_width = gdeg.empty() ? 0 : *std::max_element(gdeg.begin(), gdeg.end());
        const bool far_above = max_width > 0 && greedy_width >= max_width + 3;
        if (order_trials > 0 && !far_above)
            for (int32_t t = 0; t <= order_trials / 4; ++t) {
                const uint64_t seed = t == 0 ? 0 : 0xD1B54A32D192ED03ull * (uint64_t)t + (uint64_t)V;
                keep(minfill_order(lg, removed, seed, &torder, &tdeg));
            }
    };
    best_order();
    auto width = [&]() { return gdeg.empty() ? 0 : *std::max_element(gdeg.begin(), gdeg.end()); };
    auto out_of_budget = [&](const char* how) {
        *err = "compile: width " + std::to_string(width()) + " still >= " + std::to_string(max_width) +
               " after " + how + " slicing of at most " + std::to_string(slice_budget) + " variables (" +
               std::to_string(1ll << slice_budget) + " slices per circuit)";
        return QTB_ERR_UNSUPPORTED;
    };
    // a width far above the target is out of reach of any slicing within
    // the budget (the greedy loop below applies the same bound per step)
    if (max_width > 0 && slicing != QTB_SLICE_GREEDY && width() - max_width + 1 > 2 * slice_budget)
        return out_of_budget(slicing == QTB_SLICE_LATE ? "late" : "tree-trimming");
    if (max_width > 0 && width() >= max_width && slicing == QTB_SLICE_TREE_TRIM) {
        // TreeTrimSplitter's choice of variables, then the order search on
        // the sliced graph (the reference reorders greedily; with trials the
        // cheaper candidates compete as for an unsliced circuit)
        std::vector<char> none(V, 0);
        line_graph(V, cliques, none, &lg);
        const bool ok = tree_trim_slicing(lg, none, max_width - 1, slice_budget, &gorder, &gdeg, &par);
        for (int32_t x : par) removed[x] = 1;
        if (!ok) return out_of_budget("tree-trimming");
        if (order_trials > 0) best_order();
    } else if (max_width > 0 && width() >= max_width && slicing == QTB_SLICE_LATE) {
        // LateParOptimizer's sliced variables and order (prefix contracted
        // before each slice, then the greedy order of the sliced rest)
        MultiGraph mg;
        mg.init(V, tnodes);
        int late_width = 0;
        const bool ok = late_slicing(mg, max_width - 1, slice_budget, &gorder, &par, &late_width);
        for (int32_t x : par) removed[x] = 1;
        line_graph(V, cliques, removed, &lg);
        if (!ok) {
            greedy_order(lg, removed, 0, &gorder, &gdeg);
            return out_of_budget("late");
        }
        order_width(lg, removed, gorder, &gdeg);
    }
    while (max_width > 0 && width() >= max_width && slicing == QTB_SLICE_GREEDY) {
        if (abort && abort->load(std::memory_order_relaxed)) return kCompileAborted;
        // removing one variable lowers the treewidth by at most one, so a
        // width more than twice the remaining budget above the target is
        // out of reach: fail now instead of after the whole budget
        const int remaining = slice_budget - (int)par.size();
        if (remaining <= 0 || width() - max_width + 1 > 2 * remaining) {
            *err = "compile: width " + std::to_string(width()) + " still >= " + std::to_string(max_width) +
                   " after slicing " + std::to_string(par.size()) + " variables (at most " +
                   std::to_string(1ll << slice_budget) + " slices per circuit)";
            return QTB_ERR_UNSUPPORTED;
        }
        // distinct-neighbour degree in the graph with the sliced nodes
        // removed: the line graph of the last order search
        int best = -1, best_deg = -1;
        for (int x = 0; x < V; ++x) {
            if (removed[x]) continue;
            const int d = lg.deg[x];
            if (d > best_deg) {
                best_deg = d;
                best = x;
            }
        }
        if (best < 0) break;
        removed[best] = 1;
        par.push_back(best);
        best_order();
    }
    std::vector<int32_t> peo;
    for (int q = 0; q < nq; ++q) peo.push_back(ket_start + q);
    for (int q = 0; q < nq; ++q) peo.push_back(q);
    for (int32_t x : gorder) peo.push_back(var_of[x]);
    for (int32_t x : par) peo.push_back(var_of[x]);
    if ((int32_t)peo.size() != n_vars) {
        *err = "compile: elimination order does not cover every variable";
        return QTB_ERR_ARG;
    }
    std::vector<int32_t> perm(n_vars);
    for (int32_t i = 0; i < n_vars; ++i) perm[peo[i]] = i;
    // sliced variables (new ids): ket and bra fixed to 0, sliced ones per slice
    std::vector<char> sliced(n_vars, 0);
    for (int32_t i = 0; i < 2 * nq; ++i) sliced[i] = 1;
    for (size_t i = 0; i < par.size(); ++i) sliced[perm[var_of[par[i]]]] = 1;

    // Per circuit, in bucket order: each tensor's variables in elimination
    // order (new ids, ascending), the native axis each came from, and the
    // slice-independent part of its gate-table key (kind, expression, rank,
    // sliced axes, kept-axis permutation), interned as a base id.  Only the
    // values of the sliced axes differ between the networks of the circuit.
    struct TView {
        int32_t off, rank, base;
        uint8_t sliced_mask;
    };
    std::vector<TView> tview;
    std::vector<int32_t> tvars;     // pool: tensor variables, then op results
    std::vector<int8_t> taxes;
    std::vector<EntryKey> bases;    // sliced_value 0
    {
        std::map<EntryKey, int32_t> base_index;
        EntryKey key;
        std::vector<int> axes;
        for (const auto& b : buckets)
            for (int32_t ti : b) {
                const TRec& t = tensors[ti];
                const int r = (int)t.vars.size();
                axes.resize(r);
                std::iota(axes.begin(), axes.end(), 0);
                std::sort(axes.begin(), axes.end(),
                          [&](int x, int y) { return perm[t.vars[x]] < perm[t.vars[y]]; });
                TView v{(int32_t)tvars.size(), r, -1, 0};
                key.kind = t.kind;
                key.expr = t.expr;
                key.rank_in = (int8_t)r;
                key.sliced_mask = 0;
                key.sliced_value = 0;
                key.perm.clear();
                for (int a : axes) {
                    const int32_t nv = perm[t.vars[a]];
                    tvars.push_back(nv);
                    taxes.push_back((int8_t)a);
                    if (sliced[nv]) key.sliced_mask |= (uint8_t)(1u << a);
                    else key.perm.push_back((int8_t)a);
                }
                v.sliced_mask = key.sliced_mask;
                auto it = base_index.find(key);
                if (it == base_index.end()) {
                    it = base_index.emplace(key, (int32_t)bases.size()).first;
                    bases.push_back(key);
                }
                v.base = it->second;
                tview.push_back(v);
            }
    }
    const size_t tensor_pool = tvars.size();

    // one network per assignment of the sliced (parallel) variables, per
    // output bitstring of the first batch_vars qubits (their bra variables,
    // new ids nq + q, take the bits of `amp`, qubit 0 most significant)
    uint64_t amp = 0;
    // per-build working arrays, kept across the networks of the circuit
    std::vector<char> value(n_vars);
    std::vector<int32_t> head(n_vars), tail(n_vars), live_pos(n_vars, -1);
    std::vector<std::vector<std::pair<uint8_t, int32_t>>> local_of(bases.size());
    std::vector<Ref> refs;
    std::vector<OpRec> ops;
    std::vector<uint8_t> in_table;
    std::vector<int32_t> in_id;
    std::vector<uint32_t> in_mask;
    std::vector<int32_t> U, liveU, scalars, by_level;
    auto build = [&](uint64_t slice_bits, Network* out) -> int {
        std::fill(value.begin(), value.end(), 0);
        for (int32_t q = 0; q < batch_vars; ++q) value[nq + q] = (char)((amp >> (batch_vars - 1 - q)) & 1u);
        for (size_t i = 0; i < par.size(); ++i)
            value[perm[var_of[par[i]]]] = (char)((slice_bits >> (par.size() - 1 - i)) & 1u);
        // ---- reorder + slice: tensors become references to gate-table
        // entries, listed per bucket (head/tail/next) in arrival order
        tvars.resize(tensor_pool);
        std::fill(head.begin(), head.end(), -1);
        std::fill(tail.begin(), tail.end(), -1);
        for (auto& l : local_of) l.clear();
        refs.clear();
        auto append = [&](int32_t bucket, const Ref& r) {
            const int32_t idx = (int32_t)refs.size();
            refs.push_back(r);
            refs.back().next = -1;
            if (tail[bucket] < 0) head[bucket] = idx;
            else refs[tail[bucket]].next = idx;
            tail[bucket] = idx;
        };
        out->checks = checks;
        out->peo = peo;
        out->entries.clear();
        for (const TView& v : tview) {
            uint8_t sv = 0;
            for (int32_t i = 0; i < v.rank; ++i) {
                const int32_t nv = tvars[v.off + i];
                if (sliced[nv] && value[nv]) sv |= (uint8_t)(1u << taxes[v.off + i]);
            }
            int32_t id = -1;
            for (const auto& e : local_of[v.base])
                if (e.first == sv) id = e.second;
            if (id < 0) {
                id = (int32_t)out->entries.size();
                local_of[v.base].emplace_back(sv, id);
                out->entries.push_back(bases[v.base]);
                out->entries.back().sliced_value = sv;
            }
            append(tvars[v.off], Ref{true, id, v.off, v.rank, -1});
        }

        // ---- symbolic bucket elimination
        ops.clear();
        in_table.clear();
        in_id.clear();
        in_mask.clear();
        scalars.clear();
        double ref_flops = 0.0;
        int32_t max_rank = 0;
        for (int32_t n = 0; n < n_vars; ++n) {
            if (head[n] < 0) continue;
            U.clear();
            int32_t count = 0;
            for (int32_t r = head[n]; r >= 0; r = refs[r].next, ++count)
                U.insert(U.end(), tvars.begin() + refs[r].off, tvars.begin() + refs[r].off + refs[r].len);
            std::sort(U.begin(), U.end());
            U.erase(std::unique(U.begin(), U.end()), U.end());
            if (U.empty() || U[0] != n) {
                *err = "compile: bucket " + std::to_string(n) + " holds a tensor without its variable";
                return QTB_ERR_ARG;
            }
            ref_flops += std::ldexp(1.0, (int)U.size() - 1) * (double)(1 + count);
            const int32_t out_off = (int32_t)tvars.size(), out_len = (int32_t)U.size() - 1;
            tvars.insert(tvars.end(), U.begin() + 1, U.end());
            Ref res;
            const bool live = !sliced[n];
            if (count == 1 && !live) {
                res = refs[head[n]];   // product of one tensor over a size-1 variable: a copy
            } else {
                OpRec op;
                liveU.clear();
                for (int32_t v : U)
                    if (!sliced[v]) {
                        live_pos[v] = (int32_t)liveU.size();
                        liveU.push_back(v);
                    }
                op.u = (int32_t)liveU.size();
                op.sum = live ? 1 : 0;
                op.w = op.u - op.sum;
                if (op.u > QTB_MAX_BUCKET_VARS) {
                    *err = "compile: bucket of " + std::to_string(op.u) + " variables exceeds the limit";
                    return QTB_ERR_UNSUPPORTED;
                }
                max_rank = std::max(max_rank, op.u);
                if (ops.size() >= 65535) {
                    *err = "compile: network has more than 65535 bucket operations";
                    return QTB_ERR_UNSUPPORTED;
                }
                op.in_begin = (int32_t)in_id.size();
                op.k = count;
                for (int32_t r = head[n]; r >= 0; r = refs[r].next) {
                    uint32_t m = 0;
                    for (int32_t i = 0; i < refs[r].len; ++i) {
                        const int32_t v = tvars[refs[r].off + i];
                        if (!sliced[v]) m |= 1u << (op.u - 1 - live_pos[v]);
                    }
                    in_mask.push_back(m);
                    in_table.push_back(refs[r].table ? 1 : 0);
                    in_id.push_back(refs[r].id);
                }
                res.table = false;
                res.id = (int32_t)ops.size();
                ops.push_back(op);
            }
            res.off = out_off;
            res.len = out_len;
            if (out_len == 0) scalars.push_back((int32_t)refs.size());
            if (out_len == 0) refs.push_back(res);
            else append(tvars[out_off], res);
        }
        if (scalars.empty()) {
            *err = "compile: network has no scalar result";
            return QTB_ERR_ARG;
        }
        Ref result;
        if (scalars.size() == 1) {
            result = refs[scalars[0]];
        } else {
            OpRec op;
            op.u = op.sum = op.w = 0;
            op.in_begin = (int32_t)in_id.size();
            op.k = (int32_t)scalars.size();
            for (int32_t s : scalars) {
                in_table.push_back(refs[s].table ? 1 : 0);
                in_id.push_back(refs[s].id);
                in_mask.push_back(0);
            }
            result.table = false;
            result.id = (int32_t)ops.size();
            ops.push_back(op);
        }

        // ---- dependency levels, arena intervals
        int32_t max_level = 0;
        for (OpRec& op : ops) {
            int32_t lv = 0;
            for (int32_t t = op.in_begin; t < op.in_begin + op.k; ++t)
                if (!in_table[t]) lv = std::max(lv, ops[in_id[t]].level);
            op.level = lv + 1;
            max_level = std::max(max_level, op.level);
        }
        for (OpRec& op : ops)
            for (int32_t t = op.in_begin; t < op.in_begin + op.k; ++t)
                if (!in_table[t]) ops[in_id[t]].consumer_level = op.level;
        if (!result.table) ops[result.id].consumer_level = max_level + 1;
        by_level.resize(ops.size());
        std::iota(by_level.begin(), by_level.end(), 0);
        // within a level the widest op first: every op of a phase then starts
        // at a multiple of its own (power-of-two) size
        std::stable_sort(by_level.begin(), by_level.end(), [&](int32_t x, int32_t y) {
            return ops[x].level != ops[y].level ? ops[x].level < ops[y].level : ops[x].w > ops[y].w;
        });
        // Offsets are computed in 64 bits: an arena (and a phase) must stay
        // below kMaxArenaElems, since arena offsets share their word with
        // the kSrcTable flag and the executors index elements in 32 bits.
        struct Live { uint64_t off, size; int32_t end; };
        std::vector<Live> active;
        uint64_t arena = 0;
        uint32_t max_elems = 1;
        // `active` stays sorted by offset: first fit over the live intervals.
        // Ops come in level order and an interval placed at a level ends
        // after it, so expired intervals are swept once per level.
        int32_t swept = -1;
        for (int32_t oi : by_level) {
            OpRec& op = ops[oi];
            if (op.level != swept) {
                active.erase(std::remove_if(active.begin(), active.end(),
                                            [&](const Live& l) { return l.end < op.level; }),
                             active.end());
                swept = op.level;
            }
            const uint64_t size = uint64_t(1) << op.w;
            max_elems = (uint32_t)std::max<uint64_t>(max_elems, size);
            const uint64_t need = (size + 3u) & ~uint64_t(3);
            uint64_t off = 0;
            for (const Live& l : active) {
                if (off + need <= l.off) break;
                off = std::max(off, l.off + l.size);
            }
            op.dst = (uint32_t)off;
            const Live item{off, need, op.consumer_level};
            active.insert(std::upper_bound(active.begin(), active.end(), item,
                                           [](const Live& a, const Live& b) { return a.off < b.off; }),
                          item);
            arena = std::max(arena, off + need);
            if (arena > kMaxArenaElems) {
                *err = "compile: network needs an arena of more than " + std::to_string(kMaxArenaElems) +
                       " complex64 elements (width " + std::to_string(op.w) +
                       "); slice it (qtb_plan_set_max_width)";
                return QTB_ERR_UNSUPPORTED;
            }
        }

        // ---- device images: ops in phase order
        out->ops.clear();
        out->ins.clear();
        out->phases.clear();
        double alg_bytes = 0.0, alg_flops = 0.0;
        size_t cursor = 0;
        for (int32_t lv = 1; lv <= max_level; ++lv) {
            DevPhase ph{};
            ph.op_first = (uint32_t)out->ops.size();
            uint32_t elems = 0;
            while (cursor < by_level.size() && ops[by_level[cursor]].level == lv) {
                const OpRec& op = ops[by_level[cursor++]];
                DevOp d{};
                d.u = (uint8_t)op.u;
                d.sum = (uint8_t)op.sum;
                d.k = (uint8_t)op.k;
                d.dst = op.dst;
                d.elem_begin = elems;
                d.in_begin = (uint32_t)out->ins.size();
                for (int32_t t = op.in_begin; t < op.in_begin + op.k; ++t) {
                    DevIn in{};
                    in.mask = in_mask[t];
                    in.src = in_table[t] ? (kSrcTable | (uint32_t)in_id[t]) : ops[in_id[t]].dst;
                    in.runs = encode_runs(in.mask, (uint32_t)op.w);
                    out->ins.push_back(in);
                    alg_bytes += 8.0 * std::ldexp(1.0, __builtin_popcount(in.mask));
                }
                alg_bytes += 8.0 * std::ldexp(1.0, op.w);
                alg_flops += 6.0 * (double)(op.k - 1) * std::ldexp(1.0, op.u) +
                             (op.sum ? 2.0 * std::ldexp(1.0, op.w) : 0.0);
                elems += 1u << op.w;
                out->ops.push_back(d);
            }
            ph.op_count = (uint32_t)out->ops.size() - ph.op_first;
            ph.total_elems = elems;
            out->phases.push_back(ph);
        }
        out->result_src = result.table ? (kSrcTable | (uint32_t)result.id) : ops[result.id].dst;
        out->max_elems = max_elems;
        qtb_network_info& info = out->info;
        info.n_qubits = nq;
        info.n_vars = n_vars;
        info.treewidth = gdeg.empty() ? 0 : *std::max_element(gdeg.begin(), gdeg.end());
        info.n_slices = 1 << (int)par.size();
        info.max_rank = max_rank;
        info.n_ops = (int32_t)out->ops.size();
        info.n_phases = (int32_t)out->phases.size();
        info.arena_elems = (int32_t)arena;
        info.angle_specific = angle_specific ? 1 : 0;
        info.alg_bytes = alg_bytes;
        info.alg_flops = alg_flops;
        info.ref_flops = ref_flops;
        return QTB_OK;
    };
    const uint64_t n_slices = 1ull << par.size();
    const uint64_t n_amps = 1ull << batch_vars;
    outs->resize(n_amps * n_slices);
    for (amp = 0; amp < n_amps; ++amp)
        for (uint64_t sl = 0; sl < n_slices; ++sl) {
            int rc = build(sl, &(*outs)[amp * n_slices + sl]);
            if (rc) return rc;
        }
    return QTB_OK;
}
// ------------------------------------------------------ native lightcone
int build_lightcone(int32_t n_nodes, const int64_t* indptr, const int32_t* indices, int32_t u,
                    int32_t v, int32_t p, int32_t composer, std::vector<qtb_gate>* gates,
                    int32_t* n_qubits, std::string* err) {
    if (n_nodes <= 0 || !indptr || !indices || u < 0 || v < 0 || u >= n_nodes || v >= n_nodes ||
        u == v || p < 0 || composer < 0 || composer > 2) {
        *err = "lightcone: invalid arguments";
        return QTB_ERR_ARG;
    }
    // BFS from the edge, radius p.  Distances and qubit numbers live in
    // per-thread node arrays (-1 = outside the cone), reset after each edge,
    // so an edge costs its cone's size, not the graph's.
    static thread_local std::vector<int32_t> dist, qubit;
    if ((int32_t)dist.size() < n_nodes) {
        dist.resize(n_nodes, -1);
        qubit.resize(n_nodes, -1);
    }
    std::vector<int32_t> frontier = {u, v}, cone = {u, v};
    struct Reset {
        std::vector<int32_t>& cone;
        ~Reset() {
            for (int32_t x : cone) dist[x] = qubit[x] = -1;
        }
    } reset{cone};
    dist[u] = dist[v] = 0;
    for (int d = 1; d <= p; ++d) {
        std::vector<int32_t> next;
        for (int32_t x : frontier)
            for (int64_t e = indptr[x]; e < indptr[x + 1]; ++e) {
                const int32_t y = indices[e];
                if (y < 0 || y >= n_nodes) {
                    *err = "lightcone: neighbour id out of range";
                    return QTB_ERR_ARG;
                }
                if (dist[y] < 0) {
                    dist[y] = d;
                    next.push_back(y);
                    cone.push_back(y);
                }
            }
        frontier.swap(next);
    }
    std::sort(cone.begin(), cone.end());
    for (size_t i = 0; i < cone.size(); ++i) qubit[cone[i]] = (int32_t)i;
    const int32_t nq = (int32_t)cone.size();
    std::vector<qtb_gate> ansatz;
    auto add = [&](int32_t kind, int32_t a, int32_t b, int32_t param, double coef) {
        ansatz.push_back(qtb_gate{kind, a, b, param, coef});
    };
    for (int32_t q = 0; q < nq; ++q) add(QTB_GATE_H, q, -1, -1, 0.0);
    for (int32_t l = 0; l < p; ++l) {
        const int32_t radius = p - l;
        for (int32_t x : cone) {
            if (dist[x] > radius) continue;
            std::vector<int32_t> nb;
            for (int64_t e = indptr[x]; e < indptr[x + 1]; ++e) {
                const int32_t y = indices[e];
                if (y > x && y < n_nodes && dist[y] >= 0 && dist[y] <= radius) nb.push_back(y);
            }
            std::sort(nb.begin(), nb.end());
            nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
            for (int32_t y : nb) {
                const int32_t a = qubit[x], b = qubit[y];
                if (composer == 2) {
                    add(QTB_GATE_CX, a, b, -1, 0.0);
                    add(QTB_GATE_ZPHASE, b, -1, l, 2.0);
                    add(QTB_GATE_CX, a, b, -1, 0.0);
                } else {
                    add(QTB_GATE_ZZ, a, b, l, 2.0);
                }
            }
        }
        for (int32_t x : cone)
            if (dist[x] <= radius) add(QTB_GATE_XPHASE, qubit[x], -1, p + l, 2.0);
    }
    gates->clear();
    gates->insert(gates->end(), ansatz.begin(), ansatz.end());
    gates->push_back(qtb_gate{QTB_GATE_Z, qubit[u], -1, -1, 0.0});
    gates->push_back(qtb_gate{QTB_GATE_Z, qubit[v], -1, -1, 0.0});
    for (auto it = ansatz.rbegin(); it != ansatz.rend(); ++it) {
        qtb_gate g = *it;
        g.coef = -g.coef;   // G(alpha)^+ = G(-alpha) for ZZ / XPhase / ZPhase
        gates->push_back(g);
    }
    *n_qubits = nq;
    return QTB_OK;
}

// ------------------------------------------------------ lightcone classes
// Structural key of an edge's lightcone: the cone (nodes within distance p
// of u or v) with every node's distance, every edge among cone nodes, and
// u and v in their roles, written in a canonical numbering.  Two edges with
// equal keys have isomorphic lightcones through a map that keeps distances
// and sends u to u and v to v, so their circuits are relabelings of each
// other and contract to the same <Z_u Z_v>: one compiled network serves
// both.  Equality of the full keys is what proves it; the numbering only
// decides how often isomorphic cones get equal keys.  It comes from colour
// refinement (distance, role, then the multiset of neighbour colours until
// the classes stop splitting) and a level-by-level order: distance, colour,
// the sorted ranks of the node's neighbours one level closer, then the
// node id.  On trees this numbers isomorphic cones alike; on cones with
// cycles, ties broken by node id may give distinct keys (a missed share,
// never a wrong one).
// Coarse invariant of an edge's lightcone, cheap to compute: cone size,
// number of edges among cone nodes, and the (distance, degree in the cone)
// histogram.  Isomorphic cones (as cone_key defines them) have equal
// invariants, so an edge whose invariant no other edge has cannot share and
// skips cone_key.
void cone_invariant(int32_t n_nodes, const int64_t* indptr, const int32_t* indices, int32_t u, int32_t v,
                    int32_t p, std::vector<int32_t>* inv) {
    static thread_local std::vector<int32_t> dist;
    if ((int32_t)dist.size() < n_nodes) dist.resize(n_nodes, -1);
    std::vector<int32_t> cone = {u, v};
    struct Reset {
        std::vector<int32_t>& cone;
        ~Reset() {
            for (int32_t x : cone) dist[x] = -1;
        }
    } reset{cone};
    dist[u] = dist[v] = 0;
    for (size_t head = 0; head < cone.size(); ++head) {
        const int32_t x = cone[head];
        if (dist[x] == p) continue;
        for (int64_t e = indptr[x]; e < indptr[x + 1]; ++e) {
            const int32_t y = indices[e];
            if (y >= 0 && y < n_nodes && dist[y] < 0) {
                dist[y] = dist[x] + 1;
                cone.push_back(y);
            }
        }
    }
    std::vector<int64_t> cells;   // distance * 2^32 + degree, one per node
    int64_t twice_edges = 0;
    for (int32_t x : cone) {
        int32_t deg = 0;
        int32_t prev = -1;
        std::vector<int32_t> nb;
        for (int64_t e = indptr[x]; e < indptr[x + 1]; ++e) {
            const int32_t y = indices[e];
            if (y >= 0 && y < n_nodes && y != x && dist[y] >= 0) nb.push_back(y);
        }
        std::sort(nb.begin(), nb.end());
        for (int32_t y : nb)
            if (y != prev) {
                ++deg;
                prev = y;
            }
        twice_edges += deg;
        cells.push_back(((int64_t)dist[x] << 32) | (int64_t)deg);
    }
    std::sort(cells.begin(), cells.end());
    inv->clear();
    inv->push_back((int32_t)cone.size());
    inv->push_back((int32_t)(twice_edges / 2));
    for (int64_t c : cells) {
        inv->push_back((int32_t)(c >> 32));
        inv->push_back((int32_t)(c & 0xffffffff));
    }
}

void cone_key(int32_t n_nodes, const int64_t* indptr, const int32_t* indices, int32_t u, int32_t v,
              int32_t p, std::vector<int32_t>* key) {
    static thread_local std::vector<int32_t> dist, loc;
    if ((int32_t)dist.size() < n_nodes) {
        dist.resize(n_nodes, -1);
        loc.resize(n_nodes, -1);
    }
    std::vector<int32_t> cone = {u, v};
    struct Reset {
        std::vector<int32_t>& cone;
        ~Reset() {
            for (int32_t x : cone) dist[x] = loc[x] = -1;
        }
    } reset{cone};
    dist[u] = dist[v] = 0;
    for (size_t head = 0; head < cone.size(); ++head) {
        const int32_t x = cone[head];
        if (dist[x] == p) continue;
        for (int64_t e = indptr[x]; e < indptr[x + 1]; ++e) {
            const int32_t y = indices[e];
            if (y >= 0 && y < n_nodes && dist[y] < 0) {
                dist[y] = dist[x] + 1;
                cone.push_back(y);
            }
        }
    }
    const int n = (int)cone.size();
    for (int i = 0; i < n; ++i) loc[cone[i]] = i;
    // induced subgraph in CSR form, local indices
    std::vector<int32_t> off(n + 1, 0), adj;
    for (int i = 0; i < n; ++i) {
        const int32_t x = cone[i];
        const auto begin = (std::ptrdiff_t)adj.size();
        for (int64_t e = indptr[x]; e < indptr[x + 1]; ++e) {
            const int32_t y = indices[e];
            if (y >= 0 && y < n_nodes && y != x && loc[y] >= 0) adj.push_back(loc[y]);
        }
        std::sort(adj.begin() + begin, adj.end());
        adj.erase(std::unique(adj.begin() + begin, adj.end()), adj.end());
        off[i + 1] = (int32_t)adj.size();
    }
    // colour refinement to a stable partition.  A round's colour is a hash
    // of the node's colour and its neighbours' sorted colours; a collision
    // could only merge classes and cost a share, because keys are compared
    // in full.
    std::vector<int32_t> color(n);
    std::vector<uint64_t> h(n);
    std::vector<int32_t> idx(n), nc;
    auto relabel = [&]() {
        std::iota(idx.begin(), idx.end(), 0);
        std::sort(idx.begin(), idx.end(), [&](int a, int b) { return h[a] < h[b]; });
        int classes = 0;
        for (int k = 0; k < n; ++k) {
            if (k > 0 && h[idx[k]] != h[idx[k - 1]]) ++classes;
            color[idx[k]] = classes;
        }
        return classes + 1;
    };
    auto mix = [](uint64_t x, uint64_t y) {
        x ^= y + 0x9E3779B97F4A7C15ull + (x << 6) + (x >> 2);
        x *= 0xff51afd7ed558ccdull;
        return x ^ (x >> 33);
    };
    for (int i = 0; i < n; ++i)
        h[i] = mix((uint64_t)dist[cone[i]], (uint64_t)(i == 0 ? 1 : (i == 1 ? 2 : 0)));
    int classes = relabel();
    for (int round = 0; round < n; ++round) {
        for (int i = 0; i < n; ++i) {
            nc.clear();
            for (int32_t k = off[i]; k < off[i + 1]; ++k) nc.push_back(color[adj[k]]);
            std::sort(nc.begin(), nc.end());
            uint64_t x = mix(0x51ED270Bull, (uint64_t)color[i]);
            for (int32_t c : nc) x = mix(x, (uint64_t)c);
            h[i] = mix(x, nc.size());
        }
        const int next = relabel();
        if (next == classes) break;
        classes = next;
    }
    // level-by-level canonical ranks
    std::vector<int32_t> rank(n, -1), order;
    rank[0] = 0;
    rank[1] = 1;
    order = {0, 1};
    std::vector<int32_t> level, up, up_begin(n), up_end(n);   // ranks of the neighbours one level closer
    for (int d = 1; d <= p; ++d) {
        level.clear();
        up.clear();
        for (int i = 0; i < n; ++i)
            if (dist[cone[i]] == d) {
                level.push_back(i);
                up_begin[i] = (int32_t)up.size();
                for (int32_t k = off[i]; k < off[i + 1]; ++k)
                    if (dist[cone[adj[k]]] == d - 1) up.push_back(rank[adj[k]]);
                up_end[i] = (int32_t)up.size();
                std::sort(up.begin() + up_begin[i], up.end());
            }
        std::sort(level.begin(), level.end(), [&](int a, int b) {
            if (color[a] != color[b]) return color[a] < color[b];
            const bool ab = std::lexicographical_compare(up.begin() + up_begin[a], up.begin() + up_end[a],
                                                         up.begin() + up_begin[b], up.begin() + up_end[b]);
            const bool ba = std::lexicographical_compare(up.begin() + up_begin[b], up.begin() + up_end[b],
                                                         up.begin() + up_begin[a], up.begin() + up_end[a]);
            if (ab != ba) return ab;
            return cone[a] < cone[b];
        });
        for (int32_t i : level) {
            rank[i] = (int32_t)order.size();
            order.push_back(i);
        }
    }
    key->clear();
    key->push_back(n);
    key->push_back(p);
    for (int32_t i : order) key->push_back(dist[cone[i]]);
    std::vector<std::pair<int32_t, int32_t>> edges;
    for (int i = 0; i < n; ++i)
        for (int32_t k = off[i]; k < off[i + 1]; ++k)
            if (rank[i] < rank[adj[k]]) edges.emplace_back(rank[i], rank[adj[k]]);
    std::sort(edges.begin(), edges.end());
    for (const auto& e : edges) {
        key->push_back(e.first);
        key->push_back(e.second);
    }
}

// ------------------------------------------------------ plan assembly
void merge_network(qtb_plan* plan, Network&& net, int32_t group) {
    net.info.group = group;
    std::vector<uint32_t> table_off(net.entries.size());
    for (size_t i = 0; i < net.entries.size(); ++i) {
        const EntryKey& key = net.entries[i];
        auto it = plan->entry_index.find(key);
        if (it == plan->entry_index.end()) {
            DevEntry e{};
            e.kind = key.kind;
            e.expr_begin = (int32_t)plan->terms.size();
            e.expr_count = (int32_t)key.expr.size();
            for (const auto& t : key.expr) plan->terms.push_back(DevTerm{t.first, 0, t.second});
            e.off = plan->table_elems;
            e.rank_in = key.rank_in;
            e.rank_out = (int8_t)key.perm.size();
            e.sliced_mask = key.sliced_mask;
            e.sliced_value = key.sliced_value;
            for (int a = 0; a < 4; ++a) e.perm[a] = a < (int)key.perm.size() ? key.perm[a] : -1;
            plan->table_elems += 1u << e.rank_out;
            it = plan->entry_index.emplace(key, (int32_t)plan->entries.size()).first;
            plan->entries.push_back(e);
        }
        table_off[i] = plan->entries[it->second].off;
    }
    for (DevIn& in : net.ins)
        if (in.src & kSrcTable) in.src = kSrcTable | table_off[in.src & ~kSrcTable];
    if (net.result_src & kSrcTable) net.result_src = kSrcTable | table_off[net.result_src & ~kSrcTable];
    for (AngleCheck& c : net.checks)   // networks of a circuit, and shared edges, repeat decisions
        if (plan->check_index.emplace(c.must_be_small, c.expr).second) plan->checks.push_back(c);
    net.entries.clear();
    net.entries.shrink_to_fit();
    plan->nets.push_back(std::move(net));
    plan->uploaded = false;
    plan->images_valid = false;
    plan->flat_valid = false;
}

void flatten_plan(qtb_plan* plan) {
    plan->dnets.clear();
    plan->dops.clear();
    plan->dins.clear();
    plan->dphases.clear();
    for (const Network& n : plan->nets) {
        DevNet d{};
        d.op_begin = (uint32_t)plan->dops.size();
        d.n_ops = (uint32_t)n.ops.size();
        d.phase_begin = (uint32_t)plan->dphases.size();
        d.n_phases = (uint32_t)n.phases.size();
        d.arena_elems = (uint32_t)n.info.arena_elems;
        d.result_src = n.result_src;
        d.max_elems = n.max_elems;
        const uint32_t in_base = (uint32_t)plan->dins.size();
        for (DevOp op : n.ops) {
            op.in_begin += in_base;
            plan->dops.push_back(op);
        }
        plan->dins.insert(plan->dins.end(), n.ins.begin(), n.ins.end());
        for (DevPhase ph : n.phases) {
            ph.op_first += d.op_begin;
            plan->dphases.push_back(ph);
        }
        plan->dnets.push_back(d);
    }
}

// CPUs this process may run on: the hardware threads, bounded by its
// affinity mask and by a cgroup CPU quota (cgroup v2 cpu.max, v1
// cfs_quota_us / cfs_period_us).  In a container the hardware count is the
// host's; threads beyond the quota are throttled in bursts, which showed as
// compile latencies of seconds.
static int available_cpus() {
    static const int n = [] {
        int c = (int)std::max(1u, std::thread::hardware_concurrency());
        cpu_set_t set;
        CPU_ZERO(&set);
        if (sched_getaffinity(0, sizeof(set), &set) == 0) c = std::min(c, std::max(1, CPU_COUNT(&set)));
        auto quota_cpus = [](double quota, double period) {
            return (quota > 0 && period > 0) ? std::max(1, (int)std::ceil(quota / period)) : 0;
        };
        if (FILE* f = std::fopen("/sys/fs/cgroup/cpu.max", "r")) {
            char q[32] = {0};
            double period = 0;
            if (std::fscanf(f, "%31s %lf", q, &period) == 2 && std::strcmp(q, "max") != 0) {
                const int qc = quota_cpus(std::atof(q), period);
                if (qc) c = std::min(c, qc);
            }
            std::fclose(f);
        } else if (FILE* fq = std::fopen("/sys/fs/cgroup/cpu/cpu.cfs_quota_us", "r")) {
            double quota = -1, period = 0;
            if (std::fscanf(fq, "%lf", &quota) != 1) quota = -1;
            std::fclose(fq);
            if (FILE* fp = std::fopen("/sys/fs/cgroup/cpu/cpu.cfs_period_us", "r")) {
                if (std::fscanf(fp, "%lf", &period) != 1) period = 0;
                std::fclose(fp);
            }
            const int qc = quota_cpus(quota, period);
            if (qc) c = std::min(c, qc);
        }
        return c;
    }();
    return n;
}

// Runs fn(i) for i in [0, n) on up to n_threads threads (0 = every CPU the
// process may use).
template <typename Fn>
static void parallel_for(int32_t n, int32_t n_threads, Fn fn) {
    std::atomic<int32_t> next{0};
    auto worker = [&]() {
        for (int32_t i; (i = next.fetch_add(1)) < n;) fn(i);
    };
    int nt = n_threads > 0 ? n_threads : available_cpus();
    nt = std::max(1, std::min(nt, std::max(1, n)));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

// Bits of x selected by m, packed from bit 0 up.
static uint32_t pext_bits(uint32_t x, uint32_t m) {
    uint32_t r = 0, bit = 1;
    while (m) {
        const uint32_t lo = m & (0u - m);
        if (x & lo) r |= bit;
        bit <<= 1;
        m ^= lo;
    }
    return r;
}

// Largest operand count of a phase's ops.
static uint32_t phase_kmax(const Network& n, const DevPhase& ph) {
    uint32_t kmax = 1;
    for (uint32_t o = ph.op_first; o < ph.op_first + ph.op_count; ++o) kmax = std::max<uint32_t>(kmax, n.ops[o].k);
    return kmax;
}

// Words of a network's element records (layout at DevNetRun), or 0 when it
// cannot have them: an op without operands or with more than kRecMaxK, an
// arena past the shared-memory window (`smem_elems` complex64 elements
// beside the gate table), or window offsets past 16 bits.
// Format of a network's element records (kRecCompact when its window and
// operand counts allow, else kRecWide), or 0 when it cannot have them.
static uint32_t record_format(const Network& n, uint32_t table_pad, uint64_t smem_elems) {
    const uint64_t arena = n.info.arena_elems;
    if (arena > smem_elems || table_pad + arena > 0xffffu) return 0;
    uint32_t kmax = 0;
    for (const DevOp& op : n.ops) {
        if (op.k < 1 || op.k > kRecMaxK) return 0;
        kmax = std::max<uint32_t>(kmax, op.k);
    }
    return (table_pad + arena <= kRecCompactWindow && kmax <= kRecCompactMaxK) ? kRecCompact : kRecWide;
}

static uint32_t record_words(const Network& n, uint32_t format) {
    uint64_t words = 2 * n.phases.size();
    if (format == kRecCompact) {
        words = (words + 3) & ~uint64_t(3);
        for (const DevPhase& ph : n.phases) words += 4 * (uint64_t)ph.total_elems;
    } else {
        for (const DevPhase& ph : n.phases) words += (uint64_t)(phase_kmax(n, ph) + 1) * ph.total_elems;
    }
    return words > 0xffffffffu ? 0 : (uint32_t)words;
}

// Offsets of operand d of an op (output bits `low`, summed bit w) for every
// output element j, passed to emit(j, offset at summed variable 0, stride
// to its offset at 1 or 0).  Gathers the low byte of j from a table.
template <typename Emit>
static void operand_offsets(const DevOp& op, const DevIn& d, uint32_t table_pad, uint32_t* lo_tab, Emit emit) {
    const uint32_t w = (uint32_t)op.u - op.sum;
    const uint32_t low = (1u << w) - 1u;
    const uint32_t m = d.mask & low;
    const uint32_t src = (d.src & kSrcTable) ? (d.src & ~kSrcTable) : table_pad + d.src;
    const uint32_t stride = (op.sum && ((d.mask >> w) & 1u)) ? 1u << (__builtin_popcount(d.mask) - 1) : 0u;
    const uint32_t m_lo = m & 0xffu, shift = (uint32_t)__builtin_popcount(m_lo);
    const uint32_t n_lo = std::min(low, 255u) + 1u;
    for (uint32_t x = 0; x < n_lo; ++x) lo_tab[x] = pext_bits(x, m_lo);
    for (uint32_t hi = 0; hi <= (low >> 8); ++hi) {
        const uint32_t hoff = src + (pext_bits(hi, m >> 8) << shift);
        for (uint32_t x = 0; x < n_lo; ++x) emit((hi << 8) | x, hoff + lo_tab[x], stride);
    }
}

// First record of every op of a phase (indexed from op_first): the ops in
// order of decreasing operand count (stable), so that the 32 elements a
// warp takes mostly share it and its loop over operands.  Each record
// names its own output, so the order is free.
static void record_positions(const Network& n, const DevPhase& ph, std::vector<uint32_t>& pos) {
    std::vector<uint32_t> order(ph.op_count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        return n.ops[ph.op_first + x].k > n.ops[ph.op_first + y].k;
    });
    pos.assign(ph.op_count, 0u);
    uint32_t next = 0;
    for (uint32_t x : order) {
        const DevOp& op = n.ops[ph.op_first + x];
        pos[x] = next;
        next += 1u << ((uint32_t)op.u - op.sum);
    }
}

// One phase of compact records (layout at kRecCompact), 8 fields per element.
static void fill_compact_phase(const Network& n, const DevPhase& ph, uint32_t table_pad, uint16_t* f,
                               uint32_t* lo_tab) {
    std::vector<uint32_t> pos;
    record_positions(n, ph, pos);
    for (uint32_t o = ph.op_first; o < ph.op_first + ph.op_count; ++o) {
        const DevOp& op = n.ops[o];
        const uint32_t low = (1u << ((uint32_t)op.u - op.sum)) - 1u;
        uint16_t* r = f + 8 * (size_t)pos[o - ph.op_first];
        for (uint32_t j = 0; j <= low; ++j)
            r[8 * j] = (uint16_t)((table_pad + op.dst + j) | (uint32_t)(op.k - 1) << 12 | (uint32_t)op.sum << 15);
        for (uint32_t t = 0; t < op.k; ++t)
            operand_offsets(op, n.ins[op.in_begin + t], table_pad, lo_tab, [&](uint32_t j, uint32_t o0, uint32_t stride) {
                const uint32_t code = stride ? (uint32_t)__builtin_ctz(stride) + 1u : 0u;
                r[8 * j + 1 + t] = (uint16_t)(o0 | code << 12);
            });
    }
}

// Writes a network's element records into rec (record_words words, zeroed),
// with the gate table's padded size `table_pad` as the arena's offset in
// the shared window.  The offsets are the bit gathers compute_element
// would do, resolved once: the bits of element j that the operand's mask
// selects, packed, plus its source; the summed variable is the operand's
// top axis.
static void fill_records(const Network& n, uint32_t table_pad, uint32_t format, uint32_t* rec) {
    const size_t n_ph = n.phases.size();
    const bool compact = format == kRecCompact;
    uint32_t payload = (uint32_t)(compact ? (2 * n_ph + 3) & ~size_t(3) : 2 * n_ph);
    uint32_t lo_tab[256];
    for (size_t p = 0; p < n_ph; ++p) {
        const DevPhase& ph = n.phases[p];
        const uint32_t kmax = phase_kmax(n, ph);
        const uint32_t total = ph.total_elems;
        rec[2 * p] = payload;
        rec[2 * p + 1] = total | kmax << 24;
        if (compact) {
            fill_compact_phase(n, ph, table_pad, reinterpret_cast<uint16_t*>(rec + payload), lo_tab);
            payload += 4 * total;
            continue;
        }
        uint32_t* row = rec + payload;
        std::vector<uint32_t> pos;
        record_positions(n, ph, pos);
        for (uint32_t o = ph.op_first; o < ph.op_first + ph.op_count; ++o) {
            const DevOp& op = n.ops[o];
            const uint32_t first = pos[o - ph.op_first];
            const uint32_t w = (uint32_t)op.u - op.sum;
            const uint32_t low = (1u << w) - 1u;
            for (uint32_t t = 0; t < op.k; ++t) {
                const DevIn& d = n.ins[op.in_begin + t];
                const uint32_t m = d.mask & low;
                const uint32_t src = (d.src & kSrcTable) ? (d.src & ~kSrcTable) : table_pad + d.src;
                const uint32_t stride = (op.sum && ((d.mask >> w) & 1u)) ? 1u << (__builtin_popcount(d.mask) - 1) : 0u;
                uint32_t* r = row + (size_t)(t + 1) * total + first;
                // j = hi << 8 | lo: the gather of the low byte from a table
                const uint32_t m_lo = m & 0xffu, shift = (uint32_t)__builtin_popcount(m_lo);
                const uint32_t n_lo = std::min(low, 255u) + 1u;
                for (uint32_t x = 0; x < n_lo; ++x) lo_tab[x] = pext_bits(x, m_lo);
                for (uint32_t hi = 0; hi <= (low >> 8); ++hi) {
                    const uint32_t hoff = src + (pext_bits(hi, m >> 8) << shift);
                    uint32_t* rh = r + (hi << 8);
                    for (uint32_t x = 0; x < n_lo; ++x) {
                        const uint32_t o0 = hoff + lo_tab[x];
                        rh[x] = o0 | (o0 + stride) << 16;
                    }
                }
            }
            uint32_t* r0 = row + first;
            const uint32_t head = (uint32_t)op.k << 16 | (uint32_t)op.sum << 24;
            for (uint32_t j = 0; j <= low; ++j) r0[j] = (table_pad + op.dst + j) | head;
        }
        payload += (kmax + 1) * total;
    }
}

// Per-network blobs with network-local indices (see DevNetRun).
// Networks whose blobs are byte-identical (edges that shared a compile, or
// equal slices) point at one copy: each is still contracted on its own, but
// the plan image holds one blob, which the executors then stage from L2.
// Element records follow the blobs: one copy per distinct blob, for plans
// whose gate table fits shared memory, up to kRecMaxWords words per plan.
void build_blobs(qtb_plan* plan) {
    plan->druns.clear();
    plan->dblobs.clear();
    plan->drecs.clear();
    const bool records = plan->records && plan->table_elems <= kSmemTableLimitElems;
    const uint32_t table_pad = (plan->table_elems + 1u) & ~1u;
    // shared memory left for an arena beside the staged gate entries,
    // angle terms and gate table (an upper bound on what any launch has)
    const uint64_t fixed = 16 + ((plan->entries.size() * sizeof(DevEntry) + 15) & ~size_t(15)) +
                           plan->terms.size() * sizeof(DevTerm) + 8 * (uint64_t)table_pad;
    const uint64_t smem_elems = fixed < kSmemLimitBytes ? (kSmemLimitBytes - fixed) / 8 : 0;
    uint64_t rec_total = 0;
    std::vector<std::pair<int32_t, uint32_t>> rec_todo;   // (network, first word)
    std::unordered_map<uint64_t, std::vector<uint32_t>> seen;   // hash -> blob offsets (16 B units)
    for (const Network& n : plan->nets) {
        DevNetRun r{};
        r.blob_off16 = (uint32_t)(plan->dblobs.size() / 16);
        r.n_phases = (uint32_t)n.phases.size();
        r.arena_elems = (uint32_t)n.info.arena_elems;
        r.result_src = n.result_src;
        r.max_elems = n.max_elems;
        r.tail_start = (uint32_t)n.phases.size();
        while (r.tail_start > 0 && n.phases[r.tail_start - 1].total_elems <= 32) --r.tail_start;
        const size_t ph_bytes = n.phases.size() * sizeof(DevPhase);
        const size_t op_bytes = n.ops.size() * sizeof(DevOp);
        const size_t in_bytes = n.ins.size() * sizeof(DevIn);
        r.ins_off = (uint32_t)(ph_bytes + op_bytes);
        // chunk tables: op of every kChunkElems-th flattened element, for
        // the executors that keep the arena in shared memory (a network
        // whose arena cannot be there runs in waves or clusters, which find
        // ops by search; its tables would grow with its elements)
        std::vector<DevPhase> phases = n.phases;
        std::vector<uint16_t> chunks;
        size_t chunk_base = ph_bytes + op_bytes + in_bytes;
        const bool chunked = 8 * (uint64_t)n.info.arena_elems <= kSmemLimitBytes;
        for (DevPhase& ph : phases) {
            ph.chunk_off = chunked ? (uint32_t)(chunk_base + chunks.size() * sizeof(uint16_t)) : 0u;
            if (!chunked) continue;
            uint32_t oi = ph.op_first;
            for (uint32_t e = 0; e < ph.total_elems; e += kChunkElems) {
                while (oi + 1 < ph.op_first + ph.op_count && n.ops[oi + 1].elem_begin <= e) ++oi;
                chunks.push_back((uint16_t)oi);
            }
        }
        const size_t total = (chunk_base + chunks.size() * sizeof(uint16_t) + 15) & ~size_t(15);
        r.blob_bytes = (uint32_t)total;
        const size_t base = plan->dblobs.size();
        plan->dblobs.resize(base + total, 0);
        uint8_t* dst = plan->dblobs.data() + base;
        std::memcpy(dst, phases.data(), ph_bytes);     // op_first already network-local
        std::memcpy(dst + ph_bytes, n.ops.data(), op_bytes);   // in_begin network-local
        std::memcpy(dst + ph_bytes + op_bytes, n.ins.data(), in_bytes);
        if (!chunks.empty())
            std::memcpy(dst + chunk_base, chunks.data(), chunks.size() * sizeof(uint16_t));
        uint64_t h = 0x9E3779B97F4A7C15ull ^ total;   // blobs are whole 16-byte units
        for (size_t b = 0; b < total; b += 8) {
            uint64_t word;
            std::memcpy(&word, dst + b, 8);
            h = (h ^ word) * 0xff51afd7ed558ccdull;
            h ^= h >> 32;
        }
        auto& offs = seen[h];
        for (uint32_t o : offs) {
            const DevNetRun& prev = plan->druns[o];
            if (prev.blob_bytes == total &&
                std::memcmp(plan->dblobs.data() + 16 * (size_t)prev.blob_off16, dst, total) == 0) {
                r.blob_off16 = prev.blob_off16;
                r.rec_off = prev.rec_off;
                r.rec_words = prev.rec_words;
                r.rec_format = prev.rec_format;
                plan->dblobs.resize(base);
                break;
            }
        }
        if (r.blob_off16 == (uint32_t)(base / 16)) {
            offs.push_back((uint32_t)plan->druns.size());
            const uint32_t format = records ? record_format(n, table_pad, smem_elems) : 0u;
            const uint32_t words = format ? record_words(n, format) : 0u;
            // each network's records start on 16 bytes: the executor reads
            // phase headers as 8-byte pairs and compact records as 16 bytes
            const uint64_t start = (rec_total + 3) & ~uint64_t(3);
            if (words && start + words <= kRecMaxWords) {
                r.rec_off = (uint32_t)start;
                r.rec_words = words;
                r.rec_format = format;
                rec_total = start + words;
                rec_todo.emplace_back((int32_t)plan->druns.size(), r.rec_off);
            }
        }
        plan->druns.push_back(r);
    }
    plan->drecs.assign(rec_total, 0u);
    parallel_for((int32_t)rec_todo.size(), 0, [&](int32_t t) {
        const auto& job = rec_todo[t];
        fill_records(plan->nets[job.first], table_pad, plan->druns[job.first].rec_format,
                     plan->drecs.data() + job.second);
    });
}

void ensure_images(qtb_plan* plan) {
    if (plan->images_valid) return;
    build_blobs(plan);
    plan->images_valid = true;
}

void ensure_flat(qtb_plan* plan) {
    if (plan->flat_valid) return;
    flatten_plan(plan);
    plan->flat_valid = true;
}

}  // namespace qtb

// =================================================================== C ABI
using namespace qtb;

// Most int32 words of cone invariants and keys one lightcone call may hold
// (256 MiB); past it, edges are compiled without sharing.
constexpr size_t kShareKeyLimit = size_t(1) << 26;


extern "C" {

int qtb_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return QTB_ERR_ARG;
    std::strncpy(buf, g_err.c_str(), len - 1);
    buf[len - 1] = '\0';
    return QTB_OK;
}

int qtb_plan_create(int32_t n_params, qtb_plan** out) {
    if (!out || n_params < 0) return fail(QTB_ERR_ARG, "plan_create: bad arguments");
    qtb_plan* p = new qtb_plan();
    p->n_params = n_params;
    *out = p;
    return QTB_OK;
}

int qtb_plan_add_circuit(qtb_plan* plan, int32_t n_qubits, const qtb_gate* gates, int32_t n_gates,
                         int32_t simplify_passes, const double* params, int32_t* net_index) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_add_circuit: null plan");
    std::vector<Network> nets;
    std::string err;
    int rc = compile_circuit(n_qubits, gates, n_gates, simplify_passes, params, plan->n_params,
                             plan->order_trials, plan->max_width, plan->max_slices, plan->slicing, 0, &nets, &err);
    if (rc) return fail(rc, err);
    std::lock_guard<std::mutex> lock(plan->mu);
    if (net_index) *net_index = (int32_t)plan->nets.size();
    const int32_t group = plan->n_groups++;
    for (auto& n : nets) merge_network(plan, std::move(n), group);
    return QTB_OK;
}

int qtb_plan_add_circuit_batch(qtb_plan* plan, int32_t n_qubits, const qtb_gate* gates, int32_t n_gates,
                               int32_t simplify_passes, const double* params, int32_t batch_vars,
                               int32_t* net_index, int32_t* first_group) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_add_circuit_batch: null plan");
    std::vector<Network> nets;
    std::string err;
    int rc = compile_circuit(n_qubits, gates, n_gates, simplify_passes, params, plan->n_params,
                             plan->order_trials, plan->max_width, plan->max_slices, plan->slicing, batch_vars,
                             &nets, &err);
    if (rc) return fail(rc, err);
    const size_t n_amps = size_t(1) << batch_vars;
    const size_t per_amp = nets.size() / n_amps;
    std::lock_guard<std::mutex> lock(plan->mu);
    if (net_index) *net_index = (int32_t)plan->nets.size();
    if (first_group) *first_group = plan->n_groups;
    const int32_t group0 = plan->n_groups;
    plan->n_groups += (int32_t)n_amps;
    for (size_t i = 0; i < nets.size(); ++i) merge_network(plan, std::move(nets[i]), group0 + (int32_t)(i / per_amp));
    return QTB_OK;
}

int qtb_plan_add_lightcone(qtb_plan* plan, int32_t n_nodes, const int64_t* indptr,
                           const int32_t* indices, int32_t u, int32_t v, int32_t p,
                           int32_t composer, const double* params, int32_t* net_index) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_add_lightcone: null plan");
    if (plan->n_params != 2 * p) return fail(QTB_ERR_ARG, "plan_add_lightcone: plan needs 2*p params");
    std::vector<qtb_gate> gates;
    int32_t nq = 0;
    std::string err;
    int rc = build_lightcone(n_nodes, indptr, indices, u, v, p, composer, &gates, &nq, &err);
    if (rc) return fail(rc, err);
    return qtb_plan_add_circuit(plan, nq, gates.data(), (int32_t)gates.size(),
                                composer == 0 ? 2 : 0, params, net_index);
}

int qtb_plan_add_lightcones(qtb_plan* plan, int32_t n_nodes, const int64_t* indptr,
                            const int32_t* indices, const int32_t* edges, int32_t n_edges,
                            int32_t p, int32_t composer, const double* params, int32_t n_threads,
                            int32_t* first_net_index) {
    if (!plan || !edges || n_edges < 0) return fail(QTB_ERR_ARG, "plan_add_lightcones: bad arguments");
    if (plan->n_params != 2 * p) return fail(QTB_ERR_ARG, "plan_add_lightcones: plan needs 2*p params");
    if (n_edges > 0 && (n_nodes <= 0 || !indptr || !indices))
        return fail(QTB_ERR_ARG, "plan_add_lightcones: bad graph");
    std::vector<std::vector<Network>> nets(n_edges);
    std::vector<int> codes(n_edges, 0);
    std::vector<std::string> errs(n_edges);
    // edges whose lightcones are isomorphic share one compile: the first
    // edge of each class (in edge order, so plans do not depend on thread
    // timing) is compiled, the others copy its networks
    std::vector<int32_t> rep(n_edges);
    std::iota(rep.begin(), rep.end(), 0);
    if (plan->share_lightcones && n_edges > 1) {
        auto valid = [&](int32_t i) {
            const int32_t a = edges[2 * i], b = edges[2 * i + 1];
            return a >= 0 && b >= 0 && a < n_nodes && b < n_nodes && a != b && p >= 0;
        };
        // coarse invariants first: only edges whose invariant recurs can share
        std::vector<std::vector<int32_t>> keys(n_edges);
        parallel_for(n_edges, n_threads, [&](int32_t i) {
            if (valid(i)) cone_invariant(n_nodes, indptr, indices, edges[2 * i], edges[2 * i + 1], p, &keys[i]);
        });
        size_t held = 0;
        for (const auto& k : keys) held += k.size();
        if (held > kShareKeyLimit) {   // very large cones: compile every edge, hold no keys
            keys.clear();
            keys.shrink_to_fit();
            keys.resize(n_edges);
        } else {
            std::unordered_map<uint64_t, std::vector<int32_t>> seen;
            std::vector<char> recurs(n_edges, 0);
            for (int32_t i = 0; i < n_edges; ++i) {
                if (keys[i].empty()) continue;
                uint64_t h = 1469598103934665603ull;
                for (int32_t x : keys[i]) h = (h ^ (uint32_t)x) * 1099511628211ull;
                auto& firsts = seen[h];   // first edge of every distinct invariant
                bool found = false;
                for (int32_t r : firsts)
                    if (keys[r] == keys[i]) {
                        recurs[r] = recurs[i] = 1;
                        found = true;
                        break;
                    }
                if (!found) firsts.push_back(i);
            }
            for (int32_t i = 0; i < n_edges; ++i)
                if (!recurs[i]) keys[i].clear();
            parallel_for(n_edges, n_threads, [&](int32_t i) {
                if (recurs[i]) cone_key(n_nodes, indptr, indices, edges[2 * i], edges[2 * i + 1], p, &keys[i]);
            });
        }
        std::unordered_map<uint64_t, std::vector<int32_t>> classes;
        for (int32_t i = 0; i < n_edges; ++i) {
            if (keys[i].empty()) continue;   // no key (invalid edge, or a cone no other matches): alone
            uint64_t h = 1469598103934665603ull;
            for (int32_t x : keys[i]) h = (h ^ (uint32_t)x) * 1099511628211ull;
            auto& members = classes[h];
            for (int32_t r : members)
                if (keys[r] == keys[i]) {
                    rep[i] = r;
                    break;
                }
            if (rep[i] == i) members.push_back(i);
        }
    }
    std::vector<int32_t> todo;
    for (int32_t i = 0; i < n_edges; ++i)
        if (rep[i] == i) todo.push_back(i);
    std::atomic<bool> failed{false};   // one failing edge fails the call: stop early
    parallel_for((int32_t)todo.size(), n_threads, [&](int32_t t) {
        const int32_t i = todo[t];
        if (failed.load(std::memory_order_relaxed)) {
            codes[i] = kCompileAborted;
            return;
        }
        static thread_local std::vector<qtb_gate> gates;
        int32_t nq = 0;
        int rc = build_lightcone(n_nodes, indptr, indices, edges[2 * i], edges[2 * i + 1], p,
                                 composer, &gates, &nq, &errs[i]);
        if (!rc)
            rc = compile_circuit(nq, gates.data(), (int32_t)gates.size(), composer == 0 ? 2 : 0,
                                 params, plan->n_params, plan->order_trials, plan->max_width,
                                 plan->max_slices, plan->slicing, 0, &nets[i], &errs[i], &failed);
        codes[i] = rc;
        if (rc && rc != kCompileAborted) failed.store(true, std::memory_order_relaxed);
    });
    for (int32_t i = 0; i < n_edges; ++i)   // the first genuine failure (not an abort)
        if (codes[rep[i]] && codes[rep[i]] != kCompileAborted)
            return fail(codes[rep[i]], "edge " + std::to_string(i) + ": " + errs[rep[i]]);
    for (int32_t i = 0; i < n_edges; ++i)
        if (rep[i] != i) nets[i] = nets[rep[i]];
    std::lock_guard<std::mutex> lock(plan->mu);
    if (first_net_index) *first_net_index = (int32_t)plan->nets.size();
    for (auto& circuit : nets) {
        const int32_t group = plan->n_groups++;
        for (auto& n : circuit) merge_network(plan, std::move(n), group);
    }
    return QTB_OK;
}

int qtb_plan_set_max_width(qtb_plan* plan, int32_t max_width, int32_t max_slices) {
    if (!plan || max_width < 0 || max_slices < 1)
        return fail(QTB_ERR_ARG, "plan_set_max_width: bad arguments");
    plan->max_width = max_width;
    plan->max_slices = max_slices;
    return QTB_OK;
}

int qtb_plan_set_slicing(qtb_plan* plan, int32_t method) {
    if (!plan || method < QTB_SLICE_GREEDY || method > QTB_SLICE_LATE)
        return fail(QTB_ERR_ARG, "plan_set_slicing: unknown method");
    plan->slicing = method;
    return QTB_OK;
}

int qtb_plan_set_share_lightcones(qtb_plan* plan, int32_t enable) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_set_share_lightcones: null plan");
    plan->share_lightcones = enable != 0;
    return QTB_OK;
}

int qtb_plan_set_records(qtb_plan* plan, int32_t enable) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_set_records: null plan");
    std::lock_guard<std::mutex> lock(plan->mu);
    if (plan->uploaded) return fail(QTB_ERR_ARG, "plan_set_records: set before qtb_plan_upload");
    if (plan->records != (enable != 0)) plan->images_valid = false;
    plan->records = enable != 0;
    return QTB_OK;
}

int qtb_plan_set_order_trials(qtb_plan* plan, int32_t trials) {
    if (!plan || trials < 0) return fail(QTB_ERR_ARG, "plan_set_order_trials: bad arguments");
    plan->order_trials = trials;
    return QTB_OK;
}

int qtb_plan_n_networks(const qtb_plan* plan, int32_t* n) {
    if (!plan || !n) return fail(QTB_ERR_ARG, "plan_n_networks: bad arguments");
    *n = (int32_t)plan->nets.size();
    return QTB_OK;
}

int qtb_plan_network_info(const qtb_plan* plan, int32_t net, qtb_network_info* info) {
    if (!plan || !info || net < 0 || net >= (int32_t)plan->nets.size())
        return fail(QTB_ERR_ARG, "plan_network_info: bad arguments");
    *info = plan->nets[net].info;
    return QTB_OK;
}

int qtb_plan_network_peo(const qtb_plan* plan, int32_t net, int32_t* peo, int32_t cap, int32_t* n) {
    if (!plan || !n || net < 0 || net >= (int32_t)plan->nets.size())
        return fail(QTB_ERR_ARG, "plan_network_peo: bad arguments");
    const auto& src = plan->nets[net].peo;
    *n = (int32_t)src.size();
    if (peo) std::copy(src.begin(), src.begin() + std::min<size_t>(src.size(), (size_t)std::max(cap, 0)), peo);
    return QTB_OK;
}

int qtb_plan_check_params(const qtb_plan* plan, const double* params, int32_t* valid) {
    if (!plan || !valid || (plan->n_params > 0 && !params))
        return fail(QTB_ERR_ARG, "plan_check_params: bad arguments");
    *valid = 1;
    for (const AngleCheck& c : plan->checks) {
        double x = 0.0;
        for (const auto& t : c.expr) x += t.second * params[t.first];
        const bool small = std::fabs(x) < 1e-5;
        if (small != c.must_be_small) {
            *valid = 0;
            break;
        }
    }
    return QTB_OK;
}

int qtb_plan_export(qtb_plan* plan, int32_t which, void* buf, size_t cap, size_t* size) {
    if (!plan || !size) return fail(QTB_ERR_ARG, "plan_export: bad arguments");
    std::lock_guard<std::mutex> lock(plan->mu);
    ensure_images(plan);
    ensure_flat(plan);
    const void* src = nullptr;
    size_t n = 0;
    switch (which) {
        case 0: src = plan->dnets.data(); n = plan->dnets.size() * sizeof(DevNet); break;
        case 1: src = plan->dops.data(); n = plan->dops.size() * sizeof(DevOp); break;
        case 2: src = plan->dins.data(); n = plan->dins.size() * sizeof(DevIn); break;
        case 3: src = plan->dphases.data(); n = plan->dphases.size() * sizeof(DevPhase); break;
        case 4: src = plan->entries.data(); n = plan->entries.size() * sizeof(DevEntry); break;
        case 5: src = plan->terms.data(); n = plan->terms.size() * sizeof(DevTerm); break;
        case 6: src = plan->druns.data(); n = plan->druns.size() * sizeof(DevNetRun); break;
        case 7: src = plan->dblobs.data(); n = plan->dblobs.size(); break;
        case 8: src = plan->drecs.data(); n = plan->drecs.size() * sizeof(uint32_t); break;
        default: return fail(QTB_ERR_ARG, "plan_export: unknown array");
    }
    *size = n;
    if (buf && n) std::memcpy(buf, src, std::min(cap, n));
    return QTB_OK;
}

int qtb_plan_table_elems(const qtb_plan* plan, int64_t* n) {
    if (!plan || !n) return fail(QTB_ERR_ARG, "plan_table_elems: bad arguments");
    *n = plan->table_elems;
    return QTB_OK;
}

}  // extern "C"
