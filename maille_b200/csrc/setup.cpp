// setup.cpp -- host-side symbolic analysis: kept nodes, node graph, ordering (RCM or multicolour),
// level sets, the full 3x3-block CSR pattern and the deterministic element-to-slot scatter map.
//
// Reference counterparts: FreeSystem::new numbers the free DOFs, builds the DOF graph
// (Graph::from_elements, iterative.rs:38-76), orders it by reverse_cuthill_mckee (solve.rs:200-245)
// and allocates the lower-triangular CSR profile (Csr::zeros, iterative.rs:91-114); each element
// matrix entry is then added by a binary search (Csr::add, iterative.rs:121-128). Here the same
// work is done once per mesh topology on nodes instead of scalar DOFs, and the binary searches
// are replaced by a precomputed scatter map that the GPU reduces in a fixed order.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <thread>

#include "common.hpp"

namespace maille {
namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Runs fn(begin, end) over [0, n) split into contiguous chunks on the host's cores.
template <typename F>
void parallel_for(int64_t n, F&& fn) {
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t chunks = std::min<int64_t>(hw, std::max<int64_t>(1, n / 4096));
    if (chunks <= 1) {
        fn(int64_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    for (int64_t c = 0; c < chunks; ++c) {
        const int64_t b = n * c / chunks, e = n * (c + 1) / chunks;
        pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto& t : pool) t.join();
}

struct NodeGraph {
    std::vector<int64_t> off;   // [n + 1]
    std::vector<int32_t> adj;   // neighbours, self excluded, by ascending kept index
    int64_t degree(int32_t v) const { return off[v + 1] - off[v]; }
    // asks the cache for vertex v's neighbour list ahead of its use: the searches below visit
    // vertices far from memory order, so each list would otherwise cost a DRAM miss
    void prefetch(int32_t v) const {
        const int32_t* a = adj.data() + off[v];
        __builtin_prefetch(a);
        __builtin_prefetch(a + 16);
    }
    void prefetch_offset(int32_t v) const { __builtin_prefetch(off.data() + v); }
};
constexpr int64_t kAhead = 16;
constexpr int kIteratedPasses = 2;  // MULTICOLOR_ITERATED: two passes restore the classes' direction  // vertices ahead of the one being visited (lists; offsets 2x)

// Vertex sets as bit sets: 64 KB for half a million vertices, so the random tests of a
// breadth-first search stay in the core's cache.
struct Bits {
    std::vector<uint64_t> w;
    explicit Bits(int64_t n = 0) : w((size_t)((n + 63) / 64), 0ull) {}
    bool test(int64_t i) const { return (w[(size_t)(i >> 6)] >> (i & 63)) & 1ull; }
    void set(int64_t i) { w[(size_t)(i >> 6)] |= 1ull << (i & 63); }
};

// Breadth-first search from `start` that does not enter `excluded` vertices (bfs_levels,
// solve.rs:248-270), on flat buffers reused across calls: returns the number of levels and keeps
// the last level, in discovery order, in `last`.
struct Bfs {
    std::vector<int32_t> queue, last;
    Bits seen;
    explicit Bfs(int32_t n) : queue(n), seen(n) {}
    int32_t run(const NodeGraph& g, int32_t start, const Bits& excluded) {
        seen = excluded;
        int64_t head = 0, tail = 0;
        queue[tail++] = start;
        seen.set(start);
        int32_t levels = 0;
        int64_t level_begin = 0;
        for (;;) {
            const int64_t level_end = tail;
            ++levels;
            for (head = level_begin; head < level_end; ++head) {
                const int32_t v = queue[head];
                if (head + kAhead < tail) g.prefetch(queue[head + kAhead]);
                if (head + 2 * kAhead < tail) g.prefetch_offset(queue[head + 2 * kAhead]);
                for (int64_t p = g.off[v]; p < g.off[v + 1]; ++p) {
                    const int32_t w = g.adj[p];
                    if (!seen.test(w)) {
                        seen.set(w);
                        queue[tail++] = w;
                    }
                }
            }
            if (tail == level_end) {
                last.assign(queue.begin() + level_begin, queue.begin() + level_end);
                return levels;
            }
            level_begin = level_end;
        }
    }
};

// Reverse Cuthill-McKee with a George-Liu pseudo-peripheral start and neighbours visited by
// increasing degree (stable), one connected component at a time; the algorithm of
// reverse_cuthill_mckee (solve.rs:200-245), applied to the node graph. order[new] = old.
std::vector<int32_t> rcm(const NodeGraph& g) {
    const int32_t n = (int32_t)g.off.size() - 1;
    std::vector<int32_t> deg(n);
    for (int32_t v = 0; v < n; ++v) deg[v] = (int32_t)g.degree(v);
    Bits visited(n);
    std::vector<int32_t> order;
    order.reserve(n);
    Bfs bfs(n);
    std::vector<int32_t> next;
    int32_t scan = 0;
    for (;;) {
        while (scan < n && visited.test(scan)) ++scan;
        int32_t seed = -1;
        for (int32_t v = scan; v < n; ++v)
            if (!visited.test(v) && (seed < 0 || deg[v] < deg[seed])) seed = v;
        if (seed < 0) break;
        int32_t start = seed;
        int32_t depth = bfs.run(g, start, visited);
        for (;;) {
            int32_t far = -1;
            for (int32_t v : bfs.last)
                if (far < 0 || deg[v] < deg[far]) far = v;
            if (far < 0) break;
            const std::vector<int32_t> keep_last = bfs.last;
            const int32_t far_depth = bfs.run(g, far, visited);
            if (far_depth <= depth) {
                bfs.last = keep_last;
                break;
            }
            start = far;
            depth = far_depth;
        }
        size_t head = order.size();
        visited.set(start);
        order.push_back(start);
        while (head < order.size()) {
            if (head + kAhead < order.size()) g.prefetch(order[head + kAhead]);
            if (head + 2 * kAhead < order.size()) g.prefetch_offset(order[head + 2 * kAhead]);
            const int32_t v = order[head++];
            next.clear();
            for (int64_t p = g.off[v]; p < g.off[v + 1]; ++p)
                if (!visited.test(g.adj[p])) next.push_back(g.adj[p]);
            // stable insertion sort by degree (neighbour lists are short)
            for (size_t i = 1; i < next.size(); ++i) {
                const int32_t x = next[i];
                const int32_t dx = deg[x];
                size_t j = i;
                while (j > 0 && deg[next[j - 1]] > dx) {
                    next[j] = next[j - 1];
                    --j;
                }
                next[j] = x;
            }
            for (int32_t w : next)
                if (!visited.test(w)) {
                    visited.set(w);
                    order.push_back(w);
                }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// The visit order of the MULTICOLOR_BFS ordering's greedy colouring: a breadth-first search from
// a minimum-degree vertex (the first minimum by index), neighbours in adjacency order, one
// connected component at a time, reversed. Measured with the oracle's IC(0)-PCG on the
// lognormal Tet10 cube (10^3, 16^3, 24^3 cells): one colour fewer than colouring in RCM order
// (16-17 against 18) and 7 % fewer FP64 iterations, for one breadth-first pass instead of RCM's
// pseudo-peripheral searches and degree sorts. On Tet10 40^3 on the GPU: plain FP64 8 % fewer
// iterations, the thermal step 12 % fewer, but the mixed form 5 % more (its FP32 Krylov space
// converges differently), so the elastic solves keep MULTICOLOR.
std::vector<int32_t> reverse_bfs(const NodeGraph& g) {
    const int32_t n = (int32_t)g.off.size() - 1;
    std::vector<int32_t> order;
    order.reserve(n);
    Bits visited(n);
    int32_t scan = 0;
    for (;;) {
        while (scan < n && visited.test(scan)) ++scan;
        if (scan >= n) break;
        int32_t seed = scan;
        for (int32_t v = scan + 1; v < n; ++v)
            if (!visited.test(v) && g.degree(v) < g.degree(seed)) seed = v;
        visited.set(seed);
        size_t head = order.size();
        order.push_back(seed);
        while (head < order.size()) {
            if (head + kAhead < order.size()) g.prefetch(order[head + kAhead]);
            if (head + 2 * kAhead < order.size()) g.prefetch_offset(order[head + 2 * kAhead]);
            const int32_t v = order[head++];
            for (int64_t p = g.off[v]; p < g.off[v + 1]; ++p) {
                const int32_t w = g.adj[p];
                if (!visited.test(w)) {
                    visited.set(w);
                    order.push_back(w);
                }
            }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// Greedy colouring visiting vertices in `visit` order (smallest colour no visited neighbour
// holds); returns colours. A colour never exceeds the vertex degree, so while every degree is
// below 255 the colours are kept in bytes, which keeps the neighbour lookups in cache.
template <typename C>
void greedy_colour_into(const NodeGraph& g, const std::vector<int32_t>& visit, std::vector<int32_t>& out) {
    const int32_t n = (int32_t)visit.size();
    const C none = (C)~(C)0;
    std::vector<C> colour(n, none);
    std::vector<int32_t> stamp;  // stamp[c] == v: colour c used by a neighbour of v
    for (int32_t i = 0; i < n; ++i) {
        const int32_t v = visit[i];
        if (i + kAhead < n) g.prefetch(visit[i + kAhead]);
        if (i + 2 * kAhead < n) g.prefetch_offset(visit[i + 2 * kAhead]);
        for (int64_t p = g.off[v]; p < g.off[v + 1]; ++p) {
            const C c = colour[g.adj[p]];
            if (c != none) {
                if ((size_t)c >= stamp.size()) stamp.resize((size_t)c + 1, -1);
                stamp[c] = v;
            }
        }
        int32_t c = 0;
        while ((size_t)c < stamp.size() && stamp[c] == v) ++c;
        colour[v] = (C)c;
    }
    out.resize(n);
    for (int32_t v = 0; v < n; ++v) out[v] = (int32_t)colour[v];
}
std::vector<int32_t> greedy_colour(const NodeGraph& g, const std::vector<int32_t>& visit) {
    int64_t maxdeg = 0;
    for (size_t v = 0; v + 1 < g.off.size(); ++v) maxdeg = std::max<int64_t>(maxdeg, g.degree((int32_t)v));
    std::vector<int32_t> colour;
    if (maxdeg < 255) greedy_colour_into<uint8_t>(g, visit, colour);
    else greedy_colour_into<int32_t>(g, visit, colour);
    return colour;
}

// Iterated greedy (Culberson): recolours every node greedily, visiting the colour classes from
// the last to the first and, inside a class, in the order of `order`; a pass never adds a colour
// (the first node of each class finds every colour of the classes visited before it free or
// takes at most the class count). Returns the colours after `passes` passes.
std::vector<int32_t> iterated_greedy(const NodeGraph& g, const std::vector<int32_t>& order,
                                     std::vector<int32_t> colour, int passes) {
    const int32_t n = (int32_t)order.size();
    std::vector<int32_t> pos(n);
    for (int32_t i = 0; i < n; ++i) pos[order[i]] = i;
    std::vector<int32_t> visit(n);
    for (int k = 0; k < passes; ++k) {
        std::iota(visit.begin(), visit.end(), 0);
        std::sort(visit.begin(), visit.end(), [&](int32_t a, int32_t b) {
            return colour[a] != colour[b] ? colour[a] > colour[b] : pos[a] < pos[b];
        });
        colour = greedy_colour(g, visit);
    }
    return colour;
}

// elements touching a fixed DOF, and the nodes with a fixed DOF they contain
void boundary(Symbolic& s, int64_t n_nodes, int npe, int64_t n_elems, const int64_t* conn,
              const uint8_t* fixed) {
    if (!fixed) return;
    std::vector<uint8_t> bn(n_nodes, 0);
    for (int64_t e = 0; e < n_elems; ++e) {
        bool any = false;
        for (int a = 0; a < npe && !any; ++a) {
            const int64_t v = conn[e * npe + a];
            any = fixed[3 * v] || fixed[3 * v + 1] || fixed[3 * v + 2];
        }
        if (any) {
            s.belem.push_back((int32_t)e);
            for (int a = 0; a < npe; ++a) bn[conn[e * npe + a]] = 1;
        }
    }
    for (int64_t v = 0; v < n_nodes; ++v)
        if (bn[v]) s.bnodes.push_back((int32_t)v);
}

}  // namespace

bool analyse_topology(int64_t n_nodes, int npe, int64_t n_elems, const int64_t* conn, const uint8_t* fixed,
                      Symbolic& s, std::vector<int32_t>& kept, std::vector<int32_t>& kept_of, Error& err,
                      bool boundary_lists, bool incidence) {
    if (npe != 4 && npe != 10) {
        err = {MAILLE_INVALID_INPUT, "nodes_per_elem must be 4 or 10"};
        return false;
    }
    if (n_nodes <= 0 || n_elems <= 0) {
        err = {MAILLE_INVALID_INPUT, "empty mesh"};
        return false;
    }
    if (n_nodes >= (int64_t(1) << 30) || n_elems * node_pairs(npe) >= (int64_t(1) << 31)) {
        err = {MAILLE_INVALID_INPUT, "mesh too large for 32-bit element-pair indices"};
        return false;
    }
    for (int64_t k = 0; k < n_elems * npe; ++k)
        if (conn[k] < 0 || conn[k] >= n_nodes) {
            err = {MAILLE_INVALID_INPUT, "element " + std::to_string(k / npe) +
                                             " refers to unknown node " + std::to_string(conn[k])};
            return false;
        }
    s = Symbolic{};
    s.n_nodes = n_nodes;
    s.n_elems = n_elems;
    s.npe = npe;
    const int32_t N = (int32_t)n_nodes;
    // node -> (element, local) incidence, sorted by element (the run starts always: the solve
    // looks up the nodes no element touches there)
    s.inc_ptr.assign(N + 1, 0);
    for (int64_t k = 0; k < n_elems * npe; ++k) s.inc_ptr[conn[k] + 1]++;
    for (int32_t v = 0; v < N; ++v) s.inc_ptr[v + 1] += s.inc_ptr[v];
    if (incidence) {
        s.inc.resize(n_elems * npe);
        std::vector<int64_t> cur(s.inc_ptr.begin(), s.inc_ptr.end() - 1);
        for (int64_t k = 0; k < n_elems * npe; ++k) s.inc[cur[conn[k]]++] = (int32_t)k;
    }
    // kept nodes (at least one free DOF) in original order
    kept_of.assign(N, -1);
    kept.clear();
    for (int32_t v = 0; v < N; ++v) {
        const bool all = fixed && fixed[3 * v] && fixed[3 * v + 1] && fixed[3 * v + 2];
        if (!all) {
            kept_of[v] = (int32_t)kept.size();
            kept.push_back(v);
        }
    }
    for (int64_t g = 0; g < 3 * n_nodes; ++g) s.free_dofs += (fixed && fixed[g]) ? 0 : 1;
    if (kept.empty()) {
        err = {MAILLE_INVALID_INPUT, "every DOF is fixed"};
        return false;
    }
    if (boundary_lists) boundary(s, n_nodes, npe, n_elems, conn, fixed);
    return true;
}

void apply_ordering(const std::vector<int32_t>& kept, const std::vector<int32_t>& order,
                    const std::vector<int32_t>& level, const uint8_t* fixed, Symbolic& s) {
    const int32_t nk = (int32_t)kept.size();
    int32_t nl = 0;
    for (int32_t k = 0; k < nk; ++k) nl = std::max(nl, level[k] + 1);
    s.levels = nl;
    s.level_ptr.assign(s.levels + 1, 0);
    for (int32_t k = 0; k < nk; ++k) s.level_ptr[level[k] + 1]++;
    for (int32_t l = 0; l < s.levels; ++l) s.level_ptr[l + 1] += s.level_ptr[l];
    s.nb = nk;
    s.perm.resize(nk);
    s.inv.assign(s.n_nodes, -1);
    s.fixmask.assign(nk, 0);
    for (int32_t r = 0; r < nk; ++r) {
        const int32_t v = kept[order[r]];
        s.perm[r] = v;
        s.inv[v] = r;
        uint8_t m = 0;
        for (int c = 0; c < 3; ++c)
            if (fixed && fixed[3 * v + c]) m |= (uint8_t)(1u << c);
        s.fixmask[r] = m;
    }
}

bool analyse(int64_t n_nodes, int npe, int64_t n_elems, const int64_t* conn,
             const uint8_t* fixed, int ordering, Symbolic& s, Error& err, bool pattern, bool boundary_lists) {
    const double t0 = now_ms();
    const bool stage_timing = std::getenv("MAILLE_SETUP_TIMING") != nullptr;
    double t_stage = now_ms();
    auto stage = [&](const char* name) {
        if (!stage_timing) return;
        const double t = now_ms();
        std::fprintf(stderr, "maille setup %-12s %8.1f ms\n", name, t - t_stage);
        t_stage = t;
    };
    std::vector<int32_t> kept_of, kept;
    if (!analyse_topology(n_nodes, npe, n_elems, conn, fixed, s, kept, kept_of, err, boundary_lists && !pattern))
        return false;
    stage("topology");
    const int32_t nk = (int32_t)kept.size();
    NodeGraph g;
    g.off.assign(nk + 1, 0);
    {
        // neighbours of each kept node by ascending kept index (the order the device analysis
        // produces by sorting keys): a counting pass, then a filling pass that sorts each list;
        // duplicates are dropped with a per-thread mark array
        auto visit = [&](int32_t k, std::vector<int32_t>& mark, auto&& fn) {
            const int32_t v = kept[k];
            mark[k] = k;
            for (int64_t q = s.inc_ptr[v]; q < s.inc_ptr[v + 1]; ++q) {
                const int64_t e = s.inc[q] / npe;
                for (int a = 0; a < npe; ++a) {
                    const int32_t w = kept_of[conn[e * npe + a]];
                    if (w >= 0 && mark[w] != k) {
                        mark[w] = k;
                        fn(w);
                    }
                }
            }
        };
        parallel_for(nk, [&](int64_t k0, int64_t k1) {
            std::vector<int32_t> mark(nk, -1);
            for (int64_t k = k0; k < k1; ++k) {
                int64_t c = 0;
                visit((int32_t)k, mark, [&](int32_t) { ++c; });
                g.off[k + 1] = c;
            }
        });
        for (int32_t k = 0; k < nk; ++k) g.off[k + 1] += g.off[k];
        g.adj.resize(g.off[nk]);
        parallel_for(nk, [&](int64_t k0, int64_t k1) {
            std::vector<int32_t> mark(nk, -1);
            for (int64_t k = k0; k < k1; ++k) {
                int64_t q = g.off[k];
                visit((int32_t)k, mark, [&](int32_t w) { g.adj[q++] = w; });
                std::sort(g.adj.begin() + g.off[k], g.adj.begin() + g.off[k + 1]);
            }
        });
    }

    stage("graph");
    // ordering over kept nodes: order[new] = kept index
    std::vector<int32_t> order = ordering == MAILLE_ORDER_MULTICOLOR_BFS ? reverse_bfs(g) : rcm(g);
    std::vector<int32_t> level;
    if (ordering != MAILLE_ORDER_RCM) {
        level = greedy_colour(g, order);
        if (ordering == MAILLE_ORDER_MULTICOLOR_ITERATED) level = iterated_greedy(g, order, level, kIteratedPasses);
        // rows by colour, visit order inside a colour (a stable counting sort). A row's lower
        // neighbours are exactly its neighbours of smaller colours, and greedy colouring gives a
        // node colour c only when its earlier-visited neighbours hold every colour below c, so the
        // level of each row is its colour.
        int32_t nc = 0;
        for (int32_t k = 0; k < nk; ++k) nc = std::max(nc, level[k] + 1);
        std::vector<int64_t> pos((size_t)nc + 1, 0);
        for (int32_t k = 0; k < nk; ++k) pos[level[k] + 1]++;
        for (int32_t c = 0; c < nc; ++c) pos[c + 1] += pos[c];
        std::vector<int32_t> by_colour(nk);
        for (int32_t v : order) by_colour[pos[level[v]]++] = v;
        order.swap(by_colour);
    } else {
        // levels of the lower-triangular dependency graph in that order, then group rows by
        // level (a topological renumbering leaves the IC(0) factor unchanged)
        std::vector<int32_t> rank(nk);
        level.assign(nk, 0);
        for (int32_t r = 0; r < nk; ++r) rank[order[r]] = r;
        for (int32_t r = 0; r < nk; ++r) {
            const int32_t k = order[r];
            int32_t l = 0;
            for (int64_t p = g.off[k]; p < g.off[k + 1]; ++p)
                if (rank[g.adj[p]] < r) l = std::max(l, level[g.adj[p]] + 1);
            level[k] = l;
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t a, int32_t b) { return level[a] < level[b]; });
    }
    stage("ordering");
    apply_ordering(kept, order, level, fixed, s);
    stage("levels");
    if (!pattern) {
        s.ms = now_ms() - t0;
        return true;
    }
    // full block pattern in new numbering (neighbours + the diagonal), columns ascending
    s.row_ptr.assign(nk + 1, 0);
    for (int32_t r = 0; r < nk; ++r) {
        const int32_t k = kept_of[s.perm[r]];
        s.row_ptr[r + 1] = s.row_ptr[r] + (g.off[k + 1] - g.off[k]) + 1;
    }
    s.blocks = s.row_ptr[nk];
    if (s.blocks >= (int64_t(1) << 31)) {
        err = {MAILLE_INVALID_INPUT, "pattern too large for 32-bit block positions"};
        return false;
    }
    s.col.resize(s.blocks);
    s.diag.resize(nk);
    parallel_for(nk, [&](int64_t r0, int64_t r1) {
        for (int64_t r = r0; r < r1; ++r) {
            const int32_t k = kept_of[s.perm[r]];
            int64_t p = s.row_ptr[r];
            s.col[p++] = (int32_t)r;
            for (int64_t q = g.off[k]; q < g.off[k + 1]; ++q) s.col[p++] = s.inv[kept[g.adj[q]]];
            std::sort(s.col.begin() + s.row_ptr[r], s.col.begin() + s.row_ptr[r + 1]);
            s.diag[r] = std::lower_bound(s.col.begin() + s.row_ptr[r],
                                         s.col.begin() + s.row_ptr[r + 1], (int32_t)r) -
                        s.col.begin();
        }
    });
    g = NodeGraph{};
    auto find = [&](int32_t i, int32_t j) -> int64_t {
        auto b = s.col.begin() + s.row_ptr[i], e = s.col.begin() + s.row_ptr[i + 1];
        auto it = std::lower_bound(b, e, j);
        return (it != e && *it == j) ? (int64_t)(it - s.col.begin()) : -1;
    };
    stage("pattern");
    s.tpos.resize(s.blocks);
    parallel_for(nk, [&](int64_t r0, int64_t r1) {
        for (int64_t r = r0; r < r1; ++r)
            for (int64_t p = s.row_ptr[r]; p < s.row_ptr[r + 1]; ++p)
                s.tpos[p] = find(s.col[p], (int32_t)r);
    });

    stage("transpose");
    // lower slots (row by row, columns ascending) and the scatter map: for lower slot (I, J) the
    // element node pairs that couple I and J, in element order. Built row by row from the
    // node's incident elements (ascending), with a per-thread column -> slot map.
    const int64_t nl0 = 0;
    (void)nl0;
    std::vector<int64_t> lfirst(nk + 1, 0);
    for (int32_t r = 0; r < nk; ++r) lfirst[r + 1] = lfirst[r] + (s.diag[r] - s.row_ptr[r] + 1);
    const int64_t nl = lfirst[nk];
    s.lslot.resize(nl);
    for (int32_t r = 0; r < nk; ++r)
        for (int64_t p = s.row_ptr[r]; p <= s.diag[r]; ++p) s.lslot[lfirst[r] + (p - s.row_ptr[r])] = p;
    const int np = node_pairs(npe);
    auto pair_index = [npe](int a, int b) { return a * npe - a * (a - 1) / 2 + (b - a); };
    // visit(r, fn): fn(local slot, contribution) for every contribution of row r, element order
    auto visit_row = [&](int32_t r, std::vector<int32_t>& slotmap, auto&& fn) {
        for (int64_t p = s.row_ptr[r]; p <= s.diag[r]; ++p) slotmap[s.col[p]] = (int32_t)(p - s.row_ptr[r]);
        const int32_t v = s.perm[r];
        for (int64_t q = s.inc_ptr[v]; q < s.inc_ptr[v + 1]; ++q) {
            const int64_t e = s.inc[q] / npe;
            const int a = (int)(s.inc[q] - e * npe);
            for (int b = 0; b < npe; ++b) {
                const int32_t J = s.inv[conn[e * npe + b]];
                if (J < 0 || J > r) continue;
                const uint32_t k = (uint32_t)(e * np + (a <= b ? pair_index(a, b) : pair_index(b, a)));
                fn(slotmap[J], k | (a <= b ? 0u : 0x80000000u));
            }
        }
    };
    s.lptr.assign(nl + 1, 0);
    parallel_for(nk, [&](int64_t r0, int64_t r1) {
        std::vector<int32_t> slotmap(nk, -1);
        for (int64_t r = r0; r < r1; ++r)
            visit_row((int32_t)r, slotmap, [&](int32_t ls, uint32_t) { s.lptr[lfirst[r] + ls + 1]++; });
    });
    for (int64_t l = 0; l < nl; ++l) s.lptr[l + 1] += s.lptr[l];
    s.contrib.resize(s.lptr[nl]);
    parallel_for(nk, [&](int64_t r0, int64_t r1) {
        std::vector<int32_t> slotmap(nk, -1);
        std::vector<int64_t> cur;
        for (int64_t r = r0; r < r1; ++r) {
            cur.assign(s.lptr.begin() + lfirst[r], s.lptr.begin() + lfirst[r + 1]);
            visit_row((int32_t)r, slotmap, [&](int32_t ls, uint32_t c) { s.contrib[cur[ls]++] = c; });
        }
    });
    s.nl = nl;

    stage("scatter map");
    if (boundary_lists) boundary(s, n_nodes, npe, n_elems, conn, fixed);
    stage("boundary");
    s.ms = now_ms() - t0;
    return true;
}

void build_sell(const Symbolic& s, SellKind kind, int lpr, SellHost& out) {
    out = SellHost{};
    auto start = [&](int32_t i) { return kind == SELL_UPPER ? s.diag[i] + 1 : s.row_ptr[i]; };
    auto end = [&](int32_t i) { return kind == SELL_LOWER ? s.diag[i] : s.row_ptr[i + 1]; };
    if (lpr <= 0) {
        const double total = kind == SELL_FULL ? (double)s.blocks : (double)(s.blocks - s.nb) / 2.0;
        const double mean = total / std::max<int32_t>(1, s.nb);
        // K: one lane per row unless rows are very long (least padding; the SpMV has slices to
        // spare); L and U: about one step per row, which puts more and shorter slices in flight
        // for the dataflow sweeps (measured on Tet10 40^3: K 1 / L,U 4 lanes per row is best)
        lpr = 1;
        const double per_lane = kind == SELL_FULL ? 32.0 : 4.0;
        while (lpr < 4 && mean / lpr > per_lane) lpr *= 2;
    }
    out.lpr = lpr;
    const int S = 32 / lpr, per_step = 4 * lpr;
    out.level_slices.push_back(0);
    std::vector<int32_t> rows;
    std::vector<int64_t> count;
    for (int32_t l = 0; l < s.levels; ++l) {
        // the level's rows by decreasing length, stable (a counting sort: lengths are small)
        int64_t maxlen = 0;
        for (int32_t i = s.level_ptr[l]; i < s.level_ptr[l + 1]; ++i) maxlen = std::max<int64_t>(maxlen, end(i) - start(i));
        count.assign((size_t)maxlen + 2, 0);
        for (int32_t i = s.level_ptr[l]; i < s.level_ptr[l + 1]; ++i) count[(size_t)(maxlen - (end(i) - start(i))) + 1]++;
        for (size_t k = 1; k < count.size(); ++k) count[k] += count[k - 1];
        rows.resize((size_t)(s.level_ptr[l + 1] - s.level_ptr[l]));
        for (int32_t i = s.level_ptr[l]; i < s.level_ptr[l + 1]; ++i) rows[count[(size_t)(maxlen - (end(i) - start(i)))]++] = i;
        for (size_t c0 = 0; c0 < rows.size(); c0 += S) {
            const size_t c1 = std::min(rows.size(), c0 + S);
            int64_t maxlen = 0;
            for (size_t k = c0; k < c1; ++k) maxlen = std::max<int64_t>(maxlen, end(rows[k]) - start(rows[k]));
            const int64_t steps = (maxlen + per_step - 1) / per_step;
            out.off.push_back(out.off.back() + steps);
            for (int r = 0; r < S; ++r) out.rowid.push_back(c0 + r < c1 ? rows[c0 + r] : -1);
        }
        out.level_slices.push_back(out.nslices());
    }
}

void build_psell(const Symbolic& s, SellKind kind, PsellHost& out) {
    out = PsellHost{};
    constexpr int64_t kSlots = 128;
    auto start = [&](int32_t i) { return kind == SELL_UPPER ? s.diag[i] + 1 : s.row_ptr[i]; };
    auto end = [&](int32_t i) { return kind == SELL_LOWER ? s.diag[i] : s.row_ptr[i + 1]; };
    out.level_slices.push_back(0);
    out.rows.reserve(s.nb);
    std::vector<int32_t> open;  // rows of the slice being packed
    int64_t used = 0;
    auto close = [&]() {
        if (open.empty()) return;
        const int64_t g0 = out.off.back();
        const int64_t len0 = end(open[0]) - start(open[0]);
        const int64_t steps = open.size() == 1 && len0 > kSlots ? (len0 + kSlots - 1) / kSlots : 1;
        out.off.push_back(g0 + steps);
        uint32_t head[4] = {0, 0, 0, 0};
        int64_t slot = 0;
        for (int32_t i : open) {
            head[slot >> 5] |= 1u << (slot & 31);
            out.rows.push_back(i);
            out.rstart.push_back(g0 * kSlots + slot);
            slot += std::max<int64_t>(1, end(i) - start(i));
        }
        for (uint32_t w : head) out.head.push_back(w);
        out.row0.push_back((int32_t)out.rows.size());
        open.clear();
        used = 0;
    };
    // L is swept levels ascending, U levels descending: slices are stored in sweep order
    for (int32_t q = 0; q < s.levels; ++q) {
        const int32_t l = kind == SELL_UPPER ? s.levels - 1 - q : q;
        for (int32_t i = s.level_ptr[l]; i < s.level_ptr[l + 1]; ++i) {
            const int64_t need = std::max<int64_t>(1, end(i) - start(i));
            if (used + need > kSlots || open.size() == 32) close();
            open.push_back(i);
            used += need;
            if (used >= kSlots) close();
        }
        close();
        out.level_slices.push_back(out.nslices());
    }
}

void build_bsell(const Symbolic& s, SellKind kind, int rows, int sub, const std::vector<int32_t>& group,
                 BSellHost& out) {
    out = BSellHost{};
    out.rows = rows;
    out.sub = sub;
    const int slots = out.slots(), per_step = 4 * sub;
    auto start = [&](int32_t i) { return kind == SELL_UPPER ? s.diag[i] + 1 : s.row_ptr[i]; };
    auto end = [&](int32_t i) { return kind == SELL_LOWER ? s.diag[i] : s.row_ptr[i + 1]; };
    auto emit = [&](std::vector<int32_t>& rs) {
        // rows of one group: by decreasing length, `rows` per slice
        std::stable_sort(rs.begin(), rs.end(), [&](int32_t a, int32_t b) {
            return end(a) - start(a) > end(b) - start(b);
        });
        for (size_t c0 = 0; c0 < rs.size(); c0 += rows) {
            const size_t c1 = std::min(rs.size(), c0 + rows);
            int64_t maxlen = 0;
            for (size_t k = c0; k < c1; ++k) maxlen = std::max<int64_t>(maxlen, end(rs[k]) - start(rs[k]));
            const int64_t steps = (maxlen + per_step - 1) / per_step;
            const int64_t g0 = out.off.back();
            out.off.push_back(g0 + steps);
            out.inst.push_back(group[rs[c0]]);
            out.col.resize((size_t)(g0 + steps) * slots, s.nb);
            out.src.resize((size_t)(g0 + steps) * slots, -1);
            for (int r = 0; r < rows; ++r) out.rowid.push_back(c0 + r < c1 ? rs[c0 + r] : -1);
            for (size_t k = c0; k < c1; ++k) {
                const int32_t i = rs[k];
                const int r = (int)(k - c0);
                for (int64_t p = start(i), b = 0; p < end(i); ++p, ++b) {
                    const int64_t t = b / per_step, rem = b % per_step;
                    const size_t slot = (size_t)(g0 + t) * slots + 4 * (r * sub + rem / 4) + rem % 4;
                    out.col[slot] = s.col[p];
                    out.src[slot] = (int32_t)p;
                }
            }
        }
    };
    // rows bucketed by group, keeping row order inside a group
    const int32_t ngroups = group.empty() ? 0 : *std::max_element(group.begin(), group.end()) + 1;
    std::vector<std::vector<int32_t>> bucket(ngroups);
    if (kind == SELL_FULL) {
        for (int32_t i = 0; i < s.nb; ++i) bucket[group[i]].push_back(i);
        for (auto& b : bucket) emit(b);
        return;
    }
    out.level_slices.push_back(0);
    for (int32_t l = 0; l < s.levels; ++l) {
        for (auto& b : bucket) b.clear();
        for (int32_t i = s.level_ptr[l]; i < s.level_ptr[l + 1]; ++i) bucket[group[i]].push_back(i);
        for (auto& b : bucket)
            if (!b.empty()) emit(b);
        out.level_slices.push_back(out.nslices());
    }
}

// face_pressure for the tet faces (assembly.rs:650-674; face_rule tet branch 556-585; face nodes
// from Element::face_positions, mesh.rs:184-198; TRIANGLE_3 / TRIANGLE_6 rules).
bool face_pressure_loads(int64_t n_nodes, const double* coords, int npe, int64_t n_elems,
                         const int64_t* conn, int64_t n_press, const int64_t* p_elem,
                         const int32_t* p_face, const double* p_value, double* f, Error& err) {
    static const int faces[4][3] = {{0, 1, 2}, {0, 3, 1}, {1, 3, 2}, {2, 3, 0}};
    static const int edges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    static const double t3[3][3] = {{1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
                                    {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                                    {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
    const double A = 0.445948490915965, WA = 0.223381589678011 / 2.0;
    const double B = 0.091576213509771, WB = 0.109951743655322 / 2.0;
    const double t6[6][3] = {{A, A, WA}, {1.0 - 2.0 * A, A, WA}, {A, 1.0 - 2.0 * A, WA},
                             {B, B, WB}, {1.0 - 2.0 * B, B, WB}, {B, 1.0 - 2.0 * B, WB}};
    if (npe != 4 && npe != 10) {
        err = {MAILLE_INVALID_INPUT, "nodes_per_elem must be 4 or 10"};
        return false;
    }
    for (int64_t k = 0; k < n_press; ++k) {
        const int64_t e = p_elem[k];
        const int face = p_face[k];
        if (e < 0 || e >= n_elems || face < 0 || face > 3) continue;  // face_rule gives None
        int pos[6];
        const int nn = npe == 4 ? 3 : 6;
        for (int q = 0; q < 3; ++q) pos[q] = faces[face][q];
        if (npe == 10) {
            auto mid = [&](int a, int b) {
                for (int q = 0; q < 6; ++q)
                    if ((edges[q][0] == a && edges[q][1] == b) || (edges[q][0] == b && edges[q][1] == a))
                        return 4 + q;
                return 4;
            };
            pos[3] = mid(pos[0], pos[1]);
            pos[4] = mid(pos[1], pos[2]);
            pos[5] = mid(pos[2], pos[0]);
        }
        double c[6][3], corner[4][3];
        for (int q = 0; q < nn; ++q) {
            const int64_t v = conn[e * npe + pos[q]];
            if (v < 0 || v >= n_nodes) {
                err = {MAILLE_INVALID_INPUT, "pressure face refers to an unknown node"};
                return false;
            }
            for (int d = 0; d < 3; ++d) c[q][d] = coords[3 * v + d];
        }
        for (int q = 0; q < 4; ++q)
            for (int d = 0; d < 3; ++d) corner[q][d] = coords[3 * conn[e * npe + q] + d];
        double u[3], w[3];
        for (int d = 0; d < 3; ++d) {
            u[d] = c[1][d] - c[0][d];
            w[d] = c[2][d] - c[0][d];
        }
        const double cross[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2],
                                 u[0] * w[1] - u[1] * w[0]};
        const double twice_area =
            std::sqrt(cross[0] * cross[0] + cross[1] * cross[1] + cross[2] * cross[2]);
        double dot = 0.0;
        for (int d = 0; d < 3; ++d) {
            const double out = (c[0][d] + c[1][d] + c[2][d]) / 3.0 -
                               (corner[0][d] + corner[1][d] + corner[2][d] + corner[3][d]) / 4.0;
            dot += cross[d] * out;
        }
        const double sign = dot < 0.0 ? -1.0 : 1.0;
        double normal[3];
        for (int d = 0; d < 3; ++d) normal[d] = sign * cross[d] / twice_area;
        const int ng = nn == 3 ? 3 : 6;
        double forces[18] = {0};
        for (int gp = 0; gp < ng; ++gp) {
            const double xi = nn == 3 ? t3[gp][0] : t6[gp][0];
            const double eta = nn == 3 ? t3[gp][1] : t6[gp][1];
            const double wt = (nn == 3 ? t3[gp][2] : t6[gp][2]) * twice_area;
            double nv[6];
            const double l1 = 1.0 - xi - eta, l2 = xi, l3 = eta;
            if (nn == 3) {
                nv[0] = l1;
                nv[1] = l2;
                nv[2] = l3;
            } else {
                nv[0] = l1 * (2.0 * l1 - 1.0);
                nv[1] = l2 * (2.0 * l2 - 1.0);
                nv[2] = l3 * (2.0 * l3 - 1.0);
                nv[3] = 4.0 * l1 * l2;
                nv[4] = 4.0 * l2 * l3;
                nv[5] = 4.0 * l3 * l1;
            }
            for (int a = 0; a < nn; ++a)
                for (int d = 0; d < 3; ++d) forces[3 * a + d] -= p_value[k] * wt * nv[a] * normal[d];
        }
        for (int a = 0; a < nn; ++a)
            for (int d = 0; d < 3; ++d) f[3 * conn[e * npe + pos[a]] + d] += forces[3 * a + d];
    }
    return true;
}

}  // namespace maille
