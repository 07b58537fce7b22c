// Graph colourings of the vertex graph (VBD) and of the element dual graph (XPBD).
//
// The reference keeps each adjacency list as a std::multiset (octopus/include/Tools/Graph.h:
// 36-54, 56-85), so a neighbour shared through k elements appears k times and counts k
// times in the degree.  Here the adjacency is a CSR of unique neighbours with their
// multiplicity, which reproduces every quantity the colourings read (degree, per-occurrence
// counts) in a fraction of the memory; colours come out identical.
//   DSAT            Graph.h:321-371, priority (saturation, degree, vertex) largest first
//                   (:884-904); a neighbour's degree drops once per occurrence.
//   Greedy          Graph.h:200-207 with find_color_greedy :906-926.
//   Greedy_SLF      Graph.h:237-277 (smallest-last order, then greedy).
//   ColorReduction  Graph.h:941-969.
#include <algorithm>
#include <functional>
#include <queue>

#include "host.hpp"

namespace octb {

namespace {

// Builds the CSR from, for each row, the list of (possibly repeated) neighbours produced by
// `emit(row, push)`.  Two passes keep the peak memory at the size of the unique lists.
template <class Emit>
void build_csr(int n, Emit emit, PrimalGraph& g) {
    g.n = n;
    g.off.assign((size_t)n + 1, 0);
    g.degree.assign(n, 0);
    std::vector<int32_t> buf;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            for (int i = 0; i < n; ++i) g.off[i + 1] += g.off[i];
            g.nbr.resize(g.off[n]);
            g.mult.resize(g.off[n]);
        }
        for (int i = 0; i < n; ++i) {
            buf.clear();
            emit(i, buf);
            std::sort(buf.begin(), buf.end());
            int64_t w = pass == 1 ? g.off[i] : 0, uniq = 0;
            for (size_t k = 0; k < buf.size();) {
                size_t j = k;
                while (j < buf.size() && buf[j] == buf[k]) ++j;
                if (pass == 1) { g.nbr[w] = buf[k]; g.mult[w] = (int32_t)(j - k); ++w; }
                ++uniq;
                k = j;
            }
            if (pass == 0) { g.off[i + 1] = uniq; g.degree[i] = (int64_t)buf.size(); }
        }
    }
}

}  // namespace

void build_primal_graph(int ne, const int32_t* topo, int n_elem, int n_nodes, PrimalGraph& g) {
    // owners of each vertex, then each vertex's neighbours are the other nodes of its owners
    std::vector<int64_t> ooff((size_t)n_nodes + 1, 0);
    for (int64_t k = 0; k < (int64_t)n_elem * ne; ++k) ooff[topo[k] + 1]++;
    for (int i = 0; i < n_nodes; ++i) ooff[i + 1] += ooff[i];
    std::vector<int32_t> own(ooff[n_nodes]);
    std::vector<int64_t> fill(ooff.begin(), ooff.end() - 1);
    for (int e = 0; e < n_elem; ++e)
        for (int j = 0; j < ne; ++j) own[fill[topo[(int64_t)e * ne + j]]++] = e;
    build_csr(n_nodes, [&](int v, std::vector<int32_t>& out) {
        for (int64_t k = ooff[v]; k < ooff[v + 1]; ++k) {
            const int32_t* t = topo + (int64_t)own[k] * ne;
            for (int j = 0; j < ne; ++j) if (t[j] != v) out.push_back(t[j]);
            // an element lists v once, so every other node of it is one occurrence
        }
    }, g);
}

void build_dual_vertex_graph(int ne, const int32_t* topo, int n_elem, int n_nodes, PrimalGraph& g) {
    std::vector<int64_t> ooff((size_t)n_nodes + 1, 0);
    for (int64_t k = 0; k < (int64_t)n_elem * ne; ++k) ooff[topo[k] + 1]++;
    for (int i = 0; i < n_nodes; ++i) ooff[i + 1] += ooff[i];
    std::vector<int32_t> own(ooff[n_nodes]);
    std::vector<int64_t> fill(ooff.begin(), ooff.end() - 1);
    for (int e = 0; e < n_elem; ++e)
        for (int j = 0; j < ne; ++j) own[fill[topo[(int64_t)e * ne + j]]++] = e;
    build_csr(n_elem, [&](int e, std::vector<int32_t>& out) {
        const int32_t* t = topo + (int64_t)e * ne;
        for (int j = 0; j < ne; ++j)
            for (int64_t k = ooff[t[j]]; k < ooff[t[j] + 1]; ++k)
                if (own[k] != e) out.push_back(own[k]);
    }, g);
}

Coloring color_dsat(const PrimalGraph& g) {
    // key = (saturation, degree, vertex): the largest key is coloured next.  A max-heap with
    // lazy deletion: every update pushes the vertex's new key; a popped key that no longer
    // equals the vertex's current key (or belongs to a coloured vertex) is stale and skipped.
    auto key = [](int64_t sat, int64_t deg, int64_t v) {
        return ((uint64_t)sat << 51) | ((uint64_t)deg << 27) | (uint64_t)v;
    };
    Coloring c;
    c.colors.assign(g.n, -1);
    std::vector<int64_t> degree(g.degree);
    std::vector<std::vector<int32_t>> adjcols(g.n);
    std::vector<uint64_t> cur(g.n);
    std::vector<uint64_t> heap;
    heap.reserve((size_t)g.n * 4);
    for (int v = 0; v < g.n; ++v) { cur[v] = key(0, degree[v], v); heap.push_back(cur[v]); }
    std::make_heap(heap.begin(), heap.end());
    std::vector<char> used;
    int max_color = -1, remaining = g.n;
    while (remaining > 0) {
        std::pop_heap(heap.begin(), heap.end());
        const uint64_t top = heap.back();
        heap.pop_back();
        const int vid = (int)(top & ((1ull << 27) - 1));
        if (c.colors[vid] != -1 || cur[vid] != top) continue;
        --remaining;
        used.assign(max_color + 2, 0);
        for (int64_t k = g.off[vid]; k < g.off[vid + 1]; ++k) {
            const int col = c.colors[g.nbr[k]];
            if (col >= 0) used[col] = 1;
        }
        int i = 0;
        while (used[i]) ++i;   // used[max_color + 1] is always 0
        max_color = std::max(max_color, i);
        c.colors[vid] = i;
        for (int64_t k = g.off[vid]; k < g.off[vid + 1]; ++k) {
            const int v = g.nbr[k];
            if (c.colors[v] != -1) continue;
            auto& ac = adjcols[v];
            auto it = std::lower_bound(ac.begin(), ac.end(), i);
            if (it == ac.end() || *it != i) ac.insert(it, i);
            degree[v] -= g.mult[k];
            cur[v] = key((int64_t)ac.size(), degree[v], v);
            heap.push_back(cur[v]);
            std::push_heap(heap.begin(), heap.end());
        }
    }
    c.n_colors = g.n ? *std::max_element(c.colors.begin(), c.colors.end()) + 1 : 0;
    return c;
}

namespace {
void greedy_pick(const PrimalGraph& g, int i, int& nb_color, std::vector<int32_t>& colors, std::vector<char>& used) {
    used.assign(nb_color + 1, 0);
    for (int64_t k = g.off[i]; k < g.off[i + 1]; ++k) {
        const int col = colors[g.nbr[k]];
        if (col >= 0) used[col] = 1;
    }
    int c = 0;
    while (c < nb_color && used[c]) ++c;
    colors[i] = c;
    if (c == nb_color) ++nb_color;
}
}  // namespace

Coloring color_greedy(const PrimalGraph& g) {
    Coloring c;
    c.colors.assign(g.n, -1);
    std::vector<char> used;
    for (int i = 0; i < g.n; ++i) greedy_pick(g, i, c.n_colors, c.colors, used);
    return c;
}

Coloring color_greedy_slf(const PrimalGraph& g) {
    typedef std::pair<int64_t, int> PV;
    std::priority_queue<PV, std::vector<PV>, std::greater<PV>> h;
    for (int i = 0; i < g.n; ++i) h.push({g.degree[i], i});
    std::vector<int> ids(g.n, 0);
    std::vector<char> removed(g.n, 0);
    std::vector<int64_t> degree(g.degree);
    for (int i = g.n - 1; i >= 0; --i) {
        while (!h.empty() && removed[h.top().second]) h.pop();
        const int v = h.top().second;
        h.pop();
        removed[v] = 1;
        ids[i] = v;
        for (int64_t k = g.off[v]; k < g.off[v + 1]; ++k) {
            const int nb = g.nbr[k];
            if (removed[nb]) continue;
            degree[nb] -= g.mult[k];
            h.push({degree[nb], nb});
        }
    }
    Coloring c;
    c.colors.assign(g.n, -1);
    std::vector<char> used;
    for (int i : ids) greedy_pick(g, i, c.n_colors, c.colors, used);
    return c;
}

void color_reduction(const PrimalGraph& g, Coloring& c, int target) {
    std::vector<int64_t> occ(target > 0 ? target : 1);
    for (int vid = 0; vid < g.n; ++vid) {
        if (c.colors[vid] < target) continue;
        std::fill(occ.begin(), occ.end(), 0);
        for (int64_t k = g.off[vid]; k < g.off[vid + 1]; ++k) {
            const int col = c.colors[g.nbr[k]];
            if (col < target) occ[col] += g.mult[k];
        }
        c.colors[vid] = (int32_t)(std::min_element(occ.begin(), occ.begin() + target) - occ.begin());
    }
    c.n_colors = target;
}

int64_t count_conflicts(const PrimalGraph& g, const Coloring& c) {
    int64_t total = 0;
    for (int i = 0; i < g.n; ++i)
        for (int64_t k = g.off[i]; k < g.off[i + 1]; ++k)
            if (c.colors[g.nbr[k]] == c.colors[i]) total += 2 * g.mult[k];
    return total;
}

}  // namespace octb
