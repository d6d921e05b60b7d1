// Fill-reducing ordering by geometric nested dissection.
//
// Not the reference's ordering: the reference orders with its own approximate
// minimum degree (src/ordering.cpp:220-510), and where the reference is the
// caller its permutation is consumed unchanged. This ordering exists so a
// standalone caller (the benchmark, the serving loop) can analyse a mesh
// without the reference's host code. Every permutation yields a correct
// factorization; the ordering only decides fill and the shape of the tree.
//
// Recursive coordinate bisection: split the unknowns at the median of their
// widest coordinate; the unknowns of the smaller side that touch the other
// side form the separator, numbered after both halves. Halves below `leaf`
// unknowns are numbered by a greedy minimum-degree pass on their own graph.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "ordering.hpp"

namespace aphi_b200 {

namespace {

struct Graph {
    std::vector<int> ptr, adj;
};

Graph symmetric_graph(int n, const int* row_ptr, const int* col_idx) {
    Graph g;
    g.ptr.assign(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            if (c == r) continue;
            ++g.ptr[r + 1];
            ++g.ptr[c + 1];
        }
    for (int i = 0; i < n; ++i) g.ptr[i + 1] += g.ptr[i];
    g.adj.resize(g.ptr[n]);
    std::vector<int> cur(g.ptr.begin(), g.ptr.end() - 1);
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            if (c == r) continue;
            g.adj[cur[r]++] = c;
            g.adj[cur[c]++] = r;
        }
    return g;
}

struct Dissector {
    const Graph& g;
    const double* xyz;
    int leaf;
    std::vector<int> side;   // scratch: 0 = not in current set, 1 = left, 2 = right, 3 = separator
    std::vector<int> order;  // output, new -> old
    std::vector<int> mark;

    // Greedy minimum degree within a small set (degrees counted inside the set).
    void leaf_order(std::vector<int>& set) {
        const int stamp = static_cast<int>(order.size()) + 1;
        for (int v : set) mark[v] = stamp;
        std::vector<int> deg(set.size());
        for (size_t a = 0; a < set.size(); ++a) {
            int d = 0;
            const int v = set[a];
            for (int k = g.ptr[v]; k < g.ptr[v + 1]; ++k) d += mark[g.adj[k]] == stamp;
            deg[a] = d;
        }
        std::vector<int> idx(set.size());
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return deg[a] < deg[b]; });
        for (int a : idx) order.push_back(set[a]);
    }

    void dissect(std::vector<int>& set) {
        if (static_cast<int>(set.size()) <= leaf) {
            leaf_order(set);
            return;
        }
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int v : set)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], xyz[3 * v + d]);
                hi[d] = std::max(hi[d], xyz[3 * v + d]);
            }
        int ax = 0;
        for (int d = 1; d < 3; ++d)
            if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
        if (hi[ax] - lo[ax] <= 0.0) {
            leaf_order(set);
            return;
        }
        std::sort(set.begin(), set.end(), [&](int a, int b) {
            const double xa = xyz[3 * a + ax], xb = xyz[3 * b + ax];
            return xa != xb ? xa < xb : a < b;
        });
        // Split between distinct coordinate values nearest the median, so a
        // layer of equal coordinates stays on one side.
        size_t mid = set.size() / 2;
        const double xm = xyz[3 * set[mid] + ax];
        size_t a = mid, b = mid;
        while (a > 0 && xyz[3 * set[a - 1] + ax] == xm) --a;
        while (b < set.size() && xyz[3 * set[b] + ax] == xm) ++b;
        mid = (mid - a <= b - mid) ? a : b;
        if (mid == 0 || mid == set.size()) mid = set.size() / 2;
        for (size_t i = 0; i < set.size(); ++i) side[set[i]] = i < mid ? 1 : 2;
        // Boundary of each side; the smaller one becomes the separator.
        std::vector<int> bl, br;
        for (int v : set) {
            bool touches = false;
            const int other = side[v] == 1 ? 2 : 1;
            for (int k = g.ptr[v]; k < g.ptr[v + 1] && !touches; ++k) touches = side[g.adj[k]] == other;
            if (touches) (side[v] == 1 ? bl : br).push_back(v);
        }
        std::vector<int>& sep = bl.size() <= br.size() ? bl : br;
        for (int v : sep) side[v] = 3;
        std::vector<int> left, right;
        for (int v : set) {
            if (side[v] == 1) left.push_back(v);
            else if (side[v] == 2) right.push_back(v);
        }
        std::vector<int> s(sep);
        for (int v : set) side[v] = 0;
        set.clear();
        set.shrink_to_fit();
        dissect(left);
        dissect(right);
        for (int v : s) order.push_back(v);
    }
};

}  // namespace

// perm (new -> old) by nested dissection over coordinates xyz (3 per unknown).
// Unknowns with no neighbours (voltage-port rows) are numbered first.
void nested_dissection(int n, const int* row_ptr, const int* col_idx, const double* xyz, int leaf, int* perm) {
    if (n <= 0) return;
    if (!row_ptr || !col_idx || !xyz || !perm) throw Error(APHI_ERR_INVALID, "nested_dissection: null argument");
    const Graph g = symmetric_graph(n, row_ptr, col_idx);
    Dissector d{g, xyz, std::max(leaf, 1), std::vector<int>(n, 0), {}, std::vector<int>(n, 0)};
    d.order.reserve(n);
    std::vector<int> set;
    for (int v = 0; v < n; ++v) {
        if (g.ptr[v + 1] == g.ptr[v]) d.order.push_back(v);
        else set.push_back(v);
    }
    d.dissect(set);
    if (static_cast<int>(d.order.size()) != n) throw Error(APHI_ERR_PATTERN_MISMATCH, "nested_dissection: lost unknowns");
    std::copy(d.order.begin(), d.order.end(), perm);
}

}  // namespace aphi_b200
