// The reference's reverse Cuthill-McKee ordering (Ordering::ReverseCuthillMcKee,
// src/ordering.cpp:105-218 and :512-537), restated so that a standalone caller
// reproduces its permutation bit for bit. The steps that decide the
// permutation are the reference's:
//   - components in order of their lowest-numbered vertex;
//   - each started from a pseudo-peripheral vertex found by George and Liu's
//     rooted-level-structure search (at most 5 searches; the next root is the
//     first vertex of least degree in the deepest level, in visiting order;
//     stop when the depth stops growing or the root repeats);
//   - breadth first, each vertex's newly reached neighbours visited in
//     increasing degree, ties by index;
//   - the whole visiting order reversed.
// The bookkeeping is this file's own: a search clears only the marks of the
// component it visited.
#include <algorithm>
#include <vector>

#include "ordering.hpp"

namespace aphi_b200 {

namespace {

struct Graph {
    std::vector<int> off, nbr;
    int degree(int v) const { return off[v + 1] - off[v]; }
};

// Appends the breadth-first order of the component holding `root` to
// `order` and returns its depth (the last level's number).
int level_structure(const Graph& g, int root, std::vector<char>& seen, std::vector<int>& order,
                    std::vector<int>& level) {
    const size_t first = order.size();
    seen[root] = 1;
    level[root] = 0;
    order.push_back(root);
    int depth = 0;
    for (size_t head = first; head < order.size(); ++head) {
        const int v = order[head];
        const size_t fresh = order.size();
        for (int k = g.off[v]; k < g.off[v + 1]; ++k) {
            const int u = g.nbr[k];
            if (seen[u]) continue;
            seen[u] = 1;
            level[u] = level[v] + 1;
            depth = std::max(depth, level[u]);
            order.push_back(u);
        }
        std::sort(order.begin() + static_cast<long>(fresh), order.end(), [&](int a, int b) {
            const int da = g.degree(a), db = g.degree(b);
            return da != db ? da < db : a < b;
        });
    }
    return depth;
}

int pseudo_peripheral(const Graph& g, int start, std::vector<char>& seen, std::vector<int>& order,
                      std::vector<int>& level) {
    int root = start, root_depth = -1;
    for (int search = 0; search < 5; ++search) {
        order.clear();
        const int depth = level_structure(g, root, seen, order, level);
        for (int v : order) seen[v] = 0;
        if (depth <= root_depth) break;
        root_depth = depth;
        int next = root, next_degree = -1;
        for (int v : order)
            if (level[v] == depth && (next_degree < 0 || g.degree(v) < next_degree)) {
                next = v;
                next_degree = g.degree(v);
            }
        if (next == root) break;
        root = next;
    }
    return root;
}

}  // namespace

void reference_rcm(int n, const int* row_ptr, const int* col_idx, int* perm) {
    Graph g;
    adjacency_from_upper(n, row_ptr, col_idx, g.off, g.nbr);
    std::vector<char> seen(n, 0), scratch_seen(n, 0);
    std::vector<int> level(n, 0), order, scratch_order;
    order.reserve(n);
    for (int s = 0; s < n; ++s) {
        if (seen[s]) continue;
        const int root = pseudo_peripheral(g, s, scratch_seen, scratch_order, level);
        level_structure(g, root, seen, order, level);
    }
    std::reverse(order.begin(), order.end());
    std::copy(order.begin(), order.end(), perm);
}

}  // namespace aphi_b200
