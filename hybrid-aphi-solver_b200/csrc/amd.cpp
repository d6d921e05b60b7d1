// The reference's approximate-minimum-degree ordering, restated so that a
// standalone caller reproduces its permutation bit for bit.
//
// Why a restatement: the benchmark and the serving loop run where the
// reference's host code is not present, yet the permutation must be the
// reference's own (the fill, the elimination tree and the factor all follow
// from it). The algorithm below therefore takes the same steps, with the same
// tie-breaking, as src/ordering.cpp:220-510 -- quotient-graph minimum degree
// (Amestoy, Davis & Duff) with supervariables detected by hashing, degree
// buckets kept as last-in-first-out linked lists, and the three-way degree
// bound -- over the symmetric adjacency of src/ordering.cpp:58-98 (each
// list ascending, no duplicates, no diagonal). Each vertex keeps growable
// lists (its variable neighbours, its elements, an element's members, the
// supervariables merged into it), released when the vertex is absorbed.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "ordering.hpp"

namespace aphi_b200 {

namespace {

enum : char { kVar = 0, kElem = 1, kGone = 2 };

// Growable per-vertex integer lists.
struct Lists {
    std::vector<std::vector<int>> v;
    explicit Lists(int n) : v(n) {}
    std::vector<int>& operator[](int i) { return v[i]; }
    void drop(int i) {
        v[i].clear();
        v[i].shrink_to_fit();
    }
};

}  // namespace

void adjacency_from_upper(int n, const int* row_ptr, const int* col_idx, std::vector<int>& off,
                          std::vector<int>& nbr) {
    off.assign(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            if (c == r) continue;
            ++off[r + 1];
            ++off[c + 1];
        }
    for (int i = 0; i < n; ++i) off[i + 1] += off[i];
    nbr.assign(off[n], 0);
    std::vector<int> cur(off.begin(), off.end() - 1);
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            if (c == r) continue;
            nbr[cur[r]++] = c;
            nbr[cur[c]++] = r;
        }
    std::vector<int> packed;
    packed.reserve(nbr.size());
    std::vector<int> noff(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        auto b = nbr.begin() + off[i], e = nbr.begin() + off[i + 1];
        std::sort(b, e);
        e = std::unique(b, e);
        noff[i] = static_cast<int>(packed.size());
        packed.insert(packed.end(), b, e);
    }
    noff[n] = static_cast<int>(packed.size());
    off.swap(noff);
    nbr.swap(packed);
}

void reference_amd(int n, const int* row_ptr, const int* col_idx, int* perm_out) {
    std::vector<int> off, nbr;
    adjacency_from_upper(n, row_ptr, col_idx, off, nbr);

    std::vector<char> kind(n, kVar);
    Lists var_adj(n), elem_adj(n), elem_members(n), merged(n);
    std::vector<int> deg(n), weight(n, 1), elem_weight(n, 0);
    for (int i = 0; i < n; ++i) {
        var_adj[i].assign(nbr.begin() + off[i], nbr.begin() + off[i + 1]);
        deg[i] = off[i + 1] - off[i];
    }

    // Degree buckets: doubly linked, new entries at the head.
    std::vector<int> bhead(n + 1, -1), bnext(n, -1), bprev(n, -1);
    auto bucket_of = [&](int i) { return std::min(deg[i], n); };
    auto push = [&](int i) {
        const int d = bucket_of(i);
        bnext[i] = bhead[d];
        bprev[i] = -1;
        if (bhead[d] >= 0) bprev[bhead[d]] = i;
        bhead[d] = i;
    };
    auto unlink = [&](int i) {
        const int d = bucket_of(i);
        const int a = bprev[i], b = bnext[i];
        if (a >= 0) bnext[a] = b;
        else if (bhead[d] == i) bhead[d] = b;
        if (b >= 0) bprev[b] = a;
        bprev[i] = bnext[i] = -1;
    };
    for (int i = 0; i < n; ++i) push(i);

    std::vector<int> order;
    order.reserve(n);
    std::vector<int> tag(n, -1);   // >= 0: member of L_p at step k; <= -2: element seen at step k
    std::vector<int> ext(n, 0);    // |L_e \ L_p|, weighted
    std::vector<int> seen_elems, lp;
    std::vector<int> hhead(n, -1), hnext(n, -1), hbuckets, mark(n, -1);
    int dmin = 0, done = 0, step = 0;

    while (done < n) {
        while (dmin <= n && bhead[dmin] < 0) ++dmin;
        if (dmin > n) break;
        const int p = bhead[dmin];
        unlink(p);
        order.push_back(p);
        for (int q : merged[p]) order.push_back(q);
        done += weight[p];
        const int k = step++;

        // L_p: live variables adjacent to p directly or through its elements.
        lp.clear();
        for (int j : var_adj[p])
            if (kind[j] == kVar && tag[j] != k) {
                tag[j] = k;
                lp.push_back(j);
            }
        for (int e : elem_adj[p]) {
            if (kind[e] != kElem) continue;
            for (int j : elem_members[e])
                if (kind[j] == kVar && j != p && tag[j] != k) {
                    tag[j] = k;
                    lp.push_back(j);
                }
        }
        // p's elements are absorbed into the new element p.
        for (int e : elem_adj[p])
            if (kind[e] == kElem) {
                kind[e] = kGone;
                elem_members.drop(e);
            }
        // Prune the neighbours' lists; each gains element p.
        for (int i : lp) {
            std::vector<int>& a = var_adj[i];
            a.erase(std::remove_if(a.begin(), a.end(),
                                   [&](int j) { return j == p || kind[j] != kVar || tag[j] == k; }),
                    a.end());
            std::vector<int>& el = elem_adj[i];
            el.erase(std::remove_if(el.begin(), el.end(), [&](int e) { return kind[e] != kElem; }), el.end());
            el.push_back(p);
        }
        // External weights of the other elements touching L_p.
        seen_elems.clear();
        for (int i : lp)
            for (int e : elem_adj[i]) {
                if (e == p) continue;
                if (tag[e] != -2 - k) {
                    tag[e] = -2 - k;
                    ext[e] = elem_weight[e];
                    seen_elems.push_back(e);
                }
                ext[e] -= weight[i];
            }
        long long lp_w = 0;
        for (int i : lp) lp_w += weight[i];
        // Approximate degrees, bounded by the exact facts.
        for (int i : lp) {
            long long through = 0;
            for (int e : elem_adj[i])
                if (e != p) through += std::max(0, ext[e]);
            long long direct = 0;
            for (int j : var_adj[i])
                if (kind[j] == kVar) direct += weight[j];
            const long long approx = direct + (lp_w - weight[i]) + through;
            const long long left = static_cast<long long>(n) - done;
            const long long grown = static_cast<long long>(deg[i]) + lp_w - weight[i];
            const long long d = std::min(left, std::min(grown, approx));
            unlink(i);
            deg[i] = static_cast<int>(std::max(0LL, d));
            push(i);
            dmin = std::min(dmin, deg[i]);
        }
        for (int e : seen_elems) tag[e] = -1;

        // p becomes an element.
        kind[p] = kElem;
        elem_members[p] = lp;
        elem_weight[p] = static_cast<int>(lp_w);
        var_adj.drop(p);
        elem_adj.drop(p);

        // Supervariables among L_p: hash (A_i, E_i), confirm exactly.
        hbuckets.clear();
        for (int i : lp) {
            if (kind[i] != kVar) continue;
            long long h = 0;
            for (int j : var_adj[i]) h += j;
            for (int e : elem_adj[i]) h += e;
            h %= n;
            if (hhead[h] < 0) hbuckets.push_back(static_cast<int>(h));
            hnext[i] = hhead[h];
            hhead[h] = i;
        }
        for (int h : hbuckets) {
            for (int i = hhead[h]; i >= 0; i = hnext[i]) {
                if (kind[i] != kVar) continue;
                for (int j : var_adj[i]) mark[j] = i;
                for (int e : elem_adj[i]) mark[e] = i;
                for (int j = hnext[i]; j >= 0; j = hnext[j]) {
                    if (kind[j] != kVar) continue;
                    if (var_adj[j].size() != var_adj[i].size() || elem_adj[j].size() != elem_adj[i].size()) continue;
                    bool same = true;
                    for (int q : var_adj[j])
                        if (mark[q] != i) {
                            same = false;
                            break;
                        }
                    if (same)
                        for (int e : elem_adj[j])
                            if (mark[e] != i) {
                                same = false;
                                break;
                            }
                    if (!same) continue;
                    unlink(j);
                    weight[i] += weight[j];
                    merged[i].push_back(j);
                    for (int q : merged[j]) merged[i].push_back(q);
                    merged.drop(j);
                    weight[j] = 0;
                    kind[j] = kGone;
                    var_adj.drop(j);
                    elem_adj.drop(j);
                }
            }
            hhead[h] = -1;
        }
    }
    if (static_cast<int>(order.size()) != n)
        throw Error(APHI_ERR_PATTERN_MISMATCH, "approximate minimum degree: not every unknown was ordered");
    std::copy(order.begin(), order.end(), perm_out);
}

}  // namespace aphi_b200
