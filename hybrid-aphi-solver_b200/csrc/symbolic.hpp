// Supernodal symbolic analysis: from a pattern and a fill-reducing
// permutation to the schedule the device factorization follows.
//
// The reference's symbolic pass (src/symbolic.cpp:58-196) produces the
// permutation, the elimination tree and the column counts of L for an
// up-looking scalar factorization. This analysis recomputes the tree and the
// counts the same way (Liu's path-compressed tree; row subtrees for the
// counts), checks them against the reference's when given, and then
//   * post-orders the tree (an equivalent ordering: same fill, same factor
//     entries, only relabelled),
//   * groups columns into fundamental supernodes (a column joins its child
//     when that child is its only one and their structures nest exactly),
//   * relaxes them: a supernode absorbs the child that precedes it when the
//     explicit zeros added stay small,
//   * builds each supernode's row structure, the map from every stored entry
//     of A to its place in the supernode panels, and the child -> parent
//     extend-add maps of the multifrontal method,
//   * levels the supernodal tree (leaves first) and lays out device memory.
#pragma once

#include <cstdint>
#include <vector>

#include "aphi_b200.h"

namespace aphi_b200 {

struct Symbolic {
    int n = 0;
    long long nnz_a = 0;

    // Orderings. `post_of_ref[k]` = post-ordered index of the caller's
    // permuted column k; `new_of_orig[r]` = post-ordered index of original
    // unknown r; `orig_of_new` its inverse.
    std::vector<int> perm;          // caller's perm (new -> old)
    std::vector<int> ref_parent;    // etree in the caller's permuted numbering
    std::vector<int> ref_colcount;  // column counts (incl. diagonal), same numbering
    std::vector<int> post_of_ref, ref_of_post;
    std::vector<int> new_of_orig, orig_of_new;

    // Supernodes, in post order (children before parents).
    int ns = 0;
    std::vector<int> sn_first;   // first column (post-ordered numbering), ns + 1
    std::vector<int> sn_rows;    // m_s: rows of the panel (structure size)
    std::vector<int> sn_parent;  // parent supernode, -1 for roots
    std::vector<long long> sn_struct_off;  // ns + 1, into structs
    std::vector<int> structs;               // row indices, post-ordered numbering
    std::vector<long long> sn_loff;         // ns + 1, panel offsets (complex entries)
    std::vector<long long> sn_cboff;        // ns, CB offsets in the pool (-1 if none)
    std::vector<int> sn_level;
    std::vector<int> col_snode;             // column -> supernode

    // Children lists and extend-add maps.
    std::vector<int> child_ptr, child_list;   // ns + 1, children of each supernode in order
    std::vector<long long> rel_off;           // ns + 1, offsets into rel (per child supernode)
    std::vector<int> rel;                     // position in parent's structure, per CB row

    // Levels: supernodes grouped by level.
    int num_levels = 0;
    std::vector<int> level_ptr, level_list;

    // A entry k (upper CSR order, original numbering) -> panel position.
    std::vector<long long> a_dest;

    long long stored = 0;        // sum m_s * w_s
    long long cb_pool = 0;       // CB pool entries
    long long nnz_l = 0;         // sum col_count (unpadded, incl. diagonal)
    double flops = 0.0;          // 8 * sum c'(c'+1)/2, c' = col_count - 1
    int max_rows = 0, max_width = 0, num_roots = 0;
};

// Independent dense fronts (no tree): front s has rows[s] rows, of which the
// first widths[s] are its pivot columns. Its contribution block starts at zero
// and is left in the pool (the multifrontal update of the front, without a
// parent to add it to): the shape of the supernode-update microbenchmark.
Symbolic fronts_symbolic(int count, const int* rows, const int* widths);

// perm may be null (identity). parent/col_count, when non-null, are checked.
Symbolic analyze_supernodal(int n, const int* row_ptr, const int* col_idx, const int* perm,
                            const int* parent, const int* col_count, const aphi_analysis_options& opt);

}  // namespace aphi_b200
