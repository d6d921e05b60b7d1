#include "symbolic.hpp"

#include <algorithm>
#include <exception>
#include <functional>
#include <numeric>
#include <string>
#include <system_error>
#include <thread>

#include "common.cuh"

namespace aphi_b200 {

namespace {

[[noreturn]] void mismatch(const std::string& m) { throw Error(APHI_ERR_PATTERN_MISMATCH, m); }

// CB memory. Front s's contribution block is written at its own level and
// read for the last time by its parent's extend-add, so under the level
// schedule it is live from level(s) to level(parent(s)), inclusive; two
// blocks may share memory when their lifetimes are disjoint. The pool can be
// no smaller than the largest total of blocks live at one level.
//
// Placement is offline: blocks are taken in a fixed order and each goes to
// the lowest offset, rounded up to 32 entries (512 B for complex128), that is
// free at every level of its lifetime. Three orders are tried -- largest
// block first; largest size x lifetime first; latest-freed first, then
// largest -- and the one with the smallest pool is kept. On the cylinders
// and tori measured this lands within 0-4% of the bound (a level-by-level
// first fit was 20-50% above it).

// The blocks placed at one level, sorted by begin (they never overlap, so ends
// are sorted too), in runs of at most 2 * kRun; each block records the free
// gap before it and each run its largest gap, so searches skip full runs.
class LevelSpace {
public:
    // The lowest 32-aligned p >= x (x aligned) with [p, p + need) free here.
    long long fit(long long x, long long need) const {
        size_t lo = 0, hi = runs_.size();  // the first run with a block ending after x
        while (lo < hi) {
            const size_t mid = (lo + hi) / 2;
            if (runs_[mid].b.back().end > x) hi = mid;
            else lo = mid + 1;
        }
        size_t ri = lo;
        if (ri == runs_.size()) return x;
        size_t bi = std::upper_bound(runs_[ri].b.begin(), runs_[ri].b.end(), x,
                                     [](long long v, const Block& b) { return v < b.end; }) -
                    runs_[ri].b.begin();
        long long p = x;
        while (true) {
            if (ri == runs_.size() || runs_[ri].b[bi].begin >= p + need) return p;
            p = align(std::max(p, runs_[ri].b[bi].end));
            if (++bi == runs_[ri].b.size()) ++ri, bi = 0;
            // The next block with a gap of at least `need` before it (a smaller
            // gap cannot hold the block); p moves past every block skipped.
            while (ri < runs_.size()) {
                const Run& r = runs_[ri];
                while (bi < r.b.size() && r.b[bi].gap < need) p = align(std::max(p, r.b[bi++].end));
                if (bi < r.b.size()) break;
                ++ri;
                bi = 0;
                while (ri < runs_.size() && runs_[ri].max_gap < need) p = align(std::max(p, runs_[ri++].b.back().end));
            }
        }
    }
    void insert(long long begin, long long end) {
        if (runs_.empty()) {
            runs_.push_back(Run{{Block{begin, end, begin}}, begin});
            return;
        }
        size_t lo = 0, hi = runs_.size();  // the first run whose last block begins after `begin`
        while (lo < hi) {
            const size_t mid = (lo + hi) / 2;
            if (runs_[mid].b.back().begin > begin) hi = mid;
            else lo = mid + 1;
        }
        const size_t ri = std::min(lo, runs_.size() - 1);
        Run& r = runs_[ri];
        const size_t bi = std::upper_bound(r.b.begin(), r.b.end(), begin,
                                           [](long long v, const Block& b) { return v < b.begin; }) -
                          r.b.begin();
        const long long prev_end = bi > 0 ? r.b[bi - 1].end : (ri > 0 ? runs_[ri - 1].b.back().end : 0);
        r.b.insert(r.b.begin() + bi, Block{begin, end, begin - prev_end});
        if (bi + 1 < r.b.size()) {
            r.b[bi + 1].gap = r.b[bi + 1].begin - end;
        } else if (ri + 1 < runs_.size()) {
            Run& next = runs_[ri + 1];
            next.b[0].gap = next.b[0].begin - end;
            regap(next);
        }
        if (r.b.size() > 2 * kRun) {
            Run tail;
            tail.b.assign(r.b.begin() + kRun, r.b.end());
            r.b.resize(kRun);
            regap(tail);
            regap(r);
            runs_.insert(runs_.begin() + ri + 1, std::move(tail));
        } else {
            regap(r);
        }
    }

private:
    static constexpr size_t kRun = 256;
    struct Block {
        long long begin, end, gap;
    };
    struct Run {
        std::vector<Block> b;
        long long max_gap = 0;
    };
    static long long align(long long v) { return (v + 31) / 32 * 32; }
    static void regap(Run& r) {
        r.max_gap = 0;
        for (const Block& b : r.b) r.max_gap = std::max(r.max_gap, b.gap);
    }
    std::vector<Run> runs_;
};

struct CbBlock {
    int s, lo, hi;  // front, first and last level live
    long long need;
};

// Places the blocks in `order`; returns the pool size, offsets into `at`.
long long place_in_order(const std::vector<CbBlock>& blocks, const std::vector<int>& order, int levels,
                         std::vector<long long>& at) {
    std::vector<LevelSpace> space(levels);
    at.assign(blocks.size(), -1);
    long long top = 0;
    for (int i : order) {
        const CbBlock& b = blocks[i];
        long long x = 0;
        for (bool moved = true; moved;) {  // until one offset fits at every level
            moved = false;
            for (int L = b.lo; L <= b.hi; ++L) {
                const long long p = space[L].fit(x, b.need);
                if (p != x) {
                    x = p;
                    moved = true;
                }
            }
        }
        at[i] = x;
        top = std::max(top, x + b.need);
        for (int L = b.lo; L <= b.hi; ++L) space[L].insert(x, x + b.need);
    }
    return top;
}

long long place_blocks(const Symbolic& S, std::vector<long long>& off) {
    std::vector<CbBlock> blocks;
    for (int L = 0; L < S.num_levels; ++L)
        for (int k = S.level_ptr[L]; k < S.level_ptr[L + 1]; ++k) {
            const int s = S.level_list[k];
            const long long c = S.sn_rows[s] - (S.sn_first[s + 1] - S.sn_first[s]);
            if (c > 0) blocks.push_back({s, L, S.sn_parent[s] >= 0 ? S.sn_level[S.sn_parent[s]] : L, c * c});
        }
    auto span = [](const CbBlock& b) { return static_cast<long long>(b.hi - b.lo + 1); };
    const std::vector<std::function<bool(const CbBlock&, const CbBlock&)>> orders = {
        [](const CbBlock& a, const CbBlock& b) { return a.need > b.need; },
        [&](const CbBlock& a, const CbBlock& b) { return a.need * span(a) > b.need * span(b); },
        [](const CbBlock& a, const CbBlock& b) { return a.hi != b.hi ? a.hi > b.hi : a.need > b.need; },
    };
    // The orders are independent: one thread each. A thread that cannot be
    // started runs its order here instead; errors are rethrown once every
    // thread has been joined.
    std::vector<long long> top(orders.size());
    std::vector<std::vector<long long>> at(orders.size());
    std::vector<std::exception_ptr> err(orders.size());
    auto run = [&](size_t q) {
        try {
            std::vector<int> order(blocks.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(),
                             [&](int a, int b) { return orders[q](blocks[a], blocks[b]); });
            top[q] = place_in_order(blocks, order, S.num_levels, at[q]);
        } catch (...) {
            err[q] = std::current_exception();
        }
    };
    {
        std::vector<std::thread> pool;
        pool.reserve(orders.size());
        for (size_t q = 1; q < orders.size(); ++q) {
            try {
                pool.emplace_back(run, q);
            } catch (const std::system_error&) {
                run(q);
            }
        }
        run(0);
        for (std::thread& t : pool) t.join();
    }
    for (const std::exception_ptr& e : err)
        if (e) std::rethrow_exception(e);
    size_t best = 0;  // the smallest pool; on a tie, the earlier order
    for (size_t q = 1; q < orders.size(); ++q)
        if (top[q] < top[best]) best = q;
    off.assign(S.ns, -1);
    for (size_t i = 0; i < blocks.size(); ++i) off[blocks[i].s] = at[best][i];
    return std::max(top[best], 0LL);
}

}  // namespace

Symbolic analyze_supernodal(int n, const int* row_ptr, const int* col_idx, const int* perm_in,
                            const int* parent_in, const int* col_count_in, const aphi_analysis_options& opt) {
    if (n < 0 || !row_ptr || (!col_idx && n > 0))
        throw Error(APHI_ERR_INVALID, "analysis: missing pattern");
    Symbolic S;
    S.n = n;
    S.nnz_a = row_ptr[n];

    // Permutation and its inverse.
    S.perm.resize(n);
    std::vector<int> iperm(n, -1);
    for (int k = 0; k < n; ++k) {
        const int old = perm_in ? perm_in[k] : k;
        if (old < 0 || old >= n || iperm[old] >= 0)
            throw Error(APHI_ERR_BAD_SHAPE, "analysis: perm is not a permutation of 0..n-1");
        S.perm[k] = old;
        iperm[old] = k;
    }

    // Earlier neighbours of each permuted row (the strictly lower part).
    std::vector<int> lo_ptr(n + 1, 0);
    for (int r = 0; r < n; ++r) {
        if (row_ptr[r + 1] < row_ptr[r]) throw Error(APHI_ERR_BAD_SHAPE, "analysis: row_ptr decreases");
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            if (c < 0 || c >= n) throw Error(APHI_ERR_BAD_SHAPE, "analysis: column index out of range");
            if (c < r) throw Error(APHI_ERR_BAD_SHAPE, "analysis: entry below the diagonal in an upper pattern");
            if (c == r) continue;
            ++lo_ptr[std::max(iperm[r], iperm[c]) + 1];
        }
    }
    for (int i = 0; i < n; ++i) lo_ptr[i + 1] += lo_ptr[i];
    std::vector<int> lo_idx(lo_ptr[n]);
    {
        std::vector<int> cur(lo_ptr.begin(), lo_ptr.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
                const int c = col_idx[k];
                if (c == r) continue;
                const int a = iperm[r], b = iperm[c];
                lo_idx[cur[std::max(a, b)]++] = std::min(a, b);
            }
    }

    // Elimination tree, path compression through `ancestor`.
    std::vector<int>& parent = S.ref_parent;
    parent.assign(n, -1);
    {
        std::vector<int> ancestor(n, -1);
        for (int k = 0; k < n; ++k)
            for (int t = lo_ptr[k]; t < lo_ptr[k + 1]; ++t) {
                int i = lo_idx[t];
                while (i != -1 && i < k) {
                    const int next = ancestor[i];
                    ancestor[i] = k;
                    if (next == -1) parent[i] = k;
                    i = next;
                }
            }
    }
    // Post order (children in ascending order, roots ascending).
    std::vector<int> head(n, -1), next(n, -1);
    for (int j = n - 1; j >= 0; --j)
        if (parent[j] >= 0) {
            next[j] = head[parent[j]];
            head[parent[j]] = j;
        }
    S.post_of_ref.assign(n, -1);
    S.ref_of_post.assign(n, -1);
    {
        int k = 0;
        std::vector<int> stack;
        for (int r = 0; r < n; ++r) {
            if (parent[r] != -1) continue;
            ++S.num_roots;
            stack.push_back(r);
            while (!stack.empty()) {
                const int p = stack.back();
                const int c = head[p];
                if (c == -1) {
                    stack.pop_back();
                    S.ref_of_post[k] = p;
                    S.post_of_ref[p] = k++;
                } else {
                    head[p] = next[c];
                    stack.push_back(c);
                }
            }
        }
        if (k != n) mismatch("analysis: the elimination tree is not a forest");
    }
    // Column counts (Gilbert, Ng and Peyton 1994): cc[j] is the number of
    // row subtrees through j. In postorder, a neighbour k of row i is a leaf
    // of row i's subtree when k's subtree holds no earlier neighbour of row i
    // (first[k] > the last neighbour's postorder index). Each leaf adds one at
    // itself, each pair of consecutive leaves subtracts one at their least
    // common ancestor (the root of the union-find over finished nodes), and
    // row i subtracts one at its parent, so summing over a node's subtree
    // counts the rows through it exactly once; a row with no leaf adds its
    // own diagonal. O(nnz(A) alpha), equal to walking every row subtree.
    std::vector<int>& cc = S.ref_colcount;
    cc.assign(n, 0);
    {
        const std::vector<int>& post = S.post_of_ref;
        const std::vector<int>& ref = S.ref_of_post;
        std::vector<int> first(n, -1);  // smallest postorder index in each subtree, by postorder index
        for (int q = 0; q < n; ++q) {
            for (int v = ref[q]; v != -1 && first[post[v]] == -1; v = parent[v]) first[post[v]] = q;
        }
        // Rows below each column: the transpose of the earlier-neighbour lists.
        std::vector<int> up_ptr(n + 1, 0), up_idx(lo_ptr[n]);
        for (int t = 0; t < lo_ptr[n]; ++t) ++up_ptr[lo_idx[t] + 1];
        for (int j = 0; j < n; ++j) up_ptr[j + 1] += up_ptr[j];
        {
            std::vector<int> at(up_ptr.begin(), up_ptr.end() - 1);
            for (int i = 0; i < n; ++i)
                for (int t = lo_ptr[i]; t < lo_ptr[i + 1]; ++t) up_idx[at[lo_idx[t]]++] = i;
        }
        std::vector<long long> delta(n, 0);
        std::vector<int> prevleaf(n, -1), maxfirst(n, -1), uf(n);
        std::iota(uf.begin(), uf.end(), 0);
        auto find = [&](int x) {
            int r = x;
            while (uf[r] != r) r = uf[r];
            while (uf[x] != r) {
                const int nx = uf[x];
                uf[x] = r;
                x = nx;
            }
            return r;
        };
        for (int q = 0; q < n; ++q) {
            const int j = ref[q];
            for (int t = up_ptr[j]; t < up_ptr[j + 1]; ++t) {
                const int i = up_idx[t];
                if (first[q] <= maxfirst[i]) continue;  // not a leaf of row i's subtree
                maxfirst[i] = first[q];
                ++delta[j];
                if (prevleaf[i] != -1) --delta[find(prevleaf[i])];
                prevleaf[i] = j;
            }
            if (prevleaf[j] == -1) ++delta[j];  // row j has no earlier neighbour: its diagonal
            if (parent[j] != -1) {
                --delta[parent[j]];
                uf[j] = parent[j];
            }
        }
        for (int q = 0; q < n; ++q) {
            const int j = ref[q];
            const long long c = delta[j] + cc[j];
            cc[j] = static_cast<int>(c);
            if (parent[j] != -1) cc[parent[j]] += cc[j];
        }
    }
    if (parent_in)
        for (int j = 0; j < n; ++j)
            if (parent_in[j] != parent[j])
                mismatch("analysis: the elimination tree handed in differs from this pattern's at column " +
                         std::to_string(j));
    if (col_count_in)
        for (int j = 0; j < n; ++j)
            if (col_count_in[j] != cc[j])
                mismatch("analysis: the column counts handed in differ from this pattern's at column " +
                         std::to_string(j));

    S.new_of_orig.resize(n);
    S.orig_of_new.resize(n);
    for (int r = 0; r < n; ++r) {
        S.new_of_orig[r] = S.post_of_ref[iperm[r]];
        S.orig_of_new[S.new_of_orig[r]] = r;
    }
    std::vector<int> pp(n), pcc(n), nchild(n, 0);
    for (int j = 0; j < n; ++j) {
        const int q = S.post_of_ref[j];
        pp[q] = parent[j] < 0 ? -1 : S.post_of_ref[parent[j]];
        pcc[q] = cc[j];
    }
    for (int j = 0; j < n; ++j)
        if (pp[j] >= 0) ++nchild[pp[j]];
    for (int j = 0; j < n; ++j) {
        S.nnz_l += pcc[j];
        const double c = pcc[j] - 1;
        S.flops += 8.0 * c * (c + 1) / 2;
    }

    // Fundamental supernodes.
    std::vector<int> ffirst;
    for (int j = 0; j < n; ++j)
        if (!(j > 0 && pp[j - 1] == j && pcc[j - 1] == pcc[j] + 1 && nchild[j] == 1)) ffirst.push_back(j);
    const int nf = static_cast<int>(ffirst.size());
    ffirst.push_back(n);
    std::vector<int> fsn(n);
    for (int s = 0; s < nf; ++s)
        for (int j = ffirst[s]; j < ffirst[s + 1]; ++j) fsn[j] = s;

    // Relaxed amalgamation: a supernode absorbs the supernode ending just
    // before it when that one is its child and the padding stays small.
    struct Cur {
        int first, width;
        long long rows, nz;
    };
    std::vector<Cur> cur;
    for (int s = 0; s < nf; ++s) {
        Cur c{ffirst[s], ffirst[s + 1] - ffirst[s], pcc[ffirst[s]], 0};
        for (int j = ffirst[s]; j < ffirst[s + 1]; ++j) c.nz += pcc[j];
        while (!cur.empty()) {
            const Cur& q = cur.back();
            const int ql = q.first + q.width - 1;
            if (ql + 1 != c.first || pp[ql] < c.first || pp[ql] >= c.first + c.width) break;
            const long long w = q.width + c.width;
            const long long m = q.width + c.rows;
            const long long stored = w * m - w * (w - 1) / 2;
            const double zeros = static_cast<double>(stored - q.nz - c.nz) / static_cast<double>(stored);
            const bool ok = w <= opt.relax_max_width &&
                            (w <= opt.relax_small || (w <= 16 && zeros < 0.8) ||
                             (w <= 48 && zeros < 0.1) || zeros < opt.relax_fill);
            if (!ok) break;
            c = Cur{q.first, static_cast<int>(w), m, q.nz + c.nz};
            cur.pop_back();
        }
        cur.push_back(c);
    }
    S.ns = static_cast<int>(cur.size());
    const int ns = S.ns;
    S.sn_first.resize(ns + 1);
    for (int s = 0; s < ns; ++s) S.sn_first[s] = cur[s].first;
    S.sn_first[ns] = n;
    S.col_snode.resize(n);
    for (int s = 0; s < ns; ++s)
        for (int j = S.sn_first[s]; j < S.sn_first[s + 1]; ++j) S.col_snode[j] = s;
    S.sn_parent.assign(ns, -1);
    for (int s = 0; s < ns; ++s) {
        const int l = S.sn_first[s + 1] - 1;
        S.sn_parent[s] = pp[l] < 0 ? -1 : S.col_snode[pp[l]];
    }

    // Lower column lists of A in post-ordered numbering.
    std::vector<int> acol_ptr(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int a = S.new_of_orig[r], b = S.new_of_orig[col_idx[k]];
            if (a != b) ++acol_ptr[std::min(a, b) + 1];
        }
    for (int j = 0; j < n; ++j) acol_ptr[j + 1] += acol_ptr[j];
    std::vector<int> acol(acol_ptr[n]), acol_k(acol_ptr[n]);  // row, and the entry's index in A
    {
        std::vector<int> c2(acol_ptr.begin(), acol_ptr.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
                const int a = S.new_of_orig[r], b = S.new_of_orig[col_idx[k]];
                if (a == b) continue;
                const int t = c2[std::min(a, b)]++;
                acol[t] = std::max(a, b);
                acol_k[t] = k;
            }
    }

    // Children lists (ascending), then structures bottom-up.
    S.child_ptr.assign(ns + 1, 0);
    for (int s = 0; s < ns; ++s)
        if (S.sn_parent[s] >= 0) ++S.child_ptr[S.sn_parent[s] + 1];
    for (int s = 0; s < ns; ++s) S.child_ptr[s + 1] += S.child_ptr[s];
    S.child_list.resize(S.child_ptr[ns]);
    {
        std::vector<int> c2(S.child_ptr.begin(), S.child_ptr.end() - 1);
        for (int s = 0; s < ns; ++s)
            if (S.sn_parent[s] >= 0) S.child_list[c2[S.sn_parent[s]]++] = s;
    }
    S.sn_rows.assign(ns, 0);
    S.sn_struct_off.assign(ns + 1, 0);
    std::vector<int> mark(n, -1), rows;
    S.structs.clear();
    for (int s = 0; s < ns; ++s) {
        const int f = S.sn_first[s], l = S.sn_first[s + 1] - 1;
        rows.clear();
        for (int j = f; j <= l; ++j) {
            rows.push_back(j);
            mark[j] = s;
        }
        for (int j = f; j <= l; ++j)
            for (int t = acol_ptr[j]; t < acol_ptr[j + 1]; ++t) {
                const int i = acol[t];
                if (i > l && mark[i] != s) {
                    mark[i] = s;
                    rows.push_back(i);
                }
            }
        for (int t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
            const int c = S.child_list[t];
            for (long long q = S.sn_struct_off[c]; q < S.sn_struct_off[c + 1]; ++q) {
                const int i = S.structs[q];
                if (i > l && mark[i] != s) {
                    mark[i] = s;
                    rows.push_back(i);
                }
            }
        }
        std::sort(rows.begin() + (l - f + 1), rows.end());
        S.sn_rows[s] = static_cast<int>(rows.size());
        if (S.sn_rows[s] < pcc[f])
            mismatch("analysis: a supernode's structure is smaller than its first column's count");
        S.structs.insert(S.structs.end(), rows.begin(), rows.end());
        S.sn_struct_off[s + 1] = static_cast<long long>(S.structs.size());
    }
    for (int s = 0; s < ns; ++s) {
        const int w = S.sn_first[s + 1] - S.sn_first[s];
        S.max_rows = std::max(S.max_rows, S.sn_rows[s]);
        S.max_width = std::max(S.max_width, w);
    }

    // Panel offsets; each panel starts on a 32-entry (512 B) boundary.
    S.sn_loff.assign(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        const long long w = S.sn_first[s + 1] - S.sn_first[s];
        S.sn_loff[s + 1] = S.sn_loff[s] + (static_cast<long long>(S.sn_rows[s]) * w + 31) / 32 * 32;
    }
    S.stored = S.sn_loff[ns];

    // Extend-add maps (each CB row of child c -> its position in the parent's
    // structure) and A entries -> panel positions. Both look rows up in one
    // numbering of a supernode's structure: its children's CB rows, and the
    // rows of the entries of A in its columns. The diagonal entry of column j
    // sits at row j - first of its panel, since a structure opens with its own
    // columns.
    S.rel_off.assign(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        const int w = S.sn_first[s + 1] - S.sn_first[s];
        S.rel_off[s + 1] = S.rel_off[s] + (S.sn_parent[s] >= 0 ? S.sn_rows[s] - w : 0);
    }
    S.rel.assign(S.rel_off[ns], 0);
    S.a_dest.assign(S.nnz_a, -1);
    {
        std::vector<int> at_row(n), owner(n, -1);
        for (int s = 0; s < ns; ++s) {
            const int f = S.sn_first[s], l = S.sn_first[s + 1] - 1, m = S.sn_rows[s];
            const int* st = S.structs.data() + S.sn_struct_off[s];
            for (int q = 0; q < m; ++q) {
                at_row[st[q]] = q;
                owner[st[q]] = s;
            }
            for (int t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
                const int c = S.child_list[t];
                const int wc = S.sn_first[c + 1] - S.sn_first[c];
                const int* sc = S.structs.data() + S.sn_struct_off[c];
                for (int i = wc; i < S.sn_rows[c]; ++i) {
                    if (owner[sc[i]] != s) mismatch("analysis: a child's row is missing from its parent's structure");
                    S.rel[S.rel_off[c] + (i - wc)] = at_row[sc[i]];
                }
            }
            for (int j = f; j <= l; ++j) {
                const long long col0 = S.sn_loff[s] + static_cast<long long>(j - f) * m;
                for (int t = acol_ptr[j]; t < acol_ptr[j + 1]; ++t) {
                    if (owner[acol[t]] != s) mismatch("analysis: an entry of A has no place in L's structure");
                    S.a_dest[acol_k[t]] = col0 + at_row[acol[t]];
                }
            }
        }
        for (int r = 0; r < n; ++r)
            for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k)
                if (col_idx[k] == r) {
                    const int j = S.new_of_orig[r], s = S.col_snode[j], d = j - S.sn_first[s];
                    S.a_dest[k] = S.sn_loff[s] + static_cast<long long>(d) * S.sn_rows[s] + d;
                }
    }

    // Levels.
    S.sn_level.assign(ns, 0);
    for (int s = 0; s < ns; ++s)
        if (S.sn_parent[s] >= 0)
            S.sn_level[S.sn_parent[s]] = std::max(S.sn_level[S.sn_parent[s]], S.sn_level[s] + 1);
    S.num_levels = 0;
    for (int s = 0; s < ns; ++s) S.num_levels = std::max(S.num_levels, S.sn_level[s] + 1);
    S.level_ptr.assign(S.num_levels + 1, 0);
    for (int s = 0; s < ns; ++s) ++S.level_ptr[S.sn_level[s] + 1];
    for (int L = 0; L < S.num_levels; ++L) S.level_ptr[L + 1] += S.level_ptr[L];
    S.level_list.resize(ns);
    {
        std::vector<int> c2(S.level_ptr.begin(), S.level_ptr.end() - 1);
        for (int s = 0; s < ns; ++s) S.level_list[c2[S.sn_level[s]]++] = s;
    }
    S.cb_pool = place_blocks(S, S.sn_cboff);
    return S;
}

Symbolic fronts_symbolic(int count, const int* rows, const int* widths) {
    if (count < 1 || !rows || !widths) throw Error(APHI_ERR_BAD_SHAPE, "fronts: need at least one front");
    Symbolic S;
    S.ns = count;
    S.sn_first.assign(count + 1, 0);
    for (int s = 0; s < count; ++s) {
        if (widths[s] < 1 || rows[s] < widths[s])
            throw Error(APHI_ERR_BAD_SHAPE, "fronts: each front needs 1 <= width <= rows");
        S.sn_first[s + 1] = S.sn_first[s] + widths[s];
    }
    const int n = S.sn_first[count];
    S.n = n;
    S.nnz_a = 0;
    S.perm.resize(n);
    for (int j = 0; j < n; ++j) S.perm[j] = j;
    S.post_of_ref = S.ref_of_post = S.new_of_orig = S.orig_of_new = S.perm;
    S.ref_parent.assign(n, -1);
    S.ref_colcount.assign(n, 1);
    S.col_snode.assign(n, 0);
    S.sn_rows.assign(rows, rows + count);
    S.sn_parent.assign(count, -1);
    S.sn_level.assign(count, 0);
    S.sn_struct_off.assign(count + 1, 0);
    S.sn_loff.assign(count + 1, 0);
    for (int s = 0; s < count; ++s) {
        const int w = widths[s], m = rows[s], f = S.sn_first[s];
        S.sn_struct_off[s + 1] = S.sn_struct_off[s] + m;
        // Rows past the pivots belong to no column of this system; they are
        // never used as indices by the factorization.
        for (int i = 0; i < m; ++i) S.structs.push_back(i < w ? f + i : 0);
        S.sn_loff[s + 1] = S.sn_loff[s] + (static_cast<long long>(m) * w + 31) / 32 * 32;
        for (int j = 0; j < w; ++j) {
            S.col_snode[f + j] = s;
            // one column of a front: m - j - 1 entries below its diagonal
            S.ref_colcount[f + j] = m - j;
            const double c = m - j - 1;
            S.flops += 8.0 * c * (c + 1) / 2;
            S.nnz_l += m - j;
            if (j + 1 < w) S.ref_parent[f + j] = f + j + 1;
        }
        S.max_rows = std::max(S.max_rows, m);
        S.max_width = std::max(S.max_width, w);
    }
    S.stored = S.sn_loff[count];
    S.num_roots = count;
    S.child_ptr.assign(count + 1, 0);
    S.rel_off.assign(count + 1, 0);
    S.num_levels = 1;
    S.level_ptr = {0, count};
    S.level_list.resize(count);
    for (int s = 0; s < count; ++s) S.level_list[s] = s;
    S.cb_pool = place_blocks(S, S.sn_cboff);
    return S;
}

}  // namespace aphi_b200
