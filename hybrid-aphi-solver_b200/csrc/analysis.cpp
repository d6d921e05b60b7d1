#include "analysis.hpp"

#include <algorithm>

#include "common.cuh"
#include "tc_config.hpp"

namespace aphi_b200 {

namespace {

template <class T>
T* upload(const std::vector<T>& h, long long& bytes) {
    T* d = nullptr;
    const size_t n = std::max<size_t>(h.size(), 1);
    APHI_CUDA(cudaMalloc(&d, n * sizeof(T)));
    if (!h.empty()) APHI_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    bytes += static_cast<long long>(n * sizeof(T));
    return d;
}

// The factorization plans: per level, extend-add items, then one-CTA fronts,
// then the blocked steps of the large fronts. A large front is processed in
// 128-column panels; each 32-column step of a panel factors its diagonal
// block, solves the panel rows below it and updates the rest of the panel's
// own columns. Once a panel is complete, its trailing update -- every column
// to its right, K = panel width -- runs as 128 x 64 tiles: `trailing` is
// K_UPDATE_WIDE (DMMA for FP64, SIMT for FP32) or K_UPDATE_TC (tensor cores, FP32).
// Updating the trailing front once per 128 columns instead of once per 32
// reads and writes it a quarter as often.
void build_factor_plan(aphi_analysis& A, std::vector<Item>& items, int trailing, std::vector<Launch>& plan) {
    const Symbolic& S = A.S;
    auto push = [&](int kind, long long first, int kcap = kTcPanel, int wide = 0) {
        const int count = static_cast<int>(items.size() - first);
        if (count > 0) plan.push_back({kind, first, count, kcap, wide});
    };
    // The FP64 plan (and the SIMT FP32 one) runs the in-panel updates on the
    // trailing-update kernel as 128 x 64 tiles of K = 32, its columns capped
    // at the panel's end; the tensor-core plan keeps the 64 x 64 SIMT tiles.
    const bool panel_wide = trailing == K_UPDATE_WIDE;
    // Trailing updates whose operands are prepared once per front and panel
    // group (K_TC_SPLIT / K_DMMA_SCALE launches) rather than inside every tile.
    const bool staged = trailing == K_UPDATE_TC || trailing == K_UPDATE_WIDE;
    // Panels are grouped for the trailing update: after each panel but a
    // group's last only the group's remaining columns are updated; after its
    // last, the rest of the front with all of the group's panels, so every
    // trailing entry is read and written once per group instead of once per
    // 128 columns. Groups are 4 panels (K up to 512) in fronts of at least
    // group4_rows rows (8192 by default), where the trailing matrix dwarfs the
    // group's columns, 2 panels (K up to 256) in fronts of at least
    // group2_rows, and single panels below that, where the in-group updates
    // would cost more than the traffic they save. The thresholds are analysis
    // options, which the autotuner (aphi_b200.autotune) picks per mesh. Only full groups are grouped: the
    // narrow tiles then end exactly at the group's last column, and a front's
    // incomplete last group is updated panel by panel.
    // The tensor-core plan has thresholds of its own (its grouping sets the
    // FP32 factor's rounding, which the refinement depends on).
    const bool tc = trailing == K_UPDATE_TC;
    const int g4opt = tc ? A.opt.tc_group4_rows : A.opt.group4_rows, g2opt = tc ? A.opt.tc_group2_rows : A.opt.group2_rows;
    const int group4 = g4opt > 0 ? g4opt : kGroup4Rows;
    const int group2 = g2opt > 0 ? g2opt : 0;
    for (int L = 0; L < S.num_levels; ++L) {
        const int* lb = S.level_list.data() + S.level_ptr[L];
        const int* le = S.level_list.data() + S.level_ptr[L + 1];
        long long f0 = static_cast<long long>(items.size());
        for (const int* p = lb; p < le; ++p) {
            const int s = *p;
            const int w = S.sn_first[s + 1] - S.sn_first[s];
            const int m = S.sn_rows[s];
            const bool kids = S.child_ptr[s + 1] > S.child_ptr[s];
            const int c0 = kids ? 0 : w;  // without children only the CB needs zeroing
            for (int c = c0 - (c0 % kEaCols); c < m; c += kEaCols)
                if (kids || m > w) items.push_back({s, c, 0, 0});
        }
        push(K_EXTEND_ADD, f0);
        f0 = static_cast<long long>(items.size());
        std::vector<int> large;
        for (const int* p = lb; p < le; ++p) {
            if (S.sn_rows[*p] <= A.opt.small_front)
                items.push_back({*p, 0, 0, 0});
            else
                large.push_back(*p);
        }
        push(K_SMALL, f0);
        int maxw = 0;
        for (int s : large) maxw = std::max(maxw, S.sn_first[s + 1] - S.sn_first[s]);
        auto width = [&](int s) { return S.sn_first[s + 1] - S.sn_first[s]; };
        for (int k0 = 0; k0 < maxw; k0 += kStep) {
            f0 = static_cast<long long>(items.size());
            for (int s : large)
                if (k0 < width(s)) items.push_back({s, k0, 0, 0});
            push(K_DIAG, f0);
            f0 = static_cast<long long>(items.size());
            for (int s : large) {
                const int w = width(s);
                if (k0 >= w) continue;
                const int k1 = std::min(w, k0 + kStep);
                for (int r = k1; r < S.sn_rows[s]; r += kTrsmRows) items.push_back({s, k0, r, 0});
            }
            push(K_TRSM, f0);
            f0 = static_cast<long long>(items.size());
            for (int s : large) {
                const int w = width(s);
                if (k0 >= w) continue;
                const int k1 = std::min(w, k0 + kStep);
                const int m = S.sn_rows[s];
                const int jend = std::min(w, (k0 / kTcPanel) * kTcPanel + kTcPanel);
                if (panel_wide) {
                    for (int j = k1; j < jend; j += kTcN)
                        for (int i = k1; i < m; i += kTcM)
                            if (i + kTcM > j) items.push_back({s, k0, i, j});
                } else {
                    for (int j = k1; j < jend; j += kTile)
                        for (int i = j; i < m; i += kTile) items.push_back({s, k0, i, j});
                }
            }
            push(K_UPDATE_PANEL, f0, panel_wide ? kStep : kTcPanel, panel_wide ? 1 : 0);
            // A panel's trailing update follows its last 32-column step. Tiles
            // cover rows and columns [pe, jend) x ..., lower part only.
            // One launch per K cap: a group's last panel applies the whole group.
            for (int cap_group : {1, 2, 4}) {
                f0 = static_cast<long long>(items.size());
                struct SplitFront {
                    int s, p0, pe, d;
                };
                std::vector<SplitFront> split_fronts;
                long long region = 0;
                auto count_since = [&](long long first) { return static_cast<long long>(items.size()) - first; };
                for (int s : large) {
                    const int w = width(s);
                    if (k0 >= w) continue;
                    const bool panel_done = (k0 + kStep) % kTcPanel == 0 || k0 + kStep >= w;
                    if (!panel_done) continue;
                    const int m = S.sn_rows[s];
                    const int G = m >= group4 ? 4 : (m >= group2 ? 2 : 1);
                    const int q = (k0 / kTcPanel) % G;        // the panel's place in its group
                    int p0 = (k0 / kTcPanel) * kTcPanel;
                    const int pe = std::min(w, p0 + kTcPanel);
                    const int g0 = p0 - q * kTcPanel;         // the group's first column
                    const bool full = g0 + G * kTcPanel <= w;
                    const bool last = full && q == G - 1;
                    if ((last ? G : 1) != cap_group) continue;
                    int jend = m;
                    if (full && !last) jend = g0 + G * kTcPanel;  // the group's remaining columns
                    if (last) p0 = g0;                            // all of the group's panels
                    const long long before = static_cast<long long>(items.size());
                    for (int j = pe; j < jend; j += kTcN)
                        for (int i = pe; i < m; i += kTcM)
                            if (i + kTcM > j) items.push_back({s, p0, i, j});
                    if (staged && static_cast<long long>(items.size()) > before) {
                        // The front's trailing operands (rows [pe, m), the group's K
                        // columns) prepared once for all of its tiles, in a region of
                        // the launch's workspace (R = m - pe rounded up to 128):
                        //  tensor-core plan: split into TF32 planes, 10 planes x
                        //    8-column stages x R rows, 32 bytes per row and stage;
                        //  FP64 plan: W = L D, R x K complex128, column-major.
                        const int K = std::min(cap_group * kTcPanel, w - p0);
                        const long long R = (m - pe + kTcM - 1) / kTcM * kTcM;
                        const long long units = trailing == K_UPDATE_TC ? ((K + kTcK - 1) / kTcK) * kTcPlanes * R / 8
                                                                        : R * K / 16;
                        for (long long t = before; t < static_cast<long long>(items.size()); ++t)
                            items[t].d = static_cast<int>(region);
                        split_fronts.push_back({s, p0, pe, static_cast<int>(region)});
                        region += units;
                        if (region > 0x7fffffffLL)
                            throw Error(APHI_ERR_BAD_SHAPE, "the prepared operands of one launch exceed 512 GiB");
                    }
                }
                if (staged && count_since(f0) > 0) {
                    // The operand launch of every front of the launch runs just before it.
                    std::vector<Item> upd(items.begin() + f0, items.end());
                    items.resize(f0);
                    for (const auto& sf : split_fronts) {
                        const int m = S.sn_rows[sf.s];
                        for (int r0 = 0; r0 < m - sf.pe; r0 += kTcM) items.push_back({sf.s, sf.p0, r0, 0, sf.d});
                    }
                    push(trailing == K_UPDATE_TC ? K_TC_SPLIT : K_DMMA_SCALE, f0, cap_group * kTcPanel);
                    long long& units_max = trailing == K_UPDATE_TC ? A.tc_ws_units : A.dmma_ws_units;
                    units_max = std::max(units_max, region);
                    f0 = static_cast<long long>(items.size());
                    items.insert(items.end(), upd.begin(), upd.end());
                }
                split_fronts.clear();
                region = 0;
                push(trailing, f0, cap_group * kTcPanel);
            }
        }
    }
}

// The solve plans and the statistics pass.
void build_plans(aphi_analysis& A, std::vector<Item>& items) {
    const Symbolic& S = A.S;
    build_factor_plan(A, items, K_UPDATE_WIDE, A.plan_factor);
    build_factor_plan(A, items, K_UPDATE_TC, A.plan_factor_tc);
    // Statistics pass over the panels: 32 columns per item.
    {
        const long long f0 = static_cast<long long>(items.size());
        for (int s = 0; s < S.ns; ++s)
            for (int c = S.sn_first[s]; c < S.sn_first[s + 1]; c += 32) items.push_back({s, c - S.sn_first[s], 0, 0});
        A.stat_first = f0;
        A.stat_count = static_cast<int>(items.size() - f0);
    }
    // Solves. Forward, levels bottom-up: gather, then per 64-column block the
    // triangle and the rows below. Backward, levels top-down, blocks last to
    // first: partial sums over row chunks, then the triangle.
    //
    // Two forms of each. The split plans give every triangle a launch of its
    // own. The fused plans (wide = 1, the ones the solves run) fold each
    // triangle into the launch before it: the gather's CTA solves its
    // supernode's first block; of the CTAs updating the rows below block blk
    // (forward), the last to finish (a per-supernode arrival counter) solves
    // block blk + 1, whose rows they have just updated; of the CTAs forming
    // block blk's backward partial sums, the last reduces them and solves
    // block blk. A backward block with no rows below gets one empty chunk, so
    // that a CTA exists to solve it. Fused backward items carry the block's
    // first partial slot in d; the chunk count follows from the shape.
    auto nblocks = [&](int s) { return (S.sn_first[s + 1] - S.sn_first[s] + kSolveBlock - 1) / kSolveBlock; };
    auto below_of = [&](int s, int blk) { return std::min(S.sn_first[s + 1] - S.sn_first[s], (blk + 1) * kSolveBlock); };
    auto pushw = [&](std::vector<Launch>& plan, int kind, long long first, int wide) {
        const int count = static_cast<int>(items.size() - first);
        if (count > 0) plan.push_back({kind, first, count, kTcPanel, wide});
    };
    for (int fused = 0; fused < 2; ++fused) {
        std::vector<Launch>& fwd = fused ? A.plan_fwd : A.plan_fwd_split;
        for (int L = 0; L < S.num_levels; ++L) {
            const int* lb = S.level_list.data() + S.level_ptr[L];
            const int* le = S.level_list.data() + S.level_ptr[L + 1];
            long long f0 = static_cast<long long>(items.size());
            int maxb = 0;
            for (const int* p = lb; p < le; ++p) {
                items.push_back({*p, 0, 0, 0});
                maxb = std::max(maxb, nblocks(*p));
            }
            pushw(fwd, K_FWD_GATHER, f0, fused);
            for (int blk = 0; blk < maxb; ++blk) {
                if (!fused) {
                    f0 = static_cast<long long>(items.size());
                    for (const int* p = lb; p < le; ++p)
                        if (blk < nblocks(*p)) items.push_back({*p, blk, 0, 0});
                    pushw(fwd, K_FWD_DIAG, f0, 0);
                }
                f0 = static_cast<long long>(items.size());
                for (const int* p = lb; p < le; ++p) {
                    const int s = *p;
                    if (blk >= nblocks(s)) continue;
                    for (int r = below_of(s, blk); r < S.sn_rows[s]; r += kSolveRows) items.push_back({s, blk, r, 0});
                }
                pushw(fwd, K_FWD_UPDATE, f0, fused);
            }
        }
    }
    A.max_parts = 1;
    for (int fused = 0; fused < 2; ++fused) {
        std::vector<Launch>& bwd = fused ? A.plan_bwd : A.plan_bwd_split;
        for (int L = S.num_levels - 1; L >= 0; --L) {
            const int* lb = S.level_list.data() + S.level_ptr[L];
            const int* le = S.level_list.data() + S.level_ptr[L + 1];
            int maxb = 0;
            for (const int* p = lb; p < le; ++p) maxb = std::max(maxb, nblocks(*p));
            for (int blk = maxb - 1; blk >= 0; --blk) {
                long long f0 = static_cast<long long>(items.size());
                std::vector<std::pair<int, int>> slots;  // per supernode of this launch: first slot, count
                int slot = 0;
                for (const int* p = lb; p < le; ++p) {
                    const int s = *p;
                    if (blk >= nblocks(s)) continue;
                    const int first = slot;
                    for (int r = below_of(s, blk); r < S.sn_rows[s]; r += kSolveRows)
                        items.push_back({s, blk, r, slot++, first});
                    if (fused && slot == first) items.push_back({s, blk, S.sn_rows[s], slot++, first});
                    slots.push_back({first, slot - first});
                }
                A.max_parts = std::max(A.max_parts, slot);
                pushw(bwd, K_BWD_UPDATE, f0, fused);
                if (fused) continue;
                f0 = static_cast<long long>(items.size());
                int q = 0;
                for (const int* p = lb; p < le; ++p) {
                    if (blk >= nblocks(*p)) continue;
                    items.push_back({*p, blk, slots[q].first, slots[q].second});
                    ++q;
                }
                pushw(bwd, K_BWD_DIAG, f0, 0);
            }
        }
    }
}

}  // namespace

aphi_analysis* analysis_create(int n, const int* row_ptr, const int* col_idx, const int* perm,
                               const int* parent, const int* col_count, const aphi_analysis_options& o) {
    auto* A = new aphi_analysis;
    try {
        A->opt = o;
        if (A->opt.small_front < 1) A->opt.small_front = 1;
        if (A->opt.small_front > 96) A->opt.small_front = 96;
        A->S = analyze_supernodal(n, row_ptr, col_idx, perm, parent, col_count, A->opt);
        const Symbolic& S = A->S;
        build_plans(*A, A->h_items);
        A->num_items = static_cast<long long>(A->h_items.size());
        A->h_uoff.assign(S.ns + 1, 0);
        for (int s = 0; s < S.ns; ++s)
            A->h_uoff[s + 1] = A->h_uoff[s] + (S.sn_rows[s] - (S.sn_first[s + 1] - S.sn_first[s]));
        A->upool = A->h_uoff[S.ns];
        A->h_row_ptr.assign(row_ptr, row_ptr + n + 1);
        A->h_col_idx.assign(col_idx, col_idx + row_ptr[n]);
        // Both triangles, for the residual's SpMV: row r lists its upper entries
        // then the mirrors of the entries above it, in a fixed order.
        A->h_fptr.assign(n + 1, 0);
        for (int r = 0; r < n; ++r)
            for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
                ++A->h_fptr[r + 1];
                if (col_idx[k] != r) ++A->h_fptr[col_idx[k] + 1];
            }
        for (int r = 0; r < n; ++r) A->h_fptr[r + 1] += A->h_fptr[r];
        A->h_fcol.resize(A->h_fptr[n]);
        A->h_fmap.resize(A->h_fptr[n]);
        {
            std::vector<int> cur(A->h_fptr.begin(), A->h_fptr.end() - 1);
            for (int r = 0; r < n; ++r)
                for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
                    const int c = col_idx[k];
                    A->h_fcol[cur[r]] = c;
                    A->h_fmap[cur[r]++] = k;
                    if (c != r) {
                        A->h_fcol[cur[c]] = r;
                        A->h_fmap[cur[c]++] = k;
                    }
                }
        }
    } catch (...) {
        delete A;
        throw;
    }
    return A;
}

aphi_analysis* analysis_create_fronts(int count, const int* rows, const int* widths, const aphi_analysis_options& o) {
    auto* A = new aphi_analysis;
    try {
        A->opt = o;
        if (A->opt.small_front < 1) A->opt.small_front = 1;
        if (A->opt.small_front > 96) A->opt.small_front = 96;
        A->S = fronts_symbolic(count, rows, widths);
        A->fronts = true;
        build_plans(*A, A->h_items);
        A->num_items = static_cast<long long>(A->h_items.size());
        const Symbolic& S = A->S;
        A->h_uoff.assign(S.ns + 1, 0);
        for (int s = 0; s < S.ns; ++s)
            A->h_uoff[s + 1] = A->h_uoff[s] + (S.sn_rows[s] - (S.sn_first[s + 1] - S.sn_first[s]));
        A->upool = A->h_uoff[S.ns];
        A->h_row_ptr.assign(S.n + 1, 0);
        A->h_fptr.assign(S.n + 1, 0);
    } catch (...) {
        delete A;
        throw;
    }
    return A;
}

void analysis_destroy(aphi_analysis* a) { delete a; }

// Device copies are made when the first factor is created, so an analysis can
// be built and inspected on a host without a GPU.
void analysis_ensure_device(aphi_analysis* A) {
    int dev = 0;
    APHI_CUDA(cudaGetDevice(&dev));
    if (A->on_device) {
        if (dev != A->device)
            throw Error(APHI_ERR_INVALID, "the analysis's device copy lives on device " + std::to_string(A->device) +
                                              ", but device " + std::to_string(dev) + " is current");
        return;
    }
    const Symbolic& S = A->S;
    long long& b = A->device_bytes;
    DeviceSchedule& d = A->d;
    d.first = upload(S.sn_first, b);
    d.rows = upload(S.sn_rows, b);
    d.loff = upload(S.sn_loff, b);
    d.cboff = upload(S.sn_cboff, b);
    d.soff = upload(S.sn_struct_off, b);
    d.structs = upload(S.structs, b);
    d.reloff = upload(S.rel_off, b);
    d.rel = upload(S.rel, b);
    d.child_ptr = upload(S.child_ptr, b);
    d.child_list = upload(S.child_list, b);
    d.uoff = upload(A->h_uoff, b);
    d.a_dest = upload(S.a_dest, b);
    d.row_ptr = upload(A->h_row_ptr, b);
    d.col_idx = upload(A->h_col_idx, b);
    d.new_of_orig = upload(S.new_of_orig, b);
    d.orig_of_new = upload(S.orig_of_new, b);
    d.ref_of_post = upload(S.ref_of_post, b);
    d.fptr = upload(A->h_fptr, b);
    d.fcol = upload(A->h_fcol, b);
    d.fmap = upload(A->h_fmap, b);
    d.items = upload(A->h_items, b);
    A->device = dev;
    A->on_device = true;
}

const Symbolic& analysis_symbolic(const aphi_analysis* a) { return a->S; }

void analysis_info(const aphi_analysis* a, double* info) {
    const Symbolic& S = a->S;
    info[0] = S.n;
    info[1] = static_cast<double>(S.nnz_a);
    info[2] = static_cast<double>(S.nnz_l);
    info[3] = static_cast<double>(S.stored);
    info[4] = S.ns;
    info[5] = S.num_levels;
    info[6] = S.max_rows;
    info[7] = S.max_width;
    info[8] = S.flops;
    info[9] = static_cast<double>(S.cb_pool);
    info[10] = static_cast<double>((S.stored + S.cb_pool) * 16);
    info[11] = S.num_roots;
}

}  // namespace aphi_b200

aphi_analysis::~aphi_analysis() {
    for (void* w : ws)
        if (w) cudaFree(w);
    void* ptrs[] = {d.first, d.rows, d.loff, d.cboff, d.soff, d.structs, d.reloff, d.rel, d.child_ptr,
                    d.child_list, d.uoff, d.a_dest, d.row_ptr, d.col_idx, d.new_of_orig, d.orig_of_new,
                    d.ref_of_post, d.fptr, d.fcol, d.fmap, d.items};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}
