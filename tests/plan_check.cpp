// Replays the factorization and solve plans of an analysis on the host,
// without a GPU: every launch, item by item, with the arithmetic of its kernel
// (hybrid-aphi-solver_b200/csrc/factor_kernels.cuh) restated sequentially in
// FP64. Items of one launch run concurrently on the device, so each access to
// the factor panels, the contribution-block (CB) pool and the solve vectors is
// checked:
//   - it stays inside the front (or update segment) the item works on;
//   - no entry is written by two items of one launch, and none is written by
//     one item and read by another;
//   - a CB entry that is read still holds the data of the front it belongs to
//     (no other block was placed over it while it was live).
// The result is compared with the oracle (or_factorize / or_solve: the
// reference's up-looking LDL^T restated) on a random complex-symmetric,
// diagonally dominant system on the workload's pattern; for independent dense
// fronts, with a dense LDL^T of each front written out here.
//
// Test infrastructure: built by oracle/Makefile (twice: with the production
// panel-group threshold and with a lowered one), run by
// tests/test_plan_check.py.
//
//   plan_check cylinder <cells> [mistake] | torus <cells> [mistake]
//   plan_check fronts <seed> <count> <max_rows>
//   plan_check pattern <diag|dense|arrow|blocks|band|random> <n> <seed> [natural]
//
// With [mistake] (overlap, dup, rel, kcap: see plant_mistake) the plan is
// corrupted first, and the checks must fail.
// Prints one line of counts and errors; exit status 0 when every check holds.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "analysis.hpp"
#include "ordering.hpp"
#include "workload.hpp"
extern "C" {
#include "oracle.h"
}


using namespace aphi_b200;
using C = std::complex<double>;

namespace {

// One tracked array: values plus, per entry, the launch and item that last
// wrote and read it, and the front whose data it holds (CB pool only).
struct Mem {
    const char* name;
    std::vector<C> v;
    std::vector<int> wl, wi, rl, ri, owner;
    Mem(const char* nm, long long n)
        : name(nm), v(n), wl(n, -1), wi(n, -1), rl(n, -1), ri(n, -1), owner(n, -1) {}
};

struct Checker {
    int launch = 0, item = 0;
    const char* kind = "";
    long long bounds = 0, ww = 0, rw = 0, stale = 0, launches = 0, items = 0;
    int shown = 0;

    void report(const char* what, const char* arr, long long k, const std::string& more = "") {
        if (shown++ < 12)
            std::fprintf(stderr, "%s: %s[%lld], launch %d (%s), item %d %s\n", what, arr, k, launch, kind, item,
                         more.c_str());
    }
    bool inside(const Mem& m, long long k, long long lo, long long hi) {
        if (k >= lo && k < hi && k >= 0 && k < static_cast<long long>(m.v.size())) return true;
        ++bounds;
        report("out of bounds", m.name, k, "[" + std::to_string(lo) + ", " + std::to_string(hi) + ")");
        return false;
    }
    C rd(Mem& m, long long k, long long lo, long long hi, int own = -1) {
        if (!inside(m, k, lo, hi)) return 0.0;
        if (m.wl[k] == launch && m.wi[k] != item) {
            ++rw;
            report("read of an entry another item of the launch writes", m.name, k);
        }
        if (m.rl[k] == launch) {
            if (m.ri[k] != item) m.ri[k] = -2;  // several readers
        } else {
            m.rl[k] = launch;
            m.ri[k] = item;
        }
        if (own >= 0 && m.owner[k] != own) {
            ++stale;
            report("CB entry does not hold its front's data", m.name, k,
                   "(front " + std::to_string(own) + ", holds " + std::to_string(m.owner[k]) + ")");
        }
        return m.v[k];
    }
    void wr(Mem& m, long long k, C x, long long lo, long long hi, int own = -1) {
        if (!inside(m, k, lo, hi)) return;
        if (m.wl[k] == launch && m.wi[k] != item) {
            ++ww;
            report("entry written by two items of one launch", m.name, k);
        }
        if (m.rl[k] == launch && m.ri[k] != item) {
            ++rw;
            report("write of an entry another item of the launch reads", m.name, k);
        }
        m.wl[k] = launch;
        m.wi[k] = item;
        m.owner[k] = own;
        m.v[k] = x;
    }
};

// The fronts of one factorization: panel entries in L, CB entries in the pool.
struct Fronts {
    const Symbolic& S;
    Checker& ck;
    Mem L, CB;
    Fronts(const Symbolic& s, Checker& c)
        : S(s), ck(c), L("L", std::max<long long>(s.stored, 1)), CB("CB", std::max<long long>(s.cb_pool, 1)) {}

    int width(int s) const { return S.sn_first[s + 1] - S.sn_first[s]; }
    int rows(int s) const { return S.sn_rows[s]; }
    // Entry (i, j), i >= j, of front s.
    C get(int s, int i, int j) {
        const int w = width(s), m = rows(s);
        if (i < j || i >= m || j < 0) {
            ++ck.bounds;
            ck.report("entry outside the front's lower triangle", "front", s);
            return 0.0;
        }
        if (j < w) return ck.rd(L, S.sn_loff[s] + i + static_cast<long long>(j) * m, S.sn_loff[s],
                                S.sn_loff[s] + static_cast<long long>(m) * w);
        const long long cs = m - w, b = S.sn_cboff[s];
        return ck.rd(CB, b + (i - w) + (j - w) * cs, b, b + cs * cs, s);
    }
    void put(int s, int i, int j, C x) {
        const int w = width(s), m = rows(s);
        if (i < j || i >= m || j < 0) {
            ++ck.bounds;
            ck.report("entry outside the front's lower triangle", "front", s);
            return;
        }
        if (j < w) {
            ck.wr(L, S.sn_loff[s] + i + static_cast<long long>(j) * m, x, S.sn_loff[s],
                  S.sn_loff[s] + static_cast<long long>(m) * w);
            return;
        }
        const long long cs = m - w, b = S.sn_cboff[s];
        ck.wr(CB, b + (i - w) + (j - w) * cs, x, b, b + cs * cs, s);
    }
    // Entry (i, j) of child c's CB (CB-local indices, i >= j), as the parent reads it.
    C child(int c, int i, int j) {
        const long long cc = rows(c) - width(c), b = S.sn_cboff[c];
        return ck.rd(CB, b + i + j * cc, b, b + cc * cc, c);
    }
};

// k_extend_add: zero the CB columns in [c0, c0 + 32), then add the children's
// CB entries that land there, children in order.
void extend_add(Fronts& F, const Item& it) {
    const Symbolic& S = F.S;
    const int s = it.s, c0 = it.a, w = F.width(s), m = F.rows(s);
    const int c1 = std::min(c0 + kEaCols, m);
    for (int j = std::max(c0, w); j < c1; ++j)
        for (int i = j; i < m; ++i) F.put(s, i, j, 0.0);
    for (int t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
        const int c = S.child_list[t];
        const int cc = F.rows(c) - F.width(c);
        if (cc <= 0) continue;
        const int* rel = S.rel.data() + S.rel_off[c];
        for (int q = 1; q < cc; ++q)
            if (rel[q] <= rel[q - 1]) {
                ++F.ck.bounds;
                F.ck.report("extend-add map not increasing", "rel", S.rel_off[c] + q);
            }
        const int j0 = static_cast<int>(std::lower_bound(rel, rel + cc, c0) - rel);
        const int j1 = static_cast<int>(std::lower_bound(rel, rel + cc, c1) - rel);
        for (int j = j0; j < j1; ++j)
            for (int i = j; i < cc; ++i) {
                const C v = F.child(c, i, j);
                F.put(s, rel[i], rel[j], F.get(s, rel[i], rel[j]) + v);
            }
    }
}

// Dense lower-triangle LDL^T steps k in [k0, k1) of an nf x nf matrix held in
// `a` (column-major, leading dimension nf), as k_small_front and
// k_diag_block do: update with the unscaled column, then scale it.
void dense_steps(std::vector<C>& a, int nf, int k0, int k1) {
    for (int k = k0; k < k1; ++k) {
        const C inv = 1.0 / a[k + static_cast<size_t>(k) * nf];
        for (int j = k + 1; j < nf; ++j) {
            const C ljk = a[j + static_cast<size_t>(k) * nf] * inv;
            for (int i = j; i < nf; ++i) a[i + static_cast<size_t>(j) * nf] -= a[i + static_cast<size_t>(k) * nf] * ljk;
        }
        for (int i = k + 1; i < nf; ++i) a[i + static_cast<size_t>(k) * nf] *= inv;
    }
}

void small_front(Fronts& F, const Item& it) {
    const int s = it.s, w = F.width(s), m = F.rows(s);
    std::vector<C> a(static_cast<size_t>(m) * m);
    for (int j = 0; j < m; ++j)
        for (int i = j; i < m; ++i) a[i + static_cast<size_t>(j) * m] = F.get(s, i, j);
    dense_steps(a, m, 0, w);
    for (int j = 0; j < m; ++j)
        for (int i = j; i < m; ++i) F.put(s, i, j, a[i + static_cast<size_t>(j) * m]);
}

void diag_block(Fronts& F, const Item& it) {
    const int s = it.s, k0 = it.a, kb = std::min(kStep, F.width(s) - k0);
    std::vector<C> a(static_cast<size_t>(kb) * kb);
    for (int j = 0; j < kb; ++j)
        for (int i = j; i < kb; ++i) a[i + static_cast<size_t>(j) * kb] = F.get(s, k0 + i, k0 + j);
    dense_steps(a, kb, 0, kb);
    for (int j = 0; j < kb; ++j)
        for (int i = j; i < kb; ++i) F.put(s, k0 + i, k0 + j, a[i + static_cast<size_t>(j) * kb]);
}

// k_panel_trsm: rows row0 .. row0 + 127 of the panel below step k0's block.
void panel_trsm(Fronts& F, const Item& it) {
    const int s = it.s, k0 = it.a, row0 = it.b, m = F.rows(s);
    const int kb = std::min(kStep, F.width(s) - k0);
    std::vector<C> T(static_cast<size_t>(kb) * kb), dinv(kb);
    for (int j = 0; j < kb; ++j)
        for (int i = j; i < kb; ++i) T[i + static_cast<size_t>(j) * kb] = F.get(s, k0 + i, k0 + j);
    for (int j = 0; j < kb; ++j) dinv[j] = 1.0 / T[j + static_cast<size_t>(j) * kb];
    for (int i = row0; i < std::min(row0 + kTrsmRows, m); ++i) {
        std::vector<C> x(kb);
        for (int j = 0; j < kb; ++j) x[j] = F.get(s, i, k0 + j);
        for (int j = 0; j < kb; ++j)
            for (int t = 0; t < j; ++t) x[j] -= T[j + static_cast<size_t>(t) * kb] * x[t];
        for (int j = 0; j < kb; ++j) F.put(s, i, k0 + j, x[j] * dinv[j]);
    }
}

// Tile F[i, j] -= sum_{t < K} L[i, c + t] D[c + t] L[j, c + t] over rows
// [i0, i0 + tm) and columns [j0, min(j0 + tn, jcap)), i >= j, i < m. The
// operands are read once per tile, as the kernels stage them.
void update_tile(Fronts& F, int s, int c, int K, int i0, int j0, int tm, int tn, int jcap) {
    const int m = F.rows(s);
    const int ni = std::max(0, std::min(tm, m - i0)), nj = std::max(0, std::min(tn, m - j0));
    // Operand rows contiguous in t (row r of A at A[r * K]).
    std::vector<C> A(static_cast<size_t>(ni) * K), B(static_cast<size_t>(nj) * K), D(K);
    for (int t = 0; t < K; ++t) {
        D[t] = F.get(s, c + t, c + t);
        for (int r = 0; r < ni; ++r) A[static_cast<size_t>(r) * K + t] = F.get(s, i0 + r, c + t) * D[t];
        for (int r = 0; r < nj; ++r) B[static_cast<size_t>(r) * K + t] = F.get(s, j0 + r, c + t);
    }
    for (int b = 0; b < nj; ++b) {
        const int j = j0 + b;
        if (j >= jcap) continue;
        const C* bj = B.data() + static_cast<size_t>(b) * K;
        for (int a = 0; a < ni; ++a) {
            const int i = i0 + a;
            if (i < j) continue;
            const C* ai = A.data() + static_cast<size_t>(a) * K;
            double re = 0, im = 0;
            for (int t = 0; t < K; ++t) {
                re += ai[t].real() * bj[t].real() - ai[t].imag() * bj[t].imag();
                im += ai[t].real() * bj[t].imag() + ai[t].imag() * bj[t].real();
            }
            F.put(s, i, j, F.get(s, i, j) - C(re, im));
        }
    }
}

// The prepared-operand workspaces. A K_TC_SPLIT item writes 128 rows of
// every stage's ten planes of its front's region (tensor-core plan); a
// K_DMMA_SCALE item writes 128 rows of W = L D over the group's K columns
// (FP64 plan). The region must lie inside the per-entry workspace, the regions
// of different fronts in one launch must not overlap, and one front's items
// must agree on it. The trailing-update launch that follows reads, per tile,
// rows i0 - pe .. +127 (and, for the split planes, B rows j0 - pe .. +63) of
// its front's region: the launch just before it must be the operand launch
// that wrote those rows of that region, for the same panel group and K.
long long g_tc_ws_units = 0, g_dmma_ws_units = 0;
struct SplitFront {
    long long d, units;
    int p0, K;
    std::vector<char> rows;  // 128-row blocks written
};
std::map<int, SplitFront> g_split;
int g_split_launch = -1;  // ck.launch of the last operand launch

void operand_region(Fronts& F, const Launch& l, const Item& it, int w) {
    const int m = F.rows(it.s);
    const int K = std::min(l.kcap, w - it.a), pe = it.a + K;
    const long long R = (m - pe + kTcM - 1) / kTcM * kTcM;
    const bool tc = l.kind == K_TC_SPLIT;
    const long long units = tc ? ((K + kTcK - 1) / kTcK) * kTcPlanes * R / 8 : R * K / 16;
    const long long cap = tc ? g_tc_ws_units : g_dmma_ws_units;
    if (it.d < 0 || it.d + units > cap || it.b < 0 || it.b >= R || it.b % kTcM) {
        ++F.ck.bounds;
        F.ck.report("operand region outside the workspace", "d", it.d);
        return;
    }
    auto found = g_split.find(it.s);
    if (found == g_split.end()) {
        for (const auto& kv : g_split)
            if (it.d < kv.second.d + kv.second.units && kv.second.d < it.d + units) {
                ++F.ck.ww;
                F.ck.report("operand regions of two fronts overlap", "d", it.d);
            }
        found = g_split.emplace(it.s, SplitFront{it.d, units, it.a, K, std::vector<char>(R / kTcM, 0)}).first;
    } else if (found->second.d != it.d || found->second.p0 != it.a) {
        ++F.ck.bounds;
        F.ck.report("operand items of one front disagree on the region", "d", it.d);
        return;
    }
    char& blk = found->second.rows[it.b / kTcM];
    if (blk) {
        ++F.ck.ww;
        F.ck.report("operand row block written twice", "row", it.b);
    }
    blk = 1;
}

// A trailing-update tile of a plan with operand launches reads only rows that
// the operand launch just before it wrote (B rows too for the split planes).
void tile_region(Fronts& F, const Launch& l, const Item& it, int w) {
    const int K = std::min(l.kcap, w - it.a), pe = it.a + K;
    const auto found = g_split.find(it.s);
    const bool fresh = g_split_launch == F.ck.launch - 1;
    bool ok = fresh && found != g_split.end() && found->second.d == it.d && found->second.p0 == it.a &&
              found->second.K == K;
    if (ok) {
        const std::vector<char>& rows = found->second.rows;
        const int ia = (it.b - pe) / kTcM, jb = (it.c - pe) / kTcM;
        ok = it.b >= pe && it.c >= pe && ia < static_cast<int>(rows.size()) && rows[ia] &&
             (l.kind != K_UPDATE_TC || (jb < static_cast<int>(rows.size()) && rows[jb]));
    }
    if (!ok) {
        ++F.ck.rw;
        F.ck.report("trailing tile reads operands its operand launch did not write", "row", it.b);
    }
}

void run_factor_plan(Fronts& F, const std::vector<Launch>& plan, const std::vector<Item>& items) {
    static const char* names[] = {"extend_add", "small", "diag", "trsm", "update_wide", "", "", "", "", "",
                                  "update_panel", "update_tc", "tc_split", "dmma_scale"};
    Checker& ck = F.ck;
    auto has = [&](int kind) {
        return std::any_of(plan.begin(), plan.end(), [&](const Launch& l) { return l.kind == kind; });
    };
    const bool presplit = has(K_TC_SPLIT), prescaled = has(K_DMMA_SCALE);
    g_split.clear();
    g_split_launch = -1;
    for (const Launch& l : plan) {
        ++ck.launch;
        ++ck.launches;
        ck.kind = l.kind >= 0 && l.kind < 14 ? names[l.kind] : "?";
        if (l.kind == K_TC_SPLIT || l.kind == K_DMMA_SCALE) {
            g_split.clear();
            g_split_launch = ck.launch;
        }
        for (int q = 0; q < l.count; ++q) {
            ck.item = q;
            ++ck.items;
            const Item& it = items[l.first + q];
            const int w = F.width(it.s);
            switch (l.kind) {
                case K_EXTEND_ADD: extend_add(F, it); break;
                case K_SMALL: small_front(F, it); break;
                case K_DIAG: diag_block(F, it); break;
                case K_TRSM: panel_trsm(F, it); break;
                case K_UPDATE_PANEL: {
                    const int k0 = it.a, kb = std::min(kStep, w - k0);
                    const int jend = std::min(w, (k0 / kTcPanel) * kTcPanel + kTcPanel);
                    if (l.wide)  // on the trailing-update kernel: 128 x 64, K = min(kcap, w - k0)
                        update_tile(F, it.s, k0, std::min(l.kcap, w - k0), it.b, it.c, kTcM, kTcN, jend);
                    else
                        update_tile(F, it.s, k0, kb, it.b, it.c, kTile, kTile, jend);
                    break;
                }
                case K_UPDATE_WIDE:
                case K_UPDATE_TC: {
                    const int K = std::min(l.kcap, w - it.a);
                    if ((l.kind == K_UPDATE_TC && presplit) || (l.kind == K_UPDATE_WIDE && prescaled))
                        tile_region(F, l, it, w);
                    update_tile(F, it.s, it.a, K, it.b, it.c, kTcM, kTcN, F.rows(it.s));
                    break;
                }
                case K_TC_SPLIT:
                case K_DMMA_SCALE:
                    // The panel group's operands prepared in the workspace: the
                    // arithmetic is the tiles' (update_tile). The region must lie
                    // inside the analysis's per-entry workspace.
                    operand_region(F, l, it, w);
                    break;
                default:
                    ++ck.bounds;
                    ck.report("unexpected kind in a factor plan", "plan", l.kind);
            }
        }
    }
}

// The solve plans on one right-hand side: y (post-ordered), U (update
// segments), part (partial sums of the backward updates).
struct SolveMem {
    Mem y, U, part;
    SolveMem(long long n, long long upool, long long parts)
        : y("y", std::max<long long>(n, 1)), U("U", std::max<long long>(upool, 1)),
          part("part", std::max<long long>(parts * kSolveBlock * 8, 1)) {}
};

void run_solve_plan(const aphi_analysis& A, Fronts& F, SolveMem& V, const std::vector<Launch>& plan) {
    const Symbolic& S = A.S;
    Checker& ck = F.ck;
    const long long n = S.n;
    auto Lv = [&](int s, int i, int j) { return F.L.v[S.sn_loff[s] + i + static_cast<long long>(j) * S.sn_rows[s]]; };
    auto nblocks = [&](int s) { return (F.width(s) + kSolveBlock - 1) / kSolveBlock; };
    auto gather = [&](int s) {
        const int w = F.width(s), f = S.sn_first[s];
        const long long us = A.h_uoff[s], ue = A.h_uoff[s + 1];
        for (long long i = us; i < ue; ++i) ck.wr(V.U, i, 0.0, us, ue);
        for (int t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
            const int c = S.child_list[t];
            const int cc = F.rows(c) - F.width(c);
            const int* rel = S.rel.data() + S.rel_off[c];
            const long long uc = A.h_uoff[c];
            for (int i = 0; i < cc; ++i) {
                const C v = ck.rd(V.U, uc + i, uc, uc + cc);
                if (rel[i] < w) ck.wr(V.y, f + rel[i], ck.rd(V.y, f + rel[i], f, f + w) + v, f, f + w);
                else ck.wr(V.U, us + rel[i] - w, ck.rd(V.U, us + rel[i] - w, us, ue) + v, us, ue);
            }
        }
    };
    auto fdiag = [&](int s, int blk) {
        const int w = F.width(s), f = S.sn_first[s];
        const int j0 = blk * kSolveBlock, jb = std::min(kSolveBlock, w - j0);
        std::vector<C> ys(jb);
        for (int i = 0; i < jb; ++i) ys[i] = ck.rd(V.y, f + j0 + i, f, f + w);
        for (int j = 0; j < jb; ++j)
            for (int i = j + 1; i < jb; ++i) ys[i] -= Lv(s, j0 + i, j0 + j) * ys[j];
        for (int i = 0; i < jb; ++i) ck.wr(V.y, f + j0 + i, ys[i], f, f + w);
    };
    auto fupd = [&](const Item& it) {
        const int s = it.s, w = F.width(s), m = F.rows(s), f = S.sn_first[s];
        const long long us = A.h_uoff[s], ue = A.h_uoff[s + 1];
        const int j0 = it.a * kSolveBlock, jb = std::min(kSolveBlock, w - j0);
        std::vector<C> ys(jb);
        for (int j = 0; j < jb; ++j) ys[j] = ck.rd(V.y, f + j0 + j, f, f + w);
        const int r0 = it.b, r1 = std::min(it.b + kSolveRows, m);
        std::vector<C> acc(std::max(r1 - r0, 0), 0.0);  // each row's sum in column order
        for (int j = 0; j < jb; ++j)
            for (int r = r0; r < r1; ++r) acc[r - r0] += Lv(s, r, j0 + j) * ys[j];
        for (int r = r0; r < r1; ++r) {
            if (r < w) ck.wr(V.y, f + r, ck.rd(V.y, f + r, f, f + w) - acc[r - r0], f, f + w);
            else ck.wr(V.U, us + r - w, ck.rd(V.U, us + r - w, us, ue) - acc[r - r0], us, ue);
        }
    };
    auto bupd = [&](const Item& it) {
        const int s = it.s, w = F.width(s), m = F.rows(s), f = S.sn_first[s];
        const int j0 = it.a * kSolveBlock, jb = std::min(kSolveBlock, w - j0);
        const int row0 = it.b, slot = it.c, nrows = std::max(0, std::min(kSolveRows, m - row0));
        const int* st = S.structs.data() + S.sn_struct_off[s];
        std::vector<C> xs(nrows);
        for (int t = 0; t < nrows; ++t) {
            const int r = row0 + t;
            xs[t] = ck.rd(V.y, r < w ? f + r : st[r], 0, n);
        }
        const long long pb = static_cast<long long>(slot) * kSolveBlock * 8;
        for (int j = 0; j < jb; ++j) {
            C acc = 0.0;
            for (int t = 0; t < nrows; ++t) acc += Lv(s, row0 + t, j0 + j) * xs[t];
            ck.wr(V.part, pb + j * 8, acc, pb, pb + kSolveBlock * 8);
        }
    };
    auto bdiag = [&](int s, int blk, int p0, int np) {
        const int w = F.width(s), f = S.sn_first[s];
        const int j0 = blk * kSolveBlock, jb = std::min(kSolveBlock, w - j0);
        std::vector<C> z(jb);
        for (int j = 0; j < jb; ++j) {
            C sum = 0.0;
            for (int qq = 0; qq < np; ++qq) {
                const long long pb = static_cast<long long>(p0 + qq) * kSolveBlock * 8;
                sum += ck.rd(V.part, pb + j * 8, pb, pb + kSolveBlock * 8);
            }
            z[j] = ck.rd(V.y, f + j0 + j, f, f + w) / Lv(s, j0 + j, j0 + j) - sum;
        }
        for (int j = jb - 1; j >= 0; --j)
            for (int t = 0; t < j; ++t) z[t] -= Lv(s, j0 + j, j0 + t) * z[j];
        for (int j = 0; j < jb; ++j) ck.wr(V.y, f + j0 + j, z[j], f, f + w);
    };
    // The chunk count a fused kernel expects for (s, blk): its CTAs' arrivals.
    auto chunks = [&](int s, int blk, bool backward) {
        const int below = std::min(F.width(s), (blk + 1) * kSolveBlock);
        const int c = (F.rows(s) - below + kSolveRows - 1) / kSolveRows;
        return backward ? std::max(1, c) : c;
    };
    for (const Launch& l : plan) {
        ++ck.launch;
        ++ck.launches;
        ck.kind = l.wide ? "solve (fused)" : "solve";
        struct Arrivals {
            int blk = -1, count = 0, p0 = -1;
            std::vector<int> slots;
        };
        std::map<int, Arrivals> arrived;  // fused launches: per supernode
        for (int q = 0; q < l.count; ++q) {
            ck.item = q;
            ++ck.items;
            const Item& it = A.h_items[l.first + q];
            if (l.wide && l.kind != K_FWD_GATHER) {
                Arrivals& ar = arrived[it.s];
                if (ar.count > 0 && (ar.blk != it.a || (l.kind == K_BWD_UPDATE && ar.p0 != it.d))) {
                    ++ck.bounds;
                    ck.report("fused solve items of one supernode disagree on the block or first slot", "s", it.s);
                }
                ar.blk = it.a;
                ar.p0 = it.d;
                ++ar.count;
                ar.slots.push_back(it.c);
            }
            switch (l.kind) {
                case K_FWD_GATHER:
                    gather(it.s);
                    if (l.wide) fdiag(it.s, 0);  // the same CTA, after its gather
                    break;
                case K_FWD_DIAG: fdiag(it.s, it.a); break;
                case K_FWD_UPDATE: fupd(it); break;
                case K_BWD_UPDATE: bupd(it); break;
                case K_BWD_DIAG: bdiag(it.s, it.a, it.b, it.c); break;
                default:
                    ++ck.bounds;
                    ck.report("unexpected kind in a solve plan", "plan", l.kind);
            }
        }
        if (arrived.empty()) continue;
        // The last CTA of each supernode: after every other CTA of the launch
        // (a phase of its own for the race checks).
        ++ck.launch;
        ck.kind = "solve (fused, last CTA)";
        for (const auto& kv : arrived) {
            const int s = kv.first;
            const Arrivals& ar = kv.second;
            ck.item = s;
            const bool bwd = l.kind == K_BWD_UPDATE;
            if (ar.count != chunks(s, ar.blk, bwd)) {
                ++ck.bounds;
                ck.report("fused solve: the kernel's expected arrivals differ from the plan's items", "s", s);
                continue;
            }
            if (bwd) {
                std::vector<int> sl = ar.slots;
                std::sort(sl.begin(), sl.end());
                for (int k = 0; k < static_cast<int>(sl.size()); ++k)
                    if (sl[k] != ar.p0 + k) {
                        ++ck.bounds;
                        ck.report("fused backward slots are not p0 .. p0 + np - 1", "s", s);
                        break;
                    }
                bdiag(s, ar.blk, ar.p0, ar.count);
            } else if (ar.blk + 1 < nblocks(s)) {
                fdiag(s, ar.blk + 1);
            }
        }
    }
}

double rel_err(const std::vector<C>& a, const std::vector<C>& b) {
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        num = std::max(num, std::abs(a[i] - b[i]));
        den = std::max(den, std::abs(b[i]));
    }
    return den > 0 ? num / den : num;
}

// A mistake planted in this process's copy of the plan, to show that the
// checks catch it: two live CBs placed on one another ("overlap"), a tile
// updated by two items of one launch ("dup"), a child's extend-add map
// entry repeated ("rel"), a 2-panel group's trailing update cut to its last
// panel ("kcap"), a trailing tile pointed at another part of the prepared-
// operand workspace than its operand launch wrote ("region").
bool plant_mistake(aphi_analysis& A, const std::string& what) {
    Symbolic& S = A.S;
    auto cb_rows = [&](int s) { return S.sn_rows[s] - (S.sn_first[s + 1] - S.sn_first[s]); };
    if (what == "overlap") {
        for (int L = 0; L < S.num_levels; ++L) {
            int first = -1;
            for (int k = S.level_ptr[L]; k < S.level_ptr[L + 1]; ++k) {
                const int s = S.level_list[k];
                if (cb_rows(s) <= 0) continue;
                if (first < 0) {
                    first = s;
                } else {
                    S.sn_cboff[s] = S.sn_cboff[first];
                    return true;
                }
            }
        }
    } else if (what == "dup") {
        for (const Launch& l : A.plan_factor)
            if (l.kind == K_UPDATE_WIDE && l.count >= 2) {
                A.h_items[l.first + 1] = A.h_items[l.first];
                return true;
            }
    } else if (what == "rel") {
        for (int c = 0; c < S.ns; ++c)
            if (S.sn_parent[c] >= 0 && cb_rows(c) >= 2) {
                S.rel[S.rel_off[c] + 1] = S.rel[S.rel_off[c]];
                return true;
            }
    } else if (what == "kcap") {
        for (Launch& l : A.plan_factor)
            if (l.kind == K_UPDATE_WIDE && l.kcap > kTcPanel) {
                l.kcap = kTcPanel;
                return true;
            }
    } else if (what == "region") {
        bool staged = false;  // the launch before was an operand launch
        for (const Launch& l : A.plan_factor) {
            if (l.kind == K_UPDATE_WIDE && staged) {
                A.h_items[l.first].d += 16;
                return true;
            }
            staged = l.kind == K_DMMA_SCALE;
        }
    }
    return false;
}

aphi_analysis_options default_options() {
    aphi_analysis_options o{};
    o.relax_small = 4;
    o.relax_fill = 0.05;
    o.relax_max_width = 256;
    o.small_front = 96;
    o.group4_rows = kGroup4Rows;
    o.group2_rows = 0;
    o.tc_group4_rows = kGroup4Rows;
    o.tc_group2_rows = 0;
    return o;
}

// Synthetic upper CSR patterns (diagonal in every row) for edge cases of the
// elimination tree: "diag" (no off-diagonal entry), "dense", "arrow" (every
// unknown coupled to the last), "blocks" (disconnected cliques of 1-40
// unknowns), "band" (half-bandwidth 20), "random" (0-6 later neighbours per row).
void make_pattern(const std::string& shape, int n, unsigned seed, std::vector<int>& rp, std::vector<int>& ci) {
    std::mt19937 rng(seed);
    std::vector<std::vector<int>> rows(n);
    int block_end = 0;
    for (int i = 0; i < n; ++i) {
        rows[i].push_back(i);
        if (shape == "dense") {
            for (int j = i + 1; j < n; ++j) rows[i].push_back(j);
        } else if (shape == "arrow") {
            if (i + 1 < n) rows[i].push_back(n - 1);
        } else if (shape == "blocks") {
            if (i >= block_end) block_end = std::min(n, i + 1 + static_cast<int>(rng() % 40));
            for (int j = i + 1; j < block_end; ++j) rows[i].push_back(j);
        } else if (shape == "band") {
            for (int j = i + 1; j < std::min(n, i + 21); ++j) rows[i].push_back(j);
        } else if (shape == "random") {
            const int k = static_cast<int>(rng() % 7);
            for (int q = 0; q < k && i + 1 < n; ++q) rows[i].push_back(i + 1 + static_cast<int>(rng() % (n - i - 1)));
        } else if (shape != "diag") {
            throw std::invalid_argument("unknown pattern shape " + shape);
        }
        std::sort(rows[i].begin(), rows[i].end());
        rows[i].erase(std::unique(rows[i].begin(), rows[i].end()), rows[i].end());
    }
    rp.assign(1, 0);
    ci.clear();
    for (const auto& r : rows) {
        ci.insert(ci.end(), r.begin(), r.end());
        rp.push_back(static_cast<int>(ci.size()));
    }
}

int check_matrix(int n, const std::vector<int>& rp, const std::vector<int>& ci, bool natural,
                 const std::string& plant) {
    std::vector<int> perm(n);
    if (natural)
        for (int i = 0; i < n; ++i) perm[i] = i;
    else
        reference_amd(n, rp.data(), ci.data(), perm.data());
    aphi_analysis* A = analysis_create(n, rp.data(), ci.data(), perm.data(), nullptr, nullptr, default_options());
    const Symbolic& S = A->S;
    if (!plant.empty()) {
        if (!plant_mistake(*A, plant)) {
            std::printf("nothing to plant: %s\n", plant.c_str());
            analysis_destroy(A);
            return 2;
        }
        std::printf("planted %s ", plant.c_str());
    }
    // Random complex-symmetric values, diagonally dominant (no pivoting needed).
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    const long long nnz = rp[n];
    std::vector<double> vals(2 * nnz);
    std::vector<double> rowsum(n, 0.0);
    for (int r = 0; r < n; ++r)
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            if (ci[k] != r) {
                vals[2 * k] = U(rng);
                vals[2 * k + 1] = U(rng);
                const double a = std::hypot(vals[2 * k], vals[2 * k + 1]);
                rowsum[r] += a;
                rowsum[ci[k]] += a;
            }
    for (int r = 0; r < n; ++r)
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            if (ci[k] == r) {
                vals[2 * k] = 2.0 * rowsum[r] + 1.0;
                vals[2 * k + 1] = 0.5 * rowsum[r] + U(rng);
            }
    std::vector<double> b(2 * static_cast<size_t>(n));
    for (auto& x : b) x = U(rng);

    // The oracle's factor and solution.
    std::vector<int> col_ptr(n + 1);
    long long nnzl = 0;
    for (int j = 0; j < n; ++j) nnzl += std::max(S.ref_colcount[j] - 1, 0);
    std::vector<int> row_index(nnzl + 1);
    std::vector<double> lvalue(2 * (nnzl + 1)), diag(2 * static_cast<size_t>(n)), stats(6), xo(2 * static_cast<size_t>(n));
    if (or_factorize(n, rp.data(), ci.data(), vals.data(), perm.data(), S.ref_parent.data(), S.ref_colcount.data(), 0.0,
                     col_ptr.data(), row_index.data(), lvalue.data(), diag.data(), stats.data()) != 0 ||
        or_solve(n, col_ptr.data(), row_index.data(), lvalue.data(), diag.data(), perm.data(), b.data(), xo.data()) != 0) {
        std::printf("oracle factorization failed\n");
        return 2;
    }
    std::vector<C> d_or(n), x_or(n), bz(n);
    for (int k = 0; k < n; ++k) {
        d_or[k] = C(diag[2 * k], diag[2 * k + 1]);
        x_or[k] = C(xo[2 * k], xo[2 * k + 1]);
        bz[k] = C(b[2 * k], b[2 * k + 1]);
    }

    // The CB pool against its lower bound: the largest total of blocks live
    // at one level (a block from its front's level to its parent's).
    {
        std::vector<long long> live(std::max(S.num_levels, 1), 0);
        for (int s = 0; s < S.ns; ++s) {
            const long long c = S.sn_rows[s] - (S.sn_first[s + 1] - S.sn_first[s]);
            if (c <= 0) continue;
            const int hi = S.sn_parent[s] >= 0 ? S.sn_level[S.sn_parent[s]] : S.sn_level[s];
            for (int L = S.sn_level[s]; L <= hi; ++L) live[L] += c * c;
        }
        std::printf("cb_pool %lld bound %lld ", S.cb_pool, *std::max_element(live.begin(), live.end()));
    }
    int bad = 0;
    g_tc_ws_units = A->tc_ws_units;
    g_dmma_ws_units = A->dmma_ws_units;
    const std::vector<Launch>* plans[2] = {&A->plan_factor, &A->plan_factor_tc};
    const char* pname[2] = {"dmma", "tc"};
    for (int p = 0; p < 2; ++p) {
        Checker ck;
        Fronts F(S, ck);
        // k_scatter_a: one item per row of A.
        ck.kind = "scatter";
        for (int r = 0; r < n; ++r) {
            ck.item = r;
            for (int k = rp[r]; k < rp[r + 1]; ++k)
                ck.wr(F.L, S.a_dest[k], C(vals[2 * k], vals[2 * k + 1]), 0, S.stored);
        }
        run_factor_plan(F, *plans[p], A->h_items);
        std::vector<C> d(n);
        for (int s = 0; s < S.ns; ++s)
            for (int j = 0; j < F.width(s); ++j)
                d[S.ref_of_post[S.sn_first[s] + j]] = F.L.v[S.sn_loff[s] + j + static_cast<long long>(j) * F.rows(s)];
        const long long f_launches = ck.launches, f_items = ck.items;
        SolveMem V(n, A->upool, A->max_parts);
        std::vector<C> x(n), x_split(n);
        for (int form = 0; form < 2; ++form) {  // the fused plans, then the split ones
            for (int i = 0; i < n; ++i) V.y.v[i] = bz[S.orig_of_new[i]];
            run_solve_plan(*A, F, V, form ? A->plan_fwd_split : A->plan_fwd);
            run_solve_plan(*A, F, V, form ? A->plan_bwd_split : A->plan_bwd);
            for (int o = 0; o < n; ++o) (form ? x_split : x)[o] = V.y.v[S.new_of_orig[o]];
        }
        const double de = rel_err(d, d_or), xe = rel_err(x, x_or);
        // The fused and split solve plans do the same arithmetic in the same order.
        const bool same = x == x_split;
        const bool ok = !ck.bounds && !ck.ww && !ck.rw && !ck.stale && de <= 1e-12 && xe <= 1e-10 && same;
        if (!same) std::printf("fused and split solve plans differ\n");
        int caps[3] = {0, 0, 0};  // trailing-update launches applying 1, 2 and 4 panels
        for (const Launch& l : *plans[p])
            if (l.kind == K_UPDATE_WIDE || l.kind == K_UPDATE_TC) ++caps[l.kcap == kTcPanel ? 0 : l.kcap == 2 * kTcPanel ? 1 : 2];
        std::printf("%s n %d supernodes %d levels %d factor launches %lld items %lld solve launches %lld "
                    "trailing 1/2/4 panels %d/%d/%d bounds %lld ww %lld rw %lld stale %lld d_err %.3e x_err %.3e %s\n",
                    pname[p], n, S.ns, S.num_levels, f_launches, f_items, ck.launches - f_launches, caps[0], caps[1],
                    caps[2], ck.bounds, ck.ww, ck.rw, ck.stale, de, xe, ok ? "ok" : "FAIL");
        bad += !ok;
    }
    analysis_destroy(A);
    return bad ? 1 : 0;
}

// Independent dense fronts (the dense-front microbenchmark's analysis):
// random panels, CBs zeroed by the plan; each front against a dense LDL^T.
int check_fronts(unsigned seed, int count, int max_rows) {
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> R(1, max_rows);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<int> rows(count), widths(count);
    for (int k = 0; k < count; ++k) {
        rows[k] = R(rng);
        widths[k] = std::uniform_int_distribution<int>(1, rows[k])(rng);
    }
    // Make sure the interesting shapes occur: a front wider than a 4-panel
    // group, and one whose width ends inside a group.
    if (count >= 2 && max_rows >= 700) {
        rows[0] = max_rows;
        widths[0] = std::min(max_rows, 4 * kTcPanel + 77);
        rows[1] = max_rows - 1;
        widths[1] = std::min(max_rows - 1, 3 * kTcPanel + 5);
    }
    aphi_analysis* A = analysis_create_fronts(count, rows.data(), widths.data(), default_options());
    const Symbolic& S = A->S;
    Checker ck;
    Fronts F(S, ck);
    std::vector<std::vector<C>> dense(S.ns);
    ck.kind = "panels";
    for (int s = 0; s < S.ns; ++s) {
        const int w = F.width(s), m = F.rows(s);
        std::vector<C>& a = dense[s];
        a.assign(static_cast<size_t>(m) * m, 0.0);
        for (int j = 0; j < w; ++j)
            for (int i = j; i < m; ++i) {
                C v(U(rng), U(rng));
                if (i == j) v = C(2.0 * m + 1.0, 0.5 * m);
                a[i + static_cast<size_t>(j) * m] = v;
                ck.wr(F.L, S.sn_loff[s] + i + static_cast<long long>(j) * m, v, 0, S.stored);
            }
    }
    g_tc_ws_units = A->tc_ws_units;
    g_dmma_ws_units = A->dmma_ws_units;
    run_factor_plan(F, A->plan_factor, A->h_items);
    double err = 0;
    for (int s = 0; s < S.ns; ++s) {
        const int w = F.width(s), m = F.rows(s);
        std::vector<C>& a = dense[s];
        dense_steps(a, m, 0, w);
        double num = 0, den = 0;
        for (int j = 0; j < m; ++j)
            for (int i = j; i < m; ++i) {
                const C got = j < w ? F.L.v[S.sn_loff[s] + i + static_cast<long long>(j) * m]
                                    : F.CB.v[S.sn_cboff[s] + (i - w) + static_cast<long long>(j - w) * (m - w)];
                num = std::max(num, std::abs(got - a[i + static_cast<size_t>(j) * m]));
                den = std::max(den, std::abs(a[i + static_cast<size_t>(j) * m]));
            }
        err = std::max(err, den > 0 ? num / den : num);
    }
    const bool ok = !ck.bounds && !ck.ww && !ck.rw && !ck.stale && err <= 1e-12;
    int maxw = 0;
    for (int k = 0; k < count; ++k) maxw = std::max(maxw, widths[k]);
    int caps[3] = {0, 0, 0};
    for (const Launch& l : A->plan_factor)
        if (l.kind == K_UPDATE_WIDE) ++caps[l.kcap == kTcPanel ? 0 : l.kcap == 2 * kTcPanel ? 1 : 2];
    std::printf("fronts %d max_width %d launches %lld items %lld trailing 1/2/4 panels %d/%d/%d bounds %lld ww %lld "
                "rw %lld stale %lld err %.3e %s\n",
                count, maxw, ck.launches, ck.items, caps[0], caps[1], caps[2], ck.bounds, ck.ww, ck.rw, ck.stale, err,
                ok ? "ok" : "FAIL");
    analysis_destroy(A);
    return ok ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if ((mode == "cylinder" || mode == "torus") && (argc == 3 || argc == 4)) {
            Workload w;
            if (mode == "cylinder") build_cylinder(w, std::atoi(argv[2]), 1.0, 0);
            else build_torus(w, std::atoi(argv[2]), 1.0);
            std::printf("group4_rows %d ", kGroup4Rows);
            return check_matrix(w.num_total, w.row_ptr, w.col_idx, false, argc == 4 ? argv[3] : "");
        }
        if (mode == "pattern" && (argc == 5 || argc == 6)) {
            std::vector<int> rp, ci;
            const int n = std::atoi(argv[3]);
            make_pattern(argv[2], n, static_cast<unsigned>(std::atoi(argv[4])), rp, ci);
            std::printf("group4_rows %d %s ", kGroup4Rows, argv[2]);
            return check_matrix(n, rp, ci, argc == 6 && std::string(argv[5]) == "natural", "");
        }
        if (mode == "fronts" && argc == 5) {
            std::printf("group4_rows %d ", kGroup4Rows);
            return check_fronts(static_cast<unsigned>(std::atoi(argv[2])), std::atoi(argv[3]), std::atoi(argv[4]));
        }
        std::fprintf(stderr,
                     "usage: %s cylinder <cells> [mistake] | torus <cells> [mistake] | fronts <seed> <count> <max_rows>"
                     " | pattern <shape> <n> <seed> [natural]\n",
                     argv[0]);
        return 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "plan_check: %s\n", e.what());
        return 2;
    }
}
