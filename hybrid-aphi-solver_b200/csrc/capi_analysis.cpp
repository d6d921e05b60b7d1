// C ABI: analysis (supernodal schedule) creation and queries.
#include "analysis.hpp"
#include "capi_util.hpp"
#include "tc_config.hpp"

#include <algorithm>

using namespace aphi_b200;

extern "C" {

void aphi_analysis_default_options(aphi_analysis_options* o) {
    if (!o) return;
    o->relax_small = 4;
    o->relax_fill = 0.05;
    o->relax_max_width = 256;
    o->small_front = 96;
    o->group4_rows = kGroup4Rows;
    o->group2_rows = 0;
    o->tc_group4_rows = kGroup4Rows;
    o->tc_group2_rows = 0;
}

int aphi_analysis_create(int n, const int* row_ptr, const int* col_idx, const int* perm, const int* parent,
                         const int* col_count, const aphi_analysis_options* opt, aphi_analysis** out) {
    return guard([&] {
        if (!out) throw Error(APHI_ERR_INVALID, "aphi_analysis_create: null output");
        aphi_analysis_options o;
        aphi_analysis_default_options(&o);
        if (opt) o = *opt;
        *out = analysis_create(n, row_ptr, col_idx, perm, parent, col_count, o);
    });
}

int aphi_fronts_create(int count, const int* rows, const int* widths, const aphi_analysis_options* opt,
                       aphi_analysis** out) {
    return guard([&] {
        if (!out || !rows || !widths) throw Error(APHI_ERR_INVALID, "aphi_fronts_create: null argument");
        aphi_analysis_options o;
        aphi_analysis_default_options(&o);
        if (opt) o = *opt;
        *out = analysis_create_fronts(count, rows, widths, o);
    });
}

int aphi_fronts_layout(const aphi_analysis* a, int64_t* panel_offset, int64_t* cb_offset) {
    return guard([&] {
        if (!a) throw Error(APHI_ERR_INVALID, "aphi_fronts_layout: null analysis");
        const Symbolic& S = analysis_symbolic(a);
        for (int s = 0; s < S.ns; ++s) {
            if (panel_offset) panel_offset[s] = S.sn_loff[s];
            if (cb_offset) cb_offset[s] = S.sn_cboff[s];
        }
    });
}

int aphi_analysis_destroy(aphi_analysis* a) {
    return guard([&] { analysis_destroy(a); });
}

int aphi_analysis_info(const aphi_analysis* a, double* info) {
    return guard([&] {
        if (!a || !info) throw Error(APHI_ERR_INVALID, "aphi_analysis_info: null argument");
        analysis_info(a, info);
    });
}

int aphi_analysis_etree(const aphi_analysis* a, int* parent, int* col_count) {
    return guard([&] {
        if (!a) throw Error(APHI_ERR_INVALID, "aphi_analysis_etree: null argument");
        const Symbolic& S = analysis_symbolic(a);
        for (int j = 0; j < S.n; ++j) {
            if (parent) parent[j] = S.ref_parent[j];
            if (col_count) col_count[j] = S.ref_colcount[j];
        }
    });
}

int aphi_analysis_plan_stats(const aphi_analysis* a, int plan, int64_t* launches, int64_t* items, double* useful,
                             double* executed) {
    return guard([&] {
        if (!a || !launches || !items) throw Error(APHI_ERR_INVALID, "aphi_analysis_plan_stats: null argument");
        const std::vector<Launch>* plans[] = {&a->plan_factor, &a->plan_factor_tc, &a->plan_fwd, &a->plan_bwd};
        if (plan < 0 || plan > 3) throw Error(APHI_ERR_BAD_SHAPE, "aphi_analysis_plan_stats: plan is 0..3");
        const Symbolic& S = a->S;
        for (int k = 0; k < APHI_PLAN_KINDS; ++k) {
            launches[k] = items[k] = 0;
            if (useful) useful[k] = 0;
            if (executed) executed[k] = 0;
        }
        // Lower-triangle entries (i >= j) of rows [r0, r1) x columns [c0, c1).
        auto lower = [](long long r0, long long r1, long long c0, long long c1) {
            double n = 0;
            for (long long j = c0; j < c1; ++j) n += static_cast<double>(std::max(0LL, r1 - std::max(r0, j)));
            return n;
        };
        for (const Launch& l : *plans[plan]) {
            if (l.kind < 0 || l.kind >= APHI_PLAN_KINDS) continue;
            ++launches[l.kind];
            items[l.kind] += l.count;
            if (!useful && !executed) continue;
            for (long long t = l.first; t < l.first + l.count; ++t) {
                const Item& it = a->h_items[t];
                const int w = S.sn_first[it.s + 1] - S.sn_first[it.s];
                const int m = S.sn_rows[it.s];
                double u = 0, e = 0;
                if (l.kind == K_UPDATE_WIDE || l.kind == K_UPDATE_TC) {
                    const int K = std::min(l.kcap, w - it.a);
                    u = 8.0 * K * lower(it.b, std::min(m, it.b + kTcM), it.c, std::min(m, it.c + kTcN));
                    e = 8.0 * K * kTcM * kTcN;
                } else if (l.kind == K_UPDATE_PANEL) {
                    const int kb = std::min(kStep, w - it.a);
                    const int jend = std::min(w, (it.a / kTcPanel) * kTcPanel + kTcPanel);
                    const int tm = l.wide ? kTcM : kTile, tn = l.wide ? kTcN : kTile;
                    u = 8.0 * kb * lower(it.b, std::min(m, it.b + tm), it.c, std::min(jend, it.c + tn));
                    e = 8.0 * kb * tm * tn;
                }
                if (useful) useful[l.kind] += u;
                if (executed) executed[l.kind] += e;
            }
        }
    });
}

}  // extern "C"
