// C ABI: analysis (supernodal schedule) creation and queries.
#include "analysis.hpp"
#include "capi_util.hpp"

using namespace aphi_b200;

extern "C" {

void aphi_analysis_default_options(aphi_analysis_options* o) {
    if (!o) return;
    o->relax_small = 4;
    o->relax_fill = 0.05;
    o->relax_max_width = 256;
    o->small_front = 96;
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

int aphi_analysis_plan_stats(const aphi_analysis* a, int plan, int64_t* launches, int64_t* items) {
    return guard([&] {
        if (!a || !launches || !items) throw Error(APHI_ERR_INVALID, "aphi_analysis_plan_stats: null argument");
        const std::vector<Launch>* plans[] = {&a->plan_factor, &a->plan_factor_tc, &a->plan_fwd, &a->plan_bwd};
        if (plan < 0 || plan > 3) throw Error(APHI_ERR_BAD_SHAPE, "aphi_analysis_plan_stats: plan is 0..3");
        for (int k = 0; k < APHI_PLAN_KINDS; ++k) launches[k] = items[k] = 0;
        for (const Launch& l : *plans[plan]) {
            if (l.kind < 0 || l.kind >= APHI_PLAN_KINDS) continue;
            ++launches[l.kind];
            items[l.kind] += l.count;
        }
    });
}

}  // extern "C"
