// pivot_stats (hybrid-aphi-solver_b200/csrc/pivot_stats.cpp), which splits the
// batch entries over host threads, against the sequential walk restated
// here: every field of every entry bitwise equal, on random pivots with
// entries stopping at the floor at random columns, for a batch large enough
// to use threads and for a small one that does not. Test infrastructure:
// built by oracle/Makefile, run by tests/test_plan_check.py.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "pivot_stats.hpp"

using namespace aphi_b200;

namespace {

bool sequential(int n, int B, const std::vector<double>& dref, const std::vector<double>& dsc, double floor_,
                double ms, long long nnz, std::vector<aphi_factor_stats>& out, std::vector<int>& kmax) {
    bool any = false;
    for (int b = 0; b < B; ++b) {
        aphi_factor_stats s{};
        s.ok = 1;
        bool first = true;
        for (int k = 0; k < n; ++k) {
            const double mag = std::hypot(dref[2 * ((size_t)n * b + k)], dref[2 * ((size_t)n * b + k) + 1]);
            s.largest_pivot = std::max(s.largest_pivot, mag);
            if (first || mag < s.smallest_pivot) {
                s.smallest_pivot = mag;
                first = false;
            }
            s.columns_done = k + 1;
            if (!(mag > floor_)) {
                s.ok = 0;
                kmax[b] = k;
                any = true;
                break;
            }
        }
        s.nnz = nnz;
        s.milliseconds = ms;
        s.equilibration_min = n ? *std::min_element(dsc.begin() + (size_t)n * b, dsc.begin() + (size_t)n * (b + 1)) : 1.0;
        s.equilibration_max = n ? *std::max_element(dsc.begin() + (size_t)n * b, dsc.begin() + (size_t)n * (b + 1)) : 1.0;
        out[b] = s;
    }
    return any;
}

int check(int n, int B, unsigned seed) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> dref(2 * (size_t)n * B), dsc((size_t)n * B);
    for (auto& x : dref) x = U(g);
    for (auto& x : dsc) x = 1.0 + 0.5 * U(g);
    for (int b = 0; b < B; b += 3) {  // every third entry gets a pivot at the floor
        const int k = static_cast<int>(g() % n);
        dref[2 * ((size_t)n * b + k)] = 0.0;
        dref[2 * ((size_t)n * b + k) + 1] = 0.0;
    }
    std::vector<aphi_factor_stats> a(B), s(B);
    std::vector<int> ka(B, 0x7fffffff), ks(B, 0x7fffffff);
    const bool ra = pivot_stats(n, B, dref.data(), dsc.data(), 0.0, 12.5, 4242, a.data(), ka.data());
    const bool rs = sequential(n, B, dref, dsc, 0.0, 12.5, 4242, s, ks);
    const bool same = ra == rs && ka == ks && std::memcmp(a.data(), s.data(), sizeof(aphi_factor_stats) * B) == 0;
    std::printf("n %d batch %d %s\n", n, B, same ? "equal" : "DIFFERENT");
    return same ? 0 : 1;
}

}  // namespace

int main() { return check(227004, 16, 1) | check(50000, 7, 2) | check(300, 3, 3) | check(1, 1, 4); }
