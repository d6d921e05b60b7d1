#include "pivot_stats.hpp"

#include <algorithm>
#include <cmath>
#include <system_error>
#include <thread>
#include <vector>

namespace aphi_b200 {

bool pivot_stats(int n, int B, const double* dref, const double* dscale, double pivot_floor, double ms,
                 long long nnz_l, aphi_factor_stats* out, int* kmax) {
    std::vector<char> failed(B, 0);
    auto entry = [&](int b) {
        aphi_factor_stats& s = out[b];
        s = aphi_factor_stats{};
        s.ok = 1;
        bool first = true;
        for (int k = 0; k < n; ++k) {
            const double* d = dref + 2 * (static_cast<size_t>(n) * b + k);
            const double mag = std::hypot(d[0], d[1]);
            s.largest_pivot = std::max(s.largest_pivot, mag);
            if (first || mag < s.smallest_pivot) {
                s.smallest_pivot = mag;
                first = false;
            }
            s.columns_done = k + 1;
            if (!(mag > pivot_floor)) {
                s.ok = 0;
                kmax[b] = k;
                failed[b] = 1;
                break;
            }
        }
        s.nnz = nnz_l;
        s.milliseconds = ms;
        if (n > 0) {
            const double* sc = dscale + static_cast<size_t>(n) * b;
            s.equilibration_min = *std::min_element(sc, sc + n);
            s.equilibration_max = *std::max_element(sc, sc + n);
        } else {
            s.equilibration_min = s.equilibration_max = 1.0;
        }
    };
    // Entries are independent: one share per worker, entry b in share b % workers.
    const int workers = static_cast<long long>(n) * B >= (1 << 18)
                            ? std::min(B, static_cast<int>(std::max(1u, std::thread::hardware_concurrency())))
                            : 1;
    auto share = [&](int w) {
        for (int b = w; b < B; b += workers) entry(b);
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; ++w) {
        try {
            pool.emplace_back(share, w);
        } catch (const std::system_error&) {
            share(w);  // no thread: this share here
        }
    }
    share(0);
    for (std::thread& t : pool) t.join();
    return std::find(failed.begin(), failed.end(), 1) != failed.end();
}

}  // namespace aphi_b200
