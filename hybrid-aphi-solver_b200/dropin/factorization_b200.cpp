// Drop-in replacement for the reference's src/factorization.cpp: every
// function declared in include/aphi_solver/factorization.hpp, defined over
// the aphi_b200 C ABI so that the numeric work runs on the B200. Built in
// place of src/factorization.cpp against the reference's own headers; the
// rest of the reference (mesh, DOF map, sparsity, AMD, symbolic analysis,
// equilibration) is linked unchanged.
//
// Error conventions are the reference's: std::invalid_argument for size
// mismatches (src/factorization.cpp:113-120, :256-260, :298-302, :336-340),
// std::logic_error when the symbolic and numeric passes disagree or a solve
// meets a zero pivot (:180-184, :276-280), `return false` with the stats or
// report filled as far as they go when a pivot is at or below the floor
// (:203-210, :380-383). Any other failure of the device path is reported as
// std::runtime_error with the C ABI's message.
//
// Device residency. factorize_ldlt returns the reference's host
// SymmetricFactor (strictly lower CSC, padding dropped), and also keeps the
// device factor it was exported from, registered under the address of the
// SymmetricFactor it filled together with a fingerprint of its contents. A
// later solve_in_place / solve of that same, unchanged factor runs on the
// device factor; a factor from anywhere else (or modified since) is solved on
// the device from its CSC arrays (aphi_csc_solve_host). relative_residual and
// backward_error run on the device too (aphi_csr_residuals_host). No numeric
// work of these functions runs on the host.
#include <algorithm>
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "aphi_b200.h"
#include "aphi_solver/factorization.hpp"
#include "aphi_solver/symbolic.hpp"

namespace aphi_solver {

namespace {

using Complex = std::complex<double>;

void check_status(int rc, const char* where) {
    if (rc == APHI_OK) return;
    const std::string msg = std::string(where) + ": " + aphi_last_error();
    if (rc == APHI_ERR_BAD_SHAPE) throw std::invalid_argument(msg);
    if (rc == APHI_ERR_PATTERN_MISMATCH || rc == APHI_ERR_ZERO_PIVOT) throw std::logic_error(msg);
    throw std::runtime_error(msg + " (" + aphi_status_string(rc) + ")");
}

const double* as_doubles(const std::vector<Complex>& v) { return reinterpret_cast<const double*>(v.data()); }
double* as_doubles(std::vector<Complex>& v) { return reinterpret_cast<double*>(v.data()); }

// One device analysis per (pattern, permutation): the supernodal schedule is
// built once and reused by every factorization of that pattern.
struct DeviceAnalysis {
    std::vector<int> row_ptr, col_idx, perm;
    aphi_analysis* an = nullptr;
    ~DeviceAnalysis() {
        if (an) aphi_analysis_destroy(an);
    }
};

// A device factor registered under the SymmetricFactor it was exported to.
struct DeviceFactor {
    std::shared_ptr<DeviceAnalysis> analysis;
    aphi_factor* f = nullptr;
    const SymmetricFactor* host = nullptr;
    uint64_t fingerprint = 0;
    ~DeviceFactor() {
        if (f) aphi_factor_destroy(f);
    }
};

constexpr size_t kMaxAnalyses = 4;
constexpr size_t kMaxFactors = 8;

// The registries are heap objects that are never destroyed: device handles
// are not released from static destructors, which run after the CUDA runtime
// may have been torn down; the process exit reclaims them.
std::mutex& g_mutex = *new std::mutex;
std::list<std::shared_ptr<DeviceAnalysis>>& g_analyses = *new std::list<std::shared_ptr<DeviceAnalysis>>;  // MRU first
std::list<std::shared_ptr<DeviceFactor>>& g_factors = *new std::list<std::shared_ptr<DeviceFactor>>;

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

// Sizes, data addresses, every pivot and a strided sample of L's entries.
uint64_t fingerprint(const SymmetricFactor& f) {
    uint64_t h = mix(0, static_cast<uint64_t>(f.rows));
    h = mix(h, reinterpret_cast<uintptr_t>(f.value.data()));
    h = mix(h, f.value.size());
    h = mix(h, reinterpret_cast<uintptr_t>(f.diagonal.data()));
    h = mix(h, f.col_ptr.size());
    auto add = [&](const Complex& c) {
        uint64_t a, b;
        const double re = c.real(), im = c.imag();
        std::memcpy(&a, &re, 8);
        std::memcpy(&b, &im, 8);
        h = mix(mix(h, a), b);
    };
    for (const Complex& d : f.diagonal) add(d);
    const size_t stride = std::max<size_t>(1, f.value.size() / 4096);
    for (size_t t = 0; t < f.value.size(); t += stride) add(f.value[t]);
    return h;
}

std::shared_ptr<DeviceAnalysis> device_analysis(const SparseSymmetricZ& a, const std::vector<int>& perm,
                                                const std::vector<int>* parent, const std::vector<int>* col_count) {
    for (auto it = g_analyses.begin(); it != g_analyses.end(); ++it) {
        const auto& d = *it;
        if (d->perm == perm && d->row_ptr == a.row_ptr() && d->col_idx == a.col_index()) {
            g_analyses.splice(g_analyses.begin(), g_analyses, it);
            return d;
        }
    }
    auto d = std::make_shared<DeviceAnalysis>();
    d->row_ptr = a.row_ptr();
    d->col_idx = a.col_index();
    d->perm = perm;
    aphi_analysis_options opt;
    aphi_analysis_default_options(&opt);
    check_status(aphi_analysis_create(a.rows(), d->row_ptr.data(), d->col_idx.data(), d->perm.data(),
                                      parent ? parent->data() : nullptr, col_count ? col_count->data() : nullptr,
                                      &opt, &d->an),
                 "factorize_ldlt");
    g_analyses.push_front(d);
    if (g_analyses.size() > kMaxAnalyses) g_analyses.pop_back();
    return d;
}

std::shared_ptr<DeviceFactor> find_factor(const SymmetricFactor& f) {
    for (auto it = g_factors.begin(); it != g_factors.end(); ++it) {
        if ((*it)->host == &f) {
            if ((*it)->fingerprint != fingerprint(f)) return nullptr;
            g_factors.splice(g_factors.begin(), g_factors, it);
            return *it;
        }
    }
    return nullptr;
}

void forget_factor(const SymmetricFactor* f) {
    g_factors.remove_if([&](const std::shared_ptr<DeviceFactor>& d) { return d->host == f; });
}

}  // namespace

SparseMatrixZ permuted_lower(const SparseSymmetricZ& a, const Permutation& p) {
    const int n = a.rows();
    if (p.size() != n) {
        throw std::invalid_argument("permuted_lower: the permutation has " + std::to_string(p.size()) +
                                    " entries for a matrix of " + std::to_string(n) + " rows");
    }
    // Entry (r, c) of A (upper, original numbering) sits at (iperm[r], iperm[c])
    // of P A P^T; stored below the diagonal.
    SparseMatrixZ out(n, n);
    out.reserve(a.nnz());
    const auto& rp = a.row_ptr();
    const auto& ci = a.col_index();
    const auto& v = a.values();
    for (int r = 0; r < n; ++r)
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const int pr = p.iperm[r], pc = p.iperm[ci[k]];
            out.add(std::max(pr, pc), std::min(pr, pc), v[k]);
        }
    out.compress();
    return out;
}

bool factorize_ldlt(const SparseSymmetricZ& a, const SolverAnalysis& analysis, SymmetricFactor& out,
                    FactorStats& stats, double pivot_floor) {
    const auto started = std::chrono::steady_clock::now();
    const int n = a.rows();
    if (analysis.permutation.size() != n || static_cast<int>(analysis.col_count.size()) != n) {
        throw std::invalid_argument("factorize_ldlt: the analysis describes " +
                                    std::to_string(analysis.permutation.size()) +
                                    " unknowns, the matrix has " + std::to_string(n));
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    forget_factor(&out);
    auto d = device_analysis(a, analysis.permutation.perm, &analysis.parent, &analysis.col_count);
    auto rec = std::make_shared<DeviceFactor>();
    rec->analysis = d;
    check_status(aphi_factor_create(d->an, APHI_PREC_FP64, 1, &rec->f), "factorize_ldlt");
    aphi_factor_stats st{};
    const int rc = aphi_factorize_host(rec->f, as_doubles(a.values()), 0, pivot_floor, &st);
    if (rc != APHI_OK && rc != APHI_ERR_PIVOT_FLOOR) check_status(rc, "factorize_ldlt");

    size_t nl = 0;
    for (int j = 0; j < n; ++j) nl += static_cast<size_t>(std::max(0, analysis.col_count[j] - 1));
    out.rows = n;
    out.col_ptr.assign(static_cast<size_t>(n) + 1, 0);
    out.row_index.assign(nl, 0);
    out.value.assign(nl, Complex(0.0, 0.0));
    out.diagonal.assign(static_cast<size_t>(n), Complex(0.0, 0.0));
    check_status(aphi_factor_export(rec->f, 0, out.col_ptr.data(), out.row_index.data(), as_doubles(out.value),
                                    as_doubles(out.diagonal), nullptr),
                 "factorize_ldlt");
    stats = FactorStats{};
    stats.ok = st.ok != 0;
    stats.columns_done = st.columns_done;
    stats.smallest_pivot = st.smallest_pivot;
    stats.largest_pivot = st.largest_pivot;
    stats.largest_multiplier = st.largest_multiplier;
    stats.nnz = out.nnz();
    stats.milliseconds =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - started).count();
    if (rc == APHI_OK) {
        rec->host = &out;
        rec->fingerprint = fingerprint(out);
        g_factors.push_front(rec);
        if (g_factors.size() > kMaxFactors) g_factors.pop_back();
    }
    return rc == APHI_OK;
}

SparseMatrixZ reconstruct(const SymmetricFactor& f) {
    const int n = f.rows;
    // Column j of L (unit diagonal first) contributes L(r,j) D(j) L(c,j) to
    // every pair of its rows; accumulate row by row into a dense-per-row map.
    std::vector<std::vector<std::pair<int, Complex>>> cols(static_cast<size_t>(n));
    for (int j = 0; j < n; ++j) {
        cols[j].push_back({j, Complex(1.0, 0.0)});
        for (int t = f.col_ptr[j]; t < f.col_ptr[j + 1]; ++t) cols[j].push_back({f.row_index[t], f.value[t]});
    }
    std::vector<std::vector<std::pair<int, Complex>>> rows_of(static_cast<size_t>(n));  // r -> (j, L(r,j))
    for (int j = 0; j < n; ++j)
        for (const auto& e : cols[j]) rows_of[e.first].push_back({j, e.second});
    SparseMatrixZ out(n, n);
    std::vector<Complex> acc(static_cast<size_t>(n));
    std::vector<char> touched(static_cast<size_t>(n), 0);
    std::vector<int> list;
    for (int r = 0; r < n; ++r) {
        list.clear();
        for (const auto& rj : rows_of[r]) {
            const int j = rj.first;
            const Complex w = rj.second * f.diagonal[j];
            for (const auto& cj : cols[j]) {
                const int c = cj.first;
                if (c > r) continue;
                if (!touched[c]) {
                    touched[c] = 1;
                    acc[c] = Complex(0.0, 0.0);
                    list.push_back(c);
                }
                acc[c] += w * cj.second;
            }
        }
        std::sort(list.begin(), list.end());
        for (int c : list) {
            touched[c] = 0;
            if (acc[c] == Complex(0.0, 0.0)) continue;
            out.add(r, c, acc[c]);
            if (r != c) out.add(c, r, acc[c]);
        }
    }
    out.compress();
    return out;
}

void solve_in_place(const SymmetricFactor& f, std::vector<Complex>& y) {
    const int n = f.rows;
    if (static_cast<int>(y.size()) != n) {
        throw std::invalid_argument("solve_in_place: the right-hand side has " + std::to_string(y.size()) +
                                    " entries for a factor of " + std::to_string(n) + " rows");
    }
    for (int j = 0; j < n; ++j)
        if (f.diagonal[j] == Complex(0.0, 0.0))
            throw std::logic_error("solve_in_place: D[" + std::to_string(j) +
                                   "] is zero; this factor did not come from a completed factorize_ldlt");
    std::lock_guard<std::mutex> lock(g_mutex);
    auto d = find_factor(f);
    if (!d) {
        // A factor this layer did not produce (built by hand, or modified
        // since): solved on the device from its CSC arrays.
        check_status(aphi_csc_solve_host(n, f.col_ptr.data(), f.row_index.data(), as_doubles(f.value),
                                         reinterpret_cast<const double*>(f.diagonal.data()), 1, as_doubles(y)),
                     "solve_in_place");
        return;
    }
    // The device factor solves in the original numbering: y is in the
    // factorized one, so un-permute, solve, permute back.
    const std::vector<int>& perm = d->analysis->perm;
    std::vector<Complex> b(static_cast<size_t>(n)), x(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) b[perm[i]] = y[i];
    check_status(aphi_solve_host(d->f, 1, as_doubles(b), as_doubles(x)), "solve_in_place");
    for (int i = 0; i < n; ++i) y[i] = x[perm[i]];
}

std::vector<Complex> solve(const SymmetricFactor& f, const Permutation& p, const std::vector<Complex>& b) {
    const int n = f.rows;
    if (p.size() != n || static_cast<int>(b.size()) != n) {
        throw std::invalid_argument(
            "solve: the factor, the permutation and the right-hand side must all describe the same number of "
            "unknowns");
    }
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        auto d = find_factor(f);
        if (d && d->analysis->perm == p.perm) {
            std::vector<Complex> x(static_cast<size_t>(n));
            check_status(aphi_solve_host(d->f, 1, as_doubles(b), as_doubles(x)), "solve");
            return x;
        }
    }
    std::vector<Complex> y(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) y[i] = b[p.perm[i]];
    solve_in_place(f, y);
    std::vector<Complex> x(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) x[p.perm[i]] = y[i];
    return x;
}

namespace {

// relative_residual and backward_error together, on the device.
void device_residuals(const char* where, const SparseSymmetricZ& a, const std::vector<Complex>& x,
                      const std::vector<Complex>& b, double out[2]) {
    if (static_cast<int>(x.size()) != a.rows() || x.size() != b.size())
        throw std::invalid_argument(std::string(where) + ": lengths must match the matrix");
    if (a.rows() == 0) {
        out[0] = out[1] = 0.0;
        return;
    }
    check_status(aphi_csr_residuals_host(a.rows(), a.row_ptr().data(), a.col_index().data(), as_doubles(a.values()),
                                         1, as_doubles(x), as_doubles(b), out),
                 where);
}

}  // namespace

double relative_residual(const SparseSymmetricZ& a, const std::vector<Complex>& x, const std::vector<Complex>& b) {
    double out[2];
    device_residuals("relative_residual", a, x, b, out);
    return out[0];
}

double backward_error(const SparseSymmetricZ& a, const std::vector<Complex>& x, const std::vector<Complex>& b) {
    double out[2];
    device_residuals("backward_error", a, x, b, out);
    return out[1];
}

bool solve_symmetric(const SparseSymmetricZ& a, const std::vector<Complex>& b, std::vector<Complex>& x,
                     SolveReport& report, const SolveOptions& options, const SolverAnalysis* precomputed) {
    const int n = a.rows();
    if (static_cast<int>(b.size()) != n) {
        throw std::invalid_argument("solve_symmetric: the right-hand side has " + std::to_string(b.size()) +
                                    " entries for a matrix of " + std::to_string(n) + " rows");
    }
    report = SolveReport{};
    // The ordering is structural: the reference's own analysis of the pattern
    // (equilibration cannot change it), reused when the caller has one.
    const auto t0 = std::chrono::steady_clock::now();
    SolverAnalysis owned;
    if (!precomputed) owned = analyze(a, options.ordering);
    const SolverAnalysis& analysis = precomputed ? *precomputed : owned;
    report.analyze_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    std::lock_guard<std::mutex> lock(g_mutex);
    auto d = device_analysis(a, analysis.permutation.perm, &analysis.parent, &analysis.col_count);
    // Equilibrate, factorize, solve, un-scale and measure on the device.
    std::vector<Complex> xs(static_cast<size_t>(n));
    double rep[13] = {};
    const int rc = aphi_solve_symmetric_host(d->an, as_doubles(a.values()), as_doubles(b),
                                             options.equilibration_iterations, options.pivot_floor,
                                             as_doubles(xs), rep);
    if (rc != APHI_OK && rc != APHI_ERR_PIVOT_FLOOR) check_status(rc, "solve_symmetric");
    report.equilibration_min = rep[3];
    report.equilibration_max = rep[4];
    report.smallest_pivot = rep[5];
    report.largest_pivot = rep[6];
    report.largest_multiplier = rep[7];
    report.factor_nnz = static_cast<size_t>(rep[8]);
    report.columns_done = static_cast<int>(rep[9]);
    report.factorize_ms = rep[11];
    if (rc == APHI_ERR_PIVOT_FLOOR) {
        report.ok = false;
        return false;
    }
    report.solve_ms = rep[12];
    report.backward_error = rep[1];
    report.residual = rep[2];
    report.ok = true;
    x = std::move(xs);
    return true;
}

}  // namespace aphi_solver
