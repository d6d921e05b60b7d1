// C ABI: factors, factorization, solves, residuals, refinement and the
// whole solve_symmetric pipeline on host buffers.
#include <chrono>
#include <cstring>
#include <vector>

#include "capi_util.hpp"
#include "factor.hpp"

using namespace aphi_b200;

namespace {
cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

int aphi_factor_create(const aphi_analysis* an, int precision, int batch, aphi_factor** out) {
    return guard([&] {
        if (!out) throw Error(APHI_ERR_INVALID, "aphi_factor_create: null output");
        *out = factor_create(const_cast<aphi_analysis*>(an), precision, batch);
    });
}

int aphi_factor_destroy(aphi_factor* f) {
    return guard([&] { factor_destroy(f); });
}

int aphi_factorize(aphi_factor* f, const double* values_dev, int equil_iters, double pivot_floor,
                   aphi_factor_stats* stats, void* stream) {
    int rc = APHI_OK;
    const int g = guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_factorize: null factor");
        rc = factorize(f, values_dev, equil_iters, pivot_floor, stats, as_stream(stream));
        if (rc == APHI_ERR_PIVOT_FLOOR)
            set_last_error("factorize_ldlt: a pivot at or below the floor stopped the factorization");
    });
    if (g != APHI_OK) return g;
    return rc;
}

int aphi_solve(aphi_factor* f, int nrhs, const double* b_dev, double* x_dev, void* stream) {
    return guard([&] {
        if (!f || !b_dev || !x_dev) throw Error(APHI_ERR_INVALID, "aphi_solve: null argument");
        solve(f, nrhs, b_dev, x_dev, as_stream(stream));
    });
}

int aphi_factorize_fronts(aphi_factor* f, const double* panels_dev, aphi_factor_stats* stats, void* stream) {
    int rc = APHI_OK;
    const int g = guard([&] {
        if (!f || !panels_dev) throw Error(APHI_ERR_INVALID, "aphi_factorize_fronts: null argument");
        rc = factorize(f, nullptr, 0, 0.0, stats, as_stream(stream), panels_dev);
    });
    if (g != APHI_OK) return g;
    return rc;
}

int aphi_fronts_read(const aphi_factor* f, int k, double* panels_dev, double* cb_dev, void* stream) {
    return guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_fronts_read: null factor");
        fronts_read(f, k, panels_dev, cb_dev, as_stream(stream));
    });
}

int aphi_factor_set_batch(aphi_factor* f, int batch) {
    return guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_factor_set_batch: null factor");
        factor_set_batch(f, batch);
    });
}

int aphi_factor_set_tc_split(aphi_factor* f, int split) {
    return guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_factor_set_tc_split: null factor");
        if (split != 2 && split != 3) throw Error(APHI_ERR_BAD_SHAPE, "aphi_factor_set_tc_split: split must be 2 or 3");
        f->tc_split = split;
    });
}

int aphi_factor_profile(aphi_factor* f, int enable) {
    return guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_factor_profile: null factor");
        factor_profile(f, enable != 0);
    });
}

int aphi_factor_profile_kinds(aphi_factor* f, unsigned mask) {
    return guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_factor_profile_kinds: null factor");
        factor_profile(f, mask != 0, mask);
    });
}

int aphi_factor_profile_read(const aphi_factor* f, double* ms, int64_t* launches) {
    return guard([&] {
        if (!f || !ms || !launches) throw Error(APHI_ERR_INVALID, "aphi_factor_profile_read: null argument");
        for (int k = 0; k < APHI_PLAN_KINDS; ++k) {
            ms[k] = f->prof_ms[k];
            launches[k] = f->prof_launches[k];
        }
    });
}

int aphi_factor_export(const aphi_factor* f, int k, int* col_ptr, int* row_index, double* value,
                       double* diagonal, double* d_scale) {
    return guard([&] {
        if (!f) throw Error(APHI_ERR_INVALID, "aphi_factor_export: null factor");
        factor_export(f, k, col_ptr, row_index, value, diagonal, d_scale);
    });
}

int aphi_residuals(const aphi_analysis* an, int batch, int nrhs, const double* values_dev, const double* x_dev,
                   const double* b_dev, double* out, void* stream) {
    return guard([&] {
        if (!an || !values_dev || !x_dev || !b_dev || !out) throw Error(APHI_ERR_INVALID, "aphi_residuals: null argument");
        if (batch < 1 || nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "aphi_residuals: batch and nrhs must be >= 1");
        analysis_ensure_device(const_cast<aphi_analysis*>(an));
        residuals(an, batch, nrhs, values_dev, x_dev, b_dev, out, as_stream(stream));
    });
}

int aphi_spmv(const aphi_analysis* an, int batch, int nrhs, const double* values_dev, const double* x_dev,
              double* y_dev, void* stream) {
    return guard([&] {
        if (!an || !values_dev || !x_dev || !y_dev) throw Error(APHI_ERR_INVALID, "aphi_spmv: null argument");
        if (batch < 1 || nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "aphi_spmv: batch and nrhs must be >= 1");
        analysis_ensure_device(const_cast<aphi_analysis*>(an));
        spmv(an, batch, nrhs, values_dev, x_dev, y_dev, as_stream(stream));
    });
}

int aphi_residuals_noalloc(const aphi_analysis* an, int batch, int nrhs, const double* values_dev,
                           const double* x_dev, const double* b_dev, double* out, void* stream) {
    return guard([&] {
        if (!an || !values_dev || !x_dev || !b_dev || !out)
            throw Error(APHI_ERR_INVALID, "aphi_residuals_noalloc: null argument");
        if (batch < 1 || nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "aphi_residuals_noalloc: batch and nrhs must be >= 1");
        residuals_noalloc(an, batch, nrhs, values_dev, x_dev, b_dev, out, as_stream(stream));
    });
}

int aphi_solve_refined(aphi_factor* f, int nrhs, const double* values_dev, const double* b_dev, double* x_dev,
                       const aphi_ir_options* opt, int* iters, double* berr, void* stream) {
    int rc = APHI_OK;
    const int g = guard([&] {
        if (!f || !values_dev || !b_dev || !x_dev || !iters || !berr)
            throw Error(APHI_ERR_INVALID, "aphi_solve_refined: null argument");
        aphi_ir_options o{40, 1e-16, 0.5, 1, 1e-14};
        if (opt) o = *opt;
        rc = solve_refined(f, nrhs, values_dev, b_dev, x_dev, o, iters, berr, as_stream(stream));
        if (rc == APHI_ERR_IR_STALL) set_last_error("iterative refinement stalled before reaching the tolerance");
    });
    if (g != APHI_OK) return g;
    return rc;
}

namespace {
double* grow(double*& buf, size_t& have, size_t need) {
    if (have < need) {
        if (buf) cudaFree(buf);
        buf = nullptr;
        have = 0;
        APHI_CUDA(cudaMalloc(&buf, std::max<size_t>(need, 16)));
        have = need;
    }
    return buf;
}
}  // namespace

int aphi_factorize_host(aphi_factor* f, const double* values, int equil_iters, double pivot_floor,
                        aphi_factor_stats* stats) {
    int rc = APHI_OK;
    const int g = guard([&] {
        if (!f || !values) throw Error(APHI_ERR_INVALID, "aphi_factorize_host: null argument");
        const size_t bytes = sizeof(double) * 2 * static_cast<size_t>(f->an->S.nnz_a) * f->batch;
        double* dv = grow(f->hvals, f->hvals_bytes, bytes);
        APHI_CUDA(cudaMemcpy(dv, values, bytes, cudaMemcpyHostToDevice));
        rc = factorize(f, dv, equil_iters, pivot_floor, stats, nullptr);
        if (rc == APHI_ERR_PIVOT_FLOOR)
            set_last_error("factorize_ldlt: a pivot at or below the floor stopped the factorization");
    });
    if (g != APHI_OK) return g;
    return rc;
}

int aphi_solve_host(aphi_factor* f, int nrhs, const double* b, double* x) {
    return guard([&] {
        if (!f || !b || !x) throw Error(APHI_ERR_INVALID, "aphi_solve_host: null argument");
        if (nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "aphi_solve_host: nrhs must be >= 1");
        const size_t len = sizeof(double) * 2 * static_cast<size_t>(f->an->S.n) * nrhs * f->batch;
        double* d = grow(f->hvec, f->hvec_bytes, 2 * len);
        APHI_CUDA(cudaMemcpy(d, b, len, cudaMemcpyHostToDevice));
        solve(f, nrhs, d, d + len / sizeof(double), nullptr);
        APHI_CUDA(cudaMemcpy(x, d + len / sizeof(double), len, cudaMemcpyDeviceToHost));
    });
}

int aphi_residuals_host(const aphi_analysis* an_c, int batch, int nrhs, const double* values, const double* x,
                        const double* b, double* out) {
    return guard([&] {
        if (!an_c || !values || !x || !b || !out) throw Error(APHI_ERR_INVALID, "aphi_residuals_host: null argument");
        if (batch < 1 || nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "aphi_residuals_host: batch and nrhs must be >= 1");
        auto* an = const_cast<aphi_analysis*>(an_c);
        analysis_ensure_device(an);
        const size_t vb = sizeof(double) * 2 * static_cast<size_t>(an->S.nnz_a) * batch;
        const size_t xb = sizeof(double) * 2 * static_cast<size_t>(an->S.n) * nrhs * batch;
        double *dv = nullptr, *dx = nullptr, *db = nullptr;
        try {
            APHI_CUDA(cudaMalloc(&dv, std::max<size_t>(vb, 16)));
            APHI_CUDA(cudaMalloc(&dx, std::max<size_t>(xb, 16)));
            APHI_CUDA(cudaMalloc(&db, std::max<size_t>(xb, 16)));
            APHI_CUDA(cudaMemcpy(dv, values, vb, cudaMemcpyHostToDevice));
            APHI_CUDA(cudaMemcpy(dx, x, xb, cudaMemcpyHostToDevice));
            APHI_CUDA(cudaMemcpy(db, b, xb, cudaMemcpyHostToDevice));
            residuals(an, batch, nrhs, dv, dx, db, out, nullptr);
        } catch (...) {
            cudaFree(dv);
            cudaFree(dx);
            cudaFree(db);
            throw;
        }
        cudaFree(dv);
        cudaFree(dx);
        cudaFree(db);
    });
}

int aphi_csc_solve_host(int n, const int* col_ptr, const int* row_index, const double* value,
                        const double* diagonal, int nrhs, double* y) {
    return guard([&] {
        if (!col_ptr || (n > 0 && (!diagonal || !y)) || (n > 0 && col_ptr[n] > 0 && (!row_index || !value)))
            throw Error(APHI_ERR_INVALID, "aphi_csc_solve_host: null argument");
        csc_solve_host(n, col_ptr, row_index, value, diagonal, nrhs, y);
    });
}

int aphi_csr_residuals_host(int n, const int* row_ptr, const int* col_idx, const double* values, int nrhs,
                            const double* x, const double* b, double* out) {
    return guard([&] {
        if (!row_ptr || !col_idx || !values || !x || !b || !out)
            throw Error(APHI_ERR_INVALID, "aphi_csr_residuals_host: null argument");
        csr_residuals_host(n, row_ptr, col_idx, values, nrhs, x, b, out);
    });
}

int aphi_solve_symmetric_host(const aphi_analysis* an_c, const double* values, const double* b, int equil_iters,
                              double pivot_floor, double* x, double* report) {
    int rc = APHI_OK;
    const int g = guard([&] {
        if (!an_c || !values || !b || !x || !report) throw Error(APHI_ERR_INVALID, "aphi_solve_symmetric_host: null argument");
        auto* an = const_cast<aphi_analysis*>(an_c);
        const int n = an->S.n;
        const long long nnz = an->S.nnz_a;
        std::memset(report, 0, sizeof(double) * 13);
        report[3] = report[4] = 1.0;
        aphi_factor* f = factor_create(an, 64, 1);
        double *dv = nullptr, *db = nullptr, *dx = nullptr;
        try {
            APHI_CUDA(cudaMalloc(&dv, sizeof(double) * 2 * std::max<long long>(nnz, 1)));
            APHI_CUDA(cudaMalloc(&db, sizeof(double) * 2 * std::max(n, 1)));
            APHI_CUDA(cudaMalloc(&dx, sizeof(double) * 2 * std::max(n, 1)));
            APHI_CUDA(cudaMemcpy(dv, values, sizeof(double) * 2 * nnz, cudaMemcpyHostToDevice));
            APHI_CUDA(cudaMemcpy(db, b, sizeof(double) * 2 * n, cudaMemcpyHostToDevice));
            aphi_factor_stats st{};
            rc = factorize(f, dv, equil_iters, pivot_floor, &st, nullptr);
            report[3] = st.equilibration_min;
            report[4] = st.equilibration_max;
            report[5] = st.smallest_pivot;
            report[6] = st.largest_pivot;
            report[7] = st.largest_multiplier;
            report[8] = static_cast<double>(st.nnz);
            report[9] = st.columns_done;
            report[11] = st.milliseconds;
            if (rc == APHI_OK) {
                const auto s0 = std::chrono::steady_clock::now();
                solve(f, 1, db, dx, nullptr);
                APHI_CUDA(cudaDeviceSynchronize());
                report[12] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s0).count();
                double res[2];
                residuals(an, 1, 1, dv, dx, db, res, nullptr);
                report[1] = res[1];
                report[2] = res[0];
                report[0] = 1.0;
                APHI_CUDA(cudaMemcpy(x, dx, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost));
            } else {
                set_last_error("factorize_ldlt: a pivot at or below the floor stopped the factorization");
            }
        } catch (...) {
            cudaFree(dv);
            cudaFree(db);
            cudaFree(dx);
            factor_destroy(f);
            throw;
        }
        cudaFree(dv);
        cudaFree(db);
        cudaFree(dx);
        factor_destroy(f);
    });
    if (g != APHI_OK) return g;
    return rc;
}

}  // extern "C"
