// Numeric factorization state: batch x (panels + contribution-block pool) in
// FP64 or FP32 complex, the equilibration vectors, and solve scratch.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "aphi_b200.h"
#include "analysis.hpp"

struct aphi_factor {
    aphi_analysis* an = nullptr;
    int precision = 64;
    int batch = 1;             // active entries (<= capacity): what factorize/solve process
    int capacity = 1;          // entries the buffers are sized for
    size_t elem = 16;          // bytes per complex entry
    void* L = nullptr;         // batch x stored
    void* CB = nullptr;        // batch x cb_pool: the analysis's workspace, set at factorize
    double* dscale = nullptr;  // batch x n, original numbering
    unsigned long long* rowmax = nullptr;  // batch x n (equilibration scratch)
    unsigned long long* stats = nullptr;   // batch x 4 (max|L| bits, ...)
    double* dref = nullptr;    // batch x n complex128: D in the reference's permuted order
    // Solve scratch, grown on demand: y (batch x nrhs x n), U (batch x nrhs x upool).
    void* y = nullptr;
    void* U = nullptr;
    void* part = nullptr;  // backward partial sums: batch x max_parts x 64 x 8
    int nrhs_cap = 0;
    // Refinement scratch (FP64): x, r, d, per batch x nrhs x n; norms.
    double* ir = nullptr;
    int ir_cap = 0;
    double* red = nullptr;     // reduction partials
    double* norms = nullptr;   // batch x nrhs x 4
    int red_cap = 0;
    double* kr = nullptr;      // Krylov refinement scratch
    int kr_cap = 0;
    bool factored = false;
    bool use_tc = true;         // FP32: tensor-core updates (APHI_NO_TC=1 selects the SIMT kernels)
    int tc_split = 3;           // FP32 tensor-core updates: TF32 pieces per operand (3, or 2: hh + hl + lh)
    int tc_stages = 2;          // split 2: split-operand stages in flight (2 or 3; APHI_TC_STAGES)
    int tc_group = 2;           // split 2: stages per fresh main accumulator (2 or 4; APHI_TC_GROUP)
    bool presplit = true;       // split 2: operands split once per panel group (k_tc_split; APHI_TC_PRESPLIT=0: in the tile)
    int pre_stages = 3;         // plane buffers of the pre-split tile (APHI_TC_PRESTAGES=4: four; always four with tc_group 4)
    unsigned char* dws = nullptr;  // FP64: the trailing updates' scaled operands W = L D, dws_stride bytes per entry
    long long dws_stride = 0;      // (APHI_DMMA_PRESCALE=0: scaled inside every tile instead)
    unsigned char* tcws = nullptr;  // the pre-split operand planes, tcws_stride bytes per entry (capacity entries)
    long long tcws_stride = 0;
    int* err = nullptr;         // device error word (bounded waits)
    int* kmax = nullptr;        // capacity: the column where each entry's factorization stopped
    int* counters = nullptr;    // fused solve plans: arrival counters, ns per batch entry (zero between launches)
    int solve_form = -1;        // solve plans: -1 by batch (fused for one entry, split for more), 0 fused, 1 split
                                // (APHI_SOLVE_SPLIT=0 / 1)
    // Per-kind launch timing (aphi_factor_profile).
    bool profile = false;
    unsigned prof_mask = ~0u;  // kinds (bit k: kind k) timed while profiling
    std::vector<cudaEvent_t> prof_events;  // pairs, one per launch of the current factorization
    std::vector<int> prof_kinds;
    double prof_ms[APHI_PLAN_KINDS] = {};
    long long prof_launches[APHI_PLAN_KINDS] = {};
    // Host-buffer entry points stage through these (grown on demand).
    double* hvals = nullptr;
    size_t hvals_bytes = 0;
    double* hvec = nullptr;    // b then x
    size_t hvec_bytes = 0;
    std::vector<aphi_factor_stats> host_stats;
    ~aphi_factor();
};

namespace aphi_b200 {

aphi_factor* factor_create(aphi_analysis* an, int precision, int batch);
void factor_destroy(aphi_factor* f);
void factor_profile(aphi_factor* f, bool enable, unsigned mask = ~0u);
void factor_set_batch(aphi_factor* f, int batch);
int factorize(aphi_factor* f, const double* values_dev, int equil_iters, double pivot_floor,
              aphi_factor_stats* stats, cudaStream_t stream, const double* panels_dev = nullptr);
void fronts_read(const aphi_factor* f, int k, double* panels_out, double* cb_out, cudaStream_t stream);
void solve(aphi_factor* f, int nrhs, const double* b_dev, double* x_dev, cudaStream_t stream,
           const int* entries = nullptr, int nentries = 0);
void factor_export(const aphi_factor* f, int k, int* col_ptr, int* row_index, double* value,
                   double* diagonal, double* d_scale);
void residuals(const aphi_analysis* an, int batch, int nrhs, const double* values_dev, const double* x_dev,
               const double* b_dev, double* out, cudaStream_t stream);
void residuals_noalloc(const aphi_analysis* an, int batch, int nrhs, const double* values_dev,
                       const double* x_dev, const double* b_dev, double* out, cudaStream_t stream);
void spmv(const aphi_analysis* an, int batch, int nrhs, const double* values_dev, const double* x_dev, double* y_dev,
          cudaStream_t stream);
void csc_solve_host(int n, const int* col_ptr, const int* row_index, const double* value, const double* diagonal,
                    int nrhs, double* y);
void csr_residuals_host(int n, const int* row_ptr, const int* col_idx, const double* values, int nrhs,
                        const double* x, const double* b, double* out);
int solve_refined(aphi_factor* f, int nrhs, const double* values_dev, const double* b_dev, double* x_dev,
                  const aphi_ir_options& opt, int* iters, double* berr, cudaStream_t stream);

}  // namespace aphi_b200
