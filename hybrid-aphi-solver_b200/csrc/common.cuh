// Shared device/host helpers for the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "aphi_b200.h"

namespace aphi_b200 {

// Thrown inside the library, caught at the C ABI and mapped to a status code.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define APHI_CUDA(call)                                                                       \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            if (e_ == cudaErrorMemoryAllocation)                                              \
                throw ::aphi_b200::Error(APHI_ERR_OOM, std::string(#call) + ": " +            \
                                                           cudaGetErrorString(e_));           \
            throw ::aphi_b200::Error(APHI_ERR_CUDA,                                           \
                                     std::string(#call) + ": " + cudaGetErrorString(e_));     \
        }                                                                                     \
    } while (0)

// Every kernel launch site is followed by APHI_CHECK_LAUNCH(), which also
// counts the launch (aphi_launch_count()).
void count_launch();
#define APHI_CHECK_LAUNCH()               \
    do {                                  \
        ::aphi_b200::count_launch();      \
        APHI_CUDA(cudaGetLastError());    \
    } while (0)

// Complex double as two doubles. The operations below spell out the exact
// sequence of roundings the host's std::complex<double> performs (no fused
// multiply-add), so element and scatter arithmetic can reproduce the
// reference's bits.
struct cplx {
    double re, im;
};

__host__ __device__ __forceinline__ cplx cmake(double r, double i) { return cplx{r, i}; }

#ifdef __CUDACC__
__device__ __forceinline__ cplx cmul_exact(cplx a, cplx b) {
    return cplx{__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
                __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ cplx cscale_exact(cplx a, double s) {
    return cplx{__dmul_rn(a.re, s), __dmul_rn(a.im, s)};
}
__device__ __forceinline__ cplx cadd_exact(cplx a, cplx b) {
    return cplx{__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)};
}
__device__ __forceinline__ cplx cneg(cplx a) { return cplx{-a.re, -a.im}; }

// Fast versions (contractions allowed) for the factorization arithmetic.
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
#endif

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

constexpr int kNumSMs = 148;

}  // namespace aphi_b200
