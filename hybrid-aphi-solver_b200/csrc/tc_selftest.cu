// Diagnostic entry point: one tensor-core tile (tc_update.cuh) on caller
// data, so the tile's layout and split accuracy can be checked against a host
// product without a factorization around it.
#include <cuda_runtime.h>

#include <algorithm>

#include "aphi_b200.h"
#include "capi_util.hpp"
#include "common.cuh"
#include "tc_update.cuh"

namespace aphi_b200 {
namespace {

template <int Split>
__global__ void __launch_bounds__(kTcThreads) k_tc_selftest(const float2* P, int rows, int K, int i0, int j0,
                                                           const float2* d, float2* out, int* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const bool ok = tc_tile<Split>(smem_raw, P, rows, rows, K, i0, j0, d, 1,
                            [&](int r, int c0, const float(&re)[16], const float(&im)[16]) {
                                for (int c = 0; c < 16; ++c) out[r + (c0 + c) * kTcM] = make_float2(re[c], im[c]);
                            });
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
}

// A wait nothing will end: an mbarrier expecting one arrival that never
// comes, waited on by every thread with the same bounded wait the tensor-core
// tile uses. Each thread gives up after `limit` tries and the kernel returns
// normally with the error word set.
__global__ void k_wait_selftest(long long limit, int* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
    const bool done = mbar_wait(smem_u32(&bar), 0, limit);
    if (!done && threadIdx.x == 0) atomicExch(err, 1);
}

}  // namespace
}  // namespace aphi_b200

extern "C" int aphi_selftest_bounded_wait(long long spin_limit) {
    using namespace aphi_b200;
    return guard([&] {
        if (spin_limit < 1 || spin_limit > kTcSpinLimit)
            throw Error(APHI_ERR_BAD_SHAPE, "selftest: the spin limit is 1 .. the tile's own limit");
        int* derr = nullptr;
        APHI_CUDA(cudaMalloc(&derr, sizeof(int)));
        int e = 0;
        try {
            APHI_CUDA(cudaMemset(derr, 0, sizeof(int)));
            k_wait_selftest<<<1, 128>>>(spin_limit, derr);
            APHI_CHECK_LAUNCH();
            APHI_CUDA(cudaMemcpy(&e, derr, sizeof(int), cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(derr);
            throw;
        }
        cudaFree(derr);
        if (e) throw Error(APHI_ERR_TIMEOUT, "selftest: the bounded wait expired, as it must");
    });
}

extern "C" int aphi_selftest_tc_tile_split(int split, int rows, int K, int i0, int j0, const float* P,
                                           const float* d, float* out) {
    using namespace aphi_b200;
    return guard([&] {
        if (!P || !out) throw Error(APHI_ERR_INVALID, "selftest: null pointer");
        if (split != 2 && split != 3) throw Error(APHI_ERR_BAD_SHAPE, "selftest: split must be 2 or 3");
        if (rows < 1 || K < 1 || K > kTcPanel || i0 < 0 || j0 < 0)
            throw Error(APHI_ERR_BAD_SHAPE, "selftest: rows >= 1, 1 <= K <= 128, i0, j0 >= 0");
        float2 *dP = nullptr, *dd = nullptr, *dout = nullptr;
        int* derr = nullptr;
        const size_t pbytes = static_cast<size_t>(rows) * K * sizeof(float2);
        try {
            APHI_CUDA(cudaMalloc(&dP, pbytes));
            APHI_CUDA(cudaMalloc(&dout, static_cast<size_t>(kTcM) * kTcN * sizeof(float2)));
            APHI_CUDA(cudaMalloc(&derr, sizeof(int)));
            APHI_CUDA(cudaMemset(derr, 0, sizeof(int)));
            APHI_CUDA(cudaMemcpy(dP, P, pbytes, cudaMemcpyHostToDevice));
            if (d) {
                APHI_CUDA(cudaMalloc(&dd, static_cast<size_t>(K) * sizeof(float2)));
                APHI_CUDA(cudaMemcpy(dd, d, static_cast<size_t>(K) * sizeof(float2), cudaMemcpyHostToDevice));
            }
            if (split == 3) {
                APHI_CUDA(cudaFuncSetAttribute(k_tc_selftest<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               TcSmem<3>::bytes));
                k_tc_selftest<3><<<1, kTcThreads, TcSmem<3>::bytes>>>(dP, rows, K, i0, j0, dd, dout, derr);
            } else {
                APHI_CUDA(cudaFuncSetAttribute(k_tc_selftest<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               TcSmem<2>::bytes));
                k_tc_selftest<2><<<1, kTcThreads, TcSmem<2>::bytes>>>(dP, rows, K, i0, j0, dd, dout, derr);
            }
            APHI_CHECK_LAUNCH();
            int e = 0;
            APHI_CUDA(cudaMemcpy(&e, derr, sizeof(int), cudaMemcpyDeviceToHost));
            APHI_CUDA(cudaMemcpy(out, dout, static_cast<size_t>(kTcM) * kTcN * sizeof(float2),
                                 cudaMemcpyDeviceToHost));
            if (e) throw Error(APHI_ERR_TIMEOUT, "selftest: bounded wait expired");
        } catch (...) {
            cudaFree(dP);
            cudaFree(dd);
            cudaFree(dout);
            cudaFree(derr);
            throw;
        }
        cudaFree(dP);
        cudaFree(dd);
        cudaFree(dout);
        cudaFree(derr);
    });
}

extern "C" int aphi_selftest_tc_tile(int rows, int K, int i0, int j0, const float* P, const float* d, float* out) {
    return aphi_selftest_tc_tile_split(3, rows, K, i0, j0, P, d, out);
}
