// Diagnostic entry point: the arithmetic peaks the factorization kernels are
// measured against, timed on the device in use -- FP64 on the DMMA path
// (mma.sync m8n8k4) and as DFMA, FP32 FFMA, and TF32 on the tcgen05 tensor
// cores (M = 128, N = 64 and N = 256, operands in shared memory). Each is a
// register- or shared-memory-resident loop with no global traffic, 2 CTAs per
// SM, timed with CUDA events after one warm-up launch.
#include <cuda_runtime.h>

#include "aphi_b200.h"
#include "capi_util.hpp"
#include "common.cuh"

namespace aphi_b200 {
namespace {

constexpr int kPeakIters = 4096;

__global__ void k_peak_dfma(double* sink, int iters) {
    double a[16];
    for (int i = 0; i < 16; ++i) a[i] = threadIdx.x * 1e-3 + i;
    const double b = 1.0000001, c = 1e-9;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < 16; ++i) a[i] = fma(a[i], b, c);
    double s = 0;
    for (int i = 0; i < 16; ++i) s += a[i];
    if (s == 123.456) sink[0] = s;  // keeps the loop; never true for these inputs
}

__global__ void k_peak_ffma(float* sink, int iters) {
    float a[16];
    for (int i = 0; i < 16; ++i) a[i] = threadIdx.x * 1e-3f + i;
    const float b = 1.0000001f, c = 1e-9f;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < 16; ++i) a[i] = fmaf(a[i], b, c);
    float s = 0;
    for (int i = 0; i < 16; ++i) s += a[i];
    if (s == 123.456f) sink[0] = s;
}

__global__ void k_peak_dmma(double* sink, int iters) {
    double acc[8][2];
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0;
    const double a = threadIdx.x * 1e-3, b = 1.0 + threadIdx.x * 1e-4;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(acc[i][0]), "+d"(acc[i][1])
                         : "d"(a), "d"(b));
    double s = 0;
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1];
    if (s == 123.456) sink[0] = s;
}

__device__ __forceinline__ uint32_t peak_su32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// `iters` back-to-back tcgen05.mma kind::tf32 (M = 128, N = NN, K = 8) on one
// pair of shared-memory tiles, then one commit and a bounded wait.
template <int NN>
__global__ void __launch_bounds__(128) k_peak_tf32(int iters, int* err) {
    extern __shared__ __align__(16) unsigned char sm[];
    unsigned char* A = sm;
    unsigned char* B = sm + 128 * 32;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + 128 * 32 + NN * 32);
    uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
    for (int i = threadIdx.x; i < (128 + NN) * 8; i += blockDim.x) reinterpret_cast<float*>(sm)[i] = 0.5f;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(peak_su32(slot)),
                     "r"(NN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(peak_su32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *slot;
    if (threadIdx.x == 0) {
        const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(NN >> 3) << 17) |
                               (static_cast<uint32_t>(128 >> 4) << 24);
        auto desc = [](uint32_t addr) {
            return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>(128 >> 4) << 16) |
                   (static_cast<uint64_t>(256 >> 4) << 32) | (1ull << 46);
        };
        const uint64_t da = desc(peak_su32(A)), db = desc(peak_su32(B));
        for (int i = 0; i < iters; ++i) {
            const uint32_t acc = i > 0;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         peak_su32(mbar))
                     : "memory");
    }
    bool ok = false;
    for (long long i = 0; i < (1LL << 24); ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(peak_su32(mbar)), "r"(0u)
            : "memory");
        if (done) {
            ok = true;
            break;
        }
    }
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NN));
}

template <class F>
double time_ms(F launch) {
    cudaEvent_t a, b;
    APHI_CUDA(cudaEventCreate(&a));
    APHI_CUDA(cudaEventCreate(&b));
    launch();
    APHI_CUDA(cudaDeviceSynchronize());
    APHI_CUDA(cudaEventRecord(a));
    launch();
    APHI_CUDA(cudaEventRecord(b));
    APHI_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    APHI_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

}  // namespace
}  // namespace aphi_b200

extern "C" int aphi_measure_peaks(double* tflops) {
    using namespace aphi_b200;
    return guard([&] {
        if (!tflops) throw Error(APHI_ERR_INVALID, "aphi_measure_peaks: null output");
        int dev = 0, sms = 0;
        APHI_CUDA(cudaGetDevice(&dev));
        APHI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        double* sink = nullptr;
        int* err = nullptr;
        APHI_CUDA(cudaMalloc(&sink, 64));
        APHI_CUDA(cudaMalloc(&err, sizeof(int)));
        APHI_CUDA(cudaMemset(err, 0, sizeof(int)));
        const int grid = 2 * sms;
        double ms = time_ms([&] { k_peak_dmma<<<grid, 256>>>(sink, kPeakIters); });
        tflops[0] = 2.0 * 256 * 8 * kPeakIters * (256 / 32) * grid / ms / 1e9;
        ms = time_ms([&] { k_peak_dfma<<<grid, 512>>>(sink, kPeakIters); });
        tflops[1] = 2.0 * 16 * kPeakIters * 512.0 * grid / ms / 1e9;
        ms = time_ms([&] { k_peak_ffma<<<grid, 512>>>(reinterpret_cast<float*>(sink), kPeakIters); });
        tflops[2] = 2.0 * 16 * kPeakIters * 512.0 * grid / ms / 1e9;
        const int tci = 20000;
        const int s64 = 128 * 32 + 64 * 32 + 64, s256 = 128 * 32 + 256 * 32 + 64;
        APHI_CUDA(cudaFuncSetAttribute(k_peak_tf32<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
        APHI_CUDA(cudaFuncSetAttribute(k_peak_tf32<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, s256));
        ms = time_ms([&] { k_peak_tf32<64><<<grid, 128, s64>>>(tci, err); });
        tflops[3] = 2.0 * 128 * 64 * 8 * static_cast<double>(tci) * grid / ms / 1e9;
        ms = time_ms([&] { k_peak_tf32<256><<<grid, 128, s256>>>(tci, err); });
        tflops[4] = 2.0 * 128 * 256 * 8 * static_cast<double>(tci) * grid / ms / 1e9;
        int e = 0;
        APHI_CUDA(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
        cudaFree(sink);
        cudaFree(err);
        if (e) throw Error(APHI_ERR_TIMEOUT, "aphi_measure_peaks: a bounded wait expired");
    });
}
