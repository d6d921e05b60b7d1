// Tensor-core (tcgen05, sm_100a) Schur-complement update for the FP32 factor.
//
// One CTA computes a 128 x 64 complex tile of  W B^T  with W = L_rows(i) D and
// B = L_rows(j) over the K = nbp (<= 128) columns of one panel; the caller
// subtracts it from the front (panel columns or contribution block). The
// complex product is four real products,
//     Cr += Ar Br^T - Ai Bi^T        Ci += Ar Bi^T + Ai Br^T,
// the minus sign carried by the instruction's A-negate bit. Each real operand
// is split three ways into TF32 numbers, x = hi + mid + lo (exactly), and the
// six significant cross products are kept,
//     a b ~ hh + (hm + mh + hl + lh + mm),
// so every product is more accurate than an FP32 multiply (the dropped terms
// are below 2^-32 relative). The tensor core's FP32 accumulation does not
// round to nearest, and its error grows with the number of MMAs chained into
// one accumulator, so the hh products and the small correction terms go to
// separate TMEM accumulators (Cr, Ci main; Cr, Ci corrections: 4 x 64
// columns), summed with a rounded FP32 add in the epilogue: 2 MMAs per 8
// columns of K reach the main accumulator instead of 12.
//
// Pipeline: K advances 8 columns per stage, 3 shared-memory stages. All 128
// threads load the next stage's operands into registers (coalesced column
// reads of the column-major panel) while earlier stages' MMAs run, split them
// and store them in the canonical K-major no-swizzle layout (8-row x 16-byte
// core matrices: LBO = 128 B between the two K-adjacent cores, SBO = 256 B
// between 8-row groups), 16 bytes per store. Thread 0 issues the stage's 24
// tcgen05.mma (kind::tf32, M = 128, N = 64, K = 8) and commits them to the
// stage's mbarrier; a stage is rewritten once that barrier shows its MMAs
// done. Every wait is bounded: on expiry the CTA stops issuing, waits (again
// bounded) for what it issued, frees its TMEM and reports failure.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tc_config.hpp"

namespace aphi_b200 {

constexpr long long kTcSpinLimit = 1LL << 22;   // bounded mbarrier waits (a stage takes microseconds)
constexpr uint32_t kTcSbo = 8 * kTcK * 4;       // bytes between 8-row core groups

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Canonical K-major, no-swizzle offset of element (row, k) inside a plane.
__device__ __forceinline__ uint32_t plane_off(int row, int k) {
    return (row >> 3) * kTcSbo + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3FFF);
    d |= static_cast<uint64_t>(128 >> 4) << 16;      // LBO: K-adjacent core matrices
    d |= static_cast<uint64_t>(kTcSbo >> 4) << 32;   // SBO: 8-row groups
    d |= static_cast<uint64_t>(1) << 46;             // descriptor version for sm_100
    return d;                                        // base offset 0, no swizzle
}

// kind::tf32 instruction descriptor: F32 accumulate, TF32 A and B, K-major.
__device__ __forceinline__ uint32_t instr_desc(int negate_a) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(negate_a) << 13) |
           (static_cast<uint32_t>(kTcN >> 3) << 17) | (static_cast<uint32_t>(kTcM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    for (long long i = 0; i < kTcSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32 lanes x 16 consecutive columns of TMEM into registers.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
          "=r"(v[15])
        : "r"(taddr));
}

// Four values -> hi, mid, lo (each exactly a TF32 number, hi + mid + lo == v)
// stored as one 16-byte row of a core matrix in each of three planes.
__device__ __forceinline__ void split_store4(unsigned char* plane0, int plane_bytes, uint32_t off, const float (&v)[4]) {
    float4 h, m, l;
    float* hp = &h.x;
    float* mp = &m.x;
    float* lp = &l.x;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float hi = tf32_round(v[q]);
        const float r1 = v[q] - hi;
        const float mid = tf32_round(r1);
        hp[q] = hi;
        mp[q] = mid;
        lp[q] = r1 - mid;
    }
    *reinterpret_cast<float4*>(plane0 + off) = h;
    *reinterpret_cast<float4*>(plane0 + plane_bytes + off) = m;
    *reinterpret_cast<float4*>(plane0 + 2 * plane_bytes + off) = l;
}

// Operands of one stage held in registers between load and store: A row tid
// (8 columns of K, scaled later by d), B row tid % 64 (4 columns: the half of
// the stage selected by tid / 64), and the stage's 8 pivots.
struct TcRegs {
    float2 a[kTcK];
    float2 b[4];
    float2 d[kTcK];
};

__device__ __forceinline__ void tc_load(TcRegs& R, const float2* P, long long ldp, int rows, int K, int i0, int j0,
                                        const float2* dk, long long dstride, int kbase) {
    const int tid = threadIdx.x;
    const int rb = tid & (kTcN - 1), qb = tid >> 6;
#pragma unroll
    for (int k = 0; k < kTcK; ++k) {
        const int kk = kbase + k;
        R.a[k] = make_float2(0.f, 0.f);
        R.d[k] = make_float2(0.f, 0.f);
        if (kk < K) {
            if (i0 + tid < rows) R.a[k] = P[static_cast<long long>(kk) * ldp + i0 + tid];
            R.d[k] = dk ? dk[static_cast<long long>(kk) * dstride] : make_float2(1.f, 0.f);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int kk = kbase + qb * 4 + q;
        R.b[q] = make_float2(0.f, 0.f);
        if (kk < K && j0 + rb < rows) R.b[q] = P[static_cast<long long>(kk) * ldp + j0 + rb];
    }
}

__device__ __forceinline__ void tc_store(const TcRegs& R, unsigned char* stage) {
    const int tid = threadIdx.x;
    unsigned char* A = stage;                                   // Ar hi/mid/lo, Ai hi/mid/lo
    unsigned char* B = stage + 2 * kTcSplit * kTcPlaneA;        // Br hi/mid/lo, Bi hi/mid/lo
#pragma unroll
    for (int g = 0; g < kTcK / 4; ++g) {
        float re[4], im[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 v = R.a[4 * g + q], d = R.d[4 * g + q];
            re[q] = v.x * d.x - v.y * d.y;
            im[q] = v.x * d.y + v.y * d.x;
        }
        const uint32_t o = plane_off(tid, 4 * g);
        split_store4(A, kTcPlaneA, o, re);
        split_store4(A + kTcSplit * kTcPlaneA, kTcPlaneA, o, im);
    }
    const int rb = tid & (kTcN - 1), qb = tid >> 6;
    float re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        re[q] = R.b[q].x;
        im[q] = R.b[q].y;
    }
    const uint32_t o = plane_off(rb, 4 * qb);
    split_store4(B, kTcPlaneB, o, re);
    split_store4(B + kTcSplit * kTcPlaneB, kTcPlaneB, o, im);
}

// The 24 MMAs of one stage: for each kept split pair (pa, pb), the four real
// products into Cr, Ci; pair 0 (hi, hi) into the main accumulators, the rest
// into the correction accumulators.
__device__ __forceinline__ void tc_issue(uint32_t stage_addr, uint32_t tmem, bool first) {
    const uint32_t A0 = stage_addr, B0 = stage_addr + 2 * kTcSplit * kTcPlaneA;
    const uint32_t id_pos = instr_desc(0), id_neg = instr_desc(1);
    const int pa[6] = {0, 0, 1, 0, 2, 1}, pb[6] = {0, 1, 0, 2, 0, 1};
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const uint64_t ar = smem_desc(A0 + pa[t] * kTcPlaneA);
        const uint64_t ai = smem_desc(A0 + (kTcSplit + pa[t]) * kTcPlaneA);
        const uint64_t br = smem_desc(B0 + pb[t] * kTcPlaneB);
        const uint64_t bi = smem_desc(B0 + (kTcSplit + pb[t]) * kTcPlaneB);
        const uint32_t d_re = tmem + (t == 0 ? 0 : 2 * kTcN);
        const uint32_t d_im = d_re + kTcN;
        const uint32_t acc = (first && (t == 0 || t == 1)) ? 0u : 1u;
        mma_tf32(d_re, ar, br, id_pos, acc);   // Cr += Ar Br^T
        mma_tf32(d_re, ai, bi, id_neg, 1);     // Cr -= Ai Bi^T
        mma_tf32(d_im, ar, bi, id_pos, acc);   // Ci += Ar Bi^T
        mma_tf32(d_im, ai, br, id_pos, 1);     // Ci += Ai Br^T
    }
}

// The tile: acc(r, c) = sum_k (P[i0 + r, k] d_k) P[j0 + c, k] for k < K, where
// P is a column-major panel (leading dimension ldp) and d_k = dk[k * dstride]
// (the front's pivots; all ones when dk is null). Rows at or beyond `rows`
// read as zero. The result is handed to `store(r, c0, re[16], im[16])`, 16
// consecutive columns c0.. of row r at a time, by the thread that owns row r
// (warp r / 32, lane r % 32).
// Requires kTcSmem bytes of dynamic shared memory (16-byte aligned). Returns
// false if a bounded wait expired (the caller records the error).
template <class Store>
__device__ bool tc_tile(unsigned char* smem, const float2* P, long long ldp, int rows, int K, int i0, int j0,
                        const float2* dk, long long dstride, Store store) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kTcStages * kTcStage);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + kTcStages);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    const int nst = (K + kTcK - 1) / kTcK;
    bool ok = true;
    int issued = 0;  // stages whose MMAs were issued and committed
    TcRegs cur, nxt;
    tc_load(cur, P, ldp, rows, K, i0, j0, dk, dstride, 0);
    for (int c = 0; c < nst; ++c) {
        const int s = c % kTcStages;
        if (c + 1 < nst) tc_load(nxt, P, ldp, rows, K, i0, j0, dk, dstride, (c + 1) * kTcK);
        // The stage's previous MMAs (stage c - 3) must be done before it is rewritten.
        bool mine = true;
        if (c >= kTcStages) mine = mbar_wait(smem_u32(mbar + s), ((c - kTcStages) / kTcStages) & 1);
        if (mine) tc_store(cur, smem + s * kTcStage);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        ok = __syncthreads_and(mine) != 0;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (!ok) break;
        if (tid == 0) {
            tc_issue(smem_u32(smem + s * kTcStage), tmem, c == 0);
            mma_commit(smem_u32(mbar + s));
        }
        ++issued;
        cur = nxt;
    }
    // Drain: every committed stage not yet waited for, oldest first.
    bool drained = true;
    for (int c = (issued > kTcStages ? issued - kTcStages : 0); c < issued; ++c)
        drained = mbar_wait(smem_u32(mbar + c % kTcStages), (c / kTcStages) & 1) && drained;
    drained = __syncthreads_and(drained) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    ok = ok && drained;
    if (ok) {
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        const int r = warp * 32 + lane;
        for (int c0 = 0; c0 < kTcN; c0 += 16) {
            uint32_t mr[16], cr[16], mi[16], ci[16];
            tmem_ld16(tmem + lane_base + c0, mr);
            tmem_ld16(tmem + lane_base + 2 * kTcN + c0, cr);
            tmem_ld16(tmem + lane_base + kTcN + c0, mi);
            tmem_ld16(tmem + lane_base + 3 * kTcN + c0, ci);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float re[16], im[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                re[c] = __uint_as_float(mr[c]) + __uint_as_float(cr[c]);
                im[c] = __uint_as_float(mi[c]) + __uint_as_float(ci[c]);
            }
            store(r, c0, re, im);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
    return ok;
}

}  // namespace aphi_b200
