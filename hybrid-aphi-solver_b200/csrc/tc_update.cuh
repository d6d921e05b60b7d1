// Tensor-core (tcgen05, sm_100a) Schur-complement update for the FP32 factor.
//
// One CTA computes a 128 x 64 complex tile of  W B^T  with W = L_rows(i) D and
// B = L_rows(j) over the K = nbp (<= 128) columns of one panel; the caller
// subtracts it from the front (panel columns or contribution block). The
// complex product is four real products,
//     Cr += Ar Br^T - Ai Bi^T        Ci += Ar Bi^T + Ai Br^T,
// the minus sign carried by the instruction's A-negate bit. Each real operand
// is split exactly into three TF32 numbers, x = hi + mid + lo, and the six
// significant cross products are kept,
//     a b ~ hh + (hm + mh + hl + lh + mm),
// so every product is more accurate than an FP32 multiply (the dropped terms
// are below 2^-32 relative): 24 tcgen05.mma (kind::tf32, M = 128, N = 64,
// K = 8) per 8 columns of K.
//
// Accumulation. The tensor core's FP32 accumulation truncates instead of
// rounding to nearest, and the error of a long chain of MMAs into one
// accumulator is biased. So the hh products of each group of kTcGroup stages
// go to a fresh TMEM accumulator (Cr, Ci main: 2 x 64 columns), which the
// threads then read and add to a running sum in registers with rounded FP32
// adds (thread r holds row r: 64 complex); no truncating chain is longer
// than 2 kTcGroup MMAs. The correction terms, 2^-11 of the main ones and
// below, accumulate over the whole K in their own TMEM accumulator (Cr, Ci:
// 2 x 64 columns), where their truncation is negligible.
//
// Two-piece split (hi + lo; products hh, hl, lh) uses a stacked B layout:
// per piece the planes -Bi, Br, Bi lie back to back, so [Br; Bi] and
// [-Bi; Br] are 128-row operands and each kept pair costs two M128 N128 MMAs
// ([Cr | Ci] += Ar [Br | Bi]^T + Ai [-Bi | Br]^T) instead of four M128 N64
// ones: half the MMA instructions and a third less operand traffic.
//
// Pipeline: K advances 8 columns per stage. Raw operands (A rows, B rows and
// the stage's pivots, complex64) are fetched by cp.async into a ring of
// kTcRawStages buffers, two stages ahead, so no registers hold them in
// flight. Each stage, the threads split the raw stage into the canonical
// K-major no-swizzle layout (8-row x 16-byte core matrices: LBO = 128 B
// between the two K-adjacent cores, SBO = 256 B between 8-row groups; 16-byte
// stores) in one of kTcPlaneStages plane buffers; thread 0 issues the stage's
// 24 MMAs and commits them to the buffer's mbarrier, which the threads wait
// on before rewriting it. Every wait is bounded: on expiry the CTA stops
// issuing, waits (again bounded) for what it issued, frees its TMEM and
// reports failure.
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

// kind::tf32 instruction descriptor: F32 accumulate, TF32 A and B, K-major,
// M = kTcM, N = n (a multiple of 16, 16..256).
__device__ __forceinline__ uint32_t instr_desc(int negate_a, int n = kTcN) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(negate_a) << 13) |
           (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(kTcM >> 4) << 24);
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

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, long long limit = kTcSpinLimit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try(mbar, phase)) return true;
    return false;
}

// A bounded wait that also gives up as soon as another thread of the CTA
// has recorded a failure (*failed != 0): what it waits for may then never
// come.
__device__ __forceinline__ bool mbar_wait_live(uint32_t mbar, uint32_t phase, const volatile int* failed) {
    for (long long i = 0; i < kTcSpinLimit; ++i) {
        if (mbar_try(mbar, phase)) return true;
        if (*failed) return false;
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

// 8-byte global -> shared copy without a register round trip; bytes < 8
// (here 0) fills the rest of the destination with zeros.
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Four values -> their TF32 pieces, stored as one 16-byte row of a core
// matrix in each of Split planes. Split 3: hi, mid, lo, each exactly a TF32
// number, hi + mid + lo == v. Split 2: hi and lo = the rounded remainder,
// hi + lo == v to 2^-22 relative.
template <int Split, bool Negate = false>
__device__ __forceinline__ void split_store4(unsigned char* plane0, int plane_bytes, uint32_t off, const float (&v)[4],
                                             unsigned char* neg0 = nullptr) {
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
    if constexpr (Split == 3) *reinterpret_cast<float4*>(plane0 + 2 * plane_bytes + off) = l;
    if constexpr (Negate) {  // the pieces of -v: the negated pieces of v, exactly
        *reinterpret_cast<float4*>(neg0 + off) = make_float4(-h.x, -h.y, -h.z, -h.w);
        *reinterpret_cast<float4*>(neg0 + plane_bytes + off) = make_float4(-m.x, -m.y, -m.z, -m.w);
        if constexpr (Split == 3)
            *reinterpret_cast<float4*>(neg0 + 2 * plane_bytes + off) = make_float4(-l.x, -l.y, -l.z, -l.w);
    }
}

// Raw stage: A rows [k][128], B rows [k][64], pivots [k] (complex64). Thread
// tid fetches A row tid for the 8 columns, B row tid % 64 for columns
// 4 (tid / 64) .. +3, and (tid < 8) pivot tid; entries past the panel or the
// front read as zero.
__device__ __forceinline__ void tc_fetch(unsigned char* raw, const float2* P, long long ldp, int rows, int K,
                                         int i0, int j0, const float2* dk, long long dstride, int kbase) {
    const int tid = threadIdx.x;
    const uint32_t ra = smem_u32(raw), rb = ra + kTcRawA, rd = rb + kTcRawB;
#pragma unroll
    for (int k = 0; k < kTcK; ++k) {
        const int kk = kbase + k;
        const bool in = kk < K && i0 + tid < rows;
        cp_async8(ra + (k * kTcM + tid) * 8, in ? P + static_cast<long long>(kk) * ldp + i0 + tid : P, in ? 8u : 0u);
    }
    const int rowb = tid & (kTcN - 1), qb = tid >> 6;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = qb * 4 + q, kk = kbase + k;
        const bool in = kk < K && j0 + rowb < rows;
        cp_async8(rb + (k * kTcN + rowb) * 8, in ? P + static_cast<long long>(kk) * ldp + j0 + rowb : P,
                  in ? 8u : 0u);
    }
    if (tid < kTcK) {
        const int kk = kbase + tid;
        if (dk) {
            cp_async8(rd + tid * 8, kk < K ? dk + static_cast<long long>(kk) * dstride : dk, kk < K ? 8u : 0u);
        } else {
            *reinterpret_cast<float2*>(raw + kTcRawA + kTcRawB + tid * 8) = make_float2(kk < K ? 1.f : 0.f, 0.f);
        }
    }
}

// Raw stage -> split planes (A scaled by the pivots).
template <int Split>
__device__ __forceinline__ void tc_split(const unsigned char* raw, unsigned char* stage) {
    const int tid = threadIdx.x;
    const float2* rA = reinterpret_cast<const float2*>(raw);
    const float2* rB = reinterpret_cast<const float2*>(raw + kTcRawA);
    const float2* rD = reinterpret_cast<const float2*>(raw + kTcRawA + kTcRawB);
    unsigned char* A = stage;                                   // Ar pieces, then Ai pieces
    unsigned char* B = stage + 2 * Split * kTcPlaneA;           // B pieces (layout: TcLayout<Split>)
#pragma unroll
    for (int g = 0; g < kTcK / 4; ++g) {
        float re[4], im[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 v = rA[(4 * g + q) * kTcM + tid], d = rD[4 * g + q];
            re[q] = v.x * d.x - v.y * d.y;
            im[q] = v.x * d.y + v.y * d.x;
        }
        const uint32_t o = plane_off(tid, 4 * g);
        split_store4<Split>(A, kTcPlaneA, o, re);
        split_store4<Split>(A + Split * kTcPlaneA, kTcPlaneA, o, im);
    }
    const int rowb = tid & (kTcN - 1), qb = tid >> 6;
    float re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float2 v = rB[(qb * 4 + q) * kTcN + rowb];
        re[q] = v.x;
        im[q] = v.y;
    }
    const uint32_t o = plane_off(rowb, 4 * qb);
    if constexpr (TcLayout<Split>::stacked) {
        // per piece p: [-Bi_p | Br_p | Bi_p], three 64-row planes in a row
        split_store4<Split>(B + kTcPlaneB, 3 * kTcPlaneB, o, re);
        split_store4<Split, true>(B + 2 * kTcPlaneB, 3 * kTcPlaneB, o, im, B);
    } else {
        split_store4<Split>(B, kTcPlaneB, o, re);
        split_store4<Split>(B + Split * kTcPlaneB, kTcPlaneB, o, im);
    }
}

// The MMAs of one stage: for each kept split pair (pa, pb), the four real
// products into Cr, Ci; pair 0 (hi, hi) into the main accumulators (restarted
// when fresh_main), the rest into the correction accumulators (restarted when
// fresh_corr). Split 3 keeps six pairs (hh, hm, mh, hl, lh, mm: 24 MMAs),
// split 2 three (hh, hl, lh: 12 MMAs).
template <int Split>
__device__ __forceinline__ void tc_issue(uint32_t stage_addr, uint32_t tmem, bool fresh_main, bool fresh_corr) {
    const uint32_t A0 = stage_addr, B0 = stage_addr + 2 * Split * kTcPlaneA;
    const uint32_t id_pos = instr_desc(0), id_neg = instr_desc(1);
    constexpr int np = Split == 3 ? 6 : 3;
    const int pa[6] = {0, 0, 1, 0, 2, 1}, pb[6] = {0, 1, 0, 2, 0, 1};
    if constexpr (TcLayout<Split>::stacked) {
        // [Cr | Ci] (128 accumulator columns) += Ar [Br | Bi]^T + Ai [-Bi | Br]^T:
        // two M128 N128 MMAs per kept pair, the B operands 128-row stacks.
        const uint32_t id128 = instr_desc(0, 2 * kTcN);
#pragma unroll
        for (int t = 0; t < np; ++t) {
            const uint64_t ar = smem_desc(A0 + pa[t] * kTcPlaneA);
            const uint64_t ai = smem_desc(A0 + (Split + pa[t]) * kTcPlaneA);
            const uint32_t blk = B0 + pb[t] * 3 * kTcPlaneB;
            const uint64_t b_ri = smem_desc(blk + kTcPlaneB);   // [Br; Bi]
            const uint64_t b_nr = smem_desc(blk);               // [-Bi; Br]
            const uint32_t d = tmem + (t == 0 ? 0 : 2 * kTcN);
            const bool fresh = t == 0 ? fresh_main : (t == 1 && fresh_corr);
            mma_tf32(d, ar, b_ri, id128, fresh ? 0u : 1u);
            mma_tf32(d, ai, b_nr, id128, 1);
        }
        return;
    }
#pragma unroll
    for (int t = 0; t < np; ++t) {
        const uint64_t ar = smem_desc(A0 + pa[t] * kTcPlaneA);
        const uint64_t ai = smem_desc(A0 + (Split + pa[t]) * kTcPlaneA);
        const uint64_t br = smem_desc(B0 + pb[t] * kTcPlaneB);
        const uint64_t bi = smem_desc(B0 + (Split + pb[t]) * kTcPlaneB);
        const uint32_t d_re = tmem + (t == 0 ? 0 : 2 * kTcN);
        const uint32_t d_im = d_re + kTcN;
        const bool fresh = t == 0 ? fresh_main : (t == 1 && fresh_corr);
        const uint32_t acc = fresh ? 0u : 1u;
        mma_tf32(d_re, ar, br, id_pos, acc);   // Cr += Ar Br^T
        mma_tf32(d_re, ai, bi, id_neg, 1);     // Cr -= Ai Bi^T
        mma_tf32(d_im, ar, bi, id_pos, acc);   // Ci += Ar Bi^T
        mma_tf32(d_im, ai, br, id_pos, 1);     // Ci += Ai Br^T
    }
}

// Adds the main accumulators (this warp's 32 lanes, 64 columns) to the
// running sums, rounding to nearest.
__device__ __forceinline__ void tc_drain(uint32_t tmem, float (&sr)[kTcN], float (&si)[kTcN]) {
    const uint32_t lane_base = static_cast<uint32_t>((threadIdx.x >> 5) * 32) << 16;
#pragma unroll
    for (int c0 = 0; c0 < kTcN; c0 += 16) {
        uint32_t vr[16], vi[16];
        tmem_ld16(tmem + lane_base + c0, vr);
        tmem_ld16(tmem + lane_base + kTcN + c0, vi);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            sr[c0 + c] += __uint_as_float(vr[c]);
            si[c0 + c] += __uint_as_float(vi[c]);
        }
    }
}

// The tile: acc(r, c) = sum_k (P[i0 + r, k] d_k) P[j0 + c, k] for k < K, where
// P is a column-major panel (leading dimension ldp) and d_k = dk[k * dstride]
// (the front's pivots; all ones when dk is null). Rows at or beyond `rows`
// read as zero. The result is handed to `store(r, c0, re[16], im[16])`, 16
// consecutive columns c0.. of row r at a time, by the thread that owns row r
// (warp r / 32, lane r % 32). Requires kTcSmem bytes of dynamic shared
// memory (16-byte aligned). Returns false if a bounded wait expired (the
// caller records the error).
template <int Split, int Stages = kTcPlaneStages, int Group = kTcGroup, class Store>
__device__ bool tc_tile(unsigned char* smem, const float2* P, long long ldp, int rows, int K, int i0, int j0,
                        const float2* dk, long long dstride, Store store) {
    constexpr int kStage = TcBytes<Split>::stage;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    unsigned char* planes = smem;
    unsigned char* raws = smem + Stages * kStage;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(raws + kTcRawStages * kTcRawStage);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + Stages);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < Stages; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    const int nst = (K + kTcK - 1) / kTcK;
    // Two raw stages in flight before the loop.
    for (int c = 0; c < 2; ++c) {
        if (c < nst) tc_fetch(raws + c * kTcRawStage, P, ldp, rows, K, i0, j0, dk, dstride, c * kTcK);
        cp_async_commit();
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    float sr[kTcN], si[kTcN];
#pragma unroll
    for (int c = 0; c < kTcN; ++c) sr[c] = si[c] = 0.f;
    bool ok = true;
    int issued = 0;  // stages whose MMAs were issued and committed
    for (int c = 0; c < nst; ++c) {
        const int buf = c % Stages;
        if (c + 2 < nst)
            tc_fetch(raws + ((c + 2) % kTcRawStages) * kTcRawStage, P, ldp, rows, K, i0, j0, dk, dstride,
                     (c + 2) * kTcK);
        cp_async_commit();
        cp_async_wait<2>();  // this thread's copies of stage c have landed
        bool mine = true;
        // The plane buffer's previous MMAs (stage c - 2) must be done.
        if (c >= Stages)
            mine = mbar_wait(smem_u32(mbar + buf), ((c - Stages) / Stages) & 1);
        ok = __syncthreads_and(mine) != 0;  // also: every thread's raw copies of stage c are visible
        if (!ok) break;
        tc_split<Split>(raws + (c % kTcRawStages) * kTcRawStage, planes + buf * kStage);
        // Generic-proxy stores -> visible to the tensor core's async proxy.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        // A new group starts: the previous group's main products, complete
        // once stage c - 1's commit has arrived, go to the running sums
        // (after the split, so the split overlaps those MMAs).
        const bool group_start = c % Group == 0;
        if (group_start && c > 0) {
            const int p = c - 1;
            mine = mbar_wait(smem_u32(mbar + p % Stages), (p / Stages) & 1);
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (mine) tc_drain(tmem, sr, si);
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        ok = __syncthreads_and(mine) != 0;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (!ok) break;
        if (tid == 0) {
            tc_issue<Split>(smem_u32(planes + buf * kStage), tmem, group_start, c == 0);
            mma_commit(smem_u32(mbar + buf));
        }
        ++issued;
    }
    cp_async_wait<0>();
    // Drain: every committed stage not yet waited for, oldest first.
    bool drained = true;
    for (int c = (issued > Stages ? issued - Stages : 0); c < issued; ++c)
        drained = mbar_wait(smem_u32(mbar + c % Stages), (c / Stages) & 1) && drained;
    drained = __syncthreads_and(drained) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    ok = ok && drained;
    if (ok) {
        tc_drain(tmem, sr, si);  // the last group
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        const int r = warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < kTcN; c0 += 16) {
            uint32_t cr[16], ci[16];
            tmem_ld16(tmem + lane_base + 2 * kTcN + c0, cr);
            tmem_ld16(tmem + lane_base + 3 * kTcN + c0, ci);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float re[16], im[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                re[c] = sr[c0 + c] + __uint_as_float(cr[c]);
                im[c] = si[c0 + c] + __uint_as_float(ci[c]);
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

// ---------------------------------------------------------------- pre-split operands
// The two-piece tile with its operands split once per panel group instead of
// once per tile: k_tc_split writes each front's trailing rows as the tile's
// canonical planes (A = L D and B = L, hi and lo pieces, the stacked B form)
// into a workspace region, laid out so that one stage of one tile's A rows
// (four 128-row planes, 16 KB) and of its B rows (six 64-row planes, 12 KB)
// are each one contiguous block:
//   A part: [128-row block][stage][Ar hi, Ar lo, Ai hi, Ai lo]
//   B part: [64-row block][stage][-Bi hi, Br hi, Bi hi, -Bi lo, Br lo, Bi lo]
// (the B part follows the A part). The tile then only moves bytes and issues
// MMAs, in two roles that run side by side: a producer thread (warp 0, lane
// 0) stages each 8-column stage with two bulk asynchronous copies
// (cp.async.bulk, no threads moving data) into one of Stages plane buffers,
// completing on the buffer's "full" mbarrier by transaction count, as soon as
// the buffer's previous MMAs are done; an issuer thread (warp 1, lane 0)
// issues each stage's six MMAs once its buffer is full and commits them to
// the buffer's "empty" mbarrier. All threads drain the main accumulator every
// Group stages, as in tc_tile. Every wait is bounded, and gives up early once
// the other role has failed.
namespace aphi_b200 {

constexpr int kTcPreA = 2 * 2 * kTcPlaneA;  // one stage of a 128-row A block
constexpr int kTcPreB = 3 * 2 * kTcPlaneB;  // one stage of a 64-row B block
static_assert(kTcPreA + kTcPreB == TcBytes<2>::stage, "pre-split stage = the two-piece tile's plane stage");

// Byte offsets, inside a front's region (R padded trailing rows, nst stages),
// of stage c of the A block holding trailing row r (r / 128) and of the B
// block holding it (r / 64).
__device__ __forceinline__ long long pre_a_off(int R, int nst, int r, int c) {
    (void)R;
    return (static_cast<long long>(r >> 7) * nst + c) * kTcPreA;
}
__device__ __forceinline__ long long pre_b_off(int R, int nst, int r, int c) {
    return static_cast<long long>(R >> 7) * nst * kTcPreA + (static_cast<long long>(r >> 6) * nst + c) * kTcPreB;
}

// Dynamic shared memory of the pre-split tile with `Stages` plane buffers
// (three fit two CTAs per SM comfortably, four just).
template <int Stages>
struct TcPreSmem {
    static constexpr int bytes = Stages * TcBytes<2>::stage + 2 * Stages * 8 + 64;
};

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// region: the front's planes for this entry (layout above); R: the front's
// padded trailing rows; nst: stages; ra, rb: the tile's first A and B rows
// within the trailing part (ra a multiple of 128, rb of 64). Same result
// contract as tc_tile; requires kTcThreads threads.
template <int Group, int Stages, class Store>
__device__ bool tc_tile_presplit(unsigned char* smem, const unsigned char* region, int R, int nst, int ra, int rb,
                                 Store store) {
    constexpr int P = Stages;
    constexpr int kStage = TcBytes<2>::stage;
    constexpr int kProducer = 0, kIssuer = 32;
    // A group's drain waits on its last stage's commit only (s - 1, buffer
    // (s - 1) % P). That parity wait is exact as long as the buffer's previous
    // commit (stage s - 1 - P) has already arrived: with Group <= Stages that
    // stage is no later than the one the previous drain waited for, and a
    // commit arrives only once every earlier MMA of the issuing thread has
    // completed, in issue order. (Waiting on each stage of the group in turn
    // instead measured 1.7x slower on the 32^3 factorization.)
    static_assert(Group <= Stages, "an accumulator group must not span more stages than there are buffers");
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    unsigned char* planes = smem;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + P * kStage);
    uint64_t* empty = full + P;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(empty + P);
    volatile int* state = reinterpret_cast<volatile int*>(tmem_slot + 1);  // [0] failed, [1] stages committed, [2] stages loaded

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < P; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + b)));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(empty + b)));
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
        state[0] = 0;
        state[1] = 0;
        state[2] = 0;
    }
    auto load_stage = [&](int c) {  // producer
        const int b = c % P;
        const uint32_t dst = smem_u32(planes + b * kStage);
        const uint32_t fb = smem_u32(full + b);
        mbar_expect_tx(fb, kStage);
        bulk_g2s(dst, region + pre_a_off(R, nst, ra, c), kTcPreA, fb);
        bulk_g2s(dst + kTcPreA, region + pre_b_off(R, nst, rb, c), kTcPreB, fb);
    };
    __syncthreads();
    if (tid == kProducer) {
        const int pre = min(P - 1, nst);
        for (int c = 0; c < pre; ++c) load_stage(c);
        state[2] = pre;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    float sr[kTcN], si[kTcN];
#pragma unroll
    for (int c = 0; c < kTcN; ++c) sr[c] = si[c] = 0.f;
    bool ok = true;
    for (int s = 0; s < nst; ++s) {
        const int b = s % P;
        const bool group_start = s % Group == 0;
        if (group_start && s > 0) {
            // The previous group's main products are complete once stage s - 1's
            // commit has arrived: into the running sums before stage s
            // restarts the main accumulator.
            const int p = s - 1;
            bool mine = mbar_wait_live(smem_u32(empty + p % P), (p / P) & 1, state);
            mine = __all_sync(0xffffffffu, mine);  // the TMEM loads are warp-wide
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (mine) tc_drain(tmem, sr, si);
            asm volatile("tcgen05.fence::before_thread_sync;");
            ok = __syncthreads_and(mine) != 0;
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (!ok) break;
        }
        if (tid == kIssuer && !state[0]) {
            if (mbar_wait_live(smem_u32(full + b), (s / P) & 1, state)) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                tc_issue<2>(smem_u32(planes + b * kStage), tmem, group_start, s == 0);
                mma_commit(smem_u32(empty + b));
                state[1] = s + 1;
            } else {
                state[0] = 1;
            }
        }
        if (tid == kProducer && !state[0]) {
            // buffer (s + P - 1) % P was stage s - 1's: refill it once those MMAs are done
            const int t = s + P - 1;
            if (t < nst) {
                if (s == 0 || mbar_wait_live(smem_u32(empty + (s - 1) % P), ((s - 1) / P) & 1, state)) {
                    load_stage(t);
                    state[2] = t + 1;
                } else {
                    state[0] = 1;
                }
            }
        }
    }
    __syncthreads();
    const int committed = state[1], loaded = state[2];
    ok = ok && !state[0];
    // Drain: the last committed stage's MMAs (all earlier ones complete before
    // it), and any copies issued but never consumed (only after a failure).
    bool drained = true;
    if (committed > 0)
        drained = mbar_wait(smem_u32(empty + (committed - 1) % P), ((committed - 1) / P) & 1);
    if (tid == kProducer)
        for (int c = committed; c < loaded; ++c) drained = mbar_wait(smem_u32(full + c % P), (c / P) & 1) && drained;
    drained = __syncthreads_and(drained) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    ok = ok && drained && committed == nst;
    if (ok) {
        tc_drain(tmem, sr, si);  // the last group
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        const int r = warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < kTcN; c0 += 16) {
            uint32_t cr[16], ci[16];
            tmem_ld16(tmem + lane_base + 2 * kTcN + c0, cr);
            tmem_ld16(tmem + lane_base + 3 * kTcN + c0, ci);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float re[16], im[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                re[c] = sr[c0 + c] + __uint_as_float(cr[c]);
                im[c] = si[c0 + c] + __uint_as_float(ci[c]);
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
