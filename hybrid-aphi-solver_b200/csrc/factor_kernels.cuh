// Device kernels of the supernodal multifrontal complex-symmetric LDL^T and
// its solves, templated on the real type R (double: complex128 factor;
// float: complex64 factor). No conjugation anywhere: the matrices are complex
// symmetric (A = A^T), so every product below is a plain transpose product.
//
// Front layout. Supernode s owns columns [first, first + w) of the
// post-ordered matrix and the sorted row structure struct_s (m rows, the
// first w being its own columns). Its front is m x m; the first w columns
// live in the panel L_s (m x w, column-major, leading dimension m, inside the
// factor storage), the trailing (m - w) x (m - w) block -- the contribution
// block CB_s -- in the CB pool. After factorization the panel holds D on its
// diagonal and the multipliers below it.
#pragma once

#include <cuda_runtime.h>

#include "analysis.hpp"
#include "common.cuh"
#include "tc_update.cuh"

namespace aphi_b200 {

template <class R>
struct cx {
    R re, im;
};

template <class R>
__device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) {
    return {a.re + b.re, a.im + b.im};
}
template <class R>
__device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) {
    return {a.re - b.re, a.im - b.im};
}
// a - b * c
template <class R>
__device__ __forceinline__ cx<R> fms(cx<R> a, cx<R> b, cx<R> c) {
    return {a.re - b.re * c.re + b.im * c.im, a.im - b.re * c.im - b.im * c.re};
}
// 1 / d, scaled so that neither component over- nor underflows for ordinary d.
template <class R>
__device__ __forceinline__ cx<R> crecip(cx<R> d) {
    if (fabs(d.re) >= fabs(d.im)) {
        const R r = d.im / d.re;
        const R den = d.re + d.im * r;
        return {R(1) / den, -r / den};
    }
    const R r = d.re / d.im;
    const R den = d.re * r + d.im;
    return {r / den, R(-1) / den};
}
template <class R>
__device__ __forceinline__ double cabs_d(cx<R> a) {
    return hypot(static_cast<double>(a.re), static_cast<double>(a.im));
}

struct Sched {
    const int* first;
    const int* rows;
    const long long* loff;
    const long long* cboff;
    const long long* soff;
    const int* structs;
    const long long* reloff;
    const int* rel;
    const int* child_ptr;
    const int* child_list;
    const long long* uoff;
    const Item* items;
};

inline Sched sched_of(const DeviceSchedule& d) {
    return Sched{d.first, d.rows, d.loff, d.cboff, d.soff, d.structs, d.reloff, d.rel,
                 d.child_ptr, d.child_list, d.uoff, d.items};
}

// ---------------------------------------------------------------- extend-add
// Item (s, c0): front columns [c0, c0 + 32) of supernode s. Zeroes the CB
// columns in that range, then adds every child's contribution block entries
// that land in it, children in ascending order (a fixed summation order).
template <class R>
__global__ void __launch_bounds__(256) k_extend_add(Sched S, long long item0, cx<R>* Lb, cx<R>* CBb,
                                                    long long lstride, long long cbstride) {
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, c0 = it.a;
    cx<R>* L = Lb + lstride * blockIdx.y;
    cx<R>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int c1 = min(c0 + kEaCols, m);
    cx<R>* Ls = L + S.loff[s];
    cx<R>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = max(c0, w) + warp; j < c1; j += 8)
        for (int i = j + lane; i < m; i += 32) CBs[(i - w) + static_cast<long long>(j - w) * cs] = cx<R>{0, 0};
    __syncthreads();
    for (int t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
        const int c = S.child_list[t];
        const int cw = S.first[c + 1] - S.first[c];
        const int cc = S.rows[c] - cw;
        if (cc <= 0) continue;
        const int* rel = S.rel + S.reloff[c];
        const cx<R>* CBc = CB + S.cboff[c];
        // Child columns whose parent position falls in [c0, c1): binary search.
        int lo = 0, hi = cc;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (rel[mid] < c0) lo = mid + 1; else hi = mid;
        }
        const int j0 = lo;
        hi = cc;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (rel[mid] < c1) lo = mid + 1; else hi = mid;
        }
        const int j1 = lo;
        for (int j = j0 + warp; j < j1; j += 8) {
            const int pj = rel[j];
            const cx<R>* src = CBc + static_cast<long long>(j) * cc;
            if (pj < w) {
                cx<R>* dst = Ls + static_cast<long long>(pj) * m;
                for (int i = j + lane; i < cc; i += 32) dst[rel[i]] = dst[rel[i]] + src[i];
            } else {
                cx<R>* dst = CBs + static_cast<long long>(pj - w) * cs - w;
                for (int i = j + lane; i < cc; i += 32) dst[rel[i]] = dst[rel[i]] + src[i];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- small fronts
// One CTA factorizes a whole front (m <= 96) in shared memory.
template <class R>
__global__ void __launch_bounds__(256) k_small_front(Sched S, long long item0, cx<R>* Lb, cx<R>* CBb,
                                                     long long lstride, long long cbstride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* F = reinterpret_cast<cx<R>*>(smem_raw);
    const int s = S.items[item0 + blockIdx.x].s;
    cx<R>* L = Lb + lstride * blockIdx.y;
    cx<R>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    cx<R>* Ls = L + S.loff[s];
    cx<R>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const int nt = blockDim.x;
    for (int e = threadIdx.x; e < m * m; e += nt) {
        const int i = e % m, j = e / m;
        cx<R> v{0, 0};
        if (i >= j) v = (j < w) ? Ls[e] : CBs[(i - w) + static_cast<long long>(j - w) * cs];
        F[e] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = nt >> 5;
    for (int k = 0; k < w; ++k) {
        const cx<R> inv = crecip(F[k + k * m]);
        for (int j = k + 1 + warp; j < m; j += nw) {
            const cx<R> ljk = F[j + k * m] * inv;
            for (int i = j + lane; i < m; i += 32) F[i + j * m] = fms(F[i + j * m], F[i + k * m], ljk);
        }
        __syncthreads();
        for (int i = k + 1 + threadIdx.x; i < m; i += nt) F[i + k * m] = F[i + k * m] * inv;
        __syncthreads();
    }
    for (int e = threadIdx.x; e < m * m; e += nt) {
        const int i = e % m, j = e / m;
        if (i < j) continue;
        if (j < w)
            Ls[e] = F[e];
        else
            CBs[(i - w) + static_cast<long long>(j - w) * cs] = F[e];
    }
}

// ---------------------------------------------------------------- blocked fronts
// Step k0 of a large front: factor the kb x kb diagonal block in place. The
// block is staged with every thread's loads in flight. At step k warp v
// updates columns k + 1 + v, k + 5 + v, ... and lane l the entry l rows below
// each column's diagonal (the lower triangle only, no index division); each
// entry gets the same arithmetic, in the same order of k, as before.
template <class R>
__global__ void __launch_bounds__(128) k_diag_block(Sched S, long long item0, cx<R>* Lb, long long lstride) {
    static_assert(kStep == 32 && kStep * kStep % 128 == 0, "one lane per row, eight entries per thread");
    __shared__ cx<R> F[kStep * kStep];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, k0 = it.a;
    cx<R>* L = Lb + lstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int kb = min(kStep, w - k0);
    cx<R>* D = L + S.loff[s] + k0 + static_cast<long long>(k0) * m;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        cx<R> v[kStep * kStep / 128];
#pragma unroll
        for (int u = 0; u < kStep * kStep / 128; ++u) {
            const int e = tid + 128 * u, i = e % kStep, j = e / kStep;
            v[u] = i < kb && j < kb ? D[i + static_cast<long long>(j) * m] : cx<R>{0, 0};
        }
#pragma unroll
        for (int u = 0; u < kStep * kStep / 128; ++u) F[tid + 128 * u] = v[u];
    }
    __syncthreads();
    for (int k = 0; k < kb; ++k) {
        const cx<R> inv = crecip(F[k + k * kStep]);
        for (int j = k + 1 + warp; j < kb; j += 4) {
            const int i = j + lane;
            if (i < kb) F[i + j * kStep] = fms(F[i + j * kStep], F[i + k * kStep], F[j + k * kStep] * inv);
        }
        __syncthreads();
        for (int i = k + 1 + tid; i < kb; i += blockDim.x) F[i + k * kStep] = F[i + k * kStep] * inv;
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < kStep * kStep / 128; ++u) {
        const int e = tid + 128 * u, i = e % kStep, j = e / kStep;
        if (i < kb && j < kb && i >= j) D[i + static_cast<long long>(j) * m] = F[e];
    }
}

// Rows row0 .. row0+127 of the panel below the diagonal block of step k0:
// L21 = A21 L11^-T D^-1, one row per thread.
template <class R>
__global__ void __launch_bounds__(kTrsmRows) k_panel_trsm(Sched S, long long item0, cx<R>* Lb, long long lstride) {
    __shared__ cx<R> T[kStep * kStep];
    __shared__ cx<R> Dinv[kStep];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, k0 = it.a, row0 = it.b;
    cx<R>* L = Lb + lstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int kb = min(kStep, w - k0);
    cx<R>* P = L + S.loff[s] + static_cast<long long>(k0) * m;  // column k0 of the panel
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        T[i + j * kStep] = P[k0 + i + static_cast<long long>(j) * m];
    }
    __syncthreads();
    if (threadIdx.x < kb) Dinv[threadIdx.x] = crecip(T[threadIdx.x * (kStep + 1)]);
    __syncthreads();
    const int i = row0 + threadIdx.x;
    if (i >= m) return;
    cx<R> x[kStep];
#pragma unroll
    for (int j = 0; j < kStep; ++j)
        if (j < kb) x[j] = P[i + static_cast<long long>(j) * m];
#pragma unroll
    for (int j = 0; j < kStep; ++j) {
        if (j >= kb) break;
        cx<R> v = x[j];
#pragma unroll
        for (int t = 0; t < kStep; ++t) {
            if (t >= j) break;
            v = fms(v, T[j + t * kStep], x[t]);
        }
        x[j] = v;
    }
#pragma unroll
    for (int j = 0; j < kStep; ++j)
        if (j < kb) P[i + static_cast<long long>(j) * m] = x[j] * Dinv[j];
}

// In-panel update tile (i0, j0) of step k0: F[i, j] -= sum_t L[i,t] D[t] L[j,t]
// over the step's kb columns t, for i >= j >= k0 + kb and j inside the
// current 128-column panel (the columns to its right get the whole panel's
// update at once when the panel is complete).
template <class R>
__global__ void __launch_bounds__(256) k_update_panel(Sched S, long long item0, cx<R>* Lb, cx<R>* CBb,
                                                      long long lstride, long long cbstride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* As = reinterpret_cast<cx<R>*>(smem_raw);  // [kStep][kTile], scaled by D
    cx<R>* Bs = As + kStep * kTile;                  // [kStep][kTile]
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, k0 = it.a, i0 = it.b, j0 = it.c;
    cx<R>* L = Lb + lstride * blockIdx.y;
    cx<R>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int kb = min(kStep, w - k0);
    const cx<R>* P = L + S.loff[s] + static_cast<long long>(k0) * m;
    for (int e = threadIdx.x; e < kStep * kTile; e += blockDim.x) {
        const int r = e % kTile, t = e / kTile;
        cx<R> a{0, 0}, b{0, 0};
        if (t < kb) {
            const cx<R> d = P[k0 + t + static_cast<long long>(t) * m];
            if (i0 + r < m) a = P[i0 + r + static_cast<long long>(t) * m] * d;
            if (j0 + r < m) b = P[j0 + r + static_cast<long long>(t) * m];
        }
        As[t * kTile + r] = a;
        Bs[t * kTile + r] = b;
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    cx<R> acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = cx<R>{0, 0};
    for (int t = 0; t < kb; ++t) {
        cx<R> av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = As[t * kTile + tx + 16 * a];
#pragma unroll
        for (int b = 0; b < 4; ++b) bv[b] = Bs[t * kTile + ty + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                acc[a][b].re += av[a].re * bv[b].re - av[a].im * bv[b].im;
                acc[a][b].im += av[a].re * bv[b].im + av[a].im * bv[b].re;
            }
    }
    cx<R>* Ls = L + S.loff[s];
    cx<R>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const int jend = min(w, (k0 / kTcPanel) * kTcPanel + kTcPanel);
    // Read-modify-write: all 16 loads first, so their latencies overlap.
    cx<R>* dst[4][4];
    cx<R> old[4][4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = j0 + ty + 16 * b;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + tx + 16 * a;
            dst[a][b] = nullptr;
            if (j < jend && i < m && i >= j)
                dst[a][b] = (j < w) ? Ls + i + static_cast<long long>(j) * m
                                    : CBs + (i - w) + static_cast<long long>(j - w) * cs;
            if (dst[a][b]) old[a][b] = *dst[a][b];
        }
    }
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int a = 0; a < 4; ++a)
            if (dst[a][b]) *dst[a][b] = old[a][b] - acc[a][b];
}

// SIMT trailing update of a complete panel (either precision). Item
// (s, p0, i0, j0): F[i, j] -= sum_{t in panel} L[i,t] D[t] L[j,t] over the
// 128 x 64 tile at rows i0.., columns j0.. (i >= j); K is the panel width
// (<= 128), consumed 8 columns at a time through double-buffered shared
// memory, the next chunk's loads in flight while the current one is used.
// 256 threads, each an 8 x 4 block of complex accumulators (rows tx + 16a,
// columns ty + 16b): per column t a thread reads 12 shared entries for 32
// complex multiply-adds.
constexpr int kWideM = 128, kWideN = 64, kWideKC = 8;

template <class R>
constexpr int wide_smem() {
    return 2 * kWideKC * (kWideM + kWideN) * static_cast<int>(sizeof(cx<R>));
}

template <class R>
__global__ void __launch_bounds__(256) k_update_wide(Sched S, long long item0, cx<R>* Lb, cx<R>* CBb,
                                                     long long lstride, long long cbstride, int kcap, int panel) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R>* As = reinterpret_cast<cx<R>*>(smem_raw);   // [2][KC][128], scaled by D
    cx<R>* Bs = As + 2 * kWideKC * kWideM;            // [2][KC][64]
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, p0 = it.a, i0 = it.b, j0 = it.c;
    cx<R>* L = Lb + lstride * blockIdx.y;
    cx<R>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int K = min(kcap, w - p0);
    cx<R>* Ls = L + S.loff[s];
    cx<R>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const cx<R>* P = Ls + static_cast<long long>(p0) * m;
    const cx<R>* dg = Ls + p0 + static_cast<long long>(p0) * m;  // pivot t at dg[t * (m + 1)]
    const int tid = threadIdx.x;
    // Loader: A chunk entry (k = tid / 128 + 2q, r = tid % 128), q < 4; B chunk
    // entry (k = tid / 64 + 4q, r = tid % 64), q < 2.
    cx<R> pa[4], pd[4], pb[2];
    auto load = [&](int kbase) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = kbase + (tid >> 7) + 2 * q, r = tid & 127;
            pa[q] = cx<R>{0, 0};
            pd[q] = cx<R>{0, 0};
            if (k < K && i0 + r < m) {
                pa[q] = P[static_cast<long long>(k) * m + i0 + r];
                pd[q] = dg[static_cast<long long>(k) * (m + 1)];
            }
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int k = kbase + (tid >> 6) + 4 * q, r = tid & 63;
            pb[q] = cx<R>{0, 0};
            if (k < K && j0 + r < m) pb[q] = P[static_cast<long long>(k) * m + j0 + r];
        }
    };
    auto stash = [&](int buf) {
        cx<R>* A = As + buf * kWideKC * kWideM;
        cx<R>* B = Bs + buf * kWideKC * kWideN;
#pragma unroll
        for (int q = 0; q < 4; ++q) A[((tid >> 7) + 2 * q) * kWideM + (tid & 127)] = pa[q] * pd[q];
#pragma unroll
        for (int q = 0; q < 2; ++q) B[((tid >> 6) + 4 * q) * kWideN + (tid & 63)] = pb[q];
    };
    const int tx = tid & 15, ty = tid >> 4;
    cx<R> acc[8][4];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = cx<R>{0, 0};
    const int nc = (K + kWideKC - 1) / kWideKC;
    load(0);
    stash(0);
    __syncthreads();
    for (int c = 0; c < nc; ++c) {
        if (c + 1 < nc) load((c + 1) * kWideKC);
        const cx<R>* A = As + (c & 1) * kWideKC * kWideM;
        const cx<R>* B = Bs + (c & 1) * kWideKC * kWideN;
#pragma unroll
        for (int k = 0; k < kWideKC; ++k) {
            cx<R> av[8], bv[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) av[a] = A[k * kWideM + tx + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = B[k * kWideN + ty + 16 * b];
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    acc[a][b].re += av[a].re * bv[b].re - av[a].im * bv[b].im;
                    acc[a][b].im += av[a].re * bv[b].im + av[a].im * bv[b].re;
                }
        }
        if (c + 1 < nc) stash((c + 1) & 1);
        __syncthreads();
    }
    // In-panel updates (panel != 0) stop at the current panel's last column.
    const int jcap = panel ? min(w, (p0 / kTcPanel) * kTcPanel + kTcPanel) : m;
    // Read-modify-write, one column block at a time: 8 loads, then 8 stores.
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = j0 + ty + 16 * b;
        cx<R>* dst[8];
        cx<R> old[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int i = i0 + tx + 16 * a;
            dst[a] = nullptr;
            if (j < jcap && i < m && i >= j)
                dst[a] = (j < w) ? Ls + i + static_cast<long long>(j) * m
                                 : CBs + (i - w) + static_cast<long long>(j - w) * cs;
            if (dst[a]) old[a] = *dst[a];
        }
#pragma unroll
        for (int a = 0; a < 8; ++a)
            if (dst[a]) *dst[a] = old[a] - acc[a][b];
    }
}

// FP64 trailing update of complete panels on the FP64 tensor path (DMMA,
// mma.sync m8n8k4). Same items, tile and K (up to kcap = kWidePair: a group
// of 128-column panels) as k_update_wide. 8 warps in a 4 x 2
// grid, each a 32 x 32 complex block of the tile: 4 x 4 blocks of 8 x 8, each
// four real products (Cr += Ar Br - Ai Bi, Ci += Ar Bi + Ai Br; the minus by
// a negated copy of Ai's fragment).
//
// Operands stream global -> shared by cp.async, without a register round
// trip, through a ring of 3 chunks of 16 panel columns (2 in flight while one
// is consumed; one barrier a chunk). They are staged as complex pairs, k-major
// rows 130 / 66 entries apart, so that one quarter-warp's 16-byte fragment
// loads touch distinct banks. The panel's pivots sit beside the ring and scale
// the A fragments as they are read (L[i,k] * D[k], the same product, in the
// same order, as the other trailing updates). A k-step of 4 costs a warp 9
// shared loads for 64 DMMA.
//
// The result is subtracted with red.global.add.f64 (old + (-acc) rounds as
// old - acc does): every destination entry has exactly one writer in a launch,
// so the fire-and-forget reduction leaves the same bits as a read-modify-write
// and, like it, costs the destination's traffic once after the last MMA.
constexpr int kDmmaKC = 16, kDmmaStages = 3;
constexpr int kDmmaLdA = kWideM + 2, kDmmaLdB = kWideN + 2;
constexpr int kDmmaStage = kDmmaKC * (kDmmaLdA + kDmmaLdB);  // complex entries
constexpr int kDmmaSmem = (kWidePair + kDmmaStages * kDmmaStage) * 16;
static_assert(kDmmaSmem <= 227 * 1024, "DMMA ring exceeds shared memory");
static_assert(kTcPanel % kDmmaKC == 0 && kDmmaKC % 4 == 0, "chunks must tile the panel in k-steps of 4");

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// 16-byte global -> shared copy; bytes = 0 fills the destination with zeros.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void red_sub(double* p, double v) {
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(-v) : "memory");
}

// K_DMMA_SCALE item (s, p0, r0, d): rows pe + r0 .. pe + r0 + 127 of front
// s's trailing part (pe = p0 + K) times the group's pivots, W[r, k] =
// L[pe + r, p0 + k] D[k] (the product the tile forms for its A operand, in
// the same order), into region d: column-major, leading dimension R (the
// trailing rows rounded up to 128); rows past the front are zeros. One thread
// per row; blockIdx.z picks 64 of the K columns, whose loads are all in
// flight at once.
__global__ void __launch_bounds__(128) k_dmma_scale(Sched S, long long item0, const cx<double>* Lb,
                                                    long long lstride, unsigned char* ws, long long ws_stride,
                                                    int kcap) {
    constexpr int kCols = 64;
    __shared__ cx<double> piv[kCols];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, p0 = it.a, r0 = it.b;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int K = min(kcap, w - p0), pe = p0 + K;
    const long long R = (m - pe + kTcM - 1) / kTcM * kTcM;
    const int k0 = blockIdx.z * kCols;
    if (k0 >= K) return;  // the whole CTA: no barrier follows for it
    cx<double>* W = reinterpret_cast<cx<double>*>(ws + ws_stride * blockIdx.y + static_cast<long long>(it.d) * 256);
    const cx<double>* P = Lb + lstride * blockIdx.y + S.loff[s];
    if (threadIdx.x < kCols) {
        const int k = k0 + threadIdx.x;
        piv[threadIdx.x] = k < K ? P[(p0 + k) + static_cast<long long>(p0 + k) * m] : cx<double>{0, 0};
    }
    const int r = r0 + threadIdx.x;  // row within the trailing part
    const int row = pe + r;
    const bool in = row < m;
    __syncthreads();
#pragma unroll 2
    for (int c = 0; c < kCols; c += 32) {
        cx<double> v[32];
#pragma unroll
        for (int u = 0; u < 32; ++u) {
            const int k = k0 + c + u;
            v[u] = in && k < K ? P[row + static_cast<long long>(p0 + k) * m] : cx<double>{0, 0};
        }
#pragma unroll
        for (int u = 0; u < 32; ++u) {
            const int k = k0 + c + u;
            if (k < K) W[r + k * R] = v[u] * piv[c + u];
        }
    }
}

// Pre: the A operand comes scaled (W = L D, written by the launch's
// k_dmma_scale into workspace region it.d), so the tile only moves it; without
// it the A fragments are scaled by the pivots as they are read.
template <bool Pre>
__global__ void __launch_bounds__(256) k_update_wide_dmma(Sched S, long long item0, cx<double>* Lb,
                                                          cx<double>* CBb, long long lstride, long long cbstride,
                                                          int kcap, int panel, const unsigned char* ws,
                                                          long long ws_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double>* Ds = reinterpret_cast<cx<double>*>(smem_raw);  // [kWidePair] pivots of the group's panels
    cx<double>* Ring = Ds + kWidePair;                           // [stage][A: KC x ldA | B: KC x ldB]
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, p0 = it.a, i0 = it.b, j0 = it.c;
    cx<double>* L = Lb + lstride * blockIdx.y;
    cx<double>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int K = min(kcap, w - p0);
    cx<double>* Ls = L + S.loff[s];
    cx<double>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const cx<double>* P = Ls + static_cast<long long>(p0) * m;
    const cx<double>* dg = Ls + p0 + static_cast<long long>(p0) * m;
    // The A operand: W's rows i0 - pe .. (leading dimension R), or the panel's.
    const int pe = p0 + K;
    const long long ldw = Pre ? static_cast<long long>(m - pe + kTcM - 1) / kTcM * kTcM : m;
    const cx<double>* PA =
        Pre ? reinterpret_cast<const cx<double>*>(ws + ws_stride * blockIdx.y + static_cast<long long>(it.d) * 256) +
                  (i0 - pe)
            : P + i0;
    const int tid = threadIdx.x;
    const uint32_t ring = smem_u32(Ring);
    // Chunk c: panel columns 16c.. of rows i0.. (A, 128 rows) and j0.. (B, 64).
    auto fetch = [&](int c) {
        const int kbase = c * kDmmaKC;
        const uint32_t sa = ring + (c % kDmmaStages) * kDmmaStage * 16;
        const uint32_t sb = sa + kDmmaKC * kDmmaLdA * 16;
#pragma unroll
        for (int q = 0; q < kDmmaKC * kWideM / 256; ++q) {
            const int e = tid + 256 * q, k = e / kWideM, r = e % kWideM;
            const bool in = kbase + k < K && i0 + r < m;
            cp_async16(sa + (k * kDmmaLdA + r) * 16, in ? PA + static_cast<long long>(kbase + k) * ldw + r : P,
                       in ? 16u : 0u);
        }
#pragma unroll
        for (int q = 0; q < kDmmaKC * kWideN / 256; ++q) {
            const int e = tid + 256 * q, k = e / kWideN, r = e % kWideN;
            const bool in = kbase + k < K && j0 + r < m;
            cp_async16(sb + (k * kDmmaLdB + r) * 16, in ? P + static_cast<long long>(kbase + k) * m + j0 + r : P,
                       in ? 16u : 0u);
        }
    };
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp & 3, wn = warp >> 2;
    const int g = lane >> 2, t4 = lane & 3;
    double cr[4][4][2], ci[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) cr[a][b][0] = cr[a][b][1] = ci[a][b][0] = ci[a][b][1] = 0.0;
    const int nc = (K + kDmmaKC - 1) / kDmmaKC;
    fetch(0);
    cp_async_commit();
    if (nc > 1) fetch(1);
    cp_async_commit();
    if constexpr (!Pre)
        for (int t = tid; t < kWidePair; t += 256) Ds[t] = t < K ? dg[static_cast<long long>(t) * (m + 1)] : cx<double>{0, 0};
    for (int c = 0; c < nc; ++c) {
        cp_async_wait<1>();  // this thread's copies of chunk c have landed
        __syncthreads();     // everyone's have; everyone is done with chunk c - 1
        if (c + 2 < nc) fetch(c + 2);
        cp_async_commit();
        const cx<double>* A = Ring + (c % kDmmaStages) * kDmmaStage;
        const cx<double>* B = A + kDmmaKC * kDmmaLdA;
#pragma unroll
        for (int ks = 0; ks < kDmmaKC; ks += 4) {
            cx<double> af[4], bf[4];
            if constexpr (Pre) {
#pragma unroll
                for (int a = 0; a < 4; ++a) af[a] = A[(ks + t4) * kDmmaLdA + 32 * wm + 8 * a + g];
            } else {
                const cx<double> d = Ds[c * kDmmaKC + ks + t4];
#pragma unroll
                for (int a = 0; a < 4; ++a) af[a] = A[(ks + t4) * kDmmaLdA + 32 * wm + 8 * a + g] * d;
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) bf[b] = B[(ks + t4) * kDmmaLdB + 32 * wn + 8 * b + g];
            // One real product over all 16 blocks before the next, so that
            // consecutive MMAs never feed one another.
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma884(cr[a][b], af[a].re, bf[b].re);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma884(ci[a][b], af[a].re, bf[b].im);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma884(cr[a][b], -af[a].im, bf[b].im);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma884(ci[a][b], af[a].im, bf[b].re);
        }
    }
    // Thread holds C[g][2 t4 + e] of each 8 x 8 block: rows i0 + 32 wm + 8a + g,
    // columns j0 + 32 wn + 8b + 2 t4 + e. In-panel updates (panel != 0) stop
    // at the current panel's last column.
    const int jcap = panel ? min(w, (p0 / kTcPanel) * kTcPanel + kTcPanel) : m;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + 32 * wm + 8 * a + g;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int j = j0 + 32 * wn + 8 * (q >> 1) + 2 * t4 + (q & 1);
            if (j < jcap && i < m && i >= j) {
                cx<double>* dst = (j < w) ? Ls + i + static_cast<long long>(j) * m
                                          : CBs + (i - w) + static_cast<long long>(j - w) * cs;
                red_sub(&dst->re, cr[a][q >> 1][q & 1]);
                red_sub(&dst->im, ci[a][q >> 1][q & 1]);
            }
        }
    }
}

// Tensor-core trailing update of complete panels (FP32 factors). Item
// (s, p0, i0, j0): F[i, j] -= sum_{t in panels} L[i,t] D[t] L[j,t] over the
// 128 x 64 tile at rows i0.., columns j0.. (i >= j). K = min(kcap, w - p0):
// one panel (128) or a group of them (up to kWidePair). Split: TF32 pieces per
// operand (3, or 2 for the cheaper hh + hl + lh products). A bounded wait that
// expires sets err[0] and leaves the tile unchanged; the host reports it.
template <int Split, int Stages = kTcPlaneStages, int Group = kTcGroup>
__global__ void __launch_bounds__(kTcThreads) k_update_tc(Sched S, long long item0, cx<float>* Lb, cx<float>* CBb,
                                                          long long lstride, long long cbstride, int kcap, int* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, p0 = it.a, i0 = it.b, j0 = it.c;
    cx<float>* L = Lb + lstride * blockIdx.y;
    cx<float>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int K = min(kcap, w - p0);
    cx<float>* Ls = L + S.loff[s];
    cx<float>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const float2* P = reinterpret_cast<const float2*>(Ls + static_cast<long long>(p0) * m);
    const float2* dk = reinterpret_cast<const float2*>(Ls + p0 + static_cast<long long>(p0) * m);
    // Read-modify-write of 16 entries of row i: all loads first, so their
    // latencies overlap, then the stores.
    const bool ok = tc_tile<Split, Stages, Group>(smem_raw, P, m, m, K, i0, j0, dk, static_cast<long long>(m) + 1,
                            [&](int r, int c0, const float(&re)[16], const float(&im)[16]) {
                                const int i = i0 + r;
                                if (i >= m) return;
                                float2* dst[16];
                                float2 old[16];
#pragma unroll
                                for (int c = 0; c < 16; ++c) {
                                    const int j = j0 + c0 + c;
                                    dst[c] = nullptr;
                                    if (j < m && i >= j)
                                        dst[c] = reinterpret_cast<float2*>(
                                            (j < w) ? Ls + i + static_cast<long long>(j) * m
                                                    : CBs + (i - w) + static_cast<long long>(j - w) * cs);
                                    if (dst[c]) old[c] = *dst[c];
                                }
#pragma unroll
                                for (int c = 0; c < 16; ++c)
                                    if (dst[c]) *dst[c] = make_float2(old[c].x - re[c], old[c].y - im[c]);
                            });
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
}

// K_TC_SPLIT item (s, p0, r0, d): rows pe + r0 .. pe + r0 + 127 of front s's
// trailing part (pe = p0 + K, the group's K columns from p0) split into the
// pre-split tile's planes, stage by stage: A = L D (the pivots on the panel
// diagonal, the same product tc_split forms) and B = L, each as hi + lo TF32
// pieces (hi = round(x), lo = round(x - hi)); B also as -Bi. The region
// (workspace offset d) holds the A blocks (128 rows) and the B blocks (64
// rows) in the layout tc_tile_presplit reads (pre_a_off, pre_b_off), each
// plane in the canonical K-major core-matrix layout; rows past the front and
// columns past K are zeros. One thread per row; blockIdx.z picks 8 of the
// stages, so the rows' loads of those 64 columns are all in flight at once.
__global__ void __launch_bounds__(kTcThreads) k_tc_split(Sched S, long long item0, const cx<float>* Lb,
                                                         long long lstride, unsigned char* ws, long long ws_stride,
                                                         int kcap) {
    constexpr int kStagesPerCta = 8;  // blockIdx.z: this CTA's stages c0 .. c0 + 7 (64 columns)
    __shared__ cx<float> piv[kStagesPerCta * kTcK];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, p0 = it.a, r0 = it.b;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int K = min(kcap, w - p0), pe = p0 + K;
    const int R = (m - pe + kTcM - 1) / kTcM * kTcM;
    const int nst = (K + kTcK - 1) / kTcK;
    const int c0 = blockIdx.z * kStagesPerCta;
    if (c0 >= nst) return;  // the whole CTA: no barrier follows for it
    unsigned char* region = ws + ws_stride * blockIdx.y + static_cast<long long>(it.d) * 256;
    const cx<float>* P = Lb + lstride * blockIdx.y + S.loff[s];
    if (threadIdx.x < kStagesPerCta * kTcK) {
        const int k = c0 * kTcK + threadIdx.x;
        piv[threadIdx.x] = k < K ? P[(p0 + k) + static_cast<long long>(p0 + k) * m] : cx<float>{0.f, 0.f};
    }
    const int r = r0 + threadIdx.x;  // row within the trailing part
    const int row = pe + r;
    const bool in = row < m;
    // The CTA's 64 columns of this row, every load in flight before use.
    cx<float> v[kStagesPerCta * kTcK];
#pragma unroll
    for (int u = 0; u < kStagesPerCta * kTcK; ++u) {
        const int k = c0 * kTcK + u;
        v[u] = in && k < K ? P[row + static_cast<long long>(p0 + k) * m] : cx<float>{0.f, 0.f};
    }
    __syncthreads();
    const uint32_t oa = plane_off(r & 127, 0), ob = plane_off(r & 63, 0);
#pragma unroll
    for (int cc = 0; cc < kStagesPerCta; ++cc) {
        const int c = c0 + cc;
        if (c >= nst) break;
        unsigned char* A = region + pre_a_off(R, nst, r, c);
        unsigned char* B = region + pre_b_off(R, nst, r, c);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float ar[4], ai[4], br[4], bi[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const cx<float> x = v[cc * kTcK + 4 * h + q];
                const cx<float> d = piv[cc * kTcK + 4 * h + q];
                ar[q] = x.re * d.re - x.im * d.im;
                ai[q] = x.re * d.im + x.im * d.re;
                br[q] = x.re;
                bi[q] = x.im;
            }
            // A: re hi, re lo, im hi, im lo; B per piece: -Bi, Br, Bi
            split_store4<2>(A, kTcPlaneA, oa + h * 128, ar);
            split_store4<2>(A + 2 * kTcPlaneA, kTcPlaneA, oa + h * 128, ai);
            split_store4<2>(B + kTcPlaneB, 3 * kTcPlaneB, ob + h * 128, br);
            split_store4<2, true>(B + 2 * kTcPlaneB, 3 * kTcPlaneB, ob + h * 128, bi, B);
        }
    }
}

// The tensor-core trailing update on pre-split operands (K_UPDATE_TC with
// the two-piece split): item (s, p0, i0, j0, d), the front's planes in the
// workspace region d written by the launch's k_tc_split. Same tile and
// epilogue as k_update_tc.
template <int Group, int Stages>
__global__ void __launch_bounds__(kTcThreads) k_update_tc_presplit(Sched S, long long item0, cx<float>* Lb,
                                                                   cx<float>* CBb, long long lstride,
                                                                   long long cbstride, int kcap,
                                                                   const unsigned char* ws, long long ws_stride,
                                                                   int* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, p0 = it.a, i0 = it.b, j0 = it.c;
    cx<float>* L = Lb + lstride * blockIdx.y;
    cx<float>* CB = CBb + cbstride * blockIdx.y;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int K = min(kcap, w - p0), pe = p0 + K;
    const int R = (m - pe + kTcM - 1) / kTcM * kTcM;
    const int nst = (K + kTcK - 1) / kTcK;
    cx<float>* Ls = L + S.loff[s];
    cx<float>* CBs = CB + (cs > 0 ? S.cboff[s] : 0);
    const unsigned char* region = ws + ws_stride * blockIdx.y + static_cast<long long>(it.d) * 256;
    const bool ok = tc_tile_presplit<Group, Stages>(smem_raw, region, R, nst, i0 - pe, j0 - pe,
                                            [&](int r, int c0, const float(&re)[16], const float(&im)[16]) {
                                                const int i = i0 + r;
                                                if (i >= m) return;
                                                float2* dst[16];
                                                float2 old[16];
#pragma unroll
                                                for (int c = 0; c < 16; ++c) {
                                                    const int j = j0 + c0 + c;
                                                    dst[c] = nullptr;
                                                    if (j < m && i >= j)
                                                        dst[c] = reinterpret_cast<float2*>(
                                                            (j < w) ? Ls + i + static_cast<long long>(j) * m
                                                                    : CBs + (i - w) + static_cast<long long>(j - w) * cs);
                                                    if (dst[c]) old[c] = *dst[c];
                                                }
#pragma unroll
                                                for (int c = 0; c < 16; ++c)
                                                    if (dst[c]) *dst[c] = make_float2(old[c].x - re[c], old[c].y - im[c]);
                                            });
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
}

// ---------------------------------------------------------------- solves
// y, U: per batch entry, nrhs vectors of length n (post-ordered numbering) and
// upool (update vectors, one segment of m - w entries per supernode). A
// kernel handles nr <= 8 right-hand sides starting at rhs k0.
//
// Forward (L y = b), per level bottom-up: gather the children's update
// vectors into the front vector (y at the pivot rows, U_s below), then per
// 64-column block: solve the block's unit triangle, update the rows below.
// Backward (L^T x = D^-1 y), per level top-down, blocks last to first: partial
// sums of L[rows below, block]^T x over 256-row chunks, then one CTA adds them
// in chunk order, scales by D^-1 and solves the block's triangle.


struct SolveArgs {
    int n;
    int nrhs;      // vectors per batch entry in y / U
    int k0, nr;    // the rhs handled by this pass
    long long upool;
    int max_parts;
    const int* entries;  // grid.y -> batch entry (the entries still being solved); null: grid.y is the entry
    int ny;              // grid.y of the solve launches (0: the factor's batch)
    int* counters;       // fused plans: arrival counters, ns per grid row, zero between launches
    int ns;              // supernodes
};

__device__ __forceinline__ int solve_entry(const SolveArgs& a) {
    return a.entries ? a.entries[blockIdx.y] : static_cast<int>(blockIdx.y);
}

__device__ __forceinline__ long long vec_at(const SolveArgs& a, int b, int k) {
    return static_cast<long long>(b) * a.nrhs + (a.k0 + k);
}

// Loads of values that other CTAs of the same launch wrote (through L2, not
// a possibly stale L1 line).
__device__ __forceinline__ cx<double> ld_l2(const cx<double>* p) {
    const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return cx<double>{v.x, v.y};
}
__device__ __forceinline__ cx<float> ld_l2(const cx<float>* p) {
    const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
    return cx<float>{v.x, v.y};
}

// The fused solve kernels' hand-over: every CTA working on supernode s in
// this launch counts itself in, after a fence that publishes its writes; the
// one that arrives last (count == expected) resets the counter for the next
// launch and returns true. No CTA waits for another.
__device__ __forceinline__ bool last_to_arrive(int* counter, int expected) {
    __shared__ int last;
    __syncthreads();  // the CTA's writes ordered before thread 0's fence
    if (threadIdx.x == 0) {
        __threadfence();  // ... which publishes them before the arrival
        const int prev = atomicAdd(counter, 1);
        last = prev == expected - 1;
        if (last) {
            *counter = 0;
            __threadfence();  // the other CTAs' published writes before this CTA reads them
        }
    }
    __syncthreads();
    return last;
}

// A triangle's panel entries (jb x jb at P, leading dimension m) towards L2,
// ahead of the CTA that will stage them: one prefetch per 128-byte line.
template <class R>
__device__ __forceinline__ void prefetch_triangle(const cx<R>* P, long long m, int jb) {
    constexpr int kPerLine = 128 / sizeof(cx<R>);
    const int lines = (jb + kPerLine - 1) / kPerLine;
    for (int e = threadIdx.x; e < lines * jb; e += blockDim.x) {
        const int i = (e % lines) * kPerLine, j = e / lines;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(P + i + static_cast<long long>(j) * m));
    }
}

__device__ __forceinline__ int solve_nblocks(const Sched& S, int s) {
    return (S.first[s + 1] - S.first[s] + kSolveBlock - 1) / kSolveBlock;
}

// Shared memory of the solve kernels that hold a triangle: L_bb with leading
// dimension kTriLd (65: a lane's column-strided reads of the backward solve
// fall in distinct banks), and for the backward solve the partial-sum
// reduction's four sub-sums per (column, rhs).
constexpr int kTriLd = kSolveBlock + 1;
constexpr int kTriSmem = kSolveBlock * kTriLd;     // complex entries
constexpr int kRedSmem = 4 * kSolveBlock * 8;      // complex entries

// L_bb (jb x jb, leading dimension m in the panel) into shared memory T
// (leading dimension kTriLd, zeros outside the jb x jb block) by
// asynchronous copies (cp.async, zero-filled where the source size is 0), so
// the caller's own loads overlap them; the caller waits with
// triangle_wait() and a __syncthreads() before reading T.
__device__ __forceinline__ void cp_async_entry(uint32_t dst, const cx<double>* src, bool in) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16u : 0u) : "memory");
}
__device__ __forceinline__ void cp_async_entry(uint32_t dst, const cx<float>* src, bool in) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(in ? 8u : 0u) : "memory");
}
template <class R>
__device__ __forceinline__ void stage_triangle(cx<R>* T, const cx<R>* P, long long m, int jb) {
    static_assert(kSolveBlock * kSolveBlock % 256 == 0, "the block splits evenly over 256 threads");
#pragma unroll 4
    for (int e = threadIdx.x; e < kSolveBlock * kSolveBlock; e += 256) {
        const int i = e % kSolveBlock, j = e / kSolveBlock;
        const bool in = i < jb && j < jb;
        cp_async_entry(smem_u32(T + i + j * kTriLd), in ? P + i + static_cast<long long>(j) * m : P, in);
    }
    cp_async_commit();
}
__device__ __forceinline__ void triangle_wait() { cp_async_wait<0>(); }

// Forward triangle of block blk of supernode s: y[blk] = L_bb^-1 y[blk] for
// the pass's rhs, one warp per rhs, L_bb staged in shared memory (smem:
// kTriSmem entries). Lane l holds rows l and l + 32 in registers;
// step j broadcasts y_j from its owner lane and every lane below updates
// its rows, y_i = y_i - L_ij y_j, in ascending j. Every thread of the CTA
// calls it (256 threads).
template <class R>
__device__ void fwd_triangle(const Sched& S, const SolveArgs& a, int eb, const cx<R>* Lb, long long lstride,
                             cx<R>* yb, int s, int blk, unsigned char* smem) {
    static_assert(kSolveBlock == 64, "two rows per lane");
    cx<R>* T = reinterpret_cast<cx<R>*>(smem);
    const int j0 = blk * kSolveBlock;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int f = S.first[s];
    const int jb = min(kSolveBlock, w - j0);
    stage_triangle(T, Lb + lstride * eb + S.loff[s] + j0 + static_cast<long long>(j0) * m, m, jb);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    cx<R>* y = yb + vec_at(a, eb, warp) * a.n + f + j0;
    cx<R> y0{0, 0}, y1{0, 0};
    if (warp < a.nr) {
        if (lane < jb) y0 = ld_l2(y + lane);
        if (lane + 32 < jb) y1 = ld_l2(y + lane + 32);
    }
    triangle_wait();
    __syncthreads();
    if (warp < a.nr) {
        for (int j = 0; j < jb; ++j) {
            const cx<R> src = j < 32 ? y0 : y1;
            cx<R> yj;
            yj.re = __shfl_sync(0xffffffffu, src.re, j & 31);
            yj.im = __shfl_sync(0xffffffffu, src.im, j & 31);
            if (lane > j) y0 = fms(y0, T[lane + j * kTriLd], yj);
            if (lane + 32 > j && lane + 32 < jb) y1 = fms(y1, T[lane + 32 + j * kTriLd], yj);
        }
        if (lane < jb) y[lane] = y0;
        if (lane + 32 < jb) y[lane + 32] = y1;
    }
}

// Item (s): the children's update vectors added into supernode s's front
// vector (y at its pivot rows, its own update segment U_s below). Fused: the
// same CTA then solves the supernode's first block (dynamic shared memory
// kTriSmem entries).
template <class R, bool Fused>
__global__ void __launch_bounds__(256) k_fwd_gather(Sched S, long long item0, SolveArgs a, const cx<R>* Lb,
                                                    long long lstride, cx<R>* yb, cx<R>* Ub) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int eb = solve_entry(a);
    const int s = S.items[item0 + blockIdx.x].s;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int cs = m - w;
    const int f = S.first[s];
    if constexpr (Fused)  // the first block's triangle, staged after the gather
        prefetch_triangle(Lb + lstride * eb + S.loff[s], m, min(kSolveBlock, w));
    for (int k = 0; k < a.nr; ++k) {
        cx<R>* y = yb + vec_at(a, eb, k) * a.n;
        cx<R>* U = Ub + vec_at(a, eb, k) * a.upool;
        cx<R>* Us = U + S.uoff[s];
        for (int i = threadIdx.x; i < cs; i += blockDim.x) Us[i] = cx<R>{0, 0};
        __syncthreads();
        for (int t = S.child_ptr[s]; t < S.child_ptr[s + 1]; ++t) {
            const int c = S.child_list[t];
            const int cc = S.rows[c] - (S.first[c + 1] - S.first[c]);
            const int* rel = S.rel + S.reloff[c];
            const cx<R>* Uc = U + S.uoff[c];
            for (int i = threadIdx.x; i < cc; i += blockDim.x) {
                const int p = rel[i];
                if (p < w) y[f + p] = y[f + p] + Uc[i];
                else Us[p - w] = Us[p - w] + Uc[i];
            }
            __syncthreads();
        }
    }
    if constexpr (Fused) {
        __threadfence();
        __syncthreads();
        if (w > 0) fwd_triangle<R>(S, a, eb, Lb, lstride, yb, s, 0, smem_raw);
    }
}

// Item (s, blk): y[blk] = L_bb^-1 y[blk] (the split plan's triangle launch).
template <class R>
__global__ void __launch_bounds__(256) k_fwd_diag(Sched S, long long item0, SolveArgs a, const cx<R>* Lb,
                                                  long long lstride, cx<R>* yb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Item it = S.items[item0 + blockIdx.x];
    fwd_triangle<R>(S, a, solve_entry(a), Lb, lstride, yb, it.s, it.a, smem_raw);
}

// Item (s, blk, row0): rows row0 .. row0 + kSolveRows - 1 of the supernode
// minus L[rows, blk] y[blk]. Four threads per row, each over 16 of the
// block's columns with all 16 loads in flight (one round trip); the four
// column-ordered sub-sums are added in order. Fused: the last of the
// block's CTAs then solves block blk + 1 (counters: one per supernode and
// grid row; dynamic shared memory kTriSmem entries).
template <class R, bool Fused>
__global__ void __launch_bounds__(256) k_fwd_update(Sched S, long long item0, SolveArgs a, const cx<R>* Lb,
                                                    long long lstride, cx<R>* yb, cx<R>* Ub) {
    static_assert(kSolveRows * 4 == 256 && kSolveBlock == 64, "four 16-column quarters per row");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int eb = solve_entry(a);
    __shared__ cx<R> ys[8][kSolveBlock];
    __shared__ cx<R> red[3][8][kSolveRows];  // quarters 1..3's sub-sums
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, j0 = it.a * kSolveBlock, row0 = it.b;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int f = S.first[s];
    const int jb = min(kSolveBlock, w - j0);
    const int t = threadIdx.x % kSolveRows, qt = threadIdx.x / kSolveRows;
    const int r = row0 + t;
    const int c0 = 16 * qt, nc = min(16, jb - c0);
    // The panel entries first (they depend on the item only), so their round
    // trip overlaps the block's y values'.
    cx<R> l[16];
    {
        const bool live = r < m && nc > 0;
        const cx<R>* P = Lb + lstride * eb + S.loff[s] + (live ? r : 0) + static_cast<long long>(j0 + c0) * m;
#pragma unroll
        for (int u = 0; u < 16; ++u) l[u] = live && u < nc ? P[static_cast<long long>(u) * m] : cx<R>{0, 0};
    }
    // The first rhs's destination, read now (only this CTA writes these rows
    // in this launch).
    cx<R>* dst0 = r < w ? yb + vec_at(a, eb, 0) * a.n + f + r : Ub + vec_at(a, eb, 0) * a.upool + S.uoff[s] + (r - w);
    const cx<R> old0 = qt == 0 && r < m ? *dst0 : cx<R>{0, 0};
    if constexpr (Fused) {
        const int jn = j0 + kSolveBlock;  // the next block, which this launch's last CTA solves
        if (row0 == j0 + jb && jn < w)
            prefetch_triangle(Lb + lstride * eb + S.loff[s] + jn + static_cast<long long>(jn) * m, m,
                              min(kSolveBlock, w - jn));
    }
    for (int e = threadIdx.x; e < jb * a.nr; e += blockDim.x) {
        const int j = e % jb, k = e / jb;
        ys[k][j] = yb[vec_at(a, eb, k) * a.n + f + j0 + j];
    }
    __syncthreads();
    cx<R> acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = cx<R>{0, 0};
    if (r < m && nc > 0) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            if (u >= nc) break;
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (k < a.nr) acc[k] = acc[k] + l[u] * ys[k][c0 + u];
        }
    }
    if (qt > 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k < a.nr) red[qt - 1][k][t] = acc[k];
    }
    __syncthreads();
    if (qt == 0 && r < m) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k >= a.nr) break;
            const cx<R> sum = ((acc[k] + red[0][k][t]) + red[1][k][t]) + red[2][k][t];
            cx<R>* dst = r < w ? yb + vec_at(a, eb, k) * a.n + f + r
                               : Ub + vec_at(a, eb, k) * a.upool + S.uoff[s] + (r - w);
            *dst = (k == 0 ? old0 : *dst) - sum;
        }
    }
    if constexpr (Fused) {
        const int below = j0 + jb;
        const int chunks = (m - below + kSolveRows - 1) / kSolveRows;
        if (last_to_arrive(a.counters + static_cast<long long>(blockIdx.y) * a.ns + s, chunks) &&
            it.a + 1 < solve_nblocks(S, s))
            fwd_triangle<R>(S, a, eb, Lb, lstride, yb, s, it.a + 1, smem_raw);
    }
}

// Backward triangle of block blk of supernode s: x[blk] = L_bb^-T (D^-1
// y[blk] - sum of the partials in slots p0 .. p0 + np - 1) for the pass's
// rhs (smem: kTriSmem + kRedSmem entries). The partials are summed by four
// threads per (column, rhs), each over every fourth slot in slot order, the
// four sub-sums then added in order. The triangle: one warp per rhs, lane l
// holding rows l and l + 32; step j (descending) broadcasts x_j from its
// owner lane and every lane above updates its rows, z_t = z_t - L_jt x_j.
// Every thread of the CTA calls it (256 threads).
template <class R>
__device__ void bwd_triangle(const Sched& S, const SolveArgs& a, int eb, const cx<R>* Lb, long long lstride,
                             cx<R>* yb, const cx<R>* partb, int s, int blk, int p0, int np, unsigned char* smem) {
    static_assert(kSolveBlock == 64, "two rows per lane");
    cx<R>* T = reinterpret_cast<cx<R>*>(smem);
    cx<R>* red = T + kTriSmem;  // [4][8][kSolveBlock]
    const int j0 = blk * kSolveBlock;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int f = S.first[s];
    const int jb = min(kSolveBlock, w - j0);
    stage_triangle(T, Lb + lstride * eb + S.loff[s] + j0 + static_cast<long long>(j0) * m, m, jb);
    const cx<R>* part = partb + static_cast<long long>(eb) * a.max_parts * kSolveBlock * 8;
    for (int e = threadIdx.x; e < 4 * kSolveBlock * a.nr; e += blockDim.x) {
        const int g = e & 3, j = (e >> 2) % kSolveBlock, k = (e >> 2) / kSolveBlock;
        cx<R> sum{0, 0};
        if (j < jb) {
            constexpr int kU = 16;  // loads in flight per thread
            int q = g;
            for (; q + 4 * (kU - 1) < np; q += 4 * kU) {
                cx<R> v[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    v[u] = ld_l2(part + (static_cast<long long>(p0 + q + 4 * u) * kSolveBlock + j) * 8 + k);
#pragma unroll
                for (int u = 0; u < kU; ++u) sum = sum + v[u];
            }
            for (; q < np; q += 4) sum = sum + ld_l2(part + (static_cast<long long>(p0 + q) * kSolveBlock + j) * 8 + k);
        }
        red[(g * 8 + k) * kSolveBlock + j] = sum;
    }
    triangle_wait();
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < a.nr) {
        cx<R>* y = yb + vec_at(a, eb, warp) * a.n + f + j0;
        cx<R> z[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = lane + 32 * h;
            z[h] = cx<R>{0, 0};
            if (j < jb) {
                const cx<R>* rj = red + warp * kSolveBlock + j;
                const cx<R> sum = ((rj[0] + rj[8 * kSolveBlock]) + rj[16 * kSolveBlock]) + rj[24 * kSolveBlock];
                z[h] = ld_l2(y + j) * crecip(T[j * (kTriLd + 1)]) - sum;
            }
        }
        for (int j = jb - 1; j >= 0; --j) {
            const cx<R> src = j < 32 ? z[0] : z[1];
            cx<R> xj;
            xj.re = __shfl_sync(0xffffffffu, src.re, j & 31);
            xj.im = __shfl_sync(0xffffffffu, src.im, j & 31);
            if (lane < j) z[0] = fms(z[0], T[j + lane * kTriLd], xj);
            if (lane + 32 < j) z[1] = fms(z[1], T[j + (lane + 32) * kTriLd], xj);
        }
        if (lane < jb) y[lane] = z[0];
        if (lane + 32 < jb) y[lane + 32] = z[1];
    }
}

// Item (s, blk, row0, slot[, p0]): partial[slot][j][k] = sum over rows
// row0 .. row0 + kSolveRows - 1 (below the block) of L[row, j0 + j] x_k[row]
// (an empty chunk, row0 = m, gives zeros). Warp v takes columns 8v .. 8v + 7,
// lane l rows l and l + 32: all 16 loads in flight (one round trip); per
// column the lane's two rows in order, then a butterfly over the warp.
// Fused: the last of the block's CTAs then reduces the block's partials
// (slots p0 ..) and solves the block (counters: one per supernode and grid
// row; dynamic shared memory kTriSmem + kRedSmem entries).
template <class R, bool Fused>
__global__ void __launch_bounds__(256) k_bwd_update(Sched S, long long item0, SolveArgs a, const cx<R>* Lb,
                                                    long long lstride, cx<R>* yb, cx<R>* partb) {
    static_assert(kSolveRows == 64 && kSolveBlock == 64, "two rows per lane, eight columns per warp");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int eb = solve_entry(a);
    __shared__ cx<R> xs[8][kSolveRows];
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, j0 = it.a * kSolveBlock, row0 = it.b, slot = it.c;
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int f = S.first[s];
    const int jb = min(kSolveBlock, w - j0);
    const int nrows = max(0, min(kSolveRows, m - row0));
    const int* st = S.structs + S.soff[s];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // The panel entries first (they depend on the item only), so their round
    // trip overlaps the gather of x.
    if constexpr (Fused) {
        if (row0 == j0 + jb)  // the block's triangle, which this launch's last CTA stages
            prefetch_triangle(Lb + lstride * eb + S.loff[s] + j0 + static_cast<long long>(j0) * m, m, jb);
    }
    cx<R> l[8][2];
    {
        const cx<R>* P = Lb + lstride * eb + S.loff[s] + static_cast<long long>(j0) * m;
#pragma unroll
        for (int c = 0; c < 8; ++c)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = 8 * warp + c, t = lane + 32 * h;
                l[c][h] = j < jb && t < nrows ? P[row0 + t + static_cast<long long>(j) * m] : cx<R>{0, 0};
            }
    }
    for (int e = threadIdx.x; e < nrows * a.nr; e += blockDim.x) {
        const int t = e % nrows, k = e / nrows;
        const int r = row0 + t;
        const int g = r < w ? f + r : st[r];
        xs[k][t] = yb[vec_at(a, eb, k) * a.n + g];
    }
    __syncthreads();
    cx<R>* part = partb + static_cast<long long>(eb) * a.max_parts * kSolveBlock * 8 +
                  static_cast<long long>(slot) * kSolveBlock * 8;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int j = 8 * warp + c;
        if (j >= jb) break;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k >= a.nr) break;
            cx<R> v{0, 0};
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (lane + 32 * h < nrows) v = v + l[c][h] * xs[k][lane + 32 * h];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                v.re += __shfl_xor_sync(0xffffffffu, v.re, o);
                v.im += __shfl_xor_sync(0xffffffffu, v.im, o);
            }
            if (lane == 0) part[j * 8 + k] = v;
        }
    }
    if constexpr (Fused) {
        const int below = j0 + jb;
        const int chunks = max(1, (m - below + kSolveRows - 1) / kSolveRows);
        if (last_to_arrive(a.counters + static_cast<long long>(blockIdx.y) * a.ns + s, chunks))
            bwd_triangle<R>(S, a, eb, Lb, lstride, yb, partb, s, it.a, it.d, chunks, smem_raw);
    }
}

// Item (s, blk, first_slot, nslots): x[blk] = L_bb^-T (D^-1 y[blk] - sum of
// partials) (the split plan's triangle launch).
template <class R>
__global__ void __launch_bounds__(256) k_bwd_diag(Sched S, long long item0, SolveArgs a, const cx<R>* Lb,
                                                  long long lstride, cx<R>* yb, const cx<R>* partb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Item it = S.items[item0 + blockIdx.x];
    bwd_triangle<R>(S, a, solve_entry(a), Lb, lstride, yb, partb, it.s, it.a, it.b, it.c, smem_raw);
}

}  // namespace aphi_b200
