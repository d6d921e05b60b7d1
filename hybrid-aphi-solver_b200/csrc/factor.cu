// Host orchestration of the numeric factorization, the solves, the residuals
// and iterative refinement, plus the memory-bound helper kernels
// (equilibration, scatter of A into the fronts, permutations, SpMV, norms).
//
// Reference: solve_symmetric, src/factorization.cpp:332-398; factorize_ldlt
// :109-218; solve/solve_in_place :254-313; relative_residual :315-329;
// backward_error :401-416; compute_symmetric_equilibration,
// src/equilibration.cpp:94-139.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "factor.hpp"
#include "factor_kernels.cuh"
#include "pivot_stats.hpp"

namespace aphi_b200 {

namespace {

constexpr int kEqThreads = 256;

// ---------------------------------------------------------------- equilibration
// |a_ij| d_i d_j contributes to the maxima of BOTH row i and row j
// (src/equilibration.cpp:101-118): the matrix is stored as its upper
// triangle. Maxima of non-negative doubles are taken as unsigned integers,
// which orders them exactly, so the result does not depend on the order in
// which threads arrive.
__global__ void k_eq_rowmax(int n, const int* row_ptr, const int* col_idx, const double* values,
                            long long nnz, const double* d, unsigned long long* rowmax) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (r >= n) return;
    const double* v = values + 2LL * nnz * b;
    const double* db = d + static_cast<long long>(n) * b;
    unsigned long long* mx = rowmax + static_cast<long long>(n) * b;
    const double dr = db[r];
    double best = 0.0;
    for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
        const int c = col_idx[k];
        const double mag = hypot(v[2 * k], v[2 * k + 1]) * (dr * db[c]);
        best = fmax(best, mag);
        if (c != r) atomicMax(&mx[c], __double_as_longlong(mag));
    }
    atomicMax(&mx[r], __double_as_longlong(best));
}

__global__ void k_eq_update(int n, double* d, unsigned long long* rowmax) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (r >= n) return;
    const long long at = static_cast<long long>(n) * b + r;
    const double mx = __longlong_as_double(rowmax[at]);
    if (mx > 0.0) d[at] *= 1.0 / sqrt(mx);
    rowmax[at] = 0ULL;
}

__global__ void k_fill(double* p, long long n, double v) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < n) p[i] = v;
}

// Scaled A entries into their panel slots: L[dest[k]] = a_k d_r d_c.
template <class R>
__global__ void k_scatter_a(int n, const int* row_ptr, const int* col_idx, const double* values, long long nnz,
                            const double* d, const long long* dest, cx<R>* Lb, long long lstride) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (r >= n) return;
    const double* v = values + 2LL * nnz * b;
    const double* db = d + static_cast<long long>(n) * b;
    cx<R>* L = Lb + lstride * b;
    const double dr = db[r];
    for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
        const double s = dr * db[col_idx[k]];
        L[dest[k]] = cx<R>{static_cast<R>(v[2 * k] * s), static_cast<R>(v[2 * k + 1] * s)};
    }
}

// D in the caller's permuted order (complex128), for the host-side stats.
template <class R>
__global__ void k_extract_d(Sched S, int ns, const int* ref_of_post, const cx<R>* Lb, long long lstride,
                            double* dref, int n) {
    const int s = blockIdx.x;
    const int b = blockIdx.y;
    const cx<R>* L = Lb + lstride * b + S.loff[s];
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        const cx<R> v = L[j + static_cast<long long>(j) * m];
        const int k = ref_of_post[S.first[s] + j];
        dref[2 * (static_cast<long long>(n) * b + k)] = v.re;
        dref[2 * (static_cast<long long>(n) * b + k) + 1] = v.im;
    }
}

// max |L(i, j)| over the multipliers whose row (in the caller's order) is at
// most kmax[b] -- the rows the reference had computed when it stopped.
// Item (s, c0): 32 columns of one panel; one warp per column.
template <class R>
__global__ void __launch_bounds__(256) k_max_multiplier(Sched S, long long item0, const int* ref_of_post,
                                                        const cx<R>* Lb, long long lstride, const int* kmax,
                                                        unsigned long long* out) {
    const Item it = S.items[item0 + blockIdx.x];
    const int s = it.s, c0 = it.a;
    const int b = blockIdx.y;
    const cx<R>* L = Lb + lstride * b + S.loff[s];
    const int w = S.first[s + 1] - S.first[s];
    const int m = S.rows[s];
    const int* st = S.structs + S.soff[s];
    const int lim = kmax[b];
    const int n_all = lim >= 0x7fffffff;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double best = 0.0;
    for (int j = c0 + warp; j < min(c0 + 32, w); j += 8) {
        const cx<R>* col = L + static_cast<long long>(j) * m;
        for (int i = j + 1 + lane; i < m; i += 32) {
            if (!n_all && ref_of_post[st[i]] > lim) continue;
            best = fmax(best, cabs_d(col[i]));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) atomicMax(&out[b], __double_as_longlong(best));
}

// y[new] = b[orig] * d[orig]  (permute in, with the equilibration scaling).
template <class R>
__global__ void k_permute_in(int n, int nrhs, const int* orig_of_new, const double* dsc, const double* b,
                             cx<R>* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int bk = blockIdx.y;  // batch * nrhs + k
    if (i >= n) return;
    const int bb = bk / nrhs;
    const int o = orig_of_new[i];
    const double s = dsc[static_cast<long long>(n) * bb + o];
    const double* src = b + 2LL * n * bk;
    y[static_cast<long long>(n) * bk + i] = cx<R>{static_cast<R>(src[2 * o] * s), static_cast<R>(src[2 * o + 1] * s)};
}

// x[orig] = y[new] * d[orig]  (permute out, undoing the substitution x = D y).
template <class R>
__global__ void k_permute_out(int n, int nrhs, const int* new_of_orig, const double* dsc, const cx<R>* y,
                              double* x) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int bk = blockIdx.y;
    if (o >= n) return;
    const int bb = bk / nrhs;
    const double s = dsc[static_cast<long long>(n) * bb + o];
    const cx<R> v = y[static_cast<long long>(n) * bk + new_of_orig[o]];
    x[2LL * n * bk + 2 * o] = static_cast<double>(v.re) * s;
    x[2LL * n * bk + 2 * o + 1] = static_cast<double>(v.im) * s;
}

// ---------------------------------------------------------------- residuals
// r = b - A x on the original upper-stored A (both triangles through the
// mirrored CSR); per-row partial sums of |r|^2, |b|^2, |x|^2 reduced in a
// fixed order by k_norms_final.
__global__ void k_residual(int n, int nrhs, const int* fptr, const int* fcol, const long long* fmap,
                           const double* values, long long nnz, const double* x, const double* b, double* r_out,
                           double* partial) {
    __shared__ double sh[3][256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int bk = blockIdx.y;
    const int bb = bk / nrhs;
    const double* v = values + 2LL * nnz * bb;
    const double* xb = x + 2LL * n * bk;
    const double* bb_ = b + 2LL * n * bk;
    double rr = 0, b2 = 0, x2 = 0;
    if (i < n) {
        double ar = 0, ai = 0;
        for (int k = fptr[i]; k < fptr[i + 1]; ++k) {
            const long long q = fmap[k];
            const double vr = v[2 * q], vi = v[2 * q + 1];
            const double xr = xb[2 * fcol[k]], xi = xb[2 * fcol[k] + 1];
            ar += vr * xr - vi * xi;
            ai += vr * xi + vi * xr;
        }
        const double er = bb_[2 * i] - ar, ei = bb_[2 * i + 1] - ai;
        if (r_out) {
            r_out[2LL * n * bk + 2 * i] = er;
            r_out[2LL * n * bk + 2 * i + 1] = ei;
        }
        rr = er * er + ei * ei;
        b2 = bb_[2 * i] * bb_[2 * i] + bb_[2 * i + 1] * bb_[2 * i + 1];
        x2 = xb[2 * i] * xb[2 * i] + xb[2 * i + 1] * xb[2 * i + 1];
    }
    sh[0][threadIdx.x] = rr;
    sh[1][threadIdx.x] = b2;
    sh[2][threadIdx.x] = x2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) partial[(static_cast<long long>(bk) * gridDim.x + blockIdx.x) * 3 + q] = sh[q][0];
}

__global__ void k_amax(const double* values, long long nnz, unsigned long long* out) {
    const long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const int b = blockIdx.y;
    if (k >= nnz) return;
    const double* v = values + 2LL * nnz * b;
    atomicMax(&out[b], __double_as_longlong(hypot(v[2 * k], v[2 * k + 1])));
}

// norms[bk] = {||r||, ||b||, ||x||, max|A|}: fixed-order sums of the partials.
__global__ void k_norms_final(int nblocks, int nrhs, const double* partial, const unsigned long long* amax,
                              double* norms) {
    const int bk = blockIdx.x;
    __shared__ double sh[3][256];
    double acc[3] = {0, 0, 0};
    for (int t = threadIdx.x; t < nblocks; t += blockDim.x)
        for (int q = 0; q < 3; ++q) acc[q] += partial[(static_cast<long long>(bk) * nblocks + t) * 3 + q];
    for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norms[4 * bk] = sqrt(sh[0][0]);
        norms[4 * bk + 1] = sqrt(sh[1][0]);
        norms[4 * bk + 2] = sqrt(sh[2][0]);
        norms[4 * bk + 3] = __longlong_as_double(amax[bk / nrhs]);
    }
}

// x += dx (FP64).
__global__ void k_axpy(long long len, double* x, const double* dx) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < len) x[i] += dx[i];
}

template <class T>
T* dalloc(size_t n) {
    T* p = nullptr;
    APHI_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    return p;
}

template <class R>
void run_plan(const aphi_factor* f, const std::vector<Launch>& plan, cudaStream_t st, const SolveArgs* sa,
              cx<R>* y, cx<R>* U, cx<R>* part) {
    const aphi_analysis* A = f->an;
    const Sched S = sched_of(A->d);
    cx<R>* L = reinterpret_cast<cx<R>*>(f->L);
    cx<R>* CB = reinterpret_cast<cx<R>*>(f->CB);
    const long long ls = A->S.stored, cs = A->S.cb_pool;
    const int smallsm = A->opt.small_front * A->opt.small_front * static_cast<int>(sizeof(cx<R>));
    aphi_factor* fm = const_cast<aphi_factor*>(f);
    const bool prof = f->profile;
    const bool presplit = sizeof(R) == 4 && f->tc_split == 2 && f->presplit && f->tcws;
    const size_t tri_smem = kTriSmem * sizeof(cx<R>);               // forward triangles
    const size_t bwd_smem = (kTriSmem + kRedSmem) * sizeof(cx<R>);  // backward triangles
    // FP64 trailing updates on pre-scaled operands (W = L D per panel group).
    const bool prescaled = sizeof(R) == 8 && f->dws;
    for (const Launch& l : plan) {
        // Without pre-split (pre-scaled) operands the tile splits (scales) them
        // itself: no operand launch.
        if (l.kind == K_TC_SPLIT && !presplit) continue;
        if (l.kind == K_DMMA_SCALE && !prescaled) continue;
        dim3 grid(l.count, sa && sa->ny > 0 ? sa->ny : f->batch);
        const bool timed = prof && ((f->prof_mask >> l.kind) & 1u);
        if (timed) {
            cudaEvent_t e[2];
            APHI_CUDA(cudaEventCreate(&e[0]));
            APHI_CUDA(cudaEventCreate(&e[1]));
            fm->prof_events.push_back(e[0]);
            fm->prof_events.push_back(e[1]);
            fm->prof_kinds.push_back(l.kind);
            APHI_CUDA(cudaEventRecord(e[0], st));
        }
        switch (l.kind) {
            case K_EXTEND_ADD: k_extend_add<R><<<grid, 256, 0, st>>>(S, l.first, L, CB, ls, cs); break;
            case K_SMALL: k_small_front<R><<<grid, 256, smallsm, st>>>(S, l.first, L, CB, ls, cs); break;
            case K_DIAG: k_diag_block<R><<<grid, 128, 0, st>>>(S, l.first, L, ls); break;
            case K_TRSM: k_panel_trsm<R><<<grid, kTrsmRows, 0, st>>>(S, l.first, L, ls); break;
            case K_UPDATE_WIDE:
            case K_UPDATE_PANEL:
                if (l.kind == K_UPDATE_PANEL && !l.wide) {
                    k_update_panel<R><<<grid, 256, 2 * kStep * kTile * sizeof(cx<R>), st>>>(S, l.first, L, CB, ls, cs);
                    break;
                }
                if constexpr (sizeof(R) == 8) {
                    if (l.kind == K_UPDATE_WIDE && prescaled)
                        k_update_wide_dmma<true><<<grid, 256, kDmmaSmem, st>>>(S, l.first, L, CB, ls, cs, l.kcap, 0,
                                                                              f->dws, f->dws_stride);
                    else
                        k_update_wide_dmma<false><<<grid, 256, kDmmaSmem, st>>>(
                            S, l.first, L, CB, ls, cs, l.kcap, l.kind == K_UPDATE_PANEL ? 1 : 0, nullptr, 0);
                } else
                    k_update_wide<R><<<grid, 256, wide_smem<R>(), st>>>(S, l.first, L, CB, ls, cs, l.kcap,
                                                                      l.kind == K_UPDATE_PANEL ? 1 : 0);
                break;
            case K_DMMA_SCALE:
                if constexpr (sizeof(R) == 8)
                    k_dmma_scale<<<dim3(grid.x, grid.y, (l.kcap + 63) / 64), 128, 0, st>>>(S, l.first, L, ls, f->dws,
                                                                                         f->dws_stride, l.kcap);
                else
                    throw Error(APHI_ERR_INVALID, "operand scaling planned for an FP32 factor");
                break;
            case K_TC_SPLIT:
                if constexpr (sizeof(R) == 4)
                    k_tc_split<<<dim3(grid.x, grid.y, (l.kcap + 8 * kTcK - 1) / (8 * kTcK)), kTcThreads, 0, st>>>(
                        S, l.first, L, ls, f->tcws, f->tcws_stride, l.kcap);
                else
                    throw Error(APHI_ERR_INVALID, "operand split planned for an FP64 factor");
                break;
            case K_UPDATE_TC:
                if constexpr (sizeof(R) == 4) {
                    if (presplit) {
                        auto go = [&](auto kern, int smem) {
                            kern<<<grid, kTcThreads, smem, st>>>(S, l.first, L, CB, ls, cs, l.kcap, f->tcws,
                                                                 f->tcws_stride, f->err);
                        };
                        // A 4-stage accumulator group needs 4 plane buffers.
                        if (f->tc_group == 4) go(k_update_tc_presplit<4, 4>, TcPreSmem<4>::bytes);
                        else if (f->pre_stages == 4) go(k_update_tc_presplit<2, 4>, TcPreSmem<4>::bytes);
                        else go(k_update_tc_presplit<2, 3>, TcPreSmem<3>::bytes);
                        break;
                    }
                    // split 3: two plane stages (3 would leave one CTA per SM);
                    // split 2: plane stages and accumulator group as configured.
                    const int v = f->tc_split == 3 ? 0 : (f->tc_stages == 3 ? 2 : 0) + (f->tc_group == 4 ? 1 : 0) + 1;
                    switch (v) {
                        case 0: k_update_tc<3, 2, 2><<<grid, kTcThreads, TcSmem<3, 2>::bytes, st>>>(S, l.first, L, CB, ls, cs, l.kcap, f->err); break;
                        case 1: k_update_tc<2, 2, 2><<<grid, kTcThreads, TcSmem<2, 2>::bytes, st>>>(S, l.first, L, CB, ls, cs, l.kcap, f->err); break;
                        case 2: k_update_tc<2, 2, 4><<<grid, kTcThreads, TcSmem<2, 2>::bytes, st>>>(S, l.first, L, CB, ls, cs, l.kcap, f->err); break;
                        case 3: k_update_tc<2, 3, 2><<<grid, kTcThreads, TcSmem<2, 3>::bytes, st>>>(S, l.first, L, CB, ls, cs, l.kcap, f->err); break;
                        default: k_update_tc<2, 3, 4><<<grid, kTcThreads, TcSmem<2, 3>::bytes, st>>>(S, l.first, L, CB, ls, cs, l.kcap, f->err); break;
                    }
                } else
                    throw Error(APHI_ERR_INVALID, "tensor-core update planned for an FP64 factor");
                break;
            case K_FWD_GATHER:
                if (l.wide)
                    k_fwd_gather<R, true><<<grid, 256, tri_smem, st>>>(S, l.first, *sa, L, ls, y, U);
                else
                    k_fwd_gather<R, false><<<grid, 256, 0, st>>>(S, l.first, *sa, L, ls, y, U);
                break;
            case K_FWD_DIAG: k_fwd_diag<R><<<grid, 256, tri_smem, st>>>(S, l.first, *sa, L, ls, y); break;
            case K_FWD_UPDATE:
                if (l.wide)
                    k_fwd_update<R, true><<<grid, 256, tri_smem, st>>>(S, l.first, *sa, L, ls, y, U);
                else
                    k_fwd_update<R, false><<<grid, 256, 0, st>>>(S, l.first, *sa, L, ls, y, U);
                break;
            case K_BWD_UPDATE:
                if (l.wide)
                    k_bwd_update<R, true><<<grid, 256, bwd_smem, st>>>(S, l.first, *sa, L, ls, y, part);
                else
                    k_bwd_update<R, false><<<grid, 256, 0, st>>>(S, l.first, *sa, L, ls, y, part);
                break;
            case K_BWD_DIAG: k_bwd_diag<R><<<grid, 256, bwd_smem, st>>>(S, l.first, *sa, L, ls, y, part); break;
        }
        APHI_CHECK_LAUNCH();
        if (timed) APHI_CUDA(cudaEventRecord(fm->prof_events.back(), st));
    }
}

// Adds the per-launch durations of the last factorization to the totals
// (after the stream has been synchronized).
void collect_profile(aphi_factor* f) {
    for (size_t q = 0; q < f->prof_kinds.size(); ++q) {
        float ms = 0;
        APHI_CUDA(cudaEventElapsedTime(&ms, f->prof_events[2 * q], f->prof_events[2 * q + 1]));
        f->prof_ms[f->prof_kinds[q]] += ms;
        ++f->prof_launches[f->prof_kinds[q]];
    }
    for (cudaEvent_t e : f->prof_events) cudaEventDestroy(e);
    f->prof_events.clear();
    f->prof_kinds.clear();
}

// Opt-in shared-memory limits, set once per process; serialized because
// factors are used from several host threads at once (one stream each).
template <class R>
void set_smem_limits(int small_front) {
    static std::mutex mu;
    static bool done = false;
    std::lock_guard<std::mutex> lock(mu);
    if (done) return;
    APHI_CUDA(cudaFuncSetAttribute(k_small_front<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   96 * 96 * static_cast<int>(sizeof(cx<R>))));
    APHI_CUDA(cudaFuncSetAttribute(k_update_panel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   2 * kStep * kTile * static_cast<int>(sizeof(cx<R>))));
    APHI_CUDA(cudaFuncSetAttribute(k_update_wide<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, wide_smem<R>()));
    if constexpr (sizeof(R) == 8) {
        APHI_CUDA(cudaFuncSetAttribute(k_update_wide_dmma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kDmmaSmem));
        APHI_CUDA(cudaFuncSetAttribute(k_update_wide_dmma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kDmmaSmem));
    }
    if constexpr (sizeof(R) == 4)
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc<3, 2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcSmem<3, 2>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc<2, 2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcSmem<2, 2>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc<2, 2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcSmem<2, 2>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc<2, 3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcSmem<2, 3>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc<2, 3, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcSmem<2, 3>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc_presplit<2, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcPreSmem<3>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc_presplit<2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcPreSmem<4>::bytes));
        APHI_CUDA(cudaFuncSetAttribute(k_update_tc_presplit<4, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcPreSmem<4>::bytes));
    const int tri = kTriSmem * static_cast<int>(sizeof(cx<R>)), bwd = (kTriSmem + kRedSmem) * static_cast<int>(sizeof(cx<R>));
    APHI_CUDA(cudaFuncSetAttribute(k_fwd_diag<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    APHI_CUDA(cudaFuncSetAttribute(k_fwd_gather<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    APHI_CUDA(cudaFuncSetAttribute(k_fwd_update<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    APHI_CUDA(cudaFuncSetAttribute(k_bwd_diag<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd));
    APHI_CUDA(cudaFuncSetAttribute(k_bwd_update<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd));
    (void)small_front;
    done = true;
}

// Complex128 -> the factor's precision, and back (dense fronts in and out).
template <class R>
__global__ void k_narrow(long long len, const double* src, cx<R>* dst) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < len) dst[i] = cx<R>{static_cast<R>(src[2 * i]), static_cast<R>(src[2 * i + 1])};
}
template <class R>
__global__ void k_widen(long long len, const cx<R>* src, double* dst) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < len) {
        dst[2 * i] = static_cast<double>(src[i].re);
        dst[2 * i + 1] = static_cast<double>(src[i].im);
    }
}

// values: upper-CSR entries scattered into the panels; or, when `panels` is
// given, the panels themselves (complex128, batch x stored).
template <class R>
void factorize_numeric(aphi_factor* f, const double* values, const double* panels, cudaStream_t st) {
    const aphi_analysis* A = f->an;
    const int n = A->S.n;
    const dim3 g(ceil_div(std::max(n, 1), 256), f->batch);
    set_smem_limits<R>(A->opt.small_front);
    if (panels) {
        const long long len = A->S.stored * f->batch;
        k_narrow<R><<<ceil_div(std::max<long long>(len, 1), 256), 256, 0, st>>>(len, panels,
                                                                              reinterpret_cast<cx<R>*>(f->L));
        APHI_CHECK_LAUNCH();
    } else {
        APHI_CUDA(cudaMemsetAsync(f->L, 0, static_cast<size_t>(A->S.stored) * f->batch * f->elem, st));
        k_scatter_a<R><<<g, 256, 0, st>>>(n, A->d.row_ptr, A->d.col_idx, values, A->S.nnz_a, f->dscale,
                                          A->d.a_dest, reinterpret_cast<cx<R>*>(f->L), A->S.stored);
        APHI_CHECK_LAUNCH();
    }
    const bool tc = sizeof(R) == 4 && f->use_tc;
    run_plan<R>(f, tc ? A->plan_factor_tc : A->plan_factor, st, nullptr, nullptr, nullptr, nullptr);
    k_extract_d<R><<<dim3(A->S.ns, f->batch), 128, 0, st>>>(sched_of(A->d), A->S.ns, A->d.ref_of_post,
                                                          reinterpret_cast<const cx<R>*>(f->L), A->S.stored,
                                                          f->dref, n);
    APHI_CHECK_LAUNCH();
}

template <class R>
void solve_numeric(aphi_factor* f, int nrhs, const double* b, double* x, cudaStream_t st, const int* entries,
                   int nentries) {
    const aphi_analysis* A = f->an;
    const int n = A->S.n;
    if (f->nrhs_cap < nrhs) {
        if (f->y) cudaFree(f->y);
        if (f->U) cudaFree(f->U);
        if (f->part) cudaFree(f->part);
        f->y = f->U = f->part = nullptr;
        APHI_CUDA(cudaMalloc(&f->y, static_cast<size_t>(n) * nrhs * f->capacity * sizeof(cx<R>) + 16));
        APHI_CUDA(cudaMalloc(&f->U, static_cast<size_t>(std::max<long long>(A->upool, 1)) * nrhs * f->capacity *
                                        sizeof(cx<R>)));
        APHI_CUDA(cudaMalloc(&f->part, static_cast<size_t>(A->max_parts) * kSolveBlock * 8 * f->capacity * sizeof(cx<R>)));
        f->nrhs_cap = nrhs;
    }
    set_smem_limits<R>(A->opt.small_front);
    cx<R>* y = reinterpret_cast<cx<R>*>(f->y);
    cx<R>* U = reinterpret_cast<cx<R>*>(f->U);
    cx<R>* part = reinterpret_cast<cx<R>*>(f->part);
    const dim3 g(ceil_div(std::max(n, 1), 256), f->batch * nrhs);
    k_permute_in<R><<<g, 256, 0, st>>>(n, nrhs, A->d.orig_of_new, f->dscale, b, y);
    APHI_CHECK_LAUNCH();
    // The fused plans (half the launches, each triangle in the launch before
    // it) win while one entry is solved; with more, every CTA's reservation of
    // a triangle's shared memory costs occupancy and the split plans are
    // faster (32^3, FP32: 15.4 against 15.9 ms for one entry, 30.4 against
    // 25.4 ms for six).
    const int rows = entries ? nentries : f->batch;
    const bool split = f->solve_form == 1 || (f->solve_form < 0 && rows > 1);
    for (int k0 = 0; k0 < nrhs; k0 += 8) {
        const SolveArgs sa{n,       nrhs, k0, std::min(8, nrhs - k0), A->upool, A->max_parts, entries,
                           entries ? nentries : 0, f->counters, A->S.ns};
        run_plan<R>(f, split ? A->plan_fwd_split : A->plan_fwd, st, &sa, y, U, part);
        run_plan<R>(f, split ? A->plan_bwd_split : A->plan_bwd, st, &sa, y, U, part);
    }
    k_permute_out<R><<<g, 256, 0, st>>>(n, nrhs, A->d.new_of_orig, f->dscale, y, x);
    APHI_CHECK_LAUNCH();
    if (f->profile && !f->prof_kinds.empty()) {
        APHI_CUDA(cudaStreamSynchronize(st));
        collect_profile(f);
    }
}

}  // namespace

aphi_factor* factor_create(aphi_analysis* an, int precision, int batch) {
    if (!an) throw Error(APHI_ERR_INVALID, "factor: null analysis");
    if (precision != 64 && precision != 32) throw Error(APHI_ERR_BAD_SHAPE, "factor: precision must be 64 or 32");
    if (batch < 1) throw Error(APHI_ERR_BAD_SHAPE, "factor: batch must be at least 1");
    analysis_ensure_device(an);
    auto* f = new aphi_factor;
    try {
        f->an = an;
        f->precision = precision;
        f->batch = batch;
        f->capacity = batch;
        f->elem = precision == 64 ? 16 : 8;
        const char* no_tc = std::getenv("APHI_NO_TC");
        f->use_tc = !(no_tc && no_tc[0] == '1');
        const char* split = std::getenv("APHI_TC_SPLIT");
        f->tc_split = split && split[0] == '2' ? 2 : 3;
        const char* stages = std::getenv("APHI_TC_STAGES");
        f->tc_stages = stages && stages[0] == '3' ? 3 : 2;
        const char* group = std::getenv("APHI_TC_GROUP");
        f->tc_group = group && group[0] == '4' ? 4 : 2;
        const char* pre = std::getenv("APHI_TC_PRESPLIT");
        f->presplit = !(pre && pre[0] == '0');
        const char* pst = std::getenv("APHI_TC_PRESTAGES");
        f->pre_stages = pst && pst[0] == '4' ? 4 : 3;
        if (precision == 32 && an->tc_ws_units > 0) {
            f->tcws_stride = an->tc_ws_units * 256;
            APHI_CUDA(cudaMalloc(&f->tcws, static_cast<size_t>(f->tcws_stride) * batch));
        }
        const char* psc = std::getenv("APHI_DMMA_PRESCALE");
        if (precision == 64 && an->dmma_ws_units > 0 && !(psc && psc[0] == '0')) {
            f->dws_stride = an->dmma_ws_units * 256;
            APHI_CUDA(cudaMalloc(&f->dws, static_cast<size_t>(f->dws_stride) * batch));
        }
        const Symbolic& S = an->S;
        APHI_CUDA(cudaMalloc(&f->L, static_cast<size_t>(std::max<long long>(S.stored, 1)) * batch * f->elem));
        f->dscale = dalloc<double>(static_cast<size_t>(S.n) * batch);
        f->rowmax = dalloc<unsigned long long>(static_cast<size_t>(S.n) * batch);
        f->stats = dalloc<unsigned long long>(4 * static_cast<size_t>(batch));
        f->dref = dalloc<double>(2 * static_cast<size_t>(S.n) * batch);
        f->err = dalloc<int>(4);
        f->kmax = dalloc<int>(batch);
        APHI_CUDA(cudaMemset(f->err, 0, 4 * sizeof(int)));
        f->counters = dalloc<int>(static_cast<size_t>(std::max(S.ns, 1)) * batch);
        APHI_CUDA(cudaMemset(f->counters, 0, sizeof(int) * std::max(S.ns, 1) * batch));
        const char* split_solve = std::getenv("APHI_SOLVE_SPLIT");
        f->solve_form = split_solve && split_solve[0] == '1' ? 1 : (split_solve && split_solve[0] == '0' ? 0 : -1);
        f->host_stats.assign(batch, aphi_factor_stats{});
    } catch (...) {
        delete f;
        throw;
    }
    return f;
}

void factor_destroy(aphi_factor* f) { delete f; }

void fronts_read(const aphi_factor* f, int k, double* panels_out, double* cb_out, cudaStream_t st) {
    const aphi_analysis* A = f->an;
    if (!A->fronts) throw Error(APHI_ERR_INVALID, "fronts_read: not a fronts analysis");
    if (k < 0 || k >= f->batch) throw Error(APHI_ERR_BAD_SHAPE, "fronts_read: batch index out of range");
    if (!f->factored) throw Error(APHI_ERR_INVALID, "fronts_read: nothing factorized yet");
    // The contribution blocks live in the analysis's shared workspace of this
    // precision: they are those of its latest factorization.
    const int wi = f->precision == 64 ? 0 : 1;
    std::lock_guard<std::mutex> ws_lock(f->an->ws_mu[wi]);
    const long long ls = A->S.stored, cs = A->S.cb_pool;
    auto widen = [&](const void* src, long long len, double* dst) {
        if (!dst || len == 0) return;
        if (f->precision == 64)
            k_widen<double><<<ceil_div(len, 256), 256, 0, st>>>(len, static_cast<const cx<double>*>(src), dst);
        else
            k_widen<float><<<ceil_div(len, 256), 256, 0, st>>>(len, static_cast<const cx<float>*>(src), dst);
        APHI_CHECK_LAUNCH();
    };
    widen(static_cast<const char*>(f->L) + static_cast<size_t>(ls) * k * f->elem, ls, panels_out);
    widen(static_cast<const char*>(A->ws[wi]) + static_cast<size_t>(cs) * k * f->elem, cs, cb_out);
    APHI_CUDA(cudaStreamSynchronize(st));
}

void factor_set_batch(aphi_factor* f, int batch) {
    if (batch < 1 || batch > f->capacity)
        throw Error(APHI_ERR_BAD_SHAPE, "factor_set_batch: the active batch must be 1.." + std::to_string(f->capacity));
    f->batch = batch;
    f->factored = false;
}

void factor_profile(aphi_factor* f, bool enable, unsigned mask) {
    f->profile = enable;
    f->prof_mask = mask;
    for (int k = 0; k < APHI_PLAN_KINDS; ++k) {
        f->prof_ms[k] = 0;
        f->prof_launches[k] = 0;
    }
}

int factorize(aphi_factor* f, const double* values, int equil_iters, double pivot_floor,
              aphi_factor_stats* stats_out, cudaStream_t st, const double* panels) {
    const aphi_analysis* A = f->an;
    const Symbolic& S = A->S;
    const int n = S.n;
    const int B = f->batch;
    if (!values && !panels) throw Error(APHI_ERR_INVALID, "factorize: null values");
    if (panels && equil_iters != 0) throw Error(APHI_ERR_BAD_SHAPE, "factorize: dense fronts are not equilibrated");
    if (!panels && A->fronts) throw Error(APHI_ERR_INVALID, "factorize: a fronts analysis takes panels, not values");
    if (equil_iters < 0) throw Error(APHI_ERR_BAD_SHAPE, "factorize: negative equilibration iterations");
    const auto t0 = std::chrono::steady_clock::now();
    cudaEvent_t e0, e1;
    APHI_CUDA(cudaEventCreate(&e0));
    APHI_CUDA(cudaEventCreate(&e1));
    APHI_CUDA(cudaEventRecord(e0, st));

    // Equilibration (FP64 on the original values).
    const long long nd = static_cast<long long>(n) * B;
    k_fill<<<ceil_div(std::max<long long>(nd, 1), 256), 256, 0, st>>>(f->dscale, nd, 1.0);
    APHI_CHECK_LAUNCH();
    APHI_CUDA(cudaMemsetAsync(f->rowmax, 0, sizeof(unsigned long long) * std::max<long long>(nd, 1), st));
    const dim3 g(ceil_div(std::max(n, 1), kEqThreads), B);
    for (int it = 0; it < equil_iters; ++it) {
        k_eq_rowmax<<<g, kEqThreads, 0, st>>>(n, A->d.row_ptr, A->d.col_idx, values, S.nnz_a, f->dscale, f->rowmax);
        APHI_CHECK_LAUNCH();
        k_eq_update<<<g, kEqThreads, 0, st>>>(n, f->dscale, f->rowmax);
        APHI_CHECK_LAUNCH();
    }
    // The contribution-block pool is only live during a factorization, so it
    // is a workspace owned by the analysis and shared by every factor of the
    // same precision made from it (one pool per precision). A factorization
    // holds that pool's lock from here until its stream has finished with the
    // pool (the synchronize below), so factorizations of one precision from
    // several host threads, on any streams, take turns, while an FP64 and an
    // FP32 factorization can run at the same time.
    const int wi = f->precision == 64 ? 0 : 1;
    std::unique_lock<std::mutex> ws_lock(f->an->ws_mu[wi]);
    {
        aphi_analysis* an = f->an;
        const size_t need = static_cast<size_t>(std::max<long long>(S.cb_pool, 1)) * B * f->elem;
        if (an->ws_bytes[wi] < need) {
            if (an->ws[wi]) {
                APHI_CUDA(cudaDeviceSynchronize());
                cudaFree(an->ws[wi]);
                an->ws[wi] = nullptr;
                an->ws_bytes[wi] = 0;
            }
            APHI_CUDA(cudaMalloc(&an->ws[wi], need));
            an->ws_bytes[wi] = need;
        }
        f->CB = an->ws[wi];
    }
    if (f->precision == 64)
        factorize_numeric<double>(f, values, panels, st);
    else
        factorize_numeric<float>(f, values, panels, st);
    APHI_CUDA(cudaEventRecord(e1, st));

    // Stats, computed as the reference computes them: walk the pivots in its
    // column order, stop at the first at or below the floor.
    std::vector<double> dref(2 * static_cast<size_t>(n) * B), dsc(static_cast<size_t>(n) * B);
    APHI_CUDA(cudaMemcpyAsync(dref.data(), f->dref, dref.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaMemcpyAsync(dsc.data(), f->dscale, dsc.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    int err_word = 0;
    APHI_CUDA(cudaMemcpyAsync(&err_word, f->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    ws_lock.unlock();
    if (err_word != 0) {
        if (f->profile) collect_profile(f);
        APHI_CUDA(cudaMemsetAsync(f->err, 0, sizeof(int), st));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        f->factored = false;
        throw Error(APHI_ERR_TIMEOUT, "factorize: a tensor-core tile's bounded wait expired");
    }
    if (f->profile) collect_profile(f);
    float ms = 0;
    APHI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<int> kmax(B, 0x7fffffff);
    const bool any_fail = pivot_stats(n, B, dref.data(), dsc.data(), pivot_floor, ms, S.nnz_l,
                                      f->host_stats.data(), kmax.data());
    // Largest multiplier, over the rows the reference would have reached.
    int* d_kmax = f->kmax;
    APHI_CUDA(cudaMemcpyAsync(d_kmax, kmax.data(), sizeof(int) * B, cudaMemcpyHostToDevice, st));
    APHI_CUDA(cudaMemsetAsync(f->stats, 0, sizeof(unsigned long long) * 4 * B, st));
    if (A->stat_count > 0) {
        const dim3 gs(A->stat_count, B);
        if (f->precision == 64)
            k_max_multiplier<double><<<gs, 256, 0, st>>>(sched_of(A->d), A->stat_first, A->d.ref_of_post,
                                                         reinterpret_cast<const cx<double>*>(f->L), S.stored,
                                                         d_kmax, f->stats);
        else
            k_max_multiplier<float><<<gs, 256, 0, st>>>(sched_of(A->d), A->stat_first, A->d.ref_of_post,
                                                        reinterpret_cast<const cx<float>*>(f->L), S.stored,
                                                        d_kmax, f->stats);
        APHI_CHECK_LAUNCH();
    }
    std::vector<unsigned long long> mx(4 * B);
    APHI_CUDA(cudaMemcpyAsync(mx.data(), f->stats, sizeof(unsigned long long) * 4 * B, cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    for (int b = 0; b < B; ++b) {
        double v;
        std::memcpy(&v, &mx[b], sizeof(double));
        f->host_stats[b].largest_multiplier = v;
        if (stats_out) stats_out[b] = f->host_stats[b];
    }
    (void)t0;
    f->factored = true;
    return any_fail ? APHI_ERR_PIVOT_FLOOR : APHI_OK;
}

// entries (device, nentries of them): solve only these batch entries; the
// others' x is left holding their permuted, scaled b. Null: every entry.
void solve(aphi_factor* f, int nrhs, const double* b, double* x, cudaStream_t st, const int* entries,
           int nentries) {
    if (!f->factored) throw Error(APHI_ERR_INVALID, "solve: the factor holds no factorization");
    if (f->an->fronts) throw Error(APHI_ERR_INVALID, "solve: dense fronts have no system to solve");
    if (nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "solve: nrhs must be at least 1");
    for (int k = 0; k < f->batch; ++k)
        if (!f->host_stats[k].ok)
            throw Error(APHI_ERR_ZERO_PIVOT,
                        "solve_in_place: the factorization stopped at a pivot at or below the floor, so "
                        "this factor cannot be used.");
    if (f->precision == 64)
        solve_numeric<double>(f, nrhs, b, x, st, entries, nentries);
    else
        solve_numeric<float>(f, nrhs, b, x, st, entries, nentries);
}

// Per-thread device scratch that only grows: freeing device memory
// synchronizes the whole device, which would stall work other threads have
// in flight on their own streams.
struct ThreadScratch {
    double* p = nullptr;
    size_t doubles = 0;
    int device = -1;
    ~ThreadScratch() {
        if (p) cudaFree(p);
    }
    double* get(size_t need) {
        int dev = 0;
        APHI_CUDA(cudaGetDevice(&dev));
        if (need > doubles || dev != device) {
            if (p) cudaFree(p);
            p = nullptr;
            doubles = 0;
            p = dalloc<double>(need);
            doubles = need;
            device = dev;
        }
        return p;
    }
};
thread_local ThreadScratch t_residual_scratch;

constexpr long long kMaxGridY = 65535;  // grid.y limit of the residual kernels (one system per y)

void residuals(const aphi_analysis* an, int batch, int nrhs, const double* values, const double* x,
               const double* b, double* out, cudaStream_t st) {
    if (static_cast<long long>(batch) * nrhs > kMaxGridY)
        throw Error(APHI_ERR_BAD_SHAPE, "residuals: batch x nrhs exceeds the " + std::to_string(kMaxGridY) +
                                            " systems one call handles");
    const int n = an->S.n;
    const int nb = ceil_div(std::max(n, 1), 256);
    const size_t np = static_cast<size_t>(nb) * 3 * batch * nrhs;
    double* partial = t_residual_scratch.get(np + batch + 4 * static_cast<size_t>(batch) * nrhs);
    unsigned long long* amax = reinterpret_cast<unsigned long long*>(partial + np);
    double* norms = partial + np + batch;
    APHI_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * batch, st));
    k_residual<<<dim3(nb, batch * nrhs), 256, 0, st>>>(n, nrhs, an->d.fptr, an->d.fcol, an->d.fmap, values,
                                                       an->S.nnz_a, x, b, nullptr, partial);
    APHI_CHECK_LAUNCH();
    k_amax<<<dim3(ceil_div(std::max<long long>(an->S.nnz_a, 1), 256), batch), 256, 0, st>>>(values, an->S.nnz_a, amax);
    APHI_CHECK_LAUNCH();
    k_norms_final<<<batch * nrhs, 256, 0, st>>>(nb, nrhs, partial, amax, norms);
    APHI_CHECK_LAUNCH();
    std::vector<double> h(4 * static_cast<size_t>(batch) * nrhs);
    APHI_CUDA(cudaMemcpyAsync(h.data(), norms, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < batch * nrhs; ++q) {
        const double rn = h[4 * q], bn = h[4 * q + 1], xn = h[4 * q + 2], am = h[4 * q + 3];
        out[2 * q] = bn > 0.0 ? rn / bn : rn;
        const double den = am * xn + bn;
        out[2 * q + 1] = den > 0.0 ? rn / den : rn;
    }
}

// relative_residual and backward_error of a matrix held only as host CSR
// arrays (upper-stored), with x and b on the host: the mirrored pattern is
// built on the host (structure only), every product and sum runs on the
// device with the kernels above. out: nrhs x 2 (relative residual, backward
// error).
void csr_residuals_host(int n, const int* row_ptr, const int* col_idx, const double* values, int nrhs,
                        const double* x, const double* b, double* out) {
    if (n < 1 || nrhs < 1 || nrhs > kMaxGridY)
        throw Error(APHI_ERR_BAD_SHAPE, "relative_residual: n must be >= 1 and nrhs in 1..65535");
    const long long nnz = row_ptr[n];
    std::vector<int> fptr(static_cast<size_t>(n) + 1, 0), fcol;
    std::vector<long long> fmap;
    for (int r = 0; r < n; ++r)
        for (long long k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            if (c < r || c >= n) throw Error(APHI_ERR_BAD_SHAPE, "relative_residual: the pattern is not upper");
            ++fptr[r + 1];
            if (c != r) ++fptr[c + 1];
        }
    for (int r = 0; r < n; ++r) fptr[r + 1] += fptr[r];
    fcol.resize(fptr[n]);
    fmap.resize(fptr[n]);
    {
        std::vector<int> cur(fptr.begin(), fptr.end() - 1);
        for (int r = 0; r < n; ++r)
            for (long long k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
                const int c = col_idx[k];
                fcol[cur[r]] = c;
                fmap[cur[r]++] = k;
                if (c != r) {
                    fcol[cur[c]] = r;
                    fmap[cur[c]++] = k;
                }
            }
    }
    const int nb = ceil_div(n, 256);
    std::vector<void*> owned;
    auto up = [&](const void* h, size_t bytes) {
        void* d = nullptr;
        APHI_CUDA(cudaMalloc(&d, std::max<size_t>(bytes, 16)));
        owned.push_back(d);
        if (h && bytes) APHI_CUDA(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice));
        return d;
    };
    try {
        const int* d_fptr = static_cast<const int*>(up(fptr.data(), fptr.size() * sizeof(int)));
        const int* d_fcol = static_cast<const int*>(up(fcol.data(), fcol.size() * sizeof(int)));
        const long long* d_fmap = static_cast<const long long*>(up(fmap.data(), fmap.size() * sizeof(long long)));
        const double* d_v = static_cast<const double*>(up(values, 16 * static_cast<size_t>(nnz)));
        const double* d_x = static_cast<const double*>(up(x, 16 * static_cast<size_t>(n) * nrhs));
        const double* d_b = static_cast<const double*>(up(b, 16 * static_cast<size_t>(n) * nrhs));
        double* partial = static_cast<double*>(up(nullptr, sizeof(double) * 3 * static_cast<size_t>(nb) * nrhs));
        auto* amax = static_cast<unsigned long long*>(up(nullptr, sizeof(unsigned long long)));
        double* norms = static_cast<double*>(up(nullptr, sizeof(double) * 4 * static_cast<size_t>(nrhs)));
        APHI_CUDA(cudaMemset(amax, 0, sizeof(unsigned long long)));
        k_residual<<<dim3(nb, nrhs), 256>>>(n, nrhs, d_fptr, d_fcol, d_fmap, d_v, nnz, d_x, d_b, nullptr, partial);
        APHI_CHECK_LAUNCH();
        k_amax<<<dim3(ceil_div(std::max<long long>(nnz, 1), 256), 1), 256>>>(d_v, nnz, amax);
        APHI_CHECK_LAUNCH();
        k_norms_final<<<nrhs, 256>>>(nb, nrhs, partial, amax, norms);
        APHI_CHECK_LAUNCH();
        std::vector<double> h(4 * static_cast<size_t>(nrhs));
        APHI_CUDA(cudaMemcpy(h.data(), norms, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int q = 0; q < nrhs; ++q) {
            const double rn = h[4 * q], bn = h[4 * q + 1], xn = h[4 * q + 2], am = h[4 * q + 3];
            out[2 * q] = bn > 0.0 ? rn / bn : rn;
            const double den = am * xn + bn;
            out[2 * q + 1] = den > 0.0 ? rn / den : rn;
        }
    } catch (...) {
        for (void* d : owned) cudaFree(d);
        throw;
    }
    for (void* d : owned) cudaFree(d);
}

// ---------------------------------------------------------------- allocation-free residuals
// The same residual and backward-error computation as residuals() above, for
// callers that cannot allocate device memory while they run: a serving loop
// whose memory pool has already claimed the device's free memory for factors,
// or a latency-critical path that cannot absorb the device-wide
// synchronization cudaFree implies. Its scratch (per-block partial sums, the
// max|A| words and the final ratios) lives in the file-scope device array
// below, of fixed size; every GPU that loads this library holds it until the
// process exits.
//
// The array is shared by all calls: calls that overlap on the GPU (on
// different streams, or from different host threads) race on it, so a caller
// must order them. The max|A| words are cleared at the start of every call;
// everything else is fully written before it is read.
constexpr size_t kResidualScratchDoubles = size_t(1) << 20;  // 8 MiB
static __device__ __align__(256) double g_residual_scratch[kResidualScratchDoubles];

// Ratios straight into the scratch, so the host copy needs no staging buffer.
__global__ void k_norm_ratios(int q, const double* norms, double* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= q) return;
    const double rn = norms[4 * k], bn = norms[4 * k + 1], xn = norms[4 * k + 2], am = norms[4 * k + 3];
    out[2 * k] = bn > 0.0 ? rn / bn : rn;
    const double den = am * xn + bn;
    out[2 * k + 1] = den > 0.0 ? rn / den : rn;
}

namespace {

// Device address of the scratch array, looked up once per device with that
// device current. In host code the array's name stands for a host-side
// shadow, not a device address, so it is never handed to a kernel directly.
double* residual_scratch(int dev) {
    static std::mutex mu;
    static double* ptrs[64] = {};
    if (dev < 0 || dev >= 64) throw Error(APHI_ERR_INVALID, "residuals_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_residual_scratch);
        if (e != cudaSuccess || !p)
            throw Error(APHI_ERR_CUDA, std::string("residuals_noalloc: cudaGetSymbolAddress failed: ") +
                                           cudaGetErrorString(e));
        ptrs[dev] = static_cast<double*>(p);
    }
    return ptrs[dev];
}

}  // namespace

void residuals_noalloc(const aphi_analysis* an, int batch, int nrhs, const double* values, const double* x,
                       const double* b, double* out, cudaStream_t st) {
    if (!an->on_device)
        throw Error(APHI_ERR_INVALID,
                    "residuals_noalloc: the analysis has no device copy yet (create a factor from it first); "
                    "this entry point does not allocate one");
    int dev = 0;
    APHI_CUDA(cudaGetDevice(&dev));
    if (dev != an->device)
        throw Error(APHI_ERR_INVALID, "residuals_noalloc: the analysis's device copy lives on device " +
                                          std::to_string(an->device) + ", but device " + std::to_string(dev) +
                                          " is current");
    const int n = an->S.n;
    const long long nb = ceil_div(std::max(n, 1), 256);
    const long long q = static_cast<long long>(batch) * nrhs;
    if (q > kMaxGridY || batch > kMaxGridY)
        throw Error(APHI_ERR_BAD_SHAPE, "residuals_noalloc: batch x nrhs = " + std::to_string(q) +
                                            " exceeds the " + std::to_string(kMaxGridY) +
                                            " systems one call handles");
    // partial sums, max|A| words (one per batch entry), norms, ratios
    const long long need = nb * 3 * q + batch + 4 * q + 2 * q;
    if (need > static_cast<long long>(kResidualScratchDoubles))
        throw Error(APHI_ERR_BAD_SHAPE,
                    "residuals_noalloc: " + std::to_string(n) + " unknowns x " + std::to_string(q) +
                        " right-hand sides need " + std::to_string(need) + " doubles of scratch; the fixed "
                        "array holds " + std::to_string(kResidualScratchDoubles) +
                        " (use aphi_residuals, which allocates, or fewer right-hand sides per call)");
    double* scratch = residual_scratch(an->device);
    double* partial = scratch;
    unsigned long long* amax = reinterpret_cast<unsigned long long*>(scratch + nb * 3 * q);
    double* norms = scratch + nb * 3 * q + batch;
    double* ratios = norms + 4 * q;
    APHI_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * batch, st));
    k_residual<<<dim3(static_cast<unsigned>(nb), static_cast<unsigned>(q)), 256, 0, st>>>(
        n, nrhs, an->d.fptr, an->d.fcol, an->d.fmap, values, an->S.nnz_a, x, b, nullptr, partial);
    APHI_CHECK_LAUNCH();
    k_amax<<<dim3(ceil_div(std::max<long long>(an->S.nnz_a, 1), 256), batch), 256, 0, st>>>(values, an->S.nnz_a, amax);
    APHI_CHECK_LAUNCH();
    k_norms_final<<<static_cast<unsigned>(q), 256, 0, st>>>(static_cast<int>(nb), nrhs, partial, amax, norms);
    APHI_CHECK_LAUNCH();
    k_norm_ratios<<<ceil_div(q, 128), 128, 0, st>>>(static_cast<int>(q), norms, ratios);
    APHI_CHECK_LAUNCH();
    APHI_CUDA(cudaMemcpyAsync(out, ratios, sizeof(double) * 2 * q, cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
}

int solve_krylov(aphi_factor* f, int nrhs, const double* values, const double* b, double* x,
                 const aphi_ir_options& opt, int* iters, double* berr, cudaStream_t st);

int solve_refined(aphi_factor* f, int nrhs, const double* values, const double* b, double* x,
                  const aphi_ir_options& opt, int* iters, double* berr, cudaStream_t st) {
    if (opt.krylov) return solve_krylov(f, nrhs, values, b, x, opt, iters, berr, st);
    const aphi_analysis* A = f->an;
    const int n = A->S.n;
    const int B = f->batch;
    const int C = f->capacity;  // scratch is sized for the capacity, used for the active batch
    const long long len = 2LL * n * nrhs * B;
    if (f->ir_cap < nrhs) {
        if (f->ir) cudaFree(f->ir);
        f->ir = dalloc<double>(static_cast<size_t>(2LL * n * nrhs * C) * 2);
        f->ir_cap = nrhs;
    }
    double* r = f->ir;
    double* dx = f->ir + len;
    const int nb = ceil_div(std::max(n, 1), 256);
    if (f->red_cap < nrhs) {
        if (f->red) cudaFree(f->red);
        if (f->norms) cudaFree(f->norms);
        f->red = dalloc<double>(static_cast<size_t>(nb) * 3 * C * nrhs + C + 1);
        f->norms = dalloc<double>(4 * static_cast<size_t>(C) * nrhs);
        f->red_cap = nrhs;
    }
    unsigned long long* amax = reinterpret_cast<unsigned long long*>(f->red + static_cast<size_t>(nb) * 3 * B * nrhs);
    solve(f, nrhs, b, x, st);
    APHI_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * B, st));
    k_amax<<<dim3(ceil_div(std::max<long long>(A->S.nnz_a, 1), 256), B), 256, 0, st>>>(values, A->S.nnz_a, amax);
    APHI_CHECK_LAUNCH();
    const int q = B * nrhs;
    std::vector<double> prev(q, INFINITY), h(4 * static_cast<size_t>(q));
    std::vector<int> it(q, 0);
    std::vector<char> done(q, 0);
    int status = APHI_OK;
    for (int step = 0;; ++step) {
        k_residual<<<dim3(nb, q), 256, 0, st>>>(n, nrhs, A->d.fptr, A->d.fcol, A->d.fmap, values, A->S.nnz_a, x, b,
                                                r, f->red);
        APHI_CHECK_LAUNCH();
        k_norms_final<<<q, 256, 0, st>>>(nb, nrhs, f->red, amax, f->norms);
        APHI_CHECK_LAUNCH();
        APHI_CUDA(cudaMemcpyAsync(h.data(), f->norms, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        APHI_CUDA(cudaStreamSynchronize(st));
        bool all = true;
        for (int k = 0; k < q; ++k) {
            if (done[k]) continue;
            const double den = h[4 * k + 3] * h[4 * k + 2] + h[4 * k + 1];
            const double e = den > 0.0 ? h[4 * k] / den : h[4 * k];
            const double rr = h[4 * k + 1] > 0.0 ? h[4 * k] / h[4 * k + 1] : h[4 * k];
            berr[k] = e;
            iters[k] = it[k];
            if (e <= opt.tol && rr <= opt.rtol) {
                done[k] = 1;
                continue;
            }
            if (!(e < opt.stall_ratio * prev[k]) || it[k] >= opt.max_iters) {
                done[k] = 1;
                status = APHI_ERR_IR_STALL;
                continue;
            }
            prev[k] = e;
            all = false;
        }
        if (all) break;
        // One correction for every entry (converged ones get a tiny harmless step
        // from their own residual; their reported error is already frozen).
        solve(f, nrhs, r, dx, st);
        k_axpy<<<ceil_div(len, 256), 256, 0, st>>>(len, x, dx);
        APHI_CHECK_LAUNCH();
        for (int k = 0; k < q; ++k)
            if (!done[k]) ++it[k];
    }
    return status;
}

// COCG steps without a stall_ratio drop of the best relative residual before
// a system is declared stalled. COCG's residual is not monotone: near
// rho(I - M^-1 A) ~ 0.9 it can stay above half its best for three steps and
// still converge a few steps later.
constexpr int kCocgPatience = 5;

// ---------------------------------------------------------------- Krylov refinement
// Preconditioned COCG (conjugate orthogonal CG: CG with the unconjugated
// bilinear form x^T y, valid for complex symmetric A and M) in FP64 on the
// original system, with the factor as preconditioner M^-1. With an FP32
// factor this is refinement whose residual, scaling and update stay in FP64;
// the Krylov recurrence keeps it converging where plain refinement
// (x += M^-1 r) stalls because cond(A) * eps_fp32 approaches 1. The residual
// is recomputed from x every iteration (b - A x), so the reported backward
// error is the true one. Systems are advanced together and frozen one by one
// as they converge.

// y = A x for q systems.
__global__ void k_spmv(int n, int nrhs, const int* fptr, const int* fcol, const long long* fmap,
                       const double* values, long long nnz, const double* x, double* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= n) return;
    const double* v = values + 2LL * nnz * (k / nrhs);
    const double* xk = x + 2LL * n * k;
    double ar = 0, ai = 0;
    for (int t = fptr[i]; t < fptr[i + 1]; ++t) {
        const long long q = fmap[t];
        const double vr = v[2 * q], vi = v[2 * q + 1];
        const double xr = xk[2 * fcol[t]], xi = xk[2 * fcol[t] + 1];
        ar += vr * xr - vi * xi;
        ai += vr * xi + vi * xr;
    }
    y[2LL * n * k + 2 * i] = ar;
    y[2LL * n * k + 2 * i + 1] = ai;
}

// partial[k][blk] = sum over the block's entries of a_i b_i (unconjugated).
__global__ void k_dot_partial(int n, const double* a, const double* b, double* partial) {
    __shared__ double sh[2][256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    double re = 0, im = 0;
    if (i < n) {
        const double ar = a[2LL * n * k + 2 * i], ai = a[2LL * n * k + 2 * i + 1];
        const double br = b[2LL * n * k + 2 * i], bi = b[2LL * n * k + 2 * i + 1];
        re = ar * br - ai * bi;
        im = ar * bi + ai * br;
    }
    sh[0][threadIdx.x] = re;
    sh[1][threadIdx.x] = im;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * (static_cast<long long>(k) * gridDim.x + blockIdx.x)] = sh[0][0];
        partial[2 * (static_cast<long long>(k) * gridDim.x + blockIdx.x) + 1] = sh[1][0];
    }
}

__device__ __forceinline__ void cdiv_dev(double ar, double ai, double br, double bi, double& cr, double& ci) {
    if (fabs(br) >= fabs(bi)) {
        const double r = bi / br, den = br + bi * r;
        cr = (ar + ai * r) / den;
        ci = (ai - ar * r) / den;
    } else {
        const double r = br / bi, den = br * r + bi;
        cr = (ar * r + ai) / den;
        ci = (ai * r - ar) / den;
    }
}

// Fixed-order sum of the partials, then the COCG scalar of each system.
//   mode 0: rho = r^T z (start)            -> rho
//   mode 1: alpha = rho / (p^T A p)        -> alpha (0 for frozen systems)
//   mode 2: rho' = r^T z, beta = rho'/rho  -> beta, rho = rho'
__global__ void k_cocg_scalar(int nblocks, const double* partial, const int* active, double* rho, double* alpha,
                              double* beta, int mode) {
    __shared__ double sh[2][256];
    const int k = blockIdx.x;
    double re = 0, im = 0;
    for (int t = threadIdx.x; t < nblocks; t += blockDim.x) {
        re += partial[2 * (static_cast<long long>(k) * nblocks + t)];
        im += partial[2 * (static_cast<long long>(k) * nblocks + t) + 1];
    }
    sh[0][threadIdx.x] = re;
    sh[1][threadIdx.x] = im;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double sr = sh[0][0], si = sh[1][0];
    if (mode == 0) {
        rho[2 * k] = sr;
        rho[2 * k + 1] = si;
    } else if (mode == 1) {
        double ar = 0, ai = 0;
        if (active[k] && (sr != 0.0 || si != 0.0)) cdiv_dev(rho[2 * k], rho[2 * k + 1], sr, si, ar, ai);
        alpha[2 * k] = ar;
        alpha[2 * k + 1] = ai;
    } else {
        double br = 0, bi = 0;
        if (active[k] && (rho[2 * k] != 0.0 || rho[2 * k + 1] != 0.0)) cdiv_dev(sr, si, rho[2 * k], rho[2 * k + 1], br, bi);
        beta[2 * k] = br;
        beta[2 * k + 1] = bi;
        if (active[k]) {
            rho[2 * k] = sr;
            rho[2 * k + 1] = si;
        }
    }
}

// x += alpha p (per system).
__global__ void k_axpy_sys(int n, const double* alpha, const double* p, double* x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= n) return;
    const double ar = alpha[2 * k], ai = alpha[2 * k + 1];
    if (ar == 0.0 && ai == 0.0) return;
    const long long at = 2LL * n * k + 2 * i;
    const double pr = p[at], pi = p[at + 1];
    x[at] += ar * pr - ai * pi;
    x[at + 1] += ar * pi + ai * pr;
}

// p = z + beta p (active systems only).
__global__ void k_xpby_sys(int n, const int* active, const double* beta, const double* z, double* p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= n || !active[k]) return;
    const double br = beta[2 * k], bi = beta[2 * k + 1];
    const long long at = 2LL * n * k + 2 * i;
    const double pr = p[at], pi = p[at + 1];
    p[at] = z[at] + br * pr - bi * pi;
    p[at + 1] = z[at + 1] + br * pi + bi * pr;
}

int solve_krylov(aphi_factor* f, int nrhs, const double* values, const double* b, double* x,
                 const aphi_ir_options& opt, int* iters, double* berr, cudaStream_t st) {
    const aphi_analysis* A = f->an;
    const int n = A->S.n;
    const int B = f->batch;
    const int q = B * nrhs;
    const long long len = 2LL * n * q;
    const int nb = ceil_div(std::max(n, 1), 256);
    if (f->kr_cap < nrhs) {
        if (f->kr) cudaFree(f->kr);
        // r, z, p, Ap; partials (3 per block per system); norms, rho, alpha,
        // beta; max|A| words; active flags -- sized for the capacity.
        const long long qc = static_cast<long long>(f->capacity) * nrhs;
        f->kr = dalloc<double>(static_cast<size_t>(4 * 2LL * n * qc + 3LL * nb * qc + 11LL * qc + 2LL * f->capacity + 16));
        f->kr_cap = nrhs;
    }
    double* r = f->kr;
    double* z = r + len;
    double* p = z + len;
    double* Ap = p + len;
    double* partial = Ap + len;                 // 3 * nb * q
    double* norms = partial + 3LL * nb * q;     // 4 * q
    double* rho = norms + 4LL * q;              // 2 * q
    double* alpha = rho + 2LL * q;              // 2 * q
    double* beta = alpha + 2LL * q;             // 2 * q
    unsigned long long* amax = reinterpret_cast<unsigned long long*>(beta + 2LL * q);  // B
    int* active = reinterpret_cast<int*>(amax + B);                                   // q ints
    int* entries = active + q;                                                        // B ints
    const dim3 gv(nb, q);

    APHI_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * B, st));
    k_amax<<<dim3(ceil_div(std::max<long long>(A->S.nnz_a, 1), 256), B), 256, 0, st>>>(values, A->S.nnz_a, amax);
    APHI_CHECK_LAUNCH();
    std::vector<int> act(q, 1), it(q, 0), since(q, 0), ent;
    std::vector<int> restarted(q, 0), restart_now(q, 0);
    std::vector<double> h(4 * static_cast<size_t>(q)), best(q, INFINITY);
    APHI_CUDA(cudaMemcpyAsync(active, act.data(), sizeof(int) * q, cudaMemcpyHostToDevice, st));

    auto residual = [&]() {  // r = b - A x; norms to the host
        k_residual<<<gv, 256, 0, st>>>(n, nrhs, A->d.fptr, A->d.fcol, A->d.fmap, values, A->S.nnz_a, x, b, r,
                                       partial);
        APHI_CHECK_LAUNCH();
        k_norms_final<<<q, 256, 0, st>>>(nb, nrhs, partial, amax, norms);
        APHI_CHECK_LAUNCH();
        APHI_CUDA(cudaMemcpyAsync(h.data(), norms, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        APHI_CUDA(cudaStreamSynchronize(st));
    };
    auto dot = [&](const double* u, const double* v, int mode) {
        k_dot_partial<<<gv, 256, 0, st>>>(n, u, v, partial);
        APHI_CHECK_LAUNCH();
        k_cocg_scalar<<<q, 256, 0, st>>>(nb, partial, active, rho, alpha, beta, mode);
        APHI_CHECK_LAUNCH();
    };

    solve(f, nrhs, b, x, st);  // x0 = M^-1 b
    residual();
    int status = APHI_OK;
    bool started = false;
    for (;;) {
        bool any = false;
        for (int k = 0; k < q; ++k) {
            if (!act[k]) continue;
            const double den = h[4 * k + 3] * h[4 * k + 2] + h[4 * k + 1];
            const double e = den > 0.0 ? h[4 * k] / den : h[4 * k];
            const double rr = h[4 * k + 1] > 0.0 ? h[4 * k] / h[4 * k + 1] : h[4 * k];
            berr[k] = e;
            iters[k] = it[k];
            if (e <= opt.tol && rr <= opt.rtol) {
                act[k] = 0;
                continue;
            }
            if (rr < opt.stall_ratio * best[k]) {
                best[k] = rr;
                since[k] = 0;
            } else if (++since[k] >= kCocgPatience || !(rr == rr)) {
                if (rr == rr && !restarted[k]) {
                    // Once per system: restart the recurrence from the current
                    // iterate (p = z, rho = r^T z) before calling it stalled.
                    // COCG's unconjugated form can stagnate near a breakdown
                    // of its recurrence that a fresh start avoids.
                    restarted[k] = restart_now[k] = 1;
                    since[k] = 0;
                    best[k] = rr;
                } else {
                    act[k] = 0;
                    status = APHI_ERR_IR_STALL;
                    continue;
                }
            }
            if (it[k] >= opt.max_iters) {
                act[k] = 0;
                status = APHI_ERR_IR_STALL;
                continue;
            }
            any = true;
        }
        if (!any) break;
        APHI_CUDA(cudaMemcpyAsync(active, act.data(), sizeof(int) * q, cudaMemcpyHostToDevice, st));
        // The preconditioner solve runs over the entries with a system still
        // iterating; a frozen system's z is never read again (its alpha and
        // beta are zero and its updates are masked).
        ent.clear();
        for (int e = 0; e < B; ++e)
            for (int k = 0; k < nrhs; ++k)
                if (act[e * nrhs + k]) {
                    ent.push_back(e);
                    break;
                }
        const bool all = static_cast<int>(ent.size()) == B;
        if (!all)
            APHI_CUDA(cudaMemcpyAsync(entries, ent.data(), sizeof(int) * ent.size(), cudaMemcpyHostToDevice, st));
        solve(f, nrhs, r, z, st, all ? nullptr : entries, static_cast<int>(ent.size()));  // z = M^-1 r
        if (!started) {
            APHI_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * len, cudaMemcpyDeviceToDevice, st));
            dot(r, z, 0);
            started = true;
        } else {
            dot(r, z, 2);
            for (int k = 0; k < q; ++k)
                if (restart_now[k]) {  // beta = 0: p = z
                    APHI_CUDA(cudaMemsetAsync(beta + 2 * k, 0, 2 * sizeof(double), st));
                    restart_now[k] = 0;
                }
            k_xpby_sys<<<gv, 256, 0, st>>>(n, active, beta, z, p);
            APHI_CHECK_LAUNCH();
        }
        k_spmv<<<gv, 256, 0, st>>>(n, nrhs, A->d.fptr, A->d.fcol, A->d.fmap, values, A->S.nnz_a, p, Ap);
        APHI_CHECK_LAUNCH();
        dot(p, Ap, 1);
        k_axpy_sys<<<gv, 256, 0, st>>>(n, alpha, p, x);
        APHI_CHECK_LAUNCH();
        for (int k = 0; k < q; ++k)
            if (act[k]) ++it[k];
        residual();
    }
    return status;
}

void spmv(const aphi_analysis* an, int batch, int nrhs, const double* values, const double* x, double* y,
          cudaStream_t st) {
    if (static_cast<long long>(batch) * nrhs > kMaxGridY)
        throw Error(APHI_ERR_BAD_SHAPE, "spmv: batch x nrhs exceeds the 65535 systems one call handles");
    const int n = an->S.n;
    if (n == 0) return;
    k_spmv<<<dim3(ceil_div(n, 256), batch * nrhs), 256, 0, st>>>(n, nrhs, an->d.fptr, an->d.fcol, an->d.fmap, values,
                                                               an->S.nnz_a, x, y);
    APHI_CHECK_LAUNCH();
}

void factor_export(const aphi_factor* f, int k, int* col_ptr, int* row_index, double* value, double* diagonal,
                   double* d_scale) {
    const aphi_analysis* A = f->an;
    const Symbolic& S = A->S;
    const int n = S.n;
    if (k < 0 || k >= f->batch) throw Error(APHI_ERR_BAD_SHAPE, "factor_export: batch index out of range");
    if (!f->factored) throw Error(APHI_ERR_INVALID, "factor_export: nothing factorized yet");
    // Panels of entry k, widened to complex128.
    std::vector<double> Lh(2 * static_cast<size_t>(S.stored));
    if (f->precision == 64) {
        APHI_CUDA(cudaMemcpy(Lh.data(), static_cast<const char*>(f->L) + static_cast<size_t>(S.stored) * k * 16,
                             static_cast<size_t>(S.stored) * 16, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(2 * static_cast<size_t>(S.stored));
        APHI_CUDA(cudaMemcpy(tmp.data(), static_cast<const char*>(f->L) + static_cast<size_t>(S.stored) * k * 8,
                             static_cast<size_t>(S.stored) * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < tmp.size(); ++i) Lh[i] = tmp[i];
    }
    if (d_scale) APHI_CUDA(cudaMemcpy(d_scale, f->dscale + static_cast<size_t>(n) * k, sizeof(double) * n,
                                      cudaMemcpyDeviceToHost));
    // L's true column structures in the caller's numbering: row k of L is
    // what the row-subtree walk from A(k, 0:k-1) visits; rows come out in
    // increasing k, so each column is ascending.
    const std::vector<int>& parent = S.ref_parent;
    std::vector<int> iperm(n);
    for (int i = 0; i < n; ++i) iperm[S.perm[i]] = i;
    std::vector<std::vector<int>> earlier(n);
    for (int r = 0; r < n; ++r)
        for (int q = A->h_row_ptr[r]; q < A->h_row_ptr[r + 1]; ++q) {
            const int c = A->h_col_idx[q];
            if (c == r) continue;
            const int a = iperm[r], b = iperm[c];
            earlier[std::max(a, b)].push_back(std::min(a, b));
        }
    std::vector<int> cp(n + 1, 0);
    for (int j = 0; j < n; ++j) cp[j + 1] = cp[j] + S.ref_colcount[j] - 1;
    std::vector<int> fill(n, 0), mark(n, -1);
    std::vector<int> rows(cp[n]);
    for (int r = 0; r < n; ++r) {
        mark[r] = r;
        for (int j0 : earlier[r])
            for (int j = j0; j != -1 && mark[j] != r; j = parent[j]) {
                mark[j] = r;
                rows[cp[j] + fill[j]++] = r;
            }
    }
    if (col_ptr) std::copy(cp.begin(), cp.end(), col_ptr);
    for (int j = 0; j < n; ++j) {
        const int pj = S.post_of_ref[j];
        const int s = S.col_snode[pj];
        const int m = S.sn_rows[s];
        const int lc = pj - S.sn_first[s];
        const int* sb = S.structs.data() + S.sn_struct_off[s];
        const size_t base = static_cast<size_t>(S.sn_loff[s]) + static_cast<size_t>(lc) * m;
        if (diagonal) {
            diagonal[2 * j] = Lh[2 * (base + lc)];
            diagonal[2 * j + 1] = Lh[2 * (base + lc) + 1];
        }
        std::sort(rows.begin() + cp[j], rows.begin() + cp[j + 1]);
        for (int t = cp[j]; t < cp[j + 1]; ++t) {
            const int r = rows[t];
            if (row_index) row_index[t] = r;
            if (value) {
                const int pr = S.post_of_ref[r];
                const int* it = std::lower_bound(sb, sb + m, pr);
                if (it == sb + m || *it != pr) throw Error(APHI_ERR_PATTERN_MISMATCH, "factor_export: entry outside the panel");
                const size_t at = base + static_cast<size_t>(it - sb);
                value[2 * t] = Lh[2 * at];
                value[2 * t + 1] = Lh[2 * at + 1];
            }
        }
    }
}

}  // namespace aphi_b200

aphi_factor::~aphi_factor() {
    for (cudaEvent_t e : prof_events) cudaEventDestroy(e);
    void* ptrs[] = {L, dscale, rowmax, stats, dref, y, U, part, ir, red, norms, kr, err, kmax, hvals, hvec, tcws,
                    counters, dws};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}
