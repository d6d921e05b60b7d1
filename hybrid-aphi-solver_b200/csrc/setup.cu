// Per-mesh setup on the device: the sparsity pattern from the tets' DOF tables
// (build_sparsity, src/sparsity.cpp:19-136) and the scatter's maps -- each
// tet's term destinations in the scatter's emission order and their
// inversion into slot -> term lists (ScatterMap::build and its use by
// scatter_into, src/assembly.cpp:196-232, :255-422). Both are built once per
// mesh; in serving this is the cost of a cache miss.
//
// The outputs equal the host builders' exactly: a pattern row is the sorted,
// unique set of its columns, and a slot's term list is its terms in
// increasing term index -- so the order in which threads deposit entries
// (integer atomics) does not show in the result: every list is sorted after
// it is filled.
#include <algorithm>
#include <string>
#include <vector>

#include "assembly.hpp"
#include "common.cuh"
#include "setup.hpp"

namespace aphi_b200 {

namespace {

constexpr int kScanBlock = 1024;

// Exclusive scan, one block of kScanBlock entries: out[i] = sum in[0..i) of
// the block, sums[block] = the block's total.
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_block(const T* in, long long* out, long long* sums, long long n) {
    __shared__ long long sh[kScanBlock];
    const long long i = static_cast<long long>(blockIdx.x) * kScanBlock + threadIdx.x;
    const long long v = i < n ? static_cast<long long>(in[i]) : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        const long long add = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += add;
        __syncthreads();
    }
    if (i < n) out[i] = sh[threadIdx.x] - v;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void k_scan_add(long long* out, const long long* offsets, long long n) {
    const long long i = static_cast<long long>(blockIdx.x) * kScanBlock + threadIdx.x;
    if (i < n) out[i] += offsets[blockIdx.x];
}

struct DevBuf {
    std::vector<void*> p;
    template <class T>
    T* alloc(size_t n) {
        void* d = nullptr;
        APHI_CUDA(cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(T)));
        p.push_back(d);
        return static_cast<T*>(d);
    }
    ~DevBuf() {
        for (void* q : p) cudaFree(q);
    }
};

// out[0..n] = exclusive scan of in[0..n); out[n] = the total (returned).
template <class T>
long long scan_exclusive(const T* in, long long* out, long long n, cudaStream_t st) {
    if (n <= 0) {
        APHI_CUDA(cudaMemsetAsync(out, 0, sizeof(long long), st));
        return 0;
    }
    const long long nb = (n + kScanBlock - 1) / kScanBlock;
    DevBuf tmp;
    long long* sums = tmp.alloc<long long>(nb);
    k_scan_block<T><<<static_cast<unsigned>(nb), kScanBlock, 0, st>>>(in, out, sums, n);
    APHI_CHECK_LAUNCH();
    if (nb == 1) {
        APHI_CUDA(cudaMemcpyAsync(out + n, sums, sizeof(long long), cudaMemcpyDeviceToDevice, st));
    } else {
        long long* offs = tmp.alloc<long long>(nb + 1);
        scan_exclusive<long long>(sums, offs, nb, st);
        k_scan_add<<<static_cast<unsigned>(nb), kScanBlock, 0, st>>>(out, offs, n);
        APHI_CHECK_LAUNCH();
        APHI_CUDA(cudaMemcpyAsync(out + n, offs + nb, sizeof(long long), cudaMemcpyDeviceToDevice, st));
    }
    long long total = 0;
    APHI_CUDA(cudaMemcpyAsync(&total, out + n, sizeof(long long), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    return total;
}

// ---------------------------------------------------------------- pattern
// A tet's live DOFs, sorted and unique (several local DOFs may share one
// global index: a port terminal's nodes all read the port's unknown).
__device__ __forceinline__ int tet_live(const int* idx16, int (&live)[16]) {
    int n = 0;
    for (int q = 0; q < 16; ++q) {
        const int v = idx16[q];
        if (v < 0) continue;
        int at = n;
        while (at > 0 && live[at - 1] > v) {
            live[at] = live[at - 1];
            --at;
        }
        live[at] = v;
        ++n;
    }
    int u = 0;
    for (int q = 0; q < n; ++q)
        if (u == 0 || live[u - 1] != live[q]) live[u++] = live[q];
    return u;
}

__global__ void k_pattern_count(int T, int N, const int* tet_idx, int upper, int* count, int* err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    for (int q = 0; q < 16; ++q)
        if (tet_idx[16LL * t + q] >= N) {
            atomicExch(err, 1);  // refused by the host before anything is filled
            return;
        }
    int live[16];
    const int n = tet_live(tet_idx + 16LL * t, live);
    for (int i = 0; i < n; ++i) atomicAdd(&count[live[i]], upper ? n - i : n);
}

__global__ void k_pattern_diag_count(int nd, const int* rows, int* count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nd) atomicAdd(&count[rows[k]], 1);
}

__global__ void k_pattern_fill(int T, const int* tet_idx, int upper, const long long* raw_ptr, int* cursor,
                               int* raw_col) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    int live[16];
    const int n = tet_live(tet_idx + 16LL * t, live);
    for (int i = 0; i < n; ++i) {
        const int row = live[i];
        for (int j = upper ? i : 0; j < n; ++j) raw_col[raw_ptr[row] + atomicAdd(&cursor[row], 1)] = live[j];
    }
}

__global__ void k_pattern_diag_fill(int nd, const int* rows, const long long* raw_ptr, int* cursor, int* raw_col) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nd) raw_col[raw_ptr[rows[k]] + atomicAdd(&cursor[rows[k]], 1)] = rows[k];
}

// One warp per row: sort its raw columns and keep each value once, in place
// at the front of the row's raw slice; ucount[row] = unique count. Rows of
// up to kRowCap raw entries are rank-sorted in shared memory; a longer row
// (a port unknown read by many tets, full storage) is sorted in place by one
// thread.
constexpr int kRowCap = 1024;
constexpr int kSortWarps = 4;
__global__ void __launch_bounds__(32 * kSortWarps) k_pattern_sort_rows(int N, const long long* raw_ptr, int* raw_col,
                                                                       int* ucount) {
    __shared__ int sbuf[kSortWarps][2][kRowCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * kSortWarps + warp;
    if (row >= N) return;
    const long long b = raw_ptr[row];
    const int len = static_cast<int>(raw_ptr[row + 1] - b);
    int* col = raw_col + b;
    if (len > kRowCap) {
        if (lane == 0) {
            for (int i = 1; i < len; ++i) {
                const int v = col[i];
                int j = i;
                while (j > 0 && col[j - 1] > v) {
                    col[j] = col[j - 1];
                    --j;
                }
                col[j] = v;
            }
            int u = 0;
            for (int i = 0; i < len; ++i)
                if (u == 0 || col[u - 1] != col[i]) col[u++] = col[i];
            ucount[row] = u;
        }
        return;
    }
    int* s = sbuf[warp][0];
    int* t = sbuf[warp][1];
    for (int i = lane; i < len; i += 32) s[i] = col[i];
    __syncwarp();
    // Stable rank: entries smaller, plus equal entries before it.
    for (int i = lane; i < len; i += 32) {
        const int v = s[i];
        int r = 0;
        for (int k = 0; k < len; ++k) {
            const int u = s[k];
            r += (u < v) || (u == v && k < i);
        }
        t[r] = v;
    }
    __syncwarp();
    int written = 0;
    for (int i0 = 0; i0 < len; i0 += 32) {
        const int i = i0 + lane;
        const bool keep = i < len && (i == 0 || t[i] != t[i - 1]);
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (keep) col[written + __popc(mask & ((1u << lane) - 1u))] = t[i];
        written += __popc(mask);
    }
    if (lane == 0) ucount[row] = written;
}

__global__ void k_pattern_compact(int N, const long long* raw_ptr, const int* raw_col, const long long* row_ptr,
                                  int* col_idx) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * kSortWarps + warp;
    if (row >= N) return;
    const int len = static_cast<int>(row_ptr[row + 1] - row_ptr[row]);
    for (int i = lane; i < len; i += 32) col_idx[row_ptr[row] + i] = raw_col[raw_ptr[row] + i];
}

__global__ void k_to_int(long long n, const long long* in, int* out) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<int>(in[i]);
}

// ---------------------------------------------------------------- scatter maps
__device__ __forceinline__ int find_slot_dev(const int* row_ptr, const int* col_idx, int r, int c) {
    int lo = row_ptr[r], hi = row_ptr[r + 1];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (col_idx[mid] < c) lo = mid + 1; else hi = mid;
    }
    return (lo < row_ptr[r + 1] && col_idx[lo] == c) ? lo : -1;
}

// The scatter's terms of one tet in emission order (the same walk as
// k_tet_terms and assembly_create): emit(row, col), col < 0 for an rhs term.
template <class Emit>
__device__ void tet_term_walk(const int* idx, const double* fx, bool up, Emit emit) {
    auto nz = [&](int q) { return !(fx[2 * q] == 0.0 && fx[2 * q + 1] == 0.0); };
    bool need_phi = false;
    for (int q = 0; q < 10; ++q)
        if (idx[6 + q] >= 0 || nz(q)) need_phi = true;
    for (int p = 0; p < 6; ++p) {
        if (idx[p] < 0) continue;
        for (int q = 0; q < 6; ++q)
            if (idx[q] >= 0 && !(up && idx[q] < idx[p])) emit(idx[p], idx[q]);
    }
    if (!need_phi) return;
    for (int p = 0; p < 6; ++p) {
        if (idx[p] < 0) continue;
        for (int q = 0; q < 10; ++q) {
            const int col = idx[6 + q];
            if (col >= 0) {
                if (!(up && col < idx[p])) emit(idx[p], col);
            } else if (nz(q)) {
                emit(idx[p], -1);
            }
            if (col >= 0 && !(up && idx[p] < col)) emit(col, idx[p]);
        }
    }
    for (int p = 0; p < 10; ++p) {
        const int row = idx[6 + p];
        if (row < 0) continue;
        for (int q = 0; q < 10; ++q) {
            const int col = idx[6 + q];
            if (col >= 0) {
                if (!(up && col < row)) emit(row, col);
            } else if (nz(q)) {
                emit(row, -1);
            }
        }
    }
}

struct MapArgs {
    int T, N, nnz, up;
    const int* visit_tet;
    const int* tet_idx;
    const double* tet_fixed;
    const int* row_ptr;
    const int* col_idx;
    int* err;               // [0] index out of range, [1] missing slot; [2], [3] its row and column
};

__global__ void k_term_count(MapArgs a, int* count) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.T) return;
    const int t = a.visit_tet[v];
    if (t < 0 || t >= a.T) {
        atomicExch(&a.err[0], 1);
        count[v] = 0;
        return;
    }
    int idx[16];
    for (int q = 0; q < 16; ++q) {
        idx[q] = a.tet_idx[16LL * t + q];
        if (idx[q] >= a.N) atomicExch(&a.err[0], 1);
    }
    int n = 0;
    tet_term_walk(idx, a.tet_fixed + 20LL * t, a.up != 0, [&](int, int) { ++n; });
    count[v] = n;
}

__global__ void k_term_dest(MapArgs a, const long long* term_off, int* dest) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.T) return;
    const int t = a.visit_tet[v];
    if (t < 0 || t >= a.T) return;
    int idx[16];
    for (int q = 0; q < 16; ++q) idx[q] = min(a.tet_idx[16LL * t + q], a.N - 1);
    long long k = term_off[v];
    tet_term_walk(idx, a.tet_fixed + 20LL * t, a.up != 0, [&](int r, int c) {
        int d;
        if (c < 0) {
            d = a.nnz + r;
        } else {
            d = find_slot_dev(a.row_ptr, a.col_idx, r, c);
            if (d < 0) {
                if (atomicCAS(&a.err[1], 0, 1) == 0) {
                    a.err[2] = r;
                    a.err[3] = c;
                }
                d = 0;
            }
        }
        dest[k++] = d;
    });
}

__global__ void k_dest_count(long long nterms, const int* dest, int* count) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < nterms) atomicAdd(&count[dest[k]], 1);
}

__global__ void k_dest_fill(long long nterms, const int* dest, const long long* ptr, int* cursor, int* terms) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < nterms) terms[ptr[dest[k]] + atomicAdd(&cursor[dest[k]], 1)] = static_cast<int>(k);
}

// Each destination's terms in increasing term index (the reference's
// accumulation order); lists are short, one thread sorts one.
__global__ void k_dest_sort(int ndest, const long long* ptr, int* terms) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ndest) return;
    const long long b = ptr[d], e = ptr[d + 1];
    for (long long i = b + 1; i < e; ++i) {
        const int v = terms[i];
        long long j = i;
        while (j > b && terms[j - 1] > v) {
            terms[j] = terms[j - 1];
            --j;
        }
        terms[j] = v;
    }
}

template <class T>
T* upload_to(DevBuf& buf, const T* h, size_t n, cudaStream_t st) {
    T* d = buf.alloc<T>(n);
    if (n) APHI_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return d;
}

}  // namespace

long long pattern_build(int N, int T, const int* tet_idx, int nd, const int* diag_rows, bool upper, int* row_ptr,
                        int* col_idx, long long capacity) {
    if (N < 0 || T < 0 || nd < 0) throw Error(APHI_ERR_BAD_SHAPE, "build_sparsity: negative size");
    for (int k = 0; k < nd; ++k)
        if (diag_rows[k] < 0 || diag_rows[k] >= N) throw Error(APHI_ERR_BAD_SHAPE, "build_sparsity: a port row lies outside the unknowns");
    cudaStream_t st = nullptr;
    DevBuf buf;
    const int* d_idx = upload_to(buf, tet_idx, 16 * static_cast<size_t>(T), st);
    const int* d_diag = upload_to(buf, diag_rows, static_cast<size_t>(nd), st);
    int* count = buf.alloc<int>(static_cast<size_t>(N) + 1);
    int* err = buf.alloc<int>(4);
    APHI_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (static_cast<size_t>(N) + 1), st));
    APHI_CUDA(cudaMemsetAsync(err, 0, sizeof(int) * 4, st));
    if (T > 0) {
        k_pattern_count<<<ceil_div(T, 256), 256, 0, st>>>(T, N, d_idx, upper ? 1 : 0, count, err);
        APHI_CHECK_LAUNCH();
    }
    if (nd > 0) {
        k_pattern_diag_count<<<ceil_div(nd, 256), 256, 0, st>>>(nd, d_diag, count);
        APHI_CHECK_LAUNCH();
    }
    int herr[4];
    APHI_CUDA(cudaMemcpyAsync(herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    if (herr[0]) throw Error(APHI_ERR_BAD_SHAPE, "build_sparsity: a DOF index exceeds the unknowns");
    long long* raw_ptr = buf.alloc<long long>(static_cast<size_t>(N) + 1);
    const long long raw = scan_exclusive<int>(count, raw_ptr, N, st);
    int* raw_col = buf.alloc<int>(static_cast<size_t>(raw));
    APHI_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (static_cast<size_t>(N) + 1), st));  // cursors
    if (T > 0) {
        k_pattern_fill<<<ceil_div(T, 256), 256, 0, st>>>(T, d_idx, upper ? 1 : 0, raw_ptr, count, raw_col);
        APHI_CHECK_LAUNCH();
    }
    if (nd > 0) {
        k_pattern_diag_fill<<<ceil_div(nd, 256), 256, 0, st>>>(nd, d_diag, raw_ptr, count, raw_col);
        APHI_CHECK_LAUNCH();
    }
    if (N > 0) {
        k_pattern_sort_rows<<<ceil_div(N, kSortWarps), 32 * kSortWarps, 0, st>>>(N, raw_ptr, raw_col, count);
        APHI_CHECK_LAUNCH();
    }
    long long* ptr = buf.alloc<long long>(static_cast<size_t>(N) + 1);
    const long long nnz = scan_exclusive<int>(count, ptr, N, st);
    if (nnz >= (1LL << 31)) throw Error(APHI_ERR_BAD_SHAPE, "build_sparsity: more than 2^31 entries");
    if (nnz > capacity || !col_idx) return nnz;
    int* d_col = buf.alloc<int>(static_cast<size_t>(nnz));
    int* d_rp = buf.alloc<int>(static_cast<size_t>(N) + 1);
    if (N > 0) {
        k_pattern_compact<<<ceil_div(N, kSortWarps), 32 * kSortWarps, 0, st>>>(N, raw_ptr, raw_col, ptr, d_col);
        APHI_CHECK_LAUNCH();
    }
    k_to_int<<<ceil_div(N + 1LL, 256), 256, 0, st>>>(N + 1LL, ptr, d_rp);
    APHI_CHECK_LAUNCH();
    APHI_CUDA(cudaMemcpyAsync(row_ptr, d_rp, sizeof(int) * (static_cast<size_t>(N) + 1), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaMemcpyAsync(col_idx, d_col, sizeof(int) * static_cast<size_t>(nnz), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    return nnz;
}

void assembly_maps_on_device(Assembly& A, const aphi_assembly_desc& d, const int* visit_tet_host) {
    cudaStream_t st = nullptr;
    const int T = A.T, N = A.N, nnz = A.nnz;
    DevBuf buf;
    const int* d_rp = upload_to(buf, d.row_ptr, static_cast<size_t>(N) + 1, st);
    const int* d_ci = upload_to(buf, d.col_idx, static_cast<size_t>(nnz), st);
    const int* d_visit = upload_to(buf, visit_tet_host, static_cast<size_t>(T), st);
    int* err = buf.alloc<int>(4);
    int* count = buf.alloc<int>(std::max<size_t>(static_cast<size_t>(T), static_cast<size_t>(nnz) + N) + 1);
    APHI_CUDA(cudaMemsetAsync(err, 0, sizeof(int) * 4, st));
    MapArgs ma{T, N, nnz, A.upper_only ? 1 : 0, d_visit, A.d_tet_idx, A.d_tet_fixed, d_rp, d_ci, err};
    if (T > 0) {
        k_term_count<<<ceil_div(T, 256), 256, 0, st>>>(ma, count);
        APHI_CHECK_LAUNCH();
    }
    APHI_CUDA(cudaMalloc(&A.d_term_off, sizeof(long long) * (static_cast<size_t>(T) + 1)));
    const long long tet_terms = scan_exclusive<int>(count, A.d_term_off, T, st);
    int herr[4];
    APHI_CUDA(cudaMemcpyAsync(herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    if (herr[0]) throw Error(APHI_ERR_BAD_SHAPE, "refill: a DOF index or a body tet index is out of range");
    // Port terms after the tets', as assembly_create places them.
    std::vector<int> port_dest;
    auto slot_host = [&](int r, int c) {
        const int* b = d.col_idx + d.row_ptr[r];
        const int* e = d.col_idx + d.row_ptr[r + 1];
        const int* it = std::lower_bound(b, e, c);
        if (it == e || *it != c)
            throw Error(APHI_ERR_PATTERN_MISMATCH,
                        "assemble: no slot for entry (" + std::to_string(r) + ", " + std::to_string(c) + ")");
        return static_cast<int>(it - d.col_idx);
    };
    for (int p = 0; p < d.num_ports; ++p) {
        if (d.port_current[p]) {
            port_dest.push_back(nnz + d.port_row[p]);
        } else {
            port_dest.push_back(slot_host(d.port_row[p], d.port_row[p]));
            port_dest.push_back(nnz + d.port_row[p]);
        }
    }
    const long long nterms = tet_terms + static_cast<long long>(port_dest.size());
    if (nterms >= (1LL << 31)) throw Error(APHI_ERR_BAD_SHAPE, "refill: more than 2^31 element terms");
    int* dest = buf.alloc<int>(static_cast<size_t>(nterms));
    if (T > 0) {
        k_term_dest<<<ceil_div(T, 256), 256, 0, st>>>(ma, A.d_term_off, dest);
        APHI_CHECK_LAUNCH();
    }
    if (!port_dest.empty())
        APHI_CUDA(cudaMemcpyAsync(dest + tet_terms, port_dest.data(), sizeof(int) * port_dest.size(),
                                  cudaMemcpyHostToDevice, st));
    APHI_CUDA(cudaMemcpyAsync(herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    if (herr[1])
        throw Error(APHI_ERR_PATTERN_MISMATCH,
                    "assemble: no slot for entry (" + std::to_string(herr[2]) + ", " + std::to_string(herr[3]) +
                        "). The sparsity pattern and the scatter disagree about the matrix's shape; dropping the "
                        "term would give a quietly wrong matrix.");
    // Slot -> term lists, in increasing term order.
    const int ndest = nnz + N;
    APHI_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (static_cast<size_t>(ndest) + 1), st));
    if (nterms > 0) {
        k_dest_count<<<ceil_div(nterms, 256), 256, 0, st>>>(nterms, dest, count);
        APHI_CHECK_LAUNCH();
    }
    long long* ptr = buf.alloc<long long>(static_cast<size_t>(ndest) + 1);
    scan_exclusive<int>(count, ptr, ndest, st);
    APHI_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (static_cast<size_t>(ndest) + 1), st));
    APHI_CUDA(cudaMalloc(&A.d_dest_terms, sizeof(int) * std::max<long long>(nterms, 1)));
    if (nterms > 0) {
        k_dest_fill<<<ceil_div(nterms, 256), 256, 0, st>>>(nterms, dest, ptr, count, A.d_dest_terms);
        APHI_CHECK_LAUNCH();
    }
    if (ndest > 0) {
        k_dest_sort<<<ceil_div(ndest, 256), 256, 0, st>>>(ndest, ptr, A.d_dest_terms);
        APHI_CHECK_LAUNCH();
    }
    APHI_CUDA(cudaMalloc(&A.d_dest_ptr, sizeof(int) * (static_cast<size_t>(ndest) + 1)));
    k_to_int<<<ceil_div(ndest + 1LL, 256), 256, 0, st>>>(ndest + 1LL, ptr, A.d_dest_ptr);
    APHI_CHECK_LAUNCH();
    APHI_CUDA(cudaStreamSynchronize(st));
    A.tet_terms = tet_terms;
    A.num_terms = nterms;
}

}  // namespace aphi_b200
