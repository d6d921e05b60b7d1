// Device solves with a factor held only as host CSC arrays, and device
// residual measures of a matrix held only as host CSR arrays: the drop-in
// layer's paths for a SymmetricFactor that its own factorize_ldlt did not
// produce (one built by hand, or modified since), and for relative_residual /
// backward_error on a bare SparseSymmetricZ. Nothing of the numeric work runs
// on the host; the host only derives the level schedule from the pattern.
//
// Reference: solve_in_place, src/factorization.cpp:254-294 (forward by
// columns of L, scale by D, backward by columns of L^T, no conjugation);
// relative_residual :315-329, backward_error :401-416 and
// SparseSymmetric::matvec, include/aphi_solver/sparse_symmetric.hpp:120-136.
//
// Forward: y_r = b_r - sum_i L(r, i) y_i. The reference subtracts column j's
// contributions from y_r in increasing j; here one thread per row r walks
// row r of L (the CSC transposed on the host, in increasing column order)
// and subtracts in that same order, so every y_r is rounded exactly as the
// reference rounds it. Rows are grouped into levels (a row waits for the
// rows it reads); one launch per level. Backward: x_j = z_j - sum_i L(i, j)
// x_i over column j in increasing row order, as the reference's loop, one
// thread per column, levels from the last column down. This file is compiled
// without FMA contraction, like the host arithmetic it reproduces.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace aphi_b200 {

namespace {

struct Csc {
    int n;
    const int* col_ptr;    // L strictly lower, by columns (row indices ascending)
    const int* row_index;
    const cplx* value;
    const int* row_ptr;    // the same entries by rows (columns ascending)
    const int* row_col;
    const int* row_pos;    // position of each row entry in value[]
    const cplx* diag;
};

// One rhs per grid.y; y is rhs-major (y + n * k).
__global__ void k_csc_forward(Csc L, const int* rows, int count, cplx* y) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int r = rows[t];
    cplx* yk = y + static_cast<long long>(L.n) * blockIdx.y;
    cplx s = yk[r];
    for (int e = L.row_ptr[r]; e < L.row_ptr[r + 1]; ++e) s = csub(s, cmul(L.value[L.row_pos[e]], yk[L.row_col[e]]));
    yk[r] = s;
}

// y_j / D_j (Smith's ordering for finite operands of ordinary magnitude).
__global__ void k_csc_diag(int n, const cplx* d, cplx* y) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    cplx* yk = y + static_cast<long long>(n) * blockIdx.y;
    const cplx a = yk[j], b = d[j];
    if (fabs(b.re) < fabs(b.im)) {
        const double ratio = b.re / b.im;
        const double den = b.re * ratio + b.im;
        yk[j] = cplx{(a.re * ratio + a.im) / den, (a.im * ratio - a.re) / den};
    } else {
        const double ratio = b.im / b.re;
        const double den = b.re + b.im * ratio;
        yk[j] = cplx{(a.re + a.im * ratio) / den, (a.im - a.re * ratio) / den};
    }
}

__global__ void k_csc_backward(Csc L, const int* cols, int count, cplx* y) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int j = cols[t];
    cplx* yk = y + static_cast<long long>(L.n) * blockIdx.y;
    cplx s = yk[j];
    for (int e = L.col_ptr[j]; e < L.col_ptr[j + 1]; ++e) s = csub(s, cmul(L.value[e], yk[L.row_index[e]]));
    yk[j] = s;
}

template <class T>
T* to_device(const T* h, size_t n, std::vector<void*>& owned) {
    T* d = nullptr;
    APHI_CUDA(cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(T)));
    owned.push_back(d);
    if (n) APHI_CUDA(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

struct Owned {
    std::vector<void*> p;
    ~Owned() {
        for (void* q : p) cudaFree(q);
    }
};

}  // namespace

void csc_solve_host(int n, const int* col_ptr, const int* row_index, const double* value, const double* diagonal,
                    int nrhs, double* y) {
    if (n < 0 || nrhs < 1) throw Error(APHI_ERR_BAD_SHAPE, "solve_in_place: n must be >= 0 and nrhs >= 1");
    if (n == 0) return;
    if (col_ptr[0] != 0) throw Error(APHI_ERR_BAD_SHAPE, "solve_in_place: col_ptr must start at 0");
    const int nl = col_ptr[n];
    for (int j = 0; j < n; ++j) {
        if (col_ptr[j + 1] < col_ptr[j]) throw Error(APHI_ERR_BAD_SHAPE, "solve_in_place: col_ptr decreases");
        for (int e = col_ptr[j]; e < col_ptr[j + 1]; ++e)
            if (row_index[e] <= j || row_index[e] >= n)
                throw Error(APHI_ERR_BAD_SHAPE, "solve_in_place: a row index of column " + std::to_string(j) +
                                                    " is not strictly below the diagonal");
        if (diagonal[2 * j] == 0.0 && diagonal[2 * j + 1] == 0.0)
            throw Error(APHI_ERR_ZERO_PIVOT, "solve_in_place: D[" + std::to_string(j) +
                                                 "] is zero; this factor did not come from a completed "
                                                 "factorize_ldlt");
    }
    // The same entries by rows, columns ascending (a stable transpose).
    std::vector<int> rp(static_cast<size_t>(n) + 1, 0), rc(nl), rpos(nl);
    for (int e = 0; e < nl; ++e) ++rp[row_index[e] + 1];
    for (int i = 0; i < n; ++i) rp[i + 1] += rp[i];
    {
        std::vector<int> cur(rp.begin(), rp.end() - 1);
        for (int j = 0; j < n; ++j)
            for (int e = col_ptr[j]; e < col_ptr[j + 1]; ++e) {
                const int r = row_index[e];
                rc[cur[r]] = j;
                rpos[cur[r]++] = e;
            }
    }
    // Levels: forward, a row after every row it reads; backward, a column
    // after every column whose unknown it reads (rows below it).
    std::vector<int> lf(n, 0), lb(n, 0);
    int nf = 0, nbk = 0;
    for (int r = 0; r < n; ++r) {
        for (int e = rp[r]; e < rp[r + 1]; ++e) lf[r] = std::max(lf[r], lf[rc[e]] + 1);
        nf = std::max(nf, lf[r] + 1);
    }
    for (int j = n - 1; j >= 0; --j) {
        for (int e = col_ptr[j]; e < col_ptr[j + 1]; ++e) lb[j] = std::max(lb[j], lb[row_index[e]] + 1);
        nbk = std::max(nbk, lb[j] + 1);
    }
    auto bucket = [n](const std::vector<int>& lev, int count, std::vector<int>& ptr, std::vector<int>& list) {
        ptr.assign(static_cast<size_t>(count) + 1, 0);
        for (int i = 0; i < n; ++i) ++ptr[lev[i] + 1];
        for (int l = 0; l < count; ++l) ptr[l + 1] += ptr[l];
        list.resize(n);
        std::vector<int> cur(ptr.begin(), ptr.end() - 1);
        for (int i = 0; i < n; ++i) list[cur[lev[i]]++] = i;
    };
    std::vector<int> fptr, flist, bptr, blist;
    bucket(lf, nf, fptr, flist);
    bucket(lb, nbk, bptr, blist);

    Owned own;
    Csc L{n,
          to_device(col_ptr, static_cast<size_t>(n) + 1, own.p),
          to_device(row_index, static_cast<size_t>(nl), own.p),
          reinterpret_cast<const cplx*>(to_device(value, 2 * static_cast<size_t>(nl), own.p)),
          to_device(rp.data(), rp.size(), own.p),
          to_device(rc.data(), rc.size(), own.p),
          to_device(rpos.data(), rpos.size(), own.p),
          reinterpret_cast<const cplx*>(to_device(diagonal, 2 * static_cast<size_t>(n), own.p))};
    const int* d_flist = to_device(flist.data(), flist.size(), own.p);
    const int* d_blist = to_device(blist.data(), blist.size(), own.p);
    cplx* d_y = reinterpret_cast<cplx*>(to_device(y, 2 * static_cast<size_t>(n) * nrhs, own.p));
    for (int l = 0; l < nf; ++l) {
        const int cnt = fptr[l + 1] - fptr[l];
        k_csc_forward<<<dim3(ceil_div(cnt, 128), nrhs), 128>>>(L, d_flist + fptr[l], cnt, d_y);
        APHI_CHECK_LAUNCH();
    }
    k_csc_diag<<<dim3(ceil_div(n, 256), nrhs), 256>>>(n, L.diag, d_y);
    APHI_CHECK_LAUNCH();
    for (int l = 0; l < nbk; ++l) {
        const int cnt = bptr[l + 1] - bptr[l];
        k_csc_backward<<<dim3(ceil_div(cnt, 128), nrhs), 128>>>(L, d_blist + bptr[l], cnt, d_y);
        APHI_CHECK_LAUNCH();
    }
    APHI_CUDA(cudaMemcpy(y, d_y, sizeof(double) * 2 * static_cast<size_t>(n) * nrhs, cudaMemcpyDeviceToHost));
}

}  // namespace aphi_b200
