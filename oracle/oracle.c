/*
 * The oracle -- test infrastructure only (see oracle.h). A plain-C
 * restatement of the reference's algorithms for the per-frequency numeric
 * path, operation for operation, so that where the reference is deterministic
 * this is too and the two agree bit for bit. Each function cites the
 * reference code it restates.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cz;

static cz ld(const double* p) { return CMPLX(p[0], p[1]); }
static void st(double* p, cz v) {
    p[0] = creal(v);
    p[1] = cimag(v);
}
/* complex x real, as std::complex<double>::operator*(double): both parts scaled. */
static cz scl(cz a, double s) { return CMPLX(creal(a) * s, cimag(a) * s); }
static cz addc(cz a, cz b) { return CMPLX(creal(a) + creal(b), cimag(a) + cimag(b)); }
static cz subc(cz a, cz b) { return CMPLX(creal(a) - creal(b), cimag(a) - cimag(b)); }

/* include/aphi_solver/constants.hpp:12-13 */
static const double kMu0 = 4.0e-7 * 3.14159265358979323846;
static const double kEps0 = 8.8541878128e-12;
/* include/aphi_solver/mesh.hpp:44-51 */
static const int kEdge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {2, 3}, {1, 3}};

/* src/element_matrix.cpp:10-25 */
void or_coefficients(double sigma, double eps_r, double mu_r, double omega, double* out) {
    const double mu = mu_r * kMu0;
    const double eps = eps_r * kEps0;
    out[0] = 1.0 / mu;
    out[1] = -omega * omega * eps;
    out[2] = omega * sigma;
    out[3] = sigma;
    out[4] = omega * eps;
}

/* compute_tet_geometry, src/basis_functions.cpp:15-85: Gauss-Jordan inverse of
 * [1 x y z] with partial pivoting; grad(L_i) is column i of rows 1..3. */
static int geometry(const double* p, double g[4][3], double* volume) {
    double m[4][4], inv[4][4];
    for (int r = 0; r < 4; ++r) {
        m[r][0] = 1.0;
        m[r][1] = p[3 * r];
        m[r][2] = p[3 * r + 1];
        m[r][3] = p[3 * r + 2];
        for (int c = 0; c < 4; ++c) inv[r][c] = r == c ? 1.0 : 0.0;
    }
    for (int col = 0; col < 4; ++col) {
        int pr = col;
        double pv = fabs(m[col][col]);
        for (int r = col + 1; r < 4; ++r)
            if (fabs(m[r][col]) > pv) {
                pr = r;
                pv = fabs(m[r][col]);
            }
        if (pv < 1e-14) return -1;
        if (pr != col)
            for (int c = 0; c < 4; ++c) {
                double t = m[pr][c];
                m[pr][c] = m[col][c];
                m[col][c] = t;
                t = inv[pr][c];
                inv[pr][c] = inv[col][c];
                inv[col][c] = t;
            }
        const double piv = m[col][col];
        for (int c = 0; c < 4; ++c) {
            m[col][c] /= piv;
            inv[col][c] /= piv;
        }
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            const double f = m[r][col];
            if (f == 0.0) continue;
            for (int c = 0; c < 4; ++c) {
                m[r][c] -= f * m[col][c];
                inv[r][c] -= f * inv[col][c];
            }
        }
    }
    for (int i = 0; i < 4; ++i) {
        g[i][0] = inv[1][i];
        g[i][1] = inv[2][i];
        g[i][2] = inv[3][i];
    }
    /* Mesh::signed_tet_volume, src/mesh.cpp:141-151 */
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = p[3 + k] - p[k];
        b[k] = p[6 + k] - p[k];
        c[k] = p[9 + k] - p[k];
    }
    const double x = a[1] * b[2] - a[2] * b[1];
    const double y = a[2] * b[0] - a[0] * b[2];
    const double z = a[0] * b[1] - a[1] * b[0];
    *volume = fabs((x * c[0] + y * c[1] + z * c[2]) / 6.0);
    return 0;
}

static double dot(const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }

/* whitney_edge_value, src/basis_functions.cpp:95-99 */
static void whitney(double g[4][3], int e, const double* L, double* out) {
    const int i = kEdge[e][0], j = kEdge[e][1];
    for (int k = 0; k < 3; ++k) out[k] = g[j][k] * L[i] - g[i][k] * L[j];
}

/* p2_nodal_gradient, src/basis_functions.cpp:126-137 */
static void p2grad(double g[4][3], int b, const double* L, double* out) {
    if (b < 4) {
        const double s = 4.0 * L[b] - 1.0;
        for (int k = 0; k < 3; ++k) out[k] = g[b][k] * s;
        return;
    }
    const int v0 = kEdge[b - 4][0], v1 = kEdge[b - 4][1];
    const double s0 = 4.0 * L[v1], s1 = 4.0 * L[v0];
    for (int k = 0; k < 3; ++k) out[k] = g[v0][k] * s0 + g[v1][k] * s1;
}

/* kernel_AA, kernel_APhi, kernel_PhiPhi -- src/element_matrix.cpp:27-115 --
 * with the degree-2 rule of src/quadrature.cpp:16-35. */
static void blocks(double g[4][3], double volume, double nu, cz alpha, cz beta, cz* aa, cz* ap, cz* pp) {
    double curl[6][3];
    for (int e = 0; e < 6; ++e) {
        const double* u = g[kEdge[e][0]];
        const double* v = g[kEdge[e][1]];
        curl[e][0] = (u[1] * v[2] - u[2] * v[1]) * 2.0;
        curl[e][1] = (u[2] * v[0] - u[0] * v[2]) * 2.0;
        curl[e][2] = (u[0] * v[1] - u[1] * v[0]) * 2.0;
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) aa[i * 6 + j] = CMPLX(nu * volume * dot(curl[i], curl[j]), 0.0);
    for (int i = 0; i < 60; ++i) ap[i] = CMPLX(0.0, 0.0);
    for (int i = 0; i < 100; ++i) pp[i] = CMPLX(0.0, 0.0);
    const double s5 = sqrt(5.0);
    const double qa = (5.0 + 3.0 * s5) / 20.0, qb = (5.0 - s5) / 20.0;
    const int mass = !(creal(alpha) == 0.0 && cimag(alpha) == 0.0);
    const int coupling = !(creal(beta) == 0.0 && cimag(beta) == 0.0);
    for (int k = 0; k < 4; ++k) {
        double L[4];
        for (int i = 0; i < 4; ++i) L[i] = i == k ? qa : qb;
        const double w = 0.25 * volume;
        double wv[6][3];
        for (int e = 0; e < 6; ++e) whitney(g, e, L, wv[e]);
        if (mass)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) aa[i * 6 + j] = addc(aa[i * 6 + j], scl(alpha, w * dot(wv[i], wv[j])));
        if (coupling) {
            double gr[10][3];
            for (int b = 0; b < 10; ++b) p2grad(g, b, L, gr[b]);
            for (int i = 0; i < 6; ++i)
                for (int b = 0; b < 10; ++b) ap[i * 10 + b] = addc(ap[i * 10 + b], scl(beta, w * dot(wv[i], gr[b])));
            for (int a = 0; a < 10; ++a)
                for (int b = 0; b < 10; ++b) pp[a * 10 + b] = addc(pp[a * 10 + b], scl(beta, w * dot(gr[a], gr[b])));
        }
    }
}

int or_element_blocks(const double* xyz, double nu, const double* alpha, const double* beta, double* aa,
                      double* ap, double* pp) {
    double g[4][3], vol;
    if (geometry(xyz, g, &vol)) return -1;
    cz a[36], b[60], c[100];
    blocks(g, vol, nu, ld(alpha), ld(beta), a, b, c);
    for (int i = 0; i < 36; ++i) st(aa + 2 * i, a[i]);
    for (int i = 0; i < 60; ++i) st(ap + 2 * i, b[i]);
    for (int i = 0; i < 100; ++i) st(pp + 2 * i, c[i]);
    return 0;
}

/* src/assembly.cpp:12-45 */
int or_formulation_scales(int cond, double omega, double* rc) {
    cz r = CMPLX(1.0, 0.0), c = CMPLX(1.0, 0.0);
    const cz jw = CMPLX(0.0, omega);
    if (cond == 1) {
        if (omega == 0.0) return -1;
        r = CMPLX(1.0, 0.0) / jw;
    } else if (cond == 2) {
        if (omega == 0.0) return -1;
        c = jw;
    } else if (cond != 0) {
        return -1;
    }
    st(rc, r);
    st(rc + 2, c);
    return 0;
}

static int find_slot(const int* row_ptr, const int* col_idx, int r, int c) {
    int lo = row_ptr[r], hi = row_ptr[r + 1];
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (col_idx[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return (lo < row_ptr[r + 1] && col_idx[lo] == c) ? lo : -1;
}

/* scatter_into, src/assembly.cpp:255-422, symmetric storage: a pair below the
 * diagonal has no slot (its mirror is written by the transposed term). */
int or_refill(int num_tets, const double* xyz, const int* tets, const int* tet_idx, const double* tet_coeff,
              const double* tet_fixed, int num_bodies, const double* material, const int* body_ptr,
              const int* body_tets, int num_ports, const int* port_current, const int* port_row,
              const double* port_amplitude, const double* port_value, int n, const int* row_ptr,
              const int* col_idx, double omega, int cond, double* values, double* rhs) {
    (void)num_tets;
    double sc[4];
    if (cond != 1 && cond != 2) return -1; /* symmetric storage needs a symmetric conditioning */
    if (or_formulation_scales(cond, omega, sc)) return -1;
    const cz row = ld(sc), column = ld(sc + 2), jw = CMPLX(0.0, omega);
    cz* V = (cz*)calloc((size_t)row_ptr[n] + 1, sizeof(cz));
    cz* B = (cz*)calloc((size_t)n + 1, sizeof(cz));
    int rc = 0;
    for (int body = 0; body < num_bodies && !rc; ++body) {
        double co[5];
        or_coefficients(material[3 * body], material[3 * body + 1], material[3 * body + 2], omega, co);
        const double nu = co[0];
        const cz alpha = CMPLX(co[1], co[2]), beta = CMPLX(co[3], co[4]);
        for (int v = body_ptr[body]; v < body_ptr[body + 1] && !rc; ++v) {
            const int t = body_tets[v];
            double p[12];
            for (int q = 0; q < 4; ++q)
                for (int k = 0; k < 3; ++k) p[3 * q + k] = xyz[3 * tets[4 * t + q] + k];
            double g[4][3], vol;
            if (geometry(p, g, &vol)) {
                rc = -3;
                break;
            }
            cz aa[36], ap[60], pp[100];
            blocks(g, vol, nu, alpha, beta, aa, ap, pp);
            const int* idx = tet_idx + 16 * t;
            const double* cf = tet_coeff + 16 * t;
            const double* fx = tet_fixed + 20 * t;
#define SLOT(r_, c_)                                                \
    s_ = find_slot(row_ptr, col_idx, (r_), (c_));                   \
    if (s_ < 0) {                                                   \
        rc = -2;                                                    \
        goto done;                                                  \
    }
            int s_;
            for (int pi = 0; pi < 6; ++pi) {
                if (idx[pi] < 0) continue;
                for (int qi = 0; qi < 6; ++qi) {
                    if (idx[qi] < 0 || idx[qi] < idx[pi]) continue;
                    SLOT(idx[pi], idx[qi]);
                    V[s_] = addc(V[s_], scl(aa[pi * 6 + qi], cf[pi] * cf[qi]));
                }
            }
            for (int pi = 0; pi < 6; ++pi) {
                if (idx[pi] < 0) continue;
                for (int qi = 0; qi < 10; ++qi) {
                    const int col = idx[6 + qi];
                    const cz blk = ap[pi * 10 + qi];
                    if (col >= 0) {
                        if (col >= idx[pi]) {
                            SLOT(idx[pi], col);
                            V[s_] = addc(V[s_], scl(column, cf[pi] * cf[6 + qi]) * blk);
                        }
                    } else {
                        const cz given = ld(fx + 2 * qi);
                        const cz fixed = (given == 0.0) ? given : given / column;
                        if (fixed != 0.0) B[idx[pi]] = subc(B[idx[pi]], scl(column, cf[pi]) * blk * fixed);
                    }
                    if (col >= 0 && idx[pi] >= col) {
                        SLOT(col, idx[pi]);
                        V[s_] = addc(V[s_], scl(row * jw, cf[6 + qi] * cf[pi]) * blk);
                    }
                }
            }
            for (int pi = 0; pi < 10; ++pi) {
                const int r = idx[6 + pi];
                if (r < 0) continue;
                for (int qi = 0; qi < 10; ++qi) {
                    const int col = idx[6 + qi];
                    const cz blk = pp[pi * 10 + qi];
                    if (col >= 0) {
                        if (col >= r) {
                            SLOT(r, col);
                            V[s_] = addc(V[s_], scl(row * column, cf[6 + pi] * cf[6 + qi]) * blk);
                        }
                    } else {
                        const cz given = ld(fx + 2 * qi);
                        const cz fixed = (given == 0.0) ? given : given / column;
                        if (fixed != 0.0) B[r] = subc(B[r], scl(row * column, cf[6 + pi]) * blk * fixed);
                    }
                }
            }
#undef SLOT
        }
    }
    if (!rc) {
        for (int k = 0; k < num_ports; ++k) {
            const int r = port_row[k];
            if (port_current[k]) {
                B[r] = addc(B[r], row * ld(port_amplitude + 2 * k));
            } else {
                const int s = find_slot(row_ptr, col_idx, r, r);
                if (s < 0) {
                    rc = -2;
                    break;
                }
                V[s] = addc(V[s], CMPLX(1.0, 0.0));
                B[r] = addc(B[r], ld(port_value + 2 * k) / column);
            }
        }
    }
done:
    if (!rc) {
        for (int k = 0; k < row_ptr[n]; ++k) st(values + 2 * k, V[k]);
        for (int i = 0; i < n; ++i) st(rhs + 2 * i, B[i]);
    }
    free(V);
    free(B);
    return rc;
}

/* compute_symmetric_equilibration(SparseSymmetricZ), src/equilibration.cpp:94-139 */
void or_equilibration(int n, const int* row_ptr, const int* col_idx, const double* values, int iterations,
                      double* d) {
    const int nnz = row_ptr[n];
    cz* w = (cz*)malloc(((size_t)nnz + 1) * sizeof(cz));
    double* mx = (double*)malloc(((size_t)n + 1) * sizeof(double));
    double* f = (double*)malloc(((size_t)n + 1) * sizeof(double));
    for (int k = 0; k < nnz; ++k) w[k] = ld(values + 2 * k);
    for (int i = 0; i < n; ++i) d[i] = 1.0;
    for (int it = 0; it < iterations; ++it) {
        for (int i = 0; i < n; ++i) mx[i] = 0.0;
        for (int i = 0; i < n; ++i)
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                const int j = col_idx[k];
                const double m = cabs(w[k]);
                if (m > mx[i]) mx[i] = m;
                if (m > mx[j]) mx[j] = m;
            }
        for (int i = 0; i < n; ++i) {
            f[i] = mx[i] > 0.0 ? 1.0 / sqrt(mx[i]) : 1.0;
            d[i] *= f[i];
        }
        for (int i = 0; i < n; ++i)
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) w[k] = scl(w[k], f[i] * f[col_idx[k]]);
    }
    free(w);
    free(mx);
    free(f);
}

/* permuted_lower (src/factorization.cpp:13-74): P A P^T's lower triangle as
 * CSR, each row ascending. */
static void permuted_lower(int n, const int* row_ptr, const int* col_idx, const cz* values, const int* iperm,
                           int** lp, int** lc, cz** lv) {
    const int nnz = row_ptr[n];
    int* ptr = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            int a = iperm[r], b = iperm[col_idx[k]];
            ++ptr[(a > b ? a : b) + 1];
        }
    for (int r = 0; r < n; ++r) ptr[r + 1] += ptr[r];
    int* cur = (int*)malloc(((size_t)n + 1) * sizeof(int));
    memcpy(cur, ptr, sizeof(int) * (size_t)n);
    int* col = (int*)malloc(((size_t)nnz + 1) * sizeof(int));
    cz* val = (cz*)malloc(((size_t)nnz + 1) * sizeof(cz));
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            int a = iperm[r], b = iperm[col_idx[k]];
            const int row = a > b ? a : b, c = a > b ? b : a;
            col[cur[row]] = c;
            val[cur[row]++] = values[k];
        }
    /* insertion sort per row (columns are distinct) */
    for (int r = 0; r < n; ++r)
        for (int i = ptr[r] + 1; i < ptr[r + 1]; ++i) {
            const int c = col[i];
            const cz v = val[i];
            int j = i - 1;
            while (j >= ptr[r] && col[j] > c) {
                col[j + 1] = col[j];
                val[j + 1] = val[j];
                --j;
            }
            col[j + 1] = c;
            val[j + 1] = v;
        }
    free(cur);
    *lp = ptr;
    *lc = col;
    *lv = val;
}

/* factorize_ldlt, src/factorization.cpp:109-218; ereach :86-105. */
int or_factorize(int n, const int* row_ptr, const int* col_idx, const double* values, const int* perm,
                 const int* parent, const int* col_count, double pivot_floor, int* col_ptr, int* row_index,
                 double* lvalue, double* diag, double* stats) {
    const int nnz = row_ptr[n];
    cz* v = (cz*)malloc(((size_t)nnz + 1) * sizeof(cz));
    for (int k = 0; k < nnz; ++k) v[k] = ld(values + 2 * k);
    int* iperm = (int*)malloc(((size_t)n + 1) * sizeof(int));
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    int *lp, *lc;
    cz* lv;
    permuted_lower(n, row_ptr, col_idx, v, iperm, &lp, &lc, &lv);
    col_ptr[0] = 0;
    for (int j = 0; j < n; ++j) col_ptr[j + 1] = col_ptr[j] + (col_count[j] > 1 ? col_count[j] - 1 : 0);
    cz* L = (cz*)calloc((size_t)col_ptr[n] + 1, sizeof(cz));
    cz* D = (cz*)calloc((size_t)n + 1, sizeof(cz));
    cz* y = (cz*)calloc((size_t)n + 1, sizeof(cz));
    int* flag = (int*)malloc(((size_t)n + 1) * sizeof(int));
    int* stack = (int*)malloc(((size_t)n + 1) * sizeof(int));
    int* filled = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; ++i) flag[i] = -1;
    double smallest = 0.0, largest = 0.0, lmax = 0.0;
    int first = 1, done = 0, rc = 0;
    for (int k = 0; k < n; ++k) {
        /* ereach: row k's pattern in topological order */
        int top = n;
        flag[k] = k;
        for (int t = lp[k]; t < lp[k + 1]; ++t) {
            int i = lc[t];
            if (i >= k) continue;
            int len = 0;
            while (flag[i] != k) {
                stack[len++] = i;
                flag[i] = k;
                i = parent[i];
                if (i < 0) break;
            }
            while (len > 0) stack[--top] = stack[--len];
        }
        cz d = CMPLX(0.0, 0.0);
        for (int t = lp[k]; t < lp[k + 1]; ++t) {
            const int j = lc[t];
            if (j == k) d = addc(d, lv[t]);
            else if (j < k) y[j] = addc(y[j], lv[t]);
        }
        for (int s = top; s < n; ++s) {
            const int j = stack[s];
            const cz yj = y[j];
            y[j] = CMPLX(0.0, 0.0);
            const int b = col_ptr[j], e = b + filled[j];
            for (int t = b; t < e; ++t) y[row_index[t]] = subc(y[row_index[t]], L[t] * yj);
            const cz lkj = yj / D[j];
            d = subc(d, lkj * yj);
            if (e >= col_ptr[j + 1]) {
                rc = -1;
                goto out;
            }
            row_index[e] = k;
            L[e] = lkj;
            if (cabs(lkj) > lmax) lmax = cabs(lkj);
            ++filled[j];
        }
        D[k] = d;
        const double mag = cabs(d);
        if (mag > largest) largest = mag;
        if (first || mag < smallest) {
            smallest = mag;
            first = 0;
        }
        done = k + 1;
        if (!(mag > pivot_floor)) {
            rc = 1;
            break;
        }
    }
out:
    for (int t = 0; t < col_ptr[n]; ++t) st(lvalue + 2 * t, L[t]);
    for (int j = 0; j < n; ++j) st(diag + 2 * j, D[j]);
    stats[0] = rc == 0 ? 1.0 : 0.0;
    stats[1] = done;
    stats[2] = smallest;
    stats[3] = largest;
    stats[4] = lmax;
    stats[5] = (double)col_ptr[n] + n;
    free(v);
    free(iperm);
    free(lp);
    free(lc);
    free(lv);
    free(L);
    free(D);
    free(y);
    free(flag);
    free(stack);
    free(filled);
    return rc;
}

/* solve_in_place and solve, src/factorization.cpp:254-313 */
int or_solve(int n, const int* col_ptr, const int* row_index, const double* lvalue, const double* diag,
             const int* perm, const double* b, double* x) {
    cz* y = (cz*)malloc(((size_t)n + 1) * sizeof(cz));
    for (int i = 0; i < n; ++i) y[i] = ld(b + 2 * perm[i]);
    int rc = 0;
    for (int j = 0; j < n; ++j) {
        const cz yj = y[j];
        for (int t = col_ptr[j]; t < col_ptr[j + 1]; ++t) y[row_index[t]] = subc(y[row_index[t]], ld(lvalue + 2 * t) * yj);
    }
    for (int j = 0; j < n; ++j) {
        const cz d = ld(diag + 2 * j);
        if (d == 0.0) {
            rc = -1;
            break;
        }
        y[j] = y[j] / d;
    }
    if (!rc) {
        for (int j = n - 1; j >= 0; --j) {
            cz acc = y[j];
            for (int t = col_ptr[j]; t < col_ptr[j + 1]; ++t) acc = subc(acc, ld(lvalue + 2 * t) * y[row_index[t]]);
            y[j] = acc;
        }
        for (int i = 0; i < n; ++i) st(x + 2 * perm[i], y[i]);
    }
    free(y);
    return rc;
}

/* SparseSymmetric::matvec (include/aphi_solver/sparse_symmetric.hpp:120-136),
 * relative_residual and backward_error (src/factorization.cpp:315-329, :401-416) */
void or_residuals(int n, const int* row_ptr, const int* col_idx, const double* values, const double* x,
                  const double* b, double* out2) {
    cz* ax = (cz*)calloc((size_t)n + 1, sizeof(cz));
    double amax = 0.0;
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const int c = col_idx[k];
            const cz a = ld(values + 2 * k);
            ax[r] = addc(ax[r], a * ld(x + 2 * c));
            if (c != r) ax[c] = addc(ax[c], a * ld(x + 2 * r));
            if (cabs(a) > amax) amax = cabs(a);
        }
    double num = 0.0, bn = 0.0, xn = 0.0;
    for (int i = 0; i < n; ++i) {
        const cz e = subc(ax[i], ld(b + 2 * i));
        num += creal(e) * creal(e) + cimag(e) * cimag(e);
        bn += b[2 * i] * b[2 * i] + b[2 * i + 1] * b[2 * i + 1];
        xn += x[2 * i] * x[2 * i] + x[2 * i + 1] * x[2 * i + 1];
    }
    num = sqrt(num);
    out2[0] = sqrt(bn) > 0.0 ? num / sqrt(bn) : num;
    const double den = amax * sqrt(xn) + sqrt(bn);
    out2[1] = den > 0.0 ? num / den : num;
    free(ax);
}

/* solve_symmetric, src/factorization.cpp:332-398 */
int or_solve_symmetric(int n, const int* row_ptr, const int* col_idx, const double* values, const double* b,
                       const int* perm, const int* parent, const int* col_count, int equil_iters,
                       double pivot_floor, double* x, double* report) {
    const int nnz = row_ptr[n];
    double* d = (double*)malloc(((size_t)n + 1) * sizeof(double));
    for (int i = 0; i < n; ++i) d[i] = 1.0;
    if (equil_iters > 0) or_equilibration(n, row_ptr, col_idx, values, equil_iters, d);
    double dmin = 1.0, dmax = 1.0;
    for (int i = 0; i < n; ++i) {
        if (i == 0 || d[i] < dmin) dmin = d[i];
        if (i == 0 || d[i] > dmax) dmax = d[i];
    }
    double* sv = (double*)malloc(((size_t)nnz + 1) * 2 * sizeof(double));
    double* sb = (double*)malloc(((size_t)n + 1) * 2 * sizeof(double));
    for (int r = 0; r < n; ++r)
        for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            const cz a = ld(values + 2 * k);
            st(sv + 2 * k, equil_iters > 0 ? a * CMPLX(d[r] * d[col_idx[k]], 0.0) : a);
        }
    for (int i = 0; i < n; ++i) st(sb + 2 * i, equil_iters > 0 ? ld(b + 2 * i) * CMPLX(d[i], 0.0) : ld(b + 2 * i));
    long long nl = 0;
    for (int j = 0; j < n; ++j) nl += col_count[j] > 1 ? col_count[j] - 1 : 0;
    int* cp = (int*)malloc(((size_t)n + 1) * sizeof(int));
    int* ri = (int*)malloc(((size_t)nl + 1) * sizeof(int));
    double* lv = (double*)malloc(((size_t)nl + 1) * 2 * sizeof(double));
    double* dg = (double*)malloc(((size_t)n + 1) * 2 * sizeof(double));
    double stats[6];
    int rc = or_factorize(n, row_ptr, col_idx, sv, perm, parent, col_count, pivot_floor, cp, ri, lv, dg, stats);
    memset(report, 0, sizeof(double) * 10);
    report[3] = dmin;
    report[4] = dmax;
    report[5] = stats[2];
    report[6] = stats[3];
    report[7] = stats[4];
    report[8] = stats[5];
    report[9] = stats[1];
    if (rc == 0) {
        double* y = (double*)malloc(((size_t)n + 1) * 2 * sizeof(double));
        or_solve(n, cp, ri, lv, dg, perm, sb, y);
        for (int i = 0; i < n; ++i) st(x + 2 * i, equil_iters > 0 ? ld(y + 2 * i) * CMPLX(d[i], 0.0) : ld(y + 2 * i));
        free(y);
        double res[2];
        or_residuals(n, row_ptr, col_idx, values, x, b, res);
        report[0] = 1.0;
        report[1] = res[1];
        report[2] = res[0];
    }
    free(d);
    free(sv);
    free(sb);
    free(cp);
    free(ri);
    free(lv);
    free(dg);
    return rc == 0 ? 0 : 1;
}
