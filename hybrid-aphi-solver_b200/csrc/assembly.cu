// Numeric assembly on the device: element fill (K1) and deterministic scatter
// (K2) into the upper-triangle CSR of the symmetric system.
//
// Reference: refill -> scatter_into, src/assembly.cpp:255-422;
// element_coefficients and kernel_AA/APhi/PhiPhi, src/element_matrix.cpp:10-115;
// compute_tet_geometry, src/basis_functions.cpp:15-85; the degree-2 rule,
// src/quadrature.cpp:16-35.
//
// Design. The reference accumulates `values[slot] += term` while it walks
// bodies -> tets -> (AA, A-Phi/Phi-A, Phi-Phi) blocks. Here
//   K1 (k_tet_terms): one warp per tet, for every frequency of the batch,
//       stages the tet's tables and its frequency-independent geometry
//       (barycentric gradients, curls, Whitney values and P2 gradients at the
//       quadrature points) in shared memory, enumerates the tet's terms in
//       the reference's emission order, and computes (term, frequency) pairs
//       across its lanes -- each already scaled exactly as the reference forms
//       the addend -- into a term array, stored frequency-minor. Terms bound
//       for the right-hand side are stored negated (the reference subtracts
//       them).
//   K2 (k_slot_sum): one thread per (destination, frequency) -- CSR slot or
//       rhs row -- sums its terms in increasing term order through a slot ->
//       term list built once per mesh. Increasing term order IS the
//       reference's accumulation order, so the sums are bitwise those of the
//       reference: no float atomics, no order that depends on scheduling.
// This file is compiled with -fmad=false and uses explicitly rounded
// intrinsics for complex products, so every element entry and every addend is
// rounded exactly as the host's std::complex<double> arithmetic rounds it.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <vector>

#include "assembly.hpp"
#include "common.cuh"
#include "setup.hpp"

namespace aphi_b200 {

namespace {

__constant__ int c_edge_verts[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {2, 3}, {1, 3}};

// mu_0 and eps_0 as include/aphi_solver/constants.hpp:12-13 defines them.
constexpr double kMu0 = 4.0e-7 * 3.14159265358979323846;
constexpr double kEps0 = 8.8541878128e-12;

struct Geometry {
    double grad[4][3];
    double volume;
};

// Gauss-Jordan inverse of M = [1 x y z] per vertex row with partial
// pivoting; column i of M^-1 holds L_i's affine coefficients. Returns false
// for a pivot below 1e-14 (a degenerate tet).
__device__ bool tet_geometry(const double p[4][3], Geometry& g) {
    double m[4][4], inv[4][4];
    for (int r = 0; r < 4; ++r) {
        m[r][0] = 1.0;
        m[r][1] = p[r][0];
        m[r][2] = p[r][1];
        m[r][3] = p[r][2];
        for (int c = 0; c < 4; ++c) inv[r][c] = (r == c) ? 1.0 : 0.0;
    }
    for (int col = 0; col < 4; ++col) {
        int prow = col;
        double pval = fabs(m[col][col]);
        for (int r = col + 1; r < 4; ++r)
            if (fabs(m[r][col]) > pval) {
                prow = r;
                pval = fabs(m[r][col]);
            }
        if (pval < 1e-14) return false;
        if (prow != col)
            for (int c = 0; c < 4; ++c) {
                double t = m[prow][c];
                m[prow][c] = m[col][c];
                m[col][c] = t;
                t = inv[prow][c];
                inv[prow][c] = inv[col][c];
                inv[col][c] = t;
            }
        const double piv = m[col][col];
        for (int c = 0; c < 4; ++c) {
            m[col][c] = __ddiv_rn(m[col][c], piv);
            inv[col][c] = __ddiv_rn(inv[col][c], piv);
        }
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            const double f = m[r][col];
            if (f == 0.0) continue;
            for (int c = 0; c < 4; ++c) {
                m[r][c] = __dsub_rn(m[r][c], __dmul_rn(f, m[col][c]));
                inv[r][c] = __dsub_rn(inv[r][c], __dmul_rn(f, inv[col][c]));
            }
        }
    }
    for (int i = 0; i < 4; ++i) {
        g.grad[i][0] = inv[1][i];
        g.grad[i][1] = inv[2][i];
        g.grad[i][2] = inv[3][i];
    }
    // |((p1 - p0) x (p2 - p0)) . (p3 - p0)| / 6
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = __dsub_rn(p[1][k], p[0][k]);
        b[k] = __dsub_rn(p[2][k], p[0][k]);
        c[k] = __dsub_rn(p[3][k], p[0][k]);
    }
    const double x = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
    const double y = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
    const double z = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
    const double dot = __dadd_rn(__dadd_rn(__dmul_rn(x, c[0]), __dmul_rn(y, c[1])), __dmul_rn(z, c[2]));
    g.volume = fabs(__ddiv_rn(dot, 6.0));
    return true;
}

__device__ __forceinline__ double dot3(const double* u, const double* v) {
    return __dadd_rn(__dadd_rn(__dmul_rn(u[0], v[0]), __dmul_rn(u[1], v[1])), __dmul_rn(u[2], v[2]));
}

// Whitney edge function at barycentric point L: grad(L_j) L_i - grad(L_i) L_j.
__device__ __forceinline__ void whitney(const Geometry& g, int e, const double* L, double* out) {
    const int vi = c_edge_verts[e][0], vj = c_edge_verts[e][1];
    for (int k = 0; k < 3; ++k)
        out[k] = __dsub_rn(__dmul_rn(g.grad[vj][k], L[vi]), __dmul_rn(g.grad[vi][k], L[vj]));
}

// Gradient of P2 nodal function b at L.
__device__ __forceinline__ void p2_grad(const Geometry& g, int b, const double* L, double* out) {
    if (b < 4) {
        const double s = __dsub_rn(__dmul_rn(4.0, L[b]), 1.0);
        for (int k = 0; k < 3; ++k) out[k] = __dmul_rn(g.grad[b][k], s);
    } else {
        const int v0 = c_edge_verts[b - 4][0], v1 = c_edge_verts[b - 4][1];
        const double s0 = __dmul_rn(4.0, L[v1]), s1 = __dmul_rn(4.0, L[v0]);
        for (int k = 0; k < 3; ++k)
            out[k] = __dadd_rn(__dmul_rn(g.grad[v0][k], s0), __dmul_rn(g.grad[v1][k], s1));
    }
}

struct Coeff {
    double nu;
    cplx alpha, beta;
};

// element_coefficients, src/element_matrix.cpp:10-25.
__host__ __device__ inline Coeff body_coefficients(double sigma, double eps_r, double mu_r, double omega) {
    Coeff c;
#ifdef __CUDA_ARCH__
    const double mu = __dmul_rn(mu_r, kMu0);
    const double eps = __dmul_rn(eps_r, kEps0);
    c.nu = __ddiv_rn(1.0, mu);
    c.alpha = cplx{__dmul_rn(__dmul_rn(-omega, omega), eps), __dmul_rn(omega, sigma)};
    c.beta = cplx{sigma, __dmul_rn(omega, eps)};
#else
    const double mu = mu_r * kMu0;
    const double eps = eps_r * kEps0;
    c.nu = 1.0 / mu;
    c.alpha = cplx{-omega * omega * eps, omega * sigma};
    c.beta = cplx{sigma, omega * eps};
#endif
    return c;
}

// The degree-2 rule: points (a,b,b,b) and permutations, weights 1/4.
struct Quad {
    double a, b;
};

// kernel_AA, kernel_APhi, kernel_PhiPhi (src/element_matrix.cpp:27-115), with
// the same accumulation order over quadrature points.
__device__ void element_blocks(const Geometry& g, const Coeff& c, const Quad& q, bool need_phi,
                               cplx* aa, cplx* ap, cplx* pp) {
    double curl[6][3];
    for (int e = 0; e < 6; ++e) {
        const int vi = c_edge_verts[e][0], vj = c_edge_verts[e][1];
        const double* u = g.grad[vi];
        const double* v = g.grad[vj];
        curl[e][0] = __dmul_rn(__dsub_rn(__dmul_rn(u[1], v[2]), __dmul_rn(u[2], v[1])), 2.0);
        curl[e][1] = __dmul_rn(__dsub_rn(__dmul_rn(u[2], v[0]), __dmul_rn(u[0], v[2])), 2.0);
        curl[e][2] = __dmul_rn(__dsub_rn(__dmul_rn(u[0], v[1]), __dmul_rn(u[1], v[0])), 2.0);
    }
    const double nv = __dmul_rn(c.nu, g.volume);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) aa[i * 6 + j] = cplx{__dmul_rn(nv, dot3(curl[i], curl[j])), 0.0};

    const bool mass = !(c.alpha.re == 0.0 && c.alpha.im == 0.0);
    const bool coupling = need_phi && !(c.beta.re == 0.0 && c.beta.im == 0.0);
    if (need_phi) {
        for (int i = 0; i < 60; ++i) ap[i] = cplx{0.0, 0.0};
        for (int i = 0; i < 100; ++i) pp[i] = cplx{0.0, 0.0};
    }
    if (!mass && !coupling) return;
    for (int k = 0; k < 4; ++k) {
        double L[4];
        for (int i = 0; i < 4; ++i) L[i] = (i == k) ? q.a : q.b;
        const double w = __dmul_rn(0.25, g.volume);
        double wv[6][3];
        for (int e = 0; e < 6; ++e) whitney(g, e, L, wv[e]);
        if (mass) {
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) {
                    const double s = __dmul_rn(w, dot3(wv[i], wv[j]));
                    aa[i * 6 + j] = cadd_exact(aa[i * 6 + j], cscale_exact(c.alpha, s));
                }
        }
        if (coupling) {
            double gr[10][3];
            for (int b = 0; b < 10; ++b) p2_grad(g, b, L, gr[b]);
            for (int i = 0; i < 6; ++i)
                for (int b = 0; b < 10; ++b) {
                    const double s = __dmul_rn(w, dot3(wv[i], gr[b]));
                    ap[i * 10 + b] = cadd_exact(ap[i * 10 + b], cscale_exact(c.beta, s));
                }
            for (int a = 0; a < 10; ++a)
                for (int b = 0; b < 10; ++b) {
                    const double s = __dmul_rn(w, dot3(gr[a], gr[b]));
                    pp[a * 10 + b] = cadd_exact(pp[a * 10 + b], cscale_exact(c.beta, s));
                }
        }
    }
}

// Complex division in the order the host runtime uses for finite operands of
// ordinary magnitude (Smith's method), for the prescribed-value and port
// scalars: v / c.
__device__ cplx cdiv_smith(cplx a, cplx b) {
    if (fabs(b.re) < fabs(b.im)) {
        const double ratio = __ddiv_rn(b.re, b.im);
        const double denom = __dadd_rn(__dmul_rn(b.re, ratio), b.im);
        return cplx{__ddiv_rn(__dadd_rn(__dmul_rn(a.re, ratio), a.im), denom),
                    __ddiv_rn(__dsub_rn(__dmul_rn(a.im, ratio), a.re), denom)};
    }
    const double ratio = __ddiv_rn(b.im, b.re);
    const double denom = __dadd_rn(b.re, __dmul_rn(b.im, ratio));
    return cplx{__ddiv_rn(__dadd_rn(a.re, __dmul_rn(a.im, ratio)), denom),
                __ddiv_rn(__dsub_rn(a.im, __dmul_rn(a.re, ratio)), denom)};
}

struct Scales {
    cplx row, col, jw;
};

// formulation_scales, src/assembly.cpp:12-45 (omega == 0 is refused on the host).
__device__ Scales scales_of(int cond, double omega) {
    Scales s;
    s.jw = cplx{0.0, omega};
    s.row = cplx{1.0, 0.0};
    s.col = cplx{1.0, 0.0};
    if (cond == APHI_COND_ROW_SCALED) s.row = cdiv_smith(cplx{1.0, 0.0}, s.jw);
    if (cond == APHI_COND_SCALED_PHI) s.col = s.jw;
    return s;
}

struct TetArgs {
    int num_tets;
    int upper_only;
    const double* xyz;
    const int* tets;
    const int* visit_tet;
    const int* visit_body;
    const double* material;
    const int* tet_idx;
    const double* tet_coeff;
    const double* tet_fixed;
    const long long* term_off;
    int* err;          // [0] degenerate tet, [1] term count mismatch
};

struct Omegas {
    int n;
    double w[kMaxBatchOmegas];
};

// compute_tet_geometry's Gauss-Jordan inverse with every index static (the
// pivot row swap is a predicated exchange), so the 4 x 4 arrays stay in
// registers. The same operations on the same values, in the same order, as
// tet_geometry above: bitwise the same result.
__device__ __forceinline__ bool tet_geometry_reg(const double (&p)[4][3], double (&grad)[4][3], double& volume) {
    double m[4][4], inv[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        m[r][0] = 1.0;
        m[r][1] = p[r][0];
        m[r][2] = p[r][1];
        m[r][3] = p[r][2];
#pragma unroll
        for (int c = 0; c < 4; ++c) inv[r][c] = (r == c) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int col = 0; col < 4; ++col) {
        int prow = col;
        double pval = fabs(m[col][col]);
#pragma unroll
        for (int r = col + 1; r < 4; ++r)
            if (fabs(m[r][col]) > pval) {
                prow = r;
                pval = fabs(m[r][col]);
            }
        if (pval < 1e-14) return false;
#pragma unroll
        for (int r = col + 1; r < 4; ++r) {
            const bool sw = r == prow;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double a = m[r][c], b = m[col][c];
                m[r][c] = sw ? b : a;
                m[col][c] = sw ? a : b;
                const double x = inv[r][c], y = inv[col][c];
                inv[r][c] = sw ? y : x;
                inv[col][c] = sw ? x : y;
            }
        }
        const double piv = m[col][col];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            m[col][c] = __ddiv_rn(m[col][c], piv);
            inv[col][c] = __ddiv_rn(inv[col][c], piv);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            const double f = m[r][col];
            if (f == 0.0) continue;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                m[r][c] = __dsub_rn(m[r][c], __dmul_rn(f, m[col][c]));
                inv[r][c] = __dsub_rn(inv[r][c], __dmul_rn(f, inv[col][c]));
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        grad[i][0] = inv[1][i];
        grad[i][1] = inv[2][i];
        grad[i][2] = inv[3][i];
    }
    double a[3], b[3], c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a[k] = __dsub_rn(p[1][k], p[0][k]);
        b[k] = __dsub_rn(p[2][k], p[0][k]);
        c[k] = __dsub_rn(p[3][k], p[0][k]);
    }
    const double x = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
    const double y = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
    const double z = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
    const double dot = __dadd_rn(__dadd_rn(__dmul_rn(x, c[0]), __dmul_rn(y, c[1])), __dmul_rn(z, c[2]));
    volume = fabs(__ddiv_rn(dot, 6.0));
    return true;
}

// Term kinds of the scatter (src/assembly.cpp:268-394), in emission order
// within a tet: (A,A); (A,Phi) or its prescribed-Phi rhs term, then (Phi,A);
// (Phi,Phi) or its prescribed-Phi rhs term.
enum : int { T_AA = 0, T_AP = 1, T_AP_FIXED = 2, T_PA = 3, T_PP = 4, T_PP_FIXED = 5 };

constexpr int kTetWarps = 4;          // tets (warps) per block
constexpr int kTetMaxTerms = 256;     // 36 + 120 + 100 at most (full storage)

// Per-warp staging: the tet's tables, geometry and the frequency-independent
// vectors of its element blocks (curls; Whitney values and P2 gradients at
// the four quadrature points), and its term list.
struct TetStage {
    double grad[4][3];
    double curl[6][3];
    double wv[4][6][3];
    double gr[4][10][3];
    double fixed[10][2];
    double co[16];
    double p[4][3];
    double mat[3];
    double volume;
    int idx[16];
    unsigned short rec[kTetMaxTerms];  // kind << 8 | i << 4 | j
    // per frequency of the batch: the body's coefficients and the scalings
    Coeff cf[kMaxBatchOmegas];
    cplx col[kMaxBatchOmegas], rjw[kMaxBatchOmegas], rc[kMaxBatchOmegas];
};

__device__ __forceinline__ double dot3s(const double* u, const double* v) { return dot3(u, v); }

// K1: one warp per tet (in the reference's body -> tet visit order), all the
// batch's frequencies. The warp stages the tet once, enumerates its terms in
// the reference's emission order (a warp scan over the 36 + 60 + 100 block
// positions), then computes (term, frequency) pairs across its lanes: each
// pair's element entry is rebuilt from the staged vectors with the reference's
// accumulation over the quadrature points, and scaled exactly as the reference
// forms its addend. Terms are stored frequency-minor, terms[t * nf + f], so a
// warp's stores are contiguous and the slot sums read 16 * nf contiguous
// bytes per term.
__global__ void __launch_bounds__(32 * kTetWarps) k_tet_terms(TetArgs A, Omegas om, int cond, Quad quad,
                                                              cplx* terms) {
    __shared__ TetStage stage[kTetWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v = blockIdx.x * kTetWarps + warp;
    if (v >= A.num_tets) return;  // uniform per warp
    TetStage& S = stage[warp];
    const int t = A.visit_tet[v];
    const int b = A.visit_body[v];
    if (lane < 16) {
        S.idx[lane] = A.tet_idx[16LL * t + lane];
        S.co[lane] = A.tet_coeff[16LL * t + lane];
    }
    if (lane < 20) (&S.fixed[0][0])[lane] = A.tet_fixed[20LL * t + lane];
    if (lane < 12) S.p[lane / 3][lane % 3] = A.xyz[3LL * A.tets[4LL * t + lane / 3] + lane % 3];
    if (lane < 3) S.mat[lane] = A.material[3 * b + lane];
    __syncwarp();
    const bool fixed_lane = lane < 10 && !(S.fixed[lane][0] == 0.0 && S.fixed[lane][1] == 0.0);
    const unsigned fixed_mask = __ballot_sync(0xffffffffu, fixed_lane);
    const bool need_phi = __ballot_sync(0xffffffffu, lane < 10 && (S.idx[6 + lane] >= 0 || fixed_lane)) != 0;

    // Geometry: every lane computes it (uniform control flow); lane 0 stages it.
    {
        double p[4][3], grad[4][3], vol;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) p[r][k] = S.p[r][k];
        if (!tet_geometry_reg(p, grad, vol)) {
            if (lane == 0) atomicExch(&A.err[0], 1);
            return;
        }
        if (lane == 0) {
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int k = 0; k < 3; ++k) S.grad[r][k] = grad[r][k];
            S.volume = vol;
        }
    }
    __syncwarp();
    // Curls (6), Whitney values (4 points x 6 edges), P2 gradients (4 x 10).
    const int nvec = need_phi ? 70 : 30;
    for (int it = lane; it < nvec; it += 32) {
        if (it < 6) {
            const double* u = S.grad[c_edge_verts[it][0]];
            const double* w = S.grad[c_edge_verts[it][1]];
            S.curl[it][0] = __dmul_rn(__dsub_rn(__dmul_rn(u[1], w[2]), __dmul_rn(u[2], w[1])), 2.0);
            S.curl[it][1] = __dmul_rn(__dsub_rn(__dmul_rn(u[2], w[0]), __dmul_rn(u[0], w[2])), 2.0);
            S.curl[it][2] = __dmul_rn(__dsub_rn(__dmul_rn(u[0], w[1]), __dmul_rn(u[1], w[0])), 2.0);
        } else {
            const int q = it < 30 ? (it - 6) / 6 : (it - 30) / 10;
            // barycentric coordinate i of quadrature point q: (a, b, b, b) permuted
            auto L = [&](int i) { return i == q ? quad.a : quad.b; };
            if (it < 30) {
                const int e = (it - 6) % 6;
                const int vi = c_edge_verts[e][0], vj = c_edge_verts[e][1];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    S.wv[q][e][k] = __dsub_rn(__dmul_rn(S.grad[vj][k], L(vi)), __dmul_rn(S.grad[vi][k], L(vj)));
            } else {
                const int bb = (it - 30) % 10;
                if (bb < 4) {
                    const double sc = __dsub_rn(__dmul_rn(4.0, L(bb)), 1.0);
#pragma unroll
                    for (int k = 0; k < 3; ++k) S.gr[q][bb][k] = __dmul_rn(S.grad[bb][k], sc);
                } else {
                    const int v0 = c_edge_verts[bb - 4][0], v1 = c_edge_verts[bb - 4][1];
                    const double s0 = __dmul_rn(4.0, L(v1)), s1 = __dmul_rn(4.0, L(v0));
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        S.gr[q][bb][k] = __dadd_rn(__dmul_rn(S.grad[v0][k], s0), __dmul_rn(S.grad[v1][k], s1));
                }
            }
        }
    }
    // The tet's terms in emission order: block positions AA (36), then
    // (A,Phi) pairs (60, up to two terms each) and (Phi,Phi) (100).
    const bool up = A.upper_only != 0;
    const int ncand = need_phi ? 196 : 36;
    int total = 0;
    for (int c0 = 0; c0 < ncand; c0 += 32) {
        const int c = c0 + lane;
        int n = 0, r0 = 0, r1 = 0;
        if (c < 36) {
            const int pi = c / 6, qi = c % 6;
            if (S.idx[pi] >= 0 && S.idx[qi] >= 0 && !(up && S.idx[qi] < S.idx[pi])) {
                n = 1;
                r0 = T_AA << 8 | pi << 4 | qi;
            }
        } else if (c < 96) {
            const int pi = (c - 36) / 10, qi = (c - 36) % 10;
            const int row = S.idx[pi], col = S.idx[6 + qi];
            if (row >= 0) {
                if (col >= 0) {
                    if (!(up && col < row)) r0 = T_AP << 8 | pi << 4 | qi, n = 1;
                    if (!(up && row < col)) (n ? r1 : r0) = T_PA << 8 | pi << 4 | qi, ++n;
                } else if ((fixed_mask >> qi) & 1u) {
                    r0 = T_AP_FIXED << 8 | pi << 4 | qi;
                    n = 1;
                }
            }
        } else if (c < 196) {
            const int pi = (c - 96) / 10, qi = (c - 96) % 10;
            const int row = S.idx[6 + pi], col = S.idx[6 + qi];
            if (row >= 0) {
                if (col >= 0) {
                    if (!(up && col < row)) r0 = T_PP << 8 | pi << 4 | qi, n = 1;
                } else if ((fixed_mask >> qi) & 1u) {
                    r0 = T_PP_FIXED << 8 | pi << 4 | qi;
                    n = 1;
                }
            }
        }
        int incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int at = total + incl - n;
        if (n > 0) S.rec[at] = static_cast<unsigned short>(r0);
        if (n > 1) S.rec[at + 1] = static_cast<unsigned short>(r1);
        total += __shfl_sync(0xffffffffu, incl, 31);
    }
    const long long off = A.term_off[v];
    if (total != A.term_off[v + 1] - off) {
        if (lane == 0) atomicExch(&A.err[1], 1);
        return;
    }
    __syncwarp();
    const int nf = om.n;
    // The body's coefficients and the formulation's scalings, once per
    // frequency (they hold divisions), for every term of the tet.
    for (int f = lane; f < nf; f += 32) {
        const double omega = om.w[f];
        S.cf[f] = body_coefficients(S.mat[0], S.mat[1], S.mat[2], omega);
        const Scales sc = scales_of(cond, omega);
        S.col[f] = sc.col;
        S.rjw[f] = cmul_exact(sc.row, sc.jw);
        S.rc[f] = cmul_exact(sc.row, sc.col);
    }
    __syncwarp();
    const double vol = S.volume;
    const double w = __dmul_rn(0.25, vol);
    cplx* out = terms + off * nf;
    for (int it = lane; it < total * nf; it += 32) {
        const int k = it / nf, f = it - k * nf;
        const int r = S.rec[k];
        const int kind = r >> 8, i = (r >> 4) & 15, j = r & 15;
        const Coeff& c = S.cf[f];
        cplx blk{0.0, 0.0};
        if (kind == T_AA) {
            // kernel_AA: nu V curl.curl, then the mass term point by point.
            blk = cplx{__dmul_rn(__dmul_rn(c.nu, vol), dot3s(S.curl[i], S.curl[j])), 0.0};
            if (!(c.alpha.re == 0.0 && c.alpha.im == 0.0))
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    blk = cadd_exact(blk, cscale_exact(c.alpha, __dmul_rn(w, dot3s(S.wv[q][i], S.wv[q][j]))));
        } else if (!(c.beta.re == 0.0 && c.beta.im == 0.0)) {
            // kernel_APhi / kernel_PhiPhi
            const bool pp = kind >= T_PP;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double* u = pp ? S.gr[q][i] : S.wv[q][i];
                blk = cadd_exact(blk, cscale_exact(c.beta, __dmul_rn(w, dot3s(u, S.gr[q][j]))));
            }
        }
        const cplx col = S.col[f];
        cplx term;
        switch (kind) {
            case T_AA: term = cscale_exact(blk, __dmul_rn(S.co[i], S.co[j])); break;
            case T_AP: term = cmul_exact(cscale_exact(col, __dmul_rn(S.co[i], S.co[6 + j])), blk); break;
            case T_AP_FIXED: {
                const cplx fx = cdiv_smith(cplx{S.fixed[j][0], S.fixed[j][1]}, col);
                term = cneg(cmul_exact(cmul_exact(cscale_exact(col, S.co[i]), blk), fx));
                break;
            }
            case T_PA: term = cmul_exact(cscale_exact(S.rjw[f], __dmul_rn(S.co[6 + j], S.co[i])), blk); break;
            case T_PP: term = cmul_exact(cscale_exact(S.rc[f], __dmul_rn(S.co[6 + i], S.co[6 + j])), blk); break;
            default: {
                const cplx fx = cdiv_smith(cplx{S.fixed[j][0], S.fixed[j][1]}, col);
                term = cneg(cmul_exact(cmul_exact(cscale_exact(S.rc[f], S.co[6 + i]), blk), fx));
                break;
            }
        }
        out[it] = term;
    }
}

struct PortArgs {
    int num_ports;
    const int* current;
    const double* amplitude;
    const double* value;
    long long first_term;  // index of the first port term
};

// Port rows, src/assembly.cpp:396-421: a voltage port's unit diagonal and
// rhs V / c; a current port's rhs r * I. One thread per frequency.
__global__ void k_port_terms(PortArgs P, Omegas om, int cond, cplx* terms) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int nf = om.n;
    if (f >= nf) return;
    const Scales sc = scales_of(cond, om.w[f]);
    cplx* out = terms + P.first_term * nf + f;
    long long k = 0;
    for (int p = 0; p < P.num_ports; ++p) {
        if (P.current[p]) {
            out[nf * k++] = cmul_exact(sc.row, cplx{P.amplitude[2 * p], P.amplitude[2 * p + 1]});
        } else {
            out[nf * k++] = cplx{1.0, 0.0};
            out[nf * k++] = cdiv_smith(cplx{P.value[2 * p], P.value[2 * p + 1]}, sc.col);
        }
    }
}

// K2: fixed-order sum of each destination's terms (increasing term index,
// the reference's accumulation order), for every frequency of the batch.
// Thread (slot, frequency) with the frequency fastest, so one term's nf
// values are read as one contiguous run; the sums are transposed through
// shared memory so that each frequency's values are written as a contiguous
// run of slots.
constexpr int kSlotThreads = 256;
__global__ void __launch_bounds__(kSlotThreads) k_slot_sum(int ndest, int nnz, int n, int nf, const int* dest_ptr,
                                                           const int* dest_terms, const cplx* terms,
                                                           cplx* values, cplx* rhs) {
    __shared__ cplx sh[kSlotThreads];
    const int spb = kSlotThreads / nf;  // slots per block
    const int dl = threadIdx.x / nf, f = threadIdx.x - dl * nf;
    const int d0 = blockIdx.x * spb;
    const int d = d0 + dl;
    if (dl < spb && d < ndest) {
        cplx s{0.0, 0.0};
        const int e = dest_ptr[d + 1];
        for (int k = dest_ptr[d]; k < e; ++k) s = cadd_exact(s, terms[static_cast<long long>(dest_terms[k]) * nf + f]);
        sh[f * spb + dl] = s;
    }
    __syncthreads();
    const int cnt = min(spb, ndest - d0);
    for (int e = threadIdx.x; e < nf * spb; e += kSlotThreads) {
        const int ff = e / spb, x = e - ff * spb;
        if (x >= cnt) continue;
        const int dd = d0 + x;
        if (dd < nnz)
            values[static_cast<long long>(ff) * nnz + dd] = sh[e];
        else
            rhs[static_cast<long long>(ff) * n + (dd - nnz)] = sh[e];
    }
}

// Element blocks for a list of tets (parity hook).
__global__ void k_element_blocks(int ntets, const double* xyz, Coeff c, Quad q, cplx* aa, cplx* ap,
                                 cplx* pp, int* err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntets) return;
    double p[4][3];
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 3; ++k) p[i][k] = xyz[12LL * t + 3 * i + k];
    Geometry g;
    if (!tet_geometry(p, g)) {
        atomicExch(err, 1);
        return;
    }
    element_blocks(g, c, q, true, aa + 36LL * t, ap + 60LL * t, pp + 100LL * t);
}

template <class T>
T* upload(const T* h, size_t n) {
    T* d = nullptr;
    APHI_CUDA(cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(T)));
    if (n) APHI_CUDA(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

Quad quad_points() {
    const double s5 = std::sqrt(5.0);
    return Quad{(5.0 + 3.0 * s5) / 20.0, (5.0 - s5) / 20.0};
}

}  // namespace

void assembly_coefficients(double sigma, double eps_r, double mu_r, double omega, double* out5) {
    const Coeff c = body_coefficients(sigma, eps_r, mu_r, omega);
    out5[0] = c.nu;
    out5[1] = c.alpha.re;
    out5[2] = c.alpha.im;
    out5[3] = c.beta.re;
    out5[4] = c.beta.im;
}

void formulation_scales_host(int cond, double omega, std::complex<double>& row, std::complex<double>& col,
                             bool& symmetric) {
    const std::complex<double> jw(0.0, omega);
    switch (cond) {
        case APHI_COND_NATURAL:
            row = col = std::complex<double>(1.0, 0.0);
            symmetric = false;
            return;
        case APHI_COND_ROW_SCALED:
            if (omega == 0.0)
                throw Error(APHI_ERR_BAD_SHAPE,
                            "formulation_scales: the row-scaled formulation divides the Phi rows by "
                            "j*omega, which is undefined at DC. Use the natural form.");
            row = std::complex<double>(1.0, 0.0) / jw;
            col = std::complex<double>(1.0, 0.0);
            symmetric = true;
            return;
        case APHI_COND_SCALED_PHI:
            if (omega == 0.0)
                throw Error(APHI_ERR_BAD_SHAPE,
                            "formulation_scales: the scaled-potential formulation would divide a "
                            "prescribed potential by j*omega, which is undefined at DC. Use the "
                            "natural form.");
            row = std::complex<double>(1.0, 0.0);
            col = jw;
            symmetric = true;
            return;
    }
    throw Error(APHI_ERR_BAD_SHAPE, "formulation_scales: unknown formulation");
}

Assembly::~Assembly() {
    for (void* p : {(void*)d_xyz, (void*)d_tets, (void*)d_visit_tet, (void*)d_visit_body,
                    (void*)d_material, (void*)d_tet_idx, (void*)d_tet_coeff, (void*)d_tet_fixed,
                    (void*)d_term_off, (void*)d_dest_ptr, (void*)d_dest_terms, (void*)d_terms,
                    (void*)d_port_current, (void*)d_port_amp, (void*)d_port_value, (void*)d_err})
        if (p) cudaFree(p);
}

namespace {

int find_slot(const int* row_ptr, const int* col_idx, int r, int c) {
    const int* b = col_idx + row_ptr[r];
    const int* e = col_idx + row_ptr[r + 1];
    const int* it = std::lower_bound(b, e, c);
    return (it == e || *it != c) ? -1 : static_cast<int>(it - col_idx);
}

}  // namespace

std::unique_ptr<Assembly> assembly_create(const aphi_assembly_desc& d, bool device_setup) {
    if (d.num_tets < 0 || d.num_unknowns < 0 || d.num_bodies < 1 || !d.row_ptr || !d.col_idx ||
        !d.tet_idx || !d.tet_coeff || !d.tets || !d.xyz || !d.body_ptr || !d.body_tets || !d.material)
        throw Error(APHI_ERR_INVALID, "aphi_assembly_create: missing arrays in the description");
    const int N = d.num_unknowns;
    const int nnz = d.row_ptr[N];
    const int T = d.num_tets;
    if (d.body_ptr[0] != 0 || d.body_ptr[d.num_bodies] != T)
        throw Error(APHI_ERR_BAD_SHAPE,
                    "refill: the bodies must partition the tets (body_ptr runs 0 .. num_tets)");
    for (int p = 0; p < d.num_ports; ++p)
        if (d.port_row[p] < 0 || d.port_row[p] >= N)
            throw Error(APHI_ERR_BAD_SHAPE, "refill: a port row lies outside the unknowns");

    auto A = std::make_unique<Assembly>();
    A->N = N;
    A->nnz = nnz;
    A->T = T;
    A->num_bodies = d.num_bodies;
    A->num_ports = d.num_ports;
    A->upper_only = d.upper_only != 0;

    // Visit order and, per tet, the destination of every term in the order
    // the scatter produces it.
    std::vector<int> visit_tet(d.body_tets, d.body_tets + T), visit_body(T);
    for (int b = 0; b < d.num_bodies; ++b)
        for (int v = d.body_ptr[b]; v < d.body_ptr[b + 1]; ++v) visit_body[v] = b;
    std::vector<long long> term_off;
    std::vector<int> dest, port_current(d.num_ports), dptr, dterm;
    for (int p = 0; p < d.num_ports; ++p) port_current[p] = d.port_current[p] ? 1 : 0;
    const int ndest = nnz + N;
    if (!device_setup) {
        term_off.assign(static_cast<size_t>(T) + 1, 0);
        dest.reserve(static_cast<size_t>(T) * 24);
        const bool up = A->upper_only;
        auto slot_of = [&](int r, int c) {
            const int s = find_slot(d.row_ptr, d.col_idx, r, c);
            if (s < 0)
                throw Error(APHI_ERR_PATTERN_MISMATCH,
                            "assemble: no slot for entry (" + std::to_string(r) + ", " + std::to_string(c) +
                                "). The sparsity pattern and the scatter disagree about the matrix's "
                                "shape; dropping the term would give a quietly wrong matrix.");
            return s;
        };
        for (int v = 0; v < T; ++v) {
            const int t = visit_tet[v];
            if (t < 0 || t >= T) throw Error(APHI_ERR_BAD_SHAPE, "refill: body tet index out of range");
            const int* idx = d.tet_idx + 16LL * t;
            const double* fx = d.tet_fixed ? d.tet_fixed + 20LL * t : nullptr;
            for (int q = 0; q < 16; ++q)
                if (idx[q] >= N) throw Error(APHI_ERR_BAD_SHAPE, "refill: a DOF index exceeds the unknowns");
            auto nz = [&](int q) { return fx && (fx[2 * q] != 0.0 || fx[2 * q + 1] != 0.0); };
            bool need_phi = false;
            for (int q = 0; q < 10; ++q)
                if (idx[6 + q] >= 0 || nz(q)) need_phi = true;
            for (int p = 0; p < 6; ++p) {
                if (idx[p] < 0) continue;
                for (int q = 0; q < 6; ++q) {
                    if (idx[q] < 0 || (up && idx[q] < idx[p])) continue;
                    dest.push_back(slot_of(idx[p], idx[q]));
                }
            }
            if (need_phi) {
                for (int p = 0; p < 6; ++p) {
                    if (idx[p] < 0) continue;
                    for (int q = 0; q < 10; ++q) {
                        const int col = idx[6 + q];
                        if (col >= 0) {
                            if (!(up && col < idx[p])) dest.push_back(slot_of(idx[p], col));
                        } else if (nz(q)) {
                            dest.push_back(nnz + idx[p]);
                        }
                        if (col >= 0 && !(up && idx[p] < col)) dest.push_back(slot_of(col, idx[p]));
                    }
                }
                for (int p = 0; p < 10; ++p) {
                    const int row = idx[6 + p];
                    if (row < 0) continue;
                    for (int q = 0; q < 10; ++q) {
                        const int col = idx[6 + q];
                        if (col >= 0) {
                            if (!(up && col < row)) dest.push_back(slot_of(row, col));
                        } else if (nz(q)) {
                            dest.push_back(nnz + row);
                        }
                    }
                }
            }
            term_off[v + 1] = static_cast<long long>(dest.size());
        }
        A->tet_terms = static_cast<long long>(dest.size());
        for (int p = 0; p < d.num_ports; ++p) {
            if (port_current[p]) {
                dest.push_back(nnz + d.port_row[p]);
            } else {
                dest.push_back(slot_of(d.port_row[p], d.port_row[p]));
                dest.push_back(nnz + d.port_row[p]);
            }
        }
        A->num_terms = static_cast<long long>(dest.size());
        if (A->num_terms >= (1LL << 31))
            throw Error(APHI_ERR_BAD_SHAPE, "refill: more than 2^31 element terms");

        // Slot -> term lists, stable in term order.
        dptr.assign(static_cast<size_t>(ndest) + 1, 0);
        dterm.resize(dest.size());
        for (int x : dest) ++dptr[x + 1];
        for (int i = 0; i < ndest; ++i) dptr[i + 1] += dptr[i];
        {
            std::vector<int> cur(dptr.begin(), dptr.end() - 1);
            for (size_t k = 0; k < dest.size(); ++k) dterm[cur[dest[k]]++] = static_cast<int>(k);
        }
    }

    A->d_xyz = upload(d.xyz, 3LL * d.num_nodes);
    A->d_tets = upload(d.tets, 4LL * T);
    A->d_visit_tet = upload(visit_tet.data(), visit_tet.size());
    A->d_visit_body = upload(visit_body.data(), visit_body.size());
    A->d_material = upload(d.material, 3LL * d.num_bodies);
    A->d_tet_idx = upload(d.tet_idx, 16LL * T);
    A->d_tet_coeff = upload(d.tet_coeff, 16LL * T);
    std::vector<double> zeros;
    if (!d.tet_fixed) zeros.assign(20LL * T, 0.0);
    A->d_tet_fixed = upload(d.tet_fixed ? d.tet_fixed : zeros.data(), 20LL * T);
    if (device_setup) {
        assembly_maps_on_device(*A, d, visit_tet.data());
    } else {
        A->d_term_off = upload(term_off.data(), term_off.size());
        A->d_dest_ptr = upload(dptr.data(), dptr.size());
        A->d_dest_terms = upload(dterm.data(), dterm.size());
    }
    A->d_port_current = upload(port_current.data(), port_current.size());
    A->d_port_amp = upload(d.port_amplitude, 2LL * d.num_ports);
    A->d_port_value = upload(d.port_value, 2LL * d.num_ports);
    A->d_err = upload(std::vector<int>(4, 0).data(), 4);
    A->bytes = (3LL * d.num_nodes + 16LL * T + 20LL * T) * 8 + (4LL * T + 2LL * T + 16LL * T) * 4 +
               (T + 1LL) * 8 + (ndest + 1LL + A->num_terms) * 4;
    return A;
}

void assembly_refill(Assembly& A, int nfreq, const double* omegas, int cond, double* values_dev,
                     double* rhs_dev, cudaStream_t stream) {
    if (nfreq < 1) throw Error(APHI_ERR_BAD_SHAPE, "refill: no frequency given");
    for (int f = 0; f < nfreq; ++f) {
        std::complex<double> r, c;
        bool sym = false;
        formulation_scales_host(cond, omegas[f], r, c, sym);
        if (A.upper_only && !sym)
            throw Error(APHI_ERR_BAD_SHAPE,
                        "refill: this conditioning does not give a symmetric matrix, so only half of "
                        "it cannot be stored. Its (Phi,A) block is j*omega times its (A,Phi) block. "
                        "Use row_scaled or scaled_phi for symmetric storage.");
    }
    const int chunk = std::min(nfreq, kMaxBatchOmegas);
    if (A.terms_capacity < chunk) {
        if (A.d_terms) APHI_CUDA(cudaFree(A.d_terms));
        A.d_terms = nullptr;
        APHI_CUDA(cudaMalloc(&A.d_terms, static_cast<size_t>(chunk) * A.num_terms * sizeof(cplx)));
        A.terms_capacity = chunk;
    }
    TetArgs ta{A.T, A.upper_only ? 1 : 0, A.d_xyz, A.d_tets, A.d_visit_tet, A.d_visit_body,
               A.d_material, A.d_tet_idx, A.d_tet_coeff, A.d_tet_fixed, A.d_term_off, A.d_err};
    PortArgs pa{A.num_ports, A.d_port_current, A.d_port_amp, A.d_port_value, A.tet_terms};
    const Quad q = quad_points();
    for (int f0 = 0; f0 < nfreq; f0 += chunk) {
        Omegas om{};
        om.n = std::min(chunk, nfreq - f0);
        for (int i = 0; i < om.n; ++i) om.w[i] = omegas[f0 + i];
        cplx* terms = reinterpret_cast<cplx*>(A.d_terms);
        if (A.T > 0) {
            k_tet_terms<<<ceil_div(A.T, kTetWarps), 32 * kTetWarps, 0, stream>>>(ta, om, cond, q, terms);
            APHI_CHECK_LAUNCH();
        }
        if (A.num_ports > 0) {
            k_port_terms<<<1, 64, 0, stream>>>(pa, om, cond, terms);
            APHI_CHECK_LAUNCH();
        }
        const int ndest = A.nnz + A.N;
        const int spb = kSlotThreads / om.n;
        k_slot_sum<<<ceil_div(ndest, spb), kSlotThreads, 0, stream>>>(
            ndest, A.nnz, A.N, om.n, A.d_dest_ptr, A.d_dest_terms, terms,
            reinterpret_cast<cplx*>(values_dev) + static_cast<long long>(f0) * A.nnz,
            reinterpret_cast<cplx*>(rhs_dev) + static_cast<long long>(f0) * A.N);
        APHI_CHECK_LAUNCH();
    }
}

void assembly_check_errors(Assembly& A, cudaStream_t stream) {
    int h[4] = {0, 0, 0, 0};
    APHI_CUDA(cudaMemcpyAsync(h, A.d_err, sizeof(h), cudaMemcpyDeviceToHost, stream));
    APHI_CUDA(cudaStreamSynchronize(stream));
    if (h[0] || h[1]) {
        APHI_CUDA(cudaMemsetAsync(A.d_err, 0, sizeof(h), stream));
        if (h[0]) throw Error(APHI_ERR_DEGENERATE_TET, "compute_tet_geometry: degenerate (zero-volume) tet");
        throw Error(APHI_ERR_PATTERN_MISMATCH, "refill: a tet produced a different number of terms than planned");
    }
}

void element_blocks_host(int ntets, const double* xyz, double nu, const double* alpha,
                         const double* beta, double* aa, double* ap, double* pp) {
    double* d_xyz = upload(xyz, 12LL * ntets);
    cplx *d_aa = nullptr, *d_ap = nullptr, *d_pp = nullptr;
    int* d_err = nullptr;
    APHI_CUDA(cudaMalloc(&d_aa, 36LL * ntets * sizeof(cplx)));
    APHI_CUDA(cudaMalloc(&d_ap, 60LL * ntets * sizeof(cplx)));
    APHI_CUDA(cudaMalloc(&d_pp, 100LL * ntets * sizeof(cplx)));
    APHI_CUDA(cudaMalloc(&d_err, sizeof(int)));
    APHI_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    Coeff c{nu, cplx{alpha[0], alpha[1]}, cplx{beta[0], beta[1]}};
    k_element_blocks<<<ceil_div(ntets, 64), 64>>>(ntets, d_xyz, c, quad_points(), d_aa, d_ap, d_pp, d_err);
    APHI_CHECK_LAUNCH();
    int err = 0;
    APHI_CUDA(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    APHI_CUDA(cudaMemcpy(aa, d_aa, 36LL * ntets * sizeof(cplx), cudaMemcpyDeviceToHost));
    APHI_CUDA(cudaMemcpy(ap, d_ap, 60LL * ntets * sizeof(cplx), cudaMemcpyDeviceToHost));
    APHI_CUDA(cudaMemcpy(pp, d_pp, 100LL * ntets * sizeof(cplx), cudaMemcpyDeviceToHost));
    cudaFree(d_xyz);
    cudaFree(d_aa);
    cudaFree(d_ap);
    cudaFree(d_pp);
    cudaFree(d_err);
    if (err) throw Error(APHI_ERR_DEGENERATE_TET, "compute_tet_geometry: degenerate (zero-volume) tet");
}

// ---------------------------------------------------------------- post-solve fields
// compute_fields and the potential of potential_at_nodes (src/postprocess.cpp:
// 42-126, 223-486) on the device.
//   k_field_tets: one thread per tet. Geometry, A's and Phi's coefficients
//     for this tet (a cut's side already resolved by the tet's DOF table),
//     B = curl A (constant), A and E = -j w A - grad Phi at the centroid and
//     at each of the ten P2 nodes, J = sigma E. The node values go, with the
//     tet's volume, to a contribution array.
//   k_field_nodes: one thread per P2 node sums its contributions in
//     increasing tet order -- the reference's accumulation order -- with the
//     reference's side selection (E over the most conducting tets, B over the
//     most permeable), normalises each by its own weight, and forms J and H.
// Every operation is the reference's, in its order, rounded explicitly.
namespace {

constexpr int kFieldContrib = 13;  // volume, A (3 complex), E (3 complex)

struct FieldArgs {
    int T, P, nv;
    const double* xyz;
    const int* tets;
    const int* tet_edges;
    const int* body_of_tet;
    const double* material;
    const int* tet_idx;
    const double* tet_coeff;
    const double* tet_fixed;
    const cplx* x;
    cplx scale, mjw;
    double* contrib;
    const int* inc_ptr;
    const int* inc;
    const double* sig_max;
    const double* mu_max;
    const unsigned char* sig_uniform;
    const unsigned char* mu_uniform;
    int* err;
};

__device__ __forceinline__ void cross_rn(const double* a, const double* b, double* out) {
    out[0] = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
    out[1] = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
    out[2] = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
}

// A and E of one tet at barycentric point L.
__device__ void field_at(const Geometry& g, const cplx (&a)[6], const double (&sgn)[6], const cplx (&ph)[10],
                         cplx mjw, const double* L, cplx (&av)[3], cplx (&ev)[3]) {
    cplx gp[3];
    for (int i = 0; i < 3; ++i) av[i] = gp[i] = cplx{0.0, 0.0};
    for (int k = 0; k < 6; ++k) {
        double w[3];
        whitney(g, k, L, w);
        for (int i = 0; i < 3; ++i) av[i] = cadd_exact(av[i], cscale_exact(a[k], __dmul_rn(w[i], sgn[k])));
    }
    for (int n = 0; n < 10; ++n) {
        double gr[3];
        p2_grad(g, n, L, gr);
        for (int i = 0; i < 3; ++i) gp[i] = cadd_exact(gp[i], cscale_exact(ph[n], gr[i]));
    }
    for (int i = 0; i < 3; ++i) {
        const cplx t = cmul_exact(mjw, av[i]);
        ev[i] = cplx{__dsub_rn(t.re, gp[i].re), __dsub_rn(t.im, gp[i].im)};
    }
}

__global__ void __launch_bounds__(128) k_field_tets(FieldArgs A, cplx* a_tet, cplx* b_tet, cplx* e_tet, cplx* j_tet,
                                                    double* sigma_tet) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.T) return;
    double p[4][3];
    for (int q = 0; q < 4; ++q) {
        const int node = A.tets[4LL * t + q];
        for (int k = 0; k < 3; ++k) p[q][k] = A.xyz[3LL * node + k];
    }
    Geometry g;
    if (!tet_geometry(p, g)) {
        atomicExch(A.err, 1);
        return;
    }
    // A: the raw global unknown of each live edge; the edge sign goes with the
    // basis function (whitney_edge_value_global).
    cplx a[6];
    double sgn[6];
    for (int k = 0; k < 6; ++k) {
        const int idx = A.tet_idx[16LL * t + k];
        sgn[k] = A.tet_coeff[16LL * t + k];
        a[k] = idx >= 0 ? A.x[idx] : cplx{0.0, 0.0};
    }
    // Phi: (scale * coeff) * x for an unknown, the prescribed value otherwise.
    cplx ph[10];
    for (int n = 0; n < 10; ++n) {
        const int idx = A.tet_idx[16LL * t + 6 + n];
        if (idx >= 0)
            ph[n] = cmul_exact(cscale_exact(A.scale, A.tet_coeff[16LL * t + 6 + n]), A.x[idx]);
        else
            ph[n] = cplx{A.tet_fixed[20LL * t + 2 * n], A.tet_fixed[20LL * t + 2 * n + 1]};
    }
    // B = curl A = sum_e a_e * 2 (grad L_i x grad L_j) * sign_e.
    cplx b[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int k = 0; k < 6; ++k) {
        double c[3];
        cross_rn(g.grad[c_edge_verts[k][0]], g.grad[c_edge_verts[k][1]], c);
        for (int i = 0; i < 3; ++i) b[i] = cadd_exact(b[i], cscale_exact(a[k], __dmul_rn(__dmul_rn(c[i], 2.0), sgn[k])));
    }
    const int body = A.body_of_tet[t];
    const double sigma = A.material[3 * body];
    sigma_tet[t] = sigma;
    cplx av[3], ev[3];
    const double Lc[4] = {0.25, 0.25, 0.25, 0.25};
    field_at(g, a, sgn, ph, A.mjw, Lc, av, ev);
    for (int i = 0; i < 3; ++i) {
        a_tet[3LL * t + i] = av[i];
        b_tet[3LL * t + i] = b[i];
        e_tet[3LL * t + i] = ev[i];
        j_tet[3LL * t + i] = cscale_exact(ev[i], sigma);
    }
    const double vol = g.volume;
    for (int k = 0; k < 10; ++k) {
        double L[4] = {0.0, 0.0, 0.0, 0.0};
        if (k < 4) {
            L[k] = 1.0;
        } else {
            L[c_edge_verts[k - 4][0]] = 0.5;
            L[c_edge_verts[k - 4][1]] = 0.5;
        }
        field_at(g, a, sgn, ph, A.mjw, L, av, ev);
        double* o = A.contrib + (10LL * t + k) * kFieldContrib;
        o[0] = vol;
        for (int i = 0; i < 3; ++i) {
            o[1 + 2 * i] = av[i].re;
            o[2 + 2 * i] = av[i].im;
            o[7 + 2 * i] = ev[i].re;
            o[8 + 2 * i] = ev[i].im;
        }
    }
}

__global__ void __launch_bounds__(256) k_field_nodes(FieldArgs A, const cplx* b_tet, const double* sigma_tet,
                                                     cplx* phi_node, cplx* a_node, cplx* b_node, cplx* h_node,
                                                     cplx* e_node, cplx* j_node, double* vertex_weight,
                                                     unsigned char* on_interface) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= A.P) return;
    const bool sig_u = A.sig_uniform[u] != 0, mu_u = A.mu_uniform[u] != 0;
    double vw = 0.0, ew = 0.0, bw = 0.0;
    cplx an[3], en[3], bn[3];
    for (int i = 0; i < 3; ++i) an[i] = en[i] = bn[i] = cplx{0.0, 0.0};
    cplx phi{0.0, 0.0};
    bool phi_unknown = false, phi_fixed = false;
    for (int q = A.inc_ptr[u]; q < A.inc_ptr[u + 1]; ++q) {
        const int e = A.inc[q];
        const int t = e / 10, k = e % 10;
        const double* c = A.contrib + static_cast<long long>(e) * kFieldContrib;
        const double vol = c[0];
        vw = __dadd_rn(vw, vol);
        for (int i = 0; i < 3; ++i) an[i] = cadd_exact(an[i], cscale_exact(cplx{c[1 + 2 * i], c[2 + 2 * i]}, vol));
        if (sig_u || sigma_tet[t] == A.sig_max[u]) {
            ew = __dadd_rn(ew, vol);
            for (int i = 0; i < 3; ++i) en[i] = cadd_exact(en[i], cscale_exact(cplx{c[7 + 2 * i], c[8 + 2 * i]}, vol));
        }
        const double mu = __dmul_rn(kMu0, A.material[3 * A.body_of_tet[t] + 2]);
        if (mu_u || mu == A.mu_max[u]) {
            bw = __dadd_rn(bw, vol);
            for (int i = 0; i < 3; ++i) bn[i] = cadd_exact(bn[i], cscale_exact(b_tet[3LL * t + i], vol));
        }
        // Phi at the node: the unknown any incident tet reads (a cut's plus
        // side), else the first nonzero prescribed value.
        {
            const int idx = A.tet_idx[16LL * t + 6 + k];
            if (idx >= 0 && !phi_unknown) {
                phi = cmul_exact(A.scale, A.x[idx]);
                phi_unknown = true;
            } else if (idx < 0 && !phi_unknown && !phi_fixed) {
                const cplx f{A.tet_fixed[20LL * t + 2 * k], A.tet_fixed[20LL * t + 2 * k + 1]};
                if (f.re != 0.0 || f.im != 0.0) {
                    phi = f;
                    phi_fixed = true;
                }
            }
        }
    }
    phi_node[u] = phi;
    vertex_weight[u] = vw;
    on_interface[u] = (A.inc_ptr[u + 1] > A.inc_ptr[u]) && (!sig_u || !mu_u) ? 1 : 0;
    if (vw > 0.0) {
        for (int i = 0; i < 3; ++i) an[i] = cplx{__ddiv_rn(an[i].re, vw), __ddiv_rn(an[i].im, vw)};
        if (ew > 0.0)
            for (int i = 0; i < 3; ++i) en[i] = cplx{__ddiv_rn(en[i].re, ew), __ddiv_rn(en[i].im, ew)};
        if (bw > 0.0)
            for (int i = 0; i < 3; ++i) bn[i] = cplx{__ddiv_rn(bn[i].re, bw), __ddiv_rn(bn[i].im, bw)};
    }
    const double nu_node = vw > 0.0 ? __ddiv_rn(1.0, A.mu_max[u]) : 0.0;
    const double smax = vw > 0.0 ? A.sig_max[u] : 0.0;
    for (int i = 0; i < 3; ++i) {
        a_node[3LL * u + i] = an[i];
        e_node[3LL * u + i] = en[i];
        b_node[3LL * u + i] = bn[i];
        j_node[3LL * u + i] = vw > 0.0 ? cscale_exact(en[i], smax) : cplx{0.0, 0.0};
        h_node[3LL * u + i] = vw > 0.0 ? cscale_exact(bn[i], nu_node) : cplx{0.0, 0.0};
    }
}

}  // namespace

Fields::~Fields() {
    for (void* p : {(void*)d_tet_edges, (void*)d_body_of_tet, (void*)d_inc_ptr, (void*)d_inc, (void*)d_sig_max,
                    (void*)d_mu_max, (void*)d_sig_uniform, (void*)d_mu_uniform, (void*)d_contrib, (void*)d_err})
        if (p) cudaFree(p);
}

std::unique_ptr<Fields> fields_create(const Assembly& A, int num_nodes, int num_edges, const int* tet_edges) {
    if (num_nodes < 1 || num_edges < 0 || (A.T > 0 && !tet_edges))
        throw Error(APHI_ERR_BAD_SHAPE, "fields: need the mesh's node and edge counts and 6 edges per tet");
    auto F = std::make_unique<Fields>();
    F->A = &A;
    F->T = A.T;
    F->nv = num_nodes;
    F->ne = num_edges;
    F->P = num_nodes + num_edges;
    const int T = A.T, P = F->P;
    std::vector<int> tets(4LL * T), visit_tet(T), visit_body(T);
    std::vector<double> material(3LL * A.num_bodies);
    APHI_CUDA(cudaMemcpy(tets.data(), A.d_tets, tets.size() * sizeof(int), cudaMemcpyDeviceToHost));
    APHI_CUDA(cudaMemcpy(visit_tet.data(), A.d_visit_tet, visit_tet.size() * sizeof(int), cudaMemcpyDeviceToHost));
    APHI_CUDA(cudaMemcpy(visit_body.data(), A.d_visit_body, visit_body.size() * sizeof(int), cudaMemcpyDeviceToHost));
    APHI_CUDA(cudaMemcpy(material.data(), A.d_material, material.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<int> body_of_tet(T, -1);
    for (int v = 0; v < T; ++v) body_of_tet[visit_tet[v]] = visit_body[v];
    for (int t = 0; t < T; ++t) {
        if (body_of_tet[t] < 0) throw Error(APHI_ERR_BAD_SHAPE, "fields: a tet belongs to no body");
        for (int q = 0; q < 4; ++q)
            if (tets[4LL * t + q] < 0 || tets[4LL * t + q] >= num_nodes)
                throw Error(APHI_ERR_BAD_SHAPE, "fields: a tet names a node past num_nodes");
        for (int q = 0; q < 6; ++q)
            if (tet_edges[6LL * t + q] < 0 || tet_edges[6LL * t + q] >= num_edges)
                throw Error(APHI_ERR_BAD_SHAPE, "fields: a tet names an edge past num_edges");
    }
    // P2 node -> (tet, local node) in increasing tet order, and each node's
    // extreme conductivity and permeability over its tets.
    auto node_of = [&](int t, int k) { return k < 4 ? tets[4LL * t + k] : num_nodes + tet_edges[6LL * t + k - 4]; };
    std::vector<int> ptr(P + 1, 0);
    constexpr double kInf = std::numeric_limits<double>::infinity();
    std::vector<double> smin(P, kInf), smax(P, -kInf), mmin(P, kInf), mmax(P, -kInf);
    for (int t = 0; t < T; ++t) {
        const double s = material[3 * body_of_tet[t]], m = kMu0 * material[3 * body_of_tet[t] + 2];
        for (int k = 0; k < 10; ++k) {
            const int u = node_of(t, k);
            ++ptr[u + 1];
            smin[u] = std::min(smin[u], s);
            smax[u] = std::max(smax[u], s);
            mmin[u] = std::min(mmin[u], m);
            mmax[u] = std::max(mmax[u], m);
        }
    }
    for (int u = 0; u < P; ++u) ptr[u + 1] += ptr[u];
    std::vector<int> inc(ptr[P]), cur(ptr.begin(), ptr.end() - 1);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 10; ++k) inc[cur[node_of(t, k)]++] = 10 * t + k;
    std::vector<unsigned char> su(P), mu(P);
    for (int u = 0; u < P; ++u) {
        su[u] = smin[u] == smax[u];
        mu[u] = mmin[u] == mmax[u];
        if (ptr[u + 1] == ptr[u]) {
            ++F->orphans;
            smax[u] = mmax[u] = 1.0;  // no tet: never read
        } else if (!su[u] || !mu[u]) {
            ++F->interface_nodes;
        }
    }
    F->d_tet_edges = upload(tet_edges, 6LL * T);
    F->d_body_of_tet = upload(body_of_tet.data(), body_of_tet.size());
    F->d_inc_ptr = upload(ptr.data(), ptr.size());
    F->d_inc = upload(inc.data(), inc.size());
    F->d_sig_max = upload(smax.data(), smax.size());
    F->d_mu_max = upload(mmax.data(), mmax.size());
    F->d_sig_uniform = upload(su.data(), su.size());
    F->d_mu_uniform = upload(mu.data(), mu.size());
    APHI_CUDA(cudaMalloc(&F->d_contrib, std::max<size_t>(1, 10ULL * T * kFieldContrib) * sizeof(double)));
    APHI_CUDA(cudaMalloc(&F->d_err, sizeof(int)));
    APHI_CUDA(cudaMemset(F->d_err, 0, sizeof(int)));
    return F;
}

void fields_compute(Fields& F, double omega, int conditioning, const double* x, const FieldsOut& o, cudaStream_t st) {
    const Assembly& A = *F.A;
    if (!x || !o.phi_node || !o.a_tet || !o.b_tet || !o.e_tet || !o.j_tet || !o.sigma_tet || !o.a_node ||
        !o.b_node || !o.h_node || !o.e_node || !o.j_node || !o.vertex_weight || !o.on_interface)
        throw Error(APHI_ERR_INVALID, "fields: null solution or output array");
    if (conditioning != APHI_COND_NATURAL && conditioning != APHI_COND_ROW_SCALED && conditioning != APHI_COND_SCALED_PHI)
        throw Error(APHI_ERR_BAD_SHAPE, "fields: unknown conditioning");
    // Member by member: a braced initializer here (with the conditional
    // complex scale) crashed the device front end of CUDA 12.9.
    FieldArgs fa;
    fa.T = F.T;
    fa.P = F.P;
    fa.nv = F.nv;
    fa.xyz = A.d_xyz;
    fa.tets = A.d_tets;
    fa.tet_edges = F.d_tet_edges;
    fa.body_of_tet = F.d_body_of_tet;
    fa.material = A.d_material;
    fa.tet_idx = A.d_tet_idx;
    fa.tet_coeff = A.d_tet_coeff;
    fa.tet_fixed = A.d_tet_fixed;
    fa.x = reinterpret_cast<const cplx*>(x);
    fa.scale.re = conditioning == APHI_COND_SCALED_PHI ? 0.0 : 1.0;  // j omega under ScaledPhi
    fa.scale.im = conditioning == APHI_COND_SCALED_PHI ? omega : 0.0;
    fa.mjw.re = -0.0;                                                 // -(j omega)
    fa.mjw.im = -omega;
    fa.contrib = F.d_contrib;
    fa.inc_ptr = F.d_inc_ptr;
    fa.inc = F.d_inc;
    fa.sig_max = F.d_sig_max;
    fa.mu_max = F.d_mu_max;
    fa.sig_uniform = F.d_sig_uniform;
    fa.mu_uniform = F.d_mu_uniform;
    fa.err = F.d_err;
    if (F.T > 0) {
        k_field_tets<<<ceil_div(F.T, 128), 128, 0, st>>>(fa, reinterpret_cast<cplx*>(o.a_tet),
                                                        reinterpret_cast<cplx*>(o.b_tet), reinterpret_cast<cplx*>(o.e_tet),
                                                        reinterpret_cast<cplx*>(o.j_tet), o.sigma_tet);
        APHI_CHECK_LAUNCH();
    }
    k_field_nodes<<<ceil_div(std::max(F.P, 1), 256), 256, 0, st>>>(
        fa, reinterpret_cast<const cplx*>(o.b_tet), o.sigma_tet, reinterpret_cast<cplx*>(o.phi_node),
        reinterpret_cast<cplx*>(o.a_node), reinterpret_cast<cplx*>(o.b_node), reinterpret_cast<cplx*>(o.h_node),
        reinterpret_cast<cplx*>(o.e_node), reinterpret_cast<cplx*>(o.j_node), o.vertex_weight, o.on_interface);
    APHI_CHECK_LAUNCH();
    int err = 0;
    APHI_CUDA(cudaMemcpyAsync(&err, F.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    APHI_CUDA(cudaStreamSynchronize(st));
    if (err) {
        APHI_CUDA(cudaMemsetAsync(F.d_err, 0, sizeof(int), st));
        throw Error(APHI_ERR_DEGENERATE_TET, "compute_fields: degenerate (zero-volume) tet");
    }
}

}  // namespace aphi_b200
