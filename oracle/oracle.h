/*
 * The oracle: a plain-C restatement of the reference's per-frequency numeric
 * path, used ONLY as the checker by the test suite, smoke() and bench.py's
 * CPU-baseline arm. Never linked into, or called by, the product.
 *
 * Complex numbers are C99 `double complex`, whose multiplication and division
 * the compiler lowers exactly as it lowers std::complex<double>, so the
 * element kernels and the scatter reproduce the reference's bits.
 *
 * Pinned by tests/test_oracle.py against the golden fixtures in
 * tests/golden/ (made from the reference by tests/golden/make_golden.py) and
 * against the reference compiled from its own sources (oracle/_ref).
 */
#ifndef APHI_ORACLE_H
#define APHI_ORACLE_H

#include <stdint.h>

/* element_coefficients, src/element_matrix.cpp:10-25: out = nu, alpha (re, im), beta (re, im). */
void or_coefficients(double sigma, double eps_r, double mu_r, double omega, double* out5);

/* kernel_AA / kernel_APhi / kernel_PhiPhi (src/element_matrix.cpp:27-115) for
 * one tet (xyz[12]); blocks row-major, complex interleaved. Returns -1 for a
 * degenerate tet (src/basis_functions.cpp:30-32). */
int or_element_blocks(const double* xyz, double nu, const double* alpha, const double* beta, double* aa,
                      double* ap, double* pp);

/* formulation_scales, src/assembly.cpp:12-45: rc = r (re, im), c (re, im).
 * Returns -1 where the reference throws (row_scaled / scaled_phi at omega 0). */
int or_formulation_scales(int conditioning, double omega, double* rc);

/* refill(SymmetricSystem&) / scatter_into, src/assembly.cpp:255-422, over the
 * per-tet DOF tables (DofMap::local_dofs) and the upper CSR pattern. Bodies are
 * visited in order, each body's tets as listed. Returns -1 (refused
 * conditioning), -2 (no slot: pattern and scatter disagree), -3 (degenerate tet). */
int or_refill(int num_tets, const double* xyz, const int* tets, const int* tet_idx, const double* tet_coeff,
              const double* tet_fixed, int num_bodies, const double* material, const int* body_ptr,
              const int* body_tets, int num_ports, const int* port_current, const int* port_row,
              const double* port_amplitude, const double* port_value, int n, const int* row_ptr,
              const int* col_idx, double omega, int conditioning, double* values, double* rhs);

/* compute_symmetric_equilibration (upper-triangle overload),
 * src/equilibration.cpp:94-139. */
void or_equilibration(int n, const int* row_ptr, const int* col_idx, const double* values, int iterations,
                      double* d);

/* factorize_ldlt, src/factorization.cpp:109-218 (with permuted_lower :13-74
 * and ereach :86-105): up-looking LDL^T of P A P^T, no pivoting, no
 * conjugation. values are the (possibly already scaled) upper CSR values.
 * Outputs sized from col_count: col_ptr[n+1], row_index/lvalue[sum(col_count)-n],
 * diag[n]. stats[0..5]: ok, columns_done, smallest, largest, largest multiplier, nnz.
 * Returns 0, 1 (pivot at or below the floor), -1 (column overflow). */
int or_factorize(int n, const int* row_ptr, const int* col_idx, const double* values, const int* perm,
                 const int* parent, const int* col_count, double pivot_floor, int* col_ptr, int* row_index,
                 double* lvalue, double* diag, double* stats);

/* solve, src/factorization.cpp:254-313: x = A^-1 b through the factor of P A P^T.
 * Returns -1 on a zero D. */
int or_solve(int n, const int* col_ptr, const int* row_index, const double* lvalue, const double* diag,
             const int* perm, const double* b, double* x);

/* relative_residual and backward_error, src/factorization.cpp:315-329, :401-416. */
void or_residuals(int n, const int* row_ptr, const int* col_idx, const double* values, const double* x,
                  const double* b, double* out2);

/* solve_symmetric, src/factorization.cpp:332-398, given the analysis
 * (perm, parent, col_count). report[0..9]: ok, backward_error, residual,
 * equil_min, equil_max, smallest_pivot, largest_pivot, largest_multiplier,
 * factor_nnz, columns_done. Returns 0, or 1 when the factorization stopped. */
int or_solve_symmetric(int n, const int* row_ptr, const int* col_idx, const double* values, const double* b,
                       const int* perm, const int* parent, const int* col_count, int equil_iters,
                       double pivot_floor, double* x, double* report);

#endif
