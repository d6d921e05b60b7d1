// Host-side fill-reducing and bandwidth orderings (new -> old permutations).
#pragma once

#include <vector>

namespace aphi_b200 {

// The symmetric adjacency of an upper CSR pattern, as src/ordering.cpp:58-98
// builds it: each vertex's neighbours ascending, no duplicates, no diagonal.
void adjacency_from_upper(int n, const int* row_ptr, const int* col_idx, std::vector<int>& off,
                          std::vector<int>& nbr);

// The reference's approximate minimum degree (Ordering::ApproximateMinimumDegree),
// bit for bit (amd.cpp).
void reference_amd(int n, const int* row_ptr, const int* col_idx, int* perm);

// The reference's reverse Cuthill-McKee (Ordering::ReverseCuthillMcKee), bit
// for bit (rcm.cpp).
void reference_rcm(int n, const int* row_ptr, const int* col_idx, int* perm);

// Geometric nested dissection over the unknowns' positions (ordering.cpp).
void nested_dissection(int n, const int* row_ptr, const int* col_idx, const double* xyz, int leaf, int* perm);

}  // namespace aphi_b200
