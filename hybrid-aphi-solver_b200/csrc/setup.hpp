// Per-mesh setup on the device (setup.cu): the sparsity pattern and the
// scatter's slot -> term maps.
#pragma once

#include "assembly.hpp"

namespace aphi_b200 {

// build_sparsity (src/sparsity.cpp:19-136) from the tets' 16 DOF indices
// each (-1: none) plus a diagonal entry for each of diag_rows (the voltage
// ports' constraint rows). Writes row_ptr[N+1] and col_idx[nnz] when
// col_idx is non-null and capacity >= nnz; returns nnz either way.
long long pattern_build(int N, int T, const int* tet_idx, int nd, const int* diag_rows, bool upper, int* row_ptr,
                        int* col_idx, long long capacity);

// The assembly's term offsets per visited tet and its slot -> term lists,
// built on the device (A.d_tet_idx and A.d_tet_fixed already uploaded):
// fills A.d_term_off, A.d_dest_ptr, A.d_dest_terms, A.tet_terms, A.num_terms.
void assembly_maps_on_device(Assembly& A, const aphi_assembly_desc& d, const int* visit_tet_host);

}  // namespace aphi_b200
