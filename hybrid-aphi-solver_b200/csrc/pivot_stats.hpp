// Per-entry factorization statistics from the pivots, as the reference
// computes them (FactorStats, src/factorization.cpp:180-210).
#pragma once

#include "aphi_b200.h"

namespace aphi_b200 {

// dref: B x n complex pivots in the caller's column order; dscale: B x n
// equilibration scales. For each entry b: walk the pivots in column order
// until the first with |D| <= pivot_floor; out[b] gets ok, columns_done, the
// smallest and largest |D| seen, the equilibration range, nnz_l and ms, and
// kmax[b] that column (left as is when none fails). Entries run on several
// host threads when the walk is long; each entry's numbers are those of the
// sequential walk. Returns whether any entry stopped at the floor.
bool pivot_stats(int n, int B, const double* dref, const double* dscale, double pivot_floor, double ms,
                 long long nnz_l, aphi_factor_stats* out, int* kmax);

}  // namespace aphi_b200
