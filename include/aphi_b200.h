/*
 * aphi_b200 -- C ABI of the B200 (sm_100a) implementation of the A-Phi
 * solver's per-frequency numeric hot path.
 *
 * Every entry point takes plain pointers and sizes, never throws, and returns
 * an int status (APHI_OK or one of the APHI_ERR_* codes below); the message of
 * the last failure on the calling thread is in aphi_last_error(). Complex
 * numbers are interleaved (re, im) doubles or floats. "dev" pointers are CUDA
 * device pointers; "stream" is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).
 *
 * The interfaces replaced, in the reference (namespace aphi_solver):
 *   include/aphi_solver/assembly.hpp       formulation_scales, ScatterMap,
 *                                          refill (both overloads),
 *                                          make_symmetric_system, assemble
 *   include/aphi_solver/factorization.hpp  permuted_lower, factorize_ldlt,
 *                                          solve_in_place, solve,
 *                                          relative_residual, backward_error,
 *                                          solve_symmetric, reconstruct
 *   include/aphi_solver/equilibration.hpp  compute_symmetric_equilibration
 *                                          (upper-triangle overload)
 * Each declaration cites the reference function it stands in for.
 */
#ifndef APHI_B200_H
#define APHI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------
 * The drop-in C++ layer maps these back onto the reference's conventions:
 * BAD_SHAPE -> std::invalid_argument, PATTERN_MISMATCH and ZERO_PIVOT ->
 * std::logic_error, PIVOT_FLOOR -> `return false` with stats.ok == false. */
#define APHI_OK 0
#define APHI_ERR_BAD_SHAPE 1        /* sizes/shapes disagree; also refused conditioning */
#define APHI_ERR_PATTERN_MISMATCH 2 /* symbolic and numeric passes disagree (no slot, ...) */
#define APHI_ERR_PIVOT_FLOOR 3      /* |D[j]| <= pivot_floor: factorization stopped */
#define APHI_ERR_NAN 4              /* non-finite value met */
#define APHI_ERR_IR_STALL 5         /* refinement stalled (FP64 fallback is taken if enabled) */
#define APHI_ERR_TIMEOUT 6          /* a bounded device wait gave up */
#define APHI_ERR_OOM 7              /* device allocation failed */
#define APHI_ERR_ADMISSION 8        /* serving: request rejected by HBM admission */
#define APHI_ERR_CUDA 9             /* any other CUDA error */
#define APHI_ERR_ZERO_PIVOT 10      /* a solve met D[j] == 0 */
#define APHI_ERR_DEGENERATE_TET 11  /* zero-volume tetrahedron */
#define APHI_ERR_INVALID 12         /* null handle or argument */

const char* aphi_status_string(int status);
const char* aphi_last_error(void);
/* Kernels this library has launched in this process (all threads). */
int64_t aphi_launch_count(void);

/* Conditioning, as include/aphi_solver/problem.hpp:58-62 numbers it. */
#define APHI_COND_NATURAL 0
#define APHI_COND_ROW_SCALED 1
#define APHI_COND_SCALED_PHI 2

/* ---- synthetic workloads --------------------------------------------------
 * The cylinder-in-box problem generated on the host in the layouts the
 * device path consumes: n^3 cells x 6 Kuhn tets, conductor within r = 0.2 of
 * the z axis through (0.5, 0.5), voltage ports v_top on z = 1 and 0 V on
 * z = 0. Not a reference interface: the reference builds the same inputs
 * with its mesh, binding, DOF-map and sparsity passes. */
typedef struct aphi_workload aphi_workload;
int aphi_workload_cylinder(int cells, double v_top, int full_wave, aphi_workload** out);
/* The multiply-connected case: the same box and split (cells even), a copper
 * torus (major radius 0.25, minor 0.04, axis z, centred in the box) and one
 * internal current port of `current` A on the cut y = 0.5, x > 0.5 (its
 * conductor-conductor faces), current direction hint +y; Phi on the
 * conductor only. */
int aphi_workload_torus(int cells, double current, aphi_workload** out);
void aphi_workload_free(aphi_workload* w);
/* sizes[0..9]: nodes, tets, edges, unknowns, nnz_upper, num_a, num_phi,
 * num_ports, num_bodies, num_terms (0 until an assembly is built) */
int aphi_workload_sizes(const aphi_workload* w, int64_t* sizes);
/* Read-only views into the workload's arrays (valid until aphi_workload_free).
 * name: "xyz" (double, 3/node), "tets" (int, 4/tet), "tet_idx" (int, 16/tet),
 * "tet_coeff" (double, 16/tet), "tet_fixed" (double, 20/tet), "material"
 * (double, 3/body), "body_ptr" (int), "body_tets" (int), "port_current",
 * "port_row" (int), "port_amplitude", "port_value" (double, 2/port),
 * "row_ptr", "col_idx" (int), "edges" (int, 2/edge), "edge_index",
 * "phi_index" (int), "tet_edges" (int, 6/tet), "body_of_tet" (int),
 * "dof_xyz" (double, 3/unknown: edge midpoints, P2 nodes, port terminals). */
int aphi_workload_array(const aphi_workload* w, const char* name, const void** data, int64_t* count);

/* Fill-reducing permutation (new -> old) by geometric nested dissection over
 * the unknowns' positions xyz (3 per unknown); parts of at most `leaf`
 * unknowns are numbered by minimum degree. Not a reference interface: the
 * reference orders with its own AMD (src/ordering.cpp:220-510), whose
 * permutation this library consumes unchanged when it is the caller; this
 * one serves standalone callers. */
int aphi_order_nested_dissection(int n, const int* row_ptr, const int* col_idx, const double* xyz, int leaf,
                                 int* perm);

/* The reference's approximate-minimum-degree permutation (new -> old) of an
 * upper-triangle pattern, reproduced bit for bit -- compute_ordering(pattern,
 * Ordering::ApproximateMinimumDegree), src/ordering.cpp:220-510 and :539-556 --
 * so a caller without the reference's host code factorizes in the reference's
 * column order. */
int aphi_order_amd(int n, const int* row_ptr, const int* col_idx, int* perm);
/* The reference's reverse Cuthill-McKee ordering (compute_ordering with
 * Ordering::ReverseCuthillMcKee, src/ordering.cpp:105-218 and :512-537), bit
 * for bit: the same arguments and output as aphi_order_amd. */
int aphi_order_rcm(int n, const int* row_ptr, const int* col_idx, int* perm);

/* ---- assembly: element fill + deterministic scatter -----------------------
 * Replaces refill(SymmetricSystem&, ...) and refill(AssembledSystem&, ...)
 * (src/assembly.cpp:453-494, scatter at :255-422), element_coefficients and
 * the three element kernels (src/element_matrix.cpp:10-115), and
 * ScatterMap::build (src/assembly.cpp:196-232), whose role here is played by a
 * slot -> contribution list built once per mesh. */
typedef struct {
    int num_nodes, num_tets, num_unknowns;
    const double* xyz;        /* 3 per node */
    const int* tets;          /* 4 per tet */
    const int* tet_idx;       /* 16 per tet: DofMap::local_dofs indices, -1 eliminated */
    const double* tet_coeff;  /* 16 per tet: orientation signs / 1 */
    const double* tet_fixed;  /* 20 per tet: prescribed Phi (complex), 0 when none */
    int num_bodies;
    const double* material;   /* sigma, eps_r, mu_r per body */
    const int* body_ptr;      /* num_bodies + 1 */
    const int* body_tets;     /* tets grouped by body, in the order refill visits them */
    int num_ports;
    const int* port_current;  /* 1 = current driven, 0 = voltage driven */
    const int* port_row;
    const double* port_amplitude; /* complex, BoundPort::amplitude */
    const double* port_value;     /* complex, DofMap::port_value */
    int upper_only;           /* pattern stores only col >= row */
    const int* row_ptr;       /* num_unknowns + 1 */
    const int* col_idx;
} aphi_assembly_desc;

typedef struct aphi_assembly aphi_assembly;
int aphi_assembly_create(const aphi_assembly_desc* desc, aphi_assembly** out);
/* The same assembly with its per-mesh maps built on the device instead of
 * the host: each tet's term destinations in the scatter's emission order and
 * their inversion into slot -> term lists (ScatterMap::build and its use by
 * scatter_into, src/assembly.cpp:196-232, :255-422). The maps equal
 * aphi_assembly_create's exactly (each list sorted by term index after an
 * atomic fill), so refill gives the same bits. A missing slot is refused with
 * PATTERN_MISMATCH naming the entry. */
int aphi_assembly_create_device_setup(const aphi_assembly_desc* desc, aphi_assembly** out);
/* Copies of the assembly's maps (any pointer may be NULL): term_off[T+1]
 * (terms per visited tet, prefix), dest_ptr[nnz+N+1], dest_terms[num_terms]. */
int aphi_assembly_maps(const aphi_assembly* a, int64_t* term_off, int* dest_ptr, int* dest_terms);
/* build_sparsity (src/sparsity.cpp:19-136) on the device: the upper (or full)
 * CSR pattern of every pair of each tet's unique live DOFs (tet_idx: 16 per
 * tet, -1 for none) plus a diagonal entry for each of diag_rows (voltage-port
 * constraint rows); rows sorted and unique. row_ptr[n+1]; col_idx holds
 * capacity entries; *nnz is always set, and BAD_SHAPE is returned when it
 * exceeds capacity (call again with a larger buffer). */
int aphi_pattern_build(int n, int num_tets, const int* tet_idx, int num_diag, const int* diag_rows, int upper_only,
                       int* row_ptr, int* col_idx, int64_t capacity, int64_t* nnz);
int aphi_assembly_destroy(aphi_assembly* a);
/* info[0..3]: nnz, unknowns, num_terms, device bytes held */
int aphi_assembly_info(const aphi_assembly* a, int64_t* info);
/* Formulation scales r, c (complex, 4 doubles) -- formulation_scales,
 * src/assembly.cpp:12-45. Returns BAD_SHAPE for row_scaled/scaled_phi at omega == 0. */
int aphi_formulation_scales(int conditioning, double omega, double* rc, int* symmetric);
/* One frequency: values_dev[2*nnz], rhs_dev[2*N] are overwritten (cleared, then
 * accumulated in the reference's order: bodies, tets, AA, A-Phi/Phi-A, Phi-Phi,
 * then port rows). */
int aphi_refill(aphi_assembly* a, double omega, int conditioning, double* values_dev,
                double* rhs_dev, void* stream);
/* nfreq frequencies in one launch pair: values_dev[nfreq][2*nnz], rhs_dev[nfreq][2*N]. */
int aphi_refill_batch(aphi_assembly* a, int nfreq, const double* omegas, int conditioning,
                      double* values_dev, double* rhs_dev, void* stream);
/* Host-buffer form of aphi_refill (copies in and out inside). */
int aphi_refill_host(aphi_assembly* a, double omega, int conditioning, double* values,
                     double* rhs);
/* Element blocks of ntets tets on the device (test hook for
 * kernel_AA/APhi/PhiPhi): xyz[12 per tet]; coefficients nu (real), alpha,
 * beta (complex) shared by all; outputs 36/60/100 complex per tet, host. */
int aphi_element_blocks(int ntets, const double* xyz, double nu, const double* alpha,
                        const double* beta, double* aa, double* ap, double* pp);
/* Element coefficients nu, alpha, beta (5 doubles) -- src/element_matrix.cpp:10-25. */
void aphi_element_coefficients(double sigma, double eps_r, double mu_r, double omega, double* out5);

/* ---- post-solve fields ----------------------------------------------------
 * compute_fields (src/postprocess.cpp:223-486, include/aphi_solver/
 * postprocess.hpp:298) and potential_at_nodes' values (:42-126) on the device,
 * over an assembly's mesh and DOF tables. P2 nodes are numbered as DofMap
 * numbers them: the mesh's vertices, then one per edge. Per tet: A and E at
 * the centroid, B = curl A (constant), J = sigma E, sigma. Per P2 node: Phi
 * (the plus side on a cut), and A, B, H, E, J averaged over the node's tets
 * with their volumes as weights -- E and J over the most conducting tets, B
 * and H over the most permeable -- in the reference's tet order. Complex
 * arrays are interleaved (re, im); vector fields are 3 complex per entry.
 * All outputs are device arrays the caller owns. */
typedef struct aphi_fields aphi_fields;
typedef struct {
    double* phi_node;              /* P complex */
    double* a_tet;                 /* T x 3 complex */
    double* b_tet;
    double* e_tet;
    double* j_tet;
    double* sigma_tet;             /* T */
    double* a_node;                /* P x 3 complex */
    double* b_node;
    double* h_node;
    double* e_node;
    double* j_node;
    double* vertex_weight;         /* P: summed volume of each node's tets */
    unsigned char* on_interface;   /* P: 1 where the node's tets are not all one material */
} aphi_fields_out;
/* tet_edges: 6 global edge numbers per tet (host, the mesh's tet_edges);
 * num_nodes / num_edges: the mesh's. The assembly must outlive the fields. */
int aphi_fields_create(const aphi_assembly* a, int num_nodes, int num_edges, const int* tet_edges,
                       aphi_fields** out);
int aphi_fields_destroy(aphi_fields* f);
/* sizes[0..5]: tets T, P2 nodes P, vertices, edges, interface nodes, nodes without a tet */
int aphi_fields_sizes(const aphi_fields* f, int64_t* sizes);
/* x_dev: the solution, N complex, laid out [a | phi | V]; conditioning as in
 * the solve (ScaledPhi's unknown is Phi / (j omega)). */
int aphi_fields_compute(aphi_fields* f, double omega, int conditioning, const double* x_dev,
                        const aphi_fields_out* out, void* stream);

/* ---- analysis: supernodal schedule from the reference's symbolic pass -----
 * Consumes the pattern and the reference's permutation (SolverAnalysis::
 * permutation, include/aphi_solver/symbolic.hpp:69-92), recomputes the
 * elimination tree and column counts (checked against the caller's when
 * given), post-orders the tree, groups columns into relaxed supernodes and
 * lays out the device factor. */
typedef struct {
    int relax_small;       /* always merge a child into its parent when both are at most this wide */
    double relax_fill;     /* otherwise merge while padded zeros stay below this fraction */
    int relax_max_width;   /* never grow a supernode past this many columns */
    int small_front;       /* fronts up to this many rows use the one-CTA kernel */
    int group4_rows;       /* fronts this tall apply their trailing updates 4 panels at a time (<= 0: 8192) */
    int group2_rows;       /* shorter fronts this tall, 2 panels at a time; shorter still, one (<= 0: all 2) */
    /* The same two thresholds for the tensor-core (FP32) factorization plan,
     * kept apart from the FP64 plan's: the grouping changes the FP32
     * factor's rounding, and with it how many refinement steps the stiffer
     * systems of a sweep need, or whether they converge at all, so the FP64
     * plan's grouping can be tuned for speed alone. (<= 0: 8192 / all 2.) */
    int tc_group4_rows;
    int tc_group2_rows;
} aphi_analysis_options;

typedef struct aphi_analysis aphi_analysis;
void aphi_analysis_default_options(aphi_analysis_options* o);
/* perm: new -> old (the reference's Permutation::perm). parent/col_count, when
 * non-NULL, are the reference's etree and column counts in the same
 * numbering; a disagreement returns PATTERN_MISMATCH. */
int aphi_analysis_create(int n, const int* row_ptr, const int* col_idx, const int* perm,
                         const int* parent, const int* col_count, const aphi_analysis_options* opt,
                         aphi_analysis** out);
int aphi_analysis_destroy(aphi_analysis* a);
/* info[0..11]: n, nnz_upper, nnz_L (incl. diagonal, unpadded), stored
 * entries (padded), supernodes, levels, max front rows, max supernode width,
 * flops (real, unpadded: 8 * sum c'(c'+1)/2), CB pool entries, device bytes
 * per factor (fp64), num roots */
int aphi_analysis_info(const aphi_analysis* a, double* info);
/* The elimination tree and column counts the analysis computed, in the
 * caller's permuted numbering. */
int aphi_analysis_etree(const aphi_analysis* a, int* parent, int* col_count);

/* ---- numeric factorization, solves and refinement --------------------------
 * A factor holds `batch` independent factorizations sharing one analysis
 * (frequency batching). precision: 64 = complex128 throughout (the plain
 * drop-in), 32 = complex64 factor with tensor-core updates, used with FP64
 * iterative refinement. */
#define APHI_PREC_FP64 64
#define APHI_PREC_FP32 32

typedef struct aphi_factor aphi_factor;
/* A factor holds `batch` numeric factorizations of one analysis (its
 * capacity); every buffer is sized for it once. The contribution-block pool,
 * live only during a factorization, is a workspace of the analysis shared by
 * all its factors (sized for the largest): factorizations of one analysis take
 * turns, each holding it until its stream is done with the pool, so they may
 * come from several host threads and streams. */
int aphi_factor_create(const aphi_analysis* an, int precision, int batch, aphi_factor** out);
int aphi_factor_destroy(aphi_factor* f);
/* Sets how many entries (1..capacity) later calls process, without
 * reallocating: values, right-hand sides and solutions then hold `batch`
 * entries. Discards the current factorization. For continuous batching,
 * where each batch's size is known only when it is formed. */
int aphi_factor_set_batch(aphi_factor* f, int batch);
/* FP32 factors: how many TF32 pieces the tensor-core trailing update splits
 * each FP32 operand into. 3 (the default): hi + mid + lo, six cross products
 * kept, every product more accurate than an FP32 multiply. 2: hi + lo, the
 * products hh + hl + lh, half the tensor-core work, each product to about
 * 2^-21 relative. The environment variable APHI_TC_SPLIT=2 sets the default. */
int aphi_factor_set_tc_split(aphi_factor* f, int split);

typedef struct {
    int ok;                    /* FactorStats::ok */
    int columns_done;          /* FactorStats::columns_done */
    double smallest_pivot;     /* min |D| over completed columns */
    double largest_pivot;
    double largest_multiplier; /* max |L(i,j)| */
    int64_t nnz;               /* L entries plus D, as the reference counts them */
    double milliseconds;
    double equilibration_min, equilibration_max;
} aphi_factor_stats;

/* Equilibrates (equil_iters Ruiz passes, 0 = none; compute_symmetric_
 * equilibration, src/equilibration.cpp:94-139), then factorizes
 * P (D A D) P^T = L Dg L^T with no pivoting and no conjugation
 * (factorize_ldlt, src/factorization.cpp:109-218). values_dev: batch x nnz
 * complex128 upper-CSR values in the original numbering. pivot_floor stops a
 * factorization whose |D[j]| <= floor (the reference's convention). stats: one
 * per batch entry, may be NULL. Returns PIVOT_FLOOR if any entry stopped. */
int aphi_factorize(aphi_factor* f, const double* values_dev, int equil_iters, double pivot_floor,
                   aphi_factor_stats* stats, void* stream);
/* Solves A x = b for each batch entry: b_dev/x_dev are batch x nrhs x N
 * complex128 in the original numbering (solve, src/factorization.cpp:296-313
 * plus the equilibration substitution of solve_symmetric, :385-390). */
int aphi_solve(aphi_factor* f, int nrhs, const double* b_dev, double* x_dev, void* stream);
/* Copies batch entry k out in the reference's SymmetricFactor layout
 * (include/aphi_solver/factorization.hpp:34-42): strictly lower CSC of the
 * permuted, equilibrated matrix, rows ascending, padding dropped, in the
 * caller's permutation numbering. Sizes: col_ptr[N+1], row_index and
 * value[nnz_L - N], diagonal[N]. Any pointer may be NULL. d_scale[N] receives
 * the equilibration vector when non-NULL. */
int aphi_factor_export(const aphi_factor* f, int k, int* col_ptr, int* row_index, double* value,
                       double* diagonal, double* d_scale);

/* ||A x - b|| / ||b|| and ||A x - b|| / (max|A| ||x|| + ||b||) on the original
 * upper-stored A, per batch entry and rhs (relative_residual and
 * backward_error, src/factorization.cpp:315-329 and :401-416).
 * out: batch x nrhs x 2 doubles (host). */
int aphi_residuals(const aphi_analysis* an, int batch, int nrhs, const double* values_dev,
                   const double* x_dev, const double* b_dev, double* out, void* stream);

/* y = A x on the original upper-stored A (both triangles), per batch entry
 * and rhs: SparseSymmetric::matvec, include/aphi_solver/sparse_symmetric.hpp:
 * 120-136. x, y: batch x nrhs x N complex (device). */
int aphi_spmv(const aphi_analysis* an, int batch, int nrhs, const double* values_dev, const double* x_dev,
              double* y_dev, void* stream);

/* The same numbers as aphi_residuals, computed without allocating device
 * memory: for callers that cannot call cudaMalloc while they run -- a serving
 * loop whose memory pool already owns the device's free memory, or a
 * latency-critical path that cannot take cudaFree's device-wide
 * synchronization. No counterpart in the reference. Its scratch is one
 * fixed-size device array inside this library (8 MiB per GPU that loads it,
 * held until exit); sizes needing more -- ceil(N/256) * 3 * batch * nrhs +
 * batch + 6 * batch * nrhs doubles -- are refused with BAD_SHAPE, and so is
 * batch * nrhs above 65535. The analysis must already have a device copy
 * (any factor created from it makes one) on the current device, or INVALID
 * is returned. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture. Every call is synchronous on its stream: it returns once the
 * ratios are in `out`. All calls share the array: calls that overlap on the
 * GPU race on it, so callers must order them. */
int aphi_residuals_noalloc(const aphi_analysis* an, int batch, int nrhs, const double* values_dev,
                           const double* x_dev, const double* b_dev, double* out, void* stream);

/* Iterative refinement (new; include/aphi_solver/factorization.hpp:27-30 names
 * it as future work). The residual r = b - A x, the equilibration scaling and
 * the update stay in FP64 on the original system; the factor (FP32 or FP64)
 * supplies the correction. krylov = 0: plain refinement x += M^-1 r.
 * krylov = 1: preconditioned COCG (CG with the unconjugated bilinear form,
 * for complex symmetric A), which keeps converging where plain refinement
 * stalls because cond(A) * eps(FP32) approaches 1. A system is done when
 * its backward error <= tol AND its relative residual ||b - A x|| / ||b|| <=
 * rtol; one whose relative residual has not dropped by stall_ratio in 5
 * COCG steps (its residual is not monotone; plain refinement: in 1 step) --
 * COCG first restarts its recurrence once from the current iterate -- or
 * that reaches max_iters, is frozen and IR_STALL returned: the caller's cue
 * to refactorize it in FP64. iters/berr: per batch x rhs. */
typedef struct {
    int max_iters;
    double tol;               /* target backward error */
    double stall_ratio;       /* progress needed: new < stall_ratio * best relative residual */
    int krylov;               /* 0 plain refinement, 1 preconditioned COCG */
    double rtol;              /* target relative residual */
} aphi_ir_options;
int aphi_solve_refined(aphi_factor* f, int nrhs, const double* values_dev, const double* b_dev,
                       double* x_dev, const aphi_ir_options* opt, int* iters, double* berr,
                       void* stream);

/* Host-buffer forms of aphi_factorize, aphi_solve and aphi_residuals for
 * callers that hold no device memory (the drop-in C++ layer): the same
 * arguments with host pointers; the data is staged through device buffers the
 * factor keeps (grown on demand) and the calls return when the results are on
 * the host. */
int aphi_factorize_host(aphi_factor* f, const double* values, int equil_iters, double pivot_floor,
                        aphi_factor_stats* stats);
int aphi_solve_host(aphi_factor* f, int nrhs, const double* b, double* x);
int aphi_residuals_host(const aphi_analysis* an, int batch, int nrhs, const double* values, const double* x,
                        const double* b, double* out);

/* solve_in_place (src/factorization.cpp:254-294) for a factor held only as
 * host arrays in the reference's SymmetricFactor layout (strictly lower CSC,
 * rows ascending; complex D): forward by L, scale by D^-1, backward by L^T,
 * no conjugation, on the device. Each unknown is updated in the reference's
 * order (column by column forward, row by row backward), levels of the
 * pattern running in parallel. y: n x nrhs complex (rhs-major), in place.
 * BAD_SHAPE for a malformed pattern, ZERO_PIVOT for a zero D. */
int aphi_csc_solve_host(int n, const int* col_ptr, const int* row_index, const double* value,
                        const double* diagonal, int nrhs, double* y);
/* relative_residual and backward_error (src/factorization.cpp:315-329,
 * :401-416) of a matrix held only as host upper CSR arrays, computed on the
 * device; x, b: n x nrhs complex (rhs-major). out: nrhs x 2. */
int aphi_csr_residuals_host(int n, const int* row_ptr, const int* col_idx, const double* values, int nrhs,
                            const double* x, const double* b, double* out);

/* The whole solve_symmetric pipeline (src/factorization.cpp:332-398) on
 * host buffers, FP64: equilibrate, factorize, solve, unscale, measure.
 * report[0..12] as SolveReport: ok, backward_error, residual, equil_min,
 * equil_max, smallest_pivot, largest_pivot, largest_multiplier, factor_nnz,
 * columns_done, analyze_ms, factorize_ms, solve_ms. Returns PIVOT_FLOOR (x
 * untouched) when the factorization stopped. */
int aphi_solve_symmetric_host(const aphi_analysis* an, const double* values, const double* b,
                              int equil_iters, double pivot_floor, double* x, double* report);

/* ---- Dense fronts (the supernode-update microbenchmark) -----------------
 * A schedule of `count` independent dense fronts: front s has rows[s] rows,
 * of which the first widths[s] are pivot columns. A factor made from it
 * (aphi_factor_create) factorizes the fronts' panels -- diagonal blocks,
 * panel rows, and the Schur update of the trailing block -- with the same
 * kernels and plans as a sparse factorization. The trailing block (the
 * contribution block) starts at zero, as in the multifrontal method, and ends
 * as -L21 D L21^T.
 *   panels_dev: batch x stored complex128, front s's panel at panel_offset[s]
 *     (column-major, rows[s] x widths[s], leading dimension rows[s]; only
 *     entries on or below the diagonal are read).
 *   aphi_fronts_read: entry k's factored panels (D on the diagonal, L below)
 *     and contribution blocks (front s's (rows - widths)^2 block, column-major,
 *     lower triangle, at cb_offset[s]), widened to complex128, into device
 *     buffers of stored and cb_pool entries (analysis info[3], info[9]). The
 *     blocks sit in the analysis's shared workspace: they are those of its
 *     latest factorization, by this factor or another. */
int aphi_fronts_create(int count, const int* rows, const int* widths, const aphi_analysis_options* opt,
                       aphi_analysis** out);
int aphi_fronts_layout(const aphi_analysis* a, int64_t* panel_offset, int64_t* cb_offset);
int aphi_factorize_fronts(aphi_factor* f, const double* panels_dev, aphi_factor_stats* stats, void* stream);
int aphi_fronts_read(const aphi_factor* f, int k, double* panels_dev, double* cb_dev, void* stream);

/* ---- Diagnostics ---------------------------------------------------------
 * Launch plans of an analysis: plan 0 the FP64 / SIMT factorization, 1 the
 * FP32 tensor-core factorization, 2 the forward solve, 3 the backward solve.
 * launches[k], items[k] for each of the APHI_PLAN_KINDS kernel kinds: 0
 * extend-add, 1 one-CTA front, 2 diagonal block, 3 panel rows, 4 SIMT trailing
 * update tile,
 * 5-9 solve kernels (gather, forward diagonal, forward update, backward
 * update, backward diagonal), 10 panel-restricted update tile, 11
 * tensor-core update tile, 12 the operand split into TF32 planes that the
 * two-piece tensor-core tile reads, 13 the FP64 trailing update's operand
 * scaled by its pivots (W = L D) once per panel group. useful[k] (may be NULL): the real flops of the
 * update kinds' Schur-complement work, counting only lower-triangle entries
 * (8 per complex multiply-add); executed[k] (may be NULL): the flops their
 * tiles perform, padding included. */
#define APHI_PLAN_KINDS 14
int aphi_analysis_plan_stats(const aphi_analysis* a, int plan, int64_t* launches, int64_t* items, double* useful,
                             double* executed);

/* Per-kind device time of a factor's factorizations and solves: while
 * enabled, every launch of the factorization and solve plans is bracketed by
 * CUDA events on its stream and its duration added to ms[kind] (launch
 * counts in launches[kind]; the solve kinds are 5..9).
 * Enabling clears the totals. Costs two events per launch: for measurement
 * runs, not for timed ones. */
int aphi_factor_profile(aphi_factor* f, int enable);
int aphi_factor_profile_read(const aphi_factor* f, double* ms, int64_t* launches);
/* The same, timing only the kinds whose bit is set in mask (bit k: kind k of
 * aphi_analysis_plan_stats); 0 disables. Fewer events, so a timed run that
 * needs one kernel's durations perturbs the rest less. */
int aphi_factor_profile_kinds(aphi_factor* f, unsigned mask);

/* Arithmetic peaks of the current device, measured by short register- or
 * shared-memory-resident loops (2 CTAs per SM, CUDA events): tflops[0] FP64
 * on the DMMA path (mma.sync m8n8k4), [1] FP64 DFMA, [2] FP32 FFMA, [3] TF32
 * tcgen05 M128 N64, [4] TF32 tcgen05 M128 N256 (TFLOP/s, 2 per multiply-add). */
int aphi_measure_peaks(double* tflops);

/* One tensor-core update tile on host data: out (128 x 64 complex64,
 * column-major, leading dimension 128) = sum_{k<K} (P[i0+r, k] d[k])
 * P[j0+c, k], where P is rows x K complex64 column-major and d (K entries,
 * NULL for ones). Rows of P at or beyond `rows` read as zero. K <= 128. The
 * kernel the FP32 factorization uses for its trailing updates. */
int aphi_selftest_tc_tile(int rows, int K, int i0, int j0, const float* P, const float* d, float* out);
/* The same tile with the operands split into `split` (2 or 3) TF32 pieces. */
int aphi_selftest_tc_tile_split(int split, int rows, int K, int i0, int j0, const float* P, const float* d,
                                float* out);
/* The bounded device wait, exercised: one CTA waits on an mbarrier that
 * nothing will complete, with the tensor-core tile's own wait, giving up
 * after spin_limit tries (1 .. the tile's limit). Returns APHI_ERR_TIMEOUT,
 * with the context still usable; anything else is a failure of the wait. */
int aphi_selftest_bounded_wait(long long spin_limit);

#ifdef __cplusplus
}
#endif
#endif
