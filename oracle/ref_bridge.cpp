// C bridge over the reference implementation, compiled from its own sources.
//
// Test infrastructure only: the parity tests, smoke() and bench.py's CPU
// baseline arm call these functions through ctypes to obtain the reference's
// own answers (its mesh pipeline, refill, analysis and solve_symmetric) on the
// same synthetic problems the GPU path is fed. Nothing in the product links it.
//
// The synthetic problem is the cylinder-in-box of the benchmark: the unit cube
// split into n^3 hex cells, each cut into 6 Kuhn tets, a conductor (sigma =
// 5.8e7) wherever a tet centroid lies within r = 0.2 of the z axis through
// (0.5, 0.5), air elsewhere, n x A = 0 on the outer faces, and two voltage
// ports on the conductor's caps (top = V_top, bottom = 0 V). The Kuhn vertex
// order follows tools/generate_cube_mesh.py:32-39 of the reference.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "aphi_solver/assembly.hpp"
#include "aphi_solver/equilibration.hpp"
#include "aphi_solver/factorization.hpp"
#include "aphi_solver/postprocess.hpp"
#include "aphi_solver/symbolic.hpp"
#include "ref_meshes.hpp"

using namespace aphi_solver;
using Complex = std::complex<double>;

namespace {

using ref_meshes::build_cylinder_mesh;
using ref_meshes::build_torus_mesh;

thread_local std::string g_error;

struct RefProblem {
    bool has_mesh = false;
    Mesh mesh;
    BoundProblem bound;
    DofMap dofs;
    SparsityPattern pattern;
    SolverAnalysis analysis;
    std::unique_ptr<ScatterMap> map;
    SymmetricSystem system;
};

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return -1;
    } catch (const std::logic_error& e) {
        g_error = e.what();
        return -2;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -3;
    }
}

void to_complex(const double* in, std::size_t n, std::vector<Complex>& out) {
    out.resize(n);
    for (std::size_t i = 0; i < n; ++i) out[i] = Complex(in[2 * i], in[2 * i + 1]);
}

void from_complex(const std::vector<Complex>& in, double* out) {
    for (std::size_t i = 0; i < in.size(); ++i) {
        out[2 * i] = in[i].real();
        out[2 * i + 1] = in[i].imag();
    }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

/// Builds the cylinder-in-box problem through the reference's own pipeline:
/// build_topology, bind_to_mesh, build_dof_map, build_sparsity(UpperTriangle),
/// analyze(AMD), make_symmetric_system and ScatterMap::build.
void* ref_kuhn_cylinder(int n, int full_wave, double v_top, int ordering) {
    auto p = std::make_unique<RefProblem>();
    int rc = guarded([&] {
        build_cylinder_mesh(p->mesh, n);
        Problem pr;
        pr.type = AnalysisType::Frequency;
        pr.frequencies = {50.0};
        pr.formulation = full_wave ? Formulation::FullWave : Formulation::Reduced;
        pr.conditioning = Conditioning::RowScaled;
        Body w;
        w.name = "B1";
        w.volume = "wire";
        w.sigma = 5.8e7;
        Body a;
        a.name = "B2";
        a.volume = "air";
        a.sigma = 0.0;
        pr.bodies = {w, a};
        Port p1;
        p1.name = "P1";
        p1.type = PortType::BoundaryVoltage;
        p1.surface = {"wire_top"};
        p1.amplitude = v_top;
        Port p2;
        p2.name = "P2";
        p2.type = PortType::BoundaryVoltage;
        p2.surface = {"wire_bottom"};
        p2.amplitude = 0.0;
        pr.ports = {p1, p2};
        p->bound = bind_to_mesh(pr, p->mesh);
        p->dofs = build_dof_map(p->bound, p->mesh);
        p->pattern = build_sparsity(p->dofs, p->bound, p->mesh, SparsityStorage::UpperTriangle);
        // ordering < 0 skips the symbolic analysis (assembly-only use).
        if (ordering >= 0) p->analysis = analyze(p->pattern, static_cast<Ordering>(ordering));
        p->system = make_symmetric_system(p->pattern, p->dofs.num_total);
        p->map = std::make_unique<ScatterMap>(
            ScatterMap::build(p->pattern, p->dofs, p->mesh, p->bound));
        p->has_mesh = true;
        return 0;
    });
    if (rc != 0) return nullptr;
    return p.release();
}

/// The torus with one internal current port (`current` A, hint +y) through
/// the same pipeline.
void* ref_kuhn_torus(int n, double current, int ordering) {
    auto p = std::make_unique<RefProblem>();
    int rc = guarded([&] {
        build_torus_mesh(p->mesh, n);
        Problem pr;
        pr.type = AnalysisType::Frequency;
        pr.frequencies = {50.0};
        pr.formulation = Formulation::Reduced;
        pr.conditioning = Conditioning::RowScaled;
        Body w;
        w.name = "B1";
        w.volume = "torus";
        w.sigma = 5.8e7;
        Body a;
        a.name = "B2";
        a.volume = "air";
        a.sigma = 0.0;
        pr.bodies = {w, a};
        Port p1;
        p1.name = "P1";
        p1.type = PortType::InternalCurrent;
        p1.surface = {"cut"};
        p1.amplitude = current;
        p1.current_direction = Vec3(0.0, 1.0, 0.0);
        pr.ports = {p1};
        p->bound = bind_to_mesh(pr, p->mesh);
        p->dofs = build_dof_map(p->bound, p->mesh);
        p->pattern = build_sparsity(p->dofs, p->bound, p->mesh, SparsityStorage::UpperTriangle);
        if (ordering >= 0) p->analysis = analyze(p->pattern, static_cast<Ordering>(ordering));
        p->system = make_symmetric_system(p->pattern, p->dofs.num_total);
        p->map = std::make_unique<ScatterMap>(
            ScatterMap::build(p->pattern, p->dofs, p->mesh, p->bound));
        p->has_mesh = true;
        return 0;
    });
    if (rc != 0) return nullptr;
    return p.release();
}

/// A problem with only a pattern: an upper-triangle CSR handed in, analysed
/// under `ordering` (0 natural, 1 rcm, 2 amd), for the matrix-only tests.
void* ref_from_pattern(int n, const int* row_ptr, const int* col_idx, int ordering) {
    auto p = std::make_unique<RefProblem>();
    int rc = guarded([&] {
        p->pattern.rows = n;
        p->pattern.cols = n;
        p->pattern.upper_only = true;
        p->pattern.row_ptr.assign(row_ptr, row_ptr + n + 1);
        p->pattern.col_index.assign(col_idx, col_idx + row_ptr[n]);
        p->analysis = analyze(p->pattern, static_cast<Ordering>(ordering));
        p->system.matrix =
            SparseSymmetricZ::from_pattern(n, p->pattern.row_ptr, p->pattern.col_index);
        p->system.rhs.assign(static_cast<std::size_t>(n), Complex(0.0, 0.0));
        return 0;
    });
    if (rc != 0) return nullptr;
    return p.release();
}

void ref_free(void* h) { delete static_cast<RefProblem*>(h); }

/// sizes: [nodes, tets, edges, N, nnz_upper, num_a, num_phi, num_ports,
///         num_bodies, nnz_L (incl. diagonal), scatter_map_bytes, num_roots]
void ref_sizes(void* h, long long* out) {
    auto* p = static_cast<RefProblem*>(h);
    std::memset(out, 0, sizeof(long long) * 12);
    if (p->has_mesh) {
        out[0] = p->mesh.num_nodes();
        out[1] = p->mesh.num_tets();
        out[2] = p->mesh.num_edges();
        out[5] = p->dofs.num_a;
        out[6] = p->dofs.num_phi;
        out[7] = p->dofs.num_ports;
        out[8] = static_cast<long long>(p->bound.bodies.size());
        out[10] = static_cast<long long>(p->map->bytes());
    }
    out[3] = p->pattern.rows;
    out[4] = static_cast<long long>(p->pattern.nnz());
    out[9] = static_cast<long long>(p->analysis.predicted_nnz);
    out[11] = p->analysis.num_roots;
}

void ref_nodes(void* h, double* xyz) {
    auto* p = static_cast<RefProblem*>(h);
    for (int i = 0; i < p->mesh.num_nodes(); ++i) {
        xyz[3 * i] = p->mesh.nodes[i].x;
        xyz[3 * i + 1] = p->mesh.nodes[i].y;
        xyz[3 * i + 2] = p->mesh.nodes[i].z;
    }
}

/// tets[4T], tet_edges[6T], signs[6T], body_of_tet[T]
void ref_tets(void* h, int* tets, int* tet_edges, int* signs, int* body_of_tet) {
    auto* p = static_cast<RefProblem*>(h);
    for (int t = 0; t < p->mesh.num_tets(); ++t) {
        for (int q = 0; q < 4; ++q) tets[4 * t + q] = p->mesh.tets[t][q];
        for (int q = 0; q < 6; ++q) {
            tet_edges[6 * t + q] = p->mesh.tet_edges[t][q];
            signs[6 * t + q] = p->mesh.tet_edge_signs[t][q];
        }
        body_of_tet[t] = p->bound.body_of_tet[t];
    }
}

/// Mesh edges as (lo, hi) pairs, in the mesh's own numbering.
void ref_edges(void* h, int* pairs) {
    auto* p = static_cast<RefProblem*>(h);
    for (int e = 0; e < p->mesh.num_edges(); ++e) {
        pairs[2 * e] = p->mesh.edges[e].first;
        pairs[2 * e + 1] = p->mesh.edges[e].second;
    }
}

/// Per-edge / per-P2-node DOF classification: edge_index[E], phi_index[P2].
void ref_dof_arrays(void* h, int* edge_index, int* phi_index, int* tree_edge, int* dirichlet_edge) {
    auto* p = static_cast<RefProblem*>(h);
    for (int e = 0; e < p->mesh.num_edges(); ++e) {
        edge_index[e] = p->dofs.edge_index[e];
        tree_edge[e] = p->bound.gauge.is_tree_edge[e] ? 1 : 0;
        dirichlet_edge[e] = p->bound.dirichlet_edge[e] ? 1 : 0;
    }
    for (int i = 0; i < p->dofs.num_p2_nodes; ++i) phi_index[i] = p->dofs.phi_index[i];
}

/// DofMap::local_dofs for every tet: idx[16T] (6 edges then 10 Phi), coeff[16T],
/// phi_fixed[2*10T] (complex, interleaved).
void ref_tet_dofs(void* h, int* idx, double* coeff, double* phi_fixed) {
    auto* p = static_cast<RefProblem*>(h);
    for (int t = 0; t < p->mesh.num_tets(); ++t) {
        const TetDofs d = p->dofs.local_dofs(t, p->mesh, p->bound);
        for (int i = 0; i < 6; ++i) {
            idx[16 * t + i] = d.edge[i].index;
            coeff[16 * t + i] = d.edge[i].coeff;
        }
        for (int i = 0; i < 10; ++i) {
            idx[16 * t + 6 + i] = d.phi[i].index;
            coeff[16 * t + 6 + i] = d.phi[i].coeff;
            phi_fixed[20 * t + 2 * i] = d.phi_fixed[i].real();
            phi_fixed[20 * t + 2 * i + 1] = d.phi_fixed[i].imag();
        }
    }
}

/// Bodies: sigma, eps_r, mu_r, tet count; and each body's tets in order.
void ref_bodies(void* h, double* material /*3 per body*/, int* count) {
    auto* p = static_cast<RefProblem*>(h);
    for (std::size_t b = 0; b < p->bound.bodies.size(); ++b) {
        material[3 * b] = p->bound.bodies[b].sigma;
        material[3 * b + 1] = p->bound.bodies[b].eps_r;
        material[3 * b + 2] = p->bound.bodies[b].mu_r;
        count[b] = static_cast<int>(p->bound.bodies[b].tets.size());
    }
}

void ref_body_tets(void* h, int body, int* tets) {
    auto* p = static_cast<RefProblem*>(h);
    const auto& v = p->bound.bodies[static_cast<std::size_t>(body)].tets;
    std::copy(v.begin(), v.end(), tets);
}

/// Ports: current_driven[k], row[k], amplitude (re, im) [2k], port_value (re, im) [2k].
void ref_ports(void* h, int* current_driven, int* row, double* amplitude, double* value) {
    auto* p = static_cast<RefProblem*>(h);
    for (std::size_t k = 0; k < p->bound.ports.size(); ++k) {
        current_driven[k] = is_current_driven(p->bound.ports[k].type) ? 1 : 0;
        row[k] = p->dofs.port_index[k];
        amplitude[2 * k] = p->bound.ports[k].amplitude.real();
        amplitude[2 * k + 1] = p->bound.ports[k].amplitude.imag();
        value[2 * k] = p->dofs.port_value[k].real();
        value[2 * k + 1] = p->dofs.port_value[k].imag();
    }
}

void ref_pattern(void* h, int* row_ptr, int* col_idx) {
    auto* p = static_cast<RefProblem*>(h);
    std::copy(p->pattern.row_ptr.begin(), p->pattern.row_ptr.end(), row_ptr);
    std::copy(p->pattern.col_index.begin(), p->pattern.col_index.end(), col_idx);
}

void ref_analysis(void* h, int* perm, int* iperm, int* parent, int* col_count) {
    auto* p = static_cast<RefProblem*>(h);
    const int n = p->pattern.rows;
    for (int i = 0; i < n; ++i) {
        perm[i] = p->analysis.permutation.perm[i];
        iperm[i] = p->analysis.permutation.iperm[i];
        parent[i] = p->analysis.parent[i];
        col_count[i] = p->analysis.col_count[i];
    }
}

/// ScatterMap contents: live[T], pos[16T], offset[T+1] (as int64), slot[sum].
void ref_scatter_map(void* h, int* live, int* pos, long long* offset, int* slot) {
    auto* p = static_cast<RefProblem*>(h);
    const ScatterMap& m = *p->map;
    long long at = 0;
    for (int t = 0; t < m.num_tets(); ++t) {
        live[t] = m.live_count(t);
        for (int i = 0; i < 6; ++i) pos[16 * t + i] = m.edge_at(t)[i];
        for (int i = 0; i < 10; ++i) pos[16 * t + 6 + i] = m.phi_at(t)[i];
        offset[t] = at;
        const int sz = tet_block_size(m.live_count(t), m.packed());
        for (int k = 0; k < sz; ++k) slot[at + k] = m.slots(t)[k];
        at += sz;
    }
    offset[m.num_tets()] = at;
}

/// refill(SymmetricSystem&, ...) at one omega. conditioning: 0 natural,
/// 1 row_scaled, 2 scaled_phi. use_map selects the ScatterMap path.
int ref_refill(void* h, double omega, int conditioning, int use_map, double* values, double* rhs,
               double* milliseconds) {
    auto* p = static_cast<RefProblem*>(h);
    return guarded([&] {
        const auto t0 = std::chrono::steady_clock::now();
        refill(p->system, p->bound, p->mesh, p->dofs, p->pattern, omega,
               static_cast<Conditioning>(conditioning), use_map ? p->map.get() : nullptr);
        const auto t1 = std::chrono::steady_clock::now();
        if (milliseconds) *milliseconds = std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (values) from_complex(p->system.matrix.values(), values);
        if (rhs) from_complex(p->system.rhs, rhs);
        return 0;
    });
}

/// Loads caller values into the problem's symmetric matrix.
int ref_set_values(void* h, const double* values) {
    auto* p = static_cast<RefProblem*>(h);
    std::vector<Complex> v;
    to_complex(values, p->system.matrix.nnz(), v);
    std::copy(v.begin(), v.end(), p->system.matrix.mutable_values().begin());
    return 0;
}

/// solve_symmetric on the problem's matrix (as last refilled or set) with the
/// given rhs and the problem's own analysis. report[0..13]: ok, backward_error,
/// residual, equilibration_min, equilibration_max, smallest_pivot,
/// largest_pivot, largest_multiplier, factor_nnz, columns_done, analyze_ms,
/// factorize_ms, solve_ms.
int ref_solve_symmetric(void* h, const double* rhs, int equil_iters, double pivot_floor,
                        double* x, double* report) {
    auto* p = static_cast<RefProblem*>(h);
    return guarded([&] {
        std::vector<Complex> b, sol;
        to_complex(rhs, static_cast<std::size_t>(p->pattern.rows), b);
        SolveReport r;
        SolveOptions o;
        o.equilibration_iterations = equil_iters;
        o.pivot_floor = pivot_floor;
        const bool ok = solve_symmetric(p->system.matrix, b, sol, r, o, &p->analysis);
        if (ok) from_complex(sol, x);
        report[0] = r.ok ? 1.0 : 0.0;
        report[1] = r.backward_error;
        report[2] = r.residual;
        report[3] = r.equilibration_min;
        report[4] = r.equilibration_max;
        report[5] = r.smallest_pivot;
        report[6] = r.largest_pivot;
        report[7] = r.largest_multiplier;
        report[8] = static_cast<double>(r.factor_nnz);
        report[9] = r.columns_done;
        report[10] = r.analyze_ms;
        report[11] = r.factorize_ms;
        report[12] = r.solve_ms;
        return ok ? 0 : 1;
    });
}

/// compute_symmetric_equilibration on the problem's current matrix.
int ref_equilibration(void* h, int iterations, double* d) {
    auto* p = static_cast<RefProblem*>(h);
    return guarded([&] {
        const std::vector<double> v = compute_symmetric_equilibration(p->system.matrix, iterations);
        std::copy(v.begin(), v.end(), d);
        return 0;
    });
}

/// factorize_ldlt of the problem's current matrix (unscaled) with its analysis.
/// Fills L in CSC (strictly lower; col_ptr[N+1], row_index/value[nnz_L - N]),
/// D[N]; stats: ok, columns_done, smallest, largest, largest_multiplier, nnz, ms.
int ref_factorize(void* h, double pivot_floor, int* col_ptr, int* row_index, double* value,
                  double* diagonal, double* stats) {
    auto* p = static_cast<RefProblem*>(h);
    return guarded([&] {
        SymmetricFactor f;
        FactorStats s;
        const bool ok = factorize_ldlt(p->system.matrix, p->analysis, f, s, pivot_floor);
        if (col_ptr) std::copy(f.col_ptr.begin(), f.col_ptr.end(), col_ptr);
        if (row_index) std::copy(f.row_index.begin(), f.row_index.end(), row_index);
        if (value) from_complex(f.value, value);
        if (diagonal) from_complex(f.diagonal, diagonal);
        stats[0] = s.ok ? 1.0 : 0.0;
        stats[1] = s.columns_done;
        stats[2] = s.smallest_pivot;
        stats[3] = s.largest_pivot;
        stats[4] = s.largest_multiplier;
        stats[5] = static_cast<double>(s.nnz);
        stats[6] = s.milliseconds;
        return ok ? 0 : 1;
    });
}

/// The three element kernels for one tet with vertices xyz[12] and one body.
int ref_element_blocks(const double* xyz, double sigma, double eps_r, double mu_r, double omega,
                       double* aa, double* ap, double* pp) {
    return guarded([&] {
        Mesh m;
        for (int q = 0; q < 4; ++q) m.nodes.push_back(Vec3(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]));
        m.tets.push_back(TetVerts{0, 1, 2, 3});
        BoundBody b;
        b.sigma = sigma;
        b.eps_r = eps_r;
        b.mu_r = mu_r;
        const ElementCoefficients c = element_coefficients(b, omega);
        const TetGeometry g = compute_tet_geometry(m, 0);
        Complex a1[36], a2[60], a3[100];
        kernel_AA(g, c, a1);
        kernel_APhi(g, c, a2);
        kernel_PhiPhi(g, c, a3);
        for (int i = 0; i < 36; ++i) { aa[2 * i] = a1[i].real(); aa[2 * i + 1] = a1[i].imag(); }
        for (int i = 0; i < 60; ++i) { ap[2 * i] = a2[i].real(); ap[2 * i + 1] = a2[i].imag(); }
        for (int i = 0; i < 100; ++i) { pp[2 * i] = a3[i].real(); pp[2 * i + 1] = a3[i].imag(); }
        return 0;
    });
}

/// The reference's compute_fields on solution x (complex, n), copied out:
/// per tet a/b/e/j (3 complex each) and sigma; per P2 node phi (complex),
/// a/b/h/e/j (3 complex each), vertex_weight and on_material_interface;
/// counts[0..1] = num_interface_nodes, num_orphan_vertices.
int ref_compute_fields(void* h, const double* x, double omega, int conditioning, double* phi_node, double* a_tet,
                       double* b_tet, double* e_tet, double* j_tet, double* sigma_tet, double* a_node,
                       double* b_node, double* h_node, double* e_node, double* j_node, double* vertex_weight,
                       unsigned char* on_interface, int* counts) {
    return guarded([&] {
        auto* p = static_cast<RefProblem*>(h);
        Solution sol;
        to_complex(x, static_cast<std::size_t>(p->dofs.num_total), sol.x);
        sol.omega = omega;
        sol.conditioning = static_cast<Conditioning>(conditioning);
        const FieldOutput f = compute_fields(p->mesh, p->bound, p->dofs, sol);
        auto put3 = [](const std::vector<Vec3C>& v, double* out) {
            for (std::size_t i = 0; i < v.size(); ++i)
                for (int k = 0; k < 3; ++k) {
                    out[6 * i + 2 * k] = v[i][static_cast<std::size_t>(k)].real();
                    out[6 * i + 2 * k + 1] = v[i][static_cast<std::size_t>(k)].imag();
                }
        };
        from_complex(f.phi_node, phi_node);
        put3(f.a_tet, a_tet);
        put3(f.b_tet, b_tet);
        put3(f.e_tet, e_tet);
        put3(f.j_tet, j_tet);
        std::copy(f.sigma_tet.begin(), f.sigma_tet.end(), sigma_tet);
        put3(f.a_node, a_node);
        put3(f.b_node, b_node);
        put3(f.h_node, h_node);
        put3(f.e_node, e_node);
        put3(f.j_node, j_node);
        std::copy(f.vertex_weight.begin(), f.vertex_weight.end(), vertex_weight);
        std::copy(f.on_material_interface.begin(), f.on_material_interface.end(), on_interface);
        counts[0] = f.num_interface_nodes;
        counts[1] = f.num_orphan_vertices;
        return 0;
    });
}

}  // extern "C"
