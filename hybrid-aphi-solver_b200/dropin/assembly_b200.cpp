// Drop-in replacement for the reference's src/assembly.cpp: every function
// declared in include/aphi_solver/assembly.hpp, with the element fill and the
// scatter running on the B200 through the aphi_b200 C ABI. Built in place of
// src/assembly.cpp against the reference's own headers; the mesh, binding,
// DOF map and sparsity passes are the reference's, linked unchanged.
//
// refill (both overloads, src/assembly.cpp:453-494) hands the device
// assembly the per-mesh tables the reference's scatter reads on every call --
// node coordinates, tet vertices, DofMap::local_dofs for every tet, body
// materials and tet lists in the reference's visit order, port rows and
// excitations, and the pattern -- once, and then assembles each frequency on
// the device (element kernels + fixed-order slot sums, bitwise equal to the
// reference's scatter) into the caller's system. The device assembly is
// cached under the addresses and sizes of the mesh, DOF map, bound problem
// and pattern, together with their materials and port excitations, which are
// compared on every call; the tet tables are assumed not to change in place
// while those objects keep their addresses and sizes.
//
// ScatterMap is the reference's own class (its layout is fixed by the header
// and inspected by its tests): per tet, the distinct live global DOFs in
// ascending order, each local DOF's position among them (-1 when
// eliminated), and the value-array slot of every pair, laid out by
// tet_block_index. The device path does not read it -- it has its own slot
// lists -- but refill checks it against the pattern and the mesh as the
// reference does.
//
// Error conventions are the reference's: std::invalid_argument for shape
// mismatches and refused conditionings (src/assembly.cpp:431-498, :12-45),
// std::logic_error when the pattern has no slot for an entry, and
// std::runtime_error for a degenerate tet (src/basis_functions.cpp:31).
#include <algorithm>
#include <complex>
#include <cstdint>
#include <list>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "aphi_b200.h"
#include "aphi_solver/assembly.hpp"
#include "aphi_solver/dof_map.hpp"
#include "aphi_solver/mesh.hpp"
#include "aphi_solver/problem_binding.hpp"

namespace aphi_solver {

namespace {

using Complex = std::complex<double>;

void check_status(int rc, const char* where) {
    if (rc == APHI_OK) return;
    const std::string msg = std::string(where) + ": " + aphi_last_error();
    if (rc == APHI_ERR_BAD_SHAPE) throw std::invalid_argument(msg);
    if (rc == APHI_ERR_PATTERN_MISMATCH) throw std::logic_error(msg);
    if (rc == APHI_ERR_DEGENERATE_TET) throw std::runtime_error(msg);
    throw std::runtime_error(msg + " (" + aphi_status_string(rc) + ")");
}

int conditioning_code(Conditioning c) {
    switch (c) {
        case Conditioning::Natural: return APHI_COND_NATURAL;
        case Conditioning::RowScaled: return APHI_COND_ROW_SCALED;
        case Conditioning::ScaledPhi: return APHI_COND_SCALED_PHI;
    }
    throw std::invalid_argument("refill: unknown conditioning");
}

// One device assembly: the tables it was built from, kept for the desc's
// lifetime, and the identity it is cached under.
struct DeviceAssembly {
    const void *bound = nullptr, *mesh = nullptr, *dofs = nullptr, *pattern = nullptr;
    int num_tets = 0, num_nodes = 0, num_total = 0, rows = 0;
    std::size_t nnz = 0;
    bool upper = false;
    std::vector<double> xyz, tet_coeff, tet_fixed, material, port_amplitude, port_value;
    std::vector<int> tets, tet_idx, body_ptr, body_tets, port_current, port_row, row_ptr, col_idx;
    aphi_assembly* h = nullptr;
    ~DeviceAssembly() {
        if (h) aphi_assembly_destroy(h);
    }
};

// Never destroyed: device handles are not released from static destructors.
std::mutex& g_mutex = *new std::mutex;
std::list<std::shared_ptr<DeviceAssembly>>& g_cache = *new std::list<std::shared_ptr<DeviceAssembly>>;
constexpr std::size_t kMaxAssemblies = 4;

void excitations(const BoundProblem& bound, const DofMap& dofs, std::vector<double>& material,
                 std::vector<int>& port_current, std::vector<int>& port_row, std::vector<double>& port_amplitude,
                 std::vector<double>& port_value) {
    material.clear();
    for (const BoundBody& b : bound.bodies) {
        material.push_back(b.sigma);
        material.push_back(b.eps_r);
        material.push_back(b.mu_r);
    }
    port_current.clear();
    port_row.clear();
    port_amplitude.clear();
    port_value.clear();
    for (std::size_t k = 0; k < bound.ports.size(); ++k) {
        port_current.push_back(is_current_driven(bound.ports[k].type) ? 1 : 0);
        port_row.push_back(dofs.port_index[k]);
        port_amplitude.push_back(bound.ports[k].amplitude.real());
        port_amplitude.push_back(bound.ports[k].amplitude.imag());
        port_value.push_back(dofs.port_value[k].real());
        port_value.push_back(dofs.port_value[k].imag());
    }
}

std::shared_ptr<DeviceAssembly> device_assembly(const BoundProblem& bound, const Mesh& mesh, const DofMap& dofs,
                                                const SparsityPattern& pattern) {
    std::vector<double> material, port_amplitude, port_value;
    std::vector<int> port_current, port_row;
    excitations(bound, dofs, material, port_current, port_row, port_amplitude, port_value);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
        const DeviceAssembly& d = **it;
        if (d.bound == &bound && d.mesh == &mesh && d.dofs == &dofs && d.pattern == &pattern &&
            d.num_tets == mesh.num_tets() && d.num_nodes == mesh.num_nodes() && d.num_total == dofs.num_total &&
            d.rows == pattern.rows && d.nnz == pattern.nnz() && d.upper == pattern.upper_only &&
            d.material == material && d.port_current == port_current && d.port_row == port_row &&
            d.port_amplitude == port_amplitude && d.port_value == port_value) {
            g_cache.splice(g_cache.begin(), g_cache, it);
            return *g_cache.begin();
        }
    }
    auto d = std::make_shared<DeviceAssembly>();
    d->bound = &bound;
    d->mesh = &mesh;
    d->dofs = &dofs;
    d->pattern = &pattern;
    d->num_tets = mesh.num_tets();
    d->num_nodes = mesh.num_nodes();
    d->num_total = dofs.num_total;
    d->rows = pattern.rows;
    d->nnz = pattern.nnz();
    d->upper = pattern.upper_only;
    d->material = material;
    d->port_current = port_current;
    d->port_row = port_row;
    d->port_amplitude = port_amplitude;
    d->port_value = port_value;
    for (const Vec3& p : mesh.nodes) {
        d->xyz.push_back(p.x);
        d->xyz.push_back(p.y);
        d->xyz.push_back(p.z);
    }
    for (const TetVerts& t : mesh.tets) d->tets.insert(d->tets.end(), t.begin(), t.end());
    d->tet_idx.assign(16 * static_cast<std::size_t>(d->num_tets), -1);
    d->tet_coeff.assign(16 * static_cast<std::size_t>(d->num_tets), 0.0);
    d->tet_fixed.assign(20 * static_cast<std::size_t>(d->num_tets), 0.0);
    for (int t = 0; t < d->num_tets; ++t) {
        const TetDofs td = dofs.local_dofs(t, mesh, bound);
        const std::size_t o = 16 * static_cast<std::size_t>(t);
        for (int i = 0; i < 6; ++i) {
            d->tet_idx[o + i] = td.edge[i].index;
            d->tet_coeff[o + i] = td.edge[i].coeff;
        }
        for (int i = 0; i < 10; ++i) {
            d->tet_idx[o + 6 + i] = td.phi[i].index;
            d->tet_coeff[o + 6 + i] = td.phi[i].coeff;
            d->tet_fixed[20 * static_cast<std::size_t>(t) + 2 * i] = td.phi_fixed[i].real();
            d->tet_fixed[20 * static_cast<std::size_t>(t) + 2 * i + 1] = td.phi_fixed[i].imag();
        }
    }
    d->body_ptr.push_back(0);
    for (const BoundBody& b : bound.bodies) {
        d->body_tets.insert(d->body_tets.end(), b.tets.begin(), b.tets.end());
        d->body_ptr.push_back(static_cast<int>(d->body_tets.size()));
    }
    d->row_ptr = pattern.row_ptr;
    d->col_idx = pattern.col_index;
    aphi_assembly_desc desc{};
    desc.num_nodes = d->num_nodes;
    desc.num_tets = d->num_tets;
    desc.num_unknowns = pattern.rows;
    desc.xyz = d->xyz.data();
    desc.tets = d->tets.data();
    desc.tet_idx = d->tet_idx.data();
    desc.tet_coeff = d->tet_coeff.data();
    desc.tet_fixed = d->tet_fixed.data();
    desc.num_bodies = static_cast<int>(bound.bodies.size());
    desc.material = d->material.data();
    desc.body_ptr = d->body_ptr.data();
    desc.body_tets = d->body_tets.data();
    desc.num_ports = static_cast<int>(bound.ports.size());
    desc.port_current = d->port_current.data();
    desc.port_row = d->port_row.data();
    desc.port_amplitude = d->port_amplitude.data();
    desc.port_value = d->port_value.data();
    desc.upper_only = pattern.upper_only ? 1 : 0;
    desc.row_ptr = d->row_ptr.data();
    desc.col_idx = d->col_idx.data();
    check_status(aphi_assembly_create(&desc, &d->h), "refill");
    g_cache.push_front(d);
    if (g_cache.size() > kMaxAssemblies) g_cache.pop_back();
    return d;
}

// The reference's shape checks, shared by both overloads.
void check_shapes(int matrix_rows, std::size_t matrix_nnz, std::size_t rhs_size, const Mesh& mesh,
                  const DofMap& dofs, const SparsityPattern& pattern, const ScatterMap* scatter) {
    if (matrix_rows != pattern.rows || matrix_nnz != pattern.nnz())
        throw std::invalid_argument("refill: this system was not made from this pattern; their shapes must agree");
    if (rhs_size != static_cast<std::size_t>(dofs.num_total))
        throw std::invalid_argument("refill: the right-hand side is not one entry per unknown");
    if (scatter != nullptr && scatter->num_tets() != mesh.num_tets())
        throw std::invalid_argument("refill: the ScatterMap was built for a different mesh (" +
                                    std::to_string(scatter->num_tets()) + " tets against " +
                                    std::to_string(mesh.num_tets()) + ")");
    if (scatter != nullptr && scatter->packed() != pattern.upper_only)
        throw std::invalid_argument(
            "refill: the ScatterMap and the pattern disagree about which half of the matrix is stored");
}

void device_refill(std::vector<Complex>& values, std::vector<Complex>& rhs, const BoundProblem& bound,
                   const Mesh& mesh, const DofMap& dofs, const SparsityPattern& pattern, double omega,
                   Conditioning formulation) {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto d = device_assembly(bound, mesh, dofs, pattern);
    check_status(aphi_refill_host(d->h, omega, conditioning_code(formulation), reinterpret_cast<double*>(values.data()),
                                  reinterpret_cast<double*>(rhs.data())),
                 "refill");
}

}  // namespace

FormulationScales formulation_scales(Conditioning f, double omega) {
    double rc[4];
    int sym = 0;
    check_status(aphi_formulation_scales(conditioning_code(f), omega, rc, &sym), "formulation_scales");
    FormulationScales s;
    s.row = Complex(rc[0], rc[1]);
    s.column = Complex(rc[2], rc[3]);
    s.symmetric = sym != 0;
    return s;
}

ScatterMap ScatterMap::build(const SparsityPattern& pattern, const DofMap& dofs, const Mesh& mesh,
                             const BoundProblem& bound) {
    const int num_tets = mesh.num_tets();
    ScatterMap m;
    m.packed_ = pattern.upper_only;
    m.live_.assign(static_cast<std::size_t>(num_tets), 0);
    m.pos_.assign(static_cast<std::size_t>(num_tets) * 16, -1);
    m.offset_.assign(static_cast<std::size_t>(num_tets) + 1, 0);
    std::vector<std::vector<int>> live(static_cast<std::size_t>(num_tets));
    for (int t = 0; t < num_tets; ++t) {
        const TetDofs td = dofs.local_dofs(t, mesh, bound);
        std::vector<int>& g = live[t];
        for (const DofEntry& e : td.edge)
            if (e.index >= 0) g.push_back(e.index);
        for (const DofEntry& e : td.phi)
            if (e.index >= 0) g.push_back(e.index);
        std::sort(g.begin(), g.end());
        g.erase(std::unique(g.begin(), g.end()), g.end());
        auto at = [&](int index) {
            if (index < 0) return -1;
            return static_cast<int>(std::lower_bound(g.begin(), g.end(), index) - g.begin());
        };
        for (int i = 0; i < 6; ++i) m.pos_[16 * static_cast<std::size_t>(t) + i] = at(td.edge[i].index);
        for (int i = 0; i < 10; ++i) m.pos_[16 * static_cast<std::size_t>(t) + 6 + i] = at(td.phi[i].index);
        const int n = static_cast<int>(g.size());
        m.live_[t] = n;
        m.offset_[t + 1] = m.offset_[t] + static_cast<std::size_t>(tet_block_size(n, m.packed_));
    }
    m.slot_.assign(m.offset_[static_cast<std::size_t>(num_tets)], -1);
    for (int t = 0; t < num_tets; ++t) {
        const std::vector<int>& g = live[t];
        const int n = static_cast<int>(g.size());
        int* block = m.slot_.data() + m.offset_[t];
        for (int r = 0; r < n; ++r) {
            const auto rb = pattern.col_index.begin() + pattern.row_ptr[g[r]];
            const auto re = pattern.col_index.begin() + pattern.row_ptr[g[r] + 1];
            for (int c = m.packed_ ? r : 0; c < n; ++c) {
                const auto it = std::lower_bound(rb, re, g[c]);
                if (it == re || *it != g[c])
                    throw std::logic_error("ScatterMap::build: no slot for entry (" + std::to_string(g[r]) + ", " +
                                           std::to_string(g[c]) + "); the pattern and the DOF map disagree");
                block[tet_block_index(n, m.packed_, r, c)] = static_cast<int>(it - pattern.col_index.begin());
            }
        }
    }
    return m;
}

std::size_t ScatterMap::bytes() const {
    return live_.size() * sizeof(int) + pos_.size() * sizeof(int) + offset_.size() * sizeof(std::size_t) +
           slot_.size() * sizeof(int);
}

AssembledSystem make_system(const SparsityPattern& pattern, int num_unknowns) {
    AssembledSystem out;
    out.matrix = SparseMatrixZ::from_pattern(pattern.rows, pattern.cols, pattern.row_ptr, pattern.col_index);
    out.rhs.assign(static_cast<std::size_t>(num_unknowns), Complex(0.0, 0.0));
    return out;
}

SymmetricSystem make_symmetric_system(const SparsityPattern& pattern, int num_unknowns) {
    if (!pattern.upper_only)
        throw std::invalid_argument("make_symmetric_system: needs a pattern built with SparsityStorage::UpperTriangle");
    SymmetricSystem out;
    out.matrix = SparseSymmetricZ::from_pattern(pattern.rows, pattern.row_ptr, pattern.col_index);
    out.rhs.assign(static_cast<std::size_t>(num_unknowns), Complex(0.0, 0.0));
    return out;
}

void refill(AssembledSystem& system, const BoundProblem& bound, const Mesh& mesh, const DofMap& dofs,
            const SparsityPattern& pattern, double omega, Conditioning formulation, const ScatterMap* scatter) {
    check_shapes(system.matrix.rows(), system.matrix.nnz(), system.rhs.size(), mesh, dofs, pattern, scatter);
    if (pattern.upper_only)
        throw std::invalid_argument(
            "refill: this pattern holds only the upper triangle, which belongs in a SparseSymmetric");
    formulation_scales(formulation, omega);  // the reference's refusals
    device_refill(system.matrix.mutable_values(), system.rhs, bound, mesh, dofs, pattern, omega, formulation);
}

void refill(SymmetricSystem& system, const BoundProblem& bound, const Mesh& mesh, const DofMap& dofs,
            const SparsityPattern& pattern, double omega, Conditioning formulation, const ScatterMap* scatter) {
    check_shapes(system.matrix.rows(), system.matrix.nnz(), system.rhs.size(), mesh, dofs, pattern, scatter);
    if (!pattern.upper_only)
        throw std::invalid_argument(
            "refill: a SparseSymmetric holds only the upper triangle, so it needs a pattern built with "
            "SparsityStorage::UpperTriangle");
    if (!formulation_scales(formulation, omega).symmetric)
        throw std::invalid_argument(std::string("refill: conditioning = ") + conditioning_keyword(formulation) +
                                    " does not give a symmetric matrix, so only half of it cannot be stored");
    device_refill(system.matrix.mutable_values(), system.rhs, bound, mesh, dofs, pattern, omega, formulation);
}

AssembledSystem assemble(const BoundProblem& bound, const Mesh& mesh, const DofMap& dofs,
                         const SparsityPattern& pattern, double omega, Conditioning formulation) {
    AssembledSystem out = make_system(pattern, dofs.num_total);
    refill(out, bound, mesh, dofs, pattern, omega, formulation);
    return out;
}

}  // namespace aphi_solver
