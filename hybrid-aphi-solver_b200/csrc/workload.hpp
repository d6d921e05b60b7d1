// Synthetic workloads (cylinder-in-box, torus with a cut port): the host-side inputs of the numeric
// hot path (per-tet geometry, per-tet DOF tables, bodies, ports and the
// upper-triangle CSR pattern), generated directly in the layouts the device
// kernels consume.
//
// The rules follow the reference's host pipeline so that the same mesh gives
// the same unknowns, numbered the same way:
//   mesh topology         src/mesh.cpp:26-122 (edges in ascending (lo, hi) order,
//                         tet_edge_signs +1 when the local edge runs lo -> hi)
//   n x A = 0 edges       src/tree_cotree.cpp:253-263 (every edge of a boundary face)
//   tree-cotree gauge     src/tree_cotree.cpp:89-250 (surface tree first, then an
//                         interior breadth-first tree taking each surface whole)
//   DOF numbering         src/dof_map.cpp:8-119 ([a | phi | V]) and local_dofs
//                         src/dof_map.cpp:121-194
//   sparsity              src/sparsity.cpp:19-136 (per-tet live lists, all pairs,
//                         upper triangle, plus voltage-port diagonals)
// The code is this project's own; the test suite checks its output against
// the reference's pipeline entry by entry.
#pragma once

#include <cstdint>
#include <vector>

namespace aphi_b200 {

struct Workload {
    int cells = 0;       // n: cells per cube side
    int num_nodes = 0;
    int num_tets = 0;
    int num_edges = 0;

    std::vector<double> xyz;           // 3 per node
    std::vector<int> tets;             // 4 per tet
    std::vector<int> edges;            // 2 per edge (lo, hi)
    std::vector<int> tet_edges;        // 6 per tet
    std::vector<int8_t> tet_sign;      // 6 per tet
    std::vector<int> body_of_tet;      // per tet

    // Bodies in declaration order; each body's tets ascending.
    std::vector<double> material;      // sigma, eps_r, mu_r per body
    std::vector<int> body_ptr;         // bodies + 1
    std::vector<int> body_tets;        // tets grouped by body

    // Unknowns [a | phi | V].
    int num_a = 0, num_phi = 0, num_ports = 0, num_total = 0;
    std::vector<int> edge_index;       // per mesh edge, -1 when eliminated
    std::vector<int> phi_index;        // per P2 node, -1 when not an unknown
    std::vector<uint8_t> dirichlet_edge;
    std::vector<uint8_t> tree_edge;

    // DofMap::local_dofs per tet: 6 edge entries then 10 P2 entries.
    std::vector<int> tet_idx;          // 16 per tet, -1 eliminated
    std::vector<double> tet_coeff;     // 16 per tet
    std::vector<double> tet_fixed;     // 20 per tet: 10 complex prescribed Phi values

    // Ports in declaration order.
    std::vector<int> port_current;     // 1 current driven, 0 voltage driven
    std::vector<int> port_row;         // global unknown of the port
    std::vector<double> port_amplitude;  // complex, 2 per port
    std::vector<double> port_value;      // complex prescribed value, 2 per port

    // Position of every unknown (edge midpoint, P2 node, port terminal
    // centroid), 3 per unknown: what a geometric ordering cuts on.
    std::vector<double> dof_xyz;

    // Upper-triangle CSR pattern of the assembled matrix.
    std::vector<int> row_ptr;
    std::vector<int> col_idx;
};

// The cylinder-in-box: unit cube, n^3 cells x 6 Kuhn tets, conductor where the
// tet centroid is within 0.2 of the line (0.5, 0.5, z), sigma 5.8e7 there and 0
// in air (mu_r = eps_r = 1), voltage ports v_top on the conductor's z = 1 cap
// and 0 V on its z = 0 cap. full_wave = 0 puts Phi on conductor tets only.
void build_cylinder(Workload& w, int n, double v_top, int full_wave);

// The torus: the same box and split, conductor (sigma 5.8e7) where the tet
// centroid is within 0.04 of the circle of radius 0.25 about (0.5, 0.5, 0.5) in
// the plane z = 0.5, air elsewhere. One internal current port (`current` A,
// phase 0) on the cut: the conductor-conductor faces in the plane y = 0.5 with
// x > 0.5, current direction hint +y. Phi on conductor tets only. n even.
void build_torus(Workload& w, int n, double current);

}  // namespace aphi_b200
