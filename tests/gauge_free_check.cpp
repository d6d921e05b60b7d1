// The reference pipeline end to end on the cylinder-in-box, written with the
// reference's own interfaces: bind, DOF map, sparsity, refill, solve_symmetric,
// compute_fields and recover_gauge_free_potential (whose second solve is
// another solve_symmetric, src/gauge_free_potential.cpp:177). oracle/Makefile
// links this file twice: against the reference's own objects, and against the
// B200 drop-in units (refill and both solves then run on the device). Test
// infrastructure: tests/test_dropin_gpu.py compares the two outputs.
//
//   gauge_free_check <cells> <hz> <out.bin>
//
// out.bin: int32 n, int32 n_vertex, int32 n_ports, int32 converged; double
// main residual, recovered residual; then x (n complex), phi_vertex
// (n_vertex complex), port_potential (n_ports complex).
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <vector>

#include "aphi_solver/assembly.hpp"
#include "aphi_solver/dof_map.hpp"
#include "aphi_solver/factorization.hpp"
#include "aphi_solver/gauge_free_potential.hpp"
#include "aphi_solver/postprocess.hpp"
#include "aphi_solver/problem_binding.hpp"
#include "aphi_solver/sparsity.hpp"
#include "ref_meshes.hpp"

using namespace aphi_solver;

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <cells> <hz> <out.bin>\n", argv[0]);
        return 2;
    }
    try {
        const int cells = std::atoi(argv[1]);
        const double omega = 2.0 * 3.14159265358979323846 * std::atof(argv[2]);
        Mesh mesh;
        ref_meshes::build_cylinder_mesh(mesh, cells);
        Problem pr;
        pr.type = AnalysisType::Frequency;
        pr.frequencies = {omega / (2.0 * 3.14159265358979323846)};
        pr.formulation = Formulation::Reduced;
        pr.conditioning = Conditioning::RowScaled;
        Body wire;
        wire.name = "B1";
        wire.volume = "wire";
        wire.sigma = 5.8e7;
        Body air;
        air.name = "B2";
        air.volume = "air";
        air.sigma = 0.0;
        pr.bodies = {wire, air};
        Port top;
        top.name = "P1";
        top.type = PortType::BoundaryVoltage;
        top.surface = {"wire_top"};
        top.amplitude = 1.0;
        Port bottom;
        bottom.name = "P2";
        bottom.type = PortType::BoundaryVoltage;
        bottom.surface = {"wire_bottom"};
        bottom.amplitude = 0.0;
        pr.ports = {top, bottom};

        const BoundProblem bound = bind_to_mesh(pr, mesh);
        const DofMap dofs = build_dof_map(bound, mesh);
        const SparsityPattern pattern = build_sparsity(dofs, bound, mesh, SparsityStorage::UpperTriangle);
        SymmetricSystem sys = make_symmetric_system(pattern, dofs.num_total);
        refill(sys, bound, mesh, dofs, pattern, omega, Conditioning::RowScaled);

        std::vector<std::complex<double>> x;
        SolveReport rep;
        if (!solve_symmetric(sys.matrix, sys.rhs, x, rep)) {
            std::fprintf(stderr, "main solve failed\n");
            return 1;
        }
        Solution sol;
        sol.x = x;
        sol.omega = omega;
        sol.conditioning = Conditioning::RowScaled;
        const FieldOutput fields = compute_fields(mesh, bound, dofs, sol);
        const GaugeFreePotential g = recover_gauge_free_potential(mesh, bound, dofs, fields, omega);

        std::FILE* f = std::fopen(argv[3], "wb");
        if (!f) return 1;
        const int head[4] = {dofs.num_total, static_cast<int>(g.phi_vertex.size()),
                             static_cast<int>(g.port_potential.size()), g.converged ? 1 : 0};
        const double res[2] = {rep.residual, g.residual};
        std::fwrite(head, sizeof(int), 4, f);
        std::fwrite(res, sizeof(double), 2, f);
        std::fwrite(x.data(), sizeof(std::complex<double>), x.size(), f);
        std::fwrite(g.phi_vertex.data(), sizeof(std::complex<double>), g.phi_vertex.size(), f);
        std::fwrite(g.port_potential.data(), sizeof(std::complex<double>), g.port_potential.size(), f);
        std::fclose(f);
        std::printf("n %d vertices %zu converged %d residual %.3e recovered residual %.3e\n", dofs.num_total,
                    g.phi_vertex.size(), g.converged ? 1 : 0, rep.residual, g.residual);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "gauge_free_check: %s\n", e.what());
        return 1;
    }
}
