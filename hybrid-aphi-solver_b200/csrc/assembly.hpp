// Device assembly state: one per mesh (pattern + DOF tables), reused at every
// frequency. See assembly.cu for the kernels.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <memory>

#include "aphi_b200.h"

namespace aphi_b200 {

constexpr int kMaxBatchOmegas = 64;

struct Assembly {
    int N = 0, nnz = 0, T = 0, num_bodies = 0, num_ports = 0;
    bool upper_only = true;
    long long tet_terms = 0;  // terms produced by tets
    long long num_terms = 0;  // plus port terms
    long long bytes = 0;

    double* d_xyz = nullptr;
    int* d_tets = nullptr;
    int* d_visit_tet = nullptr;
    int* d_visit_body = nullptr;
    double* d_material = nullptr;
    int* d_tet_idx = nullptr;
    double* d_tet_coeff = nullptr;
    double* d_tet_fixed = nullptr;
    long long* d_term_off = nullptr;
    int* d_dest_ptr = nullptr;
    int* d_dest_terms = nullptr;
    double* d_terms = nullptr;  // complex, terms_capacity x num_terms
    int terms_capacity = 0;
    int* d_port_current = nullptr;
    double* d_port_amp = nullptr;
    double* d_port_value = nullptr;
    int* d_err = nullptr;

    ~Assembly();
};

// Post-solve fields over an assembly's mesh (compute_fields, src/postprocess.cpp:223-486).
struct Fields {
    const Assembly* A = nullptr;  // must outlive the Fields
    int T = 0, P = 0, nv = 0, ne = 0;
    int interface_nodes = 0, orphans = 0;
    int* d_tet_edges = nullptr;
    int* d_body_of_tet = nullptr;
    int* d_inc_ptr = nullptr;  // P2 node -> 10 * tet + local node, increasing tet
    int* d_inc = nullptr;
    double* d_sig_max = nullptr;
    double* d_mu_max = nullptr;
    unsigned char* d_sig_uniform = nullptr;
    unsigned char* d_mu_uniform = nullptr;
    double* d_contrib = nullptr;
    int* d_err = nullptr;
    ~Fields();
};
using FieldsOut = aphi_fields_out;
std::unique_ptr<Fields> fields_create(const Assembly& A, int num_nodes, int num_edges, const int* tet_edges);
void fields_compute(Fields& F, double omega, int conditioning, const double* x_dev, const FieldsOut& out,
                    cudaStream_t stream);

// device_setup: build the term offsets and slot -> term lists on the device
// (setup.cu) instead of on the host; the arrays are identical.
std::unique_ptr<Assembly> assembly_create(const aphi_assembly_desc& d, bool device_setup = false);
void assembly_refill(Assembly& A, int nfreq, const double* omegas, int cond, double* values_dev,
                     double* rhs_dev, cudaStream_t stream);
void assembly_check_errors(Assembly& A, cudaStream_t stream);
void element_blocks_host(int ntets, const double* xyz, double nu, const double* alpha,
                         const double* beta, double* aa, double* ap, double* pp);
void assembly_coefficients(double sigma, double eps_r, double mu_r, double omega, double* out5);
void formulation_scales_host(int cond, double omega, std::complex<double>& row,
                             std::complex<double>& col, bool& symmetric);

}  // namespace aphi_b200
