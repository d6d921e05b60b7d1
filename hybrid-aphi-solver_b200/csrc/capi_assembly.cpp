// C ABI: status strings, workloads and assembly. Every entry point catches
// everything and returns a status code.
#include <cstring>
#include <string>

#include "assembly.hpp"
#include "setup.hpp"
#include "capi_util.hpp"
#include "common.cuh"
#include "ordering.hpp"
#include "workload.hpp"

using namespace aphi_b200;

struct aphi_workload {
    Workload w;
    long long num_terms = 0;
};

struct aphi_assembly {
    std::unique_ptr<Assembly> a;
};

struct aphi_fields {
    std::unique_ptr<Fields> f;
};

#include <atomic>

namespace aphi_b200 {
thread_local char g_last_error[kLastErrorBytes];

void set_last_error(const char* msg) {
    size_t i = 0;
    for (; msg && msg[i] && i + 1 < static_cast<size_t>(kLastErrorBytes); ++i) g_last_error[i] = msg[i];
    g_last_error[i] = 0;
}
static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}

extern "C" {

const char* aphi_status_string(int s) {
    switch (s) {
        case APHI_OK: return "ok";
        case APHI_ERR_BAD_SHAPE: return "bad shape or refused argument";
        case APHI_ERR_PATTERN_MISMATCH: return "symbolic and numeric passes disagree";
        case APHI_ERR_PIVOT_FLOOR: return "pivot at or below the floor";
        case APHI_ERR_NAN: return "non-finite value";
        case APHI_ERR_IR_STALL: return "iterative refinement stalled";
        case APHI_ERR_TIMEOUT: return "bounded device wait timed out";
        case APHI_ERR_OOM: return "device out of memory";
        case APHI_ERR_ADMISSION: return "request rejected by admission";
        case APHI_ERR_CUDA: return "CUDA error";
        case APHI_ERR_ZERO_PIVOT: return "zero diagonal in a solve";
        case APHI_ERR_DEGENERATE_TET: return "degenerate tetrahedron";
        case APHI_ERR_INVALID: return "invalid argument";
    }
    return "unknown status";
}

const char* aphi_last_error(void) { return g_last_error; }

int64_t aphi_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int aphi_workload_cylinder(int cells, double v_top, int full_wave, aphi_workload** out) {
    return guard([&] {
        if (!out) throw Error(APHI_ERR_INVALID, "aphi_workload_cylinder: null output");
        auto* w = new aphi_workload;
        try {
            build_cylinder(w->w, cells, v_top, full_wave);
        } catch (...) {
            delete w;
            throw;
        }
        *out = w;
    });
}

int aphi_workload_torus(int cells, double current, aphi_workload** out) {
    return guard([&] {
        if (!out) throw Error(APHI_ERR_INVALID, "aphi_workload_torus: null output");
        auto* w = new aphi_workload;
        try {
            build_torus(w->w, cells, current);
        } catch (...) {
            delete w;
            throw;
        }
        *out = w;
    });
}

void aphi_workload_free(aphi_workload* w) { delete w; }

int aphi_workload_sizes(const aphi_workload* h, int64_t* s) {
    return guard([&] {
        if (!h || !s) throw Error(APHI_ERR_INVALID, "aphi_workload_sizes: null argument");
        const Workload& w = h->w;
        s[0] = w.num_nodes;
        s[1] = w.num_tets;
        s[2] = w.num_edges;
        s[3] = w.num_total;
        s[4] = w.row_ptr.empty() ? 0 : w.row_ptr.back();
        s[5] = w.num_a;
        s[6] = w.num_phi;
        s[7] = w.num_ports;
        s[8] = static_cast<int64_t>(w.material.size() / 3);
        s[9] = h->num_terms;
    });
}

int aphi_workload_array(const aphi_workload* h, const char* name, const void** data, int64_t* count) {
    return guard([&] {
        if (!h || !name || !data || !count) throw Error(APHI_ERR_INVALID, "aphi_workload_array: null argument");
        const Workload& w = h->w;
        auto set = [&](const auto& v) {
            *data = v.data();
            *count = static_cast<int64_t>(v.size());
        };
        const std::string n(name);
        if (n == "xyz") set(w.xyz);
        else if (n == "tets") set(w.tets);
        else if (n == "tet_idx") set(w.tet_idx);
        else if (n == "tet_coeff") set(w.tet_coeff);
        else if (n == "tet_fixed") set(w.tet_fixed);
        else if (n == "material") set(w.material);
        else if (n == "body_ptr") set(w.body_ptr);
        else if (n == "body_tets") set(w.body_tets);
        else if (n == "port_current") set(w.port_current);
        else if (n == "port_row") set(w.port_row);
        else if (n == "port_amplitude") set(w.port_amplitude);
        else if (n == "port_value") set(w.port_value);
        else if (n == "row_ptr") set(w.row_ptr);
        else if (n == "col_idx") set(w.col_idx);
        else if (n == "edges") set(w.edges);
        else if (n == "edge_index") set(w.edge_index);
        else if (n == "phi_index") set(w.phi_index);
        else if (n == "tet_edges") set(w.tet_edges);
        else if (n == "body_of_tet") set(w.body_of_tet);
        else if (n == "dof_xyz") set(w.dof_xyz);
        else throw Error(APHI_ERR_INVALID, "aphi_workload_array: unknown array '" + n + "'");
    });
}

int aphi_order_nested_dissection(int n, const int* row_ptr, const int* col_idx, const double* xyz, int leaf,
                                 int* perm) {
    return guard([&] { nested_dissection(n, row_ptr, col_idx, xyz, leaf, perm); });
}

int aphi_order_amd(int n, const int* row_ptr, const int* col_idx, int* perm) {
    return guard([&] {
        if (n < 0 || (n > 0 && (!row_ptr || !col_idx || !perm))) throw Error(APHI_ERR_INVALID, "aphi_order_amd: null argument");
        if (n > 0) reference_amd(n, row_ptr, col_idx, perm);
    });
}

int aphi_order_rcm(int n, const int* row_ptr, const int* col_idx, int* perm) {
    return guard([&] {
        if (n < 0 || (n > 0 && (!row_ptr || !col_idx || !perm))) throw Error(APHI_ERR_INVALID, "aphi_order_rcm: null argument");
        if (n > 0) reference_rcm(n, row_ptr, col_idx, perm);
    });
}

int aphi_assembly_create(const aphi_assembly_desc* desc, aphi_assembly** out) {
    return guard([&] {
        if (!desc || !out) throw Error(APHI_ERR_INVALID, "aphi_assembly_create: null argument");
        auto* h = new aphi_assembly;
        try {
            h->a = assembly_create(*desc);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int aphi_assembly_create_device_setup(const aphi_assembly_desc* desc, aphi_assembly** out) {
    return guard([&] {
        if (!desc || !out) throw Error(APHI_ERR_INVALID, "aphi_assembly_create_device_setup: null argument");
        auto* h = new aphi_assembly;
        try {
            h->a = assembly_create(*desc, true);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int aphi_assembly_maps(const aphi_assembly* h, int64_t* term_off, int* dest_ptr, int* dest_terms) {
    return guard([&] {
        if (!h) throw Error(APHI_ERR_INVALID, "aphi_assembly_maps: null assembly");
        const Assembly& A = *h->a;
        if (term_off)
            APHI_CUDA(cudaMemcpy(term_off, A.d_term_off, sizeof(long long) * (static_cast<size_t>(A.T) + 1),
                                 cudaMemcpyDeviceToHost));
        if (dest_ptr)
            APHI_CUDA(cudaMemcpy(dest_ptr, A.d_dest_ptr, sizeof(int) * (static_cast<size_t>(A.nnz) + A.N + 1),
                                 cudaMemcpyDeviceToHost));
        if (dest_terms)
            APHI_CUDA(cudaMemcpy(dest_terms, A.d_dest_terms, sizeof(int) * static_cast<size_t>(A.num_terms),
                                 cudaMemcpyDeviceToHost));
    });
}

int aphi_pattern_build(int n, int num_tets, const int* tet_idx, int num_diag, const int* diag_rows, int upper_only,
                       int* row_ptr, int* col_idx, int64_t capacity, int64_t* nnz) {
    return guard([&] {
        if (!tet_idx || !row_ptr || !nnz || (num_diag > 0 && !diag_rows))
            throw Error(APHI_ERR_INVALID, "aphi_pattern_build: null argument");
        const long long got = pattern_build(n, num_tets, tet_idx, num_diag, diag_rows, upper_only != 0, row_ptr,
                                            col_idx, capacity);
        *nnz = got;
        if (got > capacity || !col_idx)
            throw Error(APHI_ERR_BAD_SHAPE, "aphi_pattern_build: the pattern has " + std::to_string(got) +
                                                " entries, more than the capacity given");
    });
}

int aphi_assembly_destroy(aphi_assembly* a) {
    return guard([&] { delete a; });
}

int aphi_assembly_info(const aphi_assembly* h, int64_t* info) {
    return guard([&] {
        if (!h || !info) throw Error(APHI_ERR_INVALID, "aphi_assembly_info: null argument");
        info[0] = h->a->nnz;
        info[1] = h->a->N;
        info[2] = h->a->num_terms;
        info[3] = h->a->bytes + static_cast<int64_t>(h->a->terms_capacity) * h->a->num_terms * 16;
    });
}

int aphi_formulation_scales(int conditioning, double omega, double* rc, int* symmetric) {
    return guard([&] {
        std::complex<double> r, c;
        bool sym = false;
        formulation_scales_host(conditioning, omega, r, c, sym);
        if (rc) {
            rc[0] = r.real();
            rc[1] = r.imag();
            rc[2] = c.real();
            rc[3] = c.imag();
        }
        if (symmetric) *symmetric = sym ? 1 : 0;
    });
}

int aphi_refill(aphi_assembly* h, double omega, int conditioning, double* values_dev, double* rhs_dev,
                void* stream) {
    return aphi_refill_batch(h, 1, &omega, conditioning, values_dev, rhs_dev, stream);
}

int aphi_refill_batch(aphi_assembly* h, int nfreq, const double* omegas, int conditioning,
                      double* values_dev, double* rhs_dev, void* stream) {
    return guard([&] {
        if (!h || !omegas || !values_dev || !rhs_dev) throw Error(APHI_ERR_INVALID, "aphi_refill: null argument");
        assembly_refill(*h->a, nfreq, omegas, conditioning, values_dev, rhs_dev,
                        static_cast<cudaStream_t>(stream));
    });
}

int aphi_refill_host(aphi_assembly* h, double omega, int conditioning, double* values, double* rhs) {
    return guard([&] {
        if (!h || !values || !rhs) throw Error(APHI_ERR_INVALID, "aphi_refill_host: null argument");
        Assembly& A = *h->a;
        double *dv = nullptr, *dr = nullptr;
        APHI_CUDA(cudaMalloc(&dv, std::max<size_t>(1, 2ULL * A.nnz) * sizeof(double)));
        APHI_CUDA(cudaMalloc(&dr, std::max<size_t>(1, 2ULL * A.N) * sizeof(double)));
        try {
            assembly_refill(A, 1, &omega, conditioning, dv, dr, nullptr);
            assembly_check_errors(A, nullptr);
            APHI_CUDA(cudaMemcpy(values, dv, 2ULL * A.nnz * sizeof(double), cudaMemcpyDeviceToHost));
            APHI_CUDA(cudaMemcpy(rhs, dr, 2ULL * A.N * sizeof(double), cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(dv);
            cudaFree(dr);
            throw;
        }
        cudaFree(dv);
        cudaFree(dr);
    });
}

int aphi_fields_create(const aphi_assembly* a, int num_nodes, int num_edges, const int* tet_edges,
                       aphi_fields** out) {
    return guard([&] {
        if (!a || !out) throw Error(APHI_ERR_INVALID, "aphi_fields_create: null argument");
        auto* h = new aphi_fields;
        try {
            h->f = fields_create(*a->a, num_nodes, num_edges, tet_edges);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int aphi_fields_destroy(aphi_fields* f) {
    return guard([&] { delete f; });
}

int aphi_fields_sizes(const aphi_fields* h, int64_t* s) {
    return guard([&] {
        if (!h || !s) throw Error(APHI_ERR_INVALID, "aphi_fields_sizes: null argument");
        const Fields& F = *h->f;
        s[0] = F.T;
        s[1] = F.P;
        s[2] = F.nv;
        s[3] = F.ne;
        s[4] = F.interface_nodes;
        s[5] = F.orphans;
    });
}

int aphi_fields_compute(aphi_fields* h, double omega, int conditioning, const double* x_dev,
                        const aphi_fields_out* out, void* stream) {
    return guard([&] {
        if (!h || !out) throw Error(APHI_ERR_INVALID, "aphi_fields_compute: null argument");
        fields_compute(*h->f, omega, conditioning, x_dev, *out, static_cast<cudaStream_t>(stream));
    });
}

int aphi_element_blocks(int ntets, const double* xyz, double nu, const double* alpha, const double* beta,
                        double* aa, double* ap, double* pp) {
    return guard([&] {
        if (ntets < 0 || !xyz || !alpha || !beta || !aa || !ap || !pp)
            throw Error(APHI_ERR_INVALID, "aphi_element_blocks: null argument");
        if (ntets == 0) return;
        element_blocks_host(ntets, xyz, nu, alpha, beta, aa, ap, pp);
    });
}

void aphi_element_coefficients(double sigma, double eps_r, double mu_r, double omega, double* out5) {
    assembly_coefficients(sigma, eps_r, mu_r, omega, out5);
}

}  // extern "C"
