#include "workload.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>
#include <string>

namespace aphi_b200 {

namespace {

// Local edge -> local vertex pair, the order of include/aphi_solver/mesh.hpp:44-51.
constexpr int kEdgeVerts[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {2, 3}, {1, 3}};
// Local face i is opposite local vertex i (include/aphi_solver/mesh.hpp:58-63).
constexpr int kFaceVerts[4][3] = {{1, 2, 3}, {2, 3, 0}, {3, 0, 1}, {0, 1, 2}};
// Six Kuhn tets per cell, vertex offsets as in tools/generate_cube_mesh.py:32-39.
constexpr int kKuhn[6][4][3] = {{{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {1, 1, 1}},
                                {{0, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 1, 1}},
                                {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
                                {{0, 0, 0}, {0, 1, 1}, {0, 0, 1}, {1, 1, 1}},
                                {{0, 0, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}},
                                {{0, 0, 0}, {1, 0, 1}, {1, 0, 0}, {1, 1, 1}}};

struct Key3 {
    int a, b, c;
};

int64_t edge_key(int lo, int hi, int n) { return static_cast<int64_t>(lo) * n + hi; }

// Node -> incident edges, each node's list in ascending edge number (edges are
// visited in order, so appending keeps that order).
struct NodeEdges {
    std::vector<int> offset, other, edge;
};

NodeEdges node_edges(const Workload& w) {
    NodeEdges a;
    a.offset.assign(w.num_nodes + 1, 0);
    for (int e = 0; e < w.num_edges; ++e) {
        ++a.offset[w.edges[2 * e] + 1];
        ++a.offset[w.edges[2 * e + 1] + 1];
    }
    for (int i = 0; i < w.num_nodes; ++i) a.offset[i + 1] += a.offset[i];
    a.other.resize(a.offset.back());
    a.edge.resize(a.offset.back());
    std::vector<int> cur(a.offset.begin(), a.offset.end() - 1);
    for (int e = 0; e < w.num_edges; ++e) {
        const int i = w.edges[2 * e], j = w.edges[2 * e + 1];
        a.other[cur[i]] = j;
        a.edge[cur[i]++] = e;
        a.other[cur[j]] = i;
        a.edge[cur[j]++] = e;
    }
    return a;
}

void build_mesh(Workload& w, int n) {
    w.cells = n;
    const int np = n + 1;
    w.num_nodes = np * np * np;
    w.xyz.resize(3 * static_cast<size_t>(w.num_nodes));
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                const size_t id = (static_cast<size_t>(k) * np + j) * np + i;
                w.xyz[3 * id] = double(i) / n;
                w.xyz[3 * id + 1] = double(j) / n;
                w.xyz[3 * id + 2] = double(k) / n;
            }
    w.num_tets = 6 * n * n * n;
    w.tets.resize(4 * static_cast<size_t>(w.num_tets));
    size_t t = 0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int s = 0; s < 6; ++s, ++t)
                    for (int q = 0; q < 4; ++q)
                        w.tets[4 * t + q] = ((k + kKuhn[s][q][2]) * np + (j + kKuhn[s][q][1])) * np +
                                            (i + kKuhn[s][q][0]);

    // Edges: one record per (tet, local edge), sorted by the canonical
    // (lo, hi) key, then numbered in that order.
    const size_t nt = static_cast<size_t>(w.num_tets);
    std::vector<std::pair<int64_t, int>> rec(nt * 6);
    w.tet_sign.resize(nt * 6);
    for (size_t u = 0; u < nt; ++u)
        for (int le = 0; le < 6; ++le) {
            const int v0 = w.tets[4 * u + kEdgeVerts[le][0]];
            const int v1 = w.tets[4 * u + kEdgeVerts[le][1]];
            rec[6 * u + le] = {edge_key(std::min(v0, v1), std::max(v0, v1), w.num_nodes),
                               static_cast<int>(6 * u + le)};
            w.tet_sign[6 * u + le] = v0 < v1 ? 1 : -1;
        }
    std::sort(rec.begin(), rec.end());
    w.tet_edges.resize(nt * 6);
    w.edges.clear();
    for (size_t r = 0; r < rec.size(); ++r) {
        if (r == 0 || rec[r].first != rec[r - 1].first) {
            w.edges.push_back(static_cast<int>(rec[r].first / w.num_nodes));
            w.edges.push_back(static_cast<int>(rec[r].first % w.num_nodes));
        }
        w.tet_edges[rec[r].second] = static_cast<int>(w.edges.size() / 2) - 1;
    }
    w.num_edges = static_cast<int>(w.edges.size() / 2);
}

int find_edge(const Workload& w, int a, int b) {
    const int lo = std::min(a, b), hi = std::max(a, b);
    int l = 0, h = w.num_edges;
    while (l < h) {
        const int m = (l + h) / 2;
        const int ml = w.edges[2 * m], mh = w.edges[2 * m + 1];
        if (ml < lo || (ml == lo && mh < hi)) l = m + 1; else h = m;
    }
    if (l < w.num_edges && w.edges[2 * l] == lo && w.edges[2 * l + 1] == hi) return l;
    throw std::logic_error("workload: face edge not found in the edge list");
}

// Edges of faces that belong to exactly one tet: n x A = 0 there.
void boundary_edges(Workload& w) {
    const size_t nt = static_cast<size_t>(w.num_tets);
    struct F {
        int a, b, c;
        bool operator<(const F& o) const {
            return a != o.a ? a < o.a : (b != o.b ? b < o.b : c < o.c);
        }
        bool operator==(const F& o) const { return a == o.a && b == o.b && c == o.c; }
    };
    std::vector<F> faces(nt * 4);
    for (size_t u = 0; u < nt; ++u)
        for (int f = 0; f < 4; ++f) {
            int v[3] = {w.tets[4 * u + kFaceVerts[f][0]], w.tets[4 * u + kFaceVerts[f][1]],
                        w.tets[4 * u + kFaceVerts[f][2]]};
            std::sort(v, v + 3);
            faces[4 * u + f] = {v[0], v[1], v[2]};
        }
    std::sort(faces.begin(), faces.end());
    w.dirichlet_edge.assign(w.num_edges, 0);
    for (size_t i = 0; i < faces.size();) {
        size_t j = i;
        while (j < faces.size() && faces[j] == faces[i]) ++j;
        if (j - i == 1) {
            const F& f = faces[i];
            w.dirichlet_edge[find_edge(w, f.a, f.b)] = 1;
            w.dirichlet_edge[find_edge(w, f.b, f.c)] = 1;
            w.dirichlet_edge[find_edge(w, f.a, f.c)] = 1;
        }
        i = j;
    }
}

// Tree-cotree gauge: a spanning tree of each n x A = 0 surface built from its
// own edges first, then one breadth-first interior tree that enters each
// surface as a single group. Tree edges are eliminated (a = 0).
void gauge_tree(Workload& w) {
    const int n = w.num_nodes;
    const NodeEdges adj = node_edges(w);
    w.tree_edge.assign(w.num_edges, 0);

    // Surface components by union-find over surface edges.
    std::vector<int> uf(n);
    std::iota(uf.begin(), uf.end(), 0);
    auto find = [&](int x) {
        while (uf[x] != x) x = uf[x] = uf[uf[x]];
        return x;
    };
    std::vector<uint8_t> on_surface(n, 0);
    for (int e = 0; e < w.num_edges; ++e) {
        if (!w.dirichlet_edge[e]) continue;
        const int a = w.edges[2 * e], b = w.edges[2 * e + 1];
        const int ra = find(a), rb = find(b);
        if (ra != rb) uf[std::max(ra, rb)] = std::min(ra, rb);
        on_surface[a] = on_surface[b] = 1;
    }
    // Components numbered by their lowest node; members ascending.
    std::vector<int> comp(n, -1), comp_of_root(n, -1);
    int ncomp = 0;
    for (int i = 0; i < n; ++i) {
        if (!on_surface[i]) continue;
        int& c = comp_of_root[find(i)];
        if (c < 0) c = ncomp++;
        comp[i] = c;
    }
    std::vector<std::vector<int>> members(ncomp);
    for (int i = 0; i < n; ++i)
        if (comp[i] >= 0) members[comp[i]].push_back(i);

    // Surface trees, breadth first from each component's lowest node.
    std::vector<uint8_t> seen(n, 0);
    std::vector<int> queue;
    for (int c = 0; c < ncomp; ++c) {
        queue.assign(1, members[c].front());
        seen[members[c].front()] = 1;
        for (size_t h = 0; h < queue.size(); ++h) {
            const int u = queue[h];
            for (int k = adj.offset[u]; k < adj.offset[u + 1]; ++k) {
                const int e = adj.edge[k], v = adj.other[k];
                if (!w.dirichlet_edge[e] || seen[v]) continue;
                seen[v] = 1;
                w.tree_edge[e] = 1;
                queue.push_back(v);
            }
        }
    }

    // Interior tree: breadth first; a node on a surface brings its whole
    // surface into the tree at once.
    std::vector<uint8_t> visited(n, 0);
    queue.clear();
    size_t head = 0;
    auto take = [&](int node) {
        const int c = comp[node];
        if (c >= 0) {
            for (int m : members[c]) {
                visited[m] = 1;
                queue.push_back(m);
            }
        } else {
            visited[node] = 1;
            queue.push_back(node);
        }
    };
    auto drain = [&] {
        while (head < queue.size()) {
            const int u = queue[head++];
            for (int k = adj.offset[u]; k < adj.offset[u + 1]; ++k) {
                const int v = adj.other[k];
                if (visited[v]) continue;
                if (w.dirichlet_edge[adj.edge[k]])
                    throw std::logic_error("workload: interior tree reached a surface edge");
                w.tree_edge[adj.edge[k]] = 1;
                take(v);
            }
        }
    };
    take(ncomp > 0 ? members.front().front() : 0);
    drain();
    for (int s = 0; s < n; ++s)
        if (!visited[s]) {
            take(s);
            drain();
        }
}

// The unknowns, per-tet tables, positions and pattern, once the bodies, the
// gauge and the ports are known (src/dof_map.cpp:8-194, src/sparsity.cpp:19-136).
//   phi_port   P2 node -> the port claiming it (later ports win), -1 if none
//   port_cut   per port: 1 for an internal cut (two-sided), 0 for a terminal
//   tet_side   per tet: +1 on a cut's plus side, -1 on its minus side, 0 when
//              it touches no cut (empty when there are no cuts)
//   pinned     P2 nodes fixed at 0 V (floating conductors), unless a port claims them
//   port_xyz   3 per port: where its unknown sits for a geometric ordering
void finish(Workload& w, std::vector<int>& phi_port, const std::vector<uint8_t>& port_cut,
            const std::vector<int8_t>& tet_side, const std::vector<uint8_t>& pinned, int full_wave,
            const std::vector<double>& port_xyz) {
    const size_t nt = static_cast<size_t>(w.num_tets);
    const int num_p2 = w.num_nodes + w.num_edges;

    // A unknowns: edges neither on n x A = 0 nor in the tree, in edge order.
    w.edge_index.assign(w.num_edges, -1);
    for (int e = 0; e < w.num_edges; ++e)
        if (!w.dirichlet_edge[e] && !w.tree_edge[e]) w.edge_index[e] = w.num_a++;

    // Phi unknowns: P2 nodes touched by a Phi tet, minus port terminals, cut
    // nodes and pinned nodes.
    std::vector<uint8_t> present(num_p2, 0);
    for (size_t t = 0; t < nt; ++t) {
        if (!full_wave && w.material[3 * w.body_of_tet[t]] <= 0.0) continue;
        for (int q = 0; q < 4; ++q) present[w.tets[4 * t + q]] = 1;
        for (int le = 0; le < 6; ++le) present[w.num_nodes + w.tet_edges[6 * t + le]] = 1;
    }
    w.phi_index.assign(num_p2, -1);
    for (int i = 0; i < num_p2; ++i) {
        if (!present[i]) {
            phi_port[i] = -1;
            continue;
        }
        if (phi_port[i] < 0 && !pinned[i]) w.phi_index[i] = w.num_a + w.num_phi++;
    }

    // Ports: one unknown each after [a | phi].
    w.num_ports = static_cast<int>(w.port_current.size());
    w.port_row.resize(w.num_ports);
    for (int k = 0; k < w.num_ports; ++k) w.port_row[k] = w.num_a + w.num_phi + k;
    w.num_total = w.num_a + w.num_phi + w.num_ports;

    // Per-tet DOF tables.
    w.tet_idx.assign(16 * nt, -1);
    w.tet_coeff.assign(16 * nt, 0.0);
    w.tet_fixed.assign(20 * nt, 0.0);
    for (size_t t = 0; t < nt; ++t) {
        for (int le = 0; le < 6; ++le) {
            w.tet_idx[16 * t + le] = w.edge_index[w.tet_edges[6 * t + le]];
            w.tet_coeff[16 * t + le] = static_cast<double>(w.tet_sign[6 * t + le]);
        }
        for (int ln = 0; ln < 10; ++ln) {
            const int p2 = ln < 4 ? w.tets[4 * t + ln] : w.num_nodes + w.tet_edges[6 * t + ln - 4];
            if (w.phi_index[p2] >= 0) {
                w.tet_idx[16 * t + 6 + ln] = w.phi_index[p2];
                w.tet_coeff[16 * t + 6 + ln] = 1.0;
                continue;
            }
            const int k = phi_port[p2];
            if (k < 0) continue;
            // A cut's minus side reads the grounded zero (the defaults).
            if (port_cut[k] && !(tet_side.size() == nt && tet_side[t] > 0)) continue;
            if (w.port_current[k]) {
                w.tet_idx[16 * t + 6 + ln] = w.port_row[k];
                w.tet_coeff[16 * t + 6 + ln] = 1.0;
            } else {
                w.tet_fixed[20 * t + 2 * ln] = w.port_value[2 * k];
                w.tet_fixed[20 * t + 2 * ln + 1] = w.port_value[2 * k + 1];
            }
        }
    }

    // Unknown positions.
    w.dof_xyz.assign(3 * static_cast<size_t>(w.num_total), 0.0);
    auto p2_xyz = [&](int p2, double* out) {
        if (p2 < w.num_nodes) {
            for (int d = 0; d < 3; ++d) out[d] = w.xyz[3 * p2 + d];
        } else {
            const int e = p2 - w.num_nodes;
            for (int d = 0; d < 3; ++d) out[d] = 0.5 * (w.xyz[3 * w.edges[2 * e] + d] + w.xyz[3 * w.edges[2 * e + 1] + d]);
        }
    };
    for (int e = 0; e < w.num_edges; ++e)
        if (w.edge_index[e] >= 0) p2_xyz(w.num_nodes + e, &w.dof_xyz[3 * w.edge_index[e]]);
    for (int i = 0; i < num_p2; ++i)
        if (w.phi_index[i] >= 0) p2_xyz(i, &w.dof_xyz[3 * w.phi_index[i]]);
    for (int k = 0; k < w.num_ports; ++k)
        for (int d = 0; d < 3; ++d) w.dof_xyz[3 * w.port_row[k] + d] = port_xyz[3 * k + d];

    // Upper-triangle pattern: each tet's live unknowns, sorted and uniqued,
    // give every pair (i <= j); voltage-port rows get their diagonal.
    const int N = w.num_total;
    std::vector<std::vector<int>> rows(N);
    int live[16];
    for (size_t t = 0; t < nt; ++t) {
        int m = 0;
        for (int q = 0; q < 16; ++q)
            if (w.tet_idx[16 * t + q] >= 0) live[m++] = w.tet_idx[16 * t + q];
        std::sort(live, live + m);
        m = static_cast<int>(std::unique(live, live + m) - live);
        for (int i = 0; i < m; ++i)
            for (int j = i; j < m; ++j) rows[live[i]].push_back(live[j]);
    }
    for (int k = 0; k < w.num_ports; ++k)
        if (!w.port_current[k]) rows[w.port_row[k]].push_back(w.port_row[k]);
    w.row_ptr.assign(N + 1, 0);
    for (int r = 0; r < N; ++r) {
        auto& v = rows[r];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        w.row_ptr[r + 1] = w.row_ptr[r] + static_cast<int>(v.size());
    }
    w.col_idx.resize(w.row_ptr[N]);
    for (int r = 0; r < N; ++r) std::copy(rows[r].begin(), rows[r].end(), w.col_idx.begin() + w.row_ptr[r]);
}

// Bodies 0 = conductor (sigma 5.8e7), 1 = air, mu_r = eps_r = 1; a tet is
// conductor when inside(centroid), the centroid summed vertex by vertex and
// then scaled, in the reference's order.
template <class Inside>
void assign_bodies(Workload& w, Inside inside) {
    const size_t nt = static_cast<size_t>(w.num_tets);
    w.material = {5.8e7, 1.0, 1.0, 0.0, 1.0, 1.0};
    w.body_of_tet.assign(nt, 1);
    for (size_t t = 0; t < nt; ++t) {
        double c[3] = {0, 0, 0};
        for (int q = 0; q < 4; ++q)
            for (int d = 0; d < 3; ++d) c[d] += w.xyz[3 * w.tets[4 * t + q] + d];
        for (int d = 0; d < 3; ++d) c[d] *= 0.25;
        if (inside(c)) w.body_of_tet[t] = 0;
    }
    w.body_ptr.assign(3, 0);
    for (size_t t = 0; t < nt; ++t) ++w.body_ptr[w.body_of_tet[t] + 1];
    w.body_ptr[2] += w.body_ptr[1];
    w.body_tets.resize(nt);
    std::vector<int> cur(w.body_ptr.begin(), w.body_ptr.end() - 1);
    for (size_t t = 0; t < nt; ++t) w.body_tets[cur[w.body_of_tet[t]]++] = static_cast<int>(t);
}

void claim_face(const Workload& w, const int* v, int port, std::vector<int>& phi_port) {
    for (int q = 0; q < 3; ++q) phi_port[v[q]] = port;
    phi_port[w.num_nodes + find_edge(w, v[0], v[1])] = port;
    phi_port[w.num_nodes + find_edge(w, v[1], v[2])] = port;
    phi_port[w.num_nodes + find_edge(w, v[0], v[2])] = port;
}

}  // namespace

void build_cylinder(Workload& w, int n, double v_top, int full_wave) {
    if (n < 1) throw std::invalid_argument("build_cylinder: need at least one cell per side");
    w = Workload{};
    build_mesh(w, n);
    const size_t nt = static_cast<size_t>(w.num_tets);
    assign_bodies(w, [](const double* c) { return std::hypot(c[0] - 0.5, c[1] - 0.5) < 0.2; });
    if (w.body_ptr[1] == 0)
        throw std::invalid_argument("build_cylinder: no tet centroid lies inside the conductor at " +
                                    std::to_string(n) + " cells per side, so its ports have no faces");
    boundary_edges(w);
    gauge_tree(w);

    // Port terminals: faces of conductor tets with all three nodes on z = 1
    // (port 0, v_top) or z = 0 (port 1, 0 V).
    std::vector<int> phi_port(w.num_nodes + w.num_edges, -1);
    int port_faces[2] = {0, 0};
    for (size_t t = 0; t < nt; ++t) {
        if (w.body_of_tet[t] != 0) continue;
        for (int f = 0; f < 4; ++f) {
            int v[3];
            bool z0 = true, z1 = true;
            for (int q = 0; q < 3; ++q) {
                v[q] = w.tets[4 * t + kFaceVerts[f][q]];
                const double z = w.xyz[3 * v[q] + 2];
                if (z != 0.0) z0 = false;
                if (z != 1.0) z1 = false;
            }
            if (!z0 && !z1) continue;
            const int port = z1 ? 0 : 1;
            ++port_faces[port];
            claim_face(w, v, port, phi_port);
        }
    }
    if (port_faces[0] == 0 || port_faces[1] == 0)
        throw std::invalid_argument("build_cylinder: a port surface has no triangles in the mesh at " +
                                    std::to_string(n) + " cells per side");

    // Both ports voltage driven.
    w.port_current = {0, 0};
    w.port_amplitude = {v_top, 0.0, 0.0, 0.0};
    w.port_value = w.port_amplitude;
    finish(w, phi_port, {0, 0}, {}, std::vector<uint8_t>(w.num_nodes + w.num_edges, 0), full_wave,
           {0.5, 0.5, 1.0, 0.5, 0.5, 0.0});
}

void build_torus(Workload& w, int n, double current) {
    if (n < 2 || n % 2) throw std::invalid_argument("build_torus: need an even number of cells per side, so that y = 0.5 is a grid plane");
    w = Workload{};
    build_mesh(w, n);
    const size_t nt = static_cast<size_t>(w.num_tets);
    assign_bodies(w, [](const double* c) {
        return std::hypot(std::hypot(c[0] - 0.5, c[1] - 0.5) - 0.25, c[2] - 0.5) < 0.04;
    });
    if (w.body_ptr[1] == 0)
        throw std::invalid_argument("build_torus: no tet centroid lies inside the torus at " + std::to_string(n) +
                                    " cells per side");
    boundary_edges(w);
    gauge_tree(w);

    // Conductor faces, each with its tet: a face listed twice is shared by two
    // conductor tets (conduction across it), once is on the conductor's surface.
    struct FaceRec {
        int a, b, c, tet;
        bool operator<(const FaceRec& o) const {
            return a != o.a ? a < o.a : (b != o.b ? b < o.b : (c != o.c ? c < o.c : tet < o.tet));
        }
    };
    std::vector<FaceRec> faces;
    for (size_t t = 0; t < nt; ++t) {
        if (w.body_of_tet[t] != 0) continue;
        for (int f = 0; f < 4; ++f) {
            int v[3] = {w.tets[4 * t + kFaceVerts[f][0]], w.tets[4 * t + kFaceVerts[f][1]],
                        w.tets[4 * t + kFaceVerts[f][2]]};
            std::sort(v, v + 3);
            faces.push_back({v[0], v[1], v[2], static_cast<int>(t)});
        }
    }
    std::sort(faces.begin(), faces.end());

    // The cut: conductor-conductor faces in the plane y = 0.5 with x > 0.5.
    // Conduction paths: conductor tets joined across shared faces.
    std::vector<int> uf(nt);
    std::iota(uf.begin(), uf.end(), 0);
    auto find = [&](int x) {
        while (uf[x] != x) x = uf[x] = uf[uf[x]];
        return x;
    };
    std::vector<int> phi_port(w.num_nodes + w.num_edges, -1);
    std::vector<uint8_t> cut_node(w.num_nodes, 0), cut_tet(nt, 0);
    int cut_faces = 0;
    for (size_t i = 0; i + 1 < faces.size(); ++i) {
        const FaceRec& f = faces[i];
        const FaceRec& g = faces[i + 1];
        if (f.a != g.a || f.b != g.b || f.c != g.c) continue;
        const int ra = find(f.tet), rb = find(g.tet);
        if (ra != rb) uf[std::max(ra, rb)] = std::min(ra, rb);
        const int v[3] = {f.a, f.b, f.c};
        bool on_cut = true;
        for (int q = 0; q < 3; ++q)
            if (w.xyz[3 * v[q] + 1] != 0.5 || !(w.xyz[3 * v[q]] > 0.5)) on_cut = false;
        if (!on_cut) continue;
        ++cut_faces;
        claim_face(w, v, 0, phi_port);
        for (int q = 0; q < 3; ++q) cut_node[v[q]] = 1;
        cut_tet[f.tet] = cut_tet[g.tet] = 1;
    }
    if (cut_faces == 0)
        throw std::invalid_argument("build_torus: the cut plane crosses no conductor at " + std::to_string(n) +
                                    " cells per side");

    // Side of every tet touching the cut (a cut face or a cut node): the sign
    // of (centroid - origin) . d with d = +y (the current-direction hint) and
    // origin on the plane, i.e. of centroid.y - 0.5, summed in the reference's
    // order (src/problem_binding.cpp:702-737).
    std::vector<int8_t> tet_side(nt, 0);
    for (size_t t = 0; t < nt; ++t) {
        bool touches = cut_tet[t] != 0;
        for (int q = 0; q < 4 && !touches; ++q) touches = cut_node[w.tets[4 * t + q]] != 0;
        if (!touches) continue;
        double cy = 0;
        for (int q = 0; q < 4; ++q) cy += w.xyz[3 * w.tets[4 * t + q] + 1];
        cy *= 0.25;
        tet_side[t] = cy - 0.5 > 0.0 ? 1 : -1;
    }

    // A conduction path the cut does not touch is floating: its lowest node
    // is pinned at 0 V (src/problem_binding.cpp:581-690).
    std::vector<uint8_t> pinned(w.num_nodes + w.num_edges, 0);
    std::vector<int> lowest(nt, -1);
    std::vector<uint8_t> referenced(nt, 0);
    for (size_t t = 0; t < nt; ++t) {
        if (w.body_of_tet[t] != 0) continue;
        const int r = find(static_cast<int>(t));
        if (cut_tet[t]) referenced[r] = 1;
        for (int q = 0; q < 4; ++q) {
            const int v = w.tets[4 * t + q];
            if (lowest[r] < 0 || v < lowest[r]) lowest[r] = v;
        }
    }
    for (size_t r = 0; r < nt; ++r)
        if (lowest[r] >= 0 && !referenced[r] && phi_port[lowest[r]] < 0) pinned[lowest[r]] = 1;

    // One internal current port.
    w.port_current = {1};
    w.port_amplitude = {current, 0.0};
    w.port_value = {0.0, 0.0};
    finish(w, phi_port, {1}, tet_side, pinned, 0, {0.75, 0.5, 0.5});
}

}  // namespace aphi_b200
