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

}  // namespace

void build_cylinder(Workload& w, int n, double v_top, int full_wave) {
    if (n < 1) throw std::invalid_argument("build_cylinder: need at least one cell per side");
    w = Workload{};
    build_mesh(w, n);
    const size_t nt = static_cast<size_t>(w.num_tets);

    // Bodies: 0 = wire (sigma 5.8e7), 1 = air, by tet centroid distance to the axis.
    w.material = {5.8e7, 1.0, 1.0, 0.0, 1.0, 1.0};
    w.body_of_tet.assign(nt, 1);
    for (size_t t = 0; t < nt; ++t) {
        double cx = 0, cy = 0;
        for (int q = 0; q < 4; ++q) {
            cx += w.xyz[3 * w.tets[4 * t + q]];
            cy += w.xyz[3 * w.tets[4 * t + q] + 1];
        }
        // The same arithmetic order as a centroid summed vertex by vertex then scaled.
        cx *= 0.25;
        cy *= 0.25;
        if (std::hypot(cx - 0.5, cy - 0.5) < 0.2) w.body_of_tet[t] = 0;
    }
    w.body_ptr.assign(3, 0);
    for (size_t t = 0; t < nt; ++t) ++w.body_ptr[w.body_of_tet[t] + 1];
    if (w.body_ptr[1] == 0)
        throw std::invalid_argument("build_cylinder: no tet centroid lies inside the conductor at " +
                                    std::to_string(n) + " cells per side, so its ports have no faces");
    w.body_ptr[2] += w.body_ptr[1];
    w.body_tets.resize(nt);
    {
        std::vector<int> cur(w.body_ptr.begin(), w.body_ptr.end() - 1);
        for (size_t t = 0; t < nt; ++t) w.body_tets[cur[w.body_of_tet[t]]++] = static_cast<int>(t);
    }

    boundary_edges(w);
    gauge_tree(w);

    // Port terminals: faces of conductor tets with all three nodes on z = 1
    // (port 0, v_top) or z = 0 (port 1, 0 V).
    const int num_p2 = w.num_nodes + w.num_edges;
    std::vector<int> phi_port(num_p2, -1);
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
            for (int q = 0; q < 3; ++q) phi_port[v[q]] = port;
            phi_port[w.num_nodes + find_edge(w, v[0], v[1])] = port;
            phi_port[w.num_nodes + find_edge(w, v[1], v[2])] = port;
            phi_port[w.num_nodes + find_edge(w, v[0], v[2])] = port;
        }
    }

    if (port_faces[0] == 0 || port_faces[1] == 0)
        throw std::invalid_argument("build_cylinder: a port surface has no triangles in the mesh at " +
                                    std::to_string(n) + " cells per side");

    // A unknowns: edges neither on n x A = 0 nor in the tree, in edge order.
    w.edge_index.assign(w.num_edges, -1);
    for (int e = 0; e < w.num_edges; ++e)
        if (!w.dirichlet_edge[e] && !w.tree_edge[e]) w.edge_index[e] = w.num_a++;

    // Phi unknowns: P2 nodes touched by a Phi tet, minus port terminals.
    std::vector<uint8_t> present(num_p2, 0);
    for (size_t t = 0; t < nt; ++t) {
        if (!full_wave && w.body_of_tet[t] != 0) continue;
        for (int q = 0; q < 4; ++q) present[w.tets[4 * t + q]] = 1;
        for (int le = 0; le < 6; ++le) present[w.num_nodes + w.tet_edges[6 * t + le]] = 1;
    }
    w.phi_index.assign(num_p2, -1);
    for (int i = 0; i < num_p2; ++i) {
        if (!present[i]) {
            phi_port[i] = -1;
            continue;
        }
        if (phi_port[i] < 0) w.phi_index[i] = w.num_a + w.num_phi++;
    }

    // Ports: both voltage driven, one unknown each after [a | phi].
    w.num_ports = 2;
    w.port_current = {0, 0};
    w.port_row = {w.num_a + w.num_phi, w.num_a + w.num_phi + 1};
    w.port_amplitude = {v_top, 0.0, 0.0, 0.0};
    w.port_value = w.port_amplitude;
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
            } else if (phi_port[p2] >= 0) {
                const int k = phi_port[p2];
                if (w.port_current[k]) {
                    w.tet_idx[16 * t + 6 + ln] = w.port_row[k];
                    w.tet_coeff[16 * t + 6 + ln] = 1.0;
                } else {
                    w.tet_fixed[20 * t + 2 * ln] = w.port_value[2 * k];
                    w.tet_fixed[20 * t + 2 * ln + 1] = w.port_value[2 * k + 1];
                }
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
    for (int k = 0; k < w.num_ports; ++k) {
        w.dof_xyz[3 * w.port_row[k]] = 0.5;
        w.dof_xyz[3 * w.port_row[k] + 1] = 0.5;
        w.dof_xyz[3 * w.port_row[k] + 2] = k == 0 ? 1.0 : 0.0;
    }

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

}  // namespace aphi_b200
