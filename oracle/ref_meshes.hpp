// The synthetic meshes of the checkers, built with the reference's own types
// (aphi_solver::Mesh): the unit cube at n^3 cells, each split into the six
// Kuhn tets of tools/generate_cube_mesh.py:32-39, with the physical tags the
// problems bind to. Test infrastructure only.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "aphi_solver/mesh.hpp"

namespace ref_meshes {

using aphi_solver::FaceTets;
using aphi_solver::Mesh;
using aphi_solver::TaggedFace;
using aphi_solver::TetVerts;
using aphi_solver::Vec3;
using aphi_solver::kTetLocalFaceVerts;

// Kuhn split of one hex cell: six tets sharing the main diagonal (0,0,0)-(1,1,1).
inline constexpr int kKuhn[6][4][3] = {{{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {1, 1, 1}},
                            {{0, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 1, 1}},
                            {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
                            {{0, 0, 0}, {0, 1, 1}, {0, 0, 1}, {1, 1, 1}},
                            {{0, 0, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}},
                            {{0, 0, 0}, {1, 0, 1}, {1, 0, 0}, {1, 1, 1}}};

inline void build_cylinder_mesh(Mesh& m, int n) {
    auto id = [&](int i, int j, int k) { return (k * (n + 1) + j) * (n + 1) + i; };
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i)
                m.nodes.push_back(Vec3(double(i) / n, double(j) / n, double(k) / n));
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int t = 0; t < 6; ++t) {
                    TetVerts v;
                    for (int q = 0; q < 4; ++q)
                        v[q] = id(i + kKuhn[t][q][0], j + kKuhn[t][q][1], k + kKuhn[t][q][2]);
                    m.tets.push_back(v);
                }
    m.build_topology();
    m.tet_tags.assign(m.tets.size(), 2);
    for (std::size_t t = 0; t < m.tets.size(); ++t) {
        Vec3 c(0, 0, 0);
        for (int q = 0; q < 4; ++q) c = c + m.nodes[m.tets[t][q]];
        c = c * 0.25;
        if (std::hypot(c.x - 0.5, c.y - 0.5) < 0.2) m.tet_tags[t] = 1;
    }
    m.physical_names = {{3, 1, "wire"}, {3, 2, "air"}, {2, 10, "wire_bottom"}, {2, 11, "wire_top"}};
    for (std::size_t t = 0; t < m.tets.size(); ++t) {
        if (m.tet_tags[t] != 1) continue;
        for (int f = 0; f < 4; ++f) {
            std::array<int, 3> fv;
            for (int q = 0; q < 3; ++q) fv[q] = m.tets[t][kTetLocalFaceVerts[f][q]];
            bool b0 = true, b1 = true;
            for (int q = 0; q < 3; ++q) {
                if (m.nodes[fv[q]].z != 0.0) b0 = false;
                if (m.nodes[fv[q]].z != 1.0) b1 = false;
            }
            if (b0 || b1) {
                TaggedFace tf;
                tf.nodes = fv;
                std::sort(tf.nodes.begin(), tf.nodes.end());
                tf.tag = b0 ? 10 : 11;
                m.tagged_boundary_faces.push_back(tf);
            }
        }
    }
}

// The torus variant of the same box: tag 1 "torus" for tets whose centroid is
// within 0.04 of the circle of radius 0.25 about (0.5, 0.5, 0.5) in z = 0.5,
// tag 2 "air" elsewhere; tag 12 "cut" on the faces in the plane y = 0.5 with
// x > 0.5 that two torus tets share (n even).
inline void build_torus_mesh(Mesh& m, int n) {
    auto id = [&](int i, int j, int k) { return (k * (n + 1) + j) * (n + 1) + i; };
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i)
                m.nodes.push_back(Vec3(double(i) / n, double(j) / n, double(k) / n));
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int t = 0; t < 6; ++t) {
                    TetVerts v;
                    for (int q = 0; q < 4; ++q)
                        v[q] = id(i + kKuhn[t][q][0], j + kKuhn[t][q][1], k + kKuhn[t][q][2]);
                    m.tets.push_back(v);
                }
    m.build_topology();
    m.tet_tags.assign(m.tets.size(), 2);
    for (std::size_t t = 0; t < m.tets.size(); ++t) {
        Vec3 c(0, 0, 0);
        for (int q = 0; q < 4; ++q) c = c + m.nodes[m.tets[t][q]];
        c = c * 0.25;
        if (std::hypot(std::hypot(c.x - 0.5, c.y - 0.5) - 0.25, c.z - 0.5) < 0.04) m.tet_tags[t] = 1;
    }
    m.physical_names = {{3, 1, "torus"}, {3, 2, "air"}, {2, 12, "cut"}};
    for (int f = 0; f < m.num_faces(); ++f) {
        const FaceTets& ft = m.face_tets[static_cast<std::size_t>(f)];
        if (ft.count != 2 || m.tet_tags[ft.tets[0]] != 1 || m.tet_tags[ft.tets[1]] != 1) continue;
        const std::array<int, 3>& fv = m.faces[static_cast<std::size_t>(f)];
        bool on_cut = true;
        for (int q = 0; q < 3; ++q)
            if (m.nodes[fv[q]].y != 0.5 || !(m.nodes[fv[q]].x > 0.5)) on_cut = false;
        if (!on_cut) continue;
        TaggedFace tf;
        tf.nodes = fv;
        std::sort(tf.nodes.begin(), tf.nodes.end());
        tf.tag = 12;
        m.tagged_boundary_faces.push_back(tf);
    }
}

}  // namespace ref_meshes
