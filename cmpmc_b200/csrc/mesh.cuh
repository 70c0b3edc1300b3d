// mesh.cuh -- point location and field lookup in a tetrahedral finite-element mesh
// (TriLinearMesh3D, geometry/mesh_field.hpp:40-116), shared by the host helpers and the
// device transport.
//
// Each tetrahedron is one 144-byte record holding everything the facet walk touches:
// the inverse edge matrix T^-1, the coordinates of its fourth vertex, the constant field
// E = -grad V inside it and its four face neighbours. A walk step is then one record
// read (two 128-byte lines) instead of the reference's four separate arrays plus the
// vertex table, which is what matters on the device where every step of a carrier's
// walk is a dependent global load.
//
// The FP64 walk keeps the reference's arithmetic: bary[0..2] = T^-1 (p - x3) as row
// dot products summed left to right, bary[3] = 1 - b0 - b1 - b2, the first minimum
// wins ties, tolerance -1e-10, at most n_tets + 4 steps (mesh_field.hpp:66-100,
// 239-246). Translation units that need bit-identical results are compiled without FMA
// contraction.
#pragma once

#include <stdint.h>

#include "phys.cuh"

namespace cmpmc_gpu {

struct alignas(16) MeshTet {
    double tinv[9];  // row-major T^-1, T = [x0 - x3, x1 - x3, x2 - x3] (columns)
    double x3[3];    // fourth (largest-index) vertex
    double e[3];     // E = -grad V inside the tetrahedron (V/m)
    int32_t nb[4];   // neighbour across the facet opposite vertex i; -1 on the hull
};
static_assert(sizeof(MeshTet) == 144, "mesh record layout");

struct MeshView {
    const MeshTet* tet;  // nullptr: no mesh (uniform field)
    int32_t n_tets;
};

// FP32 copy of a record for the batched charge form (80 B): the same fields rounded to
// float, laid out so the walk reads them as four float4 loads.
struct alignas(16) MeshTet32 {
    float tinv[9];
    float x3[3];
    float e[3];
    int32_t nb[4];
    float pad;
};
static_assert(sizeof(MeshTet32) == 80, "FP32 mesh record layout");

struct MeshView32 {
    const MeshTet32* tet;
    int32_t n_tets;
};

// TriLinearMesh3D::bary_coord (mesh_field.hpp:239-246)
CMPMC_HD void mesh_bary(const MeshTet& t, V3 p, double b[4]) {
    const double dx = p.x - t.x3[0];
    const double dy = p.y - t.x3[1];
    const double dz = p.z - t.x3[2];
    b[0] = t.tinv[0] * dx + t.tinv[1] * dy + t.tinv[2] * dz;
    b[1] = t.tinv[3] * dx + t.tinv[4] * dy + t.tinv[5] * dz;
    b[2] = t.tinv[6] * dx + t.tinv[7] * dy + t.tinv[8] * dz;
    b[3] = 1.0 - b[0] - b[1] - b[2];
}

// TriLinearMesh3D::find_tetrahedron (mesh_field.hpp:66-100). `hint` is updated in place;
// returns false when the walk leaves the mesh through a hull facet (or runs out of steps).
CMPMC_HD bool mesh_find(const MeshView& m, V3 p, int32_t& hint, double b[4]) {
    if (m.n_tets <= 0) return false;
    if (hint < 0 || hint >= m.n_tets) hint = m.n_tets / 2;
    const int64_t max_steps = static_cast<int64_t>(m.n_tets) + 4;
    for (int64_t step = 0; step < max_steps; ++step) {
        const MeshTet& t = m.tet[hint];
        mesh_bary(t, p, b);
        double min_b = b[0];
        int min_i = 0;
        for (int i = 1; i < 4; ++i)
            if (b[i] < min_b) {
                min_b = b[i];
                min_i = i;
            }
        if (min_b >= -1e-10) return true;
        const int32_t next = t.nb[min_i];
        if (next < 0) return false;
        hint = next;
    }
    return false;
}

// TriLinearMesh3D::field_at (mesh_field.hpp:111-116): the field of the containing
// tetrahedron, zero outside the mesh.
CMPMC_HD V3 mesh_field(const MeshView& m, V3 p, int32_t& hint) {
    double b[4];
    if (!mesh_find(m, p, hint, b)) return v3(0.0, 0.0, 0.0);
    const MeshTet& t = m.tet[hint];
    return v3(t.e[0], t.e[1], t.e[2]);
}

// ---- BiLinearMesh2D (geometry/mesh_field.hpp:347-582) -----------------------------------
// A triangle mesh in (u, v) = (r, z) for an axisymmetric field, or (x, y) for a planar one.
// One 80-byte record per triangle: the inverse edge matrix, the third vertex, the constant
// field (E_u, E_v) inside it and the three edge neighbours.
struct alignas(16) MeshTri {
    double tinv[4];  // row-major 2x2 inverse of [x0 - x2, x1 - x2] (columns)
    double x2[2];
    double e[2];     // (E_u, E_v) = -grad V
    int32_t nb[3];   // neighbour across the edge opposite vertex i; -1 on the boundary
    int32_t pad;
};
static_assert(sizeof(MeshTri) == 80, "2D mesh record layout");

struct MeshView2 {
    const MeshTri* tri;  // nullptr: no 2D mesh
    int32_t n_tris;
    int32_t axisym;      // 1: (r, z) projection, field rotated back into (x, y, z)
};

// BiLinearMesh2D::project (mesh_field.hpp:488-493)
CMPMC_HD void mesh2_project(const MeshView2& m, V3 p, double& u, double& v) {
    if (m.axisym) {
        u = m_hypot(p.x, p.y);
        v = p.z;
    } else {
        u = p.x;
        v = p.y;
    }
}

// BiLinearMesh2D::find_triangle (mesh_field.hpp:376-405)
CMPMC_HD bool mesh2_find(const MeshView2& m, double u, double v, int32_t& hint, double b[3]) {
    if (m.n_tris <= 0) return false;
    if (hint < 0 || hint >= m.n_tris) hint = m.n_tris / 2;
    const int64_t max_steps = static_cast<int64_t>(m.n_tris) + 4;
    for (int64_t step = 0; step < max_steps; ++step) {
        const MeshTri& t = m.tri[hint];
        const double du = u - t.x2[0];
        const double dv = v - t.x2[1];
        b[0] = t.tinv[0] * du + t.tinv[1] * dv;
        b[1] = t.tinv[2] * du + t.tinv[3] * dv;
        b[2] = 1.0 - b[0] - b[1];
        double min_b = b[0];
        int min_i = 0;
        for (int i = 1; i < 3; ++i)
            if (b[i] < min_b) {
                min_b = b[i];
                min_i = i;
            }
        if (min_b >= -1e-10) return true;
        const int32_t next = t.nb[min_i];
        if (next < 0) return false;
        hint = next;
    }
    return false;
}

// BiLinearMesh2D::field_at (mesh_field.hpp:415-430)
CMPMC_HD V3 mesh2_field(const MeshView2& m, V3 p, int32_t& hint) {
    double u, v, b[3];
    mesh2_project(m, p, u, v);
    if (!mesh2_find(m, u, v, hint, b)) return v3(0.0, 0.0, 0.0);
    const MeshTri& t = m.tri[hint];
    if (!m.axisym) return v3(t.e[0], t.e[1], 0.0);
    if (u > 1e-15) return v3(t.e[0] * (p.x / u), t.e[0] * (p.y / u), t.e[1]);
    return v3(0.0, 0.0, t.e[1]);
}

// The 2D mesh in FP32 for the batched charge form: 48 bytes per triangle.
struct alignas(16) MeshTri32 {
    float tinv[4];
    float x2[2];
    float e[2];
    int32_t nb[3];
    int32_t pad;
};
static_assert(sizeof(MeshTri32) == 48, "FP32 2D mesh record layout");

struct MeshView2_32 {
    const MeshTri32* tri;  // nullptr: no 2D mesh
    int32_t n_tris;
    int32_t axisym;
};

}  // namespace cmpmc_gpu
