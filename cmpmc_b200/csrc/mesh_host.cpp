// mesh_host.cpp -- host construction of tetrahedral field meshes (TriLinearMesh3D,
// geometry/mesh_field.hpp:40-345) into the per-tetrahedron records of mesh.cuh.
//
// The construction keeps the reference's arithmetic, so a field looked up here or on the
// device is bit-identical to TriLinearMesh3D::field_at for the same tetrahedron:
//   * node indices of every tetrahedron sorted ascending before anything else
//     (fill_neighbors sorts them in place, mesh_field.hpp:264-266);
//   * T^-1 by cofactors times 1/det, det by the first-row expansion, |det| <= 1e-30
//     giving a zero inverse and zero field (mesh_field.hpp:288-334);
//   * E = -(T^-1)^T dV (mesh_field.hpp:337-343).
// Face neighbours are matched through a sorted list of facet keys, as the reference does.
// This file is compiled without FMA contraction (-ffp-contract=off).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "internal.hpp"
#include "mesh.cuh"

using namespace cmpmc_gpu;

namespace {

struct Facet {
    std::array<int32_t, 3> nodes;
    int32_t tet;
    int32_t slot;
    bool operator<(const Facet& o) const {
        if (nodes != o.nodes) return nodes < o.nodes;
        return tet < o.tet;
    }
};

int finish_mesh(cmpmc_mesh* m) {
    const size_t nt = m->tets.size();
    const size_t nv = m->V.size();
    for (auto& t : m->tets) {
        std::sort(t.begin(), t.end());
        for (int i = 0; i < 4; ++i)
            if (t[i] < 0 || static_cast<size_t>(t[i]) >= nv) return CMPMC_ERR_INVALID;
    }
    m->rec.assign(nt, MeshTet{});
    // face neighbours (fill_neighbors, mesh_field.hpp:260-285)
    std::vector<Facet> f;
    f.reserve(nt * 4);
    for (size_t it = 0; it < nt; ++it) {
        const auto& t = m->tets[it];
        const int32_t id = static_cast<int32_t>(it);
        f.push_back({{t[1], t[2], t[3]}, id, 0});
        f.push_back({{t[0], t[2], t[3]}, id, 1});
        f.push_back({{t[0], t[1], t[3]}, id, 2});
        f.push_back({{t[0], t[1], t[2]}, id, 3});
    }
    std::sort(f.begin(), f.end());
    for (size_t it = 0; it < nt; ++it)
        for (int i = 0; i < 4; ++i) m->rec[it].nb[i] = -1;
    for (size_t i = 0; i + 1 < f.size(); ++i) {
        if (f[i].nodes == f[i + 1].nodes) {
            m->rec[f[i].tet].nb[f[i].slot] = f[i + 1].tet;
            m->rec[f[i + 1].tet].nb[f[i + 1].slot] = f[i].tet;
            ++i;
        }
    }
    // inverse edge matrices and fields (fill_tinv_and_grad, mesh_field.hpp:288-344)
    for (size_t it = 0; it < nt; ++it) {
        const auto& t = m->tets[it];
        MeshTet& r = m->rec[it];
        const double* x3 = &m->X[3 * static_cast<size_t>(t[3])];
        r.x3[0] = x3[0];
        r.x3[1] = x3[1];
        r.x3[2] = x3[2];
        double col[3][3];
        for (int c = 0; c < 3; ++c) {
            const double* xc = &m->X[3 * static_cast<size_t>(t[c])];
            col[c][0] = xc[0] - x3[0];
            col[c][1] = xc[1] - x3[1];
            col[c][2] = xc[2] - x3[2];
        }
        const double a = col[0][0], b = col[1][0], c = col[2][0];
        const double d = col[0][1], e = col[1][1], ff = col[2][1];
        const double g = col[0][2], h = col[1][2], k = col[2][2];
        const double det = a * (e * k - ff * h) - b * (d * k - ff * g) + c * (d * h - e * g);
        if (std::fabs(det) <= 1e-30) {
            std::memset(r.tinv, 0, sizeof(r.tinv));
            std::memset(r.e, 0, sizeof(r.e));
            continue;
        }
        const double inv_det = 1.0 / det;
        double* M = r.tinv;
        M[0] = (e * k - ff * h) * inv_det;
        M[1] = -(b * k - c * h) * inv_det;
        M[2] = (b * ff - c * e) * inv_det;
        M[3] = -(d * k - ff * g) * inv_det;
        M[4] = (a * k - c * g) * inv_det;
        M[5] = -(a * ff - c * d) * inv_det;
        M[6] = (d * h - e * g) * inv_det;
        M[7] = -(a * h - b * g) * inv_det;
        M[8] = (a * e - b * d) * inv_det;
        const double v3n = m->V[t[3]];
        const double dv0 = m->V[t[0]] - v3n, dv1 = m->V[t[1]] - v3n, dv2 = m->V[t[2]] - v3n;
        // (T^-1)^T dV, then times -1
        const double gx = M[0] * dv0 + M[3] * dv1 + M[6] * dv2;
        const double gy = M[1] * dv0 + M[4] * dv1 + M[7] * dv2;
        const double gz = M[2] * dv0 + M[5] * dv1 + M[8] * dv2;
        r.e[0] = gx * -1.0;
        r.e[1] = gy * -1.0;
        r.e[2] = gz * -1.0;
    }
    return CMPMC_OK;
}

MeshView host_view(const cmpmc_mesh* m) {
    MeshView v;
    v.tet = m->rec.data();
    v.n_tets = static_cast<int32_t>(m->rec.size());
    return v;
}

struct Edge {
    std::array<int32_t, 2> nodes;
    int32_t tri;
    int32_t slot;
    bool operator<(const Edge& o) const {
        if (nodes != o.nodes) return nodes < o.nodes;
        return tri < o.tri;
    }
};

// BiLinearMesh2D::fill_neighbors / fill_tinv_and_grad (mesh_field.hpp:515-580)
int finish_mesh2d(cmpmc_mesh2d* m) {
    const size_t nt = m->tris.size(), nv = m->V.size();
    for (auto& t : m->tris) {
        std::sort(t.begin(), t.end());
        for (int i = 0; i < 3; ++i)
            if (t[i] < 0 || static_cast<size_t>(t[i]) >= nv) return CMPMC_ERR_INVALID;
    }
    m->rec.assign(nt, MeshTri{});
    std::vector<Edge> e;
    e.reserve(nt * 3);
    for (size_t it = 0; it < nt; ++it) {
        const auto& t = m->tris[it];
        const int32_t id = static_cast<int32_t>(it);
        e.push_back({{t[1], t[2]}, id, 0});
        e.push_back({{t[0], t[2]}, id, 1});
        e.push_back({{t[0], t[1]}, id, 2});
    }
    std::sort(e.begin(), e.end());
    for (size_t it = 0; it < nt; ++it)
        for (int i = 0; i < 3; ++i) m->rec[it].nb[i] = -1;
    for (size_t i = 0; i + 1 < e.size(); ++i)
        if (e[i].nodes == e[i + 1].nodes) {
            m->rec[e[i].tri].nb[e[i].slot] = e[i + 1].tri;
            m->rec[e[i + 1].tri].nb[e[i + 1].slot] = e[i].tri;
            ++i;
        }
    for (size_t it = 0; it < nt; ++it) {
        const auto& t = m->tris[it];
        MeshTri& r = m->rec[it];
        const double* x2 = &m->X[2 * static_cast<size_t>(t[2])];
        r.x2[0] = x2[0];
        r.x2[1] = x2[1];
        const double a = m->X[2 * static_cast<size_t>(t[0])] - x2[0];
        const double b = m->X[2 * static_cast<size_t>(t[1])] - x2[0];
        const double c = m->X[2 * static_cast<size_t>(t[0]) + 1] - x2[1];
        const double d = m->X[2 * static_cast<size_t>(t[1]) + 1] - x2[1];
        const double det = a * d - b * c;
        if (std::fabs(det) <= 1e-30) {
            std::memset(r.tinv, 0, sizeof(r.tinv));
            r.e[0] = r.e[1] = 0.0;
            continue;
        }
        const double inv_det = 1.0 / det;
        r.tinv[0] = d * inv_det;
        r.tinv[1] = -b * inv_det;
        r.tinv[2] = -c * inv_det;
        r.tinv[3] = a * inv_det;
        const double dv0 = m->V[t[0]] - m->V[t[2]];
        const double dv1 = m->V[t[1]] - m->V[t[2]];
        r.e[0] = -(r.tinv[0] * dv0 + r.tinv[2] * dv1);
        r.e[1] = -(r.tinv[1] * dv0 + r.tinv[3] * dv1);
    }
    return CMPMC_OK;
}

MeshView2 host_view2(const cmpmc_mesh2d* m) {
    MeshView2 v;
    v.tri = m->rec.data();
    v.n_tris = static_cast<int32_t>(m->rec.size());
    v.axisym = m->axisym;
    return v;
}

}  // namespace

extern "C" {

int cmpmc_mesh2d_create(const double* uv, const double* potentials, uint64_t n_vertices, const int32_t* tris,
                        uint64_t n_tris, int axisymmetric, cmpmc_mesh2d** out) {
    if (!out) return CMPMC_ERR_INVALID;
    *out = nullptr;
    if ((n_vertices && (!uv || !potentials)) || (n_tris && !tris) || n_tris > 0x7ffffffbull ||
        n_vertices > 0x7fffffffull)
        return CMPMC_ERR_INVALID;
    cmpmc_mesh2d* m = new (std::nothrow) cmpmc_mesh2d();
    if (!m) return CMPMC_ERR_INVALID;
    m->X.assign(uv, uv + 2 * n_vertices);
    m->V.assign(potentials, potentials + n_vertices);
    m->tris.resize(n_tris);
    for (uint64_t i = 0; i < n_tris; ++i)
        for (int j = 0; j < 3; ++j) m->tris[i][j] = tris[3 * i + j];
    m->axisym = axisymmetric ? 1 : 0;
    const int st = finish_mesh2d(m);
    if (st != CMPMC_OK) {
        delete m;
        return st;
    }
    *out = m;
    return CMPMC_OK;
}

int cmpmc_mesh2d_build_grid(double u_min, double u_max, double v_min, double v_max, int nu, int nv,
                            cmpmc_potential2d_fn potential, void* user, int axisymmetric, cmpmc_mesh2d** out) {
    if (!out || !potential) return CMPMC_ERR_INVALID;
    *out = nullptr;
    nu = std::max(1, nu);
    nv = std::max(1, nv);
    const int64_t vu = nu + 1, vv = nv + 1;
    if (vu * vv > 0x7fffffffll || 2ll * nu * nv > 0x7ffffffbll) return CMPMC_ERR_INVALID;
    cmpmc_mesh2d* m = new (std::nothrow) cmpmc_mesh2d();
    if (!m) return CMPMC_ERR_INVALID;
    m->X.resize(2 * static_cast<size_t>(vu * vv));
    m->V.resize(static_cast<size_t>(vu * vv));
    for (int i = 0; i <= nu; ++i) {
        const double u = u_min + (u_max - u_min) * (static_cast<double>(i) / nu);
        for (int j = 0; j <= nv; ++j) {
            const double v = v_min + (v_max - v_min) * (static_cast<double>(j) / nv);
            const size_t id = static_cast<size_t>(i * vv + j);
            m->X[2 * id] = u;
            m->X[2 * id + 1] = v;
            m->V[id] = potential(u, v, user);
        }
    }
    m->tris.reserve(2 * static_cast<size_t>(nu) * nv);
    for (int i = 0; i < nu; ++i)
        for (int j = 0; j < nv; ++j) {
            const int32_t v00 = static_cast<int32_t>(i * vv + j), v10 = static_cast<int32_t>((i + 1) * vv + j),
                          v01 = static_cast<int32_t>(i * vv + j + 1), v11 = static_cast<int32_t>((i + 1) * vv + j + 1);
            m->tris.push_back({v00, v10, v11});
            m->tris.push_back({v00, v01, v11});
        }
    m->axisym = axisymmetric ? 1 : 0;
    const int st = finish_mesh2d(m);
    if (st != CMPMC_OK) {
        delete m;
        return st;
    }
    *out = m;
    return CMPMC_OK;
}

void cmpmc_mesh2d_destroy(cmpmc_mesh2d* m) { delete m; }

int cmpmc_mesh2d_info(const cmpmc_mesh2d* m, uint64_t* n_vertices, uint64_t* n_tris) {
    if (!m) return CMPMC_ERR_INVALID;
    if (n_vertices) *n_vertices = m->V.size();
    if (n_tris) *n_tris = m->rec.size();
    return CMPMC_OK;
}

int cmpmc_mesh2d_field_at(const cmpmc_mesh2d* m, const double p[3], int32_t* hint, double E[3]) {
    if (!m || !p || !hint || !E) return CMPMC_ERR_INVALID;
    const V3 e = mesh2_field(host_view2(m), v3(p[0], p[1], p[2]), *hint);
    E[0] = e.x;
    E[1] = e.y;
    E[2] = e.z;
    return CMPMC_OK;
}

int cmpmc_mesh2d_potential_at(const cmpmc_mesh2d* m, const double p[3], int32_t* hint, double* V) {
    if (!m || !p || !hint || !V) return CMPMC_ERR_INVALID;
    const MeshView2 v = host_view2(m);
    double u, w, b[3];
    mesh2_project(v, v3(p[0], p[1], p[2]), u, w);
    if (!mesh2_find(v, u, w, *hint, b)) {
        *V = 0.0;
        return CMPMC_OK;
    }
    const auto& t = m->tris[*hint];
    *V = b[0] * m->V[t[0]] + b[1] * m->V[t[1]] + b[2] * m->V[t[2]];
    return CMPMC_OK;
}

int cmpmc_mesh_create(const double* vertices, const double* potentials, uint64_t n_vertices, const int32_t* tets,
                      uint64_t n_tets, double v_min_clamp, double v_max_clamp, cmpmc_mesh** out) {
    if (!out) return CMPMC_ERR_INVALID;
    *out = nullptr;
    if ((n_vertices && (!vertices || !potentials)) || (n_tets && !tets) || n_tets > 0x7ffffffbull ||
        n_vertices > 0x7fffffffull)
        return CMPMC_ERR_INVALID;
    cmpmc_mesh* m = new (std::nothrow) cmpmc_mesh();
    if (!m) return CMPMC_ERR_INVALID;
    m->X.assign(vertices, vertices + 3 * n_vertices);
    m->V.resize(n_vertices);
    for (uint64_t i = 0; i < n_vertices; ++i) m->V[i] = std::clamp(potentials[i], v_min_clamp, v_max_clamp);
    m->tets.resize(n_tets);
    for (uint64_t i = 0; i < n_tets; ++i)
        for (int j = 0; j < 4; ++j) m->tets[i][j] = tets[4 * i + j];
    const int st = finish_mesh(m);
    if (st != CMPMC_OK) {
        delete m;
        return st;
    }
    *out = m;
    return CMPMC_OK;
}

// TriLinearMesh3D::load_from_files (mesh_field.hpp:190-231): "x y z V" node lines and
// "i0 i1 i2 i3" tetrahedron lines, '#' / '%' comment lines and lines that do not parse
// skipped, coordinates and potentials scaled by the units. A file that does not open
// contributes no lines (an empty mesh, as in the reference).
int cmpmc_mesh_load_files(const char* coords_file, const char* tets_file, double coord_unit_m,
                          double potential_unit_V, cmpmc_mesh** out) {
    if (!out || !coords_file || !tets_file) return CMPMC_ERR_INVALID;
    *out = nullptr;
    std::vector<double> X, V;
    std::vector<int32_t> T;
    std::string line;
    {
        std::ifstream in(coords_file);
        while (std::getline(in, line)) {
            if (line.empty() || line[0] == '#' || line[0] == '%') continue;
            std::istringstream ls(line);
            double x, y, z, v;
            if (ls >> x >> y >> z >> v) {
                X.push_back(x * coord_unit_m);
                X.push_back(y * coord_unit_m);
                X.push_back(z * coord_unit_m);
                V.push_back(v * potential_unit_V);
            }
        }
    }
    {
        std::ifstream in(tets_file);
        while (std::getline(in, line)) {
            if (line.empty() || line[0] == '#' || line[0] == '%') continue;
            std::istringstream ls(line);
            int a, b, c, d;
            if (ls >> a >> b >> c >> d) {
                T.push_back(a);
                T.push_back(b);
                T.push_back(c);
                T.push_back(d);
            }
        }
    }
    return cmpmc_mesh_create(X.data(), V.data(), V.size(), T.data(), T.size() / 4, -1e30, 1e30, out);
}

int cmpmc_mesh_build_cartesian(double half_x, double half_y, double half_z, int nx, int ny, int nz,
                               cmpmc_potential_fn potential, void* user, cmpmc_mesh** out) {
    if (!out || !potential) return CMPMC_ERR_INVALID;
    *out = nullptr;
    nx = std::max(1, nx);
    ny = std::max(1, ny);
    nz = std::max(1, nz);
    const int64_t vx = nx + 1, vy = ny + 1, vz = nz + 1;
    if (vx * vy * vz > 0x7fffffffll || 6ll * nx * ny * nz > 0x7ffffffbll) return CMPMC_ERR_INVALID;
    auto vid = [vy, vz](int64_t i, int64_t j, int64_t k) { return static_cast<int32_t>((i * vy + j) * vz + k); };
    cmpmc_mesh* m = new (std::nothrow) cmpmc_mesh();
    if (!m) return CMPMC_ERR_INVALID;
    const size_t nv = static_cast<size_t>(vx * vy * vz);
    m->X.resize(3 * nv);
    m->V.resize(nv);
    // node coordinates and potentials (mesh_field.hpp:144-155)
    for (int i = 0; i <= nx; ++i) {
        const double x = -half_x + 2.0 * half_x * (static_cast<double>(i) / nx);
        for (int j = 0; j <= ny; ++j) {
            const double y = -half_y + 2.0 * half_y * (static_cast<double>(j) / ny);
            for (int k = 0; k <= nz; ++k) {
                const double z = -half_z + 2.0 * half_z * (static_cast<double>(k) / nz);
                const size_t id = static_cast<size_t>(vid(i, j, k));
                const double p[3] = {x, y, z};
                m->X[3 * id + 0] = x;
                m->X[3 * id + 1] = y;
                m->X[3 * id + 2] = z;
                m->V[id] = potential(p, user);
            }
        }
    }
    // six Kuhn tetrahedra per cell around the v000 -> v111 diagonal (mesh_field.hpp:157-184)
    m->tets.reserve(static_cast<size_t>(6) * nx * ny * nz);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const int32_t v000 = vid(i, j, k), v100 = vid(i + 1, j, k), v010 = vid(i, j + 1, k),
                              v110 = vid(i + 1, j + 1, k), v001 = vid(i, j, k + 1), v101 = vid(i + 1, j, k + 1),
                              v011 = vid(i, j + 1, k + 1), v111 = vid(i + 1, j + 1, k + 1);
                m->tets.push_back({v000, v100, v110, v111});
                m->tets.push_back({v000, v100, v101, v111});
                m->tets.push_back({v000, v010, v110, v111});
                m->tets.push_back({v000, v010, v011, v111});
                m->tets.push_back({v000, v001, v101, v111});
                m->tets.push_back({v000, v001, v011, v111});
            }
    const int st = finish_mesh(m);
    if (st != CMPMC_OK) {
        delete m;
        return st;
    }
    *out = m;
    return CMPMC_OK;
}

double cmpmc_recoil_potential(const double p[3], void* detector) {
    const cmpmc_detector* d = static_cast<const cmpmc_detector*>(detector);
    const double R = d->radius, h = d->half_z;
    const double rr = (p[0] * p[0] + p[1] * p[1]) / (R * R);
    return 4.0 * (p[2] + h) / (2.0 * h) + 0.2 * rr * std::sin(kPi * p[2] / (2.0 * h));
}

void cmpmc_mesh_destroy(cmpmc_mesh* m) { delete m; }

int cmpmc_mesh_info(const cmpmc_mesh* m, uint64_t* n_vertices, uint64_t* n_tets) {
    if (!m) return CMPMC_ERR_INVALID;
    if (n_vertices) *n_vertices = m->V.size();
    if (n_tets) *n_tets = m->rec.size();
    return CMPMC_OK;
}

int cmpmc_mesh_field_at(const cmpmc_mesh* m, const double p[3], int32_t* hint, double E[3]) {
    if (!m || !p || !hint || !E) return CMPMC_ERR_INVALID;
    const V3 e = mesh_field(host_view(m), v3(p[0], p[1], p[2]), *hint);
    E[0] = e.x;
    E[1] = e.y;
    E[2] = e.z;
    return CMPMC_OK;
}

int cmpmc_mesh_potential_at(const cmpmc_mesh* m, const double p[3], int32_t* hint, double* V) {
    if (!m || !p || !hint || !V) return CMPMC_ERR_INVALID;
    double b[4];
    if (!mesh_find(host_view(m), v3(p[0], p[1], p[2]), *hint, b)) {
        *V = 0.0;
        return CMPMC_OK;
    }
    const auto& t = m->tets[*hint];
    *V = b[0] * m->V[t[0]] + b[1] * m->V[t[1]] + b[2] * m->V[t[2]] + b[3] * m->V[t[3]];
    return CMPMC_OK;
}

}  // extern "C"
