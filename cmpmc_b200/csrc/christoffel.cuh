// christoffel.cuh -- group velocities from the Christoffel equation, shared by the host
// table builds and the device's per-call kinematics modes.
//
// Restates phonon/phonon_kernels.hpp:134-298 with the reference's operation order:
//  * modes_from_eigen: L = the eigenvector most parallel to k, then FT / ST by eigenvalue;
//    v_g,i = C_ijlm e_j s_l e_m / rho with the slowness s = k / v_p (134-175);
//  * solve_christoffel (the "exact" solve): cyclic Jacobi on the 3x3 matrix (182-247);
//  * solve_christoffel_cardano: trigonometric Cardano eigenvalues (Smith, CACM 4, 168
//    (1961)) and cross-product eigenvectors, the Jacobi solve near degeneracies (255-298).
// The Cardano path uses acos and cos (correctly rounded on the device); translation units
// that need bit-identical results compile without FMA contraction.
#pragma once

// Included by phys.cuh (only) after its vector helpers (V3, dot, cross, unit, m_acos, m_cos).

namespace cmpmc_gpu {

struct Stiffness {
    double C[3][3][3][3];
};

CMPMC_HD double comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// physics::christoffel_modes_from_eigen (phonon/phonon_kernels.hpp:134-175)
CMPMC_HD void modes_from_eigen(const Stiffness& S, double density, V3 k, const double evals[3], const V3 evecs[3],
                               V3 vg_out[3]) {
    const double inv_rho = 1.0 / density;
    int long_idx = 0;
    double max_dot = -1.0;
    for (int i = 0; i < 3; ++i) {
        const double d = fabs(dot(evecs[i], k));
        if (d > max_dot) {
            max_dot = d;
            long_idx = i;
        }
    }
    const int rem1 = (long_idx + 1) % 3;
    const int rem2 = (long_idx + 2) % 3;
    const int ft_idx = (evals[rem1] >= evals[rem2]) ? rem1 : rem2;
    const int st_idx = (evals[rem1] >= evals[rem2]) ? rem2 : rem1;
    const int mode_indices[3] = {long_idx, ft_idx, st_idx};
    for (int m = 0; m < 3; ++m) {
        const int idx = mode_indices[m];
        const double vp = sqrt(dmax(evals[idx], 1.0));
        const V3 e = evecs[idx];
        const V3 slow = vdiv(k, vp);
        double out[3];
        for (int dim = 0; dim < 3; ++dim) {
            double sum = 0.0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int l = 0; l < 3; ++l) sum += comp(e, i) * S.C[i][j][l][dim] * comp(slow, j) * comp(e, l);
            out[dim] = sum * inv_rho;
        }
        vg_out[m] = v3(out[0], out[1], out[2]);
    }
}

// physics::solve_christoffel_exact: cyclic Jacobi on the 3x3 Christoffel matrix
// (phonon/phonon_kernels.hpp:182-247)
CMPMC_HD void solve_christoffel(const Stiffness& S, double density, V3 k, V3 vg_out[3]) {
    double D[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const double inv_rho = 1.0 / density;
    for (int i = 0; i < 3; ++i)
        for (int l = 0; l < 3; ++l) {
            double sum = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int m = 0; m < 3; ++m) sum += S.C[i][j][l][m] * comp(k, j) * comp(k, m);
            D[i][l] = sum * inv_rho;
        }
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 12; ++sweep) {
        const double off = fabs(D[0][1]) + fabs(D[0][2]) + fabs(D[1][2]);
        if (off < 1e-15 * (fabs(D[0][0]) + fabs(D[1][1]) + fabs(D[2][2]))) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (fabs(D[p][q]) < 1e-18) continue;
                const double tau = (D[q][q] - D[p][p]) / (2.0 * D[p][q]);
                const double t = (tau >= 0.0) ? (1.0 / (tau + sqrt(1.0 + tau * tau)))
                                              : (-1.0 / (-tau + sqrt(1.0 + tau * tau)));
                const double c = 1.0 / sqrt(1.0 + t * t);
                const double s = t * c;
                const double d_pp = D[p][p];
                const double d_qq = D[q][q];
                const double d_pq = D[p][q];
                D[p][p] = c * c * d_pp - 2.0 * s * c * d_pq + s * s * d_qq;
                D[q][q] = s * s * d_pp + 2.0 * s * c * d_pq + c * c * d_qq;
                D[p][q] = D[q][p] = 0.0;
                for (int r = 0; r < 3; ++r) {
                    if (r != p && r != q) {
                        const double d_rp = D[r][p];
                        const double d_rq = D[r][q];
                        D[r][p] = D[p][r] = c * d_rp - s * d_rq;
                        D[r][q] = D[q][r] = s * d_rp + c * d_rq;
                    }
                    const double v_rp = V[r][p];
                    const double v_rq = V[r][q];
                    V[r][p] = c * v_rp - s * v_rq;
                    V[r][q] = s * v_rp + c * v_rq;
                }
            }
    }
    const double evals[3] = {D[0][0], D[1][1], D[2][2]};
    const V3 evecs[3] = {v3(V[0][0], V[1][0], V[2][0]), v3(V[0][1], V[1][1], V[2][1]),
                         v3(V[0][2], V[1][2], V[2][2])};
    modes_from_eigen(S, density, k, evals, evecs, vg_out);
}

// physics::solve_christoffel_cardano (phonon/phonon_kernels.hpp:255-298)
CMPMC_HD void solve_christoffel_cardano(const Stiffness& S, double density, V3 k, V3 vg_out[3]) {
    double D[3][3];
    const double inv_rho = 1.0 / density;
    for (int i = 0; i < 3; ++i)
        for (int l = i; l < 3; ++l) {
            double sum = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int m = 0; m < 3; ++m) sum += S.C[i][j][l][m] * comp(k, j) * comp(k, m);
            D[i][l] = D[l][i] = sum * inv_rho;
        }
    const double q = (D[0][0] + D[1][1] + D[2][2]) / 3.0;
    const double p1 = D[0][1] * D[0][1] + D[0][2] * D[0][2] + D[1][2] * D[1][2];
    const double p2 = (D[0][0] - q) * (D[0][0] - q) + (D[1][1] - q) * (D[1][1] - q) +
                      (D[2][2] - q) * (D[2][2] - q) + 2.0 * p1;
    const double p = sqrt(p2 / 6.0);
    if (!(p > 1e-12 * fabs(q))) {
        solve_christoffel(S, density, k, vg_out);
        return;
    }
    double B[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] = (D[i][j] - (i == j ? q : 0.0)) / p;
    const double detB = B[0][0] * (B[1][1] * B[2][2] - B[1][2] * B[2][1]) -
                        B[0][1] * (B[1][0] * B[2][2] - B[1][2] * B[2][0]) +
                        B[0][2] * (B[1][0] * B[2][1] - B[1][1] * B[2][0]);
    const double r = dclamp(0.5 * detB, -1.0, 1.0);
    const double phi = m_acos(r) / 3.0;
    double ev[3];
    ev[0] = q + 2.0 * p * m_cos(phi);
    ev[2] = q + 2.0 * p * m_cos(phi + 2.0943951023931957);
    ev[1] = 3.0 * q - ev[0] - ev[2];
    const double scale = fabs(ev[0]);
    const double gap_tol = 1e-4;
    if (fabs(ev[0] - ev[1]) < gap_tol * scale || fabs(ev[1] - ev[2]) < gap_tol * scale) {
        solve_christoffel(S, density, k, vg_out);
        return;
    }
    V3 evecs[3];
    for (int e = 0; e < 3; ++e) {
        const V3 r0 = v3(D[0][0] - ev[e], D[0][1], D[0][2]);
        const V3 r1 = v3(D[1][0], D[1][1] - ev[e], D[1][2]);
        const V3 r2 = v3(D[2][0], D[2][1], D[2][2] - ev[e]);
        const V3 c01 = cross(r0, r1), c02 = cross(r0, r2), c12 = cross(r1, r2);
        const double n01 = norm2(c01), n02 = norm2(c02), n12 = norm2(c12);
        const V3 best = (n01 >= n02 && n01 >= n12) ? c01 : ((n02 >= n12) ? c02 : c12);
        evecs[e] = unit(best);
    }
    modes_from_eigen(S, density, k, ev, evecs, vg_out);
}

}  // namespace cmpmc_gpu
