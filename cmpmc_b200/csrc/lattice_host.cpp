// lattice_host.cpp -- host construction of the crystal tables the device reads.
//
// Restates the table build of CrystalLattice (lattice/crystal_lattice.hpp:340-477) and
// the Voigt stiffness construction of CrystalConfig (materials/crystal_config.hpp:164-225)
// with the reference's arithmetic, so that the FP32 octahedral group-velocity table and
// the FP64 inverse-CDF tables are bit-identical to the CPU library's (checked against the
// reference's own tables by the test suite). Compiled by the host compiler without FMA
// contraction.
#include <atomic>
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>

#include "internal.hpp"

using namespace cmpmc_gpu;

namespace {

constexpr double kGPa = 1e9;
constexpr double kMeV = 1e-3;
constexpr double kElemCharge = 1.602176634e-19;
constexpr double kMeEV = 510998.950;
constexpr double kMeKg = 9.1093837015e-31;

using Voigt = std::array<std::array<double, 6>, 6>;

// CrystalConfig::build_voigt_matrix (crystal_config.hpp:164-225)
Voigt build_voigt(const cmpmc_crystal_config& c) {
    Voigt V{};
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) V[i][j] = c.C_custom[i][j];
    if (!c.has_custom_C) {
        V[0][0] = c.C11;
        V[0][1] = c.C12;
        V[0][2] = c.C13;
        V[0][3] = c.C14;
        V[0][5] = c.C16;
        V[2][2] = c.C33;
        V[3][3] = c.C44;
        V[5][5] = c.C66;
    }
    switch (c.group) {
        case 0:  // Amorphous
            V[3][3] = 0.5 * (V[0][0] - V[0][1]);
            [[fallthrough]];
        case 1: {  // Cubic
            const double c11 = V[0][0], c12 = V[0][1], c44 = V[3][3];
            for (int i = 0; i < 6; ++i)
                for (int j = i; j < 6; ++j) {
                    if (i < 3 && j < 3) V[i][j] = (i == j) ? c11 : c12;
                    else if (i == j && i >= 3) V[i][i] = c44;
                    else V[i][j] = 0.0;
                }
            break;
        }
        case 4:  // Hexagonal
            V[0][5] = 0.0;
            V[5][5] = 0.5 * (V[0][0] - V[0][1]);
            [[fallthrough]];
        case 2:  // Tetragonal
            V[1][1] = V[0][0];
            V[1][2] = V[0][2];
            V[1][5] = -V[0][5];
            V[4][4] = V[3][3];
            break;
        case 5: {  // Rhombohedral
            const double c11 = V[0][0], c12 = V[0][1], c13 = V[0][2], c14 = V[0][3];
            const double c44 = V[3][3], c66 = 0.5 * (c11 - c12);
            V[0][4] = 0.0; V[0][5] = 0.0;
            V[1][1] = c11; V[1][2] = c13; V[1][3] = -c14; V[1][4] = 0.0; V[1][5] = 0.0;
            V[2][3] = 0.0; V[2][4] = 0.0; V[2][5] = 0.0;
            V[3][4] = 0.0; V[3][5] = 0.0;
            V[4][4] = c44; V[4][5] = c14;
            V[5][5] = c66;
            break;
        }
        default:  // Orthorhombic, Monoclinic, Triclinic: as given
            break;
    }
    for (int i = 0; i < 6; ++i)
        for (int j = i + 1; j < 6; ++j) V[j][i] = V[i][j];
    return V;
}

int voigt_index(int i, int j) {
    if (i == j) return i;
    if ((i == 1 && j == 2) || (i == 2 && j == 1)) return 3;
    if ((i == 0 && j == 2) || (i == 2 && j == 0)) return 4;
    return 5;
}

// CrystalLattice::oct_decode (crystal_lattice.hpp:132-141)
V3 oct_decode(double u, double v) {
    const double kz = 1.0 - std::abs(u) - std::abs(v);
    double kx = u;
    double ky = v;
    if (kz < 0.0) {
        kx = (1.0 - std::abs(v)) * (u >= 0.0 ? 1.0 : -1.0);
        ky = (1.0 - std::abs(u)) * (v >= 0.0 ? 1.0 : -1.0);
    }
    return unit(v3(kx, ky, kz));
}

// CrystalLattice::build_single_cdf (crystal_lattice.hpp:448-477)
template <class F>
void build_single_cdf(std::vector<double>& inv_cdf, double xmin, double xmax, F&& pdf) {
    constexpr int N_INT = 4096;
    inv_cdf.assign(kNCdf, 0.0);
    std::vector<double> cdf(N_INT + 1, 0.0);
    const double dx = (xmax - xmin) / N_INT;
    double sum = 0.0;
    for (int i = 0; i < N_INT; ++i) {
        const double x_mid = xmin + (i + 0.5) * dx;
        sum += std::max(0.0, pdf(x_mid)) * dx;
        cdf[i + 1] = sum;
    }
    if (sum <= 0.0) {
        for (int k = 0; k < kNCdf; ++k) inv_cdf[k] = 0.5 * (xmin + xmax);
        return;
    }
    for (double& v : cdf) v /= sum;
    inv_cdf[0] = xmin;
    inv_cdf[kNCdf - 1] = xmax;
    int j = 0;
    for (int k = 1; k < kNCdf - 1; ++k) {
        const double target = static_cast<double>(k) / (kNCdf - 1);
        while (j < N_INT && cdf[j + 1] < target) ++j;
        const double denom = cdf[j + 1] - cdf[j];
        const double t = (denom > 1e-16) ? ((target - cdf[j]) / denom) : 0.0;
        inv_cdf[k] = xmin + (j + t) * dx;
    }
}

// physics::tamura_lt_pdf / tamura_tt_pdf (phonon/phonon_kernels.hpp:98-129)
double tamura_lt_pdf(double x, const cmpmc_crystal_config& c) {
    const double m = c.v_sound / c.v_trans;
    const double xmin = (m - 1.0) / (m + 1.0);
    if (x <= xmin || x >= 1.0) return 0.0;
    const double a = 1.0 - x * x;
    const double b = (1.0 + x) * (1.0 + x) - m * m * (1.0 - x) * (1.0 - x);
    const double cc = 1.0 + x * x - m * m * (1.0 - x) * (1.0 - x);
    return (a * a / (x * x)) * b * cc * cc;
}
double tamura_tt_pdf(double x, const cmpmc_crystal_config& c) {
    const double m = c.v_sound / c.v_trans;
    const double xmin = 0.5 * (1.0 - 1.0 / m);
    const double xmax = 0.5 * (1.0 + 1.0 / m);
    if (x <= xmin || x >= xmax) return 0.0;
    const double be = c.beta / 1e11, ga = c.gamma / 1e11, la = c.lambda / 1e11, mu = c.mu / 1e11;
    const double A = 0.5 * (1.0 - m * m) * (be + la + (1.0 + m * m) * (ga + mu));
    const double B = be + la + 2.0 * m * m * (ga + mu);
    const double C = be + la + 2.0 * (ga + mu);
    const double D = (1.0 - m * m) * (2.0 * be + 4.0 * ga + la + 3.0 * mu);
    const double X = m * x;
    const double t1 = A + B * m * X - B * X * X;
    const double t2 = C * X * (m - X) - D / (m - X) * (X - m - (1.0 - m * m) / (4.0 * X));
    return t1 * t1 + t2 * t2;
}

// the 181 x 361 bilinear (cos theta, phi) table (crystal_lattice.hpp:350-368)
void build_bilinear(cmpmc_lattice& lat) {
    const cmpmc_crystal_config& c = lat.cfg;
    lat.bil.assign(static_cast<size_t>(3) * kNCTheta * kNPhi * 3, 0.0);
    for (int i = 0; i < kNCTheta; ++i) {
        const double ctheta = -1.0 + 2.0 * (static_cast<double>(i) / (kNCTheta - 1));
        const double stheta = std::sqrt(std::max(0.0, 1.0 - ctheta * ctheta));
        for (int j = 0; j < kNPhi; ++j) {
            const double phi = kTwoPi * (static_cast<double>(j) / (kNPhi - 1));
            V3 k = v3(stheta * std::cos(phi), stheta * std::sin(phi), ctheta);
            if (stheta < 1e-7) k = unit(v3(1e-6, 0.0, ctheta));
            V3 vg[3];
            solve_christoffel(lat.stiff, c.density, k, vg);
            for (int m = 0; m < 3; ++m) {
                double* e = &lat.bil[3 * ((static_cast<size_t>(m) * kNCTheta + i) * kNPhi + j)];
                e[0] = vg[m].x;
                e[1] = vg[m].y;
                e[2] = vg[m].z;
            }
        }
    }
}

void build_tables(cmpmc_lattice& lat) {
    const cmpmc_crystal_config& c = lat.cfg;
    // stiffness tensor (crystal_lattice.hpp:340-348)
    const Voigt Vt = build_voigt(c);
    Stiffness& S = lat.stiff;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) S.C[i][j][l][m] = Vt[voigt_index(i, j)][voigt_index(l, m)];

    // octahedral table (crystal_lattice.hpp:370-392)
    lat.oct.resize(3 * kNOct * kNOct);
    for (int i = 0; i < kNOct; ++i) {
        const double u = -1.0 + 2.0 * (static_cast<double>(i) / (kNOct - 1));
        for (int j = 0; j < kNOct; ++j) {
            const double v = -1.0 + 2.0 * (static_cast<double>(j) / (kNOct - 1));
            V3 k = oct_decode(u, v);
            if (std::abs(k.x) < 1e-6 && std::abs(k.y) < 1e-6) k = unit(v3(1e-6, 0.0, k.z));
            V3 vg[3];
            solve_christoffel(S, c.density, k, vg);
            for (int m = 0; m < 3; ++m) {
                OctEntry& e = lat.oct[(m * kNOct + i) * kNOct + j];
                e.vx = static_cast<float>(vg[m].x);
                e.vy = static_cast<float>(vg[m].y);
                e.vz = static_cast<float>(vg[m].z);
                e.vmag = static_cast<float>(norm(vg[m]));
            }
        }
    }

    // decay inverse-CDF tables (crystal_lattice.hpp:440-446)
    const double m = c.v_sound / c.v_trans;
    build_single_cdf(lat.cdf_lt, (m - 1.0) / (m + 1.0), 1.0, [&](double x) { return tamura_lt_pdf(x, c); });
    build_single_cdf(lat.cdf_tt, 0.5 * (1.0 - 1.0 / m), 0.5 * (1.0 + 1.0 / m),
                     [&](double x) { return tamura_tt_pdf(x, c); });

    // Herring-Vogt tensors (crystal_lattice.hpp:394-438)
    Lattice& L = lat.view;
    const double m_xx = c.e_mass_tensor[0], m_yy = c.e_mass_tensor[1], m_zz = c.e_mass_tensor[2];
    const double m_cond_ratio = 3.0 / (1.0 / m_xx + 1.0 / m_yy + 1.0 / m_zz);
    L.e_cond_mass = m_cond_ratio * kMeEV;
    L.h_mass = c.h_mass_ratio * kMeEV;
    L.mass_ratio = v3(m_xx / m_cond_ratio, m_yy / m_cond_ratio, m_zz / m_cond_ratio);
    L.hv_sqrt = v3(std::sqrt(L.mass_ratio.x), std::sqrt(L.mass_ratio.y), std::sqrt(L.mass_ratio.z));
    L.hv_sqrt_inv = v3(1.0 / L.hv_sqrt.x, 1.0 / L.hv_sqrt.y, 1.0 / L.hv_sqrt.z);
    M3 orient;
    std::memcpy(orient.m, c.orient, sizeof(orient.m));
    L.n_valleys = c.n_valleys;
    for (int iv = 0; iv < c.n_valleys; ++iv) {
        const V3 raw = v3(c.valley_dirs[iv][0], c.valley_dirs[iv][1], c.valley_dirs[iv][2]);
        const V3 vdir = unit(mul(orient, unit(raw)));
        const double vx = vdir.x, vy = vdir.y, vz = vdir.z;
        const double f = std::sqrt(std::max(0.0, 1.0 - vz * vz));
        const double a = (std::abs(vy) < 1e-12) ? 0.0 : ((std::abs(vx) < 1e-12) ? -1.0 : -vy / f);
        const double b = (std::abs(vy) < 1e-12) ? 1.0 : ((std::abs(vx) < 1e-12) ? 0.0 : vx / f);
        const double d = -vz * b;
        const double e = vz * a;
        M3& R = L.valley_rot[iv];
        R.m[0][0] = vdir.x; R.m[0][1] = vdir.y; R.m[0][2] = vdir.z;
        R.m[1][0] = a;      R.m[1][1] = b;      R.m[1][2] = 0.0;
        R.m[2][0] = d;      R.m[2][1] = e;      R.m[2][2] = f;
    }
    auto compute_l0 = [&](double mass_ratio_me, double ac_deform_eV) -> double {
        if (ac_deform_eV <= 0.0) return 1e-6;
        const double hbar_SI = kHbar * kElemCharge;
        const double m_SI = mass_ratio_me * kMeKg;
        const double ac_SI = ac_deform_eV * kElemCharge;
        const double hbar4 = (hbar_SI * hbar_SI) * (hbar_SI * hbar_SI);
        const double m3 = m_SI * m_SI * m_SI;
        return 0.5 * kPi * hbar4 * c.density / (m3 * ac_SI * ac_SI);
    };
    L.l0_e = compute_l0(m_cond_ratio, c.ac_deform_e);
    L.l0_h = compute_l0(c.h_mass_ratio, c.ac_deform_h);
    L.k_sound_e = (L.e_cond_mass * c.v_sound) / (kCLight * kHbarC);
    L.k_sound_h = (L.h_mass * c.v_sound) / (kCLight * kHbarC);

    lat.hv = {L.e_cond_mass, L.h_mass, L.mass_ratio.x, L.mass_ratio.y, L.mass_ratio.z,
              L.hv_sqrt.x, L.hv_sqrt.y, L.hv_sqrt.z, L.hv_sqrt_inv.x, L.hv_sqrt_inv.y, L.hv_sqrt_inv.z,
              L.l0_e, L.l0_h, L.k_sound_e, L.k_sound_h, static_cast<double>(c.n_valleys)};
    for (int iv = 0; iv < c.n_valleys; ++iv)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) lat.hv.push_back(L.valley_rot[iv].m[i][j]);

    // scalar view
    L.oct = lat.oct.data();
    L.kin_mode = kKinOctahedral;
    L.density = c.density;
    L.stiff = &lat.stiff;
    L.bil = nullptr;
    L.cdf_lt = lat.cdf_lt.data();
    L.cdf_tt = lat.cdf_tt.data();
    L.orient = orient;
    L.B_iso = c.B_iso;
    L.A_anh = c.A_anh;
    L.fTT_frac = c.fTT_frac;
    L.poly_mfp = c.polycrystal_mfp_m;
    L.fLDOS = c.fLDOS;
    L.fSTDOS = c.fSTDOS;
    L.fFTDOS = c.fFTDOS;
    L.v_sound = c.v_sound;
    L.v_trans = c.v_trans;
    L.bandgap = c.bandgap;
    L.debye_energy = c.debye_freq * kHPlanck;
    L.iv_model = c.iv_model;
    L.iv_min_energy = c.iv_min_energy;
    L.iv_quad_rate = c.iv_quad_rate;
    L.iv_quad_field = c.iv_quad_field;
    L.iv_quad_power = c.iv_quad_power;
    L.iv_lin_rate0 = c.iv_lin_rate0;
    L.iv_lin_rate1 = c.iv_lin_rate1;
    L.iv_lin_power = c.iv_lin_power;
    L.e_trap_mfp = c.e_trapping_mfp_m;
    L.h_trap_mfp = c.h_trapping_mfp_m;
    L.e_ion_d0_mfp = c.e_trap_ion_d0_mfp_m;
    L.e_ion_a_mfp = c.e_trap_ion_a_mfp_m;
    L.h_ion_d_mfp = c.h_trap_ion_d_mfp_m;
    L.h_ion_a0_mfp = c.h_trap_ion_a0_mfp_m;
}

}  // namespace

extern "C" {

// CrystalConfig defaults (crystal_config.hpp:43-134) with the Germanium preset's
// Debye frequency (presets.hpp:18-25).
void cmpmc_crystal_config_germanium(cmpmc_crystal_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->group = 1;
    c->density = 5323.0;
    c->C11 = 126.0 * kGPa;
    c->C12 = 44.0 * kGPa;
    c->C44 = 67.0 * kGPa;
    c->beta = -73.2 * kGPa;
    c->gamma = -70.8 * kGPa;
    c->lambda = 37.6 * kGPa;
    c->mu = 56.1 * kGPa;
    c->B_iso = 3.67e-41;
    c->A_anh = 6.43e-55;
    c->fTT_frac = 0.74;
    c->fLDOS = 0.097834;
    c->fSTDOS = 0.535390;
    c->fFTDOS = 0.366770;
    c->debye_freq = 8.64 * 1e12;
    c->v_sound = 5324.2077;
    c->v_trans = 3258.7879;
    c->bandgap = 0.74;
    c->pair_energy = 2.96;
    c->fano_factor = 0.1057;
    c->epsilon_rel = 16.2;
    c->neutral_impurity_cm3 = 1.0e11;
    c->alpha_nonparabolic = 0.3;
    c->h_mass_ratio = 0.350;
    c->e_mass_tensor[0] = 1.588;
    c->e_mass_tensor[1] = 0.081;
    c->e_mass_tensor[2] = 0.081;
    c->n_valleys = 4;
    const double vd[4][3] = {{1, 1, 1}, {-1, 1, 1}, {-1, -1, 1}, {1, -1, 1}};
    std::memcpy(c->valley_dirs, vd, sizeof(vd));
    c->ac_deform_e = 11.0;
    c->ac_deform_h = 3.4;
    c->n_iv = 2;
    c->iv_deform_eV_m[0] = 3.0e10;
    c->iv_deform_eV_m[1] = 0.2e10;
    c->iv_energy_eV[0] = 27.3 * kMeV;
    c->iv_energy_eV[1] = 10.3 * kMeV;
    c->iv_min_energy = 10.3 * kMeV;
    c->iv_model = 0;
    c->iv_quad_rate = 6.72e-2;
    c->iv_quad_field = 217.0;
    c->iv_quad_power = 3.24;
    c->iv_lin_rate0 = 1.5e6;
    c->iv_lin_rate1 = 1.5;
    c->iv_lin_power = 4.0;
    c->orient[0][0] = c->orient[1][1] = c->orient[2][2] = 1.0;
    c->atomic_Z = 32.0;
    c->atomic_A = 72.63;
}

int cmpmc_lattice_create(const cmpmc_crystal_config* cfg, cmpmc_lattice** out) {
    if (!cfg || !out) return CMPMC_ERR_INVALID;
    *out = nullptr;
    if (cfg->n_valleys < 0 || cfg->n_valleys > CMPMC_MAX_VALLEYS || cfg->density <= 0.0) return CMPMC_ERR_INVALID;
    cmpmc_lattice* lat = new (std::nothrow) cmpmc_lattice();
    if (!lat) return CMPMC_ERR_INVALID;
    lat->cfg = *cfg;
    build_tables(*lat);
    static std::atomic<uint64_t> next_id{1};
    lat->id = next_id.fetch_add(1);
    *out = lat;
    return CMPMC_OK;
}

void cmpmc_lattice_destroy(cmpmc_lattice* lat) { delete lat; }

int cmpmc_lattice_set_kinematics_mode(cmpmc_lattice* lat, int mode) {
    if (!lat || mode < kKinOctahedral || mode > kKinBilinear) return CMPMC_ERR_INVALID;
    if (mode == kKinBilinear && lat->bil.empty()) build_bilinear(*lat);
    lat->view.bil = lat->bil.empty() ? nullptr : lat->bil.data();
    lat->view.kin_mode = mode;
    return CMPMC_OK;
}

int cmpmc_lattice_kinematics_mode(const cmpmc_lattice* lat) { return lat ? lat->view.kin_mode : -1; }

int cmpmc_lattice_tables(const cmpmc_lattice* lat, const float** oct_lut, const double** cdf_lt,
                         const double** cdf_tt, const double** hv, size_t* n_hv) {
    if (!lat) return CMPMC_ERR_INVALID;
    if (oct_lut) *oct_lut = reinterpret_cast<const float*>(lat->oct.data());
    if (cdf_lt) *cdf_lt = lat->cdf_lt.data();
    if (cdf_tt) *cdf_tt = lat->cdf_tt.data();
    if (hv) *hv = lat->hv.data();
    if (n_hv) *n_hv = lat->hv.size();
    return CMPMC_OK;
}

int cmpmc_lattice_map_k_to_vg(const cmpmc_lattice* lat, int mode, const double k_det[3], double vg_dir[3],
                              double* vg_mag) {
    if (!lat || mode < 0 || mode > 2 || !k_det || !vg_dir || !vg_mag) return CMPMC_ERR_INVALID;
    const Kin kin = map_k_to_vg(lat->view, mode, v3(k_det[0], k_det[1], k_det[2]));
    vg_dir[0] = kin.vg_dir.x;
    vg_dir[1] = kin.vg_dir.y;
    vg_dir[2] = kin.vg_dir.z;
    *vg_mag = kin.vg_mag;
    return CMPMC_OK;
}

int cmpmc_make_track(const cmpmc_lattice* lat, const double pos[3], const double k_dir[3], int mode,
                     double energy_eV, double time_s, double weight, cmpmc_phonon_track* out) {
    if (!lat || mode < 0 || mode > 2 || !pos || !k_dir || !out) return CMPMC_ERR_INVALID;
    const Track t = make_track(lat->view, v3(pos[0], pos[1], pos[2]), v3(k_dir[0], k_dir[1], k_dir[2]), mode,
                               energy_eV, time_s, weight);
    track_to_record(t, *out);
    return CMPMC_OK;
}

int cmpmc_make_charge(const cmpmc_lattice* lat, int type, const double pos[3], const double dir[3],
                      double ekin_eV, int valley, double time_s, cmpmc_charge_track* out) {
    if (!lat || (type != 1 && type != 2) || !pos || !dir || !out) return CMPMC_ERR_INVALID;
    if (type == 1 && (valley < 0 || valley >= lat->view.n_valleys)) return CMPMC_ERR_INVALID;
    const Charge c = make_charge(lat->view, type, v3(pos[0], pos[1], pos[2]), v3(dir[0], dir[1], dir[2]), ekin_eV,
                                 valley, time_s);
    charge_to_record(c, *out);
    return CMPMC_OK;
}

void cmpmc_rng_for_stream(uint64_t seed, uint64_t stream, uint64_t state[4]) {
    const Rng r = Rng::for_stream(seed, stream);
    for (int i = 0; i < 4; ++i) state[i] = r.s[i];
}

uint64_t cmpmc_rng_next_u64(uint64_t state[4]) {
    Rng r;
    for (int i = 0; i < 4; ++i) r.s[i] = state[i];
    const uint64_t x = r.next_u64();
    for (int i = 0; i < 4; ++i) state[i] = r.s[i];
    return x;
}

double cmpmc_rng_uniform(uint64_t state[4]) {
    Rng r;
    for (int i = 0; i < 4; ++i) r.s[i] = state[i];
    const double x = r.uniform();
    for (int i = 0; i < 4; ++i) state[i] = r.s[i];
    return x;
}

}  // extern "C"
