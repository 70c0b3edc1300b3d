// transport.cuh -- the per-event phonon and charge transport loops in FP64.
//
// transport_phonons restates SimulationEngine::transport (transport/engine.hpp:403-582)
// and transport_charges restates SimulationEngine::transport_charges (engine.hpp:192-380)
// with the same random-draw order, so a device thread that runs one event from the
// event's post-generator Rng state reproduces the CPU's event stream.
//
// The loops are templates over an event context `C` that owns the LIFO stacks and the
// hit sink; the device kernels supply global-memory stacks (transport_plain.cu).
#pragma once

#include "mesh.cuh"
#include "phys.cuh"

namespace cmpmc_gpu {

// Detector view (DetectorModel, engine.hpp:96-156; CylinderSolid, solids.hpp:23-26)
struct Detector {
    double radius, half_z;
    V3 e_field;
    Surface surf[3];
    uint32_t max_bounces;
    uint32_t rr_bounces;
    double rr_survival;
    double min_phonon_eV;
    double luke_sample_fraction;
    double charge_max_dk_frac, charge_dt_cap_s, charge_sampling_dk_frac;
    int charge_stepping;
    double fermi_level_above_Ev_eV;
    int charge_release;            // DetectorModel::ChargeRelease: 0 RecordOnly, 1 BulkDebye, 2 ElectrodeFilm
    double electrode_seed_max_gap;
    MeshView mesh;      // DetectorModel::mesh_field_3d on the device (tet == nullptr: uniform field)
    MeshView32 mesh32;  // the same mesh in FP32 (batched charge form)
    MeshView2 mesh2;       // DetectorModel::mesh_field_2d, used when there is no 3D mesh
    MeshView2_32 mesh2_32;  // the 2D mesh in FP32 (batched charge form)
};

// Phonon state held in registers (PhononTrack, track.hpp:62-72)
struct Track {
    V3 pos, k, vg;
    double E, vmag, t, w;
    uint32_t bounces;
    int mode;
};

// Charge state (ChargeTrack, track.hpp:75-84)
struct Charge {
    V3 pos, p;
    double ekin, t, w;
    int valley;
    int type;  // 1 electron, 2 hole
};

// Per-event counters and ledgers (SimStats fields used by the two loops)
struct EvStats {
    uint64_t total_steps, isotope_scatters, polycrystal_scatters, decays_TT, decays_LT,
        surface_refls, surface_downconversions, sensor_hits, killed_tracks;
    uint64_t charge_steps, luke_emitted, intervalley_scatters, charges_trapped, trap_ionizations,
        charge_surface_refls, charges_collected;
    double luke_eV, recomb_eV, deposited_eV, escaped_eV;
};

struct Hit {
    V3 pos;
    double t, edep, incident;
    int surf, excitation, mode;
};

// SimulationEngine::make_track (engine.hpp:171-187)
CMPMC_HD Track make_track(const Lattice& L, V3 pos, V3 k_dir, int mode, double e, double t, double w) {
    const V3 ku = unit(k_dir);
    const Kin kin = map_k_to_vg(L, mode, ku);
    Track r;
    r.pos = pos;
    r.k = ku;
    r.vg = kin.vg_dir;
    r.E = e;
    r.vmag = kin.vg_mag;
    r.t = t;
    r.w = w;
    r.bounces = 0;
    r.mode = mode;
    return r;
}

// SimulationEngine::sample_inward_wavevector (engine.hpp:927-936)
CMPMC_HD V3 sample_inward(const Lattice& L, int mode, V3 n, Rng& rng) {
    for (int trial = 0; trial < 16; ++trial) {
        const V3 kd = rng.lambertian_dir(n);
        const Kin kin = map_k_to_vg(L, mode, kd);
        if (dot(kin.vg_dir, n) > 1e-6) return kd;
    }
    return n;
}

CMPMC_HD void set_kin(Track& trk, const Kin& kin) {
    trk.vg = kin.vg_dir;
    trk.vmag = kin.vg_mag;
}

// SimulationEngine::perform_anharmonic_decay (engine.hpp:938-988)
template <class C>
CMPMC_HD void anharmonic_decay(const Lattice& L, Track& trk, C& ctx, EvStats& st, Rng& rng) {
    const V3 dir1 = trk.k;
    const V3 perp = orthogonal_unit(dir1);
    const double phi = kTwoPi * rng.uniform();
    const double c_phi = m_cos(phi);
    const double s_phi = m_sin(phi);
    if (rng.uniform() < L.fTT_frac) {
        st.decays_TT++;
        const double x = sample_cdf(L.cdf_tt, rng);
        const double th1 = decay_angle_TT(x, L.v_sound, L.v_trans);
        const double th2 = decay_angle_TT(1.0 - x, L.v_sound, L.v_trans);
        const V3 k1 = unit(rotate_around(rotate_around(dir1, perp, m_cos(th1), m_sin(th1)), dir1, c_phi, s_phi));
        const V3 k2 = unit(rotate_around(rotate_around(dir1, perp, m_cos(-th2), m_sin(-th2)), dir1, c_phi, s_phi));
        const int m1 = sample_transverse_mode(L, rng);
        const int m2 = sample_transverse_mode(L, rng);
        ctx.push(make_track(L, trk.pos, k2, m2, (1.0 - x) * trk.E, trk.t, trk.w));
        trk.E = x * trk.E;
        trk.mode = m1;
        trk.k = k1;
        set_kin(trk, map_k_to_vg(L, m1, k1));
    } else {
        st.decays_LT++;
        const double x = sample_cdf(L.cdf_lt, rng);
        const double thL = decay_angle_L_to_LT(x, L.v_sound, L.v_trans);
        const double thT = decay_angle_T_from_LT(x, L.v_sound, L.v_trans);
        const V3 kL = unit(rotate_around(rotate_around(dir1, perp, m_cos(thL), m_sin(thL)), dir1, c_phi, s_phi));
        const V3 kT = unit(rotate_around(rotate_around(dir1, perp, m_cos(-thT), m_sin(-thT)), dir1, c_phi, s_phi));
        const int mT = sample_transverse_mode(L, rng);
        ctx.push(make_track(L, trk.pos, kT, mT, (1.0 - x) * trk.E, trk.t, trk.w));
        trk.E = x * trk.E;
        trk.mode = 0;
        trk.k = kL;
        set_kin(trk, map_k_to_vg(L, 0, kL));
    }
}

// SimulationEngine::transport (engine.hpp:403-582). ctx provides
//   bool pop(Track&), void push(const Track&), void hit(const Hit&),
//   KBuf refl (kKaplanCap doubles) and double* kwork (4 * kKaplanCap doubles).
template <class C>
CMPMC_HD void transport_phonons(const Lattice& L, const Detector& D, C& ctx, EvStats& st, Rng& rng) {
    Track trk;
    while (ctx.pop(trk)) {
        for (;;) {
            if (trk.E < D.min_phonon_eV || trk.bounces >= D.max_bounces) {
                st.killed_tracks++;
                st.escaped_eV += trk.E * trk.w;
                break;
            }
            // apply_russian_roulette (transport/variance_reduction.hpp:17-29); a killed
            // track's energy is not added to the ledger (engine.hpp:423-428)
            if (D.rr_bounces != 0 && trk.bounces > D.rr_bounces && (trk.bounces - D.rr_bounces) % 32 == 0) {
                if (rng.uniform() < D.rr_survival) {
                    trk.w /= D.rr_survival;
                } else {
                    st.killed_tracks++;
                    break;
                }
            }
            st.total_steps++;
            const double rate_iso = isotope_rate(L, trk.E);
            const double rate_poly = polycrystal_rate(L, trk.vmag);
            const double rate_down = downconversion_rate(L, trk.mode, trk.E);
            const double rate_tot = rate_iso + rate_poly + rate_down;
            const double d_phys = (rate_tot > 1e-12) ? (-m_log(rng.uniform()) * (trk.vmag / rate_tot)) : kInf;
            const BHit bh = intersect_exit(D.radius, D.half_z, trk.pos, trk.vg);

            // new direction drawn after the branches below: 1 isotropic (Rng::isotropic_dir,
            // rng.hpp:78-83), 2 Lambertian about the inward normal with the inward check of
            // sample_inward_wavevector (engine.hpp:927-936). The two share one block so the
            // lanes of a warp stay together; each lane computes exactly the reference's values.
            int new_dir = 0;
            if (d_phys < bh.distance) {
                trk.pos = trk.pos + trk.vg * d_phys;
                trk.t += d_phys / trk.vmag;
                const double u_proc = rng.uniform() * rate_tot;
                if (rate_down > 0.0 && u_proc < rate_down) {
                    anharmonic_decay(L, trk, ctx, st, rng);
                } else {
                    if (u_proc < rate_down + rate_iso) st.isotope_scatters++;
                    else st.polycrystal_scatters++;
                    trk.mode = sample_dos_mode(L, rng);
                    new_dir = 1;
                }
            } else {

                trk.pos = trk.pos + trk.vg * bh.distance;
                trk.t += bh.distance / trk.vmag;
                trk.bounces++;
                const Surface& s = D.surf[bh.surf];
                // electrode mask (engine.hpp:483-488): bare crystal between pads reflects
                const int ch_id = (s.n_pads > 0) ? find_channel(s.pads, s.n_pads, trk.pos.x, trk.pos.y, rng) : -1;
                const bool active_pad = (s.n_pads == 0) || ch_id >= 0;

                if (active_pad && s.has_film && rng.uniform() < s.prob_abs) {
                    const Film& film = s.film;
                    const double p_enter = s.has_amm ? amm_transmission(s.amm_sub, s.amm_film, trk.mode == 0,
                                                                        dot(trk.k, bh.n_in))
                                                     : film.film_absorption;
                    if (rng.uniform() < p_enter) {
                        const double edep = film_absorb_phonon(film, trk.E, ctx.refl, ctx.kwork, rng);
                        if (edep > 0.0) {
                            const double wedep = edep * trk.w;
                            st.sensor_hits++;
                            st.deposited_eV += wedep;
                            Hit h;
                            h.pos = trk.pos;
                            h.t = trk.t;
                            h.edep = wedep;
                            h.incident = trk.E;
                            h.surf = bh.surf;
                            h.excitation = 0;
                            h.mode = trk.mode;
                            ctx.hit(h, ch_id);
                        }
                        double sum_refl = 0.0;
                        for (int i = 0; i < ctx.refl.n; ++i) sum_refl += ctx.refl.d[i];
                        st.escaped_eV += dmax(0.0, trk.E - edep - sum_refl) * trk.w;
                        if (ctx.refl.n == 0) break;
                        const V3 reemit = trk.pos + bh.n_in * 1e-11;
                        for (int i = 1; i < ctx.refl.n; ++i) {
                            const int m = sample_dos_mode(L, rng);
                            const V3 kd = sample_inward(L, m, bh.n_in, rng);
                            ctx.push(make_track(L, reemit, kd, m, ctx.refl.d[i], trk.t, trk.w));
                        }
                        trk.pos = reemit;
                        trk.E = ctx.refl.d[0];
                        trk.mode = sample_dos_mode(L, rng);
                        trk.k = sample_inward(L, trk.mode, bh.n_in, rng);
                        set_kin(trk, map_k_to_vg(L, trk.mode, trk.k));
                        continue;
                    }
                }

                if (rng.uniform() > s.prob_refl) {
                    st.killed_tracks++;
                    st.escaped_eV += trk.E * trk.w;
                    break;
                }
                st.surface_refls++;
                trk.pos = trk.pos + bh.n_in * 1e-11;
                const Split split = reflection_split(s, trk.E);
                const double u_refl = rng.uniform();
                if (u_refl < split.p_anh) {
                    st.surface_downconversions++;
                    const bool tt = rng.uniform() < L.fTT_frac;
                    const double x = tt ? sample_cdf(L.cdf_tt, rng) : sample_cdf(L.cdf_lt, rng);
                    const int m1 = tt ? sample_transverse_mode(L, rng) : 0;
                    const int m2 = sample_transverse_mode(L, rng);
                    const V3 k2 = sample_inward(L, m2, bh.n_in, rng);
                    ctx.push(make_track(L, trk.pos, k2, m2, (1.0 - x) * trk.E, trk.t, trk.w));
                    trk.E = x * trk.E;
                    trk.mode = m1;
                    trk.k = sample_inward(L, m1, bh.n_in, rng);
                    set_kin(trk, map_k_to_vg(L, m1, trk.k));
                } else if (u_refl < split.p_anh + split.p_spec) {
                    V3 k_refl = trk.k - bh.n_in * (2.0 * dot(trk.k, bh.n_in));
                    Kin kin = map_k_to_vg(L, trk.mode, k_refl);
                    if (dot(kin.vg_dir, bh.n_in) <= 1e-6) {
                        k_refl = sample_inward(L, trk.mode, bh.n_in, rng);
                        kin = map_k_to_vg(L, trk.mode, k_refl);
                    }
                    trk.k = k_refl;
                    set_kin(trk, kin);
                } else {
                    new_dir = 2;
                }
            }
            if (new_dir != 0) {
                const bool iso = (new_dir == 1);
                V3 ou = v3(1.0, 0.0, 0.0), ov = ou;
                if (!iso) {
                    ou = orthogonal_unit(bh.n_in);
                    ov = cross(bh.n_in, ou);
                }
                V3 kd;
                Kin kin;
                for (int trial = 0;; ++trial) {
                    const double u1 = rng.uniform();
                    const double u2 = rng.uniform();
                    double st_, ct_, phi;
                    if (iso) {
                        ct_ = 2.0 * u1 - 1.0;
                        st_ = sqrt(dmax(0.0, 1.0 - ct_ * ct_));
                        phi = kTwoPi * u2;
                    } else {
                        phi = kTwoPi * u1;
                        st_ = sqrt(u2);
                        ct_ = sqrt(dmax(0.0, 1.0 - st_ * st_));
                    }
                    const double cphi = m_cos(phi);
                    const double sphi = m_sin(phi);
                    kd = iso ? v3(st_ * cphi, st_ * sphi, ct_)
                             : unit(ou * (st_ * cphi) + ov * (st_ * sphi) + bh.n_in * ct_);
                    kin = map_k_to_vg(L, trk.mode, kd);
                    if (iso || dot(kin.vg_dir, bh.n_in) > 1e-6) break;
                    if (trial == 15) {
                        kd = bh.n_in;
                        kin = map_k_to_vg(L, trk.mode, kd);
                        break;
                    }
                }
                trk.k = kd;
                set_kin(trk, kin);
            }
        }
    }
}

// ---- Herring-Vogt kinematics (crystal_lattice.hpp:239-293) --------------------------
CMPMC_HD V3 e2s(const Lattice& L, int iv, V3 v) {
    const V3 vv = mul(L.valley_rot[iv], v);
    return v3(vv.x * L.hv_sqrt_inv.x, vv.y * L.hv_sqrt_inv.y, vv.z * L.hv_sqrt_inv.z);
}
CMPMC_HD V3 s2e(const Lattice& L, int iv, V3 v) {
    const V3 sc = v3(v.x * L.hv_sqrt.x, v.y * L.hv_sqrt.y, v.z * L.hv_sqrt.z);
    return mul_transpose(L.valley_rot[iv], sc);
}
CMPMC_HD double ekin_electron(const Lattice& L, int iv, V3 p) {
    const V3 ph = e2s(L, iv, p);
    return sqrt(norm2(ph) + L.e_cond_mass * L.e_cond_mass) - L.e_cond_mass;
}
CMPMC_HD double ekin_hole(const Lattice& L, V3 p) { return sqrt(norm2(p) + L.h_mass * L.h_mass) - L.h_mass; }
CMPMC_HD V3 vel_electron(const Lattice& L, int iv, V3 p) {
    const double ek = ekin_electron(L, iv, p);
    const V3 pv = mul(L.valley_rot[iv], p);
    const V3 vv = v3(pv.x / L.mass_ratio.x, pv.y / L.mass_ratio.y, pv.z / L.mass_ratio.z);
    return mul_transpose(L.valley_rot[iv], vv) * (kCLight / (ek + L.e_cond_mass));
}
CMPMC_HD V3 vel_hole(const Lattice& L, V3 p) {
    const double ek = ekin_hole(L, p);
    return p * (kCLight / (ek + L.h_mass));
}
CMPMC_HD V3 ekin_to_p_electron(const Lattice& L, int iv, V3 p_dir, double ek) {
    const V3 u = unit(p_dir);
    const V3 uh = e2s(L, iv, u);
    const double band_u = norm2(uh);
    if (band_u <= 0.0 || ek <= 0.0) return v3(0.0, 0.0, 0.0);
    const double p_mag = sqrt((ek * ek + 2.0 * ek * L.e_cond_mass) / band_u);
    return u * p_mag;
}
CMPMC_HD double hv_max_scale(const Lattice& L) {
    return dmax(dmax(L.hv_sqrt_inv.x, L.hv_sqrt_inv.y), L.hv_sqrt_inv.z);
}

// ChargePhysics::make_charge (charge_transport.hpp:49-70)
CMPMC_HD Charge make_charge(const Lattice& L, int type, V3 pos, V3 dir, double ek, int valley, double t) {
    const V3 u = unit(dir);
    Charge c;
    if (type == 1) {
        c.p = ekin_to_p_electron(L, valley, u, ek);
    } else {
        const double p_mag = sqrt(dmax(0.0, ek * ek + 2.0 * ek * L.h_mass));
        c.p = u * p_mag;
    }
    c.pos = pos;
    c.ekin = ek;
    c.t = t;
    c.w = 1.0;
    c.valley = valley;
    c.type = type;
    return c;
}

// charge_transport.hpp:82-106
CMPMC_HD double luke_rate(const Lattice& L, const Charge& c) {
    double k_mag, k_sound, l0;
    if (c.type == 1) {
        k_mag = norm(e2s(L, c.valley, vdiv(c.p, kHbarC)));
        k_sound = L.k_sound_e;
        l0 = L.l0_e;
    } else {
        k_mag = norm(c.p) / kHbarC;
        k_sound = L.k_sound_h;
        l0 = L.l0_h;
    }
    if (k_mag <= k_sound) return 0.0;
    const double mach = k_mag / k_sound;
    const double dm = mach - 1.0;
    const double tstep = (3.0 * l0) / L.v_sound;
    const double tau = tstep * mach / (dm * dm * dm);
    return (tau > 0.0) ? (1.0 / tau) : 0.0;
}

// charge_kernels.hpp:329-346 (Quadratic and Linear models)
CMPMC_HD double intervalley_rate(const Lattice& L, double ek, V3 E) {
    if (L.n_valleys < 2) return 0.0;
    if (ek < L.iv_min_energy) return 0.0;
    if (L.iv_model == 0) {
        const double e0 = L.iv_quad_field;
        return L.iv_quad_rate * m_pow(e0 * e0 + norm2(E), 0.5 * L.iv_quad_power);
    }
    const double e_vcm = norm(E) * 0.01;
    return L.iv_lin_rate0 + L.iv_lin_rate1 * m_pow(e_vcm, L.iv_lin_power);
}
CMPMC_HD double mfp_rate(double v, double mfp) { return (mfp > 0.0 && mfp < 1e20) ? (v / mfp) : 0.0; }

struct Rates {
    double luke, iv, trap, ion_e, ion_h, tot;
};
// SimulationEngine::charge_rates (engine.hpp:876-886)
CMPMC_HD Rates charge_rates(const Lattice& L, const Charge& c, V3 E) {
    const double v = norm(c.type == 1 ? vel_electron(L, c.valley, c.p) : vel_hole(L, c.p));
    Rates r;
    r.luke = luke_rate(L, c);
    r.iv = (c.type == 1) ? intervalley_rate(L, c.ekin, E) : 0.0;
    const bool e = (c.type == 1);
    r.trap = mfp_rate(v, e ? L.e_trap_mfp : L.h_trap_mfp);
    r.ion_e = mfp_rate(v, e ? L.e_ion_d0_mfp : L.h_ion_d_mfp);
    r.ion_h = mfp_rate(v, e ? L.e_ion_a_mfp : L.h_ion_a0_mfp);
    r.tot = r.luke + r.iv + r.trap + r.ion_e + r.ion_h;
    return r;
}

struct LukeEmit {
    bool emitted;
    V3 q_dir;
    double e_ph;
};
// ChargePhysics::emit_luke_phonon (charge_transport.hpp:109-166)
CMPMC_HD LukeEmit emit_luke(const Lattice& L, Charge& c, Rng& rng) {
    LukeEmit none;
    none.emitted = false;
    V3 k_trk;
    double k_sound;
    if (c.type == 1) {
        k_trk = e2s(L, c.valley, vdiv(c.p, kHbarC));
        k_sound = L.k_sound_e;
    } else {
        k_trk = vdiv(c.p, kHbarC);
        k_sound = L.k_sound_h;
    }
    const double k_mag = norm(k_trk);
    if (k_mag <= k_sound * 1.0001) return none;
    const V3 k_dir = vdiv(k_trk, k_mag);
    const double v = k_sound / k_mag;
    const double u = rng.uniform();
    const double cos_th = dclamp(v + (1.0 - v) * m_cbrt(1.0 - u), v, 1.0);
    const double sin_th = sqrt(dmax(0.0, 1.0 - cos_th * cos_th));
    const double phi = kTwoPi * rng.uniform();
    const double q = 2.0 * (k_mag * cos_th - k_sound);
    if (q <= 0.0) return none;
    const V3 perp = orthogonal_unit(k_dir);
    const V3 q_vec = rotate_around(rotate_around(k_dir * q, perp, cos_th, sin_th), k_dir, m_cos(phi), m_sin(phi));
    const V3 k_recoil = k_trk - q_vec;
    const double e_ph = norm(q_vec) * L.v_sound * kHbar;
    if (e_ph >= c.ekin || e_ph <= 0.0) return none;
    LukeEmit r;
    r.emitted = true;
    r.e_ph = e_ph;
    if (c.type == 2) {
        c.p = k_recoil * kHbarC;
        c.ekin = ekin_hole(L, c.p);
        r.q_dir = unit(q_vec);
    } else {
        const V3 q_cryst = unit(s2e(L, c.valley, q_vec));
        const V3 p_rec_dir = s2e(L, c.valley, k_recoil) * kHbarC;
        const double e_recoil = c.ekin - e_ph;
        c.p = ekin_to_p_electron(L, c.valley, p_rec_dir, e_recoil);
        c.ekin = e_recoil;
        r.q_dir = q_cryst;
    }
    return r;
}

// charge_transport.hpp:169-184
CMPMC_HD void scatter_intervalley(const Lattice& L, Charge& c, Rng& rng) {
    const int nv = L.n_valleys;
    if (c.type != 1 || nv < 2) return;
    const V3 k_cryst = vdiv(c.p, kHbarC);
    const V3 k_valley = mul(L.valley_rot[c.valley], k_cryst);
    const uint64_t offset = 1 + static_cast<uint64_t>(rng.uniform() * static_cast<double>(nv - 1));
    const int nvl = static_cast<int>((static_cast<uint64_t>(c.valley) + offset) % static_cast<uint64_t>(nv));
    const V3 k_new = mul_transpose(L.valley_rot[nvl], k_valley);
    const V3 p_new_dir = k_new * kHbarC;
    c.valley = nvl;
    c.p = ekin_to_p_electron(L, nvl, p_new_dir, c.ekin);
}

// charge_transport.hpp:187-199
CMPMC_HD bool should_absorb_boundary(const Charge& c, V3 n_in, double prob, double min_ke, double min_kh,
                                     Rng& rng) {
    const V3 outward = n_in * (-1.0);
    const V3 k_vec = vdiv(c.p, kHbarC);
    const double k_perp = dot(k_vec, outward);
    const double min_k = (c.type == 1) ? min_ke : min_kh;
    if (k_perp <= min_k) return false;
    return rng.uniform() < prob;
}

// charge_transport.hpp:203-241
CMPMC_HD void reflect_at_boundary(const Lattice& L, Charge& c, V3 n_in, double spec_prob, Rng& rng) {
    if (rng.uniform() < spec_prob) {
        const V3 k_dir = unit(c.p);
        const V3 k_refl = unit(k_dir - n_in * (2.0 * dot(k_dir, n_in)));
        if (c.type == 2) {
            c.p = k_refl * norm(c.p);
            return;
        }
        const V3 p_trial = ekin_to_p_electron(L, c.valley, k_refl, c.ekin);
        const V3 v_trial = vel_electron(L, c.valley, p_trial);
        if (dot(v_trial, n_in) > 1e-6) {
            c.p = p_trial;
            return;
        }
    }
    if (c.type == 2) {
        const V3 dir = rng.lambertian_dir(n_in);
        c.p = dir * norm(c.p);
    } else {
        for (int trial = 0; trial < 16; ++trial) {
            const V3 dir = rng.lambertian_dir(n_in);
            const V3 p_trial = ekin_to_p_electron(L, c.valley, dir, c.ekin);
            const V3 v_trial = vel_electron(L, c.valley, p_trial);
            if (dot(v_trial, n_in) > 1e-6) {
                c.p = p_trial;
                return;
            }
        }
        c.p = ekin_to_p_electron(L, c.valley, n_in, c.ekin);
    }
}

CMPMC_HD double charge_ekin(const Lattice& L, const Charge& c) {
    return (c.type == 1) ? ekin_electron(L, c.valley, c.p) : ekin_hole(L, c.p);
}

// SimulationEngine::emit_debye_phonons (engine.hpp:894-903): the released energy as
// Debye-energy phonons at the contact, Lambertian inward
template <class C>
CMPMC_HD void emit_debye_phonons(const Lattice& L, double e_rel, V3 pos, V3 n_in, double t, double w, C& ctx,
                                 Rng& rng) {
    const double ed = L.debye_energy;
    const int k = static_cast<int>(round(e_rel / ed));
    const int n = (k < 1) ? 1 : k;
    const V3 p0 = pos + n_in * 1e-11;
    for (int i = 0; i < n; ++i) {
        const int m = sample_dos_mode(L, rng);
        const V3 kd = sample_inward(L, m, n_in, rng);
        ctx.push(make_track(L, p0, kd, m, e_rel / n, t, w));
    }
}

// SimulationEngine::electrode_film_release (engine.hpp:906-925): the released energy enters
// the electrode's film as quanta of at most max(4, electrode_seed_max_gap) Delta (photon
// seeds); the absorbed part is the hit, escaping phonons re-enter the crystal, the rest is lost
template <class C>
CMPMC_HD double electrode_film_release(const Lattice& L, const Detector& D, const Film& film, double e_rel, V3 pos,
                                       V3 n_in, double t, double w, C& ctx, double& lost, Rng& rng) {
    const double qmax = dmax(4.0, D.electrode_seed_max_gap) * film.gap_energy;
    const int k = static_cast<int>(ceil(e_rel / qmax));
    const int n = (k < 1) ? 1 : k;
    const double q = e_rel / n;
    const V3 p0 = pos + n_in * 1e-11;
    double absorbed = 0.0, emitted = 0.0;
    for (int i = 0; i < n; ++i) {
        absorbed += film_absorb_quantum(film, q, ctx.refl, ctx.kwork, rng, true);
        for (int k = 0; k < ctx.refl.n; ++k) {
            const int m = sample_dos_mode(L, rng);
            const V3 kd = sample_inward(L, m, n_in, rng);
            ctx.push(make_track(L, p0, kd, m, ctx.refl.d[k], t, w));
            emitted += ctx.refl.d[k];
        }
    }
    lost = dmax(0.0, e_rel - absorbed - emitted);
    return absorbed;
}

// SimulationEngine::transport_charges (engine.hpp:192-380). ctx provides
//   bool pop_charge(Charge&), void push_charge(const Charge&), void push(const Track&),
//   void hit(const Hit&, int channel), V3 field(V3 pos, Charge&).
template <class C>
CMPMC_HD void transport_charges(const Lattice& L, const Detector& D, C& ctx, EvStats& st, Rng& rng) {
    const double e_gap = L.bandgap;
    const double luke_prob = dclamp(D.luke_sample_fraction, 0.0, 1.0);
    const double luke_wt_mult = (luke_prob > 0.0) ? (1.0 / luke_prob) : 0.0;
    Charge c;
    while (ctx.pop_charge(c)) {
        const double q_sign = (c.type == 1) ? -1.0 : +1.0;
        for (uint32_t step = 0; step < 20000000u; ++step) {
            st.charge_steps++;
            const V3 E = ctx.field(c.pos, c);
            const bool second = (D.charge_stepping == 1);
            const double dk_frac = second ? D.charge_sampling_dk_frac : D.charge_max_dk_frac;
            const Rates R0 = charge_rates(L, c, E);
            double r_luke = R0.luke, r_iv = R0.iv, r_trap = R0.trap, r_ion_e = R0.ion_e, r_ion_h = R0.ion_h;
            double r_tot = R0.tot;
            double dt_max = D.charge_dt_cap_s;
            if (dk_frac > 0.0) {
                const bool is_e = (c.type == 1);
                const double ks = is_e ? L.k_sound_e : L.k_sound_h;
                const double k_now = is_e ? norm(e2s(L, c.valley, vdiv(c.p, kHbarC))) : norm(c.p) / kHbarC;
                const double dk_rate = norm(E) * kCLight / kHbarC * (is_e ? hv_max_scale(L) : 1.0);
                if (dk_rate > 0.0) dt_max = dmin(dt_max, dk_frac * dmax(ks, k_now) / dk_rate);
            }
            double dt_phys;
            if (second) {
                // Leman second-order stepping (engine.hpp:235-254)
                Charge trial = c;
                trial.p = trial.p + E * (q_sign * kCLight * dt_max);
                trial.ekin = charge_ekin(L, trial);
                const double a0 = R0.tot;
                const double a1 = (charge_rates(L, trial, E).tot - a0) / dt_max;
                const double lnu = m_log(rng.uniform());
                if (fabs(a1) * dt_max <= 1e-9 * dmax(a0, 1e-300)) {
                    dt_phys = (a0 > 0.0) ? (-lnu / a0) : kInf;
                } else {
                    const double disc = a0 * a0 - 2.0 * a1 * lnu;
                    dt_phys = (disc < 0.0) ? kInf : (sqrt(disc) - a0) / a1;
                    if (!(dt_phys >= 0.0)) dt_phys = kInf;
                }
            } else {
                dt_phys = (r_tot > 1.0) ? (-m_log(rng.uniform()) / r_tot) : kInf;
            }
            const double dt = dmin(dt_phys, dt_max);
            const V3 dp = E * (q_sign * kCLight * dt);
            const V3 p_mid = c.p + dp * 0.5;
            const V3 v_mid = (c.type == 1) ? vel_electron(L, c.valley, p_mid) : vel_hole(L, p_mid);
            const double v_mid_mag = norm(v_mid);
            const double d_step = v_mid_mag * dt;

            if (v_mid_mag > 1e-6) {
                const V3 v_dir = vdiv(v_mid, v_mid_mag);
                const BHit bh = intersect_exit(D.radius, D.half_z, c.pos, v_dir);
                if (bh.distance <= d_step) {
                    const double dt_b = bh.distance / v_mid_mag;
                    c.pos = c.pos + v_dir * bh.distance;
                    c.t += dt_b;
                    c.p = c.p + E * (q_sign * kCLight * dt_b);
                    c.ekin = charge_ekin(L, c);
                    const Surface& s = D.surf[bh.surf];
                    // electrode mask (engine.hpp:284-289)
                    const int ch_id = (s.n_pads > 0) ? find_channel(s.pads, s.n_pads, c.pos.x, c.pos.y, rng) : -1;
                    const bool active_pad = (s.n_pads == 0) || ch_id >= 0;
                    if (!active_pad ||
                        !should_absorb_boundary(c, bh.n_in, s.prob_charge_abs, s.min_k_elec, s.min_k_hole, rng)) {
                        st.charge_surface_refls++;
                        c.pos = c.pos + bh.n_in * 1e-11;
                        reflect_at_boundary(L, c, bh.n_in, s.prob_charge_spec, rng);
                        continue;
                    }
                    // collection_release_energy (engine.hpp:889-893) and the release mode
                    // (engine.hpp:302-313)
                    const double muF = (D.fermi_level_above_Ev_eV >= 0.0) ? D.fermi_level_above_Ev_eV : 0.5 * e_gap;
                    const double e_rel = c.ekin + ((c.type == 1) ? (e_gap - muF) : muF);
                    st.charges_collected++;
                    double hit_eV = e_rel;
                    if (D.charge_release == 1) {
                        hit_eV = 0.0;
                        emit_debye_phonons(L, e_rel, c.pos, bh.n_in, c.t, c.w, ctx, rng);
                    } else if (D.charge_release == 2 && s.has_film) {
                        double lost = 0.0;
                        hit_eV = electrode_film_release(L, D, s.film, e_rel, c.pos, bh.n_in, c.t, c.w, ctx, lost, rng);
                        st.escaped_eV += lost * c.w;
                    }
                    const double recomb = hit_eV * c.w;
                    st.recomb_eV += recomb;
                    st.deposited_eV += recomb;
                    Hit h;
                    h.pos = c.pos;
                    h.t = c.t;
                    h.edep = recomb;
                    h.incident = e_rel;
                    h.surf = bh.surf;
                    h.excitation = c.type;
                    h.mode = 0;
                    ctx.hit(h, ch_id);
                    break;
                }
            }

            c.pos = c.pos + v_mid * dt;
            c.t += dt;
            c.p = c.p + dp;
            c.ekin = charge_ekin(L, c);

            if (dt_phys <= dt_max) {
                if (second) {
                    const Rates R = charge_rates(L, c, E);
                    r_luke = R.luke; r_iv = R.iv; r_trap = R.trap; r_ion_e = R.ion_e; r_ion_h = R.ion_h; r_tot = R.tot;
                    if (r_tot <= 0.0) continue;
                }
                const double u_proc = rng.uniform() * r_tot;
                if (u_proc < r_trap) {
                    st.charges_trapped++;
                    st.escaped_eV += (c.ekin + 0.5 * e_gap) * c.w;
                    break;
                } else if (u_proc < r_trap + r_ion_e + r_ion_h) {
                    st.trap_ionizations++;
                    const bool lib_elec = (u_proc < r_trap + r_ion_e);
                    const uint64_t n_val = (L.n_valleys > 1) ? static_cast<uint64_t>(L.n_valleys) : 1u;
                    const int kv = lib_elec ? static_cast<int>(static_cast<uint16_t>(rng.next_u64() % n_val)) : 0;
                    Charge knock = make_charge(L, lib_elec ? 1 : 2, c.pos, rng.isotropic_dir(), 1.0e-6, kv, c.t);
                    knock.w = c.w;
                    ctx.push_charge(knock);
                } else if (u_proc < r_trap + r_ion_e + r_ion_h + r_iv) {
                    scatter_intervalley(L, c, rng);
                    st.intervalley_scatters++;
                } else if (r_luke > 0.0) {
                    const LukeEmit em = emit_luke(L, c, rng);
                    if (em.emitted) {
                        st.luke_emitted++;
                        st.luke_eV += em.e_ph * c.w;
                        if (luke_prob > 0.0 && (luke_prob >= 1.0 || rng.uniform() < luke_prob)) {
                            const int m = sample_dos_mode(L, rng);
                            ctx.push(make_track(L, c.pos, em.q_dir, m, em.e_ph, c.t, c.w * luke_wt_mult));
                        }
                    }
                }
            }
        }
    }
}

}  // namespace cmpmc_gpu
