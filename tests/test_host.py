"""CPU tests of the host side: library load and exports, RNG streams, lattice tables,
generators and guards, all against the reference's golden records. No device needed."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from tests.helpers import GOLDEN, ROOT, WORKLOAD_SEED, detector_for, golden, lattice_for, workload_of


def test_library_exports_every_declared_symbol(lib):
    header = open(os.path.join(ROOT, "include", "cmpmc_gpu.h")).read()
    declared = set(re.findall(r"^\s*(?:[a-z_0-9]+\s*\*?\s+)+\*?(cmpmc_[a-z_0-9]+)\s*\(", header, re.M))
    assert len(declared) >= 20
    for name in sorted(declared):
        assert hasattr(lib, name), name
    from cmpmc_b200 import _ffi
    assert set(_ffi.EXPORTED) <= declared


def test_rng_streams_match_reference():
    from cmpmc_b200 import Rng
    from cmpmc_b200 import _ffi
    lib = _ffi.load()
    ref = json.load(open(os.path.join(GOLDEN, "rng.json")))
    for key, rec in ref.items():
        seed, stream = (int(x) for x in key.split(":"))
        r = Rng.for_stream(seed, stream)
        assert r.s == rec["state"]
        st = (ctypes.c_uint64 * 4)()
        lib.cmpmc_rng_for_stream(seed, stream, st)
        assert list(st) == rec["state"]
        assert [r.next_u64() for _ in range(8)] == rec["u64"]
        for want in rec["uniform"]:
            assert r.uniform() == float.fromhex(want)
        for want in rec["iso"]:
            assert r.isotropic_dir() == tuple(float.fromhex(x) for x in want)
        normals = [(0, 0, -1), (0, 0, 1), (-0.6, -0.8, 0)]
        for i, want in enumerate(rec["lamb"]):
            assert r.lambertian_dir(normals[i % 3]) == tuple(float.fromhex(x) for x in want)
        assert Rng(12345).s == rec["seeded_12345"]
        # the native stream continues identically
        r2 = Rng.for_stream(seed, stream)
        st2 = (ctypes.c_uint64 * 4)(*r2.s)
        assert [lib.cmpmc_rng_next_u64(st2) for _ in range(8)] == rec["u64"]


def test_lattice_tables_bit_identical_to_reference(ge_lattice):
    import hashlib
    g = golden("lattice_ge.npz")
    t = ge_lattice.tables()
    assert hashlib.sha256(t["oct"].tobytes()).hexdigest() == str(g["oct_sha256"])
    assert np.array_equal(t["cdf_lt"], g["cdf_lt"])
    assert np.array_equal(t["cdf_tt"], g["cdf_tt"])
    assert np.array_equal(t["hv"], g["hv"])
    idx = g["sample_idx"]
    assert np.array_equal(t["oct"][:, idx[:, 0], idx[:, 1], :], g["sample"])


@pytest.mark.parametrize("wl", ["c0", "c1", "c2", "tp", "tpl", "c3s", "tpt", "pub", "pubc"])
def test_native_generators_match_reference(ge_lattice, wl):
    import cmpmc_b200 as cm
    g = golden(f"{wl}_full.npz")
    n = len(g["rng_state"])
    eng = cm.SimulationEngine(lattice_for(wl, ge_lattice), detector_for(wl))
    ev = eng.generate(workload_of(wl), n, WORKLOAD_SEED[wl], threads=2)
    assert np.array_equal(ev.rng_state, g["rng_state"])
    assert np.array_equal(ev.injected_eV, g["injected"])
    assert np.array_equal(ev.phonon_offsets, g["phonon_offsets"])
    assert np.array_equal(ev.charge_offsets, g["charge_offsets"])
    assert ev.phonons.tobytes() == g["phonons"].tobytes()
    assert ev.charges.tobytes() == g["charges"].tobytes()


def test_native_generator_summary_streams(ge_lattice):
    """Post-generator Rng states of all 10,000 single-phonon events (the event-stream
    handoff to the device)."""
    import cmpmc_b200 as cm
    s = golden("c0_summary.npz")
    eng = cm.SimulationEngine(ge_lattice, detector_for("c0"))
    ev = eng.generate(cm.workloads.single_l_origin, len(s["rng_state"]), 42)
    assert np.array_equal(ev.rng_state, s["rng_state"])
    assert np.array_equal(ev.injected_eV, s["injected"])


def test_recoil_generator_streams(ge_lattice):
    """EnergyPartition::partition_deposit restated on the host: the post-generator Rng
    state and deposit of all 64 light-recoil events equal the reference's."""
    import cmpmc_b200 as cm
    s = golden("c3s_summary.npz")
    eng = cm.SimulationEngine(ge_lattice, detector_for("c3s"))
    ev = eng.generate(cm.workloads.recoil_light, len(s["rng_state"]), 13)
    assert np.array_equal(ev.rng_state, s["rng_state"])
    assert np.array_equal(ev.injected_eV, s["injected"])
    # pairs: electron then hole at the same point, charge weight n_true / n_sampled >= 1
    ch = ev.charges
    assert len(ch) % 2 == 0 and np.all(ch["type"][0::2] == 1) and np.all(ch["type"][1::2] == 2)
    assert np.array_equal(ch["pos"][0::2], ch["pos"][1::2])
    assert np.all(ev.phonons["weight"] >= 1.0)


def test_recoil_generator_full_range_counts(ge_lattice):
    """Deposits up to 10 keV: pair counts within [1, 4096] sampled per event (weights
    above the cap), at most 5000 prompt phonons, offsets consistent, sizing call first."""
    import cmpmc_b200 as cm
    eng = cm.SimulationEngine(ge_lattice, cm.DetectorModel())
    ev = eng.generate(cm.workloads.recoil, 256, 13)
    n_ch = np.diff(ev.charge_offsets)
    n_ph = np.diff(ev.phonon_offsets)
    assert n_ch.max() <= 2 * 4096 and n_ph.max() <= 5000 and n_ph.min() >= 1
    pair_e = ev.injected_eV / np.maximum(n_ch // 2, 1)
    assert 0.5 < np.median(pair_e) < 6.0  # ~2.96 eV per pair in Ge
    # prompt phonon energy: deposit minus n_true pairs x (gap + 10 meV)
    w = ev.phonons["weight"]
    assert np.all(w >= 1.0)


def test_mesh_field_bit_identical_to_reference():
    """TriLinearMesh3D::build_cartesian_grid + field_at / potential_at of the recoil
    workloads' mesh: every field and potential at 4096 points equals the reference's,
    with the walk hint carried from point to point."""
    import ctypes as C
    from tests.helpers import recoil_mesh
    g = golden("mesh_c3.npz")
    m = recoil_mesh()
    assert m.num_vertices() == int(g["n_vertices"]) and m.num_tetrahedra() == int(g["n_tets"])
    he, hv = C.c_int32(0), C.c_int32(0)
    for i, p in enumerate(g["points"]):
        assert m.field_at(p, he) == tuple(g["field"][i]), i
        assert m.potential_at(p, hv) == g["potential"][i], i


def test_mesh_from_arrays_and_cartesian_builder_agree():
    """A user mesh given as arrays (the TriLinearMesh3D constructor) equals the Cartesian
    builder's; outside the hull the field is zero; a linear potential gives its exact
    gradient."""
    import cmpmc_b200 as cm
    n = 3
    xs = np.linspace(-1.0, 1.0, n + 1)
    fn = lambda p: 2.0 * p[0] - 3.0 * p[1] + 0.5 * p[2]  # noqa: E731
    a = cm.TriLinearMesh3D.build_cartesian_grid(1.0, 1.0, 1.0, n, n, n, fn)
    verts = np.array([(x, y, z) for x in xs for y in xs for z in xs])
    pots = np.array([fn(v) for v in verts])
    vid = lambda i, j, k: (i * (n + 1) + j) * (n + 1) + k  # noqa: E731
    tets = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                c = [vid(i + di, j + dj, k + dk) for di in (0, 1) for dj in (0, 1) for dk in (0, 1)]
                v000, v001, v010, v011, v100, v101, v110, v111 = c
                tets += [(v111, v000, v100, v110), (v000, v100, v101, v111), (v000, v010, v110, v111),
                         (v000, v010, v011, v111), (v000, v001, v101, v111), (v000, v001, v011, v111)]
    b = cm.TriLinearMesh3D(verts, pots, tets)
    assert a.num_tetrahedra() == b.num_tetrahedra() == 6 * n ** 3
    rng = np.random.default_rng(1)
    for p in rng.uniform(-0.99, 0.99, size=(200, 3)):
        ea, eb = a.field_at(p), b.field_at(p)
        assert ea == eb
        np.testing.assert_allclose(ea, (-2.0, 3.0, -0.5), rtol=1e-12, atol=1e-12)
        assert a.potential_at(p) == pytest.approx(fn(p), rel=1e-12, abs=1e-12)
    assert a.field_at((3.0, 0.0, 0.0)) == (0.0, 0.0, 0.0)


def test_mesh_load_from_files_matches_reference():
    """TriLinearMesh3D::load_from_files of an irregular (jittered) mesh in millimetres and
    millivolts with comment, blank and malformed lines: node and tetrahedron counts, and the
    field and potential at 2048 points equal the reference's bit for bit. Files that do not
    open give no lines (an empty mesh, as in the reference); tetrahedra whose nodes are
    missing are an error (the reference reads past its node table there)."""
    import ctypes as C
    import cmpmc_b200 as cm
    from tests.helpers import GOLDEN
    g = golden("mesh_files.npz")
    d = os.path.join(GOLDEN, "mesh_files")
    m = cm.TriLinearMesh3D.load_from_files(os.path.join(d, "nodes.txt"), os.path.join(d, "tets.txt"), 1e-3, 1e-3)
    assert m.num_vertices() == int(g["n_vertices"]) and m.num_tetrahedra() == int(g["n_tets"])
    he, hv = C.c_int32(0), C.c_int32(0)
    for i, p in enumerate(g["points"]):
        assert m.field_at(p, he) == tuple(g["field"][i]), i
        assert m.potential_at(p, hv) == g["potential"][i], i
    empty = cm.TriLinearMesh3D.load_from_files(os.path.join(d, "missing.txt"), os.path.join(d, "missing.txt"))
    assert empty.empty() and empty.num_vertices() == 0
    assert empty.field_at((0.0, 0.0, 0.0)) == (0.0, 0.0, 0.0)
    with pytest.raises(cm.CmpmcError):
        cm.TriLinearMesh3D.load_from_files(os.path.join(d, "missing.txt"), os.path.join(d, "tets.txt"))


def test_mesh2d_field_bit_identical_to_reference():
    """BiLinearMesh2D::build_grid + field_at / potential_at, axisymmetric (r, z) and planar
    (x, y): every field and potential at 4096 points (16 on the axis) equals the
    reference's, with one walk hint per mesh and query kind carried from point to point."""
    import ctypes as C
    import cmpmc_b200 as cm
    from tests.helpers import axisym_mesh, planar_mesh
    g = golden("mesh2d.npz")
    det = cm.DetectorModel()
    ax, pl = axisym_mesh(det), planar_mesh(det)
    assert ax.num_vertices() == int(g["axisym_vertices"]) and ax.num_triangles() == int(g["axisym_triangles"])
    assert pl.num_vertices() == int(g["planar_vertices"]) and pl.num_triangles() == int(g["planar_triangles"])
    h = [C.c_int32(0) for _ in range(4)]
    for i, p in enumerate(g["points"]):
        assert ax.field_at(p, h[0]) == tuple(g["axisym_field"][i]), i
        assert ax.potential_at(p, h[1]) == g["axisym_potential"][i], i
        assert pl.field_at(p, h[2]) == tuple(g["planar_field"][i]), i
        assert pl.potential_at(p, h[3]) == g["planar_potential"][i], i


def test_mesh2d_from_arrays_matches_grid_builder():
    """A user mesh given as arrays (the BiLinearMesh2D constructor, triangle nodes in any
    order) equals the grid builder's; a linear potential gives its exact gradient; the
    field is zero outside the hull and along the axis only E_z remains."""
    import cmpmc_b200 as cm
    n = 4
    fn = lambda u, v: 2.0 * u - 3.0 * v  # noqa: E731
    a = cm.BiLinearMesh2D.build_grid(0.0, 1.0, -1.0, 1.0, n, n, fn, True)
    us, vs = np.linspace(0.0, 1.0, n + 1), np.linspace(-1.0, 1.0, n + 1)
    verts = np.array([(u, v) for u in us for v in vs])
    vid = lambda i, j: i * (n + 1) + j  # noqa: E731
    tris = []
    for i in range(n):
        for j in range(n):
            tris += [(vid(i + 1, j + 1), vid(i + 1, j), vid(i, j)), (vid(i, j + 1), vid(i + 1, j + 1), vid(i, j))]
    b = cm.BiLinearMesh2D(verts, [fn(u, v) for u, v in verts], tris, axisymmetric_rz=True)
    assert a.num_triangles() == b.num_triangles() == 2 * n * n
    rng = np.random.default_rng(3)
    for p in rng.uniform(-0.7, 0.7, size=(200, 3)):
        ea, eb = a.field_at(p), b.field_at(p)
        assert ea == eb
        r = float(np.hypot(p[0], p[1]))
        np.testing.assert_allclose(ea, (-2.0 * p[0] / r, -2.0 * p[1] / r, 3.0), rtol=1e-12, atol=1e-12)
    assert a.field_at((0.0, 0.0, 0.3)) == pytest.approx((0.0, 0.0, 3.0), rel=1e-12)
    assert a.field_at((2.0, 0.0, 0.0)) == (0.0, 0.0, 0.0)
    planar = cm.BiLinearMesh2D.build_grid(-1.0, 1.0, -1.0, 1.0, n, n, fn, False)
    np.testing.assert_allclose(planar.field_at((0.3, -0.2, 5.0)), (-2.0, 3.0, 0.0), rtol=1e-12, atol=1e-12)


def test_electrode_masks_match_reference():
    """SuperCDMS QET preset with fill fraction 0.8 (find_channel drawing from the same
    stream as the reference) and a 4 x 4 rectangular pad grid at 4096 points of a face."""
    import cmpmc_b200 as cm
    g = golden("mask_channels.npz")
    R = cm.DetectorModel().solid.radius
    qet = cm.ElectrodePatternMask.supercdms_qet_mask(R, 0.8)
    grid = cm.ElectrodePatternMask.rectangular_grid_mask(4, 4, 1.5e-2, 1.5e-2, 0.6e-2, 0.5e-2)
    assert qet.num_pads() == 5 and grid.num_pads() == 16
    rng = cm.Rng.for_stream(9, 0)
    for i in range(len(g["x"])):
        x = (2.0 * rng.uniform() - 1.0) * R
        y = (2.0 * rng.uniform() - 1.0) * R
        assert (x, y) == (g["x"][i], g["y"][i])
        assert qet.find_channel((x, y, 0.0), rng) == g["qet"][i], i
        one = cm.Rng(1)
        assert grid.find_channel((x, y, 0.0), one) == g["grid"][i], i
    assert set(np.unique(g["qet"])) == {-1, 0, 1, 2, 3, 4}


def test_kaplan_surrogate_matches_reference():
    """KaplanSurrogateLUT of the default Al film (seed 1337): 2000 lookups over sub-gap,
    in-table and above-table energies equal the reference's (absorbed energy and every
    re-emitted energy), drawing from the same stream."""
    import cmpmc_b200 as cm
    g = golden("kaplan_surrogate.npz")
    film = cm.AluminumFilm()
    lut = cm.KaplanSurrogateLUT(film)
    rng = cm.Rng.for_stream(3, 0)
    off = 0
    for i in range(len(g["energy"])):
        E = film.gap_energy * (1.0 + 45.0 * rng.uniform())
        assert E == g["energy"][i]
        edep, refl = lut.absorb_phonon_fast(E, rng)
        k = int(g["n_refl"][i])
        assert edep == g["edep"][i], i
        assert refl == list(g["refl"][off:off + k]), i
        off += k


def test_amm_transmission_matches_reference():
    """IsotropicAMMInterface (Ge substrate -> Al film): the L and transverse transmission at
    400 incidence angles equal the reference's (phonon/interface_transmission.hpp:74-130)."""
    import cmpmc_b200 as cm
    g = golden("amm_transmission.npz")
    a = cm.IsotropicAMMInterface(cm.IsotropicMedium(5323.0, 5324.2077, 3258.7879),
                                 cm.IsotropicMedium(2700.0, 6420.0, 3040.0))
    n = len(g["longitudinal"])
    for i in range(n):
        c = (i + 0.5) / n
        assert a.transmission(True, c) == g["longitudinal"][i], i
        assert a.transmission(False, c) == g["transverse"][i], i
    # flux conservation holds in the reference's model: transmission within [0, 1]
    assert 0.0 <= g["longitudinal"].min() and g["transverse"].max() <= 1.0


def test_kinematics_modes_match_reference():
    """CrystalLattice::map_k_to_vg in the Exact (Cardano per call) and Bilinear (181 x 361
    table) modes: group-velocity directions and magnitudes of 1000 directions x 3 modes equal
    the reference's; the native generator's make_track follows the lattice's mode."""
    import cmpmc_b200 as cm
    g = golden("kinematics_modes.npz")
    rng = cm.Rng.for_stream(21, 0)
    ks = [rng.isotropic_dir() for _ in range(1000)]
    for mode, key in ((cm.CrystalLattice.Exact, "exact"), (cm.CrystalLattice.Bilinear, "bilinear")):
        lat = cm.CrystalLattice(cm.materials.Germanium())
        lat.set_kinematics_mode(mode)
        assert lat.kinematics_mode() == mode
        for i, k in enumerate(ks):
            for m in range(3):
                d, mag = lat.map_k_to_vg(m, k)
                assert tuple(d) + (mag,) == tuple(g[key][i, m]), (key, i, m)
    for wl in ("c0x", "c0b"):
        full = golden(f"{wl}_full.npz")
        lat = lattice_for(wl, None)
        eng = cm.SimulationEngine(lat, detector_for(wl))
        ev = eng.generate(workload_of(wl), len(full["rng_state"]), WORKLOAD_SEED[wl])
        assert ev.phonons.tobytes() == full["phonons"].tobytes(), wl


def test_python_generator_matches_native(ge_lattice):
    import cmpmc_b200 as cm
    det = detector_for("tp")
    eng = cm.SimulationEngine(ge_lattice, det)
    n_val = 4

    def gen(inp):  # tests/test_parallel.cpp:110-125 of the reference
        if inp.event_id % 2 == 0:
            inp.phonons.append(eng.make_track((0, 0, 0), inp.rng.isotropic_dir(), cm.PhononMode.FT, 7.5e-3))
            inp.injected_eV += 7.5e-3
        else:
            v = int(inp.rng.uniform() * n_val) % n_val
            inp.charges.append(eng.make_charge(cm.ExcitationType.Electron, (0, 0, 0), inp.rng.isotropic_dir(), 1e-6, v))
            inp.charges.append(eng.make_charge(cm.ExcitationType.Hole, (0, 0, 0), inp.rng.isotropic_dir(), 1e-6, 0))

    a = eng.generate_python(gen, 32, 77)
    g = golden("tp_full.npz")
    assert np.array_equal(a.rng_state, g["rng_state"])
    assert a.phonons.tobytes() == g["phonons"].tobytes()
    assert a.charges.tobytes() == g["charges"].tobytes()


def test_map_k_to_vg_host_closed_form(ge_lattice):
    """Along [100] of a cubic crystal the L group velocity is sqrt(C11/rho) and parallel to k
    (the table blend reproduces it to the table's interpolation error)."""
    import math
    import cmpmc_b200 as cm
    vg, mag = ge_lattice.map_k_to_vg(cm.PhononMode.L, (1.0, 0.0, 0.0))
    cfg = ge_lattice.config()
    assert abs(mag - math.sqrt(cfg.C11 / cfg.density)) / mag < 1e-3
    assert vg[0] > 0.9999  # the [100] direction sits on the octahedral fold (u = 1)


def test_demo_surfaces_are_guarded(ge_lattice):
    import cmpmc_b200 as cm
    det = cm.DetectorModel()
    det.surfaces = [cm.SurfaceProperty.demo_polynomial_sensor_surface(),
                    cm.SurfaceProperty.demo_polynomial_sensor_surface(),
                    cm.SurfaceProperty.demo_polynomial_bare_surface()]
    with pytest.raises(cm.UnvalidatedModuleError):
        cm.SimulationEngine(ge_lattice, det)
    det.allow_unvalidated = True
    cm.SimulationEngine(ge_lattice, det)


def test_no_device_fails_loudly(ge_lattice):
    """Without a GPU the device path raises; nothing falls back to a CPU implementation."""
    from tests.helpers import has_gpu
    import cmpmc_b200 as cm
    if has_gpu():
        pytest.skip("a device is present")
    eng = cm.SimulationEngine(ge_lattice, cm.DetectorModel())
    with pytest.raises(cm.CmpmcError):
        cm.run_events(eng, 4, cm.workloads.single_l_origin, cm.RunOptions(seed=42))


def test_noalloc_refuses_non_octahedral_lattice_before_device_work(lib):
    """The allocation-free entry stages only the octahedral table in its module array, so a
    lattice in the Exact or Bilinear mode is refused with CMPMC_ERR_INVALID before any CUDA
    call (without a device, an accepted lattice gets as far as selecting the device)."""
    import ctypes as C
    from tests.helpers import has_gpu
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    det = cm.DetectorModel().to_c()
    total, n_hits = _ffi.SimStatsC(), C.c_uint64(0)

    def call(lat):
        return lib.cmpmc_gpu_run_events_noalloc(lat._h, C.byref(det), 0, 0, None, None, None, None, None, None,
                                                None, 0, None, C.byref(total), C.byref(n_hits))

    for mode in (cm.CrystalLattice.Exact, cm.CrystalLattice.Bilinear):
        lat = cm.CrystalLattice(cm.materials.Germanium())
        lat.set_kinematics_mode(mode)
        assert call(lat) == _ffi.ERR_INVALID
    octa = cm.CrystalLattice(cm.materials.Germanium())
    assert call(octa) == (_ffi.OK if has_gpu() else _ffi.ERR_NO_DEVICE)
