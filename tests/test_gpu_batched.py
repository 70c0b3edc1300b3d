"""The batched FP32 form: statistical parity with the FP64 reference.

The batched form gives every primary phonon its own random substream, so its events are
not the reference's events; what must agree are the distributions. Bar: chi^2 p > 0.01 for
the hit time (256 bins, 0-2 ms), radial position (64 bins) and energy (64 bins) histograms
against the reference (mixed-energy workload, 200,000 primaries) and against the plain
FP64 device form, and energy-ledger closure |injected - deposited - escaped| / injected
<= 1e-6. The chi^2 treats an event as the independent unit (tests/golden/records.py).
"""
import numpy as np
import pytest

from tests.helpers import WORKLOAD_SEED, detector_for, golden, workload_of
from tests.golden.records import event_histograms, hist_chi2

pytestmark = pytest.mark.gpu

P_MIN = 0.01
LEDGER_TOL = 1e-6


def _engine(ge_lattice, wl):
    import cmpmc_b200 as cm
    return cm.SimulationEngine(ge_lattice, detector_for(wl))


def _batched(eng, wl, n, seed=None, want_event_stats=False):
    import cmpmc_b200 as cm
    opt = cm.RunOptions(seed=WORKLOAD_SEED[wl], form="batched_fp32", want_event_stats=want_event_stats)
    packed = eng.generate(workload_of(wl), n, WORKLOAD_SEED[wl])
    if seed is not None:
        opt.seed = seed
    return eng.run_packed(packed, opt)


@pytest.fixture(scope="module")
def c1_batched(ge_lattice):
    eng = _engine(ge_lattice, "c1")
    return _batched(eng, "c1", 2000, want_event_stats=True)


def test_batched_histograms_match_reference(c1_batched):
    ref = dict(golden("c1_hist.npz"))
    got = event_histograms(c1_batched.hit_offsets, c1_batched.hits, tuple(ref["edep_range"]))
    for name in ("time", "radius", "edep"):
        c2, dof, p = hist_chi2(ref, got, name)
        print(f"{name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    n_ref, n_got = int(ref["n_hits"]), len(c1_batched.hits)
    assert abs(n_got - n_ref) / n_ref < 0.01


def test_batched_ledger_closes(c1_batched):
    st = c1_batched.stats
    inj = st.total_injected_eV
    assert abs(inj - st.total_deposited_eV - st.escaped_or_killed_eV) / inj <= LEDGER_TOL
    ref = golden("c1_hist.npz")
    assert abs(inj - float(ref["injected"])) / inj < 1e-12  # same generator, same primaries
    # deposited fraction agrees with the reference at the 1% level
    assert abs(st.total_deposited_eV / inj - float(ref["deposited"]) / float(ref["injected"])) < 0.01


def test_batched_event_bookkeeping(c1_batched):
    r = c1_batched
    assert len(r.hit_offsets) == 2001
    assert int(r.hit_offsets[-1]) == len(r.hits)
    assert np.all(np.diff(r.hit_offsets.astype(np.int64)) >= 0)
    ev = r.event_stats
    assert int(ev["total_steps"].sum()) == r.stats.total_steps
    assert int(ev["sensor_hits"].sum()) == len(r.hits)
    assert np.array_equal(np.diff(r.hit_offsets.astype(np.int64)), ev["sensor_hits"].astype(np.int64))
    np.testing.assert_allclose(ev["total_injected_eV"].sum(), r.stats.total_injected_eV, rtol=1e-12)


def test_batched_matches_plain_fp64_statistics(ge_lattice):
    """Single 7.5 meV L phonons in the volume: batched FP32 vs plain FP64 on the device."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c4")
    n = 20000
    plain = cm.run_events(eng, n, workload_of("c4"), cm.RunOptions(seed=17))
    batched = _batched(eng, "c4", n)
    lo = min(plain.hits["edep"].min(), batched.hits["edep"].min())
    hi = max(plain.hits["edep"].max(), batched.hits["edep"].max()) * (1 + 1e-9)
    a = event_histograms(plain.hit_offsets, plain.hits, (lo, hi))
    b = event_histograms(batched.hit_offsets, batched.hits, (lo, hi))
    for name in ("time", "radius", "edep"):
        c2, dof, p = hist_chi2(a, b, name)
        print(f"{name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    sp, sb = plain.stats, batched.stats
    for st in (sp, sb):
        assert abs(st.total_injected_eV - st.total_deposited_eV - st.escaped_or_killed_eV) / st.total_injected_eV < 1e-9
    # mean steps per primary within 2 %
    assert abs(sb.total_steps / sp.total_steps - 1.0) < 0.02


def _sorted_event_hits(res):
    out = []
    for i in range(len(res.hit_offsets) - 1):
        lo, hi = int(res.hit_offsets[i]), int(res.hit_offsets[i + 1])
        out.append(np.sort(res.hits[lo:hi], order=["time", "edep", "incident_energy"]).tobytes())
    return out


def test_batched_deterministic(ge_lattice):
    """The wavefront-split form: every unit owns its substream, so the hits of each event (as
    a set) and every integer counter are the same for any launch shape and queue size; the
    inline form also keeps the hit order."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c1")
    a = _batched(eng, "c1", 100, want_event_stats=True)
    eng2 = _engine(ge_lattice, "c1")
    eng2.configure(threads_per_block=64, blocks_per_sm=2, queue_capacity=4096)
    b = _batched(eng2, "c1", 100, want_event_stats=True)
    assert np.array_equal(a.hit_offsets, b.hit_offsets)
    assert _sorted_event_hits(a) == _sorted_event_hits(b)
    for name in a.event_stats.dtype.names:
        if a.event_stats.dtype[name].kind == "u":
            assert np.array_equal(a.event_stats[name], b.event_stats[name]), name
        else:
            np.testing.assert_allclose(a.event_stats[name], b.event_stats[name], rtol=1e-12, atol=1e-300)
    c = _batched(eng, "c1", 100, seed=12345)
    assert _sorted_event_hits(a) != _sorted_event_hits(c)
    packed = eng.generate(workload_of("c1"), 100, 7)
    i1 = eng.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32_inline"))
    i2 = eng2.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32_inline"))
    assert i1.hits.tobytes() == i2.hits.tobytes()
    assert i1.stats.record().tobytes() == i2.stats.record().tobytes()


def test_batched_inline_and_split_forms_agree(ge_lattice):
    """The two batched forms sample the same physics with different substream layouts:
    hit histograms chi^2 p > 0.01, both ledgers close."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c1")
    packed = eng.generate(workload_of("c1"), 2000, 7)
    s = eng.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32"))
    i = eng.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32_inline"))
    lo = min(s.hits["edep"].min(), i.hits["edep"].min())
    hi = max(s.hits["edep"].max(), i.hits["edep"].max()) * (1 + 1e-9)
    hs, hi_ = event_histograms(s.hit_offsets, s.hits, (lo, hi)), event_histograms(i.hit_offsets, i.hits, (lo, hi))
    for name in ("time", "radius", "edep"):
        c2, dof, p = hist_chi2(hs, hi_, name)
        print(f"split vs inline {name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    for st in (s.stats, i.stats):
        assert abs(st.total_injected_eV - st.total_deposited_eV - st.escaped_or_killed_eV) / st.total_injected_eV <= LEDGER_TOL


def test_batched_electrode_mask_channels(ge_lattice):
    """SuperCDMS QET masks (fill 0.8) on both faces: the per-event channel histogram of the
    batched form against the plain FP64 form (itself identical to the reference event by
    event), chi^2 p > 0.01; bare crystal between pads records no film hit."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c0m")
    n = 4000
    plain = cm.run_events(eng, n, workload_of("c0m"), cm.RunOptions(seed=42))
    batched = _batched(eng, "c0m", n)

    def per_event(res):
        ev = np.repeat(np.arange(n), np.diff(res.hit_offsets.astype(np.int64)))
        ch = res.hits["channel_id"].astype(np.int64)
        assert ch.min() >= 0 and ch.max() <= 4  # film hits only on pads
        counts = np.zeros((n, 5))
        np.add.at(counts, (ev, ch), 1.0)
        return {"n_events": n, "ch_sum": counts.sum(axis=0), "ch_sumsq": (counts ** 2).sum(axis=0)}

    c2, dof, p = hist_chi2(per_event(plain), per_event(batched), "ch")
    print(f"channels: chi2 {c2:.1f} dof {dof} p {p:.3f}")
    assert p > P_MIN


def test_batched_kaplan_surrogate_statistics(ge_lattice):
    """Film cascades from the KaplanSurrogateLUT table (kaplan_film.hpp:336-383) in the
    batched form against the reference's full-cascade transport: hit time and radius
    histograms chi^2 p > 0.01, deposited fraction within 3 % (the reference's own bar for
    the surrogate, tests/test_kaplan.cpp:95-107), and the ledger still closes. The per-hit
    energy spectrum is not compared: a stored outcome is rescaled from the nearest of 128
    energy nodes, which reshapes the edep histogram by design."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c1")
    packed = eng.generate(workload_of("c1"), 2000, WORKLOAD_SEED["c1"])
    res = eng.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32", kaplan_surrogate=True))
    ref = dict(golden("c1_hist.npz"))
    got = event_histograms(res.hit_offsets, res.hits, tuple(ref["edep_range"]))
    for name in ("time", "radius"):
        c2, dof, p = hist_chi2(ref, got, name)
        print(f"surrogate {name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    st = res.stats
    inj = st.total_injected_eV
    assert abs(inj - st.total_deposited_eV - st.escaped_or_killed_eV) / inj <= LEDGER_TOL
    frac_ref = float(ref["deposited"]) / float(ref["injected"])
    print(f"deposited fraction: surrogate {st.total_deposited_eV / inj:.5f} reference {frac_ref:.5f}")
    assert abs(st.total_deposited_eV / inj / frac_ref - 1.0) < 0.03


def test_batched_amm_interface_statistics(ge_lattice):
    """Ge -> Al acoustic-mismatch film entry (IsotropicAMMInterface) in the batched form
    against the plain FP64 form (identical to the reference event by event): hit
    histograms chi^2 p > 0.01 and the same deposited fraction within 1 %."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c0a")
    n = 4000
    plain = cm.run_events(eng, n, workload_of("c0a"), cm.RunOptions(seed=42))
    batched = _batched(eng, "c0a", n)
    lo = min(plain.hits["edep"].min(), batched.hits["edep"].min())
    hi = max(plain.hits["edep"].max(), batched.hits["edep"].max()) * (1 + 1e-9)
    a = event_histograms(plain.hit_offsets, plain.hits, (lo, hi))
    b = event_histograms(batched.hit_offsets, batched.hits, (lo, hi))
    for name in ("time", "radius", "edep"):
        c2, dof, p = hist_chi2(a, b, name)
        print(f"AMM {name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    fa = plain.stats.total_deposited_eV / plain.stats.total_injected_eV
    fb = batched.stats.total_deposited_eV / batched.stats.total_injected_eV
    assert abs(fb / fa - 1.0) < 0.01


@pytest.mark.parametrize("wl,n", [("c0x", 1000), ("c0b", 2000)])
def test_batched_kinematics_modes_statistics(ge_lattice, wl, n):
    """Exact (Cardano solve per call) and Bilinear kinematics in the batched form (the FP64
    maps out of line, rounded to FP32) against the plain FP64 form (identical to the
    reference event by event): hit histograms chi^2 p > 0.01 and the same deposited fraction
    within 1 %; the ledger closes."""
    import cmpmc_b200 as cm
    from tests.helpers import lattice_for
    eng = cm.SimulationEngine(lattice_for(wl, ge_lattice), detector_for(wl))
    plain = cm.run_events(eng, n, workload_of(wl), cm.RunOptions(seed=WORKLOAD_SEED[wl]))
    batched = _batched(eng, wl, n)
    lo = min(plain.hits["edep"].min(), batched.hits["edep"].min())
    hi = max(plain.hits["edep"].max(), batched.hits["edep"].max()) * (1 + 1e-9)
    a = event_histograms(plain.hit_offsets, plain.hits, (lo, hi))
    b = event_histograms(batched.hit_offsets, batched.hits, (lo, hi))
    for name in ("time", "radius", "edep"):
        c2, dof, p = hist_chi2(a, b, name)
        print(f"{wl} {name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    fa = plain.stats.total_deposited_eV / plain.stats.total_injected_eV
    fb = batched.stats.total_deposited_eV / batched.stats.total_injected_eV
    assert abs(fb / fa - 1.0) < 0.01
    st = batched.stats
    assert abs(st.total_injected_eV - st.total_deposited_eV - st.escaped_or_killed_eV) <= \
        LEDGER_TOL * st.total_injected_eV
    # the surrogate tables are built for the octahedral kinematics only
    with pytest.raises(cm.CmpmcError):
        eng.run_packed(eng.generate(workload_of(wl), 8, WORKLOAD_SEED[wl]),
                       cm.RunOptions(seed=1, form="batched_fp32", kaplan_surrogate=True))


def test_pool_and_host_driven_rounds_agree(ge_lattice):
    """The SM-phase pool (one persistent launch) and the host-driven film / transport rounds
    sample the same process (a daughter's substream differs between them): hit histograms
    chi^2 p > 0.01 on 2,000 mixed-energy events, the same deposited fraction within 1 %,
    both ledgers closed."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c1")
    packed = eng.generate(workload_of("c1"), 2000, 7)
    a = eng.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32"))
    eng2 = _engine(ge_lattice, "c1")
    eng2.configure_pool(0)
    b = eng2.run_packed(packed, cm.RunOptions(seed=7, form="batched_fp32"))
    assert a.kernel_launches < b.kernel_launches  # one transport launch against the rounds
    lo = min(a.hits["edep"].min(), b.hits["edep"].min())
    hi = max(a.hits["edep"].max(), b.hits["edep"].max()) * (1 + 1e-9)
    ha, hb = event_histograms(a.hit_offsets, a.hits, (lo, hi)), event_histograms(b.hit_offsets, b.hits, (lo, hi))
    for name in ("time", "radius", "edep"):
        c2, dof, p = hist_chi2(ha, hb, name)
        print(f"pool vs rounds {name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
        assert p > P_MIN, (name, c2, dof, p)
    for st in (a.stats, b.stats):
        assert abs(st.total_injected_eV - st.total_deposited_eV - st.escaped_or_killed_eV) / st.total_injected_eV <= LEDGER_TOL
    fa = a.stats.total_deposited_eV / a.stats.total_injected_eV
    fb = b.stats.total_deposited_eV / b.stats.total_injected_eV
    assert abs(fa / fb - 1.0) < 0.01


@pytest.mark.parametrize("form,ring", [(1, 64), (2, 64), (2, 0)])
def test_pool_forms_give_the_same_hits(ge_lattice, form, ring):
    """The two pool forms run the same step on the same substreams (a daughter's, a film
    entry's and a re-emission's keys are drawn at the same points), so the SM-phase pool and
    the warp pool give every event the same hits (as a set) and the same integer counters;
    so does a pool whose ring is too small (it overflows on the device, and the call grows it
    and reruns)."""
    eng = _engine(ge_lattice, "c1")
    a = _batched(eng, "c1", 300, want_event_stats=True)
    eng2 = _engine(ge_lattice, "c1")
    eng2.configure_pool(form, ring_capacity=ring)
    b = _batched(eng2, "c1", 300, want_event_stats=True)
    assert np.array_equal(a.hit_offsets, b.hit_offsets)
    assert _sorted_event_hits(a) == _sorted_event_hits(b)
    for name in a.event_stats.dtype.names:
        if a.event_stats.dtype[name].kind == "u":
            assert np.array_equal(a.event_stats[name], b.event_stats[name]), name


@pytest.mark.parametrize("wl,n", [("c1", 2000), ("c0x", 1000), ("c0m", 1000)])
def test_fp64_pool_statistics(ge_lattice, wl, n):
    """Pool form 3 (the SM-phase pool computed in FP64 throughout, on the FP32 pool's
    substreams) against the plain FP64 form (identical to the reference event by event) on
    the mixed-energy, Exact-kinematics and electrode-mask workloads, and against the FP32
    pool: hit histograms chi^2 p > 0.01, the same deposited fraction within 1 %, the ledgers
    closed."""
    import cmpmc_b200 as cm
    from tests.helpers import lattice_for
    eng = cm.SimulationEngine(lattice_for(wl, ge_lattice), detector_for(wl))
    plain = cm.run_events(eng, n, workload_of(wl), cm.RunOptions(seed=WORKLOAD_SEED[wl]))
    f32 = _batched(eng, wl, n)
    eng64 = cm.SimulationEngine(lattice_for(wl, ge_lattice), detector_for(wl))
    eng64.configure_pool(3)
    f64 = _batched(eng64, wl, n)
    lo = min(r.hits["edep"].min() for r in (plain, f32, f64))
    hi = max(r.hits["edep"].max() for r in (plain, f32, f64)) * (1 + 1e-9)
    h = {k: event_histograms(r.hit_offsets, r.hits, (lo, hi)) for k, r in
         (("plain", plain), ("f32", f32), ("f64", f64))}
    for other in ("plain", "f32"):
        for name in ("time", "radius", "edep"):
            c2, dof, p = hist_chi2(h["f64"], h[other], name)
            print(f"{wl} fp64 pool vs {other} {name}: chi2 {c2:.1f} dof {dof} p {p:.3f}")
            assert p > P_MIN, (other, name, c2, dof, p)
    for st in (f32.stats, f64.stats):
        assert abs(st.total_injected_eV - st.total_deposited_eV - st.escaped_or_killed_eV) <= \
            LEDGER_TOL * st.total_injected_eV
    fp = plain.stats.total_deposited_eV / plain.stats.total_injected_eV
    f6 = f64.stats.total_deposited_eV / f64.stats.total_injected_eV
    assert abs(f6 / fp - 1.0) < 0.01
    assert f64.stats.total_injected_eV == f32.stats.total_injected_eV


def test_fp64_pool_refuses_charges_and_the_surrogate(ge_lattice):
    """The FP64 pool form runs phonon-only batches with full film cascades: a batch with
    charges and a surrogate run are refused with an error, not run in another form."""
    import cmpmc_b200 as cm
    eng = _engine(ge_lattice, "c2")
    eng.configure_pool(3)
    with pytest.raises(cm.CmpmcError):
        _batched(eng, "c2", 4)
    eng = _engine(ge_lattice, "c1")
    eng.configure_pool(3)
    with pytest.raises(cm.CmpmcError):
        eng.run_packed(eng.generate(workload_of("c1"), 8, 7),
                       cm.RunOptions(seed=1, form="batched_fp32", kaplan_surrogate=True))
    eng.run_packed(eng.generate(workload_of("c1"), 8, 7), cm.RunOptions(seed=1, form="batched_fp32"))
