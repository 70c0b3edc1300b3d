"""Parity of the plain FP64 device form with the reference CPU transport.

Bar (per event): hit count, every discrete hit field (surface, excitation, mode, channel)
and every integer SimStats counter identical; hit time, energy, incident energy and
position sums within 1e-9 relative.

Two oracles (tests/golden/make_golden.py): the unmodified reference built against glibc,
and the same reference whose transport uses a correctly rounded libm (oracle/ref_crlibm.hpp).
The device's transcendentals are correctly rounded, so it must agree with the second on
every event; against the glibc build it must agree on exactly the events where the two
references agree (glibc 2.39 is not correctly rounded, and the transport amplifies a
last-bit difference into a different trajectory on some events).
"""
import numpy as np
import pytest

from tests.helpers import WORKLOAD_SEED, detector_for, golden, lattice_for, workload_of
from tests.golden.records import FP_STATS, compare_summaries, summarize

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


def _run(ge_lattice, wl, n, keep_hits=True, want_event_stats=True, packed=None):
    import cmpmc_b200 as cm
    eng = cm.SimulationEngine(lattice_for(wl, ge_lattice), detector_for(wl))
    opt = cm.RunOptions(seed=WORKLOAD_SEED[wl], keep_hits=keep_hits, want_event_stats=want_event_stats)
    if packed is None:
        return eng, cm.run_events(eng, n, workload_of(wl), opt)
    return eng, eng.run_packed(packed, opt)


_RESULTS = {}


def _device_summary(ge_lattice, wl, n):
    if (wl, n) not in _RESULTS:
        _, res = _run(ge_lattice, wl, n)
        _RESULTS[(wl, n)] = summarize(res.event_stats, res.hit_offsets, res.hits)
    return _RESULTS[(wl, n)]


ALL_WL = ["c0", "c4", "c2", "tp", "tpl", "c1", "c3s", "c0m", "tpm", "c0a", "tpd", "tpe", "c0x", "c0b", "tp2",
          "c0r", "tps", "tpt", "pub", "pubc"]


@pytest.mark.parametrize("wl", ALL_WL)
def test_event_parity_correctly_rounded_reference(ge_lattice, wl):
    ref = golden(f"{wl}_cr_summary.npz")["summary"]
    got = _device_summary(ge_lattice, wl, len(ref))
    cmp = compare_summaries(ref, got, REL_TOL)
    print(wl, {k: v for k, v in cmp.items() if k != "agree_mask"})
    assert cmp["agree"] == cmp["n"], cmp
    for j, name in enumerate(FP_STATS):
        a, b = ref["fps"][:, j], got["fps"][:, j]
        assert np.all(np.abs(a - b) <= 1e-12 * np.maximum(np.abs(a), 1e-300) + 1e-300), name


@pytest.mark.parametrize("wl", ALL_WL)
def test_event_parity_glibc_reference(ge_lattice, wl):
    ref = golden(f"{wl}_summary.npz")["summary"]
    cr = golden(f"{wl}_cr_summary.npz")
    got = _device_summary(ge_lattice, wl, len(ref))
    cmp = compare_summaries(ref, got, REL_TOL)
    print(wl, f"device vs glibc reference: {100 * cmp['frac']:.2f}% of events agree "
              f"(libm floor {100 * float(cr['floor']):.2f}%)")
    assert np.array_equal(cmp["agree_mask"], cr["floor_mask"])
    if wl in ("c0", "c4"):
        assert cmp["frac"] >= 0.985
    if wl == "pub":  # the published benchmark workload: no libm-sensitive event in 2,000
        assert cmp["frac"] == 1.0


@pytest.mark.parametrize("wl", [w for w in ALL_WL if w != "c4"])
def test_full_hit_records_match(ge_lattice, wl):
    """Hit-by-hit comparison from the reference's own initial stacks and Rng states."""
    import cmpmc_b200 as cm
    g = golden(f"{wl}_cr_full.npz")
    n = len(g["rng_state"])
    packed = cm.PackedEvents(n, 0, g["rng_state"].copy(), g["injected"].copy(), g["phonon_offsets"].copy(),
                             g["phonons"].copy(), g["charge_offsets"].copy(), g["charges"].copy())
    _, res = _run(ge_lattice, wl, n, packed=packed)
    assert np.array_equal(res.hit_offsets, g["hit_offsets"])
    h, r = res.hits, g["hits"]
    for f in ("surface_id", "excitation", "mode", "channel_id"):
        assert np.array_equal(h[f], r[f]), f
    for f in ("time", "edep", "incident_energy"):
        np.testing.assert_allclose(h[f], r[f], rtol=REL_TOL, atol=0)
    np.testing.assert_allclose(h["pos"], r["pos"], rtol=REL_TOL, atol=1e-15)
    ev = g["events"]["stats"]
    for name in ev.dtype.names:
        if name in FP_STATS:
            np.testing.assert_allclose(res.event_stats[name], ev[name], rtol=1e-12, atol=1e-300)
        else:
            assert np.array_equal(res.event_stats[name], ev[name]), name


def test_rare_branches_are_exercised(ge_lattice):
    """The parity workloads of the opt-in branches really take them: roulette kills (c0r),
    trapping and trap ionisation (tpt), and the demo polynomial surfaces' specular and
    down-converting reflections (pub)."""
    got = {}
    for wl in ("c0r", "tpt", "pub"):
        ref = golden(f"{wl}_cr_summary.npz")["summary"]
        _, res = _run(ge_lattice, wl, len(ref))
        got[wl] = res.stats
    assert got["c0r"].killed_tracks > 0
    assert got["tpt"].charges_trapped > 0 and got["tpt"].trap_ionizations > 0
    assert got["pub"].surface_downconversions > 0


def test_run_totals_and_closure(ge_lattice):
    """Totals equal the sum of the per-event records; energy closes (tests/test_parallel.cpp:126-137
    and tests/test_engine_energy_closure.cpp:14-21 of the reference, closure 1e-9)."""
    ref = golden("c0_cr_summary.npz")["summary"]
    _, res = _run(ge_lattice, "c0", 2000)
    st = res.stats
    assert st.total_steps == int(ref["ints"][:2000, 0].sum())
    assert st.sensor_hits == len(res.hits)
    assert int(res.hit_offsets[-1]) == len(res.hits)
    assert len(res.hit_offsets) == 2001
    closure = abs(st.total_deposited_eV + st.escaped_or_killed_eV - st.total_injected_eV) / st.total_injected_eV
    assert closure < 1e-9


def test_keep_hits_false_same_statistics(ge_lattice):
    _, a = _run(ge_lattice, "tp", 203)
    _, b = _run(ge_lattice, "tp", 203, keep_hits=False)
    assert len(b.hits) == 0
    assert np.all(b.hit_offsets == 0)
    ra, rb = a.stats.record(), b.stats.record()
    assert ra.tobytes() == rb.tobytes()


def test_deterministic_across_runs_and_launch_shapes(ge_lattice):
    import cmpmc_b200 as cm
    eng, a = _run(ge_lattice, "c0", 3000)
    eng.configure(threads_per_block=64, blocks_per_sm=1)
    b = cm.run_events(eng, 3000, cm.workloads.single_l_origin, cm.RunOptions(seed=42, want_event_stats=True))
    assert a.hits.tobytes() == b.hits.tobytes()
    assert a.stats.record().tobytes() == b.stats.record().tobytes()
    assert a.event_stats.tobytes() == b.event_stats.tobytes()


def test_small_capacities_grow_and_rerun(ge_lattice):
    """A stack or hit buffer that is too small is detected on the device and the run is
    repeated with more room; the result is unchanged."""
    import cmpmc_b200 as cm
    eng, a = _run(ge_lattice, "tpl", 21)
    eng2 = cm.SimulationEngine(ge_lattice, detector_for("tpl"))
    eng2.configure(stack_capacity=2, hit_capacity=16)
    b = cm.run_events(eng2, 21, cm.workloads.test_parallel, cm.RunOptions(seed=77, want_event_stats=True))
    assert a.hits.tobytes() == b.hits.tobytes()
    assert a.event_stats.tobytes() == b.event_stats.tobytes()


def test_empty_and_python_generator(ge_lattice):
    import cmpmc_b200 as cm
    eng = cm.SimulationEngine(ge_lattice, cm.DetectorModel())
    r0 = cm.run_events(eng, 0, cm.workloads.single_l_origin, cm.RunOptions(seed=42))
    assert len(r0.hits) == 0 and len(r0.hit_offsets) == 1
    # events with nothing to transport
    r1 = cm.run_events(eng, 5, lambda inp: None, cm.RunOptions(seed=3))
    assert r1.stats.total_steps == 0 and len(r1.hit_offsets) == 6

    def gen(inp):
        inp.phonons.append(eng.make_track((0, 0, 0), inp.rng.isotropic_dir(), cm.PhononMode.L, 7.5e-3))
        inp.injected_eV += 7.5e-3

    a = cm.run_events(eng, 64, gen, cm.RunOptions(seed=42))
    b = cm.run_events(eng, 64, cm.workloads.single_l_origin, cm.RunOptions(seed=42))
    assert a.hits.tobytes() == b.hits.tobytes()
