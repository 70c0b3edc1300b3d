"""The batched FP32 form with charge carriers: FP32 drift, FP64 time and energy ledgers,
tracked Luke phonons through the device queue (charges_batched.cu).

Its events are not the reference's events (every carrier and every Luke phonon owns a
substream), so what must agree are the distributions:

* electron-hole pairs drifting in the uniform 4 V field (2,000 events, Luke phonons
  counted): per-event means of the charge counters, the Luke energy, the collected
  energy and the collection time against the reference, z < 4 (event = independent unit);
* light electron recoils in the tetrahedral-mesh field with Luke phonons tracked (64
  events): per-event differences to the same events of the reference (same deposit, same
  initial carriers), z < 4;
* the queue: a queue of 2,048 entries (hundreds of park / resume phases) gives the same
  counters and the same hits as the default queue, and two launch shapes agree.
"""
import numpy as np
import pytest

from tests.helpers import WORKLOAD_SEED, detector_for, golden, workload_of
from tests.golden.records import FP_STATS, INT_STATS, summarize

pytestmark = pytest.mark.gpu

Z_MAX = 4.0


def _col(summary, name):
    if name in INT_STATS:
        return summary["ints"][:, INT_STATS.index(name)].astype(np.float64)
    if name in FP_STATS:
        return summary["fps"][:, FP_STATS.index(name)].astype(np.float64)
    return summary[name].astype(np.float64)


def _run(ge_lattice, wl, n, eng=None, seed=None, **cfg):
    import cmpmc_b200 as cm
    eng = eng or cm.SimulationEngine(ge_lattice, detector_for(wl))
    if cfg:
        eng.configure(**cfg)
    packed = eng.generate(workload_of(wl), n, WORKLOAD_SEED[wl])
    opt = cm.RunOptions(seed=WORKLOAD_SEED[wl] if seed is None else seed, form="batched_fp32",
                        want_event_stats=True)
    return eng, eng.run_packed(packed, opt)


def test_pair_drift_batched_matches_reference(ge_lattice):
    ref = golden("c2_cr_summary.npz")["summary"]
    n = len(ref)
    _, res = _run(ge_lattice, "c2", n)
    got = summarize(res.event_stats, res.hit_offsets, res.hits)
    assert np.all(got["n_hits"] == 2) and np.all(_col(got, "charges_collected") == 2)
    assert np.all(res.hits["excitation"] > 0)
    for name in ("charge_steps", "luke_phonons_emitted", "intervalley_scatters", "charge_surface_refls",
                 "total_luke_phonon_eV", "charge_recomb_edep_eV", "sum_time"):
        a, b = _col(ref, name), _col(got, name)
        z = (b.mean() - a.mean()) / np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        print(f"{name}: reference {a.mean():.6g} batched {b.mean():.6g} z {z:.2f}")
        assert abs(z) < Z_MAX, (name, z)
    # totals are the sum of the per-event records
    assert res.stats.charge_steps == int(res.event_stats["charge_steps"].sum())
    assert int(res.hit_offsets[-1]) == len(res.hits) == 2 * n


def test_recoil_batched_matches_reference(ge_lattice):
    """Mesh field, weighted prompt phonons, 5 % of the Luke phonons tracked."""
    ref = golden("c3s_cr_summary.npz")["summary"]
    n = len(ref)
    seeds = (13, 101, 202, 303)
    runs = []
    for sd in seeds:
        _, res = _run(ge_lattice, "c3s", n, seed=sd)
        runs.append(summarize(res.event_stats, res.hit_offsets, res.hits))
        st = res.stats
        assert st.total_injected_eV == pytest.approx(float(golden("c3s_summary.npz")["injected"].sum()), rel=1e-12)
    for name in ("n_hits", "charge_steps", "luke_phonons_emitted", "charges_collected", "total_steps",
                 "total_deposited_eV", "total_luke_phonon_eV", "charge_recomb_edep_eV", "sum_edep"):
        a = _col(ref, name)
        b = np.mean([_col(r, name) for r in runs], axis=0)
        d = b - a  # same events: paired differences
        if d.std(ddof=1) == 0.0:  # e.g. every carrier collected in both
            assert d.mean() == 0.0, name
            continue
        z = d.mean() / (d.std(ddof=1) / np.sqrt(n))
        print(f"{name}: reference {a.mean():.6g} batched {b.mean():.6g} z {z:.2f}")
        assert abs(z) < Z_MAX, (name, z)


def test_axisymmetric_mesh_batched_matches_reference(ge_lattice):
    """The mixed workload in the field of an axisymmetric BiLinearMesh2D (FP32 edge walk,
    the field rotated back around the axis): per-event differences to the same events of
    the reference, averaged over four seeds, z < 4."""
    ref = golden("tp2_cr_summary.npz")["summary"]
    n = len(ref)
    runs = []
    for sd in (77, 1077, 2077, 3077):
        _, res = _run(ge_lattice, "tp2", n, seed=sd)
        runs.append(summarize(res.event_stats, res.hit_offsets, res.hits))
    for name in ("n_hits", "charge_steps", "luke_phonons_emitted", "charges_collected", "total_luke_phonon_eV",
                 "charge_surface_refls", "sum_time", "sum_edep"):
        a = _col(ref, name)
        b = np.mean([_col(r, name) for r in runs], axis=0)
        d = b - a
        if d.std(ddof=1) == 0.0:
            assert d.mean() == 0.0, name
            continue
        z = d.mean() / (d.std(ddof=1) / np.sqrt(n))
        print(f"{name}: reference {a.mean():.6g} batched {b.mean():.6g} z {z:.2f}")
        assert abs(z) < Z_MAX, (name, z)


def test_queue_phases_reproduce_the_same_hits(ge_lattice):
    import cmpmc_b200 as cm
    eng, a = _run(ge_lattice, "c3s", 16)
    eng2 = cm.SimulationEngine(ge_lattice, detector_for("c3s"))
    _, b = _run(ge_lattice, "c3s", 16, eng=eng2, queue_capacity=2048, threads_per_block=64, blocks_per_sm=2)
    ea, eb = a.event_stats, b.event_stats
    for name in INT_STATS:
        assert np.array_equal(ea[name], eb[name]), name
    for name in FP_STATS:
        np.testing.assert_allclose(ea[name], eb[name], rtol=1e-12, atol=1e-300)
    assert np.array_equal(a.hit_offsets, b.hit_offsets)
    for i in range(16):
        lo, hi = int(a.hit_offsets[i]), int(a.hit_offsets[i + 1])
        ha, hb = np.sort(a.hits[lo:hi], order=["time", "edep"]), np.sort(b.hits[lo:hi], order=["time", "edep"])
        assert ha.tobytes() == hb.tobytes(), i
    assert a.stats.luke_phonons_emitted > 0 and a.stats.sensor_hits > 0


@pytest.mark.parametrize("wl", ["tpd", "tpe"])
def test_charge_release_batched_matches_plain(ge_lattice, wl):
    """BulkDebye (tpd) and ElectrodeFilm (tpe) charge release in the batched charge form (a
    release phase per round: Debye phonons, or photon-seeded film cascades whose escaping
    phonons re-enter the crystal) against the plain FP64 form, which is identical to the
    reference event by event: per-event means of the hits, the collected carriers, the
    recombination, deposited and escaped energy and the steps agree, z < 4 (independent
    samples). (The field does work on the carriers, so these events have no closed ledger.)"""
    import cmpmc_b200 as cm
    n = 2000
    eng = cm.SimulationEngine(ge_lattice, detector_for(wl))
    packed = eng.generate(workload_of(wl), n, WORKLOAD_SEED[wl])
    plain = eng.run_packed(packed, cm.RunOptions(seed=WORKLOAD_SEED[wl], want_event_stats=True))
    _, bat = _run(ge_lattice, wl, n, eng=eng)
    ps = summarize(plain.event_stats, plain.hit_offsets, plain.hits)
    bs = summarize(bat.event_stats, bat.hit_offsets, bat.hits)
    for name in ("n_hits", "charges_collected", "charge_recomb_edep_eV", "total_deposited_eV", "escaped_or_killed_eV",
                 "total_steps", "luke_phonons_emitted", "sum_edep"):
        a, b = _col(ps, name), _col(bs, name)
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        if se == 0.0:
            assert a.mean() == b.mean(), name
            continue
        z = (b.mean() - a.mean()) / se
        print(f"{wl} {name}: plain {a.mean():.6g} batched {b.mean():.6g} z {z:.2f}")
        assert abs(z) < Z_MAX, (name, z)
    if wl == "tpd":  # every collected carrier's energy becomes phonons: the collection hits carry none
        assert np.all(bat.hits["edep"][bat.hits["excitation"] > 0] == 0.0)


def test_release_queue_grows_on_overflow(ge_lattice):
    """A phonon queue too small for the released phonons is enlarged and the call rerun."""
    import cmpmc_b200 as cm
    eng = cm.SimulationEngine(ge_lattice, detector_for("tpe"))
    eng.configure(queue_capacity=64)
    packed = eng.generate(workload_of("tpe"), 64, WORKLOAD_SEED["tpe"])
    res = eng.run_packed(packed, cm.RunOptions(seed=5, form="batched_fp32", want_event_stats=True))
    assert res.stats.charges_collected == int(res.event_stats["charges_collected"].sum()) > 0
