"""CPU tests of the input side (partition_host.cpp): ionisation yields, partition_deposit
and HitMerger against the reference's own outputs (tests/golden/partition.npz, written by
oracle/ref_driver.cpp `yield`, `partition` and `merge`). Everything is compared bit for
bit, including the position of the random stream after each call."""
import dataclasses
import hashlib

import numpy as np
import pytest

from tests.helpers import golden


@pytest.fixture(scope="module")
def g():
    return golden("partition.npz")


@pytest.fixture(scope="module")
def lattice():
    import cmpmc_b200 as cm
    return cm.CrystalLattice(cm.materials.Germanium())


def test_ionization_yields_match_reference(g):
    """niel_models.hpp:43-176: the five models at 400 energies from 1 eV to 10 MeV for Ge
    and Si (Z 14, A 28.085), Empirical with a fixed k, and Lindhard with a projectile."""
    import cmpmc_b200 as cm
    ge = cm.materials.Germanium()
    si = dataclasses.replace(ge, atomic_Z=14.0, atomic_A=28.085)
    E = 10.0 ** (7.0 * np.arange(400) / 399.0)
    fixed = cm.EmpiricalNIELParams(energy_dependent_k=False)
    part = cm.EnergyPartition(cm.CrystalLattice(ge))
    for c, cfg in enumerate((ge, si)):
        for col in range(7):
            for i, e in enumerate(E):
                e = float(10.0 ** (7.0 * i / 399.0))
                if col < 5:
                    y = cm.physics.compute_ionization_yield(cm.NIELModel(col), e, cfg)
                elif col == 5:
                    y = cm.physics.compute_ionization_yield(cm.NIELModel.Empirical, e, cfg, fixed)
                else:
                    y = cm.physics.lindhard_ionization_yield(e, cfg, 2.0, 4.0) if c == 1 else \
                        part.lindhard_ionization_yield(e, 2.0, 4.0)
                assert y == g["yields"][c, col, i], (c, col, i, y, g["yields"][c, col, i])


def _case_options(i):
    import cmpmc_b200 as cm
    o = cm.PartitionOptions(max_sampled_pairs=100, max_sampled_phonons=150)
    if i % 4 == 1:
        o.use_fano_fluctuations = False
    if i % 4 == 2:
        o.use_charge_cloud = False
        o.max_sampled_pairs = 16
    if i % 4 == 3:
        o.niel_model = cm.NIELModel.Empirical
        o.max_sampled_phonons = 7
    return o


def test_partition_deposit_matches_reference(g, lattice):
    """energy_partition.hpp:78-167 for 48 deposits of 10 eV-100 keV (electron and nuclear
    recoils, Fano on / off, charge cloud on / off, sampling caps): the Result, the carrier and
    phonon records and the stream position equal the reference's."""
    import cmpmc_b200 as cm
    part = cm.EnergyPartition(lattice)
    res = g["results"]
    off_c = off_p = 0
    for i in range(48):
        rng = cm.Rng.for_stream(8, i)
        r, ch, ph = part.partition_deposit((1e-3 * i, -2e-3, 3e-3), 1e-9 * i, 10.0 ** (1.0 + 4.0 * i / 47.0),
                                           i % 2 == 1, rng, _case_options(i))
        for name in res.dtype.names:
            assert getattr(r, name) == res[i][name], (i, name, getattr(r, name), res[i][name])
        assert len(ch) == int(g["n_charges"][i]) and len(ph) == int(g["n_phonons"][i]), i
        assert hashlib.sha256(ch.tobytes()).hexdigest() == str(g["sha_charges"][i]), i
        assert hashlib.sha256(ph.tobytes()).hexdigest() == str(g["sha_phonons"][i]), i
        if i < 12:
            assert ch.tobytes() == g["charges_0_11"][off_c:off_c + 128 * len(ch)].tobytes(), i
            assert ph.tobytes() == g["phonons_0_11"][off_p:off_p + 128 * len(ph)].tobytes(), i
            off_c += 128 * len(ch)
            off_p += 128 * len(ph)
        assert rng.next_u64() == int(g["next_u64"][i]), i
    # carriers are e-/h+ pairs with the shared weight; nuclear recoils keep part of the energy
    assert res["lindhard_yield"][1::2].max() < 1.0 and np.all(res["lindhard_yield"][0::2] == 1.0)


def _merge_steps():
    """The synthetic primary tracks of oracle/ref_driver.cpp `merge`."""
    import cmpmc_b200 as cm
    steps = []
    for t in range(3):
        p = (-5e-3 + 4e-3 * t, 1e-3 * t, -4e-3)
        for k in range(12):
            start = p
            ln = 1e-4 * (2 + (k * 7 + t * 3) % 6)
            p = (p[0] + 0.6 * ln, p[1] + 0.3 * ln, p[2] + 0.74161984870956632 * ln)
            steps.append(cm.PrimaryStepInput(
                track_id=t + 1, start_pos=start, end_pos=p, time_s=1e-12 * (10 * t + k),
                edep_eV=20.0 * (k % 3) if t == 2 else 40.0 + 15.0 * ((k * 5 + t) % 7),
                eniel_eV=300.0 + 50.0 * (k % 4) if t == 2 else 0.0, is_charged=(t != 1),
                hit_boundary=(k == 7 and t == 0), track_stopped=(k == 11)))
    return steps


def test_hit_merger_matches_reference(g, lattice):
    """energy_partition.hpp:229-323: a charged, a neutral and a nuclear-recoil-like track of
    12 steps through HitMerger(1 mm): the flush flags per step, the final flush's Result, all
    merged records (positions spread along the chords) and the stream position."""
    import cmpmc_b200 as cm
    m = cm.HitMerger(lattice, 1.0 * cm.units.mm, cm.PartitionOptions(max_sampled_pairs=64, max_sampled_phonons=64))
    rng = cm.Rng.for_stream(9, 0)
    flags = [m.process_step(s, rng) for s in _merge_steps()]
    assert flags == [bool(f) for f in g["merge_flags"]]
    r = m.flush(rng)
    want = g["merge_result"][0]
    for name in want.dtype.names:
        assert getattr(r, name) == want[name], name
    ch, ph = m.take()
    assert ch.tobytes() == g["merge_charges"].tobytes()
    assert ph.tobytes() == g["merge_phonons"].tobytes()
    assert rng.next_u64() == int(g["merge_next_u64"])
    # the batch entry point gives the same records; take() empties the merger
    m2 = cm.HitMerger(lattice, 1.0 * cm.units.mm, cm.PartitionOptions(max_sampled_pairs=64, max_sampled_phonons=64))
    rng2 = cm.Rng.for_stream(9, 0)
    assert m2.process_steps(_merge_steps(), rng2) == sum(flags)
    m2.flush(rng2)
    ch2, ph2 = m2.take()
    assert ch2.tobytes() == ch.tobytes() and ph2.tobytes() == ph.tobytes()
    e1, e2 = m2.take()
    assert len(e1) == 0 and len(e2) == 0


def test_fano_sampler_moments(lattice):
    """sample_fano_binomial (niel_models.hpp:202-263): mean and variance F * mean for
    Ge (F 0.13 in the defaults) in the interpolated-binomial regime and the Gaussian one."""
    import cmpmc_b200 as cm
    fano = lattice.config().fano_factor
    for mean in (5.0, 40.0, 3000.0):
        rng = cm.Rng.for_stream(21, int(mean))
        x = np.array([cm.physics.sample_fano_binomial(mean, fano, rng) for _ in range(4000)], dtype=np.float64)
        assert abs(x.mean() - mean) < 5 * np.sqrt(fano * mean / len(x)) + 0.5
        assert 0.5 * fano * mean < x.var() < 2.0 * fano * mean + 0.5


def test_non_finite_deposits_are_refused():
    """The Sarkis knot search is bounded (a NaN energy returns instead of walking past the
    last knot), and partition_deposit refuses a non-finite energy, position or time before
    drawing (the generator state is left alone)."""
    import math
    import cmpmc_b200 as cm
    si = dataclasses.replace(cm.materials.Germanium(), atomic_Z=14.0, atomic_A=28.085)
    assert math.isnan(cm.physics.sarkis_ionization_yield(float("nan"), si))
    assert cm.physics.sarkis_ionization_yield(1e3, si) > 0.0
    part = cm.EnergyPartition(cm.CrystalLattice(cm.materials.Germanium()))
    for pos, t, e in (((0.0, 0.0, 0.0), 0.0, float("nan")), ((0.0, 0.0, 0.0), 0.0, float("inf")),
                      ((float("nan"), 0.0, 0.0), 0.0, 100.0), ((0.0, 0.0, 0.0), float("nan"), 100.0)):
        r = cm.Rng.for_stream(8, 0)
        before = list(r.s)
        with pytest.raises(cm.CmpmcError):
            part.partition_deposit(pos, t, e, False, r)
        assert r.s == before
