"""EnergyPartition::partition_deposit on the device (cmpmc_gpu_partition_deposits) against
the host partition, which is bit-identical to the reference (tests/test_partition.py).

The device runs the same code (partition.cuh) without FMA contraction, from the same
generator states; its transcendentals are correctly rounded where the host's platform libm
is not always (cbrt in the charge-cloud radius and the Lindhard yield, sin/cos of the
directions), so a record may differ in the last bits and, rarely, a comparison on such a
value may take the other branch. Bar: at least 99 % of the deposits give the same record
counts and the same final generator state, and their records agree to 1e-12 relative with
every integer field equal.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 1024


def _deposits(seed):
    """Electron and nuclear recoils of 10 eV-10 keV at points of the default cylinder, each
    with the generator state left after three draws of its own stream."""
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    dep = np.zeros(N, dtype=_ffi.DEPOSIT_DTYPE)
    states = np.zeros((N, 4), dtype=np.uint64)
    R, h = 0.0381, 0.0127
    for i in range(N):
        r = cm.Rng.for_stream(seed, i)
        u = r.uniform()
        rr, phi, z = R * np.sqrt(r.uniform()), 2 * np.pi * r.uniform(), h * (2 * r.uniform() - 1)
        dep[i]["pos"] = (rr * np.cos(phi), rr * np.sin(phi), z)
        dep[i]["time_s"] = 1e-9 * i
        dep[i]["edep_eV"] = 10.0 * 10.0 ** (3.0 * u)
        dep[i]["is_nuclear_recoil"] = i % 3 == 2
        states[i] = r.s
    return dep, states


@pytest.mark.parametrize("variant", ["defaults", "no_fano_empirical"])
def test_device_partition_matches_host(ge_lattice, variant):
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    opts = cm.PartitionOptions(max_sampled_pairs=4096, max_sampled_phonons=200)
    if variant == "no_fano_empirical":
        opts = cm.PartitionOptions(niel_model=cm.NIELModel.Empirical, use_fano_fluctuations=False,
                                   use_charge_cloud=True, max_sampled_pairs=64, max_sampled_phonons=50)
    dep, states = _deposits(13 if variant == "defaults" else 29)
    eng = cm.SimulationEngine(ge_lattice, cm.DetectorModel())
    coff, ch, poff, ph, st_out = cm.partition_deposits_on_device(eng, dep, states, opts)
    assert len(coff) == N + 1 and int(coff[-1]) == len(ch) and int(poff[-1]) == len(ph)
    part = cm.EnergyPartition(ge_lattice)
    same = 0
    for i in range(N):
        r = cm.Rng.from_state([int(x) for x in states[i]])
        _, hc, hp = part.partition_deposit(tuple(dep[i]["pos"]), float(dep[i]["time_s"]), float(dep[i]["edep_eV"]),
                                           bool(dep[i]["is_nuclear_recoil"]), r, opts)
        dc = ch[int(coff[i]):int(coff[i + 1])]
        dp = ph[int(poff[i]):int(poff[i + 1])]
        if len(dc) != len(hc) or len(dp) != len(hp) or [int(x) for x in st_out[i]] != r.s:
            continue
        same += 1
        for a, b in ((dc, hc), (dp, hp)):
            for name in a.dtype.names:
                if name.startswith("_pad"):
                    continue
                if a.dtype[name].base.kind == "f":
                    np.testing.assert_allclose(a[name], b[name], rtol=1e-12, atol=1e-300, err_msg=f"{i} {name}")
                else:
                    assert np.array_equal(a[name], b[name]), (i, name)
    print(f"{variant}: {same} of {N} deposits with the host's counts and final state; "
          f"{len(ch)} carriers, {len(ph)} phonons")
    assert same >= 0.99 * N


def test_device_partition_capacity_and_transport(ge_lattice):
    """A short record capacity reports the totals and leaves the generator states alone;
    the device records feed the transport directly (one deposit per event)."""
    import ctypes as C
    import torch
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    dep, states = _deposits(13)
    dep, states = dep[:64], states[:64]
    det = cm.DetectorModel()
    det.e_field = cm.UniformElectricField.from_bias(4.0, 2.54 * cm.units.cm)
    det.luke_sample_fraction = 0.0
    eng = cm.SimulationEngine(ge_lattice, det)
    lib = _ffi.load()
    h = eng.context(0)
    t_dep = torch.from_numpy(dep.view(np.uint8).reshape(-1).copy()).to("cuda:0")
    t_rng = torch.from_numpy(states.view(np.int64).copy()).to("cuda:0")
    t_off = torch.zeros(2 * 65, dtype=torch.int64, device="cuda:0")
    o = cm.PartitionOptions(max_sampled_pairs=4096, max_sampled_phonons=200).to_c()
    nc, nph = C.c_uint64(0), C.c_uint64(0)
    st = lib.cmpmc_gpu_partition_deposits(h, t_dep.data_ptr(), 64, C.byref(o), t_rng.data_ptr(), t_off.data_ptr(),
                                          t_off.data_ptr() + 65 * 8, None, 0, None, 0, C.byref(nc), C.byref(nph))
    assert st == 4 and nc.value > 0 and nph.value > 0
    assert np.array_equal(t_rng.cpu().numpy().view(np.uint64), states)
    coff, ch, poff, ph, st_out = cm.partition_deposits_on_device(eng, dep, states,
                                                                 cm.PartitionOptions(max_sampled_pairs=4096,
                                                                                     max_sampled_phonons=200))
    assert len(ch) == nc.value and len(ph) == nph.value
    injected = dep["edep_eV"].astype(np.float64)
    packed = cm.PackedEvents(64, 0, st_out.copy(), injected, poff.copy(), ph, coff.copy(), ch)
    # the deposits here reach 10 keV (3,400 pairs); 64 events drift a few 1e5 carriers
    res = eng.run_packed(packed, cm.RunOptions(seed=13, form="batched_fp32", want_event_stats=True))
    assert res.stats.charge_steps > 0 and res.stats.total_steps > 0
    assert res.stats.charges_collected > 0


def test_device_partition_refuses_non_finite_deposit(ge_lattice):
    """One deposit with a NaN energy makes the call return CMPMC_ERR_INVALID before the fill:
    no record is written and every generator state is left as it was."""
    import ctypes as C
    import torch
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    dep, states = _deposits(13)
    dep, states = dep[:64].copy(), states[:64].copy()
    dep[17]["edep_eV"] = np.nan
    eng = cm.SimulationEngine(ge_lattice, cm.DetectorModel())
    lib = _ffi.load()
    h = eng.context(0)
    t_dep = torch.from_numpy(dep.view(np.uint8).reshape(-1).copy()).to("cuda:0")
    t_rng = torch.from_numpy(states.view(np.int64).copy()).to("cuda:0")
    t_off = torch.zeros(2 * 65, dtype=torch.int64, device="cuda:0")
    t_ch = torch.zeros(4096 * 128, dtype=torch.uint8, device="cuda:0")
    t_ph = torch.zeros(4096 * 128, dtype=torch.uint8, device="cuda:0")
    nc, nph = C.c_uint64(0), C.c_uint64(0)
    st = lib.cmpmc_gpu_partition_deposits(h, t_dep.data_ptr(), 64, None, t_rng.data_ptr(), t_off.data_ptr(),
                                          t_off.data_ptr() + 65 * 8, t_ch.data_ptr(), 4096, t_ph.data_ptr(), 4096,
                                          C.byref(nc), C.byref(nph))
    assert st == _ffi.ERR_INVALID
    assert np.array_equal(t_rng.cpu().numpy().view(np.uint64), states)
    assert int(t_ch.count_nonzero()) == 0 and int(t_ph.count_nonzero()) == 0
