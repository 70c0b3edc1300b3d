"""Multi-rank host path on CPU: two gloo ranks shard the events, transport them with a
stand-in runner (the device is not needed to check the sharding and the merge), gather
and merge on rank 0; the merged result must equal a single-process run over all events,
and the timing reduction must return the maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

N_PER_RANK = 24


def fake_runner(packed, options):
    """Deterministic stand-in for the device: one hit per initial phonon (time = energy)."""
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    ph = packed.phonons
    hits = np.zeros(len(ph), dtype=_ffi.HIT_DTYPE)
    hits["pos"] = ph["pos"]
    hits["time"] = ph["energy"]
    hits["edep"] = ph["energy"] * 0.5
    hits["incident_energy"] = ph["energy"]
    hits["mode"] = ph["mode"]
    hits["channel_id"] = -1
    st = cm.SimStats()
    st._r["total_steps"] = len(ph) * 3
    st._r["sensor_hits"] = len(ph)
    st._r["total_injected_eV"] = packed.injected_eV.sum()
    st._r["total_deposited_eV"] = hits["edep"].sum()
    return cm.RunResult(stats=st, hits=hits, hit_offsets=packed.phonon_offsets.copy())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    import cmpmc_b200 as cm
    from cmpmc_b200 import dist as cdist
    eng = cm.SimulationEngine(cm.CrystalLattice(cm.materials.Germanium()), cm.DetectorModel())
    part = cdist.run_sharded(eng, cm.workloads.mixed_energy, N_PER_RANK, cm.RunOptions(seed=7), rank, fake_runner)
    merged = cdist.gather_to_root(part)
    t = cdist.max_over_ranks(1.0 + rank)
    if rank == 0:
        np.savez(out_path, hits=merged["hits"], offsets=merged["hit_offsets"],
                 stats=np.array(merged["stats"]).reshape(1).view(np.uint8), tmax=t)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_and_merge(tmp_path):
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    out = str(tmp_path / "merged.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    got = np.load(out)
    eng = cm.SimulationEngine(cm.CrystalLattice(cm.materials.Germanium()), cm.DetectorModel())
    packed = eng.generate(cm.workloads.mixed_energy, 2 * N_PER_RANK, 7)
    want = fake_runner(packed, cm.RunOptions(seed=7))
    assert got["hits"].tobytes() == want.hits.tobytes()
    assert np.array_equal(got["offsets"], want.hit_offsets)
    st = got["stats"].view(_ffi.STATS_DTYPE)[0]
    assert int(st["total_steps"]) == want.stats.total_steps
    assert int(st["sensor_hits"]) == want.stats.sensor_hits
    np.testing.assert_allclose(float(st["total_injected_eV"]), want.stats.total_injected_eV, rtol=1e-12)
    assert float(got["tmax"]) == 2.0
