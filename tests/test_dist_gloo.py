"""Multi-rank path on CPU: gloo ranks shard the events, transport them with a stand-in
runner (the device is not needed to check the sharding and the exchange), and merge them
with the same collectives the GPU ranks use over NCCL (cmpmc_b200.dist.exchange: all-gather
of the per-event hit counts and the SimStats records, hits sent to the root in rank order).
The merged result must equal a single-process run over all events; uneven ranks (one with no
events, one with no hits) merge the same way; the adjoint's all-reduce sums the ranks'
estimates; the timing reduction returns the maximum over ranks."""
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


def _uneven_part(rank):
    """Rank 0: 5 events with hits; rank 1: no events; rank 2: 4 events, no hits; rank 3: 3
    events with hits (records of the device's layout)."""
    from cmpmc_b200 import _ffi
    n_ev = [5, 0, 4, 3][rank]
    per = [[2, 0, 3, 1, 4], [], [0, 0, 0, 0], [1, 5, 2]][rank]
    offs = np.zeros(n_ev + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(per)
    hits = np.zeros(int(offs[-1]), dtype=_ffi.HIT_DTYPE)
    hits["time"] = 1e-6 * (100 * rank + np.arange(len(hits)))
    hits["edep"] = 1e-3 * (rank + 1)
    hits["surface_id"] = rank % 3
    hits["channel_id"] = rank - 1
    st = np.zeros((), dtype=_ffi.STATS_DTYPE)
    st["total_steps"] = 1000 + rank
    st["sensor_hits"] = len(hits)
    st["total_injected_eV"] = 0.1 * (rank + 1)
    st["total_deposited_eV"] = float(hits["edep"].sum())
    return {"hits": hits, "hit_offsets": offs, "stats": st}


def _uneven_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    from cmpmc_b200 import dist as cdist
    import cmpmc_b200 as cm
    merged = cdist.gather_to_root(_uneven_part(rank))
    # the adjoint: every rank's estimate is a sum over its own primaries
    res = cm.AdjointResult(hist=np.full(8, 1.0 + rank), value=2.0 * rank, grad=np.arange(4.0) * (rank + 1),
                           value_var=0.5, grad_var=np.full(4, 0.25), stats=cm.SimStats(_uneven_part(rank)["stats"]),
                           n_primaries=10 * (rank + 1), kernel_ms=1.0, total_ms=1.0, kernel_launches=1)
    tot = cdist.allreduce_adjoint(res)
    if rank == 0:
        np.savez(out_path, hits=merged["hits"], offsets=merged["hit_offsets"],
                 stats=np.array(merged["stats"]).reshape(1).view(np.uint8), hist=tot.hist, value=tot.value,
                 grad=tot.grad, value_var=tot.value_var, grad_var=tot.grad_var, n_primaries=tot.n_primaries,
                 steps=tot.stats.total_steps)
    dist.barrier()
    dist.destroy_process_group()


def test_exchange_uneven_ranks_and_adjoint_allreduce(tmp_path):
    from cmpmc_b200 import _ffi
    from cmpmc_b200 import dist as cdist
    out = str(tmp_path / "uneven.npz")
    mp.start_processes(_uneven_main, args=(4, _free_port(), out), nprocs=4, start_method="spawn", join=True)
    got = np.load(out)
    want = cdist.merge_results([_uneven_part(r) for r in range(4)])
    assert got["hits"].tobytes() == want["hits"].tobytes()
    assert np.array_equal(got["offsets"], want["hit_offsets"])
    assert len(got["offsets"]) == 5 + 0 + 4 + 3 + 1
    st = got["stats"].view(_ffi.STATS_DTYPE)[0]
    assert int(st["total_steps"]) == 4006 and int(st["sensor_hits"]) == len(want["hits"])
    np.testing.assert_allclose(float(st["total_injected_eV"]), 1.0, rtol=1e-15)
    np.testing.assert_array_equal(got["hist"], np.full(8, 10.0))
    assert float(got["value"]) == 12.0
    np.testing.assert_array_equal(got["grad"], np.arange(4.0) * 10.0)
    assert float(got["value_var"]) == 2.0 and np.all(got["grad_var"] == 1.0)
    assert int(got["n_primaries"]) == 100 and int(got["steps"]) == 4006
