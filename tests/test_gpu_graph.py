"""Launch machinery of the batched form: CUDA-graph replay of device-resident calls and the
autotuner. Neither may change a result: batched units own their substreams, so hits and
counters are the same for any launch shape, and a replayed graph repeats the eager call."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import WORKLOAD_SEED, detector_for, workload_of

pytestmark = pytest.mark.gpu


def _device_desc(packed, seed, keep):
    import torch
    from cmpmc_b200 import _ffi

    def dev(a):
        t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to("cuda:0")
        keep.append(t)
        return t.data_ptr()

    d = _ffi.RunDescC()
    d.n_events = packed.n_events
    d.rng_state, d.injected_eV = dev(packed.rng_state), dev(packed.injected_eV)
    d.phonon_offsets, d.phonons = dev(packed.phonon_offsets), dev(packed.phonons)
    d.inputs_on_device = d.outputs_on_device = 1
    d.keep_hits = 1
    d.want_event_stats = 1
    d.form = _ffi.FORM_BATCHED_FP32_INLINE
    d.seed = seed
    return d


def _run(lib, h, d):
    from cmpmc_b200 import _ffi
    out = _ffi.RunOutC()
    assert lib.cmpmc_gpu_run_events(h, C.byref(d), C.byref(out)) == 0
    n, nh = d.n_events, int(out.n_hits)
    # the outputs stay on the device: copy them to the host
    hits = np.zeros(nh, dtype=_ffi.HIT_DTYPE)
    offs = np.zeros(n + 1, dtype=np.uint64)
    assert lib.cmpmc_gpu_memcpy(hits.ctypes.data, out.hits, nh * _ffi.HIT_DTYPE.itemsize) == 0
    assert lib.cmpmc_gpu_memcpy(offs.ctypes.data, out.hit_offsets, (n + 1) * 8) == 0
    return out, hits, offs


def test_graph_replay_repeats_the_eager_call(ge_lattice):
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    lib = _ffi.load()
    eng = cm.SimulationEngine(ge_lattice, detector_for("c1"))
    packed = eng.generate(workload_of("c1"), 200, WORKLOAD_SEED["c1"])
    keep = []
    d = _device_desc(packed, 7, keep)
    h = eng.context(0)
    eager, h0, o0 = _run(lib, h, d)
    eng.configure_graph(True)
    first, h1, o1 = _run(lib, h, d)    # eager, then captured
    replay, h2, o2 = _run(lib, h, d)   # one graph launch
    replay2, h3, o3 = _run(lib, h, d)
    for hh, oo, rr in ((h1, o1, first), (h2, o2, replay), (h3, o3, replay2)):
        assert hh.tobytes() == h0.tobytes() and np.array_equal(oo, o0)
        assert bytes(rr.stats) == bytes(eager.stats)
    assert replay.kernel_ms > 0 and replay.kernel_launches == replay2.kernel_launches
    # a different seed is a different call: captured anew, different hits
    d2 = _device_desc(packed, 8, keep)
    other, h4, _ = _run(lib, h, d2)
    assert h4.tobytes() != h0.tobytes()
    again, h5, _ = _run(lib, h, d2)
    assert h5.tobytes() == h4.tobytes()
    eng.configure_graph(False)


def _event_sets(hits, offs):
    """the hits of every event as a sorted multiset of records (the pool forms write an
    event's hits in no fixed order)"""
    raw = hits.view(np.uint8).reshape(len(hits), -1)
    out = []
    for e in range(len(offs) - 1):
        rows = raw[int(offs[e]):int(offs[e + 1])]
        out.append(sorted(r.tobytes() for r in rows))
    return out


@pytest.mark.parametrize("pool", [1, 2])
def test_pool_graph_replay_repeats_the_eager_call(ge_lattice, pool):
    """SM-phase pool (1) and warp pool (2): the call (counter resets, unit map, the persistent
    transport launch, the merge) captured after a clean eager call and replayed as one graph
    launch gives every event the same hits and the same integer counters."""
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi
    lib = _ffi.load()
    eng = cm.SimulationEngine(ge_lattice, detector_for("c1"))
    packed = eng.generate(workload_of("c1"), 300, WORKLOAD_SEED["c1"])
    keep = []
    d = _device_desc(packed, 7, keep)
    d.form = _ffi.FORM_BATCHED_FP32
    h = eng.context(0)
    eng.configure_pool(pool)
    eager, h0, o0 = _run(lib, h, d)
    ref = _event_sets(h0, o0)
    eng.configure_graph(True)
    runs = [_run(lib, h, d) for _ in range(3)]  # eager + capture, then two graph launches
    ints = [n for n, t in _ffi.SimStatsC._fields_ if t is C.c_uint64]
    for out, hh, oo in runs:
        assert np.array_equal(oo, o0)
        assert _event_sets(hh, oo) == ref
        for name in ints:
            assert getattr(out.stats, name) == getattr(eager.stats, name), name
        inj, dep = out.stats.total_injected_eV, out.stats.total_deposited_eV
        assert abs(dep - eager.stats.total_deposited_eV) <= 1e-12 * inj
        assert out.kernel_ms > 0
    assert runs[1][0].kernel_launches == runs[2][0].kernel_launches
    # another configuration drops the captured call: the next call runs eagerly again
    eng.configure_staging(False)
    after, h4, o4 = _run(lib, h, d)
    assert _event_sets(h4, o4) == ref
    eng.configure_staging(True)
    eng.configure_graph(False)


def test_autotune_keeps_results(ge_lattice):
    import cmpmc_b200 as cm
    eng = cm.SimulationEngine(ge_lattice, detector_for("c1"))
    packed = eng.generate(workload_of("c1"), 300, WORKLOAD_SEED["c1"])
    opt = cm.RunOptions(seed=7, form="batched_fp32", want_event_stats=True)
    before = eng.run_packed(packed, opt)
    tune = eng.autotune(packed, opt, repeats=1)
    print(tune)
    assert tune["threads_per_block"] in (64, 128) or tune["threads_per_block"] == 128
    assert len(tune["tried"]) >= 4 and tune["best_ms"] <= tune["first_ms"]
    after = eng.run_packed(packed, opt)
    # the split form fixes each event's hits as a set (their order within the event is free)
    assert np.array_equal(after.hit_offsets, before.hit_offsets)
    for i in range(len(after.hit_offsets) - 1):
        lo, hi = int(after.hit_offsets[i]), int(after.hit_offsets[i + 1])
        assert np.sort(after.hits[lo:hi], order=["time", "edep"]).tobytes() == \
            np.sort(before.hits[lo:hi], order=["time", "edep"]).tobytes(), i
    for name in after.event_stats.dtype.names:
        if after.event_stats.dtype[name].kind == "u":
            assert np.array_equal(after.event_stats[name], before.event_stats[name]), name


def test_autotune_charge_queue(ge_lattice):
    import cmpmc_b200 as cm
    eng = cm.SimulationEngine(ge_lattice, detector_for("c3s"))
    packed = eng.generate(workload_of("c3s"), 8, WORKLOAD_SEED["c3s"])
    opt = cm.RunOptions(seed=13, form="batched_fp32", want_event_stats=True)
    before = eng.run_packed(packed, opt)
    tune = eng.autotune(packed, opt, repeats=1)
    assert tune["queue_capacity"] in (1 << 20, 1 << 22, 1 << 24)
    assert any(t["queue_capacity"] == 1 << 20 for t in tune["tried"])
    after = eng.run_packed(packed, opt)
    for name in after.event_stats.dtype.names:
        if after.event_stats.dtype[name].kind == "u":
            assert np.array_equal(after.event_stats[name], before.event_stats[name]), name
