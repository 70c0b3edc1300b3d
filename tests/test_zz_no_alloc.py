"""The allocation-free entry point (cmpmc_gpu_run_events_noalloc).

It serves callers that cannot call cudaMalloc -- code inside a framework whose caching
allocator owns the device memory, code with a fixed memory budget, latency-critical loops
-- so it takes every input and output as caller-owned device memory and keeps its scratch
in a fixed array of the library. Here the caller's buffers come from torch; the results of
two calls in a row must equal those of the regular entry point (same kernel arithmetic:
hits, offsets and per-event records bit for bit, run totals to 1e-12), and the second call
must leave the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_entry_point_on_two_calls(ge_lattice):
    import torch
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi

    lib = _ffi.load()
    det = cm.DetectorModel()
    eng = cm.SimulationEngine(ge_lattice, det)
    n = 512
    packed = eng.generate(cm.workloads.single_l_origin, n, 42)
    ref = eng.run_packed(packed, cm.RunOptions(seed=42, want_event_stats=True))

    dev = torch.device("cuda:0")

    def on_device(a):
        return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(dev)

    rng, inj = on_device(packed.rng_state), on_device(packed.injected_eV)
    off, ph = on_device(packed.phonon_offsets), on_device(packed.phonons)
    cap = len(ref.hits) + 1024
    ev_stats = torch.zeros(n * _ffi.STATS_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    hit_off = torch.zeros((n + 1) * 8, dtype=torch.uint8, device=dev)
    hits = torch.zeros(cap * _ffi.HIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    cdet = det.to_c()
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize(dev)

    free_before = None
    for call in range(2):
        if call == 1:
            torch.cuda.synchronize(dev)
            free_before = torch.cuda.mem_get_info(dev)[0]
        total = _ffi.SimStatsC()
        n_hits = C.c_uint64(0)
        st = lib.cmpmc_gpu_run_events_noalloc(ge_lattice._h, C.byref(cdet), 0, n, rng.data_ptr(), inj.data_ptr(),
                                              off.data_ptr(), ph.data_ptr(), ev_stats.data_ptr(), hit_off.data_ptr(),
                                              hits.data_ptr(), cap, C.c_void_p(stream), C.byref(total),
                                              C.byref(n_hits))
        assert st == 0, st
        torch.cuda.synchronize(dev)
        if call == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        assert n_hits.value == len(ref.hits)
        got_hits = hits[: n_hits.value * _ffi.HIT_DTYPE.itemsize].cpu().numpy().view(_ffi.HIT_DTYPE)
        assert got_hits.tobytes() == ref.hits.tobytes()
        got_off = hit_off.cpu().numpy().view(np.uint64)
        assert np.array_equal(got_off, ref.hit_offsets)
        got_ev = ev_stats.cpu().numpy().view(_ffi.STATS_DTYPE)
        assert got_ev.tobytes() == ref.event_stats.tobytes()
        got_total = np.frombuffer(bytes(total), dtype=_ffi.STATS_DTYPE)[0]
        want_total = ref.stats.record()
        for name in _ffi.STATS_DTYPE.names:
            a, b = float(got_total[name]), float(want_total[name])
            if _ffi.STATS_DTYPE[name].kind == "u":
                assert a == b, name
            else:
                assert abs(a - b) <= 1e-12 * max(abs(b), 1e-300), name


def test_noalloc_rejects_too_small_hit_buffer(ge_lattice):
    import torch
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi

    lib = _ffi.load()
    det = cm.DetectorModel()
    eng = cm.SimulationEngine(ge_lattice, det)
    n = 64
    packed = eng.generate(cm.workloads.single_l_origin, n, 42)
    dev = torch.device("cuda:0")

    def on_device(a):
        return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(dev)

    rng, inj = on_device(packed.rng_state), on_device(packed.injected_eV)
    off, ph = on_device(packed.phonon_offsets), on_device(packed.phonons)
    ev_stats = torch.zeros(n * _ffi.STATS_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    hit_off = torch.zeros((n + 1) * 8, dtype=torch.uint8, device=dev)
    hits = torch.zeros(16 * _ffi.HIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    cdet = det.to_c()
    total = _ffi.SimStatsC()
    n_hits = C.c_uint64(0)
    st = lib.cmpmc_gpu_run_events_noalloc(ge_lattice._h, C.byref(cdet), 0, n, rng.data_ptr(), inj.data_ptr(),
                                          off.data_ptr(), ph.data_ptr(), ev_stats.data_ptr(), hit_off.data_ptr(),
                                          hits.data_ptr(), 16, C.c_void_p(torch.cuda.current_stream(dev).cuda_stream),
                                          C.byref(total), C.byref(n_hits))
    assert st == _ffi.ERR_CAPACITY
    assert n_hits.value > 16
