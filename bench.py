"""Benchmark of the transport hot path (run_events over phonon tracks) on B200.

Workload (the mixed-energy phonon batch): 10,000 events x 100 phonons = 1,000,000 primary
tracks per GPU, energies log-uniform on [1, 30] meV, modes L/ST/FT 0.10/0.36/0.54, origins
uniform in the Ge cylinder (R 3.81 cm, half height 1.27 cm), isotropic directions, seed 7;
default Ge lattice and detector (Al Kaplan films on both faces). One step = one run_events
pass over the whole batch in the batched FP32 form (FP32 geometry, FP64 energy ledger and
time of flight; the SM-phase pool: one persistent launch, one block per SM alternating a
transport phase, whose warps refill their lanes from the block's ring of pending phonons and
the batch's primaries, and a film phase that runs the waiting film cascades, until every
track is absorbed or lost), hits kept. The launch shape comes
from the library's autotuner (results do not depend on it).

  value  primary phonon tracks / s, inputs resident on the device, device-timed (CUDA
         events on the library's stream), max over ranks
  e2e    the same through the public API with host buffers: pinned host inputs copied in
         and every hit, the hit offsets and the statistics copied back, each step, one call
         at a time (e2e_with_generator adds the host generator's time per step; --overlap
         adds e2e_overlapped_copies: two contexts in turn, each step's output copy on a copy
         stream beside the next step's call, checked against the device-resident call;
         --pipeline adds e2e_two_calls_in_flight: two contexts on two host threads)
  plain_fp64  the plain FP64 form (bit-exact event streams) on the same workload, one step
  batched_fp64  the same SM-phase pool computed in FP64 throughout on the same substreams
         (pool form 3), one step: fp32_over_fp64 is what the FP32 form gains
  matched     after the timed region: chi^2 p-values of the per-event hit histograms (time
         256 bins over 0-2 ms, radius 64, edep 64) of one timed batched call against the
         plain FP64 run and against the reference's histograms of the same 10,000 events
         (tests/golden/c1_hist_full.npz), and the energy-ledger closure of both forms
  published   the reference's published benchmark workload (benchmarks/cmpmc_bench.cpp:
         demo polynomial surfaces, max_bounces 100, one 7.5 meV phonon per event) on the
         device in both forms, beside the published CPU figures

Multi-GPU (torchrun): every rank runs its own 10,000 events (events rank*10000 + i), no
collective on the data path (weak scaling); barrier and max-over-ranks timing through
torch.distributed.

`--impl reference` times the reference's own CPU run_events (oracle/_ref/cmpmc_ref, the
unmodified reference built from its headers) on all host cores, on a bounded sample of the
same workload per step, and prints the same metric.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "phonon tracks/s, 1 B200: batched FP32 vs plain FP64 at matched hit stats"
UNIT = "primary phonon tracks/s"
EVENTS = 10000
PER_EVENT = 100
SEED = 7
BYTES_PER_STEP = 192  # algorithmic FP32 track state read + written per transport step: 2 x 96 B
# the reference's published phonon benchmark (benchmarks/README.md:55, 71): 4-core Xeon 2.10 GHz
PUBLISHED_MS_PER_EVENT_1T = 0.581
PUBLISHED_EVENTS_PER_S_4T = 6190.0


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(form: str):
    """DRAM bytes per transport step of the batched kernels from the committed ncu summary."""
    name = {"sm_pool": "batched_fp32_sm_pool_mixed_energy.json", "warp_pool": "batched_fp32_warp_pool_mixed_energy.json",
            "rounds": "batched_fp32_split_mixed_energy.json", "inline": "batched_fp32_inline_mixed_energy.json"}[form]
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return float(json.load(f)["dram_bytes_per_step"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix=f"cmpmc_clocks{index}_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        sms, maxs, reasons = [], [], set()
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                sms.append(float(p[1]))
                maxs.append(float(p[2]))
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                   p[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        except Exception:
            pass
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
                "samples": len(sms)}


def reference_arm(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    exe = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cmpmc_ref is not built (make -C oracle ref)"}))
        return
    sample_events = args.ref_events
    cores = os.cpu_count() or 1

    def one(first):
        out = subprocess.run([exe, "time", "c1", str(first), str(sample_events), "0"], check=True,
                             capture_output=True, text=True).stdout
        return json.loads(out.strip().splitlines()[-1])

    for w in range(args.warmup):
        one(w * sample_events)
    walls, prim, steps = 0.0, 0, 0
    for k in range(args.steps):
        r = one((args.warmup + k) * sample_events)
        walls += r["wall_seconds"]
        prim += r["primaries"]
        steps += r["total_steps"]
    value = prim / walls
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * walls / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": "mixed_energy_phonons", "events_per_step": sample_events, "primaries_per_event": PER_EVENT,
                   "seed": SEED, "threads": cores},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{sample_events} events x {PER_EVENT} primaries per step (events advance "
                                   f"through the seed-{SEED} stream), reference run_events on all cores",
                         "steps_per_s": steps / walls},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(sample_events: int):
    exe = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref")
    if not os.path.exists(exe):
        return None
    out = subprocess.run([exe, "time", "c1", "0", str(sample_events), "0"], check=True, capture_output=True,
                         text=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    return {"value": r["primaries"] / r["wall_seconds"], "unit": UNIT, "cores": r["threads"], "kind": "reference",
            "sample": f"events 0-{sample_events - 1} of the workload ({r['primaries']} primaries), reference "
                      f"run_events (oracle/_ref/cmpmc_ref, unmodified reference) on {r['threads']} threads",
            "steps_per_s": r["total_steps"] / r["wall_seconds"], "wall_seconds": r["wall_seconds"]}


def matched_statistics(batched: dict, plain, first_event: int, fp64=None) -> dict:
    """chi^2 of the batched call's per-event hit histograms against the plain FP64 form's on
    the same events, against the batched form computed in FP64 on the same substreams and
    against the reference's (10,000-event fixture, rank 0's events), and the ledger closures."""
    from tests.golden.records import event_histograms, hist_chi2
    path = os.path.join(ROOT, "tests", "golden", "c1_hist_full.npz")
    ref = dict(np.load(path)) if os.path.exists(path) else None
    rng = tuple(ref["edep_range"]) if ref is not None else (
        float(batched["hits"]["edep"].min()), float(batched["hits"]["edep"].max()) * (1 + 1e-9))
    hb = event_histograms(batched["offsets"], batched["hits"], rng)
    out = {"bins": {"time": "256 over 0-2 ms", "radius": "64 over 0-R", "edep": "64 over the reference range"},
           "events": int(hb["n_events"]), "batched_hits": int(len(batched["hits"])),
           "ledger_closure_batched": abs(batched["injected"] - batched["deposited"] - batched["escaped"]) /
                                     batched["injected"]}
    if plain is not None:
        hp = event_histograms(plain["offsets"], plain["hits"], rng)
        out["p_vs_plain_fp64"] = {k: round(hist_chi2(hb, hp, k)[2], 4) for k in ("time", "radius", "edep")}
        out["plain_hits"] = int(len(plain["hits"]))
        out["ledger_closure_plain_fp64"] = abs(plain["injected"] - plain["deposited"] - plain["escaped"]) / \
            plain["injected"]
    if fp64 is not None:
        hf = event_histograms(fp64["offsets"], fp64["hits"], rng)
        out["p_vs_batched_fp64"] = {k: round(hist_chi2(hb, hf, k)[2], 4) for k in ("time", "radius", "edep")}
        out["batched_fp64_hits"] = int(len(fp64["hits"]))
        out["ledger_closure_batched_fp64"] = abs(fp64["injected"] - fp64["deposited"] - fp64["escaped"]) / \
            fp64["injected"]
    if ref is not None and first_event == 0 and int(ref["n_events"]) == hb["n_events"]:
        out["p_vs_reference_cpu"] = {k: round(hist_chi2(hb, ref, k)[2], 4) for k in ("time", "radius", "edep")}
        out["reference_hits"] = int(ref["n_hits"])
    return out


def published_workload(cm, lat, dev: int, n: int, lib) -> dict:
    """The reference's published phonon benchmark workload (benchmarks/cmpmc_bench.cpp:45-67):
    n events, device-resident inputs, hits not kept (as the benchmark), both forms; and the
    reference's own CPU run_events on this host's cores on a sample of the same events."""
    det = cm.DetectorModel.published_benchmark()
    eng = cm.SimulationEngine(lat, det)
    packed = eng.generate(cm.workloads.published_phonon, n, 12345)
    out = {"workload": "published phonon benchmark (demo surfaces, max_bounces 100, 7.5 meV, seed 12345)",
           "events": n, "reference_published_ms_per_event_1_thread": PUBLISHED_MS_PER_EVENT_1T,
           "reference_published_events_per_s_4_threads": PUBLISHED_EVENTS_PER_S_4T}
    for form in ("plain_fp64", "batched_fp32"):
        opt = cm.RunOptions(seed=12345, form=form, keep_hits=False, device=dev)
        eng.run_packed(packed, opt)  # warm-up (buffers, tables)
        r = eng.run_packed(packed, opt)
        out[form] = {"events_per_s": n / (r.device_ms * 1e-3), "us_per_event": 1e3 * r.device_ms / n,
                     "steps": int(r.stats.total_steps), "sensor_hits": int(r.stats.sensor_hits)}
    exe = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref")
    if os.path.exists(exe):
        m = min(n, 20000)
        r = json.loads(subprocess.run([exe, "time", "pub", "0", str(m), "0"], check=True, capture_output=True,
                                      text=True).stdout.strip().splitlines()[-1])
        out["reference_cpu_this_host"] = {"events_per_s": m / r["wall_seconds"], "threads": r["threads"],
                                          "sample_events": m}
    return out


class _DevView:
    """A device allocation of the library seen as a flat uint8 array (CUDA array interface),
    so that torch can queue a copy of it on one of its streams without owning it."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 2}


def overlapped_e2e(args, cm, lat, det, dev: int, lib, h, run_on, hp, packed, desc, ref) -> dict:
    """End-to-end steps whose output copies overlap the next step's transport: two contexts in
    turn, inputs copied from pinned host memory into the context's device input buffers, the
    call leaving its outputs on the device, and the copy of the hits and offsets to pinned host
    memory queued on a copy stream while the other context's call runs."""
    import torch
    eng_b = cm.SimulationEngine(lat, det)
    h_b = eng_b.context(dev)
    if args.queue_capacity or args.stack_capacity:
        eng_b.configure(dev, stack_capacity=args.stack_capacity, queue_capacity=args.queue_capacity)
    eng_b.configure_pool({"sm_pool": 1, "warp_pool": 2, "rounds": 0}[args.launch], device=dev)
    if args.no_stage:
        eng_b.configure_staging(False, device=dev)
    ctxs = (h, h_b)
    n = args.events
    cuda = f"cuda:{dev}"
    dev_in = [[torch.empty(t.numel(), dtype=torch.uint8, device=cuda) for t in hp] for _ in range(2)]
    descs = []
    for s in range(2):
        d = desc(True)
        d.rng_state, d.injected_eV = dev_in[s][0].data_ptr(), dev_in[s][1].data_ptr()
        d.phonon_offsets, d.phonons = dev_in[s][2].data_ptr(), dev_in[s][3].data_ptr()
        descs.append(d)
    h2d_s, d2h_s = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    kChunk = 16 << 20

    def inputs(s):
        with torch.cuda.stream(h2d_s):
            for k in range(4):
                dev_in[s][k].copy_(hp[k], non_blocking=True)
        h2d_s.synchronize()

    n_hits0 = 0
    for s in range(2):  # warm-up: the contexts size their buffers
        inputs(s)
        n_hits0 = max(n_hits0, int(run_on(ctxs[s], descs[s]).n_hits))
    cap = (n_hits0 + n_hits0 // 8 + 1024) * 56
    host_hits = [torch.empty(cap, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    host_offs = [torch.empty((n + 1) * 8, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    done = [None, None]
    last = None
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(args.steps):
        s = i % 2
        if done[s] is not None:
            done[s].synchronize()  # this context's previous copy has finished
        inputs(s)
        o = run_on(ctxs[s], descs[s])
        nh = int(o.n_hits) * 56
        if nh > cap:
            raise RuntimeError("host hit buffer too small")
        with torch.cuda.stream(d2h_s):
            # in 16 MiB pieces: the next call's own small device-to-host reads (the batch's
            # track count, its counters) take the same copy engine and would otherwise wait
            # behind the whole 1.5 GB copy
            if nh:
                hv = torch.as_tensor(_DevView(o.hits, nh), device=cuda)
                for a0 in range(0, nh, kChunk):
                    a1 = min(nh, a0 + kChunk)
                    host_hits[s][a0:a1].copy_(hv[a0:a1], non_blocking=True)
            host_offs[s].copy_(torch.as_tensor(_DevView(o.hit_offsets, (n + 1) * 8), device=cuda), non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(d2h_s)
        done[s] = ev
        last = (s, int(o.n_hits))
    for ev in done:
        if ev is not None:
            ev.synchronize()
    ms = 1e3 * (time.perf_counter() - t0) / args.steps
    s, nh = last
    offs = host_offs[s].numpy().view(np.uint64)
    checked = None
    if ref is not None:
        # the offsets exactly, the hits as an order-free checksum (a modular sum of their 8-byte
        # words: the hits of an event come in no fixed order)
        got = host_hits[s][:nh * 56].numpy().view(np.uint64)
        want = np.ascontiguousarray(ref["hits"]).view(np.uint8).reshape(-1).view(np.uint64)
        checked = bool(np.array_equal(offs, ref["offsets"]) and nh == len(ref["hits"]) and
                       int(got.sum(dtype=np.uint64)) == int(want.sum(dtype=np.uint64)))
        if not checked:
            raise RuntimeError("overlapped e2e outputs differ from the device-resident call")
    return {"value": int(packed.phonon_offsets[-1]) / (ms * 1e-3), "unit": UNIT,
            "h2d_bytes_per_step": int(sum(t.numel() for t in hp)), "d2h_bytes_per_step": nh * 56 + (n + 1) * 8 + 208,
            "ms_per_step": ms, "checked_against_device_resident_call": checked,
            "how": "two contexts in turn on one host thread; each step's hit and offset copy to pinned host "
                   "memory runs on a copy stream during the next step's call; wall clock over all K steps"}


def recoil_batch(cm, lat, dev: int, n: int) -> None:
    """The uneven recoil batch (electron recoils of 10 eV-10 keV, log-uniform, split by
    EnergyPartition::partition_deposit with up to 4,096 pairs, every Luke phonon tracked, in
    the 201,898-node tetrahedral-mesh field; seed 13) in one call of the batched form, hits
    not kept (the batch makes billions). Prints one JSON line: primaries (deposits) per
    second, carriers and phonon steps per second."""
    det = cm.DetectorModel()
    det.mesh_field_3d = cm.TriLinearMesh3D.recoil_mesh(det)
    det.luke_sample_fraction = 1.0
    eng = cm.SimulationEngine(lat, det)
    t0 = time.perf_counter()
    packed = eng.generate(cm.workloads.recoil, n, 13)
    t_gen = time.perf_counter() - t0
    opt = cm.RunOptions(seed=13, form="batched_fp32", keep_hits=False, device=dev)
    warm = eng.generate(cm.workloads.recoil, 8, 13)
    eng.run_packed(warm, opt)  # tables, mesh and buffers
    r = eng.run_packed(packed, opt)
    st = r.stats
    ms = r.device_ms
    print(json.dumps({
        "workload": "recoil_batch", "events": n, "seed": 13, "form": "batched_fp32", "keep_hits": False,
        "device_ms": ms, "kernel_ms": r.kernel_ms, "events_per_s": n / (ms * 1e-3),
        "charges": int(packed.charge_offsets[-1]), "initial_phonons": int(packed.phonon_offsets[-1]),
        "charge_steps": int(st.charge_steps), "phonon_steps": int(st.total_steps),
        "luke_phonons": int(st.luke_phonons_emitted), "sensor_hits": int(st.sensor_hits),
        "steps_per_s": (st.charge_steps + st.total_steps) / (ms * 1e-3),
        "generator_s": t_gen, "launches": int(r.kernel_launches)}), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--events", type=int, default=EVENTS)
    ap.add_argument("--ref-events", type=int, default=400)
    ap.add_argument("--cpu-events", type=int, default=1000)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-configuration autotuner")
    ap.add_argument("--no-graph", action="store_true", help="eager launches instead of CUDA-graph replay")
    ap.add_argument("--form", default="batched_fp32", choices=["batched_fp32", "batched_fp32_inline"])
    ap.add_argument("--queue-capacity", type=int, default=0, help="phonon queue entries (0: library default)")
    ap.add_argument("--stack-capacity", type=int, default=0, help="tracks per device thread (0: library default)")
    ap.add_argument("--launch", default="sm_pool", choices=["sm_pool", "warp_pool", "rounds"],
                    help="launch form of the batched phonon transport")
    ap.add_argument("--no-matched", action="store_true", help="skip the matched-statistics check")
    ap.add_argument("--pipeline", action="store_true",
                    help="also time e2e with two calls in flight (two contexts on two host threads)")
    ap.add_argument("--overlap", action="store_true",
                    help="also time e2e with each step's output copy beside the next step's call")
    ap.add_argument("--no-fp64", action="store_true", help="skip the batched FP64 comparison step")
    ap.add_argument("--no-stage", action="store_true",
                    help="decay CDF tables read from global memory instead of the TMA-staged shared copy")
    ap.add_argument("--recoil", type=int, default=0,
                    help="instead of the headline line: time the recoil batch of this many events once")
    ap.add_argument("--surrogate", action="store_true",
                    help="film cascades from the KaplanSurrogateLUT table (not the headline configuration)")
    ap.add_argument("--pub-events", type=int, default=100000, help="events of the published workload (0: skip)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
        return

    import torch
    import torch.distributed as dist
    import cmpmc_b200 as cm
    from cmpmc_b200 import _ffi

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = local
    torch.cuda.set_device(dev)

    lat = cm.CrystalLattice(cm.materials.Germanium())
    if args.recoil:
        if rank == 0:
            recoil_batch(cm, lat, dev, args.recoil)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    det = cm.DetectorModel()
    eng = cm.SimulationEngine(lat, det)
    first = rank * args.events
    t_gen = time.perf_counter()
    packed = eng.generate(cm.workloads.mixed_energy, args.events, SEED, first_event=first)
    t_gen = time.perf_counter() - t_gen
    n_prim = int(packed.phonon_offsets[-1])
    lib = _ffi.load()
    h = eng.context(dev)
    if args.queue_capacity or args.stack_capacity:
        eng.configure(dev, stack_capacity=args.stack_capacity, queue_capacity=args.queue_capacity)
    form_id = _ffi.FORM_BATCHED_FP32 if args.form == "batched_fp32" else _ffi.FORM_BATCHED_FP32_INLINE
    eng.configure_pool({"sm_pool": 1, "warp_pool": 2, "rounds": 0}[args.launch], device=dev)
    if args.no_stage:
        eng.configure_staging(False, device=dev)
    launch_form = "inline" if args.form != "batched_fp32" else args.launch

    # device-resident inputs (torch owns the memory)
    def to_dev(a):
        t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(f"cuda:{dev}")
        return t
    d_rng, d_inj = to_dev(packed.rng_state), to_dev(packed.injected_eV)
    d_off, d_ph = to_dev(packed.phonon_offsets), to_dev(packed.phonons)
    torch.cuda.synchronize(dev)

    def desc(on_device: bool, host=None):
        d = _ffi.RunDescC()
        d.n_events = args.events
        d.first_event = first
        d.keep_hits = 1
        d.form = form_id
        d.seed = SEED
        d.kaplan_surrogate = 1 if args.surrogate else 0
        if on_device:
            d.rng_state, d.injected_eV = d_rng.data_ptr(), d_inj.data_ptr()
            d.phonon_offsets, d.phonons = d_off.data_ptr(), d_ph.data_ptr()
            d.inputs_on_device = 1
            d.outputs_on_device = 1
        else:
            d.rng_state, d.injected_eV, d.phonon_offsets, d.phonons = host
        return d

    def run_on(hh, d):
        out = _ffi.RunOutC()
        st = lib.cmpmc_gpu_run_events(hh, C.byref(d), C.byref(out))
        if st != 0:
            buf = C.create_string_buffer(512)
            lib.cmpmc_gpu_last_error(hh, buf, 512)
            raise RuntimeError(buf.value.decode())
        return out

    def run(d):
        return run_on(h, d)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")  # 256 MiB > 126 MB L2

    def fetch(out):
        """hit offsets, hits and totals of a call whose outputs stayed on the device"""
        n_h = int(out.n_hits)
        offs = np.zeros(args.events + 1, dtype=np.uint64)
        hits = np.zeros(n_h, dtype=_ffi.HIT_DTYPE)
        lib.cmpmc_gpu_memcpy(offs.ctypes.data, C.c_void_p(out.hit_offsets), offs.nbytes)
        if n_h:
            lib.cmpmc_gpu_memcpy(hits.ctypes.data, C.c_void_p(out.hits), hits.nbytes)
        st = out.stats
        return {"offsets": offs, "hits": hits, "injected": st.total_injected_eV,
                "deposited": st.total_deposited_eV, "escaped": st.escaped_or_killed_eV}

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    dd = desc(True)
    # launch configuration from the project's autotuner (results do not depend on it), then
    # CUDA-graph replay of the device-resident call
    tune = None
    # the SM-phase pool has one launch shape (one 512-thread block per SM): nothing to tune
    if not args.no_tune and launch_form != "sm_pool":
        tr = _ffi.TuneResultC()
        if lib.cmpmc_gpu_autotune(h, C.byref(dd), 1, C.byref(tr)) != 0:
            buf = C.create_string_buffer(512)
            lib.cmpmc_gpu_last_error(h, buf, 512)
            raise RuntimeError(buf.value.decode())
        tune = {"threads_per_block": tr.threads_per_block, "blocks_per_sm": tr.blocks_per_sm,
                "phase_steps": tr.phase_steps,
                "best_kernel_ms": tr.best_ms, "default_kernel_ms": tr.first_ms,
                "tried": [[tr.tried_tpb[i], tr.tried_bps[i], round(tr.tried_ms[i], 2)] for i in range(tr.n_tried)]}
    # graph replay covers the pool forms' call (counter resets, unit map, the persistent
    # transport launch, merge) and the inline form's; the host-driven rounds depend on the
    # queue counts, so they run eagerly
    use_graph = not args.no_graph and launch_form != "rounds"
    if use_graph:
        lib.cmpmc_gpu_configure_graph(h, 1)
    for _ in range(args.warmup):
        flush.zero_()
        run(dd)
    barrier()
    ms, kms, launches, steps_total, hits_total = [], [], 0, 0, 0
    with ClockSampler(dev) as clocks:
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            o = run(dd)
            ms.append(o.total_ms)
            kms.append(o.kernel_ms)
            launches += o.kernel_launches
            steps_total += o.stats.total_steps
            hits_total += o.n_hits
        barrier()
        wall = time.perf_counter() - t0
    # the last timed call's outputs (device memory of the context) for the matched check
    batched_res = fetch(o) if not args.no_matched else None
    step_ms = max_over_ranks(sum(ms) / args.steps)
    kernel_ms = max_over_ranks(sum(kms) / args.steps)
    value = world * n_prim / (step_ms * 1e-3)

    # e2e: host buffers (pinned), H2D of the inputs and D2H of every output inside the call
    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = a.view(np.uint8).reshape(-1)
        return t
    hp = [pinned(packed.rng_state), pinned(packed.injected_eV), pinned(packed.phonon_offsets), pinned(packed.phonons)]
    hd = desc(False, tuple(t.data_ptr() for t in hp))
    if world > 1:
        # several GPUs: the outputs stay on each rank's device and are merged on rank 0 over
        # NCCL (cmpmc_b200.dist.exchange), which then copies the merged hits to the host
        from cmpmc_b200 import dist as cdist
        hd.outputs_on_device = 1
        out_host = None

        def merge_to_root(o):
            nonlocal out_host
            d_hits = torch.empty(max(int(o.n_hits), 1) * 56, dtype=torch.uint8, device=f"cuda:{dev}")[:int(o.n_hits) * 56]
            d_offs = torch.empty(args.events + 1, dtype=torch.int64, device=f"cuda:{dev}")
            if o.n_hits:
                lib.cmpmc_gpu_memcpy(C.c_void_p(d_hits.data_ptr()), C.c_void_p(o.hits), int(o.n_hits) * 56)
            lib.cmpmc_gpu_memcpy(C.c_void_p(d_offs.data_ptr()), C.c_void_p(o.hit_offsets), (args.events + 1) * 8)
            st = torch.from_numpy(np.frombuffer(bytes(o.stats), dtype=np.uint8).copy()).to(f"cuda:{dev}")
            m = cdist.exchange(d_hits, d_offs, st)
            if m["hits"] is not None:
                if out_host is None or out_host.numel() < m["hits"].numel():
                    out_host = torch.empty(m["hits"].numel(), dtype=torch.uint8, pin_memory=True)
                out_host[:m["hits"].numel()].copy_(m["hits"])
                torch.cuda.synchronize(dev)
                return m["hits"].numel() + m["hit_offsets"].numel() * 8 + 208
            return 0
    lib.cmpmc_gpu_configure_graph(h, 0)
    o = run(hd)
    if world > 1:
        merge_to_root(o)
    barrier()
    e2e_ms = []
    d2h = 0
    for _ in range(args.steps):
        flush.zero_()
        barrier()
        t1 = time.perf_counter()
        o = run(hd)
        if world > 1:
            d2h = merge_to_root(o)
        e2e_ms.append(1e3 * (time.perf_counter() - t1))
    e2e_step = max_over_ranks(sum(e2e_ms) / args.steps)
    gen_ms = max_over_ranks(1e3 * t_gen)
    h2d = sum(t.numel() for t in hp)
    if world == 1:
        d2h = int(o.n_hits) * 56 + (args.events + 1) * 8 + 208

    # e2e with two calls in flight: a second context (its own stream, device buffers and pinned
    # output buffers) on a second host thread, the K steps taken in turn from a shared counter,
    # so that one call's input and hit copies run while the other call's transport runs; every
    # step still copies its inputs in and its hits, offsets and totals out
    e2e_pipe = None
    if world == 1 and args.pipeline:
        eng_b = cm.SimulationEngine(lat, det)
        h_b = eng_b.context(dev)
        if args.queue_capacity or args.stack_capacity:
            eng_b.configure(dev, stack_capacity=args.stack_capacity, queue_capacity=args.queue_capacity)
        eng_b.configure_pool({"sm_pool": 1, "warp_pool": 2, "rounds": 0}[args.launch], device=dev)
        run_on(h_b, hd)  # sizes the second context's buffers
        lock = threading.Lock()
        left = [args.steps]
        errors = []

        def worker(hh):
            while True:
                with lock:
                    if left[0] == 0:
                        return
                    left[0] -= 1
                try:
                    run_on(hh, hd)
                except Exception as e:  # reported after the join
                    errors.append(e)
                    return
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        threads = [threading.Thread(target=worker, args=(x,)) for x in (h, h_b)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall_pipe = time.perf_counter() - t1
        if errors:
            raise errors[0]
        pipe_ms = 1e3 * wall_pipe / args.steps
        e2e_pipe = {"value": n_prim / (pipe_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": pipe_ms, "calls_in_flight": 2,
                    "how": "two contexts on two host threads, steps taken in turn; wall clock over all K steps"}

    # e2e with each step's output copy overlapping the next step's transport (one host thread,
    # two contexts in turn): a step copies its inputs from pinned host memory into the device
    # input buffers of its context, calls run_events with the outputs left on the device, and
    # queues the device-to-host copy of its hits and offsets on a copy stream; the next step's
    # call (the other context, whose buffers the copy does not touch) runs meanwhile. A context
    # is reused only after its previous copy has finished. Checked against the device-resident
    # call: the same offsets and hit count.
    e2e_overlap = None
    if world == 1 and args.overlap:
        try:
            e2e_overlap = overlapped_e2e(args, cm, lat, det, dev, lib, h, run_on, hp, packed, desc, batched_res)
        except Exception as e:  # reported in the line; the one-call-at-a-time figure stands
            e2e_overlap = {"error": str(e)}

    # plain FP64 form on the same workload (bit-exact event streams), one step
    plain = None
    plain_res = None
    if not args.no_plain:
        dp = desc(True)
        dp.form = _ffi.FORM_PLAIN_FP64
        o = run(dp)
        p_ms = max_over_ranks(o.total_ms)
        plain = {"value": world * n_prim / (p_ms * 1e-3), "unit": UNIT, "ms_per_step": p_ms,
                 "steps_per_s": o.stats.total_steps / (o.kernel_ms * 1e-3)}
        if batched_res is not None:
            plain_res = fetch(o)
    # the same SM-phase pool computed in FP64 on the same substreams (pool form 3), one step
    fp64 = None
    fp64_res = None
    if not args.no_fp64 and launch_form == "sm_pool" and not args.surrogate:
        eng.configure_pool(3, device=dev)
        run(dd)  # warm-up (its ring and film buffers)
        flush.zero_()
        torch.cuda.synchronize(dev)
        o = run(dd)
        f_ms = max_over_ranks(o.total_ms)
        f_kms = max_over_ranks(o.kernel_ms)
        fp64 = {"value": world * n_prim / (f_ms * 1e-3), "unit": UNIT, "ms_per_step": f_ms,
                "kernel_ms_per_step": f_kms, "steps_per_s": o.stats.total_steps / (o.kernel_ms * 1e-3),
                "hits": int(o.n_hits)}
        if batched_res is not None:
            fp64_res = fetch(o)
        eng.configure_pool(1, device=dev)
    matched = matched_statistics(batched_res, plain_res, first, fp64_res) if batched_res is not None else None
    published = None
    if args.pub_events and rank == 0:
        try:
            published = published_workload(cm, lat, dev, args.pub_events, lib)
        except Exception as e:  # reported in the line; the headline figures above stand
            published = {"error": str(e)}

    e2e_one = {"value": world * n_prim / (e2e_step * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step, "calls_in_flight": 1}
    peak, peak_kind = measured_peaks()
    steps_per_launch = steps_total / args.steps
    achieved = steps_per_launch * BYTES_PER_STEP / (sum(kms) / args.steps * 1e-3) / 1e9
    tps = profile_traffic(launch_form)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "mixed_energy_phonons", "events": args.events * world, "primaries_per_event": PER_EVENT,
                   "primaries": n_prim * world, "form": args.form, "seed": SEED,
                   "film_cascades": "surrogate table" if args.surrogate else "full Kaplan cascade",
                   "energy": "log-uniform 1-30 meV", "modes": "L/ST/FT 0.10/0.36/0.54",
                   "decay_tables": "global memory" if args.no_stage else "shared memory (TMA bulk copy)",
                   "l2": "256 MiB buffer written between timed steps (L2 126 MB); inputs 128 MB, hits ~1.5 GB per step"},
        "kernel_ms_per_step": kernel_ms,
        "steps_per_s": world * steps_per_launch / (kernel_ms * 1e-3),
        "hits_per_step": hits_total / args.steps,
        "e2e": e2e_one,
        "e2e_with_generator": {"value": world * n_prim / ((e2e_step + gen_ms) * 1e-3), "unit": UNIT,
                               "ms_per_step": e2e_step + gen_ms, "generator_ms": gen_ms},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_step": BYTES_PER_STEP,
                     "traffic": (tps * steps_per_launch if tps else None)},
        "gpu_launches": launches,
        "launch": {"form": {"sm_pool": "sm_phase_pool", "warp_pool": "warp_pool", "rounds": "host_rounds",
                            "inline": "inline"}[launch_form],
                   "graph": use_graph, "transport_launches_per_call": launches / args.steps,
                   "host_syncs_per_call": 1 if launch_form != "rounds" else None, "autotune": tune},
        "clocks": clocks.summary(),
        "wall_s_timed": wall,
        "generator_s": t_gen,
    }
    if e2e_pipe is not None:
        line["e2e_two_calls_in_flight"] = e2e_pipe
    if e2e_overlap is not None:
        line["e2e_overlapped_copies"] = e2e_overlap
    if plain is not None:
        line["plain_fp64"] = plain
        line["batched_over_plain"] = value / plain["value"]
    if fp64 is not None:
        line["batched_fp64"] = fp64
        line["fp32_over_fp64"] = value / fp64["value"]
    if matched is not None:
        line["matched"] = matched
    if published is not None:
        line["published"] = published
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.cpu_events)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
