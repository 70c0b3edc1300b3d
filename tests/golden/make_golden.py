"""Regenerates the golden fixtures in this directory from the reference CMPMC build.

Runs oracle/_ref/cmpmc_ref and oracle/_ref/cmpmc_ref_tables (the unmodified reference,
compiled from its own headers by `make -C oracle ref`) and stores compact records:

  rng.json              Rng::for_stream / next_u64 / uniform / isotropic_dir / lambertian_dir vectors
  lattice_ge.npz        sha256 of the reference's octahedral table, its CDF tables and
                        Herring-Vogt tensors, and a sample of table entries
  <workload>_full.npz   per-event records for a few events: post-generator Rng state,
                        initial tracks, per-event SimStats and every SensorHit
  <workload>_summary.npz per-event summaries for many events (hit count, integer counters,
                        sums over the hits, hash of the discrete hit fields)
  c1_hist.npz           per-event hit histograms (time, radius, energy) of 2000 mixed-energy
                        events (200,000 primaries), for the batched FP32 form's chi^2 tests
  c1_hist_full.npz      the same over all 10,000 events of the benchmark batch (1,000,000
                        primaries; histfull), for the bench's matched-statistics check
  <workload>_cr_*.npz   the same from oracle/_ref/cmpmc_ref_crlibm: the reference whose
                        transport uses a correctly rounded libm (oracle/ref_crlibm.hpp);
                        `floor` = fraction of events on which it agrees with the glibc build
  mask_channels.npz     channels of the SuperCDMS QET mask (fill 0.8, with its draws) and of
                        a 4 x 4 pad grid at 4096 points of a face
  kinematics_modes.npz  map_k_to_vg in the Exact and Bilinear modes (1000 directions x 3 modes)
  amm_transmission.npz  IsotropicAMMInterface (Ge -> Al) transmission of L and transverse
                        phonons at 400 incidence angles
  kaplan_surrogate.npz  KaplanSurrogateLUT (default Al film, seed 1337) lookups at 2000 energies
                        on [Delta, 46 Delta] with the reference's draws
  mesh_c3.npz           the recoil workloads' field mesh (TriLinearMesh3D::build_cartesian_grid,
                        201,898 nodes): field_at and potential_at at 4096 points in the cylinder

Usage: python tests/golden/make_golden.py [--only NAME,...]   (needs the reference build;
       takes a few minutes; NAME is a workload of PLAN, rng, lattice, hist, histfull, kin, amm, kaplan,
       mask or mesh)
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from tests.golden.records import compare_summaries, event_histograms, read_dump, summarize  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref")
REF_TABLES = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref_tables")
REF_CR = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref_crlibm")

# workload -> (full events, summary events)
PLAN = {
    "c0": (64, 10000),
    "c4": (0, 2000),
    "c1": (3, 40),
    "c2": (64, 2000),
    "tp": (32, 203),
    "tpl": (2, 21),
    "c3s": (1, 64),
    "c0m": (16, 2000),
    "tpm": (8, 203),
    "c0a": (16, 2000),
    "tpd": (8, 203),
    "tpe": (8, 203),
    "c0x": (8, 1000),
    "c0b": (8, 2000),
    "tp2": (8, 1000),
    "c0r": (16, 2000),
    "tps": (8, 203),
    "tpt": (8, 203),
    "pub": (16, 2000),
    "pubc": (8, 203),
}


def dump(workload: str, first: int, n: int, tmp: str, exe: str = REF):
    prefix = os.path.join(tmp, f"{workload}_{first}_{n}_{os.path.basename(exe)}")
    subprocess.run([exe, "dump", workload, str(first), str(n), "0", prefix], check=True)
    return read_dump(prefix, n)


def main() -> None:
    if not (os.path.exists(REF) and os.path.exists(REF_TABLES)):
        sys.exit("build the reference first: make -C oracle ref")
    only = None
    if len(sys.argv) > 2 and sys.argv[1] == "--only":
        only = set(sys.argv[2].split(","))

    def want(name: str) -> bool:
        return only is None or name in only

    with tempfile.TemporaryDirectory() as tmp:
        if want("mesh"):
            path = os.path.join(tmp, "mesh.bin")
            info = json.loads(subprocess.run([REF, "mesh", "4096", path], check=True, capture_output=True,
                                             text=True).stdout)
            rec = np.fromfile(path, dtype=np.float64).reshape(-1, 7)
            np.savez_compressed(os.path.join(HERE, "mesh_c3.npz"), points=rec[:, 0:3], field=rec[:, 3:6],
                                potential=rec[:, 6], n_vertices=info["vertices"], n_tets=info["tetrahedra"])
        if want("mesh2"):
            path = os.path.join(tmp, "mesh2.bin")
            info = json.loads(subprocess.run([REF, "mesh2", "4096", path], check=True, capture_output=True,
                                             text=True).stdout)
            rec = np.fromfile(path, dtype=np.float64).reshape(-1, 11)
            np.savez_compressed(os.path.join(HERE, "mesh2d.npz"), points=rec[:, 0:3], axisym_field=rec[:, 3:6],
                                axisym_potential=rec[:, 6], planar_field=rec[:, 7:10], planar_potential=rec[:, 10],
                                **{k: v for k, v in info.items()})
        if want("partition"):
            _partition(tmp)
        if want("meshfile"):
            _mesh_files(tmp)
        if want("mask"):
            path = os.path.join(tmp, "mask.bin")
            subprocess.run([REF, "mask", "4096", path], check=True)
            rec = np.fromfile(path, dtype=np.dtype([("x", "<f8"), ("y", "<f8"), ("qet", "<i4"), ("grid", "<i4")]))
            np.savez_compressed(os.path.join(HERE, "mask_channels.npz"), x=rec["x"], y=rec["y"], qet=rec["qet"],
                                grid=rec["grid"])
        if want("kin"):
            path = os.path.join(tmp, "kin.bin")
            subprocess.run([REF, "kin", "1000", path], check=True)
            rec = np.fromfile(path, dtype=np.float64).reshape(2, 1000, 3, 4)
            np.savez_compressed(os.path.join(HERE, "kinematics_modes.npz"), exact=rec[0], bilinear=rec[1])
        if want("amm"):
            path = os.path.join(tmp, "amm.bin")
            subprocess.run([REF, "amm", "400", path], check=True)
            t = np.fromfile(path, dtype=np.float64).reshape(2, -1)
            np.savez_compressed(os.path.join(HERE, "amm_transmission.npz"), longitudinal=t[0], transverse=t[1])
        if want("kaplan"):
            path = os.path.join(tmp, "kaplan.bin")
            subprocess.run([REF, "kaplan", "2000", path], check=True)
            raw = open(path, "rb").read()
            E, edep, cnt, refl = [], [], [], []
            off = 0
            while off < len(raw):
                e, d = np.frombuffer(raw, dtype="<f8", count=2, offset=off)
                c = int(np.frombuffer(raw, dtype="<u4", count=1, offset=off + 16)[0])
                off += 20
                refl.append(np.frombuffer(raw, dtype="<f8", count=c, offset=off))
                off += 8 * c
                E.append(e)
                edep.append(d)
                cnt.append(c)
            np.savez_compressed(os.path.join(HERE, "kaplan_surrogate.npz"), energy=np.array(E), edep=np.array(edep),
                                n_refl=np.array(cnt, dtype=np.uint32), refl=np.concatenate(refl))
        if want("rng"):
            _rng_vectors()
        if want("lattice"):
            _lattice(tmp)
        _workloads(tmp, want)
        if want("hist"):
            _hist(tmp)
        if want("histfull"):
            _hist_full(tmp)
    gl = subprocess.run(["ldd", "--version"], capture_output=True, text=True).stdout.split("\n")[0]
    with open(os.path.join(HERE, "PROVENANCE.txt"), "w") as f:
        f.write("Generated by tests/golden/make_golden.py from the unmodified reference CMPMC\n"
                "(oracle/_ref, g++ -O3 -std=c++20, no -march=native).\n"
                f"host libm: {gl}\n")


RESULT_DTYPE = np.dtype([("total_edep_eV", "<f8"), ("ionizing_eV", "<f8"), ("niel_eV", "<f8"),
                         ("lindhard_yield", "<f8"), ("n_pairs_true", "<u8"), ("n_pairs_sampled", "<u8"),
                         ("n_phonons_true", "<u8"), ("n_phonons_sampled", "<u8"), ("charge_weight", "<f8"),
                         ("phonon_weight", "<f8"), ("prompt_phonon_eV", "<f8")])


def _zero_padding(b: bytes, dtype) -> bytes:
    """The reference leaves the padding of its records uninitialised: zero it."""
    a = np.frombuffer(b, dtype=dtype).copy()
    for name in a.dtype.names:
        if name.startswith("_pad"):
            a[name] = 0
    return a.tobytes()


def _read_records(raw: bytes, off: int):
    from cmpmc_b200._ffi import CHARGE_DTYPE, PHONON_DTYPE
    nc, nph = np.frombuffer(raw, dtype="<u8", count=2, offset=off)
    off += 16
    ch = _zero_padding(raw[off:off + 128 * int(nc)], CHARGE_DTYPE)
    off += 128 * int(nc)
    ph = _zero_padding(raw[off:off + 128 * int(nph)], PHONON_DTYPE)
    off += 128 * int(nph)
    nxt = int(np.frombuffer(raw, dtype="<u8", count=1, offset=off)[0])
    return ch, ph, nxt, off + 8


def _partition(tmp: str) -> None:
    """Yields of the five NIEL models (Ge and Si), 48 partition_deposit cases and a
    HitMerger run of the reference (oracle/ref_driver.cpp `yield`, `partition`, `merge`)."""
    path = os.path.join(tmp, "yield.bin")
    subprocess.run([REF, "yield", path], check=True)
    y = np.fromfile(path, dtype=np.float64).reshape(2, 7, 400)
    path = os.path.join(tmp, "partition.bin")
    subprocess.run([REF, "partition", path], check=True)
    raw = open(path, "rb").read()
    off = 0
    res, nc, nph, nxt, h_ch, h_ph, full_ch, full_ph = [], [], [], [], [], [], [], []
    for i in range(48):
        res.append(np.frombuffer(raw, dtype=RESULT_DTYPE, count=1, offset=off)[0])
        off += RESULT_DTYPE.itemsize
        ch, ph, n, off = _read_records(raw, off)
        nc.append(len(ch) // 128)
        nph.append(len(ph) // 128)
        nxt.append(n)
        h_ch.append(hashlib.sha256(ch).hexdigest())
        h_ph.append(hashlib.sha256(ph).hexdigest())
        if i < 12:
            full_ch.append(ch)
            full_ph.append(ph)
    assert off == len(raw)
    path = os.path.join(tmp, "merge.bin")
    subprocess.run([REF, "merge", path], check=True)
    raw = open(path, "rb").read()
    flags = np.frombuffer(raw, dtype=np.uint8, count=36)
    m_res = np.frombuffer(raw, dtype=RESULT_DTYPE, count=1, offset=36)
    m_ch, m_ph, m_next, off = _read_records(raw, 36 + RESULT_DTYPE.itemsize)
    assert off == len(raw)
    np.savez_compressed(os.path.join(HERE, "partition.npz"), yields=y, results=np.array(res, dtype=RESULT_DTYPE),
                        n_charges=np.array(nc, dtype=np.uint64), n_phonons=np.array(nph, dtype=np.uint64),
                        next_u64=np.array(nxt, dtype=np.uint64), sha_charges=np.array(h_ch), sha_phonons=np.array(h_ph),
                        charges_0_11=np.frombuffer(b"".join(full_ch), dtype=np.uint8),
                        phonons_0_11=np.frombuffer(b"".join(full_ph), dtype=np.uint8),
                        merge_flags=flags, merge_result=m_res, merge_charges=np.frombuffer(m_ch, dtype=np.uint8),
                        merge_phonons=np.frombuffer(m_ph, dtype=np.uint8), merge_next_u64=np.uint64(m_next))


def _mesh_files(tmp: str) -> None:
    """A jittered Kuhn mesh of the default cylinder's bounding box written as the ASCII
    node / tetrahedron files of TriLinearMesh3D::load_from_files (millimetres, millivolts,
    with comment, blank and malformed lines), and the reference's fields at 2048 points."""
    d = os.path.join(HERE, "mesh_files")
    os.makedirs(d, exist_ok=True)
    R, h = 38.1, 12.7  # mm
    n = (6, 6, 5)
    rng = np.random.default_rng(5)
    xs = [np.linspace(-a, a, k + 1) for a, k in ((R, n[0]), (R, n[1]), (h, n[2]))]
    vid = lambda i, j, k: (i * (n[1] + 1) + j) * (n[2] + 1) + k  # noqa: E731
    with open(os.path.join(d, "nodes.txt"), "w") as f:
        f.write("# x_mm y_mm z_mm V_mV\n% exported node table\n\n")
        for i in range(n[0] + 1):
            for j in range(n[1] + 1):
                for k in range(n[2] + 1):
                    p = np.array([xs[0][i], xs[1][j], xs[2][k]])
                    inner = 0 < i < n[0] and 0 < j < n[1] and 0 < k < n[2]
                    if inner:
                        p = p + rng.uniform(-0.15, 0.15, 3) * np.array([2 * R / n[0], 2 * R / n[1], 2 * h / n[2]])
                    v = 4000.0 * (p[2] + h) / (2 * h) + 150.0 * (p[0] / R) ** 2
                    f.write(" ".join(repr(float(x)) for x in (p[0], p[1], p[2], v)) + "\n")
        f.write("not a node line\n")
    with open(os.path.join(d, "tets.txt"), "w") as f:
        f.write("# i0 i1 i2 i3\n")
        for i in range(n[0]):
            for j in range(n[1]):
                for k in range(n[2]):
                    c = [vid(i + a, j + b, k + e) for a in (0, 1) for b in (0, 1) for e in (0, 1)]
                    v000, v001, v010, v011, v100, v101, v110, v111 = c
                    for t in ((v111, v000, v100, v110), (v000, v100, v101, v111), (v000, v010, v110, v111),
                              (v000, v010, v011, v111), (v000, v001, v101, v111), (v000, v001, v011, v111)):
                        f.write(" ".join(str(x) for x in t) + "\n")
        f.write("%\n")
    path = os.path.join(tmp, "meshfile.bin")
    info = json.loads(subprocess.run([REF, "meshfile", os.path.join(d, "nodes.txt"), os.path.join(d, "tets.txt"),
                                      "1e-3", "1e-3", "2048", path], check=True, capture_output=True,
                                     text=True).stdout)
    rec = np.fromfile(path, dtype=np.float64).reshape(-1, 7)
    np.savez_compressed(os.path.join(HERE, "mesh_files.npz"), points=rec[:, 0:3], field=rec[:, 3:6],
                        potential=rec[:, 6], n_vertices=info["vertices"], n_tets=info["tetrahedra"])


def _rng_vectors() -> None:
    rng = {}
    for seed, stream in ((42, 0), (7, 12345), (17, 999999)):
        out = subprocess.run([REF, "rng", str(seed), str(stream), "8"], check=True, capture_output=True,
                             text=True).stdout.split("\n")
        rec = {"state": [], "u64": [], "uniform": [], "iso": [], "lamb": [], "seeded_12345": []}
        for line in out:
            if not line:
                continue
            k, *v = line.split()
            if k == "state":
                rec["state"] = [int(x) for x in v]
            elif k == "seeded":
                rec["seeded_12345"] = [int(x) for x in v]
            elif k == "u64":
                rec["u64"].append(int(v[0]))
            elif k == "uniform":
                rec["uniform"].append(float.hex(float(v[0])))
            else:
                rec[k].append([float.hex(float(x)) for x in v])
        rng[f"{seed}:{stream}"] = rec
    with open(os.path.join(HERE, "rng.json"), "w") as f:
        json.dump(rng, f, indent=1)


def _lattice(tmp: str) -> None:
    prefix = os.path.join(tmp, "ge")
    subprocess.run([REF_TABLES, prefix], check=True)
    oct_b = open(prefix + ".oct", "rb").read()
    cdf = np.fromfile(prefix + ".cdf", dtype=np.float64)
    hv = np.fromfile(prefix + ".hv", dtype=np.float64)
    octa = np.frombuffer(oct_b, dtype=np.float32).reshape(3, 256, 256, 4)
    idx = np.random.default_rng(0).integers(0, 256, size=(64, 2))
    np.savez_compressed(os.path.join(HERE, "lattice_ge.npz"), oct_sha256=np.array(hashlib.sha256(oct_b).hexdigest()),
                        cdf_lt=cdf[:1024], cdf_tt=cdf[1024:], hv=hv, sample_idx=idx,
                        sample=octa[:, idx[:, 0], idx[:, 1], :])


def _workloads(tmp: str, want) -> None:
    # workloads: the reference (glibc libm) and the reference with a correctly rounded
    # libm in the transport (cmpmc_ref_crlibm); "floor" is the fraction of events on
    # which the two agree (the device's transcendentals are correctly rounded)
    for wl, (n_full, n_sum) in PLAN.items():
        if not want(wl):
            continue
        if n_full:
            d = dump(wl, 0, n_full, tmp)
            np.savez_compressed(os.path.join(HERE, f"{wl}_full.npz"), **d)
            dc = dump(wl, 0, n_full, tmp, REF_CR)
            np.savez_compressed(os.path.join(HERE, f"{wl}_cr_full.npz"), **dc)
        d = dump(wl, 0, n_sum, tmp)
        s = summarize(d["events"], d["hit_offsets"], d["hits"])
        np.savez_compressed(os.path.join(HERE, f"{wl}_summary.npz"), summary=s,
                            injected=d["injected"], rng_state=d["rng_state"])
        dc = dump(wl, 0, n_sum, tmp, REF_CR)
        sc = summarize(dc["events"], dc["hit_offsets"], dc["hits"])
        floor = compare_summaries(s, sc)
        np.savez_compressed(os.path.join(HERE, f"{wl}_cr_summary.npz"), summary=sc,
                            floor_mask=floor["agree_mask"], floor=np.array(floor["frac"]))
        print(wl, n_full, n_sum, int(d["hit_offsets"][-1]), "hits; glibc vs correctly rounded agree on",
              f"{100 * floor['frac']:.2f}% of events")


def _hist(tmp: str) -> None:
    # mixed-energy batch: per-event hit histograms of the reference (2000 events,
    # 200,000 primaries) for the statistical parity of the batched FP32 form
    d = dump("c1", 0, 2000, tmp)
    lo, hi = float(d["hits"]["edep"].min()), float(d["hits"]["edep"].max())
    h = event_histograms(d["hit_offsets"], d["hits"], (lo, hi * (1 + 1e-9)))
    st = d["events"]["stats"]
    np.savez_compressed(os.path.join(HERE, "c1_hist.npz"), **h,
                        injected=d["injected"].sum(), deposited=st["total_deposited_eV"].sum(),
                        escaped=st["escaped_or_killed_eV"].sum(), steps=st["total_steps"].sum(),
                        n_hits=len(d["hits"]))
    print("c1 histograms from", len(d["hits"]), "hits")


def _hist_full(tmp: str) -> None:
    """The same histograms over the whole mixed-energy batch of the benchmark (10,000 events,
    1,000,000 primaries), in chunks of 2,000 events, with the edep range of c1_hist.npz."""
    rng = tuple(np.load(os.path.join(HERE, "c1_hist.npz"))["edep_range"])
    tot, inj, dep, esc, steps, n_hits = None, 0.0, 0.0, 0.0, 0, 0
    for first in range(0, 10000, 2000):
        d = dump("c1", first, 2000, tmp)
        h = event_histograms(d["hit_offsets"], d["hits"], rng)
        if tot is None:
            tot = h
        else:
            for k, v in h.items():
                if k != "edep_range":
                    tot[k] = tot[k] + v
        st = d["events"]["stats"]
        inj += float(d["injected"].sum())
        dep += float(st["total_deposited_eV"].sum())
        esc += float(st["escaped_or_killed_eV"].sum())
        steps += int(st["total_steps"].sum())
        n_hits += len(d["hits"])
        for f in os.listdir(tmp):  # the hit dumps are large
            os.remove(os.path.join(tmp, f))
    np.savez_compressed(os.path.join(HERE, "c1_hist_full.npz"), **tot, injected=inj, deposited=dep, escaped=esc,
                        steps=steps, n_hits=n_hits)
    print("c1 histograms (10,000 events) from", n_hits, "hits")


if __name__ == "__main__":
    main()
