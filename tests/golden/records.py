"""Readers and summaries of per-event transport records (shared by the fixture script and
the tests). Record layouts are those of the reference's PhononTrack / ChargeTrack /
SensorHit / SimStats (core/track.hpp, transport/engine.hpp), mirrored in include/cmpmc_gpu.h."""
from __future__ import annotations

import numpy as np

PHONON_DTYPE = np.dtype([("pos", "<f8", 3), ("k_dir", "<f8", 3), ("vg_dir", "<f8", 3), ("energy", "<f8"),
                         ("vg_mag", "<f8"), ("time", "<f8"), ("weight", "<f8"), ("bounces", "<u4"),
                         ("mode", "u1"), ("_pad", "u1", 19)])
CHARGE_DTYPE = np.dtype([("pos", "<f8", 3), ("p_eV", "<f8", 3), ("ekin", "<f8"), ("time", "<f8"),
                         ("weight", "<f8"), ("valley", "<u2"), ("type", "u1"), ("alive", "u1"),
                         ("_pad", "u1", 52)])
HIT_DTYPE = np.dtype([("pos", "<f8", 3), ("time", "<f8"), ("edep", "<f8"), ("incident_energy", "<f8"),
                      ("surface_id", "u1"), ("excitation", "u1"), ("mode", "u1"), ("_pad", "u1"),
                      ("channel_id", "<i4")])
_STATS = [
    ("total_steps", "u8"), ("isotope_scatters", "u8"), ("polycrystal_scatters", "u8"),
    ("decays_L_to_TT", "u8"), ("decays_L_to_LT", "u8"), ("surface_refls", "u8"),
    ("surface_downconversions", "u8"), ("sensor_hits", "u8"), ("killed_tracks", "u8"),
    ("charge_steps", "u8"), ("luke_phonons_emitted", "u8"), ("intervalley_scatters", "u8"),
    ("charges_trapped", "u8"), ("trap_ionizations", "u8"), ("charge_surface_refls", "u8"),
    ("charges_collected", "u8"), ("total_luke_phonon_eV", "f8"), ("charge_recomb_edep_eV", "f8"),
    ("sc_pair_breakings", "u8"), ("qp_diffusion_steps", "u8"), ("qp_phonons_radiated", "u8"),
    ("qp_recombinations", "u8"), ("qp_local_traps", "u8"), ("total_injected_eV", "f8"),
    ("total_deposited_eV", "f8"), ("escaped_or_killed_eV", "f8"),
]
STATS_DTYPE = np.dtype([(n, "<" + t) for n, t in _STATS])
INT_STATS = [n for n, t in _STATS if t == "u8"]
FP_STATS = [n for n, t in _STATS if t == "f8"]
EVENT_DTYPE = np.dtype([("n_hits", "<u8"), ("stats", STATS_DTYPE)])
SUMMARY_DTYPE = np.dtype([("n_hits", "<u8"), ("ints", "<u8", len(INT_STATS)), ("fps", "<f8", len(FP_STATS)),
                          ("sum_time", "<f8"), ("sum_edep", "<f8"), ("sum_incident", "<f8"), ("sum_pos", "<f8", 3),
                          ("discrete_hash", "<u8")])


def read_dump(prefix: str, n: int) -> dict:
    """Reads the .init / .events / .hits files written by `cmpmc_ref dump`."""
    init = open(prefix + ".init", "rb").read()
    rng_state = np.zeros((n, 4), dtype=np.uint64)
    injected = np.zeros(n, dtype=np.float64)
    po, co = [0], [0]
    phs, chs = [], []
    off = 0
    for i in range(n):
        rng_state[i] = np.frombuffer(init, dtype=np.uint64, count=4, offset=off)
        injected[i] = np.frombuffer(init, dtype=np.float64, count=1, offset=off + 32)[0]
        nph, nch = np.frombuffer(init, dtype=np.uint64, count=2, offset=off + 40)
        off += 56
        phs.append(np.frombuffer(init, dtype=PHONON_DTYPE, count=int(nph), offset=off))
        off += 128 * int(nph)
        chs.append(np.frombuffer(init, dtype=CHARGE_DTYPE, count=int(nch), offset=off))
        off += 128 * int(nch)
        po.append(po[-1] + int(nph))
        co.append(co[-1] + int(nch))
    events = np.fromfile(prefix + ".events", dtype=EVENT_DTYPE, count=n)
    hits = np.fromfile(prefix + ".hits", dtype=HIT_DTYPE)
    hit_offsets = np.concatenate([[0], np.cumsum(events["n_hits"])]).astype(np.uint64)
    phonons = np.concatenate(phs) if phs else np.zeros(0, PHONON_DTYPE)
    charges = np.concatenate(chs) if chs else np.zeros(0, CHARGE_DTYPE)
    phonons = phonons.copy()
    charges = charges.copy()
    phonons["_pad"] = 0
    charges["_pad"] = 0
    hits = hits.copy()
    hits["_pad"] = 0
    return {"rng_state": rng_state, "injected": injected, "phonon_offsets": np.array(po, dtype=np.uint64),
            "phonons": phonons, "charge_offsets": np.array(co, dtype=np.uint64), "charges": charges,
            "events": events, "hits": hits, "hit_offsets": hit_offsets}


def _hash_discrete(h: np.ndarray) -> int:
    x = 0xCBF29CE484222325
    for s, e, m, c in zip(h["surface_id"].tolist(), h["excitation"].tolist(), h["mode"].tolist(),
                          h["channel_id"].tolist()):
        x ^= (s | (e << 8) | (m << 16) | ((c & 0xFFFFFFFF) << 24))
        x = (x * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return x


def summarize(events_stats: np.ndarray, hit_offsets: np.ndarray, hits: np.ndarray) -> np.ndarray:
    """Per-event summary. events_stats is either EVENT_DTYPE (n_hits + stats) or STATS_DTYPE."""
    n = len(hit_offsets) - 1
    st = events_stats["stats"] if events_stats.dtype.names and "stats" in events_stats.dtype.names else events_stats
    out = np.zeros(n, dtype=SUMMARY_DTYPE)
    out["n_hits"] = np.diff(hit_offsets.astype(np.int64))
    for j, name in enumerate(INT_STATS):
        out["ints"][:, j] = st[name]
    for j, name in enumerate(FP_STATS):
        out["fps"][:, j] = st[name]
    for i in range(n):
        h = hits[int(hit_offsets[i]):int(hit_offsets[i + 1])]
        if len(h) == 0:
            continue
        out["sum_time"][i] = h["time"].sum()
        out["sum_edep"][i] = h["edep"].sum()
        out["sum_incident"][i] = h["incident_energy"].sum()
        out["sum_pos"][i] = h["pos"].sum(axis=0)
        out["discrete_hash"][i] = _hash_discrete(h)
    return out


def compare_summaries(ref: np.ndarray, got: np.ndarray, rel_tol: float = 1e-9) -> dict:
    """Event-by-event parity: discrete fields exact, continuous sums within rel_tol."""
    assert len(ref) == len(got)
    same_n = ref["n_hits"] == got["n_hits"]
    same_hash = ref["discrete_hash"] == got["discrete_hash"]
    same_ints = (ref["ints"] == got["ints"]).all(axis=1)

    def close(a, b):
        return np.abs(a - b) <= rel_tol * np.maximum(np.abs(a), 1e-300) + 1e-300

    cont = close(ref["sum_time"], got["sum_time"]) & close(ref["sum_edep"], got["sum_edep"]) & \
        close(ref["sum_incident"], got["sum_incident"])
    cont &= (np.abs(ref["sum_pos"] - got["sum_pos"]) <= rel_tol * np.maximum(np.abs(ref["sum_pos"]), 1e-6)).all(axis=1)
    agree = same_n & same_hash & same_ints & cont
    return {"n": int(len(ref)), "agree": int(agree.sum()), "frac": float(agree.mean()) if len(ref) else 1.0,
            "same_n_hits": int(same_n.sum()), "same_hash": int(same_hash.sum()), "same_ints": int(same_ints.sum()),
            "cont_close": int(cont.sum()), "agree_mask": agree}


# ---- histogram statistics (hit time, radial position, energy) ---------------------------
HIST_SPEC = {
    "time": (256, 0.0, 2e-3),          # s
    "radius": (64, 0.0, 3.81e-2),      # m
    "edep": (64, None, None),          # eV, range from the reference sample
}


def event_histograms(hit_offsets: np.ndarray, hits: np.ndarray, edep_range: tuple) -> dict:
    """Per-bin sum and sum of squares over events of the per-event hit histograms.

    Hits of one event are correlated, so comparisons treat the event as the independent
    unit: the mean per-event count in a bin and its variance across events."""
    n = len(hit_offsets) - 1
    ev = np.repeat(np.arange(n), np.diff(hit_offsets.astype(np.int64)))
    out = {"n_events": n}
    values = {"time": hits["time"], "radius": np.hypot(hits["pos"][:, 0], hits["pos"][:, 1]), "edep": hits["edep"]}
    for name, (nb, lo, hi) in HIST_SPEC.items():
        if name == "edep":
            lo, hi = edep_range
        b = np.floor((values[name] - lo) / (hi - lo) * nb).astype(np.int64)
        ok = (b >= 0) & (b < nb)
        counts = np.bincount(ev[ok] * nb + b[ok], minlength=n * nb).astype(np.float64).reshape(n, nb)
        out[name + "_sum"] = counts.sum(axis=0)
        out[name + "_sumsq"] = (counts * counts).sum(axis=0)
    out["edep_range"] = np.array(edep_range, dtype=np.float64)
    return out


def hist_chi2(a: dict, b: dict, name: str, min_count: float = 20.0):
    """chi^2 of the difference of mean per-event histograms, with per-bin variances
    estimated from the spread across events. Returns (chi2, dof, p)."""
    from scipy.stats import chi2 as chi2_dist
    na, nb = a["n_events"], b["n_events"]
    sa, qa = a[name + "_sum"], a[name + "_sumsq"]
    sb, qb = b[name + "_sum"], b[name + "_sumsq"]
    ma, mb = sa / na, sb / nb
    va = np.maximum(qa / na - ma * ma, 0.0) / na
    vb = np.maximum(qb / nb - mb * mb, 0.0) / nb
    use = (sa + sb >= min_count) & (va + vb > 0)
    c2 = float(np.sum((ma[use] - mb[use]) ** 2 / (va[use] + vb[use])))
    dof = int(use.sum())
    return c2, dof, float(chi2_dist.sf(c2, dof))
