"""Host-side parts of bench.py, without a device: the matched-statistics summary of the bench
line (chi^2 of per-event hit histograms and ledger closures) and the reference arm, which
runs the reference's own CPU run_events through the oracle program."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tests.helpers import ROOT
from tests.golden.records import HIT_DTYPE

sys.path.insert(0, ROOT)


def _fake_result(seed: int, n_events: int = 400, per_event: int = 30) -> dict:
    """hits of one process: times exponential, radii uniform in area, energies uniform"""
    g = np.random.default_rng(seed)
    counts = g.poisson(per_event, n_events).astype(np.uint64)
    offs = np.zeros(n_events + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(counts)
    n = int(offs[-1])
    hits = np.zeros(n, dtype=HIT_DTYPE)
    r = 0.0381 * np.sqrt(g.random(n))
    phi = 2 * np.pi * g.random(n)
    hits["pos"][:, 0], hits["pos"][:, 1] = r * np.cos(phi), r * np.sin(phi)
    hits["time"] = g.exponential(3e-4, n)
    hits["edep"] = g.uniform(1e-4, 3e-2, n)
    dep = float(hits["edep"].sum())
    return {"offsets": offs, "hits": hits, "injected": 2.0 * dep, "deposited": dep, "escaped": dep}


def test_matched_statistics_of_one_process():
    import bench
    a, b, c = _fake_result(1), _fake_result(2), _fake_result(3)
    out = bench.matched_statistics(a, b, 1, c)  # first_event 1: no reference fixture comparison
    assert out["events"] == 400 and out["batched_hits"] == len(a["hits"])
    for key in ("p_vs_plain_fp64", "p_vs_batched_fp64"):
        assert set(out[key]) == {"time", "radius", "edep"}
        assert all(0.0 <= p <= 1.0 for p in out[key].values())
        # two samples of one process: no histogram may look different at the 1e-3 level
        assert min(out[key].values()) > 1e-3, out[key]
    assert out["ledger_closure_batched"] == 0.0 and out["ledger_closure_plain_fp64"] == 0.0
    assert "p_vs_reference_cpu" not in out


def test_matched_statistics_detects_a_shift():
    import bench
    a, b = _fake_result(1), _fake_result(2)
    b["hits"]["time"] *= 1.2  # a 20 % slower process
    out = bench.matched_statistics(a, b, 1)
    assert out["p_vs_plain_fp64"]["time"] < 1e-6
    assert out["p_vs_plain_fp64"]["radius"] > 1e-3


def test_reference_arm_prints_the_metric():
    exe = os.path.join(ROOT, "oracle", "_ref", "cmpmc_ref")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/cmpmc_ref not built (make -C oracle ref needs the reference headers)")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--ref-events", "20"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["unit"] == "primary phonon tracks/s" and line["warmup"] >= 3
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
