"""Regenerates tests/golden/adjoint_c4.npz: the CPU side of the adjoint checks.

Runs oracle/_ref/adjoint_ref (built by `make -C oracle ref` from the unmodified reference
headers) on events of the single-L-phonon volume workload (one L phonon of 7.5 meV per
event, origin uniform in the cylinder, isotropic; seed 17):

  check      the CPU restatement of the transport loop reproduces the reference's hits bit
             for bit on N_CHECK events (its score bookkeeping rides on an exact copy of the
             reference's decisions)
  hist0/hist_target   the reference's hit-time histograms (64 bins over [0, 1 ms]) at theta0
             and at 1.1 theta0 on N events
  w          fixed bin weights 2 (hist0 - hist_target) / N (the loss gradient per primary)
  est_*      the score-function estimator on the restated loop at theta0 with weights w:
             per-primary mean and standard error of value = sum_b w_b h_b and of
             d value / d theta_k
  fd_*       central finite differences with common random numbers on the reference's own
             transport: per-primary mean and standard error of
             (value(theta_k (1 + step)) - value(theta_k (1 - step))) / (2 step theta_k)

theta0 = (B_iso, A_anh, p_d, f_abs) = (3.67e-41, 6.43e-55, 0.9, 0.2): the germanium defaults,
the default film absorption, and p_d moved from the default 1 (pure diffuse, on the edge of
the range) to 0.9 so that both +-10 % and the finite-difference steps stay inside (0, 1].

Usage: python tests/golden/make_adjoint_golden.py   (needs the reference build; ~4 min on 8 cores)
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "adjoint_ref")

THETA0 = np.array([3.67e-41, 6.43e-55, 0.9, 0.2])
SCALE_TARGET = 1.1
N_BINS = 64
T_MAX = 1e-3
N = 200_000
N_CHECK = 20_000
FD_STEP = 1e-3


def _run(cmd: str, theta, n: int, weights: np.ndarray | None, cols: int, tmp: str):
    wpath = "-"
    if weights is not None:
        wpath = os.path.join(tmp, "w.bin")
        np.asarray(weights, dtype=np.float64).tofile(wpath)
    out = os.path.join(tmp, "out.bin")
    args = [EXE, cmd] + [repr(float(t)) for t in theta] + ["0", str(n), "0", str(N_BINS), repr(T_MAX), wpath, out]
    subprocess.run(args, check=True)
    raw = np.fromfile(out, dtype=np.float64)
    return raw[:N_BINS], raw[N_BINS:].reshape(n, cols)


def main() -> None:
    if not os.path.exists(EXE):
        sys.exit("build the reference first: make -C oracle ref")
    chk = subprocess.run([EXE, "check"] + [repr(float(t)) for t in THETA0] + ["0", str(N_CHECK), "0"],
                         check=True, capture_output=True, text=True).stdout
    check = json.loads(chk)
    assert check["mismatched_events"] == 0, check
    with tempfile.TemporaryDirectory() as tmp:
        hist0, _ = _run("values", THETA0, N, None, 1, tmp)
        hist_t, _ = _run("values", THETA0 * SCALE_TARGET, N, None, 1, tmp)
        w = 2.0 * (hist0 - hist_t) / N
        _, rows = _run("estimate", THETA0, N, w, 5, tmp)
        est_mean = rows.mean(axis=0)
        est_se = rows.std(axis=0, ddof=1) / np.sqrt(N)
        fd_mean, fd_se = np.zeros(4), np.zeros(4)
        for k in range(4):
            tp, tm = THETA0.copy(), THETA0.copy()
            tp[k] *= 1.0 + FD_STEP
            tm[k] *= 1.0 - FD_STEP
            _, vp = _run("values", tp, N, w, 1, tmp)
            _, vm = _run("values", tm, N, w, 1, tmp)
            c = (vp[:, 0] - vm[:, 0]) / (2.0 * FD_STEP * THETA0[k])
            fd_mean[k] = c.mean()
            fd_se[k] = c.std(ddof=1) / np.sqrt(N)
    np.savez_compressed(os.path.join(HERE, "adjoint_c4.npz"), theta0=THETA0, scale_target=SCALE_TARGET,
                        n_bins=N_BINS, t_max=T_MAX, n=N, fd_step=FD_STEP, check_events=check["events"],
                        check_mismatched=check["mismatched_events"], hist0=hist0, hist_target=hist_t, w=w,
                        est_mean=est_mean, est_se=est_se, fd_mean=fd_mean, fd_se=fd_se)
    for k in range(4):
        z = (est_mean[1 + k] - fd_mean[k]) / np.hypot(est_se[1 + k], fd_se[k])
        print(f"theta_{k}: estimator {est_mean[1 + k]:.6g} +- {est_se[1 + k]:.3g}   "
              f"FD {fd_mean[k]:.6g} +- {fd_se[k]:.3g}   z = {z:.2f}")


if __name__ == "__main__":
    main()
