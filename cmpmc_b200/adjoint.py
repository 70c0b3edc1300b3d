"""Adjoint of the binned sensor-arrival histogram with respect to four transport parameters.

theta = (B_iso, A_anh, p_d, f_abs):
  B_iso  isotope-scattering coefficient (CrystalConfig::B_iso, materials/crystal_config.hpp:71)
  A_anh  anharmonic-decay coefficient (CrystalConfig::A_anh, crystal_config.hpp:72)
  p_d    diffuse fraction of every surface: SurfaceProperty::reflection_split
         (geometry/surface_property.hpp:72-86) returns p_spec = 1 - p_d, p_diff = p_d, p_anh = 0
         when spec_coeffs = {1 - p_d}, diff_coeffs = {p_d}, anh_coeffs = {} and
         spec_prob_const = 1 - p_d, at every frequency
  f_abs  film entry probability (SuperconductorFilmConfig::film_absorption,
         crystal_config.hpp:241, used at transport/engine.hpp:495)

h_b(theta) is the weighted count of SensorHits whose time falls in bin b. Given bin weights
w_b = dLoss/dh_b, the device returns value = sum_b w_b h_b and d value / d theta from the
score-function estimator: each theta-dependent decision of a track (an exponential free
flight through the isotope and anharmonic channels, the specular/diffuse choice, film
entry) adds its d log p / d theta to the track's score, daughters start with their
parent's score, and each binned hit contributes w_b * score. The hit time is a function of
the sampled path alone, so with every theta-dependent draw scored it carries no extra
pathwise term. The backward call recomputes every track from its RNG substream.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _ffi
from .api import PackedEvents, SimStats, SimulationEngine, _check

THETA_NAMES = ("B_iso", "A_anh", "diffuse_fraction", "film_absorption")


@dataclass
class AdjointResult:
    hist: np.ndarray          # [n_bins] weighted hit counts
    value: float              # sum_b w_b hist_b
    grad: np.ndarray          # [4] d value / d theta
    value_var: float          # variance estimate of value (spread over primaries)
    grad_var: np.ndarray      # [4] variance estimates of grad
    stats: SimStats
    n_primaries: int
    kernel_ms: float
    total_ms: float
    kernel_launches: int
    per_primary: Optional[np.ndarray] = None  # [n_primaries, 5]: value, d value / d theta_k


def default_theta(engine: SimulationEngine, diffuse_fraction: float = 0.9) -> np.ndarray:
    """theta at the engine's lattice and film defaults; the default surfaces are fully
    diffuse (p_d = 1), on the boundary of the parameter range, so p_d is moved inside."""
    cfg = engine.lattice.config()
    films = [s.kaplan_sensor for s in engine.detector.surfaces if s.kaplan_sensor is not None]
    f_abs = films[0].film_absorption if films else 1.0
    return np.array([cfg.B_iso, cfg.A_anh, diffuse_fraction, f_abs], dtype=np.float64)


class HistogramAdjoint:
    """h(theta) and the adjoint of w . h(theta) for a fixed batch of primaries."""

    def __init__(self, engine: SimulationEngine, packed: PackedEvents, seed: int, n_bins: int = 64,
                 t_range: Sequence[float] = (0.0, 1e-3), device: int = 0):
        if not 1 <= n_bins <= _ffi.ADJ_MAX_BINS:
            raise ValueError(f"n_bins must be in [1, {_ffi.ADJ_MAX_BINS}]")
        self.engine = engine
        self.packed = packed
        self.seed = int(seed)
        self.n_bins = int(n_bins)
        self.t_range = (float(t_range[0]), float(t_range[1]))
        self.device = int(device)
        self._lib = _ffi.load()
        self._ph = packed.phonons if packed.phonons.size else np.zeros(1, dtype=_ffi.PHONON_DTYPE)

    @property
    def n_primaries(self) -> int:
        return int(self.packed.phonon_offsets[-1])

    def run(self, theta: Sequence[float], bin_weight: Optional[Sequence[float]] = None,
            per_primary: bool = False) -> AdjointResult:
        h = self.engine.context(self.device)
        d = _ffi.AdjointDescC()
        d.n_events = self.packed.n_events
        d.first_event = self.packed.first_event
        d.seed = self.seed
        d.phonon_offsets = self.packed.phonon_offsets.ctypes.data
        d.phonons = self._ph.ctypes.data
        d.n_bins = self.n_bins
        d.t_min, d.t_max = self.t_range
        for k in range(4):
            d.theta[k] = float(theta[k])
        w = None
        if bin_weight is not None:
            w = np.ascontiguousarray(bin_weight, dtype=np.float64)
            if w.shape != (self.n_bins,):
                raise ValueError("bin_weight must have n_bins entries")
            d.bin_weight = w.ctypes.data
        rows = None
        if per_primary:
            rows = np.zeros((max(self.n_primaries, 1), 5), dtype=np.float64)
            d.per_primary = rows.ctypes.data
        out = _ffi.AdjointOutC()
        _check(self._lib.cmpmc_gpu_adjoint(h, C.byref(d), C.byref(out)), h)
        stats = SimStats(np.frombuffer(bytes(out.stats), dtype=_ffi.STATS_DTYPE)[0])
        return AdjointResult(
            hist=np.array(out.hist[:self.n_bins]), value=out.value, grad=np.array(out.grad[:]),
            value_var=out.value_var, grad_var=np.array(out.grad_var[:]), stats=stats,
            n_primaries=int(out.n_primaries), kernel_ms=out.kernel_ms, total_ms=out.total_ms,
            kernel_launches=int(out.kernel_launches),
            per_primary=rows[:self.n_primaries] if rows is not None else None)

    def histogram(self, theta: Sequence[float]) -> np.ndarray:
        return self.run(theta).hist

    def loss_and_grad(self, theta: Sequence[float], target: np.ndarray):
        """Loss sum_b (h_b(theta) - target_b)^2 and its gradient: the forward pass gives h,
        the backward pass replays the tracks with w = 2 (h - target)."""
        hist = self.histogram(theta)
        w = 2.0 * (hist - target)
        res = self.run(theta, w)
        return float(np.sum((hist - target) ** 2)), res.grad, res
