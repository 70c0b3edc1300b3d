"""The input side of the transport: ionisation-yield models, the energy partition of a
deposit into carriers and prompt phonons, and the hit merger for primary-particle steps
(charge/niel_models.hpp, charge/energy_partition.hpp). Everything runs natively on the
host (partition_host.cpp) with the reference's draw and operation order; the records it
returns are the initial stacks the device transport takes (PHONON_DTYPE / CHARGE_DTYPE)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Iterable, Optional, Sequence, Tuple

import numpy as np

from . import _ffi
from .api import CmpmcError, CrystalConfig, CrystalLattice, Rng, _check, units


class NIELModel(IntEnum):
    """physics::NIELModel (niel_models.hpp:28-34)."""
    Lindhard = 0
    LewinSmith = 1
    Sarkis = 2
    ImpactTUNL = 3
    Empirical = 4


@dataclass
class EmpiricalNIELParams:
    """physics::EmpiricalNIELParams (niel_models.hpp:36-43): CDMSlite k(E)."""
    energy_dependent_k: bool = True
    k_fixed: float = 0.157
    k_low: float = 0.080
    k_high: float = 0.157
    e_low_eV: float = 100.0 * units.eV
    e_high_eV: float = 2000.0 * units.eV


@dataclass
class PartitionOptions:
    """PartitionOptions (energy_partition.hpp:22-29)."""
    niel_model: NIELModel = NIELModel.Lindhard
    empirical_niel: EmpiricalNIELParams = field(default_factory=EmpiricalNIELParams)
    use_fano_fluctuations: bool = True
    use_charge_cloud: bool = True
    max_sampled_pairs: int = 1000
    max_sampled_phonons: int = 5000

    def to_c(self) -> _ffi.PartitionOptionsC:
        if self.max_sampled_pairs <= 0 or self.max_sampled_phonons <= 0:
            raise ValueError("max_sampled_pairs and max_sampled_phonons must be positive")
        e = self.empirical_niel
        return _ffi.PartitionOptionsC(int(self.niel_model), int(bool(self.use_fano_fluctuations)),
                                      int(bool(self.use_charge_cloud)), int(self.max_sampled_pairs),
                                      int(self.max_sampled_phonons), int(bool(e.energy_dependent_k)), float(e.k_fixed),
                                      float(e.k_low), float(e.k_high), float(e.e_low_eV), float(e.e_high_eV))


@dataclass
class PartitionResult:
    """EnergyPartition::Result (energy_partition.hpp:36-48)."""
    total_edep_eV: float = 0.0
    ionizing_eV: float = 0.0
    niel_eV: float = 0.0
    lindhard_yield: float = 1.0
    n_pairs_true: int = 0
    n_pairs_sampled: int = 0
    n_phonons_true: int = 0
    n_phonons_sampled: int = 0
    charge_weight: float = 1.0
    phonon_weight: float = 1.0
    prompt_phonon_eV: float = 0.0

    @staticmethod
    def from_c(r: _ffi.PartitionResultC) -> "PartitionResult":
        return PartitionResult(**{name: getattr(r, name) for name, _t in _ffi.PartitionResultC._fields_})


def _state(rng: Rng):
    return (C.c_uint64 * 4)(*rng.s)


class physics:
    """Yield models and the pair-number sampler (niel_models.hpp:43-263)."""

    @staticmethod
    def compute_ionization_yield(model: NIELModel, energy_eV: float, cfg: CrystalConfig,
                                 emp: Optional[EmpiricalNIELParams] = None) -> float:
        o = PartitionOptions(empirical_niel=emp or EmpiricalNIELParams()).to_c()
        c = cfg.to_c()
        return _ffi.load().cmpmc_ionization_yield(C.byref(c), int(model), float(energy_eV), C.byref(o))

    @staticmethod
    def lindhard_ionization_yield(energy_eV: float, cfg: CrystalConfig, z1: float = 0.0, a1: float = 0.0) -> float:
        c = cfg.to_c()
        return _ffi.load().cmpmc_lindhard_yield(C.byref(c), float(energy_eV), float(z1), float(a1))

    @staticmethod
    def lewin_smith_ionization_yield(energy_eV: float, cfg: CrystalConfig) -> float:
        return physics.compute_ionization_yield(NIELModel.LewinSmith, energy_eV, cfg)

    @staticmethod
    def sarkis_ionization_yield(energy_eV: float, cfg: CrystalConfig) -> float:
        return physics.compute_ionization_yield(NIELModel.Sarkis, energy_eV, cfg)

    @staticmethod
    def impact_tunl_ionization_yield(energy_eV: float, cfg: CrystalConfig) -> float:
        return physics.compute_ionization_yield(NIELModel.ImpactTUNL, energy_eV, cfg)

    @staticmethod
    def empirical_ionization_yield(energy_eV: float, cfg: CrystalConfig,
                                   emp: Optional[EmpiricalNIELParams] = None) -> float:
        return physics.compute_ionization_yield(NIELModel.Empirical, energy_eV, cfg, emp)

    @staticmethod
    def sample_fano_binomial(mean: float, fano: float, rng: Rng) -> int:
        st = _state(rng)
        n = _ffi.load().cmpmc_sample_fano_binomial(float(mean), float(fano), st)
        rng.s = list(st)
        return int(n)


class EnergyPartition:
    """EnergyPartition (energy_partition.hpp:31-171) of a lattice (which must outlive it)."""

    def __init__(self, lattice: CrystalLattice):
        self.lattice = lattice
        self._lib = _ffi.load()

    def lindhard_ionization_yield(self, energy_eV: float, z1: float = 0.0, a1: float = 0.0) -> float:
        return physics.lindhard_ionization_yield(energy_eV, self.lattice.config(), z1, a1)

    def partition_deposit(self, pos: Sequence[float], time_s: float, total_edep_eV: float,
                          is_nuclear_recoil: bool, rng: Rng, opts: Optional[PartitionOptions] = None
                          ) -> Tuple[PartitionResult, np.ndarray, np.ndarray]:
        """(result, charges, phonons): 2 n_pairs_sampled carriers (e-, h+ interleaved) and
        n_phonons_sampled prompt Debye phonons, drawn from rng (advanced in place)."""
        o = (opts or PartitionOptions()).to_c()
        q = (C.c_double * 3)(*pos)
        nc, nph = C.c_uint64(0), C.c_uint64(0)
        res = _ffi.PartitionResultC()
        cap_c = 2 * min(int(o.max_sampled_pairs), 4096)
        cap_p = min(int(o.max_sampled_phonons), 4096)
        for _ in range(2):
            ch = np.zeros(cap_c, dtype=_ffi.CHARGE_DTYPE)
            ph = np.zeros(cap_p, dtype=_ffi.PHONON_DTYPE)
            st = _state(rng)
            status = self._lib.cmpmc_partition_deposit(self.lattice._h, q, float(time_s), float(total_edep_eV),
                                                       int(bool(is_nuclear_recoil)), C.byref(o), st, ch.ctypes.data,
                                                       cap_c, C.byref(nc), ph.ctypes.data, cap_p, C.byref(nph),
                                                       C.byref(res))
            if status == 4:  # CMPMC_ERR_CAPACITY: nothing drawn, retry with the exact sizes
                cap_c, cap_p = int(nc.value), int(nph.value)
                continue
            _check(status, what="partition_deposit")
            rng.s = list(st)
            return PartitionResult.from_c(res), ch[:nc.value].copy(), ph[:nph.value].copy()
        raise CmpmcError("partition_deposit: capacity retry failed")


@dataclass
class PrimaryStepInput:
    """PrimaryStepInput (energy_partition.hpp:182-192)."""
    track_id: int = 1
    start_pos: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    end_pos: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    time_s: float = 0.0
    edep_eV: float = 0.0
    eniel_eV: float = 0.0
    is_charged: bool = True
    hit_boundary: bool = False
    track_stopped: bool = False

    def to_c(self) -> _ffi.PrimaryStepC:
        return _ffi.PrimaryStepC(int(self.track_id), int(bool(self.is_charged)), (C.c_double * 3)(*self.start_pos),
                                 (C.c_double * 3)(*self.end_pos), float(self.time_s), float(self.edep_eV),
                                 float(self.eniel_eV), int(bool(self.hit_boundary)), int(bool(self.track_stopped)))


class HitMerger:
    """HitMerger (energy_partition.hpp:229-323): merges the steps of a primary track within
    combining_step_length and partitions each merged deposit. The secondaries accumulate in
    the merger (the reference appends them to the caller's vectors); take() hands them over."""

    def __init__(self, lattice: CrystalLattice, combining_step_length_m: float = 1.0 * units.mm,
                 opts: Optional[PartitionOptions] = None):
        self._lib = _ffi.load()
        self.lattice = lattice  # kept alive: the merger points at its tables
        o = (opts or PartitionOptions()).to_c()
        h = C.c_void_p()
        _check(self._lib.cmpmc_hit_merger_create(lattice._h, float(combining_step_length_m), C.byref(o), C.byref(h)),
               what="hit merger")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.cmpmc_hit_merger_destroy(h)
            self._h = None

    def process_steps(self, steps: Iterable[PrimaryStepInput], rng: Rng) -> int:
        """process_step for each step in order; returns how many of them flushed."""
        arr = [s.to_c() for s in steps]
        buf = (_ffi.PrimaryStepC * max(1, len(arr)))(*arr)
        st = _state(rng)
        n = C.c_uint64(0)
        _check(self._lib.cmpmc_hit_merger_process_steps(self._h, buf, len(arr), st, C.byref(n)), what="process_step")
        rng.s = list(st)
        return int(n.value)

    def process_step(self, step: PrimaryStepInput, rng: Rng) -> bool:
        """HitMerger::process_step: True when the step flushed the accumulated deposit."""
        return self.process_steps([step], rng) == 1

    def flush(self, rng: Rng) -> PartitionResult:
        st = _state(rng)
        res = _ffi.PartitionResultC()
        _check(self._lib.cmpmc_hit_merger_flush(self._h, st, C.byref(res)), what="flush")
        rng.s = list(st)
        return PartitionResult.from_c(res)

    def take(self) -> Tuple[np.ndarray, np.ndarray]:
        """(charges, phonons) accumulated since the last take()."""
        nc, nph = C.c_uint64(0), C.c_uint64(0)
        status = self._lib.cmpmc_hit_merger_take(self._h, None, 0, C.byref(nc), None, 0, C.byref(nph))
        if status not in (0, 4):  # CMPMC_ERR_CAPACITY: the counts are set
            _check(status, what="take")
        ch = np.zeros(nc.value, dtype=_ffi.CHARGE_DTYPE)
        ph = np.zeros(nph.value, dtype=_ffi.PHONON_DTYPE)
        _check(self._lib.cmpmc_hit_merger_take(self._h, ch.ctypes.data, len(ch), C.byref(nc), ph.ctypes.data, len(ph),
                                               C.byref(nph)), what="take")
        return ch, ph


def partition_deposits_on_device(engine, deposits, rng_state, opts: Optional[PartitionOptions] = None,
                                 device: int = 0):
    """EnergyPartition::partition_deposit for every deposit on the engine's device
    (cmpmc_gpu_partition_deposits): deposit i draws from rng_state[i] (n x 4 uint64).
    deposits: a DEPOSIT_DTYPE array (pos, time_s, edep_eV, is_nuclear_recoil). Returns the
    CSR offsets and records of the carriers and phonons per deposit and the advanced
    generator states, as host arrays. Device buffers come from torch, which this helper
    imports; C callers pass their own device memory."""
    import torch
    lib = _ffi.load()
    dep = np.ascontiguousarray(deposits, dtype=_ffi.DEPOSIT_DTYPE)
    n = len(dep)
    st = np.ascontiguousarray(rng_state, dtype=np.uint64).reshape(n, 4)
    dev = f"cuda:{device}"
    t_dep = torch.from_numpy(dep.view(np.uint8).reshape(-1).copy()).to(dev)
    t_rng = torch.from_numpy(st.view(np.int64).copy()).to(dev)
    t_coff = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    t_poff = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    h = engine.context(device)
    o = (opts or PartitionOptions()).to_c()
    nc, nph = C.c_uint64(0), C.c_uint64(0)
    args = (h, t_dep.data_ptr(), n, C.byref(o), t_rng.data_ptr(), t_coff.data_ptr(), t_poff.data_ptr())
    status = lib.cmpmc_gpu_partition_deposits(*args, None, 0, None, 0, C.byref(nc), C.byref(nph))
    if status not in (0, 4):
        _check(status, h)
    t_ch = torch.zeros(max(1, nc.value) * 128, dtype=torch.uint8, device=dev)
    t_ph = torch.zeros(max(1, nph.value) * 128, dtype=torch.uint8, device=dev)
    _check(lib.cmpmc_gpu_partition_deposits(*args, t_ch.data_ptr(), nc.value, t_ph.data_ptr(), nph.value,
                                            C.byref(nc), C.byref(nph)), h)
    ch = t_ch.cpu().numpy().view(_ffi.CHARGE_DTYPE)[:nc.value].copy()
    ph = t_ph.cpu().numpy().view(_ffi.PHONON_DTYPE)[:nph.value].copy()
    return (t_coff.cpu().numpy().view(np.uint64), ch, t_poff.cpu().numpy().view(np.uint64), ph,
            t_rng.cpu().numpy().view(np.uint64).reshape(n, 4))

