"""Python mirror of CMPMC's transport API, running on the B200 through the C ABI.

Names, fields and defaults follow the reference's C++ API so that code and tests read the
same: CrystalConfig / materials.Germanium (materials/crystal_config.hpp, presets.hpp),
CrystalLattice (lattice/crystal_lattice.hpp), SurfaceProperty (geometry/surface_property.hpp),
DetectorModel and SimulationEngine (transport/engine.hpp), EventInput / RunOptions /
RunResult / run_events (transport/parallel.hpp), Rng (core/rng.hpp).

run_events runs the generator on the host, one Rng.for_stream(seed, i) per event, exactly
as the reference does (parallel.hpp:102-109), then transports every event on the device.
The generator is either a Python callable taking an EventInput (as in the reference), or a
`Workload` naming one of the canonical generators, which run in the native library.
"""
from __future__ import annotations

import copy
import ctypes as C
import math
import os
import time
from dataclasses import dataclass, field, replace
from enum import IntEnum
from typing import Callable, Optional, Sequence

import numpy as np

from . import _ffi

# ---- units (core/units.hpp:26-72) -------------------------------------------------------


class units:
    pi = math.pi
    two_pi = 2.0 * math.pi
    half_pi = 0.5 * math.pi
    m, cm, mm, um, nm = 1.0, 1e-2, 1e-3, 1e-6, 1e-9
    s, ms, us, ns, ps = 1.0, 1e-3, 1e-6, 1e-9, 1e-12
    Hz, MHz, GHz, THz = 1.0, 1e6, 1e9, 1e12
    eV, keV, MeV, meV, ueV = 1.0, 1e3, 1e6, 1e-3, 1e-6
    GPa = 1e9
    c_light = 299792458.0
    h_Planck = 4.135667696e-15
    hbar_Planck = 6.582119569e-16
    hbarc = hbar_Planck * c_light
    k_Boltzmann = 8.617333262e-5


class PhononMode(IntEnum):
    L = 0
    FT = 1
    ST = 2


class SurfaceId(IntEnum):
    TopFace = 0
    BottomFace = 1
    SideWall = 2


class ExcitationType(IntEnum):
    Phonon = 0
    Electron = 1
    Hole = 2


class UnvalidatedModuleError(Exception):
    """A guarded (experimental) module was used without allow_unvalidated
    (core/validation.hpp:20-29)."""


class CmpmcError(RuntimeError):
    """A device-side failure reported through the C ABI."""


def _check(status: int, ctx=None, what: str = "") -> None:
    if status == _ffi.OK:
        return
    lib = _ffi.load()
    buf = C.create_string_buffer(1024)
    lib.cmpmc_gpu_last_error(ctx, buf, len(buf))
    msg = buf.value.decode() or what
    if status == _ffi.ERR_UNVALIDATED:
        raise UnvalidatedModuleError(msg)
    raise CmpmcError(f"status {status}: {msg}")


# ---- Rng (core/rng.hpp:17-97) -------------------------------------------------------------

_M64 = (1 << 64) - 1


def _splitmix(x: int) -> int:
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M64
    return x ^ (x >> 31)


def _mix64(x: int) -> int:
    return _splitmix((x + 0x9E3779B97F4A7C15) & _M64)


class Rng:
    """xoshiro256** with splitmix64 seeding; bit-identical to the reference's Rng."""

    __slots__ = ("s",)

    def __init__(self, seed: int = 0x853C49E6748FEA9B):
        z = seed & _M64
        s = []
        for _ in range(4):
            z = (z + 0x9E3779B97F4A7C15) & _M64
            s.append(_splitmix(z))
        self.s = s

    @staticmethod
    def for_stream(seed: int, stream: int) -> "Rng":
        return Rng(_mix64(seed & _M64) ^ _mix64((stream + 0x632BE59BD9B4E019) & _M64))

    @classmethod
    def from_state(cls, state: Sequence[int]) -> "Rng":
        r = cls.__new__(cls)
        r.s = [int(x) & _M64 for x in state]
        return r

    def next_u64(self) -> int:
        s = self.s
        x = (s[1] * 5) & _M64
        result = ((((x << 7) | (x >> 57)) & _M64) * 9) & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = ((s[3] << 45) | (s[3] >> 19)) & _M64
        return result

    def uniform(self, a: Optional[float] = None, b: Optional[float] = None) -> float:
        u = float((self.next_u64() >> 11) | 1) * (1.0 / 9007199254740992.0)
        if a is None:
            return u
        return a + (b - a) * u

    def normal(self) -> float:
        u1 = self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(units.two_pi * u2)

    def isotropic_dir(self) -> tuple[float, float, float]:
        ct = 2.0 * self.uniform() - 1.0
        st = math.sqrt(max(0.0, 1.0 - ct * ct))
        phi = units.two_pi * self.uniform()
        return (st * math.cos(phi), st * math.sin(phi), ct)

    def lambertian_dir(self, n: Sequence[float]) -> tuple[float, float, float]:
        phi = units.two_pi * self.uniform()
        st = math.sqrt(self.uniform())
        ct = math.sqrt(max(0.0, 1.0 - st * st))
        a = (1.0, 0.0, 0.0) if abs(n[0]) < 0.9 else (0.0, 1.0, 0.0)
        u = _unit(_cross(n, a))
        v = _cross(n, u)
        cp, sp = st * math.cos(phi), st * math.sin(phi)
        return _unit(tuple(u[i] * cp + v[i] * sp + n[i] * ct for i in range(3)))


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _unit(a):
    n2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2]
    if n2 <= 0.0:
        return (0.0, 0.0, 1.0)
    inv = 1.0 / math.sqrt(n2)
    return (a[0] * inv, a[1] * inv, a[2] * inv)


# ---- configuration -------------------------------------------------------------------------


@dataclass
class CrystalConfig:
    """CrystalConfig (materials/crystal_config.hpp:43-226); SI units, energies in eV."""
    name: str = "Ge"
    group: int = 1
    density: float = 5323.0
    C11: float = 126.0 * units.GPa
    C12: float = 44.0 * units.GPa
    C13: float = 0.0
    C14: float = 0.0
    C16: float = 0.0
    C33: float = 0.0
    C44: float = 67.0 * units.GPa
    C66: float = 0.0
    C_custom: Optional[np.ndarray] = None
    beta: float = -73.2 * units.GPa
    gamma: float = -70.8 * units.GPa
    lambda_: float = 37.6 * units.GPa
    mu: float = 56.1 * units.GPa
    B_iso: float = 3.67e-41
    A_anh: float = 6.43e-55
    fTT_frac: float = 0.74
    polycrystal_mfp_m: float = 0.0
    fLDOS: float = 0.097834
    fSTDOS: float = 0.535390
    fFTDOS: float = 0.366770
    debye_freq: float = 2.0 * units.THz
    v_sound: float = 5324.2077
    v_trans: float = 3258.7879
    bandgap: float = 0.74
    pair_energy: float = 2.96
    fano_factor: float = 0.1057
    epsilon_rel: float = 16.2
    neutral_impurity_cm3: float = 1.0e11
    alpha_nonparabolic: float = 0.3
    h_mass_ratio: float = 0.350
    e_mass_tensor: tuple = (1.588, 0.081, 0.081)
    valley_dirs: tuple = ((1, 1, 1), (-1, 1, 1), (-1, -1, 1), (1, -1, 1))
    ac_deform_e: float = 11.0
    ac_deform_h: float = 3.4
    iv_deform_eV_m: tuple = (3.0e10, 0.2e10)
    iv_energy_eV: tuple = (27.3 * units.meV, 10.3 * units.meV)
    iv_min_energy: float = 10.3 * units.meV
    iv_model: int = 0
    iv_quad_rate: float = 6.72e-2
    iv_quad_field: float = 217.0
    iv_quad_power: float = 3.24
    iv_lin_rate0: float = 1.5e6
    iv_lin_rate1: float = 1.5
    iv_lin_power: float = 4.0
    e_trapping_mfp_m: float = 0.0
    h_trapping_mfp_m: float = 0.0
    e_trap_ion_d0_mfp_m: float = 0.0
    e_trap_ion_a_mfp_m: float = 0.0
    h_trap_ion_d_mfp_m: float = 0.0
    h_trap_ion_a0_mfp_m: float = 0.0
    orient: tuple = ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0))
    atomic_Z: float = 32.0
    atomic_A: float = 72.63

    def to_c(self) -> _ffi.CrystalConfigC:
        c = _ffi.CrystalConfigC()
        for f, _t in _ffi.CrystalConfigC._fields_:
            if f in ("C_custom", "has_custom_C", "e_mass_tensor", "valley_dirs", "n_valleys", "iv_deform_eV_m",
                     "iv_energy_eV", "n_iv", "orient", "_pad0"):
                continue
            setattr(c, f, getattr(self, f))
        if self.C_custom is not None:
            c.has_custom_C = 1
            for i in range(6):
                for j in range(6):
                    c.C_custom[i][j] = float(self.C_custom[i][j])
        for i in range(3):
            c.e_mass_tensor[i] = self.e_mass_tensor[i]
        if len(self.valley_dirs) > _ffi.MAX_VALLEYS:
            raise ValueError("too many valleys")
        c.n_valleys = len(self.valley_dirs)
        for k, d in enumerate(self.valley_dirs):
            for i in range(3):
                c.valley_dirs[k][i] = float(d[i])
        n_iv = min(len(self.iv_deform_eV_m), len(self.iv_energy_eV), _ffi.MAX_IV)
        c.n_iv = n_iv
        for i in range(n_iv):
            c.iv_deform_eV_m[i] = self.iv_deform_eV_m[i]
            c.iv_energy_eV[i] = self.iv_energy_eV[i]
        for i in range(3):
            for j in range(3):
                c.orient[i][j] = float(self.orient[i][j])
        return c


class materials:
    @staticmethod
    def Germanium() -> CrystalConfig:
        """presets.hpp:18-25: defaults with the Debye frequency 8.64 THz."""
        return CrystalConfig(debye_freq=8.64 * units.THz)


@dataclass
class SuperconductorFilmConfig:
    """SuperconductorFilmConfig (crystal_config.hpp:240-257)."""
    film_absorption: float = 0.20
    film_thickness: float = 600.0 * units.nm
    v_sound: float = 3260.0
    gap_energy: float = 173.715 * units.ueV
    phonon_lifetime: float = 242.0 * units.ps
    phonon_lifetime_slope: float = 0.29
    low_qp_limit: float = 3.0
    high_qp_limit: float = 0.0
    subgap_absorption: float = 0.10
    absorber_gap: float = 0.0
    absorber_eff: float = 1.0
    absorber_eff_slope: float = 0.0
    temperature: float = 0.05e-3
    keep_all_phonons: bool = True
    loss_model: int = 0
    phonon_loss_time: float = 0.0

    def to_c(self) -> _ffi.FilmConfigC:
        f = _ffi.FilmConfigC()
        for name, _t in _ffi.FilmConfigC._fields_:
            v = getattr(self, name)
            setattr(f, name, int(v) if name in ("keep_all_phonons", "loss_model") else float(v))
        return f


KaplanFilm = SuperconductorFilmConfig


def AluminumFilm() -> SuperconductorFilmConfig:
    return SuperconductorFilmConfig()


@dataclass
class IsotropicMedium:
    """IsotropicMedium (phonon/interface_transmission.hpp:36-49)."""
    rho: float = 0.0
    vL: float = 0.0
    vT: float = 0.0

    @staticmethod
    def from_lame(rho: float, lam_Pa: float, mu_Pa: float) -> "IsotropicMedium":
        return IsotropicMedium(rho, math.sqrt((lam_Pa + 2.0 * mu_Pa) / rho), math.sqrt(mu_Pa / rho))

    @staticmethod
    def from_bulk_shear(rho: float, K_Pa: float, G_Pa: float) -> "IsotropicMedium":
        return IsotropicMedium(rho, math.sqrt((K_Pa + 4.0 * G_Pa / 3.0) / rho), math.sqrt(G_Pa / rho))


@dataclass
class IsotropicAMMInterface:
    """IsotropicAMMInterface (phonon/interface_transmission.hpp:123-140): acoustic-mismatch
    transmission substrate -> film; on a SurfaceProperty it replaces the film's
    film_absorption as the film-entry probability."""
    substrate: IsotropicMedium = field(default_factory=IsotropicMedium)
    film: IsotropicMedium = field(default_factory=IsotropicMedium)

    def transmission(self, longitudinal: bool, cos_theta: float) -> float:
        sub = (C.c_double * 3)(self.substrate.rho, self.substrate.vL, self.substrate.vT)
        fil = (C.c_double * 3)(self.film.rho, self.film.vL, self.film.vT)
        return _ffi.load().cmpmc_amm_transmission(sub, fil, int(bool(longitudinal)), float(cos_theta))


class KaplanSurrogateLUT:
    """KaplanSurrogateLUT (superconductor/kaplan_film.hpp:336-383), built natively on the
    host; the batched form uses the same table on the device (RunOptions.kaplan_surrogate)."""

    def __init__(self, film: "SuperconductorFilmConfig", seed: int = 1337):
        self._lib = _ffi.load()
        self._film = film.to_c()
        h = C.c_void_p()
        _check(self._lib.cmpmc_kaplan_surrogate_create(C.byref(self._film), int(seed), C.byref(h)), what="surrogate")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.cmpmc_kaplan_surrogate_destroy(h)
            self._h = None

    def absorb_phonon_fast(self, energy: float, rng: "Rng"):
        """(absorbed energy, re-emitted energies), drawing from rng like the reference."""
        st = (C.c_uint64 * 4)(*rng.s)
        buf = (C.c_double * 256)()
        n, e = C.c_uint64(), C.c_double()
        _check(self._lib.cmpmc_kaplan_surrogate_absorb(self._h, float(energy), st, buf, 256, C.byref(n), C.byref(e)))
        rng.s = list(st)
        return e.value, list(buf[:n.value])


@dataclass
class ElectrodePad:
    """ElectrodePad (geometry/electrode_pattern.hpp:23-63). shape: 0 disk, 1 annular sector,
    2 rectangle (r_min / r_max are then the half-width / half-height)."""
    shape: int = 0
    channel_id: int = 0
    cx: float = 0.0
    cy: float = 0.0
    r_min: float = 0.0
    r_max: float = 0.0
    phi_min: float = 0.0
    phi_max: float = units.two_pi
    fill_fraction: float = 1.0

    Disk, AnnularSector, Rectangle = 0, 1, 2

    def to_c(self) -> _ffi.ElectrodePadC:
        return _ffi.ElectrodePadC(int(self.shape), int(self.channel_id), self.cx, self.cy, self.r_min, self.r_max,
                                  self.phi_min, self.phi_max, self.fill_fraction)


class ElectrodePatternMask:
    """ElectrodePatternMask (geometry/electrode_pattern.hpp:65-187): readout pads on a face;
    attached to a SurfaceProperty as electrode_mask and evaluated on the device."""

    def __init__(self, pads=None):
        self.pads = list(pads or [])

    def empty(self) -> bool:
        return not self.pads

    def num_pads(self) -> int:
        return len(self.pads)

    def add_pad(self, pad: ElectrodePad) -> None:
        self.pads.append(pad)

    def to_c(self):
        arr = (_ffi.ElectrodePadC * max(len(self.pads), 1))()
        for i, p in enumerate(self.pads):
            arr[i] = p.to_c()
        return arr

    @staticmethod
    def _from_c(arr, n) -> "ElectrodePatternMask":
        return ElectrodePatternMask([ElectrodePad(a.shape, a.channel_id, a.cx, a.cy, a.r_min, a.r_max, a.phi_min,
                                                  a.phi_max, a.fill_fraction) for a in arr[:n]])

    @staticmethod
    def supercdms_qet_mask(crystal_radius_m: float, fill_fraction: float = 1.0) -> "ElectrodePatternMask":
        arr = (_ffi.ElectrodePadC * 5)()
        _check(_ffi.load().cmpmc_mask_supercdms_qet(crystal_radius_m, fill_fraction, arr))
        return ElectrodePatternMask._from_c(arr, 5)

    @staticmethod
    def rectangular_grid_mask(nx: int, ny: int, pitch_x: float, pitch_y: float, pad_half_w: float,
                              pad_half_h: float, fill_fraction: float = 1.0) -> "ElectrodePatternMask":
        n = max(nx * ny, 1)
        arr = (_ffi.ElectrodePadC * n)()
        cnt = C.c_uint64()
        _check(_ffi.load().cmpmc_mask_rectangular_grid(nx, ny, pitch_x, pitch_y, pad_half_w, pad_half_h,
                                                       fill_fraction, arr, n, C.byref(cnt)))
        return ElectrodePatternMask._from_c(arr, cnt.value)

    def find_channel(self, pos, rng: "Rng") -> int:
        """The channel at (pos.x, pos.y), drawing from rng like the reference (host)."""
        st = (C.c_uint64 * 4)(*rng.s)
        ch = C.c_int32()
        q = (C.c_double * 3)(*pos)
        _check(_ffi.load().cmpmc_mask_find_channel(self.to_c(), len(self.pads), q, st, C.byref(ch)))
        rng.s = list(st)
        return ch.value


@dataclass
class SurfaceProperty:
    """SurfaceProperty (geometry/surface_property.hpp:23-45); interface models are not
    available on the device."""
    prob_abs: float = 0.0
    prob_refl: float = 1.0
    refl_cutoff: float = 350.0
    anh_cutoff: float = 520.0
    prob_charge_abs: float = 1.0
    prob_charge_spec: float = 0.0
    min_k_elec: float = 0.0
    min_k_hole: float = 0.0
    spec_coeffs: tuple = (1.0,)
    diff_coeffs: tuple = (0.0,)
    anh_coeffs: tuple = (0.0,)
    kaplan_sensor: Optional[SuperconductorFilmConfig] = None
    spec_prob_const: float = 0.0
    demo_values: bool = False
    electrode_mask: Optional[ElectrodePatternMask] = None
    amm_interface: Optional[IsotropicAMMInterface] = None

    @staticmethod
    def diffuse_bare_surface() -> "SurfaceProperty":
        return SurfaceProperty(prob_abs=0.0, prob_refl=1.0, spec_coeffs=(0.0,), diff_coeffs=(1.0,),
                               anh_coeffs=(), spec_prob_const=0.0)

    @staticmethod
    def diffuse_al_sensor_surface() -> "SurfaceProperty":
        s = SurfaceProperty.diffuse_bare_surface()
        s.prob_abs = 1.0
        s.kaplan_sensor = AluminumFilm()
        return s

    @staticmethod
    def demo_polynomial_bare_surface() -> "SurfaceProperty":
        return SurfaceProperty(prob_abs=0.0, prob_refl=1.0, anh_cutoff=520.0, refl_cutoff=350.0,
                               spec_coeffs=(0.928, -2.03e-4, -3.21e-6, 3.1e-9, 2.9e-13),
                               diff_coeffs=(5.88e-2, 7.83e-4, -2.47e-6, 1.71e-8, -2.98e-11),
                               anh_coeffs=(0.0, 0.0, 0.0, 0.0, 0.0, 1.51e-14), demo_values=True)

    @staticmethod
    def demo_polynomial_sensor_surface() -> "SurfaceProperty":
        s = SurfaceProperty.demo_polynomial_bare_surface()
        s.prob_abs = 1.0
        s.kaplan_sensor = AluminumFilm()
        return s

    def to_c(self) -> _ffi.SurfaceC:
        s = _ffi.SurfaceC()
        for name in ("prob_abs", "prob_refl", "refl_cutoff", "anh_cutoff", "prob_charge_abs", "prob_charge_spec",
                     "min_k_elec", "min_k_hole", "spec_prob_const"):
            setattr(s, name, float(getattr(self, name)))
        for name, dst, cnt in (("spec_coeffs", "spec_coeffs", "n_spec"), ("diff_coeffs", "diff_coeffs", "n_diff"),
                               ("anh_coeffs", "anh_coeffs", "n_anh")):
            v = list(getattr(self, name))
            if len(v) > _ffi.MAX_POLY:
                raise ValueError(f"{name}: at most {_ffi.MAX_POLY} coefficients")
            setattr(s, cnt, len(v))
            arr = getattr(s, dst)
            for i, x in enumerate(v):
                arr[i] = float(x)
        s.demo_values = int(self.demo_values)
        if self.amm_interface is not None:
            s.has_amm = 1
            m1, m2 = self.amm_interface.substrate, self.amm_interface.film
            for i, v in enumerate((m1.rho, m1.vL, m1.vT)):
                s.amm_substrate[i] = float(v)
            for i, v in enumerate((m2.rho, m2.vL, m2.vT)):
                s.amm_film[i] = float(v)
        if self.kaplan_sensor is not None:
            s.has_film = 1
            s.film = self.kaplan_sensor.to_c()
        return s


@dataclass
class UniformElectricField:
    """UniformElectricField (charge/charge_transport.hpp:19-33)."""
    field_Vm: tuple = (0.0, 0.0, 0.0)

    @staticmethod
    def from_bias(bias_volts: float, thickness_m: float) -> "UniformElectricField":
        return UniformElectricField((0.0, 0.0, -bias_volts / thickness_m))


@dataclass
class CylinderSolid:
    """CylinderSolid (geometry/solids.hpp:23-26)."""
    radius: float = 3.81 * units.cm
    half_z: float = 1.27 * units.cm


def _default_surfaces():
    return [SurfaceProperty.diffuse_al_sensor_surface(), SurfaceProperty.diffuse_al_sensor_surface(),
            SurfaceProperty.diffuse_bare_surface()]


class TriLinearMesh3D:
    """TriLinearMesh3D (geometry/mesh_field.hpp:40-345): a tetrahedral mesh of node
    potentials whose field is constant inside each tetrahedron. Built on the host by the
    native library (face neighbours, inverse edge matrices and fields with the reference's
    arithmetic); attached to a DetectorModel as mesh_field_3d it is copied to the device and
    walked there by every charge step."""

    def __init__(self, vertices=None, potentials=None, tetrahedra=None, V_min_clamp: float = -1e30,
                 V_max_clamp: float = 1e30, _handle=None):
        self._lib = _ffi.load()
        self._hint = C.c_int32(0)
        if _handle is not None:
            self._h = _handle
            return
        x = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(potentials, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(tetrahedra, dtype=np.int32).reshape(-1, 4)
        if len(v) != len(x):
            raise ValueError("one potential per vertex")
        h = C.c_void_p()
        _check(self._lib.cmpmc_mesh_create(x.ctypes.data, v.ctypes.data, len(x), t.ctypes.data, len(t),
                                           float(V_min_clamp), float(V_max_clamp), C.byref(h)), what="mesh")
        self._h = h

    @staticmethod
    def build_cartesian_grid(half_x: float, half_y: float, half_z: float, nx: int, ny: int, nz: int,
                             potential_fn: Callable) -> "TriLinearMesh3D":
        """Kuhn-triangulated box, 6 tetrahedra per cell (mesh_field.hpp:131-189);
        potential_fn((x, y, z)) gives the node potential in volts."""
        lib = _ffi.load()
        cb = _ffi.POTENTIAL_FN(lambda p, _u: float(potential_fn((p[0], p[1], p[2]))))
        h = C.c_void_p()
        _check(lib.cmpmc_mesh_build_cartesian(half_x, half_y, half_z, nx, ny, nz, cb, None, C.byref(h)),
               what="mesh")
        return TriLinearMesh3D(_handle=h)

    @staticmethod
    def load_from_files(coords_file: str, tets_file: str, coord_unit_m: float = 1.0,
                        potential_unit_V: float = 1.0) -> "TriLinearMesh3D":
        """G4CMP-style ASCII mesh (mesh_field.hpp:190-231): "x y z V" node lines and
        "i0 i1 i2 i3" tetrahedron lines, '#' / '%' comments; parsed natively. A file that
        cannot be opened gives an empty mesh, as in the reference."""
        lib = _ffi.load()
        h = C.c_void_p()
        _check(lib.cmpmc_mesh_load_files(os.fsencode(coords_file), os.fsencode(tets_file), float(coord_unit_m),
                                         float(potential_unit_V), C.byref(h)), what="mesh")
        return TriLinearMesh3D(_handle=h)

    @staticmethod
    def recoil_mesh(detector: "DetectorModel") -> "TriLinearMesh3D":
        """The recoil workloads' mesh: build_cartesian_grid(R, R, h, 58, 58, 57) with
        V = 4 V (z + h) / 2h + 0.2 V (r / R)^2 sin(pi z / 2h), built natively."""
        lib = _ffi.load()
        cdet = detector.to_c()
        h = C.c_void_p()
        _check(lib.cmpmc_recoil_mesh(C.byref(cdet), C.byref(h)), what="mesh")
        return TriLinearMesh3D(_handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.cmpmc_mesh_destroy(h)
            self._h = None

    def _info(self):
        nv, nt = C.c_uint64(), C.c_uint64()
        _check(self._lib.cmpmc_mesh_info(self._h, C.byref(nv), C.byref(nt)))
        return nv.value, nt.value

    def num_vertices(self) -> int:
        return self._info()[0]

    def num_tetrahedra(self) -> int:
        return self._info()[1]

    def empty(self) -> bool:
        return self.num_tetrahedra() == 0

    def field_at(self, p, tet_hint: Optional[C.c_int32] = None):
        """E(p) in V/m from the containing tetrahedron (zero outside); the walk starts from
        and updates tet_hint (a ctypes int32), or the mesh's own hint (as at())."""
        hint = self._hint if tet_hint is None else tet_hint
        q = (C.c_double * 3)(*p)
        e = (C.c_double * 3)()
        _check(self._lib.cmpmc_mesh_field_at(self._h, q, C.byref(hint), e))
        return (e[0], e[1], e[2])

    def potential_at(self, p, tet_hint: Optional[C.c_int32] = None) -> float:
        hint = self._hint if tet_hint is None else tet_hint
        q = (C.c_double * 3)(*p)
        v = C.c_double()
        _check(self._lib.cmpmc_mesh_potential_at(self._h, q, C.byref(hint), C.byref(v)))
        return v.value

    def at(self, p):
        return self.field_at(p)


class BiLinearMesh2D:
    """BiLinearMesh2D (geometry/mesh_field.hpp:347-582): a triangle mesh in (r, z) for an
    axisymmetric field (rotated back around the z axis) or in (x, y) for a planar one, the
    field constant inside each triangle. Built on the host by the native library with the
    reference's arithmetic; attached to a DetectorModel as mesh_field_2d (and no 3D mesh)
    it is copied to the device and walked there by every charge step."""

    def __init__(self, vertices=None, potentials=None, triangles=None, axisymmetric_rz: bool = True,
                 _handle=None):
        self._lib = _ffi.load()
        self._hint = C.c_int32(0)
        if _handle is not None:
            self._h = _handle
            return
        x = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 2)
        v = np.ascontiguousarray(potentials, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(triangles, dtype=np.int32).reshape(-1, 3)
        if len(v) != len(x):
            raise ValueError("one potential per vertex")
        h = C.c_void_p()
        _check(self._lib.cmpmc_mesh2d_create(x.ctypes.data, v.ctypes.data, len(x), t.ctypes.data, len(t),
                                             int(bool(axisymmetric_rz)), C.byref(h)), what="mesh")
        self._h = h

    @staticmethod
    def build_grid(u_min: float, u_max: float, v_min: float, v_max: float, nu: int, nv: int,
                   potential_fn: Callable, axisymmetric_rz: bool = True) -> "BiLinearMesh2D":
        """nu x nv cells of two triangles each (mesh_field.hpp:438-479); potential_fn(u, v)
        gives the node potential in volts."""
        lib = _ffi.load()
        cb = _ffi.POTENTIAL2D_FN(lambda u, v, _u: float(potential_fn(u, v)))
        h = C.c_void_p()
        _check(lib.cmpmc_mesh2d_build_grid(float(u_min), float(u_max), float(v_min), float(v_max), int(nu), int(nv),
                                           cb, None, int(bool(axisymmetric_rz)), C.byref(h)), what="mesh")
        return BiLinearMesh2D(_handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.cmpmc_mesh2d_destroy(h)
            self._h = None

    def _info(self):
        nv, nt = C.c_uint64(), C.c_uint64()
        _check(self._lib.cmpmc_mesh2d_info(self._h, C.byref(nv), C.byref(nt)))
        return nv.value, nt.value

    def num_vertices(self) -> int:
        return self._info()[0]

    def num_triangles(self) -> int:
        return self._info()[1]

    def empty(self) -> bool:
        return self.num_triangles() == 0

    def field_at(self, p, tri_hint: Optional[C.c_int32] = None):
        """E(p) in V/m from the containing triangle (zero outside); the walk starts from and
        updates tri_hint (a ctypes int32), or the mesh's own hint (as at())."""
        hint = self._hint if tri_hint is None else tri_hint
        q = (C.c_double * 3)(*p)
        e = (C.c_double * 3)()
        _check(self._lib.cmpmc_mesh2d_field_at(self._h, q, C.byref(hint), e))
        return (e[0], e[1], e[2])

    def potential_at(self, p, tri_hint: Optional[C.c_int32] = None) -> float:
        hint = self._hint if tri_hint is None else tri_hint
        q = (C.c_double * 3)(*p)
        v = C.c_double()
        _check(self._lib.cmpmc_mesh2d_potential_at(self._h, q, C.byref(hint), C.byref(v)))
        return v.value

    def at(self, p):
        return self.field_at(p)


@dataclass
class DetectorModel:
    """DetectorModel (transport/engine.hpp:96-156)."""
    solid: CylinderSolid = field(default_factory=CylinderSolid)
    e_field: UniformElectricField = field(default_factory=lambda: UniformElectricField.from_bias(0.0, 2.54 * units.cm))
    mesh_field_3d: Optional[TriLinearMesh3D] = None
    mesh_field_2d: Optional[BiLinearMesh2D] = None
    surfaces: list = field(default_factory=_default_surfaces)
    max_bounces: int = 5000
    min_phonon_eV: float = 10.0 * units.ueV
    luke_sample_fraction: float = 1.0
    charge_max_dk_frac: float = 0.05
    charge_dt_cap_s: float = 100.0 * units.ps
    charge_stepping: int = 0  # 0 FirstOrderDkCap, 1 LemanSecondOrder
    charge_sampling_dk_frac: float = 0.25
    charge_release: int = 0
    fermi_level_above_Ev_eV: float = -1.0
    electrode_seed_max_gap: float = 80.0
    jump_to_ballistic: bool = False
    allow_unvalidated: bool = False
    russian_roulette_bounces: int = 0
    russian_roulette_survival: float = 0.5

    @staticmethod
    def published_benchmark(voltage_V: float = 0.0, luke_sample_fraction: float = 1.0) -> "DetectorModel":
        """The detector of the reference's published benchmark (benchmarks/cmpmc_bench.cpp:45-57):
        demo polynomial surfaces (sensor faces with prob_abs 1, a bare side wall; guarded, so
        allow_unvalidated is set), max_bounces 100, a uniform field of voltage_V over 2.54 cm."""
        sensor = SurfaceProperty.demo_polynomial_sensor_surface()
        sensor.prob_abs = 1.0
        return DetectorModel(e_field=UniformElectricField.from_bias(voltage_V, 2.54 * units.cm),
                             surfaces=[sensor, copy.deepcopy(sensor), SurfaceProperty.demo_polynomial_bare_surface()],
                             max_bounces=100, luke_sample_fraction=luke_sample_fraction, allow_unvalidated=True)

    def to_c(self) -> _ffi.DetectorC:
        d = _ffi.DetectorC()
        d.radius = self.solid.radius
        d.half_z = self.solid.half_z
        for i in range(3):
            d.e_field[i] = float(self.e_field.field_Vm[i])
        for i, s in enumerate(self.surfaces):
            d.surfaces[i] = s.to_c()
        for name in ("max_bounces", "russian_roulette_bounces", "charge_stepping", "charge_release"):
            setattr(d, name, int(getattr(self, name)))
        for name in ("russian_roulette_survival", "min_phonon_eV", "luke_sample_fraction", "charge_max_dk_frac",
                     "charge_dt_cap_s", "charge_sampling_dk_frac", "fermi_level_above_Ev_eV",
                     "electrode_seed_max_gap"):
            setattr(d, name, float(getattr(self, name)))
        d.allow_unvalidated = int(self.allow_unvalidated)
        d.jump_to_ballistic = int(self.jump_to_ballistic)
        return d


# ---- lattice and engine ----------------------------------------------------------------------


class CrystalLattice:
    """CrystalLattice (lattice/crystal_lattice.hpp:24-478): host-built tables, device queries."""

    N_OCT = 256
    N_CDF = 1024

    def __init__(self, cfg: CrystalConfig):
        self._lib = _ffi.load()
        self.cfg = cfg
        self._ccfg = cfg.to_c()
        h = C.c_void_p()
        _check(self._lib.cmpmc_lattice_create(C.byref(self._ccfg), C.byref(h)), what="lattice build")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.cmpmc_lattice_destroy(h)
            self._h = None

    def config(self) -> CrystalConfig:
        return self.cfg

    def tables(self) -> dict:
        """Copies of the octahedral table (float32 [3,256,256,4]), the decay inverse-CDF tables
        and the flattened Herring-Vogt tensors."""
        o, a, b, hv = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        n = C.c_size_t()
        _check(self._lib.cmpmc_lattice_tables(self._h, C.byref(o), C.byref(a), C.byref(b), C.byref(hv), C.byref(n)))
        oct_ = np.ctypeslib.as_array(C.cast(o, C.POINTER(C.c_float)), shape=(3 * 256 * 256 * 4,)).copy()
        return {
            "oct": oct_.reshape(3, 256, 256, 4),
            "cdf_lt": np.ctypeslib.as_array(C.cast(a, C.POINTER(C.c_double)), shape=(1024,)).copy(),
            "cdf_tt": np.ctypeslib.as_array(C.cast(b, C.POINTER(C.c_double)), shape=(1024,)).copy(),
            "hv": np.ctypeslib.as_array(C.cast(hv, C.POINTER(C.c_double)), shape=(n.value,)).copy(),
        }

    # CrystalLattice::KinematicsMode (crystal_lattice.hpp:63-74)
    Octahedral, Exact, Bilinear = 0, 1, 2

    def set_kinematics_mode(self, mode: int) -> None:
        """Octahedral (default), Exact (Cardano solve per call) or Bilinear (181 x 361
        table). Applies to make_track, the generators and every device context created
        afterwards from this lattice (engines made before keep their contexts)."""
        _check(self._lib.cmpmc_lattice_set_kinematics_mode(self._h, int(mode)), what="kinematics mode")

    def kinematics_mode(self) -> int:
        return self._lib.cmpmc_lattice_kinematics_mode(self._h)

    def map_k_to_vg(self, mode: int, k_det: Sequence[float]):
        k = (C.c_double * 3)(*k_det)
        vg = (C.c_double * 3)()
        mag = C.c_double()
        _check(self._lib.cmpmc_lattice_map_k_to_vg(self._h, int(mode), k, vg, C.byref(mag)))
        return (vg[0], vg[1], vg[2]), mag.value


@dataclass
class EventInput:
    """EventInput (transport/parallel.hpp:38-44)."""
    event_id: int
    rng: Rng
    phonons: list
    charges: list
    injected_eV: float = 0.0


@dataclass
class RunOptions:
    """RunOptions (transport/parallel.hpp:46-51) plus the device-side choices."""
    threads: int = 0
    seed: int = 1
    events_per_chunk: int = 16
    keep_hits: bool = True
    form: str = "plain_fp64"  # "batched_fp32" (wavefront split) or "batched_fp32_inline"
    device: int = 0
    want_event_stats: bool = False
    first_event: int = 0
    # batched form: film cascades from the KaplanSurrogateLUT table (kaplan_film.hpp:336-383)
    kaplan_surrogate: bool = False


class SimStats:
    """SimStats (transport/engine.hpp:29-93) as a numpy record with attribute access."""

    def __init__(self, rec: Optional[np.ndarray] = None):
        self._r = np.zeros((), dtype=_ffi.STATS_DTYPE) if rec is None else np.array(rec, dtype=_ffi.STATS_DTYPE)

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        v = self._r[name]
        return int(v) if v.dtype.kind == "u" else float(v)

    def __iadd__(self, other: "SimStats") -> "SimStats":
        for n in _ffi.STATS_DTYPE.names:
            self._r[n] = self._r[n] + other._r[n]
        return self

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n in _ffi.STATS_DTYPE.names}

    def record(self) -> np.ndarray:
        return self._r.copy()


@dataclass
class RunResult:
    """RunResult (transport/parallel.hpp:53-59) plus device timings."""
    stats: SimStats
    hits: np.ndarray
    hit_offsets: np.ndarray
    threads_used: int = 1
    wall_seconds: float = 0.0
    kernel_ms: float = 0.0
    device_ms: float = 0.0
    kernel_launches: int = 0
    event_stats: Optional[np.ndarray] = None


@dataclass(frozen=True)
class Workload:
    """A canonical generator that runs in the native library (cmpmc_generate)."""
    kind: int
    primaries_per_event: int
    name: str


class workloads:
    single_l_origin = Workload(_ffi.WL_SINGLE_L_ORIGIN, 1, "single_L_7.5meV_origin")
    mixed_energy = Workload(_ffi.WL_MIXED_ENERGY, 100, "mixed_energy_100_per_event")
    pair_drift = Workload(_ffi.WL_PAIR_DRIFT, 2, "pair_drift")
    single_l_volume = Workload(_ffi.WL_SINGLE_L_VOLUME, 1, "single_L_7.5meV_volume")
    test_parallel = Workload(_ffi.WL_TEST_PARALLEL, 1, "test_parallel_mixed")
    # electron recoils split by EnergyPartition::partition_deposit; the detector needs
    # TriLinearMesh3D.recoil_mesh as mesh_field_3d and luke_sample_fraction 1 (recoil) or
    # 0.05 (recoil_light)
    recoil = Workload(_ffi.WL_RECOIL, 1, "electron_recoil_10eV_10keV")
    recoil_light = Workload(_ffi.WL_RECOIL_LIGHT, 1, "electron_recoil_10eV_100eV_light")
    # the reference's published benchmark (benchmarks/cmpmc_bench.cpp:45-71): run them with
    # DetectorModel.published_benchmark() (demo polynomial surfaces, max_bounces 100)
    published_phonon = Workload(_ffi.WL_PUBLISHED_PHONON, 1, "published_phonon_7.5meV_dos_mode")
    published_pair = Workload(_ffi.WL_PUBLISHED_PAIR, 2, "published_pair_origin")


@dataclass
class PackedEvents:
    """Host arrays of generated events, ready for the C ABI."""
    n_events: int
    first_event: int
    rng_state: np.ndarray
    injected_eV: np.ndarray
    phonon_offsets: np.ndarray
    phonons: np.ndarray
    charge_offsets: np.ndarray
    charges: np.ndarray


class SimulationEngine:
    """SimulationEngine (transport/engine.hpp:161-989): holds the lattice and detector, owns
    one device context per device."""

    def __init__(self, lattice: CrystalLattice, detector: DetectorModel):
        self._lib = _ffi.load()
        self.lattice = lattice
        self.detector = detector
        self._cdet = detector.to_c()
        if any(s.demo_values for s in detector.surfaces) and not detector.allow_unvalidated:
            raise UnvalidatedModuleError(
                "CMPMC: 'SurfaceProperty::demo_polynomial_*' is not validated (demonstration reflection/"
                "down-conversion polynomials, not physically motivated). Set allow_unvalidated = true to run it "
                "anyway.")
        self._ctx = {}

    def __del__(self):
        for h in getattr(self, "_ctx", {}).values():
            self._lib.cmpmc_gpu_destroy(h)
        self._ctx = {}

    def context(self, device: int = 0):
        h = self._ctx.get(device)
        if h is None:
            h = C.c_void_p()
            _check(self._lib.cmpmc_gpu_create(self.lattice._h, C.byref(self._cdet), int(device), C.byref(h)),
                   what="device context")
            self._ctx[device] = h
            if self.detector.mesh_field_3d is not None:
                _check(self._lib.cmpmc_gpu_set_mesh(h, self.detector.mesh_field_3d._h), h)
            elif self.detector.mesh_field_2d is not None:
                _check(self._lib.cmpmc_gpu_set_mesh2d(h, self.detector.mesh_field_2d._h), h)
            for i, sp in enumerate(self.detector.surfaces):
                if sp.electrode_mask is not None and not sp.electrode_mask.empty():
                    m = sp.electrode_mask
                    _check(self._lib.cmpmc_gpu_set_electrode_mask(h, i, m.to_c(), m.num_pads()), h)
        return h

    def configure(self, device: int = 0, threads_per_block: int = 0, blocks_per_sm: int = 0,
                  stack_capacity: int = 0, hit_capacity: int = 0, queue_capacity: int = 0) -> None:
        h = self.context(device)
        _check(self._lib.cmpmc_gpu_configure(h, threads_per_block, blocks_per_sm, stack_capacity, hit_capacity), h)
        if queue_capacity:
            _check(self._lib.cmpmc_gpu_configure_queue(h, int(queue_capacity)), h)

    def configure_pool(self, form=1, ring_capacity: int = 0, device: int = 0) -> None:
        """Launch form of the batched phonon transport (cmpmc_gpu_configure_pool): 1 (or True)
        the SM-phase pool, one persistent launch (the default); 2 the warp pool; 0 (or False)
        the host-driven film / transport rounds; 3 the SM-phase pool computed in FP64 on the
        same substreams (phonon-only batches, full film cascades)."""
        h = self.context(device)
        _check(self._lib.cmpmc_gpu_configure_pool(h, int(form), int(ring_capacity)), h)

    def configure_staging(self, enable: bool = True, device: int = 0) -> None:
        """Decay CDF tables staged in shared memory by a TMA bulk copy (default) or read from
        global memory (cmpmc_gpu_configure_staging); the results are identical."""
        h = self.context(device)
        _check(self._lib.cmpmc_gpu_configure_staging(h, int(enable)), h)

    def configure_graph(self, enable: bool = True, device: int = 0) -> None:
        """Replay repeated batched calls on device-resident inputs as one CUDA graph."""
        h = self.context(device)
        _check(self._lib.cmpmc_gpu_configure_graph(h, int(enable)), h)

    def autotune(self, ev: "PackedEvents", options: "RunOptions", repeats: int = 2) -> dict:
        """Times the launch-configuration candidates on this batch and keeps the fastest
        (cmpmc_gpu_autotune); returns the choice and every candidate's kernel time."""
        h = self.context(options.device)
        keep = []
        d = self._desc(ev, options, keep)
        r = _ffi.TuneResultC()
        _check(self._lib.cmpmc_gpu_autotune(h, C.byref(d), int(repeats), C.byref(r)), h, "autotune")
        tried = [{"threads_per_block": r.tried_tpb[i], "blocks_per_sm": r.tried_bps[i],
                  "queue_capacity": r.tried_queue[i], "kernel_ms": r.tried_ms[i]} for i in range(r.n_tried)]
        return {"threads_per_block": r.threads_per_block, "blocks_per_sm": r.blocks_per_sm,
                "queue_capacity": r.queue_capacity, "phase_steps": r.phase_steps, "best_ms": r.best_ms,
                "first_ms": r.first_ms, "tried": tried}

    def make_track(self, pos, k_dir, mode, energy_eV, time_s=0.0, weight=1.0) -> np.ndarray:
        out = np.zeros((), dtype=_ffi.PHONON_DTYPE)
        p = (C.c_double * 3)(*pos)
        k = (C.c_double * 3)(*k_dir)
        _check(self._lib.cmpmc_make_track(self.lattice._h, p, k, int(mode), float(energy_eV), float(time_s),
                                          float(weight), out.ctypes.data))
        return out

    def make_charge(self, type_, pos, direction, ekin_eV, valley, time_s=0.0) -> np.ndarray:
        """ChargePhysics::make_charge (charge/charge_transport.hpp:49-70)."""
        out = np.zeros((), dtype=_ffi.CHARGE_DTYPE)
        p = (C.c_double * 3)(*pos)
        d = (C.c_double * 3)(*direction)
        _check(self._lib.cmpmc_make_charge(self.lattice._h, int(type_), p, d, float(ekin_eV), int(valley),
                                           float(time_s), out.ctypes.data))
        return out

    # -- event generation --------------------------------------------------------------------
    def generate(self, workload: Workload, n_events: int, seed: int, first_event: int = 0,
                 threads: int = 0) -> PackedEvents:
        n = int(n_events)
        rng_state = np.zeros((n, 4), dtype=np.uint64)
        inj = np.zeros(n, dtype=np.float64)
        po = np.zeros(n + 1, dtype=np.uint64)
        co = np.zeros(n + 1, dtype=np.uint64)
        np_, nc_ = C.c_uint64(), C.c_uint64()
        st = self._lib.cmpmc_generate(self.lattice._h, C.byref(self._cdet), workload.kind, seed, first_event, n,
                                      threads, rng_state.ctypes.data, inj.ctypes.data, po.ctypes.data, None, 0,
                                      C.byref(np_), co.ctypes.data, None, 0, C.byref(nc_))
        if st not in (_ffi.OK, _ffi.ERR_CAPACITY):
            _check(st, what="generate")
        ph = np.zeros(max(np_.value, 1), dtype=_ffi.PHONON_DTYPE)
        ch = np.zeros(max(nc_.value, 1), dtype=_ffi.CHARGE_DTYPE)
        _check(self._lib.cmpmc_generate(self.lattice._h, C.byref(self._cdet), workload.kind, seed, first_event, n,
                                        threads, rng_state.ctypes.data, inj.ctypes.data, po.ctypes.data,
                                        ph.ctypes.data, ph.size, C.byref(np_), co.ctypes.data, ch.ctypes.data,
                                        ch.size, C.byref(nc_)), what="generate")
        return PackedEvents(n, first_event, rng_state, inj, po, ph[:np_.value], co, ch[:nc_.value])

    def generate_python(self, generate: Callable[[EventInput], None], n_events: int, seed: int,
                        first_event: int = 0) -> PackedEvents:
        n = int(n_events)
        rng_state = np.zeros((n, 4), dtype=np.uint64)
        inj = np.zeros(n, dtype=np.float64)
        po = np.zeros(n + 1, dtype=np.uint64)
        co = np.zeros(n + 1, dtype=np.uint64)
        phs, chs = [], []
        for i in range(n):
            ev = first_event + i
            rng = Rng.for_stream(seed, ev)
            inp = EventInput(ev, rng, [], [], 0.0)
            generate(inp)
            rng_state[i] = rng.s
            inj[i] = inp.injected_eV
            phs.extend(inp.phonons)
            chs.extend(inp.charges)
            po[i + 1] = len(phs)
            co[i + 1] = len(chs)
        ph = np.array(phs, dtype=_ffi.PHONON_DTYPE) if phs else np.zeros(0, dtype=_ffi.PHONON_DTYPE)
        ch = np.array(chs, dtype=_ffi.CHARGE_DTYPE) if chs else np.zeros(0, dtype=_ffi.CHARGE_DTYPE)
        return PackedEvents(n, first_event, rng_state, inj, po, ph, co, ch)

    # -- device run ----------------------------------------------------------------------------
    @staticmethod
    def _desc(ev: PackedEvents, options: RunOptions, keep: list) -> _ffi.RunDescC:
        d = _ffi.RunDescC()
        d.n_events = ev.n_events
        d.first_event = ev.first_event
        ph = ev.phonons if ev.phonons.size else np.zeros(1, dtype=_ffi.PHONON_DTYPE)
        keep.append(ph)
        d.rng_state = ev.rng_state.ctypes.data
        d.injected_eV = ev.injected_eV.ctypes.data
        d.phonon_offsets = ev.phonon_offsets.ctypes.data
        d.phonons = ph.ctypes.data
        if ev.charges.size > 0:
            d.charge_offsets = ev.charge_offsets.ctypes.data
            d.charges = ev.charges.ctypes.data
        d.keep_hits = int(options.keep_hits)
        forms = {"plain_fp64": _ffi.FORM_PLAIN_FP64, "batched_fp32": _ffi.FORM_BATCHED_FP32,
                 "batched_fp32_inline": _ffi.FORM_BATCHED_FP32_INLINE}
        if options.form not in forms:
            raise ValueError(f"unknown form {options.form!r}: one of {sorted(forms)}")
        d.form = forms[options.form]
        d.seed = options.seed
        d.want_event_stats = int(options.want_event_stats)
        d.kaplan_surrogate = int(options.kaplan_surrogate)
        return d

    def run_packed(self, ev: PackedEvents, options: RunOptions) -> RunResult:
        h = self.context(options.device)
        n = ev.n_events
        keep = []
        d = self._desc(ev, options, keep)
        out = _ffi.RunOutC()
        _check(self._lib.cmpmc_gpu_run_events(h, C.byref(d), C.byref(out)), h)
        nh = int(out.n_hits)
        hits = np.zeros(nh, dtype=_ffi.HIT_DTYPE)
        if nh:
            C.memmove(hits.ctypes.data, out.hits, nh * _ffi.HIT_DTYPE.itemsize)
        offs = np.zeros(n + 1, dtype=np.uint64)
        C.memmove(offs.ctypes.data, out.hit_offsets, (n + 1) * 8)
        evst = None
        if options.want_event_stats and n:
            evst = np.zeros(n, dtype=_ffi.STATS_DTYPE)
            C.memmove(evst.ctypes.data, out.event_stats, n * _ffi.STATS_DTYPE.itemsize)
        stats = SimStats(np.frombuffer(bytes(out.stats), dtype=_ffi.STATS_DTYPE)[0])
        return RunResult(stats=stats, hits=hits, hit_offsets=offs, threads_used=1, kernel_ms=out.kernel_ms,
                         device_ms=out.total_ms, kernel_launches=int(out.kernel_launches), event_stats=evst)


def run_events(engine: SimulationEngine, n_events: int, generate, options: Optional[RunOptions] = None) -> RunResult:
    """run_events (transport/parallel.hpp:76-148) on the device.

    Event i draws from Rng.for_stream(options.seed, options.first_event + i); its generator
    runs on the host, the transport on the device. Results are independent of how the
    device schedules events.
    """
    options = options or RunOptions()
    t0 = time.perf_counter()
    if isinstance(generate, Workload):
        packed = engine.generate(generate, n_events, options.seed, options.first_event, options.threads)
    else:
        packed = engine.generate_python(generate, n_events, options.seed, options.first_event)
    res = engine.run_packed(packed, options)
    res.wall_seconds = time.perf_counter() - t0
    return res
