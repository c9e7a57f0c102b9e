"""pequod_b200: B200-native (sm_100a) QG time-step hot path of PEQUOD.

Python mirror of the C ABI in include/pequod_b200.h.  The compute path is the
CUDA library pequod_b200/_lib/libpequod_b200.so; this module only marshals
arguments.  There is no CPU fallback: if the library is missing or cannot be
loaded the import of the native handle raises.

The interface follows the reference's routines (qg3p_helmholtz.F90 helm,
qg3p_aux.F90 pv_inversion / cabaret_*, qg3p_diagnostics.F90 energy) with
Fortran-ordered numpy arrays in the reference's layouts.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libpequod_b200.so")

PQ_OK = 0
PQ_ERR_ARG, PQ_ERR_CUDA, PQ_ERR_NAN, PQ_ERR_NOMEM, PQ_ERR_UNSUPPORTED, PQ_ERR_STATE, PQ_ERR_BUDGET, PQ_ERR_NOTFOUND = (
    1, 2, 3, 4, 5, 6, 7, 8)
PTR_HOST, PTR_DEVICE = 0, 1
SCHEME_CABARET, SCHEME_LEAPFROG = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
BC_PARTIAL_SLIP, BC_NO_SLIP, BC_FREE_SLIP = 1, 2, 3
DST_BUTTERFLY, DST_TENSOR = 1, 2
MAX_LAYERS = 8
NOALLOC_MAX_JJ = 4097  # PQ_NOALLOC_MAX_JJ: largest jj pq_energy_noalloc accepts

FIELDS = {
    "psi": 0, "zeta": 1, "rel": 2, "zeta_old": 3, "ui": 4, "uj": 5, "uimo": 6, "ujmo": 7,
    "zeta_fi": 8, "zeta_fj": 9, "res": 10, "res_beta": 11, "corr": 12,
    # leapfrog second time level
    "psi2": 13, "zeta2": 14, "rel2": 15, "zeta_old2": 16,
}

_dp = C.POINTER(C.c_double)


class PQError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pequod_b200 error {code}: {msg}")
        self.code = code


class ModelDesc(C.Structure):
    _fields_ = [
        ("ii", C.c_int), ("jj", C.c_int), ("layers", C.c_int), ("periodic_j", C.c_int),
        ("scheme", C.c_int), ("limiter", C.c_int), ("bc_type", C.c_int), ("precision", C.c_int),
        ("adapt_dt", C.c_int),
        ("alpha", C.c_double), ("dt", C.c_double), ("viscosity", C.c_double), ("visc_bot", C.c_double),
        ("target_cfl", C.c_double), ("max_dt", C.c_double), ("max_dt_increase", C.c_double),
        ("ra_nu", C.c_double), ("ra_alpha", C.c_double),
        ("beta", C.c_double * MAX_LAYERS), ("h", C.c_double * MAX_LAYERS),
        ("s1", C.c_double * MAX_LAYERS), ("s2", C.c_double * MAX_LAYERS), ("ss", C.c_double * MAX_LAYERS),
        ("m2z", C.c_double * (MAX_LAYERS * MAX_LAYERS)), ("z2m", C.c_double * (MAX_LAYERS * MAX_LAYERS)),
        ("force_wind", _dp),
    ]


class Tuning(C.Structure):
    _fields_ = [("cab_band", C.c_int), ("dst_group", C.c_int), ("cab_kernel", C.c_int), ("dst_lanes", C.c_int),
                ("dst_lanes_inv", C.c_int), ("pdl", C.c_int), ("dst_algo", C.c_int), ("reserved", C.c_int * 1)]


class Physical(C.Structure):
    _fields_ = [
        ("ii", C.c_int), ("jj", C.c_int), ("layers", C.c_int),
        ("basinscale", C.c_double), ("dt", C.c_double), ("f0", C.c_double), ("beta", C.c_double),
        ("H", C.c_double * MAX_LAYERS), ("gprime", C.c_double * MAX_LAYERS),
        ("tau", C.c_double), ("wind_asym", C.c_double), ("wind_tilt", C.c_double), ("wind_shift", C.c_double),
        ("visc", C.c_double), ("visc_bot", C.c_double), ("alpha", C.c_double), ("partial_slip", C.c_int),
        ("scheme", C.c_int), ("limiter", C.c_int), ("precision", C.c_int), ("adapt_dt", C.c_int),
        ("target_cfl", C.c_double), ("max_dt", C.c_double), ("max_dt_increase", C.c_double),
        ("u_scale", C.c_double),
    ]


# Every function the C ABI exports, with its ctypes signature.
SIGNATURES = {
    "pq_stratification": (C.c_int, [C.POINTER(ModelDesc), C.c_int, _dp, _dp, _dp, C.c_double]),
    "pq_setup_double_gyre": (C.c_int, [C.POINTER(Physical), C.POINTER(ModelDesc), _dp, _dp]),
    "pq_make_ic": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_double, _dp]),
    "pq_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(ModelDesc), C.c_int]),
    "pq_destroy": (None, [C.c_void_p]),
    "pq_last_error": (C.c_char_p, [C.c_void_p]),
    "pq_device_bytes": (C.c_size_t, [C.c_void_p]),
    "pq_helm": (C.c_int, [C.c_void_p, _dp, C.c_int]),
    "pq_pv_inversion": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    "pq_add_laplace_bc_rhs": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp, _dp, C.c_int, C.c_int]),
    "pq_apply_dirichlet_bc": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp, _dp, C.c_int, C.c_int]),
    "pq_laplace_bc_rhs": (C.c_int, [C.c_void_p, C.c_double, _dp, C.c_int]),
    "pq_init_perturb": (C.c_int, [C.c_void_p, _dp, C.c_int]),
    "pq_step": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_step_async": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_cabaret_step": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "pq_check": (C.c_int, [C.c_void_p]),
    "pq_step_exchange": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    "pq_join": (C.c_int, [C.c_void_p]),
    "pq_energy": (C.c_int, [C.c_void_p, _dp, _dp]),
    "pq_cfl": (C.c_int, [C.c_void_p, _dp]),
    "pq_get_field": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "pq_set_field": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "pq_get_scalars": (C.c_int, [C.c_void_p, _dp]),
    "pq_sync": (C.c_int, [C.c_void_p]),
    "pq_write_checkpoint": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double, C.c_double]),
    "pq_average": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "pq_get_average": (C.c_int, [C.c_void_p, _dp, _dp]),
    "pq_write_average": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_double]),
    "pq_get_quad": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "pq_write_quad": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_double]),
    "pq_read_checkpoint": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, _dp]),
    "pq_stream": (C.c_void_p, [C.c_void_p]),
    "pq_last_launch_count": (C.c_long, [C.c_void_p]),
    "pq_kernel_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "pq_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "pq_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "pq_kernel_times": (C.c_int, [C.c_void_p, _dp, C.POINTER(C.c_long)]),
    "pq_energy_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp,
                                    C.c_void_p, C.c_void_p]),
    "pq_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), _dp, C.c_int]),
    "pq_batch_create_ex": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), _dp, C.c_int, C.c_int, C.c_int]),
    "pq_batch_member_dst_algo": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_batch_destroy": (None, [C.c_void_p]),
    "pq_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "pq_batch_device_bytes": (C.c_size_t, [C.c_void_p]),
    "pq_batch_stream": (C.c_void_p, [C.c_void_p]),
    "pq_batch_set_rhs": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "pq_batch_get": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "pq_batch_solve_async": (C.c_int, [C.c_void_p]),
    "pq_batch_sync": (C.c_int, [C.c_void_p]),
    "pq_batch_helm": (C.c_int, [C.c_void_p, C.POINTER(_dp), C.c_int]),
    "pq_batch_launch_count": (C.c_int, [C.c_void_p]),
    "pq_ensemble_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(ModelDesc), C.c_int]),
    "pq_ensemble_destroy": (None, [C.c_void_p]),
    "pq_ensemble_last_error": (C.c_char_p, [C.c_void_p]),
    "pq_ensemble_size": (C.c_int, [C.c_void_p]),
    "pq_ensemble_member": (C.c_void_p, [C.c_void_p, C.c_int]),
    "pq_ensemble_stream": (C.c_void_p, [C.c_void_p]),
    "pq_ensemble_init": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "pq_ensemble_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "pq_ensemble_set_dst_algo": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_ensemble_step_async": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_ensemble_sync": (C.c_int, [C.c_void_p]),
    "pq_ensemble_step": (C.c_int, [C.c_void_p, C.c_int]),
    "pq_server_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t, C.c_int]),
    "pq_server_destroy": (None, [C.c_void_p]),
    "pq_server_last_error": (C.c_char_p, [C.c_void_p]),
    "pq_server_submit": (C.c_int, [C.c_void_p, C.POINTER(ModelDesc), _dp, C.c_int, C.POINTER(C.c_long)]),
    "pq_server_poll": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pq_server_status": (C.c_int, [C.c_void_p, C.c_long]),
    "pq_server_collect": (C.c_int, [C.c_void_p, C.c_long, _dp, _dp]),
    "pq_server_device_bytes": (C.c_size_t, [C.c_void_p]),
    "pq_server_clock": (C.c_double, [C.c_void_p]),
    "pq_server_launches": (C.c_long, [C.c_void_p]),
}

KERNELS = ("dst_forward", "tridiag", "dst_inverse_backproject", "cabaret_fused")

_lib = None


def lib():
    """Load the CUDA library.  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"pequod_b200 native library not built: {LIB_PATH} (run pequod_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _check(rc, ctx=None):
    if rc != PQ_OK:
        msg = lib().pq_last_error(ctx).decode() if ctx else ""
        raise PQError(rc, msg)


# ---------------------------------------------------------------------------
# Configurations


def double_gyre_physical(ii, jj=None, layers=3, dt=1800.0, dx=30.0e5, H=(3.0e4, 7.0e4, 3.0e5),
                         gprime=(1.5, 0.75), f0=9.4e-5, beta=1.8e-13, tau=0.8, visc=1.0e6, visc_bot=1.0e-7,
                         alpha=120.0e5, partial_slip=True, wind_asym=1.0, wind_tilt=0.0, wind_shift=0.0,
                         scheme=SCHEME_CABARET, limiter=1, precision=PREC_FP64, adapt_dt=0,
                         target_cfl=0.1, max_dt=86400.0, max_dt_increase=1.5) -> Physical:
    """Wind-driven closed-basin double gyre in cgs units.

    Defaults are the 3-layer 129 x 129, dx = 30 km configuration: layer depths
    300/700/3000 m, reduced gravities 0.015/0.0075 m s^-2, f0 = 9.4e-5 s^-1,
    beta = 1.8e-11 m^-1 s^-1, tau0 = 0.08 N m^-2 (0.8 cm^2 s^-2 over
    rho0 = 1000 kg m^-3) with a -cos(2 pi y / L) profile, bottom drag 1e-7 s^-1,
    lateral viscosity 100 m^2 s^-1, partial slip with alpha = 120 km.
    """
    jj = ii if jj is None else jj
    p = Physical()
    p.ii, p.jj, p.layers = ii, jj, layers
    p.basinscale = (ii - 1) * dx
    p.dt, p.f0, p.beta = dt, f0, beta
    H = list(H)
    if len(H) != layers:
        raise ValueError("len(H) != layers")
    for k in range(layers):
        p.H[k] = H[k]
    for k in range(layers - 1):
        p.gprime[k] = gprime[k]
    p.tau, p.wind_asym, p.wind_tilt, p.wind_shift = tau, wind_asym, wind_tilt, wind_shift
    p.visc, p.visc_bot, p.alpha, p.partial_slip = visc, visc_bot, alpha, int(partial_slip)
    p.scheme, p.limiter, p.precision, p.adapt_dt = scheme, limiter, precision, adapt_dt
    p.target_cfl, p.max_dt, p.max_dt_increase = target_cfl, max_dt, max_dt_increase
    p.u_scale = 1.0
    return p


class Config:
    """A non-dimensional model description plus its wind-forcing buffer."""

    def __init__(self, desc: ModelDesc, wind: np.ndarray | None, t_scale: float, physical: Physical | None = None):
        self.desc = desc
        self.wind = wind
        self.t_scale = t_scale
        self.physical = physical  # the cgs description it was set up from, if any
        if wind is not None:
            self.desc.force_wind = _p(self.wind)

    @classmethod
    def from_physical(cls, p: Physical) -> "Config":
        d = ModelDesc()
        wind = np.zeros((p.ii, p.jj), order="F")
        ts = np.zeros(1)
        _check(lib().pq_setup_double_gyre(C.byref(p), C.byref(d), _p(wind), _p(ts)))
        return cls(d, wind, float(ts[0]), p)

    @property
    def ii(self):
        return self.desc.ii

    @property
    def jj(self):
        return self.desc.jj

    @property
    def layers(self):
        return self.desc.layers

    def modal(self):
        L = self.layers
        m2z = np.array(self.desc.m2z[: L * L]).reshape((L, L), order="F")
        z2m = np.array(self.desc.z2m[: L * L]).reshape((L, L), order="F")
        return np.array(self.desc.ss[:L]), m2z, z2m


def make_ic(ii, jj, layers, seed=0, amplitude=1.0, sigma=3.0) -> np.ndarray:
    """Seeded synthetic initial PV (N(0,1) noise smoothed by a Gaussian of sigma cells)."""
    out = np.zeros((ii, jj, layers), order="F")
    _check(lib().pq_make_ic(ii, jj, layers, seed, amplitude, sigma, _p(out)))
    return out


# ---------------------------------------------------------------------------


class Model:
    """One device context: helm / pv_inversion drop-ins and the CABARET loop."""

    def __init__(self, cfg: Config, device: int = 0):
        self.cfg = cfg
        self.ctx = C.c_void_p()
        rc = lib().pq_create(C.byref(self.ctx), C.byref(cfg.desc), device)
        if rc != PQ_OK:
            msg = lib().pq_last_error(self.ctx).decode() if self.ctx else ""
            if self.ctx:
                lib().pq_destroy(self.ctx)
                self.ctx = None
            raise PQError(rc, msg)

    def close(self):
        if getattr(self, "ctx", None):
            lib().pq_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        self.close()

    @property
    def shape(self):
        return (self.cfg.ii, self.cfg.jj, self.cfg.layers)

    def helm(self, zeta: np.ndarray) -> np.ndarray:
        z = np.array(zeta, dtype=np.float64, order="F").reshape(self.shape, order="F")
        _check(lib().pq_helm(self.ctx, _p(z), PTR_HOST), self.ctx)
        return z

    def pv_inversion(self, zeta_sdata: np.ndarray) -> np.ndarray:
        z = np.asfortranarray(zeta_sdata, dtype=np.float64).reshape(self.shape, order="F")
        psi = np.zeros(self.shape, order="F")
        _check(lib().pq_pv_inversion(self.ctx, _p(z), _p(psi), PTR_HOST), self.ctx)
        return psi

    def _bc_field(self, a):
        a = np.array(a, dtype=np.float64, order="F")
        layers = 1 if a.ndim == 2 else a.shape[2]
        if a.shape[:2] != (self.cfg.ii, self.cfg.jj):
            raise ValueError("field must be (ii, jj) or (ii, jj, layers)")
        return a, layers

    @staticmethod
    def _bc_values(bc, bc_d, layers):
        b = np.ascontiguousarray(np.atleast_1d(np.asarray(bc, dtype=np.float64)))
        d = None if bc_d is None else np.ascontiguousarray(np.atleast_1d(np.asarray(bc_d, dtype=np.float64)))
        if d is not None and d.size != b.size:
            raise ValueError("bc and bc_d must have the same length")
        return b, d

    def add_laplace_bc_rhs(self, rhs: np.ndarray, bc, bc_d=None) -> np.ndarray:
        """add_laplace_bc_rhs (qg3p_laplace_bc.F90:55-190) on the device: a
        copy of rhs ((ii, jj) or (ii, jj, layers)) with the Dirichlet values
        lifted in; bc a number or one value per layer, bc_d the channel's
        wall i = ii."""
        a, layers = self._bc_field(rhs)
        b, d = self._bc_values(bc, bc_d, layers)
        _check(lib().pq_add_laplace_bc_rhs(self.ctx, _p(a), layers, _p(b), None if d is None else _p(d), b.size,
                                           PTR_HOST), self.ctx)
        return a

    def apply_dirichlet_bc(self, field: np.ndarray, bc, bc_d=None) -> np.ndarray:
        """apply_dirichlet_bc (qg3p_laplace_bc.F90:193-374) on the device."""
        a, layers = self._bc_field(field)
        b, d = self._bc_values(bc, bc_d, layers)
        _check(lib().pq_apply_dirichlet_bc(self.ctx, _p(a), layers, _p(b), None if d is None else _p(d), b.size,
                                           PTR_HOST), self.ctx)
        return a

    def laplace_bc_rhs(self, bc: float) -> np.ndarray:
        """laplace_bc_rhs (qg3p_laplace_bc.F90:42-51): (ii, jj)."""
        out = np.zeros((self.cfg.ii, self.cfg.jj), order="F")
        _check(lib().pq_laplace_bc_rhs(self.ctx, float(bc), _p(out), PTR_HOST), self.ctx)
        return out

    def init_perturb(self, zeta_ic: np.ndarray) -> None:
        """zeta_ic: (ii, jj, L), or (ii, jj, L, 2) -- both time levels -- for the leapfrog scheme."""
        shape = self.shape + ((2,) if self.cfg.desc.scheme == SCHEME_LEAPFROG else ())
        z = np.asfortranarray(zeta_ic, dtype=np.float64).reshape(shape, order="F")
        _check(lib().pq_init_perturb(self.ctx, _p(z), PTR_HOST), self.ctx)

    def step(self, n: int = 1) -> None:
        _check(lib().pq_step(self.ctx, n), self.ctx)

    def cabaret_step(self, dt: float, tweight_a: float = 0.5, tweight_u: float = 0.5) -> None:
        """One CABARET step with the caller's dt and time weights."""
        _check(lib().pq_cabaret_step(self.ctx, float(dt), float(tweight_a), float(tweight_u)), self.ctx)

    def step_async(self, n: int = 1) -> None:
        _check(lib().pq_step_async(self.ctx, n), self.ctx)

    def check(self) -> None:
        _check(lib().pq_check(self.ctx), self.ctx)

    def step_exchange(self, zeta_in_ptr, psi_out_ptr, ptr_kind=PTR_HOST) -> None:
        """One step exchanging zeta in / psi out through raw pointers (pinned host or device)."""
        _check(lib().pq_step_exchange(self.ctx, C.cast(zeta_in_ptr, _dp) if zeta_in_ptr else None,
                                      C.cast(psi_out_ptr, _dp) if psi_out_ptr else None, ptr_kind), self.ctx)

    @property
    def stream(self) -> int:
        return int(lib().pq_stream(self.ctx) or 0)

    def sync(self) -> None:
        _check(lib().pq_sync(self.ctx), self.ctx)

    def join(self) -> None:
        """Order the context's stream after the pipelined exchange copies."""
        _check(lib().pq_join(self.ctx), self.ctx)

    def energy(self):
        ekin = np.zeros(self.cfg.layers)
        epot = np.zeros(1)
        _check(lib().pq_energy(self.ctx, _p(ekin), _p(epot)), self.ctx)
        return ekin, float(epot[0])

    def cfl(self) -> float:
        out = np.zeros(1)
        _check(lib().pq_cfl(self.ctx, _p(out)), self.ctx)
        return float(out[0])

    def field_shape(self, name):
        ii, jj, L = self.shape
        if name in ("ui", "uimo", "zeta_fi"):
            return (ii + 3, jj + 2, L)
        if name in ("uj", "ujmo", "zeta_fj"):
            return (ii + 2, jj + 3, L)
        if name in ("res", "res_beta", "corr"):
            return (ii, jj, L)
        return (ii + 2, jj + 2, L)

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.field_shape(name), order="F")
        _check(lib().pq_get_field(self.ctx, FIELDS[name], _p(out)), self.ctx)
        return out

    def set(self, name: str, value: np.ndarray) -> None:
        v = np.asfortranarray(value, dtype=np.float64).reshape(self.field_shape(name), order="F")
        _check(lib().pq_set_field(self.ctx, FIELDS[name], _p(v)), self.ctx)

    def sdata(self, name: str) -> np.ndarray:
        return np.asfortranarray(self.get(name)[1:-1, 1:-1, :])

    def scalars(self):
        out = np.zeros(4)
        _check(lib().pq_get_scalars(self.ctx, _p(out)), self.ctx)
        return dict(dt=out[0], tweight_a=out[1], tweight_u=out[2], model_time=out[3])

    def write_checkpoint(self, s_path: str, supp_path: str | None = None, t_scale: float = 1.0,
                         start_time_day: float = 0.0) -> None:
        """Dump the state as the reference's qg<L>_<ii>_s.d / _s_supp.d pair."""
        supp = supp_path.encode() if supp_path else None
        _check(lib().pq_write_checkpoint(self.ctx, s_path.encode(), supp, t_scale, start_time_day), self.ctx)

    def read_checkpoint(self, s_path: str, supp_path: str | None = None) -> float:
        """START_PICKUP from a checkpoint pair; returns its total_time_day."""
        ttd = np.zeros(1)
        supp = supp_path.encode() if supp_path else None
        _check(lib().pq_read_checkpoint(self.ctx, s_path.encode(), supp, _p(ttd)), self.ctx)
        return float(ttd[0])

    QUAD = ("uu", "vv", "uu_i", "vv_i", "uv", "ur", "vr", "rr", "pr", "uz", "vz", "zz", "zr", "pp", "pz", "ut", "vt",
            "rt", "tt", "sc_ub", "sc_vb", "sc_bb", "sc_bb_i")

    def average(self, enable=True, threshold: float = 0.0) -> None:
        """Start (clearing) or stop the time average of psi (psi_av);
        enable = 2 also accumulates the quad eddy covariances."""
        _check(lib().pq_average(self.ctx, int(enable), float(threshold)), self.ctx)

    def get_quad(self, q: int) -> np.ndarray:
        """Quad accumulator q (QUAD order) / diagnostic_time, (ii, jj, layers)."""
        L = self.cfg.layers - 1 if self.QUAD[q] in ("uu_i", "vv_i", "sc_ub", "sc_vb", "sc_bb_i") else self.cfg.layers
        out = np.zeros((self.cfg.ii, self.cfg.jj, L), order="F")
        _check(lib().pq_get_quad(self.ctx, int(q), _p(out)), self.ctx)
        return out

    def write_quad(self, path: str, t_scale: float = 1.0, start_time_day: float = 0.0) -> None:
        """The reference's qg<L>_<ii>_quad_av.d file of the current sums."""
        _check(lib().pq_write_quad(self.ctx, path.encode(), t_scale, start_time_day), self.ctx)

    def get_average(self):
        """(psi_av / diagnostic_time as sdata (ii, jj, L), diagnostic_time)."""
        out = np.zeros((self.cfg.ii, self.cfg.jj, self.cfg.layers), order="F")
        t = np.zeros(1)
        _check(lib().pq_get_average(self.ctx, _p(out), _p(t)), self.ctx)
        return out, float(t[0])

    def write_average(self, path: str, t_scale: float = 1.0, start_time_day: float = 0.0) -> None:
        """The reference's qg<L>_<ii>_s_av.d file of the current average."""
        _check(lib().pq_write_average(self.ctx, path.encode(), t_scale, start_time_day), self.ctx)

    def device_bytes(self) -> int:
        return int(lib().pq_device_bytes(self.ctx))

    def last_launch_count(self) -> int:
        return int(lib().pq_last_launch_count(self.ctx))

    def set_tuning(self, **kw) -> None:
        t = Tuning()
        _check(lib().pq_get_tuning(self.ctx, C.byref(t)), self.ctx)
        for k, v in kw.items():
            setattr(t, k, int(v))
        _check(lib().pq_set_tuning(self.ctx, C.byref(t)), self.ctx)

    def get_tuning(self) -> dict:
        t = Tuning()
        _check(lib().pq_get_tuning(self.ctx, C.byref(t)), self.ctx)
        return {"cab_band": t.cab_band, "dst_group": t.dst_group, "cab_kernel": t.cab_kernel, "dst_lanes": t.dst_lanes,
                "dst_lanes_inv": t.dst_lanes_inv, "pdl": t.pdl, "dst_algo": t.dst_algo}

    def autotune(self) -> int:
        """Time the inversion with each row-DST algorithm this context
        supports, select the faster (cached per shape for the process) and
        return it (DST_BUTTERFLY or DST_TENSOR)."""
        ch = C.c_int()
        _check(lib().pq_autotune(self.ctx, C.byref(ch)), self.ctx)
        return ch.value

    def kernel_timing(self, enable: bool) -> None:
        _check(lib().pq_kernel_timing(self.ctx, int(enable)), self.ctx)

    def kernel_times(self) -> dict:
        ms = np.zeros(4)
        n = (C.c_long * 4)()
        _check(lib().pq_kernel_times(self.ctx, _p(ms), n), self.ctx)
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(KERNELS)}


class Batch:
    """Batched Helmholtz solves (pq_batch_*): member k is an (ii, jj, L) helm
    problem with per-layer constants ss[k] (a sequence of length L)."""

    def __init__(self, shapes, ss, device: int = 0, precision: int = PREC_FP64, dst_algo: int = DST_BUTTERFLY):
        n = len(shapes)
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        ii = (C.c_int * n)(*[s[0] for s in self.shapes])
        jj = (C.c_int * n)(*[s[1] for s in self.shapes])
        ll = (C.c_int * n)(*[s[2] for s in self.shapes])
        flat = np.ascontiguousarray(np.concatenate([np.asarray(v, dtype=np.float64) for v in ss]))
        if flat.size != sum(s[2] for s in self.shapes):
            raise ValueError("ss lengths must match the layer counts")
        self.ctx = C.c_void_p()
        rc = lib().pq_batch_create_ex(C.byref(self.ctx), n, ii, jj, ll, _p(flat), int(precision), int(dst_algo),
                                      device)
        if rc != PQ_OK:
            msg = lib().pq_batch_last_error(self.ctx).decode() if self.ctx else ""
            if self.ctx:
                lib().pq_batch_destroy(self.ctx)
                self.ctx = None
            raise PQError(rc, msg)

    def _chk(self, rc):
        if rc != PQ_OK:
            raise PQError(rc, lib().pq_batch_last_error(self.ctx).decode())

    def __len__(self):
        return len(self.shapes)

    def set_rhs(self, k, rhs):
        z = np.asfortranarray(rhs, dtype=np.float64).reshape(self.shapes[k], order="F")
        self._chk(lib().pq_batch_set_rhs(self.ctx, k, _p(z), PTR_HOST))

    def get(self, k):
        out = np.zeros(self.shapes[k], order="F")
        self._chk(lib().pq_batch_get(self.ctx, k, _p(out), PTR_HOST))
        self._chk(lib().pq_batch_sync(self.ctx))
        return out

    def solve_async(self):
        self._chk(lib().pq_batch_solve_async(self.ctx))

    def sync(self):
        self._chk(lib().pq_batch_sync(self.ctx))

    def helm(self, rhs_list):
        """Solve every member; returns the solutions (helm in-place semantics)."""
        arrs = [np.array(np.asfortranarray(r, dtype=np.float64).reshape(self.shapes[k], order="F"), order="F")
                for k, r in enumerate(rhs_list)]
        ptrs = (_dp * len(arrs))(*[_p(a) for a in arrs])
        self._chk(lib().pq_batch_helm(self.ctx, ptrs, PTR_HOST))
        return arrs

    @property
    def stream(self):
        return lib().pq_batch_stream(self.ctx)

    def device_bytes(self):
        return int(lib().pq_batch_device_bytes(self.ctx))

    def launch_count(self):
        return int(lib().pq_batch_launch_count(self.ctx))

    def member_dst_algo(self, k: int) -> int:
        """DST_BUTTERFLY or DST_TENSOR: the row-DST algorithm of member k's FP32 layers."""
        return int(lib().pq_batch_member_dst_algo(self.ctx, int(k)))

    def close(self):
        if self.ctx:
            lib().pq_batch_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Member(Model):
    """A view of one ensemble member's context (owned by the ensemble)."""

    def __init__(self, cfg, ctx):  # noqa: D107 - no context of its own
        self.cfg = cfg
        self.ctx = ctx

    def close(self):
        self.ctx = None


class Ensemble:
    """n runs of one configuration stepped together (pq_ensemble_*): one
    launch per kernel over all members, replayed as CUDA graphs."""

    def __init__(self, cfg: Config, n: int, device: int = 0):
        self.cfg = cfg
        self.ctx = C.c_void_p()
        rc = lib().pq_ensemble_create(C.byref(self.ctx), int(n), C.byref(cfg.desc), device)
        if rc != PQ_OK:
            msg = lib().pq_ensemble_last_error(self.ctx).decode() if self.ctx else ""
            if self.ctx:
                lib().pq_ensemble_destroy(self.ctx)
                self.ctx = None
            raise PQError(rc, msg)
        self.members = [_Member(cfg, C.c_void_p(lib().pq_ensemble_member(self.ctx, k))) for k in range(n)]

    def _chk(self, rc):
        if rc != PQ_OK:
            raise PQError(rc, lib().pq_ensemble_last_error(self.ctx).decode())

    def __len__(self):
        return len(self.members)

    def init(self, k: int, zeta_ic) -> None:
        z = np.asfortranarray(zeta_ic, dtype=np.float64).reshape((self.cfg.ii, self.cfg.jj, self.cfg.layers),
                                                                  order="F")
        self._chk(lib().pq_ensemble_init(self.ctx, int(k), _p(z), PTR_HOST))

    def autotune(self) -> int:
        ch = C.c_int()
        self._chk(lib().pq_ensemble_autotune(self.ctx, C.byref(ch)))
        return ch.value

    def set_dst_algo(self, algo: int) -> None:
        self._chk(lib().pq_ensemble_set_dst_algo(self.ctx, int(algo)))

    def cabaret_step(self, dt: float, tweight_a: float = 0.5, tweight_u: float = 0.5) -> None:
        """One CABARET step with the caller's dt and time weights."""
        _check(lib().pq_cabaret_step(self.ctx, float(dt), float(tweight_a), float(tweight_u)), self.ctx)

    def step_async(self, n: int = 1) -> None:
        self._chk(lib().pq_ensemble_step_async(self.ctx, int(n)))

    def sync(self) -> None:
        self._chk(lib().pq_ensemble_sync(self.ctx))

    def step(self, n: int = 1) -> None:
        self._chk(lib().pq_ensemble_step(self.ctx, int(n)))

    @property
    def stream(self) -> int:
        return int(lib().pq_ensemble_stream(self.ctx) or 0)

    def close(self):
        if getattr(self, "ctx", None):
            for m in self.members:
                m.ctx = None
            lib().pq_ensemble_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuously batched serving of many runs (pq_server_*)."""

    def __init__(self, hbm_budget_bytes: int, device: int = 0):
        self.ctx = C.c_void_p()
        self.shapes = {}
        rc = lib().pq_server_create(C.byref(self.ctx), int(hbm_budget_bytes), device)
        if rc != PQ_OK:
            msg = lib().pq_server_last_error(self.ctx).decode() if self.ctx else ""
            if self.ctx:
                lib().pq_server_destroy(self.ctx)
                self.ctx = None
            raise PQError(rc, msg)

    def _chk(self, rc):
        if rc != PQ_OK:
            raise PQError(rc, lib().pq_server_last_error(self.ctx).decode())

    def submit(self, cfg: Config, zeta_ic, nsteps: int) -> int:
        z = np.asfortranarray(zeta_ic, dtype=np.float64).reshape((cfg.ii, cfg.jj, cfg.layers), order="F")
        rid = C.c_long()
        self._chk(lib().pq_server_submit(self.ctx, C.byref(cfg.desc), _p(z), int(nsteps), C.byref(rid)))
        self.shapes[rid.value] = (cfg.ii, cfg.jj, cfg.layers)
        return rid.value

    def poll(self, max_steps: int = 32):
        a, q = C.c_int(), C.c_int()
        self._chk(lib().pq_server_poll(self.ctx, int(max_steps), C.byref(a), C.byref(q)))
        return a.value, q.value

    def status(self, rid: int) -> int:
        return int(lib().pq_server_status(self.ctx, rid))

    def collect(self, rid: int):
        """(psi, (t_submit, t_start, t_done)) of a finished run; releases it.
        A failed run (status 3) raises PQError with the run's own error code
        and message (and is released too)."""
        psi = np.zeros(self.shapes[rid], order="F")
        t3 = np.zeros(3)
        rc = lib().pq_server_collect(self.ctx, rid, _p(psi), _p(t3))
        msg = lib().pq_server_last_error(self.ctx).decode() if rc != PQ_OK else ""
        if self.status(rid) == -1:  # released (finished or failed)
            self.shapes.pop(rid, None)
        if rc != PQ_OK:
            raise PQError(rc, msg)
        return psi, tuple(t3)

    def run_until_done(self, max_steps: int = 32):
        while True:
            a, q = self.poll(max_steps)
            if a == 0 and q == 0:
                return

    def clock(self) -> float:
        return float(lib().pq_server_clock(self.ctx))

    def device_bytes(self) -> int:
        return int(lib().pq_server_device_bytes(self.ctx))

    def launches(self) -> int:
        return int(lib().pq_server_launches(self.ctx))

    def close(self):
        if self.ctx:
            lib().pq_server_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
