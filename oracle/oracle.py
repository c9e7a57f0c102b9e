"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU FP64 oracle.

The oracle (pq_oracle.cpp) is a line-by-line C++ restatement of PEQUOD's
serial QG time-step path.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module, and only as the checker; the
pequod_b200 product never imports it.

Arrays follow the reference's Fortran conventions: numpy arrays in Fortran
(column-major) order, i fastest; sdata (ii, jj, L), full data arrays
(ii+2, jj+2, L), FLUX_II (ii+3, jj+2, L), FLUX_JJ (ii+2, jj+3, L).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libpq_oracle.so")

BC_PARTIAL_SLIP, BC_NO_SLIP, BC_FREE_SLIP = 1, 2, 3

_dp = C.POINTER(C.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, no fast-math, no FMA)."""
    src = os.path.join(_HERE, "pq_oracle.cpp")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_SO)
        L.or_helm_create.restype = C.c_void_p
        L.or_helm_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_int]
        L.or_helm_destroy.argtypes = [C.c_void_p]
        L.or_helm.argtypes = [C.c_void_p, _dp]
        L.or_sint.argtypes = [C.c_void_p, _dp]
        L.or_add_laplace_bc_rhs.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp]
        L.or_apply_dirichlet_bc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp]
        L.or_mean.restype = C.c_double
        L.or_mean.argtypes = [C.c_int, C.c_int, C.c_int, _dp]
        L.or_energy.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.or_strat_l2.argtypes = [C.c_double] * 3 + [_dp, _dp]
        L.or_strat_l3.argtypes = [C.c_double] * 5 + [_dp] * 4
        L.or_strat_from_parameters.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double] + [_dp] * 6
        L.or_strat_from_rd.argtypes = [C.c_int, _dp, _dp, C.c_double] + [_dp] * 6
        L.or_eigen_real_tridiag.argtypes = [C.c_int, _dp, _dp, _dp]
        L.or_inverse.argtypes = [C.c_int, _dp, _dp]
        L.or_solve.argtypes = [C.c_int, _dp, _dp, _dp]
        L.or_determinant.restype = C.c_double
        L.or_determinant.argtypes = [C.c_int, _dp]
        L.or_model_create.restype = C.c_void_p
        L.or_model_create.argtypes = [C.c_void_p]
        L.or_model_destroy.argtypes = [C.c_void_p]
        L.or_model_init.argtypes = [C.c_void_p, _dp]
        L.or_model_step.argtypes = [C.c_void_p, C.c_int]
        L.or_model_get.restype = C.c_long
        L.or_model_get.argtypes = [C.c_void_p, C.c_char_p, _dp]
        L.or_model_set.restype = C.c_long
        L.or_model_set.argtypes = [C.c_void_p, C.c_char_p, _dp]
        L.or_model_scalars.argtypes = [C.c_void_p, _dp]
        L.or_model_energy.argtypes = [C.c_void_p, _dp, _dp]
        L.or_model_cfl.restype = C.c_double
        L.or_model_cfl.argtypes = [C.c_void_p]
        L.or_pv_inversion.argtypes = [C.c_void_p, _dp, _dp]
        L.or_model_pickup.argtypes = [C.c_void_p, C.c_double]
        L.or_model_step_to_dump.argtypes = [C.c_void_p]
        L.or_model_average.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.or_model_get_average.restype = C.c_double
        L.or_model_get_average.argtypes = [C.c_void_p, _dp]
        L.or_model_get_quad.restype = C.c_long
        L.or_model_get_quad.argtypes = [C.c_void_p, C.c_int, _dp]
        L.or_model_finish_step.argtypes = [C.c_void_p]
        L.or_setup_double_gyre.argtypes = [C.c_void_p, C.c_void_p, _dp]
        L.or_make_ic.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_double, C.c_double, _dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1)
    return a.ctypes.data_as(_dp)


def farray(shape, fill=0.0):
    return np.full(shape, fill, dtype=np.float64, order="F")


class Helm:
    """helm_cache + helm (qg3p_helmholtz.F90:292-386, 614-769)."""

    def __init__(self, ii, jj, layers, ss, periodic_j=False):
        ss = np.ascontiguousarray(np.asarray(ss, dtype=np.float64).reshape(layers))
        self.ii, self.jj, self.layers = ii, jj, layers
        self.h = lib().or_helm_create(ii, jj, layers, _p(ss), int(periodic_j))
        if not self.h:
            raise ValueError("or_helm_create failed")

    def __call__(self, zeta: np.ndarray) -> np.ndarray:
        z = np.asfortranarray(zeta, dtype=np.float64).reshape((self.ii, self.jj, self.layers), order="F").copy(order="F")
        rc = lib().or_helm(self.h, _p(z))
        if rc:
            raise RuntimeError(f"or_helm rc={rc}")
        return z

    def sint(self, x: np.ndarray) -> np.ndarray:
        x = np.array(x, dtype=np.float64)
        assert x.size == self.ii - 1
        rc = lib().or_sint(self.h, _p(x))
        if rc:
            raise RuntimeError(f"or_sint rc={rc}")
        return x

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_helm_destroy(self.h)
            self.h = None


def add_laplace_bc_rhs(rhs, bc, bc_d=None, periodic_j=False):
    r = np.asfortranarray(rhs, dtype=np.float64).copy(order="F")
    ii, jj = r.shape[0], r.shape[1]
    L = 1 if r.ndim == 2 else r.shape[2]
    lib().or_add_laplace_bc_rhs(ii, jj, L, int(periodic_j), bc, bc if bc_d is None else bc_d, _p(r))
    return r


def apply_dirichlet_bc(z, bc, bc_d=None, periodic_j=False):
    r = np.asfortranarray(z, dtype=np.float64).copy(order="F")
    ii, jj = r.shape[0], r.shape[1]
    L = 1 if r.ndim == 2 else r.shape[2]
    lib().or_apply_dirichlet_bc(ii, jj, L, int(periodic_j), bc, bc if bc_d is None else bc_d, _p(r))
    return r


def mean(psi, periodic_j=False):
    p = np.asfortranarray(psi, dtype=np.float64)
    return lib().or_mean(p.shape[0], p.shape[1], int(periodic_j), _p(p))


def energy(psi_data, h, s2, periodic_j=False):
    p = np.asfortranarray(psi_data, dtype=np.float64)
    ii, jj, L = p.shape[0] - 2, p.shape[1] - 2, p.shape[2]
    ekin = np.zeros(L)
    epot = np.zeros(1)
    lib().or_energy(ii, jj, L, int(periodic_j), _p(np.ascontiguousarray(h, dtype=np.float64)),
                    _p(np.ascontiguousarray(s2, dtype=np.float64)), _p(p), _p(ekin), _p(epot))
    return ekin, float(epot[0])


def strat_from_parameters(h, s1, s2, l_scale=1.0):
    """allocate_stratification_parameters: h[L], s1[L-1] (=s1(2:L)), s2[L-1]."""
    L = len(h)
    out = [np.zeros(L) for _ in range(4)] + [np.zeros((L, L), order="F") for _ in range(2)]
    s1a = np.ascontiguousarray(s1 if L > 1 else [0.0], dtype=np.float64)
    s2a = np.ascontiguousarray(s2 if L > 1 else [0.0], dtype=np.float64)
    rc = lib().or_strat_from_parameters(L, _p(np.ascontiguousarray(h, dtype=np.float64)), _p(s1a), _p(s2a),
                                        l_scale, *[_p(o) for o in out])
    if rc:
        raise RuntimeError(f"or_strat_from_parameters rc={rc}")
    keys = ["h", "s1", "s2", "ss", "m2z", "z2m"]
    return dict(zip(keys, out))


def strat_from_rd(rd, h, l_scale=1.0):
    L = len(h)
    out = [np.zeros(L) for _ in range(4)] + [np.zeros((L, L), order="F") for _ in range(2)]
    rda = np.ascontiguousarray(list(rd) + [0.0], dtype=np.float64)
    rc = lib().or_strat_from_rd(L, _p(rda), _p(np.ascontiguousarray(h, dtype=np.float64)), l_scale,
                                *[_p(o) for o in out])
    if rc:
        raise RuntimeError(f"or_strat_from_rd rc={rc}")
    return dict(zip(["h", "s1", "s2", "ss", "m2z", "z2m"], out))


def eigen(a):
    a = np.asfortranarray(a, dtype=np.float64)
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n), order="F")
    rc = lib().or_eigen_real_tridiag(n, _p(a), _p(w), _p(v))
    if rc:
        raise RuntimeError("eigen failed")
    return w, v


def inverse(a):
    a = np.asfortranarray(a, dtype=np.float64)
    out = np.zeros_like(a, order="F")
    if lib().or_inverse(a.shape[0], _p(a), _p(out)):
        raise RuntimeError("singular")
    return out


def solve(a, rhs):
    a = np.asfortranarray(a, dtype=np.float64)
    x = np.zeros(a.shape[0])
    lib().or_solve(a.shape[0], _p(a), _p(np.ascontiguousarray(rhs, dtype=np.float64)), _p(x))
    return x


def determinant(a):
    a = np.asfortranarray(a, dtype=np.float64)
    return lib().or_determinant(a.shape[0], _p(a))



class _Physical(C.Structure):
    _fields_ = [
        ("ii", C.c_int), ("jj", C.c_int), ("layers", C.c_int),
        ("basinscale", C.c_double), ("dt", C.c_double), ("f0", C.c_double), ("beta", C.c_double),
        ("H", C.c_double * 8), ("gprime", C.c_double * 8), ("tau", C.c_double),
        ("wind_asym", C.c_double), ("wind_tilt", C.c_double), ("wind_shift", C.c_double),
        ("visc", C.c_double), ("visc_bot", C.c_double), ("alpha", C.c_double), ("partial_slip", C.c_int),
        ("max_dt", C.c_double), ("u_scale", C.c_double),
    ]


class _Setup(C.Structure):
    _fields_ = [
        ("l_scale", C.c_double), ("t_scale", C.c_double), ("dt", C.c_double), ("max_dt", C.c_double),
        ("alpha", C.c_double), ("viscosity", C.c_double), ("visc_bot", C.c_double), ("bc_type", C.c_int),
        ("beta", C.c_double * 8), ("h", C.c_double * 8), ("s1", C.c_double * 8), ("s2", C.c_double * 8),
        ("ss", C.c_double * 8), ("m2z", C.c_double * 64), ("z2m", C.c_double * 64),
    ]


PHYSICAL_KEYS = ("ii", "jj", "layers", "basinscale", "dt", "f0", "beta", "H", "gprime", "tau", "wind_asym",
                 "wind_tilt", "wind_shift", "visc", "visc_bot", "alpha", "partial_slip", "max_dt", "u_scale")


def setup_double_gyre(phys) -> dict:
    """The double-gyre driver's set-up (qg3.F90:150-307) computed by the
    oracle from physical (cgs) parameters alone: a dict with the keys of
    PHYSICAL_KEYS (H and gprime sequences) or any object with those
    attributes.  Returns the oracle's model parameters, the wind forcing and
    t_scale."""
    get = (lambda k: phys[k]) if isinstance(phys, dict) else (lambda k: getattr(phys, k))
    p = _Physical()
    for k in PHYSICAL_KEYS:
        v = get(k)
        if k in ("H", "gprime"):
            for n, x in enumerate(list(v)[:8]):
                getattr(p, k)[n] = float(x)
        else:
            setattr(p, k, v)
    L = p.layers
    st = _Setup()
    wind = np.zeros((p.ii, p.jj), order="F")
    rc = lib().or_setup_double_gyre(C.addressof(p), C.addressof(st), _p(wind))
    if rc:
        raise RuntimeError(f"or_setup_double_gyre rc={rc}")
    m2z = np.array(st.m2z[: L * L]).reshape((L, L), order="F")
    z2m = np.array(st.z2m[: L * L]).reshape((L, L), order="F")
    return dict(ii=p.ii, jj=p.jj, layers=L, dt=st.dt, max_dt=st.max_dt, alpha=st.alpha, viscosity=st.viscosity,
                visc_bot=st.visc_bot, bc_type=st.bc_type, beta=list(st.beta[:L]), h=list(st.h[:L]),
                s1=list(st.s1[:L]), s2=list(st.s2[:L]), ss=np.array(st.ss[:L]), m2z=m2z, z2m=z2m,
                force_wind=wind, t_scale=st.t_scale, l_scale=st.l_scale,
                ra_nu=0.02, ra_alpha=0.5)  # qg3p_params.F90:31-36


def cfg_from(cfg) -> dict:
    """The oracle's configuration for a model description.

    A description built from physical parameters (it carries them as
    `physical`) is set up again here, by the oracle's own restatement of the
    driver; only the run's switches (scheme, limiter, channel, adaptive step)
    are taken from the description.  A hand-written description (no
    `physical`, e.g. a Helmholtz test problem) is taken as it stands."""
    d = cfg.desc
    L = d.layers
    out = dict(ii=d.ii, jj=d.jj, layers=L, periodic_j=d.periodic_j, scheme=d.scheme, limiter=d.limiter,
               adapt_dt=d.adapt_dt, target_cfl=d.target_cfl, max_dt_increase=d.max_dt_increase)
    phys = getattr(cfg, "physical", None)
    if phys is not None:
        st = setup_double_gyre(phys)
        st.pop("t_scale")
        st.pop("l_scale")
        out.update(st)
        return out
    m2z = np.array(d.m2z[: L * L]).reshape((L, L), order="F")
    z2m = np.array(d.z2m[: L * L]).reshape((L, L), order="F")
    out.update(dt=d.dt, beta=list(d.beta[:L]), h=list(d.h[:L]), s1=list(d.s1[:L]), s2=list(d.s2[:L]),
               ss=np.array(d.ss[:L]), m2z=m2z, z2m=z2m, viscosity=d.viscosity, visc_bot=d.visc_bot,
               bc_type=d.bc_type, alpha=d.alpha, force_wind=getattr(cfg, "wind", None), max_dt=d.max_dt,
               ra_nu=d.ra_nu, ra_alpha=d.ra_alpha)
    return out


def make_ic(ii, jj, layers, seed=0, amplitude=1.0, sigma=3.0) -> np.ndarray:
    """The seeded synthetic initial PV, (ii, jj, layers), Fortran order."""
    out = np.zeros((ii, jj, layers), order="F")
    rc = lib().or_make_ic(ii, jj, layers, seed, amplitude, sigma, _p(out))
    if rc:
        raise RuntimeError(f"or_make_ic rc={rc}")
    return out

class _Params(C.Structure):
    _fields_ = [
        ("ii", C.c_int), ("jj", C.c_int), ("layers", C.c_int),
        ("periodic_j", C.c_int), ("scheme", C.c_int), ("limiter", C.c_int), ("bc_type", C.c_int),
        ("alpha", C.c_double), ("dt", C.c_double), ("viscosity", C.c_double), ("visc_bot", C.c_double),
        ("adapt_dt", C.c_int),
        ("target_cfl", C.c_double), ("max_dt", C.c_double), ("max_dt_increase", C.c_double),
        ("ra_nu", C.c_double), ("ra_alpha", C.c_double),
        ("beta", _dp), ("h", _dp), ("s1", _dp), ("s2", _dp), ("ss", _dp), ("m2z", _dp), ("z2m", _dp),
        ("force_wind", _dp),
    ]


class Model:
    """The serial qg3 time loop (qg3.F90:590-967) on reference-layout state.

    ``cfg`` is the non-dimensional configuration dictionary of cfg_from /
    setup_double_gyre (keys: ii, jj, layers, dt, beta, h, s1, s2, ss, m2z,
    z2m, viscosity, visc_bot, bc_type, alpha, force_wind, scheme, ...).
    """

    def __init__(self, cfg: dict):
        self.cfg = cfg
        L = cfg["layers"]
        self._keep = {}

        def arr(name, shape=None):
            a = np.ascontiguousarray(np.asarray(cfg[name], dtype=np.float64).ravel(order="F"))
            self._keep[name] = a
            return _p(a)

        P = _Params()
        P.ii, P.jj, P.layers = cfg["ii"], cfg["jj"], L
        P.periodic_j = int(cfg.get("periodic_j", 0))
        P.scheme = cfg.get("scheme", 0)
        P.limiter = cfg.get("limiter", 1)
        P.bc_type = cfg.get("bc_type", BC_PARTIAL_SLIP)
        P.alpha = cfg.get("alpha", 0.0)
        P.dt = cfg["dt"]
        P.viscosity = cfg["viscosity"]
        P.visc_bot = cfg["visc_bot"]
        P.adapt_dt = cfg.get("adapt_dt", 0)
        P.target_cfl = cfg.get("target_cfl", 0.1)
        P.max_dt = cfg.get("max_dt", 1e300)
        P.max_dt_increase = cfg.get("max_dt_increase", 1.5)
        P.ra_nu = cfg.get("ra_nu", 0.02)
        P.ra_alpha = cfg.get("ra_alpha", 0.5)
        for k in ["beta", "h", "s1", "s2", "ss", "m2z", "z2m"]:
            setattr(P, k, arr(k))
        if cfg.get("force_wind") is not None:
            P.force_wind = arr("force_wind")
        self._P = P
        self.m = lib().or_model_create(C.byref(P))
        if not self.m:
            raise ValueError("or_model_create failed")

    def init(self, zeta_ic: np.ndarray) -> None:
        z = np.asfortranarray(zeta_ic, dtype=np.float64)
        rc = lib().or_model_init(self.m, _p(z))
        if rc:
            raise RuntimeError(f"or_model_init rc={rc}")

    def step(self, n: int = 1) -> None:
        rc = lib().or_model_step(self.m, n)
        if rc:
            raise RuntimeError(f"or_model_step rc={rc}")

    def shape_of(self, name):
        ii, jj, L = self.cfg["ii"], self.cfg["jj"], self.cfg["layers"]
        if name in ("ui", "uimo", "zeta_fi", "flux_i"):
            return (ii + 3, jj + 2, L)
        if name in ("uj", "ujmo", "zeta_fj", "flux_j"):
            return (ii + 2, jj + 3, L)
        if name == "corr" and self.cfg.get("periodic_j", 0):
            return (ii, jj, L, 2)
        if name in ("res", "res_beta", "corr"):
            return (ii, jj, L)
        return (ii + 2, jj + 2, L)

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.shape_of(name), order="F")
        n = lib().or_model_get(self.m, name.encode(), _p(out))
        if n < 0:
            raise KeyError(name)
        return out

    def set(self, name: str, value: np.ndarray) -> None:
        v = np.asfortranarray(value, dtype=np.float64).reshape(self.shape_of(name), order="F")
        if lib().or_model_set(self.m, name.encode(), _p(v)) < 0:
            raise KeyError(name)

    def sdata(self, name: str) -> np.ndarray:
        a = self.get(name)
        return np.asfortranarray(a[1:-1, 1:-1, :])

    def average(self, enable: bool = True, threshold: float = 0.0) -> None:
        """Start (clearing) or stop the time average of psi."""
        lib().or_model_average(self.m, int(enable), float(threshold))

    QUAD = ("uu", "vv", "uu_i", "vv_i", "uv", "ur", "vr", "rr", "pr", "uz", "vz", "zz", "zr", "pp", "pz", "ut", "vt",
            "rt", "tt", "sc_ub", "sc_vb", "sc_bb", "sc_bb_i")

    def get_quad(self, q: int):
        """Quad accumulator q divided by diagnostic_time, (ii, jj, layers)."""
        n = lib().or_model_get_quad(self.m, int(q), None)
        if n < 0:
            raise KeyError(q)
        ii, jj = self.cfg["ii"], self.cfg["jj"]
        out = np.zeros(n)
        lib().or_model_get_quad(self.m, int(q), _p(out))
        t = lib().or_model_get_average(self.m, None)
        return out.reshape((ii, jj, n // (ii * jj)), order="F") * (1.0 / t)

    def get_average(self):
        """(psi_av / diagnostic_time as (ii, jj, L), diagnostic_time)."""
        s = np.zeros((self.cfg["ii"], self.cfg["jj"], self.cfg["layers"]), order="F")
        t = lib().or_model_get_average(self.m, _p(s))
        return (s * (1.0 / t) if t > 0 else s), t

    def step_to_dump(self) -> None:
        """One CABARET step up to the reference's checkpoint point."""
        rc = lib().or_model_step_to_dump(self.m)
        if rc:
            raise RuntimeError(f"or_model_step_to_dump rc={rc}")

    def finish_step(self) -> None:
        """The rest of that step: corrector, zeta_old = zeta, time."""
        rc = lib().or_model_finish_step(self.m)
        if rc:
            raise RuntimeError(f"or_model_finish_step rc={rc}")

    def dump_fields(self) -> dict:
        """The fields a checkpoint holds, in reference layout."""
        names = ["psi", "zeta", "ui", "uj", "zeta_fi", "zeta_fj", "res", "res_beta"]
        if self.cfg.get("scheme", 0) == 1:
            names = ["psi", "zeta", "psi2", "zeta2"]
        return {n: self.get(n) for n in names}

    def pickup(self, ckpt: dict) -> None:
        """START_PICKUP from a checkpoint dictionary (read_checkpoint's
        output): load its fields, then or_model_pickup."""
        leap = self.cfg.get("scheme", 0) == 1
        names = (["psi", "zeta", "ui", "uj", "zeta_fi", "zeta_fj", "res", "res_beta"] if not leap else
                 ["psi", "psi2", "zeta", "zeta2"])
        for n in names:
            self.set(n, ckpt[n])
        rc = lib().or_model_pickup(self.m, float(ckpt.get("dt", self.cfg["dt"])))
        if rc:
            raise RuntimeError(f"or_model_pickup rc={rc}")

    def scalars(self):
        out = np.zeros(4)
        lib().or_model_scalars(self.m, _p(out))
        return dict(dt=out[0], tweight_a=out[1], tweight_u=out[2], model_time=out[3])

    def energy(self):
        L = self.cfg["layers"]
        ekin = np.zeros(L)
        epot = np.zeros(1)
        rc = lib().or_model_energy(self.m, _p(ekin), _p(epot))
        if rc:
            raise RuntimeError("NaN value encountered")
        return ekin, float(epot[0])

    def cfl(self) -> float:
        return lib().or_model_cfl(self.m)

    def pv_inversion(self, zeta_data: np.ndarray) -> np.ndarray:
        z = np.asfortranarray(zeta_data, dtype=np.float64)
        psi = np.zeros_like(z, order="F")
        rc = lib().or_pv_inversion(self.m, _p(z), _p(psi))
        if rc:
            raise RuntimeError(f"pv_inversion rc={rc}")
        return psi

    def __del__(self):
        if getattr(self, "m", None):
            lib().or_model_destroy(self.m)
            self.m = None


# ---------------------------------------------------------------------------
# Checkpoint files (qg3.F90:836-878 write, qg3p_io.F90:202-314 read).  Each
# record is Fortran unformatted stream output: a 4-byte byte count, the REAL(8)
# data column-major, the byte count again (qg3p_io.F90:574-651).
#   _s.d       model_time_day, total_time_day, L x psi sdata (ii, jj),
#              L x zeta sdata; leapfrog records hold level 1 then level 2.
#   _s_supp.d  (CABARET) model_time_day, total_time_day, dt,
#              L x ui   data(fa_i_min+1:fa_i_max,   fa_j_min+1:fa_j_max-1),
#              L x uj   data(fa_i_min+1:fa_i_max-1, fa_j_min+1:fa_j_max),
#              L x zeta_fi, L x zeta_fj (same ranges), L x res, L x res_beta.
# With one process and no neighbours the ranges are, in the 1-based indexes
# of the reference-layout arrays used here, ui / zeta_fi i in [3, ii+1],
# j in [3, jj]; uj / zeta_fj i in [3, ii], j in [3, jj+1].

def _records(path):
    raw = open(path, "rb").read()
    out, k = [], 0
    while k < len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, k)[0])
        data = np.frombuffer(raw, "<f8", n // 8, k + 4).copy()
        m = int(np.frombuffer(raw, "<i4", 1, k + 4 + n)[0])
        if m != n or n % 8:
            raise ValueError(f"{path}: bad record framing at byte {k}")
        out.append(data)
        k += 8 + n
    return out


def _write_records(path, recs):
    with open(path, "wb") as f:
        for r in recs:
            r = np.asarray(r, dtype="<f8").ravel(order="F")
            n = np.array([r.size * 8], dtype="<i4")
            f.write(n.tobytes() + r.tobytes() + n.tobytes())


def _face_ranges(ii, jj, periodic_j=False):
    # 0-based slices of the saved FLUX_II / FLUX_JJ faces (qg3.F90:864-875):
    # rows fa_j_min+1 .. fa_j_max-1 and faces fa_j_min+1 .. fa_j_max, where a
    # channel (its own j neighbour) has fa_j_min = 1, fa_j_max = jj + 2 and a
    # closed basin fa_j_min = 2, fa_j_max = jj + 1 (qg3p_base.F90:893-918).
    lo = 1 if periodic_j else 2
    hi = jj + 1 if periodic_j else jj
    return (slice(2, ii + 1), slice(lo, hi)), (slice(2, ii), slice(lo, hi + 1))


def read_checkpoint(s_path, supp_path, ii, jj, L, leapfrog=False, periodic_j=False):
    """Parse a checkpoint into reference-layout arrays and the three times."""
    rs = _records(s_path)
    out = {"model_time_day": float(rs[0][0]), "total_time_day": float(rs[1][0])}
    nlev = 2 if leapfrog else 1
    if len(rs) != 2 + 2 * L or any(r.size != ii * jj * nlev for r in rs[2:]):
        raise ValueError("unexpected _s record layout")
    for k, name in enumerate(("psi", "zeta")):
        for lv in range(nlev):
            a = np.zeros((ii + 2, jj + 2, L), order="F")
            for l in range(L):
                r = rs[2 + k * L + l]
                a[1:-1, 1:-1, l] = r[lv * ii * jj:(lv + 1) * ii * jj].reshape((ii, jj), order="F")
            out[name + ("2" if lv else "")] = a
    if leapfrog or supp_path is None:
        return out
    rp = _records(supp_path)
    if len(rp) != 3 + 6 * L:
        raise ValueError("unexpected _s_supp record layout")
    if rp[0][0] != out["model_time_day"] or rp[1][0] != out["total_time_day"]:
        raise ValueError("Input times do not match in CABARET checkpoint data")
    out["dt"] = float(rp[2][0])
    (fi_i, fi_j), (fj_i, fj_j) = _face_ranges(ii, jj, periodic_j)
    k = 3
    for name, shape, (si, sj) in (("ui", (ii + 3, jj + 2), (fi_i, fi_j)), ("uj", (ii + 2, jj + 3), (fj_i, fj_j)),
                                  ("zeta_fi", (ii + 3, jj + 2), (fi_i, fi_j)),
                                  ("zeta_fj", (ii + 2, jj + 3), (fj_i, fj_j))):
        a = np.zeros(shape + (L,), order="F")
        for l in range(L):
            a[si, sj, l] = rp[k].reshape((si.stop - si.start, sj.stop - sj.start), order="F")
            k += 1
        out[name] = a
    for name in ("res", "res_beta"):
        a = np.zeros((ii, jj, L), order="F")
        for l in range(L):
            a[:, :, l] = rp[k].reshape((ii, jj), order="F")
            k += 1
        out[name] = a
    return out


def write_checkpoint(s_path, supp_path, fields, model_time_day, total_time_day, dt=None, leapfrog=False,
                     periodic_j=False):
    """Write reference-layout arrays as a checkpoint (the reference's writer)."""
    L = fields["psi"].shape[2]
    recs = [[model_time_day], [total_time_day]]
    for name in ("psi", "zeta"):
        for l in range(L):
            r = fields[name][1:-1, 1:-1, l].ravel(order="F")
            if leapfrog:
                r = np.concatenate([r, fields[name + "2"][1:-1, 1:-1, l].ravel(order="F")])
            recs.append(r)
    _write_records(s_path, recs)
    if leapfrog or supp_path is None:
        return
    ii, jj = fields["psi"].shape[0] - 2, fields["psi"].shape[1] - 2
    (fi_i, fi_j), (fj_i, fj_j) = _face_ranges(ii, jj, periodic_j)
    recs = [[model_time_day], [total_time_day], [dt]]
    for name, (si, sj) in (("ui", (fi_i, fi_j)), ("uj", (fj_i, fj_j)), ("zeta_fi", (fi_i, fi_j)),
                           ("zeta_fj", (fj_i, fj_j))):
        for l in range(L):
            recs.append(fields[name][si, sj, l].ravel(order="F"))
    for name in ("res", "res_beta"):
        for l in range(L):
            recs.append(fields[name][:, :, l].ravel(order="F"))
    _write_records(supp_path, recs)
