"""GPU parity of the mixed-precision form (PQ_PREC_MIXED).

FP32 storage and arithmetic for the CABARET fields and the baroclinic
Helmholtz modes; FP64 for psi, the barotropic mode, the projections and the
reductions.  Bar: relative L2 error of the streamfunction <= 1e-6 against the
FP64 oracle (and against the FP64 CUDA path), per solve and after 100 steps.
"""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_PSI = 1e-6


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def double_gyre(ii, layers=3, dt=1800.0, precision=pq.PREC_MIXED, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5),
         5: (2.5e4, 5.0e4, 7.5e4, 1.0e5, 1.5e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75), 5: (1.5, 0.75, 0.375, 0.1875)}[layers]
    p = pq.double_gyre_physical(ii, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp,
                                precision=precision, **kw)
    return pq.Config.from_physical(p)


def start(cfg, seed):
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    g = pq.Model(cfg)
    g.init_perturb(ic)
    return g, ic


@pytest.mark.parametrize("ii,layers", [(33, 1), (65, 3), (257, 3), (129, 5)])
def test_mixed_pv_inversion(ii, layers):
    cfg = double_gyre(ii, layers)
    rng = np.random.default_rng(ii + 7 * layers)
    zeta = np.asfortranarray(rng.standard_normal((ii, ii, layers)))
    g = pq.Model(cfg)
    psi = g.pv_inversion(zeta)
    om = O.Model(O.cfg_from(cfg))
    zd = np.zeros((ii + 2, ii + 2, layers), order="F")
    zd[1:-1, 1:-1, :] = zeta
    ref = om.pv_inversion(zd)[1:-1, 1:-1, :]
    assert rel_l2(psi, ref) <= TOL_PSI, rel_l2(psi, ref)


def test_mixed_hundred_steps_vs_oracle():
    cfg = double_gyre(129, 3)
    g, ic = start(cfg, seed=11)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    g.step(100)
    o.step(100)
    e = rel_l2(g.get("psi"), o.get("psi"))
    assert e <= TOL_PSI, e
    assert rel_l2(g.get("zeta"), o.get("zeta")) <= 1e-5
    ek_g, ep_g = g.energy()
    ek_o, ep_o = o.energy()
    assert rel_l2(ek_g, ek_o) <= 1e-5
    assert abs(ep_g - ep_o) <= 1e-5 * abs(ep_o)


@pytest.mark.parametrize("ii", [513, 1025])
def test_mixed_vs_fp64_gpu(ii):
    """The same run in both forms on the GPU, 100 steps at dt = 900 s."""
    out = {}
    for prec in (pq.PREC_FP64, pq.PREC_MIXED):
        cfg = double_gyre(ii, 3, dt=900.0, precision=prec)
        g, _ = start(cfg, seed=3)
        g.step(100)
        out[prec] = g.get("psi")
        g.close()
    e = rel_l2(out[pq.PREC_MIXED], out[pq.PREC_FP64])
    assert e <= TOL_PSI, e


def test_mixed_adaptive_dt():
    """The non-fused step (predictor in the forward DST) in FP32 storage."""
    cfg = double_gyre(65, 3, adapt_dt=1, target_cfl=0.1, max_dt=86400.0)
    g, ic = start(cfg, seed=12)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    g.step(20)
    o.step(20)
    assert rel_l2(g.get("psi"), o.get("psi")) <= TOL_PSI
    assert abs(g.scalars()["dt"] - o.scalars()["dt"]) <= 1e-5 * o.scalars()["dt"]


def test_mixed_state_roundtrip():
    """Host reads/writes of the FP32 state convert exactly (float values)."""
    cfg = double_gyre(65, 3)
    g, _ = start(cfg, seed=13)
    g.step(3)
    for f in ("zeta", "res", "res_beta", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj"):
        a = g.get(f)
        assert np.array_equal(a, a.astype(np.float32).astype(np.float64)), f
        g.set(f, a)
        assert np.array_equal(g.get(f), a), f
