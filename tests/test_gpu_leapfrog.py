"""GPU parity of the leapfrog scheme (centred Jacobian + RAW filter) against
the oracle: both time levels of psi, zeta, rel and zeta_old.  FP64 bar:
relative L2 <= 1e-12 per step, <= 1e-9 after 100 steps."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12
TOL_100 = 1e-9
LEVEL_FIELDS = ["psi", "zeta", "rel", "zeta_old", "psi2", "zeta2", "rel2", "zeta_old2"]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def double_gyre(ii, layers=3, dt=1800.0, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5),
         5: (2.5e4, 5.0e4, 7.5e4, 1.0e5, 1.5e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75), 5: (1.5, 0.75, 0.375, 0.1875)}[layers]
    p = pq.double_gyre_physical(ii, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp,
                                scheme=pq.SCHEME_LEAPFROG, **kw)
    return pq.Config.from_physical(p)


def start(cfg, seed):
    # init_rand fills both time levels with independent draws
    ic = np.stack([pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed + 1000 * lv, amplitude=1e-7 * cfg.t_scale,
                              sigma=3.0) for lv in range(2)], axis=3)
    ic = np.asfortranarray(ic)
    g = pq.Model(cfg)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return g, o


def compare(g, o, tol):
    worst = {f: rel_l2(g.get(f), o.get(f)) for f in LEVEL_FIELDS}
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst


def test_leapfrog_init_matches_oracle():
    g, o = start(double_gyre(65, 3), seed=21)
    compare(g, o, TOL_STEP)
    assert abs(g.scalars()["model_time"] - o.scalars()["model_time"]) <= 1e-14


@pytest.mark.parametrize("ii,layers", [(33, 1), (65, 2), (129, 3), (65, 5)])
def test_leapfrog_steps_match_oracle(ii, layers):
    g, o = start(double_gyre(ii, layers), seed=22 + layers)
    for n in (1, 1, 2, 3):   # both sub-step parities, graph and eager paths
        g.step(n)
        o.step(n)
        compare(g, o, TOL_STEP * 10)


def test_leapfrog_hundred_steps_and_energy():
    g, o = start(double_gyre(129, 3), seed=25)
    g.step(100)
    o.step(100)
    compare(g, o, TOL_100)
    ek_g, ep_g = g.energy()
    ek_o, ep_o = o.energy()
    assert rel_l2(ek_g, ek_o) <= TOL_100
    assert abs(ep_g - ep_o) <= TOL_100 * abs(ep_o)
    sg, so = g.scalars(), o.scalars()
    assert abs(sg["model_time"] - so["model_time"]) <= 1e-12 * so["model_time"]


def test_leapfrog_rejects_mixed_and_adaptive():
    for kw in (dict(precision=pq.PREC_MIXED), dict(adapt_dt=1)):
        with pytest.raises(Exception):
            pq.Model(double_gyre(65, 3, **kw))
