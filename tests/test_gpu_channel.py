"""The channel (periodic in j) CABARET time step on the device against the
oracle: momentum-corrected inversion (modes_to_z_correct_momentum), the
periodic stencils of the four channel kernels, energy and the adaptive
step.  The comparison covers the nodes and faces the device stores (the
reference's halo rows are copies of them).  FP64 bar: relative L2 <= 1e-12
per step, <= 1e-9 after 100 steps; mixed form <= 1e-6 on psi."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12
TOL_100 = 1e-9


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def channel(ii, jj, layers=3, dt=1800.0, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, jj=jj, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = 1
    return cfg


def start(cfg, seed):
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    g = pq.Model(cfg)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return g, o


def owned(name, a, ii, jj):
    """The part of a reference-layout array the device stores."""
    if name in ("ui", "uimo", "zeta_fi"):
        return a[1:ii + 1, 1:jj + 1]
    if name in ("uj", "ujmo", "zeta_fj"):
        return a[1:ii + 1, 1:jj + 1]
    if name in ("res", "res_beta"):
        return a
    return a[1:-1, 1:-1]


FIELDS = ["psi", "zeta", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res", "res_beta"]


def compare(g, o, tol, fields=FIELDS):
    ii, jj = g.cfg.ii, g.cfg.jj
    worst = {f: rel_l2(owned(f, g.get(f), ii, jj), owned(f, o.get(f), ii, jj)) for f in fields}
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst
    return worst


@pytest.mark.parametrize("ii,jj,layers", [(65, 64, 3), (129, 96, 2), (33, 40, 1)])
def test_channel_init_matches_oracle(ii, jj, layers):
    g, o = start(channel(ii, jj, layers), seed=51)
    compare(g, o, TOL_STEP, ["psi", "zeta", "zeta_old", "rel"])


@pytest.mark.parametrize("partial_slip", [True, False])
def test_channel_pv_inversion_matches_oracle(partial_slip):
    cfg = channel(129, 128, 3, partial_slip=partial_slip)
    rng = np.random.default_rng(52)
    zeta = np.asfortranarray(rng.standard_normal((129, 128, 3)))
    g = pq.Model(cfg)
    psi = g.pv_inversion(zeta)
    om = O.Model(O.cfg_from(cfg))
    zd = np.zeros((131, 130, 3), order="F")
    zd[1:-1, 1:-1, :] = zeta
    ref = om.pv_inversion(zd)[1:-1, 1:-1, :]
    assert rel_l2(psi, ref) <= TOL_STEP, rel_l2(psi, ref)


@pytest.mark.parametrize("ii,jj,layers", [(65, 64, 3), (129, 96, 2), (33, 40, 1)])
def test_channel_steps_match_oracle(ii, jj, layers):
    g, o = start(channel(ii, jj, layers), seed=53)
    for n in (1, 1, 2, 3):   # eager steps, one-step and two-step graphs
        g.step(n)
        o.step(n)
        compare(g, o, TOL_STEP * 10)
    ii_, jj_ = g.cfg.ii, g.cfg.jj
    assert rel_l2(owned("rel", g.get("rel"), ii_, jj_), owned("rel", o.get("rel"), ii_, jj_)) <= TOL_STEP * 10


def test_channel_hundred_steps_energy_cfl():
    cfg = channel(129, 128, 3)
    g, o = start(cfg, seed=54)
    g.step(100)
    o.step(100)
    compare(g, o, TOL_100)
    ek_g, ep_g = g.energy()
    ek_o, ep_o = o.energy()
    assert rel_l2(ek_g, ek_o) <= TOL_100
    assert abs(ep_g - ep_o) <= TOL_100 * abs(ep_o)
    assert abs(g.cfl() - o.cfl()) <= TOL_100 * o.cfl()
    assert abs(g.scalars()["model_time"] - o.scalars()["model_time"]) <= 1e-12 * o.scalars()["model_time"]


def test_channel_adaptive_dt_matches_oracle():
    cfg = channel(65, 64, 3, adapt_dt=1, target_cfl=0.1, max_dt=86400.0)
    g, o = start(cfg, seed=55)
    g.step(20)
    o.step(20)
    compare(g, o, 1e-10)
    sg, so = g.scalars(), o.scalars()
    for k in ("dt", "tweight_a", "tweight_u"):
        assert abs(sg[k] - so[k]) <= 1e-10 * abs(so[k]), (k, sg[k], so[k])


def test_channel_mixed_precision():
    cfg = channel(129, 128, 3, precision=pq.PREC_MIXED)
    g, o = start(cfg, seed=56)
    g.step(50)
    o.step(50)
    ii, jj = cfg.ii, cfg.jj
    assert rel_l2(owned("psi", g.get("psi"), ii, jj), owned("psi", o.get("psi"), ii, jj)) <= 1e-6


def start_lf(cfg, seed):
    ic = [pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed + k, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
          for k in (0, 1000)]
    ic = np.asfortranarray(np.stack(ic, axis=3))
    g = pq.Model(cfg)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return g, o


LF = ["psi", "zeta", "rel", "zeta_old", "psi2", "zeta2", "rel2", "zeta_old2"]


@pytest.mark.parametrize("ii,jj,layers", [(65, 64, 3), (33, 40, 1)])
def test_channel_leapfrog_matches_oracle(ii, jj, layers):
    """The leapfrog channel: centred step and filter with rows wrapped, the
    momentum-corrected inversion, rel and the wall PV of each level."""
    g, o = start_lf(channel(ii, jj, layers, scheme=pq.SCHEME_LEAPFROG), seed=57)
    compare(g, o, TOL_STEP, LF)
    for n in (1, 2, 3):
        g.step(n)
        o.step(n)
        compare(g, o, TOL_STEP * 10, LF)
    g.step(40)
    o.step(40)
    compare(g, o, TOL_100, LF)
    assert abs(g.scalars()["model_time"] - o.scalars()["model_time"]) <= 1e-12 * o.scalars()["model_time"]


def test_channel_leapfrog_pickup_and_average(tmp_path):
    """A leapfrog channel checkpoint (both levels) picks up with rel from psi
    over the periodic rows; the time average and covariances follow."""
    cfg = channel(65, 64, 3, scheme=pq.SCHEME_LEAPFROG)
    g, o = start_lf(cfg, seed=58)
    g.step(4)
    o.step(4)
    s = str(tmp_path / "lfc_s.d")
    g.write_checkpoint(s, None, t_scale=cfg.t_scale)
    ck = O.read_checkpoint(s, None, 65, 64, 3, leapfrog=True)
    g2 = pq.Model(cfg)
    g2.read_checkpoint(s)
    o2 = O.Model(O.cfg_from(cfg))
    o2.pickup(ck)
    compare(g2, o2, 1e-13, LF)
    g2.average(2, 0.0)
    o2.average(2, 0.0)
    g2.step(5)
    o2.step(5)
    compare(g2, o2, TOL_STEP * 10, LF)
    a_g, t_g = g2.get_average()
    a_o, t_o = o2.get_average()
    assert abs(t_g - t_o) <= 1e-12 * t_o and rel_l2(a_g, a_o) <= 1e-12
    worst = {n: rel_l2(g2.get_quad(q), o2.get_quad(q)) for q, n in enumerate(g2.QUAD)}
    assert max(worst.values()) <= 1e-11, worst
