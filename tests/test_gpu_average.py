"""Time-averaged streamfunction (psi_av, qg3.F90:672-680, 725, 886-899) on
the device against the oracle: the sum accumulated inside the fused CABARET
kernel (tile and warp-sweep forms) and by the leapfrog sub-step, the
threshold on model time, diagnostic_time, and the _s_av file."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def double_gyre(ii, layers=3, dt=1800.0, **kw):
    H = {2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    return pq.Config.from_physical(p)


def start(cfg, seed):
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    if cfg.desc.scheme == pq.SCHEME_LEAPFROG:
        ic2 = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed + 1000, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
        ic = np.asfortranarray(np.stack([ic, ic2], axis=3))
    g = pq.Model(cfg)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return g, o


@pytest.mark.parametrize("kernel,adapt,prec", [(0, 0, pq.PREC_FP64), (1, 0, pq.PREC_FP64), (0, 1, pq.PREC_FP64),
                                               (0, 0, pq.PREC_MIXED)])
def test_cabaret_average_matches_oracle(kernel, adapt, prec):
    kw = dict(adapt_dt=1, target_cfl=0.1, max_dt=86400.0) if adapt else {}
    cfg = double_gyre(129, 3, precision=prec, **kw)
    g, o = start(cfg, seed=41)
    g.set_tuning(cab_kernel=kernel, cab_band=16, dst_group=0)
    g.step(2)
    o.step(2)
    dt = cfg.desc.dt
    thr = o.scalars()["model_time"] + 2.6 * dt   # steps 1-2 after this point are not averaged
    g.average(True, thr)
    o.average(True, thr)
    for n in (1, 2, 3, 5):   # eager steps, one-step and two-step graphs
        g.step(n)
        o.step(n)
    a_g, t_g = g.get_average()
    a_o, t_o = o.get_average()
    assert t_o > 0 and abs(t_g - t_o) <= 1e-12 * t_o, (t_g, t_o)
    tol = 1e-12 if prec == pq.PREC_FP64 else 1e-6
    assert rel_l2(a_g, a_o) <= tol, rel_l2(a_g, a_o)


def test_average_off_then_on_and_file(tmp_path):
    cfg = double_gyre(65, 2)
    g, o = start(cfg, seed=42)
    g.step(3)
    o.step(3)
    with pytest.raises(pq.PQError) as e:
        g.get_average()
    assert e.value.code == pq.PQ_ERR_STATE
    g.average(True, 0.0)
    o.average(True, 0.0)
    g.step(4)
    o.step(4)
    a_g, t_g = g.get_average()
    path = str(tmp_path / "qg2_65_s_av.d")
    g.write_average(path, t_scale=cfg.t_scale, start_time_day=2.0)
    recs = O._records(path)
    assert len(recs) == 2 + 2
    want_day = (o.scalars()["model_time"] - 0.5 * cfg.desc.dt) * cfg.t_scale / 86400.0
    assert abs(recs[0][0] - want_day) <= 1e-13 * want_day
    assert abs(recs[1][0] - (2.0 + want_day)) <= 1e-13 * recs[1][0]
    a_o, _ = o.get_average()
    for l in range(2):
        assert rel_l2(recs[2 + l].reshape((65, 65), order="F"), a_o[:, :, l]) <= 1e-12
    # Stopping the average leaves the run untouched.
    g.average(False)
    g.step(2)
    o.step(2)
    assert rel_l2(g.get("psi"), o.get("psi")) <= 1e-11


def test_leapfrog_average_matches_oracle():
    cfg = double_gyre(65, 2, scheme=pq.SCHEME_LEAPFROG)
    g, o = start(cfg, seed=43)
    g.step(2)
    o.step(2)
    thr = o.scalars()["model_time"] + 1.5 * cfg.desc.dt
    g.average(True, thr)
    o.average(True, thr)
    for n in (1, 2, 3):
        g.step(n)
        o.step(n)
    assert g.last_launch_count() == 3 * 6    # the average adds one kernel per sub-step
    a_g, t_g = g.get_average()
    a_o, t_o = o.get_average()
    assert abs(t_g - t_o) <= 1e-12 * t_o
    assert rel_l2(a_g, a_o) <= 1e-12


@pytest.mark.parametrize("kernel,partial_slip,prec", [(0, True, pq.PREC_FP64), (1, False, pq.PREC_FP64),
                                                      (0, True, pq.PREC_MIXED)])
def test_quad_covariances_match_oracle(kernel, partial_slip, prec):
    """The 23 quad eddy covariances (qg3.F90:683-721) on the device against
    the oracle, with the model-time threshold passed mid-run."""
    cfg = double_gyre(129, 3, precision=prec, partial_slip=partial_slip)
    g, o = start(cfg, seed=44)
    g.set_tuning(cab_kernel=kernel, cab_band=16, dst_group=0)
    g.step(1)
    o.step(1)
    thr = o.scalars()["model_time"] + 1.7 * cfg.desc.dt
    g.average(2, thr)
    o.average(2, thr)
    for n in (1, 2, 3):
        g.step(n)
        o.step(n)
    assert g.last_launch_count() == 3 * 5    # the covariances add one kernel per step
    tol = 1e-11 if prec == pq.PREC_FP64 else 1e-5
    worst = {}
    for q, name in enumerate(g.QUAD):
        a, b = g.get_quad(q), o.get_quad(q)
        assert a.shape == b.shape, name
        worst[name] = rel_l2(a, b)
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst
    a_g, t_g = g.get_average()
    a_o, t_o = o.get_average()
    assert abs(t_g - t_o) <= 1e-12 * t_o


def test_quad_free_slip_walls_and_file(tmp_path):
    """Free slip leaves the wall velocities NaN (the reference's nan()), so
    the velocity products are NaN on those nodes on both sides; the
    _quad_av file holds the two times and 23 whole-array records."""
    cfg = double_gyre(65, 2, partial_slip=True, alpha=1.0e300)
    assert cfg.desc.bc_type == pq.BC_FREE_SLIP
    g, o = start(cfg, seed=45)
    g.average(2, 0.0)
    o.average(2, 0.0)
    g.step(3)
    o.step(3)
    for q in range(23):
        a, b = g.get_quad(q), o.get_quad(q)
        np.testing.assert_array_equal(np.isnan(a), np.isnan(b), err_msg=g.QUAD[q])
        m = ~np.isnan(b)
        assert rel_l2(a[m], b[m]) <= 1e-11, g.QUAD[q]
    assert np.isnan(g.get_quad(0)).any() and not np.isnan(g.get_quad(13)).any()
    path = str(tmp_path / "qg2_65_quad_av.d")
    g.write_quad(path, t_scale=cfg.t_scale)
    recs = O._records(path)
    assert len(recs) == 2 + 23
    assert [r.size for r in recs[2:]] == [65 * 65 * (1 if n in ("uu_i", "vv_i", "sc_ub", "sc_vb", "sc_bb_i") else 2)
                                          for n in g.QUAD]


def channel(ii, jj, layers=3, dt=1800.0, **kw):
    H = {2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, jj=jj, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = 1
    return cfg


@pytest.mark.parametrize("partial_slip,prec", [(True, pq.PREC_FP64), (False, pq.PREC_FP64),
                                               (True, pq.PREC_MIXED)])
def test_channel_average_and_quad_match_oracle(partial_slip, prec):
    """A channel's psi_av (accumulated in its rel kernel) and quad
    covariances (v central across the periodic rows, no j walls)."""
    cfg = channel(129, 96, 3, precision=prec, partial_slip=partial_slip)
    g, o = start(cfg, seed=46)
    g.step(1)
    o.step(1)
    thr = o.scalars()["model_time"] + 1.7 * cfg.desc.dt
    g.average(2, thr)
    o.average(2, thr)
    for n in (1, 2, 3):
        g.step(n)
        o.step(n)
    assert g.last_launch_count() == 3 * 8    # seven channel kernels and the covariances
    tol = 1e-11 if prec == pq.PREC_FP64 else 1e-5
    a_g, t_g = g.get_average()
    a_o, t_o = o.get_average()
    assert t_o > 0 and abs(t_g - t_o) <= 1e-12 * t_o
    assert rel_l2(a_g, a_o) <= (1e-12 if prec == pq.PREC_FP64 else 1e-6), rel_l2(a_g, a_o)
    worst = {name: rel_l2(g.get_quad(q), o.get_quad(q)) for q, name in enumerate(g.QUAD)}
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst


def test_leapfrog_quad_matches_oracle(tmp_path):
    """The leapfrog sub-step's covariances: one kernel after its rel kernel
    on the level just inverted."""
    cfg = double_gyre(129, 3, scheme=pq.SCHEME_LEAPFROG)
    g, o = start(cfg, seed=47)
    g.step(2)
    o.step(2)
    thr = o.scalars()["model_time"] + 1.5 * cfg.desc.dt
    g.average(2, thr)
    o.average(2, thr)
    for n in (1, 2, 3):
        g.step(n)
        o.step(n)
    assert g.last_launch_count() == 3 * 7    # average + covariances per sub-step
    worst = {name: rel_l2(g.get_quad(q), o.get_quad(q)) for q, name in enumerate(g.QUAD)}
    bad = {k: v for k, v in worst.items() if not v <= 1e-11}
    assert not bad, worst
    a_g, t_g = g.get_average()
    a_o, t_o = o.get_average()
    assert abs(t_g - t_o) <= 1e-12 * t_o and rel_l2(a_g, a_o) <= 1e-12
    path = str(tmp_path / "qg3_129_quad_av.d")
    g.write_quad(path, t_scale=cfg.t_scale)
    recs = O._records(path)
    want_day = o.scalars()["model_time"] * cfg.t_scale / 86400.0
    assert abs(recs[0][0] - want_day) <= 1e-13 * want_day
