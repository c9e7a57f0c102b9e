"""Checkpoint dump and pickup through the C ABI against the oracle.

The device writes the reference's _s.d / _s_supp.d records: the state the
reference holds at its data output, inside a step before the corrector.
The files parse with the oracle's reader and match the oracle stopped at
that point.  A pickup from those files on the device and in the oracle then
runs on in step, and as the uninterrupted run.  FP64 bar: relative L2
<= 1e-12 per field."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12
CAB = ["psi", "zeta", "ui", "uj", "zeta_fi", "zeta_fj", "res", "res_beta"]
AFTER = ["psi", "zeta", "zeta_old", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res", "res_beta"]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def double_gyre(ii, layers=3, dt=1800.0, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75)}[layers]
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


def compare(g, o, names, tol):
    worst = {n: rel_l2(g.get(n), o.get(n)) for n in names}
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst


def saved_view(name, a, ii, jj):
    """The part of a reference-layout array that the checkpoint holds."""
    if name in ("psi", "zeta", "psi2", "zeta2"):
        return a[1:-1, 1:-1]
    if name in ("ui", "zeta_fi"):
        return a[2:ii + 1, 2:jj]
    if name in ("uj", "zeta_fj"):
        return a[2:ii, 2:jj + 1]
    return a


@pytest.mark.parametrize("ii,layers", [(65, 1), (129, 3)])
def test_cabaret_dump_matches_oracle_state(tmp_path, ii, layers):
    cfg = double_gyre(ii, layers)
    g, o = start(cfg, seed=31)
    g.step(7)
    o.step(6)
    o.step_to_dump()
    s, supp = str(tmp_path / f"qg{layers}_{ii}_s.d"), str(tmp_path / f"qg{layers}_{ii}_s_supp.d")
    g.write_checkpoint(s, supp, t_scale=cfg.t_scale, start_time_day=10.0)
    ck = O.read_checkpoint(s, supp, ii, ii, layers)
    so = o.scalars()
    want_day = so["model_time"] * cfg.t_scale / 86400.0
    assert abs(ck["model_time_day"] - want_day) <= 1e-14 * want_day
    assert abs(ck["total_time_day"] - (10.0 + want_day)) <= 1e-14 * ck["total_time_day"]
    assert ck["dt"] == so["dt"]
    for n in CAB:
        a = saved_view(n, ck[n], ii, ii)
        b = saved_view(n, o.get(n), ii, ii)
        assert rel_l2(a, b) <= TOL, (n, rel_l2(a, b))


@pytest.mark.parametrize("adapt", [0, 1])
def test_cabaret_pickup_matches_oracle(tmp_path, adapt):
    kw = dict(adapt_dt=1, target_cfl=0.1, max_dt=86400.0) if adapt else {}
    cfg = double_gyre(129, 3, **kw)
    g, o = start(cfg, seed=32)
    g.step(9)
    o.step(8)
    o.step_to_dump()
    s, supp = str(tmp_path / "qg3_129_s.d"), str(tmp_path / "qg3_129_s_supp.d")
    g.write_checkpoint(s, supp, t_scale=cfg.t_scale, start_time_day=3.5)
    ck = O.read_checkpoint(s, supp, 129, 129, 3)
    g2 = pq.Model(cfg)
    total = g2.read_checkpoint(s, supp)
    assert total == ck["total_time_day"]
    o2 = O.Model(O.cfg_from(cfg))
    o2.pickup(ck)
    # Both pick up from the same file: the set-up arithmetic is the same.
    compare(g2, o2, AFTER, 1e-15)
    assert g2.scalars()["model_time"] == o2.scalars()["model_time"]
    # The resumed runs continue the uninterrupted ones.
    o.finish_step()
    compare(g2, o, AFTER, TOL)
    compare(g, o, AFTER, TOL)
    for n in (1, 2, 5):
        for m in (g, g2, o, o2):
            m.step(n)
        compare(g2, o2, AFTER, TOL * 10)
        compare(g2, o, AFTER, TOL * 10)
        assert max(rel_l2(g2.get(f), g.get(f)) for f in ("psi", "zeta")) <= TOL
    sg, so = g2.scalars(), o2.scalars()
    for k in ("dt", "tweight_a", "tweight_u", "model_time"):
        assert abs(sg[k] - so[k]) <= 1e-12 * abs(so[k]), (k, sg[k], so[k])


def test_pickup_into_a_context_that_has_run(tmp_path):
    """A pickup replaces every piece of a running context's state."""
    cfg = double_gyre(65, 3)
    g, o = start(cfg, seed=33)
    g.step(4)
    o.step(4)
    s, supp = str(tmp_path / "x_s.d"), str(tmp_path / "x_s_supp.d")
    g.write_checkpoint(s, supp)
    g.step(3)   # move on, then go back to the dump
    g.read_checkpoint(s, supp)
    o2 = O.Model(O.cfg_from(cfg))
    o2.pickup(O.read_checkpoint(s, supp, 65, 65, 3))
    g.step(4)
    o2.step(4)
    compare(g, o2, AFTER, TOL * 10)


def test_leapfrog_checkpoint_round_trip(tmp_path):
    cfg = double_gyre(65, 2, scheme=pq.SCHEME_LEAPFROG)
    g, o = start(cfg, seed=34)
    g.step(3)
    with pytest.raises(pq.PQError) as e:   # mid-pair: the reference never dumps here
        g.write_checkpoint(str(tmp_path / "odd_s.d"))
    assert e.value.code == pq.PQ_ERR_STATE
    g.step(1)
    o.step(4)
    s = str(tmp_path / "qg2_65_s.d")
    g.write_checkpoint(s, None, t_scale=cfg.t_scale)
    ck = O.read_checkpoint(s, None, 65, 65, 2, leapfrog=True)
    for n in ("psi", "zeta", "psi2", "zeta2"):
        assert rel_l2(ck[n][1:-1, 1:-1], o.get(n)[1:-1, 1:-1]) <= TOL, n
    g2 = pq.Model(cfg)
    g2.read_checkpoint(s)
    o2 = O.Model(O.cfg_from(cfg))
    o2.pickup(ck)
    levels = ["psi", "zeta", "rel", "zeta_old", "psi2", "zeta2", "rel2", "zeta_old2"]
    compare(g2, o2, levels, 1e-15)
    for n in (1, 2, 3):
        g2.step(n)
        o2.step(n)
        compare(g2, o2, levels, TOL * 10)
    assert abs(g2.scalars()["model_time"] - o2.scalars()["model_time"]) <= 1e-12 * o2.scalars()["model_time"]


def test_mixed_precision_pickup(tmp_path):
    """The mixed form dumps its FP32 state widened to REAL(8) and picks up
    by rounding it back; the run then tracks the FP64 oracle within the
    mixed form's 1e-6 bar on psi."""
    cfg = double_gyre(129, 3, precision=pq.PREC_MIXED)
    g, _ = start(cfg, seed=35)
    g.step(6)
    s, supp = str(tmp_path / "m_s.d"), str(tmp_path / "m_s_supp.d")
    g.write_checkpoint(s, supp)
    ck = O.read_checkpoint(s, supp, 129, 129, 3)
    g2 = pq.Model(cfg)
    g2.read_checkpoint(s, supp)
    o2 = O.Model(O.cfg_from(cfg))
    o2.pickup(ck)
    g2.step(10)
    o2.step(10)
    assert rel_l2(g2.get("psi"), o2.get("psi")) <= 1e-6


def test_checkpoint_errors(tmp_path):
    cfg = double_gyre(33, 2)
    g, o = start(cfg, seed=36)
    g.step(2)
    s, supp = str(tmp_path / "e_s.d"), str(tmp_path / "e_s_supp.d")
    g.write_checkpoint(s, supp)
    g2 = pq.Model(cfg)
    with pytest.raises(pq.PQError) as e:
        g2.read_checkpoint(s, None)          # CABARET needs the _s_supp file
    assert e.value.code == pq.PQ_ERR_ARG
    with pytest.raises(pq.PQError) as e:
        g2.read_checkpoint(str(tmp_path / "missing_s.d"), supp)
    assert e.value.code == pq.PQ_ERR_ARG and "Failed to open" in str(e.value)
    # A _s file of another dump: the times disagree, as the reference aborts.
    fields = O.read_checkpoint(s, supp, 33, 33, 2)
    other = str(tmp_path / "o_s.d")
    O.write_checkpoint(other, None, fields, fields["model_time_day"] + 1.0, fields["total_time_day"] + 1.0)
    with pytest.raises(pq.PQError) as e:
        g2.read_checkpoint(other, supp)
    assert e.value.code == pq.PQ_ERR_ARG and "do not match" in str(e.value)
    # A file of another grid size: the first field record has the wrong length.
    small = double_gyre(17, 2)
    gs, _ = start(small, seed=37)
    s17, supp17 = str(tmp_path / "s17_s.d"), str(tmp_path / "s17_s_supp.d")
    gs.write_checkpoint(s17, supp17)
    with pytest.raises(pq.PQError) as e:
        g2.read_checkpoint(s17, supp17)
    assert e.value.code == pq.PQ_ERR_ARG and "unexpected record" in str(e.value)
    # The context is still usable after the refusals.
    g2.read_checkpoint(s, supp)
    g2.step(1)


def channel(ii, jj, layers=3, dt=1800.0, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, jj=jj, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = 1
    return cfg


def channel_saved(name, a, ii, jj):
    """The part of a channel's reference-layout array that its checkpoint
    holds: rows 2..jj+1 and faces 2..jj+2 (fa_j_min = 1, fa_j_max = jj+2)."""
    if name in ("psi", "zeta"):
        return a[1:-1, 1:-1]
    if name in ("ui", "zeta_fi"):
        return a[2:ii + 1, 1:jj + 1]
    if name in ("uj", "zeta_fj"):
        return a[2:ii, 1:jj + 2]
    return a


def channel_owned(name, a, ii, jj):
    """The part of a channel's reference-layout array the device stores (the
    halo rows are copies of it)."""
    if name in ("ui", "uimo", "zeta_fi", "uj", "ujmo", "zeta_fj"):
        return a[1:ii + 1, 1:jj + 1]
    if name in ("res", "res_beta"):
        return a
    return a[1:-1, 1:-1]


def compare_channel(g, o, names, tol):
    ii, jj = g.cfg.ii, g.cfg.jj
    worst = {n: rel_l2(channel_owned(n, g.get(n), ii, jj), channel_owned(n, o.get(n), ii, jj)) for n in names}
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst


@pytest.mark.parametrize("ii,jj,layers", [(65, 64, 3), (33, 40, 1)])
def test_channel_dump_matches_oracle_state(tmp_path, ii, jj, layers):
    """The channel's _s / _s_supp files: face jj+2 of the j faces is face 2
    of the next period, written from the device's face 2."""
    cfg = channel(ii, jj, layers)
    g, o = start(cfg, seed=35)
    g.step(7)
    o.step(6)
    o.step_to_dump()
    s, supp = str(tmp_path / "ch_s.d"), str(tmp_path / "ch_s_supp.d")
    g.write_checkpoint(s, supp, t_scale=cfg.t_scale, start_time_day=1.0)
    ck = O.read_checkpoint(s, supp, ii, jj, layers, periodic_j=True)
    so = o.scalars()
    want_day = so["model_time"] * cfg.t_scale / 86400.0
    assert abs(ck["model_time_day"] - want_day) <= 1e-14 * want_day
    assert ck["dt"] == so["dt"]
    for n in CAB:
        a = channel_saved(n, ck[n], ii, jj)
        b = channel_saved(n, o.get(n), ii, jj)
        assert rel_l2(a, b) <= TOL, (n, rel_l2(a, b))


@pytest.mark.parametrize("adapt", [0, 1])
def test_channel_pickup_matches_oracle(tmp_path, adapt):
    kw = dict(adapt_dt=1, target_cfl=0.1, max_dt=86400.0) if adapt else {}
    cfg = channel(129, 96, 3, **kw)
    g, o = start(cfg, seed=36)
    g.step(9)
    o.step(8)
    o.step_to_dump()
    s, supp = str(tmp_path / "ch3_s.d"), str(tmp_path / "ch3_s_supp.d")
    g.write_checkpoint(s, supp, t_scale=cfg.t_scale, start_time_day=2.0)
    ck = O.read_checkpoint(s, supp, 129, 96, 3, periodic_j=True)
    g2 = pq.Model(cfg)
    total = g2.read_checkpoint(s, supp)
    assert total == ck["total_time_day"]
    o2 = O.Model(O.cfg_from(cfg))
    o2.pickup(ck)
    compare_channel(g2, o2, AFTER, 1e-15)
    assert g2.scalars()["model_time"] == o2.scalars()["model_time"]
    o.finish_step()
    compare_channel(g2, o, AFTER, TOL)
    compare_channel(g, o, AFTER, TOL)
    for n in (1, 2, 5):
        for m in (g, g2, o, o2):
            m.step(n)
        compare_channel(g2, o2, AFTER, TOL * 10)
        compare_channel(g2, o, AFTER, TOL * 10)
        assert max(rel_l2(g2.get(f), g.get(f)) for f in ("psi", "zeta")) <= TOL
    sg, so = g2.scalars(), o2.scalars()
    for k in ("dt", "tweight_a", "tweight_u", "model_time"):
        assert abs(sg[k] - so[k]) <= 1e-12 * abs(so[k]), (k, sg[k], so[k])
