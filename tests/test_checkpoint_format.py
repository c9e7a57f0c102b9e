"""Checkpoint files and the pickup, on the CPU: the oracle's record format
(qg3p_io.F90:574-760) and its START_PICKUP (qg3.F90:314-363, :448-497)
against a separate numpy statement of the same steps."""
import os

import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O


def double_gyre(ii, layers=2, dt=1800.0, **kw):
    H = {2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    return pq.Config.from_physical(p)


def channel(ii, jj, layers=3, dt=1800.0, **kw):
    """A channel (periodic in j) of the double-gyre physics."""
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, jj=jj, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = 1
    return cfg


def run_oracle(cfg, steps, seed):
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    if O.cfg_from(cfg).get("scheme", 0) == 1:
        ic2 = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed + 1000, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
        ic = np.asfortranarray(np.stack([ic, ic2], axis=3))
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    o.step(steps)
    return o


CAB = ["psi", "zeta", "ui", "uj", "zeta_fi", "zeta_fj", "res", "res_beta"]


def test_record_framing(tmp_path):
    """Each record: int32 byte count, REAL(8) data, the same count."""
    s = str(tmp_path / "qg2_17_s.d")
    supp = str(tmp_path / "qg2_17_s_supp.d")
    cfg = double_gyre(17)
    o = run_oracle(cfg, 3, seed=1)
    fields = {n: o.get(n) for n in CAB}
    O.write_checkpoint(s, supp, fields, 1.25, 11.25, dt=0.5)
    ii = jj = 17
    L = 2
    raw = open(s, "rb").read()
    assert len(raw) == 2 * (8 + 8) + 2 * L * (8 + 8 * ii * jj)
    assert np.frombuffer(raw, "<i4", 1, 0)[0] == 8
    assert np.frombuffer(raw, "<f8", 1, 4)[0] == 1.25
    assert np.frombuffer(raw, "<i4", 1, 12)[0] == 8
    assert np.frombuffer(raw, "<i4", 1, 32)[0] == 8 * ii * jj
    nfi = (ii - 1) * (jj - 2)
    nfj = (ii - 2) * (jj - 1)
    assert os.path.getsize(supp) == 3 * 16 + L * (6 * 8 + 8 * (2 * nfi + 2 * nfj + 2 * ii * jj))
    back = O.read_checkpoint(s, supp, ii, jj, L)
    assert back["model_time_day"] == 1.25 and back["total_time_day"] == 11.25 and back["dt"] == 0.5
    # The saved ranges come back exactly; the unsaved boundary faces as zero.
    for n in CAB:
        a, b = back[n], fields[n]
        if n in ("psi", "zeta"):
            np.testing.assert_array_equal(a[1:-1, 1:-1], b[1:-1, 1:-1])
        elif n in ("ui", "zeta_fi"):
            np.testing.assert_array_equal(a[2:ii + 1, 2:jj], b[2:ii + 1, 2:jj])
            assert not a[:2].any() and not a[ii + 1:].any()
        elif n in ("uj", "zeta_fj"):
            np.testing.assert_array_equal(a[2:ii, 2:jj + 1], b[2:ii, 2:jj + 1])
        else:
            np.testing.assert_array_equal(a, b)


def test_mismatched_times_are_rejected(tmp_path):
    s, supp = str(tmp_path / "a_s.d"), str(tmp_path / "a_s_supp.d")
    cfg = double_gyre(9)
    o = run_oracle(cfg, 1, seed=2)
    fields = {n: o.get(n) for n in CAB}
    O.write_checkpoint(s, supp, fields, 1.0, 2.0, dt=0.5)
    s2 = str(tmp_path / "b_s.d")
    O.write_checkpoint(s2, None, fields, 1.0, 3.0)
    with pytest.raises(ValueError, match="do not match"):
        O.read_checkpoint(s2, supp, 9, 9, 2)


def numpy_cabaret_pickup(ck, dt):
    """qg3.F90:316-340 in numpy, 0-based reference-layout indexes."""
    psi, zeta = ck["psi"], ck["zeta"].copy(order="F")
    ui, uj, zfi, zfj = ck["ui"], ck["uj"], ck["zeta_fi"], ck["zeta_fj"]
    ii, jj = psi.shape[0] - 2, psi.shape[1] - 2
    pe = np.zeros_like(psi)
    # psi_edge at 1-based (i, j), i in [3, ii+1], j in [3, jj+1].
    pe[2:ii + 1, 2:jj + 1] = 0.25 * (((psi[2:ii + 1, 2:jj + 1] + psi[2:ii + 1, 1:jj]) + psi[1:ii, 2:jj + 1])
                                     + psi[1:ii, 1:jj])
    uimo = np.zeros_like(ui)
    uimo[2:ii + 1, 2:jj] = -pe[2:ii + 1, 3:jj + 1] + pe[2:ii + 1, 2:jj]
    ujmo = np.zeros_like(uj)
    ujmo[2:ii, 2:jj + 1] = pe[3:ii + 1, 2:jj + 1] - pe[2:ii, 2:jj + 1]
    fli = ui * zfi
    flj = uj * zfj
    res = ck["res"].copy(order="F")
    # corrector on nodes 1-based i, j in [3, ii] x [3, jj]
    r = -(((fli[3:ii + 1, 2:jj] - fli[2:ii, 2:jj]) + flj[2:ii, 3:jj + 1]) - flj[2:ii, 2:jj])
    res[1:ii - 1, 1:jj - 1] = r
    zeta[2:ii, 2:jj] = zeta[2:ii, 2:jj] + 0.5 * dt * r
    return dict(uimo=uimo, ujmo=ujmo, res=res, zeta=zeta, zeta_old=zeta, flux_i=fli, flux_j=flj)


@pytest.mark.parametrize("adapt", [0, 1])
def test_cabaret_pickup_matches_numpy(tmp_path, adapt):
    s, supp = str(tmp_path / "c_s.d"), str(tmp_path / "c_s_supp.d")
    kw = dict(adapt_dt=1, target_cfl=0.1, max_dt=86400.0) if adapt else {}
    cfg = double_gyre(17, 3, **kw)
    o = run_oracle(cfg, 4, seed=3)
    o.step_to_dump()     # the reference writes its checkpoint here
    fields = o.dump_fields()
    dt = o.scalars()["dt"]
    O.write_checkpoint(s, supp, fields, 0.1, 0.1, dt=dt)
    ck = O.read_checkpoint(s, supp, 17, 17, 3)
    p = O.Model(O.cfg_from(cfg))
    p.pickup(ck)
    want = numpy_cabaret_pickup(ck, dt)
    ii = jj = 17
    for n in ("uimo", "ujmo", "res", "zeta", "zeta_old"):
        got = p.get(n)
        if n == "uimo":
            got, w = got[2:ii + 1, 2:jj], want[n][2:ii + 1, 2:jj]
        elif n == "ujmo":
            got, w = got[2:ii, 2:jj + 1], want[n][2:ii, 2:jj + 1]
        else:
            w = want[n]
        np.testing.assert_array_equal(got, w, err_msg=n)
    fl = p.get("flux_i")
    np.testing.assert_array_equal(fl[2:ii + 1, 2:jj], want["flux_i"][2:ii + 1, 2:jj])
    sc = p.scalars()
    assert sc["dt"] == dt and sc["model_time"] == dt / 2 and sc["tweight_a"] == 0.5 and sc["tweight_u"] == 0.5
    # The pickup finishes the interrupted step: from here the resumed run is
    # the uninterrupted one, bit for bit (model_time restarts at dt / 2).
    o.finish_step()
    for n in ("psi", "zeta", "zeta_old", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res", "res_beta"):
        np.testing.assert_array_equal(p.get(n), o.get(n), err_msg=n)
    p.step(3)
    o.step(3)
    for n in ("psi", "zeta", "ui", "uj", "zeta_fi", "zeta_fj", "res", "res_beta"):
        np.testing.assert_array_equal(p.get(n), o.get(n), err_msg=n)
    assert p.scalars()["dt"] == o.scalars()["dt"]


@pytest.mark.parametrize("adapt", [0, 1])
def test_channel_pickup_resumes_bit_for_bit(tmp_path, adapt):
    """A channel's checkpoint (faces fa_j_min+1 .. fa_j_max with fa_j_min = 1,
    fa_j_max = jj + 2, qg3.F90:864-875) and its pickup with the periodic halo
    updates (qg3.F90:324-339): the resumed oracle is the uninterrupted one."""
    s, supp = str(tmp_path / "ch_s.d"), str(tmp_path / "ch_s_supp.d")
    kw = dict(adapt_dt=1, target_cfl=0.1, max_dt=86400.0) if adapt else {}
    cfg = channel(17, 20, 3, **kw)
    ii, jj = 17, 20
    o = run_oracle(cfg, 4, seed=8)
    o.step_to_dump()
    fields = o.dump_fields()
    O.write_checkpoint(s, supp, fields, 0.1, 0.1, dt=o.scalars()["dt"], periodic_j=True)
    recs = O._records(supp)
    assert [r.size for r in recs[3:3 + 4 * 3:3]] == [(ii - 1) * jj, (ii - 2) * (jj + 1), (ii - 1) * jj, (ii - 2) * (jj + 1)]
    ck = O.read_checkpoint(s, supp, ii, jj, 3, periodic_j=True)
    for n in ("ui", "zeta_fi"):
        np.testing.assert_array_equal(ck[n][2:ii + 1, 1:jj + 1], fields[n][2:ii + 1, 1:jj + 1])
    for n in ("uj", "zeta_fj"):
        np.testing.assert_array_equal(ck[n][2:ii, 1:jj + 2], fields[n][2:ii, 1:jj + 2])
    p = O.Model(O.cfg_from(cfg))
    p.pickup(ck)
    o.finish_step()
    for n in ("psi", "zeta", "zeta_old", "uimo", "ujmo", "zeta_fj", "res", "res_beta"):
        np.testing.assert_array_equal(p.get(n), o.get(n), err_msg=n)
    p.step(3)
    o.step(3)
    for n in ("psi", "zeta", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res", "res_beta"):
        np.testing.assert_array_equal(p.get(n), o.get(n), err_msg=n)
    assert p.scalars()["dt"] == o.scalars()["dt"]


@pytest.mark.parametrize("bc", [pq.BC_PARTIAL_SLIP, pq.BC_NO_SLIP, pq.BC_FREE_SLIP])
def test_leapfrog_pickup_rel_from_psi(tmp_path, bc):
    """rel_from_psi (qg3p_aux.F90:579-603) + apply_rel_bc on both levels."""
    s = str(tmp_path / "lf_s.d")
    cfg = double_gyre(17, 2, scheme=pq.SCHEME_LEAPFROG, partial_slip=int(bc == pq.BC_PARTIAL_SLIP))
    oc = O.cfg_from(cfg)
    oc["bc_type"] = bc
    ic = pq.make_ic(17, 17, 2, seed=4, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    o = O.Model(oc)
    o.init(np.asfortranarray(np.stack([ic, 0.5 * ic], axis=3)))
    o.step(3)
    fields = {n: o.get(n) for n in ("psi", "zeta", "psi2", "zeta2")}
    O.write_checkpoint(s, None, fields, 0.2, 0.2, leapfrog=True)
    ck = O.read_checkpoint(s, None, 17, 17, 2, leapfrog=True)
    for n in fields:
        np.testing.assert_array_equal(ck[n][1:-1, 1:-1], fields[n][1:-1, 1:-1])
    p = O.Model(oc)
    p.pickup(ck)
    alpha = oc.get("alpha", 0.0)
    for lv, suf in ((0, ""), (1, "2")):
        psi = ck["psi" + suf]
        rel = np.zeros_like(psi)
        rel[2:-2, 2:-2] = ((((-4.0 * psi[2:-2, 2:-2] + psi[1:-3, 2:-2]) + psi[2:-2, 3:-1]) + psi[3:-1, 2:-2])
                           + psi[2:-2, 1:-3])

        def edge(p0, p1, p2):
            if bc == pq.BC_PARTIAL_SLIP:
                return alpha / (alpha + 3.0) * ((-3.5 * p0 + 4.0 * p1) - 0.5 * p2)
            if bc == pq.BC_NO_SLIP:
                return 2.0 * (p1 - p0)
            return 0.0 * p0

        rel[1, 1:-1] = edge(psi[1, 1:-1], psi[2, 1:-1], psi[3, 1:-1])
        rel[-2, 1:-1] = edge(psi[-2, 1:-1], psi[-3, 1:-1], psi[-4, 1:-1])
        rel[1:-1, 1] = edge(psi[1:-1, 1], psi[1:-1, 2], psi[1:-1, 3])
        rel[1:-1, -2] = edge(psi[1:-1, -2], psi[1:-1, -3], psi[1:-1, -4])
        np.testing.assert_allclose(p.get("rel" + suf), rel, rtol=0, atol=1e-15 * np.abs(rel).max())
        np.testing.assert_array_equal(p.get("zeta_old" + suf), ck["zeta" + suf])
    assert p.scalars()["model_time"] == 0.0


@pytest.mark.parametrize("scheme,periodic", [(pq.SCHEME_CABARET, False), (pq.SCHEME_LEAPFROG, False),
                                             (pq.SCHEME_CABARET, True)])
def test_oracle_time_average(scheme, periodic):
    """psi_av (qg3.F90:672-680, 725): the sum of dt * psi over the steps whose
    model time passed the threshold, restated step by step in numpy."""
    cfg = channel(17, 20, 2) if periodic else double_gyre(17, 2, scheme=scheme)
    o = run_oracle(cfg, 0, seed=5)
    dt = O.cfg_from(cfg)["dt"]
    t0 = o.scalars()["model_time"]
    thr = t0 + 3.2 * dt          # the first steps are not averaged
    o.average(True, thr)
    want = np.zeros((cfg.ii, cfg.jj, 2), order="F")
    dtime = 0.0
    for k in range(7):
        if scheme == pq.SCHEME_CABARET:
            o.step_to_dump()
            psi, t = o.get("psi"), o.scalars()["model_time"]
            o.finish_step()
        else:
            o.step(1)
            t = o.scalars()["model_time"]
            psi = o.get("psi" if k % 2 == 0 else "psi2")   # sub-steps alternate levels 1, 2
        if t > thr:
            want += dt * psi[1:-1, 1:-1]
            dtime += dt
    got, t = o.get_average()
    assert t == dtime and dtime > 0 and dtime < 7 * dt
    np.testing.assert_allclose(got, want / dtime, rtol=1e-14, atol=0)


def numpy_quad_terms(psi, rel, zeta, cfg, periodic_j=False):
    """qg3.F90:683-721 in numpy on sdata (ii, jj, L): the 23 products.  A
    channel has no j walls: u is central on every row, v wraps in j."""
    oc = O.cfg_from(cfg)
    ii, jj, L = psi.shape
    bc, alpha = oc["bc_type"], oc["alpha"]
    s1, s2, h = np.array(oc["s1"]), np.array(oc["s2"]), np.array(oc["h"])
    u = np.zeros_like(psi)
    v = np.zeros_like(psi)
    wall = {pq.BC_PARTIAL_SLIP: None, pq.BC_NO_SLIP: 0.0, pq.BC_FREE_SLIP: np.nan}[bc]
    if periodic_j:
        u[1:-1, :] = 0.5 * (psi[2:, :] - psi[:-2, :])
        v[1:-1, :] = 0.5 * (np.roll(psi, -1, axis=1) - np.roll(psi, 1, axis=1))[1:-1, :]
        if wall is None:
            u[0, :], u[-1, :] = rel[0, :] / alpha, rel[-1, :] / alpha
        else:
            u[0, :] = u[-1, :] = wall
    else:
        u[1:-1, 1:-1] = 0.5 * (psi[2:, 1:-1] - psi[:-2, 1:-1])
        v[1:-1, 1:-1] = 0.5 * (psi[1:-1, 2:] - psi[1:-1, :-2])
        if wall is None:
            u[0, 1:-1], u[-1, 1:-1] = rel[0, 1:-1] / alpha, rel[-1, 1:-1] / alpha
            v[1:-1, 0], v[1:-1, -1] = rel[1:-1, 0] / alpha, rel[1:-1, -1] / alpha
        else:
            u[0, 1:-1] = u[-1, 1:-1] = wall
            v[1:-1, 0] = v[1:-1, -1] = wall
    t = np.zeros_like(psi)
    if L > 1:
        t[:, :, 0] = -s2[0] * (psi[:, :, 0] - psi[:, :, 1])
        t[:, :, -1] = -s1[L - 1] * (psi[:, :, -1] - psi[:, :, -2])
        for l in range(1, L - 1):
            t[:, :, l] = -s1[l] * (psi[:, :, l] - psi[:, :, l - 1]) - s2[l] * (psi[:, :, l] - psi[:, :, l + 1])
    ui = 0.5 * (u[:, :, :-1] + u[:, :, 1:])
    vi = 0.5 * (v[:, :, :-1] + v[:, :, 1:])
    dp = psi[:, :, :-1] - psi[:, :, 1:]
    scb = s2[:-1] * h[:-1] * dp
    sc_bb = np.zeros_like(psi)
    sc_bb[:, :, 0] = 0.25 * (s2[0] * (psi[:, :, 1] - psi[:, :, 0]) ** 2)
    for l in range(1, L - 1):
        sc_bb[:, :, l] = 0.25 * (s1[l] * (psi[:, :, l - 1] - psi[:, :, l]) ** 2 + s2[l] * (psi[:, :, l + 1] - psi[:, :, l]) ** 2)
    sc_bb[:, :, -1] = 0.25 * (s1[L - 1] * (psi[:, :, -2] - psi[:, :, -1]) ** 2)
    return [u * u, v * v, ui * ui, vi * vi, u * v, u * rel, v * rel, rel * rel, psi * rel, u * zeta, v * zeta,
            zeta * zeta, zeta * rel, psi * psi, psi * zeta, u * t, v * t, t * rel, t * t,
            0.5 * (u[:, :, 1:] + u[:, :, :-1]) * scb, 0.5 * (v[:, :, 1:] + v[:, :, :-1]) * scb, sc_bb,
            s2[:-1] * h[:-1] * dp ** 2 / (h[:-1] + h[1:])]


@pytest.mark.parametrize("partial_slip,periodic", [(True, False), (False, False), (True, True)])
def test_oracle_quad_diagnostics(partial_slip, periodic):
    """The quad eddy covariances (qg3.F90:683-721, qg3p_diagnostics.F90:941-1537)
    of the oracle against a numpy statement, over steps with and without the
    threshold passed; in a closed basin and in a channel."""
    cfg = channel(17, 20, 3, partial_slip=partial_slip) if periodic else double_gyre(17, 3, partial_slip=partial_slip)
    o = run_oracle(cfg, 1, seed=7)
    dt = O.cfg_from(cfg)["dt"]
    thr = o.scalars()["model_time"] + 1.2 * dt
    o.average(2, thr)
    acc = None
    dtime = 0.0
    for k in range(5):
        o.step_to_dump()
        t = o.scalars()["model_time"]
        if t > thr:
            # zeta at the diagnostics (before the forcing the dump point
            # includes): rel minus the stratification coupling, the inverse
            # of rel_from_zeta_and_psi / update_zeta_bc
            psi, rel = o.sdata("psi"), o.sdata("rel")
            oc = O.cfg_from(cfg)
            s1, s2 = np.array(oc["s1"]), np.array(oc["s2"])
            zeta = rel.copy()
            zeta[:, :, 0] -= s2[0] * (psi[:, :, 0] - psi[:, :, 1])
            zeta[:, :, 1] -= s1[1] * (psi[:, :, 1] - psi[:, :, 0]) + s2[1] * (psi[:, :, 1] - psi[:, :, 2])
            zeta[:, :, 2] -= s1[2] * (psi[:, :, 2] - psi[:, :, 1])
            terms = numpy_quad_terms(psi, rel, zeta, cfg, periodic)
            acc = [dt * x for x in terms] if acc is None else [a + dt * x for a, x in zip(acc, terms)]
            dtime += dt
        o.finish_step()
    for q, want in enumerate(acc):
        got = o.get_quad(q)
        assert got.shape == want.shape, (q, got.shape, want.shape)
        np.testing.assert_allclose(got, want / dtime, rtol=1e-9, atol=1e-12 * np.abs(want).max() / dtime,
                                   err_msg=O.Model.QUAD[q])


def test_oracle_quad_diagnostics_leapfrog():
    """The leapfrog sub-step accumulates the covariances of the level it just
    inverted (psi, rel, zeta BLEAPFROG, qg3.F90:683-721), gated on the model
    time after its increment."""
    cfg = double_gyre(17, 3, scheme=pq.SCHEME_LEAPFROG)
    o = run_oracle(cfg, 2, seed=9)
    dt = O.cfg_from(cfg)["dt"]
    thr = o.scalars()["model_time"] + 1.5 * dt
    o.average(2, thr)
    acc = None
    dtime = 0.0
    for k in range(5):
        o.step(1)
        t = o.scalars()["model_time"]
        suf = "" if k % 2 == 0 else "2"      # sub-steps alternate levels 1, 2
        if t > thr:
            terms = numpy_quad_terms(o.sdata("psi" + suf), o.sdata("rel" + suf), o.sdata("zeta" + suf), cfg)
            acc = [dt * x for x in terms] if acc is None else [a + dt * x for a, x in zip(acc, terms)]
            dtime += dt
    assert 0 < dtime < 5 * dt
    for q, want in enumerate(acc):
        np.testing.assert_allclose(o.get_quad(q), want / dtime, rtol=1e-9, atol=1e-12 * np.abs(want).max() / dtime,
                                   err_msg=O.Model.QUAD[q])
