"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Plain FP64 form tolerances: relative L2 <= 1e-12 for one solve or one step,
<= 1e-9 after 100 steps, on fields and energy diagnostics.
"""
import math

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


def helm_cfg(ii, jj, ss, periodic=False):
    """A context whose layers are Helmholtz problems with the given ss."""
    L = len(ss)
    d = pq.ModelDesc()
    d.ii, d.jj, d.layers = ii, jj, L
    d.periodic_j = int(periodic)
    d.limiter, d.bc_type, d.dt = 1, pq.BC_FREE_SLIP, 1.0
    for k in range(L):
        d.ss[k] = ss[k]
        d.h[k] = 1.0
        for m in range(L):
            d.m2z[k + L * m] = 1.0 if k == m else 0.0
            d.z2m[k + L * m] = 1.0 if k == m else 0.0
    return pq.Config(d, None, 1.0)


@pytest.mark.parametrize("ii,jj,ss", [
    (5, 5, [0.0]),
    (9, 9, [0.0, 0.5]),
    (17, 33, [0.0, 1.3, 7.0]),
    (33, 20, [0.25]),
    (65, 65, [0.0, 2.0, 9.0]),
    (129, 257, [0.0, 0.7]),
    (257, 129, [0.0, 3.0, 11.0]),
    (1025, 1025, [0.0, 1.07613857, 3.31661571]),
    (1025, 1025, [0.0, 0.4, 1.1, 2.5, 6.0]),
    (2049, 2049, [0.0, 0.3, 1.2, 4.0, 9.5]),
])
def test_helm_matches_oracle(ii, jj, ss):
    rng = np.random.default_rng(ii * 7 + jj)
    L = len(ss)
    rhs = np.asfortranarray(rng.standard_normal((ii, jj, L)))
    g = pq.Model(helm_cfg(ii, jj, ss))
    out = g.helm(rhs)
    ref = O.Helm(ii, jj, L, ss)(rhs)
    for l in range(L):
        assert rel_l2(out[:, :, l], ref[:, :, l]) <= TOL_STEP, (l, rel_l2(out[:, :, l], ref[:, :, l]))
    # Untouched entries keep the input (helm's in-place semantics).
    assert np.array_equal(out[0, :, :], rhs[0, :, :])
    assert np.array_equal(out[:, -1, :], rhs[:, -1, :])


@pytest.mark.parametrize("ss,min_order", [(0.0, 2.0), (0.5, 3.9)])
def test_helm_convergence_gpu(ss, min_order):
    """test_helmholtz.F90:27-137 through the CUDA path."""
    PI = math.pi
    sizes = (33, 65, 129, 257, 513, 1025, 2049)
    errs = []
    for g in sizes:
        i = np.arange(1, g + 1)[:, None]
        j = np.arange(1, g + 1)[None, :]
        x = (j - 1) / (g - 1)
        y = (g - i) / (g - 1)
        exact = np.sin(PI * x) * np.sin(PI * y)
        if ss == 0.0:
            rhs = -PI * PI * exact * (2.0 / (g - 1) ** 2)
        else:
            rhs = -exact * (2.0 * PI * PI / (g - 1) ** 2 + ss)
        m = pq.Model(helm_cfg(g, g, [ss]))
        out = m.helm(np.asfortranarray(rhs[:, :, None]))
        out = O.apply_dirichlet_bc(out, 0.0)
        errs.append(np.abs(out[:, :, 0] - exact).max())
        m.close()
    orders = [-math.log10(errs[n] / errs[n - 1]) / math.log10(sizes[n] / sizes[n - 1]) for n in range(1, len(errs))]
    assert min(orders) >= min_order, orders


@pytest.mark.parametrize("ii,jj,ss", [
    (33, 64, [0.0]),
    (65, 128, [0.0, 2.0]),
    (129, 40, [0.5, 0.0, 7.0]),
    (257, 512, [0.0, 1.07613857]),
])
def test_helm_periodic_matches_oracle(ii, jj, ss):
    """The channel (periodic in j): Thomas solve plus periodic_ge's cyclic
    closure, qg3p_helmholtz.F90:473-610, against the oracle."""
    rng = np.random.default_rng(ii + 3 * jj)
    L = len(ss)
    rhs = np.asfortranarray(rng.standard_normal((ii, jj, L)))
    g = pq.Model(helm_cfg(ii, jj, ss, periodic=True))
    out = g.helm(rhs)
    ref = O.Helm(ii, jj, L, ss, periodic_j=True)(rhs)
    for l in range(L):
        assert rel_l2(out[:, :, l], ref[:, :, l]) <= TOL_STEP, (l, rel_l2(out[:, :, l], ref[:, :, l]))
    assert np.array_equal(out[0, :, :], rhs[0, :, :])
    if any(s == 0.0 for s in ss[1:]):
        # free slip and ss = 0 in a baroclinic mode: no momentum correction,
        # so no channel time step on this context
        with pytest.raises(pq.PQError):
            g.init_perturb(np.zeros((ii, jj, L)))


@pytest.mark.parametrize("ss,min_order", [(0.0, 2.0), (0.5, 3.9)])
def test_helm_periodic_convergence_gpu(ss, min_order):
    """test_helmholtz.F90:249-357 (periodic channel) through the CUDA path."""
    PI = math.pi
    sizes = (33, 65, 129, 257, 513, 1025)
    errs = []
    for g in sizes:
        ii, jj = g, (g - 1) * 2
        i = np.arange(1, ii + 1)[:, None]
        j = np.arange(1, jj + 1)[None, :]
        x = (j - 1) / jj
        y = (ii - i) / (ii - 1)
        exact = np.cos(2.0 * PI * x) * np.sin(PI * y)
        if ss == 0.0:
            rhs = -PI * PI * exact * ((1.0 / (ii - 1) ** 2) + (4.0 / jj ** 2))
        else:
            rhs = -exact * ((PI * PI / (ii - 1) ** 2) + (4.0 * PI * PI / jj ** 2) + ss)
        m = pq.Model(helm_cfg(ii, jj, [ss], periodic=True))
        out = m.helm(np.asfortranarray(rhs[:, :, None]))
        out = O.apply_dirichlet_bc(out, 0.0, periodic_j=True)
        errs.append(np.abs(out[:, :, 0] - exact).max())
        m.close()
    orders = [-math.log10(errs[n] / errs[n - 1]) / math.log10(sizes[n] / sizes[n - 1]) for n in range(1, len(errs))]
    assert min(orders) >= min_order, orders


EPS = np.finfo(np.float64).eps


def fne(a, b):
    """test_tools' fne: differ by more than 10 ulp."""
    a = np.atleast_1d(np.asarray(a, dtype=np.float64))
    b = np.atleast_1d(np.asarray(b, dtype=np.float64))
    return bool(np.any(np.abs(a - b) > 10.0 * np.maximum(np.spacing(np.abs(a)), EPS)))


def test_laplace_bc_gpu():
    """test_laplace_bc.F90:21-44 entirely on the device: laplace_bc_rhs,
    helm and apply_dirichlet_bc give psi == 1 to 10 ulp for BC = 1; and the
    lifting is linear (add_laplace_bc_rhs on a RHS of ones minus the BC = 0
    solution is 1)."""
    ii = jj = 9
    m = pq.Model(helm_cfg(ii, jj, [0.0]))
    phi = m.laplace_bc_rhs(1.0)
    phi = m.apply_dirichlet_bc(m.helm(phi[:, :, None]), 1.0)
    assert not (fne(phi.min(), 1.0) or fne(phi.max(), 1.0)), (phi.min(), phi.max())
    phi0 = m.apply_dirichlet_bc(m.helm(np.ones((ii, jj, 1), order="F")), 0.0)
    phi1 = m.add_laplace_bc_rhs(np.ones((ii, jj), order="F"), 1.0)
    phi1 = m.apply_dirichlet_bc(m.helm(phi1[:, :, None]), 1.0)
    d = phi1 - phi0
    assert not (fne(d.min(), 1.0) or fne(d.max(), 1.0)), (d.min(), d.max())


def test_laplace_bc_periodic_gpu():
    """test_laplace_bc.F90:50-80 on the device: in the channel, the wall
    values (1, 0) and (0, 1) give psi linear in i, exactly."""
    ii = jj = 9
    m = pq.Model(helm_cfg(ii, jj, [0.0], periodic=True))
    i = np.arange(1, ii + 1)[:, None]
    for bc_b, bc_d in ((1.0, 0.0), (0.0, 1.0)):
        phi = m.add_laplace_bc_rhs(np.zeros((ii, jj), order="F"), bc_b, bc_d)
        phi = m.apply_dirichlet_bc(m.helm(phi[:, :, None]), bc_b, bc_d)
        exact = (ii - i) / (ii - 1) if bc_b == 1.0 else (i - 1) / (ii - 1)
        assert not fne(np.abs(phi[:, :, 0] - exact).max(), 0.0)


@pytest.mark.parametrize("ii,jj,periodic", [(33, 20, False), (65, 65, False), (17, 40, True), (129, 64, True)])
def test_laplace_bc_matches_oracle_bitwise(ii, jj, periodic):
    """Every variant (one layer; all layers with one value; one value per
    layer; the channel's two walls) equals the oracle's restatement of
    qg3p_laplace_bc.F90 to the bit, with host and device arrays."""
    import torch

    L = 3
    m = pq.Model(helm_cfg(ii, jj, [0.0, 1.0, 2.0], periodic=periodic))
    rng = np.random.default_rng(ii + jj)
    f = np.asfortranarray(rng.standard_normal((ii, jj, L)))
    bcs = np.array([0.3, -1.7, 2.9])
    bds = np.array([1.1, 0.25, -0.6]) if periodic else None
    # one layer, one value
    out = m.add_laplace_bc_rhs(f[:, :, 1], 0.7, 0.2 if periodic else None)
    ref = O.add_laplace_bc_rhs(f[:, :, 1], 0.7, 0.2 if periodic else None, periodic_j=periodic)
    assert np.array_equal(out, ref)
    out = m.apply_dirichlet_bc(f[:, :, 1], 0.7, 0.2 if periodic else None)
    ref = O.apply_dirichlet_bc(f[:, :, 1], 0.7, 0.2 if periodic else None, periodic_j=periodic)
    assert np.array_equal(out, ref)
    # all layers, one value per layer
    out_a = m.add_laplace_bc_rhs(f, bcs, bds)
    out_d = m.apply_dirichlet_bc(f, bcs, bds)
    for l in range(L):
        bd = None if bds is None else bds[l]
        assert np.array_equal(out_a[:, :, l], O.add_laplace_bc_rhs(f[:, :, l], bcs[l], bd, periodic_j=periodic))
        assert np.array_equal(out_d[:, :, l], O.apply_dirichlet_bc(f[:, :, l], bcs[l], bd, periodic_j=periodic))
    # device arrays, asynchronous on the context's stream
    dev = torch.from_numpy(np.ascontiguousarray(f.ravel(order="F"))).cuda()
    torch.cuda.synchronize()
    b = np.ascontiguousarray(bcs)
    d = None if bds is None else np.ascontiguousarray(bds)
    rc = pq.lib().pq_add_laplace_bc_rhs(m.ctx, pq.C.cast(dev.data_ptr(), pq._dp), L, pq._p(b),
                                        None if d is None else pq._p(d), L, pq.PTR_DEVICE)
    assert rc == 0
    m.sync()
    got = dev.cpu().numpy().reshape((ii, jj, L), order="F")
    assert np.array_equal(got, out_a)
    # argument checks
    with pytest.raises(pq.PQError):
        m.add_laplace_bc_rhs(np.zeros((ii, jj, 4)), 1.0)  # more layers than the context
    if not periodic:
        with pytest.raises(pq.PQError):
            m.apply_dirichlet_bc(f, 1.0, 2.0)  # a second wall value in a closed basin


def double_gyre(ii, layers=3, dt=1800.0, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5),
         5: (2.5e4, 5.0e4, 7.5e4, 1.0e5, 1.5e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75), 5: (1.5, 0.75, 0.375, 0.1875)}[layers]
    p = pq.double_gyre_physical(ii, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    return pq.Config.from_physical(p)


@pytest.mark.parametrize("ii,layers", [(33, 1), (65, 2), (129, 3), (65, 5)])
def test_pv_inversion_matches_oracle(ii, layers):
    cfg = double_gyre(ii, layers)
    rng = np.random.default_rng(ii + layers)
    zeta = np.asfortranarray(rng.standard_normal((ii, ii, layers)))
    g = pq.Model(cfg)
    psi = g.pv_inversion(zeta)
    om = O.Model(O.cfg_from(cfg))
    zd = np.zeros((ii + 2, ii + 2, layers), order="F")
    zd[1:-1, 1:-1, :] = zeta
    ref = om.pv_inversion(zd)[1:-1, 1:-1, :]
    assert rel_l2(psi, ref) <= TOL_STEP, rel_l2(psi, ref)


def start(cfg, seed=1):
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    g = pq.Model(cfg)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return g, o


FIELDS = ["psi", "zeta", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res", "res_beta"]


def compare(g, o, tol, fields=FIELDS):
    worst = {}
    for f in fields:
        a, b = g.get(f), o.get(f)
        worst[f] = rel_l2(a, b)
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, worst
    return worst


def test_init_matches_oracle():
    cfg = double_gyre(65, 3)
    g, o = start(cfg)
    compare(g, o, TOL_STEP, ["psi", "zeta", "zeta_old"])
    assert rel_l2(g.get("rel"), o.get("rel")) <= TOL_STEP


@pytest.mark.parametrize("ii,layers", [(33, 1), (65, 3), (129, 3), (65, 5)])
def test_one_step_matches_oracle(ii, layers):
    cfg = double_gyre(ii, layers)
    g, o = start(cfg)
    g.step(1)
    o.step(1)
    compare(g, o, TOL_STEP)
    assert rel_l2(g.get("rel"), o.get("rel")) <= TOL_STEP


def test_ten_steps_each_matches_oracle():
    cfg = double_gyre(129, 3)
    g, o = start(cfg, seed=2)
    for s in range(10):
        g.step(1)
        o.step(1)
        compare(g, o, TOL_STEP * 10, ["psi", "zeta"])
    compare(g, o, TOL_STEP * 10)


def test_hundred_steps_and_energy():
    cfg = double_gyre(129, 3)
    g, o = start(cfg, seed=3)
    g.step(100)
    o.step(100)
    compare(g, o, TOL_100)
    ek_g, ep_g = g.energy()
    ek_o, ep_o = o.energy()
    assert rel_l2(ek_g, ek_o) <= TOL_100
    assert abs(ep_g - ep_o) <= TOL_100 * abs(ep_o)
    assert abs(g.cfl() - o.cfl()) <= TOL_100 * o.cfl()
    sc = g.scalars()
    assert abs(sc["model_time"] - o.scalars()["model_time"]) <= 1e-12 * sc["model_time"]


def test_adaptive_dt_matches_oracle():
    cfg = double_gyre(65, 3, adapt_dt=1, target_cfl=0.1, max_dt=86400.0)
    g, o = start(cfg, seed=4)
    g.step(20)
    o.step(20)
    compare(g, o, 1e-10)
    sg, so = g.scalars(), o.scalars()
    for k in ("dt", "tweight_a", "tweight_u"):
        assert abs(sg[k] - so[k]) <= 1e-10 * abs(so[k]), (k, sg[k], so[k])


def test_energy_kats_gpu():
    """test_energy_2.F90:42-66 through the device energy reduction."""
    cfg = double_gyre(9, 2)
    g = pq.Model(cfg)
    ii = jj = 9
    psi = np.zeros((ii + 2, jj + 2, 2), order="F")
    h = np.array(cfg.desc.h[:2])
    s2 = np.array(cfg.desc.s2[:2])
    for v1, v2 in ((1.0, 0.0), (2.0, 0.0), (0.0, 0.0)):
        psi[1:-1, 1:-1, 0] = v1
        psi[1:-1, 1:-1, 1] = v2
        g.set("psi", psi)
        ek, ep = g.energy()
        ek_o, ep_o = O.energy(psi, h, s2)
        assert abs(ep - ep_o) <= 1e-14 * max(abs(ep_o), 1e-300)
        assert np.allclose(ek, ek_o, rtol=0, atol=1e-14)
    for i in range(ii):
        psi[i + 1, 1:-1, 0] = i + 1.0
        psi[i + 1, 1:-1, 1] = i + 2.0
    g.set("psi", psi)
    ek, ep = g.energy()
    ek_o, ep_o = O.energy(psi, h, s2)
    assert np.allclose(ek, ek_o, rtol=1e-13, atol=0)
    assert abs(ep - ep_o) <= 1e-13 * abs(ep_o)


@pytest.mark.parametrize("kernel,band,group,lanes", [(1, 4, 0, 0), (1, 8, 1, 16), (1, 32, 2, 0), (1, 128, 1, 32),
                                                     (0, 16, 2, 0), (0, 16, 1, 32)])
def test_tile_parameters_do_not_change_results(kernel, band, group, lanes):
    """The CABARET formulation (tiles or warp sweeps), the sweep's band height,
    the DST CTA width and the DST lanes per unit are tuning knobs: results
    must match the oracle for any choice.  At 129 x 129 the sweeps are
    mostly boundary sweeps and, with 4-row bands, more than the resident
    warps, so every warp claims several from the queue."""
    cfg = double_gyre(129, 3)
    g, o = start(cfg, seed=5)
    g.set_tuning(cab_kernel=kernel, cab_band=band, dst_group=group, dst_lanes=lanes, dst_lanes_inv=lanes)
    assert g.get_tuning() == {"cab_band": band, "dst_group": group, "cab_kernel": kernel,
                              "dst_lanes": lanes if lanes else 32, "dst_lanes_inv": lanes if lanes else 32,
                              "pdl": 0, "dst_algo": 1}
    g.step(3)
    o.step(3)
    compare(g, o, TOL_STEP * 10)


@pytest.mark.parametrize("ii,kernel,band", [(129, 1, 4), (129, 2, 4), (257, 2, 16), (65, 2, 8), (1025, 1, 16),
                                            (1025, 2, 32), (1025, 2, 16), (1025, 0, 16)])
def test_mixed_cabaret_formulations_agree(ii, kernel, band):
    """The mixed form's CABARET formulations -- tiles, sweeps with one and
    with two columns per lane (interior sweeps with vector loads and stores;
    boundary sweeps, whose last strip ends mid-lane-pair since ii is odd;
    at 65 x 65 two strips, both boundary ones).

    One step from the same state (the oracle's after 4 steps): every field
    of the formulation under test within 1e-5 of its maximum of a second
    formulation's (they differ only in how FP32 sums are rounded: 7e-7
    measured at 1025^2; the velocities come from FP64 psi and agree bit for
    bit).  Trajectories are compared with the oracle only through psi (5
    steps, 1e-6): later steps amplify last-bit differences, and where a face
    velocity is near zero its upwind face value flips, which the FP32
    residual res shows as local jumps of 1e-3 of its maximum."""
    cfg = double_gyre(ii, 3, precision=pq.PREC_MIXED)
    fields = ("psi", "zeta", "ui", "uj", "zeta_fi", "zeta_fj", "res")
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=8, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    o.step(4)
    state = {f: o.get(f) for f in ["psi", "zeta", "zeta_old", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj",
                                   "res", "res_beta", "rel"]}
    o.step(1)
    psi5 = o.get("psi")
    out = []
    for k in (kernel, 1 if kernel != 1 else 0):
        g = pq.Model(cfg)
        g.init_perturb(ic)
        g.set_tuning(cab_kernel=k, cab_band=band)
        assert g.get_tuning()["cab_kernel"] == k
        if k == kernel:
            g.step(5)
            assert rel_l2(g.get("psi"), psi5) <= 1e-6
        for f, v in state.items():
            g.set(f, v)
        g.step(1)
        out.append({f: g.get(f) for f in fields})
        g.close()
    for f in fields:
        d = np.abs(out[0][f] - out[1][f]).max()
        assert d <= 1e-5 * np.abs(out[1][f]).max(), (f, d)


def test_two_column_sweeps_refused_in_fp64():
    g = pq.Model(double_gyre(129, 3))
    with pytest.raises(pq.PQError):
        g.set_tuning(cab_kernel=2)
    g.close()


def test_state_writes_between_steps():
    """Fixed-dt steps carry the next step's predictor in the fused CABARET
    kernel; writing the state between steps must drop it and give the same
    trajectory as the oracle."""
    cfg = double_gyre(65, 3)
    g, o = start(cfg, seed=6)
    g.step(3)
    o.step(3)
    for f in ("zeta", "res", "res_beta", "ui"):
        g.set(f, g.get(f))
    g.step(2)
    o.step(2)
    compare(g, o, TOL_STEP * 10)
    assert rel_l2(g.get("rel"), o.get("rel")) <= TOL_STEP * 10


def test_odd_step_counts_match_oracle():
    """Eager steps, two-step graphs and trailing steps interleave by parity."""
    cfg = double_gyre(65, 3)
    g, o = start(cfg, seed=7)
    for n in (1, 3, 2, 5):
        g.step(n)
        o.step(n)
    compare(g, o, TOL_STEP * 10)


@pytest.mark.parametrize("ii,lanes", [(257, 64), (513, 64), (513, 16)])
def test_dst_units_of_two_warps_match_oracle(ii, lanes):
    """Row DST units spread over two warps (named barriers between the
    passes, a two-level scan) or over half warps give the oracle's results."""
    cfg = double_gyre(ii, 3)
    g, o = start(cfg, seed=8)
    g.set_tuning(dst_lanes=lanes, dst_lanes_inv=lanes)
    g.step(3)
    o.step(3)
    compare(g, o, TOL_STEP * 10)
    with pytest.raises(pq.PQError):
        g.set_tuning(dst_lanes=128)


@pytest.mark.parametrize("ii,kernel", [(129, 0), (129, 1), (513, 0)])
def test_programmatic_dependent_launch_matches_oracle(ii, kernel):
    """With pdl on, each step kernel may be scheduled before its predecessor
    ends and waits for it on the device: same results, graphs included."""
    cfg = double_gyre(ii, 3)
    g, o = start(cfg, seed=9)
    g.set_tuning(pdl=1, cab_kernel=kernel)
    for n in (1, 2, 3):
        g.step(n)
        o.step(n)
    compare(g, o, TOL_STEP * 10)


def test_pipelined_exchange_matches_oracle():
    """pq_step_exchange with host buffers overlaps its copies with the
    neighbouring steps; every step still takes its own input and returns
    its own psi."""
    cfg = double_gyre(129, 3)
    g, o = start(cfg, seed=10)
    g.step(2)
    o.step(2)
    ii, jj, L = cfg.ii, cfg.jj, cfg.layers
    rng = np.random.default_rng(10)
    inputs, outs = [], []
    for k in range(5):
        z = np.asfortranarray(o.sdata("zeta") * (1.0 + 1e-3 * rng.standard_normal((ii, jj, L))))
        inputs.append(np.ascontiguousarray(z.ravel(order="F")))
        outs.append(np.zeros(ii * jj * L))
    for k in range(5):
        g.step_exchange(inputs[k].ctypes.data, outs[k].ctypes.data, pq.PTR_HOST)
    g.sync()
    for k in range(5):
        zd = o.get("zeta")
        zd[1:-1, 1:-1] = inputs[k].reshape((ii, jj, L), order="F")
        o.set("zeta", zd)
        o.set("zeta_old", zd)
        o.step(1)
        psi = outs[k].reshape((ii, jj, L), order="F")
        assert rel_l2(psi, o.sdata("psi")) <= TOL_STEP * 10, k


@pytest.mark.parametrize("tuning", [{}, {"dst_group": 2, "dst_lanes": 32, "dst_lanes_inv": 32}])
def test_1025_steps_match_oracle(tuning):
    """1025 x 1025 x 3: the warp-sweep CABARET kernel, the unstaged
    tridiagonal kernel, and both places the mass correction psiC is summed:
    the tridiagonal kernel's last CTA when the inverse DST's grid is several
    waves (default geometry, 1025 CTAs) and the inverse DST's own CTAs when it
    is one wave (two rows per CTA, 513 CTAs)."""
    cfg = double_gyre(1025, 3)
    g, o = start(cfg, seed=9)
    if tuning:
        g.set_tuning(**tuning)
    g.step(2)
    o.step(2)
    compare(g, o, TOL_STEP * 10)


def test_cabaret_step_with_callers_dt():
    """pq_cabaret_step: the time step and weights come from the caller, as
    the reference passes them to every cabaret_* routine.  The oracle adapts
    dt itself (cabaret_adapt_dt); a fixed-dt device context stepped with the
    oracle's dt and weights of every step follows its trajectory."""
    cfg_a = double_gyre(65, 3, adapt_dt=1, target_cfl=0.1, max_dt=86400.0)
    cfg_f = double_gyre(65, 3)
    ic = pq.make_ic(65, 65, 3, seed=21, amplitude=1e-7 * cfg_a.t_scale, sigma=3.0)
    o = O.Model(O.cfg_from(cfg_a))
    o.init(ic)
    g = pq.Model(cfg_f)
    g.init_perturb(ic)
    for k in range(15):
        o.step(1)
        s = o.scalars()
        g.cabaret_step(s["dt"], s["tweight_a"], s["tweight_u"])
        sg = g.scalars()
        assert sg["dt"] == s["dt"] and sg["tweight_a"] == s["tweight_a"]
    compare(g, o, 1e-10)
    assert abs(g.scalars()["model_time"] - o.scalars()["model_time"]) <= 1e-12 * o.scalars()["model_time"]
    with pytest.raises(pq.PQError):
        g.cabaret_step(-1.0)
    with pytest.raises(pq.PQError):
        g.cabaret_step(1.0, 0.5, 1.5)
