"""The channel (periodic in j) CABARET time step of the oracle: the
momentum-corrected PV inversion (correction_function_momentum,
zeta_boundary, modes_to_z_correct_momentum, qg3p_aux.F90:233-379, 524-575),
the periodic halo updates of the time loop (qg3p_base.F90:1887-1956,
2964-3003), and properties the reference's channel has by construction."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O


def channel(ii, jj, layers=3, dt=1800.0, **kw):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, jj=jj, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp, **kw)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = 1
    return cfg


def wall_pv_means(cfg, psi_modal, ss):
    """zeta_boundary in numpy: mean wall PV of each modal field (ii, jj, L)."""
    oc = O.cfg_from(cfg)
    bc, alpha = oc["bc_type"], oc["alpha"]
    jj = psi_modal.shape[1]
    zb = np.zeros(psi_modal.shape[2])
    zd = np.zeros_like(zb)
    for l in range(psi_modal.shape[2]):
        p = psi_modal[:, :, l]
        if bc == pq.BC_PARTIAL_SLIP:
            c = alpha / (alpha + 3.0)
            zb[l] = np.sum(c * (-3.5 * p[0] + 4.0 * p[1] - 0.5 * p[2]))
            zd[l] = np.sum(c * (-3.5 * p[-1] + 4.0 * p[-2] - 0.5 * p[-3]))
        elif bc == pq.BC_NO_SLIP:
            zb[l] = np.sum(2.0 * (p[1] - p[0]))
            zd[l] = np.sum(2.0 * (p[-2] - p[-1]))
        zb[l] -= ss[l] * np.sum(p[0])
        zd[l] -= ss[l] * np.sum(p[-1])
    return zb / jj, zd / jj


def start(cfg, seed):
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return o, ic


@pytest.mark.parametrize("bc", [True, False])
def test_channel_inversion_meets_the_wall_constraints(bc):
    """After the momentum correction every baroclinic mode of psi has zero
    mean wall PV on both walls, and psi is 0 on the walls in the barotropic
    mode (no net transport through the channel)."""
    cfg = channel(33, 32, 3, partial_slip=bc)
    o, _ = start(cfg, 11)
    psi = o.sdata("psi")
    ss, m2z, z2m = cfg.modal()
    modal = np.einsum("ml,ijl->ijm", z2m, psi)
    zb, zd = wall_pv_means(cfg, modal, ss)
    scale = np.abs(modal).max()
    assert np.all(np.abs(zb[1:]) <= 1e-12 * scale) and np.all(np.abs(zd[1:]) <= 1e-12 * scale), (zb, zd)
    assert np.abs(modal[0, :, 0]).max() <= 1e-14 * scale and np.abs(modal[-1, :, 0]).max() <= 1e-14 * scale


def test_channel_is_periodic_in_j():
    """Shifting the initial PV by s rows shifts the whole run by s rows: the
    channel has no seam (up to the order of the wall sums)."""
    cfg = channel(33, 32, 3)
    ic = pq.make_ic(33, 32, 3, seed=12, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    a = O.Model(O.cfg_from(cfg))
    a.init(ic)
    b = O.Model(O.cfg_from(cfg))
    b.init(np.asfortranarray(np.roll(ic, 5, axis=1)))
    a.step(6)
    b.step(6)
    for f in ("psi", "zeta"):
        pa, pb = a.sdata(f), b.sdata(f)
        err = np.abs(np.roll(pa, 5, axis=1) - pb).max() / np.abs(pa).max()
        assert err <= 1e-12, (f, err)


def test_channel_halos_follow_the_rows():
    """The halo rows of psi and zeta hold the opposite sdata rows, and the
    seam j-faces of uj and zeta_fj agree (update_pdata / update_flux_j)."""
    cfg = channel(33, 32, 2)
    o, _ = start(cfg, 13)
    o.step(3)
    for f in ("psi", "zeta"):
        a = o.get(f)
        np.testing.assert_array_equal(a[1:-1, 0], a[1:-1, -2])
        np.testing.assert_array_equal(a[1:-1, -1], a[1:-1, 1])
    for f in ("uj", "zeta_fj"):
        a = o.get(f)   # (ii+2, jj+3, L): faces 1..jj+3 (1-based)
        np.testing.assert_array_equal(a[2:33, 0], a[2:33, 32])
        np.testing.assert_array_equal(a[2:33, -1], a[2:33, 2])
        np.testing.assert_array_equal(a[2:33, 33], a[2:33, 1])
    assert np.isfinite(o.get("psi")).all()


def test_leapfrog_channel_is_periodic_with_consistent_halos():
    """The leapfrog channel (halo updates after zeta_centred, the forward
    Euler start and the pickup, qg3.F90:355-361, 475, 625): shifting both
    levels' initial PV by s rows shifts the run, and every level's halo rows
    hold the opposite rows."""
    cfg = channel(33, 32, 3, scheme=pq.SCHEME_LEAPFROG)
    ic1 = pq.make_ic(33, 32, 3, seed=14, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    ic2 = pq.make_ic(33, 32, 3, seed=15, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    ic = np.asfortranarray(np.stack([ic1, ic2], axis=3))
    a = O.Model(O.cfg_from(cfg))
    a.init(ic)
    b = O.Model(O.cfg_from(cfg))
    b.init(np.asfortranarray(np.roll(ic, 5, axis=1)))
    a.step(7)
    b.step(7)
    for f in ("psi", "zeta", "psi2", "zeta2"):
        pa, pb = a.sdata(f), b.sdata(f)
        err = np.abs(np.roll(pa, 5, axis=1) - pb).max() / np.abs(pa).max()
        assert err <= 1e-12, (f, err)
    for f in ("psi", "zeta", "rel", "zeta_old", "psi2", "zeta2", "rel2", "zeta_old2"):
        x = a.get(f)
        np.testing.assert_array_equal(x[1:-1, 0], x[1:-1, -2], err_msg=f)
        np.testing.assert_array_equal(x[1:-1, -1], x[1:-1, 1], err_msg=f)
