"""Pin the CPU oracle against PEQUOD's own known-answer tests.

Each test restates one of the reference's unittest programs (file:line cited)
on the oracle; the expected values are the reference's.  Tolerances follow
test_tools.F90:26,86-160: fne(a, b) fails when |a - b| > 10*max(spacing(a),
epsilon).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

PI = 3.14159265358979323846
EPS = np.finfo(np.float64).eps


def fne(a, b):
    a = np.atleast_1d(np.asarray(a, dtype=np.float64))
    b = np.atleast_1d(np.asarray(b, dtype=np.float64))
    tol = 10.0 * np.maximum(np.spacing(np.abs(a)), EPS)
    return bool(np.any(np.abs(a - b) > tol))


def _manufactured(ii, jj, ss, periodic):
    """Right-hand side and exact solution of test_helmholtz.F90:45-58."""
    i = np.arange(1, ii + 1)[:, None]
    j = np.arange(1, jj + 1)[None, :]
    g_jj_int = jj if periodic else jj - 1
    x = (j - 1) / g_jj_int
    y = (ii - i) / (ii - 1)
    if periodic:
        exact = np.cos(2.0 * PI * x) * np.sin(PI * y)
        kx2 = 4.0
    else:
        exact = np.sin(PI * x) * np.sin(PI * y)
        kx2 = 1.0
    if ss == 0.0:
        rhs = -PI * PI * exact * ((1.0 / (ii - 1) ** 2) + (kx2 / g_jj_int ** 2))
    else:
        rhs = -exact * ((PI * PI / (ii - 1) ** 2) + (kx2 * PI * PI / g_jj_int ** 2) + ss)
    return np.asfortranarray(rhs[:, :, None]), exact


@pytest.mark.parametrize(
    "ss,shape,periodic,min_order",
    [
        (0.0, "square", False, 2.0),      # test_helmholtz.F90:27-82
        (0.5, "square", False, 3.9),      # :84-137
        (0.0, "nonsquare", False, 2.0),   # :139-192
        (0.5, "nonsquare", False, 3.9),   # :194-247
        (0.0, "periodic", True, 2.0),     # :249-302
        (0.5, "periodic", True, 3.9),     # :304-357
    ],
)
def test_helm_convergence(ss, shape, periodic, min_order):
    sizes = (33, 65, 129, 257, 513, 1025, 2049)
    errs = []
    for g in sizes:
        ii = g
        jj = {"square": g, "nonsquare": (g - 1) * 2 + 1, "periodic": (g - 1) * 2}[shape]
        if g == 2049 and shape != "square":
            break  # keeps the CPU suite short; 2049 square is still covered
        rhs, exact = _manufactured(ii, jj, ss, periodic)
        h = O.Helm(ii, jj, 1, [ss], periodic_j=periodic)
        out = O.apply_dirichlet_bc(h(rhs), 0.0, periodic_j=periodic)
        errs.append(np.abs(out[:, :, 0] - exact).max())
    orders = [
        -math.log10(errs[n] / errs[n - 1]) / math.log10(sizes[n] / sizes[n - 1]) for n in range(1, len(errs))
    ]
    assert min(orders) >= min_order, orders


def test_sint_definition():
    """sint is FFTPACK's unnormalised DST-I: X_k = 2 sum_m x_m sin(m k pi/(n+1))."""
    rng = np.random.default_rng(3)
    for ii in (5, 9, 17, 129, 1025):
        n = ii - 2
        h = O.Helm(ii, ii, 1, [0.0])
        x = rng.standard_normal(n)
        buf = np.zeros(n + 1)
        buf[:n] = x
        y = h.sint(buf)[:n]
        m = np.arange(1, n + 1)
        ref = 2.0 * np.sin(np.outer(m, m) * PI / (n + 1)) @ x
        assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max() * max(1.0, math.log2(n))


def test_laplace_bc():
    """test_laplace_bc.F90:21-44: BC=1 with zero RHS gives psi == 1; linearity."""
    ii = jj = 9
    h = O.Helm(ii, jj, 1, [0.0])
    phi = O.add_laplace_bc_rhs(np.zeros((ii, jj), order="F"), 1.0)
    phi = h(phi[:, :, None])
    phi = O.apply_dirichlet_bc(phi, 1.0)
    assert not (fne(phi.min(), 1.0) or fne(phi.max(), 1.0))

    phi0 = O.apply_dirichlet_bc(h(np.ones((ii, jj, 1), order="F")), 0.0)
    phi1 = O.add_laplace_bc_rhs(np.ones((ii, jj), order="F"), 1.0)
    phi1 = O.apply_dirichlet_bc(h(phi1[:, :, None]), 1.0)
    d = phi1 - phi0
    assert not (fne(d.min(), 1.0) or fne(d.max(), 1.0))


def test_laplace_bc_periodic():
    """test_laplace_bc.F90:50-80: periodic channel, psi linear in i."""
    ii = jj = 9
    h = O.Helm(ii, jj, 1, [0.0], periodic_j=True)
    for bc_b, bc_d in ((1.0, 0.0), (0.0, 1.0)):
        phi = O.add_laplace_bc_rhs(np.zeros((ii, jj), order="F"), bc_b, bc_d, periodic_j=True)
        phi = O.apply_dirichlet_bc(h(phi[:, :, None]), bc_b, bc_d, periodic_j=True)
        i = np.arange(1, ii + 1)[:, None]
        exact = (ii - i) / (ii - 1) if bc_b == 1.0 else (i - 1) / (ii - 1)
        m = np.abs(phi[:, :, 0] - exact).max()
        assert not fne(m, 0.0), m


def test_mean():
    """test_mean.F90:20-55."""
    a = np.ones((3, 3), order="F")
    assert not fne(O.mean(a), 1.0)
    a[1, 1] = 0.0
    assert not fne(O.mean(a), 0.75)
    a = np.ones((4, 4), order="F")
    assert not fne(O.mean(a), 1.0)
    a[1:3, 1:3] = 0.0
    assert not fne(O.mean(a), 5.0 / 9.0)
    a = np.ones((5, 5), order="F")
    assert not fne(O.mean(a), 1.0)
    a[1:4, 1:4] = 0.0
    assert not fne(O.mean(a), 7.0 / 16.0)


def test_energy():
    """test_energy_2.F90:27-66 on one rank with the same 5 x 9 global grid."""
    st = O.strat_from_rd([math.sqrt(0.5)], [1.0, 1.0])
    h, s2 = st["h"], st["s2"]
    ii, jj, L = 5, 9, 2
    psi = np.zeros((ii + 2, jj + 2, L), order="F")
    ekin, epot = O.energy(psi, h, s2)
    assert not fne(epot, 0.0) and not fne(ekin, [0.0, 0.0])
    psi[:] = 1.0
    ekin, epot = O.energy(psi, h, s2)
    assert not fne(epot, 0.0) and not fne(ekin, [0.0, 0.0])
    for v1, v2, ep in ((1.0, 0.0, 0.25), (0.0, 1.0, 0.25), (2.0, 0.0, 1.0)):
        psi[:, :, 0] = v1
        psi[:, :, 1] = v2
        ekin, epot = O.energy(psi, h, s2)
        assert not fne(epot, ep) and not fne(ekin, [0.0, 0.0])
    for scale, ep, ek in ((1.0, 0.25, 0.25), (2.0, 1.0, 1.0)):
        psi[:] = 0.0
        for i in range(2, ii + 2):  # fa_i_min .. fa_i_max (1-based data index)
            psi[i - 1, :, 0] = scale * (i - 1)
            psi[i - 1, :, 1] = scale * (i - 1) + scale
        ekin, epot = O.energy(psi, h, s2)
        assert not fne(epot, ep), epot
        assert not fne(ekin, [ek, ek]), ekin


def test_stratification():
    """test_stratification.F90:16-53."""
    rd1, rd2 = 20.0e5, 10.0e5
    h = [1.0e5, 2.0e5, 3.0e5]
    st = O.strat_from_rd([], [h[0]])
    assert not fne(st["ss"][0], 0.0)
    st = O.strat_from_rd([rd1], h[:2])
    assert not fne(1.0 / math.sqrt(st["ss"][1]), rd1)
    assert not fne(st["ss"][0], 0.0)
    m = st["z2m"] @ np.ones(2)
    assert not fne(m, [1.0, 0.0])
    z = m[0] + st["m2z"][:, 1:] @ m[1:]
    assert not fne(z, [1.0, 1.0])
    st = O.strat_from_rd([rd1, rd2], h)
    assert not fne(1.0 / np.sqrt(st["ss"][1:3]), [rd2, rd1])
    assert not fne(st["ss"][0], 0.0)
    m = st["z2m"] @ np.ones(3)
    assert not fne(m, [1.0, 0.0, 0.0])
    z = m[0] + st["m2z"][:, 1:] @ m[1:]
    assert not fne(z, [1.0, 1.0, 1.0])
    # modes_to_z(z_to_modes(.)) is the identity on arbitrary layer vectors.
    v = np.array([0.3, -1.7, 2.2])
    assert np.allclose(st["m2z"] @ (st["z2m"] @ v), v, rtol=0, atol=1e-14)


def test_eigendecompose():
    """test_eigendecompose.F90:27-90 (real and symmetric cases)."""
    w, v = O.eigen(np.eye(2))
    assert not fne(w, [1.0, 1.0])
    w, v = O.eigen(np.diag([1.0, 2.0]))
    assert not fne(w, [1.0, 2.0])
    for a in (np.eye(2), np.array([[4.0, 5.0], [1.0, 18.0]]), np.array([[4.0, 5.0], [5.0, 18.0]])):
        w, v = O.eigen(a)
        recomposed = v @ np.diag(w) @ np.linalg.inv(v)
        assert np.allclose(recomposed, a, rtol=0, atol=1e-13)
    st = O.strat_from_rd([20.0e5, 10.0e5], [1.0e5, 2.0e5, 3.0e5])
    assert not fne(1.0 / np.sqrt(st["ss"][1:3]), [10.0e5, 20.0e5])
    # Cross-check against numpy's bundled LAPACK.
    S = np.zeros((3, 3))
    s1, s2 = st["s1"], st["s2"]
    S[0, 0], S[0, 1] = -s2[0], s2[0]
    S[1, 0], S[1, 1], S[1, 2] = s1[1], -(s1[1] + s2[1]), s2[1]
    S[2, 1], S[2, 2] = s1[2], -s1[2]
    w, _ = O.eigen(S)
    scale = np.abs(w).max()
    assert np.allclose(np.sort(w), np.sort(np.linalg.eigvals(S).real), rtol=1e-13, atol=1e-14 * scale)


def test_inverse_and_determinant():
    """test_inverse.F90:21-48."""
    cases = [
        (np.eye(2), 1.0, np.eye(2)),
        (np.diag([1.0, 2.0]), 2.0, np.diag([1.0, 0.5])),
        (np.array([[1.0, 1.0], [0.0, 1.0]]), 1.0, np.array([[1.0, -1.0], [0.0, 1.0]])),
        (np.array([[1.0, -4.0], [1.0, 1.0]]), 5.0, np.array([[0.2, 0.8], [-0.2, 0.2]])),
    ]
    for a, det, inv in cases:
        assert not fne(O.determinant(a), det)
        assert not fne(O.inverse(a).ravel(), inv.ravel())


def test_solve():
    """test_solve.F90:18-39."""
    rhs = np.array([2.0, 3.0, 4.0])
    assert not fne(O.solve(np.eye(3), rhs), rhs)
    a = np.array([[1.0, 2.0, 3.0], [0.5, 0.25, 0.0], [4.1, 0.1, 4.0]])
    x1 = O.inverse(a) @ rhs
    x2 = O.solve(a, rhs)
    assert np.allclose(x1, x2, rtol=1e-14, atol=0)


def _one_layer_model(ii, dt):
    cfg = dict(ii=ii, jj=ii, layers=1, dt=dt, beta=[0.0], h=[1.0], s1=[0.0], s2=[0.0], ss=[0.0],
               m2z=[[1.0]], z2m=[[1.0]], viscosity=0.0, visc_bot=0.0, bc_type=O.BC_FREE_SLIP, alpha=0.0)
    return O.Model(cfg)


def test_cabaret_cfl():
    """test_cabaret_cfl.F90:17-36 (65 x 65, one layer)."""
    ii = 65
    for dt, scale in ((1.0, 1.0), (2.0, 2.0)):
        m = _one_layer_model(ii, dt)
        ui = np.ones(m.shape_of("ui"), order="F")
        uj = np.zeros(m.shape_of("uj"), order="F")
        m.set("ui", ui)
        m.set("uj", uj)
        assert not fne(m.cfl(), 1.0 * scale)
        m.set("uj", np.full(m.shape_of("uj"), 2.0, order="F"))
        assert not fne(m.cfl(), 2.0 * scale)
        ui[9, 9, 0] = 10.0
        m.set("ui", ui)
        assert not fne(m.cfl(), 10.0 * scale)
        uj = np.full(m.shape_of("uj"), 2.0, order="F")
        uj[9, 9, 0] = 20.0
        m.set("uj", uj)
        assert not fne(m.cfl(), 20.0 * scale)
