"""The C-ABI library loads and exports every symbol include/*.h declares
(no device calls), and the host-side set-up matches the oracle."""
import glob
import os
import re

import numpy as np

import pequod_b200 as pq
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        for m in re.finditer(r"PQ_API\s+[\w\s\*]+?\b(pq_\w+)\s*\(", open(h).read()):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 19
    L = pq.lib()
    for n in sorted(names):
        assert hasattr(L, n), n
    # The Python mirror binds exactly the declared ABI.
    assert set(pq.SIGNATURES) >= names


def test_stratification_matches_oracle():
    H = [3.0e4, 7.0e4, 3.0e5]
    g = [1.5, 0.75]
    f0 = 9.4e-5
    s2 = [f0 * f0 / (g[k] * H[k]) for k in range(2)]
    s1 = [f0 * f0 / (g[k] * H[k + 1]) for k in range(2)]
    l_scale = 30.0e5
    d = pq.ModelDesc()
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    rc = pq.lib().pq_stratification(d, 3, pq._p(arr(H)), pq._p(arr(s1)), pq._p(arr(s2)), l_scale)
    assert rc == 0
    st = O.strat_from_parameters(H, s1, s2, l_scale)
    ss = np.array(d.ss[:3])
    assert ss[0] == 0.0
    assert np.allclose(np.sort(ss), np.sort(st["ss"]), rtol=1e-14, atol=0)
    m2z = np.array(d.m2z[:9]).reshape((3, 3), order="F")
    z2m = np.array(d.z2m[:9]).reshape((3, 3), order="F")
    assert np.allclose(m2z @ z2m, np.eye(3), atol=1e-14)
    assert np.allclose(m2z[:, 0], 1.0)
    # The modal split diagonalises S: S m2z = m2z diag(-ss).
    S = np.zeros((3, 3))
    s1s, s2s = np.array(d.s1[:3]), np.array(d.s2[:3])
    S[0, 0], S[0, 1] = -s2s[0], s2s[0]
    S[1, 0], S[1, 1], S[1, 2] = s1s[1], -(s1s[1] + s2s[1]), s2s[1]
    S[2, 1], S[2, 2] = s1s[2], -s1s[2]
    assert np.allclose(S @ m2z, m2z @ np.diag(-ss), rtol=0, atol=1e-12 * np.abs(S).max())


def test_double_gyre_setup():
    """Non-dimensionalisation of qg3.F90:152-168 for the 129 x 129 double gyre."""
    cfg = pq.Config.from_physical(pq.double_gyre_physical(129))
    d = cfg.desc
    l_scale = 30.0e5
    t_scale = l_scale / 1.0
    assert cfg.t_scale == t_scale
    assert np.isclose(d.dt, 1800.0 / t_scale, rtol=1e-15)
    assert np.isclose(d.beta[0], 1.8e-13 * l_scale ** 2, rtol=1e-15)
    assert np.isclose(d.viscosity, 1.0e6 / l_scale, rtol=1e-15)
    assert np.isclose(d.visc_bot, 1.0e-7 * l_scale, rtol=1e-15)
    assert np.isclose(d.alpha, l_scale / 120.0e5, rtol=1e-15)
    assert d.bc_type == pq.BC_PARTIAL_SLIP
    # Symmetric wind (wind_asym = 1): 2 pi tau sin(2 pi y), y = 0.5 - (i-1)/(ii-1).
    tau = 0.8 / 128.0 / (3.0e4 / l_scale)
    i = np.arange(1, 130)
    y = 0.5 - (i - 1) / 128.0
    assert np.allclose(cfg.wind[:, 5], tau * 2 * np.pi * np.sin(2 * np.pi * y), rtol=0, atol=1e-15 * tau * 7)


def test_make_ic_is_seeded():
    a = pq.make_ic(33, 17, 2, seed=5, amplitude=2.0, sigma=3.0)
    b = pq.make_ic(33, 17, 2, seed=5, amplitude=2.0, sigma=3.0)
    c = pq.make_ic(33, 17, 2, seed=6, amplitude=2.0, sigma=3.0)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    w = pq.make_ic(64, 64, 1, seed=1, amplitude=1.0, sigma=0.0)
    assert abs(w.mean()) < 0.05 and abs(w.std() - 1.0) < 0.05
