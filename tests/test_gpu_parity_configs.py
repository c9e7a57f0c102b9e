"""GPU parity on the benchmarked configurations, against the oracle.

The oracle sets each configuration up by itself (oracle.setup_double_gyre,
its own restatement of qg3.F90:150-307), so the GPU path and its checker
share nothing but the physical parameters and the seeded initial condition.

Tolerances (plain FP64 form): relative L2 <= 1e-12 for a step from the
same inputs and along the first ten steps of a trajectory, <= 1e-9 after
100 steps, on the state fields and the energy diagnostics; the mixed form
<= 1e-6 on psi against the FP64 oracle.
"""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O
from pequod_b200.workloads import double_gyre

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12
TOL_100 = 1e-9
TOL_MIXED = 1e-6
STATE = ["psi", "zeta", "zeta_old", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res", "res_beta"]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def start(cfg, seed):
    ic = O.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    g = pq.Model(cfg)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    return g, o


def errors(g, o, fields):
    return {f: rel_l2(g.get(f), o.get(f)) for f in fields}


def energy_errors(g, o):
    ek_g, ep_g = g.energy()
    ek_o, ep_o = o.energy()
    return rel_l2(ek_g, ek_o), abs(ep_g - ep_o) / abs(ep_o)


def trajectory(cfg, seed, each, total, fields=("psi", "zeta"), energy_each=False, tol=TOL_STEP):
    """Step GPU and oracle side by side; every one of the first `each` steps
    within `tol`; returns the pair after `total` steps."""
    g, o = start(cfg, seed)
    for s in range(each):
        g.step(1)
        o.step(1)
        e = errors(g, o, fields)
        assert max(e.values()) <= tol, (s + 1, e)
        if energy_each:
            ek, ep = energy_errors(g, o)
            assert ek <= tol and ep <= tol, (s + 1, ek, ep)
    if total > each:
        g.step(total - each)
        o.step(total - each)
    return g, o


def test_513_single_steps_from_oracle_state():
    """513 x 513 x 3, dt = 900 s: after the oracle has run, the GPU takes the
    oracle's whole state and both advance one step from the same inputs; the
    step's result is within 1e-12, five times along the trajectory."""
    cfg = double_gyre(513, 3, 900.0)
    g, o = start(cfg, seed=11)
    o.step(20)
    for k in range(5):
        for f in STATE + ["rel"]:
            g.set(f, o.get(f))
        g.step(1)
        o.step(1)
        e = errors(g, o, STATE)
        assert max(e.values()) <= TOL_STEP, (k, e)
        ek, ep = energy_errors(g, o)
        assert ek <= TOL_STEP and ep <= TOL_STEP, (k, ek, ep)
        o.step(7)


def test_513_hundred_steps():
    """513 x 513 x 3, dt = 900 s (the benchmarked single-run configuration):
    each of the first ten steps within 1e-12 on psi and zeta, every state
    field, the energies, the CFL number and the model time within 1e-9 after
    100 steps."""
    cfg = double_gyre(513, 3, 900.0)
    g, o = trajectory(cfg, seed=12, each=10, total=100)
    e = errors(g, o, STATE + ["rel"])
    assert max(e.values()) <= TOL_100, e
    ek, ep = energy_errors(g, o)
    assert ek <= TOL_100 and ep <= TOL_100, (ek, ep)
    assert abs(g.cfl() - o.cfl()) <= TOL_100 * o.cfl()
    assert abs(g.scalars()["model_time"] - o.scalars()["model_time"]) <= 1e-12 * o.scalars()["model_time"]


def test_1025_ten_steps():
    """1025 x 1025 x 3, dt = 900 s (the target configuration): ten steps, each
    within 1e-12 on psi and zeta; all state fields within 1e-12 at the end."""
    cfg = double_gyre(1025, 3, 900.0)
    g, o = trajectory(cfg, seed=13, each=10, total=10)
    e = errors(g, o, STATE + ["rel"])
    assert max(e.values()) <= TOL_STEP, e


def test_2049x5_ten_steps_with_energy():
    """2049 x 2049 x 5, dt = 300 s (the large eddy-resolving configuration):
    ten steps, each within 1e-12 on psi and zeta with the energies compared
    at every step."""
    cfg = double_gyre(2049, 5, 300.0)
    g, o = trajectory(cfg, seed=14, each=10, total=10, energy_each=True)
    e = errors(g, o, STATE)
    assert max(e.values()) <= TOL_STEP, e


def test_mixed_513_five_hundred_steps_vs_oracle():
    """The mixed-precision form at 513 x 513 x 3, dt = 900 s: psi within 1e-6
    of the FP64 oracle after 500 steps (and at every 100th step on the way),
    with the energies of the same order."""
    cfg = double_gyre(513, 3, 900.0, precision=pq.PREC_MIXED)
    g, o = start(cfg, seed=15)
    for k in range(5):
        g.step(100)
        o.step(100)
        e = rel_l2(g.get("psi"), o.get("psi"))
        assert e <= TOL_MIXED, ((k + 1) * 100, e)
    ek, ep = energy_errors(g, o)
    assert ek <= TOL_MIXED and ep <= TOL_MIXED, (ek, ep)


def test_mixed_1025_hundred_steps_vs_oracle():
    """The mixed-precision form at the target size 1025 x 1025 x 3: psi within
    1e-6 of the FP64 oracle after 100 steps."""
    cfg = double_gyre(1025, 3, 900.0, precision=pq.PREC_MIXED)
    g, o = start(cfg, seed=16)
    g.step(100)
    o.step(100)
    e = rel_l2(g.get("psi"), o.get("psi"))
    assert e <= TOL_MIXED, e


def test_2049x5_energy_every_ten_steps():
    """The large eddy-resolving run's diagnostics cadence: 30 steps at
    2049 x 2049 x 5, dt = 300 s, the energies (qg3.F90:744, energy of
    qg3p_diagnostics.F90:778-863) and the CFL number taken every 10 steps
    between graph-launched steps, each within 1e-12 of the oracle's."""
    cfg = double_gyre(2049, 5, 300.0)
    g, o = start(cfg, seed=17)
    for k in range(3):
        g.step(10)
        o.step(10)
        ek, ep = energy_errors(g, o)
        assert ek <= TOL_STEP and ep <= TOL_STEP, ((k + 1) * 10, ek, ep)
        assert abs(g.cfl() - o.cfl()) <= TOL_STEP * o.cfl()
    e = errors(g, o, ["psi", "zeta"])
    assert max(e.values()) <= TOL_STEP, e
