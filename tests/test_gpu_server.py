"""The continuously batched server (pq_server_*): every run's result is
bit-identical to the same run alone (pq_init_perturb + pq_step), whatever it
was batched with and however the budget staged it."""
import numpy as np
import pytest

import pequod_b200 as pq

pytestmark = pytest.mark.gpu


def cfg_of(ii, layers, precision=pq.PREC_FP64, dt=1800.0):
    H = {1: (1.0e5,), 2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5),
         5: (2.5e4, 5.0e4, 7.5e4, 1.0e5, 1.5e5)}[layers]
    gp = {1: (), 2: (1.5,), 3: (1.5, 0.75), 5: (1.5, 0.75, 0.375, 0.1875)}[layers]
    p = pq.double_gyre_physical(ii, layers=layers, dt=dt, dx=3.84e8 / (ii - 1), H=H, gprime=gp,
                                precision=precision)
    return pq.Config.from_physical(p)


def ic_of(cfg, seed):
    return pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)


def alone(cfg, ic, n):
    m = pq.Model(cfg)
    m.init_perturb(ic)
    m.step(n)
    out = m.get("psi")[1:-1, 1:-1, :]
    m.close()
    return out


RUNS = [(65, 3, pq.PREC_FP64, 1, 7), (65, 3, pq.PREC_FP64, 2, 12), (129, 3, pq.PREC_FP64, 3, 5),
        (65, 5, pq.PREC_FP64, 4, 9), (129, 3, pq.PREC_MIXED, 5, 6), (33, 1, pq.PREC_FP64, 6, 3),
        (65, 3, pq.PREC_FP64, 7, 1)]


def test_server_mix_equals_alone():
    srv = pq.Server(8 << 30)
    ids = []
    for ii, L, prec, seed, n in RUNS:
        cfg = cfg_of(ii, L, prec)
        ids.append((srv.submit(cfg, ic_of(cfg, seed), n), cfg, seed, n))
    srv.run_until_done(max_steps=4)
    assert srv.launches() > 0
    for rid, cfg, seed, n in ids:
        assert srv.status(rid) == 2
        psi, (t0, t1, t2) = srv.collect(rid)
        assert t0 <= t1 <= t2
        assert np.array_equal(psi, alone(cfg, ic_of(cfg, seed), n)), (cfg.ii, cfg.layers, n)
        assert srv.status(rid) == -1
    srv.close()


def test_server_persistent_sweeps_equal_alone():
    """Runs above 700 rows take the persistent CABARET sweeps: in the server's
    merged launch each run's CTAs claim only that run's sweeps, so every
    result is still bit-identical to the run alone (two 1025 x 1025 runs
    of each form, different step counts)."""
    srv = pq.Server(16 << 30)
    ids = []
    for prec, seed, n in ((pq.PREC_MIXED, 21, 3), (pq.PREC_MIXED, 22, 5), (pq.PREC_FP64, 23, 4),
                          (pq.PREC_FP64, 24, 2)):
        cfg = cfg_of(1025, 3, prec)
        ids.append((srv.submit(cfg, ic_of(cfg, seed), n), cfg, seed, n))
    srv.run_until_done(max_steps=2)
    for rid, cfg, seed, n in ids:
        assert srv.status(rid) == 2
        psi, _ = srv.collect(rid)
        assert np.array_equal(psi, alone(cfg, ic_of(cfg, seed), n)), (cfg.ii, n)
    srv.close()


def test_server_budget_staging_and_pool():
    cfg = cfg_of(65, 3)
    probe = pq.Model(cfg)
    one = probe.device_bytes()
    probe.close()
    # Room for a single context: the runs go through one at a time, reusing it.
    srv = pq.Server(int(one * 1.5))
    rids = [srv.submit(cfg, ic_of(cfg, 10 + k), 4 + k) for k in range(3)]
    a, q = srv.poll(2)
    assert a == 1 and q == 2
    srv.run_until_done(max_steps=2)
    held = srv.device_bytes()
    assert 0 < held <= int(one * 1.5)
    for k, rid in enumerate(rids):
        psi, _ = srv.collect(rid)
        assert np.array_equal(psi, alone(cfg, ic_of(cfg, 10 + k), 4 + k))
    with pytest.raises(pq.PQError) as e:
        srv.submit(cfg_of(513, 5), np.zeros((513, 513, 5)), 1)
    assert e.value.code == pq.PQ_ERR_BUDGET
    srv.close()


def test_server_isolates_faulted_runs():
    """Faults injected from the host stay with their run: a NaN in one
    run's initial PV (fails at admission, where the initial inversion's psiC
    is NaN), a run whose huge initial PV overflows to NaN a few steps in
    (fails mid-run, evicted after the round that raised it), and an invalid
    grid (ii - 1 not a power of two: admission fails).  Each reports its own
    error; every other run, batched with them in the same shape groups,
    finishes bit-identical to its run alone."""
    srv = pq.Server(8 << 30)
    cfg = cfg_of(65, 3)
    good = []
    for seed, n in ((21, 9), (22, 14), (23, 6)):
        good.append((srv.submit(cfg, ic_of(cfg, seed), n), seed, n))
    nan_ic = ic_of(cfg, 24)
    nan_ic[30, 31, 1] = np.nan
    r_nan = srv.submit(cfg, nan_ic, 10)
    r_blow = srv.submit(cfg, ic_of(cfg, 25) * 1e200, 40)
    bad = cfg_of(65, 3)
    bad.desc.ii = 60
    r_bad = srv.submit(bad, np.zeros((60, 65, 3)), 5)
    mixed = cfg_of(129, 3, pq.PREC_MIXED)
    good_mixed = (srv.submit(mixed, ic_of(mixed, 26), 7), 26, 7)
    srv.run_until_done(max_steps=2)
    for rid, code in ((r_nan, pq.PQ_ERR_NAN), (r_blow, pq.PQ_ERR_NAN), (r_bad, pq.PQ_ERR_ARG)):
        assert srv.status(rid) == 3, rid
        with pytest.raises(pq.PQError) as e:
            srv.collect(rid)
        assert e.value.code == code, (rid, e.value)
        assert srv.status(rid) == -1
    for rid, seed, n in good:
        assert srv.status(rid) == 2
        psi, _ = srv.collect(rid)
        assert np.array_equal(psi, alone(cfg, ic_of(cfg, seed), n))
    rid, seed, n = good_mixed
    psi, _ = srv.collect(rid)
    assert np.array_equal(psi, alone(mixed, ic_of(mixed, seed), n))
    # The failed runs' contexts were destroyed, not pooled: only the good
    # configurations' contexts are held.
    assert srv.device_bytes() <= 4 * pq.Model(cfg).device_bytes() + 2 * pq.Model(mixed).device_bytes()
    srv.close()
