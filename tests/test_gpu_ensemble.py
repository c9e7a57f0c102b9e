"""Ensembles (pq_ensemble_*): many runs of one configuration stepped with one
launch per kernel over all members.  Each member's trajectory is the run
alone's (the kernels compute every member independently) and the oracle's."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O
from pequod_b200.workloads import double_gyre

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def ic(cfg, seed):
    return O.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)


@pytest.mark.parametrize("ii,layers,prec,algo", [(129, 3, pq.PREC_FP64, 1), (257, 5, pq.PREC_FP64, 1),
                                                 (257, 3, pq.PREC_MIXED, 1), (257, 3, pq.PREC_MIXED, 2)])
def test_ensemble_members_equal_runs_alone(ii, layers, prec, algo):
    cfg = double_gyre(ii, layers, 900.0, precision=prec)
    n = 4
    ens = pq.Ensemble(cfg, n)
    if prec == pq.PREC_MIXED:
        ens.set_dst_algo(algo)
    for k in range(n):
        ens.init(k, ic(cfg, 40 + k))
    for chunk in (1, 2, 3, 6):  # odd and even counts, first step alone
        ens.step(chunk)
    tol = 1e-12 if prec == pq.PREC_FP64 else 1e-6
    for k in range(n):
        m = pq.Model(cfg)
        if prec == pq.PREC_MIXED:
            m.set_tuning(dst_algo=algo)
        m.init_perturb(ic(cfg, 40 + k))
        m.step(12)
        for f in ("psi", "zeta", "res", "ui"):
            a, b = ens.members[k].get(f), m.get(f)
            assert rel_l2(a, b) <= (1e-13 if prec == pq.PREC_FP64 else 1e-12), (k, f, rel_l2(a, b))
        assert ens.members[k].scalars()["model_time"] == m.scalars()["model_time"]
        m.close()
    # against the oracle
    o = O.Model(O.cfg_from(cfg))
    o.init(ic(cfg, 41))
    o.step(12)
    assert rel_l2(ens.members[1].get("psi"), o.get("psi")) <= tol
    ek, ep = ens.members[1].energy()
    ek_o, ep_o = o.energy()
    assert rel_l2(ek, ek_o) <= tol * 10
    ens.close()


def test_ensemble_rules():
    cfg = double_gyre(65, 3, 900.0)
    ens = pq.Ensemble(cfg, 2)
    ens.init(0, ic(cfg, 1))
    with pytest.raises(pq.PQError):
        ens.step(1)  # member 1 not initialised
    with pytest.raises(pq.PQError) as e:
        ens.init(1, np.full((65, 65, 3), np.nan))  # the reference aborts on the NaN psiC
    assert e.value.code == pq.PQ_ERR_NAN
    ens.close()
    bad = double_gyre(65, 3, 900.0, adapt_dt=1)
    with pytest.raises(pq.PQError):
        pq.Ensemble(bad, 2)


@pytest.mark.parametrize("prec,kernel", [(pq.PREC_FP64, 1), (pq.PREC_MIXED, 1), (pq.PREC_MIXED, 2)])
def test_ensemble_persistent_sweeps_equal_runs_alone(prec, kernel):
    """The CABARET step as persistent warp sweeps inside the merged launch
    (one and two columns per lane; 8-row bands at 257 x 257 give more
    sweeps than there are resident warps): each member's CTAs claim only
    that member's sweeps, from its own queue, so every member still steps
    exactly as it does alone."""
    cfg = double_gyre(257, 3, 900.0, precision=prec)
    n = 3
    ens = pq.Ensemble(cfg, n)
    for k in range(n):
        ens.members[k].set_tuning(cab_kernel=kernel, cab_band=8)
        ens.init(k, ic(cfg, 60 + k))
    ens.step(1)
    ens.step(4)
    for k in range(n):
        assert ens.members[k].get_tuning()["cab_kernel"] == kernel
        m = pq.Model(cfg)
        m.set_tuning(cab_kernel=kernel, cab_band=8)
        m.init_perturb(ic(cfg, 60 + k))
        m.step(5)
        for f in ("psi", "zeta", "res", "ui", "uj", "zeta_fi"):
            a, b = ens.members[k].get(f), m.get(f)
            assert rel_l2(a, b) <= (1e-13 if prec == pq.PREC_FP64 else 1e-12), (k, f, rel_l2(a, b))
        m.close()
    ens.close()
