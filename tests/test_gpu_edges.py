"""Edge cases of the newer entry points: the smallest grids, single-member
ensembles, the caller's time step in the mixed form, batches without FP32
layers, the Dirichlet routines on a one-layer context with device arrays."""
import ctypes as C

import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O
from pequod_b200.workloads import double_gyre

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def helm_cfg(ii, jj, ss, periodic=False):
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


@pytest.mark.parametrize("ii,jj,periodic", [(5, 5, False), (5, 7, True), (9, 6, False)])
def test_laplace_bc_smallest_grids(ii, jj, periodic):
    """The lifting ring degenerates on the smallest grids (one interior row
    or column): the corner subtractions still follow the reference's order."""
    m = pq.Model(helm_cfg(ii, jj, [0.0], periodic=periodic))
    rng = np.random.default_rng(ii * jj)
    f = np.asfortranarray(rng.standard_normal((ii, jj)))
    bd = 0.25 if periodic else None
    assert np.array_equal(m.add_laplace_bc_rhs(f, 1.5, bd),
                          O.add_laplace_bc_rhs(f, 1.5, bd, periodic_j=periodic))
    assert np.array_equal(m.apply_dirichlet_bc(f, -0.5, bd),
                          O.apply_dirichlet_bc(f, -0.5, bd, periodic_j=periodic))
    r = m.laplace_bc_rhs(2.0)
    assert np.array_equal(r, O.add_laplace_bc_rhs(np.zeros((ii, jj), order="F"), 2.0, periodic_j=periodic))


def test_dirichlet_device_array_one_layer():
    import torch

    ii, jj = 33, 20
    m = pq.Model(helm_cfg(ii, jj, [0.0]))
    f = np.asfortranarray(np.random.default_rng(3).standard_normal((ii, jj)))
    dev = torch.from_numpy(np.ascontiguousarray(f.ravel(order="F"))).cuda()
    torch.cuda.synchronize()
    bc = np.ascontiguousarray([0.75])
    rc = pq.lib().pq_apply_dirichlet_bc(m.ctx, C.cast(dev.data_ptr(), pq._dp), 1, pq._p(bc), None, 1,
                                        pq.PTR_DEVICE)
    assert rc == pq.PQ_OK
    m.sync()
    got = dev.cpu().numpy().reshape((ii, jj), order="F")
    assert np.array_equal(got, O.apply_dirichlet_bc(f, 0.75))


def test_single_member_ensemble_equals_run_alone():
    cfg = double_gyre(65, 3, 900.0)
    ic = O.make_ic(65, 65, 3, seed=51, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    e = pq.Ensemble(cfg, 1)
    e.init(0, ic)
    e.step(7)
    m = pq.Model(cfg)
    m.init_perturb(ic)
    m.step(7)
    assert rel_l2(e.members[0].get("psi"), m.get("psi")) <= 1e-13
    assert e.members[0].scalars()["model_time"] == m.scalars()["model_time"]
    e.close()


def test_cabaret_step_mixed_matches_pq_step():
    """The caller's constant dt through pq_cabaret_step gives the same
    trajectory as pq_step in the mixed form (within the mixed tolerance: the
    two paths differ only in where the predictor is computed)."""
    cfg = double_gyre(129, 3, 1800.0, precision=pq.PREC_MIXED)
    ic = O.make_ic(129, 129, 3, seed=52, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    a, b = pq.Model(cfg), pq.Model(cfg)
    a.init_perturb(ic)
    b.init_perturb(ic)
    dt = cfg.desc.dt
    for _ in range(10):
        a.cabaret_step(dt, 0.5, 0.5)
    b.step(10)
    assert rel_l2(a.get("psi"), b.get("psi")) <= 1e-6


def test_mixed_batch_without_fp32_layers():
    """One-layer members have no FP32 layers: the mixed batch solves them in
    FP64 (equal to the oracle to 1e-12) and none takes the tensor DST."""
    shapes = [(65, 65, 1), (129, 33, 1), (257, 129, 1)]
    rng = np.random.default_rng(9)
    ss = [np.array([0.0]), np.array([0.5]), np.array([3.0])]
    rhs = [np.asfortranarray(rng.standard_normal(s)) for s in shapes]
    b = pq.Batch(shapes, ss, precision=pq.PREC_MIXED, dst_algo=pq.DST_TENSOR)
    out = b.helm(rhs)
    for k, (ii, jj, L) in enumerate(shapes):
        ref = O.Helm(ii, jj, L, list(ss[k]))(rhs[k])
        assert rel_l2(out[k], ref) <= 1e-12
        assert b.member_dst_algo(k) == pq.DST_BUTTERFLY
    b.close()
