"""Batched Helmholtz solves (pq_batch_*): every member of a mixed batch
matches the oracle's helm (relative L2 <= 1e-12) and is bit-identical to the
same problem solved alone through pq_helm."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(33, 20, 1), (65, 33, 3), (129, 129, 2), (33, 65, 5), (257, 129, 3), (65, 65, 3), (129, 33, 4),
          (33, 20, 2), (513, 65, 1), (65, 257, 2)]


def rel_l2(a, b):
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def helm_cfg(ii, jj, ss):
    L = len(ss)
    d = pq.ModelDesc()
    d.ii, d.jj, d.layers = ii, jj, L
    d.limiter, d.bc_type, d.dt = 1, pq.BC_FREE_SLIP, 1.0
    for k in range(L):
        d.ss[k] = ss[k]
        d.h[k] = 1.0
        for m in range(L):
            d.m2z[k + L * m] = 1.0 if k == m else 0.0
            d.z2m[k + L * m] = 1.0 if k == m else 0.0
    return pq.Config(d, None, 1.0)


def problem(seed):
    rng = np.random.default_rng(seed)
    ss = [np.where(rng.random(s[2]) < 0.3, 0.0, rng.uniform(0.1, 20.0, s[2])) for s in SHAPES]
    rhs = [np.asfortranarray(rng.standard_normal(s)) for s in SHAPES]
    return ss, rhs


def test_batch_matches_oracle_and_alone():
    ss, rhs = problem(5)
    b = pq.Batch(SHAPES, ss)
    out = b.helm(rhs)
    assert b.launch_count() > 0
    for k, (ii, jj, L) in enumerate(SHAPES):
        ref = O.Helm(ii, jj, L, list(ss[k]))(rhs[k])
        assert rel_l2(out[k], ref) <= 1e-12, (k, rel_l2(out[k], ref))
        alone = pq.Model(helm_cfg(ii, jj, list(ss[k]))).helm(rhs[k])
        assert np.array_equal(out[k], alone), k
    b.close()


def test_batch_device_resident_resolve():
    """Solving twice from device-resident right-hand sides (graph replay)."""
    ss, rhs = problem(6)
    b = pq.Batch(SHAPES, ss)
    for k, r in enumerate(rhs):
        b.set_rhs(k, r)
    b.solve_async()
    first = [b.get(k) for k in range(len(b))]
    for k, r in enumerate(rhs):
        b.set_rhs(k, r)
    b.solve_async()
    b.sync()
    second = [b.get(k) for k in range(len(b))]
    for a, c in zip(first, second):
        assert np.array_equal(a, c)
    b.close()


@pytest.mark.parametrize("algo", [pq.DST_BUTTERFLY, pq.DST_TENSOR, 0])
def test_batch_mixed_precision_variants(algo):
    """The mixed batch: each member's first layer (here ss = 0, the
    barotropic problem) stays FP64 and matches the oracle to 1e-12; the
    other layers are transformed in FP32 -- FP32 butterfly, tensor-core DST
    (three-term BF16 split) or whichever the autotuner timed faster per
    class -- and match the FP64 oracle to FP32 accuracy."""
    shapes = [(65, 65, 3), (129, 257, 2), (257, 129, 4), (513, 513, 3), (33, 65, 2), (129, 129, 1),
              (1025, 129, 2)]
    rng = np.random.default_rng(8)
    ss = [np.concatenate([[0.0], rng.uniform(0.3, 20.0, s[2] - 1)]) for s in shapes]
    rhs = [np.asfortranarray(rng.standard_normal(s)) for s in shapes]
    b = pq.Batch(shapes, ss, precision=pq.PREC_MIXED, dst_algo=algo)
    out = b.helm(rhs)
    for k, (ii, jj, L) in enumerate(shapes):
        ref = O.Helm(ii, jj, L, list(ss[k]))(rhs[k])
        assert rel_l2(out[k][:, :, 0], ref[:, :, 0]) <= 1e-12, (k, "fp64 layer")
        for l in range(1, L):
            e = rel_l2(out[k][:, :, l], ref[:, :, l])
            assert e <= 1e-5, (k, l, e)
        used = b.member_dst_algo(k)
        if algo == pq.DST_TENSOR and L > 1 and ii >= 65:
            assert used == pq.DST_TENSOR
        elif algo == pq.DST_BUTTERFLY or L == 1 or ii < 65:
            assert used == pq.DST_BUTTERFLY
    b.close()
