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
