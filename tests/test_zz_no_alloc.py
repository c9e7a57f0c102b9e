"""pq_energy_noalloc: the energy diagnostics for callers that cannot allocate.

A host driver whose device memory is reserved up front (by an HBM budget,
or by a caching allocator that owns the whole device) cannot let the library
call cudaMalloc, and a driver that keeps its streams pipelined cannot afford
the device-wide synchronisation cudaMalloc / cudaFree may cause.  This entry
point takes the caller's own device array of psi and a caller-owned output
buffer and keeps its reduction scratch in a fixed array inside the library.
Its results must equal pq_energy's (the context-based entry point) on the
same psi, within the FP64 tolerance the other tests use, on two calls in a
row (the shared scratch keeps the previous call's contents), and the
oracle's energy() of the same field.

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _model(periodic):
    jj = 64 if periodic else 65
    p = pq.double_gyre_physical(65, jj, dx=3.84e8 / 64)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = int(periodic)
    m = pq.Model(cfg)
    ic = pq.make_ic(65, jj, 3, seed=11, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    m.init_perturb(ic)
    m.step(5)
    ekin, epot = m.energy()
    return cfg, m, m.sdata("psi"), np.append(ekin, epot)


def _call(psi_dev, ii, jj, L, ld, periodic, h, s2, out_dev):
    return pq.lib().pq_energy_noalloc(C.c_void_p(psi_dev), ii, jj, L, ld, int(periodic), pq._p(h), pq._p(s2),
                                      C.c_void_p(out_dev), None)


def _oracle_energy(psi, h, s2, periodic):
    """The oracle's energy() on the reference's full data array (with the
    channel's periodic halo rows filled)."""
    ii, jj, L = psi.shape
    full = np.zeros((ii + 2, jj + 2, L), order="F")
    full[1:-1, 1:-1] = psi
    if periodic:
        full[1:-1, 0] = psi[:, -1]
        full[1:-1, -1] = psi[:, 0]
    ek, ep = O.energy(full, h, s2, periodic_j=periodic)
    return np.append(ek, ep)


def _close(got, ref, tol=TOL):
    return bool(np.all(np.abs(got - ref) <= tol * np.abs(ref)))


@pytest.mark.parametrize("periodic", [False, True])
def test_noalloc_energy_matches_context_energy_twice(periodic):
    import torch

    cfg, m, psi, ref = _model(periodic)
    ii, jj, L = psi.shape
    h = np.ascontiguousarray(cfg.desc.h[:L])
    s2 = np.ascontiguousarray(cfg.desc.s2[:L])
    oref = _oracle_energy(psi, h, s2, periodic)
    assert _close(ref, oref), (ref, oref)
    dev = torch.device("cuda", 0)
    psi_dev = torch.from_numpy(psi.ravel(order="F").copy()).to(dev)
    out = torch.full((L + 1,), float("nan"), dtype=torch.float64, device=dev)
    for _ in range(2):
        out.fill_(float("nan"))
        assert _call(psi_dev.data_ptr(), ii, jj, L, ii, periodic, h, s2, out.data_ptr()) == pq.PQ_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert _close(got, ref), (got, ref)
        assert _close(got, oref), (got, oref)
    # A padded leading dimension gives the same answer.
    ld = ii + 7
    pad = np.zeros((ld, jj, L), order="F")
    pad[:ii] = psi
    pad_dev = torch.from_numpy(pad.ravel(order="F").copy()).to(dev)
    assert _call(pad_dev.data_ptr(), ii, jj, L, ld, periodic, h, s2, out.data_ptr()) == pq.PQ_OK
    torch.cuda.synchronize()
    assert _close(out.cpu().numpy(), ref)
    m.close()


def test_noalloc_energy_at_the_size_limit():
    """The largest jj accepted (a narrow grid keeps it cheap) against the
    oracle, closed basin and channel; one row more is refused."""
    import torch

    ii, jj, L = 9, pq.NOALLOC_MAX_JJ, 2
    rng = np.random.default_rng(4097)
    psi = np.asfortranarray(rng.standard_normal((ii, jj, L)))
    h = np.ascontiguousarray([0.3, 0.7])
    s2 = np.ascontiguousarray([2.0, 0.0])
    dev = torch.device("cuda", 0)
    psi_dev = torch.from_numpy(psi.ravel(order="F").copy()).to(dev)
    out = torch.zeros((L + 1,), dtype=torch.float64, device=dev)
    for periodic in (False, True):
        assert _call(psi_dev.data_ptr(), ii, jj, L, ii, periodic, h, s2, out.data_ptr()) == pq.PQ_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = _oracle_energy(psi, h, s2, periodic)
        assert _close(got, ref, 1e-12), (periodic, got, ref)
    assert _call(psi_dev.data_ptr(), ii, jj + 1, L, ii, False, h, s2, out.data_ptr()) == pq.PQ_ERR_ARG


def test_noalloc_energy_rejects_bad_arguments():
    h = np.ones(3)
    s2 = np.ones(3)
    assert _call(16, 5, pq.NOALLOC_MAX_JJ + 1, 3, 5, False, h, s2, 16) == pq.PQ_ERR_ARG
    assert _call(16, 5, 5, pq.MAX_LAYERS + 1, 5, False, h, s2, 16) == pq.PQ_ERR_ARG
    assert _call(16, 5, 5, 3, 4, False, h, s2, 16) == pq.PQ_ERR_ARG  # ld < ii
    assert _call(16, 5, 5, 3, 5, 2, h, s2, 16) == pq.PQ_ERR_ARG  # periodic_j not 0 / 1
