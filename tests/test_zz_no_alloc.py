"""pq_energy_noalloc: the energy diagnostics for callers that cannot allocate.

A host driver that is capturing a CUDA graph, or whose device memory is all
reserved by an HBM budget, cannot let the library call cudaMalloc.  This
entry point takes the caller's own device array of psi and a caller-owned
output buffer and keeps its reduction scratch in a fixed array inside the
library.  Its results must equal pq_energy's (the context-based entry point)
on the same psi, within the FP64 tolerance the other tests use, on two calls
in a row (the shared scratch keeps the previous call's contents).

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import pequod_b200 as pq

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _setup():
    import torch

    cfg = pq.Config.from_physical(pq.double_gyre_physical(65, dx=3.84e8 / 64))
    m = pq.Model(cfg)
    ic = pq.make_ic(65, 65, 3, seed=11, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    m.init_perturb(ic)
    m.step(5)
    psi = m.sdata("psi")  # (ii, jj, L), Fortran order
    ekin, epot = m.energy()
    return torch, cfg, m, psi, np.append(ekin, epot)


def _call(psi_dev, ii, jj, L, ld, h, s2, out_dev):
    rc = pq.lib().pq_energy_noalloc(C.c_void_p(psi_dev), ii, jj, L, ld, pq._p(h), pq._p(s2), C.c_void_p(out_dev),
                                    None)
    assert rc == pq.PQ_OK, rc


def test_noalloc_energy_matches_context_energy_twice():
    torch, cfg, m, psi, ref = _setup()
    ii, jj, L = psi.shape
    h = np.ascontiguousarray(cfg.desc.h[:L])
    s2 = np.ascontiguousarray(cfg.desc.s2[:L])
    dev = torch.device("cuda", 0)
    psi_dev = torch.from_numpy(psi.ravel(order="F").copy()).to(dev)
    out = torch.full((L + 1,), float("nan"), dtype=torch.float64, device=dev)
    for _ in range(2):
        out.fill_(float("nan"))
        _call(psi_dev.data_ptr(), ii, jj, L, ii, h, s2, out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= TOL * np.abs(ref)), (got, ref)
    # A padded leading dimension gives the same answer.
    ld = ii + 7
    pad = np.zeros((ld, jj, L), order="F")
    pad[:ii] = psi
    pad_dev = torch.from_numpy(pad.ravel(order="F").copy()).to(dev)
    _call(pad_dev.data_ptr(), ii, jj, L, ld, h, s2, out.data_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.all(np.abs(got - ref) <= TOL * np.abs(ref)), (got, ref)
    m.close()


def test_noalloc_energy_rejects_oversized_grids():
    h = np.ones(3)
    s2 = np.ones(3)
    rc = pq.lib().pq_energy_noalloc(C.c_void_p(16), 5, pq_max_jj() + 1, 3, 5, pq._p(h), pq._p(s2), C.c_void_p(16),
                                    None)
    assert rc == pq.PQ_ERR_ARG
    rc = pq.lib().pq_energy_noalloc(C.c_void_p(16), 5, 5, pq.MAX_LAYERS + 1, 5, pq._p(h), pq._p(s2),
                                    C.c_void_p(16), None)
    assert rc == pq.PQ_ERR_ARG


def pq_max_jj():
    return 4097
