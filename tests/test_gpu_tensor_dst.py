"""The tensor-core row DST of the mixed form (pq_tuning.dst_algo =
PQ_DST_TENSOR): the baroclinic modes' sine transforms as dense DST-matrix
products on the tensor cores (three-term BF16 split, FP32 accumulation),
the barotropic mode still the FP64 butterfly.  Held to the mixed form's
tolerance against the FP64 oracle (relative L2 <= 1e-6 on psi), and close
to the FP32 butterfly it replaces."""
import numpy as np
import pytest

import pequod_b200 as pq
from oracle import oracle as O
from pequod_b200.workloads import double_gyre

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def channel(ii, jj, layers=3, precision=pq.PREC_MIXED):
    H = {2: (1.0e5, 3.0e5), 3: (3.0e4, 7.0e4, 3.0e5)}[layers]
    gp = {2: (1.5,), 3: (1.5, 0.75)}[layers]
    p = pq.double_gyre_physical(ii, jj=jj, layers=layers, dt=1800.0, dx=3.84e8 / (ii - 1), H=H, gprime=gp,
                                precision=precision)
    cfg = pq.Config.from_physical(p)
    cfg.desc.periodic_j = 1
    return cfg


@pytest.mark.parametrize("ii,layers", [(65, 2), (129, 3), (257, 5), (513, 3), (1025, 3)])
def test_tensor_dst_pv_inversion_matches_oracle(ii, layers):
    cfg = double_gyre(ii, layers, 900.0, precision=pq.PREC_MIXED)
    rng = np.random.default_rng(ii + 11 * layers)
    zeta = np.asfortranarray(rng.standard_normal((ii, ii, layers)))
    g = pq.Model(cfg)
    g.set_tuning(dst_algo=pq.DST_TENSOR)
    assert g.get_tuning()["dst_algo"] == pq.DST_TENSOR
    psi_t = g.pv_inversion(zeta)
    g.set_tuning(dst_algo=pq.DST_BUTTERFLY)
    psi_b = g.pv_inversion(zeta)
    om = O.Model(O.cfg_from(cfg))
    zd = np.zeros((ii + 2, ii + 2, layers), order="F")
    zd[1:-1, 1:-1, :] = zeta
    ref = om.pv_inversion(zd)[1:-1, 1:-1, :]
    e_t, e_b = rel_l2(psi_t, ref), rel_l2(psi_b, ref)
    assert e_t <= TOL_MIXED, (e_t, e_b)
    assert rel_l2(psi_t, psi_b) <= TOL_MIXED
    # every layer, not only the norm of all of them
    for l in range(layers):
        assert rel_l2(psi_t[:, :, l], ref[:, :, l]) <= TOL_MIXED, l
    g.close()


def test_tensor_dst_channel_inversion_matches_oracle():
    cfg = channel(129, 96)
    rng = np.random.default_rng(5)
    zeta = np.asfortranarray(rng.standard_normal((129, 96, 3)))
    g = pq.Model(cfg)
    g.set_tuning(dst_algo=pq.DST_TENSOR)
    psi = g.pv_inversion(zeta)
    om = O.Model(O.cfg_from(cfg))
    zd = np.zeros((131, 98, 3), order="F")
    zd[1:-1, 1:-1, :] = zeta
    ref = om.pv_inversion(zd)[1:-1, 1:-1, :]
    assert rel_l2(psi, ref) <= TOL_MIXED


def test_tensor_dst_steps_match_oracle():
    """513 x 513 x 3 mixed with the tensor-core DST: psi within 1e-6 of the
    FP64 oracle after 200 steps (graph-captured steps, fused predictor)."""
    cfg = double_gyre(513, 3, 900.0, precision=pq.PREC_MIXED)
    ic = O.make_ic(513, 513, 3, seed=31, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    g = pq.Model(cfg)
    g.set_tuning(dst_algo=pq.DST_TENSOR)
    g.init_perturb(ic)
    o = O.Model(O.cfg_from(cfg))
    o.init(ic)
    for k in range(2):
        g.step(100)
        o.step(100)
        e = rel_l2(g.get("psi"), o.get("psi"))
        assert e <= TOL_MIXED, ((k + 1) * 100, e)


def test_autotune_keeps_the_state():
    """pq_autotune times both algorithms on the current state and leaves the
    state as it was: the trajectory afterwards is the one without it (up to
    the algorithms' difference, well inside the mixed tolerance)."""
    cfg = double_gyre(257, 3, 900.0, precision=pq.PREC_MIXED)
    ic = O.make_ic(257, 257, 3, seed=32, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    a, b = pq.Model(cfg), pq.Model(cfg)
    for m in (a, b):
        m.init_perturb(ic)
        m.step(3)
    psi0 = a.get("psi")
    sc0 = a.scalars()
    choice = a.autotune()
    assert choice in (pq.DST_BUTTERFLY, pq.DST_TENSOR)
    assert a.get_tuning()["dst_algo"] == choice
    assert np.array_equal(a.get("psi"), psi0)
    assert a.scalars() == sc0
    # cached: a second context of the same shape takes the decision
    c = pq.Model(cfg)
    assert c.autotune() == choice
    a.step(20)
    b.step(20)
    assert rel_l2(a.get("psi"), b.get("psi")) <= TOL_MIXED
    # FP64 contexts have only the butterfly
    f = pq.Model(double_gyre(129, 3, 900.0))
    assert f.autotune() == pq.DST_BUTTERFLY
    with pytest.raises(pq.PQError):
        f.set_tuning(dst_algo=pq.DST_TENSOR)
