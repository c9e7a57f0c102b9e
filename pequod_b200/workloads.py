"""Seeded synthetic workloads of the double-gyre benchmark.

The physics follows the reference's double-gyre configuration (qg3.F90:150-307
non-dimensionalisation, wind and beta; qg3p_params.F90 defaults): a basin of
3.84e8 cm (128 x 30 km) resolved by `ii` nodes, f0 = 9.4e-5 s^-1,
beta = 1.8e-13 cm^-1 s^-1, tau = 0.8 cm^2 s^-2, partial slip with alpha =
120 km, CABARET with the limiter.  Three layers use H = (300, 700, 3000) m and
g' = (1.5, 0.75) cm s^-2; five layers H = (250, 500, 750, 1000, 1500) m and
g'_k = 1.5 * 2^-k cm s^-2.  The initial condition is the seeded white-noise
vorticity smoothed by a 3-cell Gaussian (`make_ic`).

`python -m pequod_b200.workloads --size 513 --steps 6` runs the
initialisation and a few eagerly launched steps (one launch per kernel) and
prints each kernel's event-timed microseconds, the command the committed
kernel profiles were taken with; `--dst-algo 2` selects the tensor-core DST
of the mixed form, `--inversions N` runs N pv_inversions instead.
"""
from __future__ import annotations

import argparse

import numpy as np

import pequod_b200 as pq

BASIN_CM = 3.84e8
LAYERS = {
    1: ((1.0e5,), ()),
    2: ((1.0e5, 3.0e5), (1.5,)),
    3: ((3.0e4, 7.0e4, 3.0e5), (1.5, 0.75)),
    4: ((3.0e4, 7.0e4, 1.5e5, 3.0e5), (1.5, 0.75, 0.375)),
    5: ((2.5e4, 5.0e4, 7.5e4, 1.0e5, 1.5e5), (1.5, 0.75, 0.375, 0.1875)),
}


def double_gyre(ii: int, layers: int = 3, dt: float = 900.0, precision: int = pq.PREC_FP64,
                jj: int | None = None, **kw) -> "pq.Config":
    """Double gyre on an ii x jj grid over the fixed basin (dx = basin / (ii - 1))."""
    H, gp = LAYERS[layers]
    dx = BASIN_CM / (ii - 1)
    p = pq.double_gyre_physical(ii, jj, layers=layers, dt=dt, dx=dx, H=H, gprime=gp, precision=precision, **kw)
    return pq.Config.from_physical(p)


def initial_condition(cfg: "pq.Config", seed: int = 1):
    return pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)


GRID_SIZES = (65, 129, 257, 513, 1025)


def gaussian_random_field(ii: int, jj: int, layers: int, seed: int, slope: float = -3.0):
    """Seeded Gaussian random field with power spectrum |k|^slope (per layer),
    unit RMS, Fortran order (ii, jj, layers)."""
    rng = np.random.default_rng(seed)
    ki = np.fft.fftfreq(ii)[:, None]
    kj = np.fft.rfftfreq(jj)[None, :]
    k = np.sqrt(ki * ki + kj * kj)
    k[0, 0] = np.inf
    amp = k ** (slope / 2.0)
    out = np.empty((ii, jj, layers), order="F")
    for l in range(layers):
        w = np.fft.rfft2(rng.standard_normal((ii, jj)))
        f = np.fft.irfft2(w * amp, s=(ii, jj))
        out[:, :, l] = f / (np.sqrt(np.mean(f * f)) + 1e-300)
    return out


def batched_helmholtz(n: int = 512, seed: int = 2, sizes=GRID_SIZES, max_layers: int = 5):
    """The batched-Helmholtz workload: n solves with ii and jj drawn
    independently from `sizes`, L in 1..max_layers, layer depths
    H ~ U[200, 4000] m and g'_k = 1.5 * 2^-k cm s^-2, ss from the
    stratification eigenproblem of the double-gyre physics.  Returns
    (shapes, ss) for pq.Batch."""
    rng = np.random.default_rng(seed)
    shapes, ss = [], []
    for _ in range(n):
        ii = int(rng.choice(sizes))
        jj = int(rng.choice(sizes))
        L = int(rng.integers(1, max_layers + 1))
        H = tuple(float(h) for h in rng.uniform(2.0e4, 4.0e5, L))
        gp = tuple(1.5 * 2.0 ** (-k) for k in range(L - 1))
        p = pq.double_gyre_physical(ii, jj, layers=L, dt=900.0, dx=BASIN_CM / (ii - 1), H=H, gprime=gp)
        cfg = pq.Config.from_physical(p)
        shapes.append((ii, jj, L))
        ss.append(np.array(cfg.desc.ss[:L]))
    return shapes, ss


def serving_requests(rate: float = 200.0, window: float = 1.0, seed: int = 3, sizes=(129, 257, 513, 1025),
                     layers=(2, 3, 4, 5), steps=(100, 5000), dt: float = 1800.0):
    """The serving workload: Poisson arrivals at `rate` per second over
    `window` seconds; each request a double gyre on a size from `sizes`
    (square), L from `layers`, a step count uniform in `steps`, and a seeded
    1e-7 perturbation.  Returns [(arrival_s, ii, L, nsteps, seed)]."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > window:
            return out
        out.append((t, int(rng.choice(sizes)), int(rng.choice(layers)), int(rng.integers(steps[0], steps[1] + 1)),
                    int(rng.integers(1 << 30))))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--size", type=int, default=513)
    ap.add_argument("--layers", type=int, default=3)
    ap.add_argument("--dt", type=float, default=900.0)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--dst-lanes", type=int, default=0, help="lanes per row-DST unit, both directions (0: default)")
    ap.add_argument("--pdl", action="store_true", help="programmatic dependent launch of the step kernels")
    ap.add_argument("--dst-algo", type=int, default=0,
                    help="row-DST algorithm of the mixed form: 1 butterfly, 2 tensor-core DST (0: default)")
    ap.add_argument("--cab-kernel", type=int, default=-1,
                    help="CABARET formulation: 0 tiles, 1 sweeps, 2 two-column sweeps (mixed; -1: default)")
    ap.add_argument("--cab-band", type=int, default=0, help="rows per CABARET sweep (0: default)")
    ap.add_argument("--inversions", type=int, default=0,
                    help="instead of stepping: this many pv_inversions of a seeded random zeta")
    a = ap.parse_args(argv)
    cfg = double_gyre(a.size, a.layers, a.dt, pq.PREC_FP64 if a.precision == "fp64" else pq.PREC_MIXED)
    m = pq.Model(cfg)
    if a.dst_algo:
        m.set_tuning(dst_algo=a.dst_algo)
    if a.inversions:
        z = np.asfortranarray(np.random.default_rng(1).standard_normal((cfg.ii, cfg.jj, cfg.layers)))
        for _ in range(a.inversions):
            psi = m.pv_inversion(z)
        print("pv_inversion x", a.inversions, "max |psi|", float(np.abs(psi).max()))
        m.close()
        return
    m.init_perturb(initial_condition(cfg))
    if a.dst_lanes:
        m.set_tuning(dst_lanes=a.dst_lanes, dst_lanes_inv=a.dst_lanes)
    if a.pdl:
        m.set_tuning(pdl=1)
    if a.cab_kernel >= 0:
        m.set_tuning(cab_kernel=a.cab_kernel)
    if a.cab_band:
        m.set_tuning(cab_band=a.cab_band)
    m.step(4)
    m.kernel_timing(True)  # eager: one launch per kernel
    for _ in range(a.steps):
        m.step_async(1)
    m.check()
    times = m.kernel_times()
    print({k: round(v[0] / max(1, v[1]) * 1e3, 2) for k, v in times.items()}, "us per launch")
    m.close()


if __name__ == "__main__":
    main()
