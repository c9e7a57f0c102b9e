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
initialisation and a few eagerly launched steps (one launch per kernel), the
command the committed kernel profiles were taken with.
"""
from __future__ import annotations

import argparse

import pequod_b200 as pq

BASIN_CM = 3.84e8
LAYERS = {
    3: ((3.0e4, 7.0e4, 3.0e5), (1.5, 0.75)),
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


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--size", type=int, default=513)
    ap.add_argument("--layers", type=int, default=3)
    ap.add_argument("--dt", type=float, default=900.0)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    a = ap.parse_args(argv)
    cfg = double_gyre(a.size, a.layers, a.dt, pq.PREC_FP64 if a.precision == "fp64" else pq.PREC_MIXED)
    m = pq.Model(cfg)
    m.init_perturb(initial_condition(cfg))
    m.kernel_timing(True)  # eager: one launch per kernel
    for _ in range(a.steps):
        m.step_async(1)
    m.check()
    times = m.kernel_times()
    print({k: round(v[0] / max(1, v[1]) * 1e3, 2) for k, v in times.items()}, "us per launch")
    m.close()


if __name__ == "__main__":
    main()
