#!/usr/bin/env python3
"""Benchmark: CABARET QG time steps of the 3-layer 1025 x 1025 double gyre.

Workload (the single-GPU configuration the headline target is quoted on):
3-layer closed-basin wind-driven double gyre, 1025 x 1025 nodes
(dx = 3.75 km), layer depths 300/700/3000 m, reduced gravities
0.015/0.0075 m s^-2, f0 = 9.4e-5 s^-1, beta = 1.8e-11 m^-1 s^-1,
tau0 = 0.08 N m^-2, bottom drag 1e-7 s^-1, viscosity 100 m^2 s^-1, partial
slip (alpha = 120 km), CABARET with the limiter, dt = 900 s.  Initial PV:
seeded 1e-7 s^-1 N(0,1) white noise smoothed by a Gaussian of 3 cells
(synthetic; no dataset exists).  --size / --layers / --dt select the other
double-gyre configurations (513 x 513 x 3, 2049 x 2049 x 5, ...).

A step is one iteration of the reference's time loop (qg3.F90:590-957) over
the whole grid.  Metric: cell-layer-steps/s = ii * jj * L * steps / time,
for the mixed-precision form (FP32 CABARET and baroclinic transforms, FP64
psi, barotropic mode, projections and reductions) with the plain FP64 form
beside it (--precision both, the default; or one of them alone).

  value  device time of exactly K steps, state resident in HBM; the L2 cache is
         flushed (a 256 MiB memset) before every timed step and the step is
         bracketed by CUDA events on the model's stream.
  e2e    the same K steps through the public C ABI with host buffers:
         every step copies zeta (ii*jj*L doubles) from pinned host memory to
         the device, steps, and copies psi back (pq_step_exchange, whose
         copies overlap the neighbouring steps' kernels); timed as a whole.

--impl reference times the CPU restatement of the reference (the oracle; the
Fortran/MPI reference cannot be built here), set up by the oracle alone, one
single-threaded run per host core, at least 2000 steps divided among them.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): one independent replica per GPU ("replicas only": a
single domain does not shard without an exchange step), weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-layer-steps/s"
UNIT = "cell-layer-steps/s"


# Physical parameters of the double-gyre workloads (cgs), as plain values so
# that the reference arm can set its runs up without the product library:
# basin 3.84e8 cm (128 x 30 km) resolved by ii nodes, f0 = 9.4e-5 s^-1,
# beta = 1.8e-13 cm^-1 s^-1, tau = 0.8 cm^2 s^-2 (wind_asym 1), viscosity
# 1e6 cm^2 s^-1, bottom drag 1e-7 s^-1, partial slip with alpha = 120 km.
BASIN_CM = 3.84e8
LAYERS = {
    1: ((1.0e5,), ()),
    2: ((1.0e5, 3.0e5), (1.5,)),
    3: ((3.0e4, 7.0e4, 3.0e5), (1.5, 0.75)),
    4: ((3.0e4, 7.0e4, 1.5e5, 3.0e5), (1.5, 0.75, 0.375)),
    5: ((2.5e4, 5.0e4, 7.5e4, 1.0e5, 1.5e5), (1.5, 0.75, 0.375, 0.1875)),
}


def physical(ii, layers, dt):
    """The workload's physical description as a dict (oracle.PHYSICAL_KEYS)."""
    H, gp = LAYERS[layers]
    return dict(ii=ii, jj=ii, layers=layers, basinscale=BASIN_CM, dt=dt, f0=9.4e-5, beta=1.8e-13, H=H, gprime=gp,
                tau=0.8, wind_asym=1.0, wind_tilt=0.0, wind_shift=0.0, visc=1.0e6, visc_bot=1.0e-7, alpha=120.0e5,
                partial_slip=1, max_dt=86400.0, u_scale=1.0)


def workload_name(ii, layers, dt):
    return f"double_gyre_{ii}x{ii}x{layers}_dt{int(dt)}s_cabaret"


def make_config(ii, layers, dt, precision=0):
    from pequod_b200.workloads import double_gyre

    return double_gyre(ii, layers, dt, precision)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    One `nvidia-smi -lms` process samples every 50 ms; it is started, and
    its first sample awaited, before the timed region, so that no process
    start and no Python thread competes with the host's launches inside the
    region (a launch delayed there shows up as device time between the
    events).  The samples kept are the last one before the region, those
    during it and the first one after it."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._p = None
        self._f = None
        self._n0 = 0

    def _lines(self):
        self._f.seek(0)
        return [x for x in self._f.read().splitlines() if x.strip()]

    def _wait_lines(self, n, timeout):
        t = time.time() + timeout
        while time.time() < t:
            if len(self._lines()) >= n or (self._p and self._p.poll() is not None):
                break
            time.sleep(0.01)
        return self._lines()

    def __enter__(self):
        import tempfile

        self._f = tempfile.TemporaryFile(mode="w+")
        try:
            self._p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits", "-lms", "50"], stdout=self._f,
                                       stderr=subprocess.DEVNULL)
        except OSError:
            self._p = None
            return self
        self._n0 = len(self._wait_lines(1, 5.0))
        return self

    def __exit__(self, *exc):
        if self._p is None:
            return
        lines = self._wait_lines(self._n0 + 1, 1.0)
        self._p.terminate()
        try:
            self._p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self._p.kill()
            self._p.wait()
        self.samples = lines[max(0, self._n0 - 1):]
        self._f.close()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            f = [x.strip() for x in s.split(",")]
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(f) > 5 + k and f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kernel_bytes_per_cell_layer(L, mixed=False):
    """Algorithmic bytes per cell-layer of each kernel of the fixed-dt step
    (each array the kernel must touch, read or written once, at its stored
    width: FP64 everywhere, or for the mixed form FP32 layer fields and
    baroclinic spectral rows with psi, corr, wind and the barotropic mode FP64)."""
    w = 4 if mixed else 8                      # layer fields
    spec = (8 + w * (L - 1)) / L               # spectral rows, averaged over the modes
    return {
        # zeta after predictor + beta in, spectral rows out
        "dst_forward": w + spec,
        # spectral rows in and out
        "tridiag": 2 * spec,
        # spectral rows in, corr of the baroclinic modes in, psi out
        "dst_inverse_backproject": spec + 8 * (L - 1) / L + 8,
        # in: psi (FP64), wind/L (FP64), zeta, zeta_old, uimo, ujmo, zeta_fi,
        # zeta_fj, res_beta; out: zeta_old, res, ui, uj, uimo, ujmo, zeta_fi,
        # zeta_fj and the next step's zeta and res_beta
        "cabaret_fused": 8 + 8.0 / L + 17 * w,
    }


def load_traffic(workload):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(workload, {})
    except Exception:
        return {}


def cpu_baseline_sample(ii, layers, dt, seconds=10.0):
    """The oracle (single core) on a bounded sample of the same workload."""
    from oracle import oracle as O

    oc = O.setup_double_gyre(physical(ii, layers, dt))
    o = O.Model(oc)
    o.init(O.make_ic(ii, ii, layers, seed=1, amplitude=1e-7 * oc["t_scale"], sigma=3.0))
    o.step(1)
    n = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        o.step(1)
        n += 1
    secs = time.perf_counter() - t0
    return ii * ii * layers * n / secs, n, secs


def _ref_worker(args):
    """One oracle run: set up by the oracle alone (no product library), a few
    untimed steps, then `steps` timed steps."""
    ii, layers, dt, warm, steps, seed = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O

    oc = O.setup_double_gyre(physical(ii, layers, dt))
    o = O.Model(oc)
    o.init(O.make_ic(ii, ii, layers, seed=seed, amplitude=1e-7 * oc["t_scale"], sigma=3.0))
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    return time.perf_counter() - t0


REF_MIN_STEPS = 2000


def run_reference(a, rank, world):
    """The reference arm: the CPU restatement of the reference (the oracle;
    the Fortran/MPI reference cannot be built here), one single-threaded run
    per usable host core, stepping concurrently.  The sample is
    max(K, REF_MIN_STEPS) steps divided among the runs; each run times its
    own steps (set-up excluded) and the slowest run's time is the sample's."""
    import multiprocessing as mp

    if rank != 0:
        return
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    total = max(a.steps, REF_MIN_STEPS)
    procs = max(1, min(cores, total))
    per = [total // procs + (1 if r < total % procs else 0) for r in range(procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        times = pool.map(_ref_worker, [(a.size, a.layers, a.dt, min(a.warmup, 3), per[r], 100 + r)
                                       for r in range(procs)])
    wall = max(times)
    units = a.size * a.size * a.layers
    value = units * total / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": wall * 1e3 / total, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(a, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"{total} steps of the {a.size}x{a.size}x{a.layers} workload split over {procs} "
                                   f"concurrent single-threaded oracle runs ({per[0]} steps each, "
                                   f"{wall:.1f} s for the slowest; C++ restatement of the reference, set up by "
                                   f"the oracle itself; the Fortran/MPI reference cannot be built)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_config(a, world):
    return {"workload": workload_name(a.size, a.layers, a.dt), "ii": a.size, "jj": a.size, "layers": a.layers,
            "dt_s": a.dt, "precision": a.precision, "energy_every": a.diag_every,
            "l2": "flushed before every timed step (256 MiB memset)",
            "parallelism": f"replicas{world}"}


def measure_single(cfg, K, warmup, dev, dist, rank, world, seed, pdl=False, diag_every=0, force_algo=None):
    """One run of cfg on this rank: device-timed steps (value), back-to-back
    graph replay, per-kernel event times and the e2e exchange through the C
    ABI.  Returns a dict of the measurements (max over ranks)."""
    import numpy as np
    import torch

    import pequod_b200 as pq
    from pequod_b200 import multirank

    units = cfg.ii * cfg.jj * cfg.layers
    m = pq.Model(cfg, device=dev)
    if pdl:
        m.set_tuning(pdl=1)
    # The autotuner picks the row-DST algorithm (butterfly or tensor-core
    # DST for the mixed form's baroclinic modes) for this shape, unless one
    # is forced.
    if force_algo:
        m.set_tuning(dst_algo=force_algo)
        algo = force_algo
    else:
        algo = m.autotune()
    ic = pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    m.init_perturb(ic)
    m.step(max(3, warmup))
    stream = torch.cuda.ExternalStream(m.stream, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # per-kernel times: eager launches with CUDA events between kernels
    m.kernel_timing(True)
    with torch.cuda.stream(stream):
        for k in range(min(max(K, 50), 200)):
            flush.zero_()
            m.step_async(1)
    stream.synchronize()
    m.check()
    m.kernel_timing(False)
    kt = m.kernel_times()
    m.step(2)  # back to graph launches (one-step graphs of each parity)

    # timed region: K steps (one-step graphs), L2 flushed before each; with
    # diag_every, the energy diagnostics (pq_energy, which waits for the
    # step) after every diag_every-th step, inside that step's events
    barrier()
    energies = []
    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            for k in range(K):
                flush.zero_()
                ev[k][0].record(stream)
                m.step_async(1)
                if diag_every and (k + 1) % diag_every == 0:
                    energies.append(m.energy())
                ev[k][1].record(stream)
        stream.synchronize()
    barrier()
    m.check()
    total_ms = multirank.max_over_ranks(dist, [float(sum(s.elapsed_time(e) for s, e in ev))], device=dev)[0]

    # back-to-back steps (CUDA graphs, L2 warm), informational
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        m.step_async(K)
        e1.record(stream)
    stream.synchronize()
    m.check()
    b2b_ms = e0.elapsed_time(e1)

    # e2e: host buffers through the public C ABI.  The exchange pipelines its
    # copies on the model's own copy streams, so the K steps are timed as a
    # whole: from an event before the first call (which every copy follows)
    # to one after pq_join (which follows every copy).  No L2 flush: every
    # step's zeta arrives from host memory.
    zin = torch.empty(units, dtype=torch.float64, pin_memory=True)
    pout = torch.empty(units, dtype=torch.float64, pin_memory=True)
    zin.numpy()[:] = np.asfortranarray(m.sdata("zeta")).ravel(order="F")
    e2e_s, e2e_e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m.step_exchange(zin.data_ptr(), pout.data_ptr(), pq.PTR_HOST)  # staging buffers and copy streams
    m.sync()
    barrier()
    with torch.cuda.stream(stream):
        e2e_s.record(stream)
        for k in range(K):
            m.step_exchange(zin.data_ptr(), pout.data_ptr(), pq.PTR_HOST)
        m.join()
        e2e_e.record(stream)
    stream.synchronize()
    m.check()
    e2e_ms = multirank.max_over_ranks(dist, [float(e2e_s.elapsed_time(e2e_e))], device=dev)[0]
    psi = m.sdata("psi")
    m.step(1)
    m_launches = m.last_launch_count()
    m.close()
    return {"units": units, "total_ms": total_ms, "value": world * units * K / (total_ms * 1e-3),
            "ms_per_step": total_ms / K, "b2b_ms": b2b_ms, "e2e_ms": e2e_ms,
            "e2e": world * units * K / (e2e_ms * 1e-3), "kt": kt, "clocks": clk.summary(), "psi": psi,
            "dst_algo": "tensor" if algo == pq.DST_TENSOR else "butterfly",
            "launches_per_step": m_launches, "diagnostics": len(energies)}


def measure_ensemble(cfg, n, K, warmup, dev, dist, rank, world, seed):
    """n runs of cfg stepped together (pq_ensemble: one launch per kernel
    over all members, CUDA graphs): device time of K steps of every member,
    L2 flushed before each step."""
    import torch

    import pequod_b200 as pq
    from pequod_b200 import multirank

    ens = pq.Ensemble(cfg, n, device=dev)
    algo = ens.autotune()
    for k in range(n):
        ens.init(k, pq.make_ic(cfg.ii, cfg.jj, cfg.layers, seed=seed + 1000 * k, amplitude=1e-7 * cfg.t_scale,
                               sigma=3.0))
    ens.step(max(3, warmup))
    stream = torch.cuda.ExternalStream(ens.stream, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            ev[k][0].record(stream)
            ens.step_async(1)
            ev[k][1].record(stream)
    stream.synchronize()
    ens.sync()
    ms = multirank.max_over_ranks(dist, [float(sum(a.elapsed_time(b) for a, b in ev))], device=dev)[0]
    units = n * cfg.ii * cfg.jj * cfg.layers
    launches = ens.members[0].last_launch_count()
    ens.close()
    return {"members": n, "value": world * units * K / (ms * 1e-3), "ms_per_step": ms / K,
            "dst_algo": "tensor" if algo == pq.DST_TENSOR else "butterfly"}


def roofline_of(res, layers, mixed):
    peak, peak_kind = peaks()
    kt = res["kt"]
    bpc = kernel_bytes_per_cell_layer(layers, mixed=mixed)
    dom = max(kt, key=lambda k: kt[k][0])
    dom_ms = kt[dom][0] / max(1, kt[dom][1])
    alg = bpc[dom] * res["units"]
    achieved = alg / (dom_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "alg_bytes_per_launch": alg, "ms_per_launch": dom_ms}


def step_alg_bytes(layers, mixed):
    """Compulsory bytes of one fused step per cell-layer (every array read or
    written once): 8 (22 + 1/L) in FP64; 4 (20 + 1/L) + 8 * 2 when all but
    psi is stored in FP32."""
    return 4 * (20 + 1.0 / layers) + 16 if mixed else 8 * (22 + 1.0 / layers)


def run_ours(a, rank, world, local_rank):
    """Single runs of the workload: the mixed-precision form (the headline
    value) and the plain FP64 form beside it, the same seeded initial
    condition for both; psi of the mixed run is compared with the FP64 run's
    after the same steps."""
    import numpy as np
    import torch

    from pequod_b200 import multirank

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = multirank.init(world)
    K = a.steps
    seed = multirank.rank_seed(1, rank)
    forms = {"mixed": 1, "fp64": 0} if a.precision == "both" else {a.precision: 0 if a.precision == "fp64" else 1}
    res = {}
    for name, prec in forms.items():
        cfg = make_config(a.size, a.layers, a.dt, precision=prec)
        res[name] = measure_single(cfg, K, a.warmup, dev, dist, rank, world, seed, pdl=a.pdl,
                                   diag_every=a.diag_every)
    # The mixed form with the other row-DST algorithm than the autotuner's
    # choice (the tensor-core DST when it chose the butterfly), reported
    # beside it.
    other = None
    if "mixed" in res:
        from pequod_b200 import DST_BUTTERFLY, DST_TENSOR
        alt = DST_TENSOR if res["mixed"]["dst_algo"] == "butterfly" else DST_BUTTERFLY
        cfg = make_config(a.size, a.layers, a.dt, precision=1)
        other = measure_single(cfg, K, a.warmup, dev, dist, rank, world, seed, pdl=a.pdl, force_algo=alt)
    batched = {}
    if a.ensemble > 0:
        # The batched form: an ensemble of runs of the same configuration
        # stepped together, each precision (every rank takes part).
        for name, prec in forms.items():
            cfg = make_config(a.size, a.layers, a.dt, precision=prec)
            batched[name] = measure_ensemble(cfg, a.ensemble, K, a.warmup, dev, dist, rank, world, seed)
    if rank != 0:
        multirank.close(dist)
        return
    head_name = "mixed" if "mixed" in res else "fp64"
    head = res[head_name]
    mixed = head_name == "mixed"
    units = head["units"]
    traffic = load_traffic(workload_name(a.size, a.layers, a.dt) + ("_mixed" if mixed else ""))
    roof = roofline_of(head, a.layers, mixed)
    roof["traffic"] = traffic.get(roof["kernel"])
    step_alg = step_alg_bytes(a.layers, mixed) * units
    peak = roof["peak"]
    kt = head["kt"]
    shares = {k: round(v[0] / max(1e-30, sum(x[0] for x in kt.values())), 4) for k, v in kt.items()}
    cpu = None
    if world == 1 and not a.no_cpu_baseline:
        v, n, secs = cpu_baseline_sample(a.size, a.layers, a.dt, seconds=a.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{n} steps of the same {a.size}x{a.size}x{a.layers} workload in {secs:.1f} s "
                         f"(C++ restatement of the reference, one core)"}
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": K, "warmup": a.warmup,
        "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64" if mixed else "f64", "data": "synthetic",
        "config": bench_config(a, world),
        "roofline": roof,
        "step_roofline": {"alg_bytes_per_step": step_alg,
                          "achieved_gbs": step_alg / (head["ms_per_step"] * 1e-3) / 1e9,
                          "frac": step_alg / (head["ms_per_step"] * 1e-3) / 1e9 / peak},
        "kernel_shares": shares,
        "cpu_baseline": cpu,
        "e2e": {"value": head["e2e"], "unit": UNIT, "h2d_bytes_per_step": units * 8, "d2h_bytes_per_step": units * 8,
                "timing": "K pq_step_exchange calls (pinned host zeta in, psi out, FP64 reference layout, copies "
                          "pipelined on the model's copy streams) between two events, the second after pq_join"},
        "gpu_launches": K * head["launches_per_step"],
        "dst_algo": head["dst_algo"],
        "back_to_back": {"value": world * units * K / (head["b2b_ms"] * 1e-3), "ms_per_step": head["b2b_ms"] / K,
                         "note": "CUDA-graph replay, L2 not flushed"},
        "clocks": head["clocks"],
    }
    if other is not None:
        line["mixed_other_dst"] = {"dst_algo": other["dst_algo"], "value": other["value"],
                                   "ms_per_step": other["ms_per_step"],
                                   "kernel_ms": {k: v[0] / max(1, v[1]) for k, v in other["kt"].items()},
                                   "note": "the same mixed run with the row-DST algorithm the autotuner did not pick"}
    if batched:
        line["batched"] = batched
        if "mixed" in batched and "fp64" in res:
            line["batched_mixed_over_fp64_single"] = line["batched"]["mixed"]["value"] / res["fp64"]["value"]
    if "mixed" in res and "fp64" in res:
        f64 = res["fp64"]
        p64, pmx = f64["psi"], res["mixed"]["psi"]
        line["fp64"] = {"value": f64["value"], "ms_per_step": f64["ms_per_step"], "e2e": f64["e2e"],
                        "roofline": roofline_of(f64, a.layers, False),
                        "back_to_back_ms_per_step": f64["b2b_ms"] / K, "clocks": f64["clocks"]}
        line["mixed_over_fp64"] = head["value"] / f64["value"]
        line["mixed_psi_rel_l2_vs_fp64"] = float(np.linalg.norm(pmx - p64) / np.linalg.norm(p64))
        line["mixed_psi_note"] = (f"after the {max(3, a.warmup) + 2 + min(max(K, 50), 200) + 2 * K + 1} steps each "
                                  f"run took; parity against the FP64 oracle is tested separately")
    print(json.dumps(line), flush=True)
    multirank.close(dist)


def run_batched(a, rank, world, local_rank):
    """Batched Helmholtz: 512 solves of mixed sizes (65..1025)^2 x 1..5 modes,
    k^-3 Gaussian-random-field right-hand sides; one step = one solve of the
    whole batch (device-resident data, graph replay).  Replicas for N > 1."""
    import numpy as np
    import torch

    import pequod_b200 as pq
    from pequod_b200.workloads import batched_helmholtz, gaussian_random_field

    from pequod_b200 import multirank

    torch.cuda.set_device(local_rank)
    dist = multirank.init(world)
    # One batch for the whole job; each rank solves its share of the members
    # (balanced by ii * jj * L, no exchange while solving).
    all_shapes, all_ss = batched_helmholtz(a.batch, seed=2)
    total_units = sum(i * j * l for i, j, l in all_shapes)
    mine = multirank.partition([i * j * l for i, j, l in all_shapes], world)[rank]
    shapes = [all_shapes[k] for k in mine]
    ss = [all_ss[k] for k in mine]
    b = pq.Batch(shapes, ss, device=local_rank)
    # One right-hand side per distinct shape (the timing does not depend on the values).
    rhs_of = {}
    for k, sh in enumerate(shapes):
        if sh not in rhs_of:
            rhs_of[sh] = torch.from_numpy(np.asfortranarray(gaussian_random_field(*sh, seed=k)).ravel(order="F"))
            rhs_of[sh] = rhs_of[sh].pin_memory()
    for k, sh in enumerate(shapes):
        lib = pq.lib()
        lib.pq_batch_set_rhs(b.ctx, k, dptr(rhs_of[sh]), pq.PTR_HOST)
    b.sync()
    units = sum(i * j * l for i, j, l in shapes)
    stream = torch.cuda.ExternalStream(b.stream, device=local_rank)
    for _ in range(a.warmup):
        b.solve_async()
    b.sync()
    K = a.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for k in range(K):
            ev[k][0].record(stream)
            b.solve_async()
            ev[k][1].record(stream)
        b.sync()
    ms = float(sum(s_.elapsed_time(e_) for s_, e_ in ev))
    # e2e: host right-hand sides in, solutions out, through pq_batch_helm.
    arrs = [rhs_of[sh].clone().pin_memory() for sh in shapes]
    ptrs = (pq._dp * len(arrs))(*[dptr(t) for t in arrs])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    KE = max(1, min(K, 5))
    for _ in range(KE):
        for k, sh in enumerate(shapes):
            arrs[k].copy_(rhs_of[sh])
        rc = pq.lib().pq_batch_helm(b.ctx, ptrs, pq.PTR_HOST)
        assert rc == 0, pq.lib().pq_batch_last_error(b.ctx)
    e2e_s = (time.perf_counter() - t0) / KE
    ms, e2e_s = multirank.max_over_ranks(dist, [ms, e2e_s], device=f"cuda:{local_rank}")
    # The mixed-precision variants of the same batch (first layer FP64, the
    # others FP32): FP32 butterfly, tensor-core DST, and the per-class
    # autotuner's choice; accuracy against this FP64 solve (which equals the
    # oracle's helm to 1e-12, tests/test_gpu_batch.py).
    ref = [b.get(k) for k in range(len(shapes))]  # the e2e pass above solved the right-hand sides once
    variants = {}
    for vname, algo in (("fp32_butterfly", pq.DST_BUTTERFLY), ("bf16x3_tensor", pq.DST_TENSOR),
                        ("mixed_autotuned", 0)):
        bv = pq.Batch(shapes, ss, device=local_rank, precision=pq.PREC_MIXED, dst_algo=algo)
        for k, sh in enumerate(shapes):
            pq.lib().pq_batch_set_rhs(bv.ctx, k, dptr(rhs_of[sh]), pq.PTR_HOST)
        for _ in range(a.warmup):
            bv.solve_async()
        bv.sync()
        evv = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        sv = torch.cuda.ExternalStream(bv.stream, device=local_rank)
        for k in range(K):
            evv[k][0].record(sv)
            bv.solve_async()
            evv[k][1].record(sv)
        bv.sync()
        msv = float(sum(x.elapsed_time(y) for x, y in evv))
        # helm works in place: solve the right-hand sides once more for the
        # accuracy check (the timed solves re-solved their own outputs)
        for k, sh in enumerate(shapes):
            pq.lib().pq_batch_set_rhs(bv.ctx, k, dptr(rhs_of[sh]), pq.PTR_HOST)
        bv.solve_async()
        bv.sync()
        worst = 0.0
        for k in range(len(shapes)):
            o = bv.get(k)
            for l in range(1, shapes[k][2]):
                den = np.linalg.norm(ref[k][:, :, l])
                if den > 0:
                    worst = max(worst, float(np.linalg.norm(o[:, :, l] - ref[k][:, :, l]) / den))
        ntensor = sum(1 for k in range(len(shapes)) if bv.member_dst_algo(k) == pq.DST_TENSOR)
        msv = multirank.max_over_ranks(dist, [msv], device=f"cuda:{local_rank}")[0]
        variants[vname] = {"value": total_units * K / (msv * 1e-3), "ms_per_step": msv / K,
                           "max_rel_l2_fp32_layers_vs_fp64": worst, "members_on_tensor_dst": ntensor,
                           "launches_per_solve": bv.launch_count()}
        bv.close()
    if rank == 0:
        peak, peak_kind = peaks()
        per_solve_s = ms / K * 1e-3
        alg = 48.0 * units  # forward DST 16 B, tridiagonal 16 B, inverse DST 16 B per cell-layer
        cpu = None
        if world == 1 and not a.no_cpu_baseline:
            from oracle import oracle as O

            t0 = time.perf_counter()
            done_units, nsolve = 0, 0
            order = sorted(range(len(shapes)), key=lambda k: shapes[k][0] * shapes[k][1] * shapes[k][2])
            for k in order:
                if time.perf_counter() - t0 > a.cpu_seconds:
                    break
                i, j, l = shapes[k]
                O.Helm(i, j, l, list(ss[k]))(rhs_of[shapes[k]].numpy().reshape((i, j, l), order="F"))
                done_units += i * j * l
                nsolve += 1
            secs = time.perf_counter() - t0
            cpu = {"value": done_units / secs, "unit": "cell-layer-solves/s", "cores": 1, "kind": "port",
                   "sample": f"{nsolve} smallest members solved by the oracle's helm in {secs:.1f} s"}
        line = {
            "metric": "cell-layer-solves/s", "value": total_units * K / (ms * 1e-3), "unit": "cell-layer-solves/s",
            "n_gpus": world, "steps": K, "warmup": a.warmup, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"batched_helmholtz_{len(all_shapes)}", "solves_per_step": len(all_shapes),
                       "cell_layers_per_step": total_units, "sizes": "ii, jj in {65..1025}, L in 1..5",
                       "l2": f"inputs {8 * units / 1e9:.1f} GB per rank >> L2",
                       "parallelism": f"members sharded over {world} rank(s), balanced by ii*jj*L",
                       "launches_per_solve": b.launch_count()},
            "solves_per_s": len(all_shapes) * K / (ms * 1e-3),
            "roofline": {"bound": "hbm", "kernel": "whole batch solve", "achieved": alg / per_solve_s / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg / per_solve_s / 1e9 / peak,
                         "peak_kind": peak_kind, "traffic": None, "alg_bytes_per_launch": alg},
            "cpu_baseline": cpu,
            "e2e": {"value": total_units / e2e_s, "unit": "cell-layer-solves/s",
                    "h2d_bytes_per_step": 8 * units, "d2h_bytes_per_step": 8 * units},
            "gpu_launches": b.launch_count() * K,
            "clocks": clk.summary(),
            "mixed_variants": variants,
        }
        print(json.dumps(line), flush=True)
    b.close()
    multirank.close(dist)


def dptr(t):
    """double* of a torch tensor's storage."""
    import ctypes

    import pequod_b200 as pq

    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), pq._dp)


def serve(reqs, precision, a, local_rank):
    """Serve one request stream (arrival_s, ii, L, nsteps, seed) on this GPU:
    submit each request when its arrival time has passed, poll the server
    until every run is done.  Returns, per finished run, (latency from
    arrival to result, cell-layer-steps, finish time, mean time per step
    while active), the failed-run count and the kernel launches."""
    import pequod_b200 as pq
    from pequod_b200.workloads import double_gyre, initial_condition

    cfgs = {}
    srv = pq.Server(int(a.budget_gb * (1 << 30)), device=local_rank)
    pending = list(reqs)
    ids = {}
    done, failed = [], 0
    t_start = srv.clock()
    while pending or ids:
        now = srv.clock() - t_start
        while pending and pending[0][0] <= now:
            t_arr, ii, L, n, seed = pending.pop(0)
            key = (ii, L)
            if key not in cfgs:
                cfgs[key] = double_gyre(ii, L, 1800.0, precision)
            cfg = cfgs[key]
            rid = srv.submit(cfg, initial_condition(cfg, seed), n)
            ids[rid] = (t_arr, ii * ii * L * n, n)
        if ids:
            srv.poll(a.round_steps)
        for rid in [rid for rid in ids if srv.status(rid) in (2, 3)]:
            t_arr, work, n = ids.pop(rid)
            try:
                _, t3 = srv.collect(rid)
            except pq.PQError:
                failed += 1
                continue
            done.append((t3[2] - t_start - t_arr, work, t3[2] - t_start, (t3[2] - t3[1]) / max(1, n - 1)))
        if not ids and pending:
            time.sleep(max(0.0, min(0.01, pending[0][0] - (srv.clock() - t_start))))
    launches = srv.launches()
    srv.close()
    return done, failed, launches


def run_serving(a, rank, world, local_rank):
    """Serving: one stream of Poisson arrivals at 200 runs/s over a window;
    double gyres of 129..1025 squared, 2-5 layers, 100-5000 steps; 150 GB
    HBM budget.  Multi-GPU: the requests are partitioned across the ranks
    (whole runs, balanced by ii^2 * L * steps).  Reports the per-request
    latency (arrival to result) and per-step latency (a run's active time
    over its steps) percentiles and the aggregate throughput, for the
    mixed-precision form with the FP64 form beside it."""
    import numpy as np
    import torch

    from pequod_b200.workloads import serving_requests
    from pequod_b200 import multirank
    import pequod_b200 as pq

    torch.cuda.set_device(local_rank)
    dist = multirank.init(world)
    reqs = serving_requests(rate=a.rate, window=a.window, seed=3)
    mine = multirank.partition([ii * ii * L * n for _, ii, L, n, _ in reqs], world)[rank]
    my_reqs = [reqs[k] for k in mine]
    forms = ({"mixed": pq.PREC_MIXED, "fp64": pq.PREC_FP64} if a.precision == "both"
             else {a.precision: pq.PREC_FP64 if a.precision == "fp64" else pq.PREC_MIXED})
    out = {}
    with ClockSampler(local_rank) as clk:
        for name, prec in forms.items():
            done, failed, launches = serve(my_reqs, prec, a, local_rank)
            all_done = multirank.gather_lists(dist, done)
            summary = multirank.serving_summary(all_done)
            steps_lat = np.array([d[3] for d in all_done])
            summary["step_p50_ms"] = float(np.percentile(steps_lat, 50) * 1e3)
            summary["step_p99_ms"] = float(np.percentile(steps_lat, 99) * 1e3)
            summary["failed"] = int(sum(multirank.gather_lists(dist, [failed])))
            summary["launches"] = int(sum(multirank.gather_lists(dist, [launches])))
            out[name] = summary
    head_name = "mixed" if "mixed" in out else next(iter(out))
    head = out[head_name]
    line = {
        "metric": "serving latency p50/p99 (s)", "value": head["p50_s"], "unit": "s",
        "p50_s": head["p50_s"], "p99_s": head["p99_s"],
        "step_latency_ms": {"p50": head["step_p50_ms"], "p99": head["step_p99_ms"]},
        "n_gpus": world, "steps": head["runs"], "warmup": 0, "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32/f64" if head_name == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": "serving_double_gyre", "rate_per_s": a.rate, "window_s": a.window,
                   "runs": len(reqs), "budget_gb": a.budget_gb, "round_steps": a.round_steps,
                   "precision": head_name,
                   "parallelism": f"requests sharded over {world} rank(s), balanced by ii^2*L*steps"},
        "throughput": {"value": head["throughput"], "unit": "cell-layer-steps/s"},
        "failed_runs": head["failed"],
        "gpu_launches": head["launches"], "clocks": clk.summary(),
    }
    if len(out) == 2:
        f = out["fp64"]
        line["fp64"] = {"p50_s": f["p50_s"], "p99_s": f["p99_s"],
                        "step_latency_ms": {"p50": f["step_p50_ms"], "p99": f["step_p99_ms"]},
                        "throughput": f["throughput"], "failed_runs": f["failed"], "gpu_launches": f["launches"]}
        line["mixed_over_fp64_throughput"] = head["throughput"] / f["throughput"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    multirank.close(dist)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=1025)
    ap.add_argument("--pdl", action="store_true",
                    help="launch the step kernels with programmatic dependent launch")
    ap.add_argument("--layers", type=int, default=3)
    ap.add_argument("--dt", type=float, default=900.0)
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="double-gyre", choices=["double-gyre", "batched-helm", "serving"])
    ap.add_argument("--diag-every", type=int, default=0,
                    help="double-gyre: energy diagnostics every D timed steps (0: none)")
    ap.add_argument("--ensemble", type=int, default=8,
                    help="double-gyre: members of the batched form (0: single runs only)")
    ap.add_argument("--batch", type=int, default=512, help="batched-helm: solves per batch")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: arrivals per second")
    ap.add_argument("--window", type=float, default=0.25, help="serving: seconds of arrivals")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: HBM budget")
    ap.add_argument("--round-steps", type=int, default=16, help="serving: steps per scheduling round")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.workload == "batched-helm" and a.impl == "ours":
        if a.steps == 200:
            a.steps = 20
        run_batched(a, rank, world, local_rank)
    elif a.workload == "serving" and a.impl == "ours":
        run_serving(a, rank, world, local_rank)
    elif a.impl == "reference":
        run_reference(a, rank, world)
    else:
        run_ours(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
