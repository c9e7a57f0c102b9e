"""The C ABI from a plain C program (tests/c_driver.c), as a Fortran
bind(C) module or another host language would call it: the header compiles
as C, the library links, the host-side calls agree with the Python mirror,
and on a GPU a run through C gives the same energies as through ctypes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pequod_b200 as pq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_driver(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    libdir = os.path.dirname(pq.LIB_PATH)
    exe = str(tmp_path / "c_driver")
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_driver.c"), "-L", libdir, "-lpequod_b200",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True)
    return exe


def test_c_caller_host_setup(tmp_path):
    exe = build_driver(tmp_path)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")  # host calls only: no device
    out = subprocess.run([exe, "setup"], capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.splitlines()
    f = lines[0].split()
    vals = dict(zip(f[0::2], f[1::2]))
    cfg = pq.Config.from_physical(pq.double_gyre_physical(129))
    assert float(vals["t_scale"]) == cfg.t_scale
    assert float(vals["dt"]) == cfg.desc.dt
    assert float(vals["wind"]) == cfg.wind[5, 9]
    ic = pq.make_ic(129, 129, 3, seed=7, amplitude=1e-7 * cfg.t_scale, sigma=3.0)
    assert float(vals["ic"]) == ic.ravel(order="F")[1000]
    rc = int(lines[1].split("=")[1])
    assert rc != pq.PQ_OK  # no device: a status code, no abort


@pytest.mark.gpu
def test_c_caller_runs_the_model(tmp_path):
    exe = build_driver(tmp_path)
    out = subprocess.run([exe, "run", "10"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    f = out.stdout.split()
    ek_c = np.array([float(x) for x in f[1:4]])
    ep_c = float(f[5])
    cfg = pq.Config.from_physical(pq.double_gyre_physical(129))
    m = pq.Model(cfg)
    m.init_perturb(pq.make_ic(129, 129, 3, seed=7, amplitude=1e-7 * cfg.t_scale, sigma=3.0))
    m.step(10)
    ek, ep = m.energy()
    assert np.array_equal(ek, ek_c) and ep == ep_c
