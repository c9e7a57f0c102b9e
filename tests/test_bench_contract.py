"""bench.py's reference arm runs the oracle alone: it sets its runs up from
the workload's physical parameters by the oracle's own restatement of the
driver, and maps no library of the product."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_bench_physics_is_the_workload_physics():
    """The plain parameter table bench.py hands the oracle describes the same
    double gyre as the product's workload definition."""
    from pequod_b200.workloads import double_gyre
    from oracle import oracle as O

    for ii, L, dt in ((129, 3, 1800.0), (1025, 3, 900.0), (2049, 5, 300.0)):
        cfg = double_gyre(ii, L, dt)
        ph = bench.physical(ii, L, dt)
        for k in O.PHYSICAL_KEYS:
            v = getattr(cfg.physical, k)
            if k in ("H", "gprime"):
                assert np.array_equal(np.array(v[:len(ph[k])]), np.array(ph[k])), k
            else:
                assert v == ph[k], (k, v, ph[k])


def test_reference_worker_maps_no_product_library():
    code = (
        "import sys; sys.path.insert(0, %r); import bench; "
        "t = bench._ref_worker((33, 3, 900.0, 1, 2, 5)); "
        "maps = open('/proc/self/maps').read(); "
        "assert 'libpequod_b200' not in maps, 'product library mapped'; "
        "assert 'libpq_oracle' in maps; "
        "assert not any(m == 'pequod_b200' or m.startswith('pequod_b200.') for m in sys.modules), 'product imported'; "
        "print('ok', t)" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.startswith("ok")
