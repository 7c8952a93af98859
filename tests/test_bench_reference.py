"""The benchmark's reference arm: it times the oracle on the batched workload and loads nothing
of the product (no libscatrs_b200.so), and its inputs are the GPU arm's."""

import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_workload_is_the_gpu_arms():
    import bench
    from scatrs_b200 import workloads as W

    for scale in (0.05, 1.0):
        ref = bench.reference_workload(seed=0, scale=scale)
        w = W.batched_spheres(seed=0, scale=scale)
        assert ref.n_nodes == w.n_nodes and ref.greek_order == w.greek_order
        np.testing.assert_array_equal(ref.wavelengths, w.wavelengths)
        np.testing.assert_array_equal(ref.m, w.m)
        np.testing.assert_array_equal(ref.dists["kind"], w.dists["kind"])
        np.testing.assert_array_equal(ref.dists["p"], w.dists["param"])
        np.testing.assert_allclose(ref.dists["r_lo"], w.dists["r_lo"], rtol=1e-15)
        np.testing.assert_allclose(ref.dists["r_hi"], w.dists["r_hi"], rtol=1e-15)
        # the oracle's Gauss rule and the library's agree to rounding
        np.testing.assert_allclose(ref.mu, w.mu, rtol=0, atol=4e-16)


def test_reference_arm_loads_no_product_library():
    code = (
        "import runpy, sys\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',\n"
        "            '--cpu-seconds', '0.3', '--scale', '0.02']\n"
        f"runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT_LOADED' if 'libscatrs_b200' in maps else 'PRODUCT_NOT_LOADED')\n"
        "print('ORACLE_LOADED' if 'liboracle' in maps else 'ORACLE_NOT_LOADED')\n"
        "print('SCATRS_B200_IMPORTED' if any(k.startswith('scatrs_b200') for k in sys.modules)"
        " else 'NO_PRODUCT_MODULES')\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert '"impl": "reference"' in out.stdout
    assert "PRODUCT_NOT_LOADED" in out.stdout
    assert "ORACLE_LOADED" in out.stdout
    assert "NO_PRODUCT_MODULES" in out.stdout
