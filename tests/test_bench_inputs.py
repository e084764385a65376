"""The benchmark's workload inputs and its reference arm (CPU).

The reference arm builds the scan's inputs with numpy alone and times the oracle; it must never import the
package or load its library, and its inputs must be the ones the B200 arm feeds the GPU.
"""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    sys.path.insert(0, str(ROOT))
    import bench
    return bench


def test_scan_inputs_equal_the_package_generators():
    bench = _bench()
    from classical_mcmc_spin_b200.sharding import scan_delays
    from classical_mcmc_spin_b200.states import zigzag_honeycomb
    for rank, world in ((0, 1), (1, 4)):
        wl = bench.scan_inputs(100, rank, world)
        np.testing.assert_array_equal(wl["s0"], zigzag_honeycomb(24, 24, 1, tilt_sigma=0.05, seed=2).ravel())
        np.testing.assert_array_equal(wl["pulses"][1::3, 1], scan_delays(256, 100.0, rank, world))
        assert wl["pulses"].shape == (768, 4)


def test_reference_arm_loads_only_the_oracle():
    code = (
        "import sys, json\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3', '--md-steps', '40',\n"
        "            '--cpu-seconds', '0.05', '--no-cpu-rows']\n"
        "import bench\n"
        "rc = bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'rc': rc, 'pkg': [m for m in sys.modules if m.startswith('classical_mcmc_spin_b200')],\n"
        "                  'libcmd': 'libcmd_b200' in maps, 'torch': 'torch' in sys.modules}))\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert probe == {"rc": 0, "pkg": [], "libcmd": False, "torch": False}
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"] == _bench().scan_config(40, 1)
    assert line["e2e"]["value"] == line["value"]
