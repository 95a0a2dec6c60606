"""The benchmark's reference arm runs the oracle alone: no module of the tenet package is
imported, so no native library of this build is loaded into that process."""

import json
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_imports_nothing_of_the_package():
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "bad = sorted(m for m in sys.modules if m == 'tenet' or m.startswith('tenet.'))\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('BAD', bad, 'libtenet_b200' in maps)\n")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    lines = res.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["warmup"] == 3 and line["steps"] == 1
    assert line["flops_per_matvec"] > 0
    assert lines[-1] == "BAD [] False"
