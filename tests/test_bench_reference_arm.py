"""The benchmark's reference arm times only the oracle's restatement of the
reference CPU path: it must not import the bajo_b200 package or map
libbajo_b200.so, and it prints the same `config` as the GPU arm."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_workload_generator_matches_package():
    sys.path.insert(0, ROOT)
    import bench
    from bajo_b200 import scenes
    for n, seed in ((65536, 0), (1000, 5)):
        assert np.array_equal(bench.workload_triangles(n, seed), scenes.random_triangles(n, seed=seed))


def test_reference_arm_loads_no_product_code():
    code = (
        "import sys, json, io, contextlib\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import bench\n"
        "args = bench.parse_args(['--impl', 'reference', '--steps', '2', '--warmup', '1'])\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    bench.run_reference(args)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'line': json.loads(buf.getvalue().strip().splitlines()[-1]),\n"
        "                  'imported': sorted(m for m in sys.modules if m.startswith('bajo_b200')),\n"
        "                  'mapped': 'libbajo_b200' in maps}))\n"
    )
    env = dict(os.environ, BENCH_CPU_TRACE_SECONDS="0.2")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["imported"] == []
    assert out["mapped"] is False
    line = out["line"]
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    assert line["config"] == bench.workload_config()
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
