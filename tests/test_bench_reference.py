"""bench.py's reference arm on CPU: the oracle port of the reference's CG,
each timed system solved to its own convergence at 1e-6 (no iteration
budget), without importing this package or loading its CUDA library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print(json.dumps({"package_imported": any(m == "mpsparse_b200" or m.startswith("mpsparse_b200.")
                                          for m in sys.modules),
                  "cuda_lib_loaded": "libmpsparse_b200" in maps,
                  "torch_imported": "torch" in sys.modules}))
"""


def test_reference_arm_runs_converged_without_the_package():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       timeout=600, env={**os.environ, "OMP_NUM_THREADS": str(os.cpu_count() or 1)})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    line, probe = json.loads(lines[0]), json.loads(lines[1])
    assert line["impl"] == "reference" and line["unit"] == "ms" and line["higher_is_better"] is False
    assert line["converged"] == line["steps"] == 1 and line["true_resid_max"] <= 1e-6
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert not probe["package_imported"] and not probe["cuda_lib_loaded"] and not probe["torch_imported"]
