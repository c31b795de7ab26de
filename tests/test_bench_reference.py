"""bench.py's reference arm (`--impl reference`) on the CPU: it times the
oracle port of the reference's stereo on the host cores and prints one JSON
line with the headline metric, without loading any library of the product
(the scene is rendered by the host-only renderer build under oracle/ and
planned by the oracle).  Under a multi-rank launch only rank 0 works."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RUN = r"""
import sys
sys.argv = ["bench.py", "--impl", "reference", "--config", "c1", "--steps", "1", "--warmup", "3",
            "--cpu-rows", "8"]
sys.path.insert(0, ".")
import bench
bench.main()
maps = open("/proc/self/maps").read()
print("LOADED " + " ".join(sorted({l.split()[-1].rsplit("/", 1)[-1] for l in maps.splitlines()
                                   if l.split()[-1].endswith(".so")})))
"""


def _run(env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, "-c", _RUN], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_prints_the_metric_line_and_loads_no_product_library():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    rec = json.loads(lines[-2])
    import bench  # noqa: E402  (path set by conftest)
    assert rec["impl"] == "reference" and rec["metric"] == bench.METRIC
    assert rec["unit"] == "depth maps/s" and rec["higher_is_better"] is True and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "port" and rec["cpu_baseline"]["cores"] >= 1
    assert rec["cpu_baseline"]["value"] == rec["value"]
    assert rec["e2e"] == {"value": rec["value"], "unit": "depth maps/s", "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    loaded = lines[-1].split()[1:]
    assert "libmvs_oracle.so" in loaded and "libscene_host.so" in loaded
    assert "librcmvs.so" not in loaded and "librcscene.so" not in loaded


def test_reference_arm_other_ranks_do_no_work():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1 and lines[0].startswith("LOADED")
