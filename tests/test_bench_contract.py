"""bench.py's reference arm runs on the host cores alone (the FP64 oracle: the reference has no
CPU implementation of the search), so its JSON line is checked here: the keys the measurement
contract names, the unavailable line for workloads it does not time, and that under torchrun
only rank 0 prints."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SMALL = ["--impl", "reference", "--workload", "whole_2048_t24", "--steps", "1", "--warmup", "0"]


def run(args, **env):
    e = dict(os.environ, **env)
    return subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), *args], capture_output=True, text=True,
                          timeout=300, env=e)


def last_json(r):
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_reference_arm_line():
    d = last_json(run(SMALL))
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "micrographs/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "whole_2048_t24"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # the value is extrapolated from a bounded sample whose own time is ms_per_step
    assert d["extrapolated"] is True and cb["extrapolated"] is True and cb["sample_s"] > 0
    assert abs(d["ms_per_step"] - 1000.0 * cb["sample_s"]) < 1e-6 * d["ms_per_step"]
    # no GPU here: the reference CUDA build's timing says why it is absent
    assert "unavailable" in d["reference_cuda"]


def test_reference_arm_other_ranks_print_nothing():
    r = run(SMALL, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert r.returncode == 0 and r.stdout.strip() == "", (r.stdout, r.stderr[-2000:])


def test_reference_arm_unavailable_workloads():
    for wl in ("batch_c3", "project_c5", "adjoint_c4"):
        d = last_json(run(["--impl", "reference", "--workload", wl, "--steps", "1", "--warmup", "0"]))
        assert d["impl"] == "reference" and d["unavailable"]
