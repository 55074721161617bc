"""The reference arm of bench.py (the CPU oracle timed on the host cores)
prints one JSON line with the keys of the benchmark contract; under a
multi-rank launch only rank 0 prints.  CPU only, small mesh."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "9",
                           "--steps", "2", "--warmup", "3", *args], cwd=ROOT, env=env, capture_output=True,
                          text=True, timeout=600)


def test_reference_arm_line():
    p = run({})
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "Medges/s"
    assert d["higher_is_better"] is True and d["vs_baseline"] is None
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_reference_arm_only_rank0_prints():
    p = run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--gpus", "2")
    assert p.returncode == 0, p.stderr
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]


def test_clock_sampler_brackets_a_short_timed_region(tmp_path, monkeypatch):
    # a stand-in nvidia-smi that needs half a second for its first sample
    # and reports one throttle reason: the sampler waits for that sample
    # before the timed region and for the one after it, so a region far
    # shorter than the sampling period still gets a clock record
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/bash\nsleep 0.5\nwhile true; do "
                    "echo '1965, 1965, 500.0, 0x4, Not Active, Not Active, Not Active, Active'; "
                    "sleep 0.1; done\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(None)
    c.start()
    assert c.lines, "the timed region must start after the first sample"
    clk = c.stop()
    assert clk["samples"] >= 2
    assert clk["sm_mhz"] == 1965.0 and clk["sm_max_mhz"] == 1965.0
    assert clk["reasons"] == ["sw_power_cap"]
