"""The benchmark's reference arm on the CPU: `bench.py --impl reference`
times the reference's own CPU code (oracle/_ref) on a bounded sample of the
full-pipeline workload and prints one JSON line with the contract's keys,
on the same metric, unit and workload as the GPU arm."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402


@pytest.mark.skipif(not pyoracle.reference_available(512), reason="oracle/_ref not built")
def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--reference-tracers", "32"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["n_gpus"] == 1 and line["steps"] == 2 and line["warmup"] == 1
    assert line["higher_is_better"] is True and line["value"] > 0 and line["ms_per_step"] > 0
    assert "workload" in line["config"] and "tracer-snapshot" in line["unit"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e = line["e2e"]
    assert e["value"] == line["value"] and e["unit"] == line["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


@pytest.mark.skipif(not pyoracle.reference_available(512), reason="oracle/_ref not built")
def test_reference_arm_under_torchrun_prints_one_line_from_rank_0():
    """Launched as the multi-GPU bench is (torchrun, two ranks on 127.0.0.1),
    the reference arm runs on rank 0 alone, which prints the one line; the
    other rank exits 0 without work."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
                        "--reference-tracers", "16"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0


def test_e2e_tracer_count_fits_the_host_memory_left():
    """The e2e measurement keeps every tracer when the page-locked buffers of
    the host's ranks fit in 60 % of the memory left, else the largest
    multiple of 4,096 that does; the host figure is a positive byte count
    where /proc/meminfo or the memory cgroup can be read."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    bench.load_package()
    from croma_fp_b200 import config
    cfg = config.config4()
    nt = 4194304
    per_rank = bench.e2e_tracers(cfg, nt, 3, 1, None)
    assert per_rank == nt
    assert bench.e2e_tracers(cfg, nt, 3, 1, 1.0e12) == nt
    small = bench.e2e_tracers(cfg, nt, 3, 8, 196.0e9)
    assert 4096 <= small < nt and small % 4096 == 0
    per_tracer = 8 * (2 * 512 + 4 * 64 + 8 * 5 + 4 * 4)
    assert small * per_tracer * 8 <= 0.6 * 196.0e9 < (small + 4096) * per_tracer * 8
    assert bench.e2e_tracers(cfg, nt, 3, 8, 1.0e6) == 4096
    avail = bench.host_bytes_available()
    assert avail is None or avail > 0
