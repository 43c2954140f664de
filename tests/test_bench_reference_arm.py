"""The reference arm of bench.py (the CPU restatement of the reference's path,
timed on the host cores) keeps its JSON contract on CPU: one line from rank 0,
the metric and config of the engine's arm, and every usable host thread, also
under torchrun, which sets OMP_NUM_THREADS=1 in its ranks."""
import json
import os
import socket
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--workload", "c1", "--steps", "1", "--warmup", "0", "--ref-seconds", "0.5",
        "--no-ref-cuda"]


def _threads():
    return len(os.sched_getaffinity(0))


def _lines(out):
    return [json.loads(x) for x in out.splitlines() if x.startswith("{")]


def _check(line, n_gpus):
    assert line["impl"] == "reference"
    assert line["metric"] == "self-join pairs/s" and line["unit"] == "pairs/s"
    assert line["higher_is_better"] is True and line["n_gpus"] == n_gpus
    assert line["value"] > 0 and line["config"]["workload"].startswith("c1")
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and cb["cores"] == _threads()
    assert line["e2e"] == {"value": line["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_one_process():
    r = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=REPO, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_under_torchrun_two_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--gpus", "2", *ARGS]
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1          # rank 0 alone runs and prints
    _check(lines[0], 2)


def test_rank_host_threads_share(monkeypatch):
    # one process: every usable CPU; torchrun ranks on one node: an equal share
    sys.path.insert(0, REPO)
    import bench
    n = _threads()
    for var in ("WORLD_SIZE", "LOCAL_WORLD_SIZE"):
        monkeypatch.delenv(var, raising=False)
    assert bench.rank_host_threads() == n
    monkeypatch.setenv("WORLD_SIZE", "4")
    monkeypatch.setenv("LOCAL_WORLD_SIZE", "4")
    assert bench.rank_host_threads() == max(1, n // 4)
    monkeypatch.setenv("LOCAL_WORLD_SIZE", str(4 * n))
    assert bench.rank_host_threads() == 1
