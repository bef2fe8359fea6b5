"""bench.py's reference arm on the CPU: the JSON line it prints (one rank, and
two gloo ranks under torch.distributed.run, where rank 0 alone prints)."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def _lines(out):
    return [json.loads(s) for s in out.splitlines() if s.startswith("{")]


def _check(line, n_gpus):
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and line["n_gpus"] == n_gpus
    assert line["unit"] == "Gpts/s" and line["higher_is_better"] is True and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--n", "32", "--steps", "2",
                        "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)
    assert lines[0]["steps"] == 2 and lines[0]["warmup"] == 1


def test_reference_arm_under_two_ranks_prints_from_rank_0_only():
    """Two ranks with the environment torch.distributed.run gives each
    (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_*); started directly, because
    torch.distributed.run would read bench.py's --n as an abbreviation of
    its own options."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--n", "32", "--steps", "1",
           "--warmup", "1"]
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", LOCAL_WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
        procs.append(subprocess.Popen(cmd, cwd=ROOT, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = [p.communicate(timeout=300) for p in procs]
    for p, (_, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    assert _lines(outs[1][0]) == []
    lines = _lines(outs[0][0])
    assert len(lines) == 1
    _check(lines[0], 2)


def test_cpu_sample_rotation_visits_the_sweeps_operator_mix():
    """Six consecutive CPU-sample steps apply each of the 18 family x
    direction pairs of a sweep step exactly once, three per step, one per
    direction."""
    sys.path.insert(0, ROOT)
    import bench
    for start in (0, 5):
        seen = [p for s in range(start, start + 6) for p in bench.sample_ops(s)]
        assert len(seen) == 18 and len(set(seen)) == 18
        assert {k for k, _ in seen} == {k for k, _ in bench.KINDS}
    for s in range(6):
        assert [d for _, d in bench.sample_ops(s)] == [0, 1, 2]
