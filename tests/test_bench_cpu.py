"""The benchmark's launch contract on the CPU: the reference arm (the
reference's own plane_integral compiled from its sources, timed on the host
cores) prints one JSON line, alone and under a 2-rank torchrun (rank 0
prints, rank 1 exits cleanly), and the multi-rank helper takes the maximum
over ranks through a gloo process group."""
import importlib.util
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

import oracle as O

ROOT = Path(__file__).resolve().parents[1]
needs_ref = pytest.mark.skipif(not O.Reference.available(), reason="oracle/_ref not built")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env():
    env = dict(os.environ)
    env["WRT_REF_PLANES_PER_STEP"] = "48"
    return env


@needs_ref
def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True,
                       env=_env(), timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0


@needs_ref
def test_reference_arm_under_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, env=_env(), timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1 and json.loads(lines[0])["impl"] == "reference"


def _rank_main(rank, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    d = bench.Dist(2)
    d.barrier()
    m = d.max(1.5 + rank)
    d.close()
    with open(out + f".{rank}", "w") as f:
        f.write(repr(m))


def test_dist_max_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "max")
    mp.spawn(_rank_main, args=(_free_port(), out), nprocs=2, join=True)
    assert [float(open(out + f".{r}").read()) for r in range(2)] == [2.5, 2.5]
