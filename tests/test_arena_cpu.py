"""The serving loop's device-memory arena (wrt-project_b200/csrc/arena.h) is
plain C++: compiled and exercised here on the CPU with random allocation /
release sequences (no overlap, alignment, exact accounting, coalescing)."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "wrt-project_b200" / "csrc"


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_arena_random_sequences(tmp_path):
    exe = tmp_path / "arena_check"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{CSRC}", str(HERE / "arena_check.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
