"""Drop-in programs: argument and parameter-file handling (before any device
work), checked without a GPU."""
import subprocess
from pathlib import Path

import pytest

from conftest import PKG_DIR

BIN = PKG_DIR / "bin"
PROGRAMS = ["radon_grid", "ray_grid", "radon_reduction", "radon3d_grid"]


def run(prog, *args, cwd=None):
    return subprocess.run([str(BIN / prog), *args], capture_output=True, text=True, cwd=cwd,
                          timeout=60)


@pytest.mark.parametrize("prog", PROGRAMS)
def test_no_arguments(prog):
    r = run(prog)
    assert r.returncode == 1 and "arguments required" in r.stderr


@pytest.mark.parametrize("prog", PROGRAMS)
def test_help_short_and_long(prog):
    for flag in ("-h", "--help"):
        r = run(prog, flag)
        assert r.returncode == 0 and "Usage:" in r.stdout


@pytest.mark.parametrize("prog", PROGRAMS)
def test_missing_parameter_file(prog, tmp_path):
    r = run(prog, "-p", "nope.txt", "-i", "in.txt", "-o", "out.csv", cwd=tmp_path)
    assert r.returncode == 1 and "nope.txt" in r.stderr


@pytest.mark.parametrize("prog", PROGRAMS)
def test_parameter_lines_need_trailing_text(prog, tmp_path):
    # "%d %[^\n]\n" lets a bare number's text field swallow the next line, so
    # four bare numbers fail at the third parameter, as in the reference
    (tmp_path / "p.txt").write_text("8\n8\n8\n8\n")
    r = run(prog, "-p", "p.txt", "-i", "in.txt", "-o", "out.csv", cwd=tmp_path)
    assert r.returncode == 1 and "parameters 2 : reached end of file" in r.stderr


def test_truncated_volume_file(tmp_path):
    (tmp_path / "p.txt").write_text("4 : nphi\n3 : ntheta\n5 : nshift\n6 : ngrid\n")
    (tmp_path / "v.txt").write_text("0.0\n" * 100)  # 216 expected
    r = run("radon_grid", "-p", "p.txt", "-i", "v.txt", "-o", "out.csv", cwd=tmp_path)
    assert r.returncode == 1 and "end of file" in r.stderr


def test_reduction_small_flag_takes_no_argument(tmp_path):
    (tmp_path / "p.txt").write_text("5 : nshift\n4 : nphi\n3 : ntheta\n6 : ngrid\n")
    (tmp_path / "r.txt").write_text("0.0\n" * 3)
    r = run("radon_reduction", "-p", "p.txt", "-i", "r.txt", "-s", "-o", "o.txt", cwd=tmp_path)
    assert r.returncode == 1 and "small format" in r.stdout and "end of file" in r.stderr


def test_parallel_text_reader(tmp_path):
    """The programs' chunked multi-threaded reader gives exactly the serial
    parse's values, takes the first `count` records, and refuses truncated and
    malformed files (tests/reader_check.c, compiled against cli_common.c)."""
    cli = PKG_DIR / "cli"
    exe = tmp_path / "reader_check"
    subprocess.run(["gcc", "-O2", "-std=gnu99", f"-I{cli}", f"-I{PKG_DIR.parent / 'include'}",
                    str(Path(__file__).parent / "reader_check.c"), str(cli / "cli_common.c"),
                    "-o", str(exe), f"-L{PKG_DIR / 'lib'}", "-lwrt", "-lpthread", "-lm",
                    f"-Wl,-rpath,{PKG_DIR / 'lib'}"], check=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
