"""Drop-in programs: argument and parameter-file handling (before any device
work), checked without a GPU; and the analytic programs end to end against the
reference's programs, built against a CPU stand-in of the library
(tests/analytic_cli_stub.c)."""
import os
import subprocess
from pathlib import Path

import pytest

from conftest import PKG_DIR, ROOT

BIN = PKG_DIR / "bin"
PROGRAMS = ["radon_grid", "ray_grid", "radon_reduction", "radon3d_grid"]
ANALYTIC = ["radon_analytic", "ray_analytic"]


def run(prog, *args, cwd=None):
    return subprocess.run([str(BIN / prog), *args], capture_output=True, text=True, cwd=cwd,
                          timeout=60)


@pytest.mark.parametrize("prog", PROGRAMS + ANALYTIC)
def test_no_arguments(prog):
    r = run(prog)
    assert r.returncode == 1 and "arguments required" in r.stderr


@pytest.mark.parametrize("prog", PROGRAMS + ANALYTIC)
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


@pytest.mark.parametrize("prog", ANALYTIC)
def test_analytic_programs_options(prog, tmp_path):
    """No input file (the reference's analytic programs take -p, -o, -n); the
    test function, which the reference compiles in, is chosen by --function
    among its example files."""
    r = run(prog, "-h")
    assert "--function" in r.stdout and "--input" not in r.stdout
    r = run(prog, "-p", "p.txt", "-o", "out.csv", cwd=tmp_path)
    assert r.returncode == 1 and "--function is required" in r.stderr
    r = run(prog, "-p", "p.txt", "-o", "out.csv", "--function", "gaussian", cwd=tmp_path)
    assert r.returncode == 1 and "unknown test function" in r.stderr
    r = run(prog, "-p", "p.txt", "-i", "v.txt", "-o", "out.csv", "--function", "exponential_bump",
            cwd=tmp_path)
    assert r.returncode == 1 and "Usage:" in r.stderr
    r = run(prog, "-p", "nope.txt", "-o", "out.csv", "--function", "exponential_bump", cwd=tmp_path)
    assert r.returncode == 1 and "nope.txt" in r.stderr


def test_ray_analytic_reads_three_parameters(tmp_path):
    (tmp_path / "p.txt").write_text("9 : nshift\n8 : nphi\n")
    r = run("ray_analytic", "-p", "p.txt", "-o", "out.csv", "--function", "sinusoidal_bump",
            cwd=tmp_path)
    assert r.returncode == 1 and "parameters 2 : reached end of file" in r.stderr


REF_DIR = ROOT / "oracle" / "_ref"


@pytest.fixture(scope="module")
def stubbed_analytic(tmp_path_factory):
    """The analytic programs built against a CPU stand-in of the library
    (tests/analytic_cli_stub.c) that integrates with the reference's own
    code, so that everything but the GPU call is checked here."""
    if not (REF_DIR / "radon_analytic_exp").exists():
        pytest.skip("reference analytic programs not built (oracle/_ref)")
    d = tmp_path_factory.mktemp("stubbed")
    cli = PKG_DIR / "cli"
    exes = {}
    for prog in ANALYTIC:
        exe = d / prog
        subprocess.run(["gcc", "-O2", "-std=gnu99", f"-I{ROOT / 'include'}", f"-I{cli}",
                        str(Path(__file__).parent / "analytic_cli_stub.c"), str(cli / f"{prog}.c"),
                        str(cli / "cli_common.c"), "-o", str(exe), f"-L{ROOT / 'oracle'}",
                        "-loracle", f"-Wl,-rpath,{ROOT / 'oracle'}", "-ldl", "-lpthread", "-lm"],
                       check=True)
        exes[prog] = exe
    return exes


@pytest.mark.parametrize("prog,params", [
    ("radon_analytic", [("nphi", 12), ("ntheta", 6), ("nshift", 9), ("ngrid", 24)]),
    ("ray_analytic", [("nshift", 11), ("nphi", 10), ("ngrid", 16)]),
])
@pytest.mark.parametrize("family", ["exponential_bump", "sinusoidal_bump"])
def test_analytic_programs_match_the_reference_programs(stubbed_analytic, tmp_path, prog, params,
                                                        family):
    """Same parameter file, same output and readme, byte for byte, as the
    reference's program built with that example function, with the
    integrals from the reference's own code behind the stub."""
    text = "".join(f"{v}\t\t: {k}\n" for k, v in params)
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    for d in (ours, ref):
        d.mkdir()
        (d / "cfg.txt").write_text(text)
    env = dict(os.environ, WRT_STUB_REF_DIR=str(REF_DIR))
    r = subprocess.run([str(stubbed_analytic[prog]), "-p", "cfg.txt", "-o", "out.csv", "-n", "3",
                        "--function", family], cwd=ours, capture_output=True, text=True,
                       timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    suffix = "exp" if family == "exponential_bump" else "sine"
    r = subprocess.run([str(REF_DIR / f"{prog}_{suffix}"), "-p", "cfg.txt", "-o", "out.csv",
                        "-n", "2"], cwd=ref, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert (ours / "out.csv").read_bytes() == (ref / "out.csv").read_bytes()
    assert (ours / "readme_out.csv").read_text() == (ref / "readme_out.csv").read_text()
