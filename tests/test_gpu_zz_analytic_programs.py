"""The analytic drop-in programs (radon_analytic, ray_analytic) on the GPU
against the reference's programs built with each of its example test
functions (oracle/_ref/{radon,ray}_analytic_{exp,sine}).  Where the reference
compiles its test function in, the drop-ins take it by name (--function).
Same parameter file and row order; the grid columns and readme_<OUT> are
identical, the values agree to the printed precision ("%lf") plus the FP32
tolerance of the analytic kernels.  Everything in these programs but the
library call is also checked without a GPU, byte for byte against the same
reference programs (tests/test_cli_cpu.py)."""
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import PKG_DIR

pytestmark = pytest.mark.gpu

OURS = PKG_DIR / "bin"
REF = O.HERE / "_ref"


def run(exe, args, cwd):
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, cwd=cwd, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


def table(path):
    return np.loadtxt(path, delimiter=",", ndmin=2)


@pytest.fixture
def dirs(tmp_path):
    (tmp_path / "ours").mkdir()
    (tmp_path / "ref").mkdir()
    return tmp_path


@pytest.mark.parametrize("prog,params", [
    ("radon_analytic", [("nphi", 12), ("ntheta", 6), ("nshift", 9), ("ngrid", 24)]),
    ("ray_analytic", [("nshift", 11), ("nphi", 10), ("ngrid", 16)]),
])
@pytest.mark.parametrize("family", ["exponential_bump", "sinusoidal_bump"])
def test_analytic_programs(dirs, prog, params, family):
    suffix = "exp" if family == "exponential_bump" else "sine"
    if not (REF / f"{prog}_{suffix}").exists():
        pytest.skip("reference analytic programs not built")
    (dirs / "cfg.txt").write_text("".join(f"{v}\t\t: {k}\n" for k, v in params))
    for d in ("ours", "ref"):
        shutil.copy(dirs / "cfg.txt", dirs / d / "cfg.txt")
    run(OURS / prog, ["-p", "cfg.txt", "-o", "out.csv", "-n", "2", "--function", family],
        dirs / "ours")
    run(REF / f"{prog}_{suffix}", ["-p", "cfg.txt", "-o", "out.csv", "-n", "2"], dirs / "ref")
    a, b = table(dirs / "ours" / "out.csv"), table(dirs / "ref" / "out.csv")
    assert a.shape == b.shape
    assert np.array_equal(a[:, :3], b[:, :3])  # the grid: the same doubles, printed alike
    assert np.abs(a[:, 3] - b[:, 3]).max() <= 2e-6 + 1e-5 * np.abs(b[:, 3]).max()
    assert ((dirs / "ours" / "readme_out.csv").read_text()
            == (dirs / "ref" / "readme_out.csv").read_text())
