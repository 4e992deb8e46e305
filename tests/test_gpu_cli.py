"""Drop-in contract: the programs against the reference's own programs
(compiled from the reference sources into oracle/_ref) on the same parameter
and data files.  Same argv, same file formats, same row order; values agree
to the printed precision ("%lf", 6 decimals) and readme_<OUT> is identical
(radon_grid, ray_grid and the adjoint; radon_reduction differs only where the
reference prints nothing different).  The analytic programs are in
test_gpu_zz_analytic_programs.py."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from conftest import PKG_DIR

from wrt_b200.phantom import ellipsoid_phantom

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (O.HERE / "_ref" / "radon_grid").exists(),
                                 reason="reference programs not built")]

OURS = PKG_DIR / "bin"
REF = O.HERE / "_ref"


def run(exe, args, cwd):
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, cwd=cwd, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


def write_params(path, values, labels):
    path.write_text("".join(f"{v}\t\t: {l}\n" for v, l in zip(values, labels)))


def write_volume(path, vol):
    np.savetxt(path, vol.reshape(-1), fmt="%lf")


def table(path):
    return np.loadtxt(path, delimiter=",", ndmin=2)


def compare(tmp, name, ours_out, ref_out, atol=2e-6):
    a, b = table(tmp / "ours" / ours_out), table(tmp / "ref" / ref_out)
    assert a.shape == b.shape
    assert np.abs(a - b).max() <= atol, np.abs(a - b).max()
    ra = (tmp / "ours" / f"readme_{ours_out}").read_text()
    rb = (tmp / "ref" / f"readme_{ref_out}").read_text()
    assert ra == rb


@pytest.fixture
def dirs(tmp_path):
    (tmp_path / "ours").mkdir()
    (tmp_path / "ref").mkdir()
    return tmp_path


def both(tmp, prog, files, args):
    for d in ("ours", "ref"):
        for f in files:
            shutil.copy(tmp / f, tmp / d / f)
    run(OURS / prog, args, tmp / "ours")
    run(REF / prog, args, tmp / "ref")


def test_radon_grid_program(dirs):
    n = 20
    write_params(dirs / "cfg.txt", [16, 8, 11, n], ["nphi", "ntheta", "nshift", "ngrid"])
    write_volume(dirs / "vol.txt", ellipsoid_phantom(n, 6, 31))
    both(dirs, "radon_grid", ["cfg.txt", "vol.txt"], ["-p", "cfg.txt", "-i", "vol.txt", "-o", "out.csv", "-n", "3"])
    compare(dirs, "radon_grid", "out.csv", "out.csv")


def test_ray_then_reduction_then_adjoint(dirs):
    n = 16
    write_params(dirs / "rcfg.txt", [n, n, 13, 12], ["ngrid", "nslices", "nshift", "nphi"])
    write_volume(dirs / "vol.txt", ellipsoid_phantom(n, 5, 32))
    both(dirs, "ray_grid", ["rcfg.txt", "vol.txt"], ["-p", "rcfg.txt", "-i", "vol.txt", "-o", "rays.csv", "-n", "2"])
    compare(dirs, "ray_grid", "rays.csv", "rays.csv")
    # reduction reads the reference's own ray file in both cases
    shutil.copy(dirs / "ref" / "rays.csv", dirs / "rays.csv")
    write_params(dirs / "dcfg.txt", [13, 12, 6, n], ["nshift", "nphi", "ntheta", "ngrid"])
    both(dirs, "radon_reduction", ["dcfg.txt", "rays.csv"], ["-p", "dcfg.txt", "-i", "rays.csv", "-o", "radon.txt", "-n", "2"])
    compare(dirs, "radon_reduction", "radon.txt", "radon.txt")


def test_adjoint_program(dirs):
    n = 18
    write_params(dirs / "cfg.txt", [10, 6, 9, n], ["nphi", "ntheta", "nshift", "ngrid"])
    write_volume(dirs / "vol.txt", ellipsoid_phantom(n, 4, 33))
    # Radon data in the 4-column format the adjoint reads: radon_grid's output
    run(REF / "radon_grid", ["-p", "cfg.txt", "-i", "vol.txt", "-o", "radon.csv"], dirs)
    write_params(dirs / "acfg.txt", [10, 6, 9, 8], ["nphi", "ntheta", "nshift", "ngrid"])
    both(dirs, "radon3d_grid", ["acfg.txt", "radon.csv"], ["-p", "acfg.txt", "-i", "radon.csv", "-o", "adj.txt"])
    compare(dirs, "radon3d_grid", "adj.txt", "adj.txt")
