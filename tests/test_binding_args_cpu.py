"""Python binding argument checks, on the CPU against a fake of the C library:
a volume that is not n x n x n, an output array of the wrong size or type,
and a copy larger than its device buffer are refused with ValueError before
any C call (the library would otherwise read or write past a buffer), and the
checks stay on under ``python -O``, which strips assert statements."""
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, load_package

wrt = load_package()


class RecordingLib:
    """Creates handles and records every other C call by name."""

    def __init__(self):
        self.calls = []
        self.next = 100

    def _out(self, ref):
        self.next += 1
        ref._obj.value = self.next
        return 0

    def wrt_ctx_create(self, dev, budget, out):
        return self._out(out)

    def wrt_device_alloc(self, h, n, out):
        return self._out(out)

    def wrt_server_create(self, opts, out):
        return self._out(out)

    def __getattr__(self, name):
        if not name.startswith("wrt_"):
            raise AttributeError(name)

        def call(*args):
            self.calls.append(name)
            return 0
        return call


@pytest.fixture
def fake(monkeypatch):
    """The fake library, installed while the test runs; every context and
    server the test opened is closed before the real library comes back (the
    exit hook would otherwise hand the fake handles to it)."""
    f = RecordingLib()
    before = set(wrt._live)  # real contexts other tests hold stay open
    monkeypatch.setattr(wrt, "_lib", f)
    yield f
    for obj in sorted(set(wrt._live) - before, key=lambda o: not isinstance(o, wrt.Server)):
        obj.close()


def test_context_transforms_refuse_non_cubic_volumes(fake):
    ctx = wrt.Context(0)
    for bad in (np.zeros(27), np.zeros((3, 3)), np.zeros((3, 3, 4))):
        with pytest.raises(ValueError, match="n x n x n"):
            ctx.radon_grid(bad, 4, 2, 3)
        with pytest.raises(ValueError, match="n x n x n"):
            ctx.ray_grid(bad, 3, 3, 2)
        with pytest.raises(ValueError, match="n x n x n"):
            ctx.spectral_laplacian(bad)
    assert fake.calls == []


def test_device_buffer_refuses_oversized_copies(fake):
    ctx = wrt.Context(0)
    buf = wrt.DeviceBuffer(ctx, 16)
    with pytest.raises(ValueError, match="16-byte buffer"):
        buf.upload(np.zeros(3))
    with pytest.raises(ValueError, match="at most 16 bytes"):
        buf.download(np.empty(3))
    with pytest.raises(ValueError):
        buf.download(np.empty((4, 4))[:, :1])  # not contiguous
    assert fake.calls == []
    buf.upload(np.zeros(2))
    buf.download(np.empty(2))
    assert fake.calls == ["wrt_copy_to_device", "wrt_copy_to_host"]


def test_server_refuses_bad_shapes_and_outputs(fake):
    srv = wrt.Server(0)
    vol = np.zeros((4, 4, 4), np.float32)
    with pytest.raises(ValueError, match="n x n x n"):
        srv.submit_forward(np.zeros(64, np.float32), 2, 1, 3, np.empty(6))
    with pytest.raises(ValueError, match="6 values"):
        srv.submit_forward(vol, 2, 1, 3, np.empty(7))
    with pytest.raises(ValueError, match="float64"):
        srv.submit_forward(vol, 2, 1, 3, np.empty(6, np.float32))
    with pytest.raises(ValueError, match="64 values"):
        srv.submit_adjoint(np.zeros((3, 2, 1)), 4, np.empty(63))
    with pytest.raises(ValueError, match="nshift"):
        srv.submit_adjoint(np.zeros(6), 4, np.empty(64))
    with pytest.raises(ValueError, match="n x n x n"):
        srv.submit_ray(np.zeros((4, 4, 5), np.float32), 4, 3, 2, np.empty(24))
    with pytest.raises(ValueError, match="24 values"):
        srv.submit_ray(vol, 4, 3, 2, np.empty(25))
    with pytest.raises(ValueError, match="ray data"):
        srv.submit_reduce(np.zeros(12), 5, 2, np.empty(10))
    with pytest.raises(ValueError, match="20 values"):
        srv.submit_reduce(np.zeros((4, 3, 2)), 5, 2, np.empty(10))
    assert fake.calls == []


def test_checks_survive_python_O():
    script = (
        "import importlib.util, sys, numpy as np\n"
        f"spec = importlib.util.spec_from_file_location('wrt_b200', r'{ROOT / 'wrt-project_b200' / '__init__.py'}')\n"
        "m = importlib.util.module_from_spec(spec); spec.loader.exec_module(m)\n"
        "try:\n"
        "    m._cube(np.zeros(8))\n"
        "except ValueError:\n"
        "    pass\n"
        "else:\n"
        "    sys.exit('flat volume accepted')\n"
        "try:\n"
        "    m._out_array(np.empty(3), 4, 'x')\n"
        "except ValueError:\n"
        "    print('ok')\n")
    r = subprocess.run([sys.executable, "-O", "-c", script], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
