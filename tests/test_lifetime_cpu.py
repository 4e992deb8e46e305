"""Python-side resource lifetime, on the CPU against a fake of the C library:
a context closes the resources still open in it before destroying itself (the
C library frees them through their context), a resource closed after its
context makes no C call, and the exit hook closes servers before contexts."""
import pytest

from conftest import load_package

wrt = load_package()


class FakeLib:
    def __init__(self):
        self.calls = []
        self.next = 100

    def _out(self, ref):
        self.next += 1
        ref._obj.value = self.next
        return 0

    def wrt_ctx_create(self, dev, budget, out):
        self.calls.append("ctx_create")
        return self._out(out)

    def wrt_ctx_destroy(self, h):
        self.calls.append("ctx_destroy")
        return 0

    def wrt_device_alloc(self, h, n, out):
        self.calls.append("alloc")
        return self._out(out)

    def wrt_device_free(self, h, p):
        self.calls.append("free")
        return 0

    def wrt_volume_create_storage(self, h, n, storage, out):
        self.calls.append("volume_create")
        return self._out(out)

    def wrt_volume_destroy(self, h):
        self.calls.append("volume_destroy")
        return 0

    def wrt_grid_create(self, h, a, b, c, out):
        self.calls.append("grid_create")
        return self._out(out)

    def wrt_grid_destroy(self, h):
        self.calls.append("grid_destroy")
        return 0

    def wrt_server_create(self, opts, out):
        self.calls.append("server_create")
        return self._out(out)

    def wrt_server_destroy(self, h):
        self.calls.append("server_destroy")
        return 0


@pytest.fixture
def fake(monkeypatch):
    f = FakeLib()
    monkeypatch.setattr(wrt, "_lib", f)
    yield f


def test_context_closes_its_resources_first(fake):
    ctx = wrt.Context(0)
    buf = wrt.DeviceBuffer(ctx, 64)
    vol = wrt.Volume(ctx, 8)
    grid = wrt.Grid(ctx, 2, 2, 2)
    ctx.close()
    assert fake.calls[-1] == "ctx_destroy"
    assert sorted(fake.calls[-4:-1]) == ["free", "grid_destroy", "volume_destroy"]
    n = len(fake.calls)
    buf.close(), vol.close(), grid.close(), ctx.close()
    assert len(fake.calls) == n  # nothing freed twice, nothing through a dead context


def test_resource_closed_before_context(fake):
    ctx = wrt.Context(0)
    vol = wrt.Volume(ctx, 8)
    vol.close()
    ctx.close()
    assert fake.calls == ["ctx_create", "volume_create", "volume_destroy", "ctx_destroy"]


def test_exit_hook_closes_servers_then_contexts(fake):
    ctx = wrt.Context(0)
    srv = wrt.Server(0)
    buf = wrt.DeviceBuffer(ctx, 16)  # left open, owned by the context
    wrt._close_all()
    tail = fake.calls[-3:]
    assert tail == ["server_destroy", "free", "ctx_destroy"]
    assert not ctx.handle and not srv._h and not buf._p
