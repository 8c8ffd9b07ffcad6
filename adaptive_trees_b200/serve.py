"""Serving: requests to build, update and release trees, run concurrently.

The reference's callers build and update trees one at a time.  A Server
queues requests and runs them on worker threads; every resident tree keeps
its buffers and its own copy of its coordinates on the device and runs on
its own stream, so requests on different trees overlap on the GPU.  Builds
are admitted in arrival order when their memory fits the budget; requests on
one tree run in order.  Each request gives the result it gives alone.
"""
from __future__ import annotations

import ctypes

from . import _capi as C
from .tree import TreeConfig

BUILD, UPDATE, RELEASE = 0, 1, 2


def _ptr(t):
    return t.data_ptr() if t is not None and t.numel() else None


class Server:
    def __init__(self, slots: int = 8, memory_budget_bytes: int = 120 << 30):
        h = ctypes.c_void_p()
        C.check(C.load().ao_serve_create(int(slots), int(memory_budget_bytes), ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            C.load().ao_serve_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _submit(self, req: C.AoRequest) -> int:
        t = ctypes.c_longlong()
        C.check(C.load().ao_serve_submit(self._h, ctypes.byref(req), ctypes.byref(t)))
        return t.value

    def build(self, tree: int, x, y, z, config: TreeConfig | None = None, kind: int = 0, digest: bool = False):
        """Queues Tree<Real, kind>(x, y, z, config).build() as resident tree `tree`; returns a ticket."""
        import torch
        r = C.AoRequest()
        r.op, r.tree, r.kind = BUILD, int(tree), int(kind)
        r.real_type = 0 if x.dtype == torch.float32 else 1
        r.config = (config or TreeConfig()).to_c()
        r.n = x.numel()
        r.x, r.y, r.z = _ptr(x), _ptr(y), _ptr(z)
        r.want_digest = int(digest)
        return self._submit(r)

    def update(self, tree: int, x, y, z, digest: bool = False):
        """Queues an update() of resident tree `tree` on these coordinates."""
        r = C.AoRequest()
        r.op, r.tree, r.n = UPDATE, int(tree), x.numel()
        r.x, r.y, r.z = _ptr(x), _ptr(y), _ptr(z)
        r.want_digest = int(digest)
        return self._submit(r)

    def release(self, tree: int):
        r = C.AoRequest()
        r.op, r.tree = RELEASE, int(tree)
        return self._submit(r)

    def wait(self, ticket: int) -> dict:
        """Result of a request: status 0 on success, else an ao_status with its message."""
        res = C.AoRequestResult()
        st = C.load().ao_serve_wait(self._h, int(ticket), ctypes.byref(res))
        out = {k: getattr(res, k) for k, _ in C.AoRequestResult._fields_}
        out["status"] = st
        out["message"] = C.load().ao_last_error().decode() if st else ""
        return out

    def drain(self):
        C.check(C.load().ao_serve_drain(self._h))

    def stats(self) -> dict:
        s = C.AoServeStats()
        C.check(C.load().ao_serve_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in C.AoServeStats._fields_}

    def reset_stats(self):
        C.check(C.load().ao_serve_reset_stats(self._h))


def release_cached_memory():
    """Hands the device blocks kept for reuse back to the driver."""
    C.check(C.load().ao_release_cached_memory())
