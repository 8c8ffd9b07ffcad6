"""Readers of the reference's particle files and dataset manifests.

The same inputs as the reference's tests and benchmarks (text snapshots in
charge-x-y-z or x-y-z-charge order with ESC rows for escaped particles, and
binary xyz frames), read by the library's native parser.  Escaped particles
come back as the escape coordinate (the largest double) on every axis.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C

CHARGE_XYZ, XYZ_CHARGE, BINARY_XYZ = 0, 1, 2
LAYOUTS = {"cxyz": CHARGE_XYZ, "xyzc": XYZ_CHARGE, "bin": BINARY_XYZ}
ESCAPED = np.finfo(np.float64).max


def read_particles(path: str, layout=CHARGE_XYZ):
    """(x, y, z) float64 arrays of a particle file."""
    if isinstance(layout, str):
        layout = LAYOUTS[layout]
    lib = C.load()
    px, py, pz, n = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_size_t()
    C.check(lib.ao_read_particles(str(path).encode(), int(layout), ctypes.byref(px), ctypes.byref(py),
                                  ctypes.byref(pz), ctypes.byref(n)))
    try:
        out = []
        for p in (px, py, pz):
            buf = (ctypes.c_double * n.value).from_address(p.value) if n.value else None
            out.append(np.array(buf, dtype=np.float64) if buf is not None else np.empty(0))
        return tuple(out)
    finally:
        for p in (px, py, pz):
            lib.ao_free(p)


def read_manifest(path: str) -> dict:
    """{'dataset', 'slots', 'box', 'frames': [{'index', 'id', 'layout', 'path'}]}."""
    lib = C.load()
    h = ctypes.c_void_p()
    C.check(lib.ao_read_manifest(str(path).encode(), ctypes.byref(h)))
    try:
        name, slots, frames = ctypes.c_char_p(), ctypes.c_size_t(), ctypes.c_size_t()
        box = (ctypes.c_double * 6)()
        C.check(lib.ao_manifest_info(h, ctypes.byref(name), ctypes.byref(slots), box, ctypes.byref(frames)))
        out = {"dataset": name.value.decode(), "slots": slots.value, "box": tuple(box), "frames": []}
        for i in range(frames.value):
            idx, fid, lay, fp = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int(), ctypes.c_char_p()
            C.check(lib.ao_manifest_frame(h, i, ctypes.byref(idx), ctypes.byref(fid), ctypes.byref(lay),
                                          ctypes.byref(fp)))
            out["frames"].append({"index": idx.value, "id": fid.value, "layout": lay.value,
                                  "path": fp.value.decode()})
        return out
    finally:
        lib.ao_manifest_destroy(h)


def read_frame(frame: dict):
    """(x, y, z) of one manifest frame."""
    return read_particles(frame["path"], frame["layout"])
