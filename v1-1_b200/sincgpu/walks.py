"""Walk tables (determinant list, single/double walks, hops) from the C library.

Mirror of the reference's walktype (MCTDH.SRC/main_modules.f90:245-354) as numpy
arrays with the reference's 1-based values.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import _call, load_library

TABLES = {
    "configlist": 0, "numsinglewalks": 1, "numdoublewalks": 2, "singlewalkopspf": 3,
    "singlewalkdirphase": 4, "singlewalk": 5, "doublewalkdirspf": 6, "doublewalkdirphase": 7,
    "doublewalk": 8, "singlehop_off": 9, "singlehop": 10, "singlehopwalkstart": 11,
    "singlehopwalkend": 12, "doublehop_off": 13, "doublehop": 14, "doublehopwalkstart": 15,
    "doublehopwalkend": 16, "singlediaghop": 17, "doublediaghop": 18,
}


class WalkTables:
    """Owns a sincgpu_walks handle (host memory only; no GPU needed)."""

    def __init__(self, numelec: int, nspf: int, restrictms: int = 0, nthreads: int = 0):
        self.numelec, self.nspf, self.restrictms = int(numelec), int(nspf), int(restrictms)
        self._h = C.c_void_p()
        _call("sincgpu_walks_create", C.byref(self._h), self.numelec, self.nspf, self.restrictms, int(nthreads))
        s = np.zeros(6, dtype=np.int64)
        _call("sincgpu_walks_sizes", self._h, s.ctypes.data, 6)
        (self.numconfig, self.numpart, self.totsinglewalks, self.totdoublewalks,
         self.totsinglehops, self.totdoublehops) = (int(v) for v in s)

    def close(self):
        if self._h:
            load_library().sincgpu_walks_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _len(self, name):
        nc, sw, dw, sh, dh = (self.numconfig, self.totsinglewalks, self.totdoublewalks,
                              self.totsinglehops, self.totdoublehops)
        return {
            "configlist": 2 * self.numpart * nc, "numsinglewalks": nc, "numdoublewalks": nc,
            "singlewalkopspf": 2 * sw, "singlewalkdirphase": sw, "singlewalk": sw,
            "doublewalkdirspf": 4 * dw, "doublewalkdirphase": dw, "doublewalk": dw,
            "singlehop_off": nc + 1, "singlehop": sh, "singlehopwalkstart": sh, "singlehopwalkend": sh,
            "doublehop_off": nc + 1, "doublehop": dh, "doublehopwalkstart": dh, "doublehopwalkend": dh,
            "singlediaghop": nc, "doublediaghop": nc,
        }[name]

    def table(self, name: str) -> np.ndarray:
        out = np.zeros(max(self._len(name), 1), dtype=np.int32)
        _call("sincgpu_walks_table", self._h, TABLES[name], out.ctypes.data)
        out = out[: self._len(name)]
        if name == "configlist":
            return out.reshape(self.numconfig, 2 * self.numpart)
        if name == "singlewalkopspf":
            return out.reshape(-1, 2)
        if name == "doublewalkdirspf":
            return out.reshape(-1, 4)
        return out
