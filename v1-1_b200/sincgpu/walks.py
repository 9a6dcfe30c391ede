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
    "numspinwalks": 19, "spinwalk": 20, "spinwalkdirphase": 21, "spinset_off": 22, "spinsets": 23,
    "spinsetrank": 24, "spin_eliminated": 25,
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

    def build_spin(self, spinrestrictval: int = -1):
        """Spin walks, sets and S^2 projectors (allspinproject=1); 2S defaults to |restrictms|."""
        _call("sincgpu_walks_spin", self._h, int(spinrestrictval))
        s = np.zeros(6, dtype=np.int64)
        _call("sincgpu_walks_spin_sizes", self._h, s.ctypes.data, 6)
        (self.numspinsets, self.numspinconfig, self.totspinwalks, self.spinprojsize, self.numspinelim,
         self.maxspinsetsize) = (int(v) for v in s)
        return self

    def spin_projectors(self) -> list[np.ndarray]:
        flat = np.zeros(max(self.spinprojsize, 1))
        _call("sincgpu_walks_spinprojectors", self._h, flat.ctypes.data)
        off = self.table("spinset_off")
        out, p = [], 0
        for k in range(self.numspinsets):
            m = int(off[k + 1] - off[k])
            out.append(flat[p:p + m * m].reshape(m, m))
            p += m * m
        return out

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
            "numspinwalks": nc, "spinwalk": getattr(self, "totspinwalks", 0),
            "spinwalkdirphase": getattr(self, "totspinwalks", 0),
            "spinset_off": getattr(self, "numspinsets", -1) + 1,
            "spinsets": nc - getattr(self, "numspinelim", nc), "spinsetrank": getattr(self, "numspinsets", 0),
            "spin_eliminated": getattr(self, "numspinelim", 0),
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
