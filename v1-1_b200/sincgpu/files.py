"""Orbital and A-vector files in the reference's format (gfortran unformatted
sequential records), through the C library; host arrays only."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .capi import _call, _f, _ptr


def save_spfs(path, spfs, dims):
    """spfs: (totpoints, numspf) complex, Fortran order; dims = spfdims(3)."""
    a = _f(spfs)
    d = np.asarray(dims, dtype=np.int32)
    _call("sincgpu_save_spfs", os.fsencode(path), _ptr(d), int(a.shape[1]), _ptr(a))


def load_spfs(path):
    """Returns (spfs (totpoints, numspf), dims)."""
    d = np.zeros(3, dtype=np.int32)
    n = C.c_int(0)
    _call("sincgpu_load_spfs", os.fsencode(path), _ptr(d), C.byref(n), None, 0)
    g = int(np.prod(d.astype(np.int64)))
    out = np.zeros((g, n.value), dtype=np.complex128, order="F")
    _call("sincgpu_load_spfs", os.fsencode(path), _ptr(d), C.byref(n), _ptr(out), out.size)
    return out, tuple(int(x) for x in d)


def save_avector(path, walks, avectors, allspinproject=1, spinrestrictval=None):
    """avectors: (numconfig,) or (numconfig, numvects) complex."""
    a = _f(avectors)
    if a.ndim == 1:
        a = a.reshape(-1, 1, order="F")
    srv = abs(walks.restrictms) if spinrestrictval is None else int(spinrestrictval)
    _call("sincgpu_save_avector", os.fsencode(path), walks._h, int(a.shape[1]), _ptr(a), int(allspinproject), srv)


def load_avector(path, walks, maxvects=1):
    """Returns (numconfig, numvects) complex."""
    out = np.zeros((walks.numconfig, maxvects), dtype=np.complex128, order="F")
    nv = C.c_int(0)
    _call("sincgpu_load_avector", os.fsencode(path), walks._h, int(maxvects), _ptr(out), C.byref(nv))
    return out[:, : nv.value]
