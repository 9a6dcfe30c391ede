"""Served form: Python handle of the library's device-resident request loop
(sincgpu_server_*).  Requests are copied at submit; results come back per id."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import _call, _f, load_library

_P, _I, _D = C.c_void_p, C.c_int, C.c_double


class _Request(C.Structure):
    _fields_ = [("numpoints", _I), ("spacing", _D), ("numcenters", _I), ("centershift", _P),
                ("nuccharges", _P), ("numspf", _I), ("numelec", _I), ("restrictms", _I),
                ("spinrestrictval", _I), ("npulses", _I), ("pulsetype", _P), ("pulseparams", _P),
                ("nsteps", _I), ("dt", _D), ("coulomb_fp32", _I), ("keep_state", _I), ("phi", _P),
                ("avector", _P)]


_SIGS = {
    "sincgpu_server_create": ([C.POINTER(_P), _I, C.c_longlong, _I], _I),
    "sincgpu_server_submit": ([_P, C.POINTER(_Request), C.POINTER(_I)], _I),
    "sincgpu_server_wait": ([_P, _I, _P, _P, _P, _P, _P], _I),
    "sincgpu_server_result_arrays": ([_P, _I, _P, _P, _P, _P], _I),
    "sincgpu_server_stats": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_server_timeline": ([_P, _I, _P, _P], _I),
    "sincgpu_server_destroy": ([_P], _I),
}


def _bind():
    lib = load_library()
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


class Server:
    """max_active worker slots; hbm_budget bytes (0: 85% of the free memory)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_active: int = 4):
        _bind()
        self._h = _P()
        _call("sincgpu_server_create", C.byref(self._h), int(device), int(hbm_budget), int(max_active))
        self._meta = {}

    def submit(self, numpoints, spacing, centershift, nuccharges, numspf, numelec, restrictms, phi, avector,
               nsteps, dt=0.05, pulses=(), coulomb_fp32=False, keep_state=False, spinrestrictval=-1) -> int:
        cs = np.ascontiguousarray(np.asarray(centershift, dtype=np.int32).reshape(-1))
        z = np.ascontiguousarray(np.asarray(nuccharges, dtype=np.float64).reshape(-1))
        ph = _f(phi)
        av = _f(avector).reshape(-1)
        pt = np.array([p.pulsetype for p in pulses] or [0], dtype=np.int32)
        pp = np.array([[p.omega, p.omega2, p.pulsestart, p.phaseshift, p.strength, p.longstep, p.pulsetheta, 0.0]
                       for p in pulses] or [[0.0] * 8], dtype=np.float64)
        r = _Request(int(numpoints), float(spacing), len(z), cs.ctypes.data, z.ctypes.data, int(numspf),
                     int(numelec), int(restrictms), int(spinrestrictval), len(pulses), pt.ctypes.data,
                     pp.ctypes.data, int(nsteps), float(dt), int(bool(coulomb_fp32)), int(bool(keep_state)),
                     ph.ctypes.data, av.ctypes.data)
        rid = _I(0)
        _call("sincgpu_server_submit", self._h, C.byref(r), C.byref(rid))
        self._meta[rid.value] = (ph.shape, av.size, int(nsteps), bool(keep_state))
        return rid.value

    def wait(self, rid: int) -> dict:
        e0, e, nn, d, ns = _D(), _D(), _D(), _D(), _I()
        _call("sincgpu_server_wait", self._h, int(rid), C.byref(e0), C.byref(e), C.byref(nn), C.byref(d),
              C.byref(ns))
        shape, nc, nsteps, keep = self._meta[rid]
        steps = np.zeros(max(ns.value, 1))
        energies = np.zeros(max(ns.value, 1))
        phi = np.zeros(shape, dtype=np.complex128, order="F") if keep else None
        av = np.zeros(nc, dtype=np.complex128) if keep else None
        _call("sincgpu_server_result_arrays", self._h, int(rid), steps.ctypes.data, energies.ctypes.data,
              None if phi is None else phi.ctypes.data, None if av is None else av.ctypes.data)
        times = np.zeros(4)
        starts = np.zeros(max(ns.value, 1))
        _call("sincgpu_server_timeline", self._h, int(rid), times.ctypes.data, starts.ctypes.data)
        return {"energy0": e0.value, "energy": e.value, "norm": nn.value, "dipole_z": d.value,
                "nsteps": ns.value, "step_ms": steps[:ns.value], "energies": energies[:ns.value],
                "phi": phi, "avector": av,
                "timeline_ms": dict(zip(("submitted", "admitted", "ready", "finished"), times.tolist())),
                "step_start_ms": starts[:ns.value]}

    def stats(self) -> dict:
        cnt = np.zeros(5, dtype=np.int64)
        p50, p99, sps = _D(), _D(), _D()
        _call("sincgpu_server_stats", self._h, cnt.ctypes.data, C.byref(p50), C.byref(p99), C.byref(sps))
        return {"admitted": int(cnt[0]), "completed": int(cnt[1]), "steps": int(cnt[2]),
                "peak_active": int(cnt[3]), "pending": int(cnt[4]), "p50_ms": p50.value, "p99_ms": p99.value,
                "steps_per_s": sps.value}

    def close(self):
        if self._h:
            load_library().sincgpu_server_destroy(self._h)
            self._h = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
