"""ctypes binding of libsincgpu.so and the SincProject host mirror."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
_REPO = _PKG.parent.parent
_HEADER = _REPO / "include" / "sincgpu.h"
_lib = None


class SincGpuError(RuntimeError):
    """Raised when a library call returns a non-zero status."""

    def __init__(self, code: int, func: str, msg: str):
        super().__init__(f"{func} failed with status {code}: {msg}")
        self.code = code


def library_path() -> Path:
    return _PKG / "libsincgpu.so"


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_LL = C.c_longlong

_SIGS = {
    "sincgpu_last_error": ([], C.c_char_p),
    "sincgpu_version": ([], _I),
    "sincgpu_create": ([C.POINTER(_P), _I, _D, _I, _P, _P, _I, _I, _I, _I, _I], _I),
    "sincgpu_create_from_tables": ([C.POINTER(_P), _I, _D, _I, _P, _P, _I], _I),
    "sincgpu_destroy": ([_P], _I),
    "sincgpu_get_tables": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_fft_length": ([_P], _I),
    "sincgpu_set_option": ([_P, C.c_char_p, _LL], _I),
    "sincgpu_get_option": ([_P, C.c_char_p, _P], _I),
    "sincgpu_synchronize": ([_P], _I),
    "sincgpu_host_register": ([_P, _LL], _I),
    "sincgpu_host_unregister": ([_P], _I),
    "sincgpu_call_twoe_matel00": ([_P, _I, _I, _P, _P, _P, _P], _I),
    "sincgpu_op_tinv": ([_P, _P, _P, _I, _I], _I),
    "sincgpu_mult_ke": ([_P, _P, _P, _I], _I),
    "sincgpu_mult_reducedpot": ([_P, _I, _I, _P, _P, _P], _I),
    "sincgpu_get_reducedpot": ([_P, _P, _P, _P], _I),
    "sincgpu_actreduced00": ([_P, _I, _P, _P, _P, _P, _P, _D, _D, _I, _D, _P], _I),
    "sincgpu_twoe_matel_dev": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_mult_ke_dev": ([_P, _P, _P, _I], _I),
    "sincgpu_mult_reducedpot_dev": ([_P, _P, _P, _P], _I),
    "sincgpu_mean_field_dev": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_op_tinv_noalloc_dev": ([_P, _P, _P, _I], _I),
    "sincgpu_actreduced_dev": ([_P, _I, _P, _P, _P, _P, _P, _D, _D, _I, _D, _P], _I),
    "sincgpu_set_stream": ([_P, _P], _I),
    "sincgpu_launch_count": ([], _LL),
    "sincgpu_walks_create": ([C.POINTER(_P), _I, _I, _I, _I], _I),
    "sincgpu_walks_destroy": ([_P], _I),
    "sincgpu_walks_sizes": ([_P, _P, _I], _I),
    "sincgpu_walks_table": ([_P, _I, _P], _I),
    "sincgpu_ci_attach": ([_P, _P], _I),
    "sincgpu_getdenmat": ([_P, _P, _P, _P], _I),
    "sincgpu_get_tworeducedx": ([_P, _P, _P, _P], _I),
    "sincgpu_onebody_matel": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_assemble_sparsemats": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_sparseconfigmult": ([_P, _P, _P, _D], _I),
    "sincgpu_getdenmat_dev": ([_P, _P, _P, _P, _D], _I),
    "sincgpu_get_tworeducedx_dev": ([_P, _P, _P, _P], _I),
    "sincgpu_onebody_matel_dev": ([_P, _P, _P], _I),
    "sincgpu_assemble_sparsemats_dev": ([_P, _P, _P], _I),
    "sincgpu_sparseconfigmult_dev": ([_P, _P, _P, _D], _I),
    "sincgpu_orbital_rhs_avec_dev": ([_P, _P, _P, _D, _D, _D, _P, _P, _P, _P, _P, _P], _I),
    "sincgpu_orbital_rhs_avec": ([_P, _P, _P, _D, _D, _D, _P], _I),
    "sincgpu_expoavecprop_dev": ([_P, _P, _P, _D, _D, _D, _I, _D, _D, _D, _P, _P], _I),
    "sincgpu_expoavecprop": ([_P, _P, _P, _D, _D, _D, _I, _D, _D, _D, _P, _P], _I),
    "sincgpu_profile": ([_P, _I], _I),
    "sincgpu_profile_read": ([_P, _P, _P, _I], _I),
    "sincgpu_orbital_rhs_dev": ([_P, _P, _P, _P, _P, _D, _D, _D, _P, _P, _P], _I),
    "sincgpu_orbital_rhs": ([_P, _P, _P, _P, _P, _D, _D, _D, _P, _P], _I),
    "sincgpu_expospfprop_dev": ([_P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _D, _D, _I, _D, _D, _D, _D, _P], _I),
    "sincgpu_orbprop_setup": ([_P, _I, _I, _D, _D], _I),
    "sincgpu_orbprop_state": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_spf_orthogit_dev": ([_P, _P, _P], _I),
    "sincgpu_walks_spin": ([_P, _I], _I),
    "sincgpu_walks_spin_sizes": ([_P, _P, _I], _I),
    "sincgpu_walks_spinprojectors": ([_P, _P], _I),
    "sincgpu_spin_project_dev": ([_P, _P], _I),
    "sincgpu_spin_project": ([_P, _P, _P], _I),
    "sincgpu_cmf_setup": ([_P, _D, _I, _D, _D, _I, _I, _I, _I, _D, _D, _D, _D], _I),
    "sincgpu_cmf_pulses": ([_P, _I, _P, _P], _I),
    "sincgpu_pulse_ez": ([_P, _D, _P], _I),
    "sincgpu_cmf_init_dev": ([_P, _P, _P, _P], _I),
    "sincgpu_cmf_step": ([_P, _D, _D, _P, _P, _P, _P], _I),
    "sincgpu_cmf_state_dev": ([_P, _P, _P], _I),
    "sincgpu_dipole_z_dev": ([_P, _P, _P, _P], _I),
    "sincgpu_dipole_z": ([_P, _P, _P, _P], _I),
    "sincgpu_cmf_dipole_z": ([_P, _P, _P], _I),
    "sincgpu_rhs_graph_capture": ([_P, _P, _P, _D, _D, _D, _P, _P, _P, _P, _P, _P], _I),
    "sincgpu_rhs_graph_launch": ([_P], _I),
    "sincgpu_batch_create": ([C.POINTER(_P), _P, _I], _I),
    "sincgpu_batch_launch": ([_P, _P], _I),
    "sincgpu_batch_destroy": ([_P], _I),
    "sincgpu_autotune_rhs": ([_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "sincgpu_set_sync_mode": ([_I, _I], _I),
    "sincgpu_gemm_tf32x3_dev": ([_P, _P, _P, _P, _LL, _I, _I, _P], _I),
    "sincgpu_kernel_timeouts": ([_P, _P], _I),
    "sincgpu_server_create": ([C.POINTER(_P), _I, _LL, _I], _I),
    "sincgpu_server_submit": ([_P, _P, _P], _I),
    "sincgpu_server_wait": ([_P, _I, _P, _P, _P, _P, _P], _I),
    "sincgpu_server_result_arrays": ([_P, _I, _P, _P, _P, _P], _I),
    "sincgpu_server_stats": ([_P, _P, _P, _P, _P], _I),
    "sincgpu_server_timeline": ([_P, _I, _P, _P], _I),
    "sincgpu_server_destroy": ([_P], _I),
    "sincgpu_save_spfs": ([C.c_char_p, _P, _I, _P], _I),
    "sincgpu_load_spfs": ([C.c_char_p, _P, _P, _P, _LL], _I),
    "sincgpu_save_avector": ([C.c_char_p, _P, _I, _P, _I, _I], _I),
    "sincgpu_load_avector": ([C.c_char_p, _P, _I, _P, _P], _I),
}


class Batch:
    """Captured orbital-RHS graphs of several SincProjects launched as one graph."""

    def __init__(self, projects):
        arr = (_P * len(projects))(*[p._h for p in projects])
        self._h = _P()
        self._keep = list(projects)
        _call("sincgpu_batch_create", C.byref(self._h), arr, len(projects))

    def launch(self, stream_handle: int = 0):
        _call("sincgpu_batch_launch", self._h, _P(stream_handle))

    def close(self):
        if self._h:
            load_library().sincgpu_batch_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exported_symbols() -> list[str]:
    """Function names declared in include/sincgpu.h."""
    text = _HEADER.read_text()
    return sorted(set(re.findall(r"\b(sincgpu_[a-z0-9_]+)\s*\(", text)))


def load_library(path: str | Path | None = None):
    """Loads libsincgpu.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else library_path()
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with __graft_entry__.build() "
                          "(nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(str(p))
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def _call(name, *args):
    lib = load_library()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.sincgpu_last_error().decode(errors="replace")
        raise SincGpuError(rc, name, msg)


def _f(a, dtype=np.complex128):
    """Fortran-ordered contiguous copy (or view) of `a` with the given dtype."""
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def _ptr(a) -> int:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class SincProject:
    """One sinc-DVR system on one GPU (the SINCDVR project state).

    Host methods take numpy arrays with the reference's Fortran shapes and
    return numpy arrays; ``*_dev`` methods take CUDA tensors (complex128,
    Fortran layout flattened as columns) and run on the context stream.
    """

    def __init__(self, numpoints, spacing, centershift, nuccharges, numspf,
                 toothnbig=240, toothnsmall=40, sqrt32=False, notwoflag=False, device=0,
                 _handle=None):
        self.N = int(numpoints)
        self.G = self.N ** 3
        self.nspf = int(numspf)
        self.spacing = float(spacing)
        self._h = C.c_void_p()
        if _handle is not None:
            self._h = _handle
            return
        cs = np.ascontiguousarray(np.asarray(centershift, dtype=np.int32).reshape(-1, 3))
        z = np.ascontiguousarray(np.asarray(nuccharges, dtype=np.float64).reshape(-1))
        if cs.shape[0] != z.shape[0]:
            raise ValueError("centershift and nuccharges disagree on the number of centers")
        flags = (1 if sqrt32 else 0) | (2 if notwoflag else 0)
        _call("sincgpu_create", C.byref(self._h), self.N, self.spacing, int(z.shape[0]),
              _ptr(cs), _ptr(z), self.nspf, int(toothnbig), int(toothnsmall), flags, int(device))

    @classmethod
    def from_tables(cls, numpoints, spacing, numspf, threed_two, pot, device=0):
        """Context from the reference's own threed_two((2N)^3) and pot(G)."""
        h = C.c_void_p()
        t2 = _f(threed_two).reshape(-1, order="F")
        pt = _f(pot, np.float64).reshape(-1, order="F")
        _call("sincgpu_create_from_tables", C.byref(h), int(numpoints), float(spacing),
              int(numspf), _ptr(t2), _ptr(pt), int(device))
        return cls(numpoints, spacing, None, None, numspf, _handle=h)

    def close(self):
        if self._h:
            load_library().sincgpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ setup
    @property
    def fft_length(self) -> int:
        return load_library().sincgpu_fft_length(self._h)

    def set_option(self, name: str, value: int):
        _call("sincgpu_set_option", self._h, name.encode(), int(value))

    def get_option(self, name: str) -> int:
        v = C.c_longlong(0)
        _call("sincgpu_get_option", self._h, name.encode(), C.byref(v))
        return v.value

    def synchronize(self):
        _call("sincgpu_synchronize", self._h)

    def set_stream(self, stream_handle: int):
        """Enqueue on a caller-owned CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        _call("sincgpu_set_stream", self._h, C.c_void_p(int(stream_handle)))

    @staticmethod
    def launch_count() -> int:
        return int(load_library().sincgpu_launch_count())

    STAGES = ("coul_fwd_x", "coul_fwd_y", "coul_z", "coul_inv_y", "coul_inv_x", "twoe_gemm",
              "twoe_finish", "rp_w", "rp_gemm", "ke_xy", "ke_z", "rhs_mix", "rhs_redpot",
              "rhs_proj", "ci", "other", "coul_yzy")

    def profile(self, enable: bool = True):
        _call("sincgpu_profile", self._h, 1 if enable else 0)

    def profile_read(self) -> dict:
        """{stage: (milliseconds, launches)} since the last read."""
        ms = np.zeros(len(self.STAGES))
        n = np.zeros(len(self.STAGES), dtype=np.int64)
        _call("sincgpu_profile_read", self._h, _ptr(ms), _ptr(n), len(self.STAGES))
        return {s: (float(ms[i]), int(n[i])) for i, s in enumerate(self.STAGES) if n[i]}

    def get_tables(self):
        W = 2 * self.N - 1
        t = np.zeros((W, W, W), order="F")
        pot = np.zeros(self.G)
        ke = np.zeros(W)
        nr = C.c_double()
        _call("sincgpu_get_tables", self._h, _ptr(t), _ptr(pot), _ptr(ke), C.byref(nr))
        return {"tempcoulomb": t, "pot": pot, "kevect": ke, "nucrepulsion": nr.value}

    # ----------------------------------------------------- host drop-ins
    def call_twoe_matel00(self, inspfs10, inspfs20=None, lowspf=1, highspf=None):
        """SINCDVR/coreproject.f90:945-1194 -> (twoematel(n,n,n,n), twoereduced(G,n,n))."""
        n = self.nspf
        highspf = n if highspf is None else highspf
        a = _f(inspfs10)
        b = a if inspfs20 is None else _f(inspfs20)
        mat = np.zeros((n, n, n, n), dtype=np.complex128, order="F")
        red = np.zeros((self.G, n, n), dtype=np.complex128, order="F")
        _call("sincgpu_call_twoe_matel00", self._h, int(lowspf), int(highspf), _ptr(a), _ptr(b),
              _ptr(mat), _ptr(red))
        return mat, red

    def op_tinv(self, twoeden03, circsize=None):
        """SINCDVR/coreproject.f90:250-539."""
        d = _f(twoeden03).reshape(self.G, -1, order="F")
        m = d.shape[1]
        out = np.zeros((self.G, m), dtype=np.complex128, order="F")
        _call("sincgpu_op_tinv", self._h, _ptr(d), _ptr(out), m, int(circsize or max(m, 1)))
        return out

    def mult_ke(self, inp):
        """SINCDVR/coreproject.f90:2104-2116."""
        d = _f(inp).reshape(self.G, -1, order="F")
        out = np.zeros_like(d, order="F")
        _call("sincgpu_mult_ke", self._h, _ptr(d), _ptr(out), d.shape[1])
        return out

    def mult_reducedpot(self, inspfs, reducedpot, firstspf=1, lastspf=None):
        """SINCDVR/coreproject.f90:1200-1235; reducedpot(G,n,firstspf:lastspf)."""
        lastspf = self.nspf if lastspf is None else lastspf
        ni = lastspf - firstspf + 1
        phi = _f(inspfs)
        v = _f(reducedpot)
        out = np.zeros((self.G, max(ni, 0)), dtype=np.complex128, order="F")
        _call("sincgpu_mult_reducedpot", self._h, int(firstspf), int(lastspf), _ptr(phi), _ptr(out), _ptr(v))
        return out

    def get_reducedpot(self, twoereduced, reducedpottally):
        """MCTDH.SRC/mean.f90:503-588."""
        n = self.nspf
        r = _f(twoereduced)
        t = _f(reducedpottally)
        out = np.zeros((self.G, n, n), dtype=np.complex128, order="F")
        _call("sincgpu_get_reducedpot", self._h, _ptr(r), _ptr(t), _ptr(out))
        return out

    def actreduced00(self, inspfs, projspfs, denmat, invdenmat, reducedpot, timefac=-1j,
                     dentimeflag=1, projflag=1, ztdpot=0.0):
        """MCTDH.SRC/derivs.f90:629-852 (sinc project, length gauge)."""
        phi = _f(inspfs)
        proj = _f(projspfs) if projspfs is not None else None
        dm = _f(denmat)
        inv = _f(invdenmat) if invdenmat is not None else None
        v = _f(reducedpot)
        out = np.zeros((self.G, self.nspf), dtype=np.complex128, order="F")
        tf = complex(timefac)
        _call("sincgpu_actreduced00", self._h, int(dentimeflag), _ptr(phi), _ptr(proj), _ptr(dm),
              _ptr(inv), _ptr(v), tf.real, tf.imag, int(projflag), float(ztdpot), _ptr(out))
        return out

    # ------------------------------------------------------------ CI side
    def ci_attach(self, walks):
        """Uploads the walk tables (sincgpu.WalkTables) to this context's device."""
        _call("sincgpu_ci_attach", self._h, walks._h)
        self.numconfig = walks.numconfig

    def getdenmat(self, avector):
        """MCTDH.SRC/denmat.f90:312-378 -> (denmat(n,n), invdenmat(n,n))."""
        n = self.nspf
        a = _f(avector).reshape(-1)
        den = np.zeros((n, n), dtype=np.complex128, order="F")
        inv = np.zeros((n, n), dtype=np.complex128, order="F")
        _call("sincgpu_getdenmat", self._h, _ptr(a), _ptr(den), _ptr(inv))
        return den, inv

    def get_tworeducedx(self, avector1, avector2=None):
        """MCTDH.SRC/mean.f90:14-152 -> reducedpottally(n,n,n,n)."""
        n = self.nspf
        a1 = _f(avector1).reshape(-1)
        a2 = a1 if avector2 is None else _f(avector2).reshape(-1)
        t = np.zeros((n, n, n, n), dtype=np.complex128, order="F")
        _call("sincgpu_get_tworeducedx", self._h, _ptr(a1), _ptr(a2), _ptr(t))
        return t

    def onebody_matel(self, phi):
        """(potmatel, kematel, zmatel), each <phi_i|op|phi_j> (n,n)."""
        n = self.nspf
        p = _f(phi)
        mats = [np.zeros((n, n), dtype=np.complex128, order="F") for _ in range(3)]
        _call("sincgpu_onebody_matel", self._h, _ptr(p), *(_ptr(m) for m in mats))
        return tuple(mats)

    def assemble_sparsemats(self, twoematel, potmatel, kematel, zmatel):
        # keep the converted arrays alive until the call returns
        arrs = [_f(twoematel), _f(potmatel), _f(kematel), _f(zmatel)]
        _call("sincgpu_assemble_sparsemats", self._h, *(_ptr(a) for a in arrs))

    def sparseconfigmult(self, invector, ezfield=0.0):
        """MCTDH.SRC/walkmult.f90:735-907 (sparseopt=1)."""
        a = _f(invector).reshape(-1)
        out = np.zeros_like(a)
        _call("sincgpu_sparseconfigmult", self._h, _ptr(a), _ptr(out), float(ezfield))
        return out

    def expoavecprop(self, avector, t, krylovdim=20, tol=1e-9, anorm=1.0, stepguess=None, timefac=-1j,
                     ezfield=0.0):
        """A-vector Krylov step (expo_driver.f90:827-1055): returns (avec_out, stepguess, nstep)."""
        a = _f(avector).reshape(-1)
        out = np.zeros_like(a)
        g = C.c_double(t if stepguess is None else stepguess)
        ns = C.c_int(0)
        tf = complex(timefac)
        _call("sincgpu_expoavecprop", self._h, _ptr(a), _ptr(out), float(t), tf.real, tf.imag, int(krylovdim),
              float(tol), float(anorm), float(ezfield), C.byref(g), C.byref(ns))
        return out, g.value, ns.value

    # ------------------------------------------------ orbital propagation
    def orbprop_setup(self, expodim=10, maxexpodim=100, expostepfac=1.2, first_stepsize=0.1):
        _call("sincgpu_orbprop_setup", self._h, int(expodim), int(maxexpodim), float(expostepfac),
              float(first_stepsize))

    def orbprop_state(self) -> dict:
        d, s, e, i = C.c_int(0), C.c_double(0.0), C.c_int(0), C.c_int(0)
        _call("sincgpu_orbprop_state", self._h, C.byref(d), C.byref(s), C.byref(e), C.byref(i))
        return {"thisexpodim": d.value, "tempstepsize": s.value, "exposet": e.value, "icalled": i.value}

    def expospfprop_dev(self, phi, slot0, slot1, tin, tout, firsttime, lasttime, linear=True, timefac=-1j,
                        ezfield=0.0, expotol=1e-8) -> int:
        """phi (device, advanced in place); slots are (denmat, invdenmat, reducedpot)
        device tensors.  Returns the number of Jacobian products."""
        tf = complex(timefac)
        s1 = slot1 if slot1 is not None else (None, None, None)
        it = C.c_int(0)
        _call("sincgpu_expospfprop_dev", self._h, _ptr(phi), _ptr(slot0[0]), _ptr(slot0[1]), _ptr(slot0[2]),
              _ptr(s1[0]), _ptr(s1[1]), _ptr(s1[2]), float(tin), float(tout), float(firsttime),
              float(lasttime), 1 if linear else 0, tf.real, tf.imag, float(ezfield), float(expotol),
              C.byref(it))
        return it.value

    def spf_orthogit_dev(self, phi) -> float:
        e = C.c_double(0.0)
        _call("sincgpu_spf_orthogit_dev", self._h, _ptr(phi), C.byref(e))
        return e.value

    # ------------------------------------------------- CMF propagation
    def cmf_setup(self, par_timestep=0.05, littlesteps=1, expotol=1e-8, aerror=1e-9, aorder=30, maxaorder=100,
                  expodim=10, maxexpodim=100, expostepfac=1.2, denreg=1e-10, timefac=-1j):
        tf = complex(timefac)
        _call("sincgpu_cmf_setup", self._h, float(par_timestep), int(littlesteps), float(expotol), float(aerror),
              int(aorder), int(maxaorder), int(expodim), int(maxexpodim), float(expostepfac), float(denreg),
              tf.real, tf.imag)

    def cmf_pulses(self, pulses):
        """pulses: objects with pulsetype, omega, omega2, pulsestart, phaseshift, strength,
        longstep, pulsetheta (oracle.cmf_oracle.Pulse has these fields)."""
        types = np.array([p.pulsetype for p in pulses] or [0], dtype=np.int32)
        par = np.array([[p.omega, p.omega2, p.pulsestart, p.phaseshift, p.strength, p.longstep, p.pulsetheta, 0.0]
                        for p in pulses] or [[0.0] * 8], dtype=np.float64)
        _call("sincgpu_cmf_pulses", self._h, len(pulses), _ptr(types), _ptr(par))

    def pulse_ez(self, t) -> float:
        e = C.c_double(0.0)
        _call("sincgpu_pulse_ez", self._h, float(t), C.byref(e))
        return e.value

    def cmf_init_dev(self, phi, avector) -> float:
        e = C.c_double(0.0)
        _call("sincgpu_cmf_init_dev", self._h, _ptr(phi), _ptr(avector), C.byref(e))
        return e.value

    def cmf_step(self, tin, tout) -> dict:
        e, nrm, oi, ai = C.c_double(0.0), C.c_double(0.0), C.c_int(0), C.c_int(0)
        _call("sincgpu_cmf_step", self._h, float(tin), float(tout), C.byref(e), C.byref(nrm), C.byref(oi),
              C.byref(ai))
        return {"energy": e.value, "norm": nrm.value, "orb_iters": oi.value, "avec_iters": ai.value}

    def cmf_state_dev(self, phi=None, avector=None):
        _call("sincgpu_cmf_state_dev", self._h, _ptr(phi), _ptr(avector))

    def dipole_z(self, avector):
        """(<A|Z A> + nucdip <A|A> as complex, <A|A>) with the assembled CI matrices."""
        a = _f(avector).reshape(-1)
        d = np.zeros(2)
        nn = C.c_double(0.0)
        _call("sincgpu_dipole_z", self._h, _ptr(a), _ptr(d), C.byref(nn))
        return complex(d[0], d[1]), nn.value

    def cmf_dipole_z(self):
        d = np.zeros(2)
        nn = C.c_double(0.0)
        _call("sincgpu_cmf_dipole_z", self._h, _ptr(d), C.byref(nn))
        return complex(d[0], d[1]), nn.value

    # ------------------------------------------------------- graphs
    def rhs_graph_capture(self, phi, avector, denmat, invdenmat, tally, twoematel, reducedpot, out,
                          timefac=-1j, ztdpot=0.0):
        tf = complex(timefac)
        _call("sincgpu_rhs_graph_capture", self._h, _ptr(phi), _ptr(avector), tf.real, tf.imag, float(ztdpot),
              _ptr(denmat), _ptr(invdenmat), _ptr(tally), _ptr(twoematel), _ptr(reducedpot), _ptr(out))

    def rhs_graph_launch(self):
        _call("sincgpu_rhs_graph_launch", self._h)

    def autotune_rhs(self, phi, avector, denmat, invdenmat, tally, twoematel, reducedpot, out):
        ch, ms = C.c_int(0), C.c_float(0.0)
        _call("sincgpu_autotune_rhs", self._h, _ptr(phi), _ptr(avector), _ptr(denmat), _ptr(invdenmat),
              _ptr(tally), _ptr(twoematel), _ptr(reducedpot), _ptr(out), C.byref(ch), C.byref(ms))
        return ch.value, ms.value

    def spin_project(self, avector):
        """basis_project (allspinproject=1) of a host A-vector; returns the projection."""
        a = _f(avector).reshape(-1)
        out = np.zeros_like(a)
        _call("sincgpu_spin_project", self._h, _ptr(a), _ptr(out))
        return out

    def spin_project_dev(self, avector):
        _call("sincgpu_spin_project_dev", self._h, _ptr(avector))

    def getdenmat_dev(self, avector, denmat, invdenmat, denreg=1e-10):
        _call("sincgpu_getdenmat_dev", self._h, _ptr(avector), _ptr(denmat), _ptr(invdenmat), float(denreg))

    def get_tworeducedx_dev(self, avector1, avector2, tally):
        _call("sincgpu_get_tworeducedx_dev", self._h, _ptr(avector1), _ptr(avector2), _ptr(tally))

    def onebody_matel_dev(self, phi, mats):
        _call("sincgpu_onebody_matel_dev", self._h, _ptr(phi), _ptr(mats))

    def assemble_sparsemats_dev(self, twoematel, mats):
        _call("sincgpu_assemble_sparsemats_dev", self._h, _ptr(twoematel), _ptr(mats))

    def sparseconfigmult_dev(self, invector, outvector, ezfield=0.0):
        _call("sincgpu_sparseconfigmult_dev", self._h, _ptr(invector), _ptr(outvector), float(ezfield))

    def orbital_rhs_avec(self, phi, avector, timefac=-1j, ztdpot=0.0):
        """Host arrays: orbitals (G,n) and A-vector in, orbital RHS (G,n) out."""
        p = _f(phi)
        a = _f(avector).reshape(-1)
        out = np.zeros((self.G, self.nspf), dtype=np.complex128, order="F")
        tf = complex(timefac)
        _call("sincgpu_orbital_rhs_avec", self._h, _ptr(p), _ptr(a), tf.real, tf.imag, float(ztdpot), _ptr(out))
        return out

    def orbital_rhs_avec_dev(self, phi, avector, denmat, invdenmat, tally, twoematel, reducedpot, out,
                             timefac=-1j, ztdpot=0.0):
        tf = complex(timefac)
        _call("sincgpu_orbital_rhs_avec_dev", self._h, _ptr(phi), _ptr(avector), tf.real, tf.imag,
              float(ztdpot), _ptr(denmat), _ptr(invdenmat), _ptr(tally), _ptr(twoematel),
              _ptr(reducedpot), _ptr(out))

    # --------------------------------------------------- device-resident
    def twoe_matel_dev(self, phi1, phi2, twoematel, twoereduced=None):
        _call("sincgpu_twoe_matel_dev", self._h, _ptr(phi1), _ptr(phi2), _ptr(twoematel), _ptr(twoereduced))

    def gemm_tf32x3_dev(self, a, b, out) -> int:
        """out = a b^T on the tensor cores (3xTF32, FP32 accumulation); a (M, K),
        b (N, K), out (M, N) row-major float64 device tensors.  Returns the
        timeout flag (0 when the MMAs completed)."""
        m, k = a.shape
        t = _I(0)
        _call("sincgpu_gemm_tf32x3_dev", self._h, _ptr(a), _ptr(b), _ptr(out), int(m), int(b.shape[0]), int(k),
              C.byref(t))
        return t.value

    def kernel_timeouts(self) -> list:
        """[tensor-core contraction, TMA z pass] timeout flags (0 = never)."""
        f = np.zeros(2, dtype=np.int32)
        _call("sincgpu_kernel_timeouts", self._h, f.ctypes.data)
        return f.tolist()

    def mult_ke_dev(self, inp, out, howmany):
        _call("sincgpu_mult_ke_dev", self._h, _ptr(inp), _ptr(out), int(howmany))

    def mult_reducedpot_dev(self, inspfs, outspfs, reducedpot):
        _call("sincgpu_mult_reducedpot_dev", self._h, _ptr(inspfs), _ptr(outspfs), _ptr(reducedpot))

    def mean_field_dev(self, phi, tally, twoematel, reducedpot):
        _call("sincgpu_mean_field_dev", self._h, _ptr(phi), _ptr(tally), _ptr(twoematel), _ptr(reducedpot))

    def orbital_rhs_dev(self, phi, tally, denmat, invdenmat, reducedpot, out, twoematel=None,
                        timefac=-1j, ztdpot=0.0):
        tf = complex(timefac)
        _call("sincgpu_orbital_rhs_dev", self._h, _ptr(phi), _ptr(tally), _ptr(denmat), _ptr(invdenmat),
              tf.real, tf.imag, float(ztdpot), _ptr(twoematel), _ptr(reducedpot), _ptr(out))

    def orbital_rhs(self, phi, tally, denmat, invdenmat, timefac=-1j, ztdpot=0.0, want_twoematel=True):
        """Host arrays in, host arrays out: (outspfs(G,n), twoematel(n,n,n,n) or None)."""
        n = self.nspf
        p = _f(phi)
        t = _f(tally)
        dm = _f(denmat)
        inv = _f(invdenmat)
        out = np.zeros((self.G, n), dtype=np.complex128, order="F")
        mat = np.zeros((n, n, n, n), dtype=np.complex128, order="F") if want_twoematel else None
        tf = complex(timefac)
        _call("sincgpu_orbital_rhs", self._h, _ptr(p), _ptr(t), _ptr(dm), _ptr(inv), tf.real, tf.imag,
              float(ztdpot), _ptr(mat), _ptr(out))
        return out, mat

    def actreduced_dev(self, inspfs, projspfs, denmat, invdenmat, reducedpot, out, timefac=-1j,
                       dentimeflag=1, projflag=1, ztdpot=0.0):
        tf = complex(timefac)
        _call("sincgpu_actreduced_dev", self._h, int(dentimeflag), _ptr(inspfs), _ptr(projspfs),
              _ptr(denmat), _ptr(invdenmat), _ptr(reducedpot), tf.real, tf.imag, int(projflag),
              float(ztdpot), _ptr(out))
