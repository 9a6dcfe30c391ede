"""CPU oracle for the orbital propagation step (TEST INFRASTRUCTURE ONLY).

Restates, for the sinc project with no frozen core, no constraints and no
driving term, the pieces of the reference's exponential orbital propagator
(intopt=3):
  derproject00      MCTDH.SRC/derivs.f90:53-161 (jacprojorth=0)
  jacinit0          MCTDH.SRC/expo_driver.f90:429-467
  jacoperate00      MCTDH.SRC/expo_driver.f90:40-259 (jacsymflag=0)
  spf_linear_derivs MCTDH.SRC/derivs.f90:1037-1186
  spf_orthogit      MCTDH.SRC/spfs.f90:120-196 with symorthogmat
                    (MCTDH.SRC/utils.f90:947-1023, hermitian norm build)
  expospfprop       MCTDH.SRC/expo_driver.f90:482-771 (DGPHIV branch, the
                    nodgexpthirdflag=1 hardwire) with its saved Krylov-dimension
                    and step-size state
Mean fields come as two time slots (0 = end of the CMF interval, 1 = start),
each (denmat, invdenmat, reducedpot); with the linear flag they are blended
with weights (t - first)/(last - first) and its complement, as the reference's
effective_cmf_linearflag does.
Only tests/ and the CPU legs of bench.py import this module.
"""
from __future__ import annotations

import math

import numpy as np

from . import sinc_oracle as orc
from .expokit_oracle import complexify, dgphiv, realify


def derproject00(inspfs, prospfs, prospfderivs):
    """out = pro x <proder|in> + proder x <pro|in>."""
    derdot = np.conj(prospfderivs).T @ inspfs
    mydot = np.conj(prospfs).T @ inspfs
    return prospfs @ derdot + prospfderivs @ mydot


def symorthogmat(a):
    """A^(-1/2) of a hermitian positive matrix by SVD, singular values below
    1e-10 dropped: U diag(s^-1/2) V^H."""
    u, sv, vt = np.linalg.svd(a)
    f = np.where(np.abs(sv) < 1e-10, 0.0, 1.0 / np.sqrt(np.where(sv > 0, sv, 1.0)))
    return (u * f[None, :]) @ vt


def spf_orthogit(inspfs):
    """Two Loewdin passes; returns (orbitals, error of the last overlap)."""
    phi = np.array(inspfs, dtype=np.complex128, order="F")
    error = 0.0
    for ii in range(3):
        ovl = np.conj(phi).T @ phi
        error = float(np.abs(ovl - np.eye(ovl.shape[0])).max())
        if ii < 2:
            phi = phi @ symorthogmat(ovl)
    return phi, error


class OrbPropState:
    """The saved variables of expospfprop (expo_driver.f90:498-509)."""

    def __init__(self, expodim=10, maxexpodim=100, expostepfac=1.2, first_stepsize=0.05):
        self.expodim = expodim
        self.maxexpodim = maxexpodim
        self.expostepfac = expostepfac
        self.first_stepsize = first_stepsize   # par_timestep / littlesteps
        self.icalled = 0
        self.thisexpodim = 0
        self.exposet = 0
        self.tempstepsize = -1.0


def _facs(t, first, last, linear):
    if linear:
        f0 = (t - first) / (last - first)
        return [f0, 1.0 - f0]
    return [1.0, 0.0]


def spf_linear_derivs(sysm, phi, slots, t, first, last, linear, timefac=-1j, ez=0.0):
    facs = _facs(t, first, last, linear)
    out = np.zeros_like(phi)
    for s in range(2 if linear else 1):
        den, inv, rp = slots[s]
        out = out + orc.actreduced00(sysm, phi, phi, den, inv, rp, timefac=timefac, dentimeflag=1,
                                     projflag=1, ztdpot=ez) * facs[s]
    return out


def jacinit(sysm, phi, slots, t, first, last, linear, timefac=-1j, ez=0.0):
    den, inv, rp = slots[0]
    out = orc.actreduced00(sysm, phi, None, den, inv, rp, timefac=timefac, projflag=0, ztdpot=ez)
    if linear:
        g = (t - first) / (last - first)
        den, inv, rp = slots[1]
        out = out * g + (1.0 - g) * orc.actreduced00(sysm, phi, None, den, inv, rp, timefac=timefac,
                                                     projflag=0, ztdpot=ez)
    return phi.copy(), out


def jacoperate(sysm, x, jacvect, jacvectout, slots, t, first, last, linear, timefac=-1j, ez=0.0):
    facs = _facs(t, first, last, linear)
    out = np.zeros_like(x)
    for s in range(2 if linear else 1):
        den, inv, rp = slots[s]
        work = orc.actreduced00(sysm, x, None, den, inv, rp, timefac=timefac, projflag=0, ztdpot=ez)
        out = out + work * facs[s]
        out = out - orc.project00(work, jacvect) * facs[s]
        out = out - derproject00(jacvectout, jacvect, x) * facs[s]
    return out


def expospfprop(sysm, state: OrbPropState, phi, slots, tin, tout, first, last, linear, expotol=1e-8,
                timefac=-1j, ez=0.0):
    """One orbital propagation over [tin, tout]; returns (orbitals, info)."""
    phi = np.asarray(phi, dtype=np.complex128)
    G, n = phi.shape
    tdiff = tout - tin
    midtime = 0.5 * (tin + tout)
    jacvect, jacvectout = jacinit(sysm, phi, slots, midtime, first, last, linear, timefac, ez)
    idim = 2 * G * n
    maxexpodim = min(state.maxexpodim, idim - 1)
    state.icalled += 1
    if state.icalled == 1:
        state.tempstepsize = state.first_stepsize
        state.thisexpodim = min(state.expodim, maxexpodim)
    if state.icalled % 12 == 0:
        state.exposet = 0
    if state.thisexpodim < maxexpodim:
        state.tempstepsize *= 4
    else:
        state.tempstepsize *= state.expostepfac
    aspfs = spf_linear_derivs(sysm, phi, slots, midtime, first, last, linear, timefac, ez)

    def mv(xr):
        x = complexify(xr).reshape(G, n, order="F")
        y = jacoperate(sysm, x, jacvect, jacvectout, slots, midtime, first, last, linear, timefac, ez)
        return realify(y.reshape(-1, order="F"))

    u = realify(aspfs.reshape(-1, order="F"))
    w, guess, info = dgphiv(idim, state.thisexpodim, tdiff, u, np.zeros(idim), expotol, 1.0, mv,
                            lambda a, b: float(a @ b), state.tempstepsize)
    state.tempstepsize = guess
    if info["nstep"] > 1:
        state.thisexpodim = min(maxexpodim, max(state.thisexpodim + 5, math.ceil(state.thisexpodim * 1.2)))
        state.exposet = 1
    out = phi + complexify(w).reshape(G, n, order="F")
    out, error = spf_orthogit(out)
    if state.exposet == 0:
        state.thisexpodim = max(5, math.floor(state.thisexpodim * 0.95))
    info = dict(info, numiters=info["nmult"], orth_error=error)
    return out, info
