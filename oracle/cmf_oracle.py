"""CPU oracle for one constant-mean-field propagation step (TEST INFRASTRUCTURE ONLY).

Restates, for the sinc project (numr=1, no frozen core, no constraints, no
driving term, mcscfnum=1, sparseconfigflag=1, intopt=3), the reference's
  cmf_prop_wfn        MCTDH.SRC/prop.f90:230-574 with its defaults
                      prepropflag=1, step_flag=2, postpropflag=2
                      (MCTDH.SRC/parameters.f90:287-289), improvedrelaxflag=0
  propspfs/propspfs0  MCTDH.SRC/prop.f90:132-228 (expospfprop, then a second
                      spf_orthogit)
  cmf_prop_avector    MCTDH.SRC/prop.f90:578-776 (linear blend of the two
                      Hamiltonian slots at the sub-step midpoint)
  expoavecprop        MCTDH.SRC/expo_driver.f90:827-1055 (DGEXPVxxx2 with
                      t = 1, anorm = dt, its saved order / step state)
  myconfigprop        MCTDH.SRC/configstuff.f90:235-265 (spin projection after)
  get_stuff0          MCTDH.SRC/proputils.f90:264-300 (get_allden, all_matel,
                      get_reducedpot)
  energy              MCTDH.SRC/prop.f90:926-955 (<A|P H A>/<A|A> after the step)
  length-gauge pulses MCTDH.SRC/pulse.f90:8-52, 149-170, 197-211, 230-247,
                      272-299, 337-372 (z component, pulsetheta = 0)
The Krylov for the A-vector runs on the configuration basis; the reference runs
it on the spin-adapted basis.  For a spin-projected start vector and the
spin-free Hamiltonian both span the same Krylov space, so the two agree to
rounding; the spin projection after each propagation is applied as the
reference does.
Only tests/ and the CPU legs of bench.py import this module.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import orbprop_oracle as op
from . import sinc_oracle as orc
from .expokit_oracle import complexify, dgexpv, realify
from .walks_oracle import CIWalks, SpinSets, dipole_z


@dataclass
class Pulse:
    """One pulse of the reference's &pulse namelist (length gauge)."""
    pulsetype: int = 2
    omega: float = 1.0
    omega2: float = 1.0
    pulsestart: float = 0.0
    phaseshift: float = 0.0
    strength: float = 0.5
    longstep: float = 1.0
    pulsetheta: float = 0.0


def pulse_ez(pulses, t):
    """tdpotlen0(t, which=3): z component of the field of all pulses."""
    e = 0.0
    for p in pulses:
        fac = math.cos(p.pulsetheta)
        if fac == 0.0:
            continue
        w, w2, tau = p.omega, p.omega2, t - p.pulsestart
        v = 0.0
        if p.pulsetype == 1:
            if t >= p.pulsestart and tau <= math.pi / w:
                v = p.strength * w * (math.sin(tau * w) * math.cos(tau * w + p.phaseshift)
                                      + math.sin(tau * w + p.phaseshift) * math.cos(tau * w))
        elif p.pulsetype == 2:
            if t >= p.pulsestart and tau <= math.pi / w:
                arg = (tau - math.pi / w / 2) * w2 + p.phaseshift
                v = p.strength * (2 * w * math.sin(tau * w) * math.cos(tau * w) * math.sin(arg)
                                  + math.sin(tau * w) ** 2 * w2 * math.cos(arg))
        elif p.pulsetype == 3:
            if t >= p.pulsestart and tau <= math.pi / w:
                k = 2 * p.longstep + 1
                edge = math.pi / 2.0 / w / k
                if tau <= edge or tau >= math.pi / w - edge:
                    f = 2 * w * k * math.sin(tau * w * k) * math.cos(tau * w * k)
                    f2 = math.sin(tau * w * k) ** 2
                else:
                    f, f2 = 0.0, 1.0
                v = p.strength * (f * math.sin(tau * w2 + p.phaseshift) + f2 * w2 * math.cos(tau * w2 + p.phaseshift))
        elif p.pulsetype == 4:
            if t < math.pi / w:
                v = p.strength * w2 * math.cos(t * w2 + p.phaseshift)
        elif p.pulsetype == 5:
            pp = t * w - math.pi / 2
            if pp < math.pi / 2:
                v = p.strength * (0.75 * math.cos(pp) + math.cos(3 * pp) / 4.0)
        else:
            raise ValueError(f"pulse type {p.pulsetype}")
        e += v * fac
    return e


@dataclass
class CmfParams:
    par_timestep: float = 0.05
    littlesteps: int = 1
    expotol: float = 1e-8
    aerror: float = 1e-9
    aorder: int = 30
    maxaorder: int = 100
    expodim: int = 10
    maxexpodim: int = 100
    expostepfac: float = 1.2
    denreg: float = 1e-10
    step_flag: int = 2
    timefac: complex = -1j
    pulses: list = field(default_factory=list)


class _Slot:
    def copy(self):
        s = _Slot()
        s.__dict__ = {k: (v.copy() if hasattr(v, "copy") else v) for k, v in self.__dict__.items()}
        return s


class CmfOracle:
    def __init__(self, sysm, numelec, restrictms, phi, avec, params: CmfParams, spinrestrictval=None,
                 workers=1):
        self.sysm, self.p = sysm, params
        self.workers = workers          # FFT threads of the Coulomb solves (same transforms)
        n = phi.shape[1]
        self.n = n
        self.ow = CIWalks(numelec, n, restrictms)
        self.spin = SpinSets(self.ow, spinrestrictval)
        self.nucdip = float(np.sum(sysm.nuccharges * sysm.centershift[:, 2] / 2.0 * sysm.spacing))
        self.orb = op.OrbPropState(params.expodim, params.maxexpodim, params.expostepfac,
                                   params.par_timestep / params.littlesteps)
        self.a_icalled, self.a_tempstep, self.a_dim, self.a_set = 0, -1.0, -1, 0
        self.a_maxorder = max(1, min(2 * self.spin.numspinconfig - 1, params.maxaorder))
        self.s0, self.s1 = _Slot(), _Slot()
        self.s0.spfs = np.array(phi, dtype=np.complex128)
        self.s0.avec = self.spin.project(avec)
        self.get_stuff()
        self.energy = self.expect(0.0, with_pulse=True, project=False)
        self.orb_iters = self.avec_iters = 0

    # ---- mean fields (slot 0) -------------------------------------------
    def get_allden(self):
        s = self.s0
        s.den = self.ow.getdenmat00(s.avec)
        s.inv = orc.invmatsmooth(s.den, tol=self.p.denreg)
        s.tally = self.ow.get_tworeducedx(s.avec)

    def all_matel(self):
        s, sysm = self.s0, self.sysm
        s.mat, self.twoereduced = sysm.call_twoe_matel00(s.spfs, s.spfs, workers=self.workers)
        ph = np.conj(s.spfs).T
        pot, ke, z = ph @ sysm.mult_pot(s.spfs), ph @ sysm.mult_ke(s.spfs), ph @ sysm.mult_zdipole(s.spfs)
        s.hops = (self.ow.assemble_doubles(s.mat), self.ow.assemble_singles(pot), self.ow.assemble_singles(ke),
                  self.ow.assemble_singles(z))

    def get_reducedpot(self):
        self.s0.rp = orc.get_reducedpot(self.twoereduced, self.s0.tally)

    def get_stuff(self):
        self.get_allden()
        self.all_matel()
        self.get_reducedpot()

    # ---- sigma with a (blended) Hamiltonian ------------------------------
    def sigma(self, a, hops, ez):
        xp, xo, xk, xz = hops
        return self.ow.sparsesparsemult(a, xp, xo, xk, constant=self.sysm.nucrepulsion + ez * self.nucdip,
                                        xpulse=(xz * ez if ez else None))

    def expect(self, t, with_pulse=False, project=True):
        """<A|H A>/<A|A>; after a step H A is spin projected (prop.f90:944), at the
        start it is not (prop.f90:831-838)."""
        a = self.s0.avec
        ez = pulse_ez(self.p.pulses, t) if with_pulse else 0.0
        ha = self.sigma(a, self.s0.hops, ez)
        if project:
            ha = self.spin.project(ha)
        return (np.vdot(a, ha) / np.vdot(a, a)).real

    def dipole(self):
        """z dipole of the current state with the current orbitals' matrices."""
        return dipole_z(self.ow, self.s0.hops[3], self.s0.avec, self.nucdip)

    # ---- A-vector propagation -------------------------------------------
    def expoavecprop(self, a, hops, dt, midtime):
        p = self.p
        self.a_icalled += 1
        if self.a_icalled == 1:
            self.a_tempstep = p.par_timestep / p.littlesteps
            self.a_dim = min(self.a_maxorder, p.aorder)
        if self.a_icalled % 20 == 0:
            self.a_set = 0
        self.a_tempstep *= 4 if self.a_dim < self.a_maxorder else 1.1
        ez = pulse_ez(p.pulses, midtime)
        tf = p.timefac * dt
        mv = lambda x: realify(tf * self.sigma(complexify(x), hops, ez))  # noqa: E731
        w, g, info = dgexpv(2 * self.ow.numconfig, self.a_dim, 1.0, realify(a), p.aerror,
                            p.par_timestep / p.littlesteps, mv, lambda u, v: float(u @ v), self.a_tempstep,
                            self.a_maxorder + 1)
        self.a_tempstep = g
        if self.a_set == 0 and info["nstep"] == 1 and self.a_dim > 2:
            self.a_dim = max(2, self.a_dim - 1)
        if info["nstep"] > 1:
            self.a_set = 1
            self.a_dim = min(math.floor(self.a_dim * 1.2) + 5, self.a_maxorder)
        self.avec_iters += info["nmult"]
        return complexify(w)

    def cmf_prop_avector(self, linearflag, tin, tout):
        p = self.p
        a = self.s1.avec
        for k in range(1, p.littlesteps + 1):
            ta = tin + (tout - tin) * (k - 1) / p.littlesteps
            tb = tin + (tout - tin) * k / p.littlesteps
            dt, mid = tb - ta, 0.5 * (ta + tb)
            if linearflag == 0:
                hops = self.s0.hops
            else:
                s0w = (mid - self.first) / (self.last - self.first)
                s1w = (self.last - mid) / (self.last - self.first)
                hops = tuple(s1w * h1 + s0w * h0 for h1, h0 in zip(self.s1.hops, self.s0.hops))
            a = self.spin.project(self.expoavecprop(a, hops, dt, mid))
        self.s0.avec = a

    # ---- orbital propagation ---------------------------------------------
    def propspfs(self, linearflag, tin, tout):
        p = self.p
        phi = self.s1.spfs
        slots = [(self.s0.den, self.s0.inv, self.s0.rp), (self.s1.den, self.s1.inv, self.s1.rp)]
        for k in range(1, p.littlesteps + 1):
            ta = tin + (tout - tin) * (k - 1) / p.littlesteps
            tb = tin + (tout - tin) * k / p.littlesteps
            ez = pulse_ez(p.pulses, 0.5 * (ta + tb))
            phi, info = op.expospfprop(self.sysm, self.orb, phi, slots, ta, tb, self.first, self.last,
                                       linearflag == 1, expotol=p.expotol, timefac=p.timefac, ez=ez)
            phi, _ = op.spf_orthogit(phi)
            self.orb_iters += info["numiters"]
        self.s0.spfs = phi

    # ---- one step -----------------------------------------------------------
    def step(self, tin, tout):
        self.first, self.last = tin, tout
        self.orb_iters = self.avec_iters = 0
        self.s1 = self.s0.copy()
        self.cmf_prop_avector(0, tin, tout)          # pre-prop
        self.get_allden()
        self.get_reducedpot()
        for _ in range(self.p.step_flag):            # main predictor/corrector steps
            self.propspfs(1, tin, tout)
            self.cmf_prop_avector(1, tin, tout)
            self.get_stuff()
        self.cmf_prop_avector(1, tin, tout)          # post-prop (postpropflag=2)
        self.get_allden()
        self.get_reducedpot()
        self.s0.avec = self.spin.project(self.s0.avec)
        self.energy = self.expect(tout)
        self.norm = float(np.linalg.norm(self.s0.avec))
        return self.energy
