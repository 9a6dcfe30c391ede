"""CPU oracle for the Krylov exponential propagator (TEST INFRASTRUCTURE ONLY).

Restates, from Sidje's published Expokit algorithms (ACM TOMS 24, 1998), the
variants the reference calls for the A-vector propagation:
  DGPADM       irreducible (6,6) Pade with scaling and squaring
               (MCTDH.SRC/expokit.f90:526-...)
  DGEXPVxxx20  Krylov exp(t A) v with full Arnoldi, externally supplied dot,
               initial step from the caller (stepguess), next step never shorter
               than the accepted one (MCTDH.SRC/expokit.f90:2222-2660)
  DGPHIV0      Krylov w = exp(t A) v + t phi_1(t A) u on the 3-extended
               Hessenberg (MCTDH.SRC/expokit.f90:3904-4310), with the same step
               guess conventions and plain gamma step-down on rejection
as called by expoavecprop (MCTDH.SRC/expo_driver.f90:827-1055) on the real-ified
A-vector and by expospfprop (MCTDH.SRC/expo_driver.f90:482-771) on the
real-ified orbitals (complex vectors viewed as interleaved reals).
Only tests/ and the CPU legs of bench.py import this module.
"""
from __future__ import annotations

import math

import numpy as np


def dgpadm(ideg: int, H: np.ndarray, t: float):
    """exp(t H) for a small real matrix; returns (E, ns)."""
    m = H.shape[0]
    hnorm = np.abs(H).sum(axis=1).max()   # infinity norm (row sums of |H|)
    hnorm = abs(t * hnorm)
    if hnorm == 0.0:
        return np.eye(m), 0
    ns = max(0, int(math.log(hnorm) / math.log(2.0)) + 2)
    scale = t / float(2 ** ns)
    scale2 = scale * scale
    i, j = ideg + 1, 2 * ideg + 1
    coef = [1.0]
    for k in range(1, ideg + 1):
        coef.append((coef[k - 1] * float(i - k)) / float(k * (j - k)))
    H2 = scale2 * (H @ H)
    p = coef[ideg - 1] * np.eye(m)
    q = coef[ideg] * np.eye(m)
    iodd = 1
    k = ideg - 1
    while True:
        if iodd == 1:
            q = q @ H2
            q = q + coef[k - 1] * np.eye(m)
        else:
            p = p @ H2
            p = p + coef[k - 1] * np.eye(m)
        iodd = 1 - iodd
        k -= 1
        if k <= 0:
            break
    if iodd == 1:
        q = scale * (q @ H)
    else:
        p = scale * (p @ H)
    q = q - p
    p = np.linalg.solve(q, p)
    p = 2.0 * p + np.eye(m)
    if ns == 0 and iodd == 1:
        return -p, ns
    for _ in range(ns):        # squaring removes the sign of the iodd==1 case
        p = p @ p
    return p, ns


def dgexpv(n, m, t, v, tol, anorm, matvec, dot, stepguess, maxdim, ideg=6, mxstep=1000):
    """Returns (w, new_stepguess, info) for w = exp(t A) v."""
    delta, gamma = 1.2, 0.9
    if m >= maxdim or m <= 0:
        raise ValueError("bad Krylov dimension")
    k1 = 2
    mh = m + 2
    mbrkdwn = m
    t_out = abs(t)
    t_now = 0.0
    t_step = 0.0
    t_last = 0.0
    eps = abs((4.0 / 3.0 - 1.0) * 3.0 - 1.0)
    if tol <= eps:
        tol = math.sqrt(eps)
    rndoff = eps * anorm
    break_tol = 1.0e-7
    sgn = math.copysign(1.0, t)
    w = np.array(v, dtype=np.float64)
    beta = math.sqrt(dot(w, w))
    t_new = stepguess
    xm = 1.0 / m
    sqr1 = math.sqrt(0.1)
    nstep = 0
    nmult = 0
    avnorm = 0.0
    steps = []
    while t_now < t_out:
        nstep += 1
        t_last = t_step
        t_step = min(t_out - t_now, t_new)
        V = np.zeros((m + 1, n))
        Hm = np.zeros((mh, mh))
        V[0] = w / beta
        k1 = 2
        mbrkdwn = m
        brk = False
        for j in range(m):
            nmult += 1
            p = matvec(V[j])
            for i in range(j + 1):
                hij = dot(V[i], p)
                p = p - hij * V[i]
                Hm[i, j] = hij
            hj1j = math.sqrt(dot(p, p))
            if hj1j <= break_tol:
                k1 = 0
                mbrkdwn = j + 1
                t_step = t_out - t_now
                brk = True
                break
            Hm[j + 1, j] = hj1j
            V[j + 1] = p / hj1j
        if not brk:
            nmult += 1
            p = matvec(V[m])
            avnorm = math.sqrt(dot(p, p))
        Hm[m + 1, m] = 1.0
        while True:
            mx = mbrkdwn + k1
            E, ns = dgpadm(ideg, Hm[:mx, :mx], sgn * t_step)
            exph = E[:, 0]
            if k1 == 0:
                err_loc = tol
            else:
                p1 = abs(exph[m]) * beta
                p2 = abs(exph[m + 1]) * beta * avnorm
                if p1 > 10.0 * p2:
                    err_loc = p2
                    xm = 1.0 / m
                else:
                    err_loc = p1
                    xm = 1.0 / (m - 1)
            if k1 != 0 and err_loc > delta * t_step * tol:
                t_step = gamma * t_step * (t_step * tol / err_loc) ** xm
                p1 = 10.0 ** (round_half_away(math.log10(t_step) - sqr1) - 1)
                t_step = math.trunc(t_step / p1 + 0.55) * p1
                continue
            break
        mx = mbrkdwn + max(0, k1 - 1)
        w = beta * (V[:mx].T @ exph[:mx])
        beta = math.sqrt(dot(w, w))
        t_new = gamma * t_step * (t_step * tol / err_loc) ** xm
        p1 = 10.0 ** (round_half_away(math.log10(t_new) - sqr1) - 1)
        t_new = math.trunc(t_new / p1 + 0.55) * p1
        if t_new < t_step:
            t_new = t_step
        t_now += t_step
        steps.append(t_step)
        if nstep >= mxstep:
            break
    new_guess = t_step if nstep == 1 else t_last
    return w, new_guess, {"nstep": nstep, "nmult": nmult, "steps": steps}


def dgphiv(n, m, t, u, v, tol, anorm, matvec, dot, stepguess, ideg=6, mxstep=1000):
    """Returns (w, new_stepguess, info) for w = exp(t A) v + t phi_1(t A) u,
    phi_1(z) = (exp(z) - 1)/z (MCTDH.SRC/expokit.f90:3904-4310)."""
    delta, gamma = 1.2, 0.8
    if m >= n or m <= 0:
        raise ValueError("bad Krylov dimension")
    mh = m + 3
    t_out = abs(t)
    t_now = t_step = t_last = t_new = 0.0
    eps = abs((4.0 / 3.0 - 1.0) * 3.0 - 1.0)
    if tol <= eps:
        tol = math.sqrt(eps)
    break_tol = 1.0e-7
    sgn = math.copysign(1.0, t)
    sqr1 = math.sqrt(0.1)
    w = np.array(v, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    nstep = nmult = nreject = 0
    xm = 0.0
    avnorm = 0.0
    steps = []
    while t_now < t_out:
        nmult += 1
        p = matvec(w) + u
        beta = math.sqrt(dot(p, p))
        if beta == 0.0:
            break
        V = np.zeros((m + 2, n))
        Hm = np.zeros((mh, mh))
        V[0] = p / beta
        if nstep == 0:
            t_new = stepguess
            xm = 1.0 / m
        nstep += 1
        t_last = t_step
        t_step = min(t_out - t_now, t_new)
        k1, mbrkdwn, hj1j = 3, m, 0.0
        brk = False
        for j in range(m):
            nmult += 1
            p = matvec(V[j])
            for i in range(j + 1):
                hij = dot(V[i], p)
                p = p - hij * V[i]
                Hm[i, j] = hij
            hj1j = math.sqrt(dot(p, p))
            if hj1j <= break_tol:
                k1, mbrkdwn, brk = 0, j + 1, True
                t_step = t_out - t_now
                break
            Hm[j + 1, j] = hj1j
            V[j + 1] = p / hj1j
        if not brk:
            nmult += 1
            p = matvec(V[m])
            avnorm = math.sqrt(dot(p, p))
        # the 3-extended scheme: e_1 column, h(m+1,m) taken out, shifted identity
        Hm[0, mbrkdwn] = 1.0
        Hm[m, m - 1] = 0.0
        for i in range(1, k1):
            Hm[m + i - 1, m + i] = 1.0
        while True:
            mx = mbrkdwn + max(1, k1)
            E, _ = dgpadm(ideg, Hm[:mx, :mx], sgn * t_step)
            phih = np.zeros(mx + 2)
            phih[:mx] = E[:, mbrkdwn]
            if k1 != 0:
                phih[mbrkdwn] = hj1j * E[mbrkdwn - 1, mbrkdwn + 1]
                phih[mbrkdwn + 1] = hj1j * E[mbrkdwn - 1, mbrkdwn + 2]
                p1 = abs(phih[m]) * beta
                p2 = abs(phih[m + 1]) * beta * avnorm
                if p1 > 10.0 * p2:
                    err_loc, xm = p2, 1.0 / (m + 1)
                else:
                    err_loc, xm = p1, 1.0 / m
                if err_loc > delta * t_step * tol:   # mxreject = 0: step down and retry
                    t_step = gamma * t_step
                    nreject += 1
                    continue
            else:
                err_loc = tol
            break
        mx = mbrkdwn + max(0, k1 - 2)
        w = w + beta * (V[:mx].T @ phih[:mx])
        t_new = gamma * t_step * (t_step * tol / err_loc) ** xm
        p1 = 10.0 ** (round_half_away(math.log10(t_new) - sqr1) - 1)
        t_new = math.trunc(t_new / p1 + 0.55) * p1
        if t_new < t_step:
            t_new = t_step
        t_now += t_step
        steps.append(t_step)
        if nstep >= mxstep:
            break
    new_guess = t_step if nstep == 1 else t_last
    return w, new_guess, {"nstep": nstep, "nmult": nmult, "nreject": nreject, "steps": steps}


def round_half_away(x: float) -> int:
    """Fortran NINT."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def realify(z):
    z = np.asarray(z, dtype=np.complex128)
    out = np.empty(2 * z.size)
    out[0::2] = z.real
    out[1::2] = z.imag
    return out


def complexify(x):
    return x[0::2] + 1j * x[1::2]
