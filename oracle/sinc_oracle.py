"""CPU oracle for the sinc-DVR orbital right-hand side (TEST INFRASTRUCTURE ONLY).

This module is the checker, not the product.  Only ``tests/``, the
``smoke()`` entry of ``__graft_entry__`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The CUDA library
never calls into it and the product path fails loudly when its extension
is missing.

It is a plain numpy restatement of the reference algorithm
(LBNL-AMO-MCTDHF v1.36, polyatomic SINCDVR project).  Every function cites
the reference file:line it follows; paths are relative to the reference
project root (``MCTDH.SRC/...``).  Arrays use Fortran index order and
Fortran memory order (``order='F'``) so that shapes read exactly like the
reference declarations, e.g. ``twoereduced(totpoints, numspf, numspf)``.

Parity status: the reference ships no golden vectors or fixtures for this
path and cannot be compiled here (no Fortran compiler), so this oracle is
pinned by self-checks instead (analytic Coulomb potential of a Gaussian,
symmetry identities, closed-form walk counts) -- see tests/test_oracle.py.
Parity against the reference binary itself is therefore UNPINNED.

Numerical conventions restated from the reference:
  * forward FFT is unnormalised (DFFTPACK ``zfftf`` / FFTW_FORWARD,
    COREPROJECT/ftcore.f90:140-157), which numpy.fft.fftn matches;
  * the Toeplitz solve embeds densities at octant (1,1,1) of the doubled
    (2N)^3 grid and extracts octant (2,2,2)
    (SINCDVR/coreproject.f90:450,521), circ3d_sub
    (SINCDVR/toeplitz_subs.f90:561-589);
  * the tooth.f90:165 slice ``ALLTT(-NBIG-J:NBIG-K)`` is non-conformable for
    J/=K; this oracle uses the intended symmetric form ``ALLTT(-NBIG-J:NBIG-J)``
    (same start index; a compiler that takes the loop length from the first,
    conformable term computes exactly this).
"""
from __future__ import annotations

import math
import numpy as np

PI = 4.0 * math.atan(1.0)


# ---------------------------------------------------------------------------
# a1: 1-D sinc-DVR kinetic / derivative Toeplitz vectors and grid
# ---------------------------------------------------------------------------
def sine_dvr(gridpoints: int, spacing: float):
    """SINCDVR/SineDVR.f90:3-44.

    Returns (ketot, fdtot, points) with ketot/fdtot indexed d+(gridpoints-1)
    for d in [1-gridpoints, gridpoints-1].
    """
    g = gridpoints
    points = np.arange(1, g + 1, dtype=np.float64) * spacing
    points = points - (points[0] + points[-1]) / 2.0
    d = np.arange(1 - g, g, dtype=np.int64)
    ke = np.empty(2 * g - 1)
    fd = np.empty(2 * g - 1)
    for k, i in enumerate(d):
        if i == 0:
            ke[k] = PI ** 2 / 3.0
            fd[k] = 0.0
        else:
            sgn = -1.0 if (i % 2) else 1.0
            ke[k] = 2.0 / float(i) ** 2 * sgn
            fd[k] = 1.0 / float(i) * sgn
    ke = ke / 2.0 / spacing ** 2
    fd = fd / spacing
    return ke, fd, points


def ketot_matrix(gridpoints: int, spacing: float) -> np.ndarray:
    """ketot(idim)%mat(l,1,j,1) = kevect(j-l)  (SINCDVR/init_sinc_new.f90:448-463)."""
    ke, _, _ = sine_dvr(gridpoints, spacing)
    g = gridpoints
    l = np.arange(g)[:, None]
    j = np.arange(g)[None, :]
    return ke[(j - l) + (g - 1)]


# ---------------------------------------------------------------------------
# a2: inverse 3-D kinetic operator (Coulomb Green's function), tooth.f90
# ---------------------------------------------------------------------------
def _rslab(first, second, third, delta):
    """DELTA^3/SQRT(PPOS(a)**2+PPOS(b)**2+PPOS(c)**2) with the reference's
    left-to-right association (SINCDVR/tooth.f90:141)."""
    a = (first * delta)
    b = (second * delta)
    c = (third * delta)
    s = (a * a) + (b * b)
    s = s + (c * c)
    with np.errstate(divide="ignore"):
        return delta ** 3 / np.sqrt(s)


def getinverse(nout: int, nbig: int, nsmall: int, delta: float) -> np.ndarray:
    """TINVOUT(-nout:nout,-nout:nout,-nout:nout)  (SINCDVR/tooth.f90:12-95).

    R(i,j,k) = delta^3/|r| (0 at the origin) on the big grid, plus the
    near-field correction Q on [-nsmall,nsmall]^3 solving
    (T(x)1(x)1 + 1(x)T(x)1 + 1(x)1(x)T) Q = 2*pi*delta_0 - T_big R
    through the eigendecomposition of the 1-D matrix T (tooth.f90:48-79).
    Returned in Fortran index order [i,j,k] offset by +nout.
    """
    if nbig <= nsmall:
        raise ValueError("NBIG is less than nsmall")  # tooth.f90:114-117
    big = np.arange(-nbig, nbig + 1, dtype=np.float64)
    sm = np.arange(-nsmall, nsmall + 1, dtype=np.float64)
    ns = 2 * nsmall + 1
    # ALLTT(m), m in [-NSMALL-NBIG, NSMALL+NBIG]  (tooth.f90:152-156)
    m = np.arange(-nsmall - nbig, nsmall + nbig + 1)
    d2inv = 1.0 / delta ** 2
    with np.errstate(divide="ignore"):
        alltt = np.where(m % 2 == 0, 1.0, -1.0) * d2inv / (m.astype(np.float64) ** 2)
    alltt[nsmall + nbig] = PI ** 2 / (6.0 * delta ** 2)
    off = nsmall + nbig
    # A[I,p] = ALLTT(p - I) for I in small, p in big
    A = alltt[(big[None, :].astype(np.int64) - sm[:, None].astype(np.int64)) + off]

    # term 1: sum_p ALLTT(p-I) R(p,J,K),   R(p,J,K) with (p,J,K) association
    r1 = _rslab(big[:, None, None], sm[None, :, None], sm[None, None, :], delta)
    # term 2: sum_p ALLTT(p-J) R(I,p,K)
    r2 = _rslab(sm[:, None, None], big[None, :, None], sm[None, None, :], delta)
    # term 3: sum_p ALLTT(p-K) R(I,J,p)
    r3 = _rslab(sm[:, None, None], sm[None, :, None], big[None, None, :], delta)
    for r, idx in ((r1, (nbig, nsmall, nsmall)), (r2, (nsmall, nbig, nsmall)), (r3, (nsmall, nsmall, nbig))):
        r[idx] = 0.0  # R(0,0,0) = 0  (tooth.f90:146)
    t1 = np.einsum("ip,pjk->ijk", A, r1)
    t2 = np.einsum("jp,ipk->ijk", A, r2)
    t3 = np.einsum("kp,ijp->ijk", A, r3)
    tr = -1.0 * (t1 + t2 + t3)
    tr[nsmall, nsmall, nsmall] += 2 * PI  # tooth.f90:44

    # 1-D T on the small grid (tooth.f90:48-53) and its eigendecomposition
    ii = np.arange(-nsmall, nsmall + 1)
    dif = ii[:, None] - ii[None, :]
    with np.errstate(divide="ignore"):
        T = np.where(dif % 2 == 0, 1.0, -1.0) / (delta ** 2 * dif.astype(np.float64) ** 2)
    np.fill_diagonal(T, (PI / delta) ** 2 / 6.0)
    E, W = np.linalg.eigh(T)
    eigs = E[:, None, None] + E[None, :, None] + E[None, None, :]
    # TOOTHEIGMULT(TR,QQ,W^T); QQ=QQ/EIGS; TOOTHEIGMULT(QQ,Q,W)  (tooth.f90:76-79)
    qq = np.einsum("ai,bj,ck,ijk->abc", W.T, W.T, W.T, tr, optimize=True)
    qq = qq / eigs
    q = np.einsum("ai,bj,ck,ijk->abc", W, W, W, qq, optimize=True)

    out_idx = np.arange(-nout, nout + 1, dtype=np.float64)
    tinv = _rslab(out_idx[:, None, None], out_idx[None, :, None], out_idx[None, None, :], delta)
    tinv[nout, nout, nout] = 0.0
    lo = max(-nsmall, -nout)
    hi = min(nsmall, nout)
    so = slice(lo + nout, hi + nout + 1)
    ss = slice(lo + nsmall, hi + nsmall + 1)
    tinv[so, so, so] += q[ss, ss, ss]
    return tinv


# ---------------------------------------------------------------------------
# a3: Coulomb kernel on the doubled grid and the nuclear potential
# ---------------------------------------------------------------------------
def _fortran_mod(a: int, b: int) -> int:
    return int(math.fmod(a, b))


def _fortran_div(a: int, b: int) -> int:
    return int(a / b) if a * b >= 0 else -(abs(a) // abs(b))


class SincSystem:
    """Module state of the SINCDVR project: kevect, threed_two, pot
    (SINCDVR/sincproject.f90:4-43, 119-256; sinc_extraproject.f90:260-304)."""

    def __init__(self, gridpoints, spacing, centershift, nuccharges,
                 toothnbig=240, toothnsmall=40, sqrt32=False, notwoflag=0):
        g = int(gridpoints)
        self.N = g
        self.spacing = float(spacing)
        self.G = g ** 3
        centershift = np.asarray(centershift, dtype=np.int64).reshape(-1, 3)
        nuccharges = np.asarray(nuccharges, dtype=np.float64).reshape(-1)
        self.centershift = centershift
        self.nuccharges = nuccharges
        if toothnbig < g - 1:  # sinc_extraproject.f90:273-276
            toothnbig = g - 1
        self.kevect, self.fdvect, self.points = sine_dvr(g, spacing)
        self.ketot = ketot_matrix(g, spacing)

        tinv = getinverse(g - 1, toothnbig, toothnsmall, spacing)
        tempcoulomb = tinv / spacing ** 3          # sincproject.f90:155-156
        self.tempcoulomb = tempcoulomb             # index d+(g-1)
        # threed_two(-g:g-1)^3, zero on the -g planes (sincproject.f90:182-187)
        t2 = np.zeros((2 * g, 2 * g, 2 * g))
        t2[1:, 1:, 1:] = tempcoulomb
        if notwoflag == 1:                          # sincproject.f90:330-332
            t2[:] = 0.0
        self.threed_two = np.asfortranarray(t2)

        # nuclear potential  (sincproject.f90:192-250)
        ldims = np.full(3, 1 - g)
        udims = np.full(3, g - 1)
        pps, qqs = [], []
        for c in range(len(nuccharges)):
            pp = -g + centershift[c] + 1
            qq = g + centershift[c] - 1
            for ii in range(3):
                if _fortran_mod(int(qq[ii]), 2) == 1 or _fortran_mod(int(pp[ii]), 2) == 1:
                    raise ValueError("nucleus not on the grid / half-grid parity rule")
            pp = np.array([_fortran_div(int(v), 2) for v in pp])
            qq = np.array([_fortran_div(int(v), 2) for v in qq])
            pps.append(pp)
            qqs.append(qq)
            ldims = np.minimum(ldims, pp)
            udims = np.maximum(udims, qq)
        ax = [np.arange(ldims[k], udims[k] + 1) for k in range(3)]
        isq = (ax[0][:, None, None] ** 2 + ax[1][None, :, None] ** 2 + ax[2][None, None, :] ** 2)
        with np.errstate(divide="ignore"):
            if sqrt32:
                rval = spacing * np.sqrt(isq.astype(np.float32)).astype(np.float64)
            else:
                rval = spacing * np.sqrt(isq.astype(np.float64))
            big = 1.0 / rval
        o = -ldims
        big[o[0] - (g - 1):o[0] + g, o[1] - (g - 1):o[1] + g, o[2] - (g - 1):o[2] + g] = tempcoulomb
        pot = np.zeros((g, g, g))
        for c in range(len(nuccharges)):
            pp = pps[c]
            sl = tuple(slice(pp[k] + o[k], pp[k] + o[k] + g) for k in range(3))
            pot = pot - 1.0 * nuccharges[c] * big[sl]
        self.pot = np.asfortranarray(pot).reshape(self.G, order="F")

        # nuclear repulsion (sinc_extraproject.f90:290-300)
        nr = 0.0
        for i in range(len(nuccharges)):
            for j in range(i + 1, len(nuccharges)):
                rsq = ((centershift[i] - centershift[j]) * spacing / 2) ** 2
                nr += nuccharges[i] * nuccharges[j] / math.sqrt(rsq[0] + rsq[1] + rsq[2])
        self.nucrepulsion = nr

        # z dipole = grid coordinate (SINCDVR/coreproject.f90 get_dipoles)
        z = np.broadcast_to(self.points[None, None, :], (g, g, g))
        self.zdipole = np.asfortranarray(z).reshape(self.G, order="F").copy()

    # -----------------------------------------------------------------------
    # a5: op_tinv -> circ3d_sub
    # -----------------------------------------------------------------------
    def op_tinv(self, twoeden03: np.ndarray, workers: int = 1) -> np.ndarray:
        """SINCDVR/coreproject.f90:366-537 (serial path) with circ3d_sub
        SINCDVR/toeplitz_subs.f90:561-589.  twoeden03(totpoints, allsize).
        `workers` > 1 runs the (same, forward-unnormalised) FFTs multithreaded."""
        g = self.N
        if workers > 1:
            import scipy.fft as sfft

            def fftn(a):
                return sfft.fftn(a, axes=(0, 1, 2), workers=workers)
        else:
            def fftn(a):
                return np.fft.fftn(a, axes=(0, 1, 2))
        dens = np.asarray(twoeden03, dtype=np.complex128).reshape(g, g, g, -1, order="F")
        m = dens.shape[3]
        huge = np.zeros((2 * g, 2 * g, 2 * g, m), dtype=np.complex128, order="F")
        huge[:g, :g, :g, :] = dens                       # octant (1,1,1), line 450
        ffvec = fftn(huge)
        ffmat = fftn(self.threed_two.astype(np.complex128))
        ffprod = ffvec * ffmat[:, :, :, None] / (2 * g) ** 3
        ffprod = np.conj(ffprod)
        ffback = np.conj(fftn(ffprod))
        red = ffback[g:, g:, g:, :]                      # octant (2,2,2), line 521
        return np.asfortranarray(red).reshape(self.G, m, order="F")

    # -----------------------------------------------------------------------
    # a4: call_twoe_matel00
    # -----------------------------------------------------------------------
    def call_twoe_matel00(self, inspfs10, inspfs20, workers: int = 1):
        """SINCDVR/coreproject.f90:945-1194 with fft_batchdim=1,
        fft_circbatchdim=1 (defaults, sinc_params.f90:22-23), lowspf=1,
        highspf=numspf.  Returns (twoematel(n,n,n,n), twoereduced(G,n,n))."""
        phi1 = np.asarray(inspfs10, dtype=np.complex128)
        phi2 = np.asarray(inspfs20, dtype=np.complex128)
        G, n = phi1.shape
        red = np.zeros((G, n, n), dtype=np.complex128, order="F")
        for b in range(n):                                   # lines 1042-1081
            den = phi1 * np.conj(phi2[:, b])[:, None]        # line 1063
            red[:, :, b] = self.op_tinv(den, workers=workers)
        mat = np.zeros((n, n, n, n), dtype=np.complex128, order="F")
        R = red.reshape(G, n * n, order="F")
        for b1 in range(n):                                  # lines 1089-1099
            for a1 in range(n):
                myden = phi1[:, a1] * np.conj(phi2[:, b1])
                mat[a1, b1, :, :] = (R.T @ myden).reshape(n, n, order="F")
        return mat, red

    # -----------------------------------------------------------------------
    # a8: mult_ke
    # -----------------------------------------------------------------------
    def mult_ke(self, inp):
        """SINCDVR/coreproject.f90:2104-2116 -> mult_general_withbcast
        (1321-1390) -> mult_all0 (2070-2097): out(a,j,b)=sum_l in(a,l,b) ketot(l,j)
        for each axis, summed over axes."""
        g = self.N
        x = np.asarray(inp, dtype=np.complex128).reshape(g, g, g, -1, order="F")
        K = self.ketot
        # the three contractions as tensordots (BLAS); same sums as the
        # reference's per-axis ZGEMMs, summation order aside
        out = np.tensordot(K, x, axes=([0], [0]))                               # (j, y, z, m)
        out = out + np.moveaxis(np.tensordot(x, K, axes=([1], [0])), 3, 1)      # (x, j, z, m)
        out = out + np.moveaxis(np.tensordot(x, K, axes=([2], [0])), 3, 2)      # (x, y, j, m)
        return np.asfortranarray(out).reshape(self.G, -1, order="F")

    def mult_pot(self, inp):
        """MCTDH.SRC/proputils.f90:126-140 (contact operator off)."""
        return np.asarray(inp) * self.pot[:, None]

    def mult_zdipole(self, inp):
        """z-dipole multiply used by lenmultiply (proputils.f90:157-182)."""
        return np.asarray(inp) * self.zdipole[:, None]


# ---------------------------------------------------------------------------
# a6, a9: reduced potential
# ---------------------------------------------------------------------------
def get_reducedpot(twoereduced, reducedpottally):
    """MCTDH.SRC/mean.f90:503-588: reducedpot(G,n^2) = twoereduced(G,n^2) x
    reducedpottally(n^2,n^2)  (ZGEMM, line 556-558)."""
    G, n, _ = twoereduced.shape
    R = twoereduced.reshape(G, n * n, order="F")
    T = reducedpottally.reshape(n * n, n * n, order="F")
    return np.asfortranarray(R @ T).reshape(G, n, n, order="F")


def mult_reducedpot(inspfs, reducedpot):
    """SINCDVR/coreproject.f90:1200-1235: out(:,i)=sum_k reducedpot(:,k,i)*inspfs(:,k)."""
    return np.einsum("xki,xk->xi", reducedpot, inspfs)


# ---------------------------------------------------------------------------
# a10: orbital RHS
# ---------------------------------------------------------------------------
def dot(bra, ket):
    """MCTDH.SRC/parameters.f90:43-54 hermitian dot: sum conj(bra)*ket."""
    return np.vdot(bra, ket)


def project00(inspfs, prospfs):
    """MCTDH.SRC/proputils.f90:10-61: out = prospfs x mydot, mydot(j,i)=<pro_j|in_i>."""
    mydot = np.conj(prospfs).T @ inspfs
    return prospfs @ mydot


def actreduced00(sysm: SincSystem, inspfs, projspfs, denmat, invdenmat, reducedpot,
                 timefac=-1j, dentimeflag=1, projflag=1, ztdpot=0.0):
    """MCTDH.SRC/derivs.f90:629-852 for the sinc project (numr=1,
    bondpoints=1, nonuc_checkflag=1, numfrozen=0, scalarflag=0,
    length gauge z pulse with strength ztdpot)."""
    inspfs = np.asarray(inspfs, dtype=np.complex128)
    spfinvrsq = inspfs @ denmat                       # lines 674-676
    spfmult = sysm.mult_ke(spfinvrsq)                 # line 712
    spfmult = spfmult + sysm.mult_pot(spfinvrsq)      # line 719 (spfinvr=spfinvrsq)
    if ztdpot != 0.0:                                 # lines 741-752, lenmultiply
        spfmult = spfmult + sysm.mult_zdipole(spfinvrsq) * ztdpot
    spfmult = spfmult + mult_reducedpot(inspfs, reducedpot)   # line 763
    if dentimeflag != 0:
        spfmult = timefac * (spfmult @ invdenmat)     # lines 788-790
    if projflag == 1:
        spfmult = spfmult - project00(spfmult, projspfs)   # lines 806-807
    return spfmult


def invmatsmooth(a, tol=1e-10, relflag=False):
    """MCTDH.SRC/utils.f90:533-611 regularised SVD inverse."""
    u, sv, vt = np.linalg.svd(a)
    mytol = tol * sv[0] if relflag else tol
    inv = np.zeros_like(sv)
    for k in range(len(sv)):
        if sv[k] != 0.0:
            inv[k] = 1.0 / mytol if sv[k] < mytol else 1.0 / sv[k]
    return (np.conj(vt).T * inv[None, :]) @ np.conj(u).T


# ---------------------------------------------------------------------------
# seeded inputs shared by oracle and GPU tests
# ---------------------------------------------------------------------------
def gram_schmidt(spfs):
    """MCTDH.SRC/utils.f90:275-292 style modified Gram-Schmidt in index order
    with the hermitian dot."""
    out = np.array(spfs, dtype=np.complex128, order="F")
    n = out.shape[1]
    for i in range(n):
        for j in range(i):
            out[:, i] -= out[:, j] * dot(out[:, j], out[:, i])
        out[:, i] /= math.sqrt(dot(out[:, i], out[:, i]).real)
    return out


def seeded_orbitals(sysm: SincSystem, nspf: int, seed: int, width=1.0):
    """phi_k(x) = exp(-|x|^2/(2 w^2)) * z_k(x), z ~ CN(0,1), then Gram-Schmidt."""
    rng = np.random.default_rng(seed)
    g = sysm.N
    p = sysm.points
    r2 = p[:, None, None] ** 2 + p[None, :, None] ** 2 + p[None, None, :] ** 2
    env = np.exp(-r2 / (2 * width ** 2)).reshape(sysm.G, order="F")
    z = (rng.standard_normal((sysm.G, nspf)) + 1j * rng.standard_normal((sysm.G, nspf))) / math.sqrt(2)
    return gram_schmidt(env[:, None] * z)


def seeded_hermitian_psd(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = a @ np.conj(a).T / n + 0.1 * np.eye(n)
    return np.asfortranarray(h)


def seeded_tally(n, seed):
    """A Hermitian-structured 2-RDM-like tally: Gamma(a,b,c,d) =
    conj(Gamma(b,a,d,c)), Gamma(a,b,c,d) = Gamma(c,d,a,b)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, n, n, n)) + 1j * rng.standard_normal((n, n, n, n))
    g = g + np.conj(g.transpose(1, 0, 3, 2))
    g = g + g.transpose(2, 3, 0, 1)
    return np.asfortranarray(g / 4)
