"""CPU oracle for doublyexcited's two-electron matvec and GPLMR eigensolver.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s cpu_baseline / ``--impl reference`` arm may import this module,
and only as the checker (or as the timed CPU restatement of the reference).
The product package never imports it.

It restates, loop for loop where it matters, the Fortran reference
(paths relative to ``complexscale-djhnow/code/``):

* operator set-up: ``INIT_PARAMETERS`` initmod.F90:15-51, ``INIT_HAMILTONIAN``
  initmod.F90:174-228, ``KEMATRIX`` hammod.F90:235-260, ``GETINVERSE`` /
  ``RVECTOR`` / ``TOOTHEIGMULT`` tooth.f90:14-204, ``POTENTIAL1/2``
  hammod.F90:432-582;
* the matvec ``HAMMULT`` hammod.F90:19-67 (C loops in ``de_oracle.c``);
* ``GPLMR_EIG`` gplmr.F90:9-374 with ``SOLVE_GEVP``/``EIGSORT``
  gplmr.F90:395-439,640-660 and ``PRECBLOCK``/``PRECBLOCK_BASIC``
  gplmr.F90:466-502,674-770;
* the block ops ``normalize``/``crossmult_diag``/``colnorms``/``crossmult``/
  ``cholQR`` lamod.f90:21-180;
* the inner solve ``basicblocklansolve``/``harm_orthog_oneblock``/
  ``fast_harmritz_setup``/``myhgramschmidt_many``
  harmonic_ritz_small.F90:28-324 and ``gen_cmatsub`` hr_eigen.f90:223-291;
  the alternative ``PRECBLOCK_PETSC`` gplmr.F90:507-563 as GMRES in the
  configuration ``PETSCSOLVE`` petscsolve.F90:142-279 sets (PETSc is absent:
  the published algorithm, parity with PETSc itself unpinned);
* ``GET_EXPECTS`` hammod.F90:1261-1301 and the shift rule
  doublyexcited.F90:214-219;
* the initial guess: He+ orbitals (dense, where the reference runs block
  Lanczos), ``HELIUM_ORBITALGATHER`` / ``HELIUM_ORBITAL`` /
  ``DIAGSUBSPACE`` / ``mysort`` hammod.F90:1041-1256,1658-1690.

Dense LAPACK calls go to the same routines the reference calls (``dsyev``,
``zggev``, ``zgesdd``, ``zpotrf``, ``ztrsm``) through scipy's LAPACK.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.linalg.blas as sblas
import scipy.linalg.lapack as slapack

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    """Compile ``de_oracle.c`` into ``oracle/_build/libde_oracle.so``."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "_build", "libde_oracle.so")


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "libde_oracle.so")
        src = os.path.join(_HERE, "de_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.or_kematrix.argtypes = [ctypes.c_int, ctypes.c_double, P]
        L.or_rvector.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, P, P]
        L.or_tootheigmult.argtypes = [P, P, P, ctypes.c_int]
        L.or_potential1.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, P, P]
        L.or_potential2.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, P, P]
        L.or_hammult2.argtypes = [ctypes.c_int, P, P, P, P, P, P]
        L.or_hammult1.argtypes = [ctypes.c_int, P, P, P, P]
        for f in (L.or_kematrix, L.or_rvector, L.or_tootheigmult, L.or_potential1,
                  L.or_potential2, L.or_hammult2, L.or_hammult1):
            f.restype = None
        _LIB = L
    return _LIB


def _p(a: np.ndarray) -> ctypes.c_void_p:
    assert a.flags["F_CONTIGUOUS"] or a.ndim == 1
    return ctypes.c_void_p(a.ctypes.data)


# --------------------------------------------------------------------------
# set-up


def kematrix(nn: int, delta: float) -> np.ndarray:
    """Real sinc-DVR kinetic matrix, KEMATRIX hammod.F90:235-260."""
    t = np.zeros((nn, nn), order="F")
    lib().or_kematrix(nn, float(delta), _p(t))
    return t


def getinverse(nout: int, nbig: int, nsmall: int, delta: float) -> np.ndarray:
    """Regularised inverse-Laplacian table TINV on (-nout..nout)^3.

    GETINVERSE tooth.f90:14-101: R = delta^3/|r| on the big grid, TR = -T R
    on the small grid (RVECTOR :106-172), TR(0,0,0) += 2 pi, solve
    T_3D Q = TR in the eigenbasis of the 1-D T (DSYEV('V','U'), LWORK=6*NS),
    TINV = R + Q on the small grid, cropped to +-nout.
    """
    if nbig < nout:
        raise ValueError("nbig lt nout")
    nb, ns = 2 * nbig + 1, 2 * nsmall + 1
    r = np.zeros((nb, nb, nb), order="F")
    tr = np.zeros((ns, ns, ns), order="F")
    lib().or_rvector(nbig, nsmall, float(delta), _p(r), _p(tr))
    tr[nsmall, nsmall, nsmall] += 2 * math.pi
    pi = 4.0 * math.atan(1.0)
    idx = np.arange(-nsmall, nsmall + 1)
    d = idx[:, None] - idx[None, :]
    with np.errstate(divide="ignore"):
        t = np.where(d == 0, (pi / delta) ** 2 / 6.0,
                     np.where(d % 2 == 0, 1.0, -1.0) / (delta ** 2 * d.astype(float) ** 2))
    e, w, info = slapack.dsyev(np.asfortranarray(t), compute_v=1, lower=0, lwork=6 * ns)
    if info != 0:
        raise RuntimeError(f"dsyev info={info}")
    w = np.asfortranarray(w)
    wt = np.asfortranarray(w.T)
    eigs = e[:, None, None] + e[None, :, None] + e[None, None, :]
    qq = np.zeros((ns, ns, ns), order="F")
    lib().or_tootheigmult(_p(tr), _p(qq), _p(wt), ns)
    qq = np.asfortranarray(qq / eigs)
    q = np.zeros((ns, ns, ns), order="F")
    lib().or_tootheigmult(_p(qq), _p(q), _p(w), ns)
    lo, hi = nbig - nsmall, nbig + nsmall + 1
    r[lo:hi, lo:hi, lo:hi] += q
    return np.asfortranarray(r[nbig - nout:nbig + nout + 1, nbig - nout:nbig + nout + 1,
                               nbig - nout:nbig + nout + 1])


@dataclass
class Params:
    """Grid/physics parameters (PARAMETERS, structs.F90:28-57)."""

    n: int
    delta: float = 2.0
    theta: float = 0.2
    charge: float = 2.0
    nsmall: int = 22
    tfactor: int = 4

    @property
    def nn(self) -> int:
        return 2 * self.n + 1

    @property
    def m(self) -> int:
        return self.nn ** 3

    @property
    def scale(self) -> complex:
        return complex(math.cos(self.theta), math.sin(self.theta))


@dataclass
class Hamiltonian:
    """Operator data (HAMILTONIAN, structs.F90:87-102) for NELEC = 1 or 2."""

    params: Params
    nelec: int
    t_real: np.ndarray
    tinv: np.ndarray
    t: np.ndarray = field(repr=False)
    v: np.ndarray = field(repr=False)
    _w: np.ndarray | None = field(default=None, repr=False)
    _z: np.ndarray | None = field(default=None, repr=False)
    calls: int = 0

    @property
    def dim(self) -> int:
        return self.params.m ** self.nelec

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """HAMMULT hammod.F90:19-67 (NP = 1)."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        assert x.shape == (self.dim,)
        y = np.empty_like(x)
        self.calls += 1
        if self.nelec == 2:
            if self._w is None:
                self._w = np.empty(self.dim, np.complex128)
                self._z = np.empty(self.dim, np.complex128)
            lib().or_hammult2(self.params.nn, _p(self.t), _p(self.v), _p(x), _p(y),
                              _p(self._w), _p(self._z))
        else:
            lib().or_hammult1(self.params.nn, _p(self.t), _p(self.v), _p(x), _p(y))
        return y

    def matblock(self, x: np.ndarray) -> np.ndarray:
        """MATBLOCK gplmr.F90:443-462: one HAMMULT per column."""
        out = np.empty_like(x)
        for j in range(x.shape[1]):
            out[:, j] = self.matvec(x[:, j])
        return out


_TINV_CACHE: dict = {}


def tinv_table(p: Params) -> np.ndarray:
    key = (p.nn, p.tfactor * p.nsmall, p.nsmall, p.delta)
    if key not in _TINV_CACHE:
        _TINV_CACHE[key] = getinverse(p.nn, p.nsmall * p.tfactor, p.nsmall, p.delta)
    return _TINV_CACHE[key]


def init_hamiltonian(p: Params, nelec: int = 2) -> Hamiltonian:
    """INIT_HAMILTONIAN initmod.F90:174-228 with the nucleus on the grid."""
    t_real = kematrix(p.nn, p.delta)
    t = np.asfortranarray(t_real / p.scale ** 2)
    tinv = tinv_table(p)
    if nelec == 1:
        v = np.zeros(p.m)
        lib().or_potential1(p.n, float(p.delta), float(p.charge), _p(tinv), _p(v))
    elif nelec == 2:
        v = np.zeros(p.m * p.m)
        lib().or_potential2(p.n, float(p.delta), float(p.charge), _p(tinv), _p(v))
    else:
        raise ValueError("nelec must be 1 or 2")
    v = v / p.scale
    return Hamiltonian(p, nelec, t_real, tinv, t, v.astype(np.complex128))


def dense_one_electron(h: Hamiltonian) -> np.ndarray:
    """Dense one-electron H = T(x)1(x)1 + 1(x)T(x)1 + 1(x)1(x)T + diag(V)."""
    assert h.nelec == 1
    nn = h.params.nn
    eye = np.eye(nn)
    t = h.t
    hk = (np.kron(np.kron(eye, eye), t) + np.kron(np.kron(eye, t), eye)
          + np.kron(np.kron(t, eye), eye))
    return hk + np.diag(h.v)


# --------------------------------------------------------------------------
# block operations (lamod.f90)


def hdot(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Hermitian cross products A^H B (crossmult, lamod.f90:106-125)."""
    return a.conj().T @ b


def cdot(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Unconjugated c-products A^T B (MPIDOT, hammod.F90:361-380)."""
    return a.T @ b


def colnorms(x: np.ndarray) -> np.ndarray:
    """sqrt(diag(X^H X)) via ddot on the interleaved reals (lamod.f90:78-102)."""
    return np.sqrt(np.einsum("ij,ij->j", x.real, x.real) + np.einsum("ij,ij->j", x.imag, x.imag))


class CholeskyBreakdown(RuntimeError):
    pass


def cholqr(x: np.ndarray) -> np.ndarray:
    """In-place Cholesky QR, lamod.f90:128-180: R = chol(X^H X) upper,
    X <- X R^{-1} (ztrsm 'R','U','N','N').  Returns R."""
    g = hdot(x, x)
    if np.sum(np.abs(g)) == 0.0:
        r = g
    else:
        r, info = slapack.zpotrf(g, lower=0, clean=1)
        if info != 0:
            raise CholeskyBreakdown(f"Cholesky failed {info}")
    x[:] = trsm_right_upper(x, r)
    return r


def trsm_right_upper(x: np.ndarray, r: np.ndarray) -> np.ndarray:
    """X R^{-1} for upper triangular R (ztrsm 'R','U','N','N')."""
    return sblas.ztrsm(1.0, r, x, side=1, lower=0, trans_a=0, diag=0)


# --------------------------------------------------------------------------
# inner solve (harmonic_ritz_small.F90)


def gen_cmatsub_sqrt(a: np.ndarray, tol: float = 0.0):
    """gen_cmatsub flag=2, hr_eigen.f90:223-291: SVD A = U S V^H (zgesdd),
    returns (V S^{-1/2} U^H, V S^{1/2} U^H)."""
    n = a.shape[0]
    u, s, vt, info = slapack.zgesdd(np.asfortranarray(a.copy()), compute_uv=1, full_matrices=1)
    if info != 0:
        raise RuntimeError(f"zgesdd info={info}")
    sv = s.copy()
    for k in range(n):
        if sv[k] != 0.0:
            if sv[k] < tol * s[0]:
                sv[k] = 1.0 / tol / s[0]
            else:
                sv[k] = 1.0 / sv[k]
    sv = np.sqrt(sv)
    ssave = np.sqrt(s)
    v = vt.conj().T
    uh = u.conj().T
    return (v * sv[None, :]) @ uh, (v * ssave[None, :]) @ uh


class OrthoCheckFailed(RuntimeError):
    pass


def basicblocklansolve(x: np.ndarray, order: int, maxiter: int, sigma: complex, mult):
    """Fixed-order block min-residual approximation of (H - sigma)^{-1} X.

    basicblocklansolve harmonic_ritz_small.F90:258-324 with
    harm_orthog_oneblock :161-244 and fast_harmritz_setup :86-158 (both
    multiplication callbacks are the same unshifted H, gplmr.F90:700-701).
    """
    n, nblk = x.shape
    if order <= 0:
        raise ValueError("ORDERERROR")
    if order * nblk > maxiter:
        raise ValueError("Order*lanblocknum is greater than lansize")
    thisdim = min(maxiter, order * nblk)
    # harm_orthog_oneblock
    v1 = x.copy()
    w0 = mult(v1) - sigma * v1
    g = hdot(w0, w0)
    ginv, gsq = gen_cmatsub_sqrt(g, 0.0)
    v1 = v1 @ ginv.conj().T
    w1 = mult(v1) - sigma * v1
    chk = hdot(w1, w1) - np.eye(nblk)
    if np.any(np.abs(chk) > 1e-10):
        raise OrthoCheckFailed("AACK DOTS")
    # fast_harmritz_setup
    lv = np.zeros((n, nblk, order), np.complex128, order="F")
    lq = np.zeros((n, nblk, order), np.complex128, order="F")
    for io in range(order):
        nb_here = nblk
        if (io + 1) * nblk >= maxiter:
            nb_here = maxiter - io * nblk
        if io == 0:
            lv[:, :, 0] = v1
        else:
            lv[:, :nb_here, io] = mult(lv[:, :nb_here, io - 1])
        lq[:, :nb_here, io] = mult(lv[:, :nb_here, io]) - sigma * lv[:, :nb_here, io]
        for i in range(nb_here):
            m = io * nblk + i
            prev_q = lq.reshape(n, nblk * order, order="F")[:, :m]
            prev_v = lv.reshape(n, nblk * order, order="F")[:, :m]
            q = lq[:, i, io].copy()
            v = lv[:, i, io].copy()
            for _ in range(2):
                if m:
                    dots = prev_q.conj().T @ q
                    q = q - prev_q @ dots
                    v = v - prev_v @ dots
                nrm = np.vdot(q, q)
                nrm = math.sqrt(abs(nrm))
                q = q / nrm
                v = v / nrm
            lq[:, i, io] = q
            lv[:, i, io] = v
    qf = lq.reshape(n, nblk * order, order="F")
    vf = lv.reshape(n, nblk * order, order="F")
    lanham = hdot(qf, vf)
    rhs = np.zeros((order * nblk, nblk), np.complex128)
    rhs[:nblk, :] = gsq
    solve = lanham[:thisdim, :thisdim] @ rhs[:thisdim]
    return vf[:, :thisdim] @ solve


def _refl_image(v: np.ndarray, nn: int, r: int) -> np.ndarray:
    """R_r v: the axis reflections c -> nn-1-c of every axis a with bit a of
    r set, applied to both electrons (v flat, x1 fastest)."""
    a = v.reshape((nn,) * 6)  # C order: z2, y2, x2, z1, y1, x1
    for ax in range(3):
        if (r >> ax) & 1:
            a = np.flip(np.flip(a, 5 - ax), 2 - ax)
    return a.reshape(-1)


def reflection_sectors(x: np.ndarray, nn: int, rel: float = 1e-12) -> int:
    """Bit mask of the reflection sectors the columns of x reach: sector c
    (0..7) is the eigenspace where R_r has eigenvalue (-1)^popcount(c & r);
    a column reaches it when its component there has a squared norm above
    rel of the column's.  The library keeps the preconditioned blocks of
    its mixed form and of FP64 block solves in these sectors."""
    keep = 0
    for j in range(x.shape[1]):
        v = x[:, j]
        corr = [np.vdot(v, _refl_image(v, nn, r)).real for r in range(8)]
        for c in range(8):
            n2 = sum((-1) ** bin(c & r).count("1") * corr[r] for r in range(8)) / 8
            if n2 > rel * corr[0]:
                keep |= 1 << c
    return keep


def _round_c64(z: np.ndarray) -> np.ndarray:
    """Complex64 storage of a complex128 block (the mixed form's power basis)."""
    return z.astype(np.complex64).astype(np.complex128)


def reflection_project(v: np.ndarray, nn: int, keep: int) -> np.ndarray:
    """Projection of one flat vector onto the reflection sectors in keep:
    sum over kept c of (1/8) sum_r (-1)^popcount(c & r) R_r v."""
    w = np.zeros(8)
    for c in range(8):
        if (keep >> c) & 1:
            for r in range(8):
                w[r] += (-1) ** bin(c & r).count("1")
    out = np.zeros_like(v)
    for r in range(8):
        if w[r] != 0.0:
            out += (w[r] / 8) * _refl_image(v, nn, r)
    return out


def sstep_minres(x: np.ndarray, order: int, sigma: complex, mult, store=None) -> np.ndarray:
    """The library's mixed-form inner solve: the same minimal-residual
    approximation of (H - sigma)^{-1} X over the block Krylov space
    K_order(H, X) as basicblocklansolve, from the power basis Z_0 = X,
    Z_i = (H - sigma) Z_{i-1} and one Gram: with Q = [Z_1..Z_order] the
    solution is [Z_0..Z_order-1] a, (Q^H Q) a = Q^H X, solved after diagonal
    scaling D with a 1e-13 ridge by Cholesky:
    (D^-1 Q^H Q D^-1 + 1e-13 I) y = D^-1 Q^H X, a = D^-1 y.  `store` rounds
    every basis block as the library stores it (complex64 in the mixed
    form)."""
    k = x.shape[1]
    rnd = store if store is not None else (lambda v: v)
    z = [rnd(x)]
    for _ in range(order):
        z.append(rnd(mult(z[-1]) - sigma * z[-1]))
    zf = np.concatenate(z, axis=1)
    q = zf[:, k:]
    g = q.conj().T @ zf
    gq, rhs = g[:, k:], g[:, :k]
    d = np.sqrt(np.real(np.diag(gq)))
    gs = gq / d[:, None] / d[None, :] + 1e-13 * np.eye(gq.shape[0])
    lo = np.linalg.cholesky(gs)
    y = np.linalg.solve(lo.conj().T, np.linalg.solve(lo, rhs / d[:, None]))
    return zf[:, :order * k] @ (y / d[:, None])


# --------------------------------------------------------------------------
# GPLMR (gplmr.F90)


@dataclass
class GplmrResult:
    e: np.ndarray
    x: np.ndarray
    iterations: int
    residuals: np.ndarray
    history: list
    matvecs: int


def solve_gevp(kp: np.ndarray, mp: np.ndarray, k: int, nev: int) -> np.ndarray:
    """SOLVE_GEVP gplmr.F90:395-439: ZGGEV('N','V') on the leading k x k
    pencil, sort |alpha/beta| ascending (EIGSORT :640-660, first minimum on
    ties), return the nev right eigenvectors (k x nev)."""
    a = np.asfortranarray(kp[:k, :k].copy())
    b = np.asfortranarray(mp[:k, :k].copy())
    alpha, beta, vl, vr, work, info = slapack.zggev(a, b, compute_vl=0, compute_vr=1,
                                                    lwork=10 * max(1, 2 * k))
    if info != 0:
        raise RuntimeError("SOLVE OF THE PROJECTED EIGENVALUE PROBLEM FAILED")
    lam = np.abs(alpha / beta)
    y = lam.copy()
    mx = y.max()
    idx = []
    for _ in range(nev):
        i = int(np.argmin(y))
        idx.append(i)
        y[i] = mx + 1
    return vr[:, idx]


@dataclass
class GmresResult:
    x: np.ndarray
    its: int
    rnorm: float
    reason: str


def kinetic_eigs(h: Hamiltonian) -> tuple[np.ndarray, np.ndarray]:
    """KINETIC_EIGS littlesolver.F90:709-740: W, the eigenvectors of the real
    kinetic matrix (DSYEV('V','U') of Re(T)/cos(2 theta), which is T_real),
    and the eigenvalue sums (lam_i + lam_j + lam_k) / SCALE^2 of the 3D
    operator on the (NN, NN, NN) grid (i fastest, as ALLEIGS)."""
    lam, w, info = slapack.dsyev(np.asfortranarray(h.t_real), compute_v=1, lower=0)
    if info != 0:
        raise RuntimeError(f"dsyev info {info}")
    alleigs = (lam[:, None, None] + lam[None, :, None] + lam[None, None, :]) / h.params.scale ** 2
    return np.asfortranarray(w), alleigs


def _axes_apply(x: np.ndarray, mat: np.ndarray, axes) -> np.ndarray:
    """mat applied along each of the given axes of x: y_a = sum_i mat[a, i] x_i."""
    for ax in axes:
        x = np.moveaxis(np.tensordot(mat, x, axes=([1], [ax])), 0, ax)
    return x


def msolve22(h: Hamiltonian, r: np.ndarray, shift: complex = 0.0) -> np.ndarray:
    """MSOLVECPLX22 littlesolver.F90:372-436, the PETSc path's "spectral
    decomposition" shell preconditioner (PC option 2).  With W and the
    eigenvalue sums of kinetic_eigs, P = W diag(1 / (alleigs - shift)) W^T
    on a 3D cube (EIGMULT hammod.F90:764-799 with WT, the division, EIGMULT
    with W).  One electron: z = P r.  Two: P on every column cube (electron
    1) plus P on every row cube (electron 2, through MPITRANSPOSE), added."""
    nn = h.params.nn
    w, alleigs = kinetic_eigs(h)
    dinv = 1.0 / (alleigs - shift)
    r = np.asarray(r, dtype=np.complex128)
    if h.nelec == 1:
        x3 = r.reshape((nn,) * 3, order="F")
        return _axes_apply(_axes_apply(x3, w.T, (0, 1, 2)) * dinv, w, (0, 1, 2)).reshape(-1, order="F")
    x6 = r.reshape((nn,) * 6, order="F")  # (i1, j1, k1, i2, j2, k2)
    z1 = _axes_apply(_axes_apply(x6, w.T, (0, 1, 2)) * dinv[:, :, :, None, None, None], w, (0, 1, 2))
    z2 = _axes_apply(_axes_apply(x6, w.T, (3, 4, 5)) * dinv[None, None, None, :, :, :], w, (3, 4, 5))
    return (z1 + z2).reshape(-1, order="F")


def petsc_gmres(apply, b: np.ndarray, max_it: int, rtol: float, abstol: float = 1e-50,
                restart: int = 30, haptol: float = 1e-30) -> GmresResult:
    """KSPSolve as PETSCSOLVE petscsolve.F90:142-279 configures it, called
    column by column from PRECBLOCK_PETSC gplmr.F90:507-563.  The settings:
    KSPGMRES with PETSc's defaults, restart 30, classical Gram-Schmidt
    without refinement, no preconditioner (GM_PCOPT = 0 and a shell
    operator), zero initial guess.  KSPSetTolerances(rtol = GM_TOL,
    max_it = GM_MAX_INNER_ITER).  The default test stops when the Arnoldi
    residual estimate |g_{k+1}| <= max(rtol ||b||, abstol).  Inner products
    are Hermitian.

    PETSc is a third-party library absent here: this restates the published
    GMRES algorithm in the structure of PETSc's KSPGMRESCycle (one operator
    application per iteration, Givens rotations on the Hessenberg column,
    back substitution at the end of a cycle; a restart recomputes
    r = b - A x without counting an iteration)."""
    b = np.asarray(b, dtype=np.complex128)
    x = np.zeros_like(b)
    bnorm = float(np.linalg.norm(b))
    ttol = max(rtol * bnorm, abstol)
    if bnorm <= ttol:
        return GmresResult(x, 0, bnorm, "converged_atol")
    its = 0
    r = b.copy()
    reason = ""
    res = bnorm
    while not reason:
        beta = float(np.linalg.norm(r))
        vs = [r / beta]
        hh = np.zeros((restart + 1, restart), np.complex128)
        g = np.zeros(restart + 1, np.complex128)
        g[0] = beta
        cs = np.zeros(restart, np.complex128)
        sn = np.zeros(restart, np.complex128)
        k = 0
        while k < restart and its < max_it:
            w = apply(vs[k])
            coef = np.array([np.vdot(vs[i], w) for i in range(k + 1)])  # classical: all on w
            for i in range(k + 1):
                w = w - vs[i] * coef[i]
            tt = float(np.linalg.norm(w))
            col = np.zeros(restart + 1, np.complex128)
            col[:k + 1] = coef
            col[k + 1] = tt
            for i in range(k):  # earlier rotations
                a0, a1 = col[i], col[i + 1]
                col[i] = np.conj(cs[i]) * a0 + sn[i] * a1
                col[i + 1] = -np.conj(sn[i]) * a0 + cs[i] * a1
            hap = tt < min(abs(tt / g[k]) if g[k] != 0 else haptol, haptol)
            den = math.sqrt(abs(col[k]) ** 2 + abs(col[k + 1]) ** 2)
            if den == 0.0:  # KSP_DIVERGED_NULL: keep the earlier columns
                its += 1
                reason = "diverged_null"
                break
            cs[k], sn[k] = col[k] / den, col[k + 1] / den
            col[k] = den
            col[k + 1] = 0.0
            g[k + 1] = -np.conj(sn[k]) * g[k]
            g[k] = np.conj(cs[k]) * g[k]
            hh[:, k] = col
            res = abs(g[k + 1])
            k += 1
            its += 1
            if res <= ttol:
                reason = "converged_rtol"
            elif hap:
                reason = "happy_breakdown"
            elif its >= max_it:
                reason = "diverged_its"
            if reason:
                break
            vs.append(w / tt)
        y = np.zeros(k, np.complex128)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - hh[i, i + 1:k] @ y[i + 1:k]) / hh[i, i]
        for i in range(k):
            x = x + vs[i] * y[i]
        if not reason:
            r = b - apply(x)
    return GmresResult(x, its, res, reason)


def gplmr_eig(h: Hamiltonian, x0: np.ndarray, sigma: complex, ns: int = 5, maxit: int = 100,
              tol: float = 1e-7, order: int = 5, compat_first_column_only: bool = False,
              max_inner_iter: int | None = None, verbose: bool = False, usepetscflag: int = 1,
              gm_tol: float = 1e-3, gm_shift: complex = 0.0, equilibrate: bool = True,
              symmetry_project: bool = True, mixed: bool = False, gm_pcopt: int = 0) -> GplmrResult:
    """GPLMR_EIG gplmr.F90:9-374 with the BASIC preconditioner, or with
    usepetscflag = 0 the PETSc GMRES one (PRECBLOCK gplmr.F90:466-502):
    GMRES on (H - gm_shift) per column with rtol gm_tol.  The reference's
    GMSOLVER%SHIFT is never assigned and lives in the main program's
    zero-initialised storage, so gm_shift defaults to 0.  gm_pcopt = 2
    preconditions that GMRES on the left with msolve22 (PETSc's default side
    for a shell PC: GMRES on M^-1 (H - gm_shift) and M^-1 b, the stop test
    on the preconditioned residual), the option the reference wires as
    PC_GL = GMSOLVER%PCOPT (petscsolve.F90:109-114,179) but hard-codes to
    0 (GM_PCOPT, input.F90:67).

    equilibrate (default on; off restates the reference exactly): with
    NEV > 1 the residual block handed to PRECBLOCK_BASIC is scaled to unit
    columns first.  The reference passes the raw residuals
    (gplmr.F90:95-101); once a column converges, the Gram of (H - sigma) V
    in harm_orthog_oneblock (harmonic_ritz_small.F90:187-242) has a
    condition number near the squared ratio of the column norms (4e10 at
    N=3, NEV=4, iteration 21) and the 1e-10 self-check stops the run.  The
    inner solve's output is linear in column scaling (a minimal-residual
    solve over the block Krylov space, which scaling leaves unchanged) and
    GPLMR's next step, cholQR, removes the scale, so the iteration is the
    same in exact arithmetic.  The first-column-only mode is never scaled.

    symmetry_project (default on; off restates the reference): a block
    solve (NEV > 1, BASIC path) whose start columns are all exchange-
    symmetric (or all antisymmetric) projects each preconditioned block back
    onto that sector, X <- (X +- X^T)/2, and onto the reflection sectors
    the start columns reach (reflection_sectors; a no-op for a start that
    reaches all eight).  Exact arithmetic never leaves these sectors;
    rounding does, and at N = 3, 4 with NEV = 4 a singlet start otherwise
    converges to a triplet triple nearer sigma.

    mixed: the library's mixed form.  The inner solve is sstep_minres with
    its power basis rounded to complex64 (the library's FP32 matvecs are
    emulated by rounding FP64 ones), and every preconditioned block, for
    any NEV, is projected back onto the start block's exchange sector and
    onto the reflection sectors its columns reach: complex64 rounding leaks
    into the other sectors at the 1e-7 level, and the iteration amplifies a
    leaked state that lies nearer sigma."""
    if max_inner_iter is None:
        max_inner_iter = order
    calls0 = h.calls
    x = np.array(x0, dtype=np.complex128, order="F", copy=True)
    d, nev = x.shape
    ldr = ns * nev
    nproj = (3 + ns) * nev

    def precblock(blk: np.ndarray) -> np.ndarray:
        if max_inner_iter == 1:
            return h.matblock(blk)
        if usepetscflag == 0:
            out = np.empty_like(blk)
            for j in range(blk.shape[1]):
                if gm_pcopt == 2:
                    out[:, j] = petsc_gmres(lambda v: msolve22(h, h.matvec(v) - gm_shift * v, gm_shift),
                                            msolve22(h, blk[:, j], gm_shift), max_inner_iter, gm_tol).x
                else:
                    out[:, j] = petsc_gmres(lambda v: h.matvec(v) - gm_shift * v, blk[:, j], max_inner_iter,
                                            gm_tol).x
            return out

        def mult(v: np.ndarray) -> np.ndarray:
            if compat_first_column_only:
                out = np.zeros_like(v)
                out[:, 0] = h.matvec(v[:, 0])
                return out
            return h.matblock(v)

        if mixed:
            blk = blk / colnorms(blk)[None, :]
            out = sstep_minres(blk, max_inner_iter, sigma, mult, store=_round_c64)
            return project(out)
        if equilibrate and not compat_first_column_only and blk.shape[1] > 1:
            # unit columns: the inner solve's output is linear in column
            # scaling and cholQR removes it again, so only the conditioning
            # of harm_orthog_oneblock's Gram changes (see gplmr_eig)
            blk = blk / colnorms(blk)[None, :]
        out = basicblocklansolve(blk, max_inner_iter, h.params.m ** 2, sigma, mult)
        return project(out) if blk.shape[1] > 1 else out

    def project(out: np.ndarray) -> np.ndarray:
        m = h.params.m
        for j in range(out.shape[1]):
            if exch_sign != 0.0:
                z = out[:, j].reshape(m, m, order="F")
                out[:, j] = (0.5 * (z + exch_sign * z.T)).reshape(-1, order="F")
            if refl_keep != 0xFF:
                out[:, j] = reflection_project(out[:, j], h.params.nn, refl_keep)
        return out

    x /= colnorms(x)[None, :]
    # exchange sector of the start block (+1 every column symmetric, -1
    # every column antisymmetric, 0 otherwise) and the reflection sectors its
    # columns reach, kept by block solves and by the mixed form
    exch_sign = 0.0
    refl_keep = 0xFF
    if mixed and (compat_first_column_only or usepetscflag == 0 or max_inner_iter < 2):
        raise ValueError("the mixed form is the BASIC inner solve of order >= 2")
    if (mixed or (symmetry_project and nev > 1)) and not compat_first_column_only and usepetscflag != 0 \
            and max_inner_iter > 1:
        refl_keep = reflection_sectors(x, h.params.nn)
        m = h.params.m
        signs = []
        for j in range(nev):
            z = x[:, j].reshape(m, m, order="F")
            r = float(np.vdot(z.reshape(-1), z.T.reshape(-1)).real)
            signs.append(1.0 if abs(r - 1.0) < 1e-8 else -1.0 if abs(r + 1.0) < 1e-8 else 0.0)
        exch_sign = signs[0] if all(sg == signs[0] for sg in signs) else 0.0
    ax = h.matblock(x)
    e = np.einsum("ij,ij->j", x.conj(), ax)
    w = ax - x * e[None, :]
    resnrm = colnorms(w)
    maxres = resnrm.max()
    it = 1
    p = np.zeros_like(x)
    ap = np.zeros_like(x)
    s = np.zeros((d, ldr), np.complex128, order="F")
    as_ = np.zeros((d, ldr), np.complex128, order="F")
    hist = []
    while it <= maxit and maxres > tol:
        r = cholqr(x)
        ax = trsm_right_upper(ax, r)
        if max_inner_iter > 0:
            w = precblock(w)
        r = hdot(x, w)
        w = w - x @ r
        cholqr(w)
        aw = h.matblock(w)
        if ns > 0:
            s1 = aw - w * e[None, :]
            if max_inner_iter > 0:
                s1 = precblock(s1)
            s1 = s1 - x @ hdot(x, s1)
            s1 = s1 - w @ hdot(w, s1)
            cholqr(s1)
            s[:, :nev] = s1
            as_[:, :nev] = h.matblock(s1)
            for l in range(2, ns + 1):
                j1, j2 = (l - 1) * nev, l * nev
                sl = as_[:, j1 - nev:j1] - s[:, j1 - nev:j1] * e[None, :]
                if max_inner_iter > 0:
                    sl = precblock(sl)
                sl = sl - x @ hdot(x, sl)
                sl = sl - w @ hdot(w, sl)
                sl = sl - s[:, :j1] @ hdot(s[:, :j1], sl)
                cholqr(sl)
                s[:, j1:j2] = sl
                as_[:, j1:j2] = h.matblock(sl)
        if it > 1:
            r = hdot(x, p)
            p = p - x @ r
            ap = ap - ax @ r
            r = hdot(w, p)
            p = p - w @ r
            ap = ap - aw @ r
            r = hdot(s, p)
            p = p - s @ r
            ap = ap - as_ @ r
            r = cholqr(p)
            ap = trsm_right_upper(ap, r)
        asx = ax - sigma * x
        asw = aw - sigma * w
        ass = as_ - sigma * s
        if it > 1:
            asp = ap - sigma * p
            bra = np.concatenate([asx, asw, ass, asp], axis=1)
            ket = np.concatenate([x, w, s, p], axis=1)
            k = nproj
        else:
            bra = np.concatenate([asx, asw, ass], axis=1)
            ket = np.concatenate([x, w, s], axis=1)
            k = nproj - nev
        kp = hdot(bra, bra)
        mp = hdot(bra, ket)
        vr = solve_gevp(kp, mp, k, nev)
        cx = vr[:nev]
        cw = vr[nev:2 * nev]
        cs = vr[2 * nev:2 * nev + ldr]
        if it > 1:
            cp = vr[2 * nev + ldr:nproj]
            p = p @ cp
            ap = ap @ cp
        else:
            p = np.zeros_like(x)
            ap = np.zeros_like(x)
        p = p + s @ cs
        ap = ap + as_ @ cs
        p = p + w @ cw
        ap = ap + aw @ cw
        x = x @ cx + p
        ax = ax @ cx + ap
        nrm = colnorms(x)
        x = x / nrm[None, :]
        ax = ax / nrm[None, :]
        e = np.einsum("ij,ij->j", x.conj(), ax)
        w = ax - x * e[None, :]
        resnrm = colnorms(w)
        maxres = resnrm.max()
        hist.append((it, e.copy(), resnrm.copy()))
        if verbose:
            print(f"ITERATION {it:5d}", " ".join(f"{z.real:.12f}{z.imag:+.12f}i" for z in e),
                  f"ERR {maxres:.2e}", flush=True)
        it += 1
    return GplmrResult(e, x, it - 1, resnrm, hist, h.calls - calls0)


def get_expects(h: Hamiltonian, psi: np.ndarray, cshiftopt: bool = False) -> np.ndarray:
    """GET_EXPECTS hammod.F90:1261-1301 (Hermitian quotients by default)."""
    out = []
    for j in range(psi.shape[1]):
        hp = h.matvec(psi[:, j])
        if cshiftopt:
            out.append(np.dot(psi[:, j], hp) / np.dot(psi[:, j], psi[:, j]))
        else:
            out.append(np.vdot(psi[:, j], hp) / np.vdot(psi[:, j], psi[:, j]))
    return np.array(out)


def sixd_fix(x: np.ndarray, n_in: int, n_out: int) -> np.ndarray:
    """SIXD_FIX utils.F90:186-198: a two-electron vector on the (2 n_in + 1)^6
    grid copied onto the (2 n_out + 1)^6 grid about the centre, cropped or
    zero-padded in all six indices (column-major, electron 1 fastest)."""
    a, b = 2 * n_in + 1, 2 * n_out + 1
    v = np.asarray(x, np.complex128).reshape((a,) * 6, order="F")
    out = np.zeros((b,) * 6, np.complex128, order="F")
    k = min(n_in, n_out)
    si = slice(n_in - k, n_in + k + 1)
    so = slice(n_out - k, n_out + k + 1)
    out[(so,) * 6] = v[(si,) * 6]
    return out.reshape(-1, order="F")


def gplmr_shift(expects: np.ndarray, nev: int, takerealpart: bool = True) -> complex:
    """doublyexcited.F90:214-219."""
    s = complex(np.sum(expects[:nev]) / nev)
    return complex(s.real, 0.0) if takerealpart else s


# --------------------------------------------------------------------------
# initial guess: He+ orbitals, product states, subspace diagonalisation


def heplus_orbitals(h1: Hamiltonian, numorbs: int):
    """The numorbs He+ levels of lowest real part and their right
    eigenvectors.  The reference converges them with block Lanczos
    (lanmod.F90, called from doublyexcited.F90:135-137); here a dense
    ZGEEV (np.linalg.eig) of the same operator."""
    w, v = np.linalg.eig(dense_one_electron(h1))
    idx = np.argsort(w.real, kind="stable")[:numorbs]
    return w[idx], np.asfortranarray(v[:, idx])


def orbital_gather(x: np.ndarray, hermopt: bool = False) -> np.ndarray:
    """The Gram-Schmidt of HELIUM_ORBITALGATHER hammod.F90:1084-1113:
    c-products (or Hermitian products with hermopt), modified, in order."""
    x = np.array(x, dtype=np.complex128, order="F", copy=True)
    dot = (lambda a, b: np.vdot(a, b)) if hermopt else (lambda a, b: np.dot(a, b))
    for i in range(x.shape[1]):
        for j in range(i):
            x[:, i] -= x[:, j] * dot(x[:, j], x[:, i])
        x[:, i] /= np.sqrt(dot(x[:, i], x[:, i]))
    return x


def helium_orbital(ev: np.ndarray, i: int, j: int, sign: int) -> np.ndarray:
    """HELIUM_ORBITAL hammod.F90:1041-1080: PSI(p,q) = X_i(p) X_j(q) +
    sign X_j(p) X_i(q), halved when i == j, else divided by sqrt(2);
    electron 1 (p) fastest."""
    a, b = ev[:, i], ev[:, j]
    psi = np.outer(a, b) + sign * np.outer(b, a)  # psi[p, q]
    psi = psi.reshape(-1, order="F")
    return psi / 2.0 if i == j else psi / math.sqrt(2.0)


def mysort_order(values: np.ndarray, etarget: complex) -> list:
    """mysort hammod.F90:1658-1690: repeatedly the untaken value nearest
    etarget; among equal distances the later index wins (.le.)."""
    n = len(values)
    taken = [False] * n
    order = []
    for _ in range(n):
        best, low = -1, None
        for i in range(n):
            if not taken[i]:
                d = abs(values[i] - etarget)
                if best < 0 or d <= low:
                    best, low = i, d
        taken[best] = True
        order.append(best)
    return order


def diagsubspace(h2: Hamiltonian, ev: np.ndarray, singlet: bool, hermopt: bool, etarget: complex,
                 numout: int):
    """DIAGSUBSPACE hammod.F90:1125-1256: H in the span of the symmetrised
    products of the orbitals (i <= j for singlets, i < j for triplets),
    ZGEEV of A(I,J) = psi_I . (H psi_J), eigenvalues ordered by distance to
    etarget (mysort), the first numout eigenvectors as two-electron vectors
    with unit Hermitian norm."""
    numorbs = ev.shape[1]
    sign = 1 if singlet else -1
    table = [(i, j) for i in range(numorbs) for j in range(i + (0 if singlet else 1), numorbs)]
    psi = np.empty((h2.dim, len(table)), np.complex128, order="F")
    for k, (i, j) in enumerate(table):
        psi[:, k] = helium_orbital(ev, i, j, sign)
    hpsi = h2.matblock(psi)
    a = (psi.conj().T @ hpsi) if hermopt else (psi.T @ hpsi)
    e0, vr = np.linalg.eig(a)
    order = mysort_order(e0, etarget)
    e0, vr = e0[order], vr[:, order]
    out = np.asfortranarray(psi @ vr[:, :numout])
    out /= np.sqrt(np.einsum("ij,ij->j", out.conj(), out).real)
    return e0[:numout], out, e0


# --------------------------------------------------------------------------
# seeded start vectors


def seeded_start(p: Params, nev: int, seed: int, spin: str = "singlet") -> np.ndarray:
    """Complex-Gaussian columns (N(0,1)+iN(0,1))/sqrt(2), exchange
    symmetrised X <- (X +- X^T)/sqrt(2) in (p,q), unit Hermitian norm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = p.m
    out = np.empty((m * m, nev), np.complex128, order="F")
    sgn = 1.0 if spin == "singlet" else -1.0
    for j in range(nev):
        z = (rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))) / math.sqrt(2.0)
        z = (z + sgn * z.T) / math.sqrt(2.0)
        col = z.reshape(-1, order="F")
        out[:, j] = col / np.linalg.norm(col)
    return out


def seeded_vectors(dim: int, count: int, seed: int) -> np.ndarray:
    """Plain complex-Gaussian columns (N(0,1)+iN(0,1))/sqrt(2)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    re = rng.standard_normal((count, dim))
    im = rng.standard_normal((count, dim))
    return np.asfortranarray(((re + 1j * im) / math.sqrt(2.0)).T)
