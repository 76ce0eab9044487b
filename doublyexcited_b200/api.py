"""Python mirror of the reference's operator / eigensolver interface over the
C ABI.  Arrays are numpy complex128 in the reference layout: a two-electron
vector is X(1:M, 1:M) flattened column-major (electron 1 fastest); a block
is shape (D, nev) in Fortran order."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as _l
from ._lib import check, de_complex, de_gmres, de_input, de_params, de_stats, lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _block(x: np.ndarray, dim: int) -> np.ndarray:
    x = np.asarray(x)
    if x.ndim == 1:
        x = x.reshape(-1, 1)
    x = np.asfortranarray(x, dtype=np.complex128)
    if x.shape[0] != dim:
        raise ValueError(f"vector length {x.shape[0]} != {dim}")
    return x


@dataclass
class GplmrResult:
    e: np.ndarray
    x: np.ndarray
    iterations: int
    converged: bool
    matvecs: int
    matvecs_reference: int
    max_residual: float
    t_total_s: float
    t_matvec_s: float
    t_prec_s: float
    t_dense_s: float


class Problem:
    """One operator instance (HAMILTONIAN + PARAMETERS of the reference) on
    one GPU.  Mirrors ``INIT_STRUCTS``/``INIT_HAMILTONIAN``.  precision
    "fp64" is the plain form; "mixed" runs the eigensolver's inner solve
    (PRECBLOCK_BASIC) in complex64 with FP32 matvecs while the outer
    iteration, its residuals and every MATBLOCK stay FP64."""

    def __init__(self, n: int, delta: float = 2.0, theta: float = 0.2, charge: float = 2.0,
                 nelec: int = 2, nsmall: int = 22, tfactor: int = 4, device: int = 0,
                 autodelta: bool = False, radius: float = 7.0, precision: str = "fp64"):
        L = lib()
        p = de_params()
        L.de_params_default(ctypes.byref(p))
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        p.precision = 1 if precision == "mixed" else 0
        self.precision = precision
        p.n, p.delta, p.theta, p.charge = n, delta, theta, charge
        p.nelec, p.nsmall, p.tfactor, p.device = nelec, nsmall, tfactor, device
        p.autodelta, p.radius = int(bool(autodelta)), radius
        h = ctypes.c_void_p()
        check(L.de_problem_create(ctypes.byref(p), ctypes.byref(h)), "de_problem_create")
        self._h = h
        nn = ctypes.c_int()
        m = ctypes.c_int64()
        dim = ctypes.c_int64()
        check(L.de_problem_dims(h, ctypes.byref(nn), ctypes.byref(m), ctypes.byref(dim)), "de_problem_dims")
        self.nn, self.m, self.dim = nn.value, m.value, dim.value
        self.n, self.nelec = n, nelec

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().de_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_stream(self, cuda_stream: int) -> None:
        """Run the handle's kernels on a caller's cudaStream_t, e.g.
        ``torch.cuda.current_stream().cuda_stream`` (0 is the legacy default
        stream)."""
        check(lib().de_set_stream(self._h, ctypes.c_void_p(cuda_stream)), "de_set_stream")

    def set_matvec_kernel(self, kind: str) -> None:
        """'fma' (default): the CUDA-core kernels on even/odd-split
        contractions; 'tensor': the axis contractions on the FP64 tensor
        cores where built (NN 9..19); 'stream': the earlier CUDA-core
        streaming kernels (NN 13..19); 'tf32': the complex64 matvec's
        kinetic contractions on the TF32 tensor cores with head/tail split
        operands (NN 9..15)."""
        kinds = {"fma": 0, "tensor": 1, "stream": 2, "tf32": 3}
        if kind not in kinds:
            raise ValueError(f"matvec kernel must be one of {sorted(kinds)}")
        check(lib().de_set_matvec_kernel(self._h, kinds[kind]), "de_set_matvec_kernel")

    FAMILIES = ("fma", "tensor", "stream", "tf32")

    def set_matvec_launch(self, storage: str, pass_: int, family: str, ctas_per_sm: int = 0) -> None:
        """The kernels of one matvec pass: storage 'c128' (the FP64
        matvecs) or 'c64' (the mixed form's inner solve), pass 0 (electron-2
        axes and potential) or 1 (electron-1 axes), a family of
        set_matvec_kernel and a cap on resident CTAs per SM (0: all)."""
        check(lib().de_set_matvec_launch(self._h, {"c128": 0, "c64": 1}[storage], pass_,
                                         self.FAMILIES.index(family), ctas_per_sm), "de_set_matvec_launch")

    def get_matvec_launch(self, storage: str, pass_: int) -> tuple:
        """(family, ctas_per_sm) of one pass (see set_matvec_launch)."""
        f, c = ctypes.c_int(), ctypes.c_int()
        check(lib().de_get_matvec_launch(self._h, {"c128": 0, "c64": 1}[storage], pass_, ctypes.byref(f),
                                         ctypes.byref(c)), "de_get_matvec_launch")
        return self.FAMILIES[f.value], c.value

    def set_profiling(self, on, every: int = 1) -> None:
        """Device-time accounting of the matvec passes: off, or on for every
        `every`-th MATBLOCK call of each storage (1: all of them)."""
        check(lib().de_set_profiling(self._h, max(1, int(every)) if on else 0), "de_set_profiling")

    def profile_read(self) -> dict:
        """Device ms of matvec pass A / pass B, MATBLOCK calls and vectors since
        the last read (resets)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        c, v = ctypes.c_int64(), ctypes.c_int64()
        check(lib().de_profile_read(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(v)),
              "de_profile_read")
        return {"pass_a_ms": a.value, "pass_b_ms": b.value, "calls": c.value, "vectors": v.value}

    def profile_read32(self) -> dict:
        """The same for the FP32 matvecs of the mixed form's inner solve."""
        a, b = ctypes.c_double(), ctypes.c_double()
        c, v = ctypes.c_int64(), ctypes.c_int64()
        check(lib().de_profile_read32(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(v)),
              "de_profile_read32")
        return {"pass_a_ms": a.value, "pass_b_ms": b.value, "calls": c.value, "vectors": v.value}

    # -- operator ---------------------------------------------------------
    def hammult(self, x: np.ndarray) -> np.ndarray:
        x = _block(x, self.dim)[:, 0].copy()
        y = np.empty_like(x)
        check(lib().de_hammult(self._h, _ptr(x), _ptr(y), self.dim), "de_hammult")
        return y

    def matblock(self, x: np.ndarray) -> np.ndarray:
        x = _block(x, self.dim)
        y = np.empty_like(x)
        check(lib().de_matblock(self._h, _ptr(x), _ptr(y), self.m, self.dim // self.m, x.shape[1]),
              "de_matblock")
        return y

    def matblock_d(self, x_ptr: int, y_ptr: int, nev: int) -> None:
        """Device-pointer MATBLOCK (e.g. torch tensors' data_ptr())."""
        check(lib().de_matblock_d(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), self.m,
                                  self.dim // self.m, nev), "de_matblock_d")

    def kinetic_precond_d(self, x_ptr: int, y_ptr: int, nvec: int, shift: complex = 0.0) -> None:
        """MSOLVECPLX22 (littlesolver.F90:372-436) on device vectors: the
        kinetic-eigenbasis preconditioner, y = P x (y must not alias x)."""
        check(lib().de_kinetic_precond_d(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), nvec,
                                         de_complex(shift.real, shift.imag)), "de_kinetic_precond_d")

    def set_gmres_pc(self, pcopt: int) -> None:
        """Preconditioner of the GMRES inner solve (usepetscflag = 0): 0 none
        (the reference's setting), 2 the kinetic eigenbasis on the left."""
        check(lib().de_set_gmres_pc(self._h, pcopt), "de_set_gmres_pc")

    def matblock32_d(self, x_ptr: int, y_ptr: int, nev: int) -> None:
        """Device-pointer MATBLOCK on complex64 vectors in FP32 arithmetic (the
        mixed form's inner-solve matvec)."""
        check(lib().de_matblock32_d(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), self.m,
                                    self.dim // self.m, nev), "de_matblock32_d")

    def dots(self, bras: np.ndarray, kets: np.ndarray, hermitian: bool = True) -> np.ndarray:
        b = _block(bras, bras.shape[0])
        k = _block(kets, b.shape[0])
        out = np.empty((b.shape[1], k.shape[1]), np.complex128, order="F")
        check(lib().de_dots(self._h, _ptr(b), _ptr(k), b.shape[0], b.shape[1], k.shape[1], _ptr(out),
                            int(hermitian)), "de_dots")
        return out

    def get_expects(self, psi: np.ndarray, cshiftopt: bool = False) -> np.ndarray:
        psi = _block(psi, self.dim)
        out = np.empty(psi.shape[1], np.complex128)
        check(lib().de_get_expects(self._h, _ptr(psi), psi.shape[1], int(cshiftopt), _ptr(out)),
              "de_get_expects")
        return out

    def subspace_guess(self, numorbs: int, singlet: bool = True, hermopt: bool = False,
                       etarget: complex = 0.0, numout: int = 1) -> tuple[np.ndarray, np.ndarray]:
        """The reference's GPLMR start block: (E0[:numout], X (D, numout))."""
        x = np.empty((self.dim, numout), np.complex128, order="F")
        e0 = np.empty(numout, np.complex128)
        et = complex(etarget)
        check(lib().de_subspace_guess(self._h, numorbs, int(bool(singlet)), int(bool(hermopt)),
                                      de_complex(et.real, et.imag), numout, _ptr(x), _ptr(e0)),
              "de_subspace_guess")
        return e0, x

    # -- eigensolver ----------------------------------------------------------
    def gplmr_eig(self, x0: np.ndarray, sigma: complex, ns: int = 5, maxit: int = 100, tol: float = 1e-7,
                  max_inner_iter: int = 5, usepetscflag: int = 1, compat_first_column_only: bool = False,
                  outmodulus: int = 0) -> GplmrResult:
        x = _block(x0, self.dim).copy(order="F")
        nev = x.shape[1]
        e = np.empty(nev, np.complex128)
        gm = de_gmres(max_inner_iter, usepetscflag, 1e-3, int(bool(compat_first_column_only)))
        st = de_stats()
        check(lib().de_gplmr_eig(self._h, _ptr(x), _ptr(e), self.m, self.dim // self.m,
                                 de_complex(complex(sigma).real, complex(sigma).imag), nev, ns, maxit, tol,
                                 ctypes.byref(gm), outmodulus, ctypes.byref(st)), "de_gplmr_eig")
        return GplmrResult(e, x, st.iterations, bool(st.converged), st.matvecs, st.matvecs_reference,
                           st.max_residual, st.t_total_s, st.t_matvec_s, st.t_prec_s, st.t_dense_s)


# -- configuration ---------------------------------------------------------------

def heplus_orbitals(n: int, h1: np.ndarray, numorbs: int, hermopt: bool = False) -> tuple[np.ndarray, np.ndarray]:
    """He+ levels of lowest real part and their Gram-Schmidt orthonormalised
    orbitals from a dense one-electron operator (DIAGONALIZE +
    HELIUM_ORBITALGATHER); host only.  Returns (energies, orbitals (M, numorbs))."""
    nn = 2 * n + 1
    m = nn ** 3
    h1 = np.asfortranarray(h1, dtype=np.complex128)
    if h1.shape != (m, m):
        raise ValueError(f"h1 has shape {h1.shape}, expected ({m}, {m})")
    w = np.empty(numorbs, np.complex128)
    orb = np.empty((m, numorbs), np.complex128, order="F")
    check(lib().de_heplus_orbitals(n, _ptr(h1), numorbs, int(bool(hermopt)), _ptr(w), _ptr(orb)),
          "de_heplus_orbitals")
    return w, orb


@dataclass
class RunResult:
    e: np.ndarray
    x: np.ndarray
    totget: int
    e0: np.ndarray
    expects: np.ndarray
    shift: complex
    iterations: int
    converged: bool
    max_residual: float


def _parsed_input(path: str | None, argv: list[str] | None) -> de_input:
    L = lib()
    inp = de_input()
    L.de_input_default(ctypes.byref(inp))
    args = [a.encode() for a in (argv or [])]
    arr = (ctypes.c_char_p * max(1, len(args)))(*args)
    check(L.de_read_input(path.encode() if path else None, len(args), arr, ctypes.byref(inp)),
          "de_read_input")
    return inp


def run(argv: list[str] | None = None, path: str | None = None, verbose: bool = False) -> RunResult:
    """PROGRAM ATOM (doublyexcited.F90:60-262): the input file (path, else the
    Inp= key of argv, else Input.Inp) and argv's keys, then the initial guess
    or READVECS, NUMSKIP, the shift from GET_EXPECTS, GPLMR_EIG and WRITEVECS."""
    argv = list(argv or [])
    if path is None:
        buf = ctypes.create_string_buffer(400)
        args = [a.encode() for a in argv]
        arr = (ctypes.c_char_p * max(1, len(args)))(*args)
        check(lib().de_input_file_arg(len(args), arr, buf, len(buf)), "de_input_file_arg")
        path = buf.value.decode()
    inp = _parsed_input(path, argv)
    nev = inp.gplmr_nev
    dim = (2 * inp.params.n + 1) ** 6
    x = np.empty((dim, max(nev, 1)), np.complex128, order="F")
    e = np.empty(max(nev, 1), np.complex128)
    info = _l.de_run_info()
    check(lib().de_run(ctypes.byref(inp), int(bool(verbose)), _ptr(e), _ptr(x), ctypes.byref(info)), "de_run")
    k = info.nexpects
    e0 = np.array([complex(z.re, z.im) for z in info.e0[:k]])
    ex = np.array([complex(z.re, z.im) for z in info.expects[:k]])
    st = info.stats
    return RunResult(e, x, info.totget, e0, ex, complex(info.shift.re, info.shift.im), st.iterations,
                     bool(st.converged), st.max_residual)


def read_input(path: str | None, argv: list[str] | None = None) -> dict:
    """Input.Inp namelists + command-line keys (get_input / get_args)."""
    inp = _parsed_input(path, argv)
    p = inp.params
    return {
        "N": p.n, "DELTA": p.delta, "RADIUS": p.radius, "AUTODELTA": bool(p.autodelta), "THETA": p.theta,
        "CHARGE": p.charge, "NSMALL": p.nsmall, "TFACTOR": p.tfactor,
        "GM_MAX_INNER_ITER": inp.gmres.max_inner_iter, "GM_USEPETSCFLAG": inp.gmres.usepetscflag,
        "GM_TOL": inp.gmres.tol, "WRITEVECS": bool(inp.writevecs), "READVECS": bool(inp.readvecs),
        "INVECFILE": inp.invecfile.decode(), "OUTVECFILE": inp.outvecfile.decode(),
        "NUMORBS": inp.numorbs, "SINGLET": bool(inp.singlet), "NUMSKIP": inp.numskip,
        "OUTMODULUS": inp.outmodulus, "TAKEREALPART": bool(inp.takerealpart), "HERMOPT": bool(inp.hermopt),
        "CSHIFTOPT": bool(inp.cshiftopt), "GPLMR_NEV": inp.gplmr_nev, "GPLMR_NS": inp.gplmr_ns,
        "GPLMR_MAXIT": inp.gplmr_maxit, "GPLMR_TOL": inp.gplmr_tol,
        "GPLMR_SHIFT": complex(inp.gplmr_shift.re, inp.gplmr_shift.im),
        "KDIM": inp.kdim, "LANBLOCKSIZE": inp.lanblocksize, "CHECK": inp.check, "LANTOL": inp.lantol,
    }


def input_file_arg(argv: list[str]) -> str:
    L = lib()
    args = [a.encode() for a in argv]
    arr = (ctypes.c_char_p * max(1, len(args)))(*args)
    buf = ctypes.create_string_buffer(512)
    check(L.de_input_file_arg(len(args), arr, buf, 512), "de_input_file_arg")
    return buf.value.decode()


# -- eigenvector files ---------------------------------------------------------------

def write_vectors(path: str, psi: np.ndarray, m: int) -> None:
    psi = _block(psi, m * m)
    check(lib().de_write_vectors(path.encode(), m, psi.shape[1], _ptr(psi)), "de_write_vectors")


def read_vectors(path: str, m: int, num: int) -> np.ndarray:
    out = np.empty((m * m, num), np.complex128, order="F")
    check(lib().de_read_vectors(path.encode(), m, num, _ptr(out)), "de_read_vectors")
    return out


def vectors_header(path: str) -> tuple[int, int]:
    m = ctypes.c_int64()
    n = ctypes.c_int()
    check(lib().de_vectors_header(path.encode(), ctypes.byref(m), ctypes.byref(n)), "de_vectors_header")
    return m.value, n.value


# -- batched and served solves ---------------------------------------------------

@dataclass
class ServedResult:
    id: int
    status: int
    e: np.ndarray
    x: np.ndarray
    iterations: int
    converged: bool
    max_residual: float
    t_submit_s: float
    t_start_s: float
    t_end_s: float
    footprint_bytes: int
    worker: int
    tag: object = None
    matvecs: int = 0  # vector-matvecs of the solve, both precisions (de_stats.matvecs)

    @property
    def latency_s(self) -> float:
        return self.t_end_s - self.t_submit_s


class Server:
    """Many independent GPLMR solves on one GPU (``de_server_*``): requests
    are admitted first come, first served when a worker is free and their
    device footprint fits in ``max_bytes``; each worker runs its solves on
    its own CUDA stream, so different solves overlap on the device."""

    def __init__(self, workers: int = 4, max_bytes: int = 0, device: int = 0):
        o = _l.de_server_opts(device, workers, max_bytes)
        h = ctypes.c_void_p()
        check(lib().de_server_create(ctypes.byref(o), ctypes.byref(h)), "de_server_create")
        self._h = h
        self._live = {}  # id -> (request, x, e, tag): buffers stay alive until collected

    @staticmethod
    def request(n: int, x0: np.ndarray, sigma: complex, *, theta: float = 0.2, delta: float = 2.0,
                charge: float = 2.0, precision: str = "fp64", ns: int = 5, maxit: int = 100, tol: float = 1e-7,
                max_inner_iter: int = 5, autodelta: bool = False, radius: float = 7.0):
        """A request's buffers: the operator as :class:`Problem` builds it (the
        same keyword defaults), GPLMR settings as :meth:`Problem.gplmr_eig`."""
        p = de_params()
        lib().de_params_default(ctypes.byref(p))
        p.n, p.delta, p.theta, p.charge = n, delta, theta, charge
        p.autodelta, p.radius = int(bool(autodelta)), radius
        p.precision = 1 if precision == "mixed" else 0
        x = np.array(x0, dtype=np.complex128, order="F", copy=True)
        if x.ndim == 1:
            x = x[:, None]
        e = np.empty(x.shape[1], np.complex128)
        r = _l.de_request(p, de_complex(complex(sigma).real, complex(sigma).imag), x.shape[1], ns, maxit, tol,
                          de_gmres(max_inner_iter, 1, 1e-3, 0), x.ctypes.data, e.ctypes.data)
        return r, x, e

    @staticmethod
    def footprint(req) -> int:
        b = ctypes.c_int64()
        check(lib().de_request_footprint(ctypes.byref(req[0]), ctypes.byref(b)), "de_request_footprint")
        return b.value

    def submit(self, req, tag=None) -> int:
        r, x, e = req
        i = ctypes.c_uint64()
        check(lib().de_server_submit(self._h, ctypes.byref(r), ctypes.byref(i)), "de_server_submit")
        self._live[i.value] = (r, x, e, tag)
        return i.value

    def _result(self, res) -> ServedResult:
        r, x, e, tag = self._live.pop(res.id)
        st = res.stats
        return ServedResult(res.id, res.status, e, x, st.iterations, bool(st.converged), st.max_residual,
                            res.t_submit_s, res.t_start_s, res.t_end_s, res.footprint_bytes, res.worker, tag,
                            matvecs=int(st.matvecs))

    def wait(self, rid: int, timeout_s: float = -1.0) -> ServedResult:
        res = _l.de_result()
        check(lib().de_server_wait(self._h, rid, timeout_s, ctypes.byref(res)), "de_server_wait")
        return self._result(res)

    def wait_any(self, timeout_s: float = -1.0) -> ServedResult | None:
        res = _l.de_result()
        s = lib().de_server_wait_any(self._h, timeout_s, ctypes.byref(res))
        if s == _l.DE_E_BUSY:
            return None
        check(s, "de_server_wait_any")
        return self._result(res)

    def now(self) -> float:
        return lib().de_server_now(self._h)

    def load(self) -> tuple[int, int, int]:
        q, r, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        check(lib().de_server_load(self._h, ctypes.byref(q), ctypes.byref(r), ctypes.byref(b)), "de_server_load")
        return q.value, r.value, b.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().de_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tuning_lookup(path: str, storage: str, nn: int, pass_: int) -> tuple | None:
    """A tuning table's (family, ctas_per_sm) for storage 'c128'/'c64', grid
    NN and pass 0/1, or None when the file or the entry is missing (host
    only; see set_matvec_launch)."""
    f, c = ctypes.c_int(), ctypes.c_int()
    st = lib().de_tuning_lookup(path.encode(), {"c128": 0, "c64": 1}[storage], nn, pass_, ctypes.byref(f),
                                ctypes.byref(c))
    if st != 0:
        return None
    return Problem.FAMILIES[f.value], c.value
