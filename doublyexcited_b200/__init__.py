"""doublyexcited_b200 -- B200 (sm_100a) implementation of doublyexcited's hot
path: the complex-scaled two-electron sinc-DVR helium Hamiltonian applied to
blocks of vectors inside the GPLMR harmonic-Ritz block eigensolver.

The product is the C-ABI library ``libdoublyexcited_b200.so`` (declared in
``include/doublyexcited.h``).  This module is a thin ctypes binding over it,
mirroring the reference's entry points (paths relative to
``complexscale-djhnow/code/``):

* :meth:`Problem.hammult`   -- ``HAMMULT`` hammod.F90:19-67
* :meth:`Problem.matblock`  -- ``MATBLOCK`` gplmr.F90:443-462 / ``MYMATMUL``
* :meth:`Problem.dots`      -- ``MYDOTSUB`` doublyexcited.F90:47-59 / ``MPIDOT``
* :meth:`Problem.get_expects` -- ``GET_EXPECTS`` hammod.F90:1261-1301
* :meth:`Problem.gplmr_eig` -- ``GPLMR_EIG`` gplmr.F90:9-374
* :meth:`Problem.subspace_guess` -- the initial guess, doublyexcited.F90:135-190
  (``DIAGSUBSPACE`` hammod.F90:1125-1256), and :func:`heplus_orbitals`, its
  He+ orbital step on the host
* :func:`read_input`        -- ``get_input``/``get_args`` input.F90:143-362
* :func:`run` / ``python -m doublyexcited_b200`` -- ``PROGRAM ATOM``
  doublyexcited.F90:60-262
* :func:`write_vectors` / :func:`read_vectors` -- utils.F90:82-198
* :class:`Server` -- many independent solves on one GPU (no reference
  counterpart): admission by device footprint, concurrent streams
* ``python -m doublyexcited_b200.tune`` -- the matvec autotuner: times each
  kernel family and resident-CTA count per grid and pass on the GPU and
  writes the table the library reads (:func:`tuning_lookup`)

There is no CPU fallback: if the library is missing or no GPU is present the
calls raise.
"""
from __future__ import annotations

from ._lib import (  # noqa: F401
    DE_E_CHOLESKY,
    DE_E_CUDA,
    DE_E_NOMEM,
    DE_E_GEVP,
    DE_E_INVALID,
    DE_E_IO,
    DE_E_LAPACK,
    DE_E_NAN,
    DE_E_BUSY,
    DE_E_ORTHO,
    DE_E_PARSE,
    DE_E_SIZE,
    DE_E_UNSUPPORTED,
    DE_OK,
    DeError,
    lib,
    lib_path,
)
from .api import Problem, GplmrResult, RunResult, Server, ServedResult, heplus_orbitals, read_input, read_vectors, run, tuning_lookup, vectors_header, write_vectors  # noqa: F401,E501

__all__ = [
    "Problem",
    "GplmrResult",
    "Server",
    "ServedResult",
    "heplus_orbitals",
    "RunResult",
    "run",
    "read_input",
    "read_vectors",
    "vectors_header",
    "write_vectors",
    "tuning_lookup",
    "DeError",
    "lib",
    "lib_path",
]
