"""C-ABI library checks that need no GPU: it loads, exports every symbol the
header declares, parses Input.Inp like get_input/get_args, and reads/writes
the reference's eigenvector files (including the SIXD_FIX resize)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

HEADER = os.path.join(ROOT, "include", "doublyexcited.h")


def header_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"DE_API\s+[\w\s\*]+?\b(de_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol(de):
    syms = header_symbols()
    assert len(syms) >= 20
    L = ctypes.CDLL(de.lib_path())
    for s in syms:
        assert hasattr(L, s), s
    # and the Python binding declares exactly these
    from doublyexcited_b200._lib import SIGNATURES

    assert sorted(SIGNATURES) == syms


def test_library_exports_nothing_else(de):
    out = os.popen(f"nm -D --defined-only {de.lib_path()}").read()
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    ours = {s for s in exported if s.startswith("de_")}
    assert ours == set(header_symbols())


def test_strerror_and_version(de):
    L = de.lib()
    assert L.de_version().startswith(b"doublyexcited-b200")
    assert L.de_strerror(0) == b"ok"
    assert L.de_strerror(de.DE_E_SIZE) == b"size mismatch"


def test_defaults_are_the_reference_defaults(de):
    inp = de.read_input(None, [])
    assert inp["N"] == 2 and inp["DELTA"] == 0.5 and inp["RADIUS"] == 7.0 and inp["AUTODELTA"]
    assert inp["NSMALL"] == 22 and inp["TFACTOR"] == 4 and inp["CHARGE"] == 2.0 and inp["THETA"] == 0.0
    assert inp["GM_MAX_INNER_ITER"] == 5 and inp["GM_USEPETSCFLAG"] == 1 and inp["GM_TOL"] == 1e-3
    assert inp["NUMORBS"] == 14 and not inp["SINGLET"] and inp["NUMSKIP"] == 0
    assert inp["OUTMODULUS"] == 5 and inp["TAKEREALPART"] and inp["GPLMR_NEV"] == 1
    assert inp["GPLMR_NS"] == 5 and inp["GPLMR_MAXIT"] == 100 and inp["GPLMR_TOL"] == 1e-12
    assert inp["GPLMR_SHIFT"] == complex(-999, 0)
    assert inp["KDIM"] == 2001 and inp["LANBLOCKSIZE"] == 3 and inp["LANTOL"] == 1e-6


def test_namelist_parse(de, tmp_path):
    f = tmp_path / "Input.Inp"
    f.write_text(
        "! a comment line\n"
        "&main\n       WRITEVECS=.TRUE.\n       THETA=0.25d0  ! trailing comment\n/\n\n"
        "&grid\n  AUTODELTA=.false.\n  DELTA=1.5d0, N=4\n/\n"
        "&lanczos\n KDIM=301\n LANTOL=1D-3\n LANTOL=1D-2\n/\n"
        "&molecule\n/\n"
        "&gmres\n  gm_usepetscflag=1\n  GM_TOL=1d-4\n  GM_MAX_INNER_ITER=5\n  GM_MAX_INNER_ITER=7\n/\n"
        "&orbitals\n NUMORBS=5\n NUMORBS=9\n SINGLET=T\n/\n"
        "&gplmr\n TAKEREALPART=.FALSE.\n TAKEREALPART=.TRUE.\n GPLMR_SHIFT=(-0.5d0,0.01d0)\n"
        " GPLMR_SHIFT=(-0.76d0,0d0)\n GPLMR_MAXIT=1000000000\n GPLMR_TOL=1D-7\n GPLMR_NEV=2\n outmodulus=10\n/\n")
    inp = de.read_input(str(f), [])
    assert inp["WRITEVECS"] and inp["THETA"] == 0.25
    assert not inp["AUTODELTA"] and inp["DELTA"] == 1.5 and inp["N"] == 4
    assert inp["KDIM"] == 301 and inp["LANTOL"] == 1e-2  # last assignment wins
    assert inp["GM_TOL"] == 1e-4 and inp["GM_MAX_INNER_ITER"] == 7
    assert inp["NUMORBS"] == 9 and inp["SINGLET"]
    assert inp["TAKEREALPART"] and inp["GPLMR_SHIFT"] == complex(-0.76, 0)
    assert inp["GPLMR_MAXIT"] == 1000000000 and inp["GPLMR_TOL"] == 1e-7
    assert inp["GPLMR_NEV"] == 2 and inp["OUTMODULUS"] == 10


def test_command_line_keys(de, tmp_path):
    f = tmp_path / "Inp"
    f.write_text("&grid\n AUTODELTA=.false.\n DELTA=2d0\n/\n")
    argv = ["Read", "N=6", "Inp=whatever", "Nev=3", "Skip=4", "Trip", "Theta=0.35", "Outfile=eigvecs.S.N6",
            "Infile=eigvecs.S.N5", "Iter=20", "Gptol=1d-9", "Gmtol=1e-5", "NoPetsc", "Notakereal",
            "Shift=(-0.7,0.01)", "Norbs=6"]
    inp = de.read_input(str(f), argv)
    assert inp["N"] == 6 and inp["GPLMR_NEV"] == 3 and not inp["SINGLET"] and inp["THETA"] == 0.35
    assert inp["READVECS"] and inp["NUMSKIP"] == 4  # Skip= after Read overrides its NUMSKIP=0
    assert inp["OUTVECFILE"] == "eigvecs.S.N6" and inp["INVECFILE"] == "eigvecs.S.N5"
    assert inp["GM_MAX_INNER_ITER"] == 20 and inp["GPLMR_TOL"] == 1e-9 and inp["GM_TOL"] == 1e-5
    assert inp["GM_USEPETSCFLAG"] == 0 and not inp["TAKEREALPART"]
    assert inp["GPLMR_SHIFT"] == complex(-0.7, 0.01) and inp["NUMORBS"] == 6
    inp = de.read_input(str(f), ["R=9.0", "Sing"])
    assert inp["AUTODELTA"] and inp["RADIUS"] == 9.0 and inp["SINGLET"]
    from doublyexcited_b200.api import input_file_arg

    assert input_file_arg(["N=3", "Inp=Input.Inp.singlet"]) == "Input.Inp.singlet"
    assert input_file_arg(["N=3"]) == "Input.Inp"


def test_missing_file_keeps_defaults_and_bad_input_errors(de, tmp_path):
    assert de.read_input(str(tmp_path / "nope"), [])["N"] == 2
    f = tmp_path / "bad"
    f.write_text("&grid\n NOSUCHNAME=3\n/\n")
    with pytest.raises(de.DeError) as e:
        de.read_input(str(f), [])
    assert e.value.status == de.DE_E_PARSE
    f.write_text("&grid\n N=abc\n/\n")
    with pytest.raises(de.DeError):
        de.read_input(str(f), [])


def _sixd(x, n_in, n_out):
    """numpy SIXD_FIX: zero-pad / crop a (2n+1)^6 array about its centre."""
    nn_in, nn_out = 2 * n_in + 1, 2 * n_out + 1
    a = x.reshape((nn_in,) * 6, order="F")
    b = np.zeros((nn_out,) * 6, np.complex128)
    k = min(n_in, n_out)
    si = slice(n_in - k, n_in + k + 1)
    so = slice(n_out - k, n_out + k + 1)
    b[(so,) * 6] = a[(si,) * 6]
    return b.reshape(-1, order="F")


def test_vector_file_roundtrip_and_resize(de, tmp_path):
    rng = np.random.default_rng(0)
    m = 27
    x = rng.standard_normal((m * m, 3)) + 1j * rng.standard_normal((m * m, 3))
    path = str(tmp_path / "eigvecs.N1")
    de.write_vectors(path, x, m)
    assert de.vectors_header(path) == (m, 3)
    raw = open(path, "rb").read()
    # header record: marker 16, int32 M, int32 NUM, int64 16*M*M, marker 16
    assert np.frombuffer(raw[:4], "<i4")[0] == 16
    assert np.frombuffer(raw[4:12], "<i4").tolist() == [m, 3]
    assert np.frombuffer(raw[12:20], "<i8")[0] == 16 * m * m
    assert np.frombuffer(raw[24:28], "<i4")[0] == 16 * m * m
    y = de.read_vectors(path, m, 2)
    assert np.array_equal(y, x[:, :2])
    up = de.read_vectors(path, 125, 1)  # N=1 -> N=2: zero padding
    assert np.array_equal(up[:, 0], _sixd(x[:, 0], 1, 2))
    de.write_vectors(str(tmp_path / "big"), up, 125)
    down = de.read_vectors(str(tmp_path / "big"), 27, 1)  # N=2 -> N=1: crop
    assert np.array_equal(down[:, 0], x[:, 0])
    with pytest.raises(de.DeError):
        de.read_vectors(path, m, 4)  # more vectors than the file holds
    with pytest.raises(de.DeError):
        de.read_vectors(path, 28, 1)  # not an odd cube


def test_problem_create_fails_loudly_without_gpu(de):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(de.DeError) as e:
        de.Problem(n=2)
    assert e.value.status == 3  # DE_E_CUDA


def test_invalid_params_rejected(de):
    with pytest.raises(de.DeError) as e:
        de.Problem(n=12)  # NN=25: above the built grid sizes
    assert e.value.status == de.DE_E_UNSUPPORTED
    with pytest.raises(de.DeError) as e:
        de.Problem(n=2, nelec=3)
    assert e.value.status == de.DE_E_INVALID


def test_request_footprint_counts_the_solver_blocks(de):
    """Admission arithmetic of the server (host only): complex128 GPLMR blocks
    X AX W AW P AP S AS, the inner solve's Krylov blocks (complex64 in the
    mixed form), reduction scratch and operator tables."""
    x = np.zeros((7 ** 6, 2), np.complex128, order="F")
    req = de.Server.request(3, x, -0.78, ns=5, max_inner_iter=5)
    d, nev, ns, order = 7 ** 6, 2, 5, 5
    blocks = (6 * nev + 2 * ns * nev) * d * 16
    fp64 = de.Server.footprint(req)
    assert blocks + 2 * order * nev * d * 16 < fp64 < blocks + 2 * order * nev * d * 16 + (64 << 20)
    req_m = de.Server.request(3, x, -0.78, ns=5, max_inner_iter=5, precision="mixed")
    assert fp64 - de.Server.footprint(req_m) == order * nev * d * 16


def test_server_create_fails_loudly_without_gpu(de):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(de.DeError) as e:
        de.Server(workers=2)
    assert e.value.status == de.DE_E_CUDA


def test_server_result_carries_the_solve_stats(de):
    # the de_result -> ServedResult conversion, on a result struct filled here
    from doublyexcited_b200 import _lib as L

    srv = object.__new__(de.Server)  # no device: only the bookkeeping of collected requests
    x, e = np.zeros((4, 1), np.complex128), np.zeros(1, np.complex128)
    srv._live = {7: (None, x, e, "tag-7")}
    res = L.de_result(id=7, status=0, t_submit_s=1.0, t_start_s=1.5, t_end_s=4.0, footprint_bytes=123, worker=2)
    res.stats.iterations, res.stats.converged, res.stats.matvecs, res.stats.max_residual = 12, 1, 433, 5e-9
    r = srv._result(res)
    assert (r.id, r.status, r.iterations, r.converged, r.matvecs, r.worker, r.tag) == (7, 0, 12, True, 433, 2, "tag-7")
    assert r.x is x and r.e is e and r.latency_s == 3.0 and r.footprint_bytes == 123
    assert not srv._live


def test_tuning_table_lookup(de, tmp_path):
    """The matvec tuning table: entries by storage, grid and pass; comments,
    malformed lines and unknown families skipped; a missing entry or file
    reported as such (host only)."""
    t = tmp_path / "tuning.txt"
    t.write_text("# storage NN pass family ctas ms\n"
                 "c64 13 A tf32 2 0.1\n"
                 "c64 13 B ev 1   # comment\n"
                 "c128 13 A stream 0 0.2\n"
                 "c128 13 B bogus 0\n"
                 "c128 11\n")
    assert de.tuning_lookup(str(t), "c64", 13, 0) == ("tf32", 2)
    assert de.tuning_lookup(str(t), "c64", 13, 1) == ("fma", 1)
    assert de.tuning_lookup(str(t), "c128", 13, 0) == ("stream", 0)
    assert de.tuning_lookup(str(t), "c128", 13, 1) is None
    assert de.tuning_lookup(str(t), "c128", 11, 0) is None
    assert de.tuning_lookup(str(tmp_path / "missing.txt"), "c64", 13, 0) is None


def test_committed_tuning_table_covers_the_grids(de):
    """The committed table (written by python -m doublyexcited_b200.tune on a
    B200) has an entry for both storages and passes of every grid it
    tuned, N = 4..9, each a family the grid builds."""
    import os

    path = os.path.join(os.path.dirname(de.lib_path()), "matvec_tuning.txt")
    assert os.path.exists(path)
    for n in range(4, 10):
        nn = 2 * n + 1
        for storage in ("c128", "c64"):
            for pass_ in (0, 1):
                e = de.tuning_lookup(path, storage, nn, pass_)
                assert e is not None, (storage, nn, pass_)
                fam, ctas = e
                assert fam in ("fma", "tensor", "stream", "tf32") and 0 <= ctas <= 32
                if fam == "tf32":
                    assert storage == "c64" and nn <= 15


def test_tuner_candidates_follow_the_built_kernels():
    """The autotuner times only launch choices the library builds for a
    grid: even/odd kernels up to NN 13 (complex128) / 17 (complex64), the
    persistent streaming kernels from NN 13, DMMA on odd NN 9..19, tcgen05
    TF32 for complex64 up to NN 15; the built-in choice comes first."""
    from doublyexcited_b200.tune import candidates

    assert candidates("c128", 13)[0] == ("ev", 0) and candidates("c128", 15)[0] == ("stream", 0)
    assert candidates("c64", 17)[0] == ("ev", 0) and candidates("c64", 19)[0] == ("stream", 0)
    assert ("tf32", 0) in candidates("c64", 15) and not any(f == "tf32" for f, _ in candidates("c64", 17))
    assert not any(f == "tf32" for f, _ in candidates("c128", 13))
    assert ("dmma", 0) in candidates("c128", 19) and not any(f == "dmma" for f, _ in candidates("c128", 7))
    assert candidates("c128", 7) == [("stream", 0)]
