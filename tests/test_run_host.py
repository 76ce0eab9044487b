"""de_run (PROGRAM ATOM, doublyexcited.F90:60-262) on the host: the checks
the reference makes before any operator work, here made before any GPU
work, and the loud failure without a GPU."""
import pytest


def test_run_rejects_nev_above_the_guess_products(de, tmp_path):
    """Two orbitals give one triplet product; NEV=2 is the reference's
    "GPLRM_NEV TOO BIG FOR NUMORBS" stop (doublyexcited.F90:143-148)."""
    with pytest.raises(de.DeError) as e:
        de.run(["N=2", "Nev=2", "Norbs=2", "Trip"], path=str(tmp_path / "absent.inp"))
    assert e.value.status == de.DE_E_INVALID
    assert "TOO BIG" in str(e.value)


def test_run_rejects_more_than_16_start_vectors(de, tmp_path):
    """TOTGET = min(MAXGET, NEV+NUMSKIP+5) = 18 start vectors."""
    with pytest.raises(de.DeError) as e:
        de.run(["N=2", "Nev=8", "Skip=5", "Norbs=10", "Sing"], path=str(tmp_path / "absent.inp"))
    assert e.value.status == de.DE_E_INVALID
    assert "TOTGET" in str(e.value)


def test_run_fails_loudly_without_gpu(de, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(de.DeError) as e:
        de.run(["N=2", "Nev=1", "Norbs=3", "Sing"], path=str(tmp_path / "absent.inp"))
    assert e.value.status == de.DE_E_CUDA


def test_command_line_reports_input_errors(tmp_path):
    """python -m doublyexcited_b200 prints the reference's message and exits
    with the DE_E_* status, without a traceback."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-m", "doublyexcited_b200", "N=2", "Nev=2", "Norbs=2", "Trip"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300,
                       env={**os.environ, "PYTHONPATH": root})
    assert p.returncode == 1  # DE_E_INVALID
    assert "TOO BIG FOR NUMORBS" in p.stderr and "Traceback" not in p.stderr


def test_run_checks_the_vector_file_before_gpu_work(de, tmp_path):
    """READVECS: a missing file, or one with fewer vectors than NEV+NUMSKIP,
    is an I/O error before the operator is built."""
    import numpy as np

    with pytest.raises(de.DeError) as e:
        de.run(["N=2", "Read", "Nev=1", f"Infile='{tmp_path / 'absent'}'"], path=str(tmp_path / "absent.inp"))
    assert e.value.status == de.DE_E_IO
    f = tmp_path / "one"
    de.write_vectors(str(f), np.zeros((5 ** 6, 1), np.complex128), 5 ** 3)
    with pytest.raises(de.DeError) as e:
        de.run(["N=2", "Read", "Nev=2", f"Infile='{f}'"], path=str(tmp_path / "absent.inp"))
    assert e.value.status == de.DE_E_IO and "holds 1 vectors, 2 requested" in str(e.value)
