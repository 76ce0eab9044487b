"""python -m doublyexcited_b200 [Inp=file] [N=6 Shift=-0.78 Nev=1 ...]: the
reference program's run (PROGRAM ATOM) on one GPU, printing its report.
Exit status: 0 converged, else a DE_E_* code (DE_E_NOT_CONVERGED when GPLMR
stops at GPLMR_MAXIT)."""
import sys

from ._lib import DE_E_NOT_CONVERGED, DeError
from .api import run


def main(argv: list[str]) -> int:
    try:
        r = run(argv, verbose=True)
    except DeError as e:
        print(e, file=sys.stderr)
        return e.status
    return 0 if r.converged else DE_E_NOT_CONVERGED


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
