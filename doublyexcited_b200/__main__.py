"""python -m doublyexcited_b200 [Inp=file] [N=6 Shift=-0.78 Nev=1 ...]: the
reference program's run (PROGRAM ATOM) on one GPU, printing its report."""
import sys

from .api import run


def main(argv: list[str]) -> int:
    r = run(argv, verbose=True)
    return 0 if r.converged else 1


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
