"""Generate the golden fixtures of tests/golden from the CPU oracle.

    python tests/golden/make_golden.py

config0_hpsi.npz: configuration 0 (FCC 2-atom cell, 24^3, 725 plane waves,
8 bands, 16 projectors): the seeded starting bands, the G->grid map and the
oracle's H|psi> (FP64).  config0_davidson.npz: the oracle's Davidson
eigenvalues (Ry) at tolerance 1e-10 Ry with the reference's loop, and the
exact lowest eigenvalues from dense diagonalisation.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import davidson, hpsi  # noqa: E402
from q3_b200 import synthetic  # noqa: E402


def main():
    sy = synthetic.config(0)
    kp = sy.kpoints[0]
    psi = sy.psi0[0]
    h = hpsi.apply_h(psi, kp, sy.v_r, sy.cell.grid)
    np.savez_compressed(HERE / "config0_hpsi.npz", psi=psi, hpsi=h, g_to_grid=kp.g_to_grid)
    hd = hpsi.dense_hamiltonian(kp, sy.v_r, sy.cell.grid)
    exact = np.linalg.eigvalsh(hd)[: sy.nbands]
    res = davidson.solve(lambda x: hpsi.apply_h(x, kp, sy.v_r, sy.cell.grid), kp.ke, psi,
                         sy.nbands, tolerance=1e-10, max_iterations=100)
    np.savez_compressed(HERE / "config0_davidson.npz", eigenvalues=res.eigenvalues, exact=exact,
                        iterations=res.iterations, h_applications=res.h_applications,
                        tolerance=1e-10)
    print("config0: iterations", res.iterations, "max |eps - exact|",
          float(np.max(np.abs(res.eigenvalues - exact))))


if __name__ == "__main__":
    main()
