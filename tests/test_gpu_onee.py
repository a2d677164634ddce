"""Nuclear attraction matrix on the device (tce_nuclear_attraction) against the oracle.

* 64-cell H chain: the unit-cell rows against the committed golden rows
  (tests/golden/systems/h_chain64_onee.npz, written by the oracle), the other
  rows by translation;
* a 2D sheet and a 3D cube (s, p shells): the full matrix against the
  oracle's orc_one_electron computed here.
Tolerance 1e-10 per element (the integral tolerance of the path).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "systems")
TOL = 1e-10


def _translate_rows(rows, nfuc, ncl):
    """Rows of the unit cell -> full matrix (fill_with_symmetry)."""
    nbas = rows.shape[1]
    nx, ny, nz = ncl
    M = np.zeros((nbas, nbas))
    for i in range(nbas):
        Ri, a = divmod(i, nfuc)
        rxi, ryi, rzi = Ri % nx, (Ri // nx) % ny, Ri // (nx * ny)
        for Rj in range(nbas // nfuc):
            rxj, ryj, rzj = Rj % nx, (Rj // nx) % ny, Rj // (nx * ny)
            src = (((rzj - rzi) % nz) * ny + (ryj - ryi) % ny) * nx + (rxj - rxi) % nx
            M[i, Rj * nfuc:(Rj + 1) * nfuc] = rows[a, src * nfuc:(src + 1) * nfuc]
    return M


def test_nuclear_attraction_chain64_vs_golden():
    from william_ci_b200.engine import Engine
    from william_ci_b200.system import AOSystem
    sysm = AOSystem.load(os.path.join(GOLD, "h_chain64.npz"))
    gold = np.load(os.path.join(GOLD, "h_chain64_onee.npz"))["V"]
    eng = Engine(sysm)
    V = eng.nuclear_attraction()
    nf = sysm.nfuc
    assert np.abs(V[:nf] - gold).max() <= TOL, np.abs(V[:nf] - gold).max()
    full = _translate_rows(gold, nf, tuple(sysm.ncell))
    assert np.abs(V - full).max() <= TOL
    assert np.abs(V[:nf, :nf] - V[:nf, :nf].T).max() <= TOL     # Hermitian within the unit cell
    assert np.abs(V).max() > 1.0


@pytest.mark.parametrize("name,ncell", [("h2_sheet", (2, 2, 1)), ("li_cube", (2, 2, 2))])
def test_nuclear_attraction_2d_3d_vs_oracle(systems, name, ncell):
    import pyoracle
    from william_ci_b200.engine import Engine
    sysm = systems(name, ncell)
    _, _, Vo = pyoracle.Oracle(sysm).one_electron()
    V = Engine(sysm).nuclear_attraction()
    assert np.abs(V - Vo).max() <= TOL, np.abs(V - Vo).max()
    assert np.abs(V).max() > 0.1
