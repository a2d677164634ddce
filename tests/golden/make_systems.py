"""Write the normalised AO systems of the named workloads to tests/golden/systems/.

The reference normalises every Cartesian component on the Fortran side before
it calls the integral path (normalize_AO_toroidal_*D, called at
Tori1D.f90:82); the engine takes normalised coefficients as input.  These
fixtures hold that input, normalised by the oracle's restatement of
normalize_1D.f90:17-79 (and its 2D/3D twins), so that bench.py and smoke()
feed the engine exactly what the Fortran caller would.

    python tests/golden/make_systems.py
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from william_ci_b200 import system as S  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "systems")
ONE_ELECTRON = ("h2_ring", "h_chain64", "h_chain128")   # RHF inputs stored for the SCF / DF-MP2 timing
AUX = ("h_chain128",)   # even-tempered auxiliary basis of the DF-MP2 configuration


def main():
    os.makedirs(OUT, exist_ok=True)
    for name in ("h2_ring", "h_chain64", "h2_sheet", "li_cube", "h_chain128"):
        sysm = S.build_system(*S.workload(name))
        dev = pyoracle.normalize(sysm)
        path = os.path.join(OUT, name + ".npz")
        sysm.save(path)
        print("%-11s nbas %5d nfuc %3d  max|<phi|phi>-1| %.1e  -> %s" % (name, sysm.nbas, sysm.nfuc, dev, path))
        if name in AUX:
            from william_ci_b200 import df
            cell, _ = S.workload(name)
            aux = S.build_system(cell, df.even_tempered_aux(sysm.charges))
            dev_a = pyoracle.normalize(aux)
            aux.save(os.path.join(OUT, name + "_aux.npz"))
            print("%-11s auxiliary nbas %5d  max|<P|P>-1| %.1e" % (name, aux.nbas, dev_a))
        if name in ONE_ELECTRON:
            # S, T, V rows of the unit cell (the others follow by translation) and E_nuc,
            # the inputs RHF_SAO receives (main.f90:379-500)
            import numpy as np
            o = pyoracle.Oracle(sysm)
            S_, T_, V_ = o.one_electron()
            nf = sysm.nfuc
            np.savez(os.path.join(OUT, name + "_onee.npz"), S=S_[:nf], T=T_[:nf], V=V_[:nf],
                     enuc=pyoracle.nuclear_repulsion(sysm))


if __name__ == "__main__":
    main()
