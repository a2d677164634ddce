"""Supercell basis description: the inputs of the toroidal ERI path.

Mirrors the reference's input side so that the engine is fed exactly what
the Fortran code feeds its integral drivers:

* ``unitcell.mol`` (line 1: type; line 2: ``nx d Lx`` / ``nx ny d Lx Ly`` /
  ``nx ny nz d Lx Ly Lz``; keyword lines up to ``$$``; atoms up to ``$$``)
  -- src/geometry/super_molecule.f90:1-404.
* ``Basis`` (Dalton style, one general-contraction block per l per element,
  atoms tagged ``A <Z>``) -- src/basis/basis.f90:21-106.
* Supercell replication, cells x fastest then y then z --
  src/geometry/super_molecule.f90:124-140.
* AO list: per atom s columns, then p (px,py,pz), d (xx,xy,xz,yy,yz,zz), ...,
  zero coefficients dropped -- src/basis/class.f90:15-71, src/module/filter.f90.

The result is the flat layout of ``tce_system`` (include/tce.h): centres,
Cartesian powers, CSR primitive offsets, exponents, coefficients.
"""
from __future__ import annotations

import dataclasses
import math
import re
from typing import Dict, List, Sequence, Tuple

import numpy as np

# Cartesian component labels, class.f90:15-21
CART = {
    0: ["s"],
    1: ["px", "py", "pz"],
    2: ["dxx", "dxy", "dxz", "dyy", "dyz", "dzz"],
    3: ["fxxx", "fxxy", "fxxz", "fxyy", "fxyz", "fxzz", "fyyy", "fyyz", "fyzz", "fzzz"],
    4: ["gxxxx", "gxxxy", "gxxxz", "gxxyy", "gxxyz", "gxxzz", "gxyyy", "gxyyz", "gxyzz",
        "gxzzz", "gyyyy", "gyyyz", "gyyzz", "gyzzz", "gzzzz"],
}
SHELL_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4}

ELEMENTS = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si",
            "P", "S", "Cl", "Ar"]


def label_to_lxyz(label: str) -> Tuple[int, int, int]:
    """orbital_to_lxyz (clifford_tools.f90:793-810): count x, y, z letters."""
    s = label[1:].lower()
    return (s.count("x"), s.count("y"), s.count("z"))


def charge_of(symbol: str) -> int:
    sym = symbol.strip().capitalize()
    if sym in ELEMENTS:
        return ELEMENTS.index(sym)
    raise ValueError("unknown element %r" % symbol)


@dataclasses.dataclass
class BasisBlock:
    l: int
    exps: np.ndarray          # (ne,)
    coefs: np.ndarray         # (ne, nc)


Basis = Dict[int, List[BasisBlock]]   # nuclear charge -> blocks


@dataclasses.dataclass
class Cell:
    kind: str                 # Tori1D / Tori2D / Tori3D
    ncell: Tuple[int, int, int]
    spacing: float
    L: Tuple[float, float, float]
    atoms: List[Tuple[str, Tuple[float, float, float]]]
    keywords: List[str] = dataclasses.field(default_factory=list)

    @property
    def ndp(self) -> int:
        return {"Tori1D": 1, "Tori2D": 2, "Tori3D": 3}[self.kind]


@dataclasses.dataclass
class AOSystem:
    """Flat AO list of a supercell (column order of the reference arrays)."""
    ndp: int
    ncell: Tuple[int, int, int]
    nfuc: int
    L: Tuple[float, float, float]
    ctr: np.ndarray           # (nbas, 3)
    lxyz: np.ndarray          # (nbas, 3) int32
    prim_off: np.ndarray      # (nbas+1,) int32
    exps: np.ndarray          # (nprim_total,)
    coefs: np.ndarray         # (nprim_total,)
    labels: List[str]
    atom_of: np.ndarray       # (nbas,) atom index in the supercell
    charges: np.ndarray       # (natoms,) nuclear charges
    geometry: np.ndarray      # (natoms, 3)

    @property
    def nbas(self) -> int:
        return int(self.ctr.shape[0])

    def copy(self) -> "AOSystem":
        return dataclasses.replace(self, ctr=self.ctr.copy(), lxyz=self.lxyz.copy(),
                                   prim_off=self.prim_off.copy(), exps=self.exps.copy(),
                                   coefs=self.coefs.copy(), labels=list(self.labels),
                                   atom_of=self.atom_of.copy(), charges=self.charges.copy(),
                                   geometry=self.geometry.copy())

    def save(self, path: str) -> None:
        np.savez(path, ndp=self.ndp, ncell=np.array(self.ncell), nfuc=self.nfuc,
                 L=np.array(self.L), ctr=self.ctr, lxyz=self.lxyz, prim_off=self.prim_off,
                 exps=self.exps, coefs=self.coefs, labels=np.array(self.labels),
                 atom_of=self.atom_of, charges=self.charges, geometry=self.geometry)

    @staticmethod
    def load(path: str) -> "AOSystem":
        z = np.load(path)
        return AOSystem(ndp=int(z["ndp"]), ncell=tuple(int(x) for x in z["ncell"]),
                        nfuc=int(z["nfuc"]), L=tuple(float(x) for x in z["L"]),
                        ctr=z["ctr"].astype(np.float64), lxyz=z["lxyz"].astype(np.int32),
                        prim_off=z["prim_off"].astype(np.int32), exps=z["exps"].astype(np.float64),
                        coefs=z["coefs"].astype(np.float64), labels=[str(s) for s in z["labels"]],
                        atom_of=z["atom_of"].astype(np.int32), charges=z["charges"].astype(np.int32),
                        geometry=z["geometry"].astype(np.float64))


# ---------------------------------------------------------------------------
# parsers
# ---------------------------------------------------------------------------
def parse_unitcell(text: str) -> Cell:
    """build_super_molecule / read_2nd_line / read_keywords (super_molecule.f90)."""
    lines = text.splitlines()
    kind = lines[0].split()[0]
    nums = lines[1].replace(",", " ").split()
    if kind == "Tori1D":
        nx, d, Lx = int(nums[0]), float(nums[1]), float(nums[2])
        ncell, L = (nx, 1, 1), (Lx, 0.0, 0.0)
    elif kind == "Tori2D":
        nx, ny, d, Lx, Ly = int(nums[0]), int(nums[1]), float(nums[2]), float(nums[3]), float(nums[4])
        ncell, L = (nx, ny, 1), (Lx, Ly, 0.0)
    elif kind == "Tori3D":
        nx, ny, nz = int(nums[0]), int(nums[1]), int(nums[2])
        d, Lx, Ly, Lz = float(nums[3]), float(nums[4]), float(nums[5]), float(nums[6])
        ncell, L = (nx, ny, nz), (Lx, Ly, Lz)
    else:
        raise ValueError("unsupported calculation type %r (toroidal path only)" % kind)
    i = 2
    keywords: List[str] = []
    while i < len(lines) and lines[i].strip() != "$$":
        if lines[i].strip():
            keywords.append(lines[i].strip())
        i += 1
    if i >= len(lines):
        raise ValueError("reached end of file without the opening $$ marker")
    i += 1
    atoms = []
    while i < len(lines) and lines[i].strip() != "$$":
        parts = lines[i].split()
        if len(parts) >= 4:
            atoms.append((parts[0], (float(parts[1]), float(parts[2]), float(parts[3]))))
        i += 1
    return Cell(kind=kind, ncell=ncell, spacing=d, L=L, atoms=atoms, keywords=keywords)


def parse_basis(text: str) -> Basis:
    """read_atom_shells_gen (basis.f90:21-106)."""
    out: Basis = {}
    lines = text.splitlines()
    cur = None
    i = 0
    while i < len(lines):
        key = lines[i].strip()
        m = re.match(r"^[Aa]\s+(\d+)\s*$", key)
        if m:
            cur = int(m.group(1))
            out.setdefault(cur, [])
            i += 1
            continue
        if cur is not None and key.startswith("$") and "-TYPE FUNCTIONS" in key:
            shl = key[2:3].upper()
            if shl not in SHELL_L:
                raise ValueError("shell type not supported: %s" % key)
            ne, nc = (int(x) for x in lines[i + 1].split()[:2])
            ex = np.zeros(ne)
            co = np.zeros((ne, nc))
            for r in range(ne):
                vals = [float(x.replace("D", "E").replace("d", "e")) for x in lines[i + 2 + r].split()]
                ex[r] = vals[0]
                co[r, :] = vals[1:1 + nc]
            out[cur].append(BasisBlock(SHELL_L[shl], ex, co))
            i += 2 + ne
            continue
        i += 1
    return out


def format_basis(basis: Basis) -> str:
    parts = []
    for z, blocks in basis.items():
        parts.append("A %d" % z)
        for b in blocks:
            parts.append("$ %s-TYPE FUNCTIONS" % "SPDFG"[b.l])
            parts.append("%d %d" % (len(b.exps), b.coefs.shape[1]))
            for r in range(len(b.exps)):
                parts.append(" ".join(["%.16e" % b.exps[r]] + ["%.16e" % x for x in b.coefs[r]]))
    return "\n".join(parts) + "\n"


def format_unitcell(cell: Cell) -> str:
    nx, ny, nz = cell.ncell
    if cell.kind == "Tori1D":
        l2 = "%d %.16g %.16g" % (nx, cell.spacing, cell.L[0])
    elif cell.kind == "Tori2D":
        l2 = "%d %d %.16g %.16g %.16g" % (nx, ny, cell.spacing, cell.L[0], cell.L[1])
    else:
        l2 = "%d %d %d %.16g %.16g %.16g %.16g" % (nx, ny, nz, cell.spacing, *cell.L)
    rows = [cell.kind, l2] + cell.keywords + ["$$"]
    rows += ["%s %.16g %.16g %.16g" % (s, *xyz) for s, xyz in cell.atoms]
    rows += ["$$"]
    return "\n".join(rows) + "\n"


# ---------------------------------------------------------------------------
# supercell + AO list
# ---------------------------------------------------------------------------
def build_system(cell: Cell, basis: Basis) -> AOSystem:
    """Replicate the cell (x fastest) and classify the AOs (class.f90)."""
    nx, ny, nz = cell.ncell
    geo, chg = [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for sym, (x, y, z) in cell.atoms:
                    geo.append((x + i * cell.spacing, y + j * cell.spacing, z + k * cell.spacing))
                    chg.append(charge_of(sym))
    ctr, lxyz, poff, exps, coefs, labels, atom_of = [], [], [0], [], [], [], []
    for a, (r, z) in enumerate(zip(geo, chg)):
        if z not in basis:
            raise ValueError("no basis for atom \"A %d\" in the file Basis" % z)
        blocks = sorted(basis[z], key=lambda b: b.l)
        for b in blocks:
            for col in range(b.coefs.shape[1]):
                for lab in CART[b.l]:
                    keep = np.abs(b.coefs[:, col]) >= 1.0e-15       # filter.f90
                    ctr.append(r)
                    lxyz.append(label_to_lxyz(lab))
                    exps.extend(b.exps[keep].tolist())
                    coefs.extend(b.coefs[keep, col].tolist())
                    poff.append(len(exps))
                    labels.append(lab)
                    atom_of.append(a)
    nbas = len(ctr)
    ncell_tot = nx * ny * nz
    if nbas % ncell_tot:
        raise ValueError("basis size not a multiple of the cell count")
    return AOSystem(ndp=cell.ndp, ncell=(nx, ny, nz), nfuc=nbas // ncell_tot, L=tuple(cell.L),
                    ctr=np.array(ctr, dtype=np.float64), lxyz=np.array(lxyz, dtype=np.int32),
                    prim_off=np.array(poff, dtype=np.int32), exps=np.array(exps, dtype=np.float64),
                    coefs=np.array(coefs, dtype=np.float64), labels=labels,
                    atom_of=np.array(atom_of, dtype=np.int32), charges=np.array(chg, dtype=np.int32),
                    geometry=np.array(geo, dtype=np.float64))


# ---------------------------------------------------------------------------
# the named synthetic workloads (seeded; numpy default_rng)
# ---------------------------------------------------------------------------
STO3G_H = BasisBlock(0, np.array([3.42525091, 0.62391373, 0.16885540]),
                     np.array([[0.15432897], [0.53532814], [0.44463454]]))


def _loguniform(rng, lo, hi, n):
    return np.sort(np.exp(rng.uniform(math.log(lo), math.log(hi), n)))[::-1].copy()


def workload(name: str, seed: int = 2026) -> Tuple[Cell, Basis]:
    """The five named toroidal workloads (synthetic inputs, seeded).

    h2_ring   : Tori1D, 2 cells, spacing 1.8, L 3.6, H STO-3G s          (nbas 2)
    h_chain64 : Tori1D, 64 cells, spacing 1.8, L 115.2; per H 3 contracted
                s (4 prims log-uniform [0.1,20]) + 1 p (0.727)           (nbas 384)
    h2_sheet  : Tori2D 8x8, spacing 2.0, L 16x16; 2 H/cell; per atom
                2 s + 1 p + 1 d, exps log-uniform [0.08,50]             (nbas 1408)
    li_cube   : Tori3D 4x4x4, spacing 2.5, L 10; Z=3 at a seeded offset;
                3 s + 2 p, exps log-uniform [0.05,100]                   (nbas 576)
    h_chain128: h_chain64 geometry and basis on 128 cells, L 230.4       (nbas 768)
    """
    rng = np.random.default_rng(seed)
    if name == "h2_ring":
        return (Cell("Tori1D", (2, 1, 1), 1.8, (3.6, 0.0, 0.0), [("H", (0.0, 0.0, 0.0))]),
                {1: [STO3G_H]})
    if name in ("h_chain64", "h_chain128"):
        n = 64 if name == "h_chain64" else 128
        s_ex = _loguniform(rng, 0.1, 20.0, 4)
        s_co = rng.uniform(0.2, 1.0, (4, 3))
        basis = {1: [BasisBlock(0, s_ex, s_co), BasisBlock(1, np.array([0.727]), np.array([[1.0]]))]}
        return (Cell("Tori1D", (n, 1, 1), 1.8, (1.8 * n, 0.0, 0.0), [("H", (0.0, 0.0, 0.0))]), basis)
    if name == "h2_sheet":
        s_ex = _loguniform(rng, 0.08, 50.0, 3)
        s_co = rng.uniform(0.2, 1.0, (3, 2))
        p_ex = _loguniform(rng, 0.08, 50.0, 2)
        p_co = rng.uniform(0.2, 1.0, (2, 1))
        d_ex = _loguniform(rng, 0.08, 50.0, 1)
        basis = {1: [BasisBlock(0, s_ex, s_co), BasisBlock(1, p_ex, p_co),
                     BasisBlock(2, d_ex, np.array([[1.0]]))]}
        return (Cell("Tori2D", (8, 8, 1), 2.0, (16.0, 16.0, 0.0),
                     [("H", (0.0, 0.0, 0.0)), ("H", (1.4, 0.0, 0.0))]), basis)
    if name == "li_cube":
        off = tuple(float(x) for x in rng.uniform(-0.3, 0.3, 3))
        s_ex = _loguniform(rng, 0.05, 100.0, 4)
        s_co = rng.uniform(0.2, 1.0, (4, 3))
        p_ex = _loguniform(rng, 0.05, 100.0, 2)
        p_co = rng.uniform(0.2, 1.0, (2, 2))
        basis = {3: [BasisBlock(0, s_ex, s_co), BasisBlock(1, p_ex, p_co)]}
        return (Cell("Tori3D", (4, 4, 4), 2.5, (10.0, 10.0, 10.0), [("Li", off)]), basis)
    raise KeyError(name)


def scaled_down(cell: Cell, ncell: Sequence[int]) -> Cell:
    """Same cell and spacing on fewer cells (the torus length follows)."""
    n = tuple(int(x) for x in ncell)
    L = tuple(cell.spacing * n[d] if cell.L[d] > 0 else 0.0 for d in range(3))
    return dataclasses.replace(cell, ncell=n, L=L)
