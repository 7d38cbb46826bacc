"""Resolved AMOEBA systems: the per-atom data the energy library consumes.

An :class:`AmoebaSystem` holds exactly what Force Field X's ParticleMeshEwald and
VanDerWaals keep after parameter assignment:

* local-frame multipoles, frame type and frame-defining atoms
  (ParticleMeshEwald.assignMultipoles, ParticleMeshEwald.java:2535-2600;
  MultipoleType.multipoleTypeFactory, MultipoleType.java:545-680),
* polarizability, Thole and damping (ParticleMeshEwald.java:1395-1410;
  PolarizeType.java:138-148: pdamp = polarizability^(1/6), 0 when thole is 0),
* the 1-2 .. 1-5 lists and polarization groups (ParticleMeshEwald.java:1414-1445,
  2616-2650; Atom.get12List..get15List, Atom.java:763-843),
* vdW pair tables with the CUBIC-MEAN radius and HHG epsilon rules and hydrogen
  reduction (VanDerWaalsForm.java:355-522, VanDerWaals.java:1421-1433).

It also builds the synthetic AMOEBA water boxes used for parity and throughput.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

BOHR = 0.529177210903            # Constants.BOHR (utilities/.../Constants.java:209)
ELECTRIC = 332.0637133           # Constants.DEFAULT_ELECTRIC (Constants.java:192)

FRAME_NONE, FRAME_ZONLY, FRAME_ZTHENX, FRAME_BISECTOR, FRAME_ZTHENBISECTOR, FRAME_THREEFOLD = range(6)
POLAR_NONE, POLAR_DIRECT, POLAR_MUTUAL = range(3)
PRECISION_FP64, PRECISION_MIXED = range(2)

TERM_NAMES = ["vdw", "permanent", "polarization", "perm_real", "perm_self", "perm_recip",
              "pol_real", "pol_self", "pol_recip", "total"]
COUNT_NAMES = ["vdw", "permanent", "scf_iter", "list_builds", "list_pairs", "list_growths"]


def csr_from_lists(lists: Sequence[Sequence[int]]):
    ptr = np.zeros(len(lists) + 1, dtype=np.int32)
    for i, l in enumerate(lists):
        ptr[i + 1] = ptr[i] + len(l)
    idx = np.zeros(int(ptr[-1]), dtype=np.int32)
    for i, l in enumerate(lists):
        idx[ptr[i]:ptr[i + 1]] = np.asarray(list(l), dtype=np.int32)
    return ptr, idx


def connectivity_lists(n: int, bonds: np.ndarray):
    """1-2, 1-3, 1-4, 1-5 lists with Atom.get1nList precedence (Atom.java:763-843).

    Each list excludes atoms already in a lower-order list and the atom itself,
    and is sorted by index.  Duplicates that the reference may carry are
    irrelevant to the masks, which are set-valued.
    """
    n12: List[List[int]] = [[] for _ in range(n)]
    for a, b in np.asarray(bonds, dtype=np.int64).reshape(-1, 2):
        n12[a].append(int(b))
        n12[b].append(int(a))
    n12 = [sorted(set(l)) for l in n12]
    n13, n14, n15 = [], [], []
    for i in range(n):
        s12 = set(n12[i])
        s13 = set()
        for j in n12[i]:
            for k in n12[j]:
                if k != i and k not in s12:
                    s13.add(k)
        s14 = set()
        for j in s13:
            for k in n12[j]:
                if k != i and k not in s12 and k not in s13:
                    s14.add(k)
        s15 = set()
        for j in s14:
            for k in n12[j]:
                if k != i and k not in s12 and k not in s13 and k not in s14:
                    s15.add(k)
        n13.append(sorted(s13))
        n14.append(sorted(s14))
        n15.append(sorted(s15))
    return n12, n13, n14, n15


def combine_vdw(radius: np.ndarray, eps: np.ndarray, pairs: Optional[dict] = None):
    """Pair tables (1/Rmin, eps) for classes with diameters ``radius``.

    CUBIC-MEAN radius rule and HHG epsilon rule on half-diameters
    (VanDerWaalsForm.getCombinedRadius / getCombinedEps, VanDerWaalsForm.java:476-522);
    ``pairs`` maps (i, j) -> (rmin, eps) overrides (vdwpr, :446-470).
    """
    r = 0.5 * np.asarray(radius, dtype=np.float64)
    e = np.asarray(eps, dtype=np.float64)
    t = len(r)
    inv = np.zeros((t, t))
    ee = np.zeros((t, t))
    for i in range(t):
        for j in range(t):
            ri, rj = r[i], r[j]
            ri2, rj2 = ri * ri, rj * rj
            den = ri2 + rj2
            rad = 2.0 * (ri * ri2 + rj * rj2) / den if den > 0 else 0.0
            inv[i, j] = 1.0 / rad if rad > 0 else 0.0
            sei, sej = math.sqrt(e[i]), math.sqrt(e[j])
            ee[i, j] = 0.0 if e[i] * e[j] == 0.0 else 4.0 * (e[i] * e[j]) / ((sei + sej) * (sei + sej))
    if pairs:
        for (i, j), (rmin, ep) in pairs.items():
            for a, b in ((i, j), (j, i)):
                inv[a, b] = 1.0 / rmin if rmin > 0 else 0.0
                ee[a, b] = ep
    return inv, ee


@dataclasses.dataclass
class AmoebaParams:
    """Hot-path keys and their Force Field X defaults (see the key table in
    ForceFieldEnergy.java:858-895, EwaldParameters.java:55-71, PCGSolver.java:300-345)."""
    box: Sequence[float]
    vdw_cutoff: float = 12.0
    vdw_taper: float = 0.9
    ewald_cutoff: float = 7.0
    ewald_alpha: float = 0.545
    list_buffer: float = 2.0
    pme_grid: Optional[Sequence[int]] = None
    pme_mesh_density: float = 1.2
    pme_order: int = 5
    polar_eps: float = 1.0e-6
    max_scf_iter: int = 1000
    polarization: int = POLAR_MUTUAL
    precond_cutoff: float = 4.5
    precond_scale: float = 2.0
    electric: float = ELECTRIC
    m12: float = 0.0
    m13: float = 0.0
    m14: float = 0.4
    m15: float = 0.8
    p12: float = 0.0
    p13: float = 0.0
    p14: float = 1.0
    p15: float = 1.0
    intra14: float = 0.5
    d11: float = 0.0
    v12: float = 0.0
    v13: float = 0.0
    v14: float = 1.0
    precision: int = PRECISION_FP64
    angles: Sequence[float] = (90.0, 90.0, 90.0)   # alpha, beta, gamma (degrees)

    def grid(self):
        if self.pme_grid is not None:
            return [int(g) for g in self.pme_grid]
        return [pme_grid_dim(a, self.pme_mesh_density) for a in self.box]


def preferred_dimension(dim: int) -> bool:
    """Complex.preferredDimension (N/fft/Complex.java:371-383): factors 7,6,5,4,3,2."""
    if dim < 2:
        return False
    for f in (7, 6, 5, 4, 3, 2):
        while dim % f == 0:
            dim //= f
    return dim <= 1


def pme_grid_dim(edge: float, density: float, grid_min: int = 16) -> int:
    """ReciprocalSpace.initConvolution grid sizing (ReciprocalSpace.java:909-975)."""
    n = int(math.floor(edge * density)) + 1
    if n % 2 != 0:
        n += 1
    while not preferred_dimension(n):
        n += 2
    return max(n, grid_min)


@dataclasses.dataclass
class AmoebaSystem:
    xyz: np.ndarray                 # [n,3]
    multipole: np.ndarray           # [n,10] e, e*A, e*A^2
    frame: np.ndarray               # [n]
    axis: np.ndarray                # [n,3]
    polarizability: np.ndarray      # [n]
    thole: np.ndarray               # [n]
    pdamp: np.ndarray               # [n]
    vdw_type: np.ndarray            # [n]
    red_parent: np.ndarray          # [n]
    red_factor: np.ndarray          # [n]
    vdw_inv_rmin: np.ndarray        # [t,t]
    vdw_eps: np.ndarray             # [t,t]
    n12: list
    n13: list
    n14: list
    n15: list
    ip11: list
    molecule: Optional[np.ndarray] = None
    name: str = ""

    @property
    def n_atoms(self) -> int:
        return int(self.xyz.shape[0])

    # ------------------------------------------------------------------
    def c_struct(self, lib_types):
        """Fill a ctypes ffxg_system; the returned keep-alive list must outlive it."""
        keep = []

        def arr(a, dtype, ctype):
            a = np.ascontiguousarray(a, dtype=dtype)
            keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(ctype))

        s = lib_types.FfxgSystem()
        s.n_atoms = self.n_atoms
        s.xyz = arr(self.xyz, np.float64, ctypes.c_double)
        s.multipole = arr(self.multipole, np.float64, ctypes.c_double)
        s.frame = arr(self.frame, np.int32, ctypes.c_int32)
        s.axis = arr(self.axis, np.int32, ctypes.c_int32)
        s.polarizability = arr(self.polarizability, np.float64, ctypes.c_double)
        s.thole = arr(self.thole, np.float64, ctypes.c_double)
        s.pdamp = arr(self.pdamp, np.float64, ctypes.c_double)
        s.vdw_type = arr(self.vdw_type, np.int32, ctypes.c_int32)
        s.red_parent = arr(self.red_parent, np.int32, ctypes.c_int32)
        s.red_factor = arr(self.red_factor, np.float64, ctypes.c_double)
        s.n_vdw_types = int(self.vdw_inv_rmin.shape[0])
        s.vdw_inv_rmin = arr(self.vdw_inv_rmin, np.float64, ctypes.c_double)
        s.vdw_eps = arr(self.vdw_eps, np.float64, ctypes.c_double)
        for name, lists in (("mask12", self.n12), ("mask13", self.n13), ("mask14", self.n14),
                            ("mask15", self.n15), ("ip11", self.ip11)):
            ptr, idx = csr_from_lists(lists)
            if idx.size == 0:
                idx = np.zeros(1, dtype=np.int32)
            setattr(s, name + "_ptr", arr(ptr, np.int32, ctypes.c_int32))
            setattr(s, name + "_idx", arr(idx, np.int32, ctypes.c_int32))
        return s, keep

    def save_npz(self, path: str, **extra):
        ptrs = {}
        for name, lists in (("n12", self.n12), ("n13", self.n13), ("n14", self.n14),
                            ("n15", self.n15), ("ip11", self.ip11)):
            p, i = csr_from_lists(lists)
            ptrs[name + "_ptr"], ptrs[name + "_idx"] = p, i
        np.savez_compressed(path, xyz=self.xyz, multipole=self.multipole, frame=self.frame,
                            axis=self.axis, polarizability=self.polarizability, thole=self.thole,
                            pdamp=self.pdamp, vdw_type=self.vdw_type, red_parent=self.red_parent,
                            red_factor=self.red_factor, vdw_inv_rmin=self.vdw_inv_rmin,
                            vdw_eps=self.vdw_eps, **ptrs, **extra)

    @staticmethod
    def load_npz(path: str) -> "AmoebaSystem":
        d = np.load(path)

        def lists(name):
            p, i = d[name + "_ptr"], d[name + "_idx"]
            return [i[p[k]:p[k + 1]].tolist() for k in range(len(p) - 1)]

        return AmoebaSystem(xyz=d["xyz"], multipole=d["multipole"], frame=d["frame"], axis=d["axis"],
                            polarizability=d["polarizability"], thole=d["thole"], pdamp=d["pdamp"],
                            vdw_type=d["vdw_type"], red_parent=d["red_parent"], red_factor=d["red_factor"],
                            vdw_inv_rmin=d["vdw_inv_rmin"], vdw_eps=d["vdw_eps"], n12=lists("n12"),
                            n13=lists("n13"), n14=lists("n14"), n15=lists("n15"), ip11=lists("ip11"),
                            name=str(path))


def params_struct(params: AmoebaParams, lib_types):
    p = lib_types.FfxgParams()
    for i in range(3):
        p.box[i] = float(params.box[i])
    g = params.grid()
    for i in range(3):
        p.pme_grid[i] = int(g[i])
    for f in ("vdw_cutoff", "vdw_taper", "ewald_cutoff", "ewald_alpha", "list_buffer", "polar_eps",
              "precond_cutoff", "precond_scale", "electric", "m12", "m13", "m14", "m15", "p12", "p13",
              "p14", "p15", "intra14", "d11", "v12", "v13", "v14"):
        setattr(p, f, float(getattr(params, f)))
    p.pme_order = int(params.pme_order)
    p.max_scf_iter = int(params.max_scf_iter)
    p.polarization = int(params.polarization)
    p.precision = int(params.precision)
    for i in range(3):
        p.angles[i] = float(params.angles[i])
    return p


# ---------------------------------------------------------------------------
# AMOEBA water (P/parameters/ff/AMOEBA_WATER_2003): multipoles in Bohr units as in
# the parameter file; converted to e*A / e*A^2 by MultipoleType.bohrToElectronAngstroms.
WATER_O_MPOLE_BOHR = (-0.51966, (0.0, 0.0, 0.14279), ((0.37928, 0.0, 0.0), (0.0, -0.41809, 0.0), (0.0, 0.0, 0.03881)))
WATER_H_MPOLE_BOHR = (0.25983, (-0.03859, 0.0, -0.05818),
                      ((-0.03673, 0.0, -0.00203), (0.0, -0.10739, 0.0), (-0.00203, 0.0, 0.14412)))
WATER_POLAR = (0.837, 0.496)     # O, H (A^3)
WATER_THOLE = 0.39
WATER_VDW = ((3.405, 0.110, 0.0), (2.655, 0.0135, 0.910))  # diameter, eps, reduction


def pack_multipole_bohr(charge, dipole, quad):
    """MultipoleType.pack + bohrToElectronAngstroms (MultipoleType.java:1115-1140)."""
    b, b2 = BOHR, BOHR * BOHR
    return np.array([charge, dipole[0] * b, dipole[1] * b, dipole[2] * b,
                     quad[0][0] * b2, quad[1][1] * b2, quad[2][2] * b2,
                     quad[0][1] * b2, quad[0][2] * b2, quad[1][2] * b2])


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_box(n_side: int, edge: float, seed: int = 2026, jitter: float = 0.15,
              n_waters: Optional[int] = None) -> AmoebaSystem:
    """``n_side``^3 rigid AMOEBA waters on a seeded jittered cubic lattice in a cube
    of ``edge`` A, uniform random orientations, O-H 0.9572 A, H-O-H 104.52 deg.
    With ``n_waters`` set, that many sites of the lattice are drawn without replacement
    (``n_side`` is then the lattice size, at least the cube root of ``n_waters``)."""
    rng = np.random.default_rng(seed)
    nw = n_side ** 3
    sites = None
    if n_waters is not None:
        if n_waters > nw:
            raise ValueError("n_waters exceeds the lattice")
        sites = set(rng.choice(nw, size=n_waters, replace=False).tolist())
        nw = n_waters
    spacing = edge / n_side
    roh, theta = 0.9572, math.radians(104.52)
    local = np.array([[0.0, 0.0, 0.0],
                      [roh * math.sin(theta / 2), 0.0, roh * math.cos(theta / 2)],
                      [-roh * math.sin(theta / 2), 0.0, roh * math.cos(theta / 2)]])
    xyz = np.zeros((3 * nw, 3))
    m = 0
    site = -1
    for a in range(n_side):
        for b in range(n_side):
            for c in range(n_side):
                site += 1
                if sites is not None and site not in sites:
                    continue
                origin = (np.array([a, b, c]) + 0.5) * spacing - 0.5 * edge
                origin = origin + rng.uniform(-jitter, jitter, size=3)
                rot = _random_rotation(rng)
                xyz[3 * m:3 * m + 3] = origin + local @ rot.T
                m += 1
    n = 3 * nw
    mpo = pack_multipole_bohr(*WATER_O_MPOLE_BOHR)
    mph = pack_multipole_bohr(*WATER_H_MPOLE_BOHR)
    multipole = np.zeros((n, 10))
    frame = np.zeros(n, dtype=np.int32)
    axis = -np.ones((n, 3), dtype=np.int32)
    pol = np.zeros(n)
    vtype = np.zeros(n, dtype=np.int32)
    red_parent = np.arange(n, dtype=np.int32)
    red_factor = np.zeros(n)
    bonds = []
    for w in range(nw):
        o, h1, h2 = 3 * w, 3 * w + 1, 3 * w + 2
        bonds += [(o, h1), (o, h2)]
        multipole[o], multipole[h1], multipole[h2] = mpo, mph, mph
        frame[o] = FRAME_BISECTOR
        axis[o, :2] = (h1, h2)
        frame[h1] = frame[h2] = FRAME_ZTHENX
        axis[h1, :2] = (o, h2)
        axis[h2, :2] = (o, h1)
        pol[o], pol[h1], pol[h2] = WATER_POLAR[0], WATER_POLAR[1], WATER_POLAR[1]
        vtype[h1] = vtype[h2] = 1
        red_parent[h1] = red_parent[h2] = o
        red_factor[h1] = red_factor[h2] = WATER_VDW[1][2]
    thole = np.full(n, WATER_THOLE)
    pdamp = np.where(thole == 0.0, 0.0, pol ** (1.0 / 6.0))
    inv, ee = combine_vdw([WATER_VDW[0][0], WATER_VDW[1][0]], [WATER_VDW[0][1], WATER_VDW[1][1]])
    n12, n13, n14, n15 = connectivity_lists(n, np.array(bonds))
    ip11 = [[3 * (i // 3), 3 * (i // 3) + 1, 3 * (i // 3) + 2] for i in range(n)]
    return AmoebaSystem(xyz=xyz, multipole=multipole, frame=frame, axis=axis, polarizability=pol,
                        thole=thole, pdamp=pdamp, vdw_type=vtype, red_parent=red_parent,
                        red_factor=red_factor, vdw_inv_rmin=inv, vdw_eps=ee, n12=n12, n13=n13,
                        n14=n14, n15=n15, ip11=ip11, molecule=np.arange(n) // 3,
                        name=f"water{nw}")


def small_water_box(n_atoms: int, seed: int = 2026) -> Tuple[AmoebaSystem, float]:
    """A water box of ``n_atoms`` (a multiple of 3) at 29.915 A^3 per molecule, the
    density of the batched small-system workload: returns (system, edge)."""
    if n_atoms % 3:
        raise ValueError("n_atoms must be a multiple of 3")
    nw = n_atoms // 3
    edge = (nw * 29.915) ** (1.0 / 3.0)
    n_side = int(math.ceil(nw ** (1.0 / 3.0) - 1e-9))
    return water_box(n_side, edge, seed=seed, n_waters=nw, jitter=0.1), edge


def replicate(system: AmoebaSystem, edge, reps=(2, 2, 2)) -> AmoebaSystem:
    """The replicate supercell of an orthorhombic box: copies of every atom at lattice
    translations t = (i a, j b, k c), 0 <= i < reps[0] ..., with connectivity and frame
    indices offset per copy (the expansion C/ReplicatesCrystal.java:172-202 describes).
    Copy m = (k * reps[1] + j) * reps[0] + i holds atoms m*n .. m*n + n - 1."""
    edge = np.broadcast_to(np.asarray(edge, dtype=np.float64), (3,))
    copies = [(i, j, k) for k in range(reps[2]) for j in range(reps[1]) for i in range(reps[0])]
    xyz = np.concatenate([system.xyz + np.array(c) * edge for c in copies])
    return tile_system(system, xyz, len(copies))


def tile_system(system: AmoebaSystem, xyz: np.ndarray, nc: int) -> AmoebaSystem:
    """``nc`` copies of a system with the given coordinates ([nc * n, 3], copy after copy):
    per-atom parameters repeated, connectivity and frame indices offset per copy.  Local
    frame multipoles need no change (each copy's frames follow its own atoms)."""
    n = system.n_atoms
    tile = lambda a: np.concatenate([a] * nc)  # noqa: E731
    axis = np.concatenate([np.where(system.axis >= 0, system.axis + m * n, -1) for m in range(nc)]).astype(np.int32)
    red_parent = np.concatenate([system.red_parent + m * n for m in range(nc)]).astype(np.int32)
    shift_lists = lambda L: [[k + m * n for k in row] for m in range(nc) for row in L]  # noqa: E731
    mol = None
    if system.molecule is not None:
        nm = int(np.max(system.molecule)) + 1
        mol = np.concatenate([system.molecule + m * nm for m in range(nc)])
    return AmoebaSystem(xyz=xyz, multipole=tile(system.multipole), frame=tile(system.frame), axis=axis,
                        polarizability=tile(system.polarizability), thole=tile(system.thole),
                        pdamp=tile(system.pdamp), vdw_type=tile(system.vdw_type), red_parent=red_parent,
                        red_factor=tile(system.red_factor), vdw_inv_rmin=system.vdw_inv_rmin,
                        vdw_eps=system.vdw_eps, n12=shift_lists(system.n12), n13=shift_lists(system.n13),
                        n14=shift_lists(system.n14), n15=shift_lists(system.n15), ip11=shift_lists(system.ip11),
                        molecule=mol, name=f"{system.name}x{nc}")


def water_params(edge: float, **kw) -> AmoebaParams:
    """The keys of the water configurations: 7 A real space, 9 A vdW, alpha 0.545, order 5."""
    base = dict(box=(edge, edge, edge), vdw_cutoff=9.0, ewald_cutoff=7.0, ewald_alpha=0.545,
                pme_order=5, polar_eps=1.0e-6)
    base.update(kw)
    return AmoebaParams(**base)


@dataclasses.dataclass
class Alchemy:
    """Soft atoms and vdW softcore keys (the reference's Atom.applyLambda flags and the
    vdw-lambda-* / *-softcore keys, VanDerWaals.java:336-357)."""
    soft: np.ndarray                      # [n] bool / 0-1
    molecule: Optional[np.ndarray] = None  # [n] molecule index, or None (every atom its own)
    vdw_lambda_alpha: float = 0.25
    vdw_lambda_exponent: float = 3.0
    vdw_lambda_end: float = 1.0
    intermolecular_softcore: bool = False
    intramolecular_softcore: bool = False
    # Electrostatics (elec-lambdaterm, OST mode; AlchemicalParameters.java:60-190 defaults).
    elec: bool = False
    permanent_lambda_alpha: float = 2.0
    permanent_lambda_exponent: float = 3.0
    permanent_lambda_start: float = 0.4
    permanent_lambda_end: float = 1.0
    polarization_lambda_start: float = 0.75
    polarization_lambda_end: float = 1.0
    polarization_lambda_exponent: float = 3.0
    ligand_vapor_elec: bool = True
    no_ligand_condensed_scf: bool = True

    def c_struct(self, cabi):
        soft = np.ascontiguousarray(self.soft, dtype=np.int32)
        mol = None if self.molecule is None else np.ascontiguousarray(self.molecule, dtype=np.int32)
        ptr = lambda a: a.ctypes.data_as(cabi._I) if a is not None else cabi._I()  # noqa: E731
        a = cabi.FfxgAlchemy(ptr(soft), ptr(mol), float(self.vdw_lambda_alpha), float(self.vdw_lambda_exponent),
                             float(self.vdw_lambda_end), int(self.intermolecular_softcore),
                             int(self.intramolecular_softcore), int(self.elec),
                             float(self.permanent_lambda_alpha), float(self.permanent_lambda_exponent),
                             float(self.permanent_lambda_start), float(self.permanent_lambda_end),
                             float(self.polarization_lambda_start), float(self.polarization_lambda_end),
                             float(self.polarization_lambda_exponent), int(self.ligand_vapor_elec),
                             int(self.no_ligand_condensed_scf))
        return a, (soft, mol)


# The two named water workloads.
WATER_24K = dict(n_side=20, edge=62.08, grid=(64, 64, 64))   # 8,000 waters, 24,000 atoms
WATER_648 = dict(n_side=6, edge=18.643, grid=(20, 20, 20))  # 216 waters, 648 atoms
