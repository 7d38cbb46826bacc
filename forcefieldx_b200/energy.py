"""Host-side mirror of Force Field X's ForceFieldEnergy for the AMOEBA vdW + PME path.

Method names and meanings follow the reference
(modules/potential/src/main/java/ffx/potential/ForceFieldEnergy.java):

=============================  ===========================================================
this class                     reference
=============================  ===========================================================
energy(x)                      ForceFieldEnergy.energy(double[])            :1806-1830
energy_and_gradient(x, g)      ForceFieldEnergy.energyAndGradient(x, g)     :1843-1890
set_coordinates(x)             ForceFieldEnergy.setCoordinates             :2629
set_crystal(box, grid)         ForceFieldEnergy.setCrystal                  :2650-2666
update_parameters(system)      OpenMMEnergy.updateParameters (openmm/OpenMMEnergy.java:623)
get_permanent_multipole_energy getPermanentMultipoleEnergy                  :2294
get_polarization_energy        getPolarizationEnergy                        :2322
get_vdw_energy                 getVanDerWaalsEnergy
get_induced_dipoles            ParticleMeshEwald.inducedDipole[0] / inducedDipoleCR[0]
=============================  ===========================================================

Every call goes through libffxcuda.so (include/ffxcuda.h).  There is no CPU
fallback: a missing library or device raises.  A nonzero status raises
EnergyException, as the reference throws it from PCGSolver.java:554-568 and
RealSpaceEnergyRegion.java:384-391.
"""
from __future__ import annotations

import ctypes
import dataclasses
import warnings
from typing import Optional

import numpy as np

from . import cabi
from .system import COUNT_NAMES, TERM_NAMES, AmoebaParams, AmoebaSystem, params_struct


class EnergyException(RuntimeError):
    """ffx.potential.utils.EnergyException: the evaluation failed (status code attached)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{cabi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_LIB = None


def library() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = cabi.load_library()
    return _LIB


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class ForceFieldEnergy:
    """AMOEBA vdW + PME energy and gradient on one B200 (one handle, one CUDA stream)."""

    def __init__(self, system: AmoebaSystem, params: AmoebaParams, _handle=None):
        self.lib = library()
        self.system = system
        self.params = params
        self.n = system.n_atoms
        self._owned = _handle is None
        if _handle is None:
            s, self._keep = system.c_struct(cabi)
            p = params_struct(params, cabi)
            h = ctypes.c_void_p()
            st = self.lib.ffxg_create(ctypes.byref(s), ctypes.byref(p), ctypes.byref(h))
            if st != 0:
                raise EnergyException(st, self.lib.ffxg_last_error(None).decode())
        else:
            h = ctypes.c_void_p(_handle)      # a batch's system handle, owned by the batch
        self._h = h
        self.terms = np.zeros(cabi.N_TERMS)
        self.counts = np.zeros(cabi.N_COUNTS, dtype=np.int64)
        self._x = np.ascontiguousarray(system.xyz, dtype=np.float64).copy()

    # ------------------------------------------------------------------
    def _check(self, st: int):
        """Nonzero status -> EnergyException, except RANGE (the mixed form's fixed-point sums
        left their exact range: outputs complete, not bitwise reproducible), which warns."""
        self.last_status = st
        if st == cabi.STATUS_RANGE:
            warnings.warn(self.lib.ffxg_last_error(self._h).decode(), RuntimeWarning, stacklevel=3)
        elif st != 0:
            raise EnergyException(st, self.lib.ffxg_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            if self._owned:
                self.lib.ffxg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------
    def set_coordinates(self, x) -> None:
        self._x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(self.n, 3))
        self._check(self.lib.ffxg_set_coordinates(self._h, _dp(self._x)))

    def set_crystal(self, box, pme_grid=None, angles=None) -> None:
        """A new cell: edges, optionally angles (alpha, beta, gamma; None: 90) and PME mesh
        dimensions (None keeps the mesh)."""
        b = np.ascontiguousarray(np.broadcast_to(np.asarray(box, dtype=np.float64), (3,)))
        ang = np.ascontiguousarray(angles if angles is not None else (90.0, 90.0, 90.0), dtype=np.float64)
        g = None if pme_grid is None else np.ascontiguousarray(pme_grid, dtype=np.int32)
        self._check(self.lib.ffxg_set_box(self._h, _dp(b), _dp(ang),
                                          g.ctypes.data_as(cabi._I) if g is not None else None))
        grid = tuple(self.params.grid()) if g is None else tuple(int(v) for v in g)
        self.params = dataclasses.replace(self.params, box=tuple(float(v) for v in b), pme_grid=grid,
                                          angles=tuple(float(v) for v in ang))

    def update_parameters(self, system: AmoebaSystem) -> None:
        """New multipole, polarization, damping, reduction and vdW-table values for the same
        atoms and topology (in place on the device)."""
        s, keep = system.c_struct(cabi)
        self._check(self.lib.ffxg_update_parameters(self._h, ctypes.byref(s)))
        self.system = system

    def energy(self, x=None) -> float:
        if x is not None:
            self.set_coordinates(x)
        else:
            self._check(self.lib.ffxg_set_coordinates(self._h, _dp(self._x)))
        self._check(self.lib.ffxg_energy(self._h, 0, _dp(self.terms), None,
                                         self.counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return float(self.terms[9])

    def energy_and_gradient(self, x=None, g: Optional[np.ndarray] = None):
        """Returns (energy, gradient[n,3]); fills ``g`` in place when given."""
        if x is not None:
            self._x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(self.n, 3))
        out = np.zeros((self.n, 3)) if g is None else g
        buf = out if (out.flags.c_contiguous and out.dtype == np.float64) else np.zeros((self.n, 3))
        self._check(self.lib.ffxg_energy_and_gradient(
            self._h, _dp(self._x), _dp(self.terms), _dp(buf),
            self.counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        if buf is not out:
            out[...] = buf.reshape(out.shape)
        return float(self.terms[9]), out

    def energy_device(self, d_xyz: int, d_grad: int = 0) -> float:
        """Device-resident evaluation: d_xyz / d_grad are device pointers ([n][3] float64)."""
        self._check(self.lib.ffxg_energy_device(self._h, ctypes.c_void_p(d_xyz),
                                                ctypes.c_void_p(d_grad) if d_grad else None,
                                                _dp(self.terms),
                                                self.counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return float(self.terms[9])

    # ------------------------------------------------------------------
    def term(self, name: str) -> float:
        return float(self.terms[TERM_NAMES.index(name)])

    def count(self, name: str) -> int:
        return int(self.counts[COUNT_NAMES.index(name)])

    def get_vdw_energy(self) -> float:
        return self.term("vdw")

    def get_permanent_multipole_energy(self) -> float:
        return self.term("permanent")

    def get_polarization_energy(self) -> float:
        return self.term("polarization")

    def get_induced_dipoles(self):
        u = np.zeros((self.n, 3))
        ucr = np.zeros((self.n, 3))
        self._check(self.lib.ffxg_get_induced_dipoles(self._h, _dp(u), _dp(ucr)))
        return u, ucr

    def get_global_multipoles(self):
        m = np.zeros((self.n, 10))
        self._check(self.lib.ffxg_get_global_multipoles(self._h, _dp(m)))
        return m

    def get_permanent_potential(self):
        """ParticleMeshEwald.cartesianMultipolePhi: the permanent multipoles' reciprocal-space
        potential and its derivatives at each atom, [n, 20]."""
        phi = np.zeros((self.n, 20))
        self._check(self.lib.ffxg_get_permanent_potential(self._h, _dp(phi)))
        return phi

    def neighbor_pairs(self) -> np.ndarray:
        cnt = ctypes.c_int64(0)
        self._check(self.lib.ffxg_get_neighbor_pairs(self._h, None, ctypes.byref(cnt)))
        out = np.zeros((cnt.value, 2), dtype=np.int32)
        self._check(self.lib.ffxg_get_neighbor_pairs(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                     ctypes.byref(cnt)))
        return out

    def neighbor_images(self) -> np.ndarray:
        """Rows (i, k, nx, ny, nz), one per image pair of the buffered list (k > i, or k == i
        with n > 0); n is the lattice shift of x_k + n L - x_i, zero for minimum-image lists."""
        cnt = ctypes.c_int64(0)
        self._check(self.lib.ffxg_get_neighbor_images(self._h, None, ctypes.byref(cnt)))
        out = np.zeros((cnt.value, 5), dtype=np.int32)
        self._check(self.lib.ffxg_get_neighbor_images(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                      ctypes.byref(cnt)))
        return out

    def param_gradients(self):
        """(dE/dM [n, 10] of each atom's local-frame multipole, dE/dalpha [n]) of the last
        evaluation (Thole damping fixed)."""
        dM = np.zeros((self.n, 10))
        dA = np.zeros(self.n)
        self._check(self.lib.ffxg_param_grad(self._h, _dp(dM), _dp(dA)))
        return dM, dA

    @staticmethod
    def per_type(values: np.ndarray, types: np.ndarray) -> dict:
        """Sum per-atom parameter gradients over atoms of each type: {type: sum}."""
        types = np.asarray(types)
        return {int(t): values[types == t].sum(axis=0) for t in np.unique(types)}

    def set_image_mode(self, all_images: bool) -> None:
        """Force lists of every lattice image (True) or return to the automatic choice."""
        self._check(self.lib.ffxg_set_image_mode(self._h, 1 if all_images else 0))

    @property
    def stream(self) -> int:
        return int(self.lib.ffxg_stream(self._h) or 0)

    def set_alchemy(self, alchemy) -> None:
        """Soft atoms and vdW softcore keys (an Alchemy, or None to clear)."""
        if alchemy is None:
            self._check(self.lib.ffxg_set_alchemy(self._h, None))
            return
        a, keep = alchemy.c_struct(cabi)
        self._check(self.lib.ffxg_set_alchemy(self._h, ctypes.byref(a)))

    def set_lambda(self, lam: float) -> None:
        """LambdaInterface.setLambda for the vdW softcore."""
        self._check(self.lib.ffxg_set_lambda(self._h, float(lam)))

    def get_dEdL(self):
        """(dU/dL, d2U/dL2, dU/dX dL [n, 3]) of the last evaluation."""
        d1 = ctypes.c_double()
        d2 = ctypes.c_double()
        g = np.zeros((self.n, 3))
        self._check(self.lib.ffxg_get_dEdL(self._h, ctypes.byref(d1), ctypes.byref(d2), _dp(g)))
        return d1.value, d2.value, g

    def md_setup(self, mass, settle=None, d1: float = 0.0, d2: float = 0.0) -> None:
        """Masses (amu) and rigid three-site molecules [(centre, partner, partner), ...] for md_run."""
        self._md_mass = np.ascontiguousarray(mass, dtype=np.float64)
        self._md_settle = None if settle is None else np.ascontiguousarray(settle, dtype=np.int32).reshape(-1, 3)
        ns = 0 if self._md_settle is None else self._md_settle.shape[0]
        md = cabi.FfxgMd(_dp(self._md_mass), ns,
                         self._md_settle.ctypes.data_as(cabi._I) if ns else cabi._I(), float(d1), float(d2))
        self._check(self.lib.ffxg_md_setup(self._h, ctypes.byref(md)))

    def md_run(self, xyz, vel, dt: float, n_steps: int):
        """Velocity Verlet on the device; returns (xyz, vel, epot[n_steps], ekin[n_steps])."""
        x = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        v = np.ascontiguousarray(vel, dtype=np.float64).copy()
        ep = np.zeros(n_steps)
        ek = np.zeros(n_steps)
        self._check(self.lib.ffxg_md_run(self._h, float(dt), int(n_steps), _dp(x), _dp(v), _dp(ep), _dp(ek)))
        return x, v, ep, ek

    def set_scf_predictor(self, aspc: bool) -> None:
        """Start each PCG solve from the ASPC prediction (the scf-predictor key) or not."""
        self._check(self.lib.ffxg_set_scf_predictor(self._h, 1 if aspc else 0))

    def set_graph_mode(self, on: bool) -> None:
        """Replay the evaluation as one captured CUDA graph (default) or launch directly."""
        self._check(self.lib.ffxg_set_graph_mode(self._h, 1 if on else 0))

    def launch_count(self) -> int:
        return int(self.lib.ffxg_last_launch_count(self._h))

    def list_builds(self) -> int:
        """Neighbour-list builds since the handle was created."""
        return int(self.lib.ffxg_list_builds(self._h))


class CrystalEnergy:
    """Energy and gradient of an asymmetric unit in a space group (any cell: params.angles),
    evaluated as the P1 unit cell of its symmetry mates (forcefieldx_b200.ffxio): the
    reference sums the asymmetric unit's interactions with its mates
    (ParticleMeshEwald / NeighborList symmetry loops); the cell of mates has the same
    energy per asymmetric unit, and the asymmetric unit's gradient is the first mate's."""

    def __init__(self, asu_system: AmoebaSystem, params: AmoebaParams, space_group: str):
        from .ffxio import SPACE_GROUPS, expand_system
        self.space_group = space_group.upper().replace(" ", "")
        self.n_asu = asu_system.n_atoms
        self.n_symm = len(SPACE_GROUPS[self.space_group])
        self.box = params.box
        self.angles = tuple(params.angles)
        self.cell = expand_system(asu_system, params.box, self.space_group, self.angles)
        self.ffe = ForceFieldEnergy(self.cell, params)

    def close(self):
        self.ffe.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def energy_and_gradient(self, x_asu=None):
        """(energy per asymmetric unit, gradient [n_asu, 3]) at the asymmetric unit's coordinates."""
        from .ffxio import expand_coordinates
        x = None if x_asu is None else expand_coordinates(x_asu, self.box, self.space_group, self.angles)
        e, g = self.ffe.energy_and_gradient(x)
        return e / self.n_symm, g[:self.n_asu].copy()

    @property
    def terms(self) -> np.ndarray:
        return self.ffe.terms / self.n_symm
