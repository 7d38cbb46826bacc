"""ctypes binding of liboracle.so, the CPU FP64 restatement of the reference path.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from forcefieldx_b200 import cabi
from forcefieldx_b200.system import AmoebaParams, AmoebaSystem, params_struct

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or \
            os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "ffx_oracle.cpp")):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        D = ctypes.POINTER(ctypes.c_double)
        L.oracle_energy.restype = ctypes.c_int
        L.oracle_energy.argtypes = [ctypes.POINTER(cabi.FfxgSystem), ctypes.POINTER(cabi.FfxgParams), D,
                                    ctypes.c_int, ctypes.c_int, D, D, ctypes.POINTER(ctypes.c_int64), D, D, D]
        L.oracle_neighbor_pairs.restype = ctypes.c_int64
        L.oracle_neighbor_pairs.argtypes = [ctypes.POINTER(cabi.FfxgSystem), ctypes.POINTER(cabi.FfxgParams), D,
                                            ctypes.POINTER(ctypes.c_int32)]
        L.oracle_neighbor_images.restype = ctypes.c_int64
        L.oracle_neighbor_images.argtypes = [ctypes.POINTER(cabi.FfxgSystem), ctypes.POINTER(cabi.FfxgParams), D,
                                             ctypes.POINTER(ctypes.c_int32)]
        L.oracle_param_grad.restype = ctypes.c_int
        L.oracle_param_grad.argtypes = [ctypes.POINTER(cabi.FfxgSystem), ctypes.POINTER(cabi.FfxgParams), D, D, D]
        L.oracle_set_images.restype = None
        L.oracle_set_images.argtypes = [ctypes.c_int]
        L.oracle_set_alchemy.restype = None
        L.oracle_set_alchemy.argtypes = [ctypes.POINTER(cabi.FfxgAlchemy), ctypes.c_int, ctypes.c_double]
        L.oracle_get_dEdL.restype = None
        L.oracle_get_dEdL.argtypes = [D, D, D]
        L.oracle_erfc.restype = ctypes.c_double
        L.oracle_erfc.argtypes = [ctypes.c_double]
        L.oracle_bspline.restype = None
        L.oracle_bspline.argtypes = [ctypes.c_double, ctypes.c_int, D]
        L.oracle_fft3d.restype = None
        L.oracle_fft3d.argtypes = [D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def energy(system: AmoebaSystem, params: AmoebaParams, xyz=None, gradient=True, nthreads=0, alchemy=None,
           lam=1.0, all_images=False):
    """Returns dict(terms, grad, counts, induced, induced_cr, global_mpole, status), and with
    an Alchemy also dEdL, d2EdL2 and dEdXdL (the vdW softcore at lambda `lam`).
    all_images=True forces multi-image lists where the minimum image would suffice."""
    L = lib()
    L.oracle_set_images(1 if all_images else 0)
    if alchemy is not None:
        a, keep_a = alchemy.c_struct(cabi)
        L.oracle_set_alchemy(ctypes.byref(a), system.n_atoms, float(lam))
    else:
        L.oracle_set_alchemy(None, system.n_atoms, 1.0)
    s, keep = system.c_struct(cabi)
    p = params_struct(params, cabi)
    n = system.n_atoms
    x = np.ascontiguousarray(system.xyz if xyz is None else xyz, dtype=np.float64)
    terms = np.zeros(cabi.N_TERMS)
    grad = np.zeros((n, 3))
    counts = np.zeros(cabi.N_COUNTS, dtype=np.int64)
    ind = np.zeros((n, 3))
    indcr = np.zeros((n, 3))
    gm = np.zeros((n, 10))
    st = L.oracle_energy(ctypes.byref(s), ctypes.byref(p), _dp(x), 1 if gradient else 0, int(nthreads),
                         _dp(terms), _dp(grad), counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         _dp(ind), _dp(indcr), _dp(gm))
    out = dict(terms=terms, grad=grad, counts=counts, induced=ind, induced_cr=indcr, global_mpole=gm,
               status=int(st))
    L.oracle_set_images(0)
    if alchemy is not None:
        d1 = ctypes.c_double()
        d2 = ctypes.c_double()
        lg = np.zeros((n, 3))
        L.oracle_get_dEdL(ctypes.byref(d1), ctypes.byref(d2), _dp(lg))
        out.update(dEdL=d1.value, d2EdL2=d2.value, dEdXdL=lg)
        L.oracle_set_alchemy(None, n, 1.0)
    return out


def neighbor_pairs(system: AmoebaSystem, params: AmoebaParams, xyz=None) -> np.ndarray:
    L = lib()
    s, keep = system.c_struct(cabi)
    p = params_struct(params, cabi)
    x = np.ascontiguousarray(system.xyz if xyz is None else xyz, dtype=np.float64)
    n = L.oracle_neighbor_pairs(ctypes.byref(s), ctypes.byref(p), _dp(x), None)
    out = np.zeros((n, 2), dtype=np.int32)
    L.oracle_neighbor_pairs(ctypes.byref(s), ctypes.byref(p), _dp(x),
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return out


def neighbor_images(system: AmoebaSystem, params: AmoebaParams, xyz=None, all_images=False) -> np.ndarray:
    """Rows (i, k, nx, ny, nz): one per image pair of the buffered list (i < k, or i == k
    with n > 0), n the lattice shift of x_k + n L - x_i (zero outside multi-image mode)."""
    L = lib()
    L.oracle_set_images(1 if all_images else 0)
    s, keep = system.c_struct(cabi)
    p = params_struct(params, cabi)
    x = np.ascontiguousarray(system.xyz if xyz is None else xyz, dtype=np.float64)
    n = L.oracle_neighbor_images(ctypes.byref(s), ctypes.byref(p), _dp(x), None)
    out = np.zeros((n, 5), dtype=np.int32)
    L.oracle_neighbor_images(ctypes.byref(s), ctypes.byref(p), _dp(x),
                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    L.oracle_set_images(0)
    return out


def param_gradients(system: AmoebaSystem, params: AmoebaParams, xyz=None):
    """(dE/dM [n,10] w.r.t. each atom's local multipole, dE/dalpha [n])."""
    L = lib()
    L.oracle_set_alchemy(None, system.n_atoms, 1.0)
    s, keep = system.c_struct(cabi)
    p = params_struct(params, cabi)
    x = np.ascontiguousarray(system.xyz if xyz is None else xyz, dtype=np.float64)
    dM = np.zeros((system.n_atoms, 10))
    dA = np.zeros(system.n_atoms)
    st = L.oracle_param_grad(ctypes.byref(s), ctypes.byref(p), _dp(x), _dp(dM), _dp(dA))
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    return dM, dA


def erfc(x: float) -> float:
    return lib().oracle_erfc(float(x))


def bspline(x: float, order: int = 5) -> np.ndarray:
    out = np.zeros((order, 4))
    lib().oracle_bspline(float(x), int(order), _dp(out))
    return out


def fft3d(data: np.ndarray, sign: int) -> np.ndarray:
    """data: complex128 array of shape (nz, ny, nx)."""
    nz, ny, nx = data.shape
    buf = np.ascontiguousarray(np.stack([data.real, data.imag], axis=-1), dtype=np.float64)
    lib().oracle_fft3d(_dp(buf), nx, ny, nz, int(sign))
    return buf[..., 0] + 1j * buf[..., 1]
