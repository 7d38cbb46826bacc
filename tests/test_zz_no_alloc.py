"""The allocation-free reciprocal-space entry point against the handle-based path.

ffxg_pme_recip_permanent_noalloc serves callers that may not allocate device
memory (their GPU memory belongs to another allocator, or they must not pay
cudaMalloc's synchronisation).  This test plays such a caller: it owns every
buffer, makes two calls in a row through the C ABI, and checks each against what
ffxg_energy computes for the same coordinates and multipoles, within the parity
tolerance of the other GPU tests: the permanent reciprocal energy, and the potential
with its first and second derivatives against the handle's Cartesian potential
(ParticleMeshEwald.cartesianMultipolePhi).  Meshes: an even cube, an odd mesh, and a
non-cubic mesh at the 64-point limit with ~28,000 atoms on a stream the caller
created.  The file sorts last so a run that stops at the first failure has run every
other test already.
"""
import ctypes

import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy, library
from forcefieldx_b200.system import water_box, water_params

pytestmark = pytest.mark.gpu

E_REL = 1.0e-8
PHI_REL = 1.0e-8      # of the largest magnitude of each potential component


def _call(lib, d_xyz, d_mp, n, box, grid, alpha, electric, d_phi, d_e, stream=None):
    b = (ctypes.c_double * 3)(*box)
    g = (ctypes.c_int32 * 3)(*grid)
    return lib.ffxg_pme_recip_permanent_noalloc(ctypes.c_void_p(d_xyz), ctypes.c_void_p(d_mp), n, b, g, alpha,
                                                electric, ctypes.c_void_p(d_phi) if d_phi else None,
                                                ctypes.c_void_p(d_e), ctypes.c_void_p(stream) if stream else None)


def _check(n_side, edge, grid, seed, user_stream):
    import torch

    s = water_box(n_side, edge, seed=seed)
    p = water_params(edge, pme_grid=grid, vdw_cutoff=9.0, ewald_cutoff=7.0, list_buffer=2.0)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.energy(s.xyz)
        ref = ffe.term("perm_recip")
        gm = ffe.get_global_multipoles()
        cphi = ffe.get_permanent_potential()[:, :10]
    lib = library()
    n = s.n_atoms
    st = torch.cuda.Stream() if user_stream else None
    handle = st.cuda_stream if st is not None else None
    d_xyz = torch.tensor(s.xyz, dtype=torch.float64, device="cuda")
    d_mp = torch.tensor(gm, dtype=torch.float64, device="cuda")
    d_phi = torch.empty((n, 10), dtype=torch.float64, device="cuda")
    d_e = torch.empty(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    scale = np.maximum(np.abs(cphi).max(axis=0), 1e-300)
    phis = []
    for _ in range(2):
        d_phi.fill_(float("nan"))
        d_e.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = _call(lib, d_xyz.data_ptr(), d_mp.data_ptr(), n, p.box, p.grid(), p.ewald_alpha, p.electric,
                   d_phi.data_ptr(), d_e.data_ptr(), handle)
        torch.cuda.synchronize()
        assert rc == 0
        e = float(d_e.item())
        assert abs(e - ref) <= E_REL * max(1.0, abs(ref)), (e, ref)
        phi = d_phi.cpu().numpy()
        err = np.abs(phi - cphi) / scale
        assert err.max() <= PHI_REL, (grid, err.max(axis=0))
        phis.append(phi)
    assert np.max(np.abs(phis[0] - phis[1]) / scale) <= 1e-12


def test_no_alloc_matches_handle_path_twice():
    _check(8, 24.8, (30, 30, 30), 31, False)


def test_no_alloc_odd_mesh():
    _check(7, 21.7, (45, 27, 35), 37, False)


def test_no_alloc_mesh_with_prime_factors_above_seven():
    _check(7, 21.7, (22, 26, 33), 39, False)     # 2 x 11, 2 x 13, 3 x 11: the general radix pass


def test_no_alloc_non_cubic_mesh_at_the_limit_on_a_user_stream():
    _check(21, 65.184, (64, 48, 60), 41, True)     # 9,261 waters: 27,783 atoms


def test_no_alloc_rejects_sizes_beyond_its_maximum():
    import torch

    lib = library()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = d.data_ptr()
    assert _call(lib, ptr, ptr, 40000, (40.0, 40.0, 40.0), (32, 32, 32), 0.545, 332.0637133, 0, ptr) == 6
    assert _call(lib, ptr, ptr, 100, (40.0, 40.0, 40.0), (80, 32, 32), 0.545, 332.0637133, 0, ptr) == 6
    assert _call(lib, ptr, ptr, 100, (40.0, 40.0, 40.0), (4, 32, 32), 0.545, 332.0637133, 0, ptr) == 1
