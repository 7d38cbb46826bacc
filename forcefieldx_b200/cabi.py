"""ctypes mirror of include/ffxcuda.h (structs, enums and function prototypes)."""
from __future__ import annotations

import ctypes
import os

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)
_L = ctypes.POINTER(ctypes.c_int64)

N_TERMS = 10
N_COUNTS = 6

STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "CUDA", 3: "SCF_DIVERGED", 4: "SCF_MAXITER",
                5: "NONFINITE", 6: "CAPACITY", 7: "RANGE"}
STATUS_RANGE = 7


class FfxgSystem(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int32),
        ("xyz", _D), ("multipole", _D), ("frame", _I), ("axis", _I),
        ("polarizability", _D), ("thole", _D), ("pdamp", _D),
        ("vdw_type", _I), ("red_parent", _I), ("red_factor", _D),
        ("n_vdw_types", ctypes.c_int32), ("vdw_inv_rmin", _D), ("vdw_eps", _D),
        ("mask12_ptr", _I), ("mask12_idx", _I),
        ("mask13_ptr", _I), ("mask13_idx", _I),
        ("mask14_ptr", _I), ("mask14_idx", _I),
        ("mask15_ptr", _I), ("mask15_idx", _I),
        ("ip11_ptr", _I), ("ip11_idx", _I),
    ]


class FfxgParams(ctypes.Structure):
    _fields_ = [
        ("box", ctypes.c_double * 3),
        ("vdw_cutoff", ctypes.c_double), ("vdw_taper", ctypes.c_double),
        ("ewald_cutoff", ctypes.c_double), ("ewald_alpha", ctypes.c_double),
        ("list_buffer", ctypes.c_double),
        ("pme_grid", ctypes.c_int32 * 3), ("pme_order", ctypes.c_int32),
        ("polar_eps", ctypes.c_double), ("max_scf_iter", ctypes.c_int32),
        ("polarization", ctypes.c_int32),
        ("precond_cutoff", ctypes.c_double), ("precond_scale", ctypes.c_double),
        ("electric", ctypes.c_double),
        ("m12", ctypes.c_double), ("m13", ctypes.c_double), ("m14", ctypes.c_double), ("m15", ctypes.c_double),
        ("p12", ctypes.c_double), ("p13", ctypes.c_double), ("p14", ctypes.c_double), ("p15", ctypes.c_double),
        ("intra14", ctypes.c_double), ("d11", ctypes.c_double),
        ("v12", ctypes.c_double), ("v13", ctypes.c_double), ("v14", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("angles", ctypes.c_double * 3),
    ]


class FfxgAlchemy(ctypes.Structure):
    _fields_ = [
        ("soft", _I), ("molecule", _I),
        ("vdw_lambda_alpha", ctypes.c_double), ("vdw_lambda_exponent", ctypes.c_double),
        ("vdw_lambda_end", ctypes.c_double),
        ("intermolecular_softcore", ctypes.c_int32), ("intramolecular_softcore", ctypes.c_int32),
        ("elec", ctypes.c_int32),
        ("permanent_lambda_alpha", ctypes.c_double), ("permanent_lambda_exponent", ctypes.c_double),
        ("permanent_lambda_start", ctypes.c_double), ("permanent_lambda_end", ctypes.c_double),
        ("polarization_lambda_start", ctypes.c_double), ("polarization_lambda_end", ctypes.c_double),
        ("polarization_lambda_exponent", ctypes.c_double),
        ("ligand_vapor_elec", ctypes.c_int32), ("no_ligand_condensed_scf", ctypes.c_int32),
    ]


class FfxgMd(ctypes.Structure):
    _fields_ = [("mass", _D), ("n_settle", ctypes.c_int32), ("settle", _I), ("settle_d1", ctypes.c_double),
                ("settle_d2", ctypes.c_double)]


# Every symbol include/ffxcuda.h declares, with its ctypes signature.
PROTOTYPES = {
    "ffxg_create": (ctypes.c_int, [ctypes.POINTER(FfxgSystem), ctypes.POINTER(FfxgParams),
                                   ctypes.POINTER(ctypes.c_void_p)]),
    "ffxg_destroy": (None, [ctypes.c_void_p]),
    "ffxg_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "ffxg_set_coordinates": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "ffxg_set_box": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _I]),
    "ffxg_update_parameters": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FfxgSystem)]),
    "ffxg_energy": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _D, _D, _L]),
    "ffxg_energy_and_gradient": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D, _L]),
    "ffxg_energy_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _D, _L]),
    "ffxg_get_induced_dipoles": (ctypes.c_int, [ctypes.c_void_p, _D, _D]),
    "ffxg_get_global_multipoles": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "ffxg_get_permanent_potential": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "ffxg_get_neighbor_pairs": (ctypes.c_int, [ctypes.c_void_p, _I, _L]),
    "ffxg_get_neighbor_images": (ctypes.c_int, [ctypes.c_void_p, _I, _L]),
    "ffxg_set_image_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ffxg_param_grad": (ctypes.c_int, [ctypes.c_void_p, _D, _D]),
    "ffxg_batch_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(FfxgSystem), ctypes.POINTER(FfxgParams),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "ffxg_batch_energy": (ctypes.c_int, [ctypes.c_void_p, _D, ctypes.c_int, _D, _D, _L, _I]),
    "ffxg_batch_set_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ffxg_batch_atoms": (ctypes.c_int64, [ctypes.c_void_p, _L]),
    "ffxg_batch_system": (ctypes.c_void_p, [ctypes.c_void_p, ctypes.c_int32]),
    "ffxg_batch_graph_builds": (ctypes.c_int64, [ctypes.c_void_p]),
    "ffxg_batch_stages": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int]),
    "ffxg_batch_tuning": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), _D]),
    "ffxg_batch_set_groups": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "ffxg_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "ffxg_batch_destroy": (None, [ctypes.c_void_p]),
    "ffxg_set_alchemy": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FfxgAlchemy)]),
    "ffxg_set_lambda": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "ffxg_get_dEdL": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D]),
    "ffxg_md_setup": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FfxgMd)]),
    "ffxg_md_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int32, _D, _D, _D, _D]),
    "ffxg_set_scf_predictor": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ffxg_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "ffxg_list_builds": (ctypes.c_int64, [ctypes.c_void_p]),
    "ffxg_last_launch_count": (ctypes.c_int64, [ctypes.c_void_p]),
    "ffxg_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ffxg_set_graph_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ffxg_get_timings": (ctypes.c_int, [ctypes.c_void_p, _D, _L, ctypes.c_int]),
    "ffxg_pme_recip_permanent_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, _D, _I,
                                                        ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                                        ctypes.c_void_p, ctypes.c_void_p]),
}

STAGE_NAMES = ["lists", "vdw", "multipoles", "perm_recip", "perm_field", "ind_recip", "ind_field",
               "precond", "pcg_vector", "real_energy", "recip_energy", "gradient"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libffxcuda.so")


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libffxcuda.so and attach prototypes.  Raises if it is missing: there is
    no CPU fallback for the product path."""
    if not os.path.exists(path):
        raise RuntimeError(f"libffxcuda.so not built at {path}; run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
