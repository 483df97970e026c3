"""ctypes binding of librspace_b200.so (the C ABI of include/rspace_b200.h).

The library is the product: every call here runs sm_100a kernels.  There is
no CPU fallback -- if the shared object is missing or cannot be loaded the
import fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librspace_b200.so")

_i = C.c_int
_l = C.c_long
_d = C.c_double
_p = C.c_void_p
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

class SolverPrm(C.Structure):
    """rs_solver_prm: kukan namelist parameters of the band solvers."""
    _fields_ = [("northo", _i), ("nsdmax", _i), ("nprecon_cg", _i), ("nprecon_diis", _i),
                ("ndiismax", _i), ("nrrz", _i), ("nchange", _i), ("ncgscf", _i),
                ("nretcg", _i), ("epssd", _d), ("eps_eig_diis", _d), ("alambda_diis", _d),
                ("alambda_min", _d), ("alambda_max", _d)]


def solver_prm(northo=1, nsdmax=4, nprecon_cg=1, nprecon_diis=1, ndiismax=4, nrrz=1,
               nchange=1, ncgscf=200, nretcg=2000, epssd=1e-6, eps_eig_diis=1e-14,
               alambda_diis=0.5, alambda_min=0.1, alambda_max=1.0) -> SolverPrm:
    """kukan's defaults (read_input_kukan8f.F90:198-249)."""
    return SolverPrm(northo, nsdmax, nprecon_cg, nprecon_diis, ndiismax, nrrz, nchange, ncgscf,
                     nretcg, epssd, eps_eig_diis, alambda_diis, alambda_min, alambda_max)


_sp = C.POINTER(SolverPrm)

# name -> argtypes (restype int unless noted)
SIGNATURES = {
    "rs_last_error": [C.c_char_p, _i],
    "rs_sphere_lists": [_i, _dp, _dp, _dp, _dp, _i, _i, _i, _d, _d, _d, _i, _i, _i, _i, _i,
                        _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip],
    "rs_geom_create": [C.POINTER(_p), _i, _i, _i, _i, _d, _d, _d, _i, _i, _i, _ip, _ip, _ip,
                       _dp],
    "rs_geom_destroy": [_p],
    "rs_vloc_soft": [_i, _dp, _dp, _i, _i, _i, _d, _d, _d, _d, _d, _d, _d, _i, _i, _i, _p, _p],
    "rs_vloc_hard_add": [_i, _dp, _ip, _i, _dp, _ip, _i, _dp, _i, _i, _i, _d, _d, _d, _d, _d, _d,
                         _i, _i, _i, _i, _d, _d, _i, _p, _p],
    "rs_ewald": [_i, _dp, _dp, _d, _d, _d, _d, _i, _i, _i, _dp, _dp, _p],
    "rs_force_local": [_i, _dp, _dp, _ip, _i, _dp, _ip, _i, _dp, _i, _i, _i, _d, _d, _d, _d, _d,
                       _d, _d, _i, _i, _i, _i, _i, _i, _i, _d, _d, _i, _p, _p, _dp, _p],
    "rs_force_adjoint_f64": [_i, _i, _i, _dp, _ip, _ip, _ip, _ip, _i, _i, _d, _dp, _ip, _ip, _ip,
                             _d, _i, _i, _i, _d, _d, _d, _p, _p, _p, _p, _p, _i, _dp, _p, _p],
    "rs_force_adjoint_f32": [_i, _i, _i, _dp, _ip, _ip, _ip, _ip, _i, _i, _d, _dp, _ip, _ip, _ip,
                             _d, _i, _i, _i, _d, _d, _d, _p, _p, _p, _p, _p, _i, _dp, _p, _p],
    "rs_initial_wave_f64": [_i, _dp, _dp, _i, _i, _i, _i, _d, _d, _d, _d, _d, _d, _p, _p],
    "rs_initial_wave_f32": [_i, _dp, _dp, _i, _i, _i, _i, _d, _d, _d, _d, _d, _d, _p, _p],
    "rs_kslaplacian_f64": [_p, _p, _p, _p, _i, _p],
    "rs_kslaplacian_f32": [_p, _p, _p, _p, _i, _p],
    "rs_nonlocal_dot_f64": [_p, _p, _i, _p, _p],
    "rs_nonlocal_dot_f32": [_p, _p, _i, _p, _p],
    "rs_nonlocal_apply_f64": [_p, _p, _p, _i, _p, _p],
    "rs_hpsi_f64": [_p, _p, _p, _p, _p, _p, _i, _p],
    "rs_hpsi_f32": [_p, _p, _p, _p, _p, _p, _i, _p],
    "rs_hpsi_f32_tuning": [_p, _ip, _ip],
    "rs_hpsi_f32_staging": [_p, _i, _i, _ip],
    "rs_spsi_f64": [_p, _p, _p, _p, _p, _i, _p],
    "rs_spsi_f32": [_p, _p, _p, _p, _p, _i, _p],
    "rs_hpsi_host_f32": [_p, _p, _p, _p, _p, _p, _i, _i, _p],
    "rs_precondition_f64": [_p, _p, _p, _i, _p],
    "rs_precondition_f32": [_p, _p, _p, _i, _p],
    "rs_density_f64": [_l, _i, _p, _p, _p, _p],
    "rs_density_f32": [_l, _i, _p, _p, _p, _p],
    "rs_interp_c2d": [_i, _i, _i, _i, _p, _p, _p],
    "rs_hartree_laplacian": [_i, _i, _i, _i, _d, _d, _d, _p, _p, _p],
    "rs_hartree_cg": [_i, _i, _i, _i, _d, _d, _d, _d, _i, _i, _i, _p, _p, _ip, _dp, _p],
    "rs_gram_f32": [_i, _i, _l, _p, _l, _p, _l, _d, _p, _l, _i, _p],
    "rs_gram_f64": [_i, _i, _l, _p, _l, _p, _l, _d, _p, _l, _p],
    "rs_rotate_f32": [_l, _i, _i, _p, _l, _p, _l, _p, _l, _p],
    "rs_rotate_f64": [_l, _i, _i, _p, _l, _p, _l, _p, _l, _p],
    "rs_syev_f64": [_i, _p, _p, _p, _ip, _p],
    "rs_chol_inv_t": [_i, _p, _p, _p],
    "rs_orthogonalize_f64": [_p, _p, _i, _p, _p, _p, _i, _p],
    "rs_orthogonalize_f32": [_p, _p, _i, _p, _p, _p, _i, _p],
    "rs_orthogonalize_band_f64": [_p, _p, _i, _i, _p, _p, _p, _i, _p],
    "rs_orthogonalize_band_f32": [_p, _p, _i, _i, _p, _p, _p, _i, _p],
    "rs_rayleighritz_f64": [_p, _p, _p, _p, _i, _p, _p, _p, _p, _i, _dp, _p],
    "rs_rayleighritz_f32": [_p, _p, _p, _p, _i, _p, _p, _p, _p, _i, _dp, _p],
    "rs_kscg_f64": [_p, _p, _p, _p, _sp, _i, _p, _p, _p, _p, _dp, _dp, _ip, _p],
    "rs_kscg_f32": [_p, _p, _p, _p, _sp, _i, _p, _p, _p, _p, _dp, _dp, _ip, _p],
    "rs_ksdiis_f64": [_p, _p, _p, _p, _sp, _i, _i, _p, _p, _p, _p, _dp, _dp, _ip, _p],
    "rs_ksdiis_f32": [_p, _p, _p, _p, _sp, _i, _i, _p, _p, _p, _p, _dp, _dp, _ip, _p],
    "rs_reorder_f64": [_p, _p, _i, _p, _p, _p, _dp, _dp, _p],
    "rs_reorder_f32": [_p, _p, _i, _p, _p, _p, _dp, _dp, _p],
    "rs_scf_diag_f64": [_p, _p, _p, _p, _sp, _i, _i, _p, _p, _p, _p, _dp, _dp, _ip, _ip, _p],
    "rs_scf_diag_f32": [_p, _p, _p, _p, _sp, _i, _i, _p, _p, _p, _p, _dp, _dp, _ip, _ip, _p],
    "rs_hartree_cg_noalloc": [_i, _i, _i, _i, _d, _d, _d, _d, _i, _i, _i, _p, _p, _ip, _dp, _p],
    "rs_interp_d2c": [_i, _i, _i, _i, _p, _p, _p],
    "rs_vxc_pz": [_l, _p, _p, _p, _p],
    "rs_veff_sum": [_l, _p, _p, _p, _p, _p, _p],
    "rs_diffcharge": [_l, _p, _p, _d, _d, _d, _d, _d, _d, _dp, _p],
    "rs_mixer_create": [C.POINTER(_p), _l, _i, _d],
    "rs_mixer_step": [_p, _p, _p, _d, _p],
    "rs_mixer_destroy": [_p],
    "rs_force_nl_f64": [_p, _p, _p, _p, _p, _p, _i, _p, _p],
    "rs_force_nl_f32": [_p, _p, _p, _p, _p, _p, _i, _p, _p],
    "rs_dot_f64": [_l, _p, _p, _p, _p],
    "rs_dot_f32": [_l, _p, _p, _p, _p],
    "rs_atomicocc": [_p, _p, _p, _i, _p, _p],
    "rs_double_grid_weights": [_i, _i, _dp],
    "rs_create": [C.POINTER(_p), _i, _i, _i, _i, _i, _d, _d, _d, _i, _p],
    "rs_upload_geometry": [_p, _i, _i, _i, _ip, _ip, _ip, _dp, _dp, _dp],
    "rs_set_potential": [_p, _dp],
    "rs_upload_bands": [_p, _p],
    "rs_orthogonalize": [_p, _i],
    "rs_hpsi": [_p],
    "rs_diag_step": [_p, _sp, _i, _dp, _dp, _ip, _ip],
    "rs_density": [_p, _dp, _dp],
    "rs_download_bands": [_p, _p],
    "rs_state_arrays": [_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p), C.POINTER(_dp),
                        C.POINTER(_p)],
    "rs_destroy": [_p],
    "rs_projector_tables": [_i, _i, _i, _i, _i, _i, _d, _d, _d, _i, _i, _i, _i, _i, _dp, _dp,
                            _dp, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _i, _i, _dp, _d,
                            _d, _d, _d, _i, _d, _dp, _dp, _p],
    "rs_hartree_cg_f32": [_i, _i, _i, _i, _d, _d, _d, _d, _i, _i, _i, _p, _p, _ip, _dp, _p],
    "rs_hpsi_batch_create": [C.POINTER(_p), _i, C.POINTER(_p), _ip],
    "rs_hpsi_batch_set_f32": [_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p), C.POINTER(_p),
                              C.POINTER(_p)],
    "rs_hpsi_batch_run_f32": [_p, _i, _p],
    "rs_hpsi_batch_info": [_p, _ip, _ip, _ip],
    "rs_hpsi_batch_set_shape": [_p, _i, _i, _i],
    "rs_hpsi_batch_destroy": [_p],
}
RESTYPES = {"rs_version": C.c_char_p, "rs_geom_entries": _l}

_lib = None


class RsError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Loads the shared object and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RsError(f"{path} is missing: build it with `python -m rspacedist_b200.build`")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _i
    for name, rt in RESTYPES.items():
        getattr(lib, name).restype = rt
    lib.rs_geom_entries.argtypes = [_p]
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().rs_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = ""):
    if rc != 0:
        raise RsError(f"{what}: status {rc}: {last_error()}")
    return rc


def call(name: str, *args):
    return check(getattr(load(), name)(*args), name)
