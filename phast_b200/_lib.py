"""ctypes binding of the C ABI in ``include/phastb.h`` (``phast_b200/_lib/libphastb.so``).

The library is the product: every operator and solver in this package calls it.
There is no CPU or PyTorch fallback -- if the library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libphastb.so")

OK, ERR_ARG, ERR_CUDA, NONCONVERGED, DIVERGED, BREAKDOWN, NONFINITE, ERR_WORKSPACE, UNSUPPORTED, ERR_CAPACITY = range(10)
F64, F32 = 0, 1
SPLITS = {"linear": 0, "isotropic": 1, "amor": 2, "spectral": 3, "star_convex": 4, "spectral_stress": 5}
DRIVER_NONE, DRIVER_FULL, DRIVER_SPECTRAL = 0, 1, 2
MAX_SLOTS = 8

vp, ip, dp, sz = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t
fp = C.POINTER(C.c_float)


class Q4Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("hx", C.c_double), ("hy", C.c_double)]


class Q4Material(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("lam", C.c_double), ("mu", C.c_double),
                ("kappa", C.c_double), ("eta", C.c_double), ("spectral_eps", C.c_double),
                ("plane_stress", C.c_int), ("stress_split", C.c_int), ("psi_split", C.c_int)]


class VoxelGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("px", C.c_int), ("py", C.c_int),
                ("pz", C.c_int), ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double)]


class VoxelMaterial(C.Structure):
    _fields_ = [("n_slots", C.c_int), ("isotropic", C.c_int), ("C", (C.c_double * 36) * MAX_SLOTS),
                ("lam", C.c_double * MAX_SLOTS), ("mu", C.c_double * MAX_SLOTS), ("Gc", C.c_double * MAX_SLOTS),
                ("driver", C.c_int * MAX_SLOTS), ("kappa", C.c_double), ("ell", C.c_double)]


class PfczmLaw(C.Structure):
    _fields_ = [("a1", C.c_double * MAX_SLOTS), ("a2", C.c_double), ("a3", C.c_double), ("p", C.c_double)]


class MechOpts(C.Structure):
    _fields_ = [("precond", C.c_int), ("mixed", C.c_int), ("levels", C.c_int), ("smooth_degree", C.c_int),
                ("coarse_degree", C.c_int), ("power_iters", C.c_int), ("lmax_safety", C.c_double),
                ("inner_rtol", C.c_double),
                ("max_refine", C.c_int)]


class T3Mesh(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("n_elems", C.c_int), ("n_colors", C.c_int), ("reserved", C.c_int),
                ("elem", C.c_void_p), ("order", C.c_void_p), ("color_off", C.POINTER(C.c_int)),
                ("grad", C.c_void_p), ("areas", C.c_void_p)]


class T3DamageModel(C.Structure):
    _fields_ = [("nodal_h", C.c_int), ("reserved", C.c_int), ("gcl0", C.c_double), ("gc_over_l0", C.c_double),
                ("source", C.c_double), ("gcl0_e", C.c_void_p), ("gc_over_l0_e", C.c_void_p),
                ("source_e", C.c_void_p)]


Q4G, Q4M, VG, VM = C.POINTER(Q4Grid), C.POINTER(Q4Material), C.POINTER(VoxelGrid), C.POINTER(VoxelMaterial)
T3DM = C.POINTER(T3DamageModel)
T3M = C.POINTER(T3Mesh)
MO = C.POINTER(MechOpts)
PL = C.POINTER(PfczmLaw)

# name -> (restype, argtypes)
SIGNATURES = {
    "phastb_version": (C.c_char_p, []),
    "phastb_launch_count": (C.c_longlong, []),
    "phastb_launch_count_reset": (None, []),
    "phastb_reduce_workspace_bytes": (sz, []),
    "phastb_q4_strain": (C.c_int, [Q4G, C.c_int, vp, vp, vp, vp, vp]),
    "phastb_q4_internal_force": (C.c_int, [Q4G, Q4M, C.c_int, vp, vp, vp, vp]),
    "phastb_q4_stiffness_diagonal": (C.c_int, [Q4G, Q4M, C.c_int, vp, vp, vp]),
    "phastb_q4_psi_grad_t": (C.c_int, [Q4G, Q4M, vp, vp, vp, vp]),
    "phastb_q4_force_dd_t": (C.c_int, [Q4G, Q4M, vp, vp, vp, vp, vp]),
    "phastb_q4_psi_history": (C.c_int, [Q4G, Q4M, C.c_int, vp, vp, vp, vp, vp]),
    "phastb_q4_damage_apply": (C.c_int, [Q4G, vp, vp, C.c_double, C.c_double, vp, C.c_double, vp, vp, vp]),
    "phastb_q4_damage_prepare": (C.c_int, [Q4G, vp, C.c_double, vp, C.c_double, vp, vp, vp, vp]),
    "phastb_q4_damage_solve_workspace_bytes": (sz, [C.c_int]),
    "phastb_q4_damage_solve": (C.c_int, [Q4G, vp, C.c_double, vp, C.c_double, vp, vp, vp, vp, vp, C.c_double,
                                         C.c_int, C.c_int, vp, ip, vp, sz, vp]),
    "phastb_q4_damage_linear_workspace_bytes": (C.c_size_t, [C.c_int]),
    "phastb_q4_damage_linear_solve": (C.c_int, [Q4G, vp, C.c_double, vp, C.c_double, vp, vp, vp, vp, vp, C.c_double,
                                                C.c_int, C.c_int, vp, ip, dp, vp, sz, vp]),
    "phastb_q4_damage_adjoint_grads": (C.c_int, [Q4G, vp, vp, C.c_double, vp, vp, vp, vp, vp]),
    "phastb_q4_explicit_adjoint_step": (C.c_int, [Q4G, Q4M, C.c_double, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                                  vp, vp, vp]),
    "phastb_t3_internal_force": (C.c_int, [T3M, Q4M, vp, vp, vp, vp]),
    "phastb_t3_psi_history": (C.c_int, [T3M, Q4M, vp, vp, vp, vp, vp]),
    "phastb_t3_damage_apply": (C.c_int, [T3M, vp, vp, C.c_double, vp, C.c_double, vp, vp, vp]),
    "phastb_t3_damage_prepare": (C.c_int, [T3M, vp, C.c_double, vp, C.c_double, vp, vp, vp, vp]),
    "phastb_t3_damage_solve_workspace_bytes": (C.c_size_t, [C.c_int]),
    "phastb_t3_damage_solve": (C.c_int, [T3M, vp, C.c_double, vp, C.c_double, vp, vp, vp, vp, vp, C.c_double, C.c_int,
                                         C.c_int, vp, ip, vp, sz, vp]),
    "phastb_t3_psi_grad_t": (C.c_int, [T3M, Q4M, vp, vp, vp, vp]),
    "phastb_t3_force_dd_t": (C.c_int, [T3M, Q4M, vp, vp, vp, vp, vp]),
    "phastb_t3_damage_adjoint_grads": (C.c_int, [T3M, vp, vp, C.c_double, vp, vp, vp, vp, vp]),
    "phastb_t3_damage_linear_workspace_bytes": (C.c_size_t, [C.c_int]),
    "phastb_t3_damage_linear_solve": (C.c_int, [T3M, vp, C.c_double, vp, C.c_double, vp, vp, vp, vp, vp, C.c_double,
                                                C.c_int, C.c_int, vp, ip, dp, vp, sz, vp]),
    "phastb_t3_qs_workspace_bytes": (sz, [C.c_int]),
    "phastb_t3_qs_solve": (C.c_int, [T3M, Q4M, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.c_double, C.c_double, ip, vp, sz, vp]),
    "phastb_q4_explicit_step": (C.c_int, [Q4G, Q4M, C.c_int, C.c_double, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                          vp, vp, vp, vp]),
    "phastb_q4_tangent_apply": (C.c_int, [Q4G, Q4M, vp, vp, vp, vp, vp]),
    "phastb_q4_energy_sums": (C.c_int, [Q4G, Q4M, vp, vp, vp, dp, vp, sz, vp]),
    "phastb_q4_reaction_workspace_bytes": (sz, [C.c_int]),
    "phastb_q4_reaction": (C.c_int, [Q4G, Q4M, vp, vp, vp, C.c_int, C.c_int, vp, dp, vp, sz, vp]),
    "phastb_q4_qs_workspace_bytes": (sz, [C.c_int]),
    "phastb_q4_qs_solve": (C.c_int, [Q4G, Q4M, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.c_double, C.c_double, ip, vp, sz, vp]),
    "phastb_h8_scratch_bytes": (sz, [VG, C.c_int]),
    "phastb_h8_degradation": (C.c_int, [VG, C.c_int, vp, C.c_double, vp, vp]),
    "phastb_h8_mech_apply": (C.c_int, [VG, VM, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]),
    "phastb_h8_mech_apply_noalloc": (C.c_int, [VG, VM, vp, C.c_int, vp, vp, vp, vp, vp, vp]),
    "phastb_h8_tile_shape": (C.c_int, [VG, C.c_int, C.c_int, ip]),
    "phastb_h8_autotune": (C.c_int, [VG, VM, C.c_int, vp, vp, vp, vp, vp, sz, ip, fp, vp]),
    "phastb_h8_mech_diagonal": (C.c_int, [VG, VM, vp, C.c_int, vp, vp, vp, vp, vp]),
    "phastb_h8_stress_energy": (C.c_int, [VG, VM, vp, vp, vp, vp, dp, dp, vp, vp]),
    "phastb_h8_driving_history": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, vp]),
    "phastb_h8_damage_apply": (C.c_int, [VG, VM, vp, vp, vp, C.c_double, vp, vp, vp]),
    "phastb_h8_damage_rhs_diag": (C.c_int, [VG, VM, vp, vp, C.c_double, vp, vp, vp, vp]),
    "phastb_h8_mech_solve_workspace_bytes": (sz, [VG, C.c_int]),
    "phastb_h8_mech_solve": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int,
                                       vp, ip, dp, vp, sz, vp]),
    "phastb_h8_mech_solve_ex_workspace_bytes": (sz, [VG, MO]),
    "phastb_h8_mech_solve_ex": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int, MO,
                                          dp, vp, ip, dp, vp, sz, vp]),
    "phastb_h8_mech_solve_ex_g_workspace_bytes": (sz, [VG, MO]),
    "phastb_h8_mech_solve_ex_g": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int,
                                            MO, dp, vp, ip, dp, vp, sz, vp]),
    "phastb_h8_box_kkt_workspace_bytes": (sz, [VG]),
    "phastb_h8_damage_box_kkt": (C.c_int, [VG, VM, vp, vp, C.c_double, vp, C.c_double, vp, C.c_double, C.c_double,
                                           C.c_int, C.c_int, vp, ip, vp, sz, vp]),
    "phastb_h8_stagger_change": (C.c_int, [C.c_int, vp, vp, C.c_int, vp, vp, dp, vp, sz, vp]),
    "phastb_h8_record_workspace_bytes": (sz, [VG]),
    "phastb_h8_increment_record": (C.c_int, [VG, VM, vp, vp, vp, vp, C.c_double, dp, vp, sz, vp]),
    "phastb_h8_increment_record_ex": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, C.c_double, PL, dp, vp, sz, vp]),
    "phastb_t3_tangent_apply": (C.c_int, [T3M, Q4M, vp, vp, vp, vp, vp]),
    "phastb_anderson_workspace_bytes": (sz, [C.c_int]),
    "phastb_anderson_step": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, vp, ip, vp,
                                       sz, vp]),
    "phastb_anderson_projected": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, C.c_double,
                                            C.c_double, vp, ip, vp, sz, vp]),
    "phastb_h8_closure_workspace_bytes": (sz, [VG]),
    "phastb_h8_closure_pattern": (C.c_int, [VG, VM, vp, vp, vp, vp]),
    "phastb_h8_closure_pattern_change": (C.c_int, [VG, VM, vp, vp, vp, vp, C.c_double, vp, ip, vp, sz, vp]),
    "phastb_h8_closure_apply_add": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "phastb_h8_closure_diagonal_add": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, sz, vp]),
    "phastb_h8_closure_energy": (C.c_int, [VG, VM, vp, vp, vp, vp, dp, vp, sz, vp]),
    "phastb_h8_kinematic_guard": (C.c_int, [VG, vp, vp, C.c_double, dp, vp, sz, vp]),
    "phastb_h8_mech_solve_closure_workspace_bytes": (sz, [VG]),
    "phastb_h8_mech_solve_closure": (C.c_int, [VG, VM, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int,
                                               C.c_int, vp, ip, dp, vp, sz, vp]),
    "phastb_h8_pfczm_degradation": (C.c_int, [VG, VM, PL, vp, vp, vp, vp]),
    "phastb_h8_pfczm_workspace_bytes": (sz, [VG]),
    "phastb_h8_pfczm_energy": (C.c_int, [VG, VM, PL, vp, vp, vp, dp, vp, sz, vp]),
    "phastb_h8_pfczm_gradient": (C.c_int, [VG, VM, PL, vp, vp, vp, C.c_double, vp, vp, sz, vp]),
    "phastb_h8_pfczm_tangent_weights": (C.c_int, [VG, VM, PL, vp, vp, vp, vp, vp]),
    "phastb_h8_pfczm_tangent_apply": (C.c_int, [VG, VM, vp, vp, vp, C.c_double, vp, vp, sz, vp]),
    "phastb_h8_pfczm_tangent_diagonal": (C.c_int, [VG, VM, vp, vp, C.c_double, vp, vp, sz, vp]),
    "phastb_h8_pfczm_solve_workspace_bytes": (sz, [VG]),
    "phastb_h8_pfczm_damage_solve": (C.c_int, [VG, VM, PL, vp, vp, C.c_double, vp, vp, C.c_double, C.c_double,
                                               C.c_int, C.c_int, C.c_int, vp, ip, dp, vp, sz, vp]),
    "phastb_h8_damage_residual_workspace_bytes": (sz, [VG]),
    "phastb_h8_damage_residual_norm": (C.c_int, [VG, VM, vp, vp, C.c_double, vp, dp, vp, sz, vp]),
    "phastb_scale_set": (C.c_int, [C.c_int, vp, C.c_double, C.c_int, C.c_double, vp, vp]),
    "phastb_test_grid_barrier": (C.c_int, [C.c_int, C.c_int, C.c_double, ip, ip]),
    "phastb_h8_tma_staging": (C.c_int, [VG, C.c_int]),
    "phastb_batch_create": (vp, [C.c_int, VG, dp, dp, C.c_int, C.c_int, C.c_int]),
    "phastb_batch_destroy": (None, [vp]),
    "phastb_batch_sizes": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
    "phastb_batch_bind": (C.c_int, [vp, vp, sz, vp]),
    "phastb_batch_apply_workspace_bytes": (sz, [vp]),
    "phastb_batch_mech_apply": (C.c_int, [vp, VM, vp, C.c_int, vp, vp, vp, vp, dp, vp, sz, vp]),
    "phastb_batch_damage_apply": (C.c_int, [vp, VM, vp, vp, vp, C.c_int, vp, vp, vp, sz, vp]),
    "phastb_batch_mech_solve_workspace_bytes": (sz, [vp, C.c_int]),
    "phastb_batch_mech_solve": (C.c_int, [vp, VM, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int,
                                          C.c_int, C.c_double, C.c_int, ip, vp, ip, dp, vp, sz, vp]),
    "phastb_batch_mech_solve_ex_workspace_bytes": (sz, [vp, MO]),
    "phastb_batch_mech_solve_ex": (C.c_int, [vp, VM, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int,
                                             MO, C.c_int, ip, vp, ip, dp, vp, sz, vp]),
    "phastb_batch_box_kkt_workspace_bytes": (sz, [vp]),
    "phastb_batch_damage_box_kkt": (C.c_int, [vp, VM, vp, vp, vp, C.c_double, vp, C.c_double, C.c_double,
                                              C.c_double, C.c_int, C.c_int, C.c_int, ip, vp, ip, dp, vp, sz, vp]),
    "phastb_batch_predictor": (C.c_int, [vp, vp, C.c_double, C.c_int, C.c_double, vp, vp, vp]),
    "phastb_t3_damage_apply_ex": (C.c_int, [T3M, T3DM, vp, vp, vp, vp]),
    "phastb_t3_damage_prepare_ex": (C.c_int, [T3M, T3DM, vp, vp, vp, vp]),
    "phastb_t3_damage_solve_ex": (C.c_int, [T3M, T3DM, vp, vp, vp, vp, vp, C.c_double, C.c_int, C.c_int, vp, ip,
                                            vp, sz, vp]),
    "phastb_t3_check_mesh": (C.c_int, [C.c_int, C.c_int, ip, ip, C.c_int, ip]),
    "phastb_batch_change_workspace_bytes": (sz, [vp]),
    "phastb_batch_stagger_change": (C.c_int, [vp, vp, vp, vp, vp, dp, vp, sz, vp]),
}
RECORD_WORDS = 27
PFCZM_ENERGY_WORDS = 4 + MAX_SLOTS

_lock = threading.Lock()
_lib = None


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"phast_b200 CUDA library not found at {LIB_PATH}; build it with "
                    "`python -m phast_b200.build` (needs nvcc)")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


class PhastbError(RuntimeError):
    def __init__(self, fn, status):
        super().__init__(f"{fn} failed with status {status}")
        self.status = status


def check(status, fn):
    """Map a C-ABI status to PhAST's exception contract."""
    if status == OK:
        return
    if status == ERR_ARG:
        raise ValueError(f"{fn}: invalid argument")
    if status == UNSUPPORTED:
        raise NotImplementedError(f"{fn}: option not implemented by the B200 backend")
    raise PhastbError(fn, status)


def call(name, *args):
    """Call an entry point and raise on any non-OK status."""
    st = getattr(load(), name)(*args)
    check(st, name)
    return st


def raw(name, *args):
    """Call an entry point and return its status (solvers report convergence this way)."""
    return getattr(load(), name)(*args)


def ptr(t):
    """Device pointer of a contiguous tensor (or None)."""
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("phast_b200 kernels need contiguous tensors")
    if t.data_ptr() % 16:
        raise ValueError("phast_b200 kernels need 16-byte aligned tensors (vectorised loads)")
    return C.c_void_p(t.data_ptr())


def stream(device=None):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(t, name="tensor"):
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise ValueError(f"{name} must be a CUDA tensor: the B200 backend has no CPU path")


class Workspace:
    """Grow-only device scratch buffer reused across calls (caller-owned memory for the C ABI)."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.buf = None

    def get(self, nbytes):
        nbytes = int(nbytes)
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        return C.c_void_p(self.buf.data_ptr()), C.c_size_t(self.buf.numel())
