"""ctypes binding of libjxb (the C ABI declared in include/jxb.h).

The library is built in-tree by `jaxley_pytorch_b200/build.py` (nvcc, sm_100a). It
is the only compute path of this package: if it is missing, every entry point raises
instead of falling back to another implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libjxb.so")

JXB_OK = 0
JXB_NONFINITE = 1  # bit of JxbSimArgs.status: a launch produced a value that is not finite
JXB_TIMEOUT = 2  # bit of JxbSimArgs.status: a bounded wait of a launch gave up
F32, F64 = 0, 1
SCHEME_BWD_EULER, SCHEME_CN = 0, 1  # JxbSimArgs.scheme

_p = C.c_void_p
_i32p = C.c_void_p


class JxbTreeSchedule(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int32), ("n_blocks", C.c_int32), ("max_block_nodes", C.c_int32),
        ("max_levels", C.c_int32),
        ("block_info", _p), ("block_levels", _p), ("perm", _p), ("chain_top", _p),
        ("chain_len", _p), ("chain_ptop", _p), ("chain_cptr", _p), ("chain_child", _p),
        ("level_ptr", _p),
    ]


class JxbRegSchedule(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int32), ("n_blocks", C.c_int32), ("regs_per_lane", C.c_int32),
        ("num_slots", C.c_int32),
        ("block_info", _p), ("rel_parent", _p), ("rel_height", _p), ("rel_depth", _p),
        ("rel_children", _p),
    ]


class JxbSimArgs(C.Structure):
    _fields_ = [
        ("dtype", C.c_int32), ("batch", C.c_int32),
        ("n_nodes", C.c_int32), ("n_slots", C.c_int32), ("n_pslots", C.c_int32), ("n_cols", C.c_int32),
        ("n_items", C.c_int32), ("n_steps", C.c_int32),
        ("t0", C.c_int32), ("max_rows", C.c_int32),
        ("max_nodes", C.c_int32), ("max_slots", C.c_int32),
        ("max_chains", C.c_int32), ("max_child", C.c_int32),
        ("max_levels", C.c_int32), ("max_pslots", C.c_int32),
        ("threads", C.c_int32), ("pad3", C.c_int32),
        ("dt", C.c_double),
        ("node_class", _p), ("soff", _p), ("poff", _p),
        ("a_low", _p), ("a_up", _p), ("gsum", _p), ("cm", _p),
        ("cls_ptr", _p), ("cls_comp", _p), ("cls_prog", _p), ("entries", _p),
        ("n_classes", C.c_int32), ("n_entries", C.c_int32),
        ("pbase", _p), ("pcol", _p), ("pscale", _p),
        ("blocks", _p), ("items", _p),
        ("chain_top", _p), ("chain_len", _p), ("chain_ptop", _p), ("chain_cptr", _p),
        ("chain_child", _p), ("level_ptr", _p),
        ("gk", _p), ("gbase", _p), ("max_gslots", C.c_int32), ("wide", C.c_int32),
        ("parent", _p), ("kid_ptr", _p), ("kid", _p),
        ("stim_ptr", _p), ("stim_idx", _p), ("area", _p), ("stim", _p),
        ("n_stim", C.c_int32), ("stim_steps", C.c_int32), ("stim_rows", C.c_int32), ("pad0", C.c_int32),
        ("syn_lin", _p), ("syn_const", _p),
        ("rec_ptr", _p), ("rec_slot", _p), ("rec_col", _p), ("rec_out", _p),
        ("n_rec", C.c_int32), ("pad1", C.c_int32),
        ("state", _p), ("ckpt", _p),
        ("ckpt_every", C.c_int32), ("ckpt_base", C.c_int32),
        ("traj", _p), ("traj_piv", _p),
        ("adj", _p), ("rec_grad", _p), ("pgrad", _p),
        ("mode", C.c_int32), ("traj_stored", C.c_int32),
        ("gscratch", _p), ("gscratch_stride", C.c_int64),
        ("sched_ptr", _p), ("sched", _p), ("sched_warps", C.c_int32), ("pad5", C.c_int32),
        ("gacc", _p), ("gacc_stride", C.c_int64),
        ("multi", _p), ("multi_items", _p),
        ("syn_ptr", _p), ("syn_off", _p), ("syn_rs", _p), ("g_syn_lin", _p), ("g_syn_const", _p),
        ("clamp_ptr", _p), ("clamp_slot", _p), ("clamp_col", _p), ("clamp", _p),
        ("n_clamp", C.c_int32), ("clamp_steps", C.c_int32), ("clamp_rows", C.c_int32), ("pad6", C.c_int32),
        ("status", _p), ("scheme", C.c_int32), ("pad7", C.c_int32),
    ]


class JxbSynArgs(C.Structure):
    _fields_ = [
        ("dtype", C.c_int32), ("model", C.c_int32),
        ("batch", C.c_int32), ("n_nodes", C.c_int32), ("n_syn", C.c_int32), ("k", C.c_int32),
        ("targets_are_nodes", C.c_int32), ("store_current", C.c_int32),
        ("v", _p), ("s", _p), ("pre", _p), ("targets", _p),
        ("p", _p * 6), ("area", _p), ("scalars", _p),
        ("s_new", _p), ("current", _p), ("lin", _p), ("cst", _p),
        ("g_s_new", _p), ("g_current", _p), ("g_lin", _p), ("g_const", _p),
        ("g_s", _p), ("g_v", _p), ("g_params", _p), ("g_pre", _p), ("g_post", _p),
        ("need", C.c_int32), ("inv_width", C.c_int32), ("n_pre_nodes", C.c_int32), ("accumulate", C.c_int32),
        ("inv", _p), ("pre_nodes", _p),
    ]


EXPORTED = [
    "jxb_tree_solve_levels",
    "jxb_tree_solve_registers",
    "jxb_sim_forward",
    "jxb_sim_backward",
    "jxb_sim_backward_noalloc",
    "jxb_sim_smem_bytes",
    "jxb_sim_tangent",
    "jxb_sim_tangent_smem_bytes",
    "jxb_sim_forward_multi",
    "jxb_sim_backward_multi",
    "jxb_sim_multi_scratch_bytes",
    "jxb_synapse_forward",
    "jxb_synapse_backward",
    "jxb_last_error",
    "jxb_version",
]

_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libjxb (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libjxb is not built ({path} is missing): run `python -m jaxley_pytorch_b200.build`"
        )
    lib = C.CDLL(path)
    lib.jxb_last_error.restype = C.c_char_p
    lib.jxb_version.restype = C.c_int
    lib.jxb_sim_smem_bytes.restype = C.c_int64
    lib.jxb_sim_smem_bytes.argtypes = [C.POINTER(JxbSimArgs), C.c_int]
    lib.jxb_sim_tangent_smem_bytes.restype = C.c_int64
    lib.jxb_sim_tangent_smem_bytes.argtypes = [C.POINTER(JxbSimArgs)]
    for name in ["jxb_sim_forward", "jxb_sim_backward", "jxb_sim_backward_noalloc", "jxb_sim_tangent"]:
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = [C.POINTER(JxbSimArgs), C.c_void_p]
    for name in ["jxb_sim_forward_multi", "jxb_sim_backward_multi"]:
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = [C.POINTER(JxbSimArgs), C.POINTER(JxbSimArgs), C.c_int, _p, C.c_int, _p,
                       C.c_int64, C.c_void_p]
    lib.jxb_sim_multi_scratch_bytes.restype = C.c_int64
    lib.jxb_sim_multi_scratch_bytes.argtypes = [C.c_int, C.c_int]
    for name in ["jxb_synapse_forward", "jxb_synapse_backward"]:
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = [C.POINTER(JxbSynArgs), C.c_void_p]
    lib.jxb_tree_solve_levels.restype = C.c_int
    lib.jxb_tree_solve_levels.argtypes = [C.c_int, _p, _p, _p, _p, _p, C.c_int64,
                                          C.POINTER(JxbTreeSchedule), C.c_void_p]
    lib.jxb_tree_solve_registers.restype = C.c_int
    lib.jxb_tree_solve_registers.argtypes = [C.c_int, _p, _p, _p, _p, _p, C.c_int64,
                                             C.POINTER(JxbRegSchedule), C.c_void_p]
    _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != JXB_OK:
        msg = load().jxb_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed with status {rc}: {msg}")
