"""ctypes binding of the C ABI in include/zsme.h (libzsme.so).

The library is built in-tree (``csrc/Makefile`` -> ``libzsme.so`` next to this
file).  Loading fails loudly if it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libzsme.so")

ZSME_LIMITER_NONE, ZSME_LIMITER_TVD = 0, 1
ZSME_GRADIENT_GREEN_GAUSS, ZSME_GRADIENT_LSQ = 0, 1
ZSME_POSITIVITY_NONE, ZSME_POSITIVITY_ZHANG_SHU, ZSME_POSITIVITY_MOOD = 0, 1, 2
ZSME_TIME_SPLITTING, ZSME_TIME_IMEX, ZSME_TIME_IMPLICIT = 0, 1, 2
TIME_INTEGRATION = {"splitting": ZSME_TIME_SPLITTING, "imex": ZSME_TIME_IMEX, "implicit": ZSME_TIME_IMPLICIT}
POSITIVITY = {"none": ZSME_POSITIVITY_NONE, "zhang_shu": ZSME_POSITIVITY_ZHANG_SHU, "mood": ZSME_POSITIVITY_MOOD}
KERNEL_KINDS = ("begin_step", "prep", "flux", "finalize", "end_step", "gather", "finalize_fallback", "mood")


class ZsmeMesh(ct.Structure):
    _fields_ = [
        ("dim", ct.c_int32), ("n_cells", ct.c_int32), ("n_faces", ct.c_int32), ("max_faces", ct.c_int32),
        ("cell_centroid", ct.c_void_p), ("cell_volume", ct.c_void_p), ("cell_faces", ct.c_void_p),
        ("face_cells", ct.c_void_p), ("face_centroid", ct.c_void_p), ("face_normal", ct.c_void_p),
        ("face_bc", ct.c_void_p), ("cell_cfl_skip", ct.c_void_p),
    ]


class ZsmeSettings(ct.Structure):
    _fields_ = [
        ("cfl", ct.c_double), ("t_end", ct.c_double), ("min_dt", ct.c_double),
        ("reconstruction_order", ct.c_int32), ("limiter", ct.c_int32), ("gradient", ct.c_int32),
        ("ssp_stages", ct.c_int32), ("source", ct.c_int32), ("block_size", ct.c_int32),
        ("positivity", ct.c_int32), ("refresh_derivative_aux", ct.c_int32), ("time_integration", ct.c_int32),
        ("reserved", ct.c_int32 * 3),
        ("wet_dry_eps", ct.c_double),
    ]


class ZsmeDiag(ct.Structure):
    _fields_ = [
        ("steps", ct.c_int64), ("time", ct.c_double), ("dt", ct.c_double), ("n_nonfinite", ct.c_int32),
        ("n_negative_depth", ct.c_int32), ("n_newton_unconverged", ct.c_int32), ("n_mood_cells", ct.c_int32),
        ("n_newton_deferred", ct.c_int32),
    ]


def make_mesh_struct(abi: dict):
    """zsme_mesh over the arrays of Mesh.as_abi_arrays(); returns (struct,
    arrays) -- keep the tuple alive while the struct is in use."""
    keep = {k: v for k, v in abi.items() if isinstance(v, np.ndarray)}
    m = ZsmeMesh()
    m.dim, m.n_cells, m.n_faces, m.max_faces = abi["dim"], abi["n_cells"], abi["n_faces"], abi["max_faces"]
    for k in ("cell_centroid", "cell_volume", "cell_faces", "face_cells", "face_centroid", "face_normal",
              "face_bc"):
        setattr(m, k, keep[k].ctypes.data)
    if "cell_cfl_skip" in keep:
        keep["cell_cfl_skip"] = np.ascontiguousarray(keep["cell_cfl_skip"], dtype=np.uint8)
        m.cell_cfl_skip = keep["cell_cfl_skip"].ctypes.data
    return (m, keep)


_lib = None


class ZsmeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("zsme error %d: %s" % (code, msg))
        self.code = code


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libzsme.so is not built (run __graft_entry__.build() or make -C csrc): "
                          + LIB_PATH)
    lib = ct.CDLL(LIB_PATH)
    P = ct.POINTER(ct.c_double)
    vp = ct.c_void_p
    lib.zsme_version.restype = ct.c_char_p
    lib.zsme_last_error.restype = ct.c_char_p
    lib.zsme_model_name.restype = ct.c_char_p
    lib.zsme_model_name.argtypes = [ct.c_int]
    lib.zsme_model_info.argtypes = [ct.c_char_p] + [ct.POINTER(ct.c_int32)] * 4
    lib.zsme_create.argtypes = [ct.c_char_p, vp, vp, P, ct.c_int, ct.POINTER(vp)]
    lib.zsme_destroy.argtypes = [vp]
    lib.zsme_mesh_tiles.argtypes = [vp, ct.c_int32, ct.POINTER(ct.c_int32)]
    lib.zsme_set_state.argtypes = [vp, P, ct.c_double]
    lib.zsme_get_state.argtypes = [vp, P]
    lib.zsme_get_aux.argtypes = [vp, P]
    lib.zsme_set_state_device.argtypes = [vp, vp, ct.c_double]
    lib.zsme_get_state_device.argtypes = [vp, vp]
    lib.zsme_get_cells.argtypes = [vp, ct.c_int32, vp, vp, ct.c_int32]
    lib.zsme_set_cells.argtypes = [vp, ct.c_int32, vp, vp, ct.c_int32]
    lib.zsme_set_state_async.argtypes = [vp, vp, ct.c_double]
    lib.zsme_get_state_async.argtypes = [vp, vp]
    lib.zsme_stream_wait_copies.argtypes = [vp]
    lib.zsme_rhs.argtypes = [vp, ct.c_double, P, P]
    lib.zsme_implicit_function.argtypes = [vp, ct.c_double, P, P, P]
    lib.zsme_implicit_jacobian.argtypes = [vp, ct.c_double, P, ct.c_double, P, P]
    lib.zsme_implicit_stats.argtypes = [vp, ct.POINTER(ct.c_int32)]
    lib.zsme_update_state.argtypes = [vp]
    lib.zsme_source.argtypes = [vp, ct.c_double]
    lib.zsme_compute_dt.argtypes = [vp, P]
    lib.zsme_step.argtypes = [vp, ct.c_int32]
    lib.zsme_step_dt.argtypes = [vp, ct.c_int32, P]
    lib.zsme_step_dt_device.argtypes = [vp, ct.c_int32, vp]
    lib.zsme_get_time_device.argtypes = [vp, vp, vp]
    lib.zsme_sync.argtypes = [vp]
    lib.zsme_get_diag.argtypes = [vp, ct.POINTER(ZsmeDiag)]
    lib.zsme_get_time.argtypes = [vp, P, P]
    lib.zsme_set_params.argtypes = [vp, P]
    lib.zsme_stream.argtypes = [vp]
    lib.zsme_stream.restype = vp
    lib.zsme_device.argtypes = [vp, ct.POINTER(ct.c_int32)]
    lib.zsme_launches_per_step.argtypes = [vp, ct.POINTER(ct.c_int32)]
    lib.zsme_set_profiling.argtypes = [vp, ct.c_int]
    lib.zsme_read_profile.argtypes = [vp, P, ct.POINTER(ct.c_int64)]
    lib.zsme_compute_dt_noalloc.argtypes = [ct.c_char_p, ct.c_int32, vp, vp, vp, vp, ct.c_double, vp, vp]
    lib.zsme_fp64_fma_peak.argtypes = [ct.c_int, P]
    lib.zsme_batch_create.argtypes = [ct.c_char_p, ct.c_int32, vp, vp, P, ct.c_int, ct.POINTER(vp)]
    lib.zsme_batch_size.argtypes = [vp, ct.POINTER(ct.c_int32)]
    lib.zsme_batch_set_state.argtypes = [vp, ct.c_int32, P, ct.c_double]
    lib.zsme_batch_get_state.argtypes = [vp, ct.c_int32, P]
    lib.zsme_batch_get_time.argtypes = [vp, ct.c_int32, P, P]
    lib.zsme_set_launch.argtypes = [vp, ct.POINTER(ct.c_int32)]
    lib.zsme_get_launch.argtypes = [vp, ct.POINTER(ct.c_int32)]
    I32 = ct.POINTER(ct.c_int32)
    lib.zsme_adjoint.argtypes = [vp, ct.c_int32, ct.c_int32, ct.c_int32, I32, I32, I32, P, P, P, P, P, P]
    lib.zsme_adjoint_phases.argtypes = [vp, P]
    lib.zsme_adjoint_overlapped.argtypes = [vp, I32]
    _lib = lib
    return lib


def check(rc):
    if rc != 0:
        raise ZsmeError(rc, load().zsme_last_error().decode())


def mesh_tiles(mesh, tile_faces: int) -> dict:
    """The fused face + gather kernel's tiling of `mesh` (a mesh.Mesh) at
    tile_faces, computed on the host (zsme_mesh_tiles)."""
    lib = load()
    m, keep = make_mesh_struct(mesh.as_abi_arrays())
    st = (ct.c_int32 * 5)()
    check(lib.zsme_mesh_tiles(ct.byref(m), int(tile_faces), st))
    return dict(tiles=st[0], max_faces=st[1], incoming=st[2], covered=st[3], flux_slots=st[4])


def model_names():
    lib = load()
    return [lib.zsme_model_name(i).decode() for i in range(lib.zsme_num_models())]


def model_info(model: str):
    lib = load()
    v = [ct.c_int32() for _ in range(4)]
    check(lib.zsme_model_info(model.encode(), *[ct.byref(x) for x in v]))
    return dict(n_dof_q=v[0].value, n_dof_qaux=v[1].value, n_parameters=v[2].value, dimension=v[3].value)
