"""ctypes binding of the CUDA library ``libmhs_b200.so`` (the C ABI in
``include/mhs_b200.h``).  The library is built in-tree by ``build.py``; if it
is missing the package refuses to run rather than falling back to anything
else."""
from __future__ import annotations

import ctypes
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().with_name("libmhs_b200.so")

# enum mhs_kind
DISP, STRESS, TOTAL_STRESS, EIGENSTRESS, STRAIN, TRACTION, INTERACTION = range(7)
# enum mhs_precision
FP64, MIXED = 0, 1
# device status bits
DEV_FOLD_GRID_OVERFLOW = 1


class Request(ctypes.Structure):
    """Mirror of ``struct mhs_request``."""

    _fields_ = [
        ("kind", ctypes.c_int),
        ("order", ctypes.c_int),
        ("fold", ctypes.c_int),
        ("subtract_eigenstress", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("out_f32", ctypes.c_int),
        ("n_obs", ctypes.c_int64),
        ("n_src", ctypes.c_int64),
        ("obs", ctypes.c_void_p),
        ("tris", ctypes.c_void_p),
        ("eps", ctypes.c_void_p),
        ("mu", ctypes.c_double),
        ("lam", ctypes.c_double),
        ("normals", ctypes.c_void_p),
        ("rec_basis", ctypes.c_void_p),
        ("src_basis", ctypes.c_void_p),
        ("n_a", ctypes.c_int),
        ("n_b", ctypes.c_int),
        ("ids", ctypes.c_void_p),
        ("n_cols", ctypes.c_int64),
        ("col_ptr", ctypes.c_void_p),
        ("col_ent", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t),
        ("slip", ctypes.c_void_p),
    ]


class Tune(ctypes.Structure):
    """Mirror of ``struct mhs_tune``."""

    _fields_ = [("pair_tb", ctypes.c_int), ("final_tb", ctypes.c_int),
                ("far_mult", ctypes.c_int), ("near_mult", ctypes.c_int)]


#: Symbols the header declares; a test checks the library exports each.
EXPORTS = ("mhs_workspace_bytes", "mhs_assemble", "mhs_read_status", "mhs_column_plan",
           "mhs_last_error", "mhs_version", "mhs_profile_enable", "mhs_profile_read",
           "mhs_fp_peak", "mhs_debug_terms", "mhs_assemble_noalloc", "mhs_census_enable",
           "mhs_census_read", "mhs_kernel_count", "mhs_batch_create", "mhs_batch_workspace_bytes",
           "mhs_batch_bind", "mhs_submit_batch", "mhs_poll", "mhs_batch_destroy", "mhs_autotune",
           "mhs_set_tune", "mhs_get_tune", "mhs_batch_pass_bytes", "mhs_fullspace_influence")

class FullspaceRequest(ctypes.Structure):
    """struct mhs_fullspace_request (include/mhs_b200.h)."""
    _fields_ = [("order", ctypes.c_int), ("want", ctypes.c_int), ("far_field", ctypes.c_int),
                ("pad", ctypes.c_int), ("n_obs", ctypes.c_int64), ("obs", ctypes.c_void_p),
                ("tri", ctypes.c_double * 9), ("mu", ctypes.c_double), ("nu", ctypes.c_double),
                ("eps", ctypes.c_double), ("U", ctypes.c_void_p), ("H", ctypes.c_void_p),
                ("E", ctypes.c_void_p), ("G", ctypes.c_void_p), ("S", ctypes.c_void_p)]


_lib = None


def load() -> ctypes.CDLL:
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH.name} is not built: run `python -c \"import __graft_entry__ as g; "
            f"g.build()\"` (or mhs_b200.build.build()) first. There is no CPU fallback.")
    lib = ctypes.CDLL(str(LIB_PATH))
    R = ctypes.POINTER(Request)
    lib.mhs_workspace_bytes.argtypes = [R, ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_size_t)]
    lib.mhs_workspace_bytes.restype = ctypes.c_int
    lib.mhs_assemble.argtypes = [R, ctypes.c_void_p]
    lib.mhs_assemble.restype = ctypes.c_int
    lib.mhs_read_status.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    lib.mhs_read_status.restype = ctypes.c_int
    lib.mhs_column_plan.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.mhs_column_plan.restype = ctypes.c_int
    lib.mhs_last_error.argtypes = []
    lib.mhs_last_error.restype = ctypes.c_char_p
    lib.mhs_version.argtypes = []
    lib.mhs_version.restype = ctypes.c_char_p
    lib.mhs_profile_enable.argtypes = [ctypes.c_int]
    lib.mhs_profile_enable.restype = ctypes.c_int
    lib.mhs_profile_read.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    lib.mhs_profile_read.restype = ctypes.c_int
    lib.mhs_fp_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                ctypes.c_void_p]
    lib.mhs_fp_peak.restype = ctypes.c_int
    lib.mhs_debug_terms.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.mhs_debug_terms.restype = ctypes.c_int
    lib.mhs_census_enable.argtypes = [ctypes.c_int]
    lib.mhs_census_enable.restype = ctypes.c_int
    lib.mhs_census_read.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
    lib.mhs_census_read.restype = ctypes.c_int
    lib.mhs_kernel_count.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
    lib.mhs_kernel_count.restype = ctypes.c_int
    V = ctypes.c_void_p
    lib.mhs_batch_create.argtypes = [R, ctypes.c_int, ctypes.POINTER(V)]
    lib.mhs_batch_workspace_bytes.argtypes = [V, ctypes.POINTER(ctypes.c_size_t)]
    lib.mhs_batch_bind.argtypes = [V, V, ctypes.c_size_t, V]
    lib.mhs_submit_batch.argtypes = [V, V]
    lib.mhs_poll.argtypes = [V, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.mhs_batch_destroy.argtypes = [V]
    lib.mhs_batch_pass_bytes.argtypes = [R, ctypes.POINTER(ctypes.c_size_t),
                                         ctypes.POINTER(ctypes.c_size_t)]
    lib.mhs_fullspace_influence.argtypes = [ctypes.POINTER(FullspaceRequest), V]
    lib.mhs_fullspace_influence.restype = ctypes.c_int
    lib.mhs_autotune.argtypes = [R, V, ctypes.POINTER(Tune), ctypes.POINTER(ctypes.c_double)]
    lib.mhs_set_tune.argtypes = [R, ctypes.POINTER(Tune)]
    lib.mhs_get_tune.argtypes = [R, ctypes.POINTER(Tune)]
    for f in ("mhs_batch_create", "mhs_batch_workspace_bytes", "mhs_batch_bind", "mhs_submit_batch",
              "mhs_poll", "mhs_batch_destroy", "mhs_autotune", "mhs_set_tune", "mhs_get_tune",
              "mhs_batch_pass_bytes"):
        getattr(lib, f).restype = ctypes.c_int
    _lib = lib
    return lib


STAGES = ("prep", "pair", "imageq", "fold", "final", "fold_plan", "fold_nodes", "fold_far",
          "fold_near", "fold_accum", "pair_direct", "pair_image_r")


def profile(on: bool) -> None:
    check(load().mhs_profile_enable(1 if on else 0))


def profile_read() -> dict:
    """Per-stage milliseconds and launch counts since the last read."""
    ms = (ctypes.c_double * len(STAGES))()
    n = (ctypes.c_int * len(STAGES))()
    check(load().mhs_profile_read(ms, n))
    return {s: (ms[i], n[i]) for i, s in enumerate(STAGES)}


CENSUS = ("pairs", "panels", "near", "far12", "far8", "edge_closed", "edge_small", "edge_large",
          "q_pairs", "q_points")


def census(on: bool) -> None:
    """Start (clearing the counters) or stop the work census."""
    check(load().mhs_census_enable(1 if on else 0))


def census_read() -> dict:
    """Work units counted since the last read (synchronises the device)."""
    c = (ctypes.c_ulonglong * len(CENSUS))()
    check(load().mhs_census_read(c))
    return {k: int(c[i]) for i, k in enumerate(CENSUS)}


def kernel_count() -> int:
    """Kernels the library queued since the last call (the count resets)."""
    n = ctypes.c_ulonglong()
    check(load().mhs_kernel_count(ctypes.byref(n)))
    return int(n.value)


def fp_peak(fp64: bool = True, iters: int = 1 << 16, stream=None) -> float:
    """Measured FMA issue ceiling of the current device, TFLOP/s."""
    t = ctypes.c_double()
    check(load().mhs_fp_peak(1 if fp64 else 0, iters, ctypes.byref(t), stream))
    return t.value


def check(rc: int) -> None:
    if rc != 0:
        msg = load().mhs_last_error().decode(errors="replace")
        raise RuntimeError(f"mhs_b200 native call failed (code {rc}): {msg}")
