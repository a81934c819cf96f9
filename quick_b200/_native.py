"""ctypes binding of libquick_b200.so (the C ABI declared in include/quick_b200.h).

The library is the product's only compute path: if it is missing the import of
this module fails with an error naming the build step; there is no fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libquick_b200.so")

# every symbol include/quick_b200.h declares
EXPORTED = [
    "gpu_new_", "gpu_set_device_", "gpu_init_device_", "gpu_allocate_scratch_",
    "gpu_deallocate_scratch_", "gpu_setup_", "gpu_upload_method_", "gpu_upload_xyz_",
    "gpu_upload_atom_and_chg_", "gpu_upload_basis_", "gpu_upload_cutoff_matrix_",
    "gpu_upload_calculated_", "gpu_upload_cutoff_", "gpu_get_cshell_eri_", "gpu_delete_",
    "qk_last_status", "qk_status_string", "qk_set_maxprim", "qk_max_l", "qk_create",
    "qk_destroy", "qk_default_ctx", "qk_set_basis", "qk_schwarz", "qk_set_schwarz",
    "qk_set_cutoffs", "qk_fock2e_device", "qk_fock2e_host", "qk_density_cutoff_device",
    "qk_last_work", "qk_launches_per_build", "qk_oei_host", "qk_set_profiling",
    "qk_class_profile", "qk_fp64_peak", "qk_fock2e_device_noalloc", "qk_set_precision",
    "qk_last_work_mixed", "qk_batch_create", "qk_batch_destroy", "qk_batch_fock2e",
    "qk_device_bytes", "qk_prepare", "qk_small_solve", "qk_sp2_step", "qk_set_shard", "qk_fock2e_device_accumulate", "qk_finalize_fixed", "qk_set_streams",
    "qk_set_class_launch", "qk_class_launch", "qk_batch_reserve_sms", "qk_boys", "qk_set_boys", "qk_set_worklist_builder",
    "gpu_upload_calculated_beta_", "gpu_get_oshell_eri_", "qk_fock2e_uhf_device", "qk_fock2e_uhf_host",
    "qk_stream_create", "qk_stream_destroy", "qk_sp2_run", "qk_set_merge_sp",
]

_lib = None


class QuickError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: status {status} ({status_string(status)})")


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m quick_b200.build` "
                          f"(or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    PI = ctypes.POINTER(ctypes.c_int)
    L.qk_status_string.restype = ctypes.c_char_p
    L.qk_status_string.argtypes = [I]
    L.qk_last_status.restype = I
    L.qk_set_maxprim.argtypes = [I]
    L.qk_max_l.restype = I
    L.qk_create.restype = P
    L.qk_create.argtypes = [I, PI]
    L.qk_destroy.argtypes = [P]
    L.qk_default_ctx.restype = P
    L.qk_set_basis.argtypes = [P, I, P, I, I, I] + [P] * 12 + [I]
    L.qk_schwarz.argtypes = [P, P, P]
    L.qk_set_schwarz.argtypes = [P, P, P]
    L.qk_set_cutoffs.argtypes = [P, D, D]
    L.qk_fock2e_device.argtypes = [P, P, P, P, P]
    L.qk_boys.argtypes = [P, I, P, I, P, P]
    L.qk_set_boys.argtypes = [P, I]
    L.qk_set_worklist_builder.argtypes = [P, I]
    L.qk_set_merge_sp.argtypes = [P, I]
    L.qk_stream_create.argtypes = [I, I, ctypes.POINTER(ctypes.c_void_p)]
    L.qk_stream_destroy.argtypes = [P]
    L.qk_fock2e_uhf_device.argtypes = [P, P, P, P, P, P, P]
    L.qk_fock2e_uhf_host.argtypes = [P, P, P, P, P, P]
    L.qk_fock2e_host.argtypes = [P, P, P, P]
    L.qk_density_cutoff_device.argtypes = [P, P, P, P]
    L.qk_last_work.argtypes = [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong), PI]
    L.qk_launches_per_build.argtypes = [P]
    L.qk_launches_per_build.restype = I
    L.qk_oei_host.argtypes = [I, I, P, P, I, I, P, P, P, P, P, I, P, P, P, P, P]
    L.qk_oei_host.restype = I
    L.qk_set_profiling.argtypes = [P, I, I]
    L.qk_class_profile.argtypes = [P, I, P, P, P, P, P, P, P, P]
    L.qk_class_profile.restype = I
    L.qk_fp64_peak.argtypes = [I, ctypes.POINTER(ctypes.c_double)]
    L.qk_fock2e_device_noalloc.argtypes = [P, P, P, P, P]
    L.qk_fock2e_device_noalloc.restype = I
    L.qk_set_precision.argtypes = [P, D]
    L.qk_last_work_mixed.argtypes = [P, ctypes.POINTER(ctypes.c_longlong)]
    L.qk_batch_create.restype = P
    L.qk_batch_create.argtypes = [I, PI]
    L.qk_batch_destroy.argtypes = [P]
    L.qk_batch_fock2e.argtypes = [P, I, P, P, P, P, P]
    L.qk_batch_reserve_sms.argtypes = [P, I]
    L.qk_prepare.argtypes = [P]
    L.qk_set_streams.argtypes = [P, I]
    L.qk_set_class_launch.argtypes = [P, I, I, I]
    L.qk_class_launch.argtypes = [P, I, PI, PI, PI, PI]
    L.qk_small_solve.argtypes = [P, P, I, P, P, P]
    L.qk_sp2_step.argtypes = [P, P, P, I, ctypes.c_double, P]
    L.qk_sp2_run.argtypes = [P, P, P, I, ctypes.c_double, I, P]
    L.qk_set_shard.argtypes = [P, I, I]
    L.qk_fock2e_device_accumulate.argtypes = [P, P, P, P, P]
    L.qk_finalize_fixed.argtypes = [P, I, P, P]
    L.qk_device_bytes.argtypes = [P, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)]
    for name in EXPORTED:
        if name.startswith("gpu_"):
            getattr(L, name).restype = None
    _lib = L
    return L


def status_string(status: int) -> str:
    try:
        return lib().qk_status_string(int(status)).decode()
    except Exception:
        return "?"


def check(status: int, what: str = "quick_b200"):
    if status != 0:
        raise QuickError(status, what)


_free_streams = {}          # (device, high_priority) -> streams given back by free_stream
_streams_lock = None


def own_stream(device: int, high_priority: bool = True):
    """A torch view of a stream created for the caller alone (qk_stream_create).

    torch's ``torch.cuda.Stream`` hands out streams from a fixed pool per priority,
    round robin, so two threads can be given the same stream; a thread that captures
    a CUDA graph on a shared stream has its capture invalidated (or other work
    captured into it) when another thread enqueues there.  Give the stream back with
    :func:`free_stream` once its work is done: it is kept for the next caller, not
    destroyed, since torch's allocators keep per-stream state for as long as the
    process runs."""
    global _streams_lock
    import threading
    import torch
    if _streams_lock is None:
        _streams_lock = threading.Lock()
    key = (int(device), bool(high_priority))
    with _streams_lock:
        free = _free_streams.get(key)
        if free:
            return free.pop()
    p = ctypes.c_void_p()
    check(lib().qk_stream_create(int(device), 1 if high_priority else 0, ctypes.byref(p)), "qk_stream_create")
    s = torch.cuda.ExternalStream(p.value, device=torch.device("cuda", int(device)))
    s._qk_key = key
    return s


def free_stream(stream) -> None:
    """Give a stream from :func:`own_stream` back for reuse (its queued work
    must be finished or ordered before the next owner's)."""
    with _streams_lock:
        _free_streams.setdefault(stream._qk_key, []).append(stream)
