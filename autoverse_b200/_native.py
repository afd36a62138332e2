"""ctypes binding of ``libflowlenia_cuda.so`` (include/flowlenia_cuda.h).

The library is loaded from the package's in-tree ``_lib`` directory.  There is
no fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FLOWLENIA_LIB") or os.path.join(HERE, "_lib", "libflowlenia_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "flowlenia_cuda.h")

FLP_OK = 0
ERRORS = {
    -1: "INVALID_CONFIG",
    -2: "INVALID_ARGUMENT",
    -3: "OOM",
    -4: "CUDA_ERROR",
    -5: "TIMEOUT",
    -6: "NONFINITE",
    -7: "UNSUPPORTED",
}
CONV_AUTO, CONV_DIRECT, CONV_FFT = 0, 1, 2


class FlpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class ConfigError(FlpError, ValueError):
    """Invalid SimulationConfig (the reference's ConfigError, src/schema/config.rs:168-180)."""


class Info(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32), ("channels", C.c_int32),
                ("n_kernels", C.c_int32), ("conv_mode", C.c_int32), ("time", C.c_float), ("step", C.c_uint64)]


_lib: C.CDLL | None = None

P = C.c_void_p
I = C.c_int
Z = C.c_size_t
S = C.c_char_p
F = C.c_float
U64 = C.c_uint64
PP = C.POINTER(C.c_void_p)

SIGNATURES = {
    "flp_last_error": (S, []),
    "flp_create": (I, [S, PP]),
    "flp_destroy": (I, [P]),
    "flp_state_from_seed": (I, [P, S]),
    "flp_seed_generate": (I, [S, S, P, Z]),
    "flp_write_state": (I, [P, P, Z, F, U64]),
    "flp_read_state": (I, [P, P, Z, C.POINTER(F), C.POINTER(U64)]),
    "flp_step": (I, [P]),
    "flp_run": (I, [P, U64]),
    "flp_step_host": (I, [P, P, Z, C.POINTER(F), C.POINTER(U64), U64]),
    "flp_synchronize": (I, [P]),
    "flp_synchronize_for": (I, [P, C.c_double]),
    "flp_total_mass": (I, [P, C.POINTER(C.c_double)]),
    "flp_total_mass_f32": (I, [P, C.POINTER(F)]),
    "flp_get_info": (I, [P, C.POINTER(Info)]),
    "flp_set_conv_mode": (I, [P, I]),
    "flp_get_tuning": (I, [P, C.POINTER(C.c_int32), I]),
    "flp_set_tuning": (I, [P, C.POINTER(C.c_int32), I]),
    "flp_stream": (P, [P]),
    "flp_device_state": (P, [P]),
    "flp_device_info": (I, [C.c_char_p, I, C.POINTER(I), C.POINTER(Z)]),
    "flp_host_alloc": (I, [Z, PP]),
    "flp_host_free": (I, [P]),
    "flp_profile_run": (I, [P, I, I, C.POINTER(F), I, C.POINTER(I), C.c_char_p, Z, C.POINTER(F)]),
    "flp_debug_affinity": (I, [P, P, Z]),
    "flp_affinity_noalloc": (I, [S, P, P, P]),
    "flp_batch_create": (I, [C.POINTER(C.c_char_p), I, PP]),
    "flp_batch_stats": (I, [P, P, Z]),
    "flp_batch_reserve_snapshots": (I, [P, I]),
    "flp_batch_snapshot": (I, [P, I]),
    "flp_batch_similarity": (I, [P, I, I, P, I]),
    "flp_adj_create": (I, [C.POINTER(C.c_char_p), I, PP]),
    "flp_adj_destroy": (I, [P]),
    "flp_adj_write_state": (I, [P, I, P, Z]),
    "flp_adj_state_from_seed": (I, [P, I, S]),
    "flp_adj_forward": (I, [P, I, I]),
    "flp_adj_read_final": (I, [P, I, P, Z]),
    "flp_adj_param_count": (I, [P, I, C.POINTER(I)]),
    "flp_adj_backward": (I, [P, P, Z, P, Z, P, Z]),
    "flp_adj_timings": (I, [P, C.POINTER(F), C.POINTER(F)]),
    "flp_batch_destroy": (I, [P]),
    "flp_batch_state_from_seed": (I, [P, I, S]),
    "flp_batch_states_from_seeds": (I, [P, C.POINTER(C.c_char_p), I]),
    "flp_batch_reconfigure": (I, [P, C.POINTER(C.c_char_p), I]),
    "flp_batch_write_world": (I, [P, I, P, Z]),
    "flp_batch_read_world": (I, [P, I, P, Z, C.POINTER(F), C.POINTER(U64)]),
    "flp_batch_run": (I, [P, U64]),
    "flp_batch_synchronize": (I, [P]),
    "flp_batch_synchronize_for": (I, [P, C.c_double]),
    "flp_batch_total_mass": (I, [P, P, I]),
    "flp_batch_info": (I, [P, C.POINTER(I), C.POINTER(Z), C.POINTER(Z)]),
    "flp_batch_stream": (P, [P]),
    "flp_batch_kernel_spectra": (I, [P, C.POINTER(I), C.POINTER(Z)]),
    "flp_batch_profile_run": (I, [P, I, I, C.POINTER(F), C.POINTER(F)]),
    "flp_debug_transport": (I, [P, P, P, P, Z]),
    "flp_twin64_step": (I, [S, P, P, P]),
    "flp_emb_create": (I, [S, PP]),
    "flp_emb_destroy": (I, [P]),
    "flp_emb_state_from_seed": (I, [P, S]),
    "flp_emb_write_state": (I, [P, P, Z, P, Z, F, U64]),
    "flp_emb_read_state": (I, [P, P, Z, P, Z, C.POINTER(F), C.POINTER(U64)]),
    "flp_emb_step": (I, [P]),
    "flp_emb_run": (I, [P, U64]),
    "flp_emb_synchronize": (I, [P]),
    "flp_emb_total_mass": (I, [P, C.POINTER(C.c_double)]),
    "flp_emb_profile_run": (I, [P, U64, C.POINTER(F), C.POINTER(F)]),
    "flp_emb_stream": (P, [P]),
    "flp_rec_create": (I, [P, S, I, C.c_uint32, U64, PP]),
    "flp_rec_record": (I, [P, C.POINTER(I)]),
    "flp_rec_run": (I, [P, U64]),
    "flp_rec_frames_written": (I, [P, C.POINTER(U64)]),
    "flp_rec_finalize": (I, [P, C.POINTER(U64), C.POINTER(U64), C.POINTER(U64)]),
    "flp_debug_fail_device_alloc": (I, [C.c_int64]),
    "flp_debug_live_device_allocs": (I, [C.POINTER(C.c_int64)]),
}


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(flp_\w+)\s*\(", text, re.M)))


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FlpError(-7, f"engine library not built: {LIB_PATH} (run autoverse_b200/build.py)")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def device_info() -> dict:
    bus = C.create_string_buffer(64)
    sms = C.c_int()
    l2 = C.c_size_t()
    check(lib().flp_device_info(bus, 64, C.byref(sms), C.byref(l2)))
    return {"pci_bus_id": bus.value.decode(), "sm_count": sms.value, "l2_bytes": l2.value}


def check(rc: int) -> None:
    if rc != FLP_OK:
        msg = lib().flp_last_error().decode(errors="replace")
        if rc == -1:
            raise ConfigError(rc, msg)
        raise FlpError(rc, msg)
