"""ctypes binding of libgjxl_b200.so (the C ABI declared in include/gjxl_b200.h).

The library is built in-tree by gjxl_b200.build. There is no fallback: if the
shared library is missing or fails to load, every entry point raises.
"""

from __future__ import annotations

import ctypes
from ctypes import c_char_p, c_double, c_float, c_int, c_size_t, c_uint32, c_void_p
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libgjxl_b200.so"

P = c_void_p  # device or host pointer
Z = c_size_t
F = c_float
I = c_int

# name -> argument types; every function returns int (StatusCode numbering)
# unless listed in _RESTYPES.
SIGNATURES: dict[str, list] = {
    "gjxl_b200_last_error": [],
    "gjxl_b200_version": [],
    "gjxl_b200_prepare_input": [P, Z, Z, Z, I, F, P, Z, Z, P, Z, Z, Z, Z, P, P],
    "gjxl_b200_matrix_scale_stats": [P, Z, Z, Z, Z, P, P],
    "gjxl_b200_initial_quant_scratch_bytes": [Z, Z],
    "gjxl_b200_initial_quant_field": [P, Z, Z, Z, Z, F, F, P, P, P, Z, P, Z, P, P],
    "gjxl_b200_initial_quant_field_noalloc": [P, Z, Z, Z, Z, F, F, P, P, P, Z, P, P],
    "gjxl_b200_gaborish_inverse": [P, Z, Z, P, Z, Z, Z, Z, P, P, P],
    "gjxl_b200_initial_cfl": [P, Z, Z, Z, Z, P, P, P],
    "gjxl_b200_dc_token_sizes": [Z, Z, P, P, P, P],
    "gjxl_b200_ac_strategy_candidate_costs": [I, P, Z, Z, P, Z, Z, Z, P, Z, P, P, P, P, F, I, P, P,
                                              P],
    "gjxl_b200_batch_create": [I, P, P],
    "gjxl_b200_cnn_param_count": [],
    "gjxl_b200_cnn_workspace_bytes": [I],
    "gjxl_b200_cnn_train_scratch_bytes": [I],
    "gjxl_b200_cnn_gather": [P, Z, Z, Z, Z, P, I, F, P, P],
    "gjxl_b200_cnn_forward": [P, I, P, P, I, P],
    "gjxl_b200_cnn_train_step": [P, I, P, P, P, P, F, P, P, P, P],
    "gjxl_b200_cnn_adamw": [P, P, P, P, I, F, F, F, F, F, P],
    "gjxl_b200_session_device_bytes": [Z, Z, P, P],
    "gjxl_b200_session_create_in": [Z, Z, P, P, Z, P],
    "gjxl_b200_batch_destroy": None,
    "gjxl_b200_batch_set_schedule": [P, I, I],
    "gjxl_b200_batch_analyze": [P, P, Z, I, P, P],
    "gjxl_b200_batch_autotune": [P, P, Z, P, Z, P, P],
    "gjxl_b200_batch_schedule": [Z, P, I, I, P, P],
    "gjxl_b200_batch_device_bytes": [P],
    "gjxl_b200_dc_tokenize": [P, Z, P, P, P, P, P, Z, Z, I, P, P, P, P, P, Z, P, P],
    "gjxl_b200_quant_matrix": [I, I, P, P, Z],
    "gjxl_b200_ac_strategy_cost_bytes": [Z, Z],
    "gjxl_b200_ac_strategy_costs": [P, Z, Z, Z, Z, P, P, Z, P, P, F, I, I, P, P, P],
    "gjxl_b200_ac_strategy_search": [P, Z, Z, Z, Z, P, P, Z, P, P, F, I, I, P, P, P, P],
    "gjxl_b200_butteraugli_create": [Z, Z, F, P],
    "gjxl_b200_butteraugli_destroy": None,
    "gjxl_b200_butteraugli_prepare": [P, P, Z, Z, P],
    "gjxl_b200_butteraugli_compare": [P, P, Z, Z, P, Z, P, P, P],
    "gjxl_b200_ac_token_capacity": [Z, Z],
    "gjxl_b200_ac_tokens_create": [Z, Z, P],
    "gjxl_b200_ac_tokens_destroy": None,
    "gjxl_b200_ac_tokenize": [P, P, P, P, Z, Z, P, I, P, P],
    # Session entry points are bound with their struct types in session.py.
    "gjxl_b200_default_options": None,
    "gjxl_b200_session_create": None,
    "gjxl_b200_session_destroy": None,
    "gjxl_b200_session_set_butteraugli_target": None,
    "gjxl_b200_session_analyze": None,
    "gjxl_b200_session_analyze_host": None,
    "gjxl_b200_session_outputs": None,
    "gjxl_b200_session_stage_times": None,
    "gjxl_b200_stage_name": None,
    "gjxl_b200_session_kernel_count": None,
    "gjxl_b200_fp64_throughput": [P, P, P],
    "gjxl_b200_check_device_error": [P, Z, P],
    "gjxl_b200_butteraugli_pnorm_scratch_bytes": [],
    "gjxl_b200_butteraugli_pnorm": [P, Z, Z, Z, c_double, P, Z, P, P],
    "gjxl_b200_test_arm_failure": [I, I],
    "gjxl_b200_entropy_slot_words": [I, Z, Z],
    "gjxl_b200_entropy_write_sections": [P, P, P, Z, P, P, Z, P, P, P],
    "gjxl_b200_entropy_count_sections": [P, c_uint32, P, P, P, P],
}
_RESTYPES = {"gjxl_b200_last_error": c_char_p,
             "gjxl_b200_initial_quant_scratch_bytes": c_size_t,
             "gjxl_b200_ac_strategy_cost_bytes": c_size_t,
             "gjxl_b200_ac_token_capacity": c_size_t,
             "gjxl_b200_butteraugli_pnorm_scratch_bytes": c_size_t,
             "gjxl_b200_batch_device_bytes": c_size_t,
             "gjxl_b200_cnn_param_count": c_size_t,
             "gjxl_b200_cnn_workspace_bytes": c_size_t,
             "gjxl_b200_cnn_train_scratch_bytes": c_size_t,
             "gjxl_b200_entropy_slot_words": c_size_t}

STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "UNSUPPORTED", 3: "UNAVAILABLE",
    4: "OUT_OF_MEMORY", 5: "FAILED_PRECONDITION", 6: "SUBMISSION_FAILED",
    7: "DEVICE_ERROR", 8: "INTERNAL",
}


class GjxlB200Error(RuntimeError):
    def __init__(self, code: int, function: str, message: str):
        super().__init__(f"{function} failed with {STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


_lib = None


def load() -> ctypes.CDLL:
    """Loads the library (once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `python -m gjxl_b200.build`")
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            if args is None:
                continue
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, c_int)
        _lib = lib
    return _lib


def call(name: str, *args) -> None:
    """Calls an entry point and raises GjxlB200Error on a nonzero status."""
    lib = load()
    code = getattr(lib, name)(*args)
    if code != 0:
        raise GjxlB200Error(code, name, lib.gjxl_b200_last_error().decode())
