"""ctypes binding of the in-tree CUDA library (include/meikey_b200.h).

There is no CPU fallback: if ``libmeikey_b200.so`` is missing, loading raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmeikey_b200.so")

# status codes (enum mk_status)
OK = 0
ERR_DRIVER_NOT_FOUND = 1
ERR_NO_DEVICE = 2
ERR_OUT_OF_RANGE = 3
ERR_SELF_CHECK = 4
ERR_NO_SETTINGS = 5
ERR_CUDA = 6
ERR_NOT_BUILT = 7
ERR_BAD_ARG = 8
ERR_OUT_OF_MEMORY = 9
ERR_STOPPED = 10
ERR_HIT_RING_FULL = 11
ERR_PATTERN = 12

STATUS_NAMES = {
    OK: "OK", ERR_DRIVER_NOT_FOUND: "DriverNotFound", ERR_NO_DEVICE: "NoDevice",
    ERR_OUT_OF_RANGE: "OutOfRange", ERR_SELF_CHECK: "SelfCheck", ERR_NO_SETTINGS: "NoSettings",
    ERR_CUDA: "Driver", ERR_NOT_BUILT: "NotBuilt", ERR_BAD_ARG: "BadArg",
    ERR_OUT_OF_MEMORY: "OutOfMemory", ERR_STOPPED: "Stopped", ERR_HIT_RING_FULL: "HitRingFull",
    ERR_PATTERN: "Pattern",
}

SEED_CHACHA20 = 0
SEED_COUNTER = 1
SEED_INCREMENTAL = 2
MODE_CONTAINS = 0
MODE_SUFFIX = 1
MODE_REGEX = 2


class Options(ctypes.Structure):
    _fields_ = [
        ("table_rows", ctypes.c_uint32),
        ("keys_per_thread", ctypes.c_uint32),
        ("block", ctypes.c_uint32),
        ("blocks_per_sm", ctypes.c_uint32),
        ("self_check", ctypes.c_uint32),
        ("hit_capacity", ctypes.c_uint32),
        ("hash_warps", ctypes.c_uint32),
        ("inverter_rotates", ctypes.c_uint32),
        ("inversion_batch", ctypes.c_uint32),
        ("table_in_smem", ctypes.c_uint32),
        ("hash_interleave", ctypes.c_uint32),
    ]


class TuneEntryC(ctypes.Structure):
    _fields_ = [("options", Options), ("status", ctypes.c_int), ("stage", ctypes.c_uint32),
                ("keys_per_s", ctypes.c_double)]


class SearchConfigC(ctypes.Structure):
    _fields_ = [("first", ctypes.c_uint64), ("max_tries", ctypes.c_uint64), ("time_limit_s", ctypes.c_double),
                ("iters", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class OutcomeC(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("needle", ctypes.c_uint32), ("index", ctypes.c_uint64),
                ("tries", ctypes.c_uint64), ("elapsed_s", ctypes.c_double), ("secret", ctypes.c_uint8 * 32),
                ("pk", ctypes.c_uint8 * 32)]


class ServerOptionsC(ctypes.Structure):
    _fields_ = [("max_jobs", ctypes.c_uint32), ("iters_per_tick", ctypes.c_uint32), ("budget", ctypes.c_uint64),
                ("hit_capacity", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64)]


class JobResultC(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int), ("reserved", ctypes.c_uint32),
                ("admit_index", ctypes.c_uint64), ("index", ctypes.c_uint64), ("tries", ctypes.c_uint64),
                ("expected_tries", ctypes.c_double), ("secret", ctypes.c_uint8 * 32), ("pk", ctypes.c_uint8 * 32)]


PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double)


class NeedleC(ctypes.Structure):
    _fields_ = [
        ("bytes", ctypes.POINTER(ctypes.c_uint8)),
        ("len", ctypes.c_uint32),
        ("fold", ctypes.c_uint32),
        ("mode", ctypes.c_uint32),
    ]


class HitC(ctypes.Structure):
    _fields_ = [("index", ctypes.c_uint64), ("needle", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class InfoC(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int),
        ("sms", ctypes.c_uint32),
        ("grid", ctypes.c_uint32),
        ("block", ctypes.c_uint32),
        ("keys_per_thread", ctypes.c_uint32),
        ("table_rows", ctypes.c_uint32),
        ("table_bytes", ctypes.c_uint64),
        ("keys_per_iter", ctypes.c_uint64),
        ("name", ctypes.c_char * 96),
        ("inversion_batch", ctypes.c_uint32),
        ("table_in_smem", ctypes.c_uint32),
    ]


# (name, restype, argtypes) of every exported function
SIGNATURES = [
    ("mk_abi_version", ctypes.c_uint32, []),
    ("mk_device_count", ctypes.c_int, []),
    ("mk_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_void_p)]),
    ("mk_ctx_destroy", None, [ctypes.c_void_p]),
    ("mk_last_error", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    ("mk_ctx_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(InfoC)]),
    ("mk_keys_per_iter", ctypes.c_uint64, [ctypes.c_void_p]),
    ("mk_job_prepare", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(NeedleC),
                                      ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("mk_job_destroy", None, [ctypes.c_void_p]),
    ("mk_job_launch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_uint64)]),
    ("mk_job_hits", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(HitC), ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)]),
    ("mk_job_update", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(NeedleC), ctypes.c_uint32]),
    ("mk_job_graph_create", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    ("mk_graph_launch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_uint64)]),
    ("mk_graph_enqueue", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("mk_graph_destroy", None, [ctypes.c_void_p]),
    ("mk_job_confirm", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("mk_job_enqueue", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32]),
    ("mk_ctx_sync", ctypes.c_int, [ctypes.c_void_p]),
    ("mk_ctx_record", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("mk_ctx_elapsed", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("mk_derive", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.c_void_p]),
    ("mk_table_entry", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                      ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_job_io_bytes", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                       ctypes.POINTER(ctypes.c_uint64)]),
    ("mk_ctx_work_per_key", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double)]),
    ("mk_measure_imad_rates", ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_double)] * 4),
    ("mk_measure_mad_peaks", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]),
    ("mk_regex_compile", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_uint32), ctypes.c_char_p, ctypes.c_size_t]),
    ("mk_regex_compile_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32,
                                               ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_char_p,
                                               ctypes.c_size_t]),
    ("mk_autotune", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(TuneEntryC), ctypes.c_uint32, ctypes.c_uint32,
                                   ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_autotune_job", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(TuneEntryC), ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(NeedleC),
                                       ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_measure_field_mul", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("mk_measure_field_mul_forms", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                                  ctypes.POINTER(ctypes.c_double)]),
    ("mk_field_mul_pairs", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    ("mk_job_stop", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("mk_job_collect", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint64)]),
    ("mk_job_first_matches", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(OutcomeC), ctypes.c_uint32]),
    ("mk_needles_check", ctypes.c_int, [ctypes.POINTER(NeedleC), ctypes.c_uint32]),
    ("mk_job_keys_per_iter", ctypes.c_uint64, [ctypes.c_void_p]),
    ("mk_expected_tries", ctypes.c_double, [ctypes.POINTER(NeedleC)]),
    ("mk_search", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SearchConfigC), PROGRESS_FN, ctypes.c_void_p,
                                 ctypes.POINTER(OutcomeC)]),
    ("mk_search_many", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, PROGRESS_FN, ctypes.c_void_p,
                                      ctypes.POINTER(OutcomeC), ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_search_both", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SearchConfigC), ctypes.c_uint32, ctypes.c_uint64,
                                      PROGRESS_FN, ctypes.c_void_p, ctypes.POINTER(OutcomeC),
                                      ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_server_create", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ServerOptionsC),
                                        ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("mk_server_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(NeedleC), ctypes.c_uint64]),
    ("mk_server_tick", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_server_results", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(JobResultC), ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_uint32)]),
    ("mk_server_position", ctypes.c_uint64, [ctypes.c_void_p]),
    ("mk_server_destroy", None, [ctypes.c_void_p]),
    ("mk_openssh_public", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t,
                                         ctypes.POINTER(ctypes.c_size_t)]),
    ("mk_openssh_private", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_char_p,
                                          ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    ("mk_derive_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint64,
                                         ctypes.c_uint64, ctypes.c_void_p]),
]

# largest n of mk_derive_noalloc (its fixed device staging holds this many 32-byte keys)
NOALLOC_MAX_KEYS = 1 << 16

_lib = None


def load():
    """The loaded library; raises OSError when the CUDA build is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(
            f"{LIB_PATH} is missing: build the CUDA library first (python -m meikey_b200.build); "
            "there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib
