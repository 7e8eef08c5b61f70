"""ctypes binding of libempanada_b200.so (the C ABI declared in include/empanada.h).

Loading fails loudly when the library has not been built: there is no
fallback implementation of the overlap path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libempanada_b200.so")

EMP_OK = 0
EMP_E_INVAL = -1
EMP_E_NOMEM = -2
EMP_E_CUDA = -3
EMP_E_TIMEOUT = -4
EMP_E_FORMAT = -5
EMP_E_STATE = -6
EMP_E_IO = -7
EMP_E_UNSUPPORTED = -8
EMP_E_HANG = -9
MAX_ROUNDS = 512

# every function include/empanada.h declares, with its ctypes signature
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p


class Params(ctypes.Structure):
    _fields_ = [
        ("min_ovlp", ctypes.c_int32),
        ("map_mem", ctypes.c_uint64),
        ("reduce_mem", ctypes.c_uint64),
        ("base_blocksz", ctypes.c_uint64),
        ("kv_chunksz", ctypes.c_uint64),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("round_driver", ctypes.c_int32),
        ("bucket_mean", ctypes.c_uint32),
        ("region_cap", ctypes.c_uint32),
        ("dedup_driver", ctypes.c_int32),
        ("edge_cap", ctypes.c_uint64),
        ("wait_limit_ns", ctypes.c_uint64),
        ("block_next_wait", ctypes.c_int32),
        ("map_streams", ctypes.c_uint32),
    ]

    def to_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if not f.startswith("reserved")}


class GraphStats(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.c_uint64),
        ("edges", ctypes.c_uint64),
        ("unitigs", ctypes.c_uint64),
        ("long_unitigs", ctypes.c_uint64),
        ("cycles", ctypes.c_uint64),
        ("ms_build", ctypes.c_double),
    ]

    def to_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


# int (*emp_edge_sink)(void *user, int32_t ovlp_len, uint64_t n, const uint32_t *from, const uint32_t *to)
EDGE_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint64,
                             ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32))


class ServerParams(ctypes.Structure):
    _fields_ = [
        ("rounds_per_launch", ctypes.c_int32),
        ("max_jobs", ctypes.c_int32),
        ("hbm_budget_bytes", ctypes.c_uint64),
        ("rounds_per_launch_idle", ctypes.c_int32),
        ("batch_max_entries", ctypes.c_uint64),
        ("share_min_entries", ctypes.c_uint64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_uint64),
        ("admitted", ctypes.c_uint64),
        ("launches", ctypes.c_uint64),
        ("rounds", ctypes.c_uint64),
        ("batch_jobs", ctypes.c_uint64),
        ("ms_kernel", ctypes.c_double),
        ("ms_admit", ctypes.c_double),
        ("ms_map", ctypes.c_double),
        ("ms_alone", ctypes.c_double),
        ("alone", ctypes.c_uint64),
        ("ms_wait", ctypes.c_double),
        ("ms_results", ctypes.c_double),
        ("ms_launch", ctypes.c_double),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_reads", ctypes.c_uint64),
        ("read_len", ctypes.c_int32),
        ("n_rounds", ctypes.c_int32),
        ("n_unique", ctypes.c_uint64),
        ("n_edges", ctypes.c_uint64),
        ("n_records", ctypes.c_uint64),
        ("fastq_bytes", ctypes.c_uint64),
        ("output_bytes", ctypes.c_uint64),
        ("gpu_launches", ctypes.c_uint64),
        ("ms_h2d", ctypes.c_double),
        ("ms_map", ctypes.c_double),
        ("ms_dedup", ctypes.c_double),
        ("ms_rounds", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("ms_sort_passes", ctypes.c_double),
        ("sort_passes", ctypes.c_uint64),
        ("sort_pass_elems", ctypes.c_uint64),
        ("ms_update", ctypes.c_double),
        ("update_launches", ctypes.c_uint64),
        ("update_bytes", ctypes.c_uint64),
        ("ms_round_kernel", ctypes.c_double),
        ("round_kernel_bytes", ctypes.c_uint64),
        ("sfx_live", ctypes.c_uint64 * MAX_ROUNDS),
        ("pfx_live", ctypes.c_uint64 * MAX_ROUNDS),
        ("edges", ctypes.c_uint64 * MAX_ROUNDS),
    ]

    def to_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_[:22]}
        r = self.n_rounds
        d["sfx_live"] = list(self.sfx_live[:r])
        d["pfx_live"] = list(self.pfx_live[:r])
        d["edges"] = list(self.edges[:r])
        return d


SIGNATURES = {
    "emp_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "emp_abi_version": (ctypes.c_int, []),
    "emp_params_default": (ctypes.c_int, [ctypes.POINTER(Params)]),
    "emp_parse_size": (ctypes.c_int, [ctypes.c_char_p, _u64p]),
    "emp_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "emp_ctx_destroy": (ctypes.c_int, [_vp]),
    "emp_tuning_default": (ctypes.c_int, [ctypes.POINTER(Tuning)]),
    "emp_ctx_set_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(Tuning)]),
    "emp_ctx_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(Tuning)]),
    "emp_job_create": (ctypes.c_int, [_vp, ctypes.POINTER(Params), ctypes.POINTER(_vp)]),
    "emp_job_destroy": (ctypes.c_int, [_vp]),
    "emp_job_feed_fastq": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_int]),
    "emp_job_feed_fastq_device": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_int]),
    "emp_job_feed_fastq_async": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_int]),
    "emp_job_reserve": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "emp_job_reset": (ctypes.c_int, [_vp]),
    "emp_job_trim": (ctypes.c_int, [_vp]),
    "emp_job_run": (ctypes.c_int, [_vp, _vp]),
    "emp_batch_run": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.c_int, _vp]),
    "emp_job_status": (ctypes.c_int, [_vp]),
    "emp_server_params_default": (ctypes.c_int, [ctypes.POINTER(ServerParams)]),
    "emp_server_create": (ctypes.c_int, [_vp, ctypes.POINTER(ServerParams), ctypes.POINTER(_vp)]),
    "emp_server_destroy": (ctypes.c_int, [_vp]),
    "emp_server_submit": (ctypes.c_int, [_vp, _vp]),
    "emp_server_step": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "emp_server_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ServerStats)]),
    "emp_server_counts": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)]),
    "emp_job_output_size": (ctypes.c_int, [_vp, _u64p]),
    "emp_job_output_copy": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64]),
    "emp_job_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats)]),
    "emp_job_edges": (ctypes.c_int, [_vp, EDGE_SINK, _vp]),
    "emp_job_fingerprints": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, _u64p]),
    "emp_run_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(Params), ctypes.c_int,
                                    ctypes.POINTER(Stats)]),
    "emp_run_files": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_char_p,
                                     ctypes.POINTER(Params), ctypes.c_int, ctypes.POINTER(Stats)]),
    "emp_job_feed_files": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]),
    "emp_fastq_load": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.POINTER(_vp), _u64p]),
    "emp_free": (None, [_vp]),
    "emp_measure_l2_read": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]),
    "emp_graph_build": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "emp_graph_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(GraphStats)]),
    "emp_graph_unitigs": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, _vp, ctypes.c_uint64]),
    "emp_graph_write_gfa": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int32]),
    "emp_graph_destroy": (ctypes.c_int, [_vp]),
    "emp_sort_pairs": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint64, _vp]),
    "emp_sort_pairs_static": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, _vp]),
}
SORT_STATIC_MAX_PAIRS = 1 << 20  # EMP_SORT_STATIC_MAX_PAIRS

_lib = None


class EmpError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = status_string(code) if _lib is not None else str(code)
        super().__init__(f"{what}: {msg} ({code})" if what else f"{msg} ({code})")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"native library {LIB_PATH} is missing: run __graft_entry__.build() "
                               "(the overlap path has no CPU fallback)")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def status_string(code: int) -> str:
    return lib().emp_status_string(code).decode()


def check(code: int, what: str = "") -> None:
    if code != EMP_OK:
        raise EmpError(code, what)
