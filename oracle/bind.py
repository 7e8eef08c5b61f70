"""ctypes binding of oracle/_build/libempanada_oracle.so (the CPU restatement).

Test infrastructure: the checker the CUDA path is compared against.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libempanada_oracle.so")
REF_CPU = os.path.join(HERE, "_ref", "empanada_ref_cpu")
REF_GPU = os.path.join(HERE, "_ref", "empanada_ref_gpu")
MAX_ROUNDS = 512

OK, E_INVAL, E_NOMEM, E_FORMAT, E_UNSUPPORTED, E_HANG = 0, -1, -2, -5, -8, -9


class OracleStats(ctypes.Structure):
    _fields_ = [
        ("n_reads", ctypes.c_uint64),
        ("read_len", ctypes.c_int32),
        ("n_rounds", ctypes.c_int32),
        ("n_unique", ctypes.c_uint64),
        ("n_edges", ctypes.c_uint64),
        ("n_records", ctypes.c_uint64),
        ("sfx_live", ctypes.c_uint64 * MAX_ROUNDS),
        ("pfx_live", ctypes.c_uint64 * MAX_ROUNDS),
        ("edges", ctypes.c_uint64 * MAX_ROUNDS),
    ]

    def to_dict(self) -> dict:
        r = self.n_rounds
        return {"n_reads": self.n_reads, "read_len": self.read_len, "n_rounds": r, "n_unique": self.n_unique,
                "n_edges": self.n_edges, "n_records": self.n_records, "sfx_live": list(self.sfx_live[:r]),
                "pfx_live": list(self.pfx_live[:r]), "edges": list(self.edges[:r])}


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        l = ctypes.CDLL(LIB_PATH)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        l.emp_oracle_run.restype = ctypes.c_int
        l.emp_oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.POINTER(OracleStats)]
        l.emp_oracle_run_var.restype = ctypes.c_int
        l.emp_oracle_run_var.argtypes = l.emp_oracle_run.argtypes
        l.emp_oracle_fingerprints.restype = ctypes.c_int
        l.emp_oracle_fingerprints.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_uint64,
                                              u64p, ctypes.POINTER(ctypes.c_int32)]
        l.emp_oracle_hash.restype = ctypes.c_uint64
        l.emp_oracle_hash.argtypes = [ctypes.c_char_p, ctypes.c_int32]
        l.emp_oracle_next_sfx.restype = ctypes.c_uint64
        l.emp_oracle_next_sfx.argtypes = [ctypes.c_uint64, ctypes.c_char, ctypes.c_int32]
        l.emp_oracle_prev_pfx.restype = ctypes.c_uint64
        l.emp_oracle_prev_pfx.argtypes = [ctypes.c_uint64, ctypes.c_char]
        l.emp_oracle_radix_inv.restype = ctypes.c_uint32
        l.emp_oracle_radix_inv.argtypes = [ctypes.c_int]
        l.emp_oracle_free.restype = None
        l.emp_oracle_free.argtypes = [ctypes.c_void_p]
        l.emp_oracle_gfa.restype = ctypes.c_int
        l.emp_oracle_gfa.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int32,
                                     ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]
        l.emp_oracle_unitigs.restype = ctypes.c_int
        l.emp_oracle_unitigs.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_void_p,
                                         ctypes.c_void_p, u64p]
        _lib = l
    return _lib


def _host_bytes(ptr, n: int) -> bytes:
    """n bytes at ptr, of any size (the ctypes helper for this takes a C int size)."""
    return (ctypes.c_char * n).from_address(ptr).raw if n else b""


def _buf(fastq):
    if isinstance(fastq, np.ndarray):
        a = np.ascontiguousarray(fastq, dtype=np.uint8)
        return a, a.ctypes.data, a.size
    b = bytes(fastq)
    return b, ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p).value, len(b)


class OracleError(RuntimeError):
    def __init__(self, code: int):
        self.code = code
        super().__init__(f"oracle status {code}")


def run(fastq, min_ovlp: int = 31, reduce_mem: int = 1 << 30, variable: bool = False) -> tuple[bytes, dict]:
    """FASTQ bytes -> (output.bin bytes, stats); raises OracleError on a non-zero status.
    variable=True runs the variable-length extension (emp_oracle_run_var)."""
    keep, ptr, n = _buf(fastq)
    out = ctypes.c_void_p()
    out_len = ctypes.c_size_t()
    st = OracleStats()
    fn = lib().emp_oracle_run_var if variable else lib().emp_oracle_run
    rc = fn(ptr, n, min_ovlp, reduce_mem, ctypes.byref(out), ctypes.byref(out_len), ctypes.byref(st))
    del keep
    if rc != OK:
        raise OracleError(rc)
    data = _host_bytes(out.value, out_len.value)
    lib().emp_oracle_free(out)
    return data, st.to_dict()


def fingerprints(fastq) -> tuple[np.ndarray, int, int]:
    """-> (keys of all read-ends indexed by id, n_reads, read_len)."""
    keep, ptr, n = _buf(fastq)
    cap = max(2, n // 2)
    keys = np.zeros(cap, dtype=np.uint64)
    nr = ctypes.c_uint64()
    L = ctypes.c_int32()
    rc = lib().emp_oracle_fingerprints(ptr, n, keys.ctypes.data, cap, ctypes.byref(nr), ctypes.byref(L))
    del keep
    if rc != OK:
        raise OracleError(rc)
    return keys[: 2 * nr.value].copy(), int(nr.value), int(L.value)


def gfa(output_bin: bytes, n_reads: int, read_len: int) -> bytes:
    """The unitig layer's GFA text for an output.bin (the checker of emp_graph_write_gfa)."""
    keep, ptr, n = _buf(output_bin)
    text = ctypes.c_void_p()
    ln = ctypes.c_size_t()
    rc = lib().emp_oracle_gfa(ptr, n, n_reads, read_len, ctypes.byref(text), ctypes.byref(ln))
    del keep
    if rc != 0:
        raise OracleError(rc)
    out = _host_bytes(text.value, ln.value)
    lib().emp_oracle_free(text)
    return out


def unitigs(output_bin: bytes, n_reads: int) -> tuple[np.ndarray, np.ndarray]:
    """-> (read-ends in unitig order, start of every unitig + the end)."""
    keep, ptr, n = _buf(output_bin)
    order = np.zeros(max(1, 2 * n_reads), dtype=np.uint32)
    starts = np.zeros(2 * n_reads + 1, dtype=np.uint64)
    nu = ctypes.c_uint64()
    rc = lib().emp_oracle_unitigs(ptr, n, n_reads, order.ctypes.data, starts.ctypes.data, ctypes.byref(nu))
    del keep
    if rc != 0:
        raise OracleError(rc)
    return order[: 2 * n_reads].copy(), starts[: nu.value + 1].copy()


def hash_of(s: str) -> int:
    return int(lib().emp_oracle_hash(s.encode(), len(s)))


def next_sfx(key: int, base: str, length: int) -> int:
    return int(lib().emp_oracle_next_sfx(key, base.encode(), length))


def prev_pfx(key: int, base: str) -> int:
    return int(lib().emp_oracle_prev_pfx(key, base.encode()))


def radix_inv(which: int) -> int:
    return int(lib().emp_oracle_radix_inv(which))


def run_reference_cpu(input_path: str, output_path: str, args: list[str], threads: int | None = None,
                      cwd: str | None = None, timeout: float | None = None) -> subprocess.CompletedProcess:
    """Run the reference's own sources built as a CPU program (oracle/_ref)."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    return subprocess.run([REF_CPU, input_path, output_path] + list(args), stdout=subprocess.PIPE,
                          stderr=subprocess.PIPE, env=env, cwd=cwd, timeout=timeout)
