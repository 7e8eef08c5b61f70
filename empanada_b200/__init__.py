"""empanada_b200 -- B200-native drop-in for empanada's read-overlap path.

The product is the native library (``libempanada_b200.so``, C ABI in
``include/empanada.h``) and the ``empanada`` command built beside it.  This
module is the host-side mirror of the reference's interface for that path:

* :func:`parse_args` / :class:`Config` -- the reference's option parser
  (config.h:10-140): ``input.fastq output.bin -o -m -r -b -c``;
* :func:`run_file` -- the reference program (main.cu:9-77): FASTQ file in,
  ``output.bin`` out;
* :func:`run_bytes` / :class:`Engine` -- the same on in-memory or
  device-resident FASTQ bytes;
* :func:`decode_output` -- the ``output.bin`` record format
  (overlap.cu:148-161): ``u64 n | i32 ovlp_len | u32 from[n] | u32 to[n]``.

Every entry point calls the CUDA path; there is no CPU fallback.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import dataclasses
import struct
from typing import Iterable

import numpy as np

from . import _native
from ._native import EmpError, check

__all__ = ["Config", "parse_args", "parse_size", "Engine", "Job", "Graph", "run_bytes", "run_file", "decode_output",
           "EmpError", "UsageExit"]

DEFAULTS = {"o": "31", "m": "1g", "r": "1g", "b": "32m", "c": "64m"}
_OPTIONS = [  # (shortname, longname, description, default) as in config.h:120-140
    ("o", "min-overlap", "minimum overlap length", "31"),
    ("m", "map-mem", "device memory during the fingerprint generation phase", "1g"),
    ("r", "reduce-mem", "device memory during the overlap-detection phase", "1g"),
    ("b", "base-blocksz", "block size (count) of transposed bases", "32m"),
    ("c", "kv-chunksz", "block size (count) of key-value pairs", "64m"),
]


class UsageExit(SystemExit):
    """The reference prints its usage and exits 0 (config.h:21-35)."""

    def __init__(self, message: str):
        super().__init__(0)
        self.message = message


def usage_text() -> str:
    lines = ["Usage: assembly_v3 [input fastq] [output gfa] [options]", "Options:"]
    for s, l, d, dv in _OPTIONS:
        lines.append(f"  -{s} or --{l}, {d}, default = {dv}")
    return "\n".join(lines) + "\n"


def parse_size(s: str) -> int:
    """hmsize2bytes (config.h:75-100) through the native parser."""
    v = ctypes.c_uint64(0)
    rc = _native.lib().emp_parse_size(s.encode(), ctypes.byref(v))
    if rc == _native.EMP_E_INVAL and s and not s[-1].isdigit():
        inner = ctypes.c_uint64(0)
        if _native.lib().emp_parse_size(s[:-1].encode(), ctypes.byref(inner)) == _native.EMP_OK:
            return int(inner.value)  # unknown unit: logged and ignored by the reference
    check(rc, f"size {s!r}")
    return int(v.value)


@dataclasses.dataclass
class Config:
    """Config::init (config.h:120-140)."""
    input: str
    output: str
    min_ovlp: int = 31
    map_mem: int = 1 << 30
    reduce_mem: int = 1 << 30
    base_blocksz: int = 32 << 20
    kv_chunksz: int = 64 << 20

    def params(self) -> _native.Params:
        return _native.Params(self.min_ovlp, self.map_mem, self.reduce_mem, self.base_blocksz, self.kv_chunksz)


def parse_args(argv: Iterable[str]) -> Config:
    """parse_args (config.h:37-73) with the reference's quirks: options are
    matched on their second character, long options are rejected, and a
    missing positional or an unknown option raises :class:`UsageExit`."""
    args = list(argv)
    positional: list[str] = []
    values: dict[str, str] = {}
    i = 0
    while i < len(args):
        arg = args[i]
        if len(positional) < 2:
            positional.append(arg)
            i += 1
            continue
        second = arg[1] if len(arg) > 1 else ""
        found = False
        for s, _l, _d, _dv in _OPTIONS:
            if second == s:
                if i + 1 >= len(args):
                    raise ValueError(f"option {arg} needs a value")
                values[s] = args[i + 1]
                i += 2
                found = True
                break
        if not found:
            raise UsageExit(f"Invalid option {arg}\n" + usage_text())
    if len(positional) < 2:
        raise UsageExit(usage_text())
    get = lambda k: parse_size(values.get(k, DEFAULTS[k]))
    o = get("o")
    o = ((o + 2**31) % 2**32) - 2**31  # int conversion of config.h:127
    return Config(positional[0], positional[1], o, get("m"), get("r"), get("b"), get("c"))


def _params(min_ovlp=31, map_mem="1g", reduce_mem="1g", base_blocksz="32m", kv_chunksz="64m") -> _native.Params:
    conv = lambda v: parse_size(v) if isinstance(v, str) else int(v)
    return _native.Params(int(min_ovlp), conv(map_mem), conv(reduce_mem), conv(base_blocksz), conv(kv_chunksz))


class Engine:
    """An emp_ctx: one device, its stream and hash tables."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._lib = _native.lib()
        h = ctypes.c_void_p()
        check(self._lib.emp_ctx_create(device, hbm_budget_bytes, ctypes.byref(h)), "emp_ctx_create")
        self.handle = h

    def close(self):
        if self.handle:
            self._lib.emp_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def job(self, **params) -> "Job":
        return Job(self, _params(**params))

    def run_batch(self, jobs: "list[Job]", stream: int = 0) -> None:
        """Run independent jobs of this engine as one batch (emp_batch_run):
        each job's output equals what Job.run gives it alone."""
        if not jobs:
            return
        arr = (ctypes.c_void_p * len(jobs))(*[j.handle for j in jobs])
        check(self._lib.emp_batch_run(self.handle, arr, len(jobs), stream or None), "emp_batch_run")

    def sort_pairs(self, keys_ptr: int, vals_ptr: int, n: int, stream: int = 0) -> None:
        """Stable device sort of (u64 fingerprint, u32 value) pairs in place."""
        check(self._lib.emp_sort_pairs(self.handle, keys_ptr, vals_ptr, n, stream or None), "emp_sort_pairs")

    def tuning(self) -> dict:
        """The context's engine choices (emp_ctx_get_tuning), defaults filled in."""
        t = _native.Tuning()
        check(self._lib.emp_ctx_get_tuning(self.handle, ctypes.byref(t)), "emp_ctx_get_tuning")
        return t.to_dict()

    def set_tuning(self, **choices) -> None:
        """Change some engine choices (emp_ctx_set_tuning); the others keep
        their current values.  Every choice gives the same output.bin."""
        t = _native.Tuning()
        check(self._lib.emp_ctx_get_tuning(self.handle, ctypes.byref(t)), "emp_ctx_get_tuning")
        for k, v in choices.items():
            if k not in t.to_dict():
                raise KeyError(f"unknown tuning field {k!r}")
            setattr(t, k, int(v))
        check(self._lib.emp_ctx_set_tuning(self.handle, ctypes.byref(t)), "emp_ctx_set_tuning")

    @contextlib.contextmanager
    def tuned(self, **choices):
        """set_tuning for the duration of a with-block, then the previous choices."""
        before = self.tuning()
        self.set_tuning(**choices)
        try:
            yield self
        finally:
            self.set_tuning(**before)


class Job:
    def __init__(self, engine: Engine, params: _native.Params):
        self.engine = engine
        self._lib = engine._lib
        h = ctypes.c_void_p()
        check(self._lib.emp_job_create(engine.handle, ctypes.byref(params), ctypes.byref(h)), "emp_job_create")
        self.handle = h

    def close(self):
        if self.handle:
            self._lib.emp_job_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reserve(self, nbytes: int) -> None:
        check(self._lib.emp_job_reserve(self.handle, nbytes), "emp_job_reserve")

    def reset(self) -> None:
        """Drop the fed input and last result; keep the device buffers."""
        check(self._lib.emp_job_reset(self.handle), "emp_job_reset")

    def trim(self) -> None:
        """Drop the fed input and last result; give the device buffers back to the engine's pool."""
        check(self._lib.emp_job_trim(self.handle), "emp_job_trim")

    def feed(self, data, last: bool = True) -> None:
        """Append host FASTQ bytes (bytes, bytearray or a uint8 numpy array)."""
        if isinstance(data, np.ndarray):
            arr = np.ascontiguousarray(data, dtype=np.uint8)
            check(self._lib.emp_job_feed_fastq(self.handle, arr.ctypes.data, arr.size, int(last)), "feed")
        else:
            buf = bytes(data)
            check(self._lib.emp_job_feed_fastq(self.handle, ctypes.c_char_p(buf), len(buf), int(last)), "feed")

    def feed_async(self, arr: np.ndarray, last: bool = True) -> None:
        """feed() without waiting for the copy; arr (uint8, contiguous, ideally
        page-locked) must stay unchanged until the job's next run starts."""
        if arr.dtype != np.uint8 or not arr.flags.c_contiguous:
            raise ValueError("feed_async takes a contiguous uint8 array")
        self._async_keep = arr
        check(self._lib.emp_job_feed_fastq_async(self.handle, arr.ctypes.data, arr.size, int(last)), "feed_async")

    def feed_files(self, paths) -> None:
        """Append the FASTQ of files in order (plain, gzip or BGZF) and mark
        the end of the input (emp_job_feed_files)."""
        arr = _path_array(paths)
        check(self._lib.emp_job_feed_files(self.handle, arr, len(arr)), "feed_files")

    def feed_device(self, ptr: int, nbytes: int, last: bool = True) -> None:
        check(self._lib.emp_job_feed_fastq_device(self.handle, ptr, nbytes, int(last)), "feed_device")

    def run(self, stream: int = 0) -> None:
        check(self._lib.emp_job_run(self.handle, stream or None), "emp_job_run")

    def status(self) -> int:
        """Status of the last run (EMP_E_STATE while there is none)."""
        return int(self._lib.emp_job_status(self.handle))

    def output(self) -> bytes:
        n = ctypes.c_uint64()
        check(self._lib.emp_job_output_size(self.handle, ctypes.byref(n)), "output_size")
        buf = ctypes.create_string_buffer(max(1, n.value))
        check(self._lib.emp_job_output_copy(self.handle, buf, n.value), "output_copy")
        return buf.raw[: n.value]

    def output_into(self, arr: np.ndarray) -> int:
        n = ctypes.c_uint64()
        check(self._lib.emp_job_output_size(self.handle, ctypes.byref(n)), "output_size")
        if arr.nbytes < n.value:
            raise ValueError("output array too small")
        check(self._lib.emp_job_output_copy(self.handle, arr.ctypes.data, arr.nbytes), "output_copy")
        return int(n.value)

    def edges(self) -> list[tuple[int, np.ndarray, np.ndarray]]:
        """The last run's records through emp_job_edges: (ovlp_len, from, to) each."""
        out = []

        def sink(_user, ovlp, n, frm, to):
            out.append((int(ovlp), np.ctypeslib.as_array(frm, (n,)).copy() if n else np.zeros(0, np.uint32),
                        np.ctypeslib.as_array(to, (n,)).copy() if n else np.zeros(0, np.uint32)))
            return 0

        cb = _native.EDGE_SINK(sink)
        check(self._lib.emp_job_edges(self.handle, cb, None), "emp_job_edges")
        return out

    def stats(self) -> dict:
        st = _native.Stats()
        check(self._lib.emp_job_stats(self.handle, ctypes.byref(st)), "stats")
        return st.to_dict()

    def fingerprints(self) -> np.ndarray:
        n = ctypes.c_uint64()
        check(self._lib.emp_job_fingerprints(self.handle, None, 0, ctypes.byref(n)), "fingerprints")
        out = np.empty(n.value, dtype=np.uint64)
        if n.value:
            check(self._lib.emp_job_fingerprints(self.handle, out.ctypes.data, out.size, ctypes.byref(n)),
                  "fingerprints")
        return out


class Server:
    """An emp_server: continuous batching of submitted jobs on one Engine.

    submit() takes a fed Job; step() runs one scheduling step and returns the
    jobs that finished (each with status() set).  A job belongs to the server
    from submit() until a step returns it."""

    def __init__(self, engine: Engine, rounds_per_launch: int = 16, max_jobs: int = 256,
                 hbm_budget_bytes: int = 0, rounds_per_launch_idle: int = 64, batch_max_entries: int = 0,
                 share_min_entries: int = 8_000_000):
        self.engine = engine
        self._lib = engine._lib
        p = _native.ServerParams(int(rounds_per_launch), int(max_jobs), int(hbm_budget_bytes),
                                 int(rounds_per_launch_idle), int(batch_max_entries), int(share_min_entries))
        h = ctypes.c_void_p()
        check(self._lib.emp_server_create(engine.handle, ctypes.byref(p), ctypes.byref(h)), "emp_server_create")
        self.handle = h
        self._held: dict[int, "Job"] = {}
        self._out = (ctypes.c_void_p * 1024)()

    def submit(self, job: "Job") -> None:
        check(self._lib.emp_server_submit(self.handle, job.handle), "emp_server_submit")
        self._held[job.handle.value] = job

    def step(self) -> list["Job"]:
        n = ctypes.c_int()
        rc = self._lib.emp_server_step(self.handle, self._out, len(self._out), ctypes.byref(n))
        done = [self._held.pop(self._out[i]) for i in range(n.value)]
        check(rc, "emp_server_step")
        return done

    def stats(self) -> dict:
        st = _native.ServerStats()
        check(self._lib.emp_server_get_stats(self.handle, ctypes.byref(st)), "emp_server_get_stats")
        return {f: getattr(st, f) for f, _ in st._fields_}

    def counts(self) -> tuple[int, int, int]:
        q, f, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.emp_server_counts(self.handle, ctypes.byref(q), ctypes.byref(f), ctypes.byref(d)),
              "emp_server_counts")
        return q.value, f.value, d.value

    def close(self):
        if self.handle:
            self._lib.emp_server_destroy(self.handle)
            self.handle = None
            self._held.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Graph:
    """Unitigs of the overlap graph in an output.bin (emp_graph_*): read-ends
    as nodes, the records' edges; a unitig is a maximal path of edges
    u -> v with out-degree(u) = in-degree(v) = 1."""

    def __init__(self, engine: Engine, output_bin: bytes, n_reads: int):
        self._lib = engine._lib
        self.n_reads = int(n_reads)
        h = ctypes.c_void_p()
        buf = bytes(output_bin)
        check(self._lib.emp_graph_build(engine.handle, buf, len(buf), self.n_reads, ctypes.byref(h)),
              "emp_graph_build")
        self.handle = h

    def close(self):
        if self.handle:
            self._lib.emp_graph_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self) -> dict:
        st = _native.GraphStats()
        check(self._lib.emp_graph_get_stats(self.handle, ctypes.byref(st)), "emp_graph_get_stats")
        return st.to_dict()

    def unitigs(self) -> tuple[np.ndarray, np.ndarray]:
        """(read-ends in unitig order, each unitig's first position + the end)."""
        st = self.stats()
        order = np.zeros(max(1, st["nodes"]), dtype=np.uint32)
        starts = np.zeros(st["unitigs"] + 1, dtype=np.uint64)
        check(self._lib.emp_graph_unitigs(self.handle, order.ctypes.data, order.size, starts.ctypes.data,
                                          starts.size), "emp_graph_unitigs")
        return order[: st["nodes"]], starts

    def write_gfa(self, path: str, read_len: int) -> None:
        check(self._lib.emp_graph_write_gfa(self.handle, path.encode(), int(read_len)), "emp_graph_write_gfa")


SORT_STATIC_MAX_PAIRS = _native.SORT_STATIC_MAX_PAIRS


def sort_pairs_static(keys_ptr: int, vals_ptr: int, n: int, stream: int = 0) -> None:
    """Engine.sort_pairs on the current device without any allocation: the
    working set is the library's static device array, so n is at most
    SORT_STATIC_MAX_PAIRS, and calls whose GPU work overlaps race on it."""
    check(_native.lib().emp_sort_pairs_static(keys_ptr, vals_ptr, n, stream or None), "emp_sort_pairs_static")


def run_bytes(fastq, device: int = 0, engine: Engine | None = None, **params) -> tuple[bytes, dict]:
    """FASTQ bytes in host memory -> (output.bin bytes, stats)."""
    eng = engine or Engine(device)
    try:
        with eng.job(**params) as job:
            job.feed(fastq, last=True)
            job.run()
            return job.output(), job.stats()
    finally:
        if engine is None:
            eng.close()


def run_file(input_path: str, output_path: str, device: int = -1, **params) -> dict:
    """The reference program: read input_path, write output_path (main.cu:9-77)."""
    p = _params(**params)
    st = _native.Stats()
    check(_native.lib().emp_run_file(input_path.encode(), output_path.encode(), ctypes.byref(p), device,
                                     ctypes.byref(st)), "emp_run_file")
    return st.to_dict()


def _path_array(paths):
    if isinstance(paths, (str, bytes, os.PathLike)):
        paths = [paths]
    enc = [os.fsencode(p) for p in paths]
    return (ctypes.c_char_p * len(enc))(*enc)


def run_files(input_paths, output_path: str, device: int = -1, **params) -> dict:
    """run_file over the FASTQ of several files in order, each plain, gzip or BGZF."""
    p = _params(**params)
    st = _native.Stats()
    arr = _path_array(input_paths)
    check(_native.lib().emp_run_files(arr, len(arr), os.fsencode(output_path), ctypes.byref(p), device,
                                      ctypes.byref(st)), "emp_run_files")
    return st.to_dict()


def host_bytes(ptr: int, n: int) -> bytes:
    """A copy of n bytes of host memory at ptr, of any size (ctypes.string_at
    takes its size as a C int, so it fails from 2 GiB on)."""
    return (ctypes.c_char * n).from_address(ptr).raw if n else b""


def load_fastq(paths) -> bytes:
    """The FASTQ of files as a job reads them (plain, gzip, BGZF; in order,
    a newline added between files where one is missing), on the host."""
    arr = _path_array(paths)
    data = ctypes.c_void_p()
    n = ctypes.c_uint64()
    lib = _native.lib()
    check(lib.emp_fastq_load(arr, len(arr), ctypes.byref(data), ctypes.byref(n)), "emp_fastq_load")
    if not data.value:
        return b""
    try:
        return host_bytes(data.value, n.value)
    finally:
        lib.emp_free(data)


def measure_l2_read(nbytes: int = 64 << 20, device: int = -1) -> float:
    """The device's L2 read bandwidth in GB/s (emp_measure_l2_read)."""
    g = ctypes.c_double()
    check(_native.lib().emp_measure_l2_read(device, nbytes, ctypes.byref(g)), "emp_measure_l2_read")
    return g.value


def decode_output(data: bytes) -> list[tuple[int, np.ndarray, np.ndarray]]:
    """output.bin -> [(ovlp_len, from, to), ...] in file order."""
    recs = []
    off = 0
    mv = memoryview(data)
    while off < len(data):
        if off + 12 > len(data):
            raise ValueError("truncated record header")
        n, ovlp = struct.unpack_from("<Qi", data, off)
        off += 12
        if off + 8 * n > len(data):
            raise ValueError("truncated record body")
        frm = np.frombuffer(mv[off: off + 4 * n], dtype=np.uint32)
        to = np.frombuffer(mv[off + 4 * n: off + 8 * n], dtype=np.uint32)
        off += 8 * n
        recs.append((ovlp, frm, to))
    return recs
