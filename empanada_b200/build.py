"""In-tree build of the native parts (nvcc for sm_100a, g++, gcc).

Outputs (git-ignored, shipped with the tree):
  empanada_b200/libempanada_b200.so   kernels + C ABI (include/empanada.h)
  empanada_b200/_build/empanada       the command-line driver
  empanada_b200/libempanada_synth.so  seeded FASTQ generator (bench/test input)
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libempanada_b200.so")
CLI = os.path.join(BUILD, "empanada")
SYNTH = os.path.join(HERE, "libempanada_synth.so")

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
CU_SOURCES = ["k_scan.cu", "k_map.cu", "k_sort.cu", "k_sort_static.cu", "k_round.cu",
              "k_bucket.cu", "k_chunked.cu", "k_dedup.cu", "k_graph.cu", "k_probe.cu", "engine.cu"]
CXX_SOURCES = ["ingest.cpp"]  # FASTQ files: plain, gzip, BGZF (zlib)


def _run(cmd: list[str]) -> str:
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{p.stdout}")
    return p.stdout


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(ROOT, "include", "empanada.h")]


def build_native(verbose: bool = False, ptxas_info: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_info:
            cmd = [NVCC] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            jobs.append(cmd)
    for src in CXX_SOURCES:  # host-only parts (g++)
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cpp", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include"), "-c", s,
                         "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz"])
    cli_src = os.path.join(CSRC, "cli.cpp")
    if _stale(CLI, [cli_src, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), cli_src, "-o", CLI,
              "-L", HERE, "-lempanada_b200", "-Wl,-rpath,$ORIGIN/.."])
    synth_src = os.path.join(CSRC, "synth_reads.c")
    if _stale(SYNTH, [synth_src]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-o", SYNTH, synth_src])


def build_oracle(with_reference: bool | None = None) -> None:
    """Checker side: the C restatement, and the reference itself when its sources are present."""
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"])
    # the reference's sources: EMP_REFERENCE_DIR, else a `reference` directory beside the repository
    ref = os.environ.get("EMP_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")
    if with_reference is None:
        with_reference = os.path.isdir(ref)
    if with_reference and shutil.which("g++"):
        _run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-cpu", f"REF={ref}"])
        if os.path.exists(NVCC):
            _run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-gpu", f"REF={ref}"])


if __name__ == "__main__":
    build_native(verbose=True)
    build_oracle()
