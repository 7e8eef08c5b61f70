"""The drop-in command (empanada_b200/_build/empanada, the reference's
`input.fastq output.bin -o/-m/-r/-b/-c` CLI, main.cu:9-77 and
config.h:120-140) and emp_run_file on a GPU: exit status, output.bin bytes
against the digests of the reference's own build (tests/golden), the
timings.csv side file, and the error exits."""
import ctypes
import hashlib
import json
import os
import subprocess

import pytest

from cases import BY_NAME, CASES

import empanada_b200
from empanada_b200 import _native, build

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))
CLI_CASES = [c.name for c in CASES if (not c.big or c.name == "small") and c.name in GOLDEN
             and GOLDEN[c.name].get("sha256")]


def _cli(args, cwd):
    return subprocess.run([build.CLI] + list(args), cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                          text=True, timeout=600)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CLI_CASES)
def test_cli_writes_the_reference_output(tmp_path, name):
    case = BY_NAME[name]
    fq = tmp_path / "in.fq"
    fq.write_bytes(case.fastq())
    p = _cli([str(fq), "out.bin"] + list(case.args), cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr
    out = (tmp_path / "out.bin").read_bytes()
    g = GOLDEN[name]
    assert len(out) == g["size"]
    assert hashlib.sha256(out).hexdigest() == g["sha256"]
    t = (tmp_path / "timings.csv").read_text().splitlines()
    assert t[0].startswith("## ") and t[1] == "Phase,Time (us)"
    assert {line.split(",")[0] for line in t[2:]} >= {"read_input_h2d", "map_phase", "sort_unique", "overlap_rounds",
                                                     "total_device"}
    assert not p.stderr.strip(), p.stderr


@pytest.mark.gpu
def test_cli_missing_input_gives_empty_output(tmp_path):
    """A missing input file reads as empty, as the reference's ifstream does."""
    p = _cli([str(tmp_path / "absent.fq"), "out.bin"], cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr
    assert (tmp_path / "out.bin").read_bytes() == b""


@pytest.mark.gpu
def test_cli_unreadable_input_and_output_fail(tmp_path):
    """An input path that is not a readable file (a directory), or an output
    that cannot be created, exits 1 with one ERROR line and no output."""
    (tmp_path / "dir.fq").mkdir()
    p = _cli([str(tmp_path / "dir.fq"), "out.bin"], cwd=str(tmp_path))
    assert p.returncode == 1
    errs = [line for line in p.stderr.splitlines() if "ERROR" in line]
    assert len(errs) == 1, p.stderr
    assert not (tmp_path / "out.bin").exists()
    fq = tmp_path / "in.fq"
    fq.write_bytes(BY_NAME["tiny"].fastq())
    p = _cli([str(fq), str(tmp_path / "no_such_dir" / "out.bin")], cwd=str(tmp_path))
    assert p.returncode == 1
    assert len([line for line in p.stderr.splitlines() if "ERROR" in line]) == 1, p.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "split_r128k", "out_of_core_r4k", "n_reads", "empty_input"])
def test_run_file_matches_reference(tmp_path, name):
    """emp_run_file (the C ABI's whole program) on a file, read in chunks
    through two pinned buffers."""
    case = BY_NAME[name]
    fq = tmp_path / "in.fq"
    fq.write_bytes(case.fastq())
    out = tmp_path / "out.bin"
    st = empanada_b200.run_file(str(fq), str(out), device=0, **dict(
        min_ovlp=case.min_ovlp(), reduce_mem=case.reduce_mem()))
    data = out.read_bytes()
    g = GOLDEN[name]
    assert hashlib.sha256(data).hexdigest() == g["sha256"]
    assert st["output_bytes"] == len(data)


@pytest.mark.gpu
def test_run_file_in_many_chunks(tmp_path):
    """A FASTQ larger than one 128 MiB read chunk goes through both pinned
    buffers several times (the golden 1.2M x 250 bp workload, 616 MB)."""
    case = BY_NAME["larger"]
    fq = tmp_path / "in.fq"
    fq.write_bytes(case.fastq())
    out = tmp_path / "out.bin"
    params = _native.Params()
    lib = _native.lib()
    assert lib.emp_params_default(ctypes.byref(params)) == 0
    a = list(case.args)
    params.min_ovlp = int(a[a.index("-o") + 1])
    params.map_mem = empanada_b200.parse_size(a[a.index("-m") + 1])
    params.reduce_mem = empanada_b200.parse_size(a[a.index("-r") + 1])
    params.base_blocksz = empanada_b200.parse_size(a[a.index("-b") + 1])
    params.kv_chunksz = empanada_b200.parse_size(a[a.index("-c") + 1])
    st = _native.Stats()
    rc = lib.emp_run_file(str(fq).encode(), str(out).encode(), ctypes.byref(params), 0, ctypes.byref(st))
    assert rc == 0
    data = out.read_bytes()
    assert hashlib.sha256(data).hexdigest() == GOLDEN["larger"]["sha256"]


def _records_split(data: bytes, parts: int) -> list[bytes]:
    """data cut into `parts` pieces at record boundaries (every fourth newline)."""
    nl = [i for i, c in enumerate(data) if c == 10][3::4]
    cuts = [nl[len(nl) * k // parts] + 1 for k in range(1, parts)] if len(nl) >= parts else []
    bounds = [0] + cuts + [len(data)]
    return [data[a:b] for a, b in zip(bounds, bounds[1:])]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["gzip", "bgzf"])
def test_cli_reads_compressed_input(tmp_path, kind):
    """The drop-in command on gzip and BGZF input writes the same output.bin
    as the reference on the plain file."""
    import gzip

    from test_ingest import bgzf

    case = BY_NAME["small"]
    data = case.fastq()
    fq = tmp_path / "in.fq.gz"
    fq.write_bytes(gzip.compress(data) if kind == "gzip" else bgzf(data))
    p = _cli([str(fq), "out.bin"] + list(case.args), cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr
    out = (tmp_path / "out.bin").read_bytes()
    assert hashlib.sha256(out).hexdigest() == GOLDEN["small"]["sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "n_reads", "split_r128k"])
def test_run_files_and_feed_files_match_reference(tmp_path, name):
    """emp_run_files and emp_job_feed_files over the case's FASTQ cut into a
    plain, a gzip and a BGZF file (at record boundaries)."""
    import gzip

    from test_ingest import bgzf

    case = BY_NAME[name]
    parts = _records_split(case.fastq(), 3)
    paths = []
    for k, (piece, enc) in enumerate(zip(parts, (lambda b: b, gzip.compress, bgzf))):
        q = tmp_path / f"part{k}"
        q.write_bytes(enc(piece))
        paths.append(str(q))
    g = GOLDEN[name]
    out = tmp_path / "out.bin"
    params = dict(min_ovlp=case.min_ovlp(), reduce_mem=case.reduce_mem())
    empanada_b200.run_files(paths, str(out), **params)
    assert hashlib.sha256(out.read_bytes()).hexdigest() == g["sha256"]
    with empanada_b200.Engine(0) as eng, eng.job(**params) as job:
        job.feed_files(paths)
        job.run()
        assert hashlib.sha256(job.output()).hexdigest() == g["sha256"]
