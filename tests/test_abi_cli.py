"""Host-side checks that need no GPU: the C ABI library loads and exports every
function include/empanada.h declares, the size parser and defaults follow
config.h, and the `empanada` command reproduces the reference's argument
handling (config.h:10-140)."""
import ctypes
import os
import re
import subprocess

import pytest

import empanada_b200
from empanada_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "empanada.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(emp_[a-z_0-9]+)\s*\(", text, flags=re.M)))


def test_header_declarations_are_exported():
    names = declared_functions()
    assert len(names) >= 18
    lib = ctypes.CDLL(_native.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_native.SIGNATURES), "binding table out of sync with the header"


def test_abi_version_and_status_strings():
    lib = _native.lib()
    assert lib.emp_abi_version() == 6
    for code in range(0, -10, -1):
        assert lib.emp_status_string(code)
    assert _native.status_string(_native.EMP_E_FORMAT).startswith("reads of unequal length")


def test_params_default_matches_config_h():
    p = _native.Params()
    assert _native.lib().emp_params_default(ctypes.byref(p)) == 0
    assert (p.min_ovlp, p.map_mem, p.reduce_mem, p.base_blocksz, p.kv_chunksz) == (31, 1 << 30, 1 << 30, 32 << 20,
                                                                                   64 << 20)


def test_tuning_defaults_and_validation_without_a_gpu():
    """emp_tuning_default fills every choice; the context setters reject a
    missing context before touching a device."""
    t = _native.Tuning()
    lib = _native.lib()
    assert lib.emp_tuning_default(ctypes.byref(t)) == 0
    assert t.to_dict() == {"round_driver": 0, "bucket_mean": 2900, "region_cap": 2048, "dedup_driver": 0, "edge_cap": 0,
                           "wait_limit_ns": 20_000_000_000, "block_next_wait": 0, "map_streams": 8}
    assert lib.emp_tuning_default(None) == _native.EMP_E_INVAL
    assert lib.emp_ctx_set_tuning(None, ctypes.byref(t)) == _native.EMP_E_INVAL
    assert lib.emp_ctx_get_tuning(None, ctypes.byref(t)) == _native.EMP_E_INVAL


@pytest.mark.parametrize("s,v", [("31", 31), ("0", 0), ("1k", 1024), ("1K", 1024), ("16m", 16 << 20),
                                 ("12g", 12 << 30), ("8G", 8 << 30), ("5x", 5)])
def test_parse_size(s, v):
    assert empanada_b200.parse_size(s) == v


def test_parse_size_rejects_garbage():
    with pytest.raises(empanada_b200.EmpError):
        empanada_b200.parse_size("abc")


def test_python_parse_args_quirks():
    c = empanada_b200.parse_args(["in.fq", "out.bin"])
    assert (c.min_ovlp, c.reduce_mem, c.base_blocksz) == (31, 1 << 30, 32 << 20)
    c = empanada_b200.parse_args(["in.fq", "out.bin", "-o", "75", "-m", "8g", "-r", "12g", "-b", "16m", "-c", "64m"])
    assert (c.min_ovlp, c.map_mem, c.reduce_mem, c.base_blocksz, c.kv_chunksz) == (75, 8 << 30, 12 << 30, 16 << 20,
                                                                                   64 << 20)
    c = empanada_b200.parse_args(["in.fq", "out.bin", "xo", "40"])  # matched on the 2nd character
    assert c.min_ovlp == 40
    with pytest.raises(empanada_b200.UsageExit):
        empanada_b200.parse_args(["in.fq"])
    with pytest.raises(empanada_b200.UsageExit):
        empanada_b200.parse_args(["in.fq", "out.bin", "-z", "1"])
    with pytest.raises(empanada_b200.UsageExit):
        empanada_b200.parse_args(["in.fq", "out.bin", "--min-overlap", "1"])


def _cli(args, cwd=None):
    return subprocess.run([build.CLI] + args, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=cwd,
                          timeout=60)


def test_cli_usage_exits_zero():
    for args in ([], ["in.fq"], ["in.fq", "out.bin", "-z", "3"], ["in.fq", "out.bin", "--min-overlap", "3"]):
        p = _cli(args)
        assert p.returncode == 0, args
        assert p.stdout.strip().endswith("default = 64m")
        assert "Usage: assembly_v3 [input fastq] [output gfa] [options]" in p.stdout
    p = _cli(["in.fq", "out.bin", "-z", "3"])
    assert p.stdout.startswith("Invalid option -z")
    p = _cli(["in.fq", "out.bin", "--min-overlap", "3"])
    assert "Not implemented yet. Use short forms instead." in p.stderr


def test_cli_option_without_value_fails():
    p = _cli(["in.fq", "out.bin", "-o"])
    assert p.returncode == 1


def _gpu_usable() -> bool:
    ctx = ctypes.c_void_p()
    if _native.lib().emp_ctx_create(0, 0, ctypes.byref(ctx)) != 0:
        return False
    _native.lib().emp_ctx_destroy(ctx)
    return True


def test_cli_without_gpu_fails_cleanly(tmp_path):
    if _gpu_usable():
        pytest.skip("GPU present: the CLI runs under the GPU tests")
    fq = tmp_path / "in.fq"
    fq.write_bytes(b"@r0\nACGT\n+\nIIII\n")
    p = _cli([str(fq), str(tmp_path / "out.bin")], cwd=str(tmp_path))
    assert p.returncode == 1
    assert "CUDA error" in p.stderr


def test_engine_without_gpu_raises():
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("GPU present")
    with pytest.raises(empanada_b200.EmpError):
        empanada_b200.Engine(0)


def test_server_and_batch_arguments_without_a_gpu():
    """The serving and batch entry points validate their arguments before
    touching a device."""
    import ctypes

    from empanada_b200 import _native

    lib = _native.lib()
    p = _native.ServerParams()
    assert lib.emp_server_params_default(ctypes.byref(p)) == 0
    assert (p.rounds_per_launch, p.max_jobs, p.hbm_budget_bytes, p.rounds_per_launch_idle,
            p.batch_max_entries) == (16, 256, 0, 64, 0)
    out = ctypes.c_void_p()
    assert lib.emp_server_create(None, ctypes.byref(p), ctypes.byref(out)) == _native.EMP_E_INVAL
    assert lib.emp_server_submit(None, None) == _native.EMP_E_INVAL
    assert lib.emp_server_step(None, None, 0, None) == _native.EMP_E_INVAL
    assert lib.emp_server_destroy(None) == _native.EMP_E_INVAL
    assert lib.emp_batch_run(None, None, 0, None) == _native.EMP_E_INVAL
    assert lib.emp_job_status(None) == _native.EMP_E_INVAL


def test_l2_probe_rejects_a_tiny_buffer():
    """emp_measure_l2_read checks its arguments before touching a device."""
    g = ctypes.c_double()
    assert _native.lib().emp_measure_l2_read(-1, 8, ctypes.byref(g)) == -1  # EMP_E_INVAL
    assert _native.lib().emp_measure_l2_read(-1, 1 << 20, None) == -1


def test_integration_notes_cover_every_entry_point():
    """Every function include/empanada.h declares is described in INTEGRATION.md."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = [n for n in declared_functions() if n not in text]
    assert not missing, missing
