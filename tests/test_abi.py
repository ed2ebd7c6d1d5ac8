"""The C-ABI library loads and exports every entry point include/astrosim.h
declares; argument checking works without a GPU (no compute calls here)."""
import ctypes as C
import os
import re
import subprocess

import pytest

import astrosimgpu_cuda_b200 as asg
from astrosimgpu_cuda_b200 import abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(REPO, "include", f) for f in sorted(os.listdir(os.path.join(REPO, "include")))
           if f.endswith(".h")]


@pytest.fixture(scope="module")
def L():
    if not os.path.exists(asg.LIB_PATH):
        asg.build()
    return asg.lib()


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(astrosim_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_header_declares_core_entry_points():
    names = declared_functions()
    for core in ("astrosim_create", "astrosim_step", "astrosim_summary", "astrosim_destroy"):
        assert core in names


def test_library_exports_every_declared_symbol(L):
    out = subprocess.run(["nm", "-D", "--defined-only", asg.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(L, n)


def test_config_layout_and_defaults(L):
    cfg = abi.Config()
    L.astrosim_config_default(C.byref(cfg))
    assert cfg.struct_size == C.sizeof(abi.Config)
    ref = abi.default_config()
    for name, _ in abi.Config._fields_:
        a, b = getattr(cfg, name), getattr(ref, name)
        if name == "reserved":
            assert list(a) == list(b)
        elif isinstance(a, float) and a != a:
            assert b != b
        else:
            assert a == b, name
    assert L.astrosim_abi_version() == abi.ABI_VERSION


def test_null_and_bad_arguments_return_status(L):
    assert L.astrosim_step(None, 1) == abi.ERR_INVALID_ARG
    assert b"null" in L.astrosim_last_error()
    assert L.astrosim_summary(None, None) == abi.ERR_INVALID_ARG
    assert L.astrosim_destroy(None) == abi.OK
    shared = C.c_int(7)
    assert L.astrosim_ensemble_shared_constants(None, C.byref(shared)) == abi.ERR_INVALID_ARG
    assert shared.value == 7
    h = C.c_void_p()
    cfg = abi.default_config()
    cfg.struct_size = 4
    assert L.astrosim_create(C.byref(cfg), C.byref(h)) == abi.ERR_INVALID_ARG
    assert not h.value
    cfg = abi.default_config()
    cfg.reserved[0] = 1
    assert L.astrosim_create(C.byref(cfg), C.byref(h)) == abi.ERR_INVALID_ARG


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_no_device(L):
    h = C.c_void_p()
    cfg = abi.default_config(n_total=500)
    rc = L.astrosim_create(C.byref(cfg), C.byref(h))
    assert rc == abi.ERR_NO_DEVICE
    assert not h.value
    assert L.astrosim_device_info(0, None, 0, None, None) == abi.ERR_NO_DEVICE
    with pytest.raises(asg.AstrosimError):
        asg.Simulation(n_total=500)


def test_cli_help_and_unknown_flag():
    if not os.path.exists(asg.CLI_PATH):
        asg.build()
    r = subprocess.run([asg.CLI_PATH, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--n N_total" in r.stdout
    r = subprocess.run([asg.CLI_PATH, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown argument: --bogus" in r.stderr
    r = subprocess.run([asg.CLI_PATH, "--precision", "fp16"], capture_output=True, text=True)
    assert r.returncode == 1


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_cli_without_device_exits_1():
    r = subprocess.run([asg.CLI_PATH, "--n", "500", "--sim-ms", "1"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "N_total=500  N_E=400  N_I=100  N_A=100  p_primary=0.2" in r.stdout
