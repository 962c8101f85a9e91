"""CPU tests of the C ABI boundary (include/fip.h, libfip_b200.so).

No GPU needed: the library must load, export every entry point the header
declares (FIpipe with its C++ linkage, the reference's symbol), and reject
invalid arguments with a status before any device work.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import fastimagingpipe_b200 as fip

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "fip.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fip_\w+|FIpipe)\s*\(", text)))


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", fip.LIB_PATH], check=True,
                         capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_library_loads():
    assert fip.lib() is not None
    assert re.match(r"\d+\.\d+\.\d+", fip.version())


def test_every_declared_function_is_exported():
    syms = exported_symbols()
    names = declared_functions()
    assert "FIpipe" in names and len(names) > 15
    for name in names:
        if name == "FIpipe":
            # Same C++ signature as pipe_interface.cpp:8 -> same mangled name.
            assert "_Z6FIpipePfS_S_S_S_mmmfm" in syms
        else:
            assert name in syms, f"{name} declared in fip.h but not exported"


def test_status_strings():
    L = fip.lib()
    assert L.fip_status_string(0) == b"ok"
    assert L.fip_status_string(1) == b"invalid argument"
    assert L.fip_status_string(99) == b"unknown status"


@pytest.mark.parametrize("kw,needle", [
    (dict(image_size=6), "multiple of 4"),
    (dict(image_size=510), "multiple of 4"),
    (dict(unit_size=0), "unit_size"),
    (dict(unit_size=1024), "unit_size larger"),
    (dict(cell_size=0.0), "cell_size"),
    (dict(num_snapshots=2), "num_snapshots"),
    (dict(num_baselines=0), "num_baselines"),
])
def test_fipipe_rejects_bad_arguments(kw, needle):
    args = dict(num_baselines=10, image_size=64, num_snapshots=3, cell_size=1e-3, unit_size=16)
    args.update(kw)
    nb = max(args["num_baselines"], 1)
    ns = max(args["num_snapshots"], 1)
    vr = np.zeros(nb * ns, np.float32)
    B = np.zeros(nb * ns * 2, np.float32)
    V = np.tile(np.eye(3, dtype=np.float32).ravel(), ns)
    out = np.zeros(4096, np.float32)
    L = fip.lib()
    st = L.fip_pipe(vr.ctypes.data, vr.ctypes.data, B.ctypes.data, V.ctypes.data,
                    out.ctypes.data, args["num_baselines"], args["image_size"],
                    args["num_snapshots"], args["cell_size"], args["unit_size"])
    assert st == 1
    assert needle in L.fip_last_error().decode()


def test_null_pointers_rejected():
    L = fip.lib()
    assert L.fip_pipe(None, None, None, None, None, 10, 64, 3, 1e-3, 16) == 1
    assert L.fip_imager_destroy(None) == 0
    assert L.fip_trigger(None, None, None, None, None, None, None) == 1
    assert L.fip_plane_project(None, None, 1, 1, None, None, None) == 1


def test_imager_config_validation_before_device():
    cfg = fip.ImagerConfig(102, 10, 16, 1e-3, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    assert fip.lib().fip_imager_create(ctypes.byref(h), ctypes.byref(cfg)) == 1
    cfg = fip.ImagerConfig(64, 0, 16, 1e-3, 0, 0, 0, 0)
    assert fip.lib().fip_imager_create(ctypes.byref(h), ctypes.byref(cfg)) == 1
    cfg = fip.ImagerConfig(64, 10, 16, 1e-3, 7, 0, 0, 0)
    assert fip.lib().fip_imager_create(ctypes.byref(h), ctypes.byref(cfg)) == 1


def test_server_rejects_bad_arguments():
    h = ctypes.c_void_p()
    L = fip.lib()
    assert L.fip_server_create(ctypes.byref(h), 0, 1 << 30, 0, 16) == 1
    assert L.fip_server_create(None, 0, 1 << 30, 1, 16) == 1
    assert L.fip_server_destroy(None) == 0


def test_python_mirror_validates_sizes():
    with pytest.raises(ValueError):
        fip.FIpipe(np.zeros(5), np.zeros(5), np.zeros(10), np.zeros(27), 10, 64, 3, 1e-3, 16)


def test_cli_binary_is_built():
    assert os.access(fip.CLI_PATH, os.X_OK)
    r = subprocess.run([fip.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
