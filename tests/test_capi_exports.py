"""The C-ABI shared library loads on a machine without a GPU and exports every entry
point declared in include/*.h; the Python binding binds exactly those names."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

import sph_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(sph_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(sph_b200.LIB_PATH), "build the engine first (make)"
    lib = ctypes.CDLL(sph_b200.LIB_PATH)  # loads without a GPU
    declared = declared_functions()
    assert len(declared) >= 30
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", sph_b200.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T sph_" in l}
    assert declared <= exported
    assert set(sph_b200.EXPORTS) <= declared


def test_status_strings_without_a_device():
    lib = sph_b200.lib()
    for code in range(10):
        assert lib.sph_status_string(code)


def test_create_fails_loudly_without_a_device(tmp_path):
    # no CPU fallback: on a machine without a usable GPU sph_create reports SPH_ERR_CUDA
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import sph_input

    path = str(tmp_path / "input")
    sph_input.write_input(path, N=(16, 16), overlap=4.0)
    with pytest.raises(sph_b200.SphError) as e:
        sph_b200.System(path)
    assert e.value.status == "SPH_ERR_CUDA"


def test_class_system_shim_exports_every_member_function():
    """libsph_class_system.so defines every member function include/sph_class_system.h
    declares (the reference's class_system interface, src/class_system.h:145-650)."""
    shim = os.path.join(os.path.dirname(sph_b200.LIB_PATH), "libsph_class_system.so")
    assert os.path.exists(shim), "build the engine first (make)"
    ctypes.CDLL(shim)  # loads (and finds libsph_b200.so) without a GPU
    text = open(os.path.join(ROOT, "include", "sph_class_system.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = text[text.index("struct class_system {"):]
    methods = set(re.findall(r"^\s+(?:int|void|sph_ctx\*)\s+(\w+)\(", body, flags=re.M))
    assert {"read_input", "initialize", "neighbours_search", "calculate_forces",
            "V_Verlet_step1", "V_Verlet_step2", "print_output", "destructor"} <= methods
    out = subprocess.run(["nm", "-DC", "--defined-only", shim], capture_output=True, text=True,
                         check=True).stdout
    defined = set(re.findall(r"class_system::(\w+)\(", out))
    assert methods <= defined, sorted(methods - defined)


def test_drivers_are_built():
    lib_dir = os.path.dirname(sph_b200.LIB_PATH)
    assert os.access(os.path.join(lib_dir, "sph_run"), os.X_OK)
