"""The C ABI: every function include/*.h declares is exported by the library
that implements it (no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENGINE = os.path.join(REPO, "higflow_b200", "lib", "libhigflow_b200.so")
BINDING = os.path.join(REPO, "oracle", "_ref", "libhigflow_ref2d.so")


def _declared(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*\b(hf_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def _exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_engine_library_loads_and_exports_its_header():
    if not os.path.exists(ENGINE):
        pytest.skip("engine library not built")
    C.CDLL(ENGINE)   # loads without a GPU: the CUDA driver is opened on first use
    names = _declared("higflow_b200.h")
    assert len(names) > 30
    missing = sorted(set(names) - _exported(ENGINE))
    assert not missing, missing


def test_binding_exports_the_higflow_facing_header():
    if not os.path.exists(BINDING):
        pytest.skip("binding build (oracle/_ref) not present")
    names = _declared("higflow_b200_higflow.h")
    assert set(names) >= {"hf_flatten", "hf_attach", "hf_step", "hf_sync_to_host", "hf_sync_to_device", "hf_detach",
                          "hf_solver_step"}
    missing = sorted(set(names) - _exported(BINDING))
    assert not missing, missing
    # the link-time interposition targets for the case main loop
    assert {"__wrap_higflow_solver_step", "__wrap_higflow_solver_step_viscoelastic"} <= _exported(BINDING)
