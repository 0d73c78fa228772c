"""CPU checks of the C ABI: the library builds, loads and exports every declared entry point.

No compute is issued: without a GPU only host-side calls run.
"""
import ctypes
import os
import re
import subprocess

import pytest

from solunar_b200 import build as slf_build
from solunar_b200.abi import CReport, CSettings, FluidSettings

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "solunar_fluid.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(slf_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    return slf_build.build()


def test_every_declared_entry_point_is_exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (slf_[a-z0-9_]+)$", out, flags=re.M))
    declared = declared_functions()
    assert declared, "no declarations parsed"
    missing = [f for f in declared if f not in exported]
    assert not missing, missing


def test_the_library_loads_and_links_no_shared_cudart(lib_path):
    L = ctypes.CDLL(lib_path)
    for name in declared_functions():
        assert hasattr(L, name), name
    deps = subprocess.run(["ldd", lib_path], capture_output=True, text=True).stdout
    assert "libcudart" not in deps


def test_the_settings_struct_matches_the_header(lib_path):
    L = ctypes.CDLL(lib_path)
    L.slf_settings_default.argtypes = [ctypes.POINTER(CSettings)]
    c = CSettings()
    assert L.slf_settings_default(ctypes.byref(c)) == 0
    d = FluidSettings.from_c(c)
    # FluidSettings::default (src/fluid/mod.rs:80-95) and the DFSPH constants (dfsph.rs:8-16)
    ref = FluidSettings()
    for field in ("spacing", "rest_density", "support", "max_particles", "sound_speed", "viscosity", "courant",
                  "max_substeps", "min_iterations", "max_iterations"):
        assert getattr(d, field) == pytest.approx(getattr(ref, field)), field
    assert d.gravity == pytest.approx((0.0, -9.81, 0.0))
    assert d.divergence_tolerance == pytest.approx(1e-3) and d.density_tolerance == pytest.approx(5e-4)
    assert ctypes.sizeof(CSettings) == 88  # sizeof(slf_settings) as gcc lays it out
    assert ctypes.sizeof(CReport) == 40


def test_null_arguments_are_refused_without_a_device(lib_path):
    L = ctypes.CDLL(lib_path)
    L.slf_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.slf_last_error.restype = ctypes.c_char_p
    assert L.slf_create(None, None) == 9
    assert b"null" in L.slf_last_error()
