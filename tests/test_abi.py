"""The C-ABI library loads and exports every entry point of include/jfb200.h;
the ctypes struct mirrors match the C layouts (CPU only, no GPU calls)."""

import ctypes
import os
import re
import subprocess

import pytest

from jaxfun_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "jfb200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jfb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_abi():
    names = declared_functions()
    assert "jfb_kmm_advance" in names and "jfb_wavenumber_solve" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert lib.jfb_version() >= 1


def test_argument_errors_are_reported_without_a_gpu():
    lib = _lib.load()
    cfg = _lib.KMMConfig()
    cfg.nx, cfg.ny, cfg.nz = 3, 16, 16  # invalid nx: rejected before any CUDA call
    h = ctypes.c_void_p()
    st = lib.jfb_kmm_create(ctypes.byref(cfg), ctypes.byref(h))
    assert st == _lib.JFB_ERR_ARG
    assert b"out of range" in lib.jfb_last_error() or b"family" in lib.jfb_last_error()


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("abi")
    exe = str(d / "abi_layout")
    subprocess.run(["gcc", "-O1", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "abi_layout.c")], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return dict(line.split() for line in out.strip().splitlines())


@pytest.mark.parametrize("cname, cls", [("jfb_kmm_config", _lib.KMMConfig),
                                        ("jfb_kmm_state", _lib.KMMStateC),
                                        ("jfb_kmm_info", _lib.KMMInfo),
                                        ("jfb_mhd_state", _lib.MHDStateC),
                                        ("jfb_mhd_params", _lib.MHDParams),
                                        ("jfb_tps_config", _lib.TPSConfig),
                                        ("jfb_kmm_variant", _lib.KMMVariant)])
def test_struct_layouts_match_c(c_layout, cname, cls):
    assert int(c_layout[cname]) == ctypes.sizeof(cls)
    for key, off in c_layout.items():
        if key.startswith(cname + "."):
            field = key.split(".", 1)[1]
            assert getattr(cls, field).offset == int(off), key


def test_mhd_argument_errors_are_reported_without_a_gpu():
    lib = _lib.load()
    cfg = _lib.KMMConfig()
    cfg.nx, cfg.ny, cfg.nz = 17, 16, 16
    cfg.nonlinear_form = _lib.JFB_NONLINEAR_GRADIENT
    h = ctypes.c_void_p()
    prm = _lib.MHDParams()
    prm.eta = 1.0 / 400.0
    assert lib.jfb_mhd_create(ctypes.byref(cfg), ctypes.byref(prm), ctypes.byref(h)) == _lib.JFB_ERR_ARG
    assert b"rotational" in lib.jfb_last_error()
    cfg.nonlinear_form = _lib.JFB_NONLINEAR_ROTATIONAL
    prm.eta = -1.0
    assert lib.jfb_mhd_create(ctypes.byref(cfg), ctypes.byref(prm), ctypes.byref(h)) == _lib.JFB_ERR_ARG
    assert b"eta" in lib.jfb_last_error()
    assert lib.jfb_ensemble_create(None, 0, ctypes.byref(h)) == _lib.JFB_ERR_ARG
