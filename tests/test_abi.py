"""The C-ABI library loads without a GPU and exports every function include/c3d_b200.h and
include/c3d_solver.h declare (no compute calls here)."""
import ctypes
import os
import re

import c3d

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(name="c3d_b200.h"):
    text = open(os.path.join(REPO, "include", name)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip and not n.isupper()})


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(c3d.LIB_PATH)
    declared = header_functions()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(c3d.HEADER_SYMBOLS) == declared


def test_library_exports_solver_header_symbols():
    lib = ctypes.CDLL(c3d.LIB_PATH)
    declared = [n for n in header_functions("c3d_solver.h") if n.startswith("c3d_solver_")]
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(c3d.SOLVER_SYMBOLS) == declared


def test_no_device_reports_error_not_abort():
    """Without a device, creating a context returns an error code (no abort, no fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            return
    except Exception:
        pass
    q = c3d.quadrature(1, 4)
    try:
        c3d.Context(nx=4, ny=4, nz=4, nm=q["nm"], nq=q["nq"], dx=0.5, dy=0.5, dz=0.5, M=q["M"],
                    w=q["w"], xi=q["xi"], eta=q["eta"], mu=q["mu"])
    except c3d.C3DError as e:
        assert "NO_DEVICE" in str(e) or "CUDA" in str(e)
    else:
        raise AssertionError("context creation without a device must fail")


def test_library_exports_serve_header_symbols():
    lib = ctypes.CDLL(c3d.LIB_PATH)
    declared = [n for n in header_functions("c3d_serve.h") if n.startswith("c3d_server_")]
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(c3d.SERVE_SYMBOLS) == declared


def test_serve_footprint_estimate():
    """The admission test's device-memory estimate grows with the grid and the order."""
    from oracle_lib import deck_text
    small = c3d.Server.estimate(deck_text(NX=8, NY=8, NZ=8, MOMENT_ORDER=1, QUAD_ORDER=4))
    big = c3d.Server.estimate(deck_text(NX=32, NY=32, NZ=32, MOMENT_ORDER=5, QUAD_ORDER=16))
    assert 0 < small < big
