"""Gaunt tables built on the device (c3d_gaunt_build) against the host build of the
reference's algorithm (src/init.cpp:288-336, restated in host/tables.c and built into the
C oracle):

* the dense table within 1e-13 of the largest |beta| (the device sums in another order);
* the CSR at the sparse deck's threshold 1e-13: the same row pointers, columns and values
  (within the same bound), every entry far from the threshold on both builds;
* a closure on the device-built sparse table against the oracle on the host-built one:
  iteration counts equal except rounding ties, multipliers within 1e-10.
"""
import numpy as np
import pytest

import c3d
from oracle_lib import log_ties, make_opts, tie_cells
from test_gpu_kernels import _ctx, _setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,Q", [(2, 12), (4, 12), (6, 28)])
def test_gaunt_tables_match_host_build(oracle, N, Q):
    T = oracle.tables(N, Q, gaunt=True)
    nm, nm2, nq = T["nm"], T["nm2"], T["nq"]
    beta, row, col, val = c3d.gaunt_build(nm, nm2, nq, T["M2"], 1e-13)
    ref = T["beta"].reshape(nm * nm, nm2)
    scale = np.abs(ref).max()
    assert np.abs(beta - ref).max() <= 1e-13 * scale, np.abs(beta - ref).max() / scale
    # no host entry lies within the bound above of the threshold, so both builds keep the
    # same entries (the largest dropped noise entry is 1.1e-14 at N = 6)
    near = (np.abs(ref) > 5e-14) & (np.abs(ref) < 2e-13)
    assert not near.any(), int(near.sum())
    assert np.array_equal(row, T["betaRow"])
    nnz = int(row[-1])
    assert np.array_equal(col, T["betaCol"][:nnz])
    assert np.abs(val - T["betaVal"][:nnz]).max() <= 1e-13 * scale


def test_gaunt_build_count_only_and_capacity(oracle):
    T = oracle.tables(2, 12, gaunt=True)
    nm, nm2, nq = T["nm"], T["nm2"], T["nq"]
    L = c3d.lib()
    nnz = c3d.ctypes.c_longlong(-1)
    M2 = np.ascontiguousarray(T["M2"])
    st = L.c3d_gaunt_build(nm, nm2, nq, M2.ctypes.data_as(c3d._dp), 1e-13, None, None, 0, None,
                           None, c3d.ctypes.byref(nnz))
    assert st == c3d.C3D_OK and nnz.value == int(T["betaRow"][-1])
    row = np.zeros(nm * nm + 1, np.int32)
    col, val = np.zeros(4, np.int32), np.zeros(4)
    st = L.c3d_gaunt_build(nm, nm2, nq, M2.ctypes.data_as(c3d._dp), 1e-13, None,
                           row.ctypes.data_as(c3d._ip), 4, col.ctypes.data_as(c3d._ip),
                           val.ctypes.data_as(c3d._dp), c3d.ctypes.byref(nnz))
    assert c3d.STATUS_NAMES[st] == "INVALID" and b"capacity" in L.c3d_last_error()


def test_closure_on_device_built_tables(oracle):
    N, Q = 4, 12
    S = _setup(oracle, N=N, Q=Q, steps_before=2)
    T = oracle.tables(N, Q, gaunt=True)
    S["T"] = T
    ctx = _ctx(S)
    _, row, col, val = c3d.gaunt_build(T["nm"], T["nm2"], T["nq"], T["M2"], 1e-13)
    ctx.set_gaunt(T["nm2"], T["M2"], row, col, val)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    ctx.sync()
    ug, ag = ctx.get_state()
    rec = ctx.records()
    nm = S["nm"]
    uo = S["u"].reshape(-1, nm).copy()
    ao = S["alpha"].reshape(-1, nm).copy()
    out = oracle.closure(make_opts(nm, S["nq"], nm2=T["nm2"], hess_mode=2), T, uo, ao)
    assert (rec["status"] == 0).all()
    ties = tie_cells(out)
    mism = rec["iters"] != out["totalIter"]
    log_ties("test_closure_on_device_built_tables", ties, mism)
    assert not (mism & ~ties).any(), np.nonzero(mism & ~ties)[0][:10]
    ok = ~ties & (rec["regIndex"] == out["regIndex"])
    ag = ag.reshape(-1, nm)
    rel = np.linalg.norm(ag[ok] - ao[ok], axis=1) / np.linalg.norm(ao[ok], axis=1)
    assert rel.max() < 1e-10, rel.max()
    ctx.close()
