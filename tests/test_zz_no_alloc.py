"""The allocation-free closure entry point (c3d_closure_vectors_noalloc).

It serves callers that may not call cudaMalloc themselves, such as an application
that owns all device memory through its own pre-reserved pool, or a latency-critical
caller that must avoid the implicit synchronisation of cudaMalloc/cudaFree. Its scratch
lives in a static device array of at most C3D_NOALLOC_SCRATCH_BYTES, which limits it to
nm <= 64 moments and nq <= 2048 directions.

The test allocates the inputs and outputs (the caller's job), calls the entry point
through the C ABI twice in a row on different vectors, and checks each call against the
context-based c3d_closure_vectors on the same inputs: identical Newton iteration counts
and statuses, multipliers and moments within 1e-10 relative (the tolerance of the
closure parity tests). It also checks that a call leaves the device's free memory and
torch's reserved pool unchanged, compares a call with the C oracle on its own (iteration
counts except rounding ties, multipliers 1e-10), runs the largest sizes the static array accepts
(nm = 64, nq = 2048, which fill it to its last byte), and reads a call's outcome with
c3d_closure_vectors_noalloc_check. This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import c3d

pytestmark = pytest.mark.gpu


class ClosureOpts(ctypes.Structure):
    _fields_ = [("batched", ctypes.c_int), ("maxIter", ctypes.c_int), ("tol", ctypes.c_double),
                ("tolGamma", ctypes.c_double), ("condHMax", ctypes.c_double),
                ("nreg", ctypes.c_int), ("reg", ctypes.c_double * 16)]


LADDER = (0.0, 1e-3, 1e-2, 1e-1, 5e-1)


def _vectors(q, n, seed):
    """Realizable moment vectors u = <m e^{alpha.m}> from seeded multipliers."""
    rng = np.random.default_rng(seed)
    nm, nq = q["nm"], q["nq"]
    M = q["M"].reshape(nq, nm)
    a = rng.standard_normal((n, nm)) * np.exp(rng.uniform(np.log(0.05), np.log(1.5), (n, 1)))
    a[:, 0] = 0.0
    u = (np.exp(a @ M.T) * q["w"]) @ M
    u *= np.exp(rng.uniform(-3, 3, (n, 1)))  # arbitrary densities
    a0 = np.zeros((n, nm))
    a0[:, 0] = np.sqrt(4 * np.pi) * np.log(u[:, 0] / np.sqrt(4 * np.pi))
    return u, a0


def _existing(q, u, a0):
    import torch
    n, nm = u.shape
    ctx = c3d.Context(nx=1, ny=1, nz=1, nm=nm, nq=q["nq"], dx=1.0, dy=1.0, dz=1.0, M=q["M"],
                      w=q["w"], xi=q["xi"], eta=q["eta"], mu=q["mu"], ladder=LADDER, tol=1e-8)
    ctx.set_engine(1)  # the persistent direct-form kernel, which the allocation-free entry runs
    du = torch.tensor(u, device="cuda")
    da = torch.tensor(a0, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.closure_vectors_device(n, du.data_ptr(), da.data_ptr(), it.data_ptr(), None, None,
                               st.data_ptr())
    ctx.sync()
    out = du.cpu().numpy(), da.cpu().numpy(), it.cpu().numpy(), st.cpu().numpy()
    ctx.close()
    return out


def _lib():
    L = c3d.lib()
    L.c3d_closure_vectors_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_longlong,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.POINTER(ClosureOpts),
                                              ctypes.c_void_p]
    L.c3d_closure_vectors_noalloc_check.argtypes = [ctypes.c_void_p,
                                                    ctypes.POINTER(ctypes.c_longlong)]
    return L


def _opts():
    o = ClosureOpts()
    o.batched, o.maxIter, o.tol, o.tolGamma, o.condHMax = 1, 100, 1e-8, 1.1, 1e10
    o.nreg = len(LADDER)
    for i, r in enumerate(LADDER):
        o.reg[i] = r
    return o


def _check(L, stream):
    failed = ctypes.c_longlong(-1)
    rc = L.c3d_closure_vectors_noalloc_check(stream, ctypes.byref(failed))
    return rc, failed.value


def _noalloc(q, u, a0, dM, dw):
    import torch
    L = _lib()
    n, nm = u.shape
    du = torch.tensor(u, device="cuda")
    da = torch.tensor(a0, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    o = _opts()
    stream = torch.cuda.current_stream()
    rc = L.c3d_closure_vectors_noalloc(nm, q["nq"], dM.data_ptr(), dw.data_ptr(), n,
                                       du.data_ptr(), da.data_ptr(), it.data_ptr(),
                                       st.data_ptr(), ctypes.byref(o), stream.cuda_stream)
    c3d.check(rc, "c3d_closure_vectors_noalloc")
    rc, failed = _check(L, stream.cuda_stream)
    c3d.check(rc, "c3d_closure_vectors_noalloc_check")
    assert failed == 0
    torch.cuda.synchronize()
    return du.cpu().numpy(), da.cpu().numpy(), it.cpu().numpy(), st.cpu().numpy()


def _compare(q, n, seed, dM, dw):
    u, a0 = _vectors(q, n, seed)
    ue, ae, ite, ste = _existing(q, u, a0)
    un, an, itn, stn = _noalloc(q, u, a0, dM, dw)
    assert (stn == ste).all()
    assert (stn >= 0).all()
    assert np.array_equal(itn, ite)
    for x, y in ((an, ae), (un, ue)):
        rel = np.linalg.norm(x - y, axis=1) / np.linalg.norm(y, axis=1)
        assert rel.max() <= 1e-10, rel.max()
    return ite


def test_noalloc_matches_existing_entry_point_twice():
    import torch
    q = c3d.quadrature(4, 20)  # M_4: 25 moments, 800 directions
    dM = torch.tensor(q["M"], device="cuda")
    dw = torch.tensor(q["w"], device="cuda")
    for call, seed in enumerate((11, 12)):  # two calls in a row, different vectors
        ite = _compare(q, 3000, seed, dM, dw)
        assert ite.max() > 1, call  # the vectors need real Newton work


def test_noalloc_matches_oracle(oracle):
    """The entry point against the C oracle (the reference's batched closure restated) on 400
    M_4 vectors, on its own: identical Newton iteration counts and statuses except rounding
    ties (the oracle's margins), multipliers within 1e-10 relative on the other vectors."""
    import torch
    from oracle_lib import log_ties, make_opts, tie_cells
    q = c3d.quadrature(4, 20)
    T = oracle.tables(4, 20)
    assert np.array_equal(T["M"], q["M"])
    dM = torch.tensor(q["M"], device="cuda")
    dw = torch.tensor(q["w"], device="cuda")
    u, a0 = _vectors(q, 400, 13)
    un, an, itn, stn = _noalloc(q, u, a0, dM, dw)
    uo, ao = u.copy(), a0.copy()
    ro = oracle.closure(make_opts(q["nm"], q["nq"], batched=True, tol=1e-8, ladder=LADDER), T,
                        uo, ao)
    ties = tie_cells(ro)
    assert np.array_equal(stn, ro["status"])
    mism = itn != ro["totalIter"]
    log_ties("test_noalloc_matches_oracle", ties, mism)
    assert not (mism & ~ties).any(), int((mism & ~ties).sum())
    ok = ~ties & (ro["status"] == 0)
    rel = np.linalg.norm(an[ok] - ao[ok], axis=1) / np.linalg.norm(ao[ok], axis=1)
    assert ok.sum() > 150, (int(ok.sum()), int(ties.sum()))  # ~1/3 are ties at MN_TOL 1e-8
    assert rel.max() <= 1e-10, rel.max()
    assert itn.max() > 1


def test_noalloc_largest_sizes():
    """nm = 64 (M_7) and nq = 2048 (Q = 32): the basis fills the static array to its end."""
    import torch
    q = c3d.quadrature(7, 32)
    assert (q["nm"], q["nq"]) == (64, 2048)
    dM = torch.tensor(q["M"], device="cuda")
    dw = torch.tensor(q["w"], device="cuda")
    for seed in (21, 22):
        _compare(q, 300, seed, dM, dw)


def test_noalloc_allocates_nothing():
    """After a first call, a second call changes neither the device's free memory
    (cudaMemGetInfo) nor torch's reserved pool."""
    import torch
    L = _lib()
    q = c3d.quadrature(4, 20)
    u, a0 = _vectors(q, 2000, 31)
    n, nm = u.shape
    dM = torch.tensor(q["M"], device="cuda")
    dw = torch.tensor(q["w"], device="cuda")
    du = torch.tensor(u, device="cuda")
    da = torch.tensor(a0, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    o = _opts()
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        rc = L.c3d_closure_vectors_noalloc(nm, q["nq"], dM.data_ptr(), dw.data_ptr(), n,
                                           du.data_ptr(), da.data_ptr(), it.data_ptr(),
                                           st.data_ptr(), ctypes.byref(o), stream)
        c3d.check(rc, "c3d_closure_vectors_noalloc")
        c3d.check(_check(L, stream)[0], "c3d_closure_vectors_noalloc_check")

    call()  # first call: set-up (symbol address) and module loading
    du.copy_(torch.tensor(u, device="cuda"))
    da.copy_(torch.tensor(a0, device="cuda"))
    torch.cuda.synchronize()
    free1, reserved1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
    call()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free1
    assert torch.cuda.memory_reserved() == reserved1
    assert (st.cpu().numpy() == 0).all()


def test_noalloc_reports_failed_cells():
    """A vector with u0 <= 0 gets status 1 and the call's outcome is C3D_ERR_CLOSURE with
    one failed cell; the check clears the record, so the next check reports C3D_OK."""
    import torch
    L = _lib()
    q = c3d.quadrature(2, 12)
    u, a0 = _vectors(q, 64, 41)
    u[5, 0] = -1.0
    n, nm = u.shape
    dM = torch.tensor(q["M"], device="cuda")
    dw = torch.tensor(q["w"], device="cuda")
    du = torch.tensor(u, device="cuda")
    da = torch.tensor(a0, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.c3d_closure_vectors_noalloc(nm, q["nq"], dM.data_ptr(), dw.data_ptr(), n,
                                       du.data_ptr(), da.data_ptr(), None, st.data_ptr(),
                                       ctypes.byref(_opts()), stream)
    c3d.check(rc, "c3d_closure_vectors_noalloc")
    rc, failed = _check(L, stream)
    assert rc == 4 and failed == 1, (rc, failed)  # C3D_ERR_CLOSURE
    s = st.cpu().numpy()
    assert s[5] == 1 and (np.delete(s, 5) == 0).all()
    assert _check(L, stream) == (0, 0)


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    L = _lib()
    o = _opts()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    rc = L.c3d_closure_vectors_noalloc(81, 800, p, p, 1, p, p, None, None, ctypes.byref(o), None)
    assert rc == 1 and "nm must be in [1, 64]" in L.c3d_last_error().decode()
    rc = L.c3d_closure_vectors_noalloc(25, 4096, p, p, 1, p, p, None, None, ctypes.byref(o), None)
    assert rc == 1 and "2048" in L.c3d_last_error().decode()
    for field, bad in (("maxIter", 0), ("tol", 0.0), ("tol", float("nan")), ("condHMax", -1.0),
                       ("tolGamma", float("inf"))):
        o = _opts()
        setattr(o, field, bad)
        rc = L.c3d_closure_vectors_noalloc(25, 800, p, p, 1, p, p, None, None, ctypes.byref(o),
                                           None)
        assert rc == 1 and "positive and finite" in L.c3d_last_error().decode(), field
