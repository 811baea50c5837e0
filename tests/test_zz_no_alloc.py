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
closure parity tests). This file is named to be collected last.
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


def _noalloc(q, u, a0, dM, dw):
    import torch
    L = c3d.lib()
    L.c3d_closure_vectors_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_longlong,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.POINTER(ClosureOpts),
                                              ctypes.c_void_p]
    n, nm = u.shape
    du = torch.tensor(u, device="cuda")
    da = torch.tensor(a0, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    o = ClosureOpts()
    o.batched, o.maxIter, o.tol, o.tolGamma, o.condHMax = 1, 100, 1e-8, 1.1, 1e10
    o.nreg = len(LADDER)
    for i, r in enumerate(LADDER):
        o.reg[i] = r
    stream = torch.cuda.current_stream()
    rc = L.c3d_closure_vectors_noalloc(nm, q["nq"], dM.data_ptr(), dw.data_ptr(), n,
                                       du.data_ptr(), da.data_ptr(), it.data_ptr(),
                                       st.data_ptr(), ctypes.byref(o), stream.cuda_stream)
    c3d.check(rc, "c3d_closure_vectors_noalloc")
    torch.cuda.synchronize()
    return du.cpu().numpy(), da.cpu().numpy(), it.cpu().numpy(), st.cpu().numpy()


def test_noalloc_matches_existing_entry_point_twice():
    import torch
    q = c3d.quadrature(4, 20)  # M_4: 25 moments, 800 directions
    dM = torch.tensor(q["M"], device="cuda")
    dw = torch.tensor(q["w"], device="cuda")
    for call, seed in enumerate((11, 12)):  # two calls in a row, different vectors
        u, a0 = _vectors(q, 3000, seed)
        ue, ae, ite, ste = _existing(q, u, a0)
        un, an, itn, stn = _noalloc(q, u, a0, dM, dw)
        assert (stn == ste).all(), call
        assert (stn >= 0).all(), call
        assert np.array_equal(itn, ite), call
        for x, y in ((an, ae), (un, ue)):
            rel = np.linalg.norm(x - y, axis=1) / np.linalg.norm(y, axis=1)
            assert rel.max() <= 1e-10, (call, rel.max())
        assert ite.max() > 1  # the vectors need real Newton work


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    L = c3d.lib()
    L.c3d_closure_vectors_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_longlong,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.POINTER(ClosureOpts),
                                              ctypes.c_void_p]
    o = ClosureOpts()
    o.nreg, o.maxIter = 1, 10
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    rc = L.c3d_closure_vectors_noalloc(81, 800, p, p, 1, p, p, None, None, ctypes.byref(o), None)
    assert rc == 1 and "nm must be in [1, 64]" in L.c3d_last_error().decode()
    rc = L.c3d_closure_vectors_noalloc(25, 4096, p, p, 1, p, p, None, None, ctypes.byref(o), None)
    assert rc == 1 and "2048" in L.c3d_last_error().decode()
