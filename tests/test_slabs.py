"""x-slab decomposition: the halo exchange of c3d_slabs on two gloo ranks (CPU, host
buffers) against the periodic ghost fill of the whole grid, and (GPU) two slab contexts on
one device, exchanging planes through device buffers, against the single-domain step."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import c3d_slabs


class _HostSlab:
    """Host stand-in for a slab context: u as [nx + 4][ny + 4][nz + 4][nm]."""

    def __init__(self, u):
        self.u = np.ascontiguousarray(u)

    def copy_x_planes(self, field, i0, count, ptr, to_buf, device):
        assert field == 0 and not device
        plane = self.u[0].size
        a = self.u.reshape(self.u.shape[0], plane)[i0:i0 + count]
        if to_buf:
            ctypes.memmove(ptr, a.ctypes.data, a.nbytes)
        else:
            b = np.ctypeslib.as_array((ctypes.c_double * a.size).from_address(ptr))
            self.u.reshape(self.u.shape[0], plane)[i0:i0 + count] = b.reshape(count, plane)

    def sync(self):
        pass


class _HostStageSlab(_HostSlab):
    """_HostSlab with the split stage of c3d_stage_part: part 0 changes the interior planes
    (as a closure may regularise moments), part 1 records whether the x ghosts hold the
    neighbours' planes from before their part 0 -- want[stage]."""

    def __init__(self, u, n, want):
        super().__init__(u)
        self.n, self.want, self.ok = n, want, []

    def stage_part(self, stage, dt, part):
        n = self.n
        if part == 0:
            self.u[2:n + 2] *= 2.0
        else:
            ghosts = np.concatenate([self.u[0:2], self.u[n + 2:n + 4]])
            ref = np.concatenate([self.want[stage][0:2], self.want[stage][n + 2:n + 4]])
            self.ok.append(bool(np.array_equal(ghosts, ref)))


def _global_periodic(u, nx):
    g = u.copy()
    g[0:2] = u[nx:nx + 2]
    g[nx + 2:nx + 4] = u[2:4]
    return g


def _worker(rank, world, port, nx, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        ny, nz, nm = 3, 4, 2
        u = rng.standard_normal((nx + 4, ny + 4, nz + 4, nm))
        x0, n = c3d_slabs.slab_bounds(nx, world, rank)
        slab = _HostSlab(u[x0:x0 + n + 4].copy())
        slab.u[0:2] = np.nan
        slab.u[n + 2:n + 4] = np.nan
        h = c3d_slabs.XHaloExchange(slab, n, (ny + 4) * (nz + 4) * nm, rank, world, device=False)
        h.exchange()
        want = _global_periodic(u, nx)[x0:x0 + n + 4]
        ok = bool(np.array_equal(slab.u, want))
        # the overlapped step: planes packed before part 0, exchanged while it runs, the
        # ghosts filled before part 1 (stage s sees the planes of 2^s u)
        wants = [_global_periodic(f * u, nx)[x0:x0 + n + 4] for f in (1.0, 2.0)]
        st = _HostStageSlab(u[x0:x0 + n + 4].copy(), n, wants)
        st.u[0:2] = np.nan
        st.u[n + 2:n + 4] = np.nan
        hs = c3d_slabs.XHaloExchange(st, n, (ny + 4) * (nz + 4) * nm, rank, world, device=False)
        c3d_slabs.step_slab(st, hs, 0.1, overlap=True)
        q.put((rank, ok and st.ok == [True, True]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nx", [(2, 9), (3, 7)])
def test_halo_exchange_gloo(world, nx):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nx, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res[r] for r in range(world)), res


def test_slab_bounds():
    assert [c3d_slabs.slab_bounds(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]


@pytest.mark.gpu
@pytest.mark.parametrize("overlap", [False, True])
def test_two_slabs_on_one_gpu_equal_single_domain(oracle, overlap):
    """Two x-slabs of an 8^3 M_2 grid, stepped with the halo exchange (overlap: the split
    stage, c3d_stage_part, with the planes exchanged between its parts): interiors bit for bit
    equal to the single-domain run after two steps."""
    from test_gpu_kernels import _setup
    import c3d
    S = _setup(oracle, N=2, Q=12, steps_before=1)
    n, nm, T = S["n"], S["nm"], S["T"]
    ladder = (0.0, 1e-3, 1e-2, 1e-1, 5e-1)
    kw = dict(nm=nm, nq=S["nq"], dx=S["dx"], dy=S["dx"], dz=S["dx"], M=T["M"], w=T["w"],
              xi=T["xi"], eta=T["eta"], mu=T["mu"], ladder=ladder)
    U = S["u"].reshape(n + 4, n + 4, n + 4, nm)
    A = S["alpha"].reshape(n + 4, n + 4, n + 4, nm)
    sig = S["sig"].reshape(n + 4, n + 4, n + 4)
    g = c3d.Context(nx=n, ny=n, nz=n, **kw)
    g.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    with pytest.raises(c3d.C3DError, match="slab"):
        g.stage_part(0, S["dt"], 0)  # the split stage belongs to slab contexts
    ctxs, halos, bounds = [], [], []
    for r in range(2):
        x0, nl = c3d_slabs.slab_bounds(n, 2, r)
        c = c3d.Context(nx=nl, ny=n, nz=n, **kw)
        c.set_x_halo_external(True)
        sl = slice(x0, x0 + nl + 4)
        c.set_state(u=U[sl].ravel(), alpha=A[sl].ravel(), sig_t=sig[sl].ravel(),
                    sig_s=sig[sl].ravel())
        ctxs.append(c)
        halos.append(c3d_slabs.XHaloExchange(c, nl, (n + 4) * (n + 4) * nm, device=True))
        bounds.append((x0, nl))
    for _ in range(2):
        g.step(S["dt"])
        c3d_slabs.step_slabs_local(ctxs, halos, S["dt"], overlap=overlap)
    g.sync()
    ug, _ = g.get_state()
    ug = ug.reshape(n + 4, n + 4, n + 4, nm)
    inner = slice(2, n + 2)
    for c, (x0, nl) in zip(ctxs, bounds):
        c.sync()
        us, _ = c.get_state()
        us = us.reshape(nl + 4, n + 4, n + 4, nm)
        assert np.array_equal(us[2:nl + 2, inner, inner], ug[2 + x0:2 + x0 + nl, inner, inner])
        c.close()
    g.close()
