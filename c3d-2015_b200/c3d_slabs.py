"""x-slab decomposition of the M_N / P_N grid over ranks (one process per GPU).

The reference splits its grid into blocks over MPI ranks (src/init.cpp:125-186) and swaps
two ghost planes per face each RK stage (communicateBoundaries, src/comm.cpp:170-276). Here
the grid is split along x into slabs, one context per rank (c3d_set_x_halo_external), and
before each stage every slab sends its two first interior x-planes to its left neighbour's
high ghost planes and its two last interior planes to its right neighbour's low ghost planes
(periodic in x); the y and z ghosts are filled on the device as on one GPU. x-planes are
contiguous in the reference's layout, so the planes cross as single buffers (NCCL point to
point on device buffers, or gloo on host buffers). Only u crosses: the multipliers of the ghost
cells follow from solving them with the same moments and warm starts as their owners.
"""
import torch

__all__ = ["slab_bounds", "XHaloExchange", "exchange_local", "step_slabs_local", "step_slab"]


def slab_bounds(nx, world, rank):
    """Interior x-range [x0, x0 + n) of slab `rank` of `world` (sizes differ by at most 1)."""
    base, extra = divmod(nx, world)
    n = base + (1 if rank < extra else 0)
    return rank * base + min(rank, extra), n


class XHaloExchange:
    """Halo buffers and exchange of one slab context.

    ctx: a c3d.Context (or any object with copy_x_planes(field, i0, count, ptr, to_buf,
    device) and sync()); nx_local: the slab's interior x-size; plane_doubles:
    (ny + 4)(nz + 4) nm; device: buffers on the current GPU (NCCL) or on the host (gloo)."""

    TO_LOW, TO_HIGH = 0, 1  # message tags: planes bound for the receiver's low / high ghosts

    def __init__(self, ctx, nx_local, plane_doubles, rank=0, world=1, device=True):
        self.ctx, self.nx, self.rank, self.world, self.device = ctx, nx_local, rank, world, device
        self.left, self.right = (rank - 1) % world, (rank + 1) % world
        dev = torch.device("cuda", torch.cuda.current_device()) if device else torch.device("cpu")
        n = 2 * plane_doubles
        self.send_lo, self.send_hi, self.recv_lo, self.recv_hi = (
            torch.empty(n, dtype=torch.float64, device=dev) for _ in range(4))

    def pack(self):
        """Interior planes 2, 3 -> send_lo; nx, nx + 1 -> send_hi (ghost indices)."""
        c = self.ctx
        c.copy_x_planes(0, 2, 2, self.send_lo.data_ptr(), True, self.device)
        c.copy_x_planes(0, self.nx, 2, self.send_hi.data_ptr(), True, self.device)
        c.sync()

    def unpack(self):
        """recv_lo -> ghost planes 0, 1; recv_hi -> ghost planes nx + 2, nx + 3."""
        c = self.ctx
        c.copy_x_planes(0, 0, 2, self.recv_lo.data_ptr(), False, self.device)
        c.copy_x_planes(0, self.nx + 2, 2, self.recv_hi.data_ptr(), False, self.device)

    def start(self):
        """Starts the exchange of the packed planes with the neighbouring ranks
        (torch.distributed must be set up for world > 1) and returns its requests. Sends and
        receives are issued in the same order on every rank, so that with two ranks
        (left == right) they pair up correctly whatever the backend."""
        if self.world == 1:
            self.recv_lo.copy_(self.send_hi)
            self.recv_hi.copy_(self.send_lo)
            return []
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, self.send_hi, self.right, tag=self.TO_LOW),
               dist.P2POp(dist.irecv, self.recv_lo, self.left, tag=self.TO_LOW),
               dist.P2POp(dist.isend, self.send_lo, self.left, tag=self.TO_HIGH),
               dist.P2POp(dist.irecv, self.recv_hi, self.right, tag=self.TO_HIGH)]
        return dist.batch_isend_irecv(ops)

    def finish(self, reqs):
        """Waits for the exchange started by start() and fills the x ghost planes."""
        for r in reqs:
            r.wait()
        if self.device and reqs:
            torch.cuda.current_stream().synchronize()
        self.unpack()

    def exchange(self):
        """One halo exchange with the neighbouring ranks, blocking: pack, start, finish."""
        self.pack()
        self.finish(self.start())


def exchange_local(halos):
    """The same exchange among slabs held by one process (halos[r] for slab r): what each
    rank would receive, copied between the slabs' buffers."""
    for h in halos:
        h.pack()
    w = len(halos)
    for r, h in enumerate(halos):
        h.recv_lo.copy_(halos[(r - 1) % w].send_hi)
        h.recv_hi.copy_(halos[(r + 1) % w].send_lo)
    if halos and halos[0].device:
        torch.cuda.current_stream().synchronize()
    for h in halos:
        h.unpack()


def step_slab(ctx, halo, dt, overlap=True):
    """update(dt) of one rank's slab: a halo exchange before each RK stage. With overlap (M_N
    slab contexts) the exchange runs while the stage's first part (c3d_stage_part: the closure
    of the cells that need no halo) runs on the GPU: pack, start the exchange, part 0, finish
    the exchange (x ghosts filled), part 1. Results are the same either way."""
    for stage in (0, 1):
        if overlap:
            halo.pack()
            reqs = halo.start()
            ctx.stage_part(stage, dt, 0)
            halo.finish(reqs)
            ctx.stage_part(stage, dt, 1)
        else:
            halo.exchange()
            ctx.stage(stage, dt)


def step_slabs_local(ctxs, halos, dt, overlap=False):
    """update(dt) of all slabs held by one process (overlap: the split stage of step_slab,
    the planes packed before every slab's part 0)."""
    for stage in (0, 1):
        if not overlap:
            exchange_local(halos)
            for c in ctxs:
                c.stage(stage, dt)
            continue
        for h in halos:
            h.pack()
        for c in ctxs:
            c.stage_part(stage, dt, 0)
        w = len(halos)
        for r, h in enumerate(halos):
            h.recv_lo.copy_(halos[(r - 1) % w].send_hi)
            h.recv_hi.copy_(halos[(r + 1) % w].send_lo)
        if halos and halos[0].device:
            torch.cuda.current_stream().synchronize()
        for h in halos:
            h.unpack()
        for c in ctxs:
            c.stage_part(stage, dt, 1)
