"""Z-slab decomposition of a periodic 3-D box over ranks (one GPU per rank).

No reference counterpart: LB-Cube steps one domain on one device. Here rank
r of W owns planes [r nz/W, (r+1) nz/W) of a periodic nx x ny x nz box as an
ordinary [Q, nz/W, ny, nx] population field. Each step needs, from each
neighbour, the populations that cross the shared face (5 of 19 for D3Q19, 9 of
27 for D3Q27); the step kernel reads them from halo buffers and writes the
outgoing ones to send buffers in the same pass (lbm_step_slab_async), and one
exchange per step moves every send buffer into the neighbour's halo buffer:

    halo_lo(r) <- send_hi(r - 1)        halo_hi(r) <- send_lo(r + 1)

DistributedExchange does that with torch.distributed point-to-point (NCCL on
GPUs, gloo on CPU tensors); HostExchange stages device face buffers through
host memory for a gloo process group (ranks without NCCL, or several ranks
sharing one device); LocalExchange does it between slabs held by one process.
SlabDomain.step overlaps the exchange of step n with the interior planes of
step n + 1 on a second stream; only the two face planes wait for it. A box
stepped as slabs is bit-identical to the same box stepped whole with
lbm_step_async.

ReactiveSlabDomain does the same for the coupled fluid + A + B -> C step of
lbm_fluid_reaction_ab_async (one face buffer per side carries the fluid's
crossing populations and one D3Q7 plane per species), and reduces the
reactive statistics over ranks: each rank sums its cells into five FP64
values, an all-reduce adds them, and every rank forms the same diagnostics.
"""
from __future__ import annotations

import lbcube as E

Q_OF = {"D3Q19": 19, "D3Q27": 27}


def face_elems(lattice: str, nx: int, ny: int) -> int:
    return E.load().lbm_slab_face_elems(E.LATTICES[lattice], nx, ny)


class SlabDomain:
    """One rank's slab: extents, face buffers and the step launches."""

    def __init__(self, torch, lattice, real, collision, nx, ny, nz_global, omega, rank, world, device):
        if lattice not in Q_OF:
            raise ValueError("slab decomposition needs a 3-D fluid lattice (D3Q19, D3Q27)")
        if nz_global % world != 0:
            raise ValueError(f"nz = {nz_global} is not divisible by {world} ranks")
        self.torch = torch
        self.lattice, self.real, self.collision = lattice, real, collision
        self.nx, self.ny, self.nz = nx, ny, nz_global // world
        self.z0 = rank * self.nz
        self.rank, self.world = rank, world
        self.omega = float(omega)
        dtype = torch.float32 if real == "float" else torch.float64
        n = face_elems(lattice, nx, ny)
        self.halo_lo, self.halo_hi, self.send_lo, self.send_hi = (
            torch.empty(n, dtype=dtype, device=device) for _ in range(4))
        self.comm = torch.cuda.Stream(device=device) if torch.device(device).type == "cuda" else None

    def shape(self):
        return (Q_OF[self.lattice], self.nz, self.ny, self.nx)

    def pack(self, f, stream=None):
        """Face populations of state ``f`` into the send buffers."""
        E.check(E.load().lbm_slab_pack_async(E.LATTICES[self.lattice], E.REALS[self.real], f.data_ptr(),
                                             self.nx, self.ny, self.nz, self.send_lo.data_ptr(),
                                             self.send_hi.data_ptr(), E._stream(stream)), "slab pack")

    def launch(self, cur, nxt, z_begin, z_end, stream=None):
        E.check(E.load().lbm_step_slab_async(
            E.LATTICES[self.lattice], E.REALS[self.real], E.COLLISIONS[self.collision], cur.data_ptr(),
            nxt.data_ptr(), self.nx, self.ny, self.nz, self.omega, self.halo_lo.data_ptr(),
            self.halo_hi.data_ptr(), self.send_lo.data_ptr(), self.send_hi.data_ptr(), z_begin, z_end,
            E._stream(stream)), "slab step")

    def ranges(self):
        """(interior, faces): plane ranges that need no halo, and those that do."""
        if self.nz <= 2:
            return [], [(0, self.nz)]
        return [(1, self.nz - 1)], [(0, 1), (self.nz - 1, self.nz)]

    def compute(self, cur, nxt, stream=None):
        """All planes of one step (the halos must already hold this step's data)."""
        interior, faces = self.ranges()
        for z0, z1 in interior + faces:
            self.launch(cur, nxt, z0, z1, stream)

    def step(self, cur, nxt, exchange):
        """One step with the exchange of its face populations overlapped with
        the next step's interior planes (CUDA: compute on the current stream,
        exchange on self.comm)."""
        torch = self.torch
        if self.comm is None:
            self.compute(cur, nxt)
            exchange.exchange(self)
            return
        s = torch.cuda.current_stream()
        interior, faces = self.ranges()
        for z0, z1 in interior:
            self.launch(cur, nxt, z0, z1, s)
        s.wait_stream(self.comm)  # this step's halos have arrived, the last sends have left
        for z0, z1 in faces:
            self.launch(cur, nxt, z0, z1, s)
        self.comm.wait_stream(s)  # the sends of this step are written
        with torch.cuda.stream(self.comm):
            exchange.exchange(self)

    def prime(self, f, exchange):
        """Initial halos from the initial state (before the first step)."""
        torch = self.torch
        if self.comm is None:
            self.pack(f)
            exchange.exchange(self)
            return
        s = torch.cuda.current_stream()
        self.pack(f, s)
        self.comm.wait_stream(s)
        with torch.cuda.stream(self.comm):
            exchange.exchange(self)

    def finish(self):
        """Make the current stream wait for the exchange in flight."""
        if self.comm is not None:
            self.torch.cuda.current_stream().wait_stream(self.comm)


class ReactiveSlabDomain(SlabDomain):
    """One rank's slab of the coupled fluid + A + B -> C step
    (lbm_fluid_reaction_slab_async): the fluid, species A and B of planes
    [z0, z0 + nz) of one periodic box, one face buffer per side for all three."""

    def __init__(self, torch, lattice, real, collision, nx, ny, nz_global, omega, omega_c, k, rank, world,
                 device):
        super().__init__(torch, lattice, real, collision, nx, ny, nz_global, omega, rank, world, device)
        self.omega_c, self.k = float(omega_c), float(k)
        dtype = torch.float32 if real == "float" else torch.float64
        n = E.load().lbm_fluid_reaction_slab_face_elems(E.LATTICES[lattice], nx, ny)
        self.halo_lo, self.halo_hi, self.send_lo, self.send_hi = (
            torch.empty(n, dtype=dtype, device=device) for _ in range(4))
        self.partials_bytes = E.stats_partials_bytes(lattice, nx, ny, self.nz)
        self.partials = torch.empty(self.partials_bytes // 8, dtype=torch.float64, device=device)

    def pack(self, state, stream=None):
        """Face populations of state (fluid, a, b) into the send buffers."""
        f, a, b = state
        E.check(E.load().lbm_fluid_reaction_slab_pack_async(
            E.LATTICES[self.lattice], E.REALS[self.real], f.data_ptr(), a.data_ptr(), b.data_ptr(), self.nx,
            self.ny, self.nz, self.send_lo.data_ptr(), self.send_hi.data_ptr(), E._stream(stream)), "slab pack")

    def launch(self, cur, nxt, z_begin, z_end, stream=None, stats=False):
        (cf, ca, cb), (nf, na, nb) = cur, nxt
        E.check(E.load().lbm_fluid_reaction_slab_async(
            E.LATTICES[self.lattice], E.REALS[self.real], E.COLLISIONS[self.collision], cf.data_ptr(),
            nf.data_ptr(), ca.data_ptr(), na.data_ptr(), cb.data_ptr(), nb.data_ptr(), self.nx, self.ny,
            self.nz, self.omega, self.omega_c, self.k, self.halo_lo.data_ptr(), self.halo_hi.data_ptr(),
            self.send_lo.data_ptr(), self.send_hi.data_ptr(), z_begin, z_end,
            self.partials.data_ptr() if stats else None, self.partials_bytes if stats else 0,
            E._stream(stream)), "coupled slab step")

    def compute(self, cur, nxt, stream=None, stats=False):
        """All planes of one step; with stats, the statistics partials of the new fields too."""
        interior, faces = self.ranges()
        for z0, z1 in interior + faces:
            self.launch(cur, nxt, z0, z1, stream, stats)

    def rank_sums(self, stream=None):
        """This rank's five FP64 statistics sums (C_A, C_B, C_A^2, C_B^2, C_A C_B
        over its cells) from the partials of the last compute(..., stats=True)."""
        sums = self.torch.empty(5, dtype=self.torch.float64, device=self.partials.device)
        E.check(E.load().lbm_reactive_stats_sums_async(E.LATTICES[self.lattice], self.nx, self.ny, self.nz,
                                                       self.partials.data_ptr(), self.partials_bytes,
                                                       sums.data_ptr(), E._stream(stream)), "statistics sums")
        return sums

    def statistics(self, dist=None, group=None, stream=None):
        """The eight reactive diagnostics of the whole box: this rank's sums,
        all-reduced over the ranks when a process group is given (a gloo group
        reduces a host copy), then the diagnostics of the totals. A device
        tensor of 8 doubles, the same on every rank."""
        sums = self.rank_sums(stream)
        if dist is not None and self.world > 1:
            if dist.get_backend(group) == "gloo" and sums.is_cuda:
                host = sums.cpu()
                dist.all_reduce(host, op=dist.ReduceOp.SUM, group=group)
                sums.copy_(host)
            else:
                dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
        return diagnostics_from_sums(self.torch, self.real, sums, self.nx * self.ny * self.nz * self.world,
                                     self.k, stream)


def diagnostics_from_sums(torch, real, sums, cells, k, stream=None):
    """The eight reactive diagnostics (mean_A, mean_B, var_A, var_B, covariance,
    segregation intensity, true and mixed reaction rates) from the five FP64
    sums over `cells` cells, k taken in the population precision."""
    out = torch.empty(8, dtype=torch.float64, device=sums.device)
    E.check(E.load().lbm_reactive_stats_from_sums_async(E.REALS[real], sums.data_ptr(), float(cells), float(k),
                                                        out.data_ptr(), E._stream(stream)), "statistics")
    return out


class HostExchange:
    """Face exchange for a gloo process group whose ranks hold device face
    buffers: each send buffer is copied to host memory, moved by
    torch.distributed point-to-point (gloo), and the received faces are copied
    into the device halo buffers. For ranks without NCCL, or several ranks on
    one device (the kernels never wait on another rank: every transfer
    completes on the host between launches)."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group
        self._host = None

    def exchange(self, d: SlabDomain):
        torch = d.torch
        if self._host is None:
            self._host = [torch.empty(d.send_lo.shape, dtype=d.send_lo.dtype) for _ in range(4)]
        s_hi, s_lo, h_lo, h_hi = self._host
        s_hi.copy_(d.send_hi)
        s_lo.copy_(d.send_lo)
        if d.world == 1:
            h_lo.copy_(s_hi)
            h_hi.copy_(s_lo)
        else:
            dist = self.dist
            up, down = (d.rank + 1) % d.world, (d.rank - 1) % d.world
            ops = [dist.P2POp(dist.isend, s_hi, up, self.group), dist.P2POp(dist.isend, s_lo, down, self.group),
                   dist.P2POp(dist.irecv, h_lo, down, self.group), dist.P2POp(dist.irecv, h_hi, up, self.group)]
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        d.halo_lo.copy_(h_lo)
        d.halo_hi.copy_(h_hi)


class DistributedExchange:
    """Face exchange between ranks with torch.distributed point-to-point.

    Per pair of ranks the sends and receives are posted in the same order on
    both sides, so the k-th send to a peer lands in the k-th receive from it:
    send_hi goes up and send_lo down; halo_lo comes from below, halo_hi from
    above. With two ranks 'up' and 'down' are the same peer and the order
    (send_hi, send_lo) / (halo_lo, halo_hi) pairs them correctly."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group

    def exchange(self, d: SlabDomain):
        if d.world == 1:
            d.halo_lo.copy_(d.send_hi)
            d.halo_hi.copy_(d.send_lo)
            return
        dist = self.dist
        up, down = (d.rank + 1) % d.world, (d.rank - 1) % d.world
        ops = [dist.P2POp(dist.isend, d.send_hi, up, self.group),
               dist.P2POp(dist.isend, d.send_lo, down, self.group),
               dist.P2POp(dist.irecv, d.halo_lo, down, self.group),
               dist.P2POp(dist.irecv, d.halo_hi, up, self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class LocalExchange:
    """Face exchange between the slabs of one process (all ranks emulated on
    one device: the copies stand in for the point-to-point transfers)."""

    def __init__(self, domains):
        self.domains = domains

    def exchange_all(self):
        W = len(self.domains)
        for r, d in enumerate(self.domains):
            d.halo_lo.copy_(self.domains[(r - 1) % W].send_hi)
            d.halo_hi.copy_(self.domains[(r + 1) % W].send_lo)
