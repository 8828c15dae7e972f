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

ReactiveSlabGradient runs the checkpointed reactive gradient
(lbm_reactive_gradient_async) the same way: forward and adjoint steps on each
slab, face exchanges between them, and an all-reduce of the FP64 statistics and
gradient sums.
"""
from __future__ import annotations

import lbcube as E

Q_OF = {"D3Q19": 19, "D3Q27": 27}


def face_elems(lattice: str, nx: int, ny: int) -> int:
    return E.load().lbm_slab_face_elems(E.LATTICES[lattice], nx, ny)


class SlabDomain:
    """One rank's slab: extents, face buffers and the step launches. storage:
    None for populations in `real`, or a 16-bit format of lbcube.FORMATS
    (codes shifted by rho0; face buffers of codes)."""

    def __init__(self, torch, lattice, real, collision, nx, ny, nz_global, omega, rank, world, device,
                 storage=None, rho0=1.0):
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
        self.storage, self.rho0 = storage, float(rho0)
        dtype = (torch.float32 if real == "float" else torch.float64) if storage is None else torch.int16
        n = face_elems(lattice, nx, ny)
        self.halo_lo, self.halo_hi, self.send_lo, self.send_hi = (
            torch.empty(n, dtype=dtype, device=device) for _ in range(4))
        self.comm = torch.cuda.Stream(device=device) if torch.device(device).type == "cuda" else None

    def shape(self):
        return (Q_OF[self.lattice], self.nz, self.ny, self.nx)

    def pack(self, f, stream=None):
        """Face populations of state ``f`` into the send buffers."""
        lib = E.load()
        if self.storage is not None:
            rc = lib.lbm_slab_pack_shifted_async(E.LATTICES[self.lattice], f.data_ptr(), self.nx, self.ny, self.nz,
                                                 self.send_lo.data_ptr(), self.send_hi.data_ptr(), E._stream(stream))
        else:
            rc = lib.lbm_slab_pack_async(E.LATTICES[self.lattice], E.REALS[self.real], f.data_ptr(), self.nx,
                                         self.ny, self.nz, self.send_lo.data_ptr(), self.send_hi.data_ptr(),
                                         E._stream(stream))
        E.check(rc, "slab pack")

    def launch(self, cur, nxt, z_begin, z_end, stream=None):
        lib = E.load()
        if self.storage is not None:
            rc = lib.lbm_step_slab_shifted_async(
                E.LATTICES[self.lattice], E.FORMATS[self.storage], E.COLLISIONS[self.collision], cur.data_ptr(),
                nxt.data_ptr(), self.nx, self.ny, self.nz, self.omega, self.rho0, self.halo_lo.data_ptr(),
                self.halo_hi.data_ptr(), self.send_lo.data_ptr(), self.send_hi.data_ptr(), z_begin, z_end,
                E._stream(stream))
        else:
            rc = lib.lbm_step_slab_async(
                E.LATTICES[self.lattice], E.REALS[self.real], E.COLLISIONS[self.collision], cur.data_ptr(),
                nxt.data_ptr(), self.nx, self.ny, self.nz, self.omega, self.halo_lo.data_ptr(),
                self.halo_hi.data_ptr(), self.send_lo.data_ptr(), self.send_hi.data_ptr(), z_begin, z_end,
                E._stream(stream))
        E.check(rc, "slab step")

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


class ReactiveSlabGradient(ReactiveSlabDomain):
    """The checkpointed gradient of lbm_reactive_gradient_async on one rank's
    slab: J and dJ/dk, dJ/dtau, dJ/dtau_c of the whole box, and dJ/dA0,
    dJ/dB0, dJ/du0 on the rank's planes (native FP32 / FP64 states).

    The whole-box host sequence (adjoint_reactive.cu: reactive_gradient) runs
    on every rank with the slab entries of the C ABI; sequence() yields where
    the ranks meet: ("exchange",) for a face exchange (send -> halo buffers,
    as the forward step's), ("allreduce", t) for an in-place sum of the FP64
    device tensor t over ranks. run() serves those yields for one rank of a
    process group; run_local() steps the slabs of one process in lockstep.
    Per forward step one exchange, whose halos are kept with the state it
    produced; per adjoint step one (the adjoint scatter's sends) and an unpack
    of the received scatter faces. Given the same seed the adjoint fields and
    the initial-state gradients are bit-identical to the whole box's."""

    def __init__(self, torch, lattice, real, collision, objective, nx, ny, nz_global, tau, tau_c, k, steps, interval,
                 rank, world, device, storage=None, c0=0.5):
        super().__init__(torch, lattice, real, collision, nx, ny, nz_global, 1.0 / tau, 1.0 / tau_c, k, rank, world,
                         device)
        if steps < 1 or interval < 2:
            raise ValueError("need steps >= 1 and a checkpoint interval >= 2")
        if storage not in (None, "native") and real != "float":
            raise ValueError("16-bit states need real = 'float'")
        self.objective = objective
        self.storage = E._storage(storage)  # 0: states in `real`; else a 16-bit format code
        self.c0 = float(c0)
        self.tau, self.tau_c = float(tau), float(tau_c)
        self.steps, self.interval = int(steps), int(interval)
        self.total_cells = float(nx * ny * nz_global)
        dtype = torch.float32 if real == "float" else torch.float64
        sdtype = dtype if self.storage == 0 else torch.int16  # element of a stored state
        q = Q_OF[lattice]
        shape = (self.nz, ny, nx)
        self._dtype, self._device = dtype, device

        def field(qq, dt=dtype):
            return torch.empty((qq,) + shape, dtype=dt, device=device)

        n = E.load().lbm_fluid_reaction_slab_face_elems(E.LATTICES[lattice], nx, ny)

        def state():
            # fluid, A, B, the advecting velocity that produced it, and the two
            # halos the forward step that produced it received: every step that
            # pulls from the state (forward or adjoint) reads them, so the
            # backward sweep exchanges no state faces
            return (field(q, sdtype), field(7, sdtype), field(7, sdtype), field(3),
                    torch.empty(n, dtype=sdtype, device=device), torch.empty(n, dtype=sdtype, device=device))

        # face buffers: the states' sends (forward steps, packs; the received
        # halos land in the produced state's own halo buffers) and the
        # adjoint's scatter faces (in `real`); an exchange moves whichever set
        # is current in halo_lo / halo_hi / send_lo / send_hi
        self._lam_faces = (self.halo_lo, self.halo_hi, self.send_lo, self.send_hi)
        self._state_sends = (self.send_lo, self.send_hi) if self.storage == 0 else tuple(
            torch.empty(n, dtype=sdtype, device=device) for _ in range(2))

        nseg = (self.steps + self.interval - 1) // self.interval
        self.nseg = nseg
        self.ckpt = [state() for _ in range(nseg + 1)]
        self.seg = [state() for _ in range(self.interval)]
        self.lam = [(field(q), field(7), field(7)) for _ in range(2)]
        self.ubar = field(3)
        lib = E.load()
        L = E.LATTICES[lattice]
        self.slots_bytes = lib.lbm_reactive_slab_slots_bytes(L, nx, ny, self.nz)
        self.obj_bytes = lib.lbm_reactive_slab_objective_bytes(L, nx, ny, self.nz)
        if self.slots_bytes == 0 or self.obj_bytes == 0:
            raise ValueError("slab extents rejected by the engine")
        self.slots = torch.empty(self.slots_bytes // 8, dtype=torch.float64, device=device)
        self.obj_partials = torch.empty(self.obj_bytes // 8, dtype=torch.float64, device=device)
        self.diag = torch.zeros(8, dtype=torch.float64, device=device)
        self.sums = torch.empty(4, dtype=torch.float64, device=device)
        self.result = torch.empty(4, dtype=torch.float64, device=device)
        self._args = {}  # argument lists of the per-step entries, by buffer combination

    # ---- the per-step entries
    def _faces(self, target=None):
        """The face buffers of the next exchange: a state's (the states' sends
        in, `target`'s halos out) or, with no target, the adjoint's."""
        if target is None:
            self.halo_lo, self.halo_hi, self.send_lo, self.send_hi = self._lam_faces
        else:
            self.send_lo, self.send_hi = self._state_sends
            self.halo_lo, self.halo_hi = target[4], target[5]

    def pack(self, state, stream=None):
        """Faces of a stored state into the state send buffers (its halos come
        back into its own halo buffers at the next exchange)."""
        self._faces(state)
        f, a, b = state[:3]
        E.check(E.load().lbm_reactive_slab_pack_async(
            E.LATTICES[self.lattice], E.REALS[self.real], self.storage, f.data_ptr(), a.data_ptr(), b.data_ptr(),
            self.nx, self.ny, self.nz, self.send_lo.data_ptr(), self.send_hi.data_ptr(), E._stream(stream)),
            "reactive slab pack")

    # The argument lists of the per-step entries are built once per combination
    # of buffers (every buffer is allocated once, so its address is fixed): a
    # step then costs one foreign call, which keeps the host ahead of the GPU.
    def _call(self, key, fn, build, what):
        args = self._args.get(key)
        if args is None:
            args = self._args[key] = build()
        E.check(fn(*args), what)

    def _forward(self, cur, nxt, keep_u):
        """One step cur -> nxt (pulling across the faces from cur's halos); the
        next exchange delivers nxt's halos."""
        self._faces(nxt)
        lib = E.load()
        self._call(("f", id(cur), id(nxt), keep_u), lib.lbm_reactive_slab_forward_async, lambda: (
            E.LATTICES[self.lattice], E.REALS[self.real], self.storage, self.c0, E.COLLISIONS[self.collision],
            cur[0].data_ptr(), nxt[0].data_ptr(), cur[1].data_ptr(), nxt[1].data_ptr(), cur[2].data_ptr(),
            nxt[2].data_ptr(), nxt[3].data_ptr() if keep_u else None, self.nx, self.ny, self.nz, self.tau,
            self.tau_c, self.k, cur[4].data_ptr(), cur[5].data_ptr(), self.send_lo.data_ptr(),
            self.send_hi.data_ptr(), None), "reactive slab forward step")

    def _adjoint(self, sn, u_next, ln, l):
        # pulls from state n across the faces through its stored halos; writes the adjoint's sends
        self._faces()
        lib = E.load()
        self._call(("a", id(sn), id(u_next), id(ln), id(l)), lib.lbm_reactive_slab_adjoint_step_async, lambda: (
            E.LATTICES[self.lattice], E.REALS[self.real], self.storage, self.c0, E.COLLISIONS[self.collision],
            sn[0].data_ptr(), sn[1].data_ptr(), sn[2].data_ptr(), sn[4].data_ptr(), sn[5].data_ptr(),
            u_next.data_ptr(), ln[0].data_ptr(), ln[1].data_ptr(), ln[2].data_ptr(), l[0].data_ptr(),
            l[1].data_ptr(), l[2].data_ptr(), self.ubar.data_ptr(), self.send_lo.data_ptr(),
            self.send_hi.data_ptr(), self.nx, self.ny, self.nz, self.tau, self.tau_c, self.k, self.slots.data_ptr(),
            self.slots_bytes, None), "reactive slab adjoint step")

    def _unpack(self, l):
        self._faces()
        lib = E.load()
        self._call(("u", id(l)), lib.lbm_reactive_slab_adjoint_unpack_async, lambda: (
            E.LATTICES[self.lattice], E.REALS[self.real], self.halo_lo.data_ptr(), self.halo_hi.data_ptr(),
            l[0].data_ptr(), l[1].data_ptr(), l[2].data_ptr(), self.nx, self.ny, self.nz, None),
            "reactive slab adjoint unpack")

    def sequence(self, rho0, u0, a0, b0, grad_b0=True, grad_u0=True):
        """Generator of one rank's gradient (inputs: this rank's planes of
        rho0 [Z,Y,X], u0 [3,Z,Y,X], a0, b0 [Z,Y,X] on the device). Afterwards
        self.result holds J, dJ/dk, dJ/dtau, dJ/dtau_c and self.grad_a0 (and
        grad_b0, grad_u0 when asked) this rank's initial-state gradients."""
        torch, lib = self.torch, E.load()
        L, P = E.LATTICES[self.lattice], E.REALS[self.real]
        SL = E.LATTICES["D3Q7"]
        nx, ny, nz = self.nx, self.ny, self.nz
        steps, interval, nseg = self.steps, self.interval, self.nseg
        ckpt, seg = self.ckpt, self.seg
        for t in (rho0, a0, b0):
            assert tuple(t.shape) == (nz, ny, nx) and t.dtype == self._dtype and t.is_contiguous()
        assert tuple(u0.shape) == (3, nz, ny, nx) and u0.dtype == self._dtype and u0.is_contiguous()

        # forward: the equilibrium initial state, checkpoints every `interval`
        # steps, the last segment's states kept
        s0 = ckpt[0]
        # 16-bit states: the FP32 equilibrium in an adjoint buffer, then encoded
        fi, ai, bi = (s0[:3] if self.storage == 0 else self.lam[0])
        E.check(lib.lbm_init_equilibrium_async(L, P, rho0.data_ptr(), u0.data_ptr(), fi.data_ptr(), nx, ny, nz,
                                               None), "init")
        E.check(lib.lbm_init_equilibrium_async(SL, P, a0.data_ptr(), u0.data_ptr(), ai.data_ptr(), nx, ny, nz,
                                               None), "init")
        E.check(lib.lbm_init_equilibrium_async(SL, P, b0.data_ptr(), u0.data_ptr(), bi.data_ptr(), nx, ny, nz,
                                               None), "init")
        if self.storage != 0:
            for lat, src, dst, ref in ((L, fi, s0[0], 1.0), (SL, ai, s0[1], self.c0), (SL, bi, s0[2], self.c0)):
                E.check(lib.lbm_encode_shifted_async(lat, self.storage, P, src.data_ptr(), dst.data_ptr(), nx, ny,
                                                     nz, ref, None), "encode")
        self.pack(s0)
        yield ("exchange",)
        last0 = (nseg - 1) * interval
        cur = s0
        for n in range(steps):
            kept = True
            if n + 1 == steps or (n + 1) % interval == 0:
                nxt = ckpt[(n + interval) // interval]
            elif n + 1 > last0:
                nxt = seg[n + 1 - last0]
            else:
                nxt, kept = seg[n % 2], False
            self._forward(cur, nxt, kept)
            if n + 1 < steps:
                yield ("exchange",)
            cur = nxt

        # seed lambda^N (and the objective partials)
        lN = self.lam[steps % 2]
        if self.objective == "segregation":
            scratch = torch.empty(8, dtype=torch.float64, device=self._device)
            fa, fb = cur[1], cur[2]
            if self.storage != 0:  # statistics of the decoded final fields (the other adjoint buffer)
                tmp = self.lam[(steps + 1) % 2]
                for src, dst in ((cur[1], tmp[1]), (cur[2], tmp[2])):
                    E.check(lib.lbm_decode_shifted_async(SL, self.storage, P, src.data_ptr(), dst.data_ptr(), nx, ny,
                                                         nz, self.c0, None), "decode")
                fa, fb = tmp[1], tmp[2]
            E.check(lib.lbm_reactive_stats_async(SL, P, fa.data_ptr(), fb.data_ptr(), nx, ny, nz, self.k,
                                                 self.partials.data_ptr(), self.partials_bytes, scratch.data_ptr(),
                                                 None), "statistics")
            sums5 = self.rank_sums()
            yield ("allreduce", sums5)
            E.check(lib.lbm_reactive_stats_from_sums_async(P, sums5.data_ptr(), self.total_cells, self.k,
                                                           self.diag.data_ptr(), None), "statistics")
        obj = E.OBJECTIVES[self.objective]
        E.check(lib.lbm_reactive_slab_seed_async(
            L, P, self.storage, self.c0, obj, cur[1].data_ptr(), cur[2].data_ptr(), a0.data_ptr(), self.diag.data_ptr(), lN[0].data_ptr(),
            lN[1].data_ptr(), lN[2].data_ptr(), nx, ny, nz, self.total_cells, self.obj_partials.data_ptr(),
            self.obj_bytes, None), "reactive slab seed")
        self.slots.zero_()

        # backward sweep, segment by segment from the last
        for kk in range(nseg - 1, -1, -1):
            n0, n1 = kk * interval, min(steps, (kk + 1) * interval)
            if kk < nseg - 1:  # recompute the segment's states (and their halos) from its checkpoint
                src = ckpt[kk]
                for n in range(n0 + 1, n1):
                    self._forward(src, seg[n - n0], True)
                    yield ("exchange",)
                    src = seg[n - n0]
            for n in range(n1 - 1, n0 - 1, -1):
                sn = ckpt[kk] if n == n0 else seg[n - n0]
                sn1 = ckpt[kk + 1] if n + 1 == n1 else seg[n + 1 - n0]  # holds u^{n+1}
                ln, l = self.lam[(n + 1) % 2], self.lam[n % 2]
                self._adjoint(sn, sn1[3], ln, l)
                yield ("exchange",)
                self._unpack(l)

        # initial-state gradients and the four scalars
        l0 = self.lam[0]
        self.grad_a0 = torch.empty((nz, ny, nx), dtype=self._dtype, device=self._device)
        self.grad_b0 = torch.empty_like(self.grad_a0) if grad_b0 else None
        self.grad_u0 = torch.empty((3, nz, ny, nx), dtype=self._dtype, device=self._device) if grad_u0 else None
        E.check(lib.lbm_reactive_slab_init_gradients_async(
            L, P, obj, rho0.data_ptr(), u0.data_ptr(), a0.data_ptr(), b0.data_ptr(), l0[0].data_ptr(),
            l0[1].data_ptr(), l0[2].data_ptr(), nx, ny, nz, self.total_cells, self.grad_a0.data_ptr(),
            None if self.grad_b0 is None else self.grad_b0.data_ptr(),
            None if self.grad_u0 is None else self.grad_u0.data_ptr(), None), "reactive slab gradients")
        E.check(lib.lbm_reactive_slab_sums_async(L, nx, ny, nz, self.slots.data_ptr(), self.slots_bytes,
                                                 self.obj_partials.data_ptr(), self.obj_bytes, self.sums.data_ptr(),
                                                 None), "reactive slab sums")
        yield ("allreduce", self.sums)
        E.check(lib.lbm_reactive_slab_result_async(P, obj, self.sums.data_ptr(), self.diag.data_ptr(),
                                                   self.total_cells, self.tau_c, self.result.data_ptr(), None),
                "reactive slab result")

    def run(self, rho0, u0, a0, b0, exchange, dist=None, group=None, grad_b0=True, grad_u0=True):
        """One rank of a process group (exchange: HostExchange or
        DistributedExchange). Returns (result, grad_a0, grad_b0, grad_u0)."""
        for op in self.sequence(rho0, u0, a0, b0, grad_b0, grad_u0):
            if op[0] == "exchange":
                exchange.exchange(self)
            else:
                _all_reduce(dist, group, op[1], self.world)
        return self.result, self.grad_a0, self.grad_b0, self.grad_u0


def _all_reduce(dist, group, t, world):
    if world == 1:
        return
    if dist.get_backend(group) == "gloo" and t.is_cuda:
        host = t.cpu()
        dist.all_reduce(host, op=dist.ReduceOp.SUM, group=group)
        t.copy_(host)
    else:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def run_local(gradients, inputs, grad_b0=True, grad_u0=True):
    """The slabs of one process (every rank of the box), stepped in lockstep:
    LocalExchange for the exchanges, sums in rank order for the all-reduces.
    inputs[r] = (rho0, u0, a0, b0) of rank r's planes."""
    gens = [g.sequence(*inp, grad_b0=grad_b0, grad_u0=grad_u0) for g, inp in zip(gradients, inputs)]
    ex = LocalExchange(gradients)
    while True:
        ops = [next(gen, None) for gen in gens]
        if all(op is None for op in ops):
            break
        if any(op is None for op in ops) or len({op[0] for op in ops}) != 1:
            raise RuntimeError("slab ranks left the lockstep")
        if ops[0][0] == "exchange":
            ex.exchange_all()
        else:
            total = ops[0][1].clone()
            for op in ops[1:]:
                total += op[1]
            for op in ops:
                op[1].copy_(total)


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
        self._host = {}  # host staging buffers per (dtype, size) of face buffer

    def exchange(self, d: SlabDomain):
        torch = d.torch
        key = (d.send_lo.dtype, d.send_lo.numel())
        if key not in self._host:
            self._host[key] = [torch.empty(d.send_lo.shape, dtype=d.send_lo.dtype) for _ in range(4)]
        s_hi, s_lo, h_lo, h_hi = self._host[key]
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
        # 16-bit codes travel as float16 (the same bytes; NCCL has no int16 and
        # point-to-point transfers do no arithmetic)
        wire = (lambda t: t.view(d.torch.float16)) if d.send_lo.dtype == d.torch.int16 else (lambda t: t)
        ops = [dist.P2POp(dist.isend, wire(d.send_hi), up, self.group),
               dist.P2POp(dist.isend, wire(d.send_lo), down, self.group),
               dist.P2POp(dist.irecv, wire(d.halo_lo), down, self.group),
               dist.P2POp(dist.irecv, wire(d.halo_hi), up, self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class LocalExchange:
    """Face exchange between the slabs of one process (all ranks emulated on
    one device: the copies stand in for the point-to-point transfers)."""

    def __init__(self, domains):
        self.domains = domains

    def exchange_all(self):
        W = len(self.domains)
        first = self.domains[0]
        if first.send_lo.is_cuda and 2 * W <= 64:  # one launch for every copy (lbm_copy_buffers_async)
            src, dst = [], []
            for r, d in enumerate(self.domains):
                src += [self.domains[(r - 1) % W].send_hi, self.domains[(r + 1) % W].send_lo]
                dst += [d.halo_lo, d.halo_hi]
            E.check(E.copy_buffers_async(src, dst, first.send_lo.numel() * first.send_lo.element_size()),
                    "face copies")
            return
        for r, d in enumerate(self.domains):
            d.halo_lo.copy_(self.domains[(r - 1) % W].send_hi)
            d.halo_hi.copy_(self.domains[(r + 1) % W].send_lo)
