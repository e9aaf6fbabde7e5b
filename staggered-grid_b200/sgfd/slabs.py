"""z-slabs: one model split along z over several solver handles.

The reference runs one model on one GPU and caps it at 2^29 cells with a
32-bit `memsize` (3DGPUwithPML_1DArraySingleGPU_optimization/
ElasticWaveEquation.cu:20,143).  Here a model of GRID nx x ny x nz_total is
cut along z into slabs of whole computed planes; each slab is an sgfd handle
(sgfd_config.nz_total / z_offset) that keeps the whole model's PML bands and
compact split order.  At every cut the two slabs trade the 5 planes next to it
(the reach of the 10th-order z differences) twice per step:

    for every slab: exchange txz, tyz, tzz  (HALO_STRESS)
                    velocity half step      (PHASE_VELOCITY)
                    exchange vx, vy, vz     (HALO_VELOCITY)
                    stress half step        (PHASE_STRESS)

which gives the whole model's results bit for bit (the updates of a cell read
only its 10-cell neighbourhood, and every value a slab reads at its frame is
the neighbour's value of the same half step).  Each exchange overlaps the
inner part of the half step after it (PART_INNER: the planes 5 or more planes
from the slab's ends, which read no frame plane); the outer part runs once
the halos are unpacked.

Two forms share the plan and the step sequence:
  * SlabModel — all slabs in one process on one GPU, a stream each, halos
    moved by device copies ordered by events;
  * DistributedSlab — one slab per rank (one process per GPU, torch.distributed
    over NCCL), halos moved by send/recv to the ranks above and below
    (exchange_remote, also run on CPU tensors over gloo by the tests).
"""
from __future__ import annotations

import numpy as np

from . import (Config, Solver, HALO_LOW, HALO_HIGH, HALO_STRESS, HALO_VELOCITY, PHASE_VELOCITY, PHASE_STRESS,
               PART_INNER, PART_OUTER)

HALO = 5            # planes exchanged at a cut (the reference `order`)
MIN_PLANES = HALO   # computed planes a slab needs to fill its neighbour's frame


def plan_cuts(nz_total: int, nslabs: int, src_z: int | None = None, weights=None) -> list[tuple[int, int]]:
    """Computed-plane ranges (z_offset, planes) of nslabs slabs of a model with
    nz_total GRID planes, in z order, sized in proportion to `weights` (equal by
    default; e.g. the free memory of each slab's GPU).  A source at GRID plane
    src_z must lie 5 or more planes from every cut, because its injection is
    applied inside the owning slab only: a cut that lands closer is moved past
    it."""
    nzc = nz_total - 2 * HALO
    if nslabs < 1:
        raise ValueError("nslabs must be >= 1")
    if nzc < nslabs * MIN_PLANES:
        raise ValueError(f"{nzc} computed planes cannot make {nslabs} slabs of >= {MIN_PLANES} planes")
    w = np.ones(nslabs) if weights is None else np.asarray(weights, dtype=np.float64)
    if len(w) != nslabs or np.any(w <= 0):
        raise ValueError("one positive weight per slab")
    cuts = [int(round(nzc * float(np.sum(w[:k])) / float(np.sum(w)))) for k in range(1, nslabs)]
    if src_z is not None:
        zs = src_z - HALO
        for k, c in enumerate(cuts):
            if c - HALO <= zs < c + HALO:
                lo = cuts[k - 1] if k > 0 else 0
                hi = cuts[k + 1] if k + 1 < len(cuts) else nzc
                options = [zs - HALO, zs + HALO + 1]   # the source HALO planes above / below the cut
                ok = [o for o in options if o - lo >= MIN_PLANES and hi - o >= MIN_PLANES]
                if not ok:
                    raise ValueError(f"no cut near plane {c} keeps the source plane {src_z} {HALO} planes away")
                cuts[k] = min(ok, key=lambda o: abs(o - c))
    edges = [0] + cuts + [nzc]
    out = [(edges[k], edges[k + 1] - edges[k]) for k in range(nslabs)]
    if any(n < MIN_PLANES for _, n in out):
        raise ValueError(f"slab sizes {[n for _, n in out]}: each needs >= {MIN_PLANES} planes")
    return out


def slab_config(cfg: Config, z_offset: int, planes: int, device: int | None = None) -> Config:
    """The handle configuration of one slab of the whole model `cfg`."""
    c = Config.from_buffer_copy(cfg)
    c.nz_total = cfg.nz
    c.z_offset = z_offset
    c.nz = planes + 2 * HALO
    if device is not None:
        c.device = device
    return c


def split_receivers(cuts, xyz, comp):
    """Receivers per slab: (indices into the whole list, slab-local xyz, comp)."""
    xyz = np.asarray(xyz, dtype=np.int32).reshape(-1, 3)
    comp = np.asarray(comp, dtype=np.int32).reshape(-1)
    cz = xyz[:, 2] - HALO
    out = []
    for z0, n in cuts:
        idx = np.nonzero((cz >= z0) & (cz < z0 + n))[0]
        local = xyz[idx].copy()
        local[:, 2] -= z0
        out.append((idx, local, comp[idx]))
    return out


def source_slab(cuts, z: int) -> int:
    """Index of the slab holding GRID plane z (a computed plane)."""
    cz = z - HALO
    for k, (z0, n) in enumerate(cuts):
        if z0 <= cz < z0 + n:
            return k
    raise ValueError(f"plane {z} is not a computed plane")


def check_source(cuts, z: int):
    cz = z - HALO
    for z0, _ in cuts[1:]:
        if z0 - HALO <= cz < z0 + HALO:
            raise ValueError(f"source plane {z} lies within {HALO} planes of the cut at computed plane {z0}")


def exchange_remote(send_lo, send_hi, recv_lo, recv_hi, rank: int, world: int, group=None):
    """Trade halo buffers with the ranks below (rank - 1) and above (rank + 1):
    send_lo goes down and arrives as that rank's recv_hi, send_hi goes up and
    arrives as its recv_lo.  Tensors on the backend's device (CUDA over NCCL,
    CPU over gloo); every rank posts its sends and receives together."""
    import torch.distributed as dist
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, send_lo, rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, recv_lo, rank - 1, group))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.isend, send_hi, rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, recv_hi, rank + 1, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class _Slabs:
    """What both forms share: the plan, the per-slab inputs and the step."""

    def __init__(self, cfg: Config, cuts):
        self.cfg = cfg
        self.cuts = list(cuts)
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        self.src_slab = -1
        self.rec_parts = None
        self.nrec = 0
        self.nt = 0

    # GRID planes of slab k in the whole model: [z0, z0 + planes + 10)
    def _grid_planes(self, k):
        z0, n = self.cuts[k]
        return z0, z0 + n + 2 * HALO


class SlabModel(_Slabs):
    """All slabs of one model in this process, on one GPU (cfg.device).  Each
    slab runs on a stream of its own, so one slab's halo copies and kernels
    overlap another's; events order what must be ordered: a slab unpacks its
    neighbours' planes after they packed them, and packs again only after
    both neighbours unpacked the previous buffer.  `run` starts after, and
    ends before, the work queued on `stream`.  Slabs on several GPUs:
    DistributedSlab."""

    def __init__(self, cfg: Config, cuts):
        super().__init__(cfg, cuts)
        import torch
        self._torch = torch
        d = cfg.device
        self.slabs = []
        # per halo kind and slab: (buffer of its LOW side, buffer of its HIGH side), and the events
        # after the slab packed them and after it unpacked its neighbours' buffers
        self.bufs = [[], []]
        self.stream = torch.cuda.Stream(device=d)                 # joins every slab's stream around a run
        self.streams = [torch.cuda.Stream(device=d) for _ in self.cuts]
        self.packed = [[torch.cuda.Event() for _ in self.cuts] for _ in range(2)]
        self.unpacked = [[torch.cuda.Event() for _ in self.cuts] for _ in range(2)]
        try:
            for (z0, n), st in zip(self.cuts, self.streams):
                s = Solver(slab_config(cfg, z0, n, d))
                s.set_stream(st.cuda_stream)
                nbytes = s.halo_bytes()
                with torch.cuda.stream(st):
                    for kind in (HALO_STRESS, HALO_VELOCITY):
                        self.bufs[kind].append(tuple(torch.empty(nbytes // 4, dtype=torch.float32,
                                                                 device=f"cuda:{d}") for _ in range(2)))
                self.slabs.append(s)
        except Exception:
            self.close()
            raise

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_medium(self, b, lam, mu):
        arrs = [np.asarray(a, dtype=np.float32).reshape(self.nz, self.ny, self.nx) for a in (b, lam, mu)]
        for k, s in enumerate(self.slabs):
            g0, g1 = self._grid_planes(k)
            s.set_medium(*[a[g0:g1] for a in arrs])

    def set_source(self, x: int, y: int, z: int):
        check_source(self.cuts, z)
        self.src_slab = source_slab(self.cuts, z)
        self.slabs[self.src_slab].set_source(x, y, z - self.cuts[self.src_slab][0])

    def set_receivers(self, xyz, comp, nt: int):
        self.rec_parts = split_receivers(self.cuts, xyz, comp)
        for s, (idx, local, c) in zip(self.slabs, self.rec_parts):
            s.set_receivers(local, c, nt)
        self.nrec = len(np.asarray(comp).reshape(-1))
        self.nt = nt

    def _pack(self, kind: int):
        last = len(self.slabs) - 1
        bufs, packed, unpacked = self.bufs[kind], self.packed[kind], self.unpacked[kind]
        for k, s in enumerate(self.slabs):
            st = self.streams[k]
            for j in (k - 1, k + 1):          # the neighbours have unpacked this slab's previous buffers
                if 0 <= j <= last:
                    st.wait_event(unpacked[j])
            if k > 0:
                s.halo_pack(HALO_LOW, kind, bufs[k][0].data_ptr())
            if k < last:
                s.halo_pack(HALO_HIGH, kind, bufs[k][1].data_ptr())
            packed[k].record(st)

    def _unpack(self, kind: int):
        last = len(self.slabs) - 1
        bufs, packed, unpacked = self.bufs[kind], self.packed[kind], self.unpacked[kind]
        for k, s in enumerate(self.slabs):
            st = self.streams[k]
            if k > 0:
                st.wait_event(packed[k - 1])
                s.halo_unpack(HALO_LOW, kind, bufs[k - 1][1].data_ptr())
            if k < last:
                st.wait_event(packed[k + 1])
                s.halo_unpack(HALO_HIGH, kind, bufs[k + 1][0].data_ptr())
            unpacked[k].record(st)

    def step(self, it: int, value: float):
        """One step of the whole model (reference propagate()): each slab packs,
        runs the inner part of the half step, unpacks its neighbours' planes
        once they are packed, then runs the outer part."""
        for kind, phase in ((HALO_STRESS, PHASE_VELOCITY), (HALO_VELOCITY, PHASE_STRESS)):
            self._pack(kind)
            for s in self.slabs:
                s.step_phase(it, value, phase, PART_INNER)
            self._unpack(kind)
            for s in self.slabs:
                s.step_phase(it, value, phase, PART_OUTER)

    def run(self, it0: int, nsteps: int, wavelet):
        start = self._torch.cuda.Event()
        start.record(self.stream)
        for st in self.streams:
            st.wait_event(start)
        for it in range(it0, it0 + nsteps):
            self.step(it, float(wavelet[it]))
        for st in self.streams:
            done = self._torch.cuda.Event()
            done.record(st)
            self.stream.wait_event(done)

    def synchronize(self):
        for s in self.slabs:
            s.synchronize()

    def traces(self) -> np.ndarray:
        out = np.zeros((self.nrec, self.nt), dtype=np.float32)
        for s, (idx, _, _) in zip(self.slabs, self.rec_parts or []):
            if len(idx):
                out[idx] = s.traces()
        return out

    def field(self, fid: int) -> np.ndarray:
        """One wavefield of the whole model (GRID, frame planes zero)."""
        out = np.zeros((self.nz, self.ny, self.nx), dtype=np.float32)
        for k, s in enumerate(self.slabs):
            z0, n = self.cuts[k]
            out[HALO + z0:HALO + z0 + n] = s.field(fid)[HALO:HALO + n]
        return out


class DistributedSlab(_Slabs):
    """This rank's slab of a model cut into world_size slabs (slab r on rank r,
    its GPU the current device), halos traded with the ranks above and below
    by exchange_remote over the default process group: NCCL moves the device
    buffers themselves; a host backend (gloo) gets them staged through host
    memory, which lets several ranks share one GPU, since no kernel then waits
    on another process (the host does, in its receive)."""

    def __init__(self, cfg: Config, cuts, rank: int, world: int, device: int):
        super().__init__(cfg, cuts)
        import torch
        if len(self.cuts) != world:
            raise ValueError("one slab per rank")
        self.rank, self.world = rank, world
        z0, n = self.cuts[rank]
        self.s = Solver(slab_config(cfg, z0, n, device))
        # the slab's work and the exchanges' send/recv are ordered on this stream
        self.stream = torch.cuda.Stream(device=device)
        self.s.set_stream(self.stream.cuda_stream)
        nf = self.s.halo_bytes() // 4
        dev = f"cuda:{device}"
        with torch.cuda.stream(self.stream):
            self.send = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(2)]
            self.recv = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(2)]

    def close(self):
        self.s.close()

    def set_medium(self, b, lam, mu):
        g0, g1 = self._grid_planes(self.rank)
        self.s.set_medium(*[np.asarray(a, dtype=np.float32).reshape(self.nz, self.ny, self.nx)[g0:g1]
                            for a in (b, lam, mu)])

    def set_source(self, x: int, y: int, z: int):
        check_source(self.cuts, z)
        self.src_slab = source_slab(self.cuts, z)
        if self.src_slab == self.rank:
            self.s.set_source(x, y, z - self.cuts[self.rank][0])

    def set_receivers(self, xyz, comp, nt: int):
        self.rec_parts = split_receivers(self.cuts, xyz, comp)
        idx, local, c = self.rec_parts[self.rank]
        self.s.set_receivers(local, c, nt)
        self.nrec = len(idx)
        self.nt = nt

    def _exchange_start(self, kind: int):
        """Pack this slab's planes beside its cuts and start the transfers;
        returns what _exchange_finish waits for."""
        import torch
        import torch.distributed as dist
        if self.rank > 0:
            self.s.halo_pack(HALO_LOW, kind, self.send[0].data_ptr())
        if self.rank < self.world - 1:
            self.s.halo_pack(HALO_HIGH, kind, self.send[1].data_ptr())
        if dist.get_backend() != "nccl":
            # a host backend: device -> host after the packs, the send/recv on the host, host -> device
            with torch.cuda.stream(self.stream):
                hs = [t.to("cpu") for t in self.send]
            hr = [torch.empty_like(t) for t in hs]
            exchange_remote(hs[0], hs[1], hr[0], hr[1], self.rank, self.world)
            with torch.cuda.stream(self.stream):
                for d, h in zip(self.recv, hr):
                    d.copy_(h)
            return []
        ops = []
        for side, peer in ((0, self.rank - 1), (1, self.rank + 1)):
            if 0 <= peer < self.world:
                ops += [dist.P2POp(dist.isend, self.send[side], peer), dist.P2POp(dist.irecv, self.recv[side], peer)]
        with torch.cuda.stream(self.stream):   # NCCL starts after this stream's packs
            return dist.batch_isend_irecv(ops) if ops else []

    def _exchange_finish(self, kind: int, works):
        import torch
        with torch.cuda.stream(self.stream):   # this stream waits for the transfers
            for w in works:
                w.wait()
        if self.rank > 0:
            self.s.halo_unpack(HALO_LOW, kind, self.recv[0].data_ptr())
        if self.rank < self.world - 1:
            self.s.halo_unpack(HALO_HIGH, kind, self.recv[1].data_ptr())

    def step(self, it: int, value: float):
        """One step of the whole model: per half step, the transfers run while
        the slab's inner part is computed, the outer part after the unpack."""
        for kind, phase in ((HALO_STRESS, PHASE_VELOCITY), (HALO_VELOCITY, PHASE_STRESS)):
            works = self._exchange_start(kind)
            self.s.step_phase(it, value, phase, PART_INNER)
            self._exchange_finish(kind, works)
            self.s.step_phase(it, value, phase, PART_OUTER)

    def run(self, it0: int, nsteps: int, wavelet):
        for it in range(it0, it0 + nsteps):
            self.step(it, float(wavelet[it]))

    def synchronize(self):
        self.s.synchronize()

    def traces(self) -> np.ndarray:
        """This rank's receivers (rows in the order of rec_parts[rank][0])."""
        return self.s.traces()

    def own_planes(self, fid: int) -> tuple[int, np.ndarray]:
        """(first computed plane, the slab's computed planes of one wavefield):
        this rank's part of the whole model's field."""
        z0, n = self.cuts[self.rank]
        return z0, self.s.field(fid)[HALO:HALO + n]
