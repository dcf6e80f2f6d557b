"""Slab decomposition of one mesh along x: the data-parallel form of the 2D solver.

The reference's multi-GPU 2D solver splits the mesh into x slabs over MPI
(src/parallel/slab1d.h:55-72, src/cuda/sgn2d_cuda_mpi.cu:487-537, 605-615): each rank owns
a contiguous run of element columns, exchanges the traces across its two slab edges before
every right-hand side (a pack kernel and two MPI_Sendrecv), and takes one global reduction
of the error norm per BS3(2) attempt so that every rank makes the same accept / reject
decision. This module does the same for the 2D hot path:

* ``slab_partition`` -- the reference's column split (the first ``Nx % size`` slabs take
  one column more, src/parallel/slab1d.h:55-72), and ``neighbours``.
* ``LocalExchange`` -- every slab on one device: the exchange is device-to-device copies
  of the edge nodes and the reduction is a concatenation of the slabs' error partials.
* ``DistExchange`` -- one slab per rank over ``torch.distributed`` (NCCL between GPUs,
  gloo on the host): point-to-point sends of the edge nodes and an all-gather of the
  error partials.
* ``SlabSolver`` -- ``rhs``, ``integrate_adaptive`` (to tEnd), ``integrate_steps``
  (adaptive or frozen step sizes), ``upload`` / ``download`` of the whole mesh's state.

Each slab is a library context created with ``Nx_global`` / ``ex_offset`` (its node
coordinates and bathymetry are the whole mesh's), and its two ghost arrays
[5 fields][Ny][5 nodes] hold the neighbours' stage inputs along the edges. The fused
kernels read them in place of the periodic wrap or the wall mirror, so a slab's
right-hand side is the whole mesh's, bit for bit, on its columns. Every slab's
controller reduces the partials of all slabs, in slab order.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import (FP64_FAST, SGN2DB200, AdaptiveRKOptions, SgnbError, _DescHolder, _DeviceArray,
               _Opts, _Stats, _check, _dp, _stats, lib)

NP, NV = 5, 5


def slab_partition(Nx: int, size: int, rank: int) -> tuple[int, int]:
    """(first column, column count) of slab ``rank`` of ``size``."""
    if size < 1 or not 0 <= rank < size or Nx < size:
        raise ValueError("slab_partition: 0 <= rank < size <= Nx")
    base, rem = divmod(Nx, size)
    return rank * base + min(rank, rem), base + (1 if rank < rem else 0)


def neighbours(rank: int, size: int, periodic: bool) -> tuple[int | None, int | None]:
    """Left and right neighbour slabs (None: a domain wall)."""
    if periodic:
        return (rank - 1) % size, (rank + 1) % size
    return (rank - 1 if rank > 0 else None), (rank + 1 if rank < size - 1 else None)


def tile_count(Nx: int, Ny: int) -> int:
    """Tiles (8 x 4 elements) of one slab's fused grid = its error partial blocks."""
    return ((Nx + 7) // 8) * ((Ny + 3) // 4)


def _dev(ptr):
    return None if ptr is None else C.cast(C.c_void_p(ptr), _dp)


class _Slab:
    """One slab's context, its edge buffers and its partials."""

    def __init__(self, kw: dict, Nx_global: int, ex0: int, nx: int, device: int, torch):
        kw = dict(kw)
        args = [kw.pop(k, dflt) for k, dflt in (
            ("P", 4), ("Nx", Nx_global), ("Ny", 6), ("Lx", 10.0), ("Ly", 8.0), ("g", 9.81),
            ("c", 0.0), ("gamma", 1.5), ("nManning", 0.0), ("bc_x", 0), ("bc_y", 0),
            ("precision", FP64_FAST), ("device", device), ("bathy_kind", 0), ("bathy_par", ()),
            ("tables", None), ("bathy_arrays", None))]
        if kw:
            raise TypeError(f"SlabSolver: unknown keys {sorted(kw)}")
        if args[16] is not None:
            raise ValueError("SlabSolver: slabs build their bathymetry from bathy_kind")
        args[1] = nx
        args[12] = device
        holder = _DescHolder(*args)
        holder.desc.Nx_global = Nx_global
        holder.desc.ex_offset = ex0
        h = C.c_void_p()
        _check(lib().sgnb_create(C.byref(holder.desc), C.byref(h)))
        d = holder.desc
        self.ctx = SGN2DB200(P=d.P, Nx=nx, Ny=d.Ny, Lx=d.Lx, Ly=d.Ly, precision=d.precision,
                             device=device, _handle=h.value)
        self.ctx._owned = True
        self.ex0, self.nx, self.Ny = ex0, nx, d.Ny
        n = NV * d.Ny * NP
        dev = f"cuda:{device}"
        self.sendL = torch.zeros(n, dtype=torch.float64, device=dev)
        self.sendR = torch.zeros(n, dtype=torch.float64, device=dev)
        self.ghostL = torch.zeros(n, dtype=torch.float64, device=dev)
        self.ghostR = torch.zeros(n, dtype=torch.float64, device=dev)
        p, nb = _dp(), C.c_int()
        _check(lib().sgnb_slab_partials(self.h, C.byref(p), C.byref(nb)), self.h)
        self.nblk = nb.value
        self.partials = torch.as_tensor(
            _DeviceArray(C.cast(p, C.c_void_p).value, 3 * self.nblk), device=dev)

    @property
    def h(self):
        return self.ctx._h

    def set_ghosts(self, left: bool, right: bool):
        _check(lib().sgnb_set_ghosts(self.h, _dev(self.ghostL.data_ptr() if left else None),
                                     _dev(self.ghostR.data_ptr() if right else None)), self.h)

    def pack(self, stage: int, stream: int, in_ptr=None):
        _check(lib().sgnb_slab_pack(self.h, stage, _dev(in_ptr), _dev(self.sendL.data_ptr()),
                                    _dev(self.sendR.data_ptr()), C.c_void_p(stream)), self.h)

    def close(self):
        self.ctx.close()


class LocalExchange:
    """Every slab on one device; the copies run on the caller's (current) stream."""

    def __init__(self, nslabs: int, periodic: bool):
        self.size = nslabs
        self.links = [neighbours(r, nslabs, periodic) for r in range(nslabs)]

    def edges(self, slabs):
        for r, s in enumerate(slabs):
            left, right = self.links[r]
            if left is not None:
                s.ghostL.copy_(slabs[left].sendR)
            if right is not None:
                s.ghostR.copy_(slabs[right].sendL)

    def gather(self, slabs, torch):
        mb = max(s.nblk for s in slabs)
        out = torch.zeros(3 * mb * len(slabs), dtype=torch.float64, device=slabs[0].sendL.device)
        for r, s in enumerate(slabs):
            out[3 * mb * r: 3 * mb * r + 3 * s.nblk].copy_(s.partials)
        return out, mb * len(slabs)


class DistExchange:
    """One slab per rank over torch.distributed (the process group's backend).

    Edges: every rank first sends its right edge to the right and receives its left ghost
    from the left, then sends its left edge to the left and receives its right ghost from
    the right; with two periodic ranks the two messages between the pair keep that order.
    Gather: the all-gather of every rank's partials, zero-padded to the largest block
    count (zeros leave the sum, the maximum and the NaN count unchanged)."""

    def __init__(self, periodic: bool, group=None, max_blocks: int | None = None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.left, self.right = neighbours(self.rank, self.size, periodic)
        self.max_blocks = max_blocks

    def _peer(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def edges_of(self, slab):
        d = self.dist
        ops = []
        if self.right is not None:
            ops.append(d.P2POp(d.isend, slab.sendR, self._peer(self.right), self.group))
        if self.left is not None:
            ops.append(d.P2POp(d.irecv, slab.ghostL, self._peer(self.left), self.group))
        if self.left is not None:
            ops.append(d.P2POp(d.isend, slab.sendL, self._peer(self.left), self.group))
        if self.right is not None:
            ops.append(d.P2POp(d.irecv, slab.ghostR, self._peer(self.right), self.group))
        if ops:
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def edges(self, slabs):
        (slab,) = slabs
        self.edges_of(slab)

    def gather_of(self, slab, torch):
        if self.max_blocks is None:
            t = torch.tensor([slab.nblk], dtype=torch.int64, device=slab.sendL.device)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
            self.max_blocks = int(t.item())
        mb = self.max_blocks
        mine = torch.zeros(3 * mb, dtype=torch.float64, device=slab.sendL.device)
        mine[: 3 * slab.nblk].copy_(slab.partials)
        parts = [torch.empty_like(mine) for _ in range(self.size)]
        self.dist.all_gather(parts, mine, group=self.group)
        return torch.cat(parts), mb * self.size

    def gather(self, slabs, torch):
        (slab,) = slabs
        return self.gather_of(slab, torch)


class SlabSolver:
    """The 2D solver on x slabs: on one device (``nslabs`` slabs, LocalExchange) or one
    slab per rank of a torch.distributed group (``distributed=True``, DistExchange).

    ``kw`` are the whole mesh's SGN2DB200 arguments (Nx the global column count). All
    launches and copies of the solver run on one dedicated stream (``self.stream``)."""

    def __init__(self, kw: dict, nslabs: int = 1, device: int = 0, distributed: bool = False,
                 group=None):
        import torch

        self.torch = torch
        self.kw = dict(kw)
        self.Nx = int(kw["Nx"])
        self.Ny = int(kw["Ny"])
        periodic = int(kw.get("bc_x", 0)) == 0
        torch.cuda.set_device(device)
        self.device = device
        if distributed:
            self.exchange = DistExchange(periodic, group)
            ranks = [self.exchange.rank]
            size = self.exchange.size
        else:
            self.exchange = LocalExchange(nslabs, periodic)
            ranks = list(range(nslabs))
            size = nslabs
        self.size = size
        self.parts = [slab_partition(self.Nx, size, r) for r in range(size)]
        self.ranks = ranks
        self.slabs = []
        try:
            for r in ranks:
                a, w = self.parts[r]
                self.slabs.append(_Slab(kw, self.Nx, a, w, device, torch))
            for r, s in zip(ranks, self.slabs):
                left, right = neighbours(r, size, periodic)
                s.set_ghosts(left is not None, right is not None)
        except Exception:
            self.close()
            raise
        self.n_total = 5 * 25 * self.Nx * self.Ny
        self.stream = torch.cuda.Stream(device)
        torch.cuda.synchronize(device)

    def close(self):
        for s in getattr(self, "slabs", []):
            s.close()
        self.slabs = []

    def _sync(self):
        self.torch.cuda.synchronize(self.device)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- state transfer: the whole mesh's layout [field][ey][ex][node] -------------
    def _cols(self, U, a, w):
        U = np.asarray(U, dtype=np.float64).reshape(NV, self.Ny, self.Nx, 25)
        return np.ascontiguousarray(U[:, :, a:a + w, :]).reshape(-1)

    def upload(self, U):
        """Every local slab takes its columns of the whole mesh's state ``U``."""
        self.torch.cuda.synchronize(self.device)
        for s in self.slabs:
            s.ctx.upload(self._cols(U, s.ex0, s.nx))
        self.torch.cuda.synchronize(self.device)

    def upload_tensor(self, t):
        """Device-to-device form of ``upload`` (a float64 tensor of the whole mesh)."""
        torch = self.torch
        if t.dtype != torch.float64 or t.numel() != NV * 25 * self.Nx * self.Ny:
            raise ValueError("SlabSolver.upload_tensor: float64 whole-mesh state expected")
        v = t.reshape(NV, self.Ny, self.Nx, 25)
        self._sync()
        for s in self.slabs:
            s.ctx.state_tensor().view(NV, self.Ny, s.nx, 25).copy_(v[:, :, s.ex0:s.ex0 + s.nx, :])
        self._sync()

    def download_tensor(self):
        """The whole mesh's state as a new device tensor (single process)."""
        torch = self.torch
        if len(self.slabs) != self.size:
            raise ValueError("SlabSolver.download_tensor: one slab per rank")
        out = torch.empty((NV, self.Ny, self.Nx, 25), dtype=torch.float64,
                          device=f"cuda:{self.device}")
        self._sync()
        for s in self.slabs:
            out[:, :, s.ex0:s.ex0 + s.nx, :].copy_(s.ctx.state_tensor().view(NV, self.Ny, s.nx, 25))
        self._sync()
        return out.reshape(-1)

    def download_local(self):
        """{slab index: that slab's state} for the local slabs."""
        self.torch.cuda.synchronize(self.device)
        return {r: s.ctx.download() for r, s in zip(self.ranks, self.slabs)}

    def download(self):
        """The whole mesh's state (single process: every slab is local)."""
        if len(self.slabs) != self.size:
            raise ValueError("SlabSolver.download: one slab per rank; use download_local")
        out = np.empty((NV, self.Ny, self.Nx, 25))
        for r, U in self.download_local().items():
            a, w = self.parts[r]
            out[:, :, a:a + w, :] = U.reshape(NV, self.Ny, w, 25)
        return out.reshape(-1)

    # --- right-hand side ---------------------------------------------------------
    def _exchange(self, stage, in_ptrs=None):
        sp = self.stream.cuda_stream
        for i, s in enumerate(self.slabs):
            s.pack(stage, sp, None if in_ptrs is None else in_ptrs[i])
        with self.torch.cuda.stream(self.stream):
            self.exchange.edges(self.slabs)

    def rhs(self, U):
        """R(U) of the whole mesh through the slabs (host arrays in and out)."""
        torch = self.torch
        dev = f"cuda:{self.device}"
        ins = [torch.from_numpy(self._cols(U, s.ex0, s.nx)).to(dev) for s in self.slabs]
        outs = [torch.empty_like(t) for t in ins]
        torch.cuda.synchronize(self.device)
        self._exchange(0, [t.data_ptr() for t in ins])
        for s, t, o in zip(self.slabs, ins, outs):
            s.ctx.rhs_device(t.data_ptr(), o.data_ptr(), self.stream.cuda_stream)
        self.stream.synchronize()
        if len(self.slabs) != self.size:
            return {r: o.cpu().numpy() for r, o in zip(self.ranks, outs)}
        dU = np.empty((NV, self.Ny, self.Nx, 25))
        for r, o in zip(self.ranks, outs):
            a, w = self.parts[r]
            dU[:, :, a:a + w, :] = o.cpu().numpy().reshape(NV, self.Ny, w, 25)
        return dU.reshape(-1)

    # --- BS3(2) ------------------------------------------------------------------
    def integrate_adaptive(self, t0, tEnd, dt0, opt: AdaptiveRKOptions | None = None,
                           check_every: int = 4):
        """SGN2DCudaMpi::integrateAdaptive (src/cuda/sgn2d_cuda_mpi.h:62): adaptive BS3(2)
        of the uploaded state from t0 to tEnd."""
        return self._run(t0, tEnd, dt0, 0, opt, None, check_every, 1 << 40)

    def integrate_steps(self, t0, dt0, nsteps, opt: AdaptiveRKOptions | None = None,
                        dts=None, check_every: int = 4):
        """``nsteps`` accepted BS3(2) steps of the uploaded state: adaptive from ``dt0``,
        or with the frozen step sizes ``dts`` (one per step, every step accepted)."""
        if dts is not None and np.asarray(dts).size != nsteps:
            raise ValueError("integrate_steps: one frozen step size per step")
        return self._run(t0, float("inf"), dt0, nsteps, opt, dts, check_every,
                         64 * int(nsteps) + 4096)

    def _run(self, t0, tEnd, dt0, nsteps, opt, dts, check_every, limit):
        """Per attempt: stages 2, 3, 4, each after an edge exchange of its stage inputs,
        then the gather of all slabs' error partials and every slab's controller on them.
        The host reads the controller every ``check_every`` attempts (the kernels of
        attempts after the end return at once); ``limit`` bounds the attempts."""
        torch = self.torch
        sp = self.stream.cuda_stream
        o = _Opts(**dataclasses.asdict(opt or AdaptiveRKOptions()))
        d = None if dts is None else np.ascontiguousarray(dts, dtype=np.float64)
        torch.cuda.synchronize(self.device)
        for s in self.slabs:
            _check(lib().sgnb_slab_begin(s.h, float(t0), float(tEnd), float(dt0), int(nsteps),
                                         None if d is None else d.ctypes.data_as(_dp),
                                         C.byref(o)), s.h)
        # FSAL head: k1 = R(u)
        self._exchange(0)
        for s in self.slabs:
            _check(lib().sgnb_slab_launch(s.h, 1, C.c_void_p(sp)), s.h)
        attempts = 0
        done = C.c_int(0)
        st = _Stats()
        while True:
            for stage in (2, 3, 4):
                self._exchange(stage)
                for s in self.slabs:
                    _check(lib().sgnb_slab_launch(s.h, stage, C.c_void_p(sp)), s.h)
            with torch.cuda.stream(self.stream):
                allp, nblk = self.exchange.gather(self.slabs, torch)
            pp = C.cast(C.c_void_p(allp.data_ptr()), _dp)
            for s in self.slabs:
                _check(lib().sgnb_slab_control(s.h, pp, nblk, self.n_total, C.c_void_p(sp)), s.h)
            attempts += 1
            if attempts % check_every == 0 or attempts >= limit:
                _check(lib().sgnb_slab_status(self.slabs[0].h, C.byref(st), C.byref(done),
                                              C.c_void_p(sp)), self.slabs[0].h)
                if done.value or attempts >= limit:
                    break
        for s in self.slabs:
            _check(lib().sgnb_slab_status(s.h, C.byref(st), C.byref(done), C.c_void_p(sp)), s.h)
        if st.status == 4:
            raise SgnbError(4, "non-finite state in a slab integration")
        if not done.value:
            raise SgnbError(6, "slab integration did not finish within its attempt limit")
        return _stats(st)


class PeerSlabSolver(SlabSolver):
    """Slabs with the fused edge exchange: no send buffers and no copies.

    Every slab has a ghost array per side for each stage that reads ghosts (1: the FSAL
    head, 2, 3, 4). The packs of stages 0 and 2 (after the controller has set dt) and the
    edge tiles of the stage-2 and stage-3 kernels store the next stage's edge inputs
    straight into the neighbours' ghost arrays (sgnb_slab_stage), and each slab's
    controller reads every slab's error partials in place (sgnb_slab_control_all). Slabs
    may sit on several devices (``devices``, slab r on devices[r % len]): the stores and
    loads then cross NVLink as peer accesses, and every launch that reads ghosts or partials
    waits, through events, for the neighbours' launches that wrote them (and every end-point
    launch for all controllers of the previous attempt, which still read its partials).
    ``streams="shared"`` runs every slab on one stream (single device only)."""

    STAGES = (1, 2, 3, 4)

    def __init__(self, kw: dict, nslabs: int = 1, devices=None, streams: str = "per-slab"):
        import torch

        self.torch = torch
        self.kw = dict(kw)
        self.Nx = int(kw["Nx"])
        self.Ny = int(kw["Ny"])
        self.periodic = int(kw.get("bc_x", 0)) == 0
        self.devices = list(devices) if devices else [0]
        if streams not in ("shared", "per-slab"):
            raise ValueError("streams: 'shared' or 'per-slab'")
        if streams == "shared" and len(set(self.devices)) > 1:
            raise ValueError("a shared stream needs a single device")
        if nslabs > 32:
            raise ValueError("PeerSlabSolver: at most 32 slabs")
        self.device = self.devices[0]
        self.size = nslabs
        self.ranks = list(range(nslabs))
        self.parts = [slab_partition(self.Nx, nslabs, r) for r in range(nslabs)]
        self.links = [neighbours(r, nslabs, self.periodic) for r in range(nslabs)]
        self.exchange = None
        for a in set(self.devices):
            for b in set(self.devices):
                _check(lib().sgnb_enable_peer_access(a, b))
        self.slabs = []
        self.ghost = []  # ghost[r][stage] = (left, right) tensors on slab r's device
        try:
            for r in range(nslabs):
                dev = self.devices[r % len(self.devices)]
                a, w = self.parts[r]
                s = _Slab(kw, self.Nx, a, w, dev, torch)
                s.device = dev
                self.slabs.append(s)
                n = NV * self.Ny * NP
                self.ghost.append({st: (torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}"),
                                        torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}"))
                                   for st in self.STAGES})
        except Exception:
            self.close()
            raise
        self.n_total = 5 * 25 * self.Nx * self.Ny
        if streams == "shared":
            sh = torch.cuda.Stream(self.device)
            self.streams = [sh] * nslabs
        else:
            self.streams = [torch.cuda.Stream(s.device) for s in self.slabs]
        self.shared = streams == "shared"
        self.stream = self.streams[0]
        self._pp = (_dp * nslabs)(*[C.cast(C.c_void_p(s.partials.data_ptr()), _dp)
                                    for s in self.slabs])
        self._nb = (C.c_int * nslabs)(*[s.nblk for s in self.slabs])
        self._sync()

    def _sync(self):
        for d in set(self.devices):
            self.torch.cuda.synchronize(d)

    # --- ghost pointers ------------------------------------------------------------
    def _ghosts_in(self, r, st):
        """(left, right) ghost inputs of slab r for stage st (None at a wall)."""
        left, right = self.links[r]
        gl, gr = self.ghost[r][st]
        return (_dev(gl.data_ptr()) if left is not None else None,
                _dev(gr.data_ptr()) if right is not None else None)

    def _edges_out(self, r, st):
        """Where slab r's edges go for stage st: its left edge into the left neighbour's
        right ghost, its right edge into the right neighbour's left ghost."""
        left, right = self.links[r]
        return (_dev(self.ghost[left][st][1].data_ptr()) if left is not None else None,
                _dev(self.ghost[right][st][0].data_ptr()) if right is not None else None)

    # --- ordering between slabs ----------------------------------------------------
    def _record(self, r):
        if self.shared:
            return None
        e = self.torch.cuda.Event()
        e.record(self.streams[r])
        return e

    def _wait(self, r, events):
        if self.shared:
            return
        for e in events:
            if e is not None:
                self.streams[r].wait_event(e)

    def _nbr_events(self, r, ev):
        left, right = self.links[r]
        return [ev[q] for q in (left, right) if q is not None and q != r]

    def _pack(self, st_in, st_out, in_ptrs=None):
        """Packs of stage st_in (0 or 2) into the neighbours' ghosts of stage st_out."""
        ev = []
        for r, s in enumerate(self.slabs):
            oL, oR = self._edges_out(r, st_out)
            # a wall side writes nowhere: a scratch ghost of this slab takes it
            sc = self.ghost[r][st_out]
            sendL = oL if oL is not None else _dev(sc[0].data_ptr())
            sendR = oR if oR is not None else _dev(sc[1].data_ptr())
            _check(lib().sgnb_slab_pack(s.h, st_in, _dev(None if in_ptrs is None else in_ptrs[r]),
                                        sendL, sendR, C.c_void_p(self.streams[r].cuda_stream)), s.h)
            ev.append(self._record(r))
        return ev

    def _stage(self, st, prev_ev, extra=None):
        ev = []
        for r, s in enumerate(self.slabs):
            self._wait(r, self._nbr_events(r, prev_ev) + (extra or []))
            gL, gR = self._ghosts_in(r, st)
            oL, oR = self._edges_out(r, st + 1) if st in (2, 3) else (None, None)
            _check(lib().sgnb_slab_stage(s.h, st, gL, gR, oL, oR,
                                         C.c_void_p(self.streams[r].cuda_stream)), s.h)
            ev.append(self._record(r))
        return ev

    # --- right-hand side ---------------------------------------------------------
    def rhs(self, U):
        torch = self.torch
        ins = [torch.from_numpy(self._cols(U, s.ex0, s.nx)).to(f"cuda:{s.device}") for s in self.slabs]
        outs = [torch.empty_like(t) for t in ins]
        self._sync()
        ev = self._pack(0, 1, [t.data_ptr() for t in ins])
        for r, (s, t, o) in enumerate(zip(self.slabs, ins, outs)):
            self._wait(r, self._nbr_events(r, ev))
            gL, gR = self._ghosts_in(r, 1)
            _check(lib().sgnb_set_ghosts(s.h, gL, gR), s.h)
            s.ctx.rhs_device(t.data_ptr(), o.data_ptr(), self.streams[r].cuda_stream)
        self._sync()
        dU = np.empty((NV, self.Ny, self.Nx, 25))
        for r, o in enumerate(outs):
            a, w = self.parts[r]
            dU[:, :, a:a + w, :] = o.cpu().numpy().reshape(NV, self.Ny, w, 25)
        return dU.reshape(-1)

    def upload(self, U):
        self._sync()
        for s in self.slabs:
            s.ctx.upload(self._cols(U, s.ex0, s.nx))
        self._sync()

    def download_local(self):
        self._sync()
        return {r: s.ctx.download() for r, s in enumerate(self.slabs)}

    # --- BS3(2) ------------------------------------------------------------------
    def _run(self, t0, tEnd, dt0, nsteps, opt, dts, check_every, limit):
        """Per attempt: the stage-2 pack, stages 2, 3 (their edge tiles fill the
        neighbours' ghosts of the next stage), 4, and every slab's controller on all slabs'
        partials in place."""
        o = _Opts(**dataclasses.asdict(opt or AdaptiveRKOptions()))
        d = None if dts is None else np.ascontiguousarray(dts, dtype=np.float64)
        self._sync()
        for s in self.slabs:
            _check(lib().sgnb_slab_begin(s.h, float(t0), float(tEnd), float(dt0), int(nsteps),
                                         None if d is None else d.ctypes.data_as(_dp),
                                         C.byref(o)), s.h)
        ev = self._pack(0, 1)
        ev = self._stage(1, ev)
        ctrl_ev = []
        attempts = 0
        done = C.c_int(0)
        st = _Stats()
        while True:
            ev = self._pack(2, 2)
            ev = self._stage(2, ev)
            ev = self._stage(3, ev)
            # the end-point launch overwrites this slab's partials: every controller of
            # the previous attempt has read them
            fsal_ev = self._stage(4, ev, extra=ctrl_ev)
            ctrl_ev = []
            for r, s in enumerate(self.slabs):
                self._wait(r, fsal_ev)
                _check(lib().sgnb_slab_control_all(s.h, self._pp, self._nb, self.size, self.n_total,
                                                   C.c_void_p(self.streams[r].cuda_stream)), s.h)
                ctrl_ev.append(self._record(r))
            attempts += 1
            if attempts % check_every == 0 or attempts >= limit:
                s0 = self.slabs[0]
                _check(lib().sgnb_slab_status(s0.h, C.byref(st), C.byref(done),
                                              C.c_void_p(self.streams[0].cuda_stream)), s0.h)
                if done.value or attempts >= limit:
                    break
        self._sync()
        for r, s in enumerate(self.slabs):
            _check(lib().sgnb_slab_status(s.h, C.byref(st), C.byref(done),
                                          C.c_void_p(self.streams[r].cuda_stream)), s.h)
        if st.status == 4:
            raise SgnbError(4, "non-finite state in a slab integration")
        if not done.value:
            raise SgnbError(6, "slab integration did not finish within its attempt limit")
        return _stats(st)
