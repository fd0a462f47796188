"""One mesh decomposed into z slabs over several GPUs (single-job domain decomposition).

The reference steps one mesh block on one device (src/mesh.hpp, Stage() in src/main.cpp:46-93)
and lists domain decomposition as future work (README.md:163, :175). Here a mesh of nx3
planes is cut into nslab slabs of nx3 / nslab planes along z (chq_slab_create). Each slab
runs the stage kernels of a whole mesh on its own planes, with the whole mesh's cell widths,
coordinates and seeded noise. Per stage the slabs exchange the FOFC count (a sum), the FOFC
flags of their boundary planes (the repair of a face between two slabs needs both cells'
flags) and the nghost state planes each neighbour needs for its ghost planes; per cycle the
dt and density minima. The results are bitwise those of the whole mesh (tests/test_slabs.py).

Two exchanges move the data:
  DistExchange  - one slab per process and GPU; torch.distributed point-to-point messages to
                  the two ring neighbours (NCCL between GPUs, gloo between CPU processes) and
                  all-reductions of the step-control words. No collective touches the
                  stage arithmetic: messages are the halo planes only.
  LocalExchange - several slabs of one process on one device (all work on one stream): each
                  slab unpacks its ghosts straight from the neighbour's packed buffer.
SlabRun drives the cycle order documented in include/chq.h.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .core import ChqError, Mesh, _P, _check, load_library

HALO_STATE, HALO_FLAGS = 0, 1


def slab_planes(nx3: int, nslab: int, rank: int) -> tuple[int, int]:
    """(first global active plane, planes) of slab `rank` (nx3 a multiple of nslab)."""
    if nslab < 1 or not (0 <= rank < nslab) or nx3 % nslab:
        raise ChqError(f"z slabs: {nx3} planes do not split into {nslab} equal slabs")
    n = nx3 // nslab
    return rank * n, n


def local_slice(arr: np.ndarray, koff: int, nk: int, face: bool) -> np.ndarray:
    """The planes of a slab (nk cell planes, ghosts included; nk + 1 face planes) out of a whole
    mesh's array in the reference layout (ncomp, nk, nj, ni) or (nk, nj, ni); slab plane k is
    whole-mesh plane k + koff."""
    a = arr if arr.ndim == 4 else arr[None]
    out = a[:, koff:koff + nk + (1 if face else 0)]
    return out if arr.ndim == 4 else out[0]


class _CudaPtr:
    """A device pointer as a __cuda_array_interface__ object (zero-copy torch view)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _device_view(ptr: int, n: int, typestr: str):
    import torch
    return torch.as_tensor(_CudaPtr(ptr, n, typestr), device="cuda")


class SlabMesh(Mesh):
    """Slab `rank` of `nslab` of the mesh `cfg` describes (cfg is the whole mesh's config)."""

    def __init__(self, cfg, nslab: int, rank: int):
        self.nslab, self.rank = int(nslab), int(rank)
        super().__init__(cfg)
        info = (C.c_int * 5)()
        _check(load_library().chq_slab_info(self._h, info))
        self.zpeer = (bool(info[2]), bool(info[3]))
        self.koff = int(info[4])

    def _create(self, lib, h) -> int:
        return lib.chq_slab_create(C.byref(self.cfg), self.nslab, self.rank, C.byref(h))

    def sends(self, what: int, side: int) -> bool:
        """Whether message `what` crosses this side: the state halo wherever another slab
        borders it (the periodic wrap included), the FOFC message only across an internal
        boundary (include/chq.h)."""
        if what == HALO_FLAGS:
            return self.rank > 0 if side == 0 else self.rank < self.nslab - 1
        return self.zpeer[side]

    # ---- whole-mesh arrays <-> this slab ----
    def set_global(self, name: str, arr: np.ndarray) -> None:
        """Upload this slab's planes of a whole-mesh array (reference layout)."""
        face = name not in ("u0", "u1", "w", "bcc", "ecc", "flag")
        self.set(name, np.ascontiguousarray(local_slice(np.asarray(arr), self.koff, self.nk, face)))

    def active_planes(self, name: str) -> np.ndarray:
        """This slab's active planes of a field (cells: nx3 / nslab planes; faces: the same
        planes' lower faces), i.e. the slab's share of the whole mesh's active planes."""
        a = self.get(name)
        a4 = a if a.ndim == 4 else a[None]
        out = a4[:, self.ng:self.ng + self.nx3]
        return out if a.ndim == 4 else out[0]

    # ---- the C ABI of include/chq.h ----
    def halo_bytes(self, what: int, side: int) -> int:
        n = C.c_longlong()
        _check(load_library().chq_slab_halo_bytes(self._h, what, side, C.byref(n)))
        return int(n.value)

    def pack(self, what: int, buf: int, side: int, dev_ptr: int, stream) -> None:
        _check(load_library().chq_slab_pack(self._h, what, buf, side, _P(dev_ptr), stream))

    def unpack(self, what: int, buf: int, side: int, dev_ptr: int, stream) -> None:
        _check(load_library().chq_slab_unpack(self._h, what, buf, side, _P(dev_ptr), stream))

    def ctl_ptrs(self) -> tuple[int, int, int]:
        a, b, c = _P(), _P(), _P()
        _check(load_library().chq_slab_ctl(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def prime_part(self, t: float, part: int, stream) -> None:
        _check(load_library().chq_slab_prime(self._h, float(t), part, stream))

    def begin(self, stream) -> None:
        _check(load_library().chq_slab_begin(self._h, stream))

    def stage_part(self, stage: int, part: int, stream) -> None:
        _check(load_library().chq_slab_stage(self._h, stage, part, stream))

    def end(self, stream) -> None:
        _check(load_library().chq_slab_end(self._h, stream))


def out_buffer(stage: int, nstage: int) -> int:
    """State buffer a stage writes: u1/b?f1 before the last stage, u0/b?f0 at the last
    (src/main.cpp:250-268 for rk1, rk2, rk3 and SSPRK(4,3))."""
    return 0 if stage == nstage else 1


class LocalExchange:
    """All slabs of one mesh in this process, on one device and one stream."""

    def __init__(self, slabs, stream):
        import torch
        self.slabs = list(slabs)
        self.stream = stream
        n = len(self.slabs)
        self.buf = {}
        for r, s in enumerate(self.slabs):
            for side in (0, 1):
                for what in (HALO_STATE, HALO_FLAGS):
                    if s.sends(what, side):
                        nb = s.halo_bytes(what, side)
                        self.buf[(r, side, what)] = torch.empty(nb // 8, dtype=torch.int64, device="cuda")
        self.n = n
        ptrs = [s.ctl_ptrs() for s in self.slabs]
        self.nbad = [_device_view(p[0], 1, "<i4") for p in ptrs]
        self.mdt = [_device_view(p[1], 1, "<i8") for p in ptrs]
        self.rho = [_device_view(p[2], 1, "<i8") for p in ptrs]

    def _handle(self):
        return C.c_void_p(self.stream.cuda_stream)

    def halo(self, what: int, buf: int) -> None:
        h = self._handle()
        for r, s in enumerate(self.slabs):
            for side in (0, 1):
                if s.sends(what, side):
                    s.pack(what, buf, side, self.buf[(r, side, what)].data_ptr(), h)
        for r, s in enumerate(self.slabs):
            if s.sends(what, 0):   # lower ghosts: the lower neighbour's upward message
                s.unpack(what, buf, 0, self.buf[((r - 1) % self.n, 1, what)].data_ptr(), h)
            if s.sends(what, 1):   # upper ghosts: the upper neighbour's downward message
                s.unpack(what, buf, 1, self.buf[((r + 1) % self.n, 0, what)].data_ptr(), h)

    def _fold(self, ts, op) -> None:
        import torch
        with torch.cuda.stream(self.stream):
            acc = ts[0].clone()
            for t in ts[1:]:
                acc = op(acc, t)
            for t in ts:
                t.copy_(acc)

    def sum_nbad(self) -> None:
        import torch
        self._fold(self.nbad, torch.add)

    def min_steps(self, rho: bool) -> None:
        import torch
        self._fold(self.mdt, torch.minimum)
        if rho:
            self._fold(self.rho, torch.minimum)


class DistExchange:
    """One slab per process: ring messages and all-reductions over a torch.distributed group
    (NCCL for slabs on GPUs; the same calls work between CPU processes with gloo)."""

    def __init__(self, slab=None, stream=None, group=None, device: str = "cuda"):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.lower = (self.rank - 1) % self.world
        self.upper = (self.rank + 1) % self.world
        self.slab = slab
        self.stream = stream
        if slab is not None:
            import torch
            self.send, self.recv = {}, {}
            for side in (0, 1):
                for what in (HALO_STATE, HALO_FLAGS):
                    if slab.sends(what, side):
                        # the message this slab sends on `side`, and the one it receives there
                        # (every slab has the same shape: the neighbour's message for its
                        # other side has the size of this slab's own message for that side)
                        nsend = slab.halo_bytes(what, side)
                        nrecv = slab.halo_bytes(what, 1 - side)
                        self.send[(side, what)] = torch.empty(nsend // 8, dtype=torch.int64, device=device)
                        self.recv[(side, what)] = torch.empty(nrecv // 8, dtype=torch.int64, device=device)
            ptrs = slab.ctl_ptrs()
            self.nbad = _device_view(ptrs[0], 1, "<i4")
            self.mdt = _device_view(ptrs[1], 1, "<i8")
            self.rho = _device_view(ptrs[2], 1, "<i8")

    def ring(self, send_lo, send_hi, recv_lo, recv_hi, has_lo: bool, has_hi: bool) -> None:
        """Upward then downward messages with the ring neighbours: recv_lo <- lower's send_hi,
        recv_hi <- upper's send_lo. Two rounds, so that with two ranks the two messages
        between the same pair are never matched against each other."""
        dist = self.dist
        for up in (True, False):
            ops = []
            if up:
                if has_hi:
                    ops.append(dist.P2POp(dist.isend, send_hi, self.upper, self.group))
                if has_lo:
                    ops.append(dist.P2POp(dist.irecv, recv_lo, self.lower, self.group))
            else:
                if has_lo:
                    ops.append(dist.P2POp(dist.isend, send_lo, self.lower, self.group))
                if has_hi:
                    ops.append(dist.P2POp(dist.irecv, recv_hi, self.upper, self.group))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()

    def halo(self, what: int, buf: int) -> None:
        import torch
        s = self.slab
        h = C.c_void_p(self.stream.cuda_stream)
        lo, hi = s.sends(what, 0), s.sends(what, 1)
        for side, on in ((0, lo), (1, hi)):
            if on:
                s.pack(what, buf, side, self.send[(side, what)].data_ptr(), h)
        with torch.cuda.stream(self.stream):
            self.ring(self.send.get((0, what)), self.send.get((1, what)), self.recv.get((0, what)),
                      self.recv.get((1, what)), lo, hi)
        for side, on in ((0, lo), (1, hi)):
            if on:
                s.unpack(what, buf, side, self.recv[(side, what)].data_ptr(), h)

    def sum_nbad(self) -> None:
        import torch
        with torch.cuda.stream(self.stream):
            self.dist.all_reduce(self.nbad, op=self.dist.ReduceOp.SUM, group=self.group)

    def min_steps(self, rho: bool) -> None:
        import torch
        with torch.cuda.stream(self.stream):
            self.dist.all_reduce(self.mdt, op=self.dist.ReduceOp.MIN, group=self.group)
            if rho:
                self.dist.all_reduce(self.rho, op=self.dist.ReduceOp.MIN, group=self.group)


class SlabRun:
    """Cycles of one decomposed mesh: this process's slabs and their exchange (the order of
    include/chq.h's z-slab section). Every slab's work is queued on `stream`."""

    def __init__(self, slabs, exchange, stream):
        self.slabs = list(slabs)
        self.ex = exchange
        self.stream = stream
        s0 = self.slabs[0]
        self.nstage = s0.nstage
        self.fofc = bool(s0.cfg.fofc)
        self.diff = (s0.cfg.nu > 0) or (s0.cfg.kappa > 0) or (s0.cfg.eta > 0)

    def _h(self):
        return C.c_void_p(self.stream.cuda_stream)

    def prime(self, t: float = 0.0) -> None:
        h = self._h()
        for s in self.slabs:
            s.prime_part(t, 0, h)
        self.ex.halo(HALO_STATE, 0)
        for s in self.slabs:
            s.prime_part(t, 1, h)
        self.ex.min_steps(self.diff)
        for s in self.slabs:
            s.prime_part(t, 2, h)

    def cycles(self, n: int) -> None:
        h = self._h()
        for _ in range(int(n)):
            for s in self.slabs:
                s.begin(h)
            for st in range(1, self.nstage + 1):
                for s in self.slabs:
                    s.stage_part(st, 0, h)
                if self.fofc:
                    self.ex.sum_nbad()
                    self.ex.halo(HALO_FLAGS, out_buffer(st, self.nstage))
                for s in self.slabs:
                    s.stage_part(st, 1, h)
                self.ex.halo(HALO_STATE, out_buffer(st, self.nstage))
                for s in self.slabs:
                    s.stage_part(st, 2, h)
            self.ex.min_steps(self.diff)
            for s in self.slabs:
                s.end(h)

    def synchronize(self) -> None:
        self.stream.synchronize()
