"""Block partition of one mesh over several GPUs (one process per GPU).

The reference distributes its blocks over MPI ranks along a space-filling
curve (source/amr.f90:1730-2061), exchanges the blocks that border another
rank before each ghost fill (boundary.f90:174-291, :357-555) and reduces
the time step with MPI_ALLREDUCE(min) (hydro_solver.f90:198).  Here:

* ``make_plan`` cuts the block list, ordered along a Hilbert curve (or a
  Morton curve), into contiguous, equal-count shares; each rank's context holds its own blocks plus halo
  copies of every face neighbour another rank owns
  (``wx3d_set_mesh_halo``).
* ``Rank.step`` runs a main-loop iteration in parts (``wx3d_step_part``):
  global CFL minimum, U halo exchange, predictor, UP halo exchange,
  corrector + viscous step, source terms.  Halo blocks travel as the four
  cell layers next to each face that borders the receiver
  (``wx3d_pack_faces``), or whole.
* Transports: ``LocalGroup`` moves the blocks of several ranks that live in
  one process on one device (the test of the partitioned algorithm on a
  single GPU); ``TorchDist`` uses torch.distributed (NCCL between GPUs:
  all_reduce(MIN) for dt, batched isend/irecv of device buffers).

No kernel waits on another process: every exchange is a host-ordered
sequence of pack, transfer and unpack between the parts of the step.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .mesh import BlockTree

FACE_CELLS = 4 * 16 * 16   # cells of one face slab (wx3d_pack_faces)


def face_neighbours_by_face(tree: BlockTree, leaves: set, bid: int) -> list:
    """Active blocks across each of the six faces of ``bid`` (LEFT..TOP):
    same level, the coarser block covering the region, or the four finer
    blocks touching the face (the cases of amr.f90:539-631)."""
    out = [set() for _ in range(6)]
    for f in range(6):
        n = tree.neighbour_region(bid, f)
        if n is None:
            continue
        b = n
        while b != -1 and b not in leaves:
            b = tree.father(b)
        if b != -1:
            out[f].add(b)
            continue
        ax, side = f // 2, f % 2
        for c in tree.children(n):
            _, cx = tree.coords(c)
            if (cx[ax] & 1) == (0 if side else 1):
                out[f].add(c)
    return out


def face_neighbours(tree: BlockTree, leaves: set, bid: int) -> set:
    """Active blocks across any of the six faces of ``bid``."""
    return set().union(*face_neighbours_by_face(tree, leaves, bid))


@dataclass
class Plan:
    rank: int
    owned: list                                # bIDs, in the order of the space-filling curve
    halo: list                                 # bIDs of other ranks' blocks this rank reads
    send: dict = field(default_factory=dict)   # peer -> owned bIDs the peer needs
    recv: dict = field(default_factory=dict)   # peer -> halo bIDs that peer sends
    # the same exchange as (bID, face) slabs: the faces of each halo block
    # that border the receiver's own blocks, in the same order on both sides
    send_faces: dict = field(default_factory=dict)
    recv_faces: dict = field(default_factory=dict)

    @property
    def local_blocks(self) -> np.ndarray:
        return np.asarray(self.owned + self.halo, dtype=np.int32)

    def slot(self, bid: int) -> int:
        return self._slots[bid]

    def __post_init__(self):
        self._slots = {b: s for s, b in enumerate(self.owned + self.halo)}


def make_plan(local_blocks, nbroot, maxlev: int, nranks: int, order: str = "hilbert") -> list:
    """Equal-count contiguous shares of the block list along a space-filling
    curve ("hilbert", as the reference's doBalance, amr.f90:1730-1922; or
    "morton"), the halo of each share and the send/receive lists between
    ranks."""
    tree = BlockTree(tuple(nbroot), maxlev)
    leaves = {int(b) for b in local_blocks if b != -1}
    tree.leaves = leaves
    if order == "hilbert":
        blocks = tree.hilbert_order()
    elif order == "morton":
        blocks = tree.morton_order()
    else:
        raise ValueError(f"unknown block order {order!r}")
    owner = {}
    bounds = np.linspace(0, len(blocks), nranks + 1).round().astype(int)
    shares = [blocks[bounds[r]:bounds[r + 1]] for r in range(nranks)]
    for r, share in enumerate(shares):
        for b in share:
            owner[b] = r
    pos = {b: i for i, b in enumerate(blocks)}
    plans = []
    for r, share in enumerate(shares):
        halo = set()
        for b in share:
            halo |= {n for n in face_neighbours(tree, leaves, b) if owner[n] != r}
        plans.append(Plan(r, list(share), sorted(halo, key=pos.get)))
    for p in plans:
        for b in p.halo:
            q = owner[b]
            p.recv.setdefault(q, []).append(b)
            plans[q].send.setdefault(p.rank, []).append(b)
            for f, across in enumerate(face_neighbours_by_face(tree, leaves, b)):
                if any(owner[n] == p.rank for n in across):
                    p.recv_faces.setdefault(q, []).append((b, f))
                    plans[q].send_faces.setdefault(p.rank, []).append((b, f))
    return plans


class Rank:
    """One rank's context: its blocks plus halo copies, stepped in parts."""

    def __init__(self, prob, plan: Plan, stream_handle: int | None = None):
        from .solver import Walicxe3D
        self.plan = plan
        self.prob = prob
        lb = plan.local_blocks
        # with more ranks than blocks a share is empty: the rank still takes
        # part in the dt minimum, like a process whose localBlocks are all -1
        self.w = Walicxe3D(prob.cfg, max(1, len(lb)))
        if stream_handle is not None:
            self.w.set_stream(stream_handle)
        nh = len(plan.halo)
        halo_slots = np.arange(len(plan.owned), len(lb), dtype=np.int32)
        lib = self.w.lib
        _lib.check(lib.wx3d_set_mesh_halo(self.w.ctx, len(lb), lb.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nh,
                                          halo_slots.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
                   "wx3d_set_mesh_halo", self.w.ctx)
        self.w.nslots = len(lb)
        gslot = {int(b): s for s, b in enumerate(prob.local_blocks)}
        self.w.upload(np.ascontiguousarray(prob.U[[gslot[int(b)] for b in lb]]))
        if prob.cooltable is not None:
            self.w.set_cooltable(*prob.cooltable)
        if prob.cooltable_metal is not None:
            self.w.set_cooltable_metal(*prob.cooltable_metal)
        if prob.cooltable_schure is not None:
            self.w.set_cooltable_schure(*prob.cooltable_schure)
        if prob.winds:
            raise NotImplementedError("wind sources are not supported in a partitioned run")
        self.w.set_state(time=0.0, dt=0.0, it=0, nextout=1)
        self.neq = prob.cfg.neqtot

    # -- library calls --------------------------------------------------------
    def _slots(self, bids):
        return np.asarray([self.plan.slot(b) for b in bids], dtype=np.int32)

    def pack(self, array: int, bids, dbuf):
        s = self._slots(bids)
        _lib.check(self.w.lib.wx3d_pack_blocks(self.w.ctx, array, len(s), s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                               ctypes.c_void_p(dbuf.data_ptr())), "wx3d_pack_blocks", self.w.ctx)

    def unpack(self, array: int, bids, dbuf):
        s = self._slots(bids)
        _lib.check(self.w.lib.wx3d_unpack_blocks(self.w.ctx, array, len(s),
                                                 s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                 ctypes.c_void_p(dbuf.data_ptr())), "wx3d_unpack_blocks", self.w.ctx)

    def pack_faces(self, array: int, items, dbuf):
        s = self._slots([b for b, _ in items])
        f = np.asarray([f for _, f in items], dtype=np.int32)
        _lib.check(self.w.lib.wx3d_pack_faces(self.w.ctx, array, len(s), s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                              f.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                              ctypes.c_void_p(dbuf.data_ptr())), "wx3d_pack_faces", self.w.ctx)

    def unpack_faces(self, array: int, items, dbuf):
        s = self._slots([b for b, _ in items])
        f = np.asarray([f for _, f in items], dtype=np.int32)
        _lib.check(self.w.lib.wx3d_unpack_faces(self.w.ctx, array, len(s),
                                                s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                f.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                ctypes.c_void_p(dbuf.data_ptr())), "wx3d_unpack_faces", self.w.ctx)

    def exchange_bytes(self, faces: bool = True) -> int:
        """Bytes this rank sends per exchange (one array)."""
        if faces:
            return sum(len(v) for v in self.plan.send_faces.values()) * self.neq * FACE_CELLS * 8
        return sum(len(v) for v in self.plan.send.values()) * self.neq * 4096 * 8

    def dtmin(self) -> float:
        v = ctypes.c_double()
        _lib.check(self.w.lib.wx3d_get_dtmin(self.w.ctx, ctypes.byref(v)), "wx3d_get_dtmin", self.w.ctx)
        return v.value

    def set_dtmin(self, v: float):
        _lib.check(self.w.lib.wx3d_set_dtmin(self.w.ctx, ctypes.c_double(v)), "wx3d_set_dtmin", self.w.ctx)

    def part(self, p: int):
        _lib.check(self.w.lib.wx3d_step_part(self.w.ctx, p), "wx3d_step_part", self.w.ctx)

    def owned_state(self) -> np.ndarray:
        return self.w.download(len(self.plan.owned))


class LocalGroup:
    """Transport for several ranks in one process on one device: the halo
    face slabs (or, with faces=False, whole blocks) move by device-to-device
    copies through a staging buffer."""

    def __init__(self, ranks, faces: bool = True):
        self.ranks = ranks
        self.faces = faces

    def step(self):
        import torch
        g = min(r.dtmin() for r in self.ranks)
        for r in self.ranks:
            r.set_dtmin(g)
            r.part(0)
        self._exchange(0)
        for r in self.ranks:
            r.part(1)
        self._exchange(1)
        for r in self.ranks:
            r.part(2)
        for r in self.ranks:
            r.part(3)
        torch.cuda.synchronize()

    def _exchange(self, array: int):
        import torch
        for src in self.ranks:
            if self.faces:
                for peer, items in src.plan.send_faces.items():
                    buf = torch.empty(len(items) * src.neq * FACE_CELLS, dtype=torch.float64, device="cuda")
                    src.pack_faces(array, items, buf)
                    self.ranks[peer].unpack_faces(array, items, buf)
            else:
                for peer, bids in src.plan.send.items():
                    buf = torch.empty(len(bids) * src.neq * 4096, dtype=torch.float64, device="cuda")
                    src.pack(array, bids, buf)
                    self.ranks[peer].unpack(array, bids, buf)

    def gather(self) -> dict:
        out = {}
        for r in self.ranks:
            U = r.owned_state()
            for s, b in enumerate(r.plan.owned):
                out[b] = U[s]
        return out


class TorchDist:
    """Transport between processes through torch.distributed (NCCL between
    GPUs): all_reduce(MIN) of the CFL minimum, batched isend/irecv of the
    halo face slabs (or, with faces=False, whole blocks) in device
    buffers."""

    def __init__(self, rank: Rank, device="cuda", faces: bool = True):
        self.r = rank
        self.device = device
        self.faces = faces

    def step(self):
        import torch
        import torch.distributed as dist
        t = torch.tensor([self.r.dtmin()], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        self.r.set_dtmin(float(t.item()))
        self.r.part(0)
        self.exchange(0)
        self.r.part(1)
        self.exchange(1)
        self.r.part(2)
        self.r.part(3)

    def exchange(self, array: int):
        import torch
        import torch.distributed as dist
        plan = self.r.plan
        send, recv = (plan.send_faces, plan.recv_faces) if self.faces else (plan.send, plan.recv)
        n = self.r.neq * (FACE_CELLS if self.faces else 4096)
        pack = self.r.pack_faces if self.faces else self.r.pack
        unpack = self.r.unpack_faces if self.faces else self.r.unpack
        ops, sends, recvs = [], [], []
        for peer in sorted(set(send) | set(recv)):
            if peer in send:
                items = send[peer]
                buf = torch.empty(len(items) * n, dtype=torch.float64, device=self.device)
                pack(array, items, buf)
                sends.append(buf)
                ops.append(dist.P2POp(dist.isend, buf, peer))
            if peer in recv:
                items = recv[peer]
                buf = torch.empty(len(items) * n, dtype=torch.float64, device=self.device)
                recvs.append((items, buf))
                ops.append(dist.P2POp(dist.irecv, buf, peer))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if str(self.device).startswith("cuda"):
            torch.cuda.synchronize()
        for items, buf in recvs:
            unpack(array, items, buf)
