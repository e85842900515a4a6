"""Block partition over several ranks: the plan (CPU), the exchange
choreography between two gloo processes (CPU), and on one GPU the
partitioned step of several in-process ranks against the single-context
step."""
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from walicxe3d_b200 import config as C
from walicxe3d_b200 import problems
from walicxe3d_b200.mesh import BlockTree
from walicxe3d_b200.partition import FACE_CELLS, face_neighbours, face_neighbours_by_face, make_plan


def _amr():
    return problems.blast_amr(nroot=3, maxlev=3, shell_radius=0.1, shell_width=0.02)


def test_plan_covers_every_neighbour_and_is_symmetric():
    prob = _amr()
    for n in (2, 3, 5):
        plans = make_plan(prob.local_blocks, prob.cfg.nbroot, prob.cfg.maxlev, n)
        owned = [b for p in plans for b in p.owned]
        assert sorted(owned) == sorted(int(b) for b in prob.local_blocks)
        tree = BlockTree(prob.cfg.nbroot, prob.cfg.maxlev)
        leaves = set(owned)
        for p in plans:
            have = set(p.owned) | set(p.halo)
            for b in p.owned:
                assert face_neighbours(tree, leaves, b) <= have
            assert not set(p.halo) & set(p.owned)
            for q, bids in p.recv.items():
                assert plans[q].send[p.rank] == bids
                assert set(bids) <= set(plans[q].owned)
            # face slabs: the same halo blocks, each face bordering this rank's blocks
            for q, items in p.recv_faces.items():
                assert plans[q].send_faces[p.rank] == items
                assert {b for b, _ in items} == set(p.recv[q])
                for b, f in items:
                    assert face_neighbours_by_face(tree, leaves, b)[f] & set(p.owned)
            for b in p.owned:
                for f, across in enumerate(face_neighbours_by_face(tree, leaves, b)):
                    for h in across & set(p.halo):
                        # b reads h across h's opposite face: that slab is received
                        g = f ^ 1
                        assert (h, g) in {it for its in p.recv_faces.values() for it in its}


def test_more_ranks_than_blocks_leaves_empty_shares():
    """Six shares of Brio-Wu's four blocks: every block owned exactly once,
    two shares empty, and an empty share neither sends nor receives."""
    prob = problems.brio_wu(4)
    plans = make_plan(prob.local_blocks, prob.cfg.nbroot, prob.cfg.maxlev, 6)
    owned = [b for p in plans for b in p.owned]
    assert sorted(owned) == sorted(int(b) for b in prob.local_blocks)
    empty = [p for p in plans if not p.owned]
    assert len(empty) == 2
    for p in empty:
        assert not p.halo and not p.send and not p.recv and not p.send_faces and not p.recv_faces
        assert len(p.local_blocks) == 0
    for p in plans:
        for q in p.send:
            assert plans[q].owned


def test_face_neighbours_of_a_three_level_mesh_are_levels_apart_by_one():
    prob = _amr()
    tree = BlockTree(prob.cfg.nbroot, prob.cfg.maxlev)
    leaves = set(int(b) for b in prob.local_blocks)
    for b in leaves:
        for n in face_neighbours(tree, leaves, b):
            assert n in leaves and abs(tree.level(n) - tree.level(b)) <= 1


class _CpuRank:
    """A stand-in for Rank on the CPU: blocks are rows of a tensor."""

    def __init__(self, plan, neq, values):
        self.plan, self.neq = plan, neq
        self.data = {b: torch.full((neq * 4096,), float(values[b])) for b in plan.owned}
        self.data.update({b: torch.zeros(neq * 4096) for b in plan.halo})
        self.vals = [float(values[b]) for b in plan.owned]
        self.dt = None

    def dtmin(self):
        return min(self.vals, default=1.0e30)   # no block: getTimestep's 1e30

    def set_dtmin(self, v):
        self.dt = v

    def part(self, p):
        pass

    def pack(self, array, bids, buf):
        buf.copy_(torch.cat([self.data[b] for b in bids]))

    def unpack(self, array, bids, buf):
        for i, b in enumerate(bids):
            self.data[b] = buf[i * self.neq * 4096:(i + 1) * self.neq * 4096].clone()

    def pack_faces(self, array, items, buf):
        n = self.neq * FACE_CELLS
        buf.copy_(torch.cat([self.data[b][:n] for b, _ in items]))

    def unpack_faces(self, array, items, buf):
        n = self.neq * FACE_CELLS
        for i, (b, f) in enumerate(items):
            self.data[(b, f)] = buf[i * n:(i + 1) * n].clone()


def _free_port() -> int:
    """An ephemeral port the kernel hands out on 127.0.0.1 (released before
    the ranks bind it), so concurrent test runs do not collide."""
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, world, port, q, faces):
    import torch.distributed as dist
    from walicxe3d_b200.partition import TorchDist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob = _amr()
        plans = make_plan(prob.local_blocks, prob.cfg.nbroot, prob.cfg.maxlev, world)
        values = {int(b): float(b) for b in prob.local_blocks}
        r = _CpuRank(plans[rank], 2, values)
        TorchDist(r, device="cpu", faces=faces).exchange(0)
        if faces:
            items = [it for its in plans[rank].recv_faces.values() for it in its]
            ok = bool(items) and all(bool(torch.all(r.data[(b, f)] == float(b))) for b, f in items)
        else:
            ok = all(bool(torch.all(r.data[b] == float(b))) for b in plans[rank].halo)
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        q.put((rank, ok, len(plans[rank].halo), float(t.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("faces", [False, True])
def test_halo_exchange_between_two_gloo_processes(faces):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(r, 2, port, q, faces)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(ok and nh > 0 and m == 1.0 for _, ok, nh, m in res), res


def _step_worker(rank, world, port, q):
    import torch.distributed as dist
    from walicxe3d_b200.partition import TorchDist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob = problems.brio_wu(2)
        plans = make_plan(prob.local_blocks, prob.cfg.nbroot, prob.cfg.maxlev, world)
        values = {int(b): 10.0 + float(b) for b in prob.local_blocks}
        r = _CpuRank(plans[rank], 2, values)
        TorchDist(r, device="cpu", faces=True).step()
        items = [it for its in plans[rank].recv_faces.values() for it in its]
        ok = all(bool(torch.all(r.data[(b, f)] == values[b])) for b, f in items)
        q.put((rank, ok, len(plans[rank].owned), len(items), r.dt))
    finally:
        dist.destroy_process_group()


def test_step_choreography_with_an_empty_rank_over_gloo():
    """Three gloo processes over Brio-Wu's two blocks: the middle rank owns
    nothing, contributes getTimestep's 1e30 to the dt minimum, sends and
    receives no slab, and the step completes on every rank with the same
    dt; the two other ranks receive each other's face slab."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_step_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [n for _, _, n, _, _ in res] == [1, 0, 1]
    assert [k for _, _, _, k, _ in res] == [1, 0, 1]
    assert all(ok for _, ok, _, _, _ in res)
    assert all(dt == 11.0 for *_, dt in res)


@pytest.mark.gpu
@pytest.mark.parametrize("name,nranks,faces", [("amr", 2, True), ("amr", 3, True), ("snr-h", 2, True),
                                               ("brio-wu", 2, True), ("amr", 3, False),
                                               ("brio-wu", 6, True)])
def test_partitioned_step_equals_single_context(name, nranks, faces):
    """Ranks on one device exchanging their halo face slabs (or whole halo
    blocks) reproduce the single-context run bit for bit: same fluxes per
    block, same global dt.  Six ranks over Brio-Wu's four blocks leave two
    ranks without a block; they still take part in the dt minimum."""
    from walicxe3d_b200.partition import LocalGroup, Rank
    from walicxe3d_b200.solver import from_problem
    prob = {"amr": _amr, "snr-h": lambda: problems.snr_h(nroot=2, maxlev=2),
            "brio-wu": lambda: problems.brio_wu(4)}[name]()
    ref = from_problem(prob)
    plans = make_plan(prob.local_blocks, prob.cfg.nbroot, prob.cfg.maxlev, nranks)
    group = LocalGroup([Rank(prob, p) for p in plans], faces=faces)
    for _ in range(6):
        ref.step()
        group.step()
    U = ref.download()
    parts = group.gather()
    for s, b in enumerate(prob.local_blocks):
        assert np.array_equal(parts[int(b)], U[s]), f"block {b}"
    sr = ref.state
    for r in group.ranks:
        st = r.w.state
        assert (st.time, st.dt, st.it) == (sr.time, sr.dt, sr.it)


def test_hilbert_order_walks_face_neighbours():
    """The Hilbert keys of a uniform 2^k cube are a permutation of 0..n^3-1
    and consecutive blocks along the curve share a face (the locality the
    reference's Hilbert load balance relies on); on an AMR mesh the keys of
    the leaves are distinct."""
    from walicxe3d_b200 import problems
    from walicxe3d_b200.mesh import BlockTree
    for n in (2, 4, 8):
        t = BlockTree((n, n, n), 1).roots()
        assert sorted(t.hilbert_key(b) for b in t.leaves) == list(range(n ** 3))
        order = t.hilbert_order()
        for a, b in zip(order, order[1:]):
            xa, xb = t.coords(a)[1], t.coords(b)[1]
            assert sum(abs(i - j) for i, j in zip(xa, xb)) == 1
    prob = problems.blast_amr(nroot=4, maxlev=3)
    prob.tree.leaves = {int(b) for b in prob.local_blocks}
    keys = [prob.tree.hilbert_key(int(b)) for b in prob.local_blocks]
    assert len(set(keys)) == len(keys)
