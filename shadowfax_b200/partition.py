"""One mesh over several devices: the flux-pass side of the reference's
domain decomposition.

The reference orders particles along a Hilbert curve and splits them over
MPI ranks (ParticleVector::sort, src/utilities/ParticleVector.cpp:222-);
each rank tessellates its cells plus ghost copies (DelTess::add_mirrors,
src/DelTess_mpi.cpp:71-) and refreshes the ghosts' states, gradients and
fluxes every step (DelTess::update_Ws / update_gradients / update_dQs,
src/DelTess_mpi.cpp:1614, 1781, 2024).  Here the tessellation is global and
each part holds

* its owned cells (numbered first),
* ring 1: the cells that share a face with an owned cell (their gradients
  are computed locally, so no gradient exchange is needed),
* ring 2: the cells that share a face with ring 1 (state only),

with every face of the owned and ring-1 cells, the faces of owned cells
first, and each cell's face list in the global mesh's order.  The pass then
computes gradients for the owned and ring-1 cells, fluxes for the faces of
owned cells and updates only the owned cells (``sfx_mesh_set_ranges``),
which gives the owned cells exactly the values of a pass over the whole
mesh.  After each step the ring cells' W and mass come from their owners:
one exchange of ``S + 1`` doubles per ring cell (``sfx_mesh_pack_cells`` /
``sfx_mesh_unpack_cells``), the lists from :func:`exchange_plan`, the
transfer by :func:`exchange_records` (torch.distributed point-to-point: NCCL
over NVLink between GPUs, gloo on the CPU).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import Mesh

KIND_REAL, KIND_PERIODIC, KIND_MIRROR = 0, 1, 2


def hilbert_keys(pos: np.ndarray) -> np.ndarray:
    """Hilbert-curve index of points in [0, 1)^dim (21 bits per axis in 3D,
    31 in 2D), by J. Skilling's transpose method ("Programming the Hilbert
    curve", AIP Conf. Proc. 707, 2004), vectorised over the points."""
    n, dim = pos.shape
    bits = 21 if dim == 3 else 31
    q = np.clip(np.floor(np.asarray(pos, np.float64) * (1 << bits)), 0, (1 << bits) - 1)
    X = [q[:, i].astype(np.uint64) for i in range(dim)]
    one = np.uint64(1)
    M = np.uint64(1 << (bits - 1))
    Q = M
    while Q > one:
        P = Q - one
        for i in range(dim):
            hit = (X[i] & Q) != 0
            X[0] = np.where(hit, X[0] ^ P, X[0])
            t = np.where(hit, np.uint64(0), (X[0] ^ X[i]) & P)
            X[0] ^= t
            X[i] ^= t
        Q >>= one
    for i in range(1, dim):
        X[i] ^= X[i - 1]
    t = np.zeros(n, np.uint64)
    Q = M
    while Q > one:
        t = np.where((X[dim - 1] & Q) != 0, t ^ (Q - one), t)
        Q >>= one
    for i in range(dim):
        X[i] ^= t
    key = np.zeros(n, np.uint64)
    for b in range(bits - 1, -1, -1):
        for i in range(dim):
            key = (key << one) | ((X[i] >> np.uint64(b)) & one)
    return key


def partition(mesh: Mesh, nparts: int) -> np.ndarray:
    """Owner rank of every cell: contiguous pieces of the Hilbert order of
    the generators with about equal work (faces + 1 per cell)."""
    if nparts < 1 or nparts > mesh.n_cells:
        raise ValueError("need 1 <= nparts <= cells")
    order = np.argsort(hilbert_keys(mesh.cell_pos), kind="stable")
    cost = np.diff(mesh.cell_face_offset).astype(np.int64)[order] + 1
    cum = np.cumsum(cost)
    cuts = np.searchsorted(cum, cum[-1] * np.arange(1, nparts) / nparts, side="left")
    part_of_rank = np.zeros(mesh.n_cells, np.int32)
    for c in cuts:
        part_of_rank[c + 1:] += 1
    owner = np.empty(mesh.n_cells, np.int32)
    owner[order] = part_of_rank
    if np.bincount(owner, minlength=nparts).min() == 0:
        raise ValueError("a part without cells")
    return owner


def _neighbours(mesh: Mesh, cells: np.ndarray) -> np.ndarray:
    """cells across a real or periodic face of any of `cells` (boolean mask)"""
    L, R, K = mesh.face_left, mesh.face_right, mesh.face_kind
    link = K != KIND_MIRROR
    out = np.zeros(mesh.n_cells, bool)
    out[R[link & cells[L]]] = True
    out[L[link & cells[np.where(link, R, 0)]]] = True
    return out


@dataclass
class Part:
    """one part: its local mesh and where its cells and faces come from"""
    rank: int
    mesh: Mesh
    cells: np.ndarray      # global cell id of each local cell
    faces: np.ndarray      # global face id of each local face
    n_own: int             # owned cells: local [0, n_own)
    n_grad: int            # owned + ring 1: local [0, n_grad)
    n_flux: int            # faces of owned cells: local [0, n_flux)


def _csr_faces(mesh: Mesh, mask: np.ndarray) -> np.ndarray:
    off = mesh.cell_face_offset
    sel = np.repeat(mask, np.diff(off))
    return np.unique(mesh.cell_face_index[sel])


def _periodic_twins(mesh: Mesh) -> np.ndarray:
    """for each face across a periodic boundary, the other cell's copy of it
    (left and right swapped, image shifted the other way); -1 elsewhere"""
    twin = np.full(mesh.n_faces, -1, np.int64)
    per = np.flatnonzero(mesh.face_kind == KIND_PERIODIC)
    if per.size == 0:
        return twin
    L, R = mesh.face_left[per], mesh.face_right[per]
    shift = np.rint(mesh.face_right_pos[per] - mesh.cell_pos[R]).astype(np.int64)
    seen = {}
    for k, f in enumerate(per):
        seen[(int(L[k]), int(R[k]), tuple(shift[k]))] = f
    for k, f in enumerate(per):
        g = seen.get((int(R[k]), int(L[k]), tuple(-shift[k])))
        if g is not None:
            twin[f] = g
    return twin


def _with_twins(faces: np.ndarray, twin: np.ndarray) -> np.ndarray:
    t = twin[faces]
    return np.union1d(faces, t[t >= 0])


def _rings(mesh: Mesh, owner: np.ndarray, rank: int):
    """masks of the owned, ring-1 and ring-2 cells of a rank"""
    own = owner == rank
    r1 = _neighbours(mesh, own) & ~own
    r2 = _neighbours(mesh, r1) & ~own & ~r1
    return own, r1, r2


def build_part(mesh: Mesh, owner: np.ndarray, rank: int) -> Part:
    own, r1, r2 = _rings(mesh, owner, rank)
    cells = np.concatenate([np.flatnonzero(own), np.flatnonzero(r1), np.flatnonzero(r2)])
    n_own, n_grad = int(own.sum()), int(own.sum() + r1.sum())
    g2l = np.full(mesh.n_cells, -1, np.int64)
    g2l[cells] = np.arange(len(cells))
    # the split pass applies one copy of each periodic face pair (chosen by
    # its geometry) to both cells: a part holds both copies of every pair
    # at its owned and ring-1 cells, the pairs at owned cells in the flux range
    twin = _periodic_twins(mesh)
    flux = _with_twins(_csr_faces(mesh, own), twin)
    need = _with_twins(_csr_faces(mesh, own | r1), twin)
    faces = np.concatenate([flux, np.setdiff1d(need, flux, assume_unique=True)])
    f2l = np.full(mesh.n_faces, -1, np.int64)
    f2l[faces] = np.arange(len(faces))
    # each local cell's faces in its global order, restricted to local faces
    # (complete for owned and ring-1 cells)
    off = mesh.cell_face_offset
    cnt = np.diff(off)
    rows = np.repeat(np.arange(mesh.n_cells), cnt)
    keep = (g2l[rows] >= 0) & (f2l[mesh.cell_face_index] >= 0)
    lrow = g2l[rows[keep]]
    lface = f2l[mesh.cell_face_index[keep]]
    order = np.argsort(lrow, kind="stable")
    lcnt = np.bincount(lrow, minlength=len(cells))
    loff = np.zeros(len(cells) + 1, np.int32)
    loff[1:] = np.cumsum(lcnt)
    R = mesh.face_right[faces]
    kind = mesh.face_kind[faces]
    lright = np.where(kind == KIND_MIRROR, -1, g2l[np.where(kind == KIND_MIRROR, 0, R)])
    local = Mesh(
        dim=mesh.dim, periodic=mesh.periodic,
        cell_pos=mesh.cell_pos[cells], cell_centroid=mesh.cell_centroid[cells],
        cell_volume=mesh.cell_volume[cells], cell_total_area=mesh.cell_total_area[cells],
        cell_face_offset=loff, cell_face_index=lface[order].astype(np.int32),
        face_area=mesh.face_area[faces], face_midpoint=mesh.face_midpoint[faces],
        face_left=g2l[mesh.face_left[faces]].astype(np.int32),
        face_right=lright.astype(np.int32), face_kind=kind.copy(),
        face_right_pos=mesh.face_right_pos[faces],
        face_velocity=None if mesh.face_velocity is None else mesh.face_velocity[faces],
    ).normalized()
    if np.any(local.face_left < 0) or np.any((kind != KIND_MIRROR) & (lright < 0)):
        raise AssertionError("a needed face leaves the part")
    return Part(rank, local, cells, faces, n_own, n_grad, len(flux))


def exchange_plan(mesh: Mesh, owner: np.ndarray,
                  part: Part) -> dict[int, tuple[np.ndarray, np.ndarray]]:
    """Per peer p: (send, recv) local cell indices of this part.  The part
    sends the records of `send` (its owned cells in p's rings) to p and
    stores what it receives from p into `recv` (its ring cells owned by p);
    both sides list the cells in ascending global id, so the records line
    up, and every rank computes the plan from the global mesh and the owner
    array alone."""
    rank = part.rank
    world = int(owner.max()) + 1
    g2l = np.full(mesh.n_cells, -1, np.int64)
    g2l[part.cells] = np.arange(len(part.cells))
    ring = part.cells[part.n_own:]
    plan: dict[int, tuple[np.ndarray, np.ndarray]] = {}
    for p in range(world):
        if p == rank:
            continue
        recv_g = np.sort(ring[owner[ring] == p])
        _, r1p, r2p = _rings(mesh, owner, p)
        send_g = np.flatnonzero((r1p | r2p) & (owner == rank))
        if len(recv_g) or len(send_g):
            plan[p] = (g2l[send_g].astype(np.int32), g2l[recv_g].astype(np.int32))
    return plan


def exchange_records(send: dict, recv: dict, group=None) -> None:
    """Send send[p] to rank p and receive recv[p] from rank p for every peer,
    as one batch of point-to-point operations of the current process group
    (NCCL for CUDA tensors, gloo for CPU ones); returns when the received
    records are in place (for NCCL: ordered before later work on the current
    stream)."""
    import torch.distributed as dist
    ops = []
    for p in sorted(set(send) | set(recv)):
        if p in send and send[p].numel():
            ops.append(dist.P2POp(dist.isend, send[p], p, group))
        if p in recv and recv[p].numel():
            ops.append(dist.P2POp(dist.irecv, recv[p], p, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class PartitionedPass:
    """This rank's part of one mesh split over the ranks of a process group
    (plain FP64 or split, one GPU per rank): the local mesh with its two rings on the
    device, the pass restricted to it, and the ring exchange after every
    step.  The owned cells' W and Q equal those of a pass over the whole
    mesh, bit for bit.

    Every rank of the group constructs its PartitionedPass (the constructor
    ends with a barrier, so that the first point-to-point batch is not the
    group's first collective) and calls step() with the same arguments.  The
    context's stream becomes torch's current stream on ctx.device (set that
    device current first), for the context's other meshes too.

    Over a gloo group the records are staged through host memory and the
    status flag is a CPU tensor.  `flux_pass` replaces the device pass over
    the part (any object with FluxPass's set_ranges / set_primitive / step /
    pack_cells / unpack_cells / state working on CPU tensors); tests use it to
    run this class on CPU ranks."""

    def __init__(self, ctx, mesh: Mesh, owner: np.ndarray, rank: int, group=None,
                 flux_pass=None):
        import torch
        import torch.distributed as dist

        from .hydro import FluxPass
        self.part = build_part(mesh, owner, rank)
        self.plan = exchange_plan(mesh, owner, self.part)
        n_local = len(self.part.cells)
        for s, r in self.plan.values():
            if (len(s) and (s.min() < 0 or s.max() >= self.part.n_own)) or \
                    (len(r) and (r.min() < self.part.n_own or r.max() >= n_local)):
                raise ValueError("exchange list outside the part")
        self.group = group
        gloo = dist.is_initialized() and dist.get_backend(group) == "gloo"
        if flux_pass is None:
            self.fp = FluxPass(ctx, self.part.mesh)
            dev = torch.device("cuda", ctx.device)
            # the library's kernels on torch's current stream, so that the
            # records are packed before they are sent and stored after they
            # arrive
            ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        else:
            self.fp = flux_pass
            dev = torch.device("cpu")
        self.fp.set_ranges(self.part.n_grad, self.part.n_flux, self.part.n_own)
        # records are packed and stored on `device`; they travel from
        # `comm_device` (host memory for gloo)
        self.device = dev
        self.comm_device = torch.device("cpu") if gloo else dev
        R = mesh.dim + 3
        self.send_idx = {p: torch.as_tensor(s, device=dev) for p, (s, _) in self.plan.items()}
        self.recv_idx = {p: torch.as_tensor(r, device=dev) for p, (_, r) in self.plan.items()}
        self.send_buf = {p: torch.empty((len(s), R), dtype=torch.float64, device=dev)
                         for p, (s, _) in self.plan.items()}
        self.recv_buf = {p: torch.empty((len(r), R), dtype=torch.float64, device=dev)
                         for p, (_, r) in self.plan.items()}
        if dist.is_initialized():
            dist.barrier(group)

    def set_primitive(self, W_global: np.ndarray) -> None:
        self.fp.set_primitive(np.asarray(W_global)[self.part.cells])

    def exchange(self) -> None:
        for p, idx in self.send_idx.items():
            if idx.numel():
                self.fp.pack_cells(idx, self.send_buf[p])
        if self.comm_device == self.device:
            exchange_records(self.send_buf, self.recv_buf, self.group)
        else:
            recv = {p: b.to(self.comm_device) for p, b in self.recv_buf.items()}
            exchange_records({p: b.to(self.comm_device) for p, b in self.send_buf.items()},
                             recv, self.group)
            for p, b in recv.items():
                self.recv_buf[p].copy_(b)
        for p, idx in self.recv_idx.items():
            if idx.numel():
                self.fp.unpack_cells(idx, self.recv_buf[p])

    def step(self, dt: float, nsteps: int = 1, check: bool = True) -> None:
        """nsteps, each followed by the ring exchange.  With `check`, every
        rank reads back its step's status and the ranks agree on the worst
        one (a MAX all-reduce) before exchanging, so that a failing part
        (the reference's exceptions) stops every rank with SfxError instead
        of leaving the others waiting in the exchange."""
        import torch
        import torch.distributed as dist

        from ._lib import SfxError
        for _ in range(nsteps):
            err = None
            try:
                self.fp.step(dt, 1, stats=check)
            except SfxError as e:
                err = e
            if check and dist.is_initialized():
                flag = torch.tensor([0 if err is None else err.status], dtype=torch.int32,
                                    device=self.comm_device)
                dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=self.group)
                worst = int(flag.item())
                if worst:
                    raise err or SfxError(worst, "sfx_step on another rank")
            elif err is not None:
                raise err
            self.exchange()

    def owned_state(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(global ids, W, Q) of the owned cells"""
        W, Q = self.fp.state()
        n = self.part.n_own
        return self.part.cells[:n], W[:n], Q[:n]

