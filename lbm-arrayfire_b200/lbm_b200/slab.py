"""Slab decomposition of one lattice over ranks along its slowest axis (z for D3Q27, y for D2Q9).

The reference runs one lattice on one device; this is the layer for lattices beyond one GPU's memory
(or for strong scaling).  Rank r of R holds planes [p0, p1) of the global lattice (balanced, sizes
differ by at most one) plus two ghost planes: local plane 0 stands for global plane p0 - 1 and local
plane n + 1 for global plane p1, periodic across the ends (rank 0's lower neighbour is rank R - 1),
as the single-lattice kernels wrap.

A step pulls population i of a cell from the cell c_i behind it, so interior plane 1 reads ghost plane
0 only in the directions with c = +1 along the axis and plane n reads ghost plane n + 1 only in those
with c = -1 (Q/3 of the Q: 3 of 9, 9 of 27).  After every step each rank sends the c = +1 populations
of its plane n up and the c = -1 populations of its plane 1 down, as stored words (`face_get` /
`face_set` on the C ABI: one copy per direction, no conversion), so the decomposed run is
bit-identical to the undivided lattice.  Ghost cells take a bounce-back solid class: their own updates
are never read, and bounce-back keeps them finite.  The exchange is point-to-point
(`torch.distributed` isend/irecv; NCCL over NVLink on GPUs, gloo on CPUs) on the lattice's own stream,
and it is the only data-path communication.  Shan-Chen is not decomposed (its force needs psi of the
neighbour planes as a second exchange per step).

`Slab` is one rank's part (one process per GPU).  `SlabSet` holds every rank's part in one process and
exchanges by plain copies, for tests and for several slabs on one device.
"""
from __future__ import annotations

import numpy as np

from . import (BGK, BOUNCE, D3Q27, MAX_CLASSES, MRT, SET_RHO, SET_UX, SET_UY, SET_UZ, STORAGE_BYTES, Desc,
               Lattice, classes_of, set_classes, velocities)

__all__ = ["split_planes", "axis_dirs", "local_problem", "scatter_populations", "Slab", "SlabSet"]

def split_planes(n: int, world: int):
    """[(p0, p1)] per rank: n planes in `world` contiguous runs whose sizes differ by at most one."""
    if world < 1 or n < world:
        raise ValueError(f"{n} planes cannot be split over {world} ranks (at least one plane each)")
    base, extra = divmod(n, world)
    out, p = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((p, p + k))
        p += k
    return out


def axis_dirs(lattice: int):
    """(up, down): the directions with c = +1 and with c = -1 along the slowest axis."""
    cx, cy, cz, _, _ = velocities(lattice)
    c = np.asarray(cz if lattice == D3Q27 else cy)
    return [int(i) for i in np.flatnonzero(c == 1)], [int(i) for i in np.flatnonzero(c == -1)]


def _planes(d: Desc) -> int:
    return d.nz if d.dim == 3 else d.ny


def local_problem(desc: Desc, mask, p0: int, p1: int):
    """Descriptor and class mask of the slab [p0, p1) with its two ghost planes.

    The ghost class is appended to the descriptor's classes: full-way bounce-back with rho and u set
    to zero, as the reference's solid cells."""
    if desc.collision not in (BGK, MRT):
        raise ValueError("slab decomposition covers BGK and MRT (Shan-Chen needs a psi exchange)")
    if desc.n_classes >= MAX_CLASSES:
        raise ValueError("no class index left for the ghost planes")
    n = p1 - p0
    d = Desc.from_buffer_copy(desc)
    if d.dim == 3:
        d.nz = n + 2
    else:
        d.ny = n + 2
    ghost = d.n_classes
    classes = classes_of(desc) + [(BOUNCE | SET_RHO | SET_UX | SET_UY | SET_UZ, 0.0, 0.0, 0.0, 0.0)]
    set_classes(d, classes)
    cells = desc.cells // _planes(desc)
    m = np.full((n + 2, cells), ghost, dtype=np.uint8)
    if mask is not None:
        g = np.asarray(mask, dtype=np.uint8).ravel(order="F").reshape(_planes(desc), cells)
        m[1:n + 1] = g[p0:p1]
    else:
        m[1:n + 1] = 0
    d.mask = None
    return d, m.ravel()


def scatter_populations(desc: Desc, F, p0: int, p1: int) -> np.ndarray:
    """The slab's part of global populations F (flat [x, y(, z), i]), ghost planes included."""
    P = _planes(desc)
    G = np.asarray(F).reshape(desc.q, P, desc.cells // P)
    idx = np.arange(p0 - 1, p1 + 1) % P
    return np.ascontiguousarray(G[:, idx, :]).ravel()


def _interior(lat, n: int, dtype=np.float64) -> np.ndarray:
    F = lat.get_populations(dtype)
    return F.reshape(lat.q, n + 2, -1)[:, 1:n + 1, :]


class Slab:
    """One rank's slab of a lattice, stepped with halo exchanges over a torch.distributed group.

    lattice_factory(desc, mask) builds the local stepper (default: a GPU `Lattice`); it must offer
    step, face_get, face_set, get_populations, set_populations, set_stream and face_cells."""

    def __init__(self, desc: Desc, mask, F0, rank: int, world: int, group=None, device=None,
                 lattice_factory=None):
        import torch
        import torch.distributed as dist

        if F0 is None:
            raise ValueError("F0 (global start populations) is required")
        self.dist, self.group, self.rank, self.world = dist, group, rank, world
        self.global_desc = desc
        self.p0, self.p1 = split_planes(_planes(desc), world)[rank]
        self.n = self.p1 - self.p0
        self.desc, self.mask = local_problem(desc, mask, self.p0, self.p1)
        self.lat = (lattice_factory or Lattice)(self.desc, self.mask)
        if hasattr(self.lat, "set_cell_offset"):
            # local plane 0 is global plane p0 - 1: the slab's cells hash (stochastic rounding) like the
            # undivided lattice's
            self.lat.set_cell_offset((self.p0 - 1) * (desc.cells // _planes(desc)))
        self.up_dirs, self.down_dirs = axis_dirs(desc.lattice)
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        if self.device.type == "cuda":
            # one stream for the steps, the face copies and the NCCL transfers: ordered without events
            self.lat.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
        # faces travel as raw bytes of the stored words (NCCL has no 16-bit integer type; a
        # point-to-point transfer never touches the values); an injected stepper uses FP64 words
        k = len(self.up_dirs) * self.lat.face_cells()
        word, k = (torch.uint8, k * STORAGE_BYTES[self.desc.storage]) if lattice_factory is None else (torch.float64, k)
        self._buf = {name: torch.empty(k, dtype=word, device=self.device)
                     for name in ("send_up", "send_down", "recv_down", "recv_up")}
        self.lat.set_populations(scatter_populations(desc, F0, self.p0, self.p1))

    def _pack(self):
        self.lat.face_get(self.n, self.up_dirs, self._buf["send_up"])
        self.lat.face_get(1, self.down_dirs, self._buf["send_down"])

    def _unpack(self, from_down, from_up):
        self.lat.face_set(0, self.up_dirs, from_down)
        self.lat.face_set(self.n + 1, self.down_dirs, from_up)

    def exchange(self):
        """Fill both ghost planes from the neighbours' boundary planes (the same steps on every rank)."""
        b = self._buf
        self._pack()
        if self.world == 1:
            self._unpack(b["send_up"], b["send_down"])
            return
        dist = self.dist
        up, down = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        ops = [dist.P2POp(dist.isend, b["send_up"], up, self.group, tag=1),
               dist.P2POp(dist.irecv, b["recv_down"], down, self.group, tag=1),
               dist.P2POp(dist.isend, b["send_down"], down, self.group, tag=2),
               dist.P2POp(dist.irecv, b["recv_up"], up, self.group, tag=2)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        self._unpack(b["recv_down"], b["recv_up"])

    def step(self, n: int = 1):
        for _ in range(n):
            self.lat.step(1)
            self.exchange()

    def interior_populations(self, dtype=np.float64) -> np.ndarray:
        """This rank's planes, [Q, n, plane cells]."""
        return _interior(self.lat, self.n, dtype)

    def gather_populations(self, dtype=np.float64):
        """Global populations (flat [x, y(, z), i]) on every rank (all_gather_object: for checks)."""
        if self.world == 1:
            return self.interior_populations(dtype).ravel()
        parts = [None] * self.world
        self.dist.all_gather_object(parts, self.interior_populations(dtype), group=self.group)
        return np.concatenate(parts, axis=1).ravel()

    def close(self):
        """Release the slab's lattice (its device buffers)."""
        if hasattr(self.lat, "close"):
            self.lat.close()

    def sums(self) -> np.ndarray:
        """FP64 mass and momentum of the whole lattice (a sum over ranks)."""
        import torch
        local = torch.tensor(_sums(self.global_desc.lattice, self.interior_populations()), dtype=torch.float64,
                             device=self.device)
        if self.world > 1:
            self.dist.all_reduce(local, group=self.group)
        return local.cpu().numpy()


def _sums(lattice: int, Fi: np.ndarray) -> np.ndarray:
    cx, cy, cz, _, _ = velocities(lattice)
    per_dir = Fi.reshape(Fi.shape[0], -1).sum(axis=1)
    return np.array([per_dir.sum(), per_dir @ np.asarray(cx, float), per_dir @ np.asarray(cy, float),
                     per_dir @ np.asarray(cz, float)])


class SlabSet:
    """Every slab of a decomposed lattice in one process, exchanged by plain copies (no collective).

    The same planes, ghost classes and exchange order as `Slab`, for parity tests on one device and
    for decompositions whose slabs share a GPU."""

    def __init__(self, desc: Desc, mask, F0, parts: int, lattice_factory=None):
        self.global_desc = desc
        self.ranges = split_planes(_planes(desc), parts)
        self.up_dirs, self.down_dirs = axis_dirs(desc.lattice)
        self.lats, self.ns = [], []
        for p0, p1 in self.ranges:
            d, m = local_problem(desc, mask, p0, p1)
            lat = (lattice_factory or Lattice)(d, m)
            if hasattr(lat, "set_cell_offset"):
                lat.set_cell_offset((p0 - 1) * (desc.cells // _planes(desc)))
            lat.set_populations(scatter_populations(desc, F0, p0, p1))
            self.lats.append(lat)
            self.ns.append(p1 - p0)
        k = len(self.up_dirs) * self.lats[0].face_cells()
        word = {4: np.float32, 8: np.float64, 2: np.uint16}[STORAGE_BYTES[desc.storage]] \
            if lattice_factory is None else np.float64
        self._up = [np.empty(k, dtype=word) for _ in self.lats]
        self._down = [np.empty(k, dtype=word) for _ in self.lats]

    def exchange(self):
        R = len(self.lats)
        for r, lat in enumerate(self.lats):
            lat.face_get(self.ns[r], self.up_dirs, self._up[r])
            lat.face_get(1, self.down_dirs, self._down[r])
        for r, lat in enumerate(self.lats):
            lat.face_set(0, self.up_dirs, self._up[(r - 1) % R])
            lat.face_set(self.ns[r] + 1, self.down_dirs, self._down[(r + 1) % R])

    def step(self, n: int = 1):
        for _ in range(n):
            for lat in self.lats:
                lat.step(1)
            self.exchange()

    def gather_populations(self, dtype=np.float64) -> np.ndarray:
        return np.concatenate([_interior(lat, n, dtype) for lat, n in zip(self.lats, self.ns)], axis=1).ravel()

    def sums(self) -> np.ndarray:
        return sum(_sums(self.global_desc.lattice, _interior(lat, n)) for lat, n in zip(self.lats, self.ns))

    def close(self):
        for lat in self.lats:
            if hasattr(lat, "close"):
                lat.close()
