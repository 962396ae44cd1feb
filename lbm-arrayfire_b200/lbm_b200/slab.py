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
(`torch.distributed` isend/irecv; NCCL over NVLink on GPUs, gloo on CPUs) on the slab's stream,
and it is the only data-path communication.

Shan-Chen slabs carry two ghost planes per side.  The force at a cell needs psi = 1 - exp(-rho) of its
neighbours, and psi of a cell needs that cell's streamed density, so the update of the first interior
plane reads populations two planes below it: the adjacent ghost plane's c = 0 and c = +1 populations
(its streamed density, and what streams into the interior) and the far ghost plane's c = +1 ones (6 + 3
of the 9 per cell and side).  The ghost planes keep the global lattice's own cell classes there, since
psi of a boundary class depends on it.  The ghost planes' own updates are never read; the overlapped
step updates the two bottom and the two top rows beside the interior (`lbm_step_planes` runs Shan-Chen
plane sets on the one-pass window kernel).

On a GPU the exchange overlaps the interior update (`lbm_step_planes`).  Within a step the slab's
stream updates planes 2 .. n-1 in all but a few SMs, while a second (high-priority) CUDA stream, in
those few SMs (`lbm_set_reserved_sms`: the row pipeline's persistent grid would otherwise hold every
SM until it ends), updates the two boundary planes (local planes 1 and n, one strided launch), packs
their outgoing faces straight from the buffer being written, exchanges them (NCCL, or copies within
one process) and unpacks the incoming ones into that buffer's ghost planes.  The next step waits for
both streams.  D3Q27 MRT 256^3 F16S on one B200: 351 us per step with 8 SMs for the side stream
(one rank, faces copied to itself), against 470 us for step-then-exchange and 341 us for the
undivided lattice; Shan-Chen 4096^2 F32 326 us against 437 and 296.  Slabs with no plane that the
neighbours leave unread (n <= 2h: fewer than three planes, five for Shan-Chen), and steppers without
plane ranges (the oracle in the CPU tests), step whole and exchange afterwards.

`Slab` is one rank's part (one process per GPU).  `SlabSet` holds every rank's part in one process and
exchanges by plain copies, for tests and for several slabs on one device.
"""
from __future__ import annotations

import numpy as np

from . import (BGK, BOUNCE, D3Q27, MAX_CLASSES, MRT, SET_RHO, SET_UX, SET_UY, SET_UZ, SHANCHEN, STORAGE_BYTES,
               Desc, Lattice, classes_of, set_classes, velocities)

__all__ = ["split_planes", "axis_dirs", "halo_plan", "local_problem", "scatter_populations", "Slab", "SlabSet"]

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


def halo_plan(desc: Desc):
    """(h, up, down): ghost planes per side, and the face transfers of one exchange.

    A slab of n planes holds local planes 0 .. n + 2h - 1: h ghost planes, its n own planes (h .. h+n-1),
    h ghost planes.  up = [(k, dirs)]: a rank sends the populations `dirs` of its plane h + n - 1 - k to
    its upper neighbour, which stores them in its ghost plane h - 1 - k; down = [(k, dirs)]: a rank
    sends `dirs` of its plane h + k to its lower neighbour, into that one's ghost plane h + n' + k.
    BGK and MRT: one plane, the c = +1 (c = -1) populations.  Shan-Chen: two planes, the adjacent one
    with the c = 0 populations as well (psi of a ghost cell needs its streamed density)."""
    up_dirs, down_dirs = axis_dirs(desc.lattice)
    if desc.collision in (BGK, MRT):
        return 1, [(0, up_dirs)], [(0, down_dirs)]
    if desc.collision == SHANCHEN:
        c = np.asarray(velocities(desc.lattice)[2 if desc.dim == 3 else 1])
        zero = [int(i) for i in np.flatnonzero(c == 0)]
        return 2, [(0, up_dirs + zero), (1, up_dirs)], [(0, down_dirs + zero), (1, down_dirs)]
    raise ValueError("unknown collision model")


def local_problem(desc: Desc, mask, p0: int, p1: int):
    """Descriptor and class mask of the slab [p0, p1) with its ghost planes (halo_plan).

    BGK / MRT: one ghost plane per side, of a class appended to the descriptor's classes: full-way
    bounce-back with rho and u set to zero, as the reference's solid cells (its updates are never read;
    bounce-back keeps them finite).  Shan-Chen: two ghost planes per side with the global lattice's
    classes of those planes (periodic), since the interior reads psi of the adjacent ghost plane."""
    h = halo_plan(desc)[0]
    n = p1 - p0
    P = _planes(desc)
    if n < h:
        raise ValueError(f"a slab of {n} plane(s) cannot feed its neighbours' {h} ghost planes")
    d = Desc.from_buffer_copy(desc)
    if d.dim == 3:
        d.nz = n + 2 * h
    else:
        d.ny = n + 2 * h
    d.mask = None
    cells = desc.cells // P
    g = None if mask is None else np.asarray(mask, dtype=np.uint8).ravel(order="F").reshape(P, cells)
    if desc.collision == SHANCHEN:
        if g is None:
            return d, None
        return d, np.ascontiguousarray(g[np.arange(p0 - h, p1 + h) % P]).ravel()
    if desc.n_classes >= MAX_CLASSES:
        raise ValueError("no class index left for the ghost planes")
    ghost = d.n_classes
    classes = classes_of(desc) + [(BOUNCE | SET_RHO | SET_UX | SET_UY | SET_UZ, 0.0, 0.0, 0.0, 0.0)]
    set_classes(d, classes)
    m = np.full((n + 2, cells), ghost, dtype=np.uint8)
    m[1:n + 1] = 0 if g is None else g[p0:p1]
    return d, m.ravel()


def scatter_populations(desc: Desc, F, p0: int, p1: int) -> np.ndarray:
    """The slab's part of global populations F (flat [x, y(, z), i]), ghost planes included."""
    P = _planes(desc)
    h = halo_plan(desc)[0]
    G = np.asarray(F).reshape(desc.q, P, desc.cells // P)
    idx = np.arange(p0 - h, p1 + h) % P
    return np.ascontiguousarray(G[:, idx, :]).ravel()


def _device_bytes(ptr: int, nbytes: int, device):
    """A torch uint8 tensor viewing `nbytes` of device memory at `ptr` (no copy; the memory stays the
    lattice's)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_View(), device=device)


def _plane_views(lat, planes: int, device) -> dict:
    """{device pointer: [Q, planes, plane bytes] uint8 view} for both population buffers of `lat`
    (the layout is [i][plane][cell], so a plane of one direction is one contiguous run)."""
    cur, nxt, nbytes = lat.device_buffers()
    return {ptr: _device_bytes(ptr, nbytes, device).view(lat.q, planes, -1) for ptr in (cur, nxt)}


def _interior(lat, n: int, h: int = 1, dtype=np.float64) -> np.ndarray:
    F = lat.get_populations(dtype)
    return F.reshape(lat.q, n + 2 * h, -1)[:, h:n + h, :]


def _words(plan_side) -> int:
    return sum(len(dirs) for _, dirs in plan_side)


class Slab:
    """One rank's slab of a lattice, stepped with halo exchanges over a torch.distributed group.

    lattice_factory(desc, mask) builds the local stepper (default: a GPU `Lattice`); it must offer
    step, face_get, face_set, get_populations, set_populations, set_stream and face_cells.  A GPU
    stepper that also offers step_planes and device_buffers gets the overlapped step unless
    `overlap=False` (then: step, then exchange); its row pipeline then leaves `reserved_sms` SMs to
    the exchange stream (NCCL's point-to-point kernels included: limit its channels to fit them)."""

    def __init__(self, desc: Desc, mask, F0, rank: int, world: int, group=None, device=None,
                 lattice_factory=None, overlap: bool = True, reserved_sms: int = 8):
        import torch
        import torch.distributed as dist

        if F0 is None:
            raise ValueError("F0 (global start populations) is required")
        self.dist, self.group, self.rank, self.world = dist, group, rank, world
        self.global_desc = desc
        self.p0, self.p1 = split_planes(_planes(desc), world)[rank]
        self.n = self.p1 - self.p0
        self.desc, self.mask = local_problem(desc, mask, self.p0, self.p1)
        self.h, up_plan, down_plan = halo_plan(desc)
        self.lat = (lattice_factory or Lattice)(self.desc, self.mask)
        if hasattr(self.lat, "set_cell_offset"):
            # local plane 0 is global plane p0 - h: the slab's cells hash (stochastic rounding) like the
            # undivided lattice's
            self.lat.set_cell_offset((self.p0 - self.h) * (desc.cells // _planes(desc)))
        self.up_dirs, self.down_dirs = axis_dirs(desc.lattice)
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        # a stream of the slab's own orders the steps, the face copies and the NCCL transfers (torch's
        # default stream has handle 0, which the engine would read as "the lattice's own stream");
        # an overlapped step exchanges on a second stream ordered by events
        self.stream = torch.cuda.Stream(device=self.device) if self.device.type == "cuda" else None
        if self.stream is not None:
            self.lat.set_stream(self.stream.cuda_stream)
        # faces of engine lattices travel as raw bytes of the stored words (NCCL has no 16-bit integer
        # type; a point-to-point transfer never touches the values); other steppers (the oracle) use
        # FP64 words
        word, unit = (torch.uint8, STORAGE_BYTES[self.desc.storage]) if isinstance(self.lat, Lattice) \
            else (torch.float64, 1)
        cells = self.lat.face_cells()
        self._up_seg, self._down_seg = _segments(up_plan, cells, unit), _segments(down_plan, cells, unit)
        k = _words(up_plan) * cells * unit
        self._buf = {name: torch.empty(k, dtype=word, device=self.device)
                     for name in ("send_up", "send_down", "recv_down", "recv_up")}
        self.lat.set_populations(scatter_populations(desc, F0, self.p0, self.p1))
        # the overlapped step (see the module docstring): GPU steppers with plane ranges and at least
        # one plane that no neighbour reads (n > 2h)
        self.overlap = (overlap and self.device.type == "cuda" and hasattr(self.lat, "step_planes")
                        and self.n > 2 * self.h)
        if self.overlap:
            # the exchange stream runs first wherever SMs free up; the row pipeline leaves it some
            self._comm = torch.cuda.Stream(device=self.device, priority=-1)
            self.lat.set_reserved_sms(reserved_sms)
            self._views = _plane_views(self.lat, self.n + 2 * self.h, self.device)
            self._up_idx = [torch.tensor(dirs, device=self.device) for _, dirs, _, _ in self._up_seg]
            self._down_idx = [torch.tensor(dirs, device=self.device) for _, dirs, _, _ in self._down_seg]
            self._ready, self._done = torch.cuda.Event(), torch.cuda.Event()

    def _pack(self):
        _pack(self.lat, self.n, self.h, self._up_seg, self._down_seg, self._buf["send_up"], self._buf["send_down"])

    def _unpack(self, from_down, from_up):
        _unpack(self.lat, self.n, self.h, self._up_seg, self._down_seg, from_down, from_up)

    def exchange(self):
        """Fill both ghost planes from the neighbours' boundary planes (the same steps on every rank)."""
        import torch

        with torch.cuda.stream(self.stream):  # no-op without a CUDA stream
            self._exchange()

    def _exchange(self):
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
        import torch

        with torch.cuda.stream(self.stream):
            for _ in range(n):
                if self.overlap:
                    self._step_overlapped()
                else:
                    self.lat.step(1)
                    self._exchange()

    def _step_overlapped(self):
        """One step: the interior planes on the slab's stream, and beside them, on the side stream in
        the SMs the row pipeline leaves free, the boundary planes and the face exchange."""
        import torch

        dist, lat, n, h, b = self.dist, self.lat, self.n, self.h, self._buf
        main, comm = self.stream, self._comm
        self._ready.record(main)  # the previous step (and its exchange) is complete on `main`
        F = self._views[lat.device_buffers()[1]]  # the buffer this step writes
        _step_sides(lat, n, h, main, comm, self._ready)
        with torch.cuda.stream(comm):
            _pack_views(F, n, h, self._up_seg, self._down_seg, self._up_idx, self._down_idx, b["send_up"],
                        b["send_down"])
            if self.world == 1:
                from_down, from_up = b["send_up"], b["send_down"]
            else:
                up, down = (self.rank + 1) % self.world, (self.rank - 1) % self.world
                ops = [dist.P2POp(dist.isend, b["send_up"], up, self.group, tag=1),
                       dist.P2POp(dist.irecv, b["recv_down"], down, self.group, tag=1),
                       dist.P2POp(dist.isend, b["send_down"], down, self.group, tag=2),
                       dist.P2POp(dist.irecv, b["recv_up"], up, self.group, tag=2)]
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
                from_down, from_up = b["recv_down"], b["recv_up"]
            _unpack_views(F, n, h, self._up_seg, self._down_seg, self._up_idx, self._down_idx, from_down, from_up)
            self._done.record(comm)
        main.wait_event(self._done)

    def interior_populations(self, dtype=np.float64) -> np.ndarray:
        """This rank's planes, [Q, n, plane cells]."""
        return _interior(self.lat, self.n, self.h, dtype)

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


def _segments(plan_side, cells: int, unit: int):
    """[(k, dirs, start, stop)]: where each transfer of one side (halo_plan) sits in its send buffer,
    in buffer elements (`unit` elements per stored word)."""
    out, at = [], 0
    for k, dirs in plan_side:
        size = len(dirs) * cells * unit
        out.append((k, dirs, at, at + size))
        at += size
    return out


def _pack(lat, n, h, up_seg, down_seg, send_up, send_down):
    """The faces a slab of n planes sends up (from its top planes) and down (from its bottom planes)."""
    for k, dirs, a, b in up_seg:
        lat.face_get(h + n - 1 - k, dirs, send_up[a:b])
    for k, dirs, a, b in down_seg:
        lat.face_get(h + k, dirs, send_down[a:b])


def _unpack(lat, n, h, up_seg, down_seg, from_down, from_up):
    """Store what the lower neighbour sent up in the lower ghost planes and what the upper one sent
    down in the upper ghost planes."""
    for k, dirs, a, b in up_seg:
        lat.face_set(h - 1 - k, dirs, from_down[a:b])
    for k, dirs, a, b in down_seg:
        lat.face_set(h + n + k, dirs, from_up[a:b])


def _step_sides(lat, n, h, main, comm, ready):
    """One step of a slab in pieces: its interior planes (2h .. n-1, read by no neighbour) on `main`, and
    on `comm` (after `ready`) the planes its neighbours read (h .. 2h-1 and n .. n+h-1), which end the
    step.  One ghost plane: both boundary planes in one strided launch."""
    import torch

    lat.step_planes(2 * h, n - 2 * h, False, main)  # the interior first: it takes its SMs before the side
    with torch.cuda.stream(comm):
        comm.wait_event(ready)
        if h == 1:
            lat.step_planes(1, 2, True, comm, stride=n - 1)
        else:
            lat.step_planes(h, h, False, comm)
            lat.step_planes(n, h, True, comm)


def _step_sides_all(lats, ns, h, main, comm, ready):
    """_step_sides for every slab of a SlabSet: all interiors on `main` first, then the boundary planes."""
    import torch

    for lat, n in zip(lats, ns):
        lat.step_planes(2 * h, n - 2 * h, False, main)
    with torch.cuda.stream(comm):
        comm.wait_event(ready)
        for lat, n in zip(lats, ns):
            if h == 1:
                lat.step_planes(1, 2, True, comm, stride=n - 1)
            else:
                lat.step_planes(h, h, False, comm)
                lat.step_planes(n, h, True, comm)


def _pack_views(F, n, h, up_seg, down_seg, up_idx, down_idx, send_up, send_down):
    """_pack from a [Q, planes, plane bytes] view of the buffer being written (on the current stream)."""
    import torch

    for (k, dirs, a, b), idx in zip(up_seg, up_idx):
        torch.index_select(F[:, h + n - 1 - k], 0, idx, out=send_up[a:b].view(len(dirs), -1))
    for (k, dirs, a, b), idx in zip(down_seg, down_idx):
        torch.index_select(F[:, h + k], 0, idx, out=send_down[a:b].view(len(dirs), -1))


def _unpack_views(F, n, h, up_seg, down_seg, up_idx, down_idx, from_down, from_up):
    """_unpack into a [Q, planes, plane bytes] view of the buffer being written."""
    for (k, dirs, a, b), idx in zip(up_seg, up_idx):
        F[:, h - 1 - k].index_copy_(0, idx, from_down[a:b].view(len(dirs), -1))
    for (k, dirs, a, b), idx in zip(down_seg, down_idx):
        F[:, h + n + k].index_copy_(0, idx, from_up[a:b].view(len(dirs), -1))


def _sums(lattice: int, Fi: np.ndarray) -> np.ndarray:
    cx, cy, cz, _, _ = velocities(lattice)
    per_dir = Fi.reshape(Fi.shape[0], -1).sum(axis=1)
    return np.array([per_dir.sum(), per_dir @ np.asarray(cx, float), per_dir @ np.asarray(cy, float),
                     per_dir @ np.asarray(cz, float)])


class SlabSet:
    """Every slab of a decomposed lattice in one process, exchanged by plain copies (no collective).

    The same planes, ghost classes and exchange order as `Slab`, for parity tests on one device and
    for decompositions whose slabs share a GPU."""

    def __init__(self, desc: Desc, mask, F0, parts: int, lattice_factory=None, overlap: bool = False,
                 reserved_sms: int = 8):
        self.global_desc = desc
        self.ranges = split_planes(_planes(desc), parts)
        self.up_dirs, self.down_dirs = axis_dirs(desc.lattice)
        self.h, up_plan, down_plan = halo_plan(desc)
        self.lats, self.ns = [], []
        for p0, p1 in self.ranges:
            d, m = local_problem(desc, mask, p0, p1)
            lat = (lattice_factory or Lattice)(d, m)
            if hasattr(lat, "set_cell_offset"):
                lat.set_cell_offset((p0 - self.h) * (desc.cells // _planes(desc)))
            lat.set_populations(scatter_populations(desc, F0, p0, p1))
            self.lats.append(lat)
            self.ns.append(p1 - p0)
        cells = self.lats[0].face_cells()
        self._up_seg, self._down_seg = _segments(up_plan, cells, 1), _segments(down_plan, cells, 1)
        k = _words(up_plan) * cells
        word = {4: np.float32, 8: np.float64, 2: np.uint16}[STORAGE_BYTES[desc.storage]] \
            if isinstance(self.lats[0], Lattice) else np.float64
        self._up = [np.empty(k, dtype=word) for _ in self.lats]
        self._down = [np.empty(k, dtype=word) for _ in self.lats]
        # overlapped steps: every lattice on one stream of the set's own, the face copies on a second
        self.overlap = overlap and isinstance(self.lats[0], Lattice) and min(self.ns) > 2 * self.h
        if self.overlap:
            import torch

            self._dev = torch.device("cuda", desc.device)
            self.stream = torch.cuda.Stream(device=self._dev)
            for lat in self.lats:
                lat.set_stream(self.stream.cuda_stream)
                lat.set_reserved_sms(reserved_sms)
            self._comm = torch.cuda.Stream(device=self._dev, priority=-1)
            self._views = [_plane_views(lat, n + 2 * self.h, self._dev) for lat, n in zip(self.lats, self.ns)]
            self._up_idx = [torch.tensor(dirs, device=self._dev) for _, dirs, _, _ in self._up_seg]
            self._down_idx = [torch.tensor(dirs, device=self._dev) for _, dirs, _, _ in self._down_seg]
            self._ready, self._done = torch.cuda.Event(), torch.cuda.Event()

    def exchange(self):
        R = len(self.lats)
        for r, lat in enumerate(self.lats):
            _pack(lat, self.ns[r], self.h, self._up_seg, self._down_seg, self._up[r], self._down[r])
        for r, lat in enumerate(self.lats):
            _unpack(lat, self.ns[r], self.h, self._up_seg, self._down_seg, self._up[(r - 1) % R],
                    self._down[(r + 1) % R])

    def step(self, n: int = 1):
        for _ in range(n):
            if self.overlap:
                self._step_overlapped()
                continue
            for lat in self.lats:
                lat.step(1)
            self.exchange()

    def _step_overlapped(self):
        """The overlapped step of `Slab`, for every slab of one device: boundary planes, face copies
        between the slabs' next buffers on the side stream, interior planes on the main stream."""
        import torch

        main, comm, h = self.stream, self._comm, self.h
        self._ready.record(main)
        F = [v[lat.device_buffers()[1]] for lat, v in zip(self.lats, self._views)]
        R = len(self.lats)
        _step_sides_all(self.lats, self.ns, h, main, comm, self._ready)
        with torch.cuda.stream(comm):
            for r, n in enumerate(self.ns):
                lo, hi = (r - 1) % R, (r + 1) % R
                # lower ghosts from the lower slab's top planes, upper ghosts from the upper slab's bottom ones
                for (k, _, _, _), idx in zip(self._up_seg, self._up_idx):
                    F[r][:, h - 1 - k].index_copy_(0, idx, F[lo][:, h + self.ns[lo] - 1 - k].index_select(0, idx))
                for (k, _, _, _), idx in zip(self._down_seg, self._down_idx):
                    F[r][:, h + n + k].index_copy_(0, idx, F[hi][:, h + k].index_select(0, idx))
            self._done.record(comm)
        main.wait_event(self._done)

    def gather_populations(self, dtype=np.float64) -> np.ndarray:
        return np.concatenate([_interior(lat, n, self.h, dtype) for lat, n in zip(self.lats, self.ns)],
                              axis=1).ravel()

    def sums(self) -> np.ndarray:
        return sum(_sums(self.global_desc.lattice, _interior(lat, n, self.h)) for lat, n in zip(self.lats, self.ns))

    def close(self):
        for lat in self.lats:
            if hasattr(lat, "close"):
                lat.close()
