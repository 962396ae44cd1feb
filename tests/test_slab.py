"""Slab decomposition of one lattice (lbm_b200.slab): ghost planes, the per-step face exchange and the
gather must reproduce the undivided lattice bit for bit.

CPU: the oracle steps every slab (one process, and a gloo world of 2 and 3 processes exchanging
faces with isend/irecv).  GPU: the engine steps every slab of a `SlabSet` on one device (plain copies
between slabs, no collective) and matches one engine lattice of the full size.
"""
import json
import os
import socket
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import O, P, channel2d, lb, oracle_problem

from lbm_b200.slab import Slab, SlabSet, axis_dirs, halo_plan, local_problem, scatter_populations, split_planes


class OracleStepper:
    """The oracle behind the stepper interface Slab uses (FP64 populations are the stored words)."""

    def __init__(self, desc, mask):
        self.p = oracle_problem(desc, mask)
        self.q, self.n = desc.q, desc.cells
        self.planes = desc.nz if desc.dim == 3 else desc.ny
        self.F = None

    def face_cells(self):
        return self.n // self.planes

    def set_populations(self, F):
        self.F = np.array(F, dtype=np.float64)

    def get_populations(self, dtype=np.float64):
        return self.F.astype(dtype)

    def step(self, n=1):
        self.F = O.run(self.p, self.F, n, dtype=np.float64, threads=1)[0]

    def _view(self):
        return self.F.reshape(self.q, self.planes, -1)

    def face_get(self, plane, dirs, out):
        a = out.numpy() if hasattr(out, "numpy") else out
        a.reshape(len(dirs), -1)[:] = self._view()[dirs, plane, :]
        return out

    def face_set(self, plane, dirs, src):
        a = src.numpy() if hasattr(src, "numpy") else src
        self._view()[dirs, plane, :] = np.asarray(a).reshape(len(dirs), -1)

    def set_stream(self, stream):
        pass


def mrt_cavity3d(storage=lb.F64, n=(12, 8, 9)):
    d = lb.make_desc(lb.D3Q27, lb.MRT, storage, n, mrt_s=lb.mrt_rates(1.7, 1.1), mrt_basis=lb.MRT_GRAM_SCHMIDT)
    m = lb.setup_cavity3d(d, 0.05)
    _, _, _, w, _ = lb.velocities(lb.D3Q27)
    rng = np.random.default_rng(11)
    F0 = np.repeat(w, d.cells) * (1.0 + 0.01 * rng.standard_normal(27 * d.cells))
    return d, m, F0


def channel(storage=lb.F64, nx=48, ny=20):
    return channel2d(nx, ny, 0.04, 100.0, 14, 10, 4, storage=storage, config_mode=True, seed=1, noise=1e-3)


def periodic3d(storage=lb.F64, n=(8, 6, 7)):
    d = lb.make_desc(lb.D3Q27, lb.BGK, storage, n, omega=1.6)
    _, _, _, w, _ = lb.velocities(lb.D3Q27)
    rng = np.random.default_rng(12)
    return d, None, np.repeat(w, d.cells) * (1.0 + 0.02 * rng.standard_normal(27 * d.cells))


def shanchen2d(storage=lb.F64, nx=24, ny=20, G=-5.5):
    """Periodic single-component Shan-Chen in its phase-separating regime (seeded density noise)."""
    d = lb.make_desc(lb.D2Q9, lb.SHANCHEN, storage, (nx, ny), omega=1.0, sc_G=G)
    F0 = P.shanchen_start_state(P.shanchen(nx, ny, G), 0.693, 0.01, 5)
    return d, None, F0


def shanchen_walls(storage=lb.F64, nx=20, ny=17):
    """Shan-Chen between two walls (rows y = 0 and y = ny - 1: bounce-back with a prescribed wall
    density, which sets the walls' psi) and a row of forced density in the bulk: the slabs' ghost
    rows must carry those classes."""
    d, _, F0 = shanchen2d(storage, nx, ny)
    lb.set_classes(d, [(0, 0.0, 0.0, 0.0, 0.0),
                       (lb.BOUNCE | lb.SET_RHO | lb.SET_UX | lb.SET_UY, 0.4, 0.0, 0.0, 0.0),
                       (lb.SET_RHO, 0.9, 0.0, 0.0, 0.0)])
    m = np.zeros((nx, ny), dtype=np.uint8, order="F")
    m[:, 0] = m[:, ny - 1] = 1
    m[3:9, 7] = 2
    return d, m.ravel(order="F"), F0


CASES = {"mrt_cavity3d": mrt_cavity3d, "channel2d": channel, "periodic3d": periodic3d,
         "shanchen2d": shanchen2d, "shanchen_walls": shanchen_walls}


def test_split_planes_and_axis_dirs():
    for n, world in [(10, 3), (7, 7), (256, 8), (5, 1)]:
        parts = split_planes(n, world)
        sizes = [b - a for a, b in parts]
        assert parts[0][0] == 0 and parts[-1][1] == n and max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
        assert all(parts[k][1] == parts[k + 1][0] for k in range(world - 1))
    with pytest.raises(ValueError):
        split_planes(3, 4)
    for lat, k in [(lb.D3Q27, 9), (lb.D2Q9, 3)]:
        up, down = axis_dirs(lat)
        assert len(up) == len(down) == k
        opp = lb.velocities(lat)[4]
        assert sorted(int(opp[i]) for i in up) == down


def test_local_problem_ghost_planes():
    d, m, F0 = mrt_cavity3d()
    ld, lm = local_problem(d, m, 3, 7)
    assert (ld.nx, ld.ny, ld.nz) == (12, 8, 6) and ld.n_classes == d.n_classes + 1
    g = lm.reshape(6, -1)
    assert (g[0] == d.n_classes).all() and (g[-1] == d.n_classes).all()
    assert np.array_equal(g[1:5].ravel(), np.asarray(m).ravel(order="F")[3 * 96:7 * 96])
    Fl = scatter_populations(d, F0, 0, 2).reshape(27, 4, -1)
    Fg = F0.reshape(27, 9, -1)
    assert np.array_equal(Fl[:, 0], Fg[:, 8]) and np.array_equal(Fl[:, 1:3], Fg[:, 0:2])


def test_shanchen_halo_two_planes_with_the_global_classes():
    """Shan-Chen slabs: two ghost rows per side holding the global rows' classes (periodic), the
    adjacent ghost row fed with the c = 0 and c = +1 (c = -1) populations and the far one with the
    c = +1 (c = -1) ones; a slab must hold at least two rows."""
    d, m, F0 = shanchen_walls()
    h, up, down = halo_plan(d)
    cy = lb.velocities(lb.D2Q9)[1]
    assert h == 2 and [k for k, _ in up] == [0, 1] and [k for k, _ in down] == [0, 1]
    assert sorted(cy[up[0][1]]) == [0, 0, 0, 1, 1, 1] and sorted(cy[up[1][1]]) == [1, 1, 1]
    assert sorted(cy[down[0][1]]) == [-1, -1, -1, 0, 0, 0] and sorted(cy[down[1][1]]) == [-1, -1, -1]
    ld, lm = local_problem(d, m, 0, 5)
    assert (ld.nx, ld.ny) == (20, 9) and ld.n_classes == d.n_classes
    rows = np.asarray(m).reshape(17, 20)
    assert np.array_equal(lm.reshape(9, 20), rows[[15, 16, 0, 1, 2, 3, 4, 5, 6]])
    Fl = scatter_populations(d, F0, 0, 5).reshape(9, 9, -1)
    Fg = F0.reshape(9, 17, -1)
    assert np.array_equal(Fl[:, :2], Fg[:, 15:17]) and np.array_equal(Fl[:, 2:9], Fg[:, 0:7])
    assert local_problem(*shanchen2d()[:2], 2, 9)[1] is None  # no mask: none for the slab either
    with pytest.raises(ValueError):
        local_problem(d, m, 4, 5)
    with pytest.raises(ValueError):
        SlabSet(d, m, F0, 9, lattice_factory=OracleStepper)  # 17 rows over 9 slabs: one has a single row


def test_face_calls_validate_buffers_and_context():
    """Face buffers are checked on the host (size, contiguity) and the C ABI rejects a NULL context;
    nothing here reaches a GPU."""
    import ctypes as C

    class Unopened(lb.Lattice):
        def __init__(self, d):  # no lbm_create: a NULL context
            self.desc, self._h, self._mask = d, C.c_void_p(), None

    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F16S, (32, 8))
    lat = Unopened(d)
    with pytest.raises(ValueError):
        lat.face_get(0, [2, 5, 6], np.empty(10, np.uint16))
    with pytest.raises(ValueError):
        lat.face_get(0, [2, 5, 6], np.empty((192, 2), np.uint16)[:, 0])
    with pytest.raises(lb.LbmError):
        lat.face_get(0, [2, 5, 6], np.empty(96, np.uint16))
    lat._h = None


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("parts", [1, 2, 3])
def test_slabset_of_oracles_equals_undivided_oracle(case, parts):
    d, m, F0 = CASES[case]()
    ref = O.run(oracle_problem(d, m), np.array(F0, dtype=np.float64), 12, dtype=np.float64, threads=1)[0]
    s = SlabSet(d, m, F0, parts, lattice_factory=OracleStepper)
    s.step(12)
    assert np.array_equal(s.gather_populations(), ref)
    assert np.allclose(s.sums(), O.sums(oracle_problem(d, m), ref), rtol=1e-12, atol=1e-12)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _gloo_body(rank, world, port, case, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d, m, F0 = CASES[case]()
        slab = Slab(d, m, F0, rank, world, lattice_factory=OracleStepper)
        slab.step(9)
        F = slab.gather_populations()
        sums = slab.sums()
        if rank == 0:
            np.save(Path(out_dir) / "F.npy", F)
            (Path(out_dir) / "sums.json").write_text(json.dumps(list(map(float, sums))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world", [("mrt_cavity3d", 2), ("channel2d", 3), ("shanchen_walls", 3)])
def test_slab_gloo_ranks_equal_undivided_oracle(tmp_path, case, world):
    mp.start_processes(_gloo_body, args=(world, _free_port(), case, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    d, m, F0 = CASES[case]()
    ref = O.run(oracle_problem(d, m), np.array(F0, dtype=np.float64), 9, dtype=np.float64, threads=1)[0]
    assert np.array_equal(np.load(tmp_path / "F.npy"), ref)
    sums = json.loads((tmp_path / "sums.json").read_text())
    assert np.allclose(sums, O.sums(oracle_problem(d, m), ref), rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [lb.F32, lb.F16S])
@pytest.mark.parametrize("case", ["mrt_cavity3d", "channel2d", "periodic3d", "mrt_rows"])
@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("overlap", [False, True])
def test_slabset_of_engine_lattices_equals_one_lattice(storage, case, parts, overlap):
    """Slabs stepped by the engine (its kernel choice per slab: plain or row pipeline) and exchanged
    by face_get/face_set, or overlapped (boundary planes, face copies between the slabs' buffers on a
    side stream, interior planes): bit-identical to one lattice of the full size."""
    if case == "mrt_rows":
        d, m, F0 = mrt_cavity3d(storage, n=(128, 16, 24))  # row-pipeline eligible slabs
    else:
        d, m, F0 = CASES[case](storage)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(np.asarray(F0, dtype=np.float64))
        lat.step(15)
        ref = lat.get_populations(np.float32)
    s = SlabSet(d, m, F0, parts, overlap=overlap)
    assert s.overlap == (overlap and min(s.ns) >= 3)
    try:
        s.step(15)
        got = s.gather_populations(np.float32)
    finally:
        s.close()
    assert np.isfinite(got).all() and np.array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [lb.F32, lb.BF16S, lb.F64])
@pytest.mark.parametrize("case", ["shanchen2d", "shanchen_walls", "shanchen_wide"])
@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("kernel", [lb.KERNEL_AUTO, lb.KERNEL_PLAIN])
@pytest.mark.parametrize("overlap", [False, True])
def test_shanchen_slabs_on_the_gpu_equal_one_lattice(storage, case, parts, kernel, overlap):
    """Shan-Chen slabs on the engine (one-pass window kernel or the two-pass kernels, stochastic
    rounding for BF16S hashed by global cell) with two ghost rows per side, stepped then exchanged or
    overlapped (the rows the neighbours read and their exchange on a side stream beside the interior
    rows): bit-identical to one lattice of the full size after 40 steps of phase separation."""
    if case == "shanchen_wide":  # rows wider than one window strip, a ragged last strip
        d, m, F0 = shanchen2d(storage, nx=300, ny=26)
    else:
        d, m, F0 = CASES[case](storage)

    def engine(dd, mm):
        lat = lb.Lattice(dd, mm)
        lat.set_kernel(kernel)
        return lat

    dtype = np.float64 if storage == lb.F64 else np.float32
    with engine(d, m) as lat:
        lat.set_populations(np.asarray(F0, dtype=np.float64))
        lat.step(40)
        ref = lat.get_populations(dtype)
        ref_sums = lat.sums()
    s = SlabSet(d, m, F0, parts, lattice_factory=engine, overlap=overlap)
    assert s.overlap == overlap and s.h == 2
    try:
        s.step(40)
        got = s.gather_populations(dtype)
        sums = s.sums()
    finally:
        s.close()
    assert np.isfinite(got).all() and np.array_equal(got, ref)
    assert np.allclose(sums, ref_sums, rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [lb.F32, lb.BF16S])
@pytest.mark.parametrize("overlap", [False, True])
def test_one_rank_shanchen_slab_on_the_gpu_equals_one_lattice(storage, overlap):
    """The rank-side Slab for Shan-Chen: device byte buffers holding both ghost rows' transfers per
    side, filled from the rank's own far rows (periodic wrap), equal to the undivided lattice."""
    import torch

    d, m, F0 = shanchen_walls(storage, nx=96, ny=30)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(np.asarray(F0, dtype=np.float64))
        lat.step(25)
        ref = lat.get_populations(np.float32)
    slab = Slab(d, m, F0, 0, 1, device="cuda:0", overlap=overlap)
    assert slab.overlap == overlap and slab.h == 2
    assert slab._buf["send_up"].numel() == 9 * 96 * lb.STORAGE_BYTES[storage]
    slab.step(25)
    torch.cuda.synchronize()
    assert np.array_equal(slab.gather_populations(np.float32), ref)
    slab.close()


def _plane_case(name, storage):
    if name == "mrt3d":
        return mrt_cavity3d(storage, n=(128, 16, 12))
    if name == "mrt3d_seg":  # rows wider than 1024 cells: the segmented row kernel
        return mrt_cavity3d(storage, n=(1040, 4, 6))
    if name == "channel":
        return channel(storage, nx=256, ny=40)
    if name == "channel_seg":
        return channel(storage, nx=1088, ny=12)
    return periodic3d(storage, n=(64, 6, 7))


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [lb.F32, lb.F16S])
@pytest.mark.parametrize("kernel", [lb.KERNEL_PLAIN, lb.KERNEL_ROWS])
@pytest.mark.parametrize("case", ["mrt3d", "mrt3d_seg", "channel", "channel_seg", "bgk3d"])
def test_step_planes_in_pieces_equals_whole_steps(storage, kernel, case):
    """lbm_step_planes: a step cut into plane ranges (in any order; the last one finishes it) is
    bit-identical to lbm_step, for the plain kernels, the row pipeline and its segmented form, with
    stochastic rounding on for the 16-bit storage.  The ranges before the last run on a side stream,
    beside the last one (the overlapped slab's pattern), with SMs reserved from the row pipeline."""
    import torch

    d, m, F0 = _plane_case(case, storage)
    planes = d.nz if d.dim == 3 else d.ny
    F0 = np.asarray(F0, dtype=np.float64)
    main, side = torch.cuda.Stream(), torch.cuda.Stream(priority=-1)
    ready, done = torch.cuda.Event(), torch.cuda.Event()
    with lb.Lattice(d, m) as a, lb.Lattice(d, m) as b:
        for lat in (a, b):
            lat.set_kernel(kernel)
            lat.set_populations(F0)
        a.step(8)
        b.set_stream(main)
        b.set_reserved_sms(3)
        # (first, count, stride): the slab order (boundary planes in one strided launch, then the
        # interior), contiguous ranges, single planes backwards, and the odd planes then the even ones
        cuts = [[(0, 2, planes - 1), (1, planes - 2, 1)],
                [(3, planes - 3, 1), (0, 3, 1)],
                [(k, 1, 1) for k in range(planes - 1, -1, -1)],
                [(1, planes // 2, 2), (0, (planes + 1) // 2, 2)]]
        for t in range(8):
            pieces = cuts[t % len(cuts)]
            ready.record(main)
            side.wait_event(ready)
            for k, (first, count, stride) in enumerate(pieces):
                last = k == len(pieces) - 1
                b.step_planes(first, count, last, main if last else side, stride=stride)
            done.record(side)
            main.wait_event(done)
        assert b.steps_done == a.steps_done == 8
        ref, got = a.get_populations(np.float32), b.get_populations(np.float32)
        b.set_stream(None)
        b.step(2)  # whole steps with the reserved SMs
        a.step(2)
        assert np.array_equal(a.get_populations(np.float32), b.get_populations(np.float32))
    assert np.isfinite(got).all() and np.array_equal(got, ref)


@pytest.mark.gpu
def test_step_planes_rejects_bad_ranges():
    d, m, _ = mrt_cavity3d(lb.F32, n=(32, 4, 5))
    with lb.Lattice(d, m) as lat:
        for first, count, stride in ((-1, 1, 1), (0, 0, 1), (4, 2, 1), (5, 1, 1), (0, 2, 0), (1, 2, 4), (1, 3, 2)):
            with pytest.raises(lb.LbmError):
                lat.step_planes(first, count, True, stride=stride)
        assert lat.steps_done == 0


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [lb.F32, lb.BF16S, lb.F64])
@pytest.mark.parametrize("kernel", [lb.KERNEL_AUTO, lb.KERNEL_PLAIN, lb.KERNEL_ROWS])
@pytest.mark.parametrize("case", ["shanchen_walls", "shanchen_wide"])
def test_shanchen_step_planes_in_pieces_equals_whole_steps(storage, kernel, case):
    """Shan-Chen plane sets (the one-pass window kernel whatever the family: contiguous rows, strided
    rows, single rows) make the same step as lbm_step: bit-identical, stochastic rounding included,
    with the pieces before the last on a side stream beside it."""
    import torch

    d, m, F0 = shanchen2d(storage, nx=300, ny=26) if case == "shanchen_wide" else shanchen_walls(storage, nx=96, ny=30)
    planes = d.ny
    F0 = np.asarray(F0, dtype=np.float64)
    main, side = torch.cuda.Stream(), torch.cuda.Stream(priority=-1)
    ready, done = torch.cuda.Event(), torch.cuda.Event()
    dtype = np.float64 if storage == lb.F64 else np.float32
    with lb.Lattice(d, m) as a, lb.Lattice(d, m) as b:
        for lat in (a, b):
            lat.set_kernel(kernel)
            lat.set_populations(F0)
        a.step(8)
        b.set_stream(main)
        # the slab's order (two bottom rows, two top rows beside the interior), contiguous ranges,
        # single rows backwards, and the odd rows then the even ones
        cuts = [[(2, 2, 1), (planes - 4, 2, 1), (4, planes - 8, 1), (0, 2, 1), (planes - 2, 2, 1)],
                [(3, planes - 3, 1), (0, 3, 1)],
                [(k, 1, 1) for k in range(planes - 1, -1, -1)],
                [(1, planes // 2, 2), (0, (planes + 1) // 2, 2)]]
        for t in range(8):
            pieces = cuts[t % len(cuts)]
            ready.record(main)
            side.wait_event(ready)
            for k, (first, count, stride) in enumerate(pieces):
                last = k == len(pieces) - 1
                b.step_planes(first, count, last, main if last else side, stride=stride)
            done.record(side)
            main.wait_event(done)
        assert b.steps_done == a.steps_done == 8
        ref, got = a.get_populations(dtype), b.get_populations(dtype)
        b.set_stream(None)
    assert np.isfinite(got).all() and np.array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [lb.F32, lb.BF16S])
@pytest.mark.parametrize("overlap", [False, True])
def test_one_rank_slab_on_the_gpu_equals_one_lattice(storage, overlap):
    """The rank-side Slab with CUDA byte buffers on torch's stream: with one rank its ghost planes are
    filled from its own far planes (the periodic wrap), so it equals the undivided lattice.  Both the
    sequential step and the overlapped one (faces packed from the buffer being written, on a side
    stream, while the interior planes are updated)."""
    import torch

    d, m, F0 = mrt_cavity3d(storage, n=(128, 16, 12))
    with lb.Lattice(d, m) as lat:
        lat.set_populations(np.asarray(F0, dtype=np.float64))
        lat.step(10)
        ref = lat.get_populations(np.float32)
        ref_sums = lat.sums()
    slab = Slab(d, m, F0, 0, 1, device="cuda:0", overlap=overlap)
    assert slab.overlap == overlap
    assert slab._buf["send_up"].dtype == torch.uint8 and slab._buf["send_up"].is_cuda
    slab.step(10)
    torch.cuda.synchronize()
    assert np.array_equal(slab.gather_populations(np.float32), ref)
    # lbm_sums_fp64 decodes each population in FP32 before its FP64 sum; Slab.sums decodes in FP64
    assert np.allclose(slab.sums(), ref_sums, rtol=1e-6, atol=1e-6)
    slab.close()


@pytest.mark.gpu
@pytest.mark.parametrize("workload,dims", [("d3q27_mrt_gs_lid_256", "64x32x24"), ("d2q9_shanchen_1024", "256x64")])
def test_bench_slab_line(workload, dims):
    """bench.py --slab: one JSON line with the overlapped, sequential and undivided step times (D3Q27
    MRT, and Shan-Chen with its two ghost rows per side)."""
    import subprocess
    import sys

    root = Path(__file__).resolve().parents[1]
    cmd = [sys.executable, str(root / "bench.py"), "--slab", "--workload", workload, "--dims", dims, "--steps", "4",
           "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(root))
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["config"]["parallelism"] == "slab x1" and line["config"]["overlap"] is True
    assert line["value"] > 0 and line["sequential_ms_per_step"] > 0 and line["undivided_ms_per_step"] > 0
