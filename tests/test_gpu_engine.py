"""Engine behaviour on the GPU beyond parity: transfers, graph vs single-step stepping, split vs
continuous runs (checkpoint/resume), block widths, reductions, divergence detection, batched
ensembles — all through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, cavity2d, cavity3d, channel2d, lb, mrt_cavity, oracle_problem, rel_l2

pytestmark = pytest.mark.gpu


def test_population_round_trip_exact():
    d, m, F0 = cavity2d(n=64, storage=lb.F32)
    rng = np.random.default_rng(0)
    F = (F0 * (1 + 0.01 * rng.standard_normal(F0.size))).astype(np.float32)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F)
        assert np.array_equal(lat.get_populations(np.float32), F)
        lat.set_populations(F.astype(np.float64))
        assert np.array_equal(lat.get_populations(np.float64), F.astype(np.float64))
    d.storage = lb.F64
    with lb.Lattice(d, m) as lat:
        F64 = F0 * (1 + 0.01 * rng.standard_normal(F0.size))
        lat.set_populations(F64)
        assert np.array_equal(lat.get_populations(np.float64), F64)


@pytest.mark.parametrize("storage,rel", [(lb.F16S, 2.0 ** -11), (lb.BF16S, 2.0 ** -8)])
def test_shifted_round_trip_error_is_bounded(storage, rel):
    """Round-to-nearest of the stored deviation f - w: |error| <= 2^-11 (FP16) / 2^-8 (BF16) of it."""
    d, m, F0 = cavity2d(n=32, storage=storage)
    rng = np.random.default_rng(1)
    F = F0 * (1 + 0.05 * rng.standard_normal(F0.size))
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F)
        G = lat.get_populations(np.float64)
    assert np.all(np.abs(G - F) <= rel * np.abs(F - F0) * 1.0001 + 1e-11)


def test_macros_before_any_step_are_local_moments():
    d, m, F0 = cavity2d(n=32)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        rho, u = lat.macros()
    assert np.allclose(rho, 1.0, atol=1e-6)
    assert np.allclose(u, 0.0, atol=1e-6)


def test_graph_chunks_equal_single_steps():
    d, m, F0 = cavity2d(n=128)
    with lb.Lattice(d, m) as a, lb.Lattice(d, m) as b:
        a.set_populations(F0)
        b.set_populations(F0)
        a.step(777)
        for _ in range(777):
            b.step(1)
        assert np.array_equal(a.get_populations(np.float32), b.get_populations(np.float32))
        assert a.steps_done == b.steps_done == 777


def test_split_run_equals_continuous_run():
    d, m, F0 = mrt_cavity(n=16, u_lid=0.1)
    with lb.Lattice(d, m) as a:
        a.set_populations(F0)
        a.step(120)
        ref = a.get_populations(np.float32)
    with lb.Lattice(d, m) as b:
        b.set_populations(F0)
        b.step(50)
        ckpt = b.get_populations(np.float32)
    with lb.Lattice(d, m) as c:
        c.set_populations(ckpt)
        c.step(70)
        assert np.array_equal(c.get_populations(np.float32), ref)


def test_block_width_does_not_change_results():
    d, m, F0 = cavity3d(n=(70, 12, 9), u_lid=0.1, omega=1.4)
    out = []
    for bx in (32, 64, 128, 256):
        with lb.Lattice(d, m) as lat:
            lat.set_block(bx)
            lat.set_populations(F0)
            lat.step(21)
            assert lat.block() == bx
            out.append(lat.get_populations(np.float32))
    for o in out[1:]:
        assert np.array_equal(o, out[0])


def test_autotune_picks_a_legal_block():
    d, m, F0 = cavity2d(n=256)
    with lb.Lattice(d, m) as lat:
        lat.step(4)
        assert lat.block() in (32, 64, 128, 256, 512)
        assert lat.last_step_ms() > 0


def test_sums_match_oracle_and_detect_nan():
    d, m, F0 = cavity2d(n=64)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        lat.step(100)
        F = lat.get_populations(np.float64)
        s = lat.sums()
        assert np.allclose(s, O.sums(oracle_problem(d, m), F), rtol=1e-12, atol=1e-12)
        F[123] = np.nan
        lat.set_populations(F)
        with pytest.raises(lb.LbmError) as e:
            lat.sums()
        assert e.value.code == -4


def test_residual_decreases_towards_steady_state():
    d, m, F0 = cavity2d(n=64, u_lid=0.05, re=50)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        with pytest.raises(lb.LbmError):
            lat.residual()
        lat.step(200)
        r1 = lat.residual()
        lat.step(5000)
        r2 = lat.residual()
    assert r2 < r1 and r2 < 1e-4


def test_device_pointer_transfers_with_torch():
    torch = pytest.importorskip("torch")
    d, m, F0 = cavity2d(n=64)
    with lb.Lattice(d, m) as lat:
        t = torch.tensor(F0, dtype=torch.float32, device="cuda")
        lat.set_populations(t)
        lat.step(10)
        out = torch.empty_like(t)
        lat.get_populations(out=out)
        torch.cuda.synchronize()
        ref = lat.get_populations(np.float32)
        assert np.array_equal(out.cpu().numpy(), ref)
        rho = torch.empty(d.cells, dtype=torch.float64, device="cuda")
        u = torch.empty(2 * d.cells, dtype=torch.float64, device="cuda")
        lat.macros_into(rho, u)
        r2, u2 = lat.macros()
        assert np.array_equal(rho.cpu().numpy(), r2)


def test_external_stream():
    torch = pytest.importorskip("torch")
    d, m, F0 = cavity2d(n=64)
    s = torch.cuda.Stream()
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        lat.set_stream(s.cuda_stream)
        lat.step(10)
        lat.sync()
        a = lat.get_populations(np.float32)
        lat.set_stream(None)
    with lb.Lattice(d, m) as lat2:
        lat2.set_populations(F0)
        lat2.step(10)
        assert np.array_equal(lat2.get_populations(np.float32), a)
    # torch's default stream (handle 0) becomes CUDA's legacy default stream, not the lattice's own:
    # torch work queued after the steps on that stream sees their result
    with lb.Lattice(d, m) as lat3:
        lat3.set_populations(F0)
        lat3.set_stream(torch.cuda.default_stream())
        assert lat3.stream() == 1
        ptr, nbytes = lat3.device_populations()
        lat3.step(10)
        view = torch.as_tensor(_ByteView(ptr, nbytes), device="cuda")
        snap = view.clone()  # queued on torch's default stream right behind the steps
        lat3.sync()
        assert torch.equal(snap, view)
        assert np.array_equal(lat3.get_populations(np.float32), a)
        lat3.set_stream(None)


class _ByteView:
    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


@pytest.mark.parametrize("mode", [lb.BATCH_TILES, lb.BATCH_ROWS, lb.BATCH_ROWS_PER_FAMILY])
@pytest.mark.parametrize("storage", [lb.F32, lb.F16S])
def test_batch_equals_individual_lattices(storage, mode):
    """Every member of a batch (tile kernel, or row pipeline for the members whose rows the bulk copies
    can move and tiles for the rest, in the same step) equals the lattice stepped alone."""
    members = []
    for n in (48, 80):
        d, m, F0 = cavity2d(n=n, u_lid=0.1, re=300, storage=storage)
        members.append((d, m, F0))
    d, m, F0 = cavity3d(n=(20, 14, 12), u_lid=0.05, omega=1.2, storage=storage)  # nx = 20: tiles
    members.append((d, m, F0))
    d, m, F0 = cavity3d(n=(32, 14, 12), u_lid=0.05, omega=1.2, storage=storage)
    members.append((d, m, F0))
    for nx in (40, 64):
        dd = lb.make_desc(lb.D3Q27, lb.BGK, storage, (nx, 16, 16), omega=1.6)
        mm = lb.setup_duct3d(dd, 0.04, 11, 8, 8, 4)
        solid = mm == 1
        F0 = O.init_equilibrium(oracle_problem(dd, mm), rho=np.where(solid, 0.0, 1.0),
                                u=np.concatenate([np.where(solid, 0.0, 0.04), np.zeros(2 * mm.size)]))
        members.append((dd, mm, F0))
    b = lb.Batch([x[0] for x in members], [x[1] for x in members])
    b.set_mode(mode)
    for k, (_, _, F0) in enumerate(members):
        b.set_populations(k, np.asarray(F0, dtype=np.float64))
    b.step(37)
    assert b.mode() == mode
    tx, nt = b.tile_info()
    assert tx in (64, 128, 256) and nt > 0
    for k, (d, m, F0) in enumerate(members):
        with lb.Lattice(d, m) as lat:
            lat.set_populations(np.asarray(F0, dtype=np.float64))
            lat.step(37)
            assert np.array_equal(b.get_populations(k, np.float32), lat.get_populations(np.float32)), k
            r1, u1 = b.macros(k)
            r2, u2 = lat.macros()
            assert np.array_equal(u1, u2)
    b.close()


@pytest.mark.parametrize("mode", [lb.BATCH_ROWS, lb.BATCH_ROWS_PER_FAMILY])
@pytest.mark.parametrize("storage", [lb.F32, lb.BF16S])
def test_batch_rows_many_groups_equal_individual(storage, mode):
    """Row-pipeline batch with ~10x more row groups than resident CTAs (every CTA cycles its stage ring
    over groups of different members and widths): each member equals the lattice stepped alone."""
    members = []
    for nx, ny, nz in ((256, 40, 30), (128, 33, 17), (96, 20, 9)):
        d = lb.make_desc(lb.D3Q27, lb.BGK, storage, (nx, ny, nz), omega=1.5)
        members.append((d, lb.setup_cavity3d(d, 0.06)))
    for n in (512, 64, 208):
        d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (n, n), omega=1.7)
        members.append((d, lb.setup_cavity2d(d, 0.1)))
    b = lb.Batch([x[0] for x in members], [x[1] for x in members])
    b.set_mode(mode)
    b.step(9)
    b.sync()
    assert b.mode() == mode
    # every member's rows can be copied: one launch per step in the one-launch mode
    assert b.plan()[0] == (1 if mode == lb.BATCH_ROWS else 2)
    for k, (d, m) in enumerate(members):
        with lb.Lattice(d, m) as lat:
            lat.step(9)
            assert np.array_equal(b.get_populations(k, np.float32), lat.get_populations(np.float32)), k
    b.close()


def test_duct3d_config_mode_parity():
    dd = lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, (48, 16, 16), omega=1.7)
    mm = lb.setup_duct3d(dd, 0.04, 13, 8, 8, 4)
    solid = mm == 1
    F0 = O.init_equilibrium(oracle_problem(dd, mm), rho=np.where(solid, 0.0, 1.0),
                            u=np.concatenate([np.where(solid, 0.0, 0.04), np.zeros(2 * mm.size)]))
    with lb.Lattice(dd, mm) as lat:
        lat.set_populations(F0)
        lat.step(200)
        F = lat.get_populations(np.float64)
    Fo, _, _ = O.run(oracle_problem(dd, mm), F0, 200, dtype=np.float32)
    assert rel_l2(F, Fo) < 1e-5


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S, lb.BF16S])
@pytest.mark.parametrize("coll", ["bgk_cavity", "bgk_duct", "mrt_ref", "mrt_gs", "mrt_gs_general"])
def test_row_pipeline_equals_plain_kernel(storage, coll):
    """The bulk-copy row pipeline and the one-cell-per-thread kernel run the same collision code on
    the same inputs: results must be bit-identical (lid, solid, equilibrium-inlet, zero-gradient)."""
    if coll == "bgk_cavity":
        d, m, F0 = cavity3d(n=(128, 10, 9), u_lid=0.08, omega=1.6, storage=storage)
    elif coll == "bgk_duct":
        d = lb.make_desc(lb.D3Q27, lb.BGK, storage, (128, 12, 12), omega=1.7)
        m = lb.setup_duct3d(d, 0.04, 30, 6, 6, 3)
        solid = m == 1
        F0 = O.init_equilibrium(oracle_problem(d, m), rho=np.where(solid, 0.0, 1.0),
                                u=np.concatenate([np.where(solid, 0.0, 0.04), np.zeros(2 * m.size)]))
    else:
        basis = lb.MRT_REF if coll == "mrt_ref" else lb.MRT_GRAM_SCHMIDT
        # two rates (16-bit storage: the two-rate collision) or three (the general one)
        rates = lb.mrt_rates(1.8, 1.2) if coll != "mrt_gs_general" else lb.mrt_reference_rates()
        d = lb.make_desc(lb.D3Q27, lb.MRT, storage, (256, 9, 8), mrt_s=rates, mrt_basis=basis)
        m = lb.setup_cavity3d(d, 0.05)
        F0 = np.repeat(lb.velocities(lb.D3Q27)[3], d.cells)
    out = {}
    for kind in (lb.KERNEL_PLAIN, lb.KERNEL_ROWS):
        with lb.Lattice(d, m) as lat:
            lat.set_kernel(kind)
            lat.set_populations(np.asarray(F0, dtype=np.float64))
            lat.step(25)
            lat.sync()
            assert lat.kernel() == kind
            out[kind] = lat.get_populations(np.float32)
    assert np.array_equal(out[lb.KERNEL_PLAIN], out[lb.KERNEL_ROWS])


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S])
@pytest.mark.parametrize("coll", ["bgk", "mrt_gs"])
def test_row_pipeline_ring_wraps_equal_plain_kernel(storage, coll):
    """A lattice with ~20x more row groups than resident CTAs, so every CTA cycles through its
    shared-memory stage ring many times (refills, barrier phases, short last group of each plane):
    still bit-identical to the one-cell-per-thread kernel."""
    shape = (256, 126, 48)  # 126 = 31 groups of 4 + one of 2 (16-bit), 126 groups of 1 (F32)
    if coll == "bgk":
        d = lb.make_desc(lb.D3Q27, lb.BGK, storage, shape, omega=1.7)
    else:
        d = lb.make_desc(lb.D3Q27, lb.MRT, storage, shape, mrt_s=lb.mrt_rates(1.8, 1.2),
                         mrt_basis=lb.MRT_GRAM_SCHMIDT)
    m = lb.setup_cavity3d(d, 0.08)
    out = {}
    for kind in (lb.KERNEL_PLAIN, lb.KERNEL_ROWS):
        with lb.Lattice(d, m) as lat:
            lat.set_kernel(kind)
            lat.step(12)
            lat.sync()
            out[kind] = lat.get_populations(np.float32)
    assert np.isfinite(out[lb.KERNEL_ROWS]).all()
    assert np.array_equal(out[lb.KERNEL_PLAIN], out[lb.KERNEL_ROWS])


def _rows_vs_plain(d, m, F0, steps):
    out = {}
    for kind in (lb.KERNEL_PLAIN, lb.KERNEL_ROWS):
        with lb.Lattice(d, m) as lat:
            lat.set_kernel(kind)
            if F0 is not None:
                lat.set_populations(np.asarray(F0, dtype=np.float64))
            lat.step(steps)
            lat.sync()
            assert lat.kernel() == kind
            out[kind] = lat.get_populations(np.float32)
    assert np.isfinite(out[lb.KERNEL_ROWS]).all()
    return out[lb.KERNEL_PLAIN], out[lb.KERNEL_ROWS]


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S, lb.BF16S])
@pytest.mark.parametrize("case", ["d2q9_lid_128", "d2q9_lid_64", "d2q9_channel_1024", "d3q27_duct_384",
                                  "d3q27_duct_640", "d3q27_mrt_96"])
def test_row_pipeline_other_widths_and_d2q9_equal_plain(storage, case):
    """Widths below the shared-memory row pitch (idle threads), above 512 (two x per thread), D2Q9,
    equilibrium inlets and zero-gradient outlets: bit-identical to the one-cell-per-thread kernel."""
    if case == "d2q9_lid_128":
        d, m, F0 = cavity2d(n=128, storage=storage)
    elif case == "d2q9_lid_64":
        d, m, F0 = cavity2d(n=64, re=400.0, storage=storage)
    elif case == "d2q9_channel_1024":
        d, m, F0 = channel2d(1024, 64, 0.04, 100.0, 200, 32, 10, storage=storage, config_mode=True, seed=1,
                             noise=1e-4)
    elif case in ("d3q27_duct_384", "d3q27_duct_640"):
        nx = int(case.split("_")[-1])
        d = lb.make_desc(lb.D3Q27, lb.BGK, storage, (nx, 14, 10), omega=1.7)
        m = lb.setup_duct3d(d, 0.04, nx / 3, 7, 5, 3)
        F0 = None
    else:
        d = lb.make_desc(lb.D3Q27, lb.MRT, storage, (96, 20, 9), mrt_s=lb.mrt_rates(1.8, 1.2),
                         mrt_basis=lb.MRT_GRAM_SCHMIDT)
        m = lb.setup_cavity3d(d, 0.05)
        F0 = None
    a, b = _rows_vs_plain(d, m, F0, 30)
    assert np.array_equal(a, b)


def _periodic_noise(d, seed):
    """Random near-equilibrium start on a mask-free (fully periodic) lattice: exercises the x wrap."""
    _, _, _, w, _ = lb.velocities(d.lattice)
    n = d.nx * d.ny * d.nz
    rng = np.random.default_rng(seed)
    return np.repeat(w, n) * (1.0 + 0.02 * rng.standard_normal(len(w) * n))


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S, lb.BF16S])
@pytest.mark.parametrize("case", ["d2q9_channel_2048", "d2q9_periodic_1040", "d3q27_duct_2016",
                                  "d3q27_mrt_periodic_1280", "d3q27_mrt_lid_3056"])
def test_row_pipeline_segmented_wide_rows_equal_plain(storage, case):
    """Rows wider than 1024 cells go through the segmented row kernel (1008-cell segments with 8-cell
    halos; the first and last segment fetch their halo from the row's other end).  Widths with a
    32-cell last segment (1040, 2048, 3056) and with whole segments (2016); inlets, zero-gradient
    outlets, bounce-back walls and the periodic wrap all cross segment edges: bit-identical to the
    one-cell-per-thread kernel."""
    if case == "d2q9_channel_2048":
        d, m, F0 = channel2d(2048, 40, 0.04, 100.0, 1000, 20, 8, storage=storage, config_mode=True, seed=2,
                             noise=1e-4)
    elif case == "d2q9_periodic_1040":
        d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (1040, 24), omega=1.6)
        m, F0 = None, _periodic_noise(d, 5)
    elif case == "d3q27_duct_2016":
        d = lb.make_desc(lb.D3Q27, lb.BGK, storage, (2016, 10, 6), omega=1.7)
        m = lb.setup_duct3d(d, 0.04, 1008, 5, 3, 2)
        F0 = None
    elif case == "d3q27_mrt_periodic_1280":
        d = lb.make_desc(lb.D3Q27, lb.MRT, storage, (1280, 6, 5), mrt_s=lb.mrt_rates(1.7, 1.1),
                         mrt_basis=lb.MRT_GRAM_SCHMIDT)
        m, F0 = None, _periodic_noise(d, 6)
    else:
        d = lb.make_desc(lb.D3Q27, lb.MRT, storage, (3056, 6, 5), mrt_s=lb.mrt_rates(1.8, 1.2),
                         mrt_basis=lb.MRT_REF)
        m = lb.setup_cavity3d(d, 0.05)
        F0 = None
    a, b = _rows_vs_plain(d, m, F0, 25)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S, lb.BF16S, lb.F64])
@pytest.mark.parametrize("arith", [lb.ARITH_ABSOLUTE, lb.ARITH_DEVIATION])
@pytest.mark.parametrize("shape,solid", [((128, 128), False), ((100, 50), True), ((20, 10), False),
                                         ((48, 36), True), ((200, 24), "zerograd")])
def test_shanchen_fused_equals_two_pass(storage, arith, shape, solid):
    """The one-pass Shan-Chen kernel (KERNEL_ROWS: a window sliding down y, psi of the next row in a
    shared ring) against the two-pass kernels (KERNEL_PLAIN: psi through global memory), each with
    32-bit population indices (their choice on these lattices) and with 64-bit ones (the form of
    lattices beyond 2^32 / 9 cells, forced by a test hook): bit-identical populations and fields, on full and
    partial column strips, a lattice narrower than a strip, with solid (bounce-back, set-density)
    cells, and with zero-gradient outlet columns on both sides of the first strip edge (x = 127 and
    128: the window pulls them both as its own cells and as the neighbouring strip's edge column)."""
    if arith == lb.ARITH_ABSOLUTE and storage in (lb.F16S, lb.BF16S):
        pytest.skip("absolute arithmetic is F32/F64 only")
    d = lb.make_desc(lb.D2Q9, lb.SHANCHEN, storage, shape, omega=1.0, sc_G=-4.5, arithmetic=arith)
    m = None
    n = d.cells
    if solid == "zerograd":
        lb.set_classes(d, [(0, 1.0, 0.0, 0.0, 0.0), (lb.ZEROGRAD_XP, 1.0, 0.0, 0.0, 0.0)])
        xx = np.repeat(np.arange(shape[0])[None, :], shape[1], axis=0).ravel()  # x of cell x + nx y
        m = ((xx == 127) | (xx == 128) | (xx == shape[0] - 1)).astype(np.uint8)
    elif solid:
        lb.set_classes(d, [(0, 1.0, 0.0, 0.0, 0.0), (lb.BOUNCE | lb.SET_RHO | lb.SET_UX | lb.SET_UY, 0.5, 0.0, 0.0, 0.0)])
        xx, yy = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), indexing="ij")
        m = ((xx - shape[0] // 3) ** 2 + (yy - shape[1] // 2) ** 2 <= (min(shape) // 5) ** 2).astype(np.uint8)
        m = m.ravel(order="F")
    rng = np.random.default_rng(4)
    rho = 0.693 + 0.01 * rng.uniform(-1.0, 1.0, size=n)
    out = {}
    for kind, index64 in ((lb.KERNEL_PLAIN, False), (lb.KERNEL_PLAIN, True), (lb.KERNEL_ROWS, False),
                          (lb.KERNEL_ROWS, True)):
        with lb.Lattice(d, m) as lat:
            lat.set_kernel(kind)
            if index64:
                lat.test_index64(True)
            lat.init_equilibrium(rho=rho)
            lat.step(40)
            lat.sync()
            assert lat.kernel() == kind
            r, u = lat.macros()
            out[kind, index64] = (lat.get_populations(np.float64), r, u)
    a = out[lb.KERNEL_PLAIN, False]
    for key in ((lb.KERNEL_PLAIN, True), (lb.KERNEL_ROWS, False), (lb.KERNEL_ROWS, True)):
        b = out[key]
        assert np.isfinite(b[0]).all()
        for x, y in zip(a, b):
            assert np.array_equal(x, y), key


def _index_case(case, storage):
    if case == "cavity2d":
        return cavity2d(n=64, u_lid=0.1, re=300, storage=storage)
    if case == "channel2d":  # equilibrium inlet, zero-gradient outlet, cylinder
        return channel2d(96, 40, 0.04, 100.0, 24, 20, 6, storage=storage, config_mode=True, seed=1, noise=1e-3)
    if case == "channel2d_wide":  # rows wider than 1024 cells: the segmented row kernel
        return channel2d(1088, 12, 0.04, 100.0, 300, 6, 3, storage=storage, config_mode=True, seed=1, noise=1e-3)
    if case == "cavity3d":
        return cavity3d(n=(32, 14, 12), u_lid=0.05, omega=1.3, storage=storage)
    if case == "mrt_wide":  # D3Q27 rows wider than 1024 cells
        d = lb.make_desc(lb.D3Q27, lb.MRT, storage, (1040, 4, 6), mrt_s=lb.mrt_rates(1.7, 1.1),
                         mrt_basis=lb.MRT_GRAM_SCHMIDT)
        m = lb.setup_cavity3d(d, 0.05)
        w = lb.velocities(lb.D3Q27)[3]
        rng = np.random.default_rng(13)
        return d, m, np.repeat(w, d.cells) * (1.0 + 0.01 * rng.standard_normal(27 * d.cells))
    rates = lb.mrt_rates(1.7, 1.2) if case == "mrt_two_rate" else None
    basis = lb.MRT_REF if case == "mrt_ref" else lb.MRT_GRAM_SCHMIDT
    return mrt_cavity(n=16, u_lid=0.1, storage=storage, basis=basis, rates=rates)


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S, lb.BF16S, lb.F64])
@pytest.mark.parametrize("case", ["cavity2d", "channel2d", "channel2d_wide", "cavity3d", "mrt_ref", "mrt_gs",
                                  "mrt_two_rate", "mrt_wide"])
@pytest.mark.parametrize("arith", [lb.ARITH_DEVIATION, lb.ARITH_ABSOLUTE])
def test_plain_kernels_32_and_64_bit_indices_agree(storage, case, arith):
    """The plain step kernels (BGK, MRT in both bases, the two-rate MRT of 16-bit storage) with 32-bit
    population indices (their choice on lattices with Q N <= 2^32) and with 64-bit ones (forced by a
    test hook): bit-identical populations, with bounce-back, lid, inlet and zero-gradient classes, on
    rows narrower and wider than 1024 cells."""
    if arith == lb.ARITH_ABSOLUTE and (storage in (lb.F16S, lb.BF16S) or case.startswith("mrt")):
        pytest.skip("absolute arithmetic: F32/F64 BGK only")
    kernel = lb.KERNEL_PLAIN
    d, m, F0 = _index_case(case, storage)
    d.arithmetic = arith
    out = []
    for index64 in (False, True):
        with lb.Lattice(d, m) as lat:
            lat.set_kernel(kernel)
            if index64:
                lat.test_index64(True)
            lat.set_populations(np.asarray(F0, dtype=np.float64))
            lat.step(30)
            assert lat.kernel() == kernel
            out.append(lat.get_populations(np.float64))
    assert np.isfinite(out[0]).all() and np.array_equal(out[0], out[1])


def test_row_pipeline_needs_eligible_shape():
    rejected = [
        lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, (100, 8, 8), omega=1.3),  # 100-byte mask rows
        lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (2056, 8), omega=1.3),  # segmented, but 2056 % 16 != 0
        lb.make_desc(lb.D3Q27, lb.BGK, lb.F64, (128, 8, 8), omega=1.3),  # FP64 storage
        lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (128, 8), omega=1.3, arithmetic=lb.ARITH_ABSOLUTE),
    ]
    for d in rejected:
        with lb.Lattice(d, None) as lat:
            with pytest.raises(lb.LbmError) as e:
                lat.set_kernel(lb.KERNEL_ROWS)
            assert e.value.code == -5
            lat.step(3)
            assert lat.kernel() == lb.KERNEL_PLAIN
    # nx = 112 (a multiple of 16 below the 128-cell row pitch): eligible, and equal to the plain kernel
    d, m, F0 = cavity3d(n=(112, 8, 8), storage=lb.F16S)
    a, b = _rows_vs_plain(d, m, F0, 7)
    assert np.array_equal(a, b)


def test_batch_one_launch_autotuned_and_stall_recovers():
    """AUTO picks among tiles, one launch for both families and one launch per family; a stalled row
    stage (test hook) makes lbm_batch_sync report LBM_ERR_TIMEOUT once, and the batch steps on
    correctly after its populations are set again."""
    members = []
    for n in (64, 128):
        d, m, F0 = cavity2d(n=n, u_lid=0.1, re=300, storage=lb.F16S)
        members.append((d, m, F0))
    d, m, F0 = cavity3d(n=(64, 24, 20), u_lid=0.05, omega=1.2, storage=lb.F16S)
    members.append((d, m, F0))
    # the batch has stepped further than the lattices it is compared with at the end: rounding to
    # nearest keeps that comparison bit-exact (stochastic rounding draws on the step number)
    for d, _, _ in members:
        d.rounding = lb.ROUND_NEAREST
    b = lb.Batch([x[0] for x in members], [x[1] for x in members])
    for k, (_, _, F0) in enumerate(members):
        b.set_populations(k, np.asarray(F0, dtype=np.float64))
    b.step(2)
    b.sync()
    assert b.mode() in (lb.BATCH_TILES, lb.BATCH_ROWS, lb.BATCH_ROWS_PER_FAMILY)
    b.set_mode(lb.BATCH_ROWS)
    b.step(1)
    b.sync()
    launches, g2, g3 = b.plan()
    assert launches == 1 and g2 > 0 and g3 > 0
    b.test_stall_next_step(item=3, wait_clocks=1 << 21)
    b.step(2)
    assert lb.lib().lbm_batch_sync(b._h) == -8
    assert lb.lib().lbm_batch_sync(b._h) == 0
    for k, (_, _, F0) in enumerate(members):
        b.set_populations(k, np.asarray(F0, dtype=np.float64))
    b.step(21)
    for k, (d, m, F0) in enumerate(members):
        with lb.Lattice(d, m) as lat:
            lat.set_populations(np.asarray(F0, dtype=np.float64))
            lat.step(21)
            assert np.array_equal(b.get_populations(k, np.float32), lat.get_populations(np.float32)), k
    b.close()


@pytest.mark.parametrize("storage,mode,tol", [(lb.F32, lb.BATCH_ROWS, 1e-5), (lb.F32, lb.BATCH_TILES, 1e-5),
                                               (lb.F64, lb.BATCH_TILES, 1e-12)])
def test_batch_members_match_the_oracle(storage, mode, tol):
    """A small mixed ensemble (D2Q9 lids of two sizes and rates, D3Q27 ducts with a sphere, an
    equilibrium inlet and a zero-gradient outlet) against the FP64 oracle run of each member: the batch
    compared with the reference's algorithm directly, not only with the single-lattice engine."""
    from helpers import P

    specs = [("lid", 64, 0.1, 300.0), ("lid", 96, 0.1, 150.0), ("duct", 32, 0.04, 20.0), ("duct", 48, 0.04, 30.0)]
    members = []
    for kind, L, u, re in specs:
        if kind == "lid":
            om = lb.omega_from_re(u, L, re, 1)
            d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (L, L), omega=om)
            m = lb.setup_cavity2d(d, u)
            p = P.cavity2d(L, L, u, om)
            F0 = P.rest_state(p)
        else:
            om = 1.0 / (3.0 * (u * (L / 4.0) / re) + 0.5)
            d = lb.make_desc(lb.D3Q27, lb.BGK, storage, (4 * L, L, L), omega=om)
            m = lb.setup_duct3d(d, u, 2.0 * L, L / 2.0, L / 2.0, L / 8.0)
            p = P.duct3d(4 * L, L, L, u, 2.0 * L, L / 2.0, L / 2.0, L / 8.0, om)
            F0 = P.channel_start_state(p, u)
        members.append((d, m, p, F0))
    b = lb.Batch([x[0] for x in members], [x[1] for x in members])
    if storage != lb.F64:
        b.set_mode(mode)
    for k, (_, _, _, F0) in enumerate(members):
        b.set_populations(k, np.asarray(F0, dtype=np.float64))
    b.step(120)
    b.sync()
    for k, (d, m, p, F0) in enumerate(members):
        Fo, _, _ = O.run(p, F0, 120)
        assert rel_l2(b.get_populations(k, np.float64), Fo) < tol, (k, rel_l2(b.get_populations(k, np.float64), Fo))
    b.close()


def _cluster_case(case, storage):
    if case == "cavity128":
        return cavity2d(n=128, storage=storage)
    if case == "cavity_odd":  # rows not a multiple of the cluster size, a short and an empty CTA
        d, m, F0 = cavity2d(n=100, storage=storage)
        return d, m, F0
    if case == "channel":  # equilibrium inlet, zero-gradient outlet, a solid circle
        return channel2d(96, 40, 0.04, 100.0, 24, 20, 6, storage=storage, config_mode=True, seed=4, noise=1e-3)
    # periodic, no mask, a thin lattice: rows 1 per CTA and a lattice one row high per CTA pair
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (48, 10), omega=1.7)
    _, _, _, w, _ = lb.velocities(lb.D2Q9)
    rng = np.random.default_rng(5)
    return d, None, np.repeat(w, d.cells) * (1.0 + 0.02 * rng.standard_normal(9 * d.cells))


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S, lb.BF16S, lb.F64])
@pytest.mark.parametrize("case", ["cavity128", "cavity_odd", "channel", "periodic_thin"])
def test_cluster_resident_kernel_equals_plain(storage, case):
    """LBM_KERNEL_CLUSTER (the lattice resident in one thread-block cluster's shared memory for many
    steps per launch) is bit-identical to the plain kernel: runs of 1, 3, 10 and 4100 steps (two
    launches), stochastic rounding for the 16-bit storage, and a step cut into plane sets (which take
    the plain kernel) in between."""
    d, m, F0 = _cluster_case(case, storage)
    F0 = np.asarray(F0, dtype=np.float64)
    with lb.Lattice(d, m) as a, lb.Lattice(d, m) as b:
        a.set_kernel(lb.KERNEL_PLAIN)
        b.set_kernel(lb.KERNEL_CLUSTER)
        for lat in (a, b):
            lat.set_populations(F0)
        for n in (1, 3, 10):
            a.step(n)
            b.step(n)
            assert b.kernel() == lb.KERNEL_CLUSTER
            assert np.array_equal(a.get_populations(np.float64), b.get_populations(np.float64)), n
            # the macros pull the previous step's populations: a multi-step launch leaves them too
            (ra, ua), (rb, ub) = a.macros(np.float64), b.macros(np.float64)
            assert np.array_equal(ra, rb) and np.array_equal(ua, ub), n
        a.step(1)
        b.step_planes(0, 1, False)
        b.step_planes(1, d.ny - 1, True)
        a.step(4100)
        b.step(4100)
        assert a.steps_done == b.steps_done == 4115
        ref, got = a.get_populations(np.float64), b.get_populations(np.float64)
        (ra, ua), (rb, ub) = a.macros(np.float64), b.macros(np.float64)
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub)
    assert np.isfinite(got).all() and np.array_equal(got, ref)


@pytest.mark.parametrize("storage", [lb.F32, lb.F16S])
def test_zouhe_boundaries_identical_in_every_family(storage):
    """Zou-He inlet and outlet cells rebuild their incoming populations inside the shared BGK collision,
    so the plain kernel, the row pipeline, the cluster-resident kernel and an ensemble member give the
    same bits."""
    d, m, F0 = channel2d(128, 48, 0.05, 20.0, 30, 24, 5, storage=storage, config_mode=2, seed=8, noise=1e-3)
    F0 = np.asarray(F0, dtype=np.float64)
    out = {}
    for kind in (lb.KERNEL_PLAIN, lb.KERNEL_ROWS, lb.KERNEL_CLUSTER):
        with lb.Lattice(d, m) as lat:
            lat.set_kernel(kind)
            lat.set_populations(F0)
            lat.step(333)
            lat.sync()
            assert lat.kernel() == kind
            out[kind] = (lat.get_populations(np.float64), *lat.macros(np.float64))
    b = lb.Batch([d], [m])
    b.set_populations(0, F0)
    b.step(333)
    b.sync()
    member = b.get_populations(0, np.float64)
    b.close()
    ref = out[lb.KERNEL_PLAIN]
    assert np.isfinite(ref[0]).all()
    for kind in (lb.KERNEL_ROWS, lb.KERNEL_CLUSTER):
        for x, y in zip(out[kind], ref):
            assert np.array_equal(x, y), kind
    assert np.array_equal(member, ref[0])


def test_cluster_kernel_is_refused_where_it_does_not_fit():
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (1024, 256), omega=1.2)
    with lb.Lattice(d, None) as lat:
        with pytest.raises(lb.LbmError):
            lat.set_kernel(lb.KERNEL_CLUSTER)
    d = lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, (16, 16, 16), omega=1.2)
    with lb.Lattice(d, None) as lat:
        with pytest.raises(lb.LbmError):
            lat.set_kernel(lb.KERNEL_CLUSTER)


def test_cluster_kernel_contexts_of_different_sizes_interleaved():
    """The cluster kernel's shared-memory size is a per-kernel attribute: a context set up after a
    larger one (which lowers it) must not break the larger one's next launch."""
    big, small = cavity2d(n=128), cavity2d(n=64)
    with lb.Lattice(big[0], big[1]) as a, lb.Lattice(big[0], big[1]) as ref:
        ref.set_kernel(lb.KERNEL_PLAIN)
        a.set_kernel(lb.KERNEL_CLUSTER)
        for lat in (a, ref):
            lat.set_populations(big[2])
            lat.step(5)
        with lb.Lattice(small[0], small[1]) as b:
            b.set_kernel(lb.KERNEL_CLUSTER)
            b.set_populations(small[2])
            b.step(5)
            a.step(7)
            ref.step(7)
            b.step(3)
            b.sync()
            a.sync()
        assert np.array_equal(a.get_populations(np.float64), ref.get_populations(np.float64))


def test_autotune_picks_the_cluster_kernel_for_the_128_cavity():
    d, m, F0 = cavity2d(n=128)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        lat.step(2)
        assert lat.kernel() == lb.KERNEL_CLUSTER
