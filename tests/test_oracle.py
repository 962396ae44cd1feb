"""The CPU oracle against the golden fixtures (literal emulation of the reference's array programs)
and against the invariants the reference's physics must keep.  CPU only."""
import numpy as np
import pytest

from helpers import E, O, cavity2d, cavity3d, channel2d, lb, load_golden, mrt_cavity, oracle_problem, rel_l2


def _check_golden(name, d, m, F0, steps):
    g = load_golden(name)
    p = oracle_problem(d, m)
    for tag, dt, tol in (("f64", np.float64, 1e-13), ("f32", np.float32, 2e-6)):
        F, rho, u = O.run(p, F0, steps, dtype=dt)
        if tag == "f64":
            assert np.max(np.abs(F - g["F_f64"])) < tol
            assert np.max(np.abs(rho - g["rho_f64"])) < tol
            assert np.max(np.abs(u[:d.cells] - g["ux_f64"])) < tol
        else:
            assert rel_l2(F, g["F_f32"]) < tol
            assert rel_l2(u[:d.cells], g["ux_f32"]) < 20 * tol


def test_golden_d2q9_lid():
    d, m, F0 = cavity2d(n=16, u_lid=0.1, re=100.0)
    # the fixture is 16x12: rebuild with that shape
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (16, 12), omega=1 / 0.884)
    m = lb.setup_cavity2d(d, 0.1)
    F0 = np.repeat(lb.velocities(lb.D2Q9)[3], 16 * 12)
    _check_golden("d2q9_lid_16x12", d, m, F0, 200)


def test_golden_d2q9_channel():
    om = 1 / (3 * (0.1 * 2 * 3 / 20) + 0.5)
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (60, 24), omega=om)
    m = lb.setup_channel2d(d, 0.1, 13, 12, 3, False)
    solid = np.isin(m, [1, 4])
    F0 = O.init_equilibrium(oracle_problem(d, m), rho=np.where(solid, 0.0, 1.0),
                            u=np.concatenate([np.where(solid, 0.0, 0.1), np.zeros(m.size)]))
    _check_golden("d2q9_channel_60x24", d, m, F0, 100)


def test_golden_d3q27_bgk_lid():
    d, m, F0 = cavity3d(n=(8, 9, 10), u_lid=0.1, omega=1.3)
    _check_golden("d3q27_bgk_lid_8x9x10", d, m, F0, 40)


def test_golden_d3q27_mrt_lid():
    d, m, F0 = mrt_cavity(n=8, u_lid=0.1)
    g = load_golden("d3q27_mrt_lid_8")
    p = oracle_problem(d, m)
    F, rho, u = O.run(p, F0, 40, dtype=np.float64)
    assert np.max(np.abs(F - g["F_f64"])) < 1e-12
    F, rho, u = O.run(p, F0, 40, dtype=np.float32)
    assert rel_l2(F, g["F_f32"]) < 5e-6


@pytest.mark.parametrize("shape", [(9, 7), (5, 13)])
def test_oracle_vs_emulation_odd_sizes(shape):
    nx, ny = shape
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F64, shape, omega=1.7)
    m = lb.setup_cavity2d(d, 0.05)
    F0 = np.repeat(lb.velocities(lb.D2Q9)[3], nx * ny)
    Fo, ro, uo = O.run(oracle_problem(d, m), F0, 30)
    Fe, De, Ue, Ve = E.d2q9_lid(nx, ny, 0.05, 1.7, 30)
    assert np.max(np.abs(Fo - Fe)) < 1e-14
    assert np.max(np.abs(uo[nx * ny:] - E.flat(Ve))) < 1e-14


def _periodic(lattice, collision, shape, **kw):
    return O.Problem(lattice, collision, shape, **kw)


def _random_state(p, seed, amp=0.02):
    rng = np.random.default_rng(seed)
    rho = 1.0 + rng.uniform(-amp, amp, p.n)
    u = rng.uniform(-amp, amp, p.dim * p.n)
    return O.init_equilibrium(p, rho=rho, u=u)


def test_rest_state_is_kept():
    p = _periodic("D2Q9", "BGK", (12, 10), omega=1.4)
    F0 = O.init_equilibrium(p)
    F, rho, u = O.run(p, F0, 50)
    assert np.max(np.abs(F - F0)) < 1e-15
    # the reference MRT's rest state is M^-1 meq(rho=1, u=0) of its own equilibrium table
    p3 = _periodic("D3Q27", "MRT", (5, 6, 7), s=E.REF_RATES)
    M, Mi = O.mrt_matrices("ref")
    meq = np.zeros(27)
    meq[0], meq[7], meq[17:20], meq[26] = 1.0, 1.0, 1.0 / 9.0, 1.0 / 27.0
    F0 = np.repeat(Mi @ meq, p3.n)
    F1, _, _ = O.run(p3, F0, 6)
    assert np.max(np.abs(F1 - F0)) < 1e-14


@pytest.mark.parametrize("collision,lattice,extra", [
    ("BGK", "D2Q9", {"omega": 1.3}), ("BGK", "D3Q27", {"omega": 0.8}),
    ("MRT", "D3Q27", {"s": [1.2] * 27, "mrt_basis": "gs"}),
    ("MRT", "D3Q27", {"s": E.REF_RATES, "mrt_basis": "gs"}),
    ("SC", "D2Q9", {"omega": 1.0, "G": -5.5}),
])
def test_mass_conserved_periodic(collision, lattice, extra):
    shape = (11, 9) if lattice == "D2Q9" else (6, 5, 7)
    p = _periodic(lattice, collision, shape, **extra)
    F0 = _random_state(p, 3)
    F, _, _ = O.run(p, F0, 40)
    s0, s1 = O.sums(p, F0), O.sums(p, F)
    assert abs(s1[0] - s0[0]) / s0[0] < 1e-13
    if collision != "SC":
        assert np.max(np.abs(s1[1:] - s0[1:])) < 1e-12


def test_transpose_symmetry_d2q9():
    # swapping x and y maps direction i to the direction with (cy, cx)
    cx, cy, _, _, _ = O.velocities("D2Q9")
    perm = [next(j for j in range(9) if cx[j] == cy[i] and cy[j] == cx[i]) for i in range(9)]
    nx, ny = 10, 7
    p = _periodic("D2Q9", "BGK", (nx, ny), omega=1.6)
    pt = _periodic("D2Q9", "BGK", (ny, nx), omega=1.6)
    F0 = _random_state(p, 5).reshape(9, ny, nx)       # [i][y][x]
    F0t = np.empty((9, nx, ny))
    for i in range(9):
        F0t[perm[i]] = F0[i].T
    F, rho, u = O.run(p, F0.ravel(), 25)
    Ft, rhot, ut = O.run(pt, F0t.ravel(), 25)
    assert np.allclose(rho.reshape(ny, nx).T, rhot.reshape(nx, ny), atol=1e-14)
    assert np.allclose(u[:nx * ny].reshape(ny, nx).T, ut[nx * ny:].reshape(nx, ny), atol=1e-14)


def test_mrt_gram_schmidt_with_one_rate_is_bgk():
    om = 1.37
    pm = _periodic("D3Q27", "MRT", (6, 5, 4), s=[om] * 27, mrt_basis="gs")
    pb = _periodic("D3Q27", "BGK", (6, 5, 4), omega=om)
    F0 = _random_state(pb, 7)
    Fm, _, _ = O.run(pm, F0, 10)
    Fb, _, _ = O.run(pb, F0, 10)
    assert np.max(np.abs(Fm - Fb)) < 1e-13


def test_gram_schmidt_rows_are_orthogonal():
    M, Mi = O.mrt_matrices("gs")
    G = M @ M.T
    assert np.max(np.abs(G - np.diag(np.diag(G)))) < 1e-12
    Mr, _ = O.mrt_matrices("ref")
    # same nested spans as the reference rows (Gram-Schmidt in row order)
    for k in range(1, 27):
        a = np.linalg.matrix_rank(np.vstack([Mr[:k + 1], M[:k + 1]]), tol=1e-9)
        assert a == k + 1


def test_closed_box_conserves_mass():
    # cavity without lid motion: every population stays inside the box
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F64, (14, 11), omega=1.2)
    m = lb.setup_cavity2d(d, 0.0)
    p = oracle_problem(d, m)
    rng = np.random.default_rng(11)
    fluid = m.ravel() != 1
    rho = np.where(fluid, 1.0 + rng.uniform(-0.01, 0.01, m.size), 0.0)
    F0 = O.init_equilibrium(p, rho=rho)
    F, _, _ = O.run(p, F0, 60)
    assert abs(O.sums(p, F)[0] - O.sums(p, F0)[0]) < 1e-12


def test_zero_gradient_outlet_copies_upstream_column():
    # a uniform flow through an open channel (no walls) is a fixed point of the config-mode BCs
    nx, ny, u0 = 20, 6, 0.05
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F64, (nx, ny), omega=1.1)
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.EQUILIBRIUM | lb.SET_RHO | lb.SET_UX | lb.SET_UY | lb.SET_UZ, 1, u0, 0, 0),
                       (lb.ZEROGRAD_XP, 1, 0, 0, 0)])
    m = np.zeros((ny, nx), np.uint8)
    m[:, 0] = 1
    m[:, nx - 1] = 2
    p = oracle_problem(d, m.ravel())
    F0 = O.init_equilibrium(p, u=np.concatenate([np.full(nx * ny, u0), np.zeros(nx * ny)]))
    F, rho, u = O.run(p, F0, 30)
    assert np.max(np.abs(F - F0)) < 1e-14


def _zouhe_channel(nx, ny, u_in, omega, steps, dtype=np.float64):
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F64, (nx, ny), omega=omega)
    m = lb.setup_channel2d(d, u_in, -100.0, -100.0, 0.0, 2)  # Zou-He inlet and outlet, no obstacle
    p = oracle_problem(d, m)
    F0 = O.init_equilibrium(p, rho=np.where(m == 1, 0.0, 1.0))
    F, rho, u = O.run(p, F0, steps, dtype=dtype)
    return m.reshape(ny, nx), rho.reshape(ny, nx), u[:nx * ny].reshape(ny, nx), u[nx * ny:].reshape(ny, nx)


def test_zouhe_channel_develops_poiseuille_flow():
    """Zou-He velocity inlet (uniform u_in) and pressure outlet (rho = 1) on a walled channel: the inlet
    cells carry exactly the prescribed velocity and the outlet cells the prescribed density, the volume
    flux is the same through every column, and the developed profile is the Poiseuille parabola
    between walls halfway between the solid and the first fluid rows."""
    nx, ny, u_in = 64, 18, 0.02
    m, rho, ux, uy = _zouhe_channel(nx, ny, u_in, 1.0 / 0.8, 8000)
    fluid = slice(1, ny - 1)
    assert np.max(np.abs(ux[fluid, 0] - u_in)) < 1e-13
    assert np.max(np.abs(uy[fluid, 0])) < 1e-13
    assert np.max(np.abs(rho[fluid, nx - 1] - 1.0)) < 1e-13
    flux = (rho * ux)[fluid, :].sum(axis=0)
    assert np.max(np.abs(flux / flux[0] - 1.0)) < 2e-3
    y = np.arange(ny, dtype=np.float64)[fluid]
    shape = (y - 0.5) * (ny - 1.5 - y)  # walls at y = 0.5 and y = ny - 1.5
    prof = ux[fluid, 3 * nx // 4]
    fit = shape * (prof @ shape) / (shape @ shape)
    assert rel_l2(prof, fit) < 2e-2
    assert abs(prof.mean() / u_in - 1.0) < 2e-2


def test_zouhe_uniform_flow_is_kept():
    """A uniform flow u_in through an open periodic-in-y channel with a Zou-He inlet (u_in) and outlet
    (rho = 1) is a fixed point: the rebuilt populations are the equilibrium ones."""
    nx, ny, u0 = 20, 6, 0.05
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F64, (nx, ny), omega=1.1)
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.ZOUHE_VEL_XM, 1, u0, 0, 0), (lb.ZOUHE_RHO_XP, 1, 0, 0, 0)])
    m = np.zeros((ny, nx), np.uint8)
    m[:, 0] = 1
    m[:, nx - 1] = 2
    p = oracle_problem(d, m.ravel())
    F0 = O.init_equilibrium(p, u=np.concatenate([np.full(nx * ny, u0), np.zeros(nx * ny)]))
    F, rho, u = O.run(p, F0, 30)
    assert np.max(np.abs(F - F0)) < 1e-14
