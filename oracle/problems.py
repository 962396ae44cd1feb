"""The reference drivers' problems, restated on the oracle side (numpy only).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference legs import this module.  It builds the loop-invariant state of each reference driver --
the solid mask ``BOUND``, the boundary overwrites as per-cell classes, the relaxation rules and the
start state -- directly from the reference's definitions, without the engine's set-up helpers, so the
engine's ``lbm_setup_*`` output is checked against an independent restatement (tests/test_problems.py)
and the reference arm of bench.py never loads the engine library.

Class semantics (flags and values) are the oracle's: BOUNCE, SET_RHO, SET_UX, SET_UY, SET_UZ,
EQUILIBRIUM, ZEROGRAD_XP in ``oracle.py``; a solid node of the reference (``ON = where(BOUND)``) is
BOUNCE with rho = u = 0 forced, the lid row forces u, and the channel ends force rho / u_x in the
order the reference assigns them.
"""
from __future__ import annotations

import numpy as np

import oracle as O

SOLID = O.BOUNCE | O.SET_RHO | O.SET_UX | O.SET_UY | O.SET_UZ
FORCE_U = O.SET_UX | O.SET_UY | O.SET_UZ
EQ_INLET = O.EQUILIBRIUM | O.SET_RHO | O.SET_UX | O.SET_UY | O.SET_UZ


def omega_from_re(u: float, L: float, re: float, rule: int = 0) -> float:
    """tau = 3 nu + 1/2 with nu = u L / Re (C++ drivers, cpp/d2q9_bgk_lid.cpp:45) or nu = u 2 L / Re
    (Rust drivers, rust/examples/d2q9_bgk_lid.rs:52); omega = 1 / tau."""
    nu = u * 2.0 * L / re if rule == 1 else u * L / re
    return 1.0 / (3.0 * nu + 0.5)


def mrt_reference_rates():
    """S of rust/examples/d3q27_mrt_lid.rs:111-150 (s0 = s1 = 1.3, sv = 1.1, sb = 0.9, s3 = 1.2,
    s3b = 0.9, s4 = 1.2, s4b = 1.2, s5 = s6 = 1.1) in the reference's row order."""
    s0, s1, sv, sb, s3, s3b, s4, s4b, s5, s6 = 1.3, 1.3, 1.1, 0.9, 1.2, 0.9, 1.2, 1.2, 1.1, 1.1
    return [s0, s1, s1, s1, sv, sv, sv, sb, sv, sv, s3, s3, s3, s3, s3, s3, s3b, s4, s4, s4,
            s4b, s4b, s4b, s5, s5, s5, s6]


def mrt_rates(sv: float, other: float):
    """Shear rate sv on the five shear rows (4-6: ex ey, ex ez, ey ez; 8, 9: ex^2 - ey^2,
    ex^2 - ez^2) and `other` on every other row."""
    s = [other] * 27
    for k in (4, 5, 6, 8, 9):
        s[k] = sv
    return s


def _grid2(nx, ny):
    x = np.arange(nx)[:, None] * np.ones((1, ny), dtype=np.int64)
    y = np.ones((nx, 1), dtype=np.int64) * np.arange(ny)[None, :]
    return x, y


def _grid3(nx, ny, nz):
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return x, y, z


def _flat(a):
    return np.ascontiguousarray(a).ravel(order="F").astype(np.uint8)


def cavity2d(nx: int, ny: int, u_lid: float, omega: float) -> O.Problem:
    """cpp/d2q9_bgk_lid.cpp: BOUND = 1; BOUND(1..nx-2, 1..ny-1) = 0 (:90-91); the lid row
    UX(1..nx-2, ny-1) = u_lid, UY = 0 (:141-142); UX/UY/DENSITY(ON) = 0 (:144-146)."""
    BOUND = np.ones((nx, ny), dtype=bool)
    BOUND[1:nx - 1, 1:] = False
    cls = np.where(BOUND, 1, 0)
    cls[1:nx - 1, ny - 1] = 2
    classes = [(0, 1.0, 0.0, 0.0, 0.0), (SOLID, 0.0, 0.0, 0.0, 0.0), (FORCE_U, 1.0, u_lid, 0.0, 0.0)]
    return O.Problem("D2Q9", "BGK", (nx, ny), omega=omega, classes=classes, mask=_flat(cls))


def channel2d(nx: int, ny: int, u_in: float, ox: float, oy: float, r: float, omega: float,
              config_mode: int = 0) -> O.Problem:
    """cpp/d2q9_bgk_channel_packed.cpp: solid circle (x-ox)^2 + (y-oy)^2 <= r^2 and rows y = 0,
    y = ny-1 (:37-39).  Reference BCs (:64-69), in order: UX(0,:) = u_max; UX/UY/DENSITY(ON) = 0;
    DENSITY(0,:) = DENSITY(nx-1,:) = 1 -- so solid cells of the end columns keep rho = 1.  Config mode
    1: an equilibrium inlet (rho = 1, u = (u_in, 0)) at x = 0 and a zero-gradient outlet at x = nx-1.
    Config mode 2: a Zou-He velocity inlet (u = (u_in, 0)) and a Zou-He pressure outlet (rho = 1,
    uy = 0), the open boundaries of Zou & He (1997)."""
    x, y = _grid2(nx, ny)
    solid = ((x - ox) ** 2 + (y - oy) ** 2 <= r * r) | (y == 0) | (y == ny - 1)
    end = (x == 0) | (x == nx - 1)
    cls = np.zeros((nx, ny), dtype=np.int64)
    cls[(x == 0) & ~solid] = 2
    cls[(x == nx - 1) & ~solid] = 3
    cls[solid] = 1
    if config_mode == 2:
        classes = [(0, 1.0, 0.0, 0.0, 0.0), (SOLID, 0.0, 0.0, 0.0, 0.0), (O.ZOUHE_VEL_XM, 1.0, u_in, 0.0, 0.0),
                   (O.ZOUHE_RHO_XP, 1.0, 0.0, 0.0, 0.0)]
    elif config_mode:
        classes = [(0, 1.0, 0.0, 0.0, 0.0), (SOLID, 0.0, 0.0, 0.0, 0.0), (EQ_INLET, 1.0, u_in, 0.0, 0.0),
                   (O.ZEROGRAD_XP, 1.0, 0.0, 0.0, 0.0)]
    else:
        cls[solid & end] = 4
        classes = [(0, 1.0, 0.0, 0.0, 0.0), (SOLID, 0.0, 0.0, 0.0, 0.0),
                   (O.SET_UX | O.SET_RHO, 1.0, u_in, 0.0, 0.0), (O.SET_RHO, 1.0, 0.0, 0.0, 0.0),
                   (SOLID, 1.0, 0.0, 0.0, 0.0)]
    return O.Problem("D2Q9", "BGK", (nx, ny), omega=omega, classes=classes, mask=_flat(cls))


def cavity3d(nx: int, ny: int, nz: int, u_lid: float, omega: float = 1.0, collision: str = "BGK",
             s=None, mrt_basis: str = "ref") -> O.Problem:
    """cpp/d3q27_bgk_lid.cpp: fluid (1..nx-2, 1..ny-2, 1..nz-1), solid elsewhere (:119-120); the lid
    plane z = nz-1 forces u = (u_lid, 0, 0) (:179-186); rust/examples/d3q27_mrt_lid.rs uses the same
    geometry for the MRT cavity."""
    BOUND = np.ones((nx, ny, nz), dtype=bool)
    BOUND[1:nx - 1, 1:ny - 1, 1:] = False
    cls = np.where(BOUND, 1, 0)
    cls[1:nx - 1, 1:ny - 1, nz - 1] = 2
    classes = [(0, 1.0, 0.0, 0.0, 0.0), (SOLID, 0.0, 0.0, 0.0, 0.0), (FORCE_U, 1.0, u_lid, 0.0, 0.0)]
    return O.Problem("D3Q27", collision, (nx, ny, nz), omega=omega, s=s, mrt_basis=mrt_basis,
                     classes=classes, mask=_flat(cls))


def duct3d(nx: int, ny: int, nz: int, u_in: float, ox: float, oy: float, oz: float, r: float,
           omega: float) -> O.Problem:
    """D3Q27 channel (the config-5 member): walls y = 0, ny-1, z = 0, nz-1, a solid sphere of radius r
    at (ox, oy, oz), an equilibrium inlet (u = (u_in, 0, 0)) at x = 0 and a zero-gradient outlet at
    x = nx-1.  The reference's pipe/sphere channels (cpp/d3q27_bgk_channel.cpp:120-124,181-187) force
    the inlet by equilibrium the same way."""
    x, y, z = _grid3(nx, ny, nz)
    solid = (((x - ox) ** 2 + (y - oy) ** 2 + (z - oz) ** 2 <= r * r) | (y == 0) | (y == ny - 1) |
             (z == 0) | (z == nz - 1))
    cls = np.zeros((nx, ny, nz), dtype=np.int64)
    cls[x == 0] = 2
    cls[x == nx - 1] = 3
    cls[solid] = 1
    classes = [(0, 1.0, 0.0, 0.0, 0.0), (SOLID, 0.0, 0.0, 0.0, 0.0), (EQ_INLET, 1.0, u_in, 0.0, 0.0),
               (O.ZEROGRAD_XP, 1.0, 0.0, 0.0, 0.0)]
    return O.Problem("D3Q27", "BGK", (nx, ny, nz), omega=omega, classes=classes, mask=_flat(cls))


def shanchen(nx: int, ny: int, G: float, tau: float = 1.0) -> O.Problem:
    """Single-component Shan-Chen, fully periodic (the standard model; the reference's
    cpp/d2q9_shanchen.cpp is an unfinished two-component draft)."""
    return O.Problem("D2Q9", "SC", (nx, ny), omega=1.0 / tau, G=G)


# ---- start states ---------------------------------------------------------------------------

def rest_state(p: O.Problem) -> np.ndarray:
    """DENSITY = 1, U = 0 in every cell, solids included (cpp/d2q9_bgk_lid.cpp:100-107)."""
    return O.init_equilibrium(p)


def mrt_start_state(p: O.Problem) -> np.ndarray:
    """rust/examples/d3q27_mrt_lid.rs:228-287: uniform f = 1/27 in every cell, collided once towards
    meq(rho = 1, u = 0) with the relaxation rates S: f = M^-1 (m - S (m - meq)), m = M f."""
    M, Mi = O.mrt_matrices(p.mrt_basis)
    f = np.full(27, 1.0 / 27.0)
    m = M @ f
    if p.mrt_basis == "ref":
        cs2 = 1.0 / 3.0
        meq = np.zeros(27)
        meq[0] = 1.0
        meq[7] = 1.0
        meq[17] = meq[18] = meq[19] = cs2 * cs2
        meq[26] = cs2 ** 3
    else:
        _, _, _, w, _ = O.velocities("D3Q27")
        meq = M @ w
    s = np.asarray(p.s, dtype=np.float64)
    f_init = Mi @ (m - s * (m - meq))
    return np.repeat(f_init, p.n)


def channel_start_state(p: O.Problem, u_in: float, seed=None, noise: float = 0.0) -> np.ndarray:
    """Equilibrium of rho = 1, u = (u_in, 0) in fluid cells and rho = u = 0 in solid ones; config 2
    adds a seeded uniform perturbation U(-noise, noise) to u_x of the fluid (numpy PCG64)."""
    m = np.asarray(p.mask).ravel()
    flags = np.array([c[0] for c in p.classes])[m]
    solid = (flags & O.BOUNCE) != 0
    rho = np.where(solid, 0.0, 1.0)
    ux = np.where(solid, 0.0, u_in)
    if seed is not None and noise > 0:
        rng = np.random.default_rng(seed)
        ux = np.where(solid, 0.0, ux + rng.uniform(-noise, noise, ux.shape))
    uy = np.zeros_like(ux)
    u = np.concatenate([ux, uy] if p.dim == 2 else [ux, uy, np.zeros_like(ux)])
    return O.init_equilibrium(p, rho=rho, u=u)


def shanchen_start_state(p: O.Problem, rho0: float, amp: float, seed: int) -> np.ndarray:
    """rho = rho0 + U(-amp, amp) per cell (numpy PCG64 seeded), u = 0."""
    rng = np.random.default_rng(seed)
    return O.init_equilibrium(p, rho=rho0 + rng.uniform(-amp, amp, p.n))


# ---- the benchmark configurations ------------------------------------------------------------

def config_lid128():
    """D2Q9 lid cavity 128^2, lid 0.1, Re 100 with the C++ viscosity rule."""
    return cavity2d(128, 128, 0.1, omega_from_re(0.1, 128, 100.0, 0))


def config_channel(nx=1024, ny=256):
    """D2Q9 channel 1024 x 256, cylinder d = 40 at (200, 128), inlet 0.04, zero-gradient outlet,
    nu from Re 200 on the diameter."""
    nu = 0.04 * 40 / 200.0
    return channel2d(nx, ny, 0.04, 200, 128, 20, 1.0 / (3 * nu + 0.5), config_mode=True)


def config_shanchen(n=1024):
    return shanchen(n, n, -5.5, 1.0)


def config_mrt_lid(shape=(256, 256, 256)):
    """D3Q27 MRT lid cavity (Gram-Schmidt basis), lid 0.05 on the z-top face, shear rate from Re 1000
    at L = 256, every other rate 1.2."""
    sv = 1.0 / (3.0 * (0.05 * 256 / 1000.0) + 0.5)
    nx, ny, nz = shape
    return cavity3d(nx, ny, nz, 0.05, collision="MRT", s=mrt_rates(sv, 1.2), mrt_basis="gs")


def config_bgk_lid3d(shape=(256, 256, 256)):
    nx, ny, nz = shape
    return cavity3d(nx, ny, nz, 0.05, omega=omega_from_re(0.05, nx, 1000.0, 0))


def ensemble_spec(seed: int = 3):
    """Config 5: 48 D2Q9 BGK lid cavities (L uniform in {64, 128, ..., 1024}, Re uniform in [100, 1000],
    lid 0.1, the Rust examples' viscosity rule nu = u 2 L / Re) and 16 D3Q27 BGK channels (4L, L, L), L uniform in
    {64, 96, 128, 160, 192}, sphere of diameter L/4 at (2L, L/2, L/2), equilibrium inlet 0.04,
    zero-gradient outlet, nu from Re 100 on the sphere diameter.  numpy PCG64 seeded with `seed`.
    Returns (name, shape, omega) per member, in order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(48):
        L = int(rng.integers(1, 17)) * 64
        re = float(rng.uniform(100.0, 1000.0))
        out.append((f"d2q9_lid_{L}", (L, L), omega_from_re(0.1, L, re, 1)))
    for _ in range(16):
        L = int(rng.choice([64, 96, 128, 160, 192]))
        nu = 0.04 * (L / 4.0) / 100.0
        out.append((f"d3q27_channel_{L}", (4 * L, L, L), 1.0 / (3.0 * nu + 0.5)))
    return out


def ensemble_problem(name, shape, omega) -> O.Problem:
    if name.startswith("d2q9_lid"):
        return cavity2d(shape[0], shape[1], 0.1, omega)
    L = shape[1]
    return duct3d(shape[0], shape[1], shape[2], 0.04, 2.0 * L, L / 2.0, L / 2.0, L / 8.0, omega)


def cell_semantics(p: O.Problem):
    """Per-cell (flags, rho, ux, uy, uz) of a problem: what every cell does, independent of how the
    class ids are numbered."""
    m = np.zeros(p.n, dtype=np.int64) if p.mask is None else np.asarray(p.mask, dtype=np.int64).ravel()
    table = np.array([[c[0], c[1], c[2], c[3], c[4]] for c in p.classes], dtype=np.float64)
    return table[m]
