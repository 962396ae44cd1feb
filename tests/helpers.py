"""Shared test helpers: build the same problem for the engine (via its C-ABI set-up helpers) and
for the CPU oracle (oracle/problems.py, an independent restatement of the reference drivers' set-up),
check that both describe the same cells, and produce the reference drivers' start states."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "lbm-arrayfire_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import lbm_b200 as lb  # noqa: E402
import oracle as O  # noqa: E402
import af_emulation as E  # noqa: E402
import problems as P  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def oracle_problem(d: "lb.Desc", mask) -> O.Problem:
    coll = {lb.BGK: "BGK", lb.MRT: "MRT", lb.SHANCHEN: "SC"}[d.collision]
    return O.Problem("D2Q9" if d.lattice == lb.D2Q9 else "D3Q27", coll, (d.nx, d.ny, d.nz), omega=d.omega,
                     s=list(d.mrt_s), G=d.sc_G, mrt_basis="ref" if d.mrt_basis == lb.MRT_REF else "gs",
                     classes=lb.classes_of(d), mask=None if mask is None else np.asarray(mask).ravel())


def same_problem(d: "lb.Desc", mask, p: O.Problem) -> None:
    """The engine's descriptor + mask (from lbm_setup_*) and the oracle's independent restatement give
    every cell the same behaviour (flags, forced rho/u), the same relaxation and the same extents."""
    q = oracle_problem(d, mask)
    assert q.shape == p.shape and q.lattice == p.lattice and q.collision == p.collision
    assert q.omega == p.omega and list(q.s) == list(p.s) and q.G == p.G
    if q.collision == "MRT":
        assert q.mrt_basis == p.mrt_basis
    assert np.array_equal(P.cell_semantics(q), P.cell_semantics(p))


# ---- the reference drivers' problems (engine set-up checked against the oracle's) -----------

def cavity2d(n=128, u_lid=0.1, re=100.0, storage=lb.F32, rule=0):
    """cpp/d2q9_bgk_lid.cpp with the C++ viscosity rule (rule 0) or the Rust one (rule 1)."""
    om = lb.omega_from_re(u_lid, n, re, rule)
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (n, n), omega=om)
    m = lb.setup_cavity2d(d, u_lid)
    p = P.cavity2d(n, n, u_lid, P.omega_from_re(u_lid, n, re, rule))
    same_problem(d, m, p)
    F0 = P.rest_state(p)  # DENSITY = 1, U = 0 everywhere, solids included (:100-107)
    return d, m, F0


def channel2d(nx, ny, u_in, re, ox, oy, r, storage=lb.F32, config_mode=False, seed=None, noise=0.0):
    """cpp/d2q9_bgk_channel_packed.cpp (config_mode=False) or the config-mode channel."""
    nu = u_in * 2 * r / re
    om = 1.0 / (3 * nu + 0.5)
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (nx, ny), omega=om)
    m = lb.setup_channel2d(d, u_in, ox, oy, r, config_mode)
    p = P.channel2d(nx, ny, u_in, ox, oy, r, om, config_mode)
    same_problem(d, m, p)
    F0 = P.channel_start_state(p, u_in, seed, noise)
    return d, m, F0


def cavity3d(n=(16, 16, 16), u_lid=0.1, omega=1.3, storage=lb.F32):
    d = lb.make_desc(lb.D3Q27, lb.BGK, storage, n, omega=omega)
    m = lb.setup_cavity3d(d, u_lid)
    p = P.cavity3d(n[0], n[1], n[2], u_lid, omega=omega)
    same_problem(d, m, p)
    F0 = P.rest_state(p)
    return d, m, F0


def mrt_cavity(n=16, u_lid=0.1, storage=lb.F32, basis=lb.MRT_REF, rates=None):
    """rust/examples/d3q27_mrt_lid.rs: cube, lid on z = n-1, reference rates and start state."""
    s = lb.mrt_reference_rates() if rates is None else np.asarray(rates)
    d = lb.make_desc(lb.D3Q27, lb.MRT, storage, (n, n, n), mrt_s=s, mrt_basis=basis)
    m = lb.setup_cavity3d(d, u_lid)
    p = P.cavity3d(n, n, n, u_lid, collision="MRT", s=list(s), mrt_basis="ref" if basis == lb.MRT_REF else "gs")
    same_problem(d, m, p)
    # start state: uniform 1/27 collided once towards meq(rho=1, u=0) in every cell (:228-287)
    F0 = P.mrt_start_state(p)
    return d, m, F0


def shanchen(n=64, G=-5.5, rho0=0.693, amp=0.01, seed=2, storage=lb.F32, tau=1.0):
    d = lb.make_desc(lb.D2Q9, lb.SHANCHEN, storage, (n, n), omega=1.0 / tau, sc_G=G)
    p = P.shanchen(n, n, G, tau)
    same_problem(d, None, p)
    F0 = P.shanchen_start_state(p, rho0, amp, seed)
    return d, None, F0


def load_golden(name):
    return np.load(GOLDEN / f"{name}.npz")
