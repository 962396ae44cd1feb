"""Parity of the CUDA engine (called through its C ABI) with the CPU oracle and the golden
fixtures.  Tolerances: FP32 storage vs FP32 oracle <= 1e-5 relative L2;
F64 storage vs FP64 oracle <= 1e-12; 16-bit shifted storage vs the FP64 run <= 1e-3 on velocity."""
import numpy as np
import pytest

from helpers import (O, cavity2d, cavity3d, channel2d, lb, load_golden, mrt_cavity, oracle_problem, rel_l2,
                     shanchen)

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-5
TOL_F64 = 1e-12


def run_engine(d, m, F0, steps, storage=None):
    if storage is not None:
        d.storage = storage
    with lb.Lattice(d, m) as lat:
        lat.set_populations(np.asarray(F0, dtype=np.float64))
        lat.step(steps)
        F = lat.get_populations(np.float64)
        rho, u = lat.macros(np.float64)
    return F, rho, u


def run_oracle(d, m, F0, steps, dtype=np.float64):
    return O.run(oracle_problem(d, m), F0, steps, dtype=dtype)


@pytest.mark.parametrize("storage", [lb.F32, lb.F64])
def test_golden_fixtures(storage):
    tag = "f64" if storage == lb.F64 else "f32"
    tol = TOL_F64 if storage == lb.F64 else TOL_F32
    # D2Q9 lid 16x12
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (16, 12), omega=1 / 0.884)
    m = lb.setup_cavity2d(d, 0.1)
    F, rho, u = run_engine(d, m, np.repeat(lb.velocities(lb.D2Q9)[3], 192), 200)
    g = load_golden("d2q9_lid_16x12")
    assert rel_l2(F, g[f"F_{tag}"]) < tol
    assert rel_l2(u[:192], g[f"ux_{tag}"]) < 10 * tol
    # D2Q9 channel 60x24 (reference BCs)
    om = 1 / (3 * (0.1 * 2 * 3 / 20) + 0.5)
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (60, 24), omega=om)
    m = lb.setup_channel2d(d, 0.1, 13, 12, 3, False)
    solid = np.isin(m, [1, 4])
    F0 = O.init_equilibrium(oracle_problem(d, m), rho=np.where(solid, 0.0, 1.0),
                            u=np.concatenate([np.where(solid, 0.0, 0.1), np.zeros(m.size)]))
    F, rho, u = run_engine(d, m, F0, 100)
    g = load_golden("d2q9_channel_60x24")
    assert rel_l2(F, g[f"F_{tag}"]) < tol
    assert rel_l2(rho, g[f"rho_{tag}"]) < tol
    # D3Q27 BGK lid 8x9x10
    d, m, F0 = cavity3d(n=(8, 9, 10), u_lid=0.1, omega=1.3, storage=storage)
    F, rho, u = run_engine(d, m, F0, 40)
    assert rel_l2(F, load_golden("d3q27_bgk_lid_8x9x10")[f"F_{tag}"]) < tol
    # D3Q27 MRT lid 8^3 (Rust reference basis)
    d, m, F0 = mrt_cavity(n=8, u_lid=0.1, storage=storage)
    F, rho, u = run_engine(d, m, F0, 40)
    g = load_golden("d3q27_mrt_lid_8")
    assert rel_l2(F, g[f"F_{tag}"]) < (1e-11 if storage == lb.F64 else tol)
    assert rel_l2(u[:512], g[f"ux_{tag}"]) < (1e-10 if storage == lb.F64 else 10 * tol)


def test_cavity2d_128_10k_steps_fp32():
    """Config 1: D2Q9 lid 128^2, u_lid 0.1, Re 100 (C++ viscosity rule), 10,000 steps."""
    d, m, F0 = cavity2d(n=128, u_lid=0.1, re=100.0, storage=lb.F32)
    F, rho, u = run_engine(d, m, F0, 10000)
    Fo, ro, uo = run_oracle(d, m, F0, 10000, np.float32)
    fluid = m != 1
    n = 128 * 128
    assert rel_l2(F, Fo) < TOL_F32
    assert rel_l2(rho[fluid], ro[fluid]) < TOL_F32
    assert rel_l2(u[:n][fluid], uo[:n][fluid]) < TOL_F32
    assert rel_l2(u[n:][fluid], uo[n:][fluid]) < TOL_F32
    F64, r64, u64 = run_oracle(d, m, F0, 10000, np.float64)
    assert rel_l2(u[:n][fluid], u64[:n][fluid]) < TOL_F32


def test_cavity2d_fp64_storage_is_the_fp64_oracle():
    d, m, F0 = cavity2d(n=64, u_lid=0.1, re=100.0, storage=lb.F64)
    F, rho, u = run_engine(d, m, F0, 2000)
    Fo, ro, uo = run_oracle(d, m, F0, 2000)
    assert rel_l2(F, Fo) < TOL_F64
    assert rel_l2(u, uo) < TOL_F64


@pytest.mark.parametrize("config_mode", [False, True])
def test_channel2d(config_mode):
    if config_mode:
        # config 2 geometry: 1024x256, circle d=40 at (200,128), inlet 0.04, Re 200 on d, seeded noise
        d, m, F0 = channel2d(1024, 256, 0.04, 200.0, 200, 128, 20, config_mode=True, seed=1, noise=1e-4)
        steps = 400
    else:
        d, m, F0 = channel2d(200, 64, 0.1, 20.0, 41, 34, 6, config_mode=False)
        steps = 1000
    F, rho, u = run_engine(d, m, F0, steps)
    Fo, ro, uo = run_oracle(d, m, F0, steps, np.float32)
    fluid = ~np.isin(m, [1, 4])
    n = d.cells
    assert np.all(np.isfinite(F))
    assert rel_l2(F, Fo) < TOL_F32
    assert rel_l2(u[:n][fluid], uo[:n][fluid]) < TOL_F32
    assert rel_l2(rho[fluid], ro[fluid]) < TOL_F32


def test_cavity3d_bgk():
    d, m, F0 = cavity3d(n=(24, 20, 22), u_lid=0.1, omega=1.5)
    F, rho, u = run_engine(d, m, F0, 300)
    Fo, ro, uo = run_oracle(d, m, F0, 300, np.float32)
    assert rel_l2(F, Fo) < TOL_F32
    fluid = m != 1
    assert rel_l2(u[:d.cells][fluid], uo[:d.cells][fluid]) < TOL_F32


@pytest.mark.parametrize("basis", [lb.MRT_REF, lb.MRT_GRAM_SCHMIDT])
@pytest.mark.parametrize("storage", [lb.F32, lb.F64])
def test_mrt_cavity(basis, storage):
    n = 20
    rates = None
    if basis == lb.MRT_GRAM_SCHMIDT:
        # config 4 rates: shear from Re 1000 at lid 0.05, every other rate 1.2
        sv = 1.0 / (3 * (0.05 * 256 / 1000) + 0.5)
        rates = lb.mrt_rates(sv, 1.2)
    d, m, F0 = mrt_cavity(n=n, u_lid=0.05, storage=storage, basis=basis, rates=rates)
    F, rho, u = run_engine(d, m, F0, 300)
    Fo, ro, uo = run_oracle(d, m, F0, 300, np.float64 if storage == lb.F64 else np.float32)
    tol = 1e-11 if storage == lb.F64 else TOL_F32
    assert rel_l2(F, Fo) < tol
    fluid = m != 1
    assert rel_l2(u[:d.cells][fluid], uo[:d.cells][fluid]) < tol


def test_shanchen_periodic():
    d, m, F0 = shanchen(n=128, G=-5.5, rho0=0.693, amp=0.01, seed=2)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        s0 = lat.sums()
        lat.step(500)
        F = lat.get_populations(np.float64)
        rho, u = lat.macros()
        s1 = lat.sums()
    Fo, ro, uo = run_oracle(d, m, F0, 500, np.float32)
    assert rel_l2(F, Fo) < TOL_F32
    assert rel_l2(rho, ro) < TOL_F32
    assert rel_l2(u, uo) < 1e-4  # velocities are O(1e-4) noise here
    assert abs(s1[0] - s0[0]) / s0[0] < 1e-6
    # FP64 engine run against the FP64 oracle
    F64, r64, u64 = run_engine(d, m, F0, 500, storage=lb.F64)
    Fo64, _, _ = run_oracle(d, m, F0, 500)
    assert rel_l2(F64, Fo64) < TOL_F64


@pytest.mark.parametrize("storage,tol", [(lb.F16S, 1e-3), (lb.BF16S, 2e-2)])
def test_shifted_storage_accuracy_cavity(storage, tol):
    d, m, F0 = cavity2d(n=128, u_lid=0.1, re=100.0, storage=lb.F64)
    F64, r64, u64 = run_engine(d, m, F0, 3000)
    Fs, rs, us = run_engine(d, m, F0, 3000, storage=storage)
    fluid = m != 1
    n = d.cells
    err_u = rel_l2(np.concatenate([us[:n][fluid], us[n:][fluid]]), np.concatenate([u64[:n][fluid], u64[n:][fluid]]))
    err_rho = rel_l2(rs[fluid], r64[fluid])
    assert err_u < tol, err_u
    assert err_rho < tol, err_rho


def test_f16s_mrt_accuracy():
    sv = 1.0 / (3 * (0.05 * 32 / 100) + 0.5)
    d, m, F0 = mrt_cavity(n=32, u_lid=0.05, storage=lb.F64, basis=lb.MRT_GRAM_SCHMIDT, rates=lb.mrt_rates(sv, 1.2))
    F64, r64, u64 = run_engine(d, m, F0, 1000)
    Fs, rs, us = run_engine(d, m, F0, 1000, storage=lb.F16S)
    fluid = m != 1
    n = d.cells
    err = rel_l2(np.concatenate([us[k * n:(k + 1) * n][fluid] for k in range(3)]),
                 np.concatenate([u64[k * n:(k + 1) * n][fluid] for k in range(3)]))
    assert err < 1e-3, err
