"""The engine's set-up helpers (lbm_setup_*, relaxation rules, rates) against the oracle's independent
restatement of the reference drivers' set-up (oracle/problems.py).  Host code only: no GPU needed.

A set-up bug in the engine would otherwise show up on both sides of every parity test; here each
helper's mask and class table are compared cell by cell (what every cell does: flags and the forced
rho/u) with masks built straight from the reference's BOUND definitions, at the benchmark
configurations' sizes and at odd ones."""
import numpy as np
import pytest

from helpers import P, lb, oracle_problem, same_problem


@pytest.mark.parametrize("n", [(3, 2), (11, 9), (128, 128), (257, 130)])
def test_cavity2d_setup_matches_reference(n):
    nx, ny = n
    om = lb.omega_from_re(0.1, nx, 100.0, 0)
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (nx, ny), omega=om)
    m = lb.setup_cavity2d(d, 0.1)
    same_problem(d, m, P.cavity2d(nx, ny, 0.1, P.omega_from_re(0.1, nx, 100.0, 0)))


@pytest.mark.parametrize("config_mode", [0, 1, 2])
@pytest.mark.parametrize("geom", [(60, 24, 13, 12, 3), (1024, 256, 200, 128, 20), (97, 41, 30.5, 20.25, 7.3)])
def test_channel2d_setup_matches_reference(geom, config_mode):
    nx, ny, ox, oy, r = geom
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (nx, ny), omega=1.2)
    m = lb.setup_channel2d(d, 0.04, ox, oy, r, config_mode)
    same_problem(d, m, P.channel2d(nx, ny, 0.04, ox, oy, r, 1.2, config_mode))


@pytest.mark.parametrize("n", [(3, 3, 2), (6, 7, 8), (64, 64, 64), (40, 17, 9)])
def test_cavity3d_setup_matches_reference(n):
    d = lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, n, omega=1.1)
    m = lb.setup_cavity3d(d, 0.05)
    same_problem(d, m, P.cavity3d(*n, 0.05, omega=1.1))


@pytest.mark.parametrize("L", [64, 96])
def test_duct3d_setup_matches_reference(L):
    nu = 0.04 * (L / 4.0) / 100.0
    om = 1.0 / (3.0 * nu + 0.5)
    d = lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, (4 * L, L, L), omega=om)
    m = lb.setup_duct3d(d, 0.04, 2.0 * L, L / 2.0, L / 2.0, L / 8.0)
    same_problem(d, m, P.duct3d(4 * L, L, L, 0.04, 2.0 * L, L / 2.0, L / 2.0, L / 8.0, om))


def test_rates_and_rules_match_reference():
    assert list(lb.mrt_reference_rates()) == P.mrt_reference_rates()
    sv = 1.0 / (3.0 * (0.05 * 256 / 1000.0) + 0.5)
    assert list(lb.mrt_rates(sv, 1.2)) == P.mrt_rates(sv, 1.2)
    for rule in (0, 1):
        assert lb.omega_from_re(0.1, 128, 100.0, rule) == P.omega_from_re(0.1, 128, 100.0, rule)


@pytest.mark.parametrize("basis", [lb.MRT_REF, lb.MRT_GRAM_SCHMIDT])
def test_mrt_start_state_matches_engine_host_collision(basis):
    s = lb.mrt_reference_rates()
    d = lb.make_desc(lb.D3Q27, lb.MRT, lb.F64, (4, 4, 4), mrt_s=s, mrt_basis=basis)
    f_engine = lb.mrt_collide_host(d, np.full(27, 1.0 / 27.0), 1.0, [0.0, 0.0, 0.0])
    p = P.cavity3d(4, 4, 4, 0.1, collision="MRT", s=list(s), mrt_basis="ref" if basis == lb.MRT_REF else "gs")
    f_oracle = P.mrt_start_state(p)[::p.n]
    assert np.max(np.abs(f_engine - f_oracle)) < 1e-15


def test_benchmark_ensemble_spec_matches_the_engine_side():
    import bench

    members = bench.ensemble_members(lb, lb.F16S)
    spec = P.ensemble_spec(3)
    assert len(members) == len(spec) == 64
    for (d, _, name), (name_o, shape, omega) in zip(members, spec):
        assert name == name_o and tuple(d.shape) == tuple(shape) and d.omega == omega
    # per-cell set-up of the smallest member of each family
    for fam in ("d2q9", "d3q27"):
        k = min((i for i, s in enumerate(spec) if s[0].startswith(fam)), key=lambda i: np.prod(spec[i][1]))
        d, m, _ = members[k]
        same_problem(d, m, P.ensemble_problem(*spec[k]))


def test_benchmark_workloads_match_the_oracle_configs():
    import bench

    for wl, oracle_cfg in (("d2q9_lid_128", P.config_lid128()), ("d2q9_channel_1024x256", P.config_channel()),
                           ("d2q9_shanchen_1024", P.config_shanchen())):
        d, m = bench.WORKLOADS[wl][0](lb, lb.F32)
        same_problem(d, m, oracle_cfg)
    d, m = bench.wl_mrt256(lb, lb.F32, (32, 24, 16))
    same_problem(d, m, P.config_mrt_lid((32, 24, 16)))
    assert oracle_problem(d, m).mrt_basis == "gs"
