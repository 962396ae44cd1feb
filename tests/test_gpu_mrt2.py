"""The two-rate Gram-Schmidt MRT collision (mrt2_collide, used for 16-bit storage when the shear rows
relax at one rate and every other row at another) against the general factorised collision.

Both evaluate the same map f* = M^-1 (m - S (m - meq)); they differ only in FP32 rounding, which the
16-bit storage rounds away except where a value sits next to a rounding boundary.  The general path is
selected by moving one non-shear rate by 1e-13 (no longer two-valued), which changes the physics by
far less than either rounding."""
import numpy as np
import pytest

from helpers import O, lb, mrt_cavity, oracle_problem, rel_l2

pytestmark = pytest.mark.gpu


def _run(d, m, F0, steps, kernel):
    with lb.Lattice(d, m) as lat:
        lat.set_kernel(kernel)
        lat.set_populations(F0)
        lat.step(steps)
        lat.sync()
        return lat.get_populations(np.float64)


@pytest.mark.parametrize("storage", [lb.F16S, lb.BF16S])
@pytest.mark.parametrize("kernel", [lb.KERNEL_PLAIN, lb.KERNEL_ROWS])
def test_two_rate_equals_general_collision(storage, kernel):
    sv = 1.0 / (3 * (0.05 * 48 / 100) + 0.5)
    rates = lb.mrt_rates(sv, 1.2)
    d, m, F0 = mrt_cavity(n=48, u_lid=0.05, storage=storage, basis=lb.MRT_GRAM_SCHMIDT, rates=rates)
    w = np.repeat(lb.velocities(lb.D3Q27)[3], d.cells)
    general = np.array(rates)
    general[7] += 1e-13
    dg = lb.make_desc(lb.D3Q27, lb.MRT, storage, d.shape, mrt_s=general, mrt_basis=lb.MRT_GRAM_SCHMIDT)
    mg = lb.setup_cavity3d(dg, 0.05)
    ulp = 2.0 ** -11 if storage == lb.F16S else 2.0 ** -8
    for steps, tol in ((1, ulp), (60, 4 * ulp)):
        F2 = _run(d, m, F0, steps, kernel)
        Fg = _run(dg, mg, F0, steps, kernel)
        assert rel_l2(F2 - w, Fg - w) < tol, (steps, rel_l2(F2 - w, Fg - w))


def test_two_rate_f16s_against_fp64_oracle():
    """Config-4 rates (shear from Re 1000 at L = 256, every other rate 1.2) on a 40^3 cavity: F16S with
    the two-rate collision against the FP64 oracle (the reference's dense MRT)."""
    sv = 1.0 / (3.0 * (0.05 * 256 / 1000.0) + 0.5)
    d, m, F0 = mrt_cavity(n=40, u_lid=0.05, storage=lb.F16S, basis=lb.MRT_GRAM_SCHMIDT, rates=lb.mrt_rates(sv, 1.2))
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        lat.step(400)
        rho, u = lat.macros()
    _, ro, uo = O.run(oracle_problem(d, m), F0, 400)
    fluid = m != 1
    n = d.cells
    vel = lambda x: np.concatenate([x[k * n:(k + 1) * n][fluid] for k in range(3)])  # noqa: E731
    assert rel_l2(vel(u), vel(uo)) < 1e-3
    assert rel_l2(rho[fluid], ro[fluid]) < 1e-4
