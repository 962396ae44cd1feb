"""lbm_sums_fp64_noalloc: the allocation-free FP64 conservation sums.

It exists for callers that cannot let a library call cudaMalloc/cudaFree (device memory owned by
another allocator or a pool reserved up front).  It must give the same sums as lbm_sums_fp64 (which
uses the context's scratch buffer), call after call, although every call reuses one fixed scratch
array in the library's device image.  This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from helpers import cavity2d, lb, mrt_cavity

pytestmark = pytest.mark.gpu


def sums_noalloc(lat):
    ptr, _ = lat.device_populations()
    d = lat.desc
    out = np.zeros(4)
    rc = lb.lib().lbm_sums_fp64_noalloc(C.c_void_p(ptr), d.lattice, d.storage, d.nx, d.ny, d.nz, d.storage_scale,
                                        C.c_void_p(lat.stream()), C.c_void_p(out.ctypes.data))
    return rc, out


def close(a, b):
    # FP64 sums in another summation order: the tolerance of the other FP64 sum tests
    return np.allclose(a, b, rtol=1e-12, atol=1e-12 * abs(b[0]))


@pytest.mark.parametrize("case", ["d2q9_f32", "d3q27_mrt_f16s", "d3q27_mrt_f64"])
def test_noalloc_sums_equal_lbm_sums_fp64_on_two_calls_in_a_row(case):
    if case == "d2q9_f32":
        d, m, F0 = cavity2d(n=96, u_lid=0.1, re=100.0, storage=lb.F32)
    elif case == "d3q27_mrt_f16s":
        d, m, F0 = mrt_cavity(n=24, u_lid=0.05, storage=lb.F16S, basis=lb.MRT_GRAM_SCHMIDT)
    else:
        d, m, F0 = mrt_cavity(n=16, u_lid=0.05, storage=lb.F64)
    with lb.Lattice(d, m) as lat:
        lat.set_populations(F0)
        lat.step(37)
        lat.sync()
        ref = lat.sums()
        rc1, first = sums_noalloc(lat)
        rc2, second = sums_noalloc(lat)
        assert rc1 == 0 and rc2 == 0, lb.lib().lbm_last_error()
        assert close(first, ref)
        assert close(second, ref)
        assert np.array_equal(first, second)  # same data, same fixed block assignment
        # the array keeps the last call's contents: a later call on new data must not see them
        lat.step(11)
        lat.sync()
        rc3, third = sums_noalloc(lat)
        assert rc3 == 0
        assert close(third, lat.sums())


def test_noalloc_rejects_lattices_beyond_its_scratch():
    d, m, F0 = cavity2d(n=32)
    with lb.Lattice(d, m) as lat:
        ptr, _ = lat.device_populations()
        out = np.zeros(4)
        rc = lb.lib().lbm_sums_fp64_noalloc(C.c_void_p(ptr), lb.D3Q27, lb.F32, 4096, 4096, 5, 0.0, None,
                                            C.c_void_p(out.ctypes.data))
        assert rc == -1
        assert b"LBM_NOALLOC_MAX_CELLS" in lb.lib().lbm_last_error()


def test_noalloc_reports_nan():
    d, m, F0 = cavity2d(n=40)
    with lb.Lattice(d, m) as lat:
        F = np.array(F0, dtype=np.float64)
        F[17] = np.nan
        lat.set_populations(F)
        rc, out = sums_noalloc(lat)
        assert rc == -4
