"""C-ABI checks that need no GPU: the library loads and exports every entry point of include/lbm.h,
descriptor validation, the set-up helpers against the reference's own masks, and the factorised
MRT collision (host instantiation of the kernel's code) against the dense 27x27 form."""
import ctypes as C
import re

import numpy as np
import pytest

from helpers import E, O, ROOT, lb

HEADER = ROOT / "include" / "lbm.h"


def header_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = lb.lib()
    declared = header_functions()
    assert len(declared) >= 40
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(lb.EXPORTED_SYMBOLS) == declared
    assert L.lbm_abi_version() == 1


def test_velocity_sets_match_reference():
    cx, cy, cz, w, opp = lb.velocities(lb.D2Q9)
    assert list(cx) == list(E.D2_CX) and list(cy) == list(E.D2_CY)
    assert np.allclose(w, E._d2_weights(np.float64))
    assert list(opp[1:]) == list(E.D2_NBIDX + 1)
    cx, cy, cz, w, opp = lb.velocities(lb.D3Q27)
    assert list(cx) == list(E.D3_CX) and list(cy) == list(E.D3_CY) and list(cz) == list(E.D3_CZ)
    assert np.allclose(w, E._d3_weights(np.float64))
    assert abs(w.sum() - 1) < 1e-15
    assert list(opp[1:]) == list(E.D3_NBIDX + 1)
    for i in range(27):
        assert (cx[opp[i]], cy[opp[i]], cz[opp[i]]) == (-cx[i], -cy[i], -cz[i])


def test_cavity_masks_match_reference_bound():
    nx, ny = 11, 9
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (nx, ny))
    m = lb.setup_cavity2d(d, 0.1).reshape(ny, nx).T
    BOUND = np.ones((nx, ny))
    BOUND[1:nx - 1, 1:] = 0
    assert np.array_equal(m == 1, BOUND == 1)
    assert np.all(m[1:nx - 1, ny - 1] == 2) and (m == 2).sum() == nx - 2
    assert lb.classes_of(d)[2][2] == pytest.approx(0.1)
    d3 = lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, (6, 7, 8))
    m3 = lb.setup_cavity3d(d3, 0.05).reshape(8, 7, 6).transpose(2, 1, 0)
    B3 = E._d3_cavity_bound(6, 7, 8)
    assert np.array_equal(m3 == 1, B3 == 1)
    assert np.all(m3[1:5, 1:6, 7] == 2)


def test_channel_mask_matches_reference_bound():
    nx, ny, ox, oy, r = 60, 24, 13, 12, 3
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (nx, ny))
    m = lb.setup_channel2d(d, 0.1, ox, oy, r, False).reshape(ny, nx).T
    x = np.tile(np.arange(nx)[:, None], (1, ny))
    y = np.tile(np.arange(ny)[None, :], (nx, 1))
    B = ((x - ox) ** 2 + (y - oy) ** 2 <= r ** 2)
    B[:, 0] = True
    B[:, ny - 1] = True
    assert np.array_equal(np.isin(m, [1, 4]), B)
    assert np.all(m[0, 1:ny - 1] == 2) and np.all(m[nx - 1, 1:ny - 1] == 3)
    assert m[0, 0] == 4 and m[nx - 1, ny - 1] == 4
    fl = [c[0] for c in lb.classes_of(d)]
    assert fl[2] == lb.SET_UX | lb.SET_RHO and fl[3] == lb.SET_RHO


def test_index_list_shim_matches_where():
    nx, ny = 10, 8
    BOUND = np.ones((nx, ny))
    BOUND[1:nx - 1, 1:] = 0
    ON = E.af_where(BOUND)
    m = lb.mask_from_index_list(nx * ny, ON, 1)
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (nx, ny))
    ref = lb.setup_cavity2d(d, 0.0)
    assert np.array_equal(m == 1, ref == 1)
    with pytest.raises(lb.LbmError):
        lb.mask_from_index_list(nx * ny, [nx * ny], 1)


def test_relaxation_rules():
    assert lb.omega_from_re(0.1, 128, 100, 0) == pytest.approx(1 / (3 * 0.1 * 128 / 100 + 0.5))
    assert lb.omega_from_re(0.05, 256, 100, 1) == pytest.approx(1 / (3 * 0.05 * 2 * 256 / 100 + 0.5))
    assert np.allclose(lb.mrt_reference_rates(), E.REF_RATES)
    s = lb.mrt_rates(1.8, 1.2)
    assert s[4] == s[5] == s[6] == s[8] == s[9] == 1.8 and s[7] == 1.2 and s[0] == 1.2


@pytest.mark.parametrize("basis", [lb.MRT_REF, lb.MRT_GRAM_SCHMIDT])
def test_factorised_mrt_equals_dense(basis):
    rng = np.random.default_rng(basis + 1)
    s = rng.uniform(0.6, 1.9, 27)
    d = lb.make_desc(lb.D3Q27, lb.MRT, lb.F64, (4, 4, 4), mrt_s=s, mrt_basis=basis)
    M, Mi = O.mrt_matrices("ref" if basis == lb.MRT_REF else "gs")
    cx, cy, cz, w, _ = lb.velocities(lb.D3Q27)
    for _ in range(5):
        f = w * (1 + rng.uniform(-0.2, 0.2, 27))
        rho = rng.uniform(0.8, 1.2)
        u = rng.uniform(-0.1, 0.1, 3)
        if basis == lb.MRT_REF:
            cs2 = 1 / 3
            ux, uy, uz = u
            meq = np.zeros(27)
            meq[0], meq[1], meq[2], meq[3] = rho, rho * ux, rho * uy, rho * uz
            meq[4], meq[5], meq[6] = rho * ux * uy, rho * ux * uz, rho * uy * uz
            meq[7] = rho + rho * (ux * ux + uy * uy + uz * uz)
            meq[8], meq[9] = rho * (ux * ux - uy * uy), rho * (ux * ux - uz * uz)
            meq[10:16] = rho * cs2 * np.array([ux, ux, uy, uz, uy, uz])
            meq[17] = rho * cs2 * (cs2 + ux * ux + uy * uy)
            meq[18] = rho * cs2 * (cs2 + ux * ux + uz * uz)
            meq[19] = rho * cs2 * (cs2 + uy * uy + uz * uz)
            meq[20:23] = rho * cs2 * np.array([uy * uz, ux * uz, ux * uy])
            meq[23:26] = rho * cs2 * cs2 * np.array([ux, uy, uz])
            meq[26] = (ux * ux + uy * uy + uz * uz) + rho * cs2 ** 3
        else:
            eu = cx * u[0] + cy * u[1] + cz * u[2]
            feq = w * rho * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * (u @ u))
            meq = M @ feq
        m = M @ f
        dense = Mi @ (m - s * (m - meq))
        fact = lb.mrt_collide_host(d, f, rho, u)
        assert np.max(np.abs(fact - dense)) < 1e-14


def test_descriptor_validation_precedes_device():
    bad = []
    d = lb.make_desc(lb.D2Q9, lb.MRT, lb.F32, (8, 8))
    bad.append((d, -5))
    d = lb.make_desc(lb.D3Q27, lb.SHANCHEN, lb.F32, (8, 8, 8))
    bad.append((d, -5))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8, 2))
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (0, 8))
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8), omega=2.5)
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F16S, (8, 8), storage_scale=1000.0)
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, 7, (8, 8))
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8))
    d.n_classes = 0
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8))
    d.classes[0].flags = 0x200
    bad.append((d, -1))
    # Zou-He classes: D2Q9 BGK only, one side per class, an inlet slower than 1, an outlet denser than 0
    d = lb.make_desc(lb.D3Q27, lb.BGK, lb.F32, (8, 8, 8))
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.ZOUHE_VEL_XM, 1, 0.05, 0, 0)])
    bad.append((d, -5))
    d = lb.make_desc(lb.D2Q9, lb.SHANCHEN, lb.F32, (8, 8), sc_G=-5.5)
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.ZOUHE_RHO_XP, 1, 0, 0, 0)])
    bad.append((d, -5))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8))
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.ZOUHE_VEL_XM | lb.ZOUHE_RHO_XP, 1, 0.05, 0, 0)])
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8))
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.ZOUHE_VEL_XM, 1, 1.0, 0, 0)])
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8))
    lb.set_classes(d, [(0, 1, 0, 0, 0), (lb.ZOUHE_RHO_XP, 0.0, 0, 0, 0)])
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F32, (8, 8), arithmetic=7)
    bad.append((d, -1))
    d = lb.make_desc(lb.D2Q9, lb.BGK, lb.F16S, (8, 8), arithmetic=lb.ARITH_ABSOLUTE)
    bad.append((d, -5))
    d = lb.make_desc(lb.D3Q27, lb.MRT, lb.F32, (8, 8, 8), arithmetic=lb.ARITH_ABSOLUTE)
    bad.append((d, -5))
    for desc, code in bad:
        h = C.c_void_p()
        assert lb.lib().lbm_create(C.byref(desc), C.byref(h)) == code
        assert not h.value
        assert lb.lib().lbm_last_error()


def test_statuses_have_names():
    for code in range(0, -8, -1):
        assert lb.lib().lbm_strerror(code).decode() != "unknown status"
    assert lb.lib().lbm_strerror(-99).decode() == "unknown status"
    assert lb.lib().lbm_q(lb.D2Q9) == 9 and lb.lib().lbm_q(lb.D3Q27) == 27 and lb.lib().lbm_q(5) == 0


def test_null_handles_are_rejected():
    L = lb.lib()
    assert L.lbm_step(None, 1) == -1
    assert L.lbm_sync(None) == -1
    assert L.lbm_sums_fp64(None, None) == -1
    assert L.lbm_batch_step(None, 1) == -1
    assert L.lbm_steps_done(None) == -1
    assert L.lbm_step_planes(None, 0, 1, 1, 1, None) == -1
    assert L.lbm_set_reserved_sms(None, 2) == -1
    assert L.lbm_device_buffers(None, None, None, None) == -1
    assert L.lbm_set_cell_offset(None, 0) == -1
    L.lbm_destroy(None)
    L.lbm_batch_destroy(None)


@pytest.mark.parametrize("ext", [(1 << 22, 1 << 22, 1 << 22), (1 << 26, 1 << 26, 1 << 12),
                                 (1 << 25, 3, 1), (8193, 8192, 1), (1 << 13, 1 << 13, 2)])
def test_noalloc_rejects_extent_products_beyond_its_scratch(ext):
    # each extent alone is within LBM_NOALLOC_MAX_CELLS, the product is not (some of them wrap a
    # 64-bit product to 0 or to a small positive count): rejected before any device work
    nx, ny, nz = ext
    out = np.zeros(4)
    lattice = lb.D2Q9 if nz == 1 else lb.D3Q27
    rc = lb.lib().lbm_sums_fp64_noalloc(C.c_void_p(16), lattice, lb.F32, nx, ny, nz, 0.0, None,
                                        C.c_void_p(out.ctypes.data))
    assert rc == -1
    assert b"LBM_NOALLOC_MAX_CELLS" in lb.lib().lbm_last_error()
