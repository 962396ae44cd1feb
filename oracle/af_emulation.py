"""Literal numpy emulation of the reference's ArrayFire array programs (small sizes only).

TEST INFRASTRUCTURE ONLY: it pins the C oracle (lbm_oracle.c) and generates the golden fixtures in
tests/golden/.  It reproduces each reference driver's index tables and its per-iteration sequence of
array expressions one by one, with ArrayFire's documented semantics restated in numpy:

* ``shift(a, s0, s1, ...)`` is circular with ``out[i] = in[i - s]``      -> ``np.roll(a, s, axis)``
* ``flat`` / ``moddims`` are column-major                               -> ``ravel/reshape(order="F")``
* ``where(a)`` / ``locate(a)`` return ascending column-major indices    -> ``np.flatnonzero(a.ravel("F"))``
* ``tile(a, n)`` repeats along dimension 0
* ``batchFunc(row, col, mul)`` is an outer product broadcast

The reference indexes populations through an f32 index array (exact below 2**24 entries); these
emulations use int64 indices and only run sizes far below that bound.
"""
from __future__ import annotations

import numpy as np


def flat(a):
    return np.asarray(a).ravel(order="F")


def moddims(a, *dims):
    return np.asarray(a).reshape(dims, order="F")


def af_shift(a, *s):
    out = a
    for ax, k in enumerate(s):
        if k:
            out = np.roll(out, k, axis=ax)
    return out


def af_where(a):
    return np.flatnonzero(flat(a))


def _div(a, b):
    """Elementwise a / b; solid cells divide by a zero density and are overwritten right after."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return a / b


def _rowsum(F2, dtype):
    """sum(F_2D, 1): accumulate the direction columns in order."""
    acc = np.zeros(F2.shape[0], dtype=dtype)
    for i in range(F2.shape[1]):
        acc = acc + F2[:, i]
    return acc


# ---------------------------------------------------------------------------------------------
# D2Q9 BGK lid-driven cavity: cpp/d2q9_bgk_lid.cpp:30-155 (window and timer omitted)
# ---------------------------------------------------------------------------------------------
D2_CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
D2_CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
D2_NBIDX = np.array([2, 3, 0, 1, 6, 7, 4, 5])


def _d2_weights(dt):
    t1, t2, t3 = dt(4.0 / 9.0), dt(1.0 / 9.0), dt(1.0 / 36.0)
    return np.array([t1, t2, t2, t2, t2, t3, t3, t3, t3], dtype=dt)


def _d2_tables(nx, ny, BOUND):
    total = nx * ny
    CI = (np.arange(8) + 1) * total                                   # :81
    NBI = CI[D2_NBIDX]                                                # :84
    main_index = moddims(np.arange(total * 9), nx, ny, 9)            # :86
    nb = main_index.copy()
    for i in range(1, 9):                                             # stream(), :18-28
        nb[:, :, i] = af_shift(main_index, D2_CX[i], D2_CY[i])[:, :, i]
    nb_index = flat(nb)                                               # :87
    ON = af_where(BOUND)                                              # :94
    TO_REFLECT = flat(np.tile(ON, 8)) + flat(np.tile(CI[None, :], (ON.size, 1)))   # :97
    REFLECTED = flat(np.tile(ON, 8)) + flat(np.tile(NBI[None, :], (ON.size, 1)))   # :98
    return nb_index, ON, TO_REFLECT, REFLECTED


def _d2_feq(w, DENSITY, UX, UY, dt):
    u_sq = flat(UX ** 2 + UY ** 2)
    eu = flat(np.outer(flat(UX), D2_CX.astype(dt)) + np.outer(flat(UY), D2_CY.astype(dt)))
    return flat(np.outer(flat(DENSITY), w)) * (dt(1.0) + dt(3.0) * eu + dt(4.5) * eu ** 2
                                               - dt(1.5) * np.tile(u_sq, 9))


def d2q9_lid(nx, ny, u_lid, omega, steps, dtype=np.float64, F0=None):
    """Returns (F, DENSITY, UX, UY) after `steps` iterations of cpp/d2q9_bgk_lid.cpp's loop."""
    dt = np.dtype(dtype).type
    w = _d2_weights(dt)
    omega = dt(omega)
    u_lid = dt(u_lid)
    BOUND = np.ones((nx, ny))
    BOUND[1:nx - 1, 1:] = 0                                           # :90-91
    nb_index, ON, TO_REFLECT, REFLECTED = _d2_tables(nx, ny, BOUND)
    DENSITY = np.full((nx, ny), 1.0, dtype=dt)                        # :100-102
    UX = np.zeros((nx, ny), dtype=dt)
    UY = np.zeros((nx, ny), dtype=dt)
    F = _d2_feq(w, DENSITY, UX, UY, dt) if F0 is None else np.array(F0, dtype=dt)   # :105-107
    total = nx * ny
    for _ in range(steps):
        Fs = F[nb_index]                                              # :124
        BOUNCEDBACK = Fs[TO_REFLECT]                                  # :126
        F2 = moddims(Fs, total, 9)                                    # :128
        rho = _rowsum(F2, dt)                                         # :131
        DENSITY = moddims(rho, nx, ny)
        UX = moddims(_div(_rowsum(F2 * D2_CX.astype(dt), dt), rho), nx, ny)   # :134-138
        UY = moddims(_div(_rowsum(F2 * D2_CY.astype(dt), dt), rho), nx, ny)
        UX[1:nx - 1, ny - 1] = u_lid                                  # :141
        UY[1:nx - 1, ny - 1] = dt(0)                                  # :142
        UXf, UYf, Df = flat(UX).copy(), flat(UY).copy(), flat(DENSITY).copy()
        UXf[ON] = 0                                                   # :144-146
        UYf[ON] = 0
        Df[ON] = 0
        UX, UY, DENSITY = moddims(UXf, nx, ny), moddims(UYf, nx, ny), moddims(Df, nx, ny)
        FEQ = _d2_feq(w, DENSITY, UX, UY, dt)                          # :149-151
        F = omega * FEQ + (dt(1) - omega) * Fs                        # :153
        F[REFLECTED] = BOUNCEDBACK                                    # :155
    return F, DENSITY, UX, UY


def d2q9_channel(nx, ny, u_max, omega, ox, oy, r, steps, dtype=np.float64):
    """cpp/d2q9_bgk_channel_packed.cpp:8-74 (correct ey); returns (F, DENSITY, UX, UY)."""
    dt = np.dtype(dtype).type
    w = _d2_weights(dt)
    omega = dt(omega)
    u_max = dt(u_max)
    x = np.tile(np.arange(nx)[:, None], (1, ny)).astype(dt)          # :21
    y = np.tile(np.arange(ny)[None, :], (nx, 1)).astype(dt)          # :22
    BOUND = ((x - ox) ** 2 + (y - oy) ** 2 <= r ** 2).astype(np.float64)   # :37
    BOUND[:, 0] = 1                                                   # :38
    BOUND[:, ny - 1] = 1                                              # :39
    nb_index, ON, TO_REFLECT, REFLECTED = _d2_tables(nx, ny, BOUND)
    total = nx * ny
    Df = np.full(total, 1.0, dtype=dt)
    UXf = np.full(total, u_max, dtype=dt)
    UYf = np.zeros(total, dtype=dt)
    UXf[ON] = 0                                                       # :46
    Df[ON] = 0                                                        # :47
    F = _d2_feq(w, moddims(Df, nx, ny), moddims(UXf, nx, ny), moddims(UYf, nx, ny), dt)  # :48-50
    DENSITY = UX = UY = None
    for _ in range(steps):
        Fs = F[nb_index]                                              # :54
        BOUNCEDBACK = Fs[TO_REFLECT]                                  # :55
        F2 = moddims(Fs, total, 9)
        rho = _rowsum(F2, dt)                                         # :58
        UX = moddims(_div(_rowsum(F2 * D2_CX.astype(dt), dt), rho), nx, ny)   # :60-62
        UY = moddims(_div(_rowsum(F2 * D2_CY.astype(dt), dt), rho), nx, ny)   # :63
        DENSITY = moddims(rho, nx, ny).copy()
        UX[0, :] = u_max                                              # :64
        UXf, UYf, Df = flat(UX).copy(), flat(UY).copy(), flat(DENSITY).copy()
        UXf[ON] = 0                                                   # :65
        UYf[ON] = 0                                                   # :66
        Df[ON] = 0                                                    # :67
        UX, UY, DENSITY = moddims(UXf, nx, ny), moddims(UYf, nx, ny), moddims(Df, nx, ny)
        DENSITY[0, :] = 1                                             # :68
        DENSITY[nx - 1, :] = 1                                        # :69
        FEQ = _d2_feq(w, DENSITY, UX, UY, dt)                          # :70-72
        F = omega * FEQ + (dt(1) - omega) * Fs                        # :73
        F[REFLECTED] = BOUNCEDBACK                                    # :74
    return F, DENSITY, UX, UY


# ---------------------------------------------------------------------------------------------
# D3Q27
# ---------------------------------------------------------------------------------------------
D3_CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
D3_CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1])
D3_CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1])
D3_NBIDX = np.array([1, 0, 3, 2, 5, 4, 9, 8, 7, 6, 13, 12, 11, 10, 17, 16, 15, 14, 25, 24, 23, 22, 21, 20,
                     19, 18])


def _d3_weights(dt):
    t1, t2, t3, t4 = dt(8.0 / 27.0), dt(2.0 / 27.0), dt(1.0 / 54.0), dt(1.0 / 216.0)
    return np.array([t1] + [t2] * 6 + [t3] * 12 + [t4] * 8, dtype=dt)


def _d3_tables(nx, ny, nz, BOUND):
    total = nx * ny * nz
    CI = (np.arange(26) + 1) * total                                  # cpp/d3q27_bgk_lid.cpp:109
    NBI = CI[D3_NBIDX]                                                # :113
    main_index = moddims(np.arange(total * 27), nx, ny, nz, 27)       # :115
    nb = main_index.copy()
    for i in range(1, 27):                                            # stream(), :20-55
        nb[:, :, :, i] = af_shift(main_index, D3_CX[i], D3_CY[i], D3_CZ[i])[:, :, :, i]
    nb_index = flat(nb)
    ON = af_where(BOUND)                                              # :123
    TO_REFLECT = flat(np.tile(ON, 26)) + flat(np.tile(CI[None, :], (ON.size, 1)))   # :126
    REFLECTED = flat(np.tile(ON, 26)) + flat(np.tile(NBI[None, :], (ON.size, 1)))   # :127
    return nb_index, ON, TO_REFLECT, REFLECTED


def _d3_cavity_bound(nx, ny, nz):
    BOUND = np.ones((nx, ny, nz))
    BOUND[1:nx - 1, 1:ny - 1, 1:] = 0                                 # cpp/d3q27_bgk_lid.cpp:119-120
    return BOUND


def _d3_moments(Fs, total, dt):
    F2 = moddims(Fs, total, 27)
    rho = _rowsum(F2, dt)
    ux = _div(_rowsum(F2 * D3_CX.astype(dt), dt), rho)
    uy = _div(_rowsum(F2 * D3_CY.astype(dt), dt), rho)
    uz = _div(_rowsum(F2 * D3_CZ.astype(dt), dt), rho)
    return F2, rho, ux, uy, uz


def _d3_lid_overwrite(nx, ny, nz, ON, rho, ux, uy, uz, u_lid, dt):
    UX, UY, UZ = moddims(ux, nx, ny, nz).copy(), moddims(uy, nx, ny, nz).copy(), moddims(uz, nx, ny, nz).copy()
    UX[1:nx - 1, 1:ny - 1, nz - 1] = u_lid                            # cpp/d3q27_bgk_lid.cpp:179-181
    UY[1:nx - 1, 1:ny - 1, nz - 1] = 0
    UZ[1:nx - 1, 1:ny - 1, nz - 1] = 0
    UXf, UYf, UZf, Df = flat(UX).copy(), flat(UY).copy(), flat(UZ).copy(), rho.copy()
    for A in (UXf, UYf, UZf, Df):                                     # :183-186
        A[ON] = 0
    return Df, UXf, UYf, UZf


def d3q27_bgk_lid(nx, ny, nz, u_lid, omega, steps, dtype=np.float64):
    """cpp/d3q27_bgk_lid.cpp:57-195; returns (F, DENSITY, UX, UY, UZ) (flat column-major)."""
    dt = np.dtype(dtype).type
    w = _d3_weights(dt)
    omega = dt(omega)
    u_lid = dt(u_lid)
    BOUND = _d3_cavity_bound(nx, ny, nz)
    nb_index, ON, TO_REFLECT, REFLECTED = _d3_tables(nx, ny, nz, BOUND)
    total = nx * ny * nz

    def feq(Df, UXf, UYf, UZf):                                       # :140-142, :189-191
        u_sq = UXf ** 2 + UYf ** 2 + UZf ** 2
        eu = flat(np.outer(UXf, D3_CX.astype(dt)) + np.outer(UYf, D3_CY.astype(dt))
                  + np.outer(UZf, D3_CZ.astype(dt)))
        return flat(np.outer(Df, w)) * (dt(1.0) + dt(3.0) * eu + dt(4.5) * eu ** 2
                                        - dt(1.5) * np.tile(u_sq, 27))

    Df = np.full(total, 1.0, dtype=dt)
    Z = np.zeros(total, dtype=dt)
    F = feq(Df, Z, Z, Z)
    UXf = UYf = UZf = Z
    for _ in range(steps):
        Fs = F[nb_index]                                              # :160
        BOUNCEDBACK = Fs[TO_REFLECT]                                  # :162
        _, rho, ux, uy, uz = _d3_moments(Fs, total, dt)               # :164-176
        Df, UXf, UYf, UZf = _d3_lid_overwrite(nx, ny, nz, ON, rho, ux, uy, uz, u_lid, dt)
        F = omega * feq(Df, UXf, UYf, UZf) + (dt(1) - omega) * Fs     # :193
        F[REFLECTED] = BOUNCEDBACK                                    # :195
    return F, Df, UXf, UYf, UZf


def mrt_reference_matrix(dt=np.float64):
    """The transformation matrix of rust/examples/d3q27_mrt_lid.rs:167-193."""
    ex, ey, ez = D3_CX.astype(dt), D3_CY.astype(dt), D3_CZ.astype(dt)
    tm = np.ones((27, 27), dtype=dt)
    rows = [ex, ey, ez, ex * ey, ex * ez, ey * ez, ex * ex + ey * ey + ez * ez, ex * ex - ey * ey,
            ex * ex - ez * ez, ex * ey * ey, ex * ez * ez, ey * ex * ex, ez * ex * ex, ey * ez * ez,
            ez * ey * ey, ex * ey * ez, ex * ex * ey * ey, ex * ex * ez * ez, ey * ey * ez * ez,
            ex * ex * ey * ez, ex * ey * ey * ez, ex * ey * ez * ez, ex * ey * ey * ez * ez,
            ex * ex * ey * ez * ez, ex * ex * ey * ey * ez, ex * ex * ey * ey * ez * ez]
    for k, r in enumerate(rows, start=1):
        tm[k, :] = r
    return tm


REF_RATES = [1.3, 1.3, 1.3, 1.3, 1.1, 1.1, 1.1, 0.9, 1.1, 1.1, 1.2, 1.2, 1.2, 1.2, 1.2, 1.2, 0.9,
             1.2, 1.2, 1.2, 1.2, 1.2, 1.2, 1.1, 1.1, 1.1, 1.1]   # rust/examples/d3q27_mrt_lid.rs:111-150


def _mrt_meq(rho_1d, ux_1d, uy_1d, uz_1d, dt):
    """rust/examples/d3q27_mrt_lid.rs:343-383, column by column."""
    c_squ = dt(1.0) / dt(3.0)
    cs_2, cs_4, cs_6 = c_squ, c_squ * c_squ, c_squ * c_squ * c_squ
    rvx, rvy, rvz = rho_1d * ux_1d, rho_1d * uy_1d, rho_1d * uz_1d
    rc2, rc4, rc6 = cs_2 * rho_1d, cs_4 * rho_1d, cs_6 * rho_1d
    vx2, vy2, vz2 = ux_1d * ux_1d, uy_1d * uy_1d, uz_1d * uz_1d
    v2 = vx2 + vy2 + vz2
    meq = np.zeros((rho_1d.size, 27), dtype=dt)
    cols = {0: rho_1d, 1: rvx, 2: rvy, 3: rvz, 4: rvx * uy_1d, 5: rvx * uz_1d, 6: rvy * uz_1d,
            7: rho_1d + rvx * ux_1d + rvy * uy_1d + rvz * uz_1d, 8: rho_1d * (vx2 - vy2),
            9: rho_1d * (vx2 - vz2), 10: rc2 * ux_1d, 11: rc2 * ux_1d, 12: rc2 * uy_1d,
            13: rc2 * uz_1d, 14: rc2 * uy_1d, 15: rc2 * uz_1d, 17: rc2 * (cs_2 + vx2 + vy2),
            18: rc2 * (cs_2 + vx2 + vz2), 19: rc2 * (cs_2 + vy2 + vz2), 20: rc2 * uy_1d * uz_1d,
            21: rc2 * ux_1d * uz_1d, 22: rc2 * ux_1d * uy_1d, 23: rc4 * ux_1d, 24: rc4 * uy_1d,
            25: rc4 * uz_1d, 26: v2 + rc6}
    for k, v in cols.items():
        meq[:, k] = v
    return meq


def d3q27_mrt_lid(n, u_lid, steps, rates=None, dtype=np.float64):
    """rust/examples/d3q27_mrt_lid.rs:62-389 for a cube of side n (lid on z = n-1); returns
    (F flat column-major [N,27], DENSITY, UX, UY, UZ)."""
    dt = np.dtype(dtype).type
    nx = ny = nz = n
    total = n ** 3
    rates = REF_RATES if rates is None else rates
    S_t = np.diag(np.array(rates, dtype=dt)).T                        # :151-155
    tm = mrt_reference_matrix(dt)
    tm_inv = np.linalg.inv(tm).astype(dt)                             # :196
    tm_t, tm_inv_t = tm.T, tm_inv.T
    BOUND = _d3_cavity_bound(nx, ny, nz)                              # :201-209
    nb_index, ON, TO_REFLECT, REFLECTED = _d3_tables(nx, ny, nz, BOUND)
    u_lid = dt(u_lid)
    # start state: uniform rho0/27 collided once towards meq(rho=1, u=0) (:220-287)
    f = np.full((total, 27), dt(1.0) / dt(27.0), dtype=dt)
    m = f @ tm_t
    ones = np.full(total, 1.0, dtype=dt)
    zeros = np.zeros(total, dtype=dt)
    meq = _mrt_meq(ones, zeros, zeros, zeros, dt)
    f = (m - (m - meq) @ S_t) @ tm_inv_t
    F = flat(f)
    Df = UXf = UYf = UZf = None
    for _ in range(steps):
        Fs = F[nb_index]                                              # :304
        BOUNCEDBACK = Fs[TO_REFLECT]                                  # :306
        F2, rho, ux, uy, uz = _d3_moments(Fs, total, dt)              # :308-320
        Df, UXf, UYf, UZf = _d3_lid_overwrite(nx, ny, nz, ON, rho, ux, uy, uz, u_lid, dt)  # :323-330
        m = F2 @ tm_t                                                 # :336
        meq = _mrt_meq(Df, UXf, UYf, UZf, dt)                         # :338-383
        f = (m - (m - meq) @ S_t) @ tm_inv_t                          # :385-387
        F = flat(f)
        F[REFLECTED] = BOUNCEDBACK                                    # :389
    return F, Df, UXf, UYf, UZf
