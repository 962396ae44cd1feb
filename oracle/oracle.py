"""ctypes bridge to the CPU oracle (liblbm_oracle.so).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference legs import this module, and only as the checker or the CPU baseline; the engine in
``lbm-arrayfire_b200/`` never imports it.

The oracle restates the reference's time-step loop (cpp/d2q9_bgk_lid.cpp:121-155,
cpp/d2q9_bgk_channel_packed.cpp:53-74, cpp/d3q27_bgk_lid.cpp:157-195,
rust/examples/d3q27_mrt_lid.rs:302-389) as per-cell loops in C; see lbm_oracle.h for the parity
status (unpinned against the reference itself; pinned to oracle/af_emulation.py and invariants).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liblbm_oracle.so"

BOUNCE, SET_RHO, SET_UX, SET_UY, SET_UZ, EQUILIBRIUM, ZEROGRAD_XP = 1, 2, 4, 8, 16, 32, 64
ZOUHE_VEL_XM, ZOUHE_RHO_XP = 128, 256


class OrcDesc(C.Structure):
    _fields_ = [
        ("lattice", C.c_int32),
        ("collision", C.c_int32),
        ("mrt_basis", C.c_int32),
        ("n_classes", C.c_int32),
        ("nx", C.c_int64),
        ("ny", C.c_int64),
        ("nz", C.c_int64),
        ("omega", C.c_double),
        ("s", C.c_double * 27),
        ("G", C.c_double),
        ("cls_flags", C.c_uint32 * 16),
        ("cls_rho", C.c_double * 16),
        ("cls_ux", C.c_double * 16),
        ("cls_uy", C.c_double * 16),
        ("cls_uz", C.c_double * 16),
        ("mask", C.POINTER(C.c_uint8)),
    ]


_lib = None


def build() -> Path:
    """Compile liblbm_oracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        try:
            L = C.CDLL(str(LIB_PATH))
        except OSError:
            # built for another host: rebuild in place with the local compiler
            subprocess.run(["make", "-s", "-B", "-C", str(HERE)], check=True)
            L = C.CDLL(str(LIB_PATH))
        dp = C.POINTER(C.c_double)
        fp = C.POINTER(C.c_float)
        L.orc_run_f64.argtypes = [C.POINTER(OrcDesc), dp, C.c_int64, dp, dp, C.c_int]
        L.orc_run_f32.argtypes = [C.POINTER(OrcDesc), fp, C.c_int64, fp, fp, C.c_int]
        L.orc_init_eq_f64.argtypes = [C.POINTER(OrcDesc), dp, dp, dp]
        L.orc_mrt_matrices.argtypes = [C.c_int, dp, dp]
        L.orc_sums_f64.argtypes = [C.POINTER(OrcDesc), dp, dp]
        L.orc_velocities.argtypes = [C.c_int] + [C.POINTER(C.c_int)] * 3 + [dp, C.POINTER(C.c_int)]
        _lib = L
    return _lib


class Problem:
    """Plain-Python problem description the oracle runs (mirrors the engine's descriptor fields)."""

    def __init__(self, lattice: str, collision: str, shape, omega=1.0, s=None, G=0.0,
                 mrt_basis: str = "ref", classes=None, mask=None):
        self.lattice = lattice  # "D2Q9" | "D3Q27"
        self.collision = collision  # "BGK" | "MRT" | "SC"
        nx, ny = shape[0], shape[1]
        nz = shape[2] if len(shape) > 2 else 1
        self.shape = (nx, ny, nz)
        self.omega = float(omega)
        self.s = list(s) if s is not None else [1.0] * 27
        self.G = float(G)
        self.mrt_basis = mrt_basis
        # classes: list of (flags, rho, ux, uy, uz); class 0 defaults to plain fluid
        self.classes = classes if classes is not None else [(0, 1.0, 0.0, 0.0, 0.0)]
        self.mask = mask  # uint8 array of N (column-major) or None

    @property
    def q(self) -> int:
        return 9 if self.lattice == "D2Q9" else 27

    @property
    def n(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    @property
    def dim(self) -> int:
        return 2 if self.lattice == "D2Q9" else 3

    def to_c(self):
        d = OrcDesc()
        d.lattice = 0 if self.lattice == "D2Q9" else 1
        d.collision = {"BGK": 0, "MRT": 1, "SC": 2}[self.collision]
        d.mrt_basis = 0 if self.mrt_basis == "ref" else 1
        d.n_classes = len(self.classes)
        d.nx, d.ny, d.nz = self.shape
        d.omega = self.omega
        for i in range(27):
            d.s[i] = self.s[i]
        d.G = self.G
        for k, (fl, r, ux, uy, uz) in enumerate(self.classes):
            d.cls_flags[k] = fl
            d.cls_rho[k], d.cls_ux[k], d.cls_uy[k], d.cls_uz[k] = r, ux, uy, uz
        keep = None
        if self.mask is not None:
            keep = np.ascontiguousarray(self.mask, dtype=np.uint8).ravel(order="F")
            assert keep.size == self.n
            d.mask = keep.ctypes.data_as(C.POINTER(C.c_uint8))
        return d, keep


def velocities(lattice: str):
    q = 9 if lattice == "D2Q9" else 27
    cx, cy, cz, opp = [(C.c_int * 27)() for _ in range(4)]
    w = (C.c_double * 27)()
    lib().orc_velocities(0 if lattice == "D2Q9" else 1, cx, cy, cz, w, opp)
    return (np.array(cx[:q]), np.array(cy[:q]), np.array(cz[:q]), np.array(w[:q]),
            np.array(opp[:q]))


def mrt_matrices(basis: str = "ref"):
    M = np.zeros(27 * 27)
    Mi = np.zeros(27 * 27)
    rc = lib().orc_mrt_matrices(0 if basis == "ref" else 1,
                                M.ctypes.data_as(C.POINTER(C.c_double)),
                                Mi.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError("singular MRT matrix")
    return M.reshape(27, 27), Mi.reshape(27, 27)


def init_equilibrium(p: Problem, rho=None, u=None) -> np.ndarray:
    """F = feq(rho, u) in the reference layout (flat, column-major [nx,ny,nz,Q]), FP64."""
    F = np.zeros(p.n * p.q)
    d, keep = p.to_c()
    r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64).ravel(order="F")
    uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64).ravel()
    dp = C.POINTER(C.c_double)
    lib().orc_init_eq_f64(C.byref(d), F.ctypes.data_as(dp),
                          None if r is None else r.ctypes.data_as(dp),
                          None if uu is None else uu.ctypes.data_as(dp))
    del keep
    return F


def run(p: Problem, F: np.ndarray, steps: int, dtype=np.float64, threads: int = 0):
    """Advance a copy of F by `steps`; returns (F, rho, u) in `dtype` (float64 or float32)."""
    dtype = np.dtype(dtype)
    F = np.array(F, dtype=dtype, copy=True).ravel()
    assert F.size == p.n * p.q
    rho = np.zeros(p.n, dtype=dtype)
    u = np.zeros(p.dim * p.n, dtype=dtype)
    d, keep = p.to_c()
    if dtype == np.float64:
        ptr = C.POINTER(C.c_double)
        rc = lib().orc_run_f64(C.byref(d), F.ctypes.data_as(ptr), steps, rho.ctypes.data_as(ptr),
                               u.ctypes.data_as(ptr), threads)
    elif dtype == np.float32:
        ptr = C.POINTER(C.c_float)
        rc = lib().orc_run_f32(C.byref(d), F.ctypes.data_as(ptr), steps, rho.ctypes.data_as(ptr),
                               u.ctypes.data_as(ptr), threads)
    else:
        raise TypeError(dtype)
    del keep
    if rc != 0:
        raise RuntimeError("oracle rejected the problem")
    return F, rho, u


def sums(p: Problem, F: np.ndarray) -> np.ndarray:
    out = np.zeros(4)
    d, keep = p.to_c()
    Fd = np.ascontiguousarray(F, dtype=np.float64)
    lib().orc_sums_f64(C.byref(d), Fd.ctypes.data_as(C.POINTER(C.c_double)),
                       out.ctypes.data_as(C.POINTER(C.c_double)))
    del keep
    return out


def threads_available() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
