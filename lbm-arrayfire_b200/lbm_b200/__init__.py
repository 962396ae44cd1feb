"""Python binding of liblbm_b200.so (the B200 Lattice Boltzmann engine) over its C ABI.

The binding is a thin ctypes layer: every call goes through the ``extern "C"`` entry points declared
in ``include/lbm.h``; there is no Python or CPU fallback.  If the shared library is missing the
import fails with a message saying how to build it.

The objects mirror the reference drivers' state (michaltakac/lbm-arrayfire ``cpp/*.cpp``,
``rust/examples/*.rs``): a population array ``F`` in column-major ``[nx, ny(, nz), Q]`` layout,
a solid/lid/inlet mask and the scalar relaxation parameters; ``Lattice.step(n)`` replaces ``n``
iterations of the reference's ``while`` loop body (e.g. cpp/d2q9_bgk_lid.cpp:123-155).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

__all__ = [
    "LIB_PATH", "lib", "LbmError", "Desc", "CellClass", "Lattice", "Batch",
    "D2Q9", "D3Q27", "BGK", "MRT", "SHANCHEN", "F32", "F16S", "BF16S", "F64",
    "MRT_REF", "MRT_GRAM_SCHMIDT", "BOUNCE", "SET_RHO", "SET_UX", "SET_UY", "SET_UZ",
    "EQUILIBRIUM", "ZEROGRAD_XP", "ZOUHE_VEL_XM", "ZOUHE_RHO_XP", "velocities", "omega_from_re",
    "mrt_reference_rates", "mrt_rates",
    "mrt_collide_host", "setup_cavity2d", "setup_cavity3d", "setup_channel2d", "setup_duct3d",
    "mask_from_index_list", "EXPORTED_SYMBOLS", "ROUND_STOCHASTIC", "ROUND_NEAREST",
]

LIB_PATH = Path(os.environ.get("LBM_B200_LIB", Path(__file__).resolve().parent / "liblbm_b200.so"))

D2Q9, D3Q27 = 0, 1
BGK, MRT, SHANCHEN = 0, 1, 2
F32, F16S, BF16S, F64 = 0, 1, 2, 3
STORAGE_BYTES = {F32: 4, F16S: 2, BF16S: 2, F64: 8}  # bytes of one stored population
MRT_REF, MRT_GRAM_SCHMIDT = 0, 1
ARITH_DEVIATION, ARITH_ABSOLUTE = 0, 1
ROUND_STOCHASTIC, ROUND_NEAREST = 0, 1
KERNEL_AUTO, KERNEL_PLAIN, KERNEL_ROWS, KERNEL_CLUSTER = 0, 1, 2, 3
BATCH_AUTO, BATCH_TILES, BATCH_ROWS, BATCH_ROWS_PER_FAMILY = 0, 1, 2, 3
DTYPE_F32, DTYPE_F64 = 0, 1
HOST, DEVICE = 0, 1
BOUNCE, SET_RHO, SET_UX, SET_UY, SET_UZ, EQUILIBRIUM, ZEROGRAD_XP = 1, 2, 4, 8, 16, 32, 64
ZOUHE_VEL_XM, ZOUHE_RHO_XP = 128, 256  # Zou-He velocity inlet (x = 0), pressure outlet (x = nx-1); D2Q9 BGK
MAX_CLASSES = 16

ERRORS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "diverged",
          -5: "unsupported", -6: "no device", -7: "invalid state", -8: "device wait timed out"}


def _stream_handle(stream):
    """cudaStream_t handle of a torch.cuda.Stream or a raw handle; None stays None.  Torch's default
    stream (handle 0) becomes CUDA's legacy default stream (handle 1, cudaStreamLegacy), since the C
    calls read NULL as "the lattice's own stream"."""
    h = getattr(stream, "cuda_stream", stream)
    return 1 if stream is not None and h == 0 else h


class LbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)} ({code}): {msg}")
        self.code = code


class CellClass(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("reserved", C.c_uint32), ("rho", C.c_double), ("ux", C.c_double),
                ("uy", C.c_double), ("uz", C.c_double)]


class Desc(C.Structure):
    _fields_ = [
        ("lattice", C.c_int32), ("collision", C.c_int32), ("storage", C.c_int32), ("mrt_basis", C.c_int32),
        ("arithmetic", C.c_int32), ("rounding", C.c_int32),
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("omega", C.c_double), ("mrt_s", C.c_double * 27), ("sc_G", C.c_double),
        ("storage_scale", C.c_double), ("n_classes", C.c_int32), ("device", C.c_int32),
        ("classes", CellClass * MAX_CLASSES), ("mask", C.POINTER(C.c_uint8)),
    ]

    @property
    def q(self) -> int:
        return 9 if self.lattice == D2Q9 else 27

    @property
    def dim(self) -> int:
        return 2 if self.lattice == D2Q9 else 3

    @property
    def cells(self) -> int:
        return int(self.nx * self.ny * self.nz)

    @property
    def shape(self):
        return (self.nx, self.ny) if self.lattice == D2Q9 else (self.nx, self.ny, self.nz)


# name -> (restype, argtypes); the complete ABI of include/lbm.h
_P = C.c_void_p
_DP = C.POINTER(Desc)
_SIGS = {
    "lbm_abi_version": (C.c_int, []),
    "lbm_strerror": (C.c_char_p, [C.c_int]),
    "lbm_last_error": (C.c_char_p, []),
    "lbm_desc_init": (None, [_DP, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64]),
    "lbm_q": (C.c_int, [C.c_int]),
    "lbm_velocities": (C.c_int, [C.c_int, _P, _P, _P, _P, _P]),
    "lbm_create": (C.c_int, [_DP, C.POINTER(_P)]),
    "lbm_destroy": (None, [_P]),
    "lbm_set_populations": (C.c_int, [_P, _P, C.c_int, C.c_int]),
    "lbm_get_populations": (C.c_int, [_P, _P, C.c_int, C.c_int]),
    "lbm_init_equilibrium": (C.c_int, [_P, _P, _P]),
    "lbm_step": (C.c_int, [_P, C.c_int64]),
    "lbm_sync": (C.c_int, [_P]),
    "lbm_get_macros": (C.c_int, [_P, _P, _P, C.c_int, C.c_int]),
    "lbm_sums_fp64": (C.c_int, [_P, _P]),
    "lbm_residual_fp64": (C.c_int, [_P, _P]),
    "lbm_last_step_ms": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "lbm_steps_done": (C.c_int64, [_P]),
    "lbm_stream": (_P, [_P]),
    "lbm_set_stream": (C.c_int, [_P, _P]),
    "lbm_device_populations": (_P, [_P, C.POINTER(C.c_size_t)]),
    "lbm_face_get": (C.c_int, [_P, C.c_int64, C.POINTER(C.c_int32), C.c_int32, _P, C.c_int]),
    "lbm_face_set": (C.c_int, [_P, C.c_int64, C.POINTER(C.c_int32), C.c_int32, _P, C.c_int]),
    "lbm_get_desc": (C.c_int, [_P, _DP]),
    "lbm_set_block": (C.c_int, [_P, C.c_int]),
    "lbm_get_block": (C.c_int, [_P]),
    "lbm_set_kernel": (C.c_int, [_P, C.c_int]),
    "lbm_get_kernel": (C.c_int, [_P]),
    "lbm_test_stall_next_step": (C.c_int, [_P, C.c_int64, C.c_int64]),
    "lbm_test_index64": (C.c_int, [_P, C.c_int]),
    "lbm_set_cell_offset": (C.c_int, [_P, C.c_int64]),
    "lbm_step_planes": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int, _P]),
    "lbm_set_reserved_sms": (C.c_int, [_P, C.c_int]),
    "lbm_device_buffers": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "lbm_sums_fp64_noalloc": (C.c_int, [_P, C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64, C.c_double, _P, _P]),
    "lbm_batch_create": (C.c_int, [_DP, C.c_int, C.POINTER(_P)]),
    "lbm_batch_destroy": (None, [_P]),
    "lbm_batch_size": (C.c_int, [_P]),
    "lbm_batch_step": (C.c_int, [_P, C.c_int64]),
    "lbm_batch_sync": (C.c_int, [_P]),
    "lbm_batch_get_populations": (C.c_int, [_P, C.c_int, _P, C.c_int, C.c_int]),
    "lbm_batch_set_populations": (C.c_int, [_P, C.c_int, _P, C.c_int, C.c_int]),
    "lbm_batch_get_macros": (C.c_int, [_P, C.c_int, _P, _P, C.c_int, C.c_int]),
    "lbm_batch_sums_fp64": (C.c_int, [_P, C.c_int, _P]),
    "lbm_batch_set_mode": (C.c_int, [_P, C.c_int]),
    "lbm_batch_get_mode": (C.c_int, [_P]),
    "lbm_batch_cells": (C.c_int64, [_P]),
    "lbm_batch_stream": (_P, [_P]),
    "lbm_batch_tile_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
    "lbm_batch_plan": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "lbm_batch_test_stall_next_step": (C.c_int, [_P, C.c_int64, C.c_int64]),
    "lbm_setup_cavity2d": (C.c_int, [_DP, _P, C.c_double]),
    "lbm_setup_cavity3d": (C.c_int, [_DP, _P, C.c_double]),
    "lbm_setup_channel2d": (C.c_int, [_DP, _P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]),
    "lbm_setup_duct3d": (C.c_int, [_DP, _P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
    "lbm_mask_from_index_list": (C.c_int, [_P, C.c_int64, _P, C.c_int64, C.c_uint8]),
    "lbm_omega_from_re": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_int]),
    "lbm_mrt_reference_rates": (None, [_P]),
    "lbm_mrt_rates": (None, [_P, C.c_double, C.c_double]),
    "lbm_mrt_collide_host": (C.c_int, [_DP, _P, C.c_double, _P, _P]),
}
EXPORTED_SYMBOLS = tuple(_SIGS)

_lib = None


def lib():
    """Load liblbm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C lbm-arrayfire_b200` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise LbmError(rc, lib().lbm_last_error().decode())


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _torch_ptr(t):
    return C.c_void_p(t.data_ptr())


def velocities(lattice: int):
    q = 9 if lattice == D2Q9 else 27
    cx, cy, cz, opp = (np.zeros(q, np.int32) for _ in range(4))
    w = np.zeros(q)
    _check(lib().lbm_velocities(lattice, _ptr(cx), _ptr(cy), _ptr(cz), _ptr(w), _ptr(opp)))
    return cx, cy, cz, w, opp


def omega_from_re(u: float, L: float, re: float, rule: int = 0) -> float:
    return lib().lbm_omega_from_re(u, L, re, rule)


def mrt_reference_rates() -> np.ndarray:
    s = np.zeros(27)
    lib().lbm_mrt_reference_rates(_ptr(s))
    return s


def mrt_rates(sv: float, other: float) -> np.ndarray:
    s = np.zeros(27)
    lib().lbm_mrt_rates(_ptr(s), sv, other)
    return s


def make_desc(lattice: int, collision: int, storage: int, shape, *, omega: float = 1.0, mrt_s=None,
              mrt_basis: int = MRT_REF, sc_G: float = 0.0, storage_scale: float = 0.0, device: int = 0,
              arithmetic: int = ARITH_DEVIATION, rounding: int = 0) -> Desc:
    """rounding (16-bit storage): ROUND_STOCHASTIC (0, default) or ROUND_NEAREST (1)."""
    d = Desc()
    nx, ny = int(shape[0]), int(shape[1])
    nz = int(shape[2]) if len(shape) > 2 else 1
    lib().lbm_desc_init(C.byref(d), lattice, collision, storage, nx, ny, nz)
    d.arithmetic = arithmetic
    d.rounding = rounding
    d.omega = omega
    if mrt_s is not None:
        for i, v in enumerate(mrt_s):
            d.mrt_s[i] = float(v)
    d.mrt_basis = mrt_basis
    d.sc_G = sc_G
    d.storage_scale = storage_scale
    d.device = device
    return d


def set_classes(d: Desc, classes):
    """classes: list of (flags, rho, ux, uy, uz)."""
    d.n_classes = len(classes)
    for k, (fl, r, ux, uy, uz) in enumerate(classes):
        d.classes[k].flags, d.classes[k].rho = fl, r
        d.classes[k].ux, d.classes[k].uy, d.classes[k].uz = ux, uy, uz


def classes_of(d: Desc):
    return [(d.classes[k].flags, d.classes[k].rho, d.classes[k].ux, d.classes[k].uy, d.classes[k].uz)
            for k in range(d.n_classes)]


def _mask_buf(d: Desc) -> np.ndarray:
    return np.zeros(d.cells, dtype=np.uint8)


def setup_cavity2d(d: Desc, u_lid: float) -> np.ndarray:
    m = _mask_buf(d)
    _check(lib().lbm_setup_cavity2d(C.byref(d), _ptr(m), u_lid))
    return m


def setup_cavity3d(d: Desc, u_lid: float) -> np.ndarray:
    m = _mask_buf(d)
    _check(lib().lbm_setup_cavity3d(C.byref(d), _ptr(m), u_lid))
    return m


def setup_channel2d(d: Desc, u_in: float, ox: float, oy: float, r: float, config_mode: int) -> np.ndarray:
    """config_mode 0: the reference's boundaries; 1: equilibrium inlet, zero-gradient outlet; 2: Zou-He
    velocity inlet and pressure outlet."""
    m = _mask_buf(d)
    _check(lib().lbm_setup_channel2d(C.byref(d), _ptr(m), u_in, ox, oy, r, int(config_mode)))
    return m


def setup_duct3d(d: Desc, u_in: float, ox: float, oy: float, oz: float, r: float) -> np.ndarray:
    m = _mask_buf(d)
    _check(lib().lbm_setup_duct3d(C.byref(d), _ptr(m), u_in, ox, oy, oz, r))
    return m


def mask_from_index_list(n_cells: int, on, cls: int, mask=None) -> np.ndarray:
    m = np.zeros(n_cells, np.uint8) if mask is None else mask
    on = np.ascontiguousarray(on, dtype=np.int64)
    _check(lib().lbm_mask_from_index_list(_ptr(m), n_cells, _ptr(on), on.size, cls))
    return m


def mrt_collide_host(d: Desc, f_in, rho: float, u) -> np.ndarray:
    f_in = np.ascontiguousarray(f_in, dtype=np.float64)
    uu = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(27)
    _check(lib().lbm_mrt_collide_host(C.byref(d), _ptr(f_in), rho, _ptr(uu), _ptr(out)))
    return out


class Lattice:
    """One lattice on one GPU (an ``lbm_ctx``)."""

    def __init__(self, desc: Desc, mask: np.ndarray | None = None):
        self._mask = None
        if mask is not None:
            self._mask = np.ascontiguousarray(mask, dtype=np.uint8).ravel(order="F") \
                if mask.ndim > 1 else np.ascontiguousarray(mask, dtype=np.uint8)
            desc.mask = self._mask.ctypes.data_as(C.POINTER(C.c_uint8))
        self.desc = desc
        h = C.c_void_p()
        _check(lib().lbm_create(C.byref(desc), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def q(self):
        return self.desc.q

    @property
    def n(self):
        return self.desc.cells

    @property
    def dim(self):
        return self.desc.dim

    def step(self, n: int = 1):
        _check(lib().lbm_step(self._h, n))

    def sync(self):
        _check(lib().lbm_sync(self._h))

    def last_step_ms(self) -> float:
        ms = C.c_float()
        _check(lib().lbm_last_step_ms(self._h, C.byref(ms)))
        return ms.value

    @property
    def steps_done(self) -> int:
        return lib().lbm_steps_done(self._h)

    def stream(self) -> int:
        return lib().lbm_stream(self._h) or 0

    def set_stream(self, stream):
        """Run the lattice's work on `stream`: a torch.cuda.Stream, a cudaStream_t handle, or None for
        the lattice's own stream.  Torch's default stream (handle 0) is passed as CUDA's legacy
        default stream (handle 1, cudaStreamLegacy), since lbm_set_stream reads NULL as "own stream"."""
        _check(lib().lbm_set_stream(self._h, C.c_void_p(_stream_handle(stream) or 0)))

    def set_block(self, threads_x: int):
        _check(lib().lbm_set_block(self._h, threads_x))

    def block(self) -> int:
        return lib().lbm_get_block(self._h)

    def set_kernel(self, kind: int):
        """KERNEL_AUTO, KERNEL_PLAIN, KERNEL_ROWS (bulk-copy row pipeline) or KERNEL_CLUSTER (small D2Q9
        BGK lattices resident in one thread-block cluster's shared memory)."""
        _check(lib().lbm_set_kernel(self._h, kind))

    def kernel(self) -> int:
        return lib().lbm_get_kernel(self._h)

    def step_planes(self, first: int, count: int, finish: bool, stream=None, stride: int = 1):
        """One step over planes first + k * stride, k < count, of the slowest axis (lbm_step_planes),
        on `stream` (a torch.cuda.Stream or cudaStream_t handle; None: the lattice's stream)."""
        h = _stream_handle(stream)
        _check(lib().lbm_step_planes(self._h, first, count, stride, 1 if finish else 0, C.c_void_p(h or 0)))

    def set_reserved_sms(self, sms: int):
        """SMs the row pipeline's persistent grid leaves free for kernels on other streams."""
        _check(lib().lbm_set_reserved_sms(self._h, sms))

    def device_buffers(self):
        """(current, next, bytes): device pointers of both population buffers."""
        cur, nxt, nb = _P(), _P(), C.c_size_t()
        _check(lib().lbm_device_buffers(self._h, C.byref(cur), C.byref(nxt), C.byref(nb)))
        return cur.value, nxt.value, nb.value

    def set_cell_offset(self, offset: int):
        """Index of this lattice's cell 0 in the lattice it is a slab of (stochastic rounding's hash)."""
        _check(lib().lbm_set_cell_offset(self._h, offset))

    def test_stall_next_step(self, item: int = 0, wait_clocks: int = 1 << 21):
        """Test hook: the next step's row pipeline leaves work item `item` unfilled and gives its waits
        `wait_clocks` clocks; lbm_sync then reports LBM_ERR_TIMEOUT (see lbm_test_stall_next_step)."""
        _check(lib().lbm_test_stall_next_step(self._h, item, wait_clocks))

    def test_index64(self, on: bool = True):
        """Test hook: the plain step kernels and the one-pass Shan-Chen kernel index populations in 64
        bits (see lbm_test_index64)."""
        _check(lib().lbm_test_index64(self._h, int(bool(on))))

    def device_populations(self):
        nbytes = C.c_size_t()
        p = lib().lbm_device_populations(self._h, C.byref(nbytes))
        return p, nbytes.value

    def face_cells(self) -> int:
        """Cells of one plane of the slowest axis (nx*ny for D3Q27, nx for D2Q9)."""
        return self.n // (self.desc.nz if self.dim == 3 else self.desc.ny)

    def _face(self, fn, plane: int, dirs, buf):
        dirs = [int(i) for i in dirs]
        want = len(dirs) * self.face_cells() * STORAGE_BYTES[self.desc.storage]
        if hasattr(buf, "data_ptr"):
            if not buf.is_contiguous():
                raise ValueError("face buffer must be contiguous")
            got, ptr, mem = buf.numel() * buf.element_size(), _torch_ptr(buf), DEVICE if buf.is_cuda else HOST
        else:
            if not buf.flags["C_CONTIGUOUS"]:
                raise ValueError("face buffer must be contiguous")
            got, ptr, mem = buf.nbytes, _ptr(buf), HOST
        if got != want:
            raise ValueError(f"face buffer holds {got} bytes, {want} needed")
        _check(fn(self._h, plane, (C.c_int32 * len(dirs))(*dirs), len(dirs), ptr, mem))
        return buf

    def face_get(self, plane: int, dirs, out):
        """Populations of directions `dirs` on plane `plane` of the slowest axis (z for D3Q27, y for
        D2Q9) as stored words into `out` (numpy array or torch tensor of len(dirs) * face_cells()
        words of the storage type; CUDA copies are asynchronous on the lattice's stream)."""
        return self._face(lib().lbm_face_get, plane, dirs, out)

    def face_set(self, plane: int, dirs, src):
        """Inverse of face_get: write stored words into plane `plane` of the current buffer."""
        return self._face(lib().lbm_face_set, plane, dirs, src)

    def init_equilibrium(self, rho=None, u=None):
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64).ravel(order="F")
        uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64).ravel()
        _check(lib().lbm_init_equilibrium(self._h, None if r is None else _ptr(r), None if uu is None else _ptr(uu)))

    def set_populations(self, F):
        """F: host numpy (float32/float64, flat column-major N*Q) or a CUDA torch tensor."""
        if hasattr(F, "data_ptr"):
            dt = DTYPE_F32 if str(F.dtype) == "torch.float32" else DTYPE_F64
            _check(lib().lbm_set_populations(self._h, _torch_ptr(F), dt, DEVICE if F.is_cuda else HOST))
            return
        F = np.ascontiguousarray(F)
        if F.dtype not in (np.float32, np.float64):
            F = F.astype(np.float64)
        assert F.size == self.n * self.q
        _check(lib().lbm_set_populations(self._h, _ptr(F), DTYPE_F32 if F.dtype == np.float32 else DTYPE_F64, HOST))

    def get_populations(self, dtype=np.float64, out=None):
        if out is not None and hasattr(out, "data_ptr"):
            dt = DTYPE_F32 if str(out.dtype) == "torch.float32" else DTYPE_F64
            _check(lib().lbm_get_populations(self._h, _torch_ptr(out), dt, DEVICE if out.is_cuda else HOST))
            return out
        F = np.empty(self.n * self.q, dtype=dtype) if out is None else out
        _check(lib().lbm_get_populations(self._h, _ptr(F), DTYPE_F32 if F.dtype == np.float32 else DTYPE_F64, HOST))
        return F

    def macros(self, dtype=np.float64):
        """(rho[N], u[dim*N]) — the fields the last step's collision used."""
        rho = np.empty(self.n, dtype=dtype)
        u = np.empty(self.dim * self.n, dtype=dtype)
        _check(lib().lbm_get_macros(self._h, _ptr(rho), _ptr(u), DTYPE_F32 if dtype == np.float32 else DTYPE_F64,
                                    HOST))
        return rho, u

    def macros_into(self, rho, u):
        """Write the macros into host or device buffers (numpy arrays or torch tensors)."""
        def p(a):
            if a is None:
                return None, HOST, DTYPE_F64
            if hasattr(a, "data_ptr"):
                return _torch_ptr(a), DEVICE if a.is_cuda else HOST, \
                    DTYPE_F32 if str(a.dtype) == "torch.float32" else DTYPE_F64
            return _ptr(a), HOST, DTYPE_F32 if a.dtype == np.float32 else DTYPE_F64
        pr, mr, dr = p(rho)
        pu, mu, du = p(u)
        _check(lib().lbm_get_macros(self._h, pr, pu, dr if rho is not None else du, mr if rho is not None else mu))

    def sums(self) -> np.ndarray:
        out = np.zeros(4)
        _check(lib().lbm_sums_fp64(self._h, _ptr(out)))
        return out

    def residual(self) -> float:
        out = C.c_double()
        _check(lib().lbm_residual_fp64(self._h, C.byref(out)))
        return out.value


class Batch:
    """Many independent lattices advanced by one launch per step (an ``lbm_batch``)."""

    def __init__(self, descs, masks):
        self._masks = []
        arr = (Desc * len(descs))()
        for k, (d, m) in enumerate(zip(descs, masks)):
            if m is not None:
                mm = np.ascontiguousarray(m, dtype=np.uint8).ravel(order="F") if m.ndim > 1 else \
                    np.ascontiguousarray(m, dtype=np.uint8)
                self._masks.append(mm)
                d.mask = mm.ctypes.data_as(C.POINTER(C.c_uint8))
            arr[k] = d
        self.descs = list(descs)
        h = C.c_void_p()
        _check(lib().lbm_batch_create(arr, len(descs), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return lib().lbm_batch_size(self._h)

    @property
    def cells(self) -> int:
        return lib().lbm_batch_cells(self._h)

    def step(self, n: int = 1):
        _check(lib().lbm_batch_step(self._h, n))

    def sync(self):
        _check(lib().lbm_batch_sync(self._h))

    def stream(self) -> int:
        return lib().lbm_batch_stream(self._h) or 0

    def set_mode(self, mode: int):
        """BATCH_AUTO (time the candidates), BATCH_TILES (tile kernel only), BATCH_ROWS (one row-pipeline
        launch for both families) or BATCH_ROWS_PER_FAMILY (one row-pipeline launch per family)."""
        _check(lib().lbm_batch_set_mode(self._h, mode))

    def mode(self) -> int:
        return lib().lbm_batch_get_mode(self._h)

    def plan(self):
        """(kernel launches per step, D2Q9 and D3Q27 row-group copy bytes of the one-launch mode)."""
        n, g2, g3 = C.c_int(), C.c_int(), C.c_int()
        _check(lib().lbm_batch_plan(self._h, C.byref(n), C.byref(g2), C.byref(g3)))
        return n.value, g2.value, g3.value

    def test_stall_next_step(self, item: int = 0, wait_clocks: int = 1 << 21):
        """Test hook: the next step leaves row work item `item` unfilled (lbm_batch_test_stall_next_step)."""
        _check(lib().lbm_batch_test_stall_next_step(self._h, item, wait_clocks))

    def tile_info(self):
        tx = C.c_int()
        nt = C.c_int64()
        _check(lib().lbm_batch_tile_info(self._h, C.byref(tx), C.byref(nt)))
        return tx.value, nt.value

    def get_populations(self, k: int, dtype=np.float64):
        d = self.descs[k]
        F = np.empty(d.cells * d.q, dtype=dtype)
        _check(lib().lbm_batch_get_populations(self._h, k, _ptr(F), DTYPE_F32 if dtype == np.float32 else DTYPE_F64,
                                               HOST))
        return F

    def set_populations(self, k: int, F):
        F = np.ascontiguousarray(F)
        _check(lib().lbm_batch_set_populations(self._h, k, _ptr(F),
                                               DTYPE_F32 if F.dtype == np.float32 else DTYPE_F64, HOST))

    def macros(self, k: int, dtype=np.float64):
        d = self.descs[k]
        rho = np.empty(d.cells, dtype=dtype)
        u = np.empty(d.dim * d.cells, dtype=dtype)
        _check(lib().lbm_batch_get_macros(self._h, k, _ptr(rho), _ptr(u),
                                          DTYPE_F32 if dtype == np.float32 else DTYPE_F64, HOST))
        return rho, u

    def sums(self, k: int) -> np.ndarray:
        out = np.zeros(4)
        _check(lib().lbm_batch_sums_fp64(self._h, k, _ptr(out)))
        return out
