"""ctypes view of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the C restatement in ``oracle/lbm_oracle.c`` of the
reference's D3Q19 shaders (simulation/shaders/lbm_collide.comp,
lbm_stream.comp, lbm_force.comp, particle_lbm.comp) and of the host
geometry in simulation/src/lbm.c.  Only the tests, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg import this module; the product
library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblbm_oracle.so")


class OrGridStruct(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("n", C.c_int64),
        ("tau", C.c_float),
        ("useRegularized", C.c_int),
        ("useMRT", C.c_int),
        ("useSmagorinsky", C.c_int),
        ("smagorinskyCs", C.c_float),
        ("periodicYZ", C.c_int),
        ("prec", C.c_int),
        ("f", C.c_void_p),
        ("f_new", C.c_void_p),
        ("vel", C.c_void_p),
        ("solid", C.c_void_p),
        ("q", C.c_void_p),
        ("force_raw", C.c_int64 * 7),
        ("force_f64", C.c_double * 6),
        ("guard_resets", C.c_int64),
    ]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER(OrGridStruct)
        f = C.c_float
        L.or_create.restype = P
        L.or_create.argtypes = [C.c_int, C.c_int, C.c_int, f, C.c_int]
        L.or_free.argtypes = [P]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_set_solid_aabb.argtypes = [P] + [f] * 6
        L.or_set_solid_sphere.argtypes = [P, f, f, f, f, C.c_int]
        L.or_add_ground_plane.argtypes = [P, f]
        L.or_set_solid_mesh.argtypes = [P, C.c_void_p, C.c_int] + [f] * 6
        L.or_projected_area.restype = f
        L.or_projected_area.argtypes = [P, C.c_int]
        L.or_initialize_flow.restype = C.c_int
        L.or_initialize_flow.argtypes = [P, f, f, f]
        L.or_step.argtypes = [P, f, f, f]
        L.or_collide.argtypes = [P, f, f, f]
        L.or_stream.argtypes = [P]
        L.or_drag_force_decomposed.argtypes = [P, C.c_void_p]
        L.or_drag_coefficient.restype = f
        L.or_drag_coefficient.argtypes = [P, f, f]
        L.or_lift_coefficient.restype = f
        L.or_lift_coefficient.argtypes = [P, f, f]
        L.or_feq_f32.restype = f
        L.or_feq_f32.argtypes = [C.c_int, f, f, f, f]
        L.or_feq_f64.restype = C.c_double
        L.or_feq_f64.argtypes = [C.c_int] + [C.c_double] * 4
        L.or_mrt_forward_f32.argtypes = [C.c_void_p, C.c_void_p]
        L.or_mrt_inverse_f32.argtypes = [C.c_void_p, C.c_void_p]
        L.or_mrt_meq_f32.argtypes = [f, f, f, f, C.c_void_p]
        L.or_weight_f32.restype = f
        L.or_weight_f32.argtypes = [C.c_int]
        L.or_hash3.restype = C.c_uint32
        L.or_hash3.argtypes = [C.c_uint32] * 3
        L.or_uniform01.restype = f
        L.or_uniform01.argtypes = [C.c_uint32] * 3
        L.or_particles_seed_inlet.argtypes = [C.c_void_p, C.c_int, C.c_uint32]
        L.or_particles_step.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_int, f, C.c_uint32]
        L.or_write_vti.restype = C.c_int
        L.or_write_vti.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int,
                                   C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class OracleGrid:
    """One oracle grid; arrays are exposed as numpy views in the
    reference's AoS layout (f[cell, 19], vel[cell, 4], solid[cell],
    q[cell, 19]) with cell = x + NX*(y + NY*z)."""

    def __init__(self, nx: int, ny: int, nz: int, viscosity: float,
                 prec: int = 4):
        self._L = lib()
        self._g = self._L.or_create(nx, ny, nz, viscosity, prec)
        if not self._g:
            raise MemoryError("or_create failed")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        self.prec = prec

    def close(self):
        if self._g:
            self._L.or_free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- public scalar fields (mirrors LBMGrid) ----
    def __getattr__(self, name):
        if name in ("tau", "useRegularized", "useMRT", "useSmagorinsky",
                    "smagorinskyCs", "periodicYZ", "guard_resets"):
            return getattr(self._g.contents, name)
        raise AttributeError(name)

    def set(self, **kw):
        for k, v in kw.items():
            setattr(self._g.contents, k, v)
        return self

    # ---- arrays ----
    def _view(self, field, count, dtype):
        addr = getattr(self._g.contents, field)
        buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(addr)
        return np.frombuffer(buf, dtype=dtype, count=count)

    @property
    def real(self):
        return np.float32 if self.prec == 4 else np.float64

    @property
    def f(self):
        return self._view("f", 19 * self.n, self.real).reshape(self.n, 19)

    @property
    def f_new(self):
        return self._view("f_new", 19 * self.n, self.real).reshape(self.n, 19)

    @property
    def vel(self):
        return self._view("vel", 4 * self.n, self.real).reshape(self.n, 4)

    @property
    def solid(self):
        return self._view("solid", self.n, np.int32)

    @property
    def q(self):
        return self._view("q", 19 * self.n, np.float32).reshape(self.n, 19)

    @property
    def force_raw(self):
        return list(self._g.contents.force_raw)

    @property
    def force_f64(self):
        return list(self._g.contents.force_f64)

    # ---- reference entry points ----
    def set_solid_aabb(self, *b):
        self._L.or_set_solid_aabb(self._g, *b)

    def set_solid_sphere(self, cx, cy, cz, r, halfway=False):
        self._L.or_set_solid_sphere(self._g, cx, cy, cz, r, int(halfway))

    def add_ground_plane(self, z):
        self._L.or_add_ground_plane(self._g, z)

    def set_solid_mesh(self, tris: np.ndarray, bbox):
        tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 12)
        self._L.or_set_solid_mesh(self._g, _ptr(tris), tris.shape[0], *bbox)

    def projected_area(self, axis=0) -> float:
        return self._L.or_projected_area(self._g, axis)

    def initialize_flow(self, ux, uy=0.0, uz=0.0) -> int:
        return self._L.or_initialize_flow(self._g, ux, uy, uz)

    def step(self, ux, uy=0.0, uz=0.0, n=1):
        for _ in range(n):
            self._L.or_step(self._g, ux, uy, uz)

    def collide(self, ux, uy=0.0, uz=0.0):
        self._L.or_collide(self._g, ux, uy, uz)

    def stream(self):
        self._L.or_stream(self._g)

    def drag_force_decomposed(self):
        out = np.zeros(6, np.float32)
        self._L.or_drag_force_decomposed(self._g, _ptr(out))
        return out

    def drag_coefficient(self, U, A) -> float:
        return self._L.or_drag_coefficient(self._g, U, A)

    def lift_coefficient(self, U, A) -> float:
        return self._L.or_lift_coefficient(self._g, U, A)

    def links(self):
        """Canonical compacted boundary-link list: (cell, dir, q) for every
        q >= 0, sorted by (cell, dir)."""
        q = self.q
        cell, d = np.nonzero(q >= 0.0)
        return (cell.astype(np.int32), d.astype(np.int32),
                q[cell, d].astype(np.float32))


def set_threads(n: int):
    lib().or_set_threads(n)


def feq32(i, rho, ux, uy, uz) -> float:
    return lib().or_feq_f32(i, rho, ux, uy, uz)


def feq64(i, rho, ux, uy, uz) -> float:
    return lib().or_feq_f64(i, rho, ux, uy, uz)


def weight32(i) -> float:
    return lib().or_weight_f32(i)


def mrt_forward(fi: np.ndarray) -> np.ndarray:
    fi = np.ascontiguousarray(fi, np.float32)
    m = np.zeros(19, np.float32)
    lib().or_mrt_forward_f32(_ptr(fi), _ptr(m))
    return m


def mrt_inverse(m: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(m, np.float32)
    fi = np.zeros(19, np.float32)
    lib().or_mrt_inverse_f32(_ptr(m), _ptr(fi))
    return fi


def mrt_meq(rho, ux, uy, uz) -> np.ndarray:
    meq = np.zeros(19, np.float32)
    lib().or_mrt_meq_f32(rho, ux, uy, uz, _ptr(meq))
    return meq


def particles_seed_inlet(n: int, seed: int) -> np.ndarray:
    p = np.zeros((n, 8), np.float32)
    lib().or_particles_seed_inlet(_ptr(p), n, seed)
    return p


def particles_step(vel4: np.ndarray, dims, p: np.ndarray, dt: float,
                   seed: int) -> None:
    vel4 = np.ascontiguousarray(vel4, np.float32)
    assert p.dtype == np.float32 and p.flags.c_contiguous
    nx, ny, nz = dims
    lib().or_particles_step(_ptr(vel4), nx, ny, nz, _ptr(p), p.shape[0], dt,
                            seed)


def uniform01(seed, idx, k) -> float:
    return lib().or_uniform01(seed, idx, k)


def write_vti(path: str, dims, vel4: np.ndarray, solid: np.ndarray) -> bool:
    nx, ny, nz = dims
    vel4 = np.ascontiguousarray(vel4, np.float32)
    solid = np.ascontiguousarray(solid, np.int32)
    return bool(lib().or_write_vti(path.encode(), nx, ny, nz, _ptr(vel4),
                                   _ptr(solid)))
