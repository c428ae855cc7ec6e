"""ctypes binding of the C ABI in include/lattice_lbm.h.

This is the Python-side mirror of the reference's solver interface
(simulation/lib/lbm.h): the same ``LBM_*`` entry points with the same
argument meaning, plus the readback functions that replace the
reference's direct GL buffer access.  The library is the in-tree
``liblattice_lbm.so`` built by ``lattice_fluid_dynamics_b200.build``; there
is no fallback -- loading fails loudly if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblattice_lbm.so")

LBM_STORAGE_FP32 = 0
LBM_STORAGE_FP16 = 1
LBM_STORAGE_BF16 = 2
LBM_STORAGE_FP64 = 3
LBM_ARITH_EXACT = 0
LBM_ARITH_FAST = 1
STORAGE_NAMES = {"fp32": 0, "fp16": 1, "bf16": 2, "fp64": 3}


class LBMGrid(C.Structure):
    """Mirror of ``struct LBMGrid`` (public fields of simulation/lib/lbm.h:6-56)."""
    _fields_ = [
        ("sizeX", C.c_int), ("sizeY", C.c_int), ("sizeZ", C.c_int),
        ("totalCells", C.c_int),
        ("tau", C.c_float),
        ("useRegularized", C.c_int),
        ("useMRT", C.c_int),
        ("useSmagorinsky", C.c_int),
        ("smagorinskyCs", C.c_float),
        ("periodicYZ", C.c_int),
        ("storage", C.c_int),
        ("arithmetic", C.c_int),
        ("lastError", C.c_int),
        ("impl", C.c_void_p),
    ]


class LBMModel(C.Structure):
    """Mirror of ``LBMModel`` (the reference's Model, obj-file-loader/lib/model_loader.h:4-18)."""
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("faces", C.POINTER(C.c_int)),
                ("vertexCount", C.c_int), ("faceCount", C.c_int)]


class LBMCdMonitor(C.Structure):
    _fields_ = [("history", C.c_float * 100), ("historyCount", C.c_int), ("converged", C.c_int),
                ("ema", C.c_float), ("convergedMean", C.c_float),
                ("convergedRelStd", C.c_float)]


class LBMCoefficients(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("cd", "cdCorr", "cl", "cdPressure", "cdFriction")]


class LBMTunnelOptions(C.Structure):
    _fields_ = [("modelPath", C.c_char_p), ("windSpeed", C.c_float),
                ("renderDuration", C.c_int), ("reynolds", C.c_float), ("scale", C.c_float),
                ("gridX", C.c_int), ("gridY", C.c_int), ("gridZ", C.c_int),
                ("smagorinskyCs", C.c_float), ("substeps", C.c_int),
                ("latticeVelocity", C.c_float), ("vtkOutputPath", C.c_char_p),
                ("vtkInterval", C.c_int), ("logPath", C.c_char_p), ("storage", C.c_int)]


class LBMTunnelResult(C.Structure):
    _fields_ = [("frames", C.c_int), ("latticeSteps", C.c_longlong), ("cdSamples", C.c_int),
                ("cdStartFrame", C.c_int)] + \
               [(n, C.c_float) for n in ("tau", "viscosity", "reynolds", "charLength",
                                         "refArea", "blockage", "blockageFactor", "lastCd",
                                         "lastCdCorr", "lastCl", "cdEma")] + \
               [("converged", C.c_int), ("convergedMean", C.c_float), ("strouhal", C.c_float),
                ("sheddingFrequency", C.c_float), ("seconds", C.c_double),
                ("mlups", C.c_double), ("solidCells", C.c_int), ("triangles", C.c_int)]


class LBMParticle(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("x", "y", "z", "pad", "vx", "vy", "vz", "life")]


# every exported symbol with its (restype, argtypes)
_G = C.POINTER(LBMGrid)
_f = C.c_float
_vp = C.c_void_p
SIGNATURES = {
    "LBM_Create": (_G, [C.c_int, C.c_int, C.c_int, _f]),
    "LBM_CreateEx": (_G, [C.c_int, C.c_int, C.c_int, _f, C.c_int]),
    "LBM_Free": (None, [_G]),
    "LBM_SetSolidAABB": (None, [_G] + [_f] * 6),
    "LBM_InitializeFlow": (C.c_int, [_G, _f, _f, _f]),
    "LBM_Step": (None, [_G, _f, _f, _f]),
    "LBM_StepN": (None, [_G, C.c_int, _f, _f, _f]),
    "LBM_GetVelocityBuffer": (_vp, [_G]),
    "LBM_ComputeDragForce": (None, [_G, _vp, _vp, _vp]),
    "LBM_ComputeDragForceDecomposed": (None, [_G] + [_vp] * 6),
    "LBM_ComputeDragCoefficient": (_f, [_G, _f, _f]),
    "LBM_ComputeLiftCoefficient": (_f, [_G, _f, _f]),
    "LBM_SetSolidSphere": (None, [_G, _f, _f, _f, _f]),
    "LBM_SetSolidSphereHalfway": (None, [_G, _f, _f, _f, _f]),
    "LBM_AddGroundPlane": (None, [_G, _f]),
    "LBM_ComputeProjectedArea": (_f, [_G, C.c_int]),
    "LBM_SetSolidMesh": (None, [_G, _vp, C.c_int] + [_f] * 6),
    "writeVTI": (None, [_G, C.c_char_p, C.c_int]),
    "LBM_CopyVelocity": (C.c_int, [_G, _vp]),
    "LBM_CopySolid": (C.c_int, [_G, _vp]),
    "LBM_CopyPopulations": (C.c_int, [_G, _vp]),
    "LBM_CopyPostCollision": (C.c_int, [_G, _vp]),
    "LBM_CopyPopulationsF64": (C.c_int, [_G, _vp]),
    "LBM_CopyPostCollisionF64": (C.c_int, [_G, _vp]),
    "LBM_CopyQ": (C.c_int, [_G, _vp]),
    "LBM_GetBoundaryLinkCount": (C.c_longlong, [_G]),
    "LBM_CopyBoundaryLinks": (C.c_int, [_G, _vp, _vp, _vp]),
    "LBM_GetStream": (_vp, [_G]),
    "LBM_ComputeDragForceF64": (C.c_int, [_G, _vp, _vp]),
    "LBM_ComputeMassMomentum": (C.c_int, [_G, _vp]),
    "LBM_GetGuardResetCount": (C.c_longlong, [_G]),
    "LBM_MassMomentumNoAlloc": (C.c_int, [_vp, C.c_longlong, _vp, _vp]),
    "LBM_LoadPopulations": (C.c_int, [_G, _vp]),
    "LBM_InitializeFromField": (C.c_int, [_G, _vp, _vp]),
    "LBM_GetLastError": (C.c_int, [_G]),
    "LBM_GetErrorString": (C.c_char_p, [C.c_int]),
    "LBM_BytesPerUpdate": (C.c_int, [_G]),
    "LBM_SetTMAStaging": (C.c_int, [_G, C.c_int]),
    "LBM_ParticlesCreate": (_vp, [C.c_int, C.c_uint]),
    "LBM_ParticlesFree": (None, [_vp]),
    "LBM_ParticlesStep": (C.c_int, [_vp, _G, _f]),
    "LBM_ParticlesCopy": (C.c_int, [_vp, _vp]),
    "LBM_ParticlesLoad": (C.c_int, [_vp, _vp]),
    "LBM_ParticlesDevice": (_vp, [_vp]),
    "LBM_LoadOBJ": (C.c_int, [C.c_char_p, _vp]),
    "LBM_FreeModel": (None, [_vp]),
    "LBM_ModelBounds": (C.c_int, [_vp, _f, _f, _f, _f, _f, _vp]),
    "LBM_CreateTriangleBuffer": (_vp, [_vp, _f, _f, _f, _f, _f, _vp]),
    "LBM_FreeTriangles": (None, [_vp]),
    "LBM_PlaceModel": (C.c_int, [_vp, _f, _vp, _vp, _vp]),
    "LBM_ReynoldsToTau": (C.c_int, [_f, _f, _f, _vp, _vp, _vp]),
    "LBM_Strouhal": (_f, [_vp, C.c_int, C.c_int, C.c_int, _f, _f, _vp]),
    "LBM_BatchCreate": (_vp, [_vp, C.c_int]),
    "LBM_BatchFree": (None, [_vp]),
    "LBM_BatchRun": (C.c_int, [_vp, C.c_int, _vp]),
    "LBM_BatchAutotune": (C.c_int, [_vp, C.c_int]),
    "LBM_BatchGetTile": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "LBM_BatchSetTile": (C.c_int, [_vp, C.c_int, C.c_int]),
    "LBM_BatchTilesPerStep": (C.c_longlong, [_vp]),
    "LBM_BatchGetSchedule": (C.c_int, [_vp]),
    "LBM_BatchSetSchedule": (C.c_int, [_vp, C.c_int]),
    "LBM_BatchGetStream": (_vp, [_vp]),
    "LBM_NNKPad": (C.c_int, [C.c_int]),
    "LBM_NNConvForward": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, C.c_int,
                                    _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_int, _vp]),
    "LBM_NNWeightTranspose": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp]),
    "LBM_NNWgradWorkspaceBytes": (C.c_longlong, [C.c_int] * 7),
    "LBM_NNConvWeightGrad": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_int,
                                       C.c_int, _vp, C.c_int, _vp, C.c_longlong, C.c_int,
                                       C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "LBM_NNTakeError": (C.c_int, []),
    "LBM_NNSetConvPath": (C.c_int, [C.c_int]),
    "LBM_WarmNetParamCount": (C.c_longlong, []),
    "LBM_WarmNetCreate": (_vp, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint]),
    "LBM_WarmNetFree": (None, [_vp]),
    "LBM_WarmNetGetParams": (C.c_int, [_vp, _vp]),
    "LBM_WarmNetSetParams": (C.c_int, [_vp, _vp]),
    "LBM_WarmNetForward": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "LBM_WarmNetForwardDevice": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "LBM_WarmNetLossGrad": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, _vp]),
    "LBM_WarmNetLossGradDevice": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, _vp]),
    "LBM_WarmNetTrainStep": (C.c_int, [_vp, _vp, _vp, C.c_int, _f, _vp]),
    "LBM_WarmNetTrainStepDevice": (C.c_int, [_vp, _vp, _vp, C.c_int, _f, _vp]),
    "LBM_WarmNetGetStream": (_vp, [_vp]),
    "LBM_WarmNetSetOutputScaling": (C.c_int, [_vp, _vp, _vp]),
    "LBM_WarmNetSetGradClip": (C.c_int, [_vp, _f]),
    "LBM_WarmNetGridFeatures": (C.c_int, [_G, C.c_int, _f, _f, _vp]),
    "LBM_WarmNetGridTargets": (C.c_int, [_G, C.c_int, _f, _vp]),
    "LBM_InitializeFromWarmNet": (C.c_int, [_G, _vp, _f, _f, C.c_int]),
    "LBM_CdMonitorInit": (None, [_vp]),
    "LBM_CdMonitorAdd": (C.c_int, [_vp, _f, _f]),
    "LBM_TunnelCoefficients": (None, [_f, _f, _f, _f, _f, _f, _vp]),
    "LBM_TunnelCdStartFrame": (C.c_int, [C.c_int, _f, C.c_int, C.c_int]),
    "LBM_TunnelRampFactor": (_f, [C.c_int]),
    "LBM_TunnelDefaults": (None, [_vp]),
    "LBM_TunnelRun": (C.c_int, [_vp, _vp]),
    "LBM_SuperResCreate": (_vp, [C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p]),
    "LBM_SuperResCreateFromArrays": (_vp, [C.c_int, C.c_int, C.c_int, _vp, C.c_longlong, _vp,
                                           _vp]),
    "LBM_SuperResFree": (None, [_vp]),
    "LBM_SuperResUpscale": (C.c_int, [_vp, _vp, _vp]),
    "LBM_SuperResGetFineVelocity": (_vp, [_vp]),
    "LBM_SuperResGetFineSize": (None, [_vp, _vp, _vp, _vp]),
    "LBM_SuperResCopyFine": (C.c_int, [_vp, _vp]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the solver library (no fallback: raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with "
                "`python -m lattice_fluid_dynamics_b200.build`")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class Grid:
    """One solver grid.  Method names follow the reference's C API."""

    def __init__(self, nx: int, ny: int, nz: int, viscosity: float,
                 storage: int | str = LBM_STORAGE_FP32):
        self._L = load()
        if isinstance(storage, str):
            storage = STORAGE_NAMES[storage]
        self._g = self._L.LBM_CreateEx(nx, ny, nz, viscosity, storage)
        if not self._g:
            raise RuntimeError(f"LBM_CreateEx({nx},{ny},{nz}) failed")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        self.storage = storage

    # -- lifetime --
    def close(self):
        if getattr(self, "_g", None):
            self._L.LBM_Free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- public struct fields --
    @property
    def s(self) -> LBMGrid:
        return self._g.contents

    def set(self, **kw):
        for k, v in kw.items():
            setattr(self._g.contents, k, v)
        return self

    @property
    def tau(self) -> float:
        return self.s.tau

    @property
    def handle(self):
        return self._g

    def check(self):
        err = self._L.LBM_GetLastError(self._g)
        if err != 0:
            raise RuntimeError("LBM error: " + self._L.LBM_GetErrorString(err).decode())

    # -- reference API --
    def set_solid_aabb(self, minX, minY, minZ, maxX, maxY, maxZ):
        self._L.LBM_SetSolidAABB(self._g, minX, minY, minZ, maxX, maxY, maxZ)
        self.check()

    def set_solid_sphere(self, cx, cy, cz, r, halfway=False):
        fn = self._L.LBM_SetSolidSphereHalfway if halfway else self._L.LBM_SetSolidSphere
        fn(self._g, cx, cy, cz, r)
        self.check()

    def add_ground_plane(self, z):
        self._L.LBM_AddGroundPlane(self._g, z)
        self.check()

    def set_solid_mesh(self, tris: np.ndarray, bbox):
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 12)
        self._L.LBM_SetSolidMesh(self._g, _p(tris), tris.shape[0], *bbox)
        self.check()

    def projected_area(self, axis=0) -> float:
        return self._L.LBM_ComputeProjectedArea(self._g, axis)

    def initialize_flow(self, ux, uy=0.0, uz=0.0):
        if self._L.LBM_InitializeFlow(self._g, ux, uy, uz) != 1:
            self.check()
            raise RuntimeError("LBM_InitializeFlow failed")

    def initialize_from_field(self, rho: np.ndarray, u: np.ndarray):
        rho = np.ascontiguousarray(rho, np.float32).reshape(-1)
        u = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
        if self._L.LBM_InitializeFromField(self._g, _p(rho), _p(u)) != 1:
            self.check()
            raise RuntimeError("LBM_InitializeFromField failed")

    def step(self, ux, uy=0.0, uz=0.0, n: int = 1):
        if n == 1:
            self._L.LBM_Step(self._g, ux, uy, uz)
        else:
            self._L.LBM_StepN(self._g, n, ux, uy, uz)

    def step_loop(self, ux, uy=0.0, uz=0.0, n: int = 1):
        for _ in range(n):
            self._L.LBM_Step(self._g, ux, uy, uz)

    def drag_force_decomposed(self) -> np.ndarray:
        if getattr(self, "_fout", None) is None:  # one output block per grid
            self._fout = np.zeros(6, np.float32)
            base = self._fout.ctypes.data
            self._fptr = [base + 4 * k for k in range(6)]
        self._L.LBM_ComputeDragForceDecomposed(self._g, *self._fptr)
        self.check()
        return self._fout.copy()

    def drag_force_f64(self):
        out = np.zeros(6, np.float64)
        raw = np.zeros(7, np.int64)
        if not self._L.LBM_ComputeDragForceF64(self._g, _p(out), _p(raw)):
            self.check()
        return out, raw

    def drag_coefficient(self, U, A) -> float:
        return self._L.LBM_ComputeDragCoefficient(self._g, U, A)

    def lift_coefficient(self, U, A) -> float:
        return self._L.LBM_ComputeLiftCoefficient(self._g, U, A)

    def velocity_device_ptr(self) -> int:
        return self._L.LBM_GetVelocityBuffer(self._g)

    def stream_ptr(self) -> int:
        return self._L.LBM_GetStream(self._g)

    def write_vti(self, path: str, step: int):
        self._L.writeVTI(self._g, path.encode(), step)

    # -- readbacks --
    def velocity(self) -> np.ndarray:
        out = np.empty((self.n, 4), np.float32)
        assert self._L.LBM_CopyVelocity(self._g, _p(out)) == 1
        return out

    def solid(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        assert self._L.LBM_CopySolid(self._g, _p(out)) == 1
        return out

    def populations(self) -> np.ndarray:
        out = np.empty((self.n, 19), np.float32)
        assert self._L.LBM_CopyPopulations(self._g, _p(out)) == 1
        return out

    def post_collision(self) -> np.ndarray:
        out = np.empty((self.n, 19), np.float32)
        assert self._L.LBM_CopyPostCollision(self._g, _p(out)) == 1
        return out

    def populations_f64(self) -> np.ndarray:
        out = np.empty((self.n, 19), np.float64)
        assert self._L.LBM_CopyPopulationsF64(self._g, _p(out)) == 1
        return out

    def post_collision_f64(self) -> np.ndarray:
        out = np.empty((self.n, 19), np.float64)
        assert self._L.LBM_CopyPostCollisionF64(self._g, _p(out)) == 1
        return out

    def q(self) -> np.ndarray:
        out = np.empty((self.n, 19), np.float32)
        assert self._L.LBM_CopyQ(self._g, _p(out)) == 1
        return out

    def links(self):
        nl = self._L.LBM_GetBoundaryLinkCount(self._g)
        cell = np.empty(nl, np.int32)
        d = np.empty(nl, np.int32)
        q = np.empty(nl, np.float32)
        assert self._L.LBM_CopyBoundaryLinks(self._g, _p(cell), _p(d), _p(q)) == 1
        return cell, d, q

    def load_populations(self, f: np.ndarray):
        f = np.ascontiguousarray(f, np.float32).reshape(self.n, 19)
        assert self._L.LBM_LoadPopulations(self._g, _p(f)) == 1

    def mass_momentum(self) -> np.ndarray:
        out = np.zeros(4, np.float64)
        assert self._L.LBM_ComputeMassMomentum(self._g, _p(out)) == 1
        return out

    def guard_resets(self) -> int:
        return int(self._L.LBM_GetGuardResetCount(self._g))

    def bytes_per_update(self) -> int:
        return int(self._L.LBM_BytesPerUpdate(self._g))

    def set_tma_staging(self, enable: bool) -> bool:
        """Turn the TMA-staged step kernel on or off; returns whether it is on."""
        return bool(self._L.LBM_SetTMAStaging(self._g, 1 if enable else 0))


class Particles:
    def __init__(self, n: int, seed: int = 0):
        self._L = load()
        self._p = self._L.LBM_ParticlesCreate(n, seed)
        if not self._p:
            raise RuntimeError("LBM_ParticlesCreate failed")
        self.n = n

    def close(self):
        if getattr(self, "_p", None):
            self._L.LBM_ParticlesFree(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, grid: Grid, dt: float):
        assert self._L.LBM_ParticlesStep(self._p, grid.handle, dt) == 1

    def get(self) -> np.ndarray:
        out = np.empty((self.n, 8), np.float32)
        assert self._L.LBM_ParticlesCopy(self._p, _p(out)) == 1
        return out

    def set(self, arr: np.ndarray):
        arr = np.ascontiguousarray(arr, np.float32).reshape(self.n, 8)
        assert self._L.LBM_ParticlesLoad(self._p, _p(arr)) == 1


class Model:
    """An OBJ model loaded by LBM_LoadOBJ (reference loadOBJ semantics)."""

    def __init__(self, path: str):
        self._L = load()
        self._m = LBMModel()
        if self._L.LBM_LoadOBJ(os.fsencode(path), C.byref(self._m)) != 1:
            raise OSError(f"LBM_LoadOBJ could not open {path}")

    def close(self):
        if getattr(self, "_m", None) is not None:
            self._L.LBM_FreeModel(C.byref(self._m))
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def vertex_count(self) -> int:
        return self._m.vertexCount

    @property
    def face_count(self) -> int:
        return self._m.faceCount

    def vertices(self) -> np.ndarray:
        n = self._m.vertexCount
        if n == 0:
            return np.zeros((0, 3), np.float32)
        return np.ctypeslib.as_array(self._m.vertices, (n, 3)).copy()

    def faces(self) -> np.ndarray:
        n = self._m.faceCount
        if n == 0:
            return np.zeros((0, 3), np.int32)
        return np.ctypeslib.as_array(self._m.faces, (n, 3)).copy()

    def place(self, scale: float = 0.0):
        """(scale, (ox, oy, oz), rotationY) as the reference's main.c places a model."""
        s = C.c_float()
        off = (C.c_float * 3)()
        rot = C.c_float()
        if self._L.LBM_PlaceModel(C.byref(self._m), scale, C.byref(s), off, C.byref(rot)) != 1:
            raise ValueError("LBM_PlaceModel: empty model")
        return s.value, (off[0], off[1], off[2]), rot.value

    def bounds(self, scale, offset, rotation_y) -> np.ndarray:
        out = np.empty(9, np.float32)
        self._L.LBM_ModelBounds(C.byref(self._m), scale, *offset, rotation_y, _p(out))
        return out

    def triangles(self, scale, offset, rotation_y) -> np.ndarray:
        """(n, 12) float32 triangle buffer for LBM_SetSolidMesh."""
        cnt = C.c_int()
        ptr = self._L.LBM_CreateTriangleBuffer(C.byref(self._m), scale, *offset, rotation_y,
                                               C.byref(cnt))
        if not ptr:
            return np.zeros((0, 12), np.float32)
        try:
            arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)),
                                        (cnt.value, 12)).copy()
        finally:
            self._L.LBM_FreeTriangles(ptr)
        return arr


def reynolds_to_tau(lattice_velocity: float, char_length: float, reynolds: float):
    """(tau, viscosity, effective_reynolds, clamped) by the reference's rule."""
    L = load()
    t, nu, re = C.c_float(), C.c_float(), C.c_float()
    rc = L.LBM_ReynoldsToTau(lattice_velocity, char_length, reynolds, C.byref(t),
                             C.byref(nu), C.byref(re))
    if rc == 0:
        raise ValueError("LBM_ReynoldsToTau: bad arguments")
    return t.value, nu.value, re.value, rc == 2


def strouhal(cl_series, lbm_substeps: int, char_length: float, lattice_velocity: float,
             sample_interval: int = 20):
    """(St, peak frequency) of a Cl series, the reference's compute_strouhal."""
    L = load()
    cl = np.ascontiguousarray(cl_series, np.float32)
    f = C.c_float()
    st = L.LBM_Strouhal(_p(cl), len(cl), lbm_substeps, sample_interval, char_length,
                        lattice_velocity, C.byref(f))
    return st, f.value


class CdMonitor:
    """The reference driver's Cd EMA / convergence monitor (LBM_CdMonitor*)."""

    def __init__(self):
        self._L = load()
        self.m = LBMCdMonitor()
        self._L.LBM_CdMonitorInit(C.byref(self.m))

    def add(self, cd: float, cd_corr: float) -> bool:
        return bool(self._L.LBM_CdMonitorAdd(C.byref(self.m), cd, cd_corr))


def tunnel_coefficients(fx, fy, px, U, ref_area, blockage_factor) -> LBMCoefficients:
    out = LBMCoefficients()
    load().LBM_TunnelCoefficients(fx, fy, px, U, ref_area, blockage_factor, C.byref(out))
    return out


def tunnel_defaults() -> LBMTunnelOptions:
    o = LBMTunnelOptions()
    load().LBM_TunnelDefaults(C.byref(o))
    return o


def tunnel_run(**kw) -> LBMTunnelResult:
    """Run the headless wind-tunnel loop (LBM_TunnelRun); keyword arguments
    set LBMTunnelOptions fields (strings are encoded)."""
    o = tunnel_defaults()
    keep = []
    for k, v in kw.items():
        if isinstance(v, str):
            v = os.fsencode(v)
            keep.append(v)
        setattr(o, k, v)
    r = LBMTunnelResult()
    rc = load().LBM_TunnelRun(C.byref(o), C.byref(r))
    if rc != 0:
        raise RuntimeError(f"LBM_TunnelRun failed: {load().LBM_GetErrorString(rc).decode()}")
    return r


class Batch:
    """Grids advanced together, one launch per step (LBM_Batch*)."""

    def __init__(self, grids):
        self._L = load()
        self.grids = list(grids)
        arr = (C.c_void_p * len(self.grids))(*[C.cast(g._g, C.c_void_p) for g in self.grids])
        self._b = self._L.LBM_BatchCreate(arr, len(self.grids))
        if not self._b:
            raise RuntimeError("LBM_BatchCreate failed (uninitialised grid, mixed storage, "
                               "fast arithmetic or a repeated grid)")

    def close(self):
        if getattr(self, "_b", None):
            self._L.LBM_BatchFree(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n: int, inlets):
        inl = np.ascontiguousarray(inlets, np.float32).reshape(len(self.grids), 3)
        rc = self._L.LBM_BatchRun(self._b, n, _p(inl))
        if rc != 0:
            raise RuntimeError(f"LBM_BatchRun: {self._L.LBM_GetErrorString(rc).decode()}")

    def autotune(self, trial_launches: int = 10):
        rc = self._L.LBM_BatchAutotune(self._b, trial_launches)
        if rc != 0:
            raise RuntimeError(f"LBM_BatchAutotune: {self._L.LBM_GetErrorString(rc).decode()}")

    def tile(self, i: int):
        tx, ty = C.c_int(), C.c_int()
        assert self._L.LBM_BatchGetTile(self._b, i, C.byref(tx), C.byref(ty)) == 0
        return tx.value, ty.value

    def set_tile(self, i: int, tile_x: int):
        if self._L.LBM_BatchSetTile(self._b, i, tile_x) != 0:
            raise ValueError(f"tile width {tile_x}")

    @property
    def schedule(self) -> str:
        return ("fused", "graph")[self._L.LBM_BatchGetSchedule(self._b)]

    def set_schedule(self, name: str):
        if self._L.LBM_BatchSetSchedule(self._b, {"fused": 0, "graph": 1}[name]) != 0:
            raise ValueError(name)

    @property
    def tiles_per_step(self) -> int:
        return int(self._L.LBM_BatchTilesPerStep(self._b))

    @property
    def stream(self) -> int:
        return self._L.LBM_BatchGetStream(self._b) or 0


class WarmNet:
    """The warm-start network (LBM_WarmNet*); arrays are numpy float32."""

    def __init__(self, nx: int, ny: int, nz: int, max_batch: int = 1, seed: int = 0):
        self._L = load()
        self._n = self._L.LBM_WarmNetCreate(nx, ny, nz, max_batch, seed)
        if not self._n:
            raise RuntimeError("LBM_WarmNetCreate failed")
        self.dims = (nz, ny, nx)
        self.vox = nx * ny * nz
        self.max_batch = max_batch

    def close(self):
        if getattr(self, "_n", None):
            self._L.LBM_WarmNetFree(self._n)
            self._n = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._n

    @staticmethod
    def param_count() -> int:
        return int(load().LBM_WarmNetParamCount())

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {self._L.LBM_GetErrorString(rc).decode()}")

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        self._check(self._L.LBM_WarmNetGetParams(self._n, _p(out)), "LBM_WarmNetGetParams")
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.param_count()
        self._check(self._L.LBM_WarmNetSetParams(self._n, _p(p)), "LBM_WarmNetSetParams")

    def forward(self, features: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(features, np.float32)
        b = f.size // (3 * self.vox)
        out = np.empty((b, self.vox, 4), np.float32)
        self._check(self._L.LBM_WarmNetForward(self._n, _p(f), b, _p(out)), "forward")
        return out

    def loss_grad(self, features, target, want_grad=True):
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        b = f.size // (3 * self.vox)
        loss = C.c_double()
        g = np.empty(self.param_count(), np.float32) if want_grad else None
        self._check(self._L.LBM_WarmNetLossGrad(self._n, _p(f), _p(t), b, C.byref(loss),
                                                None if g is None else _p(g)), "loss_grad")
        return loss.value, g

    def train_step(self, features, target, lr: float) -> float:
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        b = f.size // (3 * self.vox)
        loss = C.c_double()
        self._check(self._L.LBM_WarmNetTrainStep(self._n, _p(f), _p(t), b, lr, C.byref(loss)),
                    "train_step")
        return loss.value

    def set_output_scaling(self, scale, shift):
        sc = np.ascontiguousarray(scale, np.float32)
        sh = np.ascontiguousarray(shift, np.float32)
        self._check(self._L.LBM_WarmNetSetOutputScaling(self._n, _p(sc), _p(sh)),
                    "LBM_WarmNetSetOutputScaling")

    def set_grad_clip(self, max_norm: float):
        self._check(self._L.LBM_WarmNetSetGradClip(self._n, max_norm), "LBM_WarmNetSetGradClip")

    def train_step_device(self, feat_ptr: int, target_ptr: int, batch: int, lr: float) -> float:
        loss = C.c_double()
        self._check(self._L.LBM_WarmNetTrainStepDevice(self._n, feat_ptr, target_ptr, batch, lr,
                                                       C.byref(loss)), "train_step_device")
        return loss.value


class SuperRes:
    """The velocity-field upscaler (LBM_SuperRes*): coarse vec4 field ->
    fine field at twice the resolution, through the tensor-core MLP."""

    def __init__(self, cx: int, cy: int, cz: int, weights=None, mean=None, std=None,
                 weights_path: str | None = None, norm_path: str | None = None):
        self._L = load()
        self.coarse = (cx, cy, cz)
        if weights_path is not None:
            self._h = self._L.LBM_SuperResCreate(
                cx, cy, cz, weights_path.encode(),
                norm_path.encode() if norm_path is not None else None)
        else:
            w = np.ascontiguousarray(weights, np.float32)
            m = np.ascontiguousarray(mean if mean is not None else np.zeros(4), np.float32)
            sd = np.ascontiguousarray(std if std is not None else np.ones(4), np.float32)
            self._h = self._L.LBM_SuperResCreateFromArrays(cx, cy, cz, _p(w), w.size, _p(m),
                                                          _p(sd))
        if not self._h:
            raise RuntimeError("LBM_SuperResCreate failed")

    def close(self):
        if getattr(self, "_h", None):
            self._L.LBM_SuperResFree(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def fine_size(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._L.LBM_SuperResGetFineSize(self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def upscale(self, coarse_device_ptr: int, stream: int = 0):
        rc = self._L.LBM_SuperResUpscale(self._h, coarse_device_ptr, stream or None)
        if rc != 0:
            raise RuntimeError(f"LBM_SuperResUpscale: {rc}")

    def fine(self) -> np.ndarray:
        fx, fy, fz = self.fine_size()
        out = np.empty((fx * fy * fz, 4), np.float32)
        rc = self._L.LBM_SuperResCopyFine(self._h, _p(out))
        if rc != 0:
            raise RuntimeError(f"LBM_SuperResCopyFine: {rc}")
        return out

    def fine_device_ptr(self) -> int:
        return self._L.LBM_SuperResGetFineVelocity(self._h) or 0
