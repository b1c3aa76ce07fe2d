"""solidfem_b200: the solve path of solidfem (larsbrubaker/solidfem) on NVIDIA B200 (sm_100a).

Python mirror of the reference's Rust API (crates/solidfem-elastic/src/study.rs and
crates/solidfem-solve): ``box_tet_mesh`` / ``Mesh`` in, ``Model`` with material, supports and
loads, ``StudyBuilder`` (resumable assembly and multigrid setup), ``StaticStudy`` (resumable,
cancellable conjugate gradient) and the displacement field out. Every call goes through the C ABI
of ``libsolidfem_b200.so`` (include/solidfem_b200.h); there is no CPU fallback: importing this
package fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libsolidfem_b200.so")

# ----------------------------------------------------------------------------- C structures


FACE_DTYPE = np.dtype([("tet", "<u4"), ("face", "<u4"), ("nodes", "<u4", (6,))])


class BoundaryFace(C.Structure):
    """A boundary face: BoundaryFace, crates/solidfem-mesh/src/boundary.rs:15-24."""
    _fields_ = [("tet", C.c_uint32), ("face", C.c_uint32), ("nodes", C.c_uint32 * 6)]

    def key(self):
        return (self.tet, self.face, tuple(self.nodes))

    def __repr__(self):
        return f"BoundaryFace(tet={self.tet}, face={self.face}, nodes={list(self.nodes)})"


class _Material(C.Structure):
    _fields_ = [("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double)]


class _Options(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_uint64), ("preconditioner", C.c_int32),
                ("neighbour_reach", C.c_double), ("coarse_dofs", C.c_uint64), ("max_levels", C.c_uint64),
                ("smoother_degree", C.c_uint64), ("smoother_range", C.c_double), ("precision", C.c_int32),
                ("threads", C.c_uint64), ("device", C.c_int32), ("use_graphs", C.c_int32),
                ("device_memory_budget", C.c_uint64), ("sell_min_rows", C.c_uint64), ("batchable", C.c_int32),
                ("coarse_tail", C.c_int32)]


class _BuildProgress(C.Structure):
    _fields_ = [("elements_done", C.c_uint64), ("elements_total", C.c_uint64), ("setup_finished", C.c_int32)]


class _Progress(C.Structure):
    _fields_ = [("iteration", C.c_uint64), ("relative_residual", C.c_double), ("at_rounding_floor", C.c_int32)]


class _StepOutcome(C.Structure):
    _fields_ = [("kind", C.c_int32), ("progress", _Progress)]


class _Report(C.Structure):
    _fields_ = [("total_dofs", C.c_uint64), ("free_dofs", C.c_uint64), ("nonzeros", C.c_uint64),
                ("at_rounding_floor", C.c_int32), ("iterations", C.c_uint64), ("relative_residual", C.c_double),
                ("assembly_seconds", C.c_double), ("preconditioner_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("recovery_seconds", C.c_double), ("has_multigrid", C.c_int32),
                ("mg_levels", C.c_uint64), ("mg_coarse_dofs", C.c_uint64),
                ("mg_operator_complexity", C.c_double), ("mg_memory_bytes", C.c_uint64)]


class PointStress(C.Structure):
    """PointStress, crates/solidfem-elastic/src/results.rs:66-79."""
    _fields_ = [("tet", C.c_uint32), ("point", C.c_uint32), ("position", C.c_double * 3),
                ("stress", C.c_double * 6), ("von_mises", C.c_double)]


class _Error(C.Structure):
    _fields_ = [("status", C.c_int32), ("tet", C.c_uint32), ("node", C.c_uint32), ("face", C.c_uint32),
                ("point", C.c_uint32), ("axis", C.c_uint32), ("row", C.c_uint64), ("level", C.c_uint64),
                ("block", C.c_uint64), ("iteration", C.c_uint64), ("rank", C.c_uint64), ("expected", C.c_uint64),
                ("found", C.c_uint64), ("pivot", C.c_double),
                ("curvature", C.c_double), ("relative_residual", C.c_double), ("determinant", C.c_double),
                ("value", C.c_double), ("message", C.c_char * 256)]


class _LevelInfo(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("row_block", C.c_uint64), ("blocks", C.c_uint64),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double), ("has_prolongator", C.c_int32),
                ("prolongator_blocks", C.c_uint64), ("has_factor", C.c_int32)]


class _DeviceTiming(C.Structure):
    _fields_ = [("step_ms", C.c_double), ("assembly_ms", C.c_double), ("setup_ms", C.c_double),
                ("kernel_launches", C.c_uint64), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("launches_per_iteration", C.c_uint64), ("coarse_tail_level", C.c_int32),
                ("coarse_tail_cluster", C.c_uint32)]


class _KernelTiming(C.Structure):
    _fields_ = [("ms_per_launch", C.c_double), ("bytes_per_launch", C.c_double), ("launches", C.c_uint64)]


class Stage(enum.IntEnum):
    """Stages of one level of the device V-cycle (SF_STAGE_*)."""
    SMOOTH = 0
    RESIDUAL = 1
    RESTRICT = 2
    PROLONG = 3
    START = 4
    SMOOTH_ADD = 5
    RESTRICT_START = 6
    RESIDUAL_START = 7


class Kernel(enum.IntEnum):
    """Solver kernels that can be timed in isolation (SF_KERNEL_*)."""
    CHEBYSHEV_STEP = 0
    LEVEL_RESIDUAL = 1
    SYSTEM_PRODUCT = 2
    RESTRICTION = 3


class _ServerOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("memory_budget", C.c_uint64), ("batch_max_dofs", C.c_uint64),
                ("max_batch", C.c_uint64), ("build_threads", C.c_uint64), ("solve_threads", C.c_uint64),
                ("setup_threads", C.c_uint64)]


class _RequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("finished", C.c_int32), ("batched", C.c_int32), ("batch_size", C.c_uint64),
                ("outcome", _StepOutcome), ("free_dofs", C.c_uint64), ("node_count", C.c_uint64),
                ("device_bytes", C.c_uint64), ("queue_seconds", C.c_double), ("build_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("latency_seconds", C.c_double), ("message", C.c_char * 160)]


class _ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("pending", C.c_uint64), ("reserved_bytes", C.c_uint64),
                ("peak_reserved_bytes", C.c_uint64), ("batches", C.c_uint64), ("batched_requests", C.c_uint64),
                ("mean_batch_size", C.c_double)]


_CANCEL = C.CFUNCTYPE(C.c_int32, C.c_void_p)
_FIELD = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.c_uint64, C.POINTER(_Material))

# Every symbol include/solidfem_b200.h declares, with (restype, argtypes).
_P = C.POINTER
_V = C.c_void_p
SIGNATURES = {
    "sf_last_error": (C.c_int, [_P(_Error)]),
    "sf_status_message": (C.c_char_p, [C.c_int]),
    "sf_abi_version": (C.c_int32, []),
    "sf_box_tet_mesh": (C.c_int, [_P(C.c_double), _P(C.c_double), _P(C.c_uint64), _P(_V)]),
    "sf_mesh_from_linear": (C.c_int, [_P(C.c_double), C.c_uint64, _P(C.c_uint32), C.c_uint64, _P(_V)]),
    "sf_box_tet_mesh_device": (C.c_int, [_P(C.c_double), _P(C.c_double), _P(C.c_uint64), C.c_int32, _P(_V)]),
    "sf_mesh_from_linear_device": (C.c_int, [_P(C.c_double), C.c_uint64, _P(C.c_uint32), C.c_uint64, C.c_int32,
                                             _P(_V)]),
    "sf_part_tet_mesh_device": (C.c_int, [_P(C.c_double), C.c_uint64, _P(C.c_double), C.c_uint64, _P(C.c_double),
                                          C.c_uint64, C.c_uint64, C.c_int32, _P(_V)]),
    "sf_mesh_device": (C.c_int32, [_V]),
    "sf_mesh_destroy": (None, [_V]),
    "sf_mesh_node_count": (C.c_uint64, [_V]),
    "sf_mesh_tet_count": (C.c_uint64, [_V]),
    "sf_mesh_vertex_count": (C.c_uint64, [_V]),
    "sf_mesh_nodes": (C.c_int, [_V, _P(C.c_double)]),
    "sf_mesh_tets": (C.c_int, [_V, _P(C.c_uint32)]),
    "sf_mesh_boundary_face_count": (C.c_uint64, [_V]),
    "sf_mesh_boundary_faces": (C.c_int, [_V, _P(BoundaryFace)]),
    "sf_model_create": (C.c_int, [_V, _Material, _P(_V)]),
    "sf_model_destroy": (None, [_V]),
    "sf_model_set_material_field": (C.c_int, [_V, _FIELD, _V]),
    "sf_model_set_shell_core": (C.c_int, [_V, _Material, _Material, _P(C.c_double), _P(C.c_double), C.c_double]),
    "sf_model_set_quadrature": (C.c_int, [_V, C.c_int32]),
    "sf_model_fix_node": (C.c_int, [_V, C.c_uint32]),
    "sf_model_fix_nodes": (C.c_int, [_V, _P(C.c_uint32), C.c_uint64]),
    "sf_model_add_nodal_force": (C.c_int, [_V, C.c_uint32, _P(C.c_double)]),
    "sf_model_add_traction": (C.c_int, [_V, _P(BoundaryFace), _P(C.c_double)]),
    "sf_model_add_tractions": (C.c_int, [_V, _P(BoundaryFace), _P(C.c_double), C.c_uint64]),
    "sf_model_prescribe_displacement": (C.c_int, [_V, C.c_uint32, C.c_uint32, C.c_double]),
    "sf_study_options_default": (None, [_P(_Options)]),
    "sf_builder_create": (C.c_int, [_V, _P(_Options), _P(_V)]),
    "sf_builder_step": (C.c_int, [_V, C.c_uint64, _CANCEL, _V, _P(_BuildProgress)]),
    "sf_builder_finish": (C.c_int, [_V, _P(_V)]),
    "sf_builder_destroy": (None, [_V]),
    "sf_study_create": (C.c_int, [_V, _P(_Options), _CANCEL, _V, _P(_V)]),
    "sf_study_step": (C.c_int, [_V, C.c_uint64, _CANCEL, _V, _P(_StepOutcome)]),
    "sf_study_progress": (C.c_int, [_V, _P(_Progress)]),
    "sf_study_displacements": (C.c_int, [_V, _P(C.c_double)]),
    "sf_study_report": (C.c_int, [_V, _P(_Report)]),
    "sf_study_solution": (C.c_int, [_V, _CANCEL, _V, _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(PointStress)]),
    "sf_study_begin_recovery": (C.c_int, [_V, _P(_V)]),
    "sf_study_continue_recovery": (C.c_int, [_V, _V, C.c_uint64, _CANCEL, _V, _P(C.c_int32)]),
    "sf_study_finish_recovery": (C.c_int, [_V, _V, _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(PointStress)]),
    "sf_recovery_destroy": (None, [_V]),
    "sf_study_destroy": (None, [_V]),
    "sf_study_matrix": (C.c_int, [_V, _P(C.c_uint64), _P(C.c_uint32), _P(C.c_double)]),
    "sf_study_rhs": (C.c_int, [_V, _P(C.c_double)]),
    "sf_study_level_count": (C.c_uint64, [_V]),
    "sf_study_level_info": (C.c_int, [_V, C.c_uint64, _P(_LevelInfo)]),
    "sf_study_level_matrix": (C.c_int, [_V, C.c_uint64, C.c_int32, _P(C.c_uint64), _P(C.c_uint32), _P(C.c_double)]),
    "sf_study_aggregates": (C.c_int, [_V, C.c_uint64, _P(C.c_uint32)]),
    "sf_study_precondition": (C.c_int, [_V, _P(C.c_double), _P(C.c_double)]),
    "sf_study_system_multiply": (C.c_int, [_V, _P(C.c_double), _P(C.c_double)]),
    "sf_study_level_stage": (C.c_int, [_V, C.c_uint64, C.c_int32, _P(C.c_double), _P(C.c_double), _P(C.c_double),
                                       _P(C.c_double)]),
    "sf_study_energy_products": (C.c_int, [_V, _V, _V, _V, C.c_uint64]),
    "sf_study_solve_batch": (C.c_int, [_P(_V), C.c_uint64, _P(_StepOutcome), _P(C.c_int)]),
    "sf_server_options_default": (None, [_P(_ServerOptions)]),
    "sf_server_create": (C.c_int, [_P(_ServerOptions), _P(_V)]),
    "sf_server_submit": (C.c_int, [_V, _V, _P(_Options), _P(C.c_uint64)]),
    "sf_server_wait": (C.c_int, [_V, C.c_uint64, C.c_uint64, _P(_RequestResult)]),
    "sf_server_take": (C.c_int, [_V, C.c_uint64, _P(C.c_double)]),
    "sf_server_statistics": (C.c_int, [_V, _P(_ServerStats)]),
    "sf_server_cancel": (C.c_int, [_V, C.c_uint64]),
    "sf_server_destroy": (None, [_V]),
    "sf_study_device_timing": (C.c_int, [_V, _P(_DeviceTiming)]),
    "sf_study_resolve": (C.c_int, [_V, _P(C.c_double)]),
    "sf_study_stream": (C.c_uint64, [_V]),
    "sf_study_time_kernel": (C.c_int, [_V, C.c_int32, C.c_uint64, _P(_KernelTiming)]),
    "sf_system_create": (C.c_int, [C.c_uint64, _P(C.c_uint64), _P(C.c_uint32), _P(C.c_double), _P(C.c_double),
                                   _P(C.c_double), C.c_uint64, _P(C.c_double), C.c_uint64, _P(_Options), _CANCEL, _V,
                                   _P(_V)]),
    "sf_system_step": (C.c_int, [_V, C.c_uint64, _CANCEL, _V, _P(_StepOutcome)]),
    "sf_system_estimate": (C.c_int, [_V, _P(C.c_double)]),
    "sf_system_progress": (C.c_int, [_V, _P(_Progress)]),
    "sf_system_level_count": (C.c_uint64, [_V]),
    "sf_system_destroy": (None, [_V]),
}

_lib = None


def library() -> C.CDLL:
    """The loaded C-ABI library. Raises when it has not been built (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(f"{LIBRARY_PATH} is missing: build it with `python -m solidfem_b200.build` "
                              "(there is no CPU fallback)")
        lib = C.CDLL(LIBRARY_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class Status(enum.IntEnum):
    OK = 0
    MESH_EMPTY = 1
    MESH_NON_FINITE_POSITION = 2
    MESH_NODE_OUT_OF_RANGE = 3
    MESH_DEGENERATE_TET = 4
    MESH_FLAT_TET = 5
    MESH_UNUSED_NODE = 6
    MESH_NON_MANIFOLD_FACE = 7
    MESH_INVALID_BOX = 8
    NO_FIXED_NODES = 20
    BODY_NOT_HELD = 21
    NODE_OUT_OF_RANGE = 22
    NON_FINITE_LOAD = 23
    FACE_NOT_ON_BOUNDARY = 24
    NO_EFFECTIVE_LOAD = 25
    ELEMENT_INVERTED_JACOBIAN = 26
    ELEMENT_INVALID_MATERIAL = 27
    JACOBI_DIAGONAL = 28
    CANCELLED = 29
    NOT_FINISHED = 30
    AXIS_OUT_OF_RANGE = 31
    PRESCRIBED_ON_FIXED_NODE = 32
    DOFS_DO_NOT_HOLD = 33
    MG_BLOCK_STRUCTURE = 40
    MG_NEAR_NULL_LENGTH = 41
    MG_NOT_POSITIVE_DEFINITE = 42
    MG_POSITION_LENGTH = 43
    MG_COARSEST_NOT_FACTORED = 44
    MG_COARSE_LENGTH = 45
    PCG_NOT_POSITIVE_DEFINITE = 50
    PCG_NOT_CONVERGED = 51
    INVALID_ARGUMENT = 60
    CUDA_ERROR = 61
    DEVICE_MEMORY_BUDGET = 62
    NO_DEVICE = 63
    DEVICE_WAIT_TIMEOUT = 64


class SolidfemError(RuntimeError):
    """A refusal or failure: the reference's ModelError / MultigridError / PcgError variants, named by
    ``status`` with their payload in ``detail``."""

    def __init__(self, status: int, detail: dict):
        self.status = Status(status)
        self.detail = detail
        super().__init__(f"{self.status.name}: {detail.get('message', '')}")


def _check(code: int) -> None:
    if code != 0:
        err = _Error()
        library().sf_last_error(C.byref(err))
        detail = {name: getattr(err, name) for name, _ in _Error._fields_ if name != "message"}
        detail["message"] = err.message.decode(errors="replace")
        raise SolidfemError(code, detail)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _uptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


# ----------------------------------------------------------------------------- mesh


class Mesh:
    """A validated 10-node tetrahedral mesh (QuadraticTetMesh, crates/solidfem-mesh/src/quadratic.rs)."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        if getattr(self, "_h", None):
            library().sf_mesh_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def node_count(self) -> int:
        return int(library().sf_mesh_node_count(self._h))

    def tet_count(self) -> int:
        return int(library().sf_mesh_tet_count(self._h))

    def vertex_count(self) -> int:
        return int(library().sf_mesh_vertex_count(self._h))

    def nodes(self) -> np.ndarray:
        out = np.empty((self.node_count(), 3))
        _check(library().sf_mesh_nodes(self._h, _dptr(out)))
        return out

    def tets(self) -> np.ndarray:
        out = np.empty((self.tet_count(), 10), dtype=np.uint32)
        _check(library().sf_mesh_tets(self._h, _uptr(out)))
        return out

    def boundary_faces(self) -> list:
        n = int(library().sf_mesh_boundary_face_count(self._h))
        arr = (BoundaryFace * max(n, 1))()
        _check(library().sf_mesh_boundary_faces(self._h, arr))
        return list(arr[:n])

    def boundary_face_array(self) -> np.ndarray:
        """The boundary faces as a structured array (tet, face, nodes[6]), in boundary_faces() order."""
        n = int(library().sf_mesh_boundary_face_count(self._h))
        arr = np.zeros(max(n, 1), dtype=FACE_DTYPE)
        _check(library().sf_mesh_boundary_faces(self._h, arr.ctypes.data_as(C.POINTER(BoundaryFace))))
        return arr[:n]

    def device(self) -> Optional[int]:
        """The CUDA device holding this mesh's ten-node arrays (a generated mesh), else None."""
        d = int(library().sf_mesh_device(self._h))
        return None if d < 0 else d

    @classmethod
    def from_linear(cls, positions, tets, device: Optional[int] = None) -> "Mesh":
        """TetMesh::new + QuadraticTetMesh::from_linear (tet.rs:59-109, quadratic.rs:24-71); on the
        given CUDA device when `device` is set (the same mesh, generated there)."""
        p = np.ascontiguousarray(positions, dtype=np.float64)
        t = np.ascontiguousarray(tets, dtype=np.uint32)
        h = C.c_void_p()
        if device is None:
            _check(library().sf_mesh_from_linear(_dptr(p), len(p), _uptr(t), len(t), C.byref(h)))
        else:
            _check(library().sf_mesh_from_linear_device(_dptr(p), len(p), _uptr(t), len(t), int(device), C.byref(h)))
        return cls(h)


def box_tet_mesh(origin, size, divisions, device: Optional[int] = None) -> Mesh:
    """box_tet_mesh (crates/solidfem-mesh/src/box_mesh.rs:22-80) upgraded to 10 nodes; generated on
    the given CUDA device when `device` is set (the same mesh, bit for bit)."""
    h = C.c_void_p()
    o, sz = (C.c_double * 3)(*origin), (C.c_double * 3)(*size)
    dv = (C.c_uint64 * 3)(*[int(d) for d in divisions])
    if device is None:
        _check(library().sf_box_tet_mesh(o, sz, dv, C.byref(h)))
    else:
        _check(library().sf_box_tet_mesh_device(o, sz, dv, int(device), C.byref(h)))
    return Mesh(h)


def part_tet_mesh(x_lines, y_lines, z_lines, wall_cells: int = 0, device: int = 0) -> Mesh:
    """The demo's part mesh (demo/wasm/src/part.rs:135-189) over grid lines per axis, the hollow
    core's cells dropped when wall_cells > 0, generated on a CUDA device."""
    lines = [np.ascontiguousarray(v, dtype=np.float64) for v in (x_lines, y_lines, z_lines)]
    h = C.c_void_p()
    _check(library().sf_part_tet_mesh_device(_dptr(lines[0]), len(lines[0]), _dptr(lines[1]), len(lines[1]),
                                             _dptr(lines[2]), len(lines[2]), int(wall_cells), int(device),
                                             C.byref(h)))
    return Mesh(h)


# ----------------------------------------------------------------------------- model


@dataclass(frozen=True)
class Material:
    """Isotropic linear elastic properties (crates/solidfem-elastic/src/material.rs:5-31)."""
    youngs_modulus: float
    poisson_ratio: float

    def _c(self):
        return _Material(self.youngs_modulus, self.poisson_ratio)


@dataclass(frozen=True)
class ShellCore:
    """A printed part's material field: points nearer than ``depth`` to a face of the box
    ``[lo, hi]`` are ``shell``, the rest ``core``; evaluated per integration point."""
    shell: Material
    core: Material
    lo: Sequence[float]
    hi: Sequence[float]
    depth: float


class Quadrature(enum.IntEnum):
    FOUR_POINT = 0
    FOURTEEN_POINT = 1


class Model:
    """A structure, its material, supports and loads (Model, study.rs:46-104)."""

    def __init__(self, mesh: Mesh, material):
        self.mesh = mesh
        self.material = material
        self.quadrature = Quadrature.FOUR_POINT
        self.fixed: list = []
        self.forces: list = []
        self.tractions: list = []
        self.face_tractions: list = []
        self.prescribed: dict = {}

    def set_quadrature(self, q: Quadrature) -> None:
        self.quadrature = Quadrature(q)

    def fix_node(self, node: int) -> None:
        self.fixed.append(int(node))

    def fix_nodes(self, nodes) -> None:
        self.fixed.extend(int(n) for n in nodes)

    def add_nodal_force(self, node: int, force) -> None:
        self.forces.append((int(node), tuple(float(f) for f in force)))

    def add_traction(self, face: BoundaryFace, traction) -> None:
        self.tractions.append((face, tuple(float(t) for t in traction)))

    def add_face_tractions(self, faces: np.ndarray, traction) -> None:
        """Adds one traction to every face of a FACE_DTYPE array (the array form of add_traction)."""
        faces = np.ascontiguousarray(faces, dtype=FACE_DTYPE)
        self.face_tractions.append((faces, np.tile(np.asarray(traction, dtype=np.float64), (len(faces), 1))))

    def prescribe_displacement(self, node: int, axis: int, value: float) -> None:
        self.prescribed[(int(node), int(axis))] = float(value)

    def _to_c(self):
        lib = library()
        h = C.c_void_p()
        mat = self.material
        base = mat if isinstance(mat, Material) else Material(1.0, 0.0)
        _check(lib.sf_model_create(self.mesh.handle, base._c(), C.byref(h)))
        keep = []
        if isinstance(mat, ShellCore):
            _check(lib.sf_model_set_shell_core(h, mat.shell._c(), mat.core._c(), (C.c_double * 3)(*mat.lo),
                                               (C.c_double * 3)(*mat.hi), mat.depth))
        elif callable(mat):
            def field(user, positions, count, out, fn=mat):
                pos = np.ctypeslib.as_array(positions, shape=(count * 3,)).reshape(count, 3)
                for i in range(count):
                    m = fn(pos[i])
                    out[i].youngs_modulus = m.youngs_modulus
                    out[i].poisson_ratio = m.poisson_ratio
            cb = _FIELD(field)
            keep.append(cb)
            _check(lib.sf_model_set_material_field(h, cb, None))
        _check(lib.sf_model_set_quadrature(h, int(self.quadrature)))
        if self.fixed:
            f = np.ascontiguousarray(self.fixed, dtype=np.uint32)
            _check(lib.sf_model_fix_nodes(h, _uptr(f), len(f)))
        for node, force in self.forces:
            _check(lib.sf_model_add_nodal_force(h, node, (C.c_double * 3)(*force)))
        if self.tractions:
            faces = (BoundaryFace * len(self.tractions))(*[f for f, _ in self.tractions])
            tr = np.ascontiguousarray([t for _, t in self.tractions], dtype=np.float64)
            _check(lib.sf_model_add_tractions(h, faces, _dptr(tr), len(self.tractions)))
        for faces, tr in self.face_tractions:
            if len(faces):
                tr = np.ascontiguousarray(tr, dtype=np.float64)
                _check(lib.sf_model_add_tractions(h, faces.ctypes.data_as(C.POINTER(BoundaryFace)), _dptr(tr),
                                                  len(faces)))
        for (node, axis), value in self.prescribed.items():
            _check(lib.sf_model_prescribe_displacement(h, node, axis, value))
        return h, keep


# ----------------------------------------------------------------------------- options


class Precision(enum.IntEnum):
    """multigrid/mod.rs:127-141, plus MIXED: the f32 cycle inside FP64 flexible CG."""
    DOUBLE = 0
    SINGLE_STORAGE = 1
    SINGLE = 2
    MIXED = 3


@dataclass
class PcgOptions:
    """pcg.rs:14-33."""
    tolerance: float = 1e-9
    max_iterations: Optional[int] = None


@dataclass
class MultigridOptions:
    """multigrid/mod.rs:143-182."""
    neighbour_reach: float = 3.0
    coarse_dofs: int = 1500
    max_levels: int = 12
    smoother_degree: int = 3
    smoother_range: float = 30.0
    precision: Precision = Precision.SINGLE_STORAGE
    threads: int = 0


class Jacobi:
    """PreconditionerChoice::Jacobi (study.rs:106-115)."""


@dataclass
class StudyOptions:
    """StudyOptions (study.rs:139-148): Jacobi unless a MultigridOptions is given."""
    pcg: PcgOptions = field(default_factory=PcgOptions)
    preconditioner: object = field(default_factory=Jacobi)
    device: int = 0
    use_graphs: bool = True
    device_memory_budget: int = 0
    sell_min_rows: int = 0
    batchable: bool = False
    coarse_tail: bool = False

    def _c(self) -> _Options:
        o = _Options()
        library().sf_study_options_default(C.byref(o))
        o.tolerance = self.pcg.tolerance
        o.max_iterations = self.pcg.max_iterations or 0
        if isinstance(self.preconditioner, MultigridOptions):
            m = self.preconditioner
            o.preconditioner = 1
            o.neighbour_reach = m.neighbour_reach
            o.coarse_dofs = m.coarse_dofs
            o.max_levels = m.max_levels
            o.smoother_degree = m.smoother_degree
            o.smoother_range = m.smoother_range
            o.precision = int(m.precision)
            o.threads = m.threads
        else:
            o.preconditioner = 0
        o.device = self.device
        o.use_graphs = 1 if self.use_graphs else 0
        o.device_memory_budget = self.device_memory_budget
        o.sell_min_rows = self.sell_min_rows
        o.batchable = 1 if self.batchable else 0
        o.coarse_tail = 1 if self.coarse_tail else 0
        return o


def _cancel_fn(cancel: Optional[Callable[[], bool]]):
    if cancel is None:
        return _CANCEL(0)
    return _CANCEL(lambda _user: 1 if cancel() else 0)


# ----------------------------------------------------------------------------- study


@dataclass
class BuildProgress:
    elements_done: int
    elements_total: int
    setup_finished: bool


@dataclass
class Progress:
    """pcg.rs:36-45."""
    iteration: int
    relative_residual: float
    at_rounding_floor: bool


class Outcome(enum.IntEnum):
    RUNNING = 0
    CONVERGED = 1
    CANCELLED = 2


@dataclass
class StepOutcome:
    """pcg.rs:47-57."""
    kind: Outcome
    progress: Progress


@dataclass
class Solution:
    """A solved study's results (Solution, crates/solidfem-elastic/src/results.rs:81-95)."""
    displacements: np.ndarray      # node_count x 3
    point_stresses: np.ndarray     # structured: tet, point, position[3], stress[6], von_mises
    nodal_stress: np.ndarray       # node_count x 6: [xx, yy, zz, xy, yz, zx]
    nodal_von_mises: np.ndarray    # node_count
    report: dict


POINT_STRESS_DTYPE = np.dtype([("tet", "<u4"), ("point", "<u4"), ("position", "<f8", 3), ("stress", "<f8", 6),
                               ("von_mises", "<f8")])


class StudyBuilder:
    """StudyBuilder (study.rs:392-656): new validates and builds the load and pattern; step adds
    element stiffness on the device and then advances the multigrid setup."""

    def __init__(self, model: Model, options: Optional[StudyOptions] = None):
        options = options or StudyOptions()
        mh, self._keep = model._to_c()
        self._mesh = model.mesh
        self._quadrature = model.quadrature
        h = C.c_void_p()
        _check(library().sf_builder_create(mh, C.byref(options._c()), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            library().sf_builder_destroy(self._h)
            self._h = None

    def step(self, max_elements: int, cancel: Optional[Callable[[], bool]] = None) -> BuildProgress:
        p = _BuildProgress()
        cb = _cancel_fn(cancel)
        _check(library().sf_builder_step(self._h, max_elements, cb, None, C.byref(p)))
        return BuildProgress(p.elements_done, p.elements_total, bool(p.setup_finished))

    def finish(self) -> "StaticStudy":
        h = C.c_void_p()
        _check(library().sf_builder_finish(self._h, C.byref(h)))
        self._h = None
        return StaticStudy(h, self._mesh, self._keep, self._quadrature)


class StaticStudy:
    """A study in progress (StaticStudy, study.rs:178-378): step runs device iterations."""

    def __init__(self, handle, mesh: Mesh, keep=(), quadrature=None):
        self._h = handle
        self.mesh = mesh
        self._keep = keep
        self._quadrature = Quadrature.FOUR_POINT if quadrature is None else quadrature

    @classmethod
    def new(cls, model: Model, options: Optional[StudyOptions] = None,
            cancel: Optional[Callable[[], bool]] = None) -> "StaticStudy":
        """StaticStudy::new (study.rs:191-199)."""
        options = options or StudyOptions()
        mh, keep = model._to_c()
        h = C.c_void_p()
        _check(library().sf_study_create(mh, C.byref(options._c()), _cancel_fn(cancel), None, C.byref(h)))
        return cls(h, model.mesh, keep, model.quadrature)

    def __del__(self):
        if getattr(self, "_h", None):
            library().sf_study_destroy(self._h)
            self._h = None

    def step(self, max_iterations: int, cancel: Optional[Callable[[], bool]] = None) -> StepOutcome:
        o = _StepOutcome()
        _check(library().sf_study_step(self._h, max_iterations, _cancel_fn(cancel), None, C.byref(o)))
        p = o.progress
        return StepOutcome(Outcome(o.kind), Progress(p.iteration, p.relative_residual, bool(p.at_rounding_floor)))

    def solve(self, slice_iterations: int = 2**62) -> StepOutcome:
        while True:
            o = self.step(slice_iterations)
            if o.kind != Outcome.RUNNING:
                return o

    def displacements(self) -> np.ndarray:
        """The current estimate (a preview until converged), node_count x 3, zero at fixed nodes."""
        out = np.empty((self.mesh.node_count(), 3))
        _check(library().sf_study_displacements(self._h, _dptr(out)))
        return out

    def progress(self) -> Progress:
        """Pcg::progress (pcg.rs:200-207)."""
        p = _Progress()
        _check(library().sf_study_progress(self._h, C.byref(p)))
        return Progress(p.iteration, p.relative_residual, bool(p.at_rounding_floor))

    def _field_buffers(self):
        n = self.mesh.node_count()
        q = 14 if self._quadrature == Quadrature.FOURTEEN_POINT else 4
        return (np.empty((n, 3)), np.empty((n, 6)), np.empty(n),
                np.empty(self.mesh.tet_count() * q, dtype=POINT_STRESS_DTYPE))

    def solution(self, cancel: Optional[Callable[[], bool]] = None) -> Solution:
        """StaticStudy::solution (study.rs:246-260): displacements and the stress field recovered on
        the device; refuses (NOT_FINISHED) until the solve has converged, CANCELLED when `cancel`
        returns true between slices of the recovery."""
        d, s6, vm, pts = self._field_buffers()
        _check(library().sf_study_solution(self._h, _cancel_fn(cancel), None, _dptr(d), _dptr(s6), _dptr(vm),
                                           pts.ctypes.data_as(C.POINTER(PointStress))))
        return Solution(d, pts, s6, vm, self.report())

    def begin_recovery(self) -> "Recovery":
        """StaticStudy::begin_recovery (study.rs:262-274): a resumable recovery of the current
        displacements (the answer once converged, else a preview)."""
        h = C.c_void_p()
        _check(library().sf_study_begin_recovery(self._h, C.byref(h)))
        return Recovery(self, h)

    def report(self) -> dict:
        r = _Report()
        _check(library().sf_study_report(self._h, C.byref(r)))
        return {name: getattr(r, name) for name, _ in _Report._fields_}

    def matrix(self):
        rep = self.report()
        n, nnz = rep["free_dofs"], rep["nonzeros"]
        rs = np.empty(n + 1, dtype=np.uint64)
        cols = np.empty(nnz, dtype=np.uint32)
        vals = np.empty(nnz)
        _check(library().sf_study_matrix(self._h, rs.ctypes.data_as(C.POINTER(C.c_uint64)), _uptr(cols), _dptr(vals)))
        return rs, cols, vals

    def rhs(self) -> np.ndarray:
        out = np.empty(self.report()["free_dofs"])
        _check(library().sf_study_rhs(self._h, _dptr(out)))
        return out

    def levels(self) -> list:
        lib = library()
        out = []
        for lv in range(int(lib.sf_study_level_count(self._h))):
            info = _LevelInfo()
            _check(lib.sf_study_level_info(self._h, lv, C.byref(info)))
            rb = info.row_block
            st = np.empty(info.rows + 1, dtype=np.uint64)
            cols = np.empty(info.blocks, dtype=np.uint32)
            vals = np.empty(info.blocks * rb * rb)
            _check(lib.sf_study_level_matrix(self._h, lv, 0, st.ctypes.data_as(C.POINTER(C.c_uint64)), _uptr(cols), _dptr(vals)))
            d = {"rows": info.rows, "row_block": rb, "starts": st, "columns": cols, "values": vals,
                 "lambda_min": info.lambda_min, "lambda_max": info.lambda_max, "has_factor": bool(info.has_factor)}
            if info.has_prolongator:
                pst = np.empty(info.rows + 1, dtype=np.uint64)
                pc = np.empty(info.prolongator_blocks, dtype=np.uint32)
                pv = np.empty(info.prolongator_blocks * rb * 6)
                _check(lib.sf_study_level_matrix(self._h, lv, 1, pst.ctypes.data_as(C.POINTER(C.c_uint64)), _uptr(pc), _dptr(pv)))
                agg = np.empty(info.rows, dtype=np.uint32)
                _check(lib.sf_study_aggregates(self._h, lv, _uptr(agg)))
                d.update({"p_starts": pst, "p_columns": pc, "p_values": pv, "aggregates": agg})
            out.append(d)
        return out

    def precondition(self, residual: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(residual, dtype=np.float64)
        z = np.empty_like(r)
        _check(library().sf_study_precondition(self._h, _dptr(r), _dptr(z)))
        return z

    def level_stage(self, level: int, stage: "Stage", in0, in1=None, out_len: Optional[int] = None):
        """One stage of a level's device V-cycle (sf_study_level_stage): returns out0, or (out0, out1)
        for the fused-start stages. out_len is the output length (the coarser level's for the
        restrictions)."""
        a = np.ascontiguousarray(in0, dtype=np.float64)
        b = None if in1 is None else np.ascontiguousarray(in1, dtype=np.float64)
        n = out_len or len(a)
        o0, o1 = np.empty(n), np.empty(n)
        _check(library().sf_study_level_stage(self._h, level, int(stage), _dptr(a), None if b is None else _dptr(b),
                                              _dptr(o0), _dptr(o1)))
        if stage in (Stage.RESTRICT_START, Stage.RESIDUAL_START):
            return o0, o1
        return o0

    def system_multiply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        _check(library().sf_study_system_multiply(self._h, _dptr(x), _dptr(y)))
        return y

    def energy_products(self, x: int, y: int, energy: int, count: int) -> None:
        """y_k = A x_k and energy[k] = x_k . y_k for count (<= 8) vectors of the caller's device memory
        (raw device addresses), enqueued on stream() without allocating device memory."""
        _check(library().sf_study_energy_products(self._h, x, y, energy, count))

    def device_timing(self) -> dict:
        t = _DeviceTiming()
        _check(library().sf_study_device_timing(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in _DeviceTiming._fields_}

    def resolve(self, rhs: Optional[np.ndarray] = None) -> None:
        """Restarts the solve from zero with a new right-hand side (free DOFs) or the resident one."""
        if rhs is None:
            _check(library().sf_study_resolve(self._h, None))
        else:
            r = np.ascontiguousarray(rhs, dtype=np.float64)
            _check(library().sf_study_resolve(self._h, _dptr(r)))

    def stream(self) -> int:
        """The CUDA stream every kernel of this study runs on (cudaStream_t as an integer)."""
        return int(library().sf_study_stream(self._h))

    def time_kernel(self, kernel: "Kernel", repeats: int) -> dict:
        t = _KernelTiming()
        _check(library().sf_study_time_kernel(self._h, int(kernel), repeats, C.byref(t)))
        return {"ms_per_launch": t.ms_per_launch, "bytes_per_launch": t.bytes_per_launch, "launches": t.launches}


@dataclass
class RecoveredField:
    """RecoveredField (crates/solidfem-elastic/src/results.rs:126-139)."""
    displacements: np.ndarray
    point_stresses: np.ndarray
    nodal_stress: np.ndarray
    nodal_von_mises: np.ndarray


class Recovery:
    """A resumable stress recovery on the device (Recovery, results.rs:97-124): continue() does up to
    max_units more elements, then vertex patch fits; finish() returns the field."""

    def __init__(self, study: StaticStudy, handle):
        self._study = study  # the study outlives its recoveries
        self._h = handle

    def __del__(self):
        if getattr(self, "_h", None):
            library().sf_recovery_destroy(self._h)
            self._h = None

    def continue_(self, max_units: int, cancel: Optional[Callable[[], bool]] = None) -> bool:
        """StaticStudy::continue_recovery (study.rs:276-296): True once every unit is done."""
        done = C.c_int32()
        _check(library().sf_study_continue_recovery(self._study._h, self._h, max_units, _cancel_fn(cancel), None,
                                                    C.byref(done)))
        return bool(done.value)

    def finish(self) -> RecoveredField:
        """StaticStudy::finish_recovery (study.rs:298-304); NOT_FINISHED while units remain."""
        d, s6, vm, pts = self._study._field_buffers()
        _check(library().sf_study_finish_recovery(self._study._h, self._h, _dptr(d), _dptr(s6), _dptr(vm),
                                                  pts.ctypes.data_as(C.POINTER(PointStress))))
        return RecoveredField(d, pts, s6, vm)


@dataclass
class ServerOptions:
    """sf_server_options: device, memory budget (bytes, 0: 150 GiB), the batching threshold in free DOFs,
    studies per batch, build threads, solver threads and setup threads per build."""
    device: int = 0
    memory_budget: int = 0
    batch_max_dofs: int = 100000
    max_batch: int = 64
    build_threads: int = 8
    solve_threads: int = 4
    setup_threads: int = 2

    def _c(self) -> _ServerOptions:
        o = _ServerOptions()
        o.device = self.device
        o.memory_budget = self.memory_budget
        o.batch_max_dofs = self.batch_max_dofs
        o.max_batch = self.max_batch
        o.build_threads = self.build_threads
        o.solve_threads = self.solve_threads
        o.setup_threads = self.setup_threads
        return o


@dataclass
class RequestResult:
    status: "Status"
    finished: bool
    batched: bool
    batch_size: int
    outcome: StepOutcome
    free_dofs: int
    node_count: int
    device_bytes: int
    queue_seconds: float
    build_seconds: float
    solve_seconds: float
    latency_seconds: float
    message: str = ""


class Server:
    """The serving loop (sf_server): requests admitted by device memory budget, built on worker threads,
    small ones solved in continuous batches, large ones on their own streams."""

    def __init__(self, options: Optional[ServerOptions] = None):
        self._h = C.c_void_p()
        _check(library().sf_server_create(C.byref((options or ServerOptions())._c()), C.byref(self._h)))
        self._keep = {}

    def submit(self, model: Model, options: Optional[StudyOptions] = None) -> int:
        mh, keep = model._to_c()
        rid = C.c_uint64()
        _check(library().sf_server_submit(self._h, mh, C.byref((options or StudyOptions())._c()), C.byref(rid)))
        self._keep[rid.value] = keep
        return rid.value

    def wait(self, rid: int, timeout: Optional[float] = None) -> RequestResult:
        r = _RequestResult()
        ms = 2**64 - 1 if timeout is None else int(timeout * 1000)
        code = library().sf_server_wait(self._h, rid, ms, C.byref(r))
        if code not in (0, int(Status.NOT_FINISHED)):
            _check(code)
        p = r.outcome.progress
        return RequestResult(Status(r.status), bool(r.finished), bool(r.batched), r.batch_size,
                             StepOutcome(Outcome(r.outcome.kind), Progress(p.iteration, p.relative_residual,
                                                                           bool(p.at_rounding_floor))),
                             r.free_dofs, r.node_count, r.device_bytes, r.queue_seconds, r.build_seconds,
                             r.solve_seconds, r.latency_seconds, r.message.decode(errors="replace"))

    def cancel(self, rid: int) -> None:
        """Stops a request at its next cancel check; it finishes as CANCELLED (sf_server_cancel)."""
        _check(library().sf_server_cancel(self._h, rid))

    def take(self, rid: int, node_count: int) -> np.ndarray:
        out = np.empty((node_count, 3), dtype=np.float64)
        try:
            _check(library().sf_server_take(self._h, rid, _dptr(out)))
        finally:
            self._keep.pop(rid, None)
        return out

    def stats(self) -> dict:
        st = _ServerStats()
        _check(library().sf_server_statistics(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in _ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().sf_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()


def _outcome(o: _StepOutcome) -> StepOutcome:
    p = o.progress
    return StepOutcome(Outcome(o.kind), Progress(p.iteration, p.relative_residual, bool(p.at_rounding_floor)))


class System:
    """A raw symmetric system solved on the device: CsrMatrix + Pcg (crates/solidfem-solve/src/pcg.rs)
    under Jacobi or the multigrid of MultigridSetup (multigrid/setup.rs), without a mesh.

    ``row_starts``/``columns``/``values`` are scalar CSR (each row's columns ascending); for multigrid
    ``near_null`` holds 6 values per unknown and ``positions`` one point per block row of three."""

    def __init__(self, row_starts, columns, values, rhs, options: Optional[StudyOptions] = None,
                 near_null=None, positions=None, cancel: Optional[Callable[[], bool]] = None):
        rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
        cols = np.ascontiguousarray(columns, dtype=np.uint32)
        vals = np.ascontiguousarray(values, dtype=np.float64)
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        n = len(rs) - 1
        if len(b) != n:
            raise ValueError(f"rhs has {len(b)} values for {n} rows")
        nn = None if near_null is None else np.ascontiguousarray(near_null, dtype=np.float64).reshape(-1)
        pos = None if positions is None else np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self.n = n
        h = C.c_void_p()
        _check(library().sf_system_create(
            n, rs.ctypes.data_as(C.POINTER(C.c_uint64)), _uptr(cols), _dptr(vals), _dptr(b),
            None if nn is None else _dptr(nn), 0 if nn is None else len(nn),
            None if pos is None else _dptr(pos), 0 if pos is None else len(pos),
            C.byref((options or StudyOptions())._c()), _cancel_fn(cancel), None, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            library().sf_system_destroy(self._h)
            self._h = None

    def step(self, max_iterations: int, cancel: Optional[Callable[[], bool]] = None) -> StepOutcome:
        """Pcg::step: raises SolidfemError (PCG_NOT_POSITIVE_DEFINITE / PCG_NOT_CONVERGED) once failed."""
        o = _StepOutcome()
        _check(library().sf_system_step(self._h, max_iterations, _cancel_fn(cancel), None, C.byref(o)))
        return _outcome(o)

    def solve(self, slice_iterations: int = 2**62) -> StepOutcome:
        while True:
            o = self.step(slice_iterations)
            if o.kind != Outcome.RUNNING:
                return o

    def estimate(self) -> np.ndarray:
        """Pcg::estimate: the current estimate of x."""
        out = np.empty(self.n)
        _check(library().sf_system_estimate(self._h, _dptr(out)))
        return out

    def progress(self) -> Progress:
        p = _Progress()
        _check(library().sf_system_progress(self._h, C.byref(p)))
        return Progress(p.iteration, p.relative_residual, bool(p.at_rounding_floor))

    def level_count(self) -> int:
        return int(library().sf_system_level_count(self._h))


def solve_batch(studies) -> list:
    """Solves resident studies together, one grid per kernel over all of them (sf_study_solve_batch).
    Returns (StepOutcome, Status) per study."""
    n = len(studies)
    handles = (_V * n)(*[st._h for st in studies])
    outs = (_StepOutcome * n)()
    stats = (C.c_int * n)()
    _check(library().sf_study_solve_batch(handles, n, outs, stats))
    res = []
    for i in range(n):
        p = outs[i].progress
        res.append((StepOutcome(Outcome(outs[i].kind), Progress(p.iteration, p.relative_residual,
                                                                 bool(p.at_rounding_floor))), Status(stats[i])))
    return res


__all__ = [
    "FACE_DTYPE", "BoundaryFace", "Mesh", "box_tet_mesh", "part_tet_mesh", "Material", "ShellCore", "Quadrature", "Model", "Precision",
    "PcgOptions", "MultigridOptions", "Jacobi", "StudyOptions", "StudyBuilder", "StaticStudy", "StepOutcome",
    "Outcome", "Progress", "BuildProgress", "PointStress", "SolidfemError", "Status", "library", "SIGNATURES", "Kernel", "Solution",
    "solve_batch", "Server", "ServerOptions", "RequestResult", "System", "Recovery", "RecoveredField", "Stage",
]
