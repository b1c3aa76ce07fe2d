"""ORACLE — test infrastructure only.

ctypes access to the CPU restatement of the reference solve path in ``oracle.cpp``. Only the tests,
``__graft_entry__.smoke()`` and the CPU baseline of ``bench.py`` import this module; the product
(``solidfem_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

ACTIVE, CONVERGED, FAILED_NOT_PD, FAILED_NOT_CONVERGED = 0, 1, 2, 3
STAGE_SMOOTH, STAGE_RESIDUAL, STAGE_RESTRICT, STAGE_PROLONG, STAGE_START, STAGE_SMOOTH_ADD = range(6)
DOUBLE, SINGLE_STORAGE, SINGLE = 0, 1, 2
JACOBI, MULTIGRID = 0, 1
UNIFORM, SHELL_CORE = 0, 1


class Material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("E", C.c_double), ("nu", C.c_double),
                ("E2", C.c_double), ("nu2", C.c_double), ("lo", C.c_double * 3),
                ("hi", C.c_double * 3), ("depth", C.c_double)]


class Options(C.Structure):
    _fields_ = [("preconditioner", C.c_int32), ("precision", C.c_int32),
                ("tolerance", C.c_double), ("max_iterations", C.c_uint64),
                ("neighbour_reach", C.c_double), ("coarse_dofs", C.c_uint64),
                ("max_levels", C.c_uint64), ("smoother_degree", C.c_uint64),
                ("smoother_range", C.c_double), ("quadrature", C.c_int32)]


class NodalForce(C.Structure):
    _fields_ = [("node", C.c_uint32), ("force", C.c_double * 3)]


class Prescribed(C.Structure):
    _fields_ = [("node", C.c_uint32), ("axis", C.c_uint32), ("value", C.c_double)]


class Face(C.Structure):
    _fields_ = [("tet", C.c_uint32), ("face", C.c_uint32), ("nodes", C.c_uint32 * 6)]


class Progress(C.Structure):
    _fields_ = [("iteration", C.c_uint64), ("relative_residual", C.c_double),
                ("at_rounding_floor", C.c_int32), ("status", C.c_int32),
                ("fail_curvature", C.c_double)]


class LevelInfo(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("row_block", C.c_uint64), ("blocks", C.c_uint64),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double),
                ("has_prolongator", C.c_int32), ("p_blocks", C.c_uint64),
                ("p_col_block", C.c_uint64), ("has_factor", C.c_int32)]


class MgStats(C.Structure):
    _fields_ = [("levels", C.c_uint64), ("coarse_dofs", C.c_uint64),
                ("operator_complexity", C.c_double), ("memory_bytes", C.c_uint64)]


class PointStress(C.Structure):
    _fields_ = [("tet", C.c_uint32), ("point", C.c_uint32), ("position", C.c_double * 3),
                ("stress", C.c_double * 6), ("von_mises", C.c_double)]


_lib = None


def build() -> None:
    """Compiles the oracle with its Makefile (no FMA contraction, OpenMP row threading)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        p = C.POINTER
        L.orc_box_mesh.argtypes = [p(C.c_double), p(C.c_double), p(C.c_uint64), p(C.c_void_p)]
        L.orc_linear_mesh.argtypes = [p(C.c_double), C.c_uint64, p(C.c_uint32), C.c_uint64, p(C.c_void_p)]
        L.orc_mesh_free.argtypes = [C.c_void_p]
        for name in ("orc_mesh_node_count", "orc_mesh_tet_count", "orc_mesh_vertex_count", "orc_mesh_face_count"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = C.c_uint64
        L.orc_mesh_nodes.argtypes = [C.c_void_p, p(C.c_double)]
        L.orc_mesh_tets.argtypes = [C.c_void_p, p(C.c_uint32)]
        L.orc_mesh_faces.argtypes = [C.c_void_p, p(Face)]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_default_threads.restype = C.c_int
        L.orc_study_new.argtypes = [C.c_void_p, p(Material), p(Options), p(C.c_uint32), C.c_uint64,
                                    p(NodalForce), C.c_uint64, p(Face), p(C.c_double), C.c_uint64,
                                    p(C.c_void_p)]
        L.orc_study_new_prescribed.argtypes = [C.c_void_p, p(Material), p(Options), p(C.c_uint32), C.c_uint64,
                                               p(NodalForce), C.c_uint64, p(Face), p(C.c_double), C.c_uint64,
                                               p(Prescribed), C.c_uint64, p(C.c_void_p)]
        L.orc_study_free.argtypes = [C.c_void_p]
        L.orc_study_step.argtypes = [C.c_void_p, C.c_uint64, p(Progress)]
        L.orc_study_displacements.argtypes = [C.c_void_p, p(C.c_double)]
        L.orc_study_fingerprint.argtypes = [C.c_void_p]
        L.orc_study_fingerprint.restype = C.c_uint64
        L.orc_study_seconds.argtypes = [C.c_void_p, p(C.c_double)]
        L.orc_study_free_dofs.argtypes = [C.c_void_p]
        L.orc_study_free_dofs.restype = C.c_uint64
        L.orc_study_nonzeros.argtypes = [C.c_void_p]
        L.orc_study_nonzeros.restype = C.c_uint64
        L.orc_study_rhs.argtypes = [C.c_void_p, p(C.c_double)]
        L.orc_study_matrix.argtypes = [C.c_void_p, p(C.c_uint64), p(C.c_uint32), p(C.c_double)]
        L.orc_study_free_numbering.argtypes = [C.c_void_p, p(C.c_uint32)]
        L.orc_mg_levels.argtypes = [C.c_void_p]
        L.orc_mg_levels.restype = C.c_uint64
        L.orc_mg_level_info.argtypes = [C.c_void_p, C.c_uint64, p(LevelInfo)]
        L.orc_mg_level_matrix.argtypes = [C.c_void_p, C.c_uint64, C.c_int, p(C.c_uint64), p(C.c_uint32), p(C.c_double)]
        L.orc_mg_level_inverse_diagonal.argtypes = [C.c_void_p, C.c_uint64, p(C.c_double)]
        L.orc_mg_level_aggregates.argtypes = [C.c_void_p, C.c_uint64, p(C.c_uint32)]
        L.orc_mg_get_stats.argtypes = [C.c_void_p, p(MgStats)]
        L.orc_precondition.argtypes = [C.c_void_p, p(C.c_double), p(C.c_double)]
        L.orc_system_multiply.argtypes = [C.c_void_p, p(C.c_double), p(C.c_double)]
        L.orc_multiply_rounding_bound.argtypes = [C.c_void_p, p(C.c_double)]
        L.orc_multiply_rounding_bound.restype = C.c_double
        L.orc_study_recover.argtypes = [C.c_void_p]
        L.orc_study_recover_with.argtypes = [C.c_void_p, p(C.c_double)]
        L.orc_study_nodal_stress.argtypes = [C.c_void_p, p(C.c_double), p(C.c_double)]
        L.orc_study_point_count.argtypes = [C.c_void_p]
        L.orc_study_point_count.restype = C.c_uint64
        L.orc_study_point_stresses.argtypes = [C.c_void_p, p(PointStress)]
        L.orc_element_stiffness.argtypes = [p(C.c_double), p(Material), C.c_int, p(C.c_double)]
        L.orc_level_stage.argtypes = [C.c_void_p, C.c_uint64, C.c_int, p(C.c_double), p(C.c_double), p(C.c_double),
                                      p(C.c_double)]
        _lib = L
    return _lib


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Mesh:
    """A Tet10 mesh built by the oracle (box_mesh.rs + quadratic.rs)."""

    def __init__(self, handle):
        self.h = handle
        L = lib()
        self.node_count = L.orc_mesh_node_count(handle)
        self.tet_count = L.orc_mesh_tet_count(handle)
        self.vertex_count = L.orc_mesh_vertex_count(handle)
        self.face_count = L.orc_mesh_face_count(handle)

    @classmethod
    def box(cls, size, divisions, origin=(0.0, 0.0, 0.0)):
        h = C.c_void_p()
        o = (C.c_double * 3)(*origin)
        s = (C.c_double * 3)(*size)
        d = (C.c_uint64 * 3)(*divisions)
        code = lib().orc_box_mesh(o, s, d, C.byref(h))
        if code:
            raise ValueError(f"box mesh refused: code {code}")
        return cls(h)

    @classmethod
    def linear(cls, positions, tets):
        positions = np.ascontiguousarray(positions, dtype=np.float64)
        tets = np.ascontiguousarray(tets, dtype=np.uint32)
        h = C.c_void_p()
        code = lib().orc_linear_mesh(_ptr(positions, C.c_double), len(positions),
                                     _ptr(tets, C.c_uint32), len(tets), C.byref(h))
        if code:
            raise ValueError(f"mesh refused: code {code}")
        return cls(h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mesh_free(self.h)
            self.h = None

    def nodes(self):
        out = np.empty((self.node_count, 3), dtype=np.float64)
        lib().orc_mesh_nodes(self.h, _ptr(out, C.c_double))
        return out

    def tets(self):
        out = np.empty((self.tet_count, 10), dtype=np.uint32)
        lib().orc_mesh_tets(self.h, _ptr(out, C.c_uint32))
        return out

    def faces(self):
        arr = (Face * self.face_count)()
        lib().orc_mesh_faces(self.h, arr)
        return [(f.tet, f.face, tuple(f.nodes)) for f in arr]


def default_options(**kw) -> Options:
    """The reference's defaults: PcgOptions (pcg.rs:26-33), MultigridOptions (mod.rs:170-182)."""
    o = Options(preconditioner=MULTIGRID, precision=SINGLE_STORAGE, tolerance=1e-9,
                max_iterations=0, neighbour_reach=3.0, coarse_dofs=1500, max_levels=12,
                smoother_degree=3, smoother_range=30.0, quadrature=0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def uniform(E, nu) -> Material:
    return Material(kind=UNIFORM, E=E, nu=nu)


def shell_core(shell, core, lo, hi, depth) -> Material:
    return Material(kind=SHELL_CORE, E=shell[0], nu=shell[1], E2=core[0], nu2=core[1],
                    lo=(C.c_double * 3)(*lo), hi=(C.c_double * 3)(*hi), depth=depth)


class Study:
    """StaticStudy::new + step + solution of the oracle (study.rs)."""

    def __init__(self, mesh: Mesh, material: Material, options: Options, fixed,
                 faces=(), tractions=(), forces=(), prescribed=()):
        self.mesh = mesh
        fixed = np.ascontiguousarray(fixed, dtype=np.uint32)
        nf = len(faces)
        farr = (Face * max(nf, 1))()
        for i, (tet, face, nodes) in enumerate(faces):
            farr[i].tet, farr[i].face = tet, face
            for k in range(6):
                farr[i].nodes[k] = nodes[k]
        tr = np.ascontiguousarray(np.asarray(tractions, dtype=np.float64).reshape(-1, 3) if nf else np.zeros((1, 3)))
        forr = (NodalForce * max(len(forces), 1))()
        for i, (node, f) in enumerate(forces):
            forr[i].node = node
            for k in range(3):
                forr[i].force[k] = f[k]
        h = C.c_void_p()
        parr = (Prescribed * max(len(prescribed), 1))(*[Prescribed(int(n), int(a), float(v)) for n, a, v in prescribed])
        code = lib().orc_study_new_prescribed(mesh.h, C.byref(material), C.byref(options),
                                              _ptr(fixed, C.c_uint32), len(fixed), forr, len(forces), farr,
                                              _ptr(tr, C.c_double), nf, parr, len(prescribed), C.byref(h))
        if code:
            raise ValueError(f"study refused: code {code}")
        self.h = h
        self.n = lib().orc_study_free_dofs(h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_study_free(self.h)
            self.h = None

    def step(self, max_iterations=2**63):
        pr = Progress()
        lib().orc_study_step(self.h, max_iterations, C.byref(pr))
        return pr

    def solve(self):
        pr = self.step()
        return pr

    def displacements(self):
        out = np.empty((self.mesh.node_count, 3), dtype=np.float64)
        lib().orc_study_displacements(self.h, _ptr(out, C.c_double))
        return out

    def fingerprint(self):
        return int(lib().orc_study_fingerprint(self.h))

    def seconds(self):
        out = np.zeros(4)
        lib().orc_study_seconds(self.h, _ptr(out, C.c_double))
        return {"assembly": out[0], "preconditioner": out[1], "solve": out[2], "recovery": out[3]}

    def rhs(self):
        out = np.empty(self.n)
        lib().orc_study_rhs(self.h, _ptr(out, C.c_double))
        return out

    def matrix(self):
        nnz = lib().orc_study_nonzeros(self.h)
        rs = np.empty(self.n + 1, dtype=np.uint64)
        cols = np.empty(nnz, dtype=np.uint32)
        vals = np.empty(nnz)
        lib().orc_study_matrix(self.h, _ptr(rs, C.c_uint64), _ptr(cols, C.c_uint32), _ptr(vals, C.c_double))
        return rs, cols, vals

    def free_numbering(self):
        out = np.empty(self.mesh.node_count, dtype=np.uint32)
        lib().orc_study_free_numbering(self.h, _ptr(out, C.c_uint32))
        return out

    def levels(self):
        L = lib()
        out = []
        for lv in range(L.orc_mg_levels(self.h)):
            info = LevelInfo()
            L.orc_mg_level_info(self.h, lv, C.byref(info))
            rb = info.row_block
            starts = np.empty(info.rows + 1, dtype=np.uint64)
            cols = np.empty(info.blocks, dtype=np.uint32)
            vals = np.empty(info.blocks * rb * rb)
            L.orc_mg_level_matrix(self.h, lv, 0, _ptr(starts, C.c_uint64), _ptr(cols, C.c_uint32), _ptr(vals, C.c_double))
            inv = np.empty(info.rows * rb * rb)
            L.orc_mg_level_inverse_diagonal(self.h, lv, _ptr(inv, C.c_double))
            d = {"rows": info.rows, "row_block": rb, "starts": starts, "columns": cols, "values": vals,
                 "inverse_diagonal": inv, "lambda_min": info.lambda_min, "lambda_max": info.lambda_max,
                 "has_factor": bool(info.has_factor)}
            if info.has_prolongator:
                pst = np.empty(info.rows + 1, dtype=np.uint64)
                pc = np.empty(info.p_blocks, dtype=np.uint32)
                pv = np.empty(info.p_blocks * rb * info.p_col_block)
                L.orc_mg_level_matrix(self.h, lv, 1, _ptr(pst, C.c_uint64), _ptr(pc, C.c_uint32), _ptr(pv, C.c_double))
                agg = np.empty(info.rows, dtype=np.uint32)
                L.orc_mg_level_aggregates(self.h, lv, _ptr(agg, C.c_uint32))
                d.update({"p_starts": pst, "p_columns": pc, "p_values": pv, "aggregates": agg})
            out.append(d)
        return out

    def stats(self):
        st = MgStats()
        lib().orc_mg_get_stats(self.h, C.byref(st))
        return {"levels": st.levels, "coarse_dofs": st.coarse_dofs,
                "operator_complexity": st.operator_complexity, "memory_bytes": st.memory_bytes}

    def precondition(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        lib().orc_precondition(self.h, _ptr(r, C.c_double), _ptr(z, C.c_double))
        return z

    def system_multiply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        lib().orc_system_multiply(self.h, _ptr(x, C.c_double), _ptr(y, C.c_double))
        return y

    def level_stage(self, level, stage, in0, in1=None, out_len=None):
        """One stage of a level's V-cycle in the study's precision and its per-entry rounding bound
        (gpu/reference.rs:256-355): returns (out, bound)."""
        a = np.ascontiguousarray(in0, dtype=np.float64)
        b = np.ascontiguousarray(in1 if in1 is not None else np.zeros(1), dtype=np.float64)
        n = out_len or len(a)
        out, bound = np.empty(n), np.empty(n)
        if lib().orc_level_stage(self.h, level, stage, _ptr(a, C.c_double), _ptr(b, C.c_double),
                                 _ptr(out, C.c_double), _ptr(bound, C.c_double)):
            raise ValueError(f"stage {stage} does not apply to level {level}")
        return out, bound

    def recover(self):
        code = lib().orc_study_recover(self.h)
        if code:
            raise ValueError(f"recovery refused: code {code}")
        n = self.mesh.node_count
        s6 = np.empty((n, 6))
        vm = np.empty(n)
        lib().orc_study_nodal_stress(self.h, _ptr(s6, C.c_double), _ptr(vm, C.c_double))
        return s6, vm

    def recover_with(self, displacements):
        """Recovery (results.rs) of the given displacements of every mesh node."""
        d = np.ascontiguousarray(displacements, dtype=np.float64)
        code = lib().orc_study_recover_with(self.h, _ptr(d, C.c_double))
        if code:
            raise ValueError(f"recovery refused: code {code}")
        n = self.mesh.node_count
        s6 = np.empty((n, 6))
        vm = np.empty(n)
        lib().orc_study_nodal_stress(self.h, _ptr(s6, C.c_double), _ptr(vm, C.c_double))
        return s6, vm

    def point_stresses(self):
        cnt = lib().orc_study_point_count(self.h)
        arr = (PointStress * cnt)()
        lib().orc_study_point_stresses(self.h, arr)
        return arr


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def default_threads() -> int:
    return int(lib().orc_default_threads())


def fnv1a(displacements: np.ndarray) -> int:
    """FNV-1a over the little-endian bits of every displacement value, in node order
    (crates/solidfem/tests/validation/multigrid_precision.rs:216-226)."""
    h = 0xcbf29ce484222325
    for byte in np.ascontiguousarray(displacements, dtype="<f8").tobytes():
        h ^= byte
        h = (h * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h


ON_PLANE = 1e-9  # crates/solidfem/tests/validation/support.rs:12


def nodes_on_plane(nodes, axis, value):
    return np.nonzero(np.abs(nodes[:, axis] - value) < ON_PLANE)[0].astype(np.uint32)


def faces_on_plane(mesh: Mesh, axis, value, nodes=None):
    """Boundary faces whose three corners lie on the plane (support.rs:30-39)."""
    if nodes is None:
        nodes = mesh.nodes()
    out = []
    for f in mesh.faces():
        if all(abs(nodes[n][axis] - value) < ON_PLANE for n in f[2][:3]):
            out.append(f)
    return out
