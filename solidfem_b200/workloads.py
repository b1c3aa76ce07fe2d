"""Synthetic solve requests: cantilever bars, square tubes and thin plates, and the seeded serving
stream of mixed-size requests (Poisson arrivals).

Every part is a structured hex grid split 6 tets per hex (box_tet_mesh) upgraded to Tet10; a tube
is the reference demo's part grid (demo/wasm/src/part.rs:135-189) with 2 cells through each wall:
a unit grid of the cells, the hollow core's tets dropped, the kept vertices numbered in order of
first appearance and placed on the grid lines. Meshes are generated on a CUDA device when one is
given (the same mesh, bit for bit), else on the host. The part is clamped at x = 0 and carries a
total force on its x = L end face, spread as a uniform traction in -z.

DOF targeting (this stream's own rule; the reference has none): the request draws a target DOF
count, then the grid spacing is chosen so the Tet10 mesh has about that many DOFs, with at least
two cells through every thin dimension. For a tube the wall fixes the spacing (two cells through
the wall), so the tube's length and outer side are scaled together to reach the target.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import solidfem_b200 as sf

KINDS = ("bar", "tube", "plate")


@dataclass
class Request:
    index: int
    arrival: float          # seconds after the stream starts
    kind: str
    target_dofs: int
    length: float           # mm, along x
    width: float            # mm: plate width, tube outer side (unused for a bar)
    thickness: float        # mm: bar side, plate thickness, tube wall
    youngs_modulus: float   # MPa
    poisson_ratio: float
    force: float            # N, total, on the x = length face


def serving_stream(count: int = 512, rate: float = 20.0, seed: int = 0,
                   dof_range: tuple = (10_000, 600_000)) -> list:
    """The serving workload: `count` requests, Poisson arrivals at `rate` per second, kinds uniform,
    DOFs log-uniform over `dof_range`, dimensions uniform in [20, 200] mm, wall or thickness uniform
    in [0.8, 10] mm, E log-uniform in [0.8, 210] GPa, nu uniform in [0.28, 0.40], force uniform in
    [10, 1000] N."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    lo, hi = math.log(dof_range[0]), math.log(dof_range[1])
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        kind = KINDS[int(rng.integers(0, 3))]
        dofs = int(round(math.exp(rng.uniform(lo, hi))))
        length = float(rng.uniform(20.0, 200.0))
        width = float(rng.uniform(20.0, 200.0))
        thickness = float(rng.uniform(0.8, 10.0))
        E = float(math.exp(rng.uniform(math.log(800.0), math.log(210000.0))))
        nu = float(rng.uniform(0.28, 0.40))
        force = float(rng.uniform(10.0, 1000.0))
        out.append(Request(i, t, kind, dofs, length, width, thickness, E, nu, force))
    return out


def _box_dofs(div) -> int:
    nx, ny, nz = div
    return 3 * (2 * nx + 1) * (2 * ny + 1) * (2 * nz + 1)


def _box_divisions(size, target, min_cells) -> tuple:
    """Divisions of a box of `size` whose Tet10 mesh has about `target` DOFs, each at least
    `min_cells` (per axis) cells."""
    def div_for(h):
        return tuple(max(m, int(round(s / h))) for s, m in zip(size, min_cells))
    lo, hi = 1e-4 * max(size), 2.0 * max(size)
    for _ in range(80):
        mid = math.sqrt(lo * hi)
        if _box_dofs(div_for(mid)) > target:
            lo = mid
        else:
            hi = mid
    a, b = div_for(lo), div_for(hi)
    return a if abs(_box_dofs(a) - target) <= abs(_box_dofs(b) - target) else b


def _tube_layout(req: Request) -> tuple:
    """Length, outer side and divisions of a square tube with 2 cells through its wall whose mesh has
    about the target DOF count."""
    h = req.thickness / 2.0
    def dofs(scale):
        # A Tet10 node is a point of the grid at half spacing covered by a kept cell: the ring's
        # cross-section holds (2 ny + 1)^2 - (2 (ny - 4) - 1)^2 of them, and one section is clamped.
        ny = max(6, int(round(req.width * scale / h)))
        nx = max(2, int(round(req.length * scale / h)))
        section = (2 * ny + 1) ** 2 - (2 * (ny - 4) - 1) ** 2
        return 3 * section * 2 * nx, nx, ny
    lo, hi = 1e-3, 1e3
    for _ in range(80):
        mid = math.sqrt(lo * hi)
        if dofs(mid)[0] > req.target_dofs:
            hi = mid
        else:
            lo = mid
    a, b = dofs(lo), dofs(hi)
    _, nx, ny = a if abs(a[0] - req.target_dofs) <= abs(b[0] - req.target_dofs) else b
    return nx * h, ny * h, (nx, ny, ny)


TUBE_WALL_CELLS = 2


def part_mesh_host(x_lines, y_lines, z_lines, wall_cells: int) -> sf.Mesh:
    """The demo's part mesh (demo/wasm/src/part.rs:135-189) built on the host: a unit box_tet_mesh of
    the cells; a tet is dropped when the cell of its centroid (summed as sum + p * 0.25 from zero,
    then floored) lies in the hollow core (part.rs:114-122); the kept vertices are numbered in order
    of first appearance in the kept tets and placed on their grid lines; then TetMesh::new and
    from_linear. sf.part_tet_mesh generates the same mesh on a device."""
    lines = [np.asarray(v, dtype=np.float64) for v in (x_lines, y_lines, z_lines)]
    cells = tuple(len(v) - 1 for v in lines)
    unit = sf.box_tet_mesh((0.0, 0.0, 0.0), tuple(float(c) for c in cells), cells)
    pos = unit.nodes()[:unit.vertex_count()]
    tets = unit.tets()[:, :4].astype(np.int64)
    centroid = np.zeros((len(tets), 3))
    for q in range(4):
        centroid = centroid + pos[tets[:, q]] * 0.25
    j, k = np.floor(centroid[:, 1]).astype(np.int64), np.floor(centroid[:, 2]).astype(np.int64)
    hollow = ((wall_cells > 0) & (j >= wall_cells) & (j < cells[1] - wall_cells) &
              (k >= wall_cells) & (k < cells[2] - wall_cells))
    kept = tets[~hollow]
    flat = kept.ravel()
    used, first = np.unique(flat, return_index=True)
    order = used[np.argsort(first, kind="stable")]  # vertices by first appearance
    number = np.empty(len(pos), dtype=np.int64)
    number[order] = np.arange(len(order))
    grid = np.round(pos[order]).astype(np.int64)
    positions = np.stack([lines[a][grid[:, a]] for a in range(3)], axis=1)
    return sf.Mesh.from_linear(positions, number[kept].astype(np.uint32))


def tube_lines(req: Request) -> tuple:
    """Grid lines of the request's square tube (uniform cells, 2 through each wall)."""
    length, side, (nx, ny, nz) = _tube_layout(req)
    x = [length * i / nx for i in range(nx + 1)]
    y = [side * j / ny for j in range(ny + 1)]
    return x, y, list(y)


def build_mesh(req: Request, device: int | None = None) -> sf.Mesh:
    """The request's Tet10 mesh, generated on CUDA device `device` when it is given."""
    if req.kind == "plate":
        size = (req.length, req.width, req.thickness)
        return sf.box_tet_mesh((0.0, 0.0, 0.0), size, _box_divisions(size, req.target_dofs, (2, 2, 2)), device)
    if req.kind == "bar":
        size = (req.length, req.thickness, req.thickness)
        return sf.box_tet_mesh((0.0, 0.0, 0.0), size, _box_divisions(size, req.target_dofs, (2, 2, 2)), device)
    x, y, z = tube_lines(req)
    if device is None:
        return part_mesh_host(x, y, z, TUBE_WALL_CELLS)
    return sf.part_tet_mesh(x, y, z, TUBE_WALL_CELLS, device)


def end_area(req: Request, mesh_nodes: np.ndarray) -> float:
    if req.kind == "plate":
        return req.width * req.thickness
    if req.kind == "bar":
        return req.thickness * req.thickness
    side = float(mesh_nodes[:, 1].max())
    return side * side - (side - 2 * req.thickness) ** 2


def build_model(req: Request, mesh: sf.Mesh | None = None, device: int | None = None) -> tuple:
    """(mesh, model): clamped at x = 0, the total force as a uniform -z traction on the x = L face;
    the mesh generated on CUDA device `device` when it is given."""
    mesh = mesh or build_mesh(req, device)
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(req.youngs_modulus, req.poisson_ratio))
    xmax = float(nodes[:, 0].max())
    tol = 1e-9 * max(1.0, xmax)
    model.fix_nodes(np.flatnonzero(np.abs(nodes[:, 0]) <= tol))
    faces = mesh.boundary_face_array()
    on_end = np.all(np.abs(nodes[faces["nodes"][:, :3], 0] - xmax) <= tol, axis=1)
    model.add_face_tractions(faces[on_end], (0.0, 0.0, -req.force / end_area(req, nodes)))
    return mesh, model
