"""Synthetic solve requests: cantilever bars, square tubes and thin plates, and the seeded serving
stream of mixed-size requests (Poisson arrivals).

Every part is a structured hex grid split 6 tets per hex (box_tet_mesh) upgraded to Tet10; a tube
drops the hollow cells of its box and keeps 2 cells through each wall, the way the reference's
demo builds tubes (demo/wasm/src/part.rs:50-189). The part is clamped at x = 0 and carries a total
force on its x = L end face, spread as a uniform traction in -z.

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


def build_mesh(req: Request) -> sf.Mesh:
    """The request's Tet10 mesh."""
    if req.kind == "plate":
        size = (req.length, req.width, req.thickness)
        return sf.box_tet_mesh((0.0, 0.0, 0.0), size, _box_divisions(size, req.target_dofs, (2, 2, 2)))
    if req.kind == "bar":
        size = (req.length, req.thickness, req.thickness)
        return sf.box_tet_mesh((0.0, 0.0, 0.0), size, _box_divisions(size, req.target_dofs, (2, 2, 2)))
    length, side, div = _tube_layout(req)
    box = sf.box_tet_mesh((0.0, 0.0, 0.0), (length, side, side), div)
    nodes, tets = box.nodes(), box.tets()[:, :4].astype(np.int64)
    centroid = nodes[tets].mean(axis=1)
    wall = req.thickness
    hollow = ((centroid[:, 1] > wall) & (centroid[:, 1] < side - wall) &
              (centroid[:, 2] > wall) & (centroid[:, 2] < side - wall))
    kept = tets[~hollow]
    used, inverse = np.unique(kept, return_inverse=True)
    return sf.Mesh.from_linear(nodes[used], inverse.reshape(kept.shape).astype(np.uint32))


def end_area(req: Request, mesh_nodes: np.ndarray) -> float:
    if req.kind == "plate":
        return req.width * req.thickness
    if req.kind == "bar":
        return req.thickness * req.thickness
    side = float(mesh_nodes[:, 1].max())
    return side * side - (side - 2 * req.thickness) ** 2


def build_model(req: Request, mesh: sf.Mesh | None = None) -> tuple:
    """(mesh, model): clamped at x = 0, the total force as a uniform -z traction on the x = L face."""
    mesh = mesh or build_mesh(req)
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(req.youngs_modulus, req.poisson_ratio))
    xmax = float(nodes[:, 0].max())
    tol = 1e-9 * max(1.0, xmax)
    model.fix_nodes(np.flatnonzero(np.abs(nodes[:, 0]) <= tol))
    faces = mesh.boundary_face_array()
    on_end = np.all(np.abs(nodes[faces["nodes"][:, :3], 0] - xmax) <= tol, axis=1)
    model.add_face_tractions(faces[on_end], (0.0, 0.0, -req.force / end_area(req, nodes)))
    return mesh, model
