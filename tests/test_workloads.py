"""The serving stream and its part builders (CPU: meshes and loads are host work)."""
import numpy as np

import solidfem_b200 as sf
from solidfem_b200 import workloads as W


def test_stream_is_seeded_and_shaped():
    a, b = W.serving_stream(), W.serving_stream()
    assert len(a) == 512
    assert [(r.kind, r.target_dofs, r.arrival) for r in a] == [(r.kind, r.target_dofs, r.arrival) for r in b]
    arrivals = np.array([r.arrival for r in a])
    assert np.all(np.diff(arrivals) > 0)
    assert 20.0 < arrivals[-1] < 32.0  # 512 Poisson arrivals at 20/s
    dofs = np.array([r.target_dofs for r in a])
    assert dofs.min() >= 10_000 and dofs.max() <= 600_000
    assert {r.kind for r in a} == set(W.KINDS)
    for r in a:
        assert 20.0 <= r.length <= 200.0 and 0.8 <= r.thickness <= 10.0
        assert 800.0 <= r.youngs_modulus <= 210000.0 and 0.28 <= r.poisson_ratio <= 0.40
        assert 10.0 <= r.force <= 1000.0


def test_parts_hit_their_dof_targets():
    reqs = [r for r in W.serving_stream() if r.target_dofs < 60_000]
    seen = set()
    for r in reqs:
        if r.kind in seen:
            continue
        seen.add(r.kind)
        mesh, model = W.build_model(r)
        free = 3 * (mesh.node_count() - len(set(model.fixed)))
        assert abs(free - r.target_dofs) <= 0.35 * r.target_dofs, (r.kind, free, r.target_dofs)
        faces = sum(len(f) for f, _ in model.face_tractions)
        assert faces > 0 and len(model.fixed) > 0
    assert seen == set(W.KINDS)


def test_tube_keeps_two_cells_through_the_wall():
    r = next(r for r in W.serving_stream() if r.kind == "tube" and r.target_dofs < 30_000)
    mesh = W.build_mesh(r)
    nodes = mesh.nodes()
    side = nodes[:, 1].max()
    # the hollow core holds no node; the wall does
    core = (nodes[:, 1] > r.thickness + 1e-9) & (nodes[:, 1] < side - r.thickness - 1e-9) & \
           (nodes[:, 2] > r.thickness + 1e-9) & (nodes[:, 2] < side - r.thickness - 1e-9)
    assert not core.any()
    assert np.isclose(np.unique(np.round(nodes[:, 1], 9))[4], r.thickness)
