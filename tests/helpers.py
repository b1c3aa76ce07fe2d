"""Shared builders for product-vs-oracle tests: the same model through both."""
import numpy as np

import solidfem_b200 as sf

ON_PLANE = 1e-9


def product_model(size, div, E, nu, clamp_axis=0, clamp_value=0.0, load_axis=0, load_value=None,
                  traction=(0.0, 3.0, -7.0), material=None):
    mesh = sf.box_tet_mesh((0, 0, 0), size, div)
    nodes = mesh.nodes()
    load_value = size[load_axis] if load_value is None else load_value
    model = sf.Model(mesh, material or sf.Material(E, nu))
    model.fix_nodes(np.nonzero(np.abs(nodes[:, clamp_axis] - clamp_value) < ON_PLANE)[0])
    for f in mesh.boundary_faces():
        if all(abs(nodes[n][load_axis] - load_value) < ON_PLANE for n in list(f.nodes)[:3]):
            model.add_traction(f, traction)
    return mesh, model


def oracle_study(O, size, div, E, nu, options, clamp_axis=0, clamp_value=0.0, load_axis=0, load_value=None,
                 traction=(0.0, 3.0, -7.0), material=None):
    mesh = O.Mesh.box(size, div)
    nodes = mesh.nodes()
    load_value = size[load_axis] if load_value is None else load_value
    fixed = O.nodes_on_plane(nodes, clamp_axis, clamp_value)
    faces = O.faces_on_plane(mesh, load_axis, load_value, nodes)
    return O.Study(mesh, material or O.uniform(E, nu), options, fixed, faces, [list(traction)] * len(faces))


def mg_options(precision, tolerance=1e-9, coarse_dofs=100, sell_min_rows=0, batchable=False, **kw):
    return sf.StudyOptions(pcg=sf.PcgOptions(tolerance=tolerance), sell_min_rows=sell_min_rows, batchable=batchable,
                           preconditioner=sf.MultigridOptions(coarse_dofs=coarse_dofs, precision=precision, **kw))
