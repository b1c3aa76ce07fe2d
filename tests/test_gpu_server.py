"""The serving loop (sf_server) on a small mixed stream (needs a B200): every request's answer in
the mix equals its answer alone in the same operator layout (also with the requests' meshes
generated on the device), one answer of each part kind matches
the oracle's FP64 solve, a request cancelled in the middle of a batch leaves the others' answers
unchanged, and the memory budget holds.
"""
import time

import numpy as np
import pytest

import solidfem_b200 as sf
from solidfem_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-8
BATCH_MAX_DOFS = 30_000
# A request alone and in the mix runs the same arithmetic per row, and every reduction has a fixed
# grid per study, so the answers come out with the same bits (measured); the bar leaves room only
# for a batch whose members' thread blocks differ in shape, which would regroup the partial sums
# of a dot product (about 1e-16 relative each).
MIX_BAR = 1e-12


def options(batchable=False):
    return sf.StudyOptions(pcg=sf.PcgOptions(tolerance=TOL), batchable=batchable,
                           preconditioner=sf.MultigridOptions(precision=sf.Precision.MIXED))


def stream():
    return W.serving_stream(count=12, rate=400.0, seed=7, dof_range=(4_000, 60_000))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def solo_answers(reqs, batch_max_dofs=BATCH_MAX_DOFS):
    """Each request alone, laid out as the server lays it out (batchable below the threshold)."""
    out = []
    for r in reqs:
        mesh, model = W.build_model(r)
        free = 3 * (mesh.node_count() - len(set(model.fixed)))
        st = sf.StaticStudy.new(model, options(batchable=free < batch_max_dofs))
        assert st.solve().kind == sf.Outcome.CONVERGED
        out.append(st.displacements())
    return out


def serve(reqs, server_options, cancel_index=None, device=None):
    server = sf.Server(server_options)
    try:
        models = [W.build_model(r, device=device) for r in reqs]
        start = time.perf_counter()
        ids = []
        for r, (mesh, model) in zip(reqs, models):
            delay = r.arrival - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            ids.append((server.submit(model, options()), mesh.node_count()))
        cancelled_in_batch = None
        if cancel_index is not None:
            rid = ids[cancel_index][0]
            while True:  # wait until it runs inside a batch, then cancel it
                res = server.wait(rid, timeout=0.0)
                if res.finished or res.batch_size > 0:
                    break
                time.sleep(0.0005)
            cancelled_in_batch = not res.finished
            server.cancel(rid)
        results = [server.wait(rid) for rid, _ in ids]
        answers = []
        for i, (rid, n) in enumerate(ids):
            if i == cancel_index and results[i].status == sf.Status.CANCELLED:
                with pytest.raises(sf.SolidfemError) as err:
                    server.take(rid, n)
                assert err.value.status == sf.Status.CANCELLED
                answers.append(None)
            else:
                answers.append(server.take(rid, n))
        return results, answers, server.stats(), cancelled_in_batch
    finally:
        server.close()


def test_served_answers_equal_solo_answers():
    reqs = stream()
    solo = solo_answers(reqs)
    results, answers, stats, _ = serve(reqs, sf.ServerOptions(batch_max_dofs=BATCH_MAX_DOFS, build_threads=3))
    assert stats["completed"] == len(reqs)
    assert any(r.batched for r in results) and any(not r.batched for r in results)
    for r, res, a, s in zip(reqs, results, answers, solo):
        assert res.status == sf.Status.OK and res.outcome.kind == sf.Outcome.CONVERGED
        d = rel(a, s)
        print(f"request {r.index} {r.kind} batched {res.batched}: served vs alone {d:.2e}")
        if res.batched:
            assert d <= MIX_BAR, (r.index, r.kind, d)
        else:  # solved on its own stream exactly as alone
            assert np.array_equal(a.view(np.uint64), s.view(np.uint64)), (r.index, r.kind, d)
        assert res.latency_seconds >= res.solve_seconds >= 0.0


def test_served_answers_from_device_meshes_equal_solo_host_answers():
    """The serving bench generates each request's mesh on the device: the device mesh, pattern and
    traction load give the host-mesh answers (unbatched to the bit, batched within the mix bar)."""
    reqs = stream()
    solo = solo_answers(reqs)
    results, answers, stats, _ = serve(reqs, sf.ServerOptions(batch_max_dofs=BATCH_MAX_DOFS, build_threads=3),
                                       device=0)
    assert stats["completed"] == len(reqs)
    for r, res, a, s in zip(reqs, results, answers, solo):
        assert res.status == sf.Status.OK and res.outcome.kind == sf.Outcome.CONVERGED
        if res.batched:
            assert rel(a, s) <= MIX_BAR, (r.index, r.kind, rel(a, s))
        else:
            assert np.array_equal(a.view(np.uint64), s.view(np.uint64)), (r.index, r.kind, rel(a, s))


def oracle_answer(O, req):
    """The oracle's FP64 solve (requested 1e-12) of the request's model: the same Tet10 mesh from the
    same linear tets, supports and end traction."""
    mesh, model = W.build_model(req)
    nodes, tets = mesh.nodes(), mesh.tets()
    om = O.Mesh.linear(nodes[:mesh.vertex_count()], tets[:, :4])
    on = om.nodes()
    xmax = float(on[:, 0].max())
    tol = 1e-9 * max(1.0, xmax)
    fixed = np.flatnonzero(np.abs(on[:, 0]) <= tol).astype(np.uint32)
    faces = [f for f in om.faces() if all(abs(on[n][0] - xmax) <= tol for n in f[2][:3])]
    traction = [0.0, 0.0, -req.force / W.end_area(req, on)]
    O.set_threads(4)
    ref = O.Study(om, O.uniform(req.youngs_modulus, req.poisson_ratio),
                  O.default_options(tolerance=1e-12, precision=O.DOUBLE), fixed, faces, [traction] * len(faces))
    ref.solve()
    return ref.displacements()


def test_one_served_answer_of_each_kind_matches_the_oracle(oracle):
    reqs = []
    for r in W.serving_stream(count=40, rate=400.0, seed=11, dof_range=(4_000, 40_000)):
        if r.kind not in {q.kind for q in reqs}:
            reqs.append(r)
    assert {r.kind for r in reqs} == set(W.KINDS)
    results, answers, stats, _ = serve(reqs, sf.ServerOptions(batch_max_dofs=BATCH_MAX_DOFS, build_threads=3))
    for r, res, a in zip(reqs, results, answers):
        assert res.status == sf.Status.OK
        ref = oracle_answer(oracle, r)
        d = rel(a, ref)
        print(f"{r.kind} ({res.free_dofs} DOFs, batched {res.batched}): served vs oracle FP64 {d:.2e}")
        assert d <= 1e-8, (r.kind, d)


def burst():
    return [W.Request(i, 0.0, "plate", 30_000 + 500 * i, 60.0 + i, 40.0, 1.0 + 0.1 * i, 2000.0 * (1 + i), 0.3,
                      100.0 + 10 * i) for i in range(8)]


def test_a_burst_of_similar_requests_shares_batches():
    reqs = burst()
    solo = solo_answers(reqs, batch_max_dofs=100_000)
    results, answers, stats, _ = serve(reqs, sf.ServerOptions(build_threads=8))
    assert stats["completed"] == len(reqs)
    assert all(r.batched for r in results)
    assert max(r.batch_size for r in results) > 1, "no two requests shared a batch"
    for res, a, s in zip(results, answers, solo):
        assert res.status == sf.Status.OK
        assert rel(a, s) <= MIX_BAR


def test_a_request_cancelled_mid_batch_leaves_the_others_unchanged():
    reqs = burst()
    solo = solo_answers(reqs, batch_max_dofs=100_000)
    victim = 3
    results, answers, stats, in_batch = serve(reqs, sf.ServerOptions(build_threads=8), cancel_index=victim)
    assert stats["completed"] == len(reqs)
    if in_batch:
        assert results[victim].status == sf.Status.CANCELLED
        assert results[victim].outcome.kind != sf.Outcome.CONVERGED
    for i, (res, a, s) in enumerate(zip(results, answers, solo)):
        if i == victim:
            continue
        assert res.status == sf.Status.OK and res.outcome.kind == sf.Outcome.CONVERGED
        d = rel(a, s)
        print(f"request {i}: served (with {victim} cancelled: {in_batch}) vs alone {d:.2e}")
        assert d <= MIX_BAR


def test_a_queued_request_is_cancelled_at_once():
    reqs = burst()[:4]
    server = sf.Server(sf.ServerOptions(build_threads=1, memory_budget=1))  # admits one request at a time
    try:
        ids = []
        for r in reqs:
            mesh, model = W.build_model(r)
            ids.append((server.submit(model, options()), mesh.node_count()))
        server.cancel(ids[-1][0])
        last = server.wait(ids[-1][0], timeout=5.0)
        assert last.finished and last.status == sf.Status.CANCELLED
        for rid, n in ids[:-1]:
            assert server.wait(rid).status == sf.Status.OK
    finally:
        server.close()


def test_memory_budget_bounds_admission():
    reqs = stream()[:6]
    # Admission reserves an estimate per free DOF until a study is built, then its real bytes: a
    # budget that fits every single request but not all of them at once must never be exceeded.
    estimates = []
    for r in reqs:
        mesh, model = W.build_model(r)
        estimates.append(3 * (mesh.node_count() - len(set(model.fixed))) * 6144)
    budget = int(1.5 * max(estimates))
    assert budget < sum(estimates)
    results, answers, stats, _ = serve(reqs, sf.ServerOptions(memory_budget=budget, batch_max_dofs=BATCH_MAX_DOFS))
    assert stats["completed"] == len(reqs)
    assert stats["peak_reserved_bytes"] <= budget
    assert stats["reserved_bytes"] == 0
    assert all(r.status == sf.Status.OK for r in results)
    assert any(r.queue_seconds > 0.0 for r in results)
