"""The serving loop (sf_server) on a small mixed stream (needs a B200): every request's answer in
the mix equals its answer alone, batched and unbatched requests both, and the memory budget holds.
"""
import time

import numpy as np
import pytest

import solidfem_b200 as sf
from solidfem_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-8


def options():
    return sf.StudyOptions(pcg=sf.PcgOptions(tolerance=TOL),
                           preconditioner=sf.MultigridOptions(precision=sf.Precision.MIXED))


def stream():
    return W.serving_stream(count=12, rate=400.0, seed=7, dof_range=(4_000, 60_000))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def solo_answers(reqs):
    out = []
    for r in reqs:
        mesh, model = W.build_model(r)
        st = sf.StaticStudy.new(model, options())
        assert st.solve().kind == sf.Outcome.CONVERGED
        out.append(st.displacements())
    return out


def serve(reqs, server_options):
    server = sf.Server(server_options)
    try:
        models = [W.build_model(r) for r in reqs]
        start = time.perf_counter()
        ids = []
        for r, (mesh, model) in zip(reqs, models):
            delay = r.arrival - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            ids.append((server.submit(model, options()), mesh.node_count()))
        results = [server.wait(rid) for rid, _ in ids]
        answers = [server.take(rid, n) for rid, n in ids]
        return results, answers, server.stats()
    finally:
        server.close()


def test_served_answers_equal_solo_answers():
    reqs = stream()
    solo = solo_answers(reqs)
    results, answers, stats = serve(reqs, sf.ServerOptions(batch_max_dofs=30_000, build_threads=3))
    assert stats["completed"] == len(reqs)
    assert any(r.batched for r in results) and any(not r.batched for r in results)
    for r, res, a, s in zip(reqs, results, answers, solo):
        assert res.status == sf.Status.OK and res.outcome.kind == sf.Outcome.CONVERGED
        assert rel(a, s) <= 1e-6, (r.index, r.kind, res.batched, rel(a, s))
        assert res.latency_seconds >= res.solve_seconds >= 0.0


def test_a_burst_of_similar_requests_shares_batches():
    base = W.serving_stream(count=1, seed=3)[0]
    reqs = [W.Request(i, 0.0, "plate", 20_000 + 500 * i, 60.0 + i, 40.0, 1.0 + 0.1 * i, 2000.0 * (1 + i), 0.3,
                      100.0 + 10 * i) for i in range(8)]
    assert base.kind in W.KINDS
    solo = solo_answers(reqs)
    results, answers, stats = serve(reqs, sf.ServerOptions(build_threads=8))
    assert stats["completed"] == len(reqs)
    assert all(r.batched for r in results)
    assert max(r.batch_size for r in results) > 1, "no two requests shared a batch"
    for res, a, s in zip(results, answers, solo):
        assert res.status == sf.Status.OK
        assert rel(a, s) <= 1e-6


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
    results, answers, stats = serve(reqs, sf.ServerOptions(memory_budget=budget, batch_max_dofs=30_000))
    assert stats["completed"] == len(reqs)
    assert stats["peak_reserved_bytes"] <= budget
    assert stats["reserved_bytes"] == 0
    assert all(r.status == sf.Status.OK for r in results)
    assert any(r.queue_seconds > 0.0 for r in results)
