"""Benchmark: the 606k-DOF gate plate solve on B200.

Workload (the gate-size plate): 100 x 100 x 0.8 mm on a 100 x 100 x 2 hex grid, six Tet10 per hex
(120,000 elements, 202,005 nodes, 603,000 free DOFs), E = 2.0 GPa, nu = 0.35, edge x = 0 clamped,
0.01 MPa pressure on the top face, solved to a relative residual of 1e-8 with the block
smoothed-aggregation V-cycle (f32 hierarchy and vectors) inside FP64 flexible CG. Every input is
generated here (synthetic, seeded by construction: the structured box builder).

A step is one complete conjugate gradient solve of the plate on the device-resident matrix and
hierarchy (restart from a zero estimate, iterate to convergence). `value` is solves per second
over all ranks; `e2e` is the same metric through the public API from the plate's description: mesh
generated on the device (host copies for the model), model, device assembly, setup, solve,
displacements back to the host. Under torchrun every
rank runs its own replica (the solve does not shard): scaling is weak.

--impl reference times the reference's CPU path (the bit-exact restatement in oracle/): each step
is one complete solve of the same plate through the reference's own sequence (assembly, multigrid
setup, conjugate gradient to convergence; iterations counted live), in the reference's default
precision (SingleStorage: f32-stored hierarchy, f64 vectors), on every host core.

The main line's `cpu_baseline` is the FP64 oracle solve the answers are checked against (Double
precision, requested 1e-12, which stops at its rounding floor): one complete solve at the
reference's default thread count, timed, with one-thread figures for the per-iteration work beside
it. Its displacements give `oracle_check`: the mixed and FP64 device answers' relative L2 and
nodal von Mises differences from the oracle's.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SIZE = (100.0, 100.0, 0.8)
DIVISIONS = (100, 100, 2)
YOUNGS, POISSON = 2000.0, 0.35
PRESSURE = 0.01
TOLERANCE = 1e-8
METRIC = "606k-DOF plate solve throughput (mixed-precision V-cycle PCG)"
UNIT = "solves/s"
ORACLE_TOLERANCE = 1e-12  # the FP64 oracle answers are checked against
ONE_THREAD_REPEATS = 3


def workload_config():
    return {"workload": "gate plate 100x100x0.8 mm, 100x100x2 hex x 6 Tet10, 603,000 free DOFs, "
                        "E 2.0 GPa nu 0.35, x=0 clamped, 0.01 MPa top pressure, rel. residual 1e-8 requested; "
                        "f64 cannot resolve 1e-8 for this plate, so every solve stops at its rounding floor "
                        "(true relative residual about 5.3e-6, reported in relative_residual)",
            "elements": 120000, "free_dofs": 603000, "precision": "f32 V-cycle in FP64 flexible CG",
            "l2": "inputs larger than L2 (f32 fine operator 207.6 MB, f64 system 394 MB)",
            "parallelism": "replicas"}


def host_cores():
    return len(os.sched_getaffinity(0))


def build_model(sf, device=None):
    """The gate plate's mesh and model; the mesh generated on CUDA device `device` when given."""
    mesh = sf.box_tet_mesh((0.0, 0.0, 0.0), SIZE, DIVISIONS, device)
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(YOUNGS, POISSON))
    model.fix_nodes(np.nonzero(np.abs(nodes[:, 0]) < 1e-9)[0])
    # the top faces (all three corners at z = thickness), as one array in boundary-face order
    faces = mesh.boundary_face_array()
    top = np.all(np.abs(nodes[faces["nodes"][:, :3], 2] - SIZE[2]) < 1e-9, axis=1)
    model.add_face_tractions(faces[top], (0.0, 0.0, -PRESSURE))
    return mesh, model


def options(sf, precision, device):
    return sf.StudyOptions(pcg=sf.PcgOptions(tolerance=TOLERANCE),
                           preconditioner=sf.MultigridOptions(precision=precision), device=device)


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the dominant kernel from its committed ncu summary, when present."""
    path = os.path.join(ROOT, "profiles", "cheb_step_fine_gate_plate.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    return None


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.build()
    return O


def oracle_plate(O, precision, tolerance):
    mesh = O.Mesh.box(SIZE, DIVISIONS)
    nodes = mesh.nodes()
    faces = O.faces_on_plane(mesh, 2, SIZE[2], nodes)
    return O.Study(mesh, O.uniform(YOUNGS, POISSON), O.default_options(tolerance=tolerance, precision=precision),
                   O.nodes_on_plane(nodes, 0, 0.0), faces, [[0.0, 0.0, -PRESSURE]] * len(faces))


def oracle_solve(O, precision, tolerance, threads):
    """One complete solve of the plate by the oracle: assembly, multigrid setup and conjugate
    gradient to convergence, timed on the host clock. Returns (seconds, study, progress, phases)."""
    O.set_threads(threads)
    t0 = time.perf_counter()
    study = oracle_plate(O, precision, tolerance)
    t1 = time.perf_counter()
    pr = study.solve()
    t2 = time.perf_counter()
    if pr.status != 1:
        raise RuntimeError(f"oracle solve did not converge: status {pr.status}")
    return t2 - t0, study, pr, {"build_seconds": t1 - t0, "solve_seconds": t2 - t1}


def per_iteration_work(O, study, threads, repeats=ONE_THREAD_REPEATS):
    """Seconds for the work of one conjugate gradient iteration at `threads` host threads: one FP64
    system product and one V-cycle of the oracle's hierarchy, measured `repeats` times (median)."""
    O.set_threads(threads)
    r = np.random.default_rng(0).standard_normal(study.n)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        study.system_multiply(r)
        study.precondition(r)
        times.append(time.perf_counter() - t0)
    return statistics.median(times)


def cpu_baseline_fp64():
    """The FP64 oracle solve (Double, requested 1e-12, stopping at its rounding floor) of the plate at
    the reference's default thread count clamp(logical / 2, 1, 8), complete and timed; one-thread
    figures for one iteration's work beside it. Returns (baseline dict, oracle study)."""
    O = _oracle()
    threads = O.default_threads()
    seconds, study, pr, phases = oracle_solve(O, O.DOUBLE, ORACLE_TOLERANCE, threads)
    work_default = per_iteration_work(O, study, threads)
    work_one = per_iteration_work(O, study, 1)
    base = {"value": 1.0 / seconds, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one complete FP64 solve by the oracle (C++ restatement, Double, requested {ORACLE_TOLERANCE:g}): "
                      f"assembly + setup {phases['build_seconds']:.2f} s, {pr.iteration} CG iterations "
                      f"{phases['solve_seconds']:.2f} s to the rounding floor (relative residual "
                      f"{pr.relative_residual:.2e}); {seconds:.1f} s",
            "iterations": int(pr.iteration), "relative_residual": pr.relative_residual,
            "seconds_per_solve": seconds, **phases,
            "iteration_work_seconds": {"what": "one FP64 system product plus one V-cycle (median of "
                                               f"{ONE_THREAD_REPEATS}), measured",
                                       f"threads_{threads}": work_default, "threads_1": work_one}}
    return base, study


def run_reference(args, rank, world):
    """The reference's CPU path on the host cores: each step one complete solve of the plate in the
    reference's default precision (SingleStorage) to the requested 1e-8, iterations counted live."""
    if rank != 0:
        return 0
    O = _oracle()
    threads = host_cores()
    seconds, iterations = [], []
    for i in range(args.warmup + args.steps):
        dt, study, pr, phases = oracle_solve(O, O.SINGLE_STORAGE, TOLERANCE, threads)
        del study
        gc.collect()
        if i >= args.warmup:
            seconds.append(dt)
            iterations.append(int(pr.iteration))
    secs = statistics.mean(seconds)
    value = 1.0 / secs
    sample = (f"{args.steps} complete solve(s) by the oracle (C++ restatement of the reference's CPU path, "
              f"SingleStorage, requested {TOLERANCE:g}): assembly, setup and {iterations[-1]} CG iterations each, "
              f"{secs:.1f} s per solve (min {min(seconds):.1f}, max {max(seconds):.1f})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 vectors / f32-stored hierarchy (SingleStorage)",
            "data": "synthetic",
            "config": {**workload_config(), "precision": "the reference's default: SingleStorage hierarchy (f32 values, "
                                                         "f64 cycle arithmetic) in standard FP64 CG"},
            "iterations": iterations[-1],
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def timed_solves(torch, study, stream, steps):
    """Solves `steps` times on the resident system; CUDA events on the study's stream."""
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    its = []
    start.record(stream)
    for _ in range(steps):
        study.resolve()
        out = study.solve()
        its.append(out.progress.iteration)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end), its, out


def run_mine(args, rank, world):
    import torch

    import solidfem_b200 as sf

    from replicas import ReplicaGroup

    group = ReplicaGroup.from_env("nccl")
    device = group.local_rank
    torch.cuda.set_device(device)

    def barrier():
        group.barrier()
        torch.cuda.synchronize()

    mesh, model = build_model(sf)
    # --- e2e through the public API from the plate's description to displacements on the host:
    # the mesh generated on the device (its arrays copied back for the host-side model), the model,
    # the study (assembly and setup), the solve and the displacements read back. The reference arm
    # times the same span (mesh, assembly, setup, iterations).
    def e2e_step():
        t0 = time.perf_counter()
        msh, m = build_model(sf, device)
        st = sf.StaticStudy.new(m, options(sf, sf.Precision.MIXED, device))
        out = st.solve()
        d = st.displacements()
        t1 = time.perf_counter()
        timing = st.device_timing()
        # the generated mesh's host copies: nodes, ten-node tets, corner tets, boundary faces
        timing["mesh_d2h_bytes"] = (24 * msh.node_count() + 56 * msh.tet_count() +
                                    32 * len(msh.boundary_face_array()))
        return t1 - t0, timing, out, d, st

    e2e_step()  # warm-up: CUDA context, module load, allocator
    e2e_steps = max(1, min(args.steps, 5))
    barrier()
    e2e_times, h2d, d2h = [], 0, 0
    study = None
    for _ in range(e2e_steps):
        # The previous step's study is released before the clock starts, so its device memory is
        # not freed inside the next timed region.
        study = None
        gc.collect()
        dt, timing, out_e2e, disp_e2e, study = e2e_step()
        e2e_times.append(dt)
        h2d, d2h = timing["h2d_bytes"], timing["d2h_bytes"] + timing["mesh_d2h_bytes"] + disp_e2e.nbytes
    barrier()
    # Median of the steps: host phases (pattern, aggregation, layouts) share the box's cores with
    # other tenants, and a step that met contention is listed in `samples` rather than averaged in.
    e2e_local = statistics.median(e2e_times)
    e2e_value = group.rate(1, e2e_local)
    e2e_sec = group.max(e2e_local)
    rep = study.report()

    # --- value: device-resident solves of the mixed path.
    stream = torch.cuda.ExternalStream(study.stream(), device=torch.device("cuda", device))
    for _ in range(args.warmup):
        study.resolve()
        study.solve()
    launches0 = study.device_timing()["kernel_launches"]
    barrier()
    with Clocks(device) as clocks:
        ms, its, out = timed_solves(torch, study, stream, args.steps)
    barrier()
    launches = study.device_timing()["kernel_launches"] - launches0
    value = group.rate(args.steps, ms / 1000.0)
    ms = group.max(ms)
    clock = clocks.summary()
    ms_per_step = ms / args.steps
    x_mixed = study.displacements()

    # --- the plain FP64 path (Precision::Double semantics) for the mixed-vs-FP64 comparison.
    double = sf.StaticStudy.new(model, options(sf, sf.Precision.DOUBLE, device))
    double.solve()
    dstream = torch.cuda.ExternalStream(double.stream(), device=torch.device("cuda", device))
    barrier()
    dms, dits, dout = timed_solves(torch, double, dstream, max(1, min(args.steps, 3)))
    barrier()
    dms = group.max(dms) / max(1, min(args.steps, 3))
    x_double = double.displacements()
    diff = float(np.linalg.norm(x_mixed - x_double) / np.linalg.norm(x_double))

    # --- roofline of the dominant kernel: the finest level's fused Chebyshev step, timed live.
    kt = study.time_kernel(sf.Kernel.CHEBYSHEV_STEP, 50)
    st = study.time_kernel(sf.Kernel.SYSTEM_PRODUCT, 50)
    peak, peak_kind = measured_peak()
    achieved = kt["bytes_per_launch"] / (kt["ms_per_launch"] * 1e-3) / 1e9
    traffic = ncu_traffic()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 cycle / f64 outer", "data": "synthetic (structured box mesh)",
            "config": workload_config(),
            "iterations": its[-1], "relative_residual": out.progress.relative_residual,
            "at_rounding_floor": out.progress.at_rounding_floor,
            "fp64_path": {"ms_per_step": dms, "iterations": dout.progress.iteration,
                          "relative_residual": dout.progress.relative_residual,
                          "mixed_speedup": dms / ms_per_step, "mixed_vs_fp64_rel_l2": diff},
            "setup": {"assembly_seconds": rep["assembly_seconds"], "preconditioner_seconds": rep["preconditioner_seconds"],
                      "levels": rep["mg_levels"], "operator_complexity": rep["mg_operator_complexity"]},
            "roofline": {"bound": "hbm", "kernel": "sell_cheb_kernel<float,float,3> (finest level, fused Chebyshev step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "bytes_per_launch": kt["bytes_per_launch"], "ms_per_launch": kt["ms_per_launch"],
                         "system_product_gbs": st["bytes_per_launch"] / (st["ms_per_launch"] * 1e-3) / 1e9},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "span": "plate description -> mesh generated on the device (host copies) -> model -> study "
                            "(assembly, setup) -> solve -> displacements on the host",
                    "seconds_per_step": e2e_sec, "samples": [round(t, 4) for t in e2e_times]},
            "gpu_launches": launches, "clocks": clock}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, ref = cpu_baseline_fp64()
        line["cpu_baseline"] = base
        line["oracle_check"] = oracle_check(study, double, ref, x_mixed, x_double)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del study, double
    group.close()
    return 0


def oracle_check(mixed, double, ref, x_mixed, x_double):
    """The device answers against the FP64 oracle's: displacement relative L2 and the largest nodal
    von Mises difference relative to the largest von Mises (the correctness bar is 1e-8 and 1e-6)."""
    xr = ref.displacements()
    _, vm_ref = ref.recover()
    vm_scale = float(np.max(np.abs(vm_ref)))
    out = {"oracle": "FP64 oracle solve of the same plate (the cpu_baseline run)", "l2_bar": 1e-8, "von_mises_bar": 1e-6}
    for name, st, x in (("mixed", mixed, x_mixed), ("fp64", double, x_double)):
        vm = st.solution().nodal_von_mises
        out[f"{name}_vs_oracle_rel_l2"] = float(np.linalg.norm(x - xr) / np.linalg.norm(xr))
        out[f"{name}_vs_oracle_von_mises"] = float(np.max(np.abs(vm - vm_ref)) / vm_scale)
    return out


def run_profile(args):
    """One warm and one further resident solve of the mixed path, for profilers (no JSON line)."""
    import solidfem_b200 as sf

    precision = sf.Precision.DOUBLE if args.profile == "double" else sf.Precision.MIXED
    _, model = build_model(sf)
    study = sf.StaticStudy.new(model, options(sf, precision, 0))
    for _ in range(2):
        study.resolve()
        out = study.solve()
    print(f"profile {precision.name}: {out.progress.iteration} iterations, residual {out.progress.relative_residual:.3e}, "
          f"{study.device_timing()['step_ms']:.1f} ms")
    return 0


def profile_extras(sf, torch, tol, note):
    """The kernels the other profiled paths never launch: mesh generation on the device (the gate
    plate's box, a hollow part grid, a study's traction load from a generated mesh), quadrature-point
    positions for a material field, the degree-1 smoother's plain add, and the energy products of a
    row-group system product."""
    plate = sf.box_tet_mesh((0.0, 0.0, 0.0), SIZE, DIVISIONS, 0)
    lines = [[40.0 * i / 160 for i in range(161)], [12.0 * j / 24 for j in range(25)], [12.0 * k / 24 for k in range(25)]]
    sf.part_tet_mesh(*lines, wall_cells=2, device=0)
    pn = plate.nodes()
    pm = sf.Model(plate, sf.Material(YOUNGS, POISSON))
    pm.fix_nodes(np.nonzero(np.abs(pn[:, 0]) < 1e-9)[0])
    pf = plate.boundary_face_array()
    pm.add_face_tractions(pf[np.all(np.abs(pn[pf["nodes"][:, :3], 2] - SIZE[2]) < 1e-9, axis=1)], (0.0, 0.0, -PRESSURE))
    sf.StudyBuilder(pm, options(sf, sf.Precision.MIXED, 0))  # numbering, pattern, device load
    m = sf.box_tet_mesh((0.0, 0.0, 0.0), (10.0, 1.0, 1.0), (20, 4, 4))
    nd = m.nodes()
    model = sf.Model(m, lambda pos: sf.Material(200000.0 if pos[0] < 5.0 else 100000.0, 0.3))
    model.fix_nodes(np.nonzero(np.abs(nd[:, 0]) < 1e-9)[0])
    faces = m.boundary_face_array()
    end = np.all(np.abs(nd[faces["nodes"][:, :3], 0] - 10.0) < 1e-9, axis=1)
    model.add_face_tractions(faces[end], (0.0, 3.0, -7.0))
    st = sf.StaticStudy.new(model, sf.StudyOptions(
        pcg=sf.PcgOptions(tolerance=tol or 1e-9),
        preconditioner=sf.MultigridOptions(coarse_dofs=100, smoother_degree=1, precision=sf.Precision.DOUBLE)))
    note("extras", st, st.solve())
    k = st.report()["free_dofs"]
    xs = torch.from_numpy(np.random.default_rng(1).standard_normal((2, k))).to("cuda:0")
    ys = torch.empty_like(xs)
    es = torch.empty(2, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    st.energy_products(xs.data_ptr(), ys.data_ptr(), es.data_ptr(), 2)
    torch.cuda.synchronize()
    return 0


def run_profile_paths(args):
    """Every kernel family of the library once, for a profiler's launch list (no JSON line): the gate
    plate's study creation (mesh upload, assembly, multigrid setup), one mixed and one FP64 solve,
    the stress recovery, the energy products and the coarse-tail cluster launch; then small studies
    for the batched grids, the Jacobi preconditioner and prescribed displacements. `--profile-cells`
    scales the plate (the gate plate has 100 cells a side); `--profile-iterations` and
    `--profile-tolerance` shorten the solves, for captures that collect more than the launch times."""
    import torch

    import solidfem_b200 as sf

    torch.cuda.set_device(0)
    cells = args.profile_cells
    tol = args.profile_tolerance

    def opts(precision):
        o = options(sf, precision, 0)
        if tol:
            o.pcg.tolerance = tol
        return o

    mesh = sf.box_tet_mesh((0.0, 0.0, 0.0), SIZE, (cells, cells, 2))
    nodes = mesh.nodes()

    def plate(extra=None):
        model = sf.Model(mesh, sf.Material(YOUNGS, POISSON))
        model.fix_nodes(np.nonzero(np.abs(nodes[:, 0]) < 1e-9)[0])
        faces = mesh.boundary_face_array()
        top = np.all(np.abs(nodes[faces["nodes"][:, :3], 2] - SIZE[2]) < 1e-9, axis=1)
        model.add_face_tractions(faces[top], (0.0, 0.0, -PRESSURE))
        if extra:
            extra(model)
        return model

    def note(name, study, out):
        print(f"profile {name}: {out.progress.iteration} iterations, residual {out.progress.relative_residual:.3e}, "
              f"{study.device_timing()['step_ms']:.1f} ms", flush=True)

    if args.profile_extras:
        return profile_extras(sf, torch, tol, note)

    def run(study):
        # --profile-iterations: a few iterations of each plate solve (the stress recovery then runs on
        # the small converged studies below)
        return study.step(args.profile_iterations) if args.profile_iterations else study.solve()

    mixed = sf.StaticStudy.new(plate(), opts(sf.Precision.MIXED))
    note("mixed", mixed, run(mixed))
    if not args.profile_iterations:
        mixed.solution()
    n = mixed.report()["free_dofs"]
    xs = torch.from_numpy(np.random.default_rng(0).standard_normal((2, n))).to("cuda:0")
    ys = torch.empty_like(xs)
    es = torch.empty(2, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    mixed.energy_products(xs.data_ptr(), ys.data_ptr(), es.data_ptr(), 2)
    torch.cuda.synchronize()
    del mixed
    gc.collect()
    double = sf.StaticStudy.new(plate(), opts(sf.Precision.DOUBLE))
    note("double", double, run(double))
    del double
    gc.collect()
    tail_opts = opts(sf.Precision.MIXED)
    tail_opts.coarse_tail = True
    tail = sf.StaticStudy.new(plate(), tail_opts)
    note("coarse tail", tail, run(tail))
    del tail
    gc.collect()

    def small(div, precision, batchable=False, prescribe=False, jacobi=False):
        m = sf.box_tet_mesh((0.0, 0.0, 0.0), (10.0, 1.0, 1.0), div)
        nd = m.nodes()
        model = sf.Model(m, sf.Material(200000.0, 0.3))
        model.fix_nodes(np.nonzero(np.abs(nd[:, 0]) < 1e-9)[0])
        faces = m.boundary_face_array()
        end = np.all(np.abs(nd[faces["nodes"][:, :3], 0] - 10.0) < 1e-9, axis=1)
        model.add_face_tractions(faces[end], (0.0, 3.0, -7.0))
        if prescribe:
            tip = np.nonzero(np.abs(nd[:, 0] - 10.0) < 1e-9)[0]
            for node in tip[:4]:
                model.prescribe_displacement(int(node), 2, -0.01)
        pre = sf.Jacobi() if jacobi else sf.MultigridOptions(coarse_dofs=100, precision=precision)
        return sf.StaticStudy.new(model, sf.StudyOptions(pcg=sf.PcgOptions(tolerance=tol or 1e-9), preconditioner=pre,
                                                         batchable=batchable))

    batch = [small(d, sf.Precision.MIXED, batchable=True) for d in ((24, 4, 4), (30, 5, 5), (36, 6, 6))]
    res = sf.solve_batch(batch)
    print("profile batch:", [r[0].progress.iteration for r in res], flush=True)
    jacobi = small((20, 4, 4), None, jacobi=True)
    note("jacobi", jacobi, run(jacobi))
    prescribed = small((20, 4, 4), sf.Precision.DOUBLE, prescribe=True)
    note("prescribed", prescribed, prescribed.solve())
    if args.profile_iterations:
        prescribed.solution()
    return 0


def percentile(values, q):
    v = sorted(values)
    if not v:
        return None
    k = (len(v) - 1) * q
    lo, hi = int(k), min(int(k) + 1, len(v) - 1)
    return v[lo] + (v[hi] - v[lo]) * (k - lo)


def run_block(args):
    """Config 4: the 60 mm two-material printed block (60^3 hexes x 6 Tet10, 5.27M free DOFs): shell
    E 2.4 GPa nu 0.36 within 2 mm of the surface, core E 0.8 GPa nu 0.30, z = 0 clamped, 0.5 MPa
    x-shear on z = 60, mixed-precision and plain FP64 device-resident solves to 1e-8, the device FP64
    assembly timed on its own, and the whole study end to end through the public API from the
    block's description (mesh generated on the device)."""
    import torch

    import solidfem_b200 as sf

    torch.cuda.set_device(0)
    n = args.block_cells

    def model(device=None):
        mesh = sf.box_tet_mesh((0.0, 0.0, 0.0), (60.0, 60.0, 60.0), (n, n, n), device)
        nodes = mesh.nodes()
        m = sf.Model(mesh, sf.ShellCore(sf.Material(2400.0, 0.36), sf.Material(800.0, 0.30), (0.0, 0.0, 0.0),
                                        (60.0, 60.0, 60.0), 2.0))
        m.fix_nodes(np.flatnonzero(nodes[:, 2] == 0.0))
        faces = mesh.boundary_face_array()
        top = np.all(nodes[faces["nodes"][:, :3], 2] == 60.0, axis=1)
        m.add_face_tractions(faces[top], (0.5, 0.0, 0.0))
        return mesh, m

    def resident(study, steps):
        stream = torch.cuda.ExternalStream(study.stream(), device=torch.device("cuda", 0))
        study.resolve()
        study.solve()
        ms, its, out = timed_solves(torch, study, stream, steps)
        return ms / steps, out

    out = {}
    model(0)  # context and module load outside the clock
    for name, precision in (("mixed", sf.Precision.MIXED), ("fp64", sf.Precision.DOUBLE)):
        # end to end from the block's description: mesh generated on the device, model, study, solve
        t0 = time.perf_counter()
        mesh, m = model(0)
        st = sf.StaticStudy.new(m, options(sf, precision, 0))
        res = st.solve()
        d = st.displacements()
        e2e = time.perf_counter() - t0
        rep, tim = st.report(), st.device_timing()
        ms, o = resident(st, max(1, min(args.steps, 5)))
        out[name] = {"ms_per_solve": ms, "iterations": o.progress.iteration,
                     "relative_residual": o.progress.relative_residual, "converged": o.kind == sf.Outcome.CONVERGED,
                     "e2e_seconds": e2e, "device_assembly_ms": tim["assembly_ms"],
                     "host_assembly_and_pattern_seconds": rep["assembly_seconds"],
                     "setup_seconds": rep["preconditioner_seconds"], "levels": rep["mg_levels"],
                     "operator_complexity": rep["mg_operator_complexity"], "free_dofs": rep["free_dofs"]}
        if name == "mixed":
            x_mixed = d
        else:
            out["mixed_vs_fp64_rel_l2"] = float(np.linalg.norm(x_mixed - d) / np.linalg.norm(d))
        del st
        gc.collect()
    line = {"metric": "5.3M-DOF printed block solve time (mixed-precision V-cycle PCG)",
            "value": out["mixed"]["ms_per_solve"], "unit": "ms", "higher_is_better": False, "n_gpus": 1,
            "config": {"workload": f"printed block 60 mm, {n}^3 hex x 6 Tet10, shell/core, z=0 clamped, "
                                   "0.5 MPa x-shear on top, rel. residual 1e-8"},
            "mixed": out["mixed"], "fp64": out["fp64"],
            "mixed_speedup": out["fp64"]["ms_per_solve"] / out["mixed"]["ms_per_solve"],
            "mixed_vs_fp64_rel_l2": out["mixed_vs_fp64_rel_l2"], "data": "synthetic (structured box mesh)"}
    print(json.dumps(line))
    return 0


def run_serving(args):
    """The serving stream (512 mixed bar / tube / plate requests, Poisson arrivals at 20/s, seed 0)
    through the serving loop: paced at the arrivals with the models built first (meshes generated
    on the device; the host-mesh build time is reported beside it), paced with each request's mesh
    and model generated on the device at its arrival (inside its latency), and all submitted at
    once; then the same stream through serial plain FP64 GPU solves. Under
    torchrun every rank serves its round-robin share of the stream on its own GPU (one server per
    GPU, no collective on the data path); rates are over all ranks, latencies pooled."""
    import concurrent.futures

    import torch

    import solidfem_b200 as sf
    from solidfem_b200 import workloads as W
    from replicas import ReplicaGroup

    group = ReplicaGroup.from_env("nccl")
    device = group.local_rank
    torch.cuda.set_device(device)
    stream = W.serving_stream(count=args.requests, rate=args.rate)
    reqs = group.shard(stream)

    def build_all(dev):
        # every request's mesh and model, meshes generated on the device (dev) or on the host (None)
        with concurrent.futures.ThreadPoolExecutor(max_workers=8) as pool:
            return list(pool.map(lambda r: W.build_model(r, device=dev), reqs))

    W.build_model(reqs[0], device=device)  # context and module load outside the clocks
    t0 = time.perf_counter()
    built = build_all(None)
    prep_host = group.max(time.perf_counter() - t0)
    del built
    gc.collect()
    t0 = time.perf_counter()
    built = build_all(device)
    prep = group.max(time.perf_counter() - t0)

    def opts(precision):
        return sf.StudyOptions(pcg=sf.PcgOptions(tolerance=TOLERANCE),
                               preconditioner=sf.MultigridOptions(precision=precision), device=device)

    # warm-up: context, module load
    w = sf.StaticStudy.new(W.build_model(reqs[0])[1], opts(sf.Precision.MIXED))
    w.solve()
    del w
    gc.collect()

    def serve(models, paced):
        """models None: each request's mesh and model are generated on the device when it arrives,
        inside its latency (the latencies then run from arrival, not from submission)."""
        server = sf.Server(sf.ServerOptions(device=device, build_threads=args.build_threads))
        group.barrier()
        start = time.perf_counter()
        ids, waited = [], []
        for i, r in enumerate(reqs):
            delay = r.arrival - (time.perf_counter() - start)
            if paced and delay > 0:
                time.sleep(delay)
            mesh, model = models[i] if models is not None else W.build_model(r, device=device)
            waited.append(max(0.0, time.perf_counter() - start - r.arrival) if models is None else 0.0)
            ids.append((server.submit(model, opts(sf.Precision.MIXED)), mesh.node_count()))
        results = [server.wait(rid) for rid, _ in ids]
        for res, w in zip(results, waited):
            res.latency_seconds += w
        makespan = time.perf_counter() - start
        stats = server.stats()
        for rid, n in ids:
            try:
                server.take(rid, n)
            except sf.SolidfemError:
                pass
        server.close()
        return results, makespan, stats

    def pooled(results, makespan, stats):
        lat = group.gather([r.latency_seconds for r in results])
        batches = group.sum(stats["batches"])
        batched = group.sum(stats["batched_requests"])
        return {"solves_per_s": group.rate(len(results), makespan), "makespan_s": group.max(makespan),
                "p50_latency_s": percentile(lat, 0.5), "p99_latency_s": percentile(lat, 0.99),
                "failed": int(group.sum(sum(1 for r in results if r.status != sf.Status.OK))),
                "batched_requests": int(batched), "batches": int(batches),
                "mean_batch_size": batched / batches if batches else 0.0,
                "peak_reserved_gb": group.max(stats["peak_reserved_bytes"]) / 1e9}

    results, makespan, stats = serve(built, True)
    mine = pooled(results, makespan, stats)
    mine.update({"iterations_mean": statistics.mean(group.gather([r.outcome.progress.iteration for r in results])),
                 "build_seconds_sum": group.sum(sum(r.build_seconds for r in results)),
                 "solve_seconds_sum": group.sum(sum(r.solve_seconds for r in results)),
                 "queue_seconds_mean": statistics.mean(group.gather([r.queue_seconds for r in results])),
                 "failures": sorted(set(group.gather(
                     [f"{r.status.name}: {r.message}" for r in results if r.status != sf.Status.OK])))})
    del built
    gc.collect()
    # each request's mesh and model generated on the device at its arrival, inside its latency
    in_request = pooled(*serve(None, True))
    mine["prep_in_request"] = {k: in_request[k] for k in ("solves_per_s", "makespan_s", "p50_latency_s",
                                                           "p99_latency_s", "failed", "mean_batch_size")}
    gc.collect()
    # the same requests all submitted at once: the loop's capacity rather than the arrival rate
    built = build_all(device)
    saturated = pooled(*serve(built, False))
    mine["saturated"] = {k: saturated[k] for k in ("solves_per_s", "makespan_s", "p50_latency_s", "p99_latency_s",
                                                   "failed", "mean_batch_size", "peak_reserved_gb")}
    del built
    gc.collect()

    config = {"workload": f"serving stream: {len(stream)} bar/tube/plate requests, Poisson {args.rate:g}/s, seed 0, "
                          "10k-600k DOF log-uniform, rel. residual 1e-8, HBM budget 150 GB, "
                          "requests under 100k DOF batched",
              "build_threads": args.build_threads, "model_prep_seconds": prep,
              "model_prep_seconds_host_meshes": prep_host,
              "parallelism": f"replicas: {group.world} server(s), round-robin request shares"}
    if args.no_serial:
        if group.leader:
            print(json.dumps({"metric": "served solves/s", "value": mine["solves_per_s"], "unit": "solves/s",
                              "n_gpus": group.world, "config": config, "mine": mine}))
        group.close()
        return 0
    # serial plain FP64 GPU solves of the same stream, one at a time in arrival order
    built = build_all(device)
    group.barrier()
    start = time.perf_counter()
    lat, serial_failed = [], 0
    for r, (mesh, model) in zip(reqs, built):
        now = time.perf_counter() - start
        if now < r.arrival:
            time.sleep(r.arrival - now)
        st = sf.StaticStudy.new(model, opts(sf.Precision.DOUBLE))
        out = st.solve()
        st.displacements()
        serial_failed += out.kind != sf.Outcome.CONVERGED
        del st
        lat.append(time.perf_counter() - start - r.arrival)
    makespan = time.perf_counter() - start
    lat = group.gather(lat)
    serial = {"solves_per_s": group.rate(len(reqs), makespan), "makespan_s": group.max(makespan),
              "p50_latency_s": percentile(lat, 0.5), "p99_latency_s": percentile(lat, 0.99),
              "failed": int(group.sum(serial_failed))}
    line = {"metric": "served solves/s (mixed-size stream, continuous batching)", "value": mine["solves_per_s"],
            "unit": "solves/s", "n_gpus": group.world, "higher_is_better": True, "scaling": "strong",
            "config": config, "mine": mine, "serial_fp64": serial,
            "speedup_throughput": mine["solves_per_s"] / serial["solves_per_s"],
            "data": "synthetic (seeded request stream)"}
    if group.leader:
        print(json.dumps(line))
    group.close()
    return 0


def main():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["mine", "reference"], default="mine")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile", choices=["mixed", "double", "paths"], default=None,
                   help="mixed / double: two resident solves of the plate for a profiler; paths: every "
                        "kernel family once (creation, solves, recovery, batches, Jacobi, ...); then exit")
    p.add_argument("--profile-cells", type=int, default=100, help="paths: plate cells a side (100: the gate plate)")
    p.add_argument("--profile-iterations", type=int, default=0,
                   help="paths: run only this many iterations of each plate solve")
    p.add_argument("--profile-extras", action="store_true",
                   help="paths: only the kernels no other path launches")
    p.add_argument("--profile-tolerance", type=float, default=None,
                   help="paths: a looser relative residual, so each solve runs only a few iterations")
    p.add_argument("--workload", choices=["plate", "serving", "block"], default="plate",
                   help="plate: the 603k-DOF gate plate (default); serving: the mixed request stream; "
                        "block: the 5.3M-DOF printed block")
    p.add_argument("--block-cells", type=int, default=60, help="block: hex cells per side")
    p.add_argument("--requests", type=int, default=512, help="serving: requests in the stream")
    p.add_argument("--rate", type=float, default=20.0, help="serving: Poisson arrival rate, requests per second")
    p.add_argument("--build-threads", type=int, default=8, help="serving: host build threads")
    p.add_argument("--no-serial", action="store_true", help="serving: skip the serial FP64 comparison")
    args = p.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.profile == "paths":
        return run_profile_paths(args)
    if args.profile:
        return run_profile(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "block":
        return run_block(args) if rank == 0 else 0
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_mine(args, rank, world)


if __name__ == "__main__":
    sys.exit(main())
