"""Benchmark: batched nonlinear magnetostatic solves per second on B200.

Workload (the nonlinear planar solve): 0.1 m square, 500 x 500 quads split into 2 P1
triangles (251,001 nodes / 500,000 triangles), interior nodes jittered by U(+/-0.3 h),
iron on the 24-point B = 2H/(200+H) table, a 5 mm magnet strip (mu_r 1.05, Hc 9e5 A/m,
seeded angle) and three series circuits at seeded currents U[-20, 20] A; Newton step gate
1e-6 with the reference's production options (inner PCG tolerance 1e-10 at the end).
One step = one batched nonlinear solve of --items samples sharing the mesh (different
currents).  Synthetic, seeded data; random currents per step and rank.

Arms:
  --impl ours       libfemmgpu through the C ABI.  ``value``: device-resident inputs
                    (fg_solve_batch_device, CUDA-event timed); ``e2e``: host buffers
                    through fg_solve_batch, H2D of currents and D2H of A, B, flux inside.
  --impl reference  the reference's CPU path (FEMM-GPU host assembler + FEMM 4.2 SSOR-PCG,
                    oracle/_ref) on all host threads; each step = one Newton iteration of
                    one sample per thread, samples restarted as they converge.

Forms (N = 1, rank 0; skipped with --no-forms): the same samples through block-Jacobi,
the FP32-inner mixed PCG (reliable updates) and the PCG started from the Newton iterate,
each with solves/s, iterations and its error against the plain FP64 solutions; and the
learned warm start on the axisymmetric plunger (about 100k nodes; --learned-train training
solves, 256 held-out samples) against the plain zero start; the rotor-stator sector
(--sector-samples samples sharing the mesh, per-sample currents and magnet strength); and
--hetero-meshes independent meshes of 5k-200k nodes in one multi-plan launch per Newton
step against solving them one plan at a time.

Multi-GPU: replicas only -- every rank solves its own batch, no collective on the data
path; ``value`` = all ranks' solves / max-over-ranks time (weak scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for sub in ("femm-gpu_b200", "oracle"):
    sys.path.insert(0, os.path.join(ROOT, sub))

METRIC = "nonlinear solves/sec & SpMV HBM GB/s; warm/mixed vs plain FP64 at 1e-8, 1 B200"
MESH_M = 500
SEED_MESH = 2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--items", type=int, default=8, help="samples per batched solve")
    p.add_argument("--mesh", type=int, default=MESH_M)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-forms", action="store_true", help="skip the mixed / block / learned forms")
    p.add_argument("--no-learned", action="store_true", help="skip the learned warm start form")
    p.add_argument("--learned-train", type=int, default=8192, help="training solves of the learned form")
    p.add_argument("--learned-held", type=int, default=4096, help="held-out samples of the learned form")
    p.add_argument("--sector-samples", type=int, default=1024, help="samples of the shared-geometry sector form")
    p.add_argument("--hetero-meshes", type=int, default=256, help="meshes of the heterogeneous-batch form")
    p.add_argument("--all-forms", action="store_true",
                   help="also the postprocess / tangent, streaming-worker and sliding-band forms")
    p.add_argument("--only-form", choices=["postprocess_tangent_sector", "streaming_worker", "sliding_band",
                                           "planar_2m", "reference_gpu", "learned", "sector", "hetero",
                                           "pcg_launch"],
                   help="run one form alone and print its JSON (profiling)")
    p.add_argument("--probe-mesh", type=int, default=MESH_M,
                   help="pcg_launch: planar square size m (0: the 40k-node rotor-stator sector)")
    p.add_argument("--probe-items", type=int, default=8, help="pcg_launch: samples per launch")
    p.add_argument("--probe-iterations", type=int, default=300, help="pcg_launch: CG iterations per launch")
    p.add_argument("--probe-launches", type=int, default=3, help="pcg_launch: launches timed")
    p.add_argument("--probe-one-reduction", action="store_true", help="pcg_launch: the one-reduction form")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def mesh_counts(model):
    """Free rows and CSR entries of a constraint-free planar mesh, counted with numpy from
    the triangles (used by both arms so their config keys agree)."""
    fixed = np.zeros(model.node_count, bool)
    fixed[model.dir_nodes] = True
    t = model.tri
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    e = e[~(fixed[e[:, 0]] | fixed[e[:, 1]])]
    e.sort(axis=1)
    edges = np.unique(e[:, 0].astype(np.int64) * model.node_count + e[:, 1]).size
    rows = int((~fixed).sum())
    return rows, rows + 2 * edges


def headline_config(model, mesh, world):
    """The config both arms print (the driver compares them key for key)."""
    rows, nnz = mesh_counts(model)
    return {"workload": f"nonlinear planar solve, jittered {mesh}x{mesh} quads ({model.node_count} nodes, "
                        f"{model.tri_count} triangles), iron B-H + PM strip + 3 circuits",
            "nodes": model.node_count, "triangles": model.tri_count, "rows": rows, "nnz": nnz,
            "precision": "fp64", "gates": "Newton step 1e-6, inner true residual 1e-10 (production options)",
            "l2": "flushed between timed GPU steps", "parallelism": f"replicas{world}"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def traffic_per_cg_iteration(workload):
    """DRAM bytes per CG iteration of the PCG kernel from the committed ncu capture of that
    workload (profiles/traffic.json; the capture's command is in the profile beside it)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None, None
    d = json.load(open(path)).get(workload)
    return (float(d["dram_bytes_per_cg_iteration"]), d["profile"]) if d else (None, None)


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 8:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def max_over_ranks(x, world, device):
    """The slowest rank's figure (replicas: every rank times its own batch), then a barrier."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def weak_value(world, items, steps, seconds):
    """Whole-job solves/s: every rank solves `items` samples per step."""
    return world * items * steps / seconds


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(model, items_seed, budget_threads=None, single_core=True):
    """Reference CPU path (oracle/_ref) on one full-size sample per host thread, plus one
    sample alone on one thread (single-core latency).  Returns the report and the
    reference's answers (currents, A, flux, status, Newton iterations) for the parity check."""
    import oracle as O
    from femm_gpu_b200 import meshes

    threads = budget_threads or os.cpu_count() or 1
    currents = meshes.seeded_currents(threads, model.circuit_count, 20.0, seed=items_seed)
    answers = None
    extra = {}
    if O.ref() is not None:
        t0 = time.perf_counter()
        a, flux, status, newton, calls, worst = O.ref_cpu_newton_batch(model, currents, threads=threads)
        dt = time.perf_counter() - t0
        kind = "reference"
        ok = int((status == 0).sum())
        answers = (currents, a, flux, status, newton)
        extra = {"max_true_residual": float(worst.max()), "newton_iterations_mean": float(newton.mean()),
                 "femm_pcg_calls_mean": float(calls.mean())}
        if single_core:
            t0 = time.perf_counter()
            O.ref_cpu_newton_batch(model, currents[:1], threads=1)
            extra["single_core_latency_s"] = time.perf_counter() - t0
    else:  # the C restatement, one Python thread per sample (ctypes releases the GIL)
        out = [None] * threads

        def run(i):
            out[i] = O.solve_batch(model, currents[i:i + 1])

        t0 = time.perf_counter()
        ths = [threading.Thread(target=run, args=(i,)) for i in range(threads)]
        [t.start() for t in ths]
        [t.join() for t in ths]
        dt = time.perf_counter() - t0
        kind = "port"
        ok = sum(1 for o in out if o[4][0].status == 0)
    report = {"value": threads / dt, "unit": "solves/s", "cores": threads, "kind": kind,
              "cpu_model": cpu_model(), "nproc": os.cpu_count(),
              "sample": f"{threads} full nonlinear solves of the {model.node_count}-node workload, "
                        f"one per host thread, {ok} converged, {dt:.1f} s wall", **extra}
    return report, answers


def parity_vs_reference(model, plan, answers):
    """The library's answers for the reference's own samples (same currents): relative
    2-norm errors of A and flux linkage, max |B| error relative to max |B|, statuses and
    Newton iteration counts."""
    import oracle as O

    currents, ra, rflux, rst, rnewton = answers
    got = plan.solve(currents)
    ea, ef, eb = [], [], []
    for i in range(len(currents)):
        ea.append(float(np.linalg.norm(got.a[i] - ra[i]) / np.linalg.norm(ra[i])))
        ef.append(float(np.linalg.norm(got.flux[i] - rflux[i]) / np.linalg.norm(rflux[i])))
        b1, b2, _ = O.finalize(model, ra[i])
        bmax = max(np.abs(b1).max(), np.abs(b2).max())
        eb.append(float(max(np.abs(got.b1[i] - b1).max(), np.abs(got.b2[i] - b2).max()) / bmax))
    return {"samples": len(currents), "a_rel_err_max": max(ea), "flux_rel_err_max": max(ef),
            "b_err_max_over_max_b": max(eb),
            "statuses_equal": bool(all(g.status == r for g, r in zip(got.info, rst))),
            "newton_iterations_equal": bool(all(g.iterations == r for g, r in zip(got.info, rnewton))),
            "reference": "the reference's host assembler + FEMM SSOR PCG (oracle/_ref), same currents"}


def run_ours(args, world, rank, local):
    import torch

    import femm_gpu_b200 as fg
    from femm_gpu_b200 import meshes

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    model = meshes.square_nonlinear(m=args.mesh, seed=SEED_MESH)
    plan = fg.Plan(model)
    k, N, E, Cc = args.items, plan.N, plan.E, plan.C
    dev = torch.device("cuda", local)
    opts = fg.production_options()
    stream = torch.cuda.current_stream(dev)
    out_a = torch.empty((k, N), dtype=torch.float64, device=dev)
    out_b1 = torch.empty((k, E), dtype=torch.float64, device=dev)
    out_b2 = torch.empty((k, E), dtype=torch.float64, device=dev)
    out_f = torch.empty((k, Cc), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    total = args.warmup + args.steps
    inputs = [torch.tensor(meshes.seeded_currents(k, Cc, 20.0, seed=100000 * rank + s), device=dev)
              for s in range(total)]
    torch.cuda.synchronize()

    def step(s):
        info = plan.solve_device(k, inputs[s].data_ptr(), options=opts, a_ptr=out_a.data_ptr(),
                                 b1_ptr=out_b1.data_ptr(), b2_ptr=out_b2.data_ptr(),
                                 flux_ptr=out_f.data_ptr(), stream=stream.cuda_stream)
        return info, plan.last_timing()

    for s in range(args.warmup):
        step(s)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    pcg_ms = 0.0
    pcg_its = 0
    item_its = 0
    launches = 0
    newton = 0
    statuses = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            flush.fill_(float(i))  # L2 flush between timed steps (outside the events)
            ev0[i].record(stream)
            info, t = step(args.warmup + i)
            ev1[i].record(stream)
            pcg_ms += t.pcg_ms
            pcg_its += t.pcg_iterations
            launches += t.kernel_launches
            newton += t.newton_iterations
            item_its += sum(x.linear_iterations for x in info)
            statuses += [x.status for x in info]
        torch.cuda.synchronize()
    ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1)), world, dev)
    value = weak_value(world, k, args.steps, ms / 1e3)

    # Roofline of the dominant kernel (the cooperative PCG).
    n, nnz = plan.rows, plan.nnz
    per_item = 8.0 * nnz + 104.0 * n  # values + vector traffic of one item's iteration
    shared = 4.0 * nnz + 4.0 * (n + 1)  # column indices + row structure, once per iteration
    alg_bytes = item_its * per_item + pcg_its * shared
    achieved = alg_bytes / (pcg_ms / 1e3) / 1e9 if pcg_ms > 0 else 0.0
    peak, peak_kind = peaks()
    # DRAM traffic of the PCG kernel from the committed ncu capture of this workload,
    # per launch of this run.
    traffic, traffic_src = None, None
    if args.mesh == MESH_M and k == 8:
        per_it, traffic_src = traffic_per_cg_iteration("square500_items8")
        if per_it is not None:
            traffic = per_it * pcg_its / max(1, newton)

    # End to end through the host-buffer C ABI (H2D currents, D2H A / B / flux / info).
    host_in = [meshes.seeded_currents(k, Cc, 20.0, seed=777000 + 100000 * rank + s) for s in range(args.steps)]
    host_out = plan.solve(host_in[0])  # warm the staging buffers; its host arrays are reused
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(args.steps):
        plan.solve(host_in[s], out=host_out)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e = {"value": weak_value(world, k, args.steps, e2e_s), "unit": "solves/s",
           "h2d_bytes_per_step": k * Cc * 8,
           "d2h_bytes_per_step": k * (N + 2 * E + Cc) * 8 + k * 40}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(model, args.mesh, world),
        "items_per_step": k, "solver": "fp64 Jacobi PCG (the drop-in form)",
        "e2e": e2e,
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "PcgKernel",
                     "traffic_source": (f"ncu capture of this workload, DRAM bytes per CG iteration x "
                                        f"iterations per launch ({traffic_src})") if traffic_src else None,
                     "algorithmic_bytes_per_launch": alg_bytes / max(1, newton),
                     "peak_source": peak_kind, "pcg_ms": pcg_ms, "pcg_iterations": pcg_its,
                     "item_pcg_iterations": item_its},
        "newton_iterations": newton,
        "pcg_shapes_autotuned": plan.pcg_shapes(),
        "statuses_ok": sum(1 for s in statuses if s == 0), "statuses_total": len(statuses),
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_forms:
        line["forms"] = run_forms(args, model, plan, dev, stream, flush, value)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], answers = cpu_baseline(model, items_seed=4242)
        if answers is not None:
            line["parity_vs_reference"] = parity_vs_reference(model, plan, answers)
            line["e2e_vs_cpu_baseline"] = e2e["value"] / line["cpu_baseline"]["value"]
    if "forms" in line:
        line["forms_summary"] = forms_summary(line["forms"])
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def forms_summary(forms):
    """The forms' key figures, printed last on the line so a truncated log keeps them."""
    out = {}

    def short(v):
        return float(f"{v:.4g}") if isinstance(v, float) else v

    def pick(name, d, *keys):
        if isinstance(d, dict):
            out[name] = {k: short(d[k]) for k in keys if k in d}

    for name in ("fp64_jacobi", "fp64_block8", "mixed_jacobi", "mixed_block8", "mixed_block8_from_iterate"):
        pick("planar_" + name, forms.get(name), "solves_per_s", "vs_fp64_jacobi", "pcg_iterations_per_item",
             "a_rel_err", "flux_rel_err")
    c4 = forms.get("planar_2m", {})
    for name, d in c4.items():
        pick("planar_2m_" + name, d, "solves_per_s", "vs_fp64_jacobi_k4", "pcg_gbs", "pcg_frac",
             "newton_iterations_per_item", "pcg_iterations_per_item", "a_rel_err", "b_rel_err", "flux_rel_err")
    sec = forms.get("shared_geometry_sector", {})
    for name, d in sec.items():
        pick("sector_" + name, d, "solves_per_s_e2e", "vs_chunk_by_chunk", "a_rel_err_vs_oracle",
             "flux_rel_err_vs_oracle", "newton_iterations_equal_oracle")
    pick("reference_gpu_executable", forms.get("reference_gpu"), "reference_gpu_solve_seconds",
         "ours_solve_seconds", "solve_speedup", "solve_flux_rel_err", "reference_gpu_batch_solves_per_s",
         "ours_batch_solves_per_s", "batch_speedup", "batch_flux_rel_err", "batch_torque_rel_err")
    pick("heterogeneous", forms.get("heterogeneous_meshes"), "meshes", "multi_solves_per_s",
         "one_plan_at_a_time_solves_per_s", "speedup", "a_rel_err_vs_single")
    lw = forms.get("learned_warm_start", {})
    for name, d in lw.items():
        pick("learned_" + name, d, "solves_per_s_e2e", "vs_fp64_zero_start", "vs_same_form_zero_start",
             "warm_starts_used",
             "newton_iterations_per_item", "pcg_iterations_per_item", "a_rel_err", "flux_rel_err")
    pick("sliding_band", forms.get("sliding_band"), "solves_per_s_e2e", "speedup_vs_cpu",
         "flux_rel_err_vs_reference")
    pick("worker", forms.get("streaming_worker"), "worker_solves_per_s", "speedup")
    return out


def time_device(plan, k, inputs, steps, warmup, dev, stream, flush):
    """Device-timed batched solves (CUDA events on the launching stream, L2 flushed
    between steps); returns solves/s, per-item info of the timed steps and their A."""
    import torch

    N, E, Cc = plan.N, plan.E, plan.C
    out_a = torch.empty((k, N), dtype=torch.float64, device=dev)
    out_f = torch.empty((k, Cc), dtype=torch.float64, device=dev)
    opts = None
    infos, a_all, f_all = [], [], []
    ms = 0.0
    for s in range(warmup + steps):
        if s >= warmup:
            flush.fill_(float(s))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        info = plan.solve_device(k, inputs[s].data_ptr(), options=opts, a_ptr=out_a.data_ptr(),
                                 flux_ptr=out_f.data_ptr(), stream=stream.cuda_stream)
        if s >= warmup:
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            infos += info
            a_all.append(out_a.cpu().numpy())
            f_all.append(out_f.cpu().numpy())
    return k * steps / (ms / 1e3), infos, np.concatenate(a_all), np.concatenate(f_all)


def run_forms(args, model, plan, dev, stream, flush, plain_value):
    """The three forms beside the plain FP64 method, at the same Newton and PCG gates:
    block-Jacobi, FP32-inner mixed precision (reliable updates) and the PCG started from the
    Newton iterate on the nonlinear planar workload; the learned warm start on the
    axisymmetric plunger (about 100k nodes), trained on FP64 solves of the plain method.
    Errors are relative 2-norms against the plain FP64 solutions of the same samples."""
    import torch

    import femm_gpu_b200 as fg
    from femm_gpu_b200 import meshes

    k, Cc = args.items, plan.C
    steps, warmup = 3, 1
    inputs = [torch.tensor(meshes.seeded_currents(k, Cc, 20.0, seed=555000 + s), device=dev)
              for s in range(warmup + steps)]
    ref_v, ref_info, ref_a, ref_f = time_device(plan, k, inputs, steps, warmup, dev, stream, flush)

    def err(a, b):
        return float(max(np.linalg.norm(a[i] - b[i]) / np.linalg.norm(b[i]) for i in range(len(b))))

    out = {"workload": "nonlinear planar solve (as value), same samples",
           "fp64_jacobi": {"solves_per_s": ref_v,
                           "pcg_iterations_per_item": float(np.mean([i.linear_iterations for i in ref_info]))}}
    for name, kw in (("fp64_block8", dict(preconditioner=1, block_size=8)),
                     ("mixed_jacobi", dict(precision=1)),
                     ("mixed_block8", dict(precision=1, preconditioner=1, block_size=8)),
                     ("mixed_block8_from_iterate", dict(precision=1, preconditioner=1, block_size=8,
                                                        from_iterate=True))):
        p = fg.Plan(model, **kw)
        v, info, a, f = time_device(p, k, inputs, steps, warmup, dev, stream, flush)
        out[name] = {"solves_per_s": v, "vs_fp64_jacobi": v / ref_v,
                     "pcg_iterations_per_item": float(np.mean([i.linear_iterations for i in info])),
                     "newton_iterations_per_item": float(np.mean([i.iterations for i in info])),
                     "a_rel_err": err(a, ref_a), "flux_rel_err": err(f, ref_f),
                     "all_converged": all(i.status == 0 for i in info)}
        p.close()
    out["planar_2m"] = planar_2m_form(dev, stream, flush)

    out["shared_geometry_sector"] = sector_form(args.sector_samples)
    out["heterogeneous_meshes"] = hetero_form(args.hetero_meshes)
    out["reference_gpu"] = reference_gpu_form(args.mesh)
    if not args.no_learned:
        out["learned_warm_start"] = learned_form(args.learned_train, args.learned_held)
    if args.all_forms:
        rng = np.random.default_rng(77)
        cur = rng.uniform(-15.0, 15.0, size=(64, 3))
        hcs = rng.uniform(8.5e5, 9.5e5, size=64) / 9.0e5
        out["postprocess_tangent_sector"] = postprocess_tangent_form(meshes.annular_sector(), cur, hcs, dev,
                                                                     stream, err)
        out["streaming_worker"] = worker_form()
        out["sliding_band"] = sliding_band_form()
    return out


def oracle_solves(models, currents):
    """The FP64 oracle (the C restatement) on one sample per model, one host thread each
    (ctypes releases the GIL): (A, flux, status, Newton iterations) per sample."""
    import oracle as O

    out = [None] * len(models)

    def run(i):
        a, _, _, f, info = O.solve_batch(models[i], currents[i:i + 1])
        out[i] = (a[0], f[0], info[0].status, info[0].iterations)

    ths = [threading.Thread(target=run, args=(i,)) for i in range(len(models))]
    [t.start() for t in ths]
    [t.join() for t in ths]
    return out


def max_rel(a, b):
    return float(max(np.linalg.norm(a[i] - b[i]) / np.linalg.norm(b[i]) for i in range(len(b))))


def sector_form(samples, check=8, fast_samples=256):
    """Shared geometry at scale: the rotor-stator sector (about 40k nodes, anti-periodic
    90-degree edges), `samples` samples with per-sample currents U[-15, 15] A and magnet
    Hc U[8.5e5, 9.5e5] A/m, solved by the plain FP64 Jacobi method through one
    fg_solve_batch call (chunks of 32 one after another, the library's default).  On the
    first `fast_samples` samples: chunk after chunk, all chunks advancing together (one
    multi-group PCG launch per Newton step, CUDA-graph replays), and the fast forms (block-Jacobi 8 and the PCG from the Newton iterate, in
    FP64 and with the FP32 inner solve).  Host-buffer API timing.  The first `check` samples
    are compared with the FP64 oracle solving each sample's own model."""
    import femm_gpu_b200 as fg
    from femm_gpu_b200 import meshes

    sector = meshes.annular_sector()
    rng = np.random.default_rng(77)
    cur = rng.uniform(-15.0, 15.0, size=(samples, 3))
    hc = rng.uniform(8.5e5, 9.5e5, size=samples)
    hcs = hc / 9.0e5
    t0 = time.perf_counter()
    ref = oracle_solves([meshes.annular_sector(hc=h) for h in hc[:check]], cur[:check])
    oracle_s = time.perf_counter() - t0
    ra = np.array([r[0] for r in ref])
    rf = np.array([r[1] for r in ref])
    out = {"workload": f"rotor-stator sector, {sector.node_count} nodes, anti-periodic 90-degree edges, "
                       f"{samples} samples with per-sample currents and magnet Hc; host-buffer API timing",
           "oracle_check_samples": check, "oracle_seconds": oracle_s,
           "oracle_all_converged": all(r[2] == 0 for r in ref)}
    saved = os.environ.get("FG_CHUNKS_TOGETHER")
    try:
        fast = dict(preconditioner=1, block_size=8, from_iterate=True)
        for name, kw, together, ks in (("fp64_jacobi", {}, "0", samples),
                                       ("fp64_jacobi_chunk_by_chunk_subset", {}, "0", fast_samples),
                                       ("fp64_jacobi_chunks_together_subset", {}, "2", fast_samples),
                                       ("fp64_block8_from_iterate_subset", fast, "0", fast_samples),
                                       ("mixed_block8_from_iterate_subset", dict(precision=1, **fast), "0",
                                        fast_samples)):
            os.environ["FG_CHUNKS_TOGETHER"] = together
            p = fg.Plan(sector, **kw)
            p.solve(cur[:64], hc_scale=hcs[:64], outputs=False)  # warm: workspaces and lanes
            t0 = time.perf_counter()
            r = p.solve(cur[:ks], hc_scale=hcs[:ks], outputs="a")
            dt = time.perf_counter() - t0
            t = p.last_timing()
            out[name] = {"samples": ks, "solves_per_s_e2e": ks / dt, "seconds": dt,
                         "newton_iterations_per_item": float(np.mean([i.iterations for i in r.info])),
                         "pcg_iterations_per_item": float(np.mean([i.linear_iterations for i in r.info])),
                         "pcg_launches": int(t.pcg_launches), "all_converged": all(i.status == 0 for i in r.info),
                         "a_rel_err_vs_oracle": max_rel(r.a[:check], ra),
                         "flux_rel_err_vs_oracle": max_rel(r.flux[:check], rf),
                         "newton_iterations_equal_oracle": all(r.info[i].iterations == ref[i][3] for i in range(check))}
            p.close()
    finally:
        if saved is None:
            os.environ.pop("FG_CHUNKS_TOGETHER", None)
        else:
            os.environ["FG_CHUNKS_TOGETHER"] = saved
    sub = out["fp64_jacobi_chunk_by_chunk_subset"]["solves_per_s_e2e"]
    for name in ("fp64_jacobi_chunks_together_subset", "fp64_block8_from_iterate_subset",
                 "mixed_block8_from_iterate_subset"):
        out[name]["vs_chunk_by_chunk"] = out[name]["solves_per_s_e2e"] / sub
    return out


def hetero_form(count):
    """Heterogeneous meshes: `count` jittered squares with node counts log-uniform in
    [5k, 200k], one sample each, in one multi-plan PCG launch per Newton step against the
    same solves one plan at a time.  Host-buffer API timing (plans built beforehand)."""
    import femm_gpu_b200 as fg
    from femm_gpu_b200 import meshes

    rng = np.random.default_rng(11)
    ns = np.exp(rng.uniform(np.log(5e3), np.log(2e5), size=count))
    models = [meshes.square_nonlinear(m=int(round(np.sqrt(n))) - 1, seed=1000 + i) for i, n in enumerate(ns)]
    curs = [meshes.seeded_currents(1, 3, 20.0, seed=3000 + i)[0] for i in range(count)]
    t0 = time.perf_counter()
    plans = [fg.Plan(mo) for mo in models]
    plan_s = time.perf_counter() - t0
    multi = fg.Multi(plans)
    multi.solve(curs, outputs=False)
    t0 = time.perf_counter()
    ma, _, _, mf, minfo = multi.solve(curs, outputs="a")
    dt_multi = time.perf_counter() - t0
    mt = multi.last_timing()
    t0 = time.perf_counter()
    single = [p.solve([c], outputs="a") for p, c in zip(plans, curs)]
    dt_single = time.perf_counter() - t0
    out = {"workload": f"{count} jittered squares, {sum(mo.node_count for mo in models)} nodes in all "
                       "(5k-200k each, log-uniform), one sample each; host-buffer API timing",
           "meshes": count, "plan_build_seconds": plan_s,
           "multi_solves_per_s": count / dt_multi, "one_plan_at_a_time_solves_per_s": count / dt_single,
           "speedup": dt_single / dt_multi, "newton_steps": int(mt.newton_steps),
           "pcg_launches": int(mt.pcg_launches), "graph_launches": int(mt.graph_launches),
           "graph_captures": int(mt.graph_captures), "max_ctas": int(mt.max_ctas),
           "all_converged": all(i.status == 0 for i in minfo),
           "a_rel_err_vs_single": max_rel(ma, [s_.a[0] for s_ in single])}
    multi.close()
    for p in plans:
        p.close()
    return out


def learned_form(ntrain, nheld, block=1024):
    """The learned warm start on the axisymmetric plunger (about 100k nodes, 2 coils
    U[-30, 30] A): POD basis + MLP trained on `ntrain` FP64 solves of the plain method, then
    `nheld` held-out samples solved three ways at the same gates -- the plain FP64 Jacobi
    method from zero; the fast form (mixed precision, block-Jacobi 8, PCG from the iterate)
    from zero; the same fast form from the network's guarded prediction.  The last two
    isolate the network's own gain.  Errors: against the plain FP64 solutions."""
    import torch
    import femm_gpu_b200 as fg
    from femm_gpu_b200 import learned, meshes

    ax = meshes.axisymmetric_plunger()
    base = fg.Plan(ax)
    train = np.random.default_rng(2024).uniform(-30, 30, size=(ntrain, 2))
    held = np.random.default_rng(2025).uniform(-30, 30, size=(nheld, 2))
    t0 = time.perf_counter()
    ws = learned.LearnedWarmStart(base, current_scale=30.0, rank=64, hidden=256, seed=1)
    ws.fit(train, pod_samples=min(512, ntrain), epochs=200, batch=256, lr=2e-3, block=block)
    fit_s = time.perf_counter() - t0
    fast = fg.Plan(ax, precision=1, preconditioner=1, block_size=8, from_iterate=True)
    w = ws.warm
    lw = learned.LearnedWarmStart(fast, 30.0)
    lw.warm = learned.WarmModel(fast, w.mean, w.basis, ws.mlp, *w._keep)
    res = {}
    for name, fn in (("fp64_jacobi_zero_start", lambda c: base.solve(c, outputs="a")),
                     ("fast_form_zero_start", lambda c: fast.solve(c, outputs="a")),
                     ("learned_fast_form", lambda c: lw.solve(c, outputs="a"))):
        fn(held[:32])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rs = [fn(held[i:i + block]) for i in range(0, nheld, block)]
        dt = time.perf_counter() - t0
        info = [i for r in rs for i in r.info]
        res[name] = {"solves_per_s_e2e": nheld / dt,
                     "newton_iterations_per_item": float(np.mean([i.iterations for i in info])),
                     "pcg_iterations_per_item": float(np.mean([i.linear_iterations for i in info])),
                     "warm_starts_used": int(sum(i.warm_start == 1 for i in info)),
                     "all_converged": all(i.status == 0 for i in info),
                     "a": np.concatenate([r.a for r in rs]), "flux": np.concatenate([r.flux for r in rs])}
    z = res["fp64_jacobi_zero_start"]
    for name in ("fast_form_zero_start", "learned_fast_form"):
        r = res[name]
        r["a_rel_err"] = max_rel(r["a"], z["a"])
        r["flux_rel_err"] = max_rel(r["flux"], z["flux"])
        r["vs_fp64_zero_start"] = r["solves_per_s_e2e"] / z["solves_per_s_e2e"]
    res["learned_fast_form"]["vs_same_form_zero_start"] = (res["learned_fast_form"]["solves_per_s_e2e"] /
                                                          res["fast_form_zero_start"]["solves_per_s_e2e"])
    for r in res.values():
        r.pop("a")
        r.pop("flux")
    out = dict(workload=f"axisymmetric plunger r-z, {ax.node_count} nodes, 2 coils U[-30,30] A; "
                        f"{ntrain} training solves, {nheld} held-out samples; host-buffer API timing",
               fit_seconds=fit_s, pod_energy=float(ws.stats["pod_energy"]),
               final_loss=float(ws.stats["final_loss"]), **res)
    fast.close()
    base.close()
    return out


def reference_gpu_form(mesh=MESH_M, items=8):
    """GPU against GPU on the headline workload: the reference's own executable built for
    sm_100a (oracle/_ref/bin/femm_gpu_ref, built by oracle/Makefile's refgpu target) and this
    library's femm_gpu answer the same request files.  --solve: one sample per process
    (wall clock, process start, artifact read and hash included), flux linkage and Newton
    iterations compared.  --motor-batch-profile: `items` samples of the posed motor form of
    the same artifact in one process (the reference's SolveBatch path, 32 items per chunk),
    its own timing block and the wall clock, every item's flux linkage and torque compared."""
    import hashlib
    import tempfile
    from femm_gpu_b200 import artifact, meshes

    theirs = os.path.join(ROOT, "oracle", "_ref", "bin", "femm_gpu_ref")
    ours = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
    if not os.path.exists(theirs):
        return {"unavailable": "the reference executable was not built (no reference checkout)"}
    tmp = tempfile.mkdtemp(prefix="fg_refgpu_")
    model = meshes.square_nonlinear(m=mesh, seed=SEED_MESH)
    text, _ = artifact.write_artifact(model, [0.0, 0.0, 0.0])
    neutral = os.path.join(tmp, "square.gpu.json")
    open(neutral, "w").write(text)
    src = json.loads(text)
    src["schema_version"] = "gpu_femm_mesh_v1"
    base = "e" * 64
    src["base_motor_fem_sha256"] = base
    src["resolved"]["base_motor_fem_sha256"] = base
    src["resolved"]["pose"] = {"rotor_angle_deg": 0, "displacement_mm": [0, 0]}
    del src["resolved"]["node_constraints"]  # a posed motor artifact carries none
    motor = os.path.join(tmp, "square_motor.gpu.json")
    open(motor, "w").write(json.dumps(src))
    sha = lambda p: hashlib.sha256(open(p, "rb").read()).hexdigest()  # noqa: E731
    cur = meshes.seeded_currents(items, 3, 20.0, seed=5150)

    def run(exe, command, body, name):
        rq, rs = os.path.join(tmp, name + ".json"), os.path.join(tmp, name + "." + os.path.basename(exe) + ".out")
        open(rq, "w").write(json.dumps(body))
        t0 = time.perf_counter()
        r = subprocess.run([exe, command, rq, rs], capture_output=True, text=True, timeout=1800)
        return r.returncode, time.perf_counter() - t0, (json.load(open(rs)) if os.path.exists(rs) else {})

    solve = {"protocol": "gpu_femm_magnetostatic_sample_v1", "mesh_artifact_path": neutral,
             "mesh_artifact_sha256": sha(neutral), "circuit_currents_A": [float(c) for c in cur[0]],
             "force_group_number": -1, "stress_air_group_number": -1, "airgap_radius_mm": 0,
             "airgap_angles_deg": [], "sliding_band_angle_deg": 0, "compute_force_torque": False,
             "include_field_solution": False}
    out = {"workload": f"nonlinear planar solve, {model.node_count} nodes; the same request files to both "
                       "executables; wall clock per process"}
    res = {}
    for name, exe in (("reference_gpu", theirs), ("ours", ours)):
        run(exe, "--solve", solve, "warm")  # page in the executable and the driver
        rc, dt, body = run(exe, "--solve", solve, "solve")
        res[name] = (rc, dt, body)
        out[f"{name}_solve_seconds"] = dt
        out[f"{name}_solve_ok"] = rc == 0 and body.get("status") == "PASS"
    fr, fo = res["reference_gpu"][2], res["ours"][2]
    if out["reference_gpu_solve_ok"] and out["ours_solve_ok"]:
        a, b = np.array(fo["circuit_flux_linkage_Wb"]), np.array(fr["circuit_flux_linkage_Wb"])
        out["solve_flux_rel_err"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
        out["solve_newton_iterations"] = [fr["convergence"]["iterations"], fo["convergence"]["iterations"]]
        out["solve_speedup"] = out["reference_gpu_solve_seconds"] / out["ours_solve_seconds"]
    batch = {"protocol": "gpu_femm_motor_batch_v1", "max_items_per_chunk": 32,
             "items": [{"task_id": f"t{i}", "request": {
                 "protocol": "gpu_femm_motor_sample_v1", "mesh_artifact_path": motor,
                 "mesh_artifact_sha256": sha(motor), "base_motor_fem_sha256": base,
                 "source_fem_sha256": src["source_fem_sha256"], "circuit_currents_A": [float(c) for c in cur[i]],
                 "selected_group_number": 1, "air_group_number": 0, "airgap_radius_mm": 0,
                 "airgap_angles_deg": [], "rotor_angle_deg": 0, "displacement_mm": [0, 0]}}
                       for i in range(items)]}
    for name, exe in (("reference_gpu", theirs), ("ours", ours)):
        rc, dt, body = run(exe, "--motor-batch-profile", batch, "batch")
        res[name] = (rc, dt, body)
        out[f"{name}_batch_seconds"] = dt
        out[f"{name}_batch_solves_per_s"] = items / dt
        tm = body.get("timing", {})
        out[f"{name}_batch_timing"] = {k: tm.get(k) for k in ("gpu_kernel_sync_seconds", "host_assembly_seconds",
                                                               "device_assembly_seconds", "postprocess_seconds",
                                                               "measured_before_response_write_seconds")}
        out[f"{name}_batch_ok"] = rc == 0 and body.get("status") == "PASS"
    if out["reference_gpu_batch_ok"] and out["ours_batch_ok"]:
        ir, io = res["reference_gpu"][2]["items"], res["ours"][2]["items"]
        out["batch_flux_rel_err"] = float(max(
            np.linalg.norm(np.subtract(a["response"]["circuit_flux_linkage_Wb"], b["response"]["circuit_flux_linkage_Wb"]))
            / np.linalg.norm(b["response"]["circuit_flux_linkage_Wb"]) for a, b in zip(io, ir)))
        out["batch_torque_rel_err"] = float(max(abs(a["response"]["torque_Nm"] - b["response"]["torque_Nm"])
                                                / max(abs(b["response"]["torque_Nm"]), 1e-300) for a, b in zip(io, ir)))
        out["batch_speedup"] = out["reference_gpu_batch_seconds"] / out["ours_batch_seconds"]
    return out


def pcg_bytes_per_item_iteration(n, nnz, precision, block):
    """Algorithmic bytes of one item's CG iteration (values + the 13 vector passes), FP64
    or the FP32 inner form; block-Jacobi adds the block inverses' read."""
    w = 8 if precision == 0 else 4
    return w * nnz + 13 * w * n + (w * block * n if block else 0)


def pcg_launch_form(dev, stream, m, k, iterations, launches, one_reduction):
    """PCG launches of a fixed length, for profiling one launch: the planar square of size m
    (m = 0: the rotor-stator sector of the shared-geometry batches, its 3 coil currents
    U[-15, 15] A), k samples, one Newton iteration whose inner PCG is capped at `iterations`
    CG iterations (tolerance 1e-30, so every launch runs exactly that many), repeated
    `launches` times on one plan.  The launch-shape autotuner is off (FG_PCG_TUNE=0: the default value ring, no
    column cache), so the PCG launches are exactly these.  Reports the CUDA-event time per CG
    iteration of each launch and the algorithmic bytes per CG iteration."""
    import torch

    import femm_gpu_b200 as fg
    from femm_gpu_b200 import meshes

    os.environ["FG_PCG_TUNE"] = "0"
    if m > 0:
        model = meshes.square_nonlinear(m=m, seed=2)
        currents = meshes.seeded_currents(k, 3, 20.0, seed=4242)
    else:
        model = meshes.annular_sector()
        currents = np.random.default_rng(5).uniform(-15.0, 15.0, size=(k, model.circuit_count))
    plan = fg.Plan(model, one_reduction=one_reduction)
    peak, source = peaks()
    cur = torch.tensor(currents, device=dev)
    out_a = torch.empty((k, plan.N), dtype=torch.float64, device=dev)
    opts = fg.production_options(max_newton_iterations=1, max_linear_iterations=iterations,
                                 linear_relative_tolerance=1e-30, adaptive_linear_tolerance=0,
                                 recover_nonconvergence=0)
    per_item = pcg_bytes_per_item_iteration(plan.rows, plan.nnz, 0, 0)
    shared = 4.0 * plan.nnz + 4.0 * (plan.rows + 1)
    runs = []
    for _ in range(launches):
        torch.cuda.synchronize()
        plan.solve_device(k, cur.data_ptr(), options=opts, a_ptr=out_a.data_ptr(), stream=stream.cuda_stream)
        torch.cuda.synchronize()
        t = plan.last_timing()
        us = 1e3 * t.pcg_ms / max(1, t.pcg_iterations)
        runs.append({"cg_iterations": int(t.pcg_iterations), "pcg_ms": t.pcg_ms, "us_per_cg_iteration": us})
    plan.close()
    best = min(r["us_per_cg_iteration"] for r in runs)
    algo = k * per_item + shared
    return {"form": "pcg_launch", "mesh": m, "nodes": model.node_count, "rows": plan.rows, "nnz": plan.nnz,
            "items": k, "one_reduction": one_reduction, "runs": runs,
            "algorithmic_bytes_per_cg_iteration": algo, "pcg_gbs": algo / best / 1e3,
            "pcg_frac": algo / best / 1e3 / peak, "peak_gbs": peak, "peak_source": source}


def planar_2m_form(dev, stream, flush, samples=4):
    """The mixed-precision-at-scale workload: the jittered planar square at m = 1414
    (2,002,225 nodes, 3,998,792 triangles, 1,996,569 rows) with the config-2 physics.
    Runs: plain FP64 Jacobi for 1 and 4 samples; the FP32-inner PCG (SpMV + 32-row
    block-Jacobi, FP64 defect correction by reliable updates) for 4 samples, from zero and
    from the Newton iterate.  Each: solves/s (CUDA events, device buffers), Newton (outer)
    and PCG (inner) iterations per sample, PCG algorithmic GB/s and fraction of the HBM
    peak, errors of A, B and flux linkage against the FP64 solutions of the same samples."""
    import torch

    import femm_gpu_b200 as fg
    from femm_gpu_b200 import meshes

    model = meshes.square_nonlinear(m=1414, seed=2)
    peak, _ = peaks()
    cur = meshes.seeded_currents(samples, 3, 20.0, seed=1414)
    runs = (("fp64_jacobi_k1", dict(), 1), ("fp64_jacobi_k4", dict(), samples),
            ("mixed_block32_k4", dict(precision=1, preconditioner=1, block_size=32), samples),
            ("mixed_block32_from_iterate_k4", dict(precision=1, preconditioner=1, block_size=32,
                                                   from_iterate=True), samples))
    out = {"workload": f"nonlinear planar solve, jittered 1414x1414 quads ({model.node_count} nodes, "
                       f"{model.tri_count} triangles)"}
    ref = None
    for name, kw, k in runs:
        p = fg.Plan(model, **kw)
        N, E = p.N, p.E
        x = torch.tensor(cur[:k], device=dev)
        out_a = torch.empty((k, N), dtype=torch.float64, device=dev)
        out_b1 = torch.empty((k, E), dtype=torch.float64, device=dev)
        out_b2 = torch.empty((k, E), dtype=torch.float64, device=dev)
        out_f = torch.empty((k, 3), dtype=torch.float64, device=dev)
        ptrs = dict(a_ptr=out_a.data_ptr(), b1_ptr=out_b1.data_ptr(), b2_ptr=out_b2.data_ptr(),
                    flux_ptr=out_f.data_ptr(), stream=stream.cuda_stream)
        # warm-up: one Newton iteration sizes every workspace of this batch width
        p.solve_device(k, x.data_ptr(), options=fg.production_options(max_newton_iterations=1), **ptrs)
        torch.cuda.synchronize()
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        info = p.solve_device(k, x.data_ptr(), **ptrs)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        t = p.last_timing()
        item_its = sum(i.linear_iterations for i in info)
        per_item = pcg_bytes_per_item_iteration(p.rows, p.nnz, kw.get("precision", 0),
                                                kw.get("block_size", 0) if kw.get("preconditioner") else 0)
        shared = 4.0 * p.nnz + 4.0 * (p.rows + 1)
        gbs = (item_its * per_item + t.pcg_iterations * shared) / (t.pcg_ms / 1e3) / 1e9
        a, b1, b2, f = (out_a.cpu().numpy(), out_b1.cpu().numpy(), out_b2.cpu().numpy(), out_f.cpu().numpy())
        r = {"samples": k, "solves_per_s": k / (ms / 1e3), "seconds": ms / 1e3,
             "newton_iterations_per_item": float(np.mean([i.iterations for i in info])),
             "pcg_iterations_per_item": item_its / k, "pcg_ms": t.pcg_ms,
             "pcg_ms_per_cg_iteration": t.pcg_ms / max(1, t.pcg_iterations),
             "pcg_gbs": gbs, "pcg_frac": gbs / peak,
             "mixed_fallbacks": int(t.mixed_fallbacks), "all_converged": all(i.status == 0 for i in info)}
        if name == "fp64_jacobi_k1":
            per_it, src = traffic_per_cg_iteration("square1414_items1")
            if per_it:
                r["dram_traffic_per_cg_iteration"] = per_it
                r["algorithmic_bytes_per_cg_iteration"] = per_item + shared
                r["traffic_source"] = src
        if name == "fp64_jacobi_k4":
            ref = (a, b1, b2, f)
        elif ref is not None:
            bmax = np.maximum(np.abs(ref[1]).max(axis=1), np.abs(ref[2]).max(axis=1))
            r["a_rel_err"] = float(max(np.linalg.norm(a[i] - ref[0][i]) / np.linalg.norm(ref[0][i])
                                       for i in range(k)))
            r["b_rel_err"] = float(max(max(np.abs(b1[i] - ref[1][i]).max(), np.abs(b2[i] - ref[2][i]).max())
                                       / bmax[i] for i in range(k)))
            r["flux_rel_err"] = float(max(np.linalg.norm(f[i] - ref[3][i]) / np.linalg.norm(ref[3][i])
                                          for i in range(k)))
        out[name] = r
        del out_a, out_b1, out_b2, out_f
        p.close()
    base = out["fp64_jacobi_k4"]["solves_per_s"]
    for name in ("mixed_block32_k4", "mixed_block32_from_iterate_k4"):
        out[name]["vs_fp64_jacobi_k4"] = out[name]["solves_per_s"] / base
    out["errors_against"] = "the plain FP64 Jacobi solutions of the same samples (the drop-in form)"
    return out


def postprocess_tangent_form(sector, cur, hcs, dev, stream, err):
    """Rotor torque, force and 45 smoothed air-gap B probes per sample of the sector
    (weighted stress on the rotor iron + magnets against air, mask solved once on the GPU),
    host form, device form (one launch for all samples) and the reference's own host
    ComputeFrozenPostprocess with its reusable plan; then the 3-circuit tangent multi-RHS
    at one operating point against central differences (6 nonlinear solves)."""
    import torch
    import femm_gpu_b200 as fg
    import oracle as O
    from femm_gpu_b200 import meshes

    sec = meshes.annular_sector()
    sec.group = np.array([0, 10, 10, 3, 4, 5, 6], np.int32)
    p = fg.Plan(sec)
    kk = 32
    r = p.solve(cur[:kk], hc_scale=hcs[:kk])
    ang = np.radians(np.linspace(1.0, 89.0, 45))
    t0 = time.perf_counter()
    pp = fg.Postprocess(p, selected_group=10, air_group=0, radius_m=0.0455, angles_rad=ang,
                        max_mask_iterations=4096)
    mask_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    host = pp.compute(r.a, r.b1, r.b2)
    host_s = time.perf_counter() - t0
    dev_in = [torch.from_numpy(x).to(dev).contiguous() for x in (r.a, r.b1, r.b2)]
    torch.cuda.synchronize()
    ptrs = [t_.data_ptr() for t_ in dev_in]
    got = pp.compute_device(kk, *ptrs, stream=stream.cuda_stream)
    reps = 50
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        pp.compute_device(kk, *ptrs, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    dev_us = 1e3 * e0.elapsed_time(e1) / reps
    E = sec.tri_count
    alg_bytes = E * (5 * 8 + kk * 2 * 8)
    out = {"workload": f"sector {sec.node_count} nodes / {E} triangles, {kk} solved samples, rotor group "
                       f"against air, {ang.size} probes at r = 45.5 mm",
           "mask_build_s_gpu_pcg": mask_s,
           "host_us_per_sample": 1e6 * host_s / kk,
           "device_api_us_per_call_all_samples": dev_us,
           "device_api_us_per_sample": dev_us / kk,
           "device_call_includes": "one kernel (force/torque partials + probe smoothing), one D2H of "
                                   "partials and samples, the ctypes call",
           "device_achieved_gbs": alg_bytes / (dev_us * 1e-6) / 1e9,
           "device_algorithmic_bytes": alg_bytes,
           "device_vs_host_force_rel_err": err(got.force, host.force),
           "device_vs_host_radial_max_abs_diff_over_max": float(np.abs(got.radial_b - host.radial_b).max()
                                                                 / np.abs(host.radial_b).max()),
           "all_ok": bool((host.status == 0).all() and (got.status == 0).all())}
    if O.ref() is not None:
        hs = O.ref_model_handle(sec)
        mask = pp.mask()
        nref = 4
        t0 = time.perf_counter()
        for i in range(nref):
            st, fx, fy, tq, rad, _ = O.ref_postprocess(hs, r.a[i], r.b1[i], r.b2[i], selected_group=10,
                                                       air_group=0, radius_m=0.0455, angles_rad=ang, mask=mask)
        # ref_postprocess rebuilds the reusable plan (geometry, probes) for each call
        out["reference_host_us_per_sample_incl_plan"] = 1e6 * (time.perf_counter() - t0) / nref
        out["host_equals_reference"] = bool(host.force[nref - 1, 0] == fx and host.torque[nref - 1] == tq
                                            and np.array_equal(host.radial_b[nref - 1], rad))
    # Tangent: differential inductances and torque sensitivities at sample 0.
    base = cur[0]
    o = fg.production_options()
    p_hc = fg.Plan(sec)  # the operating point without per-sample Hc: same magnets for +-h
    b0 = p_hc.solve([base])
    p_hc.solve_tangent(b0.a[0], base, np.eye(3), o)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    da, db1, db2, dflux, tinfo = p_hc.solve_tangent(b0.a[0], base, np.eye(3), o)
    tan_s = time.perf_counter() - t0
    h = 0.5
    cd_in = np.concatenate([base + h * np.eye(3), base - h * np.eye(3)])
    p_hc.solve(cd_in)
    t0 = time.perf_counter()
    cd = p_hc.solve(cd_in)
    cd_s = time.perf_counter() - t0
    L_cd = (cd.flux[:3] - cd.flux[3:]) / (2 * h)
    pt = fg.Postprocess(p_hc, selected_group=10, air_group=0, radius_m=0.0455, angles_rad=ang,
                        max_mask_iterations=4096)
    tq = pt.tangent(b0.b1[0], b0.b2[0], da, db1, db2)
    out["tangent"] = {"directions": 3, "tangent_ms_e2e": 1e3 * tan_s, "pcg_launches": 1,
                      "pcg_iterations": [int(i.iterations) for i in tinfo],
                      "central_difference_ms_e2e": 1e3 * cd_s, "speedup_vs_central_difference": cd_s / tan_s,
                      "inductance_rel_err_vs_central_difference": err(dflux, L_cd),
                      "dtorque_nm_per_a": [float(x) for x in tq.torque],
                      "all_ok": bool(all(i.status == 0 for i in tinfo))}
    pt.close()
    pp.close()
    p_hc.close()
    p.close()
    return out


def sliding_band_form(angles=8, items=8):
    """The native air-gap element row: the full two-pole sliding-band machine (38k nodes, the
    1 mm gap a periodic band of 240 arcs) solved over a rotor-angle sweep.  Each angle is its
    own operator (the band's pose), so each gets its own plan: the sweep is timed with host
    buffers, plan set-up and the band postprocess (torque, 45 Fourier probes) included.
    The reference CPU path (its host assembler with the band and FEMM's PCG, one sample per
    host thread) solves one angle's samples as the CPU baseline, and their flux linkages
    give the parity figure."""
    import femm_gpu_b200 as fg
    import oracle as O
    from femm_gpu_b200 import meshes

    degs = np.linspace(0.0, 30.0, angles, endpoint=False)
    cur = meshes.seeded_currents(items, 3, 10.0, seed=6100)
    probes = np.radians(np.linspace(0.0, 358.0, 45))
    warm = fg.Plan(meshes.sliding_band_machine(rotor_deg=0.0))
    warm.solve(cur[:2], outputs="a")
    warm.close()
    models = [meshes.sliding_band_machine(rotor_deg=float(d)) for d in degs]
    t0 = time.perf_counter()
    torques, statuses, first = [], [], None
    for m in models:
        p = fg.Plan(m)
        r = p.solve(cur, outputs="a")
        post = p.air_gap_postprocess(r.a, probes)
        torques.append(post.torque.tolist())
        statuses += [i.status for i in r.info] + list(post.status)
        if first is None:
            first = r
        p.close()
    sweep_s = time.perf_counter() - t0
    out = {"workload": f"full two-pole sliding-band machine, {models[0].node_count} nodes, "
                       f"{models[0].ages[0].nodes.shape[0] - 1}-arc periodic band; {angles} rotor angles x "
                       f"{items} samples, a plan per angle, host buffers, band postprocess included",
           "solves_per_s_e2e": angles * items / sweep_s, "sweep_seconds": sweep_s,
           "all_ok": all(s_ == 0 for s_ in statuses),
           "torque_nm_at_first_sample": [t[0] for t in torques]}
    # The torque-vs-angle pattern: one sample per rotor angle.  Each angle's own launch is
    # latency-bound at this size, so the angles share one multi-plan launch per Newton step
    # (what --motor-batch does for the poses of a chunk).
    sweep = [meshes.sliding_band_machine(rotor_deg=float(d)) for d in np.linspace(0.0, 30.0, 16, endpoint=False)]
    plans = [fg.Plan(m) for m in sweep]
    c1 = cur[0]
    t0 = time.perf_counter()
    one = [p.solve([c1], outputs="a") for p in plans]
    per_plan_s = time.perf_counter() - t0
    multi = fg.Multi(plans)
    multi.solve([c1] * len(plans), outputs=False)
    t0 = time.perf_counter()
    _, _, _, mflux, minfo = multi.solve([c1] * len(plans), outputs="a")
    multi_s = time.perf_counter() - t0
    out["one_sample_per_angle"] = {
        "angles": len(plans), "per_plan_solves_per_s": len(plans) / per_plan_s,
        "multi_plan_solves_per_s": len(plans) / multi_s, "speedup": per_plan_s / multi_s,
        "flux_rel_err_multi_vs_per_plan": float(max(np.linalg.norm(mflux[i] - one[i].flux[0]) /
                                                    np.linalg.norm(one[i].flux[0]) for i in range(len(plans)))),
        "all_ok": all(i.status == 0 for i in minfo) and all(r.info[0].status == 0 for r in one)}
    for p in plans:
        p.close()
    if O.ref() is not None:
        threads = min(os.cpu_count() or 1, items)
        t0 = time.perf_counter()
        a, flux, st, *_ = O.ref_cpu_newton_batch(models[0], cur[:threads], threads=threads)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": threads / cpu_s, "unit": "solves/s", "cores": threads,
                               "kind": "reference",
                               "sample": f"{threads} samples of the first angle, one per host thread"}
        out["speedup_vs_cpu"] = out["solves_per_s_e2e"] / out["cpu_baseline"]["value"]
        out["flux_rel_err_vs_reference"] = float(max(
            np.linalg.norm(first.flux[i] - flux[i]) / np.linalg.norm(flux[i]) for i in range(threads)))
        out["reference_all_converged"] = bool((st == 0).all())
    return out


def worker_form(jobs=8, items=8):
    """The JSON boundary as a service: `jobs` batch files of `items` samples on one 40,401-node
    artifact, streamed through one `femm_gpu --worker` (plans resident across jobs, the next
    job prepared while the GPU solves) against one `femm_gpu --batch` process per file."""
    import hashlib
    import subprocess
    import tempfile
    from femm_gpu_b200 import artifact, meshes

    cli = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
    tmp = tempfile.mkdtemp(prefix="fg_worker_")
    model = meshes.square_nonlinear(m=200, seed=2)
    text, _ = artifact.write_artifact(model, [10.0, -5.0, 3.0])
    art = os.path.join(tmp, "mesh.gpu.json")
    open(art, "w").write(text)
    digest = hashlib.sha256(text.encode()).hexdigest()
    files = []
    for j in range(jobs):
        cur = meshes.seeded_currents(items, 3, 20.0, seed=9000 + j)
        body = {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": items,
                "items": [{"task_id": f"j{j}i{i}", "request": {
                    "protocol": "gpu_femm_magnetostatic_sample_v1", "mesh_artifact_path": art,
                    "mesh_artifact_sha256": digest, "circuit_currents_A": [float(x) for x in cur[i]],
                    "force_group_number": -1, "stress_air_group_number": -1, "airgap_radius_mm": 0,
                    "airgap_angles_deg": [], "sliding_band_angle_deg": 0, "compute_force_torque": False,
                    "include_field_solution": False}} for i in range(items)]}
        f = os.path.join(tmp, f"b{j}.json")
        open(f, "w").write(json.dumps(body))
        files.append(f)
    session = hashlib.sha256(b"bench").hexdigest()
    lines = [json.dumps({"session": session, "sequence": j + 1, "request_path": f,
                         "response_path": os.path.join(tmp, f"w{j}.json"),
                         "request_sha256": hashlib.sha256(open(f, "rb").read()).hexdigest()})
             for j, f in enumerate(files)]
    t0 = time.perf_counter()
    r = subprocess.run([cli, "--worker"], input="\n".join(lines) + "\n", capture_output=True, text=True,
                       timeout=900)
    worker_s = time.perf_counter() - t0
    status = [json.loads(x) for x in r.stdout.strip().splitlines()]
    t0 = time.perf_counter()
    rcs = [subprocess.run([cli, "--batch", f, os.path.join(tmp, f"o{j}.json")], capture_output=True,
                          timeout=900).returncode for j, f in enumerate(files)]
    oneshot_s = time.perf_counter() - t0
    same = all(json.load(open(os.path.join(tmp, f"w{j}.json")))["items"][0]["response"]["circuit_flux_linkage_Wb"]
               == json.load(open(os.path.join(tmp, f"o{j}.json")))["items"][0]["response"]["circuit_flux_linkage_Wb"]
               for j in range(jobs))
    return {"workload": f"{jobs} batch files x {items} samples, one {model.node_count}-node artifact "
                        f"({len(text) / 1e6:.1f} MB JSON), wall clock including process start",
            "worker_solves_per_s": jobs * items / worker_s, "one_shot_solves_per_s": jobs * items / oneshot_s,
            "speedup": oneshot_s / worker_s,
            "worker_prepare_seconds": [round(s_["prepare_seconds"], 4) for s_ in status],
            "all_pass": all(s_["exit_code"] == 0 for s_ in status) and all(rc == 0 for rc in rcs),
            "responses_equal": bool(same)}


def run_reference(args, world, rank, local):
    """The reference's CPU path on every host thread, timed in bounded steps.

    One sample per host thread; one step = one Newton iteration (reference host assembly +
    FEMM 4.2 SSOR-PCG to the inner tolerance) of every sample, samples restarted with fresh
    seeded currents as they converge.  After the timed steps the unfinished samples run on,
    untimed, to convergence; solves/s = Newton iterations/s / mean Newton iterations per
    solve of the samples that finished."""
    if rank != 0:
        return
    import oracle as O
    from femm_gpu_b200 import meshes

    model = meshes.square_nonlinear(m=args.mesh, seed=SEED_MESH)
    threads = os.cpu_count() or 1
    if O.ref() is None:  # the C restatement: whole solves, one per thread
        base, _ = cpu_baseline(model, items_seed=4242, budget_threads=threads)
        value, ms, sample = base["value"], 1e3 * threads / base["value"], base["sample"]
        kind = "port"
    else:
        kind = "reference"
        rng_seed = [4242]

        def fresh():
            rng_seed[0] += 1
            return meshes.seeded_currents(1, model.circuit_count, 20.0, seed=rng_seed[0])[0]

        session = O.RefSession(model, meshes.seeded_currents(threads, model.circuit_count, 20.0,
                                                             seed=4242))
        finished = []

        def step():
            done = session.step(threads)
            status, newton = session.info()
            for i in np.nonzero(done)[0]:
                finished.append((int(status[i]), int(newton[i])))
                session.restart(int(i), fresh())

        for _ in range(args.warmup):
            step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        dt = time.perf_counter() - t0
        for _ in range(200):  # untimed: finish every running sample
            done = session.step(threads)
            if done.all():
                break
        status, newton = session.info()
        finished += [(int(status[i]), int(newton[i])) for i in range(threads)]
        session.close()
        mean_newton = float(np.mean([n for _, n in finished]))
        converged = sum(1 for s_, _ in finished if s_ == 0)
        value = threads * args.steps / dt / mean_newton
        ms = 1e3 * dt / args.steps
        sample = (f"{threads} samples on {threads} host threads; step = one Newton iteration "
                  f"(reference host assembly + FEMM SSOR-PCG) per sample; {args.steps} timed "
                  f"steps in {dt:.1f} s; {mean_newton:.2f} mean Newton iterations over "
                  f"{len(finished)} finished solves ({converged} converged)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(model, args.mesh, world), "items_per_step": threads,
            "solver": "reference host assembler + FEMM 4.2 SSOR PCG, one sample per host thread",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                             "cpu_model": cpu_model(), "nproc": os.cpu_count(), "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def only_form(args):
    import torch

    from femm_gpu_b200 import meshes

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    if args.only_form == "streaming_worker":
        out = worker_form()
    elif args.only_form == "learned":
        out = learned_form(args.learned_train, args.learned_held)
    elif args.only_form == "reference_gpu":
        out = reference_gpu_form(args.mesh)
    elif args.only_form == "sector":
        out = sector_form(args.sector_samples)
    elif args.only_form == "hetero":
        out = hetero_form(args.hetero_meshes)
    elif args.only_form == "planar_2m":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        out = planar_2m_form(dev, stream, flush)
    elif args.only_form == "sliding_band":
        out = sliding_band_form()
    elif args.only_form == "pcg_launch":
        out = pcg_launch_form(dev, stream, args.probe_mesh, args.probe_items, args.probe_iterations,
                              args.probe_launches, args.probe_one_reduction)
    else:
        rng = np.random.default_rng(77)
        cur = rng.uniform(-15.0, 15.0, size=(args.sector_samples, 3))
        hcs = rng.uniform(8.5e5, 9.5e5, size=args.sector_samples) / 9.0e5

        def err(a, b):
            return float(max(np.linalg.norm(a[i] - b[i]) / np.linalg.norm(b[i]) for i in range(len(b))))
        out = postprocess_tangent_form(meshes.annular_sector(), cur, hcs, dev, stream, err)
    print(json.dumps({"form": args.only_form, **out}))


def main():
    args = parse()
    if args.only_form:
        only_form(args)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
