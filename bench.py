"""Benchmark: element-integrations/s of the element-integration + CSR assembly path.

Headline workload (`value`): the C3D20 full-integration (27-point) linear-elastic block,
64^3 quadratic hexes of a unit cube (262,144 elements, 1,085,825 nodes, 3,219,840 free
DOF, 550,501,596 CSR values), node jitter uniform +-0.05 h, per-element E lognormal
(median 200000, sigma 0.3), nu 0.3, z=0 face clamped. Synthetic and seeded. One step =
one assembly of K_ff and the rhs (every element integrated, every CSR value written
once). `value` = mixed precision (FP32 blocks, FP64 Jacobians and accumulation),
inputs resident in HBM; the FP64 path is timed in the same run ("fp64"). e2e = the same
through the C ABI with host buffers (load vector in, K_ff + rhs out every step).

Further sections of the same JSON line:
  j2_newton  C3D8 128^3 J2 block, residual + consistent tangent of the last increment of a
             graded uniaxial ramp (~40 % of Gauss points yielding), FP64 and mixed;
  batched    256 independent models of five element types in one CUDA graph, autotuned;
  adjoint    C3D8 96x96x48 cantilever: device CG solve, then dc/dE and dc/dX per step;
  cpu_baseline  the reference's own element routine on the host cores (oracle/_ref).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--n 64]
Multi-GPU (torchrun): every rank assembles its own workloads (weak scaling, no
collective on the data path); timing is max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cxg", choices=["cxg", "reference"])
    ap.add_argument("--n", type=int, default=64, help="cells per axis of the C3D20 block")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--j2-n", type=int, default=128, help="cells per axis of the C3D8 J2 block (0: skip)")
    ap.add_argument("--batch-models", type=int, default=256, help="models of the batched workload (0: skip)")
    ap.add_argument("--adj-n", type=int, default=96, help="cells along x and y of the adjoint cantilever (0: skip)")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (no tuning sweeps; for profiler runs)")
    return ap.parse_args()


# ---- distributed plumbing -------------------------------------------------------------
def dist_init(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device(f"cuda:{local}"))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- clocks -------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            try:
                os.remove(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded or sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---- workload -----------------------------------------------------------------------------
def c3d20_model(n, seed):
    from calculixpp_b200 import meshgen as mg
    from calculixpp_b200.assembly import Material, Model
    cfg = mg.c3d20_block(n, seed=seed)
    m = cfg["mesh"]
    return Model(m, [Material(200000.0, 0.3)], None, cfg["spc"], None), cfg["f_ext"]


def j2_model(n, k, seed=0):
    """The J2 Newton workload (C3D8 n^3, graded uniaxial ramp) at increment k."""
    from calculixpp_b200 import meshgen as mg
    from calculixpp_b200.assembly import Material, Model
    cfg = mg.c3d8_j2_block(n, seed)
    u, spc = mg.j2_increment(cfg, k)
    return Model(cfg["mesh"], [Material(mg.J2_E, mg.J2_NU, cfg["table"])], None, spc, None), cfg, u


def j2_algorithmic_bytes(plan, model):
    """Compulsory bytes of one residual + consistent-tangent pass: connectivity, node
    coordinates and displacements read, E and nu per element, the isotropic-hardening
    state (plastic strain 6 + equivalent plastic strain 1 doubles per Gauss point) read
    and written, f_int and rhs written, every K_ff value written once."""
    m = model.mesh
    npe = m.conn.shape[1]
    G = m.n_elems * npe  # 2x2x2 rule: 8 points per C3D8
    return (4 * npe * m.n_elems + 24 * m.n_nodes * 3 + 16 * m.n_elems + 2 * 56 * G + 8 * plan.n_free
            + 8 * plan.nnz)


def j2_newton(args, world, dev, stream):
    """Residual + consistent tangent of one Newton iteration of the last ramp increment,
    FP64 and mixed, on the C3D8 J2 block. The committed state is that of increment 9
    (assembled and committed before timing); every timed step re-integrates all
    elements from it."""
    import torch

    from calculixpp_b200 import Plan
    model, cfg, u10 = j2_model(args.j2_n, 10)
    from calculixpp_b200 import meshgen as mg
    u9, _ = mg.j2_increment(cfg, 9)
    plan = Plan(model, "fp64")
    m = model.mesh
    vals = torch.empty(plan.nnz, dtype=torch.float64, device=dev)
    f_int = torch.empty(3 * m.n_nodes, dtype=torch.float64, device=dev)
    rhs = torch.empty(plan.n_free, dtype=torch.float64, device=dev)
    d_u9 = torch.as_tensor(u9, device=dev)
    d_u = torch.as_tensor(u10, device=dev)
    plan.assemble_tangent(d_u9, vals=vals, f_int=f_int, rhs=rhs)
    plan.commit()

    def step():
        plan.assemble_tangent(d_u, vals=vals, f_int=f_int, rhs=rhs, check=False)

    out = {}
    keep = {}
    shapes = {}
    for prec in ("fp64", "mixed"):
        plan.set_precision(prec)
        shapes[prec] = {"default": True} if args.no_tune else plan.tune(step, tangent=True)
        for _ in range(args.warmup):
            step()
        plan.check()
        torch.cuda.synchronize()
        barrier(world)
        t = max_over_ranks(time_steps(step, args.steps, stream), world)
        plan.check()
        keep[prec] = (vals.clone(), f_int.clone(), plan.state(committed=False).clone())
        out[prec] = {"value": world * m.n_elems * args.steps / t, "ms_per_step": t / args.steps * 1e3,
                     "launch_shape": shapes[prec], "windows_and_ring": plan.windows(tangent=True)}
    (v64, f64, s64), (vm, fm, sm) = keep["fp64"], keep["mixed"]
    yielded = float((s64[:, 6] > 0).double().mean())
    B = j2_algorithmic_bytes(plan, model)
    traffic = json.load(open(TRAFFIC_FILE)) if os.path.exists(TRAFFIC_FILE) else {}
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    ach = B / (out["fp64"]["ms_per_step"] * 1e-3) / 1e9
    res = {
        "workload": f"C3D8 J2 block {args.j2_n}^3, graded uniaxial ramp, increment 10 of 10, "
                    "Newton residual + consistent tangent",
        "elements": m.n_elems, "gauss_points": 8 * m.n_elems, "nnz": plan.nnz,
        "yielded_fraction": yielded,
        "fp64": out["fp64"], "mixed": out["mixed"],
        "speedup_mixed_vs_fp64": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
        "mixed_error": {"K_rel_fro": float(torch.linalg.norm(vm - v64) / torch.linalg.norm(v64)),
                        "f_int_rel_l2": float(torch.linalg.norm(fm - f64) / torch.linalg.norm(f64)),
                        "state_max_abs": float((sm - s64).abs().max())},
        "roofline_fp64": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                          "traffic": traffic.get(f"c3d8_j2_{args.j2_n}_fp64_tangent"),
                          "kernel": "p1_kernel + p2_kernel_small (element pass with J2 return + row gather), C3D8 tangent, FP64",
                          "algorithmic_bytes": B, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
        "gpu_launches_per_step": 2,
    }
    del keep, v64, vm, f64, fm, s64, sm, vals, f_int, rhs
    plan.close()
    torch.cuda.empty_cache()
    return res


def plain_fp64_per_model(models, args, dev, stream):
    """The plain FP64 drop-in path on the batched workload: one plan and one assembly
    call per model (no batching, no graph), each model's assembly timed with CUDA events
    (median of args.steps after args.warmup), summed over the models. Plans are built one
    at a time so device memory stays bounded."""
    import torch

    from calculixpp_b200 import Plan
    total = 0.0
    elems = 0
    for model in models:
        plan = Plan(model, "fp64")
        f = torch.as_tensor(model.external_load_vector(), device=dev)
        vals = torch.empty(plan.nnz, dtype=torch.float64, device=dev)
        rhs = torch.empty(plan.n_free, dtype=torch.float64, device=dev)
        for _ in range(args.warmup):
            plan.assemble_linear(f, vals=vals, rhs=rhs, check=False)
        plan.check()
        times = []
        for _ in range(max(args.steps, 1)):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            plan.assemble_linear(f, vals=vals, rhs=rhs, check=False)
            s1.record(stream)
            s1.synchronize()
            times.append(s0.elapsed_time(s1))
        plan.check()
        total += sorted(times)[len(times) // 2]
        elems += model.mesh.n_elems
        del vals, rhs, f
        plan.close()
    torch.cuda.empty_cache()
    return {"value": elems / (total * 1e-3), "ms_total": total,
            "how": "one FP64 plan per model, one assembly call each, per-model median event time summed"}


def batched(args, world, rank, dev, stream):
    """Batched mixed-element models: the autotuned batch replayed as one CUDA graph per
    step (all groups as parallel branches), mixed precision; FP64 on the same batch when
    its FP64 element buffers fit in the remaining device memory."""
    import torch

    from calculixpp_b200 import Batch, CxgError
    from calculixpp_b200 import meshgen as mg
    from calculixpp_b200.assembly import Material, Model
    n_models = args.batch_models
    work = mg.batched_workload(n_models, seed=rank)
    models = [Model(m, [Material(E, nu)], None, spc, (top, np.zeros(top.size, np.int64), np.full(top.size, 1.0 / top.size)))
              for m, spc, top, E, nu in work]
    while True:
        try:
            t0 = time.perf_counter()
            b = Batch(models, "mixed")
            t_build = time.perf_counter() - t0
            f = torch.as_tensor(b.load_vector(), device=dev)
            vals, rhs = b.buffers()
            break
        except (CxgError, torch.cuda.OutOfMemoryError):
            b = vals = rhs = None
            torch.cuda.empty_cache()
            if len(models) <= 8:
                raise
            models = models[: len(models) // 2]
    E_tot = sum(m.mesh.n_elems for m in models)
    E_all = E_tot  # elements over all ranks (each rank draws its own models)
    if world > 1:
        import torch.distributed as dist
        e = torch.tensor([float(E_tot)], dtype=torch.float64, device=dev)
        dist.all_reduce(e, op=dist.ReduceOp.SUM)
        E_all = float(e.item())
    by_type = {}
    for m in models:
        name = mg.TYPE_NAMES[m.mesh.etype]
        by_type[name] = by_type.get(name, 0) + m.mesh.n_elems

    def run(prec):
        b.set_precision(prec)
        t0 = time.perf_counter()
        cfg = [] if args.no_tune else b.tune(f, vals, rhs)
        t_tune = time.perf_counter() - t0

        def step():
            b.graph_launch(f, vals, rhs)

        for _ in range(args.warmup):
            step()
        b.check()
        torch.cuda.synchronize()
        barrier(world)
        t = max_over_ranks(time_steps(step, args.steps, stream), world)
        b.check()
        return {"value": E_all * args.steps / t, "ms_per_step": t / args.steps * 1e3,
                "tune_s": t_tune, "group_configs": cfg}

    res = {"workload": f"{len(models)} independent boxes, element counts log-uniform in [1e3, 2e5], types "
                       "C3D8/C3D8R/C3D20R/C3D6/C3D15, corner-node jitter 0.1 h (quadratic midside nodes at edge midpoints), E ~ U[7e4, 2.1e5], nu ~ U[0.25, 0.35]; "
                       "one CUDA graph per step (one element pass + one row gather per type group, groups as "
                       "parallel branches)",
           "models": len(models), "elements": E_tot, "elements_by_type": by_type, "nnz": b.nnz,
           "n_free": b.n_free, "plan_build_s": t_build}
    plain = plain_fp64_per_model(models, args, dev, stream) if world == 1 else None

    def signature():
        # sums and strided samples of the batch's values and rhs: equal outputs give equal
        # signatures (the full vals buffer is too large to keep a copy of)
        return float(vals.sum().item()), float(rhs.sum().item()), vals[::9973].clone(), rhs[::97].clone()

    def one_launch(prec, ref):
        # the same step with the whole batch as one element pass + one row gather
        b.set_launch("one_launch")
        r = run(prec)
        sig = signature()
        r["equal_to_per_group"] = bool(sig[:2] == ref[:2] and torch.equal(sig[2], ref[2]) and torch.equal(sig[3], ref[3]))
        r["how"] = "one element pass + one row gather for all groups (cxg_batch_set_launch ONE_LAUNCH), one CUDA graph"
        b.set_launch("per_group")
        del sig, ref
        torch.cuda.empty_cache()
        return r

    res["mixed"] = run("mixed")
    res["mixed_one_launch"] = one_launch("mixed", signature())
    keep = vals.clone() if b.nnz * 8 < 0.2 * torch.cuda.mem_get_info()[0] else None
    free = torch.cuda.mem_get_info()[0]
    # FP64 element buffers replace the FP32 ones group by group (each FP32 buffer is
    # released before its FP64 successor is allocated)
    # (padded 3x3 blocks: 80 B in FP64, 48 B in FP32)
    fp64_extra = sum(m.mesh.n_elems * (m.mesh.conn.shape[1] * (m.mesh.conn.shape[1] + 1) // 2) * 80 for m in models)
    fits = free + fp64_extra * 0.6 > 1.05 * fp64_extra + 4e9
    if world > 1:  # every rank takes the same branch (the FP64 run holds collectives)
        import torch.distributed as dist
        flag = torch.tensor([1.0 if fits else 0.0], device=dev)
        dist.all_reduce(flag, op=dist.ReduceOp.MIN)
        fits = bool(flag.item() > 0.5)
    if fits:
        res["fp64"] = run("fp64")
        res["fp64_one_launch"] = one_launch("fp64", signature())
        res["speedup_mixed_vs_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
        if keep is not None:
            res["mixed_K_rel_fro_vs_fp64"] = float(torch.linalg.norm(keep - vals) / torch.linalg.norm(vals))
    else:
        res["fp64"] = {"skipped": f"FP64 element buffers ({fp64_extra / 1e9:.1f} GB) exceed free device memory "
                                  f"({free / 1e9:.1f} GB) plus the FP32 buffers they replace"}
    if plain is not None:
        res["plain_fp64_per_model"] = plain
        res["speedup_batched_mixed_vs_plain_fp64"] = plain["ms_total"] / res["mixed"]["ms_per_step"]
    del keep, vals, rhs, f
    b.close()
    torch.cuda.empty_cache()
    return res


def adjoint_section(args, world, dev, stream):
    """Compliance sensitivities of the C3D8 cantilever: assembly + device CG solve once,
    then the adjoint kernel (dc/dE per element, dc/dX per node) timed per step. Checks at
    full size: sum_e E_e dc/dE_e = -c, sum_nodes dc/dX = 0, sum X.dc/dX = -c."""
    import ctypes as C

    import torch

    from calculixpp_b200 import Plan, _lib
    from calculixpp_b200 import meshgen as mg
    from calculixpp_b200.assembly import Material, Model
    nx = args.adj_n
    cfg = mg.adjoint_cantilever(nx, nx, nx // 2)
    m = cfg["mesh"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"], cfg["cloads"])
    plan = Plan(model, "fp64")
    f = torch.as_tensor(model.external_load_vector(), device=dev)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    vals, rhs = plan.assemble_linear(f)
    s0.record(stream)
    x, iters, rel = plan.solve_cg(vals, rhs, rtol=1e-10, max_iter=100000)
    s1.record(stream)
    s1.synchronize()
    t_solve = s0.elapsed_time(s1) * 1e-3
    c = float(torch.dot(rhs, x))
    u = plan.expand(x)
    dE = torch.empty(m.n_elems, dtype=torch.float64, device=dev)
    dX = torch.empty(3 * m.n_nodes, dtype=torch.float64, device=dev)
    lib = _lib.load()
    vp = C.c_void_p

    def step():
        _lib.check(lib.cxg_adjoint_compliance(plan.h, vp(u.data_ptr()), vp(dE.data_ptr()), vp(dX.data_ptr()),
                                              vp(stream.cuda_stream)))

    for _ in range(args.warmup):
        step()
    plan.check()
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(time_steps(step, args.steps, stream), world)
    plan.check()
    E = torch.as_tensor(m.young, device=dev)
    X = torch.as_tensor(m.coords, device=dev).reshape(-1)
    res = {"workload": f"C3D8 cantilever {nx}x{nx}x{nx // 2}, E = 2.1e5 rho^3, rho ~ U[0.1, 1], x=0 clamped, tip load",
           "elements": m.n_elems, "n_free": plan.n_free,
           "solve": {"kind": "Jacobi-PCG on the device", "rtol": 1e-10, "iterations": iters, "rel_residual": rel,
                     "seconds": t_solve},
           "adjoint": {"value": world * m.n_elems * args.steps / t, "unit": "element-integrations/s",
                       "ms_per_step": t / args.steps * 1e3},
           "identities": {"sum_E_dcdE_plus_c_rel": abs(float(E @ dE) + c) / abs(c),
                          "sum_dcdX_rel": float(dX.view(-1, 3).sum(0).abs().max() / dX.abs().sum()),
                          "sum_X_dcdX_plus_c_rel": abs(float(X @ dX) + c) / abs(c)}}
    del vals, rhs, x, u, dE, dX
    plan.close()
    torch.cuda.empty_cache()
    return res


def algorithmic_bytes(plan, model):
    """Compulsory bytes of one linear assembly launch: connectivity, node coordinates,
    per-element E and nu read once, every K_ff value written once."""
    m = model.mesh
    npe = m.conn.shape[1]
    return 4 * npe * m.n_elems + 24 * m.n_nodes + 16 * m.n_elems + 8 * plan.nnz


FLOPS_PER_ELEM_C3D20 = 27 * (2 * 9 * 20 + 60 + 2 * 9 * 20 + 45 * 20 * 21 // 2)


def measure_peaks():
    """cuBLAS DGEMM / SGEMM throughput (the FP64 / FP32 pipe references)."""
    import torch
    out = {}
    for name, dt in (("fp64_tflops", torch.float64), ("fp32_tflops", torch.float32)):
        torch.backends.cuda.matmul.allow_tf32 = False
        n = 8192
        a = torch.randn(n, n, dtype=dt, device="cuda")
        b = torch.randn(n, n, dtype=dt, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
        out[name] = best
        del a, b
    torch.cuda.empty_cache()
    return out


def time_steps(fn, steps, stream):
    import torch
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(steps):
        fn()
    e.record(stream)
    e.synchronize()
    return s.elapsed_time(e) * 1e-3


# ---- CPU baseline (the reference compiled from its sources, all host threads) ----------
def host_pattern(mesh, dof_eq):
    """Canonical CSR pattern (row_ptr, col_idx) of K_ff on the host: row (a, i) holds the
    free DOFs of every node sharing an element with node a, in ascending order."""
    conn = mesh.conn.astype(np.int64)
    N, npe = mesh.n_nodes, conn.shape[1]
    key = np.unique((np.repeat(conn, npe, axis=1) * N + np.tile(conn, (1, npe))).reshape(-1))
    a, b = key // N, key % N
    deq = dof_eq.reshape(N, 3)
    rows, cols = [], []
    for i in range(3):
        for j in range(3):
            r, c = deq[a, i], deq[b, j]
            keep = (r >= 0) & (c >= 0)
            rows.append(r[keep])
            cols.append(c[keep])
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    n_free = int((dof_eq >= 0).sum())
    rp = np.zeros(n_free + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n_free), out=rp[1:])
    return rp, cols.astype(np.int32)


def cpu_baseline(seconds, seed=0, as_shipped=True):
    from oracle.oracle import Port, Ref
    threads = len(os.sched_getaffinity(0))
    n = 12
    model, _ = c3d20_model(n, seed)
    dof_eq, pre, _ = model.dof_map()
    rp, ci = host_pattern(model.mesh, dof_eq)
    m = model.mesh
    if Ref.available():
        ref = Ref()
        elems, t0 = 0, time.perf_counter()
        while True:
            kv, kr = ref.assemble_csr_threads(m, dof_eq, pre, rp, ci, threads)
            elems += m.n_elems
            if time.perf_counter() - t0 >= seconds:
                break
        dt = time.perf_counter() - t0
        out = {"value": elems / dt, "unit": "element-integrations/s", "cores": threads, "kind": "reference",
               "sample": f"C3D20 {n}^3 block ({m.n_elems} elements) x {elems // m.n_elems} passes: reference "
                         f"element_stiffness (src/fem/element.cpp) on {threads} threads + exact CSR scatter"}
        if not as_shipped:
            return out
        # the reference's FP64 system of the sampled block, the checker of the GPU's
        # mixed and FP64 outputs on the same block (popped before the line is printed)
        out["_ref_system"] = {"n": n, "seed": seed, "row_ptr": rp, "col_idx": ci, "vals": kv, "rhs": kr,
                              "dof_eq": dof_eq}
        # beside it, the reference's own assembly driver as shipped: one thread, its hash-map
        # scatter and unordered COO flush (assemble_linear_static, src/fem/assembly.cpp:225-257)
        try:
            from oracle.oracle import make_material
            n2 = 8
            model2, _ = c3d20_model(n2, seed)
            m2 = model2.mesh
            mats = [make_material(float(E), 0.3) for E in m2.young]
            rm = ref.model(m2, mats, np.arange(m2.n_elems, dtype=np.int32), model2.spc, model2.cloads)
            calls, dt2 = rm.time_linear_static(max(1.0, seconds / 3))
            out["as_shipped"] = {"value": calls * m2.n_elems / dt2, "unit": "element-integrations/s", "cores": 1,
                                 "sample": f"C3D20 {n2}^3 block ({m2.n_elems} elements) x {calls} calls of the "
                                           "reference's assemble_linear_static (src/fem/assembly.cpp:225-257), "
                                           "single-threaded"}
        except Exception as exc:  # the threaded figure above stands on its own
            out["as_shipped"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        return out
    port = Port()
    from oracle.oracle import make_material
    mats = [make_material(float(E), 0.3) for E in m.young]
    em = np.arange(m.n_elems, dtype=np.int32)
    nf = int((dof_eq >= 0).sum())
    t0 = time.perf_counter()
    elems = 0
    while time.perf_counter() - t0 < seconds:
        port.assemble_linear(m, mats, em, dof_eq, pre, nf)
        elems += m.n_elems
    dt = time.perf_counter() - t0
    return {"value": elems / dt, "unit": "element-integrations/s", "cores": 1, "kind": "port",
            "sample": f"C3D20 {n}^3 block x {elems // m.n_elems} passes through the oracle's C restatement"}


def accuracy_vs_reference(sysref):
    """Errors of the GPU's FP64 and mixed outputs against the reference's own FP64
    system of the same block (its element_stiffness + exact CSR scatter): K relative
    Frobenius, and displacements relative L2 after the same host sparse direct solve."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    import torch

    from calculixpp_b200 import Plan
    model, f = c3d20_model(sysref["n"], seed=sysref["seed"])
    nf = sysref["row_ptr"].size - 1
    k_ref = sp.csr_matrix((sysref["vals"], sysref["col_idx"], sysref["row_ptr"]), shape=(nf, nf))
    deq = sysref["dof_eq"]
    f_red = np.zeros(nf)
    free = deq >= 0
    np.add.at(f_red, deq[free], np.asarray(f, dtype=np.float64)[free])
    u_ref = spla.spsolve(k_ref.tocsc(), f_red + sysref["rhs"])
    plan = Plan(model)
    rp, ci = (t.cpu().numpy() for t in plan.pattern())
    out = {"block": f"{sysref['n']}^3", "checker": "reference element_stiffness + exact CSR scatter (FP64)",
           "bar_mixed_disp": 1e-6, "bar_fp64_K": 1e-12, "bar_fp64_disp": 1e-10}
    for prec in ("fp64", "mixed"):
        plan.set_precision(prec)
        v, r = plan.assemble_linear(torch.as_tensor(f, device=plan.device))
        k = sp.csr_matrix((v.cpu().numpy(), ci, rp), shape=(plan.n_free, plan.n_free))
        u = spla.spsolve(k.tocsc(), r.cpu().numpy())
        out[prec] = {"K_rel_fro": float(spla.norm(k - k_ref) / spla.norm(k_ref)),
                     "disp_rel_l2": float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref))}
    plan.close()
    out["pass"] = bool(out["mixed"]["disp_rel_l2"] <= 1e-6 and out["fp64"]["K_rel_fro"] <= 1e-12 and
                       out["fp64"]["disp_rel_l2"] <= 1e-10)
    return out


def reference_arm(args, rank, world):
    """--impl reference: the reference's own CPU implementation on the box's host cores."""
    if rank != 0:
        return
    out = None
    t_all = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(max(1.0, args.cpu_seconds / 4), seed=0, as_shipped=False)
        if i >= args.warmup:
            t_all.append(r["value"])
        out = r
    value = statistics.median(t_all)
    line = {"impl": "reference", "metric": "element-integrations/s (K_e+f_int+J2), mixed vs FP64",
            "value": value, "unit": "element-integrations/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"C3D20 27-point linear elastic block {args.n}^3 (sampled per step on the CPU)",
                       "sample_per_step": out["sample"],
                       "cpu_baseline_sample": "per-element rate measured on a C3D20 12^3 block of the same "
                                              "generator, reported against the 64^3 workload"},
            "cpu_baseline": {"value": value, "unit": out["unit"], "cores": out["cores"], "kind": out["kind"],
                             "sample": out["sample"]},
            "e2e": {"value": value, "unit": "element-integrations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_init(args.gpus)
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    import torch

    from calculixpp_b200 import Plan
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    model, f_ext = c3d20_model(args.n, seed=rank)
    plan = Plan(model, "mixed")
    m = model.mesh
    d_f = torch.as_tensor(f_ext, device=dev)
    vals = torch.empty(plan.nnz, dtype=torch.float64, device=dev)
    rhs = torch.empty(plan.n_free, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        plan.assemble_linear(d_f, vals=vals, rhs=rhs, check=False)

    results = {}
    clocks = None
    shapes = {}
    for prec in ("fp64", "mixed"):
        plan.set_precision(prec)
        shapes[prec] = {"default": True} if args.no_tune else plan.tune(step)
        for _ in range(args.warmup):
            step()
        plan.check()
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        if prec == "mixed":
            with ClockSampler(local) as cs:
                t = time_steps(step, args.steps, stream)
            clocks = cs.summary()
        else:
            t = time_steps(step, args.steps, stream)
        torch.cuda.synchronize()
        barrier(world)
        t = max_over_ranks(t, world)
        plan.check()
        results[prec] = {"t": t, "launch_shape": shapes[prec], "windows_and_ring": plan.windows()}

    # e2e through the C ABI with host buffers (pinned): load vector in, K_ff + rhs out.
    h_f = torch.as_tensor(f_ext).pin_memory()
    h_vals = torch.empty(plan.nnz, dtype=torch.float64).pin_memory()
    h_rhs = torch.empty(plan.n_free, dtype=torch.float64).pin_memory()
    import ctypes as C

    from calculixpp_b200 import _lib
    lib = _lib.load()
    e2e_steps = args.steps

    def e2e_step():
        _lib.check(lib.cxg_assemble_linear(plan.h, C.c_void_p(h_vals.data_ptr()), C.c_void_p(h_rhs.data_ptr()),
                                           C.c_void_p(h_f.data_ptr()), C.c_void_p(stream.cuda_stream)))

    e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)

    # free the C3D20 block before the other workloads
    B = algorithmic_bytes(plan, model)
    h2d, d2h = int(h_f.numel() * 8), int((h_vals.numel() + h_rhs.numel()) * 8)
    n_free, nnz = plan.n_free, plan.nnz
    del vals, rhs, d_f, h_vals, h_rhs, h_f
    plan.close()
    torch.cuda.empty_cache()
    j2 = j2_newton(args, world, dev, stream) if args.j2_n > 0 else None
    batch = batched(args, world, rank, dev, stream) if args.batch_models > 0 else None
    adj = adjoint_section(args, world, dev, stream) if args.adj_n > 0 else None

    # accuracy of the mixed path against FP64 on a reduced block (host sparse solve)
    acc = None
    if rank == 0:
        acc = mixed_accuracy(12)

    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    pipe = measure_peaks() if rank == 0 else {}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_seconds)
        if acc is not None and "_ref_system" in cpu:
            acc["vs_reference"] = accuracy_vs_reference(cpu.pop("_ref_system"))

    if rank != 0:
        return
    E = m.n_elems
    mix, f64 = results["mixed"], results["fp64"]
    value = world * E * args.steps / mix["t"]
    # one step is exactly the element pass + row gather pair, so the step's event time is
    # the pair's time per launch
    achieved = B / (mix["t"] / args.steps) / 1e9
    traffic = None
    if os.path.exists(TRAFFIC_FILE):
        traffic = json.load(open(TRAFFIC_FILE)).get(f"c3d20_{args.n}_mixed_linear")
    line = {
        "metric": "element-integrations/s (K_e+f_int+J2), mixed vs FP64",
        "value": value,
        "unit": "element-integrations/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mix["t"] / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic (seeded C3D20 block, lognormal E)",
        "config": {"workload": f"C3D20 27-point linear elastic block {args.n}^3",
                   "elements": E, "nodes": m.n_nodes, "n_free": n_free, "nnz": nnz,
                   "precision": "mixed: FP32 gradients/Gram blocks, FP64 Jacobians, diagonal blocks and accumulation",
                   "l2": "outputs (8*nnz bytes) far larger than L2; no flush needed",
                   "parallelism": f"independent block per GPU x{world}",
                   "cpu_baseline_sample": "per-element rate measured on a C3D20 12^3 block of the same "
                                          "generator (same element type, rule and scatter), reported beside "
                                          "the 64^3 GPU figure"},
        "launch_shape": mix["launch_shape"],
        "windows_and_ring": mix["windows_and_ring"],
        "targets": targets(j2, batch),
        "fp64": {"value": world * E * args.steps / f64["t"], "ms_per_step": f64["t"] / args.steps * 1e3,
                 "launch_shape": f64["launch_shape"],
                 "windows_and_ring": f64["windows_and_ring"],
                 "fp64_pipe": {"achieved_tflops": FLOPS_PER_ELEM_C3D20 * E / (f64["t"] / args.steps) / 1e12,
                               "peak_tflops": pipe.get("fp64_tflops"),
                               "peak_kind": "cuBLAS DGEMM 8192^3 measured in this run"}},
        "speedup_mixed_vs_fp64": f64["t"] / mix["t"],
        "mixed_accuracy": acc,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic,
                     "kernel": "p1_kernel + p2_kernel (element pass + row gather), C3D20 linear, mixed",
                     "kernel_ms": mix["t"] / args.steps * 1e3,
                     "algorithmic_bytes": B, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
        "j2_newton": j2,
        "batched": batch,
        "adjoint": adj,
        "cpu_baseline": cpu,
        "e2e": {"value": world * E * e2e_steps / t_e2e, "unit": "element-integrations/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps * 2,
        "clocks": clocks,
        "measured_pipe_peaks": pipe,
    }
    print(json.dumps(line), flush=True)


def targets(j2, batch):
    """The two throughput targets of the path, each beside its measured figure: the FP64
    C3D8 J2 residual + tangent at >= 60 % of the HBM roofline, and the mixed-precision
    batched path >= 2x the plain FP64 path in element-integrations/s."""
    out = {"fp64_j2_hbm_roofline_frac": {"target": 0.60, "measured": None},
           "batched_mixed_vs_plain_fp64": {"target": 2.0, "measured": None}}
    if j2:
        out["fp64_j2_hbm_roofline_frac"]["measured"] = j2["roofline_fp64"]["frac"]
    if batch and "speedup_batched_mixed_vs_plain_fp64" in batch:
        out["batched_mixed_vs_plain_fp64"]["measured"] = batch["speedup_batched_mixed_vs_plain_fp64"]
    return out


def mixed_accuracy(n):
    """Relative L2 displacement error of the mixed path against FP64 after the same
    host sparse direct solve, on an n^3 block of the benchmark workload."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    import torch

    from calculixpp_b200 import Plan
    model, f = c3d20_model(n, seed=0)
    plan = Plan(model)
    rp, ci = (t.cpu().numpy() for t in plan.pattern())
    out = {}
    u = {}
    for prec in ("fp64", "mixed"):
        plan.set_precision(prec)
        v, r = plan.assemble_linear(torch.as_tensor(f, device=plan.device))
        A = sp.csr_matrix((v.cpu().numpy(), ci, rp), shape=(plan.n_free, plan.n_free))
        u[prec] = spla.spsolve(A.tocsc(), r.cpu().numpy())
        out[f"K_{prec}"] = v.cpu().numpy()
    err_u = float(np.linalg.norm(u["mixed"] - u["fp64"]) / np.linalg.norm(u["fp64"]))
    err_k = float(np.linalg.norm(out["K_mixed"] - out["K_fp64"]) / np.linalg.norm(out["K_fp64"]))
    plan.close()
    return {"block": f"{n}^3", "disp_rel_l2": err_u, "K_rel_fro": err_k, "bar": 1e-6, "pass": err_u <= 1e-6}


if __name__ == "__main__":
    main()
