#!/usr/bin/env python
"""Laplace3D FMM matvec throughput on B200 (one JSON line on stdout).

Workload: SphericalHarmonics(Laplace3D(); p), ppl=64, 1,000,000 points uniform in the unit cube
(seed 3), FP64 charges N(0,1), potential and gradient at the sources. A step is one matvec =
build_expansions + evaluate_at_sources (the reference's definition, bench/bench.jl:44-50), the
tree/plan built once beforehand. The headline order is p = 11: the metric asks for ≤ 1e-6
relative error, and the configured p = 10 stays above it even in FP64 (1.7e-6 against direct
sums; p = 11 gives 7.3e-7). The configured order is measured beside it (configured_order_p10).

  value      evaluations/s of the mixed path (tensor-core FP16x3 M2L, FP32 near field),
             inputs resident in HBM, device time (CUDA events on the library's stream), L2
             flushed (256 MB write) between steps, max over ranks
  e2e        the same through the host-pointer C ABI call (fmmb_matvec) with pinned host
             buffers: copies in and out inside the timed region
  fp64       the plain FP64 path on the same inputs; mixed_vs_fp64 = the ratio
  error      relative L2 error of both paths against FP64 direct sums at 4096 sampled
             sources (computed on the device, fmmb_direct_dev)
  roofline   the dominant kernel of the mixed path (the M2L) against the measured peak
  cpu_baseline  the CPU oracle (C++ restatement of the reference CPU path) on this host
  parity     the oracle's outputs of that baseline run, and of one more at p = 10, against the
             device's at all 10^6 points: tree field by field (perm included) and far pairs per
             level, FP64 path max-norm relative (1e-12 potential, 1e-11 gradient), mixed path
             relative L2 (1e-6 potential)

Every figure goes on a "bench_detail" line first; the headline line after it carries the
contract's keys and a compact copy of the rest.

--impl reference times that CPU path alone (all host threads) as the reference arm.
--gpus N: N independent replicas (the single FMM is not sharded: replicas only), one
process per GPU under torch.distributed; value = N·1e6 / max-over-ranks step time.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "flexiblefmm.jl_b200"))

METRIC = "Laplace3D 1M-pt FMM evals/s @1e-6 err, mixed vs FP64 GPU; p50/p99 latency"
UNIT = "evals/s"


def args_():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=20)
    a.add_argument("--warmup", type=int, default=3)
    a.add_argument("--impl", default="ours", choices=["ours", "reference"])
    a.add_argument("--n", type=int, default=1_000_000)
    a.add_argument("--p", type=int, default=11)
    a.add_argument("--ppl", type=int, default=64)
    a.add_argument("--samples", type=int, default=4096)
    a.add_argument("--no-cpu-baseline", action="store_true")
    a.add_argument("--no-p10", action="store_true", help="skip the side measurement at the configured order p = 10")
    a.add_argument("--serve-requests", type=int, default=4096, help="requests of the serving measurement (0: skip it)")
    a.add_argument("--serve-slots", type=int, default=3)
    a.add_argument("--stokes-instances", type=int, default=64, help="instances of the batched Stokes measurement (0: skip it)")
    a.add_argument("--ki-points", type=int, default=2_000_000, help="points of the cube KI measurement (0: skip it)")
    a.add_argument("--no-circle-ki", action="store_true", help="skip the 2D circle KI measurement")
    a.add_argument("--peaks", action="store_true",
                   help="measure the FP64 (DGEMM) and FP32 (SGEMM, no TF32) rates of this GPU and exit")
    return a.parse_args()


def workload(n, seed=3):
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3))
    tau = rng.standard_normal(n)
    return pts, tau


def config(a, extra=None):
    c = {"workload": f"Laplace3D SphericalHarmonics p={a.p}, ppl={a.ppl}, {a.n:,} points uniform in the unit cube "
                     f"(seed 3), charges N(0,1), potential+gradient at the sources; step = build_expansions + "
                     f"evaluate_at_sources", "n_points": a.n, "p": a.p, "ppl": a.ppl,
         "l2": "flushed between steps (256 MB device write)", "parallelism": f"replicas{a.gpus}"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------- the CPU oracle (baseline / reference arm)
def cpu_oracle(pts, tau, p, ppl, reps, warmup=1, keep=False):
    """The oracle's matvec on all host threads: step times; with keep, the oracle FMM (its tree)
    and the outputs of the last step too."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = oracle.set_threads(0)
    t0 = time.perf_counter()
    f = oracle.FMM(p, pts, ppl)
    t_tree = time.perf_counter() - t0
    times = []
    out = None
    for r in range(warmup + reps):
        t0 = time.perf_counter()
        f.build_expansions(pts, tau)
        out = f.evaluate_at_sources()
        dt = time.perf_counter() - t0
        if r >= warmup:
            times.append(dt)
    res = dict(times=times, threads=threads, tree_s=t_tree)
    if keep:
        res.update(fmm=f, pot=out[0], grad=out[1])
    return res


def _mrd(a, b):
    """max-norm relative difference; rows of a 2-D array are vectors"""
    if a.ndim == 2:
        return float(np.max(np.linalg.norm(a - b, axis=1)) / np.max(np.linalg.norm(b, axis=1)))
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _rl2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


TREE_FIELDS = ("cell", "level", "parent", "child_first", "plo", "phi", "leaf", "ghost", "xlist", "has_source", "colleagues",
               "point_node", "perm")


def parity(dev, orc):
    """The device results of one order against the oracle's on the same points and charges:
    the tree field by field (perm included) and the far pairs of every level as sets; the FP64
    path's potential and gradient by max-norm relative difference (bars 1e-12 / 1e-11, the
    reference's CPU-vs-device tolerances); the mixed path's by relative L2 (bar 1e-6 on the
    potential, the metric's tolerance, 1e-5 on the gradient)."""
    T = orc["fmm"].tree
    t = dev["tree"]
    bad = [k for k in TREE_FIELDS if t[k].shape != getattr(T, k).shape or not np.array_equal(t[k], getattr(T, k))]
    pairs_ok, npairs = len(dev["pairs"]) == T.L, 0
    for l in range(min(T.L, len(dev["pairs"]))):
        a, b = np.stack(dev["pairs"][l]), np.stack(T.pairs(l))
        npairs += b.shape[1]
        if a.shape != b.shape or not np.array_equal(a[:, np.lexsort(a)], b[:, np.lexsort(b)]):
            pairs_ok = False
    ou, og = orc["pot"], orc["grad"]
    fu, fg = dev["fp64"]
    mu, mg = dev["mixed"]
    r = {"tree_equal": not bad and dev["nnodes"] == T.n, "mismatched_fields": bad, "nodes": int(T.n), "levels": int(T.L),
         "far_pairs_equal": pairs_ok, "far_pairs": int(npairs),
         "fp64_vs_oracle_maxrel": {"pot": _mrd(fu, ou), "grad": _mrd(fg, og)},
         "mixed_vs_oracle_rel_l2": {"pot": _rl2(mu, ou), "grad": _rl2(mg, og)}}
    r["pass"] = bool(r["tree_equal"] and pairs_ok and r["fp64_vs_oracle_maxrel"]["pot"] < 1e-12
                     and r["fp64_vs_oracle_maxrel"]["grad"] < 1e-11 and r["mixed_vs_oracle_rel_l2"]["pot"] < 1e-6
                     and r["mixed_vs_oracle_rel_l2"]["grad"] < 1e-5)
    return r


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pts, tau = workload(a.n)
    r = cpu_oracle(pts, tau, a.p, a.ppl, reps=a.steps, warmup=a.warmup)
    ms = 1e3 * statistics.mean(r["times"])
    v = a.n / (ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": config(a, {"precision": "fp64 (the reference CPU path restated in C++/OpenMP)"}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["threads"], "kind": "port",
                             "sample": f"full {a.n:,}-point matvec per step, mean of {a.steps} after {a.warmup} warm-up; "
                                       f"tree + operators {r['tree_s']:.2f} s untimed"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- replicas
def max_over_ranks(x, dist=None, device="cpu"):
    """The largest value of x over the ranks of the process group (x itself without one)."""
    import torch
    if dist is None or not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(n_per_rank, ms_per_step, world):
    """Whole-job evaluations/s of `world` independent replicas timed at the slowest rank."""
    return world * n_per_rank / (ms_per_step / 1e3)


# ---------------------------------------------------------------- clocks during the timed region
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                                       "-i", str(device)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}



# ---------------------------------------------------------------- the serving loop
def serving_workload(count, seed=6):
    """Requests as the serving configuration draws them: Laplace3D or Yukawa3D(kappa = 5) with
    equal probability, N log-uniform in [1e3, 5e5], points uniform in the unit cube or from 4
    Gaussians (sigma = 0.02) with equal probability, charges N(0,1), tolerance from
    {1e-3, 1e-6, 1e-9}. Each request is (points, charges, tol, kappa or None)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        kappa = 5.0 if rng.random() < 0.5 else None
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
        if rng.random() < 0.5:
            pts = rng.random((n, 3))
        else:
            c = 0.1 + 0.8 * rng.random((4, 3))
            pts = np.clip(c[rng.integers(0, 4, n)] + 0.02 * rng.standard_normal((n, 3)), 0.0, 1.0)
        out.append((pts, rng.standard_normal(n), float(rng.choice([1e-3, 1e-6, 1e-9])), kappa))
    return out


def serving(fmmb, device, count, slots):
    """Throughput and latency of the request server (same-kind requests grouped into batch plans,
    `slots` groups in flight): batched (all requests submitted at once), then open-loop Poisson
    arrivals at 80 % of the batched request rate (p50/p99 latency), and the same requests one at a
    time on the plain FP64 path (one request per plan, one slot)."""
    reqs = serving_workload(count)
    total = sum(len(r[0]) for r in reqs)
    srv = fmmb.Server(device, slots=slots)
    # warm-up: the first eighth of the requests at once (operators of every order and width
    # resident, the device pool grown)
    for k in [srv.submit(pts, tau, tol=tol, kappa=kappa) for pts, tau, tol, kappa in reqs[:max(6, count // 8)]]:
        srv.wait(k)
    t0 = time.perf_counter()
    tk = [srv.submit(pts, tau, tol=tol, kappa=kappa) for pts, tau, tol, kappa in reqs]
    infos = [srv.wait(k)[2] for k in tk]
    t_batch = time.perf_counter() - t0
    # where a request's time goes: its plan (tree, lists, operators, state) on the host against its
    # matvec (host call and span on the slot's stream), summed per path over the batched pass
    per_path = {}
    for (pts, tau, tol, kappa), i in zip(reqs, infos):
        key = ("yukawa" if kappa is not None else "laplace") + "_" + i["precision"]
        d = per_path.setdefault(key, {"requests": 0, "points": 0, "plan_s": 0.0, "matvec_s": 0.0, "device_s": 0.0})
        d["requests"] += 1
        d["points"] += len(pts)
        for k in ("plan_s", "matvec_s", "device_s"):
            d[k] += i[k]
    rate = 0.8 * count / t_batch                                       # requests/s offered in the open loop
    rng = np.random.default_rng(60)
    gaps = rng.exponential(1.0 / rate, count)
    t0 = time.perf_counter()
    tk = []
    due = t0
    for (pts, tau, tol, kappa), g in zip(reqs, gaps):
        due += g
        while time.perf_counter() < due:
            time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
        tk.append(srv.submit(pts, tau, tol=tol, kappa=kappa))
    lat = [srv.wait(k)[2]["latency_s"] for k in tk]
    t_open = time.perf_counter() - t0
    srv.close()
    one = fmmb.Server(device, slots=1, group_max=1)
    for pts, tau, tol, kappa in reqs[:3]:
        one.wait(one.submit(pts, tau, tol=tol, precision="fp64", kappa=kappa))
    t0 = time.perf_counter()
    seq_lat = []
    for pts, tau, tol, kappa in reqs:
        seq_lat.append(one.wait(one.submit(pts, tau, tol=tol, precision="fp64", kappa=kappa))[2]["latency_s"])
    t_seq = time.perf_counter() - t0
    one.close()
    q = lambda v, f: float(np.quantile(np.asarray(v) * 1e3, f))
    return {"requests": count, "slots": slots, "points": total,
            "group_mean": float(np.mean([i["group"] for i in infos])),
            "workload": "Laplace3D or Yukawa3D(kappa=5) 50/50, N log-uniform [1e3, 5e5], uniform or 4-Gaussian (sigma 0.02) "
                        "points, tol in {1e-3, 1e-6, 1e-9} (p and precision path chosen from tol) (seed 6)",
            "batched": {"evals_per_s": total / t_batch, "requests_per_s": count / t_batch, "seconds": t_batch},
            "open_loop": {"offered_requests_per_s": rate, "evals_per_s": total / t_open,
                          "fraction_of_batched": (total / t_open) / (total / t_batch),
                          "latency_ms": {"p50": q(lat, 0.5), "p99": q(lat, 0.99)}},
            "one_at_a_time_fp64": {"evals_per_s": total / t_seq, "latency_ms": {"p50": q(seq_lat, 0.5), "p99": q(seq_lat, 0.99)}},
            "paths": {"mixed": sum(i["precision"] == "mixed" for i in infos), "fp64": sum(i["precision"] == "fp64" for i in infos),
                      "yukawa": sum(r[3] is not None for r in reqs)},
            "time_per_path_s": per_path,
            "host_device_s": {"plan": sum(i["plan_s"] for i in infos), "matvec": sum(i["matvec_s"] for i in infos),
                              "device": sum(i["device_s"] for i in infos)}}

# ---------------------------------------------------------------- batched Stokes
def stokes_workload(count, seed=5):
    """The batched Stokes configuration: N log-uniform in [2e4, 2e5] points on the unit sphere
    jittered by U(-0.01, 0.01)^3, Stokeslets N(0,1)^3."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(2e4), np.log(2e5))))
        v = rng.standard_normal((n, 3))
        pts = v / np.linalg.norm(v, axis=1)[:, None] + rng.uniform(-0.01, 0.01, (n, 3))
        out.append((pts, rng.standard_normal((n, 3))))
    return out


def stokes_direct(src, f, sel):
    """FP64 Stokeslet velocities (1/8pi) sum_{j != i} [f_j/r + d(d.f_j)/r^3] at the sources sel."""
    out = np.zeros((len(sel), 3))
    for a in range(0, len(sel), 16):
        idx = sel[a:a + 16]
        d = src[idx, None, :] - src[None, :, :]
        r2 = np.einsum("tsk,tsk->ts", d, d)
        r2[np.arange(len(idx)), idx] = np.inf
        ir = 1.0 / np.sqrt(r2)
        df = np.einsum("tsk,sk->ts", d, f) * ir ** 3
        out[a:a + 16] = (np.einsum("ts,sk->tk", ir, f) + np.einsum("ts,tsk->tk", df, d)) / (8 * np.pi)
    return out


def stokes_batch(fmmb, torch, ctx, count, p=16, ppl=200, samples=32, steps=3):
    """The batched Stokes configuration as ONE batch plan (fmmb_batch_plan_create):
    StokesHarmonics(Stokeslet3D(); p = 16) self plans of `count` jittered unit-sphere point sets in
    the common box [-1.02, 1.02]^3, all trees built in one tree build and all instances evaluated
    by one call (one launch per pass and level). Timed: the plan (every tree, list and operator
    table) followed by one evaluation through host arrays (a call with new geometry), the
    evaluation alone with the inputs resident on the device (CUDA events on the library's stream,
    L2 flushed between steps), and the instances one at a time (each its own plan and evaluation,
    one operator cache). Every instance's velocities are compared bitwise with its own plan's, and
    their relative L2 error against FP64 direct sums at `samples` sampled sources is reported."""
    import ctypes as C
    L = fmmb.lib()
    reqs = stokes_workload(count)
    xs, fs = [x for x, _ in reqs], [f for _, f in reqs]
    total = sum(len(x) for x in xs)
    box = ((-1.02, -1.02, -1.02), 2.04)
    cache = fmmb.OperatorCache(fmmb.StokesHarmonics(fmmb.Stokeslet3D(), p=p))
    w = fmmb.BatchStokesFMMPlan(xs[:2], ppl=ppl, bbox=box, cache=cache)      # warm-up: operators resident
    fmmb.stokes_fmm_eval(w, stokeslets=w.fmm.concat(fs[:2]))
    del w
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bp = fmmb.BatchStokesFMMPlan(xs, ppl=ppl, bbox=box, cache=cache)
    t_plan = time.perf_counter() - t0
    F = bp.fmm.concat(fs)
    tuned = fmmb.autotune(bp.state, bp.sources, F)                     # the launch shapes, on these inputs
    t0 = time.perf_counter()
    vel = fmmb.stokes_fmm_eval(bp, stokeslets=F)
    t_eval_host = time.perf_counter() - t0
    P = lambda t: C.c_void_p(t.data_ptr())
    xd, fd = torch.from_numpy(bp.sources).cuda(), torch.from_numpy(F).cuda()
    vd = torch.zeros((total, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    step = lambda: fmmb._check(L.fmmb_stokes_eval_dev(bp.state._h, P(xd), P(fd), total, P(vd)))
    step()
    torch.cuda.synchronize()
    ev = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    ms_dev = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    same_dev = bool(np.array_equal(vd.cpu().numpy(), vel))
    del xd, fd, vd, flush
    # one at a time: each instance its own plan and evaluation (the same cache, so the same box)
    one = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for x, f in zip(xs, fs):
        sp = fmmb.StokesFMMPlan(x, ppl=ppl, bbox=box, cache=cache)
        one.append(fmmb.stokes_fmm_eval(sp, stokeslets=f))
        del sp
    t_seq = time.perf_counter() - t0
    parts = bp.fmm.split(vel)
    bitwise = sum(bool(np.array_equal(a, b)) for a, b in zip(parts, one))
    rng = np.random.default_rng(50)
    errs = []
    for x, f, v in zip(xs, fs, parts):
        sel = np.sort(rng.choice(len(x), samples, replace=False))
        ud = stokes_direct(x, f, sel)
        errs.append(float(np.linalg.norm(v[sel] - ud) / np.linalg.norm(ud)))
    fm = bp.fmm
    out = {"instances": count, "points": total, "p": p, "ppl": ppl, "precision": "fp64",
           "workload": "N log-uniform [2e4, 2e5] jittered unit-sphere points, N(0,1)^3 Stokeslets (seed 5), one batch "
                       "plan over all instances in the common box [-1.02, 1.02]^3",
           "plan": {"levels": fm.nlevels, "nodes": fm.nnodes, "far_pairs": fm.npairs, "seconds": t_plan},
           "batched": {"evals_per_s": total / (t_plan + t_eval_host), "seconds": t_plan + t_eval_host,
                       "what": "batch plan + one evaluation, host arrays"},
           "eval_device": {"evals_per_s": total / (ms_dev / 1e3), "ms": ms_dev, "steps": steps,
                           "what": "one evaluation of all instances, inputs resident, CUDA events",
                           "equals_host_path": same_dev},
           "eval_host": {"evals_per_s": total / t_eval_host, "seconds": t_eval_host},
           "one_at_a_time": {"evals_per_s": total / t_seq, "seconds": t_seq},
           "bitwise_equal_instances": bitwise, "tuned": tuned,
           "error": {"samples_per_instance": samples, "max": max(errs), "median": float(np.median(errs)),
                     "per_instance": [float(f"{e:.3g}") for e in errs]}}
    del bp, one
    return out


# ---------------------------------------------------------------- the cube KI method
def cube_ki_workload(n, seed=4):
    """The adaptive configuration: n points from 16 isotropic Gaussians (centres uniform in
    [0.1, 0.9]^3, sigma = 0.01), points outside the unit box redrawn; charges U(-1, 1) rounded to
    FP32 values (the configuration's Float32 densities)."""
    rng = np.random.default_rng(seed)
    c = 0.1 + 0.8 * rng.random((16, 3))
    pts = c[rng.integers(0, 16, n)] + 0.01 * rng.standard_normal((n, 3))
    bad = np.any((pts < 0) | (pts >= 1), axis=1)
    while bad.any():
        pts[bad] = c[rng.integers(0, 16, int(bad.sum()))] + 0.01 * rng.standard_normal((int(bad.sum()), 3))
        bad = np.any((pts < 0) | (pts >= 1), axis=1)
    tau = rng.uniform(-1, 1, n).astype(np.float32).astype(np.float64)
    return pts, tau


def cube_ki(fmmb, torch, ctx, n, steps, warmup, samples=4096):
    """CubeKernelIndependent{3}(Laplace3D(); p = 8, pc = 16, d = 0.1), ppl = 64, spectral M2L: the
    matvec (potential + gradient at the sources, inputs resident on the device, CUDA events on the
    library's stream) on the FP32 far/near-field path, its relative L2 error against FP64 direct
    sums, the stage times, and the spectral M2L stage's bytes per second."""
    import ctypes as C
    L = fmmb.lib()
    pts, tau = cube_ki_workload(n)
    P = lambda t: C.c_void_p(t.data_ptr())
    xyz_d = torch.from_numpy(pts).cuda()
    tau_d = torch.from_numpy(tau).cuda()
    pot_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    grad_d = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    m = fmmb.CubeKernelIndependent(fmmb.Laplace3D(), p=8)
    t0 = time.perf_counter()
    f = fmmb.FMM(m, pts, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0))
    plan_s = time.perf_counter() - t0
    st = fmmb.FMMState(f, "mixed")
    step = lambda: fmmb._check(L.fmmb_matvec_dev(st._h, P(xyz_d), P(tau_d), n, 3, P(pot_d), P(grad_d)))
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ev = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    names = ("gather", "p2m", "m2m", "m2l", "l2l", "eval")
    runs = []
    for _ in range(3):
        msa = (C.c_double * 6)()
        nl = C.c_int()
        fmmb._check(L.fmmb_profile_matvec(st._h, P(xyz_d), P(tau_d), n, 3, P(pot_d), P(grad_d), msa, 6, C.byref(nl)))
        runs.append(list(msa))
    stages = {k: statistics.median(r[i] for r in runs) for i, k in enumerate(names)}
    step()
    torch.cuda.synchronize()
    u, g = pot_d.cpu().numpy(), grad_d.cpu().numpy()
    rng = np.random.default_rng(8)
    sel = np.sort(rng.choice(n, size=min(samples, n), replace=False)).astype(np.int64)
    sel_d = torch.from_numpy(sel).cuda()
    tg_d = xyz_d[sel_d].contiguous()
    dp = torch.zeros(len(sel), dtype=torch.float64, device="cuda")
    dg = torch.zeros((len(sel), 3), dtype=torch.float64, device="cuda")
    fmmb._check(L.fmmb_direct_dev(ctx._h, P(xyz_d), P(tau_d), n, P(tg_d), P(sel_d), len(sel), P(dp), P(dg)))
    dp_h, dg_h = dp.cpu().numpy(), dg.cpu().numpy()
    err = {"pot_rel_l2": float(np.linalg.norm(u[sel] - dp_h) / np.linalg.norm(dp_h)),
           "grad_rel_l2": float(np.linalg.norm(g[sel] - dg_h) / np.linalg.norm(dg_h))}
    nfreq = 9 * 16 * 16
    # the Hadamard pull (k_ki_hadamard), the spectral stage's largest kernel, moves 16 B per far pair
    # and frequency through the SM's L1/shared-memory data pipe: the source's spectrum (FP32
    # complex, served by L1 and L2) and the offset's table entry (shared memory). That pipe, at
    # 128 B per cycle per SM, bounds it; DRAM stays near 5 % busy.
    l1_bytes = 16.0 * nfreq * f.npairs
    l1_peak = 148 * 128 * 1.965e9
    return {"workload": f"{n:,} points from 16 Gaussians (sigma 0.01, centres U[0.1, 0.9]^3, seed 4), charges U(-1,1) "
                        "as FP32 values; CubeKernelIndependent{3}(Laplace3D; p=8, pc=16, d=0.1), ppl=64, bbox (0,1); "
                        "potential + gradient at the sources",
            "precision": "FP32 spectra, far field (surface sums) and near field; FP64 dense translations",
            "evals_per_s": n / (ms / 1e3), "ms_per_step": ms, "plan_s": plan_s, "levels": f.nlevels, "nodes": f.nnodes,
            "far_pairs": f.npairs, "stages_ms": stages, "error": {"samples": len(sel), **err},
            "spectral_m2l": {"bound": "L1/shared-memory data pipe", "l1_bytes": l1_bytes,
                             "l1_TB_per_s_over_stage": l1_bytes / (stages["m2l"] / 1e3) / 1e12,
                             "l1_peak_TB_per_s": l1_peak / 1e12,
                             "note": "16 B per far pair and frequency (source spectrum + table entry) through L1/shared "
                                     "memory, over the whole spectral stage (forward transforms + Hadamard pull + "
                                     "inverse transforms); the peak is 148 SMs x 128 B/cycle at 1965 MHz"}}


# ---------------------------------------------------------------- the 2D circle KI method
def circle_ki(fmmb, n=100_000, nt=50_000, samples=2000, reps=5):
    """The CPU-runnable configuration on the device: KernelIndependent(Laplace2D(); nequiv = 60),
    ppl = 50, bbox ((0,0), 1), n sources uniform in the unit square with N(0,1) charges (seed 1)
    and nt uniform targets (seed 2): evaluate_at_sources and evaluate at the targets (potentials,
    host arrays in and out, the build of the expansions included), best of `reps`; relative L2
    error against FP64 direct sums (numpy) at `samples` sampled sources and targets."""
    pts = np.random.default_rng(1).random((n, 2))
    tau = np.random.default_rng(1).standard_normal(n)
    tg = np.random.default_rng(2).random((nt, 2))
    m = fmmb.KernelIndependent(fmmb.Laplace2D(), nequiv=60)
    t0 = time.perf_counter()
    f = fmmb.FMM(m, pts, ppl=50, bbox=((0.0, 0.0), 1.0))
    plan_s = time.perf_counter() - t0
    st = fmmb.FMMState(f, "fp64")
    best = None
    for _ in range(reps + 1):
        t0 = time.perf_counter()
        fmmb.build_expansions_(st, f, pts, tau)
        u = fmmb.evaluate_at_sources(f, st)
        ut = fmmb.evaluate(f, st, tg)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    rng = np.random.default_rng(3)
    ss = np.sort(rng.choice(n, samples, replace=False))
    st_ = np.sort(rng.choice(nt, samples, replace=False))
    c = -1 / (4 * np.pi)

    def direct(x, excl=None):
        out = np.zeros(len(x))
        for a in range(0, len(x), 256):
            r2 = ((x[a:a + 256, None, :] - pts[None, :, :]) ** 2).sum(-1)
            if excl is not None:
                r2[np.arange(len(r2)), excl[a:a + 256]] = 1.0
            out[a:a + 256] = c * np.log(r2) @ tau
        return out

    du, dt_ = direct(pts[ss], ss), direct(tg[st_])
    return {"workload": f"KernelIndependent(Laplace2D; nequiv=60), ppl=50, bbox ((0,0),1); {n:,} sources uniform in the "
                        f"unit square, N(0,1) charges (seed 1); {nt:,} uniform targets (seed 2); potentials at the sources and "
                        "at the targets, host arrays in and out, FP64",
            "seconds": best, "evals_per_s": (n + nt) / best, "plan_s": plan_s, "levels": f.nlevels, "nodes": f.nnodes,
            "far_pairs": f.npairs,
            "error": {"samples": samples, "sources_rel_l2": float(np.linalg.norm(u[ss] - du) / np.linalg.norm(du)),
                      "targets_rel_l2": float(np.linalg.norm(ut[st_] - dt_) / np.linalg.norm(dt_))}}


# ---------------------------------------------------------------- our arm
def run_ours(a):
    import torch
    import fmmb

    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    L = fmmb.lib()
    ctx = fmmb.default_context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    pts, tau = workload(a.n)
    xyz_d = torch.from_numpy(pts).cuda()
    tau_d = torch.from_numpy(tau).cuda()
    pot_d = torch.zeros(a.n, dtype=torch.float64, device="cuda")
    grad_d = torch.zeros((a.n, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    P = lambda t: C.c_void_p(t.data_ptr())

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # FP64 direct sums at sampled sources (device), the error oracle of every path and order
    rng = np.random.default_rng(7)
    sel = np.sort(rng.choice(a.n, size=min(a.samples, a.n), replace=False)).astype(np.int64)
    sel_d = torch.from_numpy(sel).cuda()
    tg_d = xyz_d[sel_d].contiguous()
    dp = torch.zeros(len(sel), dtype=torch.float64, device="cuda")
    dg = torch.zeros((len(sel), 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fmmb._check(L.fmmb_direct_dev(ctx._h, P(xyz_d), P(tau_d), a.n, P(tg_d), P(sel_d), len(sel), P(dp), P(dg)))
    dp_h, dg_h = dp.cpu().numpy(), dg.cpu().numpy()

    def measure(p, sample_clocks):
        """Both precision paths at order p: device step times, errors, stage times, launches."""
        m = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=p)
        t0 = time.perf_counter()
        f = fmmb.FMM(m, pts, ppl=a.ppl, bbox=((0.0, 0.0, 0.0), 1.0))
        plan_s = time.perf_counter() - t0
        states = {"mixed": fmmb.FMMState(f, "mixed"), "fp64": fmmb.FMMState(f, "fp64")}
        # the launch shapes tuned on these inputs (fmmb_autotune; no result depends on them): the
        # FP64 path's chunk width and near-field warps, then the mixed path's, with the plan's M2L
        # block size, which both paths share
        tuned = {"fp64": fmmb.autotune(states["fp64"], pts, tau, tune_blocks=False),
                 "mixed": fmmb.autotune(states["mixed"], pts, tau, tune_blocks=True)}

        def step(st):
            rc = L.fmmb_matvec_dev(st._h, P(xyz_d), P(tau_d), a.n, 3, P(pot_d), P(grad_d))
            if rc:
                fmmb._check(rc)

        def timed(st, k):
            times = []
            for _ in range(k):
                with torch.cuda.stream(stream):
                    flush.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    step(st)
                    e1.record(stream)
                times.append((e0, e1))
            torch.cuda.synchronize()
            return [e0.elapsed_time(e1) for e0, e1 in times]

        for name in ("mixed", "fp64"):
            for _ in range(a.warmup):
                step(states[name])
        torch.cuda.synchronize()
        clocks = Clocks(local) if (rank == 0 and sample_clocks) else None
        barrier()
        t_mixed = timed(states["mixed"], a.steps)
        barrier()
        t_fp64 = timed(states["fp64"], a.steps)
        barrier()
        clk = clocks.stop() if clocks else None
        r = {"p": p, "f": f, "states": states, "step": step, "plan_s": plan_s, "t_mixed": t_mixed, "clocks": clk,
             "tuned": tuned,
             "ms_mixed": max_over_ranks(statistics.mean(t_mixed), dist, "cuda"),
             "ms_fp64": max_over_ranks(statistics.mean(t_fp64), dist, "cuda")}
        err = {}
        dev = {"tree": f.tree(), "pairs": [f.pairs(l) for l in range(f.nlevels)], "nnodes": f.nnodes}
        for name in ("mixed", "fp64"):
            step(states[name])
            torch.cuda.synchronize()
            dev[name] = (pot_d.cpu().numpy().copy(), grad_d.cpu().numpy().copy())
            u, g = dev[name][0][sel], dev[name][1][sel]
            err[name] = {"pot_rel_l2": float(np.linalg.norm(u - dp_h) / np.linalg.norm(dp_h)),
                         "grad_rel_l2": float(np.linalg.norm(g - dg_h) / np.linalg.norm(dg_h))}
        r["error"], r["dev"] = err, dev
        # stage times of one matvec per path (median of 3, CUDA events on the library's stream)
        stages, launches = {}, {}
        names = ("gather", "p2m", "m2m", "m2l", "l2l", "eval")
        for name in ("mixed", "fp64"):
            runs = []
            for _ in range(3):
                with torch.cuda.stream(stream):
                    flush.zero_()
                ms = (C.c_double * 6)()
                nl = C.c_int()
                fmmb._check(L.fmmb_profile_matvec(states[name]._h, P(xyz_d), P(tau_d), a.n, 3, P(pot_d), P(grad_d), ms, 6,
                                                   C.byref(nl)))
                runs.append(list(ms))
                launches[name] = nl.value
            stages[name] = {k: statistics.median(x[i] for x in runs) for i, k in enumerate(names)}
        r["stages"], r["launches"] = stages, launches
        return r

    # the configured order (p = 10) first, then the headline order
    side, dev10 = None, None
    if a.p != 10 and not a.no_p10:
        r10 = measure(10, False)
        side = {"p": 10, "value": replica_throughput(a.n, r10["ms_mixed"], world), "ms_per_step": r10["ms_mixed"],
                "fp64": {"value": replica_throughput(a.n, r10["ms_fp64"], world), "ms_per_step": r10["ms_fp64"]},
                "mixed_vs_fp64": r10["ms_fp64"] / r10["ms_mixed"], "error": {"samples": len(sel), **r10["error"]},
                "stages_ms": r10["stages"]}
        dev10 = r10["dev"]
        del r10
    R = measure(a.p, True)
    f, states, t_mixed = R["f"], R["states"], R["t_mixed"]
    ms_mixed, ms_fp64, stages, launches, err, clk = R["ms_mixed"], R["ms_fp64"], R["stages"], R["launches"], R["error"], R["clocks"]
    plan_s = R["plan_s"]

    # end to end through the host-pointer C ABI call, pinned buffers
    xyz_h = torch.from_numpy(pts).pin_memory()
    tau_h = torch.from_numpy(tau).pin_memory()
    pot_h = torch.zeros(a.n, dtype=torch.float64).pin_memory()
    grad_h = torch.zeros((a.n, 3), dtype=torch.float64).pin_memory()
    st = states["mixed"]
    for _ in range(a.warmup):
        fmmb._check(L.fmmb_matvec(st._h, P(xyz_h), P(tau_h), a.n, 3, P(pot_h), P(grad_h)))
    e2e = []
    for _ in range(a.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fmmb._check(L.fmmb_matvec(st._h, P(xyz_h), P(tau_h), a.n, 3, P(pot_h), P(grad_h)))
        e2e.append(time.perf_counter() - t0)
    barrier()
    e2e_s = max_over_ranks(statistics.mean(e2e), dist, "cuda")

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    np_ = (a.p + 1) ** 2
    m2l_flops = 2.0 * f.npairs * np_ * np_                    # the algorithmic FP64-equivalent M2L work
    t_m2l = stages["mixed"]["m2l"] / 1e3
    achieved = m2l_flops / t_m2l / 1e12
    peak = peaks.get("bf16_tflops", 1590.0)
    traffic = None
    tp = os.path.join(ROOT, "profiles", "m2l_traffic.json")
    if os.path.exists(tp):
        tj = json.load(open(tp))
        traffic = tj.get("dram_bytes_per_launch_full") or tj.get("dram_bytes_per_launch")
    lat = sorted(t_mixed)
    pct = lambda q: lat[min(len(lat) - 1, int(round(q * (len(lat) - 1))))]
    cpu, par = None, {}
    if world == 1 and not a.no_cpu_baseline:
        r = cpu_oracle(pts, tau, a.p, a.ppl, reps=2, warmup=1, keep=True)
        cpu = {"value": a.n / min(r["times"]), "unit": UNIT, "cores": r["threads"], "kind": "port",
               "sample": f"full {a.n:,}-point matvec (the same points and charges), best of 2 after 1 warm-up, "
                         f"tree + operators {r['tree_s']:.2f} s untimed"}
        par[f"p{a.p}"] = parity(R["dev"], r)
        del r
        if dev10 is not None:
            r = cpu_oracle(pts, tau, 10, a.ppl, reps=1, warmup=0, keep=True)
            par["p10"] = parity(dev10, r)
            del r
    del dev10
    R.pop("dev", None)
    serve = serving(fmmb, local, a.serve_requests, a.serve_slots) if a.serve_requests > 0 else None
    stokes = stokes_batch(fmmb, torch, ctx, a.stokes_instances) if a.stokes_instances > 0 else None
    ki = cube_ki(fmmb, torch, ctx, a.ki_points, 5, 3) if a.ki_points > 0 else None
    kic = None if a.no_circle_ki else circle_ki(fmmb)
    # every figure, on a line of its own before the headline
    detail = {"configured_order_p10": side, "serving": serve, "stokes_batched": stokes, "cube_ki": ki, "circle_ki": kic,
              "parity": par, "plan_s": plan_s, "stages_ms": stages, "error": {"samples": len(sel), **err},
              "tuned": R["tuned"]}
    print(json.dumps({"bench_detail": detail}), flush=True)
    line = {
        "metric": METRIC, "value": replica_throughput(a.n, ms_mixed, world), "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp16x3 M2L (tcgen05 kind::f16, FP32 accumulation); f32 P2M, L2P and near field (FP64 batch sums); f64 M2M/L2L (DMMA)",
        "data": "synthetic (seeded uniform points, N(0,1) charges)",
        "config": config(a, {"precision": "mixed", "levels": f.nlevels, "nodes": f.nnodes, "far_pairs": f.npairs}),
        "roofline": {"bound": "tensor", "kernel": "k_m2l_tc (M2L, all levels, one launch)", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if "bf16_tflops" in peaks else "fallback",
                     "work": f"{f.npairs:,} far pairs x 2 x {np_}^2 flop"},
        "e2e": {"value": world * a.n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": a.n * 32, "d2h_bytes_per_step": a.n * 32},
        "gpu_launches": launches["mixed"] * a.steps,
        "clocks": clk,
        "cpu_baseline": cpu,
        # the rest is a compact copy of the detail line's figures
        "latency_ms": {"p50": _sig(pct(0.5)), "p99": _sig(pct(0.99))},
        "fp64": {"value": _sig(replica_throughput(a.n, ms_fp64, world)), "ms_per_step": _sig(ms_fp64)},
        "mixed_vs_fp64": _sig(ms_fp64 / ms_mixed),
        "error": {"samples": len(sel), **_sig(err)},
        "parity": compact_parity(par),
        "side": compact_side(side, serve, stokes, ki, kic),
    }
    print(json.dumps(line), flush=True)
    del states, f
    if dist:
        dist.destroy_process_group()


def _sig(x, d=4):
    """x with floats rounded to d significant digits (nested dicts and lists too)"""
    if isinstance(x, dict):
        return {k: _sig(v, d) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_sig(v, d) for v in x]
    if isinstance(x, float):
        return float(f"{x:.{d}g}")
    return x


def compact_parity(par):
    out = {}
    for k, r in par.items():
        out[k] = {"pass": r["pass"], "fp64_maxrel": _sig(r["fp64_vs_oracle_maxrel"], 3),
                  "mixed_rel_l2": _sig(r["mixed_vs_oracle_rel_l2"], 3)}
    return out


def compact_side(p10, serve, stokes, ki, kic):
    s = {}
    if p10:
        s["p10"] = {"value": _sig(p10["value"]), "fp64": _sig(p10["fp64"]["value"]),
                    "err_mixed": _sig(p10["error"]["mixed"]["pot_rel_l2"], 3), "err_fp64": _sig(p10["error"]["fp64"]["pot_rel_l2"], 3)}
    if serve:
        s["serving"] = {"requests": serve["requests"], "batched": _sig(serve["batched"]["evals_per_s"]),
                        "open_frac": _sig(serve["open_loop"]["fraction_of_batched"], 3),
                        "p50_ms": _sig(serve["open_loop"]["latency_ms"]["p50"], 3), "p99_ms": _sig(serve["open_loop"]["latency_ms"]["p99"], 3),
                        "fp64_one": _sig(serve["one_at_a_time_fp64"]["evals_per_s"])}
    if stokes:
        s["stokes"] = {"instances": stokes["instances"], "batched": _sig(stokes["batched"]["evals_per_s"]),
                       "eval_dev": _sig(stokes["eval_device"]["evals_per_s"]), "one": _sig(stokes["one_at_a_time"]["evals_per_s"]),
                       "bitwise": stokes["bitwise_equal_instances"], "err_max": _sig(stokes["error"]["max"], 3)}
    if ki:
        s["cube_ki"] = {"value": _sig(ki["evals_per_s"]), "ms": _sig(ki["ms_per_step"]), "m2l_ms": _sig(ki["stages_ms"]["m2l"]),
                        "err": _sig(ki["error"]["pot_rel_l2"], 3)}
    if kic:
        s["circle_ki"] = {"value": _sig(kic["evals_per_s"]), "err": _sig(kic["error"]["sources_rel_l2"], 3)}
    return s


def measure_peaks(reps=10):
    """The FP64 and FP32 denominators of the FP64 kernels' rooflines: cuBLAS DGEMM (FP64 tensor
    cores, DMMA) and SGEMM with TF32 off (FP32 FMA on the CUDA cores), square n = 8192, the best
    of `reps` CUDA-event timings after three warm-ups (2n³ flop each), then the same back to back
    for about three seconds (sustained), with the SM clocks sampled meanwhile."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.backends.cudnn.allow_tf32 = False
    out = {"gpu_name": torch.cuda.get_device_name(0), "n": 8192}
    clk = Clocks(torch.cuda.current_device())
    for key, dt in (("fp64_dgemm_tflops", torch.float64), ("fp32_sgemm_tflops", torch.float32)):
        n = 8192
        g = torch.Generator(device="cuda").manual_seed(1)
        x = torch.randn(n, n, dtype=dt, device="cuda", generator=g)
        y = torch.randn(n, n, dtype=dt, device="cuda", generator=g)
        z = torch.empty(n, n, dtype=dt, device="cuda")
        for _ in range(3):
            torch.matmul(x, y, out=z)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(x, y, out=z)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k = max(1, int(3000.0 / best))
        e0.record()
        for _ in range(k):
            torch.matmul(x, y, out=z)
        e1.record()
        e1.synchronize()
        flop = 2.0 * n ** 3
        out[key] = round(flop / (best * 1e-3) / 1e12, 2)
        out[key + "_sustained"] = round(flop * k / (e0.elapsed_time(e1) * 1e-3) / 1e12, 2)
        del x, y, z
    out["clocks"] = clk.stop()
    print(json.dumps(out))


def main():
    a = args_()
    if a.peaks:
        measure_peaks()
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
