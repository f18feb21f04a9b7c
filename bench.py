#!/usr/bin/env python
"""Benchmark of the batched edge-step collision checker on one B200.

Workload (the batched plain-GPU-checker configuration): 6-DOF arm whose
links are hulls of 16 points on an ellipsoid (0.15/0.04/0.04 m), 64 hull
obstacles of 12-32 points, 2^20 uniform samples in [-pi,pi]^6, the vertex
check, then k=10 nearest free neighbours -> ~4M undirected edges of uneven
length, discretised at dq = 0.01 rad; FP32 with the FP64 band recheck
(|margin| < 1e-5 m).  All inputs are seeded synthetic data.

One step = one pass of the edge checker over the whole edge batch.
  value  nominal edge-step checks/s (sum of testnum / time) of the device
         entry point on inputs resident in HBM (CUDA events on the launch
         stream, max over ranks);
  e2e    the same through the host-buffer C ABI (indicator2): host->device
         copies of qs/qe and the device->host read of res inside the timed
         region;
  roofline  FP32 pipe: counted FP32 operations of the checked steps over
         the FP32 check kernel's event-timed duration, against the measured
         FP32 FMA peak of the device;
  cpu_baseline  GPUPRM's own CPU checker (oracle/_ref, compiled from the
         reference sources) on a bounded sample of the same edges, all host
         cores, one checker instance per thread.

Extra legs in the same line (not part of `value`):
  prm        learned-guided vs plain GPU PRM time-to-path on the same scene
             (2^20 samples, 1000 seeded queries; the predictor is trained on
             2^20 exact-checker labels by the library's BF16 kernels);
  prm_stress the same on the 7-DOF wall scene (512 obstacles, two walls with
             a 0.12 m gap, dq 0.005, k 16, 2^20 samples);
  stress_edges  checker throughput on the 7-DOF wall scene at full size
             (2^22 samples, k=16, dq 0.005): vertex checks/s and edge-step
             checks/s on 2^21 of the roadmap's edges, with the reference CPU
             checker on a bounded sample of them;
  mlp        collision-predictor inference on 2^22 rows: the fused tcgen05
             kernel against per-layer tcgen05 kernels and the training GEMMs;
             training throughput (batch 4096) with tcgen05 and mma.sync GEMMs;
  batch      256 independent problems in one graph-captured launch per kind
             against a loop of per-problem launches;
  box4_prm   the reference's own CPU planning case: 4-DOF box arm, 16 box
             obstacles, C-space radius 0.5 rad, dq 0.02 rad; GPUPRM's
             planner (oracle/_ref/prm_dropin: process_mpi5 on its CPU
             checker, and on this library's checker behind the same
             interface) against the GPU eager and lazy PRMs, 8192 samples
             upwards, on the same seeded free start/goal pairs.

--impl reference times only that CPU checker (same metric/config).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes per edge of one k_check_edges launch on this workload at full
# size (the default last-colliding-step policy, fast arithmetic; one launch
# captured by ncu with dram__bytes_read.sum and dram__bytes_write.sum:
# 159.34 MB + 29.60 MB for 2,926,333 edges).
DRAM_BYTES_PER_EDGE = 188.94e6 / 2926333

METRIC = "edge-step collision checks/s"
UNIT = "edge-steps/s"
WORKLOAD = dict(workload="hull6 batched edges: 6-DOF ellipsoid-hull arm, 64 hull obstacles, "
                         "2^20 samples, kNN k=10, dq=0.01 rad, FP64 band 1e-5 m",
                ndof=6, obstacles=64, samples=1 << 20, k=10, dq=0.01, band_m=1e-5)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--samples", type=int, default=1 << 20)
    ap.add_argument("--k", type=int, default=10)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--policy", default="all", choices=["early", "all"])
    ap.add_argument("--arith", default="fast", choices=["fast", "exact"],
                    help="FP32 arithmetic of the checks: fast (GPRM_MODE_FAST) or the reference's exact operations")
    ap.add_argument("--no-prm", action="store_true", help="skip the PRM time-to-path comparison")
    ap.add_argument("--prm-samples", type=int, default=1 << 20)
    ap.add_argument("--no-stress", action="store_true", help="skip the 7-DOF wall planner comparison")
    ap.add_argument("--stress-samples", type=int, default=1 << 20)
    ap.add_argument("--no-stress-edges", action="store_true", help="skip the 7-DOF wall checker throughput leg")
    ap.add_argument("--stress-edges", type=int, default=1 << 21, help="roadmap edges the stress leg checks")
    ap.add_argument("--no-batch", action="store_true", help="skip the many-problem batch leg")
    ap.add_argument("--no-sampler", action="store_true", help="skip the near-node sampler leg")
    ap.add_argument("--batch-problems", type=int, default=256)
    ap.add_argument("--no-box4", action="store_true", help="skip the 4-DOF reference planner comparison")
    ap.add_argument("--box4-queries", type=int, default=6)
    ap.add_argument("--no-mlp", action="store_true", help="skip the predictor inference leg")
    ap.add_argument("--mlp-rows", type=int, default=1 << 22)
    ap.add_argument("--only-mlp", action="store_true",
                    help="run only the predictor inference leg and print it (profiling)")
    return ap.parse_args()


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(prefix="gprm_clocks_", suffix=".csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU leg (GPUPRM's own CPU checker; the oracle restatement if it is absent)
# --------------------------------------------------------------------------

def cpu_reference_rate(scene, qs_np, qe_np, dq, seconds, seed=0, count_ops=True):
    """Times the reference CPU checker on a bounded sample of the edges with
    all host cores.  Returns (dict for cpu_baseline, work counts, sample):
    the work counts are the reference algorithm's FP32 operations per step
    and per pair test, counted by the oracle's instrumented restatement on
    256 of the edges (None without count_ops); the sample holds the edge
    indices timed and the reference's codes for them (kept for the verdict
    parity check)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(seed + 77)
    order = rng.permutation(qs_np.shape[0])
    orc = O.Oracle(scene)
    work = None
    if count_ops:
        cnt_idx = order[:256]
        ops = orc.count_ops_edges(qs_np[cnt_idx], qe_np[cnt_idx], dq)
        tn_cnt = orc.testnum(qs_np[cnt_idx], qe_np[cnt_idx], dq)
        flops = ops["add"] + ops["mul"] + ops["div"] + ops["sqrt"]
        work = {"ref_flops_per_step": flops / max(1, int(tn_cnt.sum())),
                "flops_per_pair_test": flops / max(1.0, ops["pairs"])}
    if O.ref_available():
        ref = O.RefChecker(scene, dq=dq, nbuf=4096)
        kind = "reference"
        run = lambda a, b: ref.check_edges_mt(a, b, cores, chunk=16)
    else:
        kind = "port"
        cores = 1
        run = lambda a, b: orc.check_edges(a, b, dq, O.FP32)[0]
    # calibrate on a small slice, then size the sample to `seconds`
    cal = order[256:256 + 64 * cores]
    t0 = time.perf_counter()
    run(qs_np[cal], qe_np[cal])
    dt = max(1e-3, time.perf_counter() - t0)
    n = int(len(cal) * seconds / dt)
    n = max(64, min(n, qs_np.shape[0]))
    idx = order[:n]
    a, b = qs_np[idx], qe_np[idx]
    steps = int(orc.testnum(a, b, dq).sum())
    t0 = time.perf_counter()
    ref_res = run(a, b)
    dt = time.perf_counter() - t0
    return ({"value": steps / dt, "unit": UNIT, "cores": cores, "kind": kind,
             "sample": f"{n} random edges of the workload ({steps} edge steps), indicator2 in chunks "
                       f"of <=4096 edges per thread, {dt:.1f} s"}, work,
            {"idx": idx, "ref_res": np.asarray(ref_res), "kind": kind, "steps": steps})


def edge_parity(scene, qs_np, qe_np, dq, band, sample, gpu_res, what):
    """Verdict parity of the GPU's edge results with the reference CPU
    checker's on the timed CPU sample: the oracle classifies every sampled
    edge as decided outside the band (free / not free) or inside it (with
    its FP32 + FP64-band result), all host threads; see oracle/parity.py."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import parity as P
    idx = sample["idx"]
    t0 = time.perf_counter()
    cls, band_res, nin = O.Oracle(scene).edge_classify(qs_np[idx], qe_np[idx], dq, O.DEVICE_TRIG, band,
                                                       threads=os.cpu_count() or 1)
    d = P.verdict_parity(gpu_res[idx], sample["ref_res"], cls, band_res, nin)
    d.update({"what": what, "reference": sample["kind"], "edge_steps": int(sample["steps"]), "band_m": band,
              "oracle_seconds": time.perf_counter() - t0, "ok": P.parity_ok(d)})
    return d


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------

def check_mode(args) -> int:
    """FP32 with the FP64 band recheck, in the requested arithmetic."""
    from gpuprm_b200._abi import GPRM_MODE_FAST, GPRM_MODE_FP64_BAND
    return GPRM_MODE_FP64_BAND | (GPRM_MODE_FAST if args.arith == "fast" else 0)


def replica_seed(seed: int, rank: int) -> int:
    """Each rank checks its own replica of the workload (independent seeded
    samples, the same scene and sizes): weak scaling, no data exchange."""
    return seed + 7919 * rank


def reduce_over_ranks(values_max, values_sum, device=None):
    """(max over ranks of each of values_max, sum over ranks of each of
    values_sum) through the default process group; the values themselves
    for a single process.  Every rank must call it with the same lengths."""
    import torch
    dist = torch.distributed
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values_max], [float(v) for v in values_sum]
    out = []
    for vals, op in ((values_max, dist.ReduceOp.MAX), (values_sum, dist.ReduceOp.SUM)):
        if len(vals):
            t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
            dist.all_reduce(t, op=op)
            out.append([float(x) for x in t.cpu().tolist()])
        else:
            out.append([])
    return out[0], out[1]


def run_ours(args, rank, world, local_rank):
    import torch
    from gpuprm_b200 import workloads
    from gpuprm_b200._abi import GPRM_EDGES_ALL_STEPS, GPRM_EDGES_EARLY_EXIT
    from gpuprm_b200.configspace import measure_fp32_peak

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    ws = workloads.edge_workload("hull6", seed=replica_seed(args.seed, rank), n_samples=args.samples, k=args.k,
                                 dq=WORKLOAD["dq"], device=str(dev))
    cs = ws["space"]
    cs.set_mode(check_mode(args))
    policy = GPRM_EDGES_EARLY_EXIT if args.policy == "early" else GPRM_EDGES_ALL_STEPS
    cs.set_edge_policy(policy)
    qs, qe = ws["qs"], ws["qe"]
    E = qs.shape[1]
    res = torch.empty(E, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(max(3, args.warmup)):
        cs.check_edges_device(qs, qe, res)
    torch.cuda.synchronize()
    barrier()
    s0 = cs.stats()
    cs.profile_enable(True)
    clk = ClockSampler(local_rank)
    clk.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        cs.check_edges_device(qs, qe, res)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t = e0.elapsed_time(e1) / 1e3
    clocks = clk.stop()
    prof = cs.profile_read()
    s1 = cs.stats()
    cs.profile_enable(False)
    nominal = (s1["edge_steps_nominal"] - s0["edge_steps_nominal"])
    executed = (s1["edge_steps_executed"] - s0["edge_steps_executed"])
    band = (s1["band_rechecks"] - s0["band_rechecks"])
    launches = s1["launches"] - s0["launches"]
    colliding = int((res != 0).sum().item())

    # max over ranks of the device time; totals over ranks
    (t_max,), (nominal_all, executed_all) = reduce_over_ranks([t], [nominal, executed], dev)
    nominal_all, executed_all = int(nominal_all), int(executed_all)

    # e2e through the host-buffer C ABI (H2D + D2H inside the timed region)
    qs_np = np.ascontiguousarray(qs.cpu().numpy())
    qe_np = np.ascontiguousarray(qe.cpu().numpy())
    res_np = np.zeros(E, np.int32)
    cs.indicator2(qs_np, qe_np, res_np, E, E)   # warm-up (allocates pinned staging)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cs.indicator2(qs_np, qe_np, res_np, E, E)
    t_e2e = time.perf_counter() - t0
    (t_e2e,), _ = reduce_over_ranks([t_e2e], [], dev)
    assert np.array_equal(res_np, res.cpu().numpy()), "host and device entry points disagree"

    if rank != 0:
        return None
    peak = measure_fp32_peak()
    cpu = None
    work = None
    parity = None
    if not args.no_cpu_baseline and world == 1:
        qs_r = np.ascontiguousarray(qs_np.T)
        qe_r = np.ascontiguousarray(qe_np.T)
        cpu, work, sample = cpu_reference_rate(ws["scene"], qs_r, qe_r, WORKLOAD["dq"], args.cpu_seconds,
                                               args.seed)
        parity = edge_parity(ws["scene"], qs_r, qe_r, WORKLOAD["dq"], WORKLOAD["band_m"], sample, res_np,
                             "headline edges (FP64 band mode, %s policy) vs the reference CPU checker"
                             % ("early-exit" if args.policy == "early" else "last-colliding-step"))
    k_ms = prof["fp32_ms"] / max(1, prof["fp32_launches"])
    per = lambda key: (s1[key] - s0[key]) / max(1, args.steps)
    full_pl, cert_pl, exec_pl = per("pairs_tested"), per("pairs_certified"), executed / max(1, args.steps)
    roof = None
    if work is not None:
        nd, ns = ws["scene"].ndof, ws["scene"].ndof
        # achieved: the reference algorithm's FP32 operations for the steps of
        # one launch (the oracle's instrumented restatement counts FK and every
        # pair iteration of the reference's edge check on a sample of the same
        # edges, per nominal step) over the FP32 check kernel's event time.
        # The separation certificates settle 98% of the pair tests without
        # running them, so this is the throughput in the reference's own
        # arithmetic; the operations the kernel actually executes are given
        # as executed_tflops.
        nominal_pl = nominal / max(1, args.steps)
        achieved = work["ref_flops_per_step"] * nominal_pl / (k_ms * 1e-3) / 1e12
        exec_flops = full_pl * work["flops_per_pair_test"] + cert_pl * 8.0 + exec_pl * (45.0 * nd + 18.0 * ns)
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": DRAM_BYTES_PER_EDGE * E,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_check_edges launch "
                                  "of this workload at full size (159.34 + 29.60 MB for 2,926,333 edges, default "
                                  "policy), per edge x this run's edges",
                "algorithmic_bytes": int(2 * qs.numel() * 4 + E * 4),
                "peak_source": "measured FP32 FMA probe on this device (2 flops/FMA); "
                               "MEASURED_PEAKS.json has no FP32 entry",
                "counting": "algorithmic: the reference algorithm's FP32 ops per nominal edge step (oracle "
                            "counter, FMA=2, add/mul=1, div/sqrt counted) x nominal steps per launch",
                "executed_tflops": exec_flops / (k_ms * 1e-3) / 1e12,
                "frac_executed": exec_flops / (k_ms * 1e-3) / 1e12 / peak,
                "frac_note": "frac counts the reference algorithm's operations for every nominal step; the "
                             "separation certificates settle 98.6% of the pair tests without running them, so "
                             "frac > 1 measures work avoided; frac_executed is the FP32 work the kernel runs",
                "ref_flops_per_step": work["ref_flops_per_step"],
                "kernel_ms": k_ms, "pairs_certified_frac": cert_pl / max(1.0, cert_pl + full_pl),
                "fp64_recheck_ms_per_launch": prof["fp64_ms"] / max(1, prof["fp32_launches"])}
    prm = prm_stress = None
    if not args.no_prm and world == 1:
        prm = prm_leg(args, "hull6", WORKLOAD["dq"], args.prm_samples, 10)
        if not args.no_stress:
            prm_stress = prm_leg(args, "wall7", 0.005, args.stress_samples, 16)
    stress_edges = None
    if not args.no_stress_edges and world == 1:
        stress_edges = stress_edges_leg(args, dev, policy)
    batch = None
    if not args.no_batch and world == 1:
        batch = batch_leg(args, dev, policy)
    sampler = None
    if not args.no_sampler and world == 1:
        sampler = sampler_leg(args, ws, dev)
    mlp = None
    if not args.no_mlp and world == 1:
        mlp = mlp_leg(args, dev)
    box4 = None
    if not args.no_box4 and world == 1:
        box4 = box4_leg(args)
    line = {
        "metric": METRIC, "value": nominal_all / t_max, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": 1e3 * t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (+f64 band)",
        "data": "synthetic (seeded)",
        "config": dict(WORKLOAD, edges_per_gpu=E, free_samples=ws["n_free"], policy=args.policy, arith=args.arith,
                       l2="inputs (qs,qe: %.0f MB) larger than L2" % (2 * qs.numel() * 4 / 1e6)),
        "executed_steps_per_s": executed_all / t_max,
        "nominal_steps_per_step": nominal // args.steps, "executed_steps_per_step": executed // args.steps,
        "colliding_edges": colliding, "band_rechecks_per_step": band / args.steps,
        "e2e": {"value": nominal_all / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(2 * qs.numel() * 4),
                "d2h_bytes_per_step": int(E * 4)},
        "roofline": roof, "cpu_baseline": cpu, "parity": parity, "clocks": clocks, "gpu_launches": launches,
        "prm": prm, "prm_stress": prm_stress, "stress_edges": stress_edges, "batch": batch, "sampler": sampler,
        "mlp": mlp, "box4_prm": box4,
    }
    return line


def prm_leg(args, kind, dq, n_samples, k):
    """Learned-guided vs plain GPU PRM on one scene: the predictor is trained
    on 2^20 exact-checker labels (10 epochs, batch 4096, lr 1e-3) by the
    library's BF16 kernels, then the planners answer 1000 seeded queries."""
    from gpuprm_b200 import planner, scenes as _sc
    from gpuprm_b200.configspace import RobotConfigspace as _RC
    psc = _sc.make_scene(kind, args.seed)
    pcs = _RC(psc, dq=dq)
    pcs.init()
    pcs.set_mode(check_mode(args))
    mlp, losses, t_lab, t_train = planner.train_predictor(pcs, psc, n_labels=1 << 20, epochs=10, batch=4096,
                                                          lr=1e-3, seed=args.seed)
    out = planner.compare_planners(pcs, psc, n_samples=n_samples, n_queries=1000, k=k, seed=args.seed, mlp=mlp,
                                   repeats=3)
    out["scene"] = {"kind": kind, "ndof": psc.ndof, "polytopes": len(psc.polys), "pairs": len(psc.pair_from)}
    out["predictor"] = {"labels": 1 << 20, "epochs": 10, "batch": 4096, "lr": 1e-3,
                        "label_seconds": t_lab, "train_seconds": t_train, "final_loss": float(losses[-1])}
    # what the network itself gains: the learned planner against the same
    # lazy planner without it, with and without the cost of its labels and
    # training spread over the query batch (the planners' times are whole
    # batches of 1000 queries); the lazy scheduling's own gain over the
    # eager planner is lazy_over_plain_time
    lz, ln = out["lazy"]["batch_seconds"], out["learned"]["batch_seconds"]
    out["network_gain"] = {
        "learned_over_lazy_time": ln / lz,
        "learned_with_training_over_lazy_time": (ln + t_lab + t_train) / lz,
        "false_free_rate": out["predictor_errors"]["false_free_rate"],
        "lazy_over_plain_time": out["lazy_over_plain_time"],
        "note": "the <= 0.5x time-to-path of the learned planner against the eager one comes from the lazy "
                "scheduling (lazy_over_plain_time); the network's own gain is learned_over_lazy_time",
    }
    return out


BOX4 = dict(workload="box4 PRM: 4-DOF revolute arm of 0.3 x 0.05 x 0.05 m box links, 16 box obstacles, "
                     "8192 uniform samples, C-space L2 radius 0.5 rad, dq=0.02 rad, start and goal free samples",
            ndof=4, obstacles=16, samples=8192, radius=0.5, dq=0.02)


def _dropin_plan(exe, checker, cfg_dir, s, g, seed):
    """One run of GPUPRM's planner (process_mpi5, 32 new nodes per step,
    nbuf 2048, distD = distH = radius, at most 5000 steps) between s and g."""
    out = tempfile.mkdtemp(prefix="box4_out_")
    cmd = [exe, "--checker", checker, "--config", cfg_dir, "--out", out, "--num", "32", "--nbuf", "2048",
           "--dq", str(BOX4["dq"]), "--distD", str(BOX4["radius"]), "--distH", str(BOX4["radius"]),
           "--maxsteps", "5000", "--seed", str(seed),
           "--start", ",".join("%.9g" % x for x in s), "--goal", ",".join("%.9g" % x for x in g)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        return {"error": "exit %d: %s" % (p.returncode, p.stderr.strip()[-200:])}
    return json.loads(p.stdout.strip().splitlines()[-1])


def box4_leg(args):
    """The reference's CPU planning case.  GPUPRM's planner grows two trees
    from the start and the goal until they meet; its time per query is
    timed per start/goal pair (one core), with its own CPU checker and with
    this library's checker behind the same Configspace<4> interface.  The
    GPU PRMs build a radius-0.5 roadmap of n uniform samples and answer the
    same pairs: n starts at 8192 and doubles until every pair is answered
    (8192 samples at this radius leave the free space in thousands of
    components).  Each GPU run is timed alone for the whole batch of pairs
    and for one pair."""
    from gpuprm_b200 import planner, scenes
    from gpuprm_b200.configspace import RobotConfigspace
    sc = scenes.make_box4(args.seed)
    cs = RobotConfigspace(sc, dq=BOX4["dq"])
    cs.init()
    cs.set_mode(check_mode(args))
    Q = max(1, args.box4_queries)
    starts, goals = planner.make_queries(cs, sc, Q, args.seed + 31)
    out = {"config": dict(BOX4, queries=Q)}
    gpu, n = [], BOX4["samples"]
    while True:
        row = {"samples": n}
        for name, fn in (("plain", planner.plain_prm), ("lazy", planner.lazy_prm)):
            fn(cs, sc, starts, goals, n, seed=args.seed, radius=BOX4["radius"])
            runs = sorted((fn(cs, sc, starts, goals, n, seed=args.seed, radius=BOX4["radius"]) for _ in range(3)),
                          key=lambda r: r.seconds)
            r = runs[1]
            one = sorted(fn(cs, sc, starts[:1], goals[:1], n, seed=args.seed, radius=BOX4["radius"]).seconds
                         for _ in range(3))[1]
            row[name] = {"success_rate": float(r.success.mean()), "batch_seconds": r.seconds,
                         "seconds_one_pair": one, "paths_verified": bool(r.info["verified"]),
                         "free_vertices": r.info["free_vertices"], "candidate_edges": r.info["candidate_edges"],
                         "edge_checks": r.edge_checks, "edge_steps": r.edge_steps}
        gpu.append(row)
        if row["plain"]["success_rate"] >= 1.0 or n >= (1 << 18):
            break
        n *= 2
    out["gpu"] = gpu
    exe = os.path.join(ROOT, "oracle", "_ref", "prm_dropin")
    if args.no_cpu_baseline or not os.path.exists(exe):
        out["cpu_baseline"] = None if args.no_cpu_baseline else {"unavailable": "oracle/_ref/prm_dropin not built"}
        return out
    cfg = tempfile.mkdtemp(prefix="box4_cfg_")
    scenes.write_config_dir(sc, cfg)
    ref = {}
    for checker in ("ref", "b200"):
        runs = [_dropin_plan(exe, checker, cfg, starts[t], goals[t], args.seed + t) for t in range(Q)]
        ok = [r for r in runs if "error" not in r]
        secs = [r["plan_seconds"] for r in ok]
        ref[checker] = {"runs": len(runs), "errors": [r["error"] for r in runs if "error" in r],
                        "success_rate": sum(r["connection_found"] for r in ok) / len(runs),
                        "median_seconds": statistics.median(secs) if secs else None,
                        "mean_seconds": sum(secs) / len(secs) if secs else None,
                        "median_nodes": statistics.median(r["num_nodes"] for r in ok) if ok else None,
                        "median_edge_steps": statistics.median(r["edge_step_checks"] for r in ok) if ok else None}
    out["cpu_baseline"] = {"kind": "reference", "cores": 1, "planner": "PRMSolver<4>::process_mpi5",
                           "sample": "%d seeded free start/goal pairs, one planner run each" % Q,
                           "reference_checker": ref["ref"], "library_checker_dropin": ref["b200"]}
    best = gpu[-1]
    if ref["ref"]["median_seconds"]:
        out["gpu_over_reference_time"] = {
            k: best[k]["batch_seconds"] / Q / ref["ref"]["median_seconds"] for k in ("plain", "lazy")}
        out["gpu_one_pair_over_reference_time"] = {
            k: best[k]["seconds_one_pair"] / ref["ref"]["median_seconds"] for k in ("plain", "lazy")}
    return out


STRESS = dict(workload="wall7 edges: 7-DOF arm of 8 32-vertex hull links, 512 hull obstacles (8-64 vertices) "
                        "in 6 Gaussian clusters forming two walls with a 0.12 m gap, 2^22 samples, kNN k=16, "
                        "dq=0.005 rad, FP64 band 1e-5 m",
              ndof=7, obstacles=512, samples=1 << 22, k=16, dq=0.005, band_m=1e-5)


def stress_edges_leg(args, dev, policy):
    """Checker throughput on the 7-DOF wall scene at full size: the vertex
    check of 2^22 samples, the kNN roadmap of the free ones (k=16), then the
    edge checker on a seeded uniform sample of the roadmap's edges (the whole
    roadmap takes ~2.5e9 edge steps, about half a minute), next to the
    reference CPU checker on a bounded sample of the same edges."""
    import torch
    from gpuprm_b200 import scenes, workloads
    from gpuprm_b200.configspace import RobotConfigspace
    sc = scenes.make_scene("wall7", args.seed)
    cs = RobotConfigspace(sc, dq=STRESS["dq"])
    cs.init()
    cs.set_mode(check_mode(args))
    cs.set_edge_policy(policy)
    n = STRESS["samples"]
    q = torch.tensor(np.ascontiguousarray(scenes.uniform_configs(sc, n, args.seed + 1000).T), device=dev)
    codes = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # warm-up: small calls, then one at full size (the handle sizes its
    # buffers to the largest call so far, outside the timed region)
    for _ in range(max(3, args.warmup)):
        cs.check_configs_device(q[:, :1 << 16].contiguous(), codes[:1 << 16])
    cs.check_configs_device(q, codes)
    torch.cuda.synchronize()
    e0.record(stream)
    cs.check_configs_device(q, codes)
    e1.record(stream)
    torch.cuda.synchronize()
    t_v = e0.elapsed_time(e1) / 1e3
    free = torch.nonzero(codes == 0).squeeze(1)
    qf = q[:, free].T.contiguous()
    t0 = time.perf_counter()
    i, j = workloads.knn_pairs(qf, STRESS["k"])
    torch.cuda.synchronize()
    t_knn = time.perf_counter() - t0
    E = int(i.numel())
    tn_all = (torch.linalg.vector_norm(qf[i] - qf[j], dim=1) / STRESS["dq"]).floor() + 1
    g = torch.Generator(device="cpu").manual_seed(args.seed + 17)
    m = min(E, args.stress_edges)
    pick = torch.randperm(E, generator=g)[:m].to(dev)
    qs = qf[i[pick]].T.contiguous()
    qe = qf[j[pick]].T.contiguous()
    res = torch.empty(m, dtype=torch.int32, device=dev)
    w = min(m, 1 << 14)
    for _ in range(max(3, args.warmup)):
        cs.check_edges_device(qs[:, :w].contiguous(), qe[:, :w].contiguous(), res[:w])
    cs.check_edges_device(qs, qe, res)
    torch.cuda.synchronize()
    s0 = cs.stats()
    e0.record(stream)
    cs.check_edges_device(qs, qe, res)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e = e0.elapsed_time(e1) / 1e3
    s1 = cs.stats()
    nominal = s1["edge_steps_nominal"] - s0["edge_steps_nominal"]
    out = {
        "config": dict(STRESS, free_samples=int(free.numel()), roadmap_edges=E,
                       roadmap_edge_steps=int(tn_all.sum().item()), sampled_edges=m,
                       policy=args.policy),
        "vertex": {"configs_per_s": n / t_v, "ms": 1e3 * t_v, "pairs_per_config": len(sc.pair_from)},
        "knn_seconds": t_knn,
        "edges": {"value": nominal / t_e, "unit": UNIT, "ms": 1e3 * t_e, "edge_steps_nominal": int(nominal),
                  "edge_steps_executed": int(s1["edge_steps_executed"] - s0["edge_steps_executed"]),
                  "colliding_edges": int((res != 0).sum().item()),
                  "band_rechecks": int(s1["band_rechecks"] - s0["band_rechecks"])},
    }
    # mid-size batches of these edges (a lazy planner's first round here is
    # about 35k edges): one warp per edge against edges split into segments
    # of 2 rounds over several warps
    split = []
    for mb in (35000, 140000):
        if mb > m:
            break
        qs_b, qe_b = qs[:, :mb].contiguous(), qe[:, :mb].contiguous()
        rb = {}
        for name, smax in (("whole", 0), ("split", mb)):
            cs.set_edge_split(smax, 2)
            rr = torch.empty(mb, dtype=torch.int32, device=dev)
            for _ in range(2):
                cs.check_edges_device(qs_b, qe_b, rr)
            torch.cuda.synchronize()
            e0.record(stream)
            cs.check_edges_device(qs_b, qe_b, rr)
            e1.record(stream)
            torch.cuda.synchronize()
            rb[name] = (e0.elapsed_time(e1), rr.clone())
        split.append({"edges": mb, "whole_ms": rb["whole"][0], "split_ms": rb["split"][0],
                      "split_over_whole_time": rb["split"][0] / rb["whole"][0],
                      "codes_identical": bool(torch.equal(rb["whole"][1], rb["split"][1]))})
    cs.set_edge_split(16384, 2)
    out["split_batches"] = split
    if not args.no_cpu_baseline:
        qs_r = np.ascontiguousarray(qs.T.cpu().numpy())
        qe_r = np.ascontiguousarray(qe.T.cpu().numpy())
        cpu, _, sample = cpu_reference_rate(sc, qs_r, qe_r, STRESS["dq"], args.cpu_seconds, args.seed,
                                            count_ops=False)
        out["cpu_baseline"] = cpu
        out["parity"] = edge_parity(sc, qs_r, qe_r, STRESS["dq"], STRESS["band_m"], sample, res.cpu().numpy(),
                                    "7-DOF wall edges (512 obstacles, FP64 band mode) vs the reference CPU checker")
    return out


# the network's own work for 6 joints: 12 inputs (sin, cos), three 256x256
# layers and the output; the first layer's operand is padded to 16 inputs
# for the MMA K step, and the padding is not counted
MLP_FLOPS_PER_ROW = 2 * (12 * 256 + 3 * 256 * 256 + 256)


def mlp_leg(args, dev):
    """Inference of the collision predictor (6 joints, 16 -> 256 x4 -> 1,
    BF16 operands, FP32 accumulation) on 2^22 uniform configurations: the
    fused tcgen05 kernel (the library default), one tcgen05 kernel per
    layer, and the training GEMMs.  FLOPs per row = 2 (12*256 + 3*256^2 +
    256) (the 12 real inputs); roofline against the measured dense BF16
    peak (burst figure: one kernel timed alone)."""
    import torch
    from gpuprm_b200.mlp import CollisionMLP
    n = args.mlp_rows
    rng = np.random.default_rng(args.seed + 11)
    q = torch.tensor(rng.uniform(-np.pi, np.pi, (6, n)).astype(np.float32), device=dev)
    mlp = CollisionMLP(6, seed=args.seed + 1)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    res = {"rows": n, "flops_per_row": MLP_FLOPS_PER_ROW}
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except Exception:
        peak = 1590.0
    for path in ("tcgen05", "tcgen05_layers", "training"):
        mlp.set_inference(path)
        for _ in range(max(3, args.warmup)):
            mlp.predict(q, out=out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            mlp.predict(q, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        tf = n * MLP_FLOPS_PER_ROW / (ms * 1e-3) / 1e12
        res[path] = {"ms": ms, "tflops": tf, "rows_per_s": n / (ms * 1e-3), "frac_of_bf16_peak": tf / peak}
    # training: 2^20 labelled rows, batch 4096, the configuration's 10
    # epochs (each call captures one epoch's 256 steps - features, forward,
    # loss, backward, Adam - into a CUDA graph and replays it per epoch).
    # ms_per_step is the replay cost: (time of 11 epochs - time of 1) / 10
    # epochs; seconds_10_epochs includes the call's capture.
    nt, bt, ep = 1 << 20, 4096, 10
    qt = torch.tensor(rng.uniform(-np.pi, np.pi, (6, nt)).astype(np.float32), device=dev)
    yt = torch.tensor((rng.random(nt) < 0.4).astype(np.float32), device=dev)
    train = {"rows": nt, "batch": bt, "epochs": ep, "flops_per_step": 3 * bt * MLP_FLOPS_PER_ROW}
    steps_ep = nt // bt

    def timed_train(m, epochs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.train(qt, yt, epochs=epochs, batch=bt)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    for path in ("tcgen05", "mma_sync"):
        m2 = CollisionMLP(6, seed=args.seed + 2)
        m2.set_training(path)
        timed_train(m2, 1)   # warm-up
        t1 = timed_train(m2, 1)
        t10 = timed_train(m2, ep)
        t11 = timed_train(m2, ep + 1)
        per = (t11 - t1) / (ep * steps_ep)
        train[path] = {"seconds_10_epochs": t10, "ms_per_step": 1e3 * per,
                       "tflops": train["flops_per_step"] / per / 1e12, "device_status": m2.device_status()}
    res["train"] = train
    res["device_status"] = mlp.device_status()
    res["peak_tflops"] = peak
    res["peak_source"] = "MEASURED_PEAKS.json bf16_tflops (burst)"
    return res


def sampler_leg(args, ws, dev):
    """Near-node sampling with the reference's acceptance rule
    (get_random_nodes2, prmsolver.cpp:2635-2698: power 2): 2^16 accepted,
    free samples near the workload's free vertices (surrnum = their kNN
    degree, D = 0.5) in batches of 2^20 candidates, against the CPU
    restatement (one core) on a bounded number of samples."""
    import torch
    from gpuprm_b200 import workloads
    from gpuprm_b200.sampler import sample_near
    cs = ws["space"]
    nodes = ws["q_soa"][:, ws["codes"] == 0].contiguous()
    i, j = workloads.knn_pairs(nodes.T.contiguous(), 10)
    surr = torch.bincount(torch.cat([i, j]), minlength=nodes.shape[1]).to(torch.int32)
    num, power, batch = 1 << 16, 2, 1 << 20
    sample_near(cs, nodes, surr, 1024, 0.5, seed=1, power=power, batch=batch)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q, par, used = sample_near(cs, nodes, surr, num, 0.5, seed=args.seed + 3, power=power, batch=batch)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    got = int(q.shape[1])
    out = {"samples": got, "requested": num, "power": power, "candidates": int(used), "seconds": dt,
           "samples_per_s": got / dt, "candidates_per_s": used / dt,
           "accepted_free_per_candidate": got / max(1, used), "nodes": int(nodes.shape[1])}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        import sampler_oracle as SO
        orc = O.Oracle(ws["scene"])
        free = lambda qq: orc.check_configs(qq, O.FP32_BAND | O.DEVICE_TRIG)[0] == 0
        nodes_np, surr_np = nodes.T.cpu().numpy(), surr.cpu().numpy()
        m = 1024
        t0 = time.perf_counter()
        SO.sample_near(nodes_np, surr_np, power, 0.5, args.seed + 3, m, free, batch=1 << 16)
        cdt = time.perf_counter() - t0
        out["cpu_port"] = {"samples": m, "seconds": cdt, "samples_per_s": m / cdt, "cores": 1,
                           "kind": "port (numpy restatement + oracle vertex check)"}
    return out


def batch_leg(args, dev, policy):
    """Many independent problems: one graph-captured batched launch per kind
    against a loop of per-problem launches (same stream, same inputs);
    results must agree bit for bit.  The launch shape (threads per block x
    resident blocks per SM) is autotuned on every 8th problem (the same mix
    of DOF and scene sizes at 1/8 of the work) and applied to the whole
    batch.  One untimed and two timed passes per arm (a full edge pass is
    several seconds of work)."""
    import torch
    from gpuprm_b200 import workloads
    from gpuprm_b200.batch import CONFIGS, EDGES, ProblemBatch
    t_build = time.perf_counter()
    ws = workloads.batch_workload(seed=args.seed, problems=args.batch_problems, device=str(dev))
    t_build = time.perf_counter() - t_build
    spaces = ws["spaces"]
    for cs in spaces:
        cs.set_edge_policy(policy)
        cs.set_mode(check_mode(args))
    B = ProblemBatch(spaces)
    Q, A, Bq = ws["q"], ws["qs"], ws["qe"]
    nv, ne = Q.shape[1], A.shape[1]
    rv = torch.zeros(nv, dtype=torch.int32, device=dev)
    re = torch.zeros(ne, dtype=torch.int32, device=dev)
    B.set_layout(CONFIGS, ws["offs_v"])
    B.set_layout(EDGES, ws["offs_e"])
    ov, oe = ws["offs_v"], ws["offs_e"]
    # the tuning sub-batch: every 8th problem, packed contiguously
    sub = list(range(0, len(spaces), 8))
    T = ProblemBatch([spaces[p] for p in sub])
    tq = torch.cat([Q[:, ov[p]:ov[p + 1]] for p in sub], 1).contiguous()
    ta = torch.cat([A[:, oe[p]:oe[p + 1]] for p in sub], 1).contiguous()
    tb = torch.cat([Bq[:, oe[p]:oe[p + 1]] for p in sub], 1).contiguous()
    T.set_layout(CONFIGS, np.concatenate([[0], np.cumsum([ov[p + 1] - ov[p] for p in sub])]))
    T.set_layout(EDGES, np.concatenate([[0], np.cumsum([oe[p + 1] - oe[p] for p in sub])]))
    t_tune = time.perf_counter()
    tune_v = T.autotune(CONFIGS, tq, None, torch.zeros(tq.shape[1], dtype=torch.int32, device=dev), reps=2)
    tune_e = T.autotune(EDGES, ta, tb, torch.zeros(ta.shape[1], dtype=torch.int32, device=dev), reps=2)
    t_tune = time.perf_counter() - t_tune
    table = {"configs": T.tune_table(CONFIGS), "edges": T.tune_table(EDGES)}
    del T, tq, ta, tb
    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / steps

    # the shape a new batch starts with, on the full set, before tuning
    default = {"configs": B.get_launch(CONFIGS), "edges": B.get_launch(EDGES)}
    t_dv = timed(lambda: B.check_configs_device(Q, rv), 1)
    t_de = timed(lambda: B.check_edges_device(A, Bq, re), 1)
    B.set_launch(CONFIGS, tune_v["threads"], tune_v["blocks_per_sm"])
    B.set_launch(EDGES, tune_e["threads"], tune_e["blocks_per_sm"])
    B.set_solo_threshold(CONFIGS, tune_v["solo"]["min_items"])
    B.set_solo_threshold(EDGES, tune_e["solo"]["min_items"])
    B.capture(CONFIGS, Q, None, rv)
    B.capture(EDGES, A, Bq, re)
    # rounds of 32 steps per edge (an edge split over warps pays only from
    # a few rounds on)
    tn = torch.floor(torch.linalg.vector_norm(Bq - A, dim=0) / workloads.MANY["dq"]) + 1
    rounds = torch.ceil(tn / 32)
    # per-problem views of the same inputs for the launch loop
    ov, oe = ws["offs_v"], ws["offs_e"]
    dofs = [sc.ndof for sc in ws["scenes"]]
    pv = [Q[:d, ov[p]:ov[p + 1]] for p, d in enumerate(dofs)]
    pa = [A[:d, oe[p]:oe[p + 1]] for p, d in enumerate(dofs)]
    pb = [Bq[:d, oe[p]:oe[p + 1]] for p, d in enumerate(dofs)]
    lv = [torch.zeros(x.shape[1], dtype=torch.int32, device=dev) for x in pv]
    le = [torch.zeros(x.shape[1], dtype=torch.int32, device=dev) for x in pa]

    def loop(kind):
        for p, cs in enumerate(spaces):
            if kind == CONFIGS and lv[p].numel():
                cs.check_configs_device(pv[p], lv[p])
            elif kind == EDGES and le[p].numel():
                cs.check_edges_device(pa[p], pb[p], le[p])

    steps = 2
    s0 = B.stats()
    t_bv = timed(lambda: B.replay(CONFIGS), steps)
    s1 = B.stats()
    t_be = timed(lambda: B.replay(EDGES), steps)
    s2 = B.stats()
    t_lv = timed(lambda: loop(CONFIGS), steps)
    t_le = timed(lambda: loop(EDGES), steps)
    reps = 1 + steps
    nominal = (s2["edge_steps_nominal"] - s1["edge_steps_nominal"]) // reps
    got_v, got_e = rv.cpu().numpy(), re.cpu().numpy()
    same_v = all(np.array_equal(got_v[ov[p]:ov[p + 1]], lv[p].cpu().numpy()) for p in range(len(spaces)))
    same_e = all(np.array_equal(got_e[oe[p]:oe[p + 1]], le[p].cpu().numpy()) for p in range(len(spaces)))
    return {
        "workload": "many problems: %d mixed scenes (DOF 4-7, 8-128 hull obstacles), 2^14-2^18 samples each, "
                    "kNN k=%d of every free sample, edges cut to a radius U[0.4,0.8], dq=%g"
                    % (len(spaces), workloads.MANY["k"], workloads.MANY["dq"]),
        "problems": len(spaces), "dof_counts": {str(d): dofs.count(d) for d in sorted(set(dofs))},
        "configs": int(nv), "edges": int(ne), "edge_steps_nominal": int(nominal),
        "batched": {"configs_per_s": nv / t_bv, "edge_steps_per_s": nominal / t_be,
                    "configs_ms": 1e3 * t_bv, "edges_ms": 1e3 * t_be, "graph_launches_per_step": 2,
                    "launch_shape": {"configs": B.get_launch(CONFIGS), "edges": B.get_launch(EDGES)},
                    "solo": {"configs": B.get_solo_threshold(CONFIGS), "edges": B.get_solo_threshold(EDGES),
                             "meaning": "problems with at least min_items items run in launches of their own "
                                        "inside the captured graph; the rest share one persistent launch"},
                    "autotune": {"sub_batch": "every 8th problem (%d)" % len(sub), "seconds": t_tune,
                                 "candidates": "threads 64/128/256/512 x resident blocks per SM all/3/4/half, "
                                               "then solo threshold none/2^18/2^16/2^14/all items",
                                 "sweep_ms_on_sub_batch": table,
                                 "not_swept": "edge split over warps: the edges are %.2f rounds of 32 steps on "
                                              "average (max %d), below the 2 rounds a segment needs; scene tables "
                                              "in shared memory: the warps of a block check different problems, "
                                              "so the tables go through L1, whose share the blocks-per-SM cap sets"
                                              % (float(rounds.mean()), int(rounds.max()))},
                    "default_shape": default,
                    "default_configs_ms": 1e3 * t_dv, "default_edges_ms": 1e3 * t_de,
                    "tuned_over_default_time": {"configs": t_bv / t_dv, "edges": t_be / t_de},
                    "timed_passes": steps},
        "per_problem_loop": {"configs_per_s": nv / t_lv, "edge_steps_per_s": nominal / t_le,
                             "configs_ms": 1e3 * t_lv, "edges_ms": 1e3 * t_le},
        "speedup": {"configs": t_lv / t_bv, "edges": t_le / t_be},
        "results_identical": bool(same_v and same_e),
        "vertex_checks_per_step": int((s1["vertex_checks"] - s0["vertex_checks"]) // reps),
        "setup_seconds": t_build,
    }


# --------------------------------------------------------------------------
# reference arm: GPUPRM's CPU checker on the same workload definition
# --------------------------------------------------------------------------

def run_reference(args):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from scipy.spatial import cKDTree
    from gpuprm_b200 import scenes
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libgprm_ref.so was not built (reference tree absent at build time)"}
    sc = scenes.make_scene("hull6", args.seed)
    dq = WORKLOAD["dq"]
    cores = os.cpu_count() or 1
    ref = O.RefChecker(sc, dq=dq, nbuf=4096)
    q = scenes.uniform_configs(sc, args.samples, args.seed + 1000)
    codes = ref.check_configs_mt(q, cores, chunk=512)
    free = q[codes == 0]
    tree = cKDTree(free.astype(np.float64))
    rng = np.random.default_rng(args.seed + 5)

    def sample_edges(m):
        src = rng.choice(free.shape[0], m, replace=False)
        _, nb = tree.query(free[src].astype(np.float64), k=args.k + 1)
        j = nb[np.arange(m), rng.integers(1, args.k + 1, m)]
        return free[src], free[j]

    # size one step to ~cpu_seconds of work
    a, b = sample_edges(64 * cores)
    t0 = time.perf_counter()
    ref.check_edges_mt(a, b, cores, chunk=16)
    per_edge = (time.perf_counter() - t0) / a.shape[0]
    m = int(max(64, min(200000, args.cpu_seconds / max(per_edge, 1e-9))))
    for _ in range(max(3, args.warmup)):
        a, b = sample_edges(min(m, 256 * cores))
        ref.check_edges_mt(a, b, cores, chunk=16)
    steps = 0
    t = 0.0
    for _ in range(args.steps):
        a, b = sample_edges(m)
        steps += int(O.Oracle(sc).testnum(a, b, dq).sum())
        t0 = time.perf_counter()
        ref.check_edges_mt(a, b, cores, chunk=16)
        t += time.perf_counter() - t0
    v = steps / t
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": dict(WORKLOAD), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{m} kNN edges per step drawn from the workload's free samples"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if args.only_mlp:
        import torch
        torch.cuda.set_device(local_rank)
        if rank == 0:
            print(json.dumps({"mlp": mlp_leg(args, torch.device("cuda", local_rank))}), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
        bad = [p["what"] for p in (line.get("parity"), (line.get("stress_edges") or {}).get("parity"))
               if p is not None and not p["ok"]]
        if bad:
            sys.stderr.write("verdict parity with the reference failed: %s\n" % "; ".join(bad))
            sys.exit(3)


if __name__ == "__main__":
    main()
