#!/usr/bin/env python
"""Throughput of the direct-summation hot path on B200.

Workload (one "step"): the precision form -- an N = 2^20 Plummer sphere with
Salpeter masses (0.1-100, slope -2.35, M = 1) and 10 % of the particles in
circular binaries (a ~ logU(1e-6, 1e-4)), Hermite 6th order; every step
predicts all j to t_i and evaluates acc/jerk/snap/pot and the nearest
neighbour on all N i-particles (N^2 interactions).  Inputs are synthetic and
seeded; the j derivatives come from an FP64 direct summation (the library's
all-FP64 kernels).

  value   interactions/s of the mixed-precision kernels with all inputs
          resident in HBM (predictor + force, CUDA events on the launching
          stream, L2 flushed between steps);
  e2e     the same metric through the public `sapporo` class with host
          buffers: j upload, i upload in n_pipes chunks, result download.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
    torchrun --nproc-per-node N bench.py --gpus N ...   (independent replicas)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOPS_4TH, FLOPS_6TH = 38, 60
METRIC = "interactions/s at N=2^20 mixed vs plain FP64, 1 GPU, acc err<=1e-6; %FP32 peak"


# DRAM bytes (read + written) of one mixed 6th-order force launch at N = 2^20,
# all i, from `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum` (one
# pass) of `bench.py --steps 1 --warmup 0 --only mixed` (spatial mode, and
# with --spatial 0), and the hash of the kernel sources that capture ran
# (kernel_source_sha).  When the sources change the figure is stale and the
# bench reports no traffic until it is captured again.
FORCE_DRAM = {"source_sha": "8d4037f0416779eb",
              "spatial": 1098467840.0 + 109549312.0, "address": 1002800384.0 + 120619520.0}
KERNEL_SOURCES = ["sapb_kernels.cu", "sapb_kernels.cuh", "sapb_pair.cuh", "sapb_internal.cuh",
                  "sapb_spatial.cu", "sapb_capi.cu"]


def kernel_source_sha() -> str:
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        h.update((ROOT / "sapporo2_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
def build_inputs(n: int, seed: int):
    from sapporo2_b200 import ic
    from sapporo2_b200.direct import fp64_direct
    cfg = ic.make_config("C3", n=n, seed=seed)
    t0 = time.time()
    acc, jrk, _ = fp64_direct(1, cfg["x"], cfg["v"], None, cfg["m"], cfg["id"], cfg["eps2"])
    _, _, snp = fp64_direct(2, cfg["x"], cfg["v"], acc, cfg["m"], cfg["id"], cfg["eps2"])
    cfg["a"], cfg["j"], cfg["s"] = acc, jrk, snp
    cfg["c"] = ic.crackle_from(cfg["x"], acc, jrk)
    cfg["px"], cfg["pv"], cfg["pa"] = ic.predict_fp64(2, cfg["ti"], cfg["t0"], cfg["x"], cfg["v"],
                                                      acc, jrk, snp, cfg["c"])
    log(f"[bench] inputs N={n} built in {time.time() - t0:.1f}s")
    return cfg


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "power_w_max": float(max(power)), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


# ---------------------------------------------------------------------------
LAUNCH = None  # (tpi, ip, slices) override for the force kernel, from --launch
LAUNCH_PREC = None  # the precision the override applies to (mixed unless --only fp64)


def device_arm(cfg, precision: int, steps: int, warmup: int, torch, flush, lists=False,
               shard=None, spatial_mode_set=None):
    """Predictor + force on all N with device-resident inputs.  Returns
    per-step predictor / force (+ combine) times (ms) and the results.

    shard = (rank, world): this rank holds the j with address % world ==
    rank (the reference's round-robin split over devices) and computes
    their partial forces on every i; the partials are combined by NCCL
    all-reduces (sum of forces, min of nearest-neighbour keys) on the same
    stream, inside the timed step.  spatial_mode_set: spatial mode of the
    handle (None: the library's default)."""
    import sapporo2_b200 as sp
    from sapporo2_b200.sharded import combine_partials
    n = cfg["n"]
    rank, world = shard if shard else (0, 1)
    jsel = np.arange(rank, n, world)
    nj = len(jsel)
    s = sp.Sapporo(order=sp.SIXTH, precision=precision)
    # a dedicated stream: the library and the timing events must share it
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    if spatial_mode_set is not None:
        s.set_spatial(spatial_mode_set, 0.0)
    if LAUNCH and precision == (LAUNCH_PREC if LAUNCH_PREC is not None else sp.DOUBLESINGLE):
        s.set_launch(*LAUNCH)
    s.set_j_particles(np.arange(nj), cfg["id"][jsel], cfg["t0"][jsel], cfg["m"][jsel],
                      cfg["x"][jsel], cfg["v"][jsel], cfg["a"][jsel], cfg["j"][jsel],
                      cfg["s"][jsel], cfg["c"][jsel])
    s.force_prediction(nj)  # uploads and scatters j (no prediction: no set_time yet)
    rec = sp.pack_i_records(2, cfg["px"], cfg["pv"], cfg["h2"], cfg["id"], cfg["pa"])
    i_dev = torch.from_numpy(rec).cuda()
    res = torch.zeros((n, sp.RES_STRIDE), dtype=torch.float64, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda") if lists else None
    lst = torch.zeros(n * sp.NGB_PB, dtype=torch.int32, device="cuda") if lists else None
    flags = sp.F_NGB_LIST if lists else 0
    lib, dev = s.lib, s.dev
    tpi, ip, ns = s.plan(n, nj)
    pred_ms, force_ms, comb_ms = [], [], []
    torch.cuda.synchronize()
    for it in range(warmup + steps):
        with torch.cuda.stream(stream):  # ordered before the timed step
            flush()
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        rc = lib.sapb_predict(dev, nj, float(cfg["ti"]))
        e1.record(stream)
        rc |= lib.sapb_force_device(dev, nj, n, i_dev.data_ptr(), float(cfg["eps2"]), flags,
                                    res.data_ptr(), cnt.data_ptr() if lists else None,
                                    lst.data_ptr() if lists else None)
        e2.record(stream)
        if rc:
            raise RuntimeError(f"device step failed: {lib.sapb_last_error(dev).decode()}")
        if world > 1:
            with torch.cuda.stream(stream):
                combine_partials(res)
        e3.record(stream)
        e3.synchronize()
        if it >= warmup:
            pred_ms.append(e0.elapsed_time(e1))
            force_ms.append(e1.elapsed_time(e2))
            comb_ms.append(e2.elapsed_time(e3))
    stream.synchronize()
    out = res.cpu().numpy()
    far_tiles, warp_tiles = s.spatial_stats(reset=True)
    s.close()
    spatial = precision == sp.DOUBLESINGLE and warp_tiles > 0
    # own kernels in the timed steps: predictor, force (+ slice reduction);
    # in spatial mode the j gather, i keys and bounds every step, plus frame
    # init, frame and j keys on the steps that re-sort j (the first call and
    # every 17th after it: the library reuses an order 16 times); the radix
    # sorts are CUB's kernels, not counted
    per = 2 + (1 if ns > 1 else 0) + (3 if spatial else 0)
    timed = range(warmup, warmup + steps)
    launches = per * steps + (3 * sum(1 for c in timed if c % 17 == 0) if spatial else 0)
    return {"pred_ms": pred_ms, "force_ms": force_ms, "comb_ms": comb_ms, "res": out,
            "plan": {"tpi": tpi, "ip": ip, "nslices": ns}, "nj_local": nj,
            "spatial": spatial,
            "far_fraction": far_tiles / warp_tiles if warp_tiles else None,
            "launches": launches}


def e2e_arm(cfg, steps: int, shard=None):
    """The public class API with host buffers, n_pipes chunks (with shard,
    the class on each rank behind ShardedSapporo: the rank's j share, NCCL
    combine of the partial results)."""
    import sapporo2_b200 as sp
    n = cfg["n"]
    s = sp.Sapporo(order=sp.SIXTH, precision=sp.DOUBLESINGLE)
    npipes = s.get_n_pipes()
    api = s
    if shard:
        from sapporo2_b200.sharded import ShardedSapporo
        api = ShardedSapporo(s, device="cuda")
    times = []
    for it in range(steps + 1):  # first pass warms the pinned buffers
        t0 = time.perf_counter()
        api.set_j_particles(np.arange(n), cfg["id"], cfg["t0"], cfg["m"], cfg["x"], cfg["v"],
                            cfg["a"], cfg["j"], cfg["s"], cfg["c"])
        api.set_time(cfg["ti"])
        for i0 in range(0, n, npipes):
            sl = slice(i0, min(n, i0 + npipes))
            api.start(n, cfg["id"][sl], cfg["px"][sl], cfg["pv"][sl], cfg["pa"][sl],
                      cfg["eps2"], cfg["h2"][sl])
            r = api.results(n, ngb=True)
        t1 = time.perf_counter()
        if it > 0:
            times.append(t1 - t0)
        del r
    s.close()
    world = shard[1] if shard else 1
    h2d = (n // world) * 22 * 8 + n * 12 * 8
    d2h = n * 12 * 8
    return {"s_per_step": float(np.mean(times)), "h2d": h2d, "d2h": d2h, "chunks": -(-n // npipes)}


def cpu_baseline_leg(cfg, nsample: int):
    """FP64 OpenMP direct summation (the project's CPU restatement of the
    reference's Hermite expressions) on a seeded sample of i against all N j,
    timed on all host threads.  Also returns the oracle answers for the
    sample, used as the FP64 truth of the accuracy figures."""
    from oracle import oracle as O
    rng = np.random.default_rng(1234)
    sel = np.sort(rng.choice(cfg["n"], nsample, replace=False)).astype(np.int32)
    # the oracle predicts the j itself (FP64), exactly as the device does
    px, pv, pa = O.predict(2, cfg["ti"], cfg["t0"], cfg["x"], cfg["v"], cfg["a"], cfg["j"],
                           cfg["s"], cfg["c"])
    threads = O.max_threads()
    t0 = time.perf_counter()
    r = O.force_subset(2, sel, cfg["px"], cfg["pv"], cfg["pa"], cfg["h2"], cfg["id"], px, pv, pa,
                       cfg["m"], cfg["id"], cfg["eps2"], nthreads=threads)
    dt = time.perf_counter() - t0
    inter = float(nsample) * cfg["n"]
    return {"value": inter / dt, "cores": threads, "seconds": dt, "sel": sel, "oracle": r,
            "interactions": inter}


def ensemble_inputs(k: int, seed: int):
    """512-cluster ensemble: N_c ~ logU[256, 16384], own t_i, active fraction
    ~ logU[1/N_c, 1], 4th order.  j acc/jerk from an FP64 direct sum done by
    one batched FP64 run over all clusters."""
    import sapporo2_b200 as sp
    from sapporo2_b200 import ic
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(256), np.log(16384), k)).astype(int)
    cl = []
    for c, n in enumerate(ns):
        x, v, m = ic.plummer(int(n), seed * 1000 + c)
        ti = 1.0 + 0.01 * c
        t0 = ti - rng.integers(0, 8, n) * 2.0 ** -10
        frac = np.exp(rng.uniform(np.log(1.0 / n), 0.0))
        active = np.sort(rng.choice(n, max(1, int(round(frac * n))), replace=False))
        cl.append({"n": int(n), "x": x, "v": v, "m": m, "ti": ti, "t0": t0, "active": active,
                   "id": np.arange(n, dtype=np.int32), "eps2": 1e-6})
    total = int(ns.sum())
    first = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int32)
    # derivatives: every particle of every cluster active, no prediction, FP64
    z = np.zeros((total, 3))
    X = np.concatenate([c["x"] for c in cl])
    V = np.concatenate([c["v"] for c in cl])
    M = np.concatenate([c["m"] for c in cl])
    ID = np.concatenate([c["id"] for c in cl])
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLE) as s:
        s.set_j_particles(np.arange(total), ID, np.zeros(total), M, X, V, z, z)
        s.force_prediction(total)
        with sp.Batch(s, k, total) as b:
            b.plan(first, ns, ns, np.zeros(k), np.full(k, 1e-6))
            b.i_stage[:total] = sp.pack_i_records(1, X, V, None, ID)
            b.run(0)
            r = b.results()
    A, J = r[:, 0:3], r[:, 4:7]
    for c, f in zip(cl, first):
        c["a"], c["j"] = A[f:f + c["n"]], J[f:f + c["n"]]
        c["px"], c["pv"], _ = ic.predict_fp64(1, c["ti"], c["t0"], c["x"], c["v"], c["a"], c["j"])
    return cl, first, ns


def ensemble_leg(torch, steps: int, warmup: int, tune_reps: int = 3) -> dict:
    """C4: 512 Plummer clusters in one persistent launch per step (batch API,
    graph replay), after the autotuner.  Device time per step: CUDA events
    around sapb_batch_run (blob upload + graph replay) on the library's
    stream; end to end: host wall time of run + results."""
    import sapporo2_b200 as sp
    t_build = time.time()
    cl, first, ns = ensemble_inputs(512, seed=4)
    build_s = time.time() - t_build
    log(f"[bench] ensemble of {len(cl)} clusters, {int(ns.sum())} particles built in {build_s:.1f}s")
    total = int(ns.sum())
    act = np.array([len(c["active"]) for c in cl])
    inter = float(np.sum(act * ns))
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLESINGLE) as s:
        stream = torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        X = np.concatenate([c["x"] for c in cl])
        s.set_j_particles(np.arange(total), np.concatenate([c["id"] for c in cl]),
                          np.concatenate([c["t0"] for c in cl]), np.concatenate([c["m"] for c in cl]),
                          X, np.concatenate([c["v"] for c in cl]),
                          np.concatenate([c["a"] for c in cl]), np.concatenate([c["j"] for c in cl]))
        s.force_prediction(total)
        with sp.Batch(s, len(cl), int(act.sum())) as b:
            b.plan(first, ns, act, [c["ti"] for c in cl], [c["eps2"] for c in cl])
            row = 0
            for c in cl:
                a = c["active"]
                b.i_stage[row:row + len(a)] = sp.pack_i_records(1, c["px"][a], c["pv"][a], None,
                                                                c["id"][a])
                row += len(a)
            tune = b.autotune(sp.F_PREDICT, reps=tune_reps)
            info = b.info()
            wall, dev = [], []
            for it in range(warmup + steps):
                e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
                t0 = time.perf_counter()
                e0.record(stream)
                b.run(sp.F_PREDICT)
                e1.record(stream)
                b.results()
                t1 = time.perf_counter()
                if it >= warmup:
                    wall.append(t1 - t0)
                    dev.append(e0.elapsed_time(e1))
        s.set_stream(None)
    dev_ms = float(np.mean(dev))
    per = float(np.mean(wall))
    return {"value": inter / (dev_ms * 1e-3), "ms_per_step": dev_ms, "steps": steps,
            "warmup": warmup, "clusters": len(cl), "particles": total,
            "active_i": int(act.sum()), "interactions_per_step": inter, "autotune": tune,
            "work_items": info["items"], "persistent_blocks": info["force_blocks"],
            "e2e": {"value": inter / per, "s_per_step": per,
                    "h2d_bytes_per_step": int(act.sum()) * 64,
                    "d2h_bytes_per_step": int(act.sum()) * 96},
            "inputs_built_s": build_s, "gpu_launches": 3 * steps}


def run_ensemble_bench(args, torch):
    r = ensemble_leg(torch, args.steps, args.warmup)
    print(json.dumps({
        "metric": "interactions/s, ensemble of 512 Plummer clusters (N~logU[256,16384], own t_i, "
                  "active~logU[1/N,1]), Hermite 4th order mixed, one persistent launch per step",
        "value": r["value"], "unit": "interactions/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 body",
        "data": "synthetic",
        "config": {"workload": "ensemble (C4)", "clusters": r["clusters"],
                   "particles": r["particles"], "active_i": r["active_i"],
                   "interactions_per_step": r["interactions_per_step"],
                   "autotune": r["autotune"], "work_items": r["work_items"],
                   "persistent_blocks": r["persistent_blocks"],
                   "device_time": "CUDA events around sapb_batch_run (blob upload + graph replay)"},
        "e2e": {"value": r["e2e"]["value"], "unit": "interactions/s",
                "s_per_step": r["e2e"]["s_per_step"],
                "h2d_bytes_per_step": r["e2e"]["h2d_bytes_per_step"],
                "d2h_bytes_per_step": r["e2e"]["d2h_bytes_per_step"],
                "api": "sapb_batch_run + sapb_batch_results (tables, i records, graph, results)"},
        "gpu_launches": r["gpu_launches"],
    }), flush=True)


def learned_h2_leg(n: int, steps: int):
    """C5: N Plummer + 10 % binaries, 6th-order block steps, neighbour lists
    on (target 32, cap 256), the same steps run with the fixed global
    radius, the count-scaled radius and the learned radius.  Returns the
    per-policy statistics and the final states."""
    from sapporo2_b200 import hermite6 as H, ic
    cfg = ic.make_config("C5", n=n, seed=5)
    policies = {"fixed": lambda: H.FixedH2(), "count_scaled": lambda: H.CountScaledH2(),
                "learned": lambda: (lambda sap: H.LearnedH2(sap, seed=5))}
    out, final = {}, {}
    for name, make in policies.items():
        t0 = time.perf_counter()
        sim = H.BlockHermite6(cfg["x"], cfg["v"], cfg["m"], cfg["eps2"], make())
        t_init = time.perf_counter() - t0
        active = []
        for _ in range(steps):
            active.append(sim.step())
        de = abs(sim.energy() - sim.e0) / abs(sim.e0)
        st = dict(sim.stats)
        ev = max(st["evaluated"], 1)
        out[name] = {
            "overflow_rate": st["overflow"] / ev, "overflows": st["overflow"],
            "retries": st["retries"], "retry_rounds": st["rounds"],
            "in_range_frac": st["in_range"] / ev, "evaluations": st["evaluated"],
            "in_25pct_frac": st["in_tight"] / ev, "mean_abs_log_count_err": st["abs_log_err"] / ev,
            "ms_per_step": 1e3 * st["step_s"] / max(st["steps"], 1),
            "force_ms_per_step": 1e3 * st["force_s"] / max(st["steps"], 1),
            "train_ms_per_step": 1e3 * getattr(sim.policy, "train_s", 0.0) / max(st["steps"], 1),
            "propose_ms_per_step": 1e3 * getattr(sim.policy, "propose_s", 0.0) / max(st["steps"], 1),
            "pretrain_s": getattr(sim.policy, "pretrain_s", 0.0),
            "init_s": t_init, "t_end": float(sim.t.max()), "rel_energy_error": de,
            "mean_active": float(np.mean(active)),
            "interactions_per_step": st["interactions"] / max(st["steps"], 1),
        }
        final[name] = (sim.x.copy(), sim.v.copy())
        log(f"[bench] learned_h2 {name}: {out[name]}")
        sim.close()
    same = all(np.array_equal(final[k][0], final["fixed"][0]) and
               np.array_equal(final[k][1], final["fixed"][1]) for k in final)
    return cfg, out, same


def run_learned_h2_bench(args):
    """The learned-h2 workload (learned_h2_leg at N = 262144, 200 block
    steps) plus how far the same steps get with other force arithmetic.
    Forces do not depend on the radius (in spatial mode too: its far test
    ignores h2), so the policies' trajectories are identical; the policies
    differ in overflows, retries and time."""
    from sapporo2_b200 import hermite6 as H
    cfg, out, same = learned_h2_leg(args.c5_n, args.c5_steps)
    fr, lr_ = out["fixed"]["retries"], out["learned"]["retries"]
    # how far the same block steps get with other force arithmetic (the
    # count-scaled radius; forces do not depend on it): tight binaries make
    # the time steps sensitive to rounding in the pair sums
    import sapporo2_b200 as sp
    variants = {"mixed_address_order": ({"SAPPORO_B200_SPATIAL": "0"}, sp.DOUBLESINGLE),
                "mixed_address_order_near_off": ({"SAPPORO_B200_SPATIAL": "0",
                                                  "SAPPORO_B200_NEAR": "0"}, sp.DOUBLESINGLE),
                "mixed_spatial_near_off": ({"SAPPORO_B200_NEAR": "0"}, sp.DOUBLESINGLE),
                "fp64": ({}, sp.DOUBLE)}
    t_end = {"mixed_default": out["count_scaled"]["t_end"]}
    for name, (env, prec) in variants.items():
        old_env = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            sim = H.BlockHermite6(cfg["x"], cfg["v"], cfg["m"], cfg["eps2"], H.CountScaledH2(),
                                  precision=prec)
            for _ in range(args.c5_steps):
                sim.step()
            t_end[name] = float(sim.t.max())
            sim.close()
        finally:
            for k, v in old_env.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        log(f"[bench] learned_h2 t_end {name}: {t_end[name]}")
    print(json.dumps({
        "metric": "neighbour-overflow retries over the block steps, fixed global h2 / learned h2 "
                  "(N=262144 Plummer + 10% binaries, 6th order, target 32, cap 256)",
        "value": fr / max(lr_, 1), "unit": "x fewer retries", "n_gpus": 1,
        "steps": args.c5_steps, "warmup": 0, "ms_per_step": out["learned"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 body, f64 corrector", "data": "synthetic",
        "config": {"workload": "learned h2 (C5)", "n": args.c5_n, "block_steps": args.c5_steps,
                   "identical_trajectories": bool(same), "policies": out,
                   "t_end_after_block_steps": t_end},
    }), flush=True)


def run_spatial_sizes_bench(args, torch):
    """Where the spatial mode pays: one call = prediction of all j + force
    on ni i (a random subset of the j, 6th order, mixed, lists on), timed on
    the device (median of the timed calls), with the spatial mode off (0)
    and on for every call (2); j = 16384, 65536, 131072 and 2^20 Plummer + 10 %
    binaries."""
    import sapporo2_b200 as sp
    from sapporo2_b200 import ic
    sizes = [512, 1024, 2048, 4096, 8192, 16384, 65536]
    rows = []
    for nj in (16384, 65536, 131072, 1 << 20):
        cfg = ic.make_config("C3", n=nj, seed=3)
        rng = np.random.default_rng(1)
        z = np.zeros((nj, 3))
        njsizes = [ni for ni in sizes if ni <= nj]
        sels = {ni: np.sort(rng.choice(nj, ni, replace=False)) for ni in njsizes}
        ms = {}
        for mode in (0, 2):
            s = sp.Sapporo(order=sp.SIXTH, precision=sp.DOUBLESINGLE)
            s.set_spatial(mode, 0.0)
            stream = torch.cuda.Stream()
            s.set_stream(stream.cuda_stream)
            s.set_j_particles(np.arange(nj), cfg["id"], np.zeros(nj), cfg["m"], cfg["x"],
                              cfg["v"], z, z, z, z)
            s.force_prediction(nj)
            lib, dev = s.lib, s.dev
            for ni in njsizes:
                sel = sels[ni]
                rec = sp.pack_i_records(2, cfg["x"][sel], cfg["v"][sel], np.full(ni, 1e-4),
                                        cfg["id"][sel], z[sel])
                i_dev = torch.from_numpy(rec).cuda()
                res = torch.zeros((ni, sp.RES_STRIDE), dtype=torch.float64, device="cuda")
                cnt = torch.zeros(ni, dtype=torch.int32, device="cuda")
                lst = torch.zeros(ni * sp.NGB_PB, dtype=torch.int32, device="cuda")
                ts = []
                for it in range(args.warmup + args.steps):
                    e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
                    e0.record(stream)
                    rc = lib.sapb_predict(dev, nj, 0.0)
                    rc |= lib.sapb_force_device(dev, nj, ni, i_dev.data_ptr(), 1e-6,
                                                sp.F_NGB_LIST, res.data_ptr(), cnt.data_ptr(),
                                                lst.data_ptr())
                    e1.record(stream)
                    e1.synchronize()
                    if rc:
                        raise RuntimeError(lib.sapb_last_error(dev).decode())
                    if it >= args.warmup:
                        ts.append(e0.elapsed_time(e1))
                ms[(mode, ni)] = float(np.median(ts))
            s.set_stream(None)
            s.close()
        for ni in njsizes:
            a, b = ms[(0, ni)], ms[(2, ni)]
            rows.append({"nj": nj, "ni": ni, "log2_pairs": round(float(np.log2(ni * nj)), 1),
                         "address_ms": a, "spatial_ms": b, "speedup": a / b})
            log(f"[bench] nj {nj} ni {ni}: address {a:.3f} ms spatial {b:.3f} ms x{a / b:.3f}")
    big = [r["speedup"] for r in rows if r["log2_pairs"] >= 33]
    print(json.dumps({
        "metric": "spatial mode / address order speed-up per call (predict + force, 6th order, "
                  "mixed, lists on), calls of >= 2^33 pairs",
        "value": float(np.mean(big)), "unit": "x", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 body + ds positions (near tiles) + f64 sums", "data": "synthetic",
        "config": {"workload": "call sizes: i random subsets of j = 16384, 65536, 131072 and "
                               "2^20 (Plummer + 10 % binaries)", "rows": rows},
    }), flush=True)


def blocksteps_leg(bs_steps: int, modes=("class", "batch")) -> dict:
    """Block time steps of one system (N = 131072 Plummer, 6th order,
    dt = 2^-k with k uniform in 3..12, lists on with h2 for ~32 neighbours):
    the first `bs_steps` block times of the 2^-12 grid, each with the active
    set its block-bin occupancy gives.  Per step the active particles' j
    records are re-staged, then the force on the active set is computed
    (a) through the sapporo class (set_time, startGravCalc, getGravResults)
    and/or (b) through the batch API (plan, i records, one graph replay,
    results).  Host wall time per step; the active particles' arrays (the
    corrector's output in an integrator) are gathered before the timed loop;
    every mode runs the steps twice and the second pass is timed."""
    import sapporo2_b200 as sp
    from sapporo2_b200 import ic
    from sapporo2_b200.direct import fp64_direct
    cfg = ic.make_config("C2")
    n, k = cfg["n"], cfg["k"]
    x, v, m, ids, eps2 = cfg["x"], cfg["v"], cfg["m"], cfg["id"], cfg["eps2"]
    a, j, _ = fp64_direct(1, x, v, None, m, ids, eps2)
    _, _, sn = fp64_direct(2, x, v, a, m, ids, eps2)
    c = ic.crackle_from(x, a, j)
    steps = []
    for st in range(1, bs_steps + 1):
        T_, t0, act = ic.block_state(k, st)
        px, pv, pa = ic.predict_fp64(2, T_, t0[act], x[act], v[act], a[act], j[act], sn[act],
                                     c[act])
        jarr = (act, ids[act], t0[act], m[act], x[act], v[act], a[act], j[act], sn[act],
                c[act])
        steps.append((T_, jarr, px, pv, pa, cfg["h2"][act]))
    inter = float(sum(len(q[1][0]) for q in steps)) * n
    out = {}
    with sp.Sapporo(order=sp.SIXTH, precision=sp.DOUBLESINGLE, n_pipes=n) as s:
        s.set_j_particles(np.arange(n), ids, np.zeros(n), m, x, v, a, j, sn, c)
        for mode in [md for md in modes for _ in range(2)]:  # second pass timed
            times = []
            b = sp.Batch(s, 1, n) if mode == "batch" else None
            for T_, jarr, px, pv, pa, h2 in steps:
                act, idact = jarr[0], jarr[1]
                t_a = time.perf_counter()
                s.set_j_particles(*jarr)
                if mode == "class":
                    s.set_time(T_)
                    s.start(n, idact, px, pv, pa, eps2, h2)
                    s.results(n)
                else:
                    s.set_no_time()  # the batch run predicts; here only the upload
                    s.force_prediction(n)
                    b.plan([0], [n], [len(act)], [T_], [eps2])
                    b.i_stage[:len(act)] = sp.pack_i_records(2, px, pv, h2, idact, pa)
                    b.run(sp.F_PREDICT | sp.F_NGB_LIST)
                    b.results()
                times.append(time.perf_counter() - t_a)
            if b is not None:
                b.close()
            out[mode] = {"s_total": float(np.sum(times)),
                         "ms_per_step": 1e3 * float(np.mean(times)),
                         "interactions_per_s": inter / float(np.sum(times))}
    act_n = np.array([len(q[1][0]) for q in steps])
    out.update({"n": n, "block_steps": bs_steps, "active_mean": float(act_n.mean()),
                "active_min": int(act_n.min()), "active_max": int(act_n.max()),
                "interactions": inter})
    return out


def run_blocksteps_bench(args):
    r = blocksteps_leg(args.bs_steps)
    print(json.dumps({
        "metric": "interactions/s over block steps (N=131072 Plummer, 6th order, dt=2^-k, "
                  "k in 3..12, lists on), host wall time per step",
        "value": r["class"]["interactions_per_s"], "unit": "interactions/s", "n_gpus": 1,
        "steps": args.bs_steps, "warmup": args.bs_steps, "ms_per_step": r["class"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 body + ds positions (near tiles) + f64 sums", "data": "synthetic",
        "config": {"workload": "block steps of one system (C2)", "n": r["n"],
                   "block_steps": args.bs_steps, "active_mean": r["active_mean"],
                   "active_min": r["active_min"], "active_max": r["active_max"],
                   "class_api": r["class"], "batch_api": r["batch"]},
    }), flush=True)


def run_fma_ceiling_bench(args):
    """What the FP32 pipe sustains for the force kernel's instruction mixes
    (bench_fma_ceiling.cu, compiled here for sm_100a): packed FFMA2 chains
    alone and with one MUFU rsqrt per 16 FFMA2 or one broadcast LDS.128 per
    32 FFMA2, at 8, 4, 3 and 2 resident 128-thread blocks per SM."""
    import re
    import tempfile
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "fma_ceiling")
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                        "-o", exe, str(ROOT / "bench_fma_ceiling.cu")], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    log(out)
    rows = []
    for ln in out.splitlines():
        m = re.match(r"(\d+) blocks/SM\s+(\S+)\s+([\d.]+) ms\s+([\d.]+) TFLOP/s\s+([\d.]+) %", ln)
        if m:
            rows.append({"blocks_per_sm": int(m.group(1)), "mix": m.group(2),
                         "tflops": float(m.group(4)), "frac_nominal": float(m.group(5)) / 100})
    ceil = {(r["blocks_per_sm"], r["mix"]): r["frac_nominal"] for r in rows}
    print(json.dumps({
        "metric": "FP32-pipe ceiling: fraction of nominal FP32 peak sustained by FFMA2 chains "
                  "with one MUFU per 16 FFMA2, 2 resident blocks/SM",
        "value": ceil.get((2, "ffma2+mufu")), "unit": "fraction of nominal", "n_gpus": 1,
        "steps": 3, "warmup": 1, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "fma_ceiling probe (bench_fma_ceiling.cu)", "rows": rows},
    }), flush=True)


def rel_stats(got, want):
    e = np.linalg.norm(got - want, axis=1) / np.maximum(np.linalg.norm(want, axis=1), 1e-300)
    return {"median": float(np.median(e)), "max": float(e.max())}


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation of the path is
    not separable from its host class, so the CPU restatement (oracle port,
    FP64 OpenMP) of the same Hermite expressions is timed on all host cores,
    on bounded samples of the same workload."""
    if rank != 0:
        return
    from sapporo2_b200 import ic
    from oracle import oracle as O
    n = args.n
    cfg = ic.make_config("C3", n=n, seed=3)
    rng = np.random.default_rng(7)
    z = np.zeros((n, 3))
    # derivatives do not change the cost of a pair evaluation; use zeros
    cfg["a"] = cfg["j"] = cfg["s"] = cfg["c"] = z
    px, pv, pa = O.predict(2, cfg["ti"], cfg["t0"], cfg["x"], cfg["v"], z, z, z, z)
    threads = O.max_threads()
    nsample = args.ref_sample
    times = []
    for it in range(args.warmup + args.steps):
        sel = np.sort(rng.choice(n, nsample, replace=False)).astype(np.int32)
        t0 = time.perf_counter()
        O.force_subset(2, sel, px, pv, pa, cfg["h2"], cfg["id"], px, pv, pa, cfg["m"], cfg["id"],
                       cfg["eps2"], nthreads=threads)
        if it >= args.warmup:
            times.append(time.perf_counter() - t0)
    per = float(nsample) * n / np.mean(times)
    sample = f"{nsample} random i x all {n} j per step (6th order, FP64)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": per, "unit": "interactions/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean(times)) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "precision form: Plummer N=2^20, Salpeter masses, 10% binaries, "
                               "Hermite 6th order", "n": n, "order": 6},
        "cpu_baseline": {"value": per, "unit": "interactions/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": per, "unit": "interactions/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def spatial_mode() -> int:
    """Spatial mode the library opens with (SAPPORO_B200_SPATIAL, default 1)."""
    v = os.environ.get("SAPPORO_B200_SPATIAL")
    return 1 if v is None else (0 if int(v) == 0 else min(int(v), 2))


def spatial_on(ni: int, nj: int) -> bool:
    """Whether a mixed-precision force call of ni x nj pairs runs in spatial
    mode (the library's rule: mode 2, or mode 1, >= 1024 i, >= 65536 j and >= 2^28
    pairs)."""
    m = spatial_mode()
    return m == 2 or (m == 1 and ni >= 1024 and nj >= 65536 and ni * nj >= 1 << 28)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sapporo_b200")
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--address-steps", type=int, default=2,
                    help="timed steps of the address-order (spatial mode off) arm")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the block-step (C2) and ensemble (C4) legs of the default run")
    ap.add_argument("--cpu-sample", type=int, default=16384,
                    help="i of the timed CPU-baseline sample (x all N j; about 10 s on 16 host threads)")
    ap.add_argument("--ref-sample", type=int, default=1024)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", choices=["precision", "ensemble", "learned_h2", "blocksteps",
                                           "spatial_sizes", "fma_ceiling"],
                    default="precision",
                    help="precision: the N=2^20 6th-order bench line; ensemble: 512 clusters; "
                         "learned_h2: block steps with fixed, count-scaled and learned h2; "
                         "blocksteps: block steps of one system, class vs batch API; "
                         "spatial_sizes: predict + force per call, address order vs spatial "
                         "mode, over call sizes; fma_ceiling: what the FP32 pipe sustains for "
                         "the force kernel's instruction mixes")
    ap.add_argument("--bs-steps", type=int, default=64)
    ap.add_argument("--multi", choices=["shard", "replicas"], default="shard",
                    help="N>1 GPUs: shard: one N-body system, j split over the ranks "
                         "(strong scaling); replicas: an independent system per rank")
    ap.add_argument("--c5-n", type=int, default=262144)
    ap.add_argument("--c5-steps", type=int, default=200)
    ap.add_argument("--launch", default=None,
                    help="force-kernel shape override tpi,ip,slices (default: planner)")
    ap.add_argument("--only", choices=["all", "mixed", "fp64"], default="all",
                    help="mixed / fp64: time only that device arm (profiling runs)")
    ap.add_argument("--spatial", type=int, choices=[0, 1, 2], default=None,
                    help="spatial mode of the mixed-precision calls (default: the library's, "
                         "SAPPORO_B200_SPATIAL or 1)")
    args = ap.parse_args()
    if args.spatial is not None:
        os.environ["SAPPORO_B200_SPATIAL"] = str(args.spatial)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "fma_ceiling":
        run_fma_ceiling_bench(args)
        return
    if args.launch:
        global LAUNCH, LAUNCH_PREC
        LAUNCH = tuple(int(v) for v in args.launch.split(","))
        LAUNCH_PREC = 2 if args.only == "fp64" else None  # 2 = DOUBLE

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    os.environ.setdefault("CUDA_VISIBLE_DEVICES_LOCAL", str(local))

    import sapporo2_b200 as sp
    if args.workload == "ensemble":
        run_ensemble_bench(args, torch)
        return
    if args.workload == "learned_h2":
        run_learned_h2_bench(args)
        return
    if args.workload == "blocksteps":
        run_blocksteps_bench(args)
        return
    if args.workload == "spatial_sizes":
        run_spatial_sizes_bench(args, torch)
        return
    n = args.n
    sharded = world > 1 and args.multi == "shard"
    shard = (rank, world) if sharded else None
    # j-shards: every rank builds the same system; replicas: one per rank
    cfg = build_inputs(n, seed=3 if sharded else 3 + rank)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    flush_rd = torch.ones(64 << 20, dtype=torch.float32, device="cuda")

    def flush():
        # write 256 MB (evicts the inputs), then read another 256 MB so the
        # dirty lines are written back before the timed step, not during it
        flush_buf.zero_()
        flush_rd.sum()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if args.only == "fp64":  # profiling runs of the all-FP64 kernels
        f = device_arm(cfg, sp.DOUBLE, args.steps, args.warmup, torch, flush, shard=shard)
        print(json.dumps({"metric": "interactions/s, all-FP64 kernels", "unit": "interactions/s",
                          "value": float(n) * n / (np.mean(f["force_ms"]) * 1e-3),
                          "force_ms": float(np.mean(f["force_ms"])), "plan": f["plan"]}))
        return
    clocks = ClockSampler(local)
    clocks.start()
    mix = device_arm(cfg, sp.DOUBLESINGLE, args.steps, args.warmup, torch, flush, shard=shard)
    clk = clocks.stop()
    torch.cuda.synchronize()
    step_ms = np.array(mix["pred_ms"]) + np.array(mix["force_ms"]) + np.array(mix["comb_ms"])
    total_ms = float(step_ms.sum())
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    inter_step = float(n) * n
    # replicas: every rank does a whole step; j-shards: the ranks share one
    jobs = 1 if sharded else world
    value = inter_step * args.steps * jobs / (total_ms * 1e-3)

    if args.only == "mixed":
        print(json.dumps({"metric": METRIC, "value": value, "unit": "interactions/s",
                          "force_ms": float(np.mean(mix["force_ms"])),
                          "pred_ms": float(np.mean(mix["pred_ms"])), "plan": mix["plan"]}))
        return
    f64 = device_arm(cfg, sp.DOUBLE, args.fp64_steps, 1, torch, flush, shard=shard)
    f64_ms = np.array(f64["pred_ms"]) + np.array(f64["force_ms"]) + np.array(f64["comb_ms"])
    if dist:
        t = torch.tensor([float(f64_ms.mean())], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        f64_ms = np.array([float(t.item())])
    f64_value = inter_step / (f64_ms.mean() * 1e-3)  # per job

    # the same mixed kernels in address order (double-single difference on
    # every pair, the reference's arithmetic), beside the spatial-mode line
    addr = None
    if mix["spatial"]:
        addr = device_arm(cfg, sp.DOUBLESINGLE, args.address_steps, 1, torch, flush, shard=shard,
                          spatial_mode_set=0)
        a_ms = np.array(addr["pred_ms"]) + np.array(addr["force_ms"]) + np.array(addr["comb_ms"])
        if dist:
            t = torch.tensor([float(a_ms.mean())], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            a_ms = np.array([float(t.item())])
        addr["value"] = inter_step * jobs / (a_ms.mean() * 1e-3)
        addr["ms_per_step"] = float(a_ms.mean())

    e2e = e2e_arm(cfg, args.e2e_steps, shard=shard)
    e2e_value = inter_step / e2e["s_per_step"]
    if dist:
        t = torch.tensor([e2e["s_per_step"]], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_value = inter_step * jobs / float(t.item())

    # short legs on one GPU: block steps of one system through the class (C2)
    # and the 512-cluster ensemble in one persistent launch (C4)
    legs = {}
    if world == 1 and not args.no_legs:
        bl = blocksteps_leg(16, modes=("class",))
        legs["blocksteps_c2"] = {
            "value": bl["class"]["interactions_per_s"], "unit": "interactions/s",
            "ms_per_step": bl["class"]["ms_per_step"], "block_steps": bl["block_steps"],
            "active_mean": bl["active_mean"], "active_min": bl["active_min"],
            "active_max": bl["active_max"], "n": bl["n"],
            "timing": "host wall time per block step through the sapporo class (j re-staged, "
                      "set_time, startGravCalc, getGravResults), second of two passes; the "
                      "active particles' arrays gathered before the timed loop"}
        _, lh, same = learned_h2_leg(262144, 200)
        legs["learned_h2_c5"] = {
            "value": lh["fixed"]["retries"] / max(lh["learned"]["retries"], 1),
            "unit": "x fewer overflow retries (fixed global h2 / learned h2)",
            "n": 262144, "block_steps": 200, "identical_trajectories": bool(same),
            "policies": {k: {q: v[q] for q in ("retries", "in_range_frac", "in_25pct_frac",
                                                "mean_abs_log_count_err", "ms_per_step",
                                                "t_end")} for k, v in lh.items()}}
        en = ensemble_leg(torch, steps=5, warmup=2, tune_reps=1)
        legs["ensemble_c4"] = {
            "value": en["value"], "unit": "interactions/s", "ms_per_step": en["ms_per_step"],
            "steps": en["steps"], "clusters": en["clusters"], "particles": en["particles"],
            "active_i": en["active_i"], "interactions_per_step": en["interactions_per_step"],
            "autotune": en["autotune"], "e2e": en["e2e"],
            "timing": "CUDA events around sapb_batch_run (blob upload + graph replay), after "
                      "the autotuner"}

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    peaks = measured_peaks()
    props = torch.cuda.get_device_properties(local)
    nsm = props.multi_processor_count
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = nsm * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s
    force_ms = float(np.mean(mix["force_ms"]))
    nj_loc = mix["nj_local"]  # j this rank's launches stream (all N on one GPU)
    achieved = FLOPS_6TH * float(n) * nj_loc / (force_ms * 1e-3) / 1e12
    clk_mhz = clk.get("sm_mhz") or sm_max
    fp32_peak_run = nsm * 128 * 2 * clk_mhz * 1e6 / 1e12
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    pred_bytes = 224.0  # FP64 inputs 19 doubles read + 9 values written, per j
    pred_read_write = (19 * 8 + 64)  # bytes actually moved by this predictor (64-B record out)
    pred_ms = float(np.mean(mix["pred_ms"]))

    sha = kernel_source_sha()
    traffic, traffic_note = None, (
        f"no ncu capture of this kernel source (sha {sha}); the last capture was of "
        f"{FORCE_DRAM['source_sha']}")
    if FORCE_DRAM["source_sha"] == sha and n == 1 << 20 and nj_loc == n:
        traffic = FORCE_DRAM["spatial" if mix["spatial"] else "address"]
        traffic_note = ("dram__bytes_read.sum + dram__bytes_write.sum of one force_kernel<6th,DS> "
                        f"launch at N=2^20 (ncu, 1 pass) of this kernel source (sha {sha})")

    result = {
        "metric": METRIC, "value": value, "unit": "interactions/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "strong" if sharded else "weak",
        "vs_baseline": None,
        "dtype": "f32 body + ds positions (near tiles) + f64 sums", "data": "synthetic",
        "config": {"workload": "precision form: Plummer N=2^20, Salpeter masses 0.1-100, 10% "
                               "circular binaries a~logU(1e-6,1e-4), Hermite 6th order, all i "
                               "active, NN on, lists off",
                   "n": n, "order": 6, "precision": "mixed (DS dr on near tiles, FP32 body, FP64 sums)",
                   "eps2": cfg["eps2"], "l2": "flushed between steps (256 MB write, then 256 MB read)",
                   "launch_plan": mix["plan"],
                   "spatial": {"mode": spatial_mode(), "used": mix["spatial"],
                               "far_tile_fraction": mix["far_fraction"],
                               "delta": 1e-6,
                               "note": "Morton-ordered j and i; (warp, j tile) pairs whose boxes "
                                       "are >= |x|max*2^-23/delta apart take the single-float "
                                       "position difference; the orderings (incl. two CUB "
                                       "radix sorts) are inside the timed force call"},
                   "parallelism": (f"j-shards x{world} (round-robin j, NCCL all-reduce of "
                                   "partial forces and nearest-neighbour keys)") if sharded
                   else f"replicas x{world}",
                   "combine_ms": float(np.mean(mix["comb_ms"])), "nj_per_rank": mix["nj_local"]},
        "gflops": value * FLOPS_6TH / 1e9,
        "fp64": {"value": f64_value * jobs, "unit": "interactions/s",
                 "ms_per_step": float(f64_ms.mean()),
                 "speedup_mixed_over_fp64": value / jobs / f64_value},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak,
                     "traffic": traffic,
                     "traffic_note": traffic_note,
                     "peak_note": f"derived: {nsm} SMs x 128 FP32 lanes x 2 x {sm_max:.0f} MHz "
                                  "(sm_max_mhz of measured peaks; no FP32 entry there)",
                     "frac_at_run_clock": achieved / fp32_peak_run,
                     "flops_per_interaction": FLOPS_6TH, "kernel": "force_kernel<6th,DS>",
                     "force_ms": force_ms},
        "roofline_predictor": {"bound": "hbm",
                               "achieved": pred_bytes * nj_loc / (pred_ms * 1e-3) / 1e9,
                               "peak": hbm, "unit": "GB/s",
                               "frac": pred_bytes * nj_loc / (pred_ms * 1e-3) / 1e9 / hbm,
                               "bytes_per_j": pred_bytes, "bytes_moved_per_j": pred_read_write,
                               "pred_ms": pred_ms, "peak_note": "hbm_gbs of measured peaks"},
        "e2e": {"value": e2e_value, "unit": "interactions/s",
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                "s_per_step": e2e["s_per_step"], "api": "sapporo class, n_pipes chunks",
                "chunks": e2e["chunks"]},
        "clocks": clk,
        "gpu_launches": mix["launches"],
    }
    # accuracy: mixed vs all-FP64 GPU kernel on all N
    fields = (("acc", slice(0, 3)), ("pot", slice(3, 4)), ("jrk", slice(4, 7)),
              ("snp", slice(7, 10)))
    rm, rd = mix["res"], f64["res"]
    result["accuracy_vs_fp64_gpu"] = {k: rel_stats(rm[:, sl], rd[:, sl]) for k, sl in fields}
    if addr is not None:
        result["address_order"] = {
            "value": addr["value"], "unit": "interactions/s", "ms_per_step": addr["ms_per_step"],
            "force_ms": float(np.mean(addr["force_ms"])), "steps": args.address_steps,
            "frac_fp32_peak": FLOPS_6TH * float(n) * nj_loc
                              / (float(np.mean(addr["force_ms"])) * 1e-3) / 1e12 / fp32_peak,
            "note": "the same mixed kernels with the spatial mode off: double-single position "
                    "difference on every pair (the reference's arithmetic)",
            "accuracy_vs_fp64_gpu": {k: rel_stats(addr["res"][:, sl], rd[:, sl])
                                     for k, sl in fields}}
    result.update(legs)
    if not args.no_cpu and world == 1:
        cb = cpu_baseline_leg(cfg, args.cpu_sample)
        o, sel = cb["oracle"], cb["sel"]
        result["cpu_baseline"] = {
            "value": cb["value"], "unit": "interactions/s", "cores": cb["cores"], "kind": "port",
            "sample": f"{len(sel)} seeded i x all {n} j, FP64 OpenMP, {cb['seconds']:.1f} s"}
        acc_m = {}
        for name, res in (("mixed", rm), ("fp64_gpu", rd)):
            acc_m[name] = {k: rel_stats(res[sel][:, s3], o[k] if k != "pot" else o[k][:, None])
                           for k, s3 in fields}
        result["accuracy_vs_fp64_oracle"] = acc_m
    print(json.dumps(result), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
