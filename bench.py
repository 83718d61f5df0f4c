"""Benchmark of the CKKS evaluator hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload prim|ctpt]

One JSON line on rank 0.  Workloads (all synthetic, seeded; RLWE ciphertexts are
uniform residues, so random limbs have the cost profile of real ones):

  prim  config-1 primitive chain on one ciphertext, N = 2^16, Q = [60] + 23x[50],
        P = 8x[60] (dnum 3): inverse+forward NTT of all limbs, HRotate by one slot,
        multiply + relinearize + rescale.  Unit: chains/s.

Multi-GPU: ciphertexts are independent, so every rank runs its own replica of
the step (weak scaling, no data-path collective); the step time is the max
over ranks.

--impl reference times the reference's CPU path for the same workload: the
reference has no CPU implementation of these operations, so this is the CPU
oracle (oracle/ckks_oracle.c, a scalar OpenMP restatement of the reference's
arithmetic), run on all host cores, one chain per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PRIM = dict(log_n=16, bits=[60] + [50] * 23 + [60] * 8, n_special=8)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str):
    """dram bytes per launch of `kernel` recorded from an ncu capture (profiles/traffic.txt)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            return float(parts[1])
    return None


class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.send_signal(2)  # SIGINT lets nvidia-smi flush its output
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.p = None

    def summary(self):
        """Median SM clock and the throttle reasons over samples taken while the GPU was loaded
        (power above idle)."""
        self.__exit__()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        idle = min(r[2] for r in rows)
        busy = [r for r in rows if r[2] > idle + 50] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in busy for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(busy), "power_w_max": max(r[2] for r in rows)}


# ---------------------------------------------------------------------------
# our arm


def run_ours(args, rank, world, dist):
    import torch

    import shmoai_b200
    from shmoai_b200.ckks import CKKSContext

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = shmoai_b200.lib()
    ctx = CKKSContext(PRIM["log_n"], bits=PRIM["bits"], n_special=PRIM["n_special"], device=dev)
    n, L, QP, dnum = ctx.n, ctx.nq, ctx.nq + ctx.np, ctx.dnum
    B = args.batch
    g = torch.Generator(device="cuda").manual_seed(0x5EED + rank)
    primes_t = torch.tensor(ctx.primes.astype(np.int64), device="cuda")

    def residues(*shape, rows_primes):
        # uniform residues: 62 random bits reduced mod the row's prime
        x = torch.randint(0, 2 ** 62, shape, device="cuda", generator=g, dtype=torch.int64)
        return torch.remainder(x, rows_primes.view(*([1] * (len(shape) - 2)), -1, 1))

    qL = primes_t[:L]
    ct = residues(B, 2, L, n, rows_primes=qL)
    ct2 = residues(B, 2, L, n, rows_primes=qL)
    gk = torch.remainder(torch.randint(0, 2 ** 62, (dnum, 2, QP, n), device="cuda", generator=g),
                         primes_t.view(1, 1, -1, 1))
    rk = torch.remainder(torch.randint(0, 2 ** 62, (dnum, 2, QP, n), device="cuda", generator=g),
                         primes_t.view(1, 1, -1, 1))
    ws = torch.empty(max(ctx.workspace_bytes("keyswitch", B, L) // 8 + B * 2 * L * n,
                         ctx.workspace_bytes("rescale", 2 * B, L) // 8), dtype=torch.int64, device="cuda")
    work = ct.clone()
    rot = torch.empty_like(ct)
    rel = torch.empty_like(ct)
    out = torch.empty(B, 2, L - 1, n, dtype=torch.int64, device="cuda")
    # L2 flush buffer (inputs of one chain are ~50 MB; the 126 MB L2 is flushed between steps)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.int64, device="cuda")

    def step(src):
        work.copy_(src)
        ctx.ntt_inverse_(work)
        ctx.ntt_forward_(work)
        ctx.rotate(work, 1, gk, out=rot, workspace=ws)
        m = ctx.multiply(rot, ct2)
        ctx.relinearize(m, rk, out=rel, workspace=ws)
        ctx.rescale(rel, out=out, workspace=ws)

    # clocks are sampled from before the warm-up (nvidia-smi needs ~0.3 s to start) through
    # the timed region; only samples taken while the GPU is busy count
    clk = ClockSampler(dev).__enter__()
    time.sleep(0.5)
    for _ in range(args.warmup):
        step(ct)
    torch.cuda.synchronize()

    # ---- device-resident timing
    launches0 = lib.shm_kernel_launches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if True:  # timed region
        for i in range(args.steps):
            flush.zero_()
            starts[i].record()
            step(ct)
            ends[i].record()
        torch.cuda.synchronize()
    launches = lib.shm_kernel_launches() - launches0
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    if dist:
        t = torch.tensor([dev_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = t.item()
    ms_per_step = dev_ms / args.steps
    value = world * B * 1000.0 / ms_per_step

    # ---- end to end through the API with host buffers (pinned), copies inside the timed region
    h_in = ct.cpu().pin_memory()
    h_out = torch.empty(out.shape, dtype=torch.int64).pin_memory()
    d_in = torch.empty_like(ct)
    e2e_s, e2e_e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        d_in.copy_(h_in, non_blocking=True)
        step(d_in)
        h_out.copy_(out, non_blocking=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2e_s.record()
    for _ in range(args.steps):
        d_in.copy_(h_in, non_blocking=True)
        step(d_in)
        h_out.copy_(out, non_blocking=True)
    e2e_e.record()
    torch.cuda.synchronize()
    e2e_ms = e2e_s.elapsed_time(e2e_e) / args.steps
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = t.item()

    # ---- dominant kernel: the batched NTT (both phases), timed alone with events
    nt = torch.empty(B * 2 * (L + ctx.np) * 3, L, n, dtype=torch.int64, device="cuda")
    nt.copy_(torch.remainder(torch.randint(0, 2 ** 62, nt.shape, device="cuda", generator=g), qL.view(1, -1, 1)))
    reps = 20
    for _ in range(3):
        ctx.ntt_forward_(nt)
    torch.cuda.synchronize()
    ks, ke = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ks.record()
    for _ in range(reps):
        ctx.ntt_forward_(nt)
    ke.record()
    torch.cuda.synchronize()
    ntt_ms = ks.elapsed_time(ke) / reps
    limbs = nt.numel() // n
    ntt_bytes = limbs * n * 8 * 2 * 2  # two phase kernels, each reads and writes every word once
    peak, peak_kind = measured_peaks()
    achieved = ntt_bytes / (ntt_ms * 1e-3) / 1e9
    tr = traffic_from_profiles("ntt_forward_pair_per_limb")

    clocks = clk.summary()
    res = {
        "metric": "config-1 primitive chains/s (NTT inv+fwd, HRotate, mult+relin+rescale; N=2^16, L=24, dnum=3)",
        "value": round(value, 3),
        "unit": "chains/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded uniform RNS residues; random key material)",
        "config": {"workload": "prim: config-1 chain, one ciphertext per GPU per step", "N": n, "L": L,
                   "special_primes": ctx.np, "dnum": dnum, "batch_per_gpu": B,
                   "l2": "flushed between timed steps (256 MiB write)"},
        "e2e": {"value": round(world * B * 1000.0 / e2e_ms, 3), "unit": "chains/s",
                "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "ntt fwd (fwd_col + fwd_blk), batch of limbs", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": None if tr is None else tr * limbs,
                     "algorithmic_bytes_per_launch_pair": ntt_bytes, "launch_pair_ms": round(ntt_ms, 4)},
        "clocks": clocks,
    }
    return res


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on host cores


def run_cpu_chain(sample_chains=1):
    from oracle import oracle as O

    o = O.Oracle.from_bits(PRIM["log_n"], PRIM["bits"], PRIM["n_special"])
    n, L, QP = o.n, o.nq, o.nq + o.np
    rows = list(o.primes[:L]) * 2
    ct, ct2 = O.fill(11, (2, L, n), rows), O.fill(12, (2, L, n), rows)
    key = np.stack([O.fill(13 + d, (2, QP, n), list(o.primes) * 2) for d in range(o.dnum)])
    t0 = time.perf_counter()
    for _ in range(sample_chains):
        w = o.ntt(o.intt(ct))
        r = o.apply_galois_ct(w, 5, key)
        m = o.tensor(r, ct2)
        o.rescale(o.relinearize(m, key))
    dt = time.perf_counter() - t0
    return sample_chains / dt, os.cpu_count()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="prim", choices=["prim"])
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        per_step = []
        for _ in range(args.warmup):
            run_cpu_chain(1)
        for _ in range(args.steps):
            v, cores = run_cpu_chain(1)
            per_step.append(1.0 / v)
        ms = 1000.0 * statistics.mean(per_step)
        value = 1000.0 / ms
        print(json.dumps({
            "impl": "reference",
            "metric": "config-1 primitive chains/s (NTT inv+fwd, HRotate, mult+relin+rescale; N=2^16, L=24, dnum=3)",
            "value": round(value, 4), "unit": "chains/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform RNS residues)",
            "config": {"workload": "prim: config-1 chain, one ciphertext per step"},
            "cpu_baseline": {"value": round(value, 4), "unit": "chains/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "one full chain per step (the reference has no CPU path; oracle/ckks_oracle.c)"},
            "e2e": {"value": round(value, 4), "unit": "chains/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    res = run_ours(args, rank, world, dist)
    if rank == 0:
        if not args.no_cpu_baseline:
            v, cores = run_cpu_chain(1)
            res["cpu_baseline"] = {"value": round(v, 4), "unit": "chains/s", "cores": cores, "kind": "port",
                                   "sample": "one config-1 chain on the CPU oracle (OpenMP over limbs)"}
        print(json.dumps(res))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
