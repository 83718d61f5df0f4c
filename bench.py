"""Benchmark of the CKKS evaluator hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload boot|prim|ctpt|serve|ntt|ks] [--batch B] [--shared n]

Prints one JSON line on rank 0.  Workloads (synthetic, seeded):

  boot  (default; the headline metric) S2C-first bootstrapping through the C++ host
        library, reference parameters N = 2^16, Q = [51] + 20x[46] + 14x[51],
        P = 5x[51] (dnum 7), Delta = 2^46, h = 192, inputs at 4 primes with 2^15 slots
        uniform in [-1, 1]^2; shared-a groups of --shared n (default 8; 0 = ordinary
        ciphertexts).  One step = one batch of B ciphertexts (default 32; the
        768-ciphertext job of the reference is 24 such steps).  Unit: bootstraps/s.
        The decryption error of the last batch is reported beside the speed.
  prim  config-1 chain on one ciphertext (N = 2^16, Q = [60] + 23x[50], P = 8x[60],
        dnum 3): inverse+forward NTT of all limbs, HRotate by one slot,
        multiply + relinearize + rescale.  Unit: chains/s.
  ctpt  config-2 rotation-free ct-pt matmul (768 -> 768 ciphertexts at 13 limbs) on
        the INT8 tensor cores.  Unit: output ciphertexts/s.
  serve config-5 serving loop: a Poisson stream of mixed jobs (rotation batches,
        matmuls, shared-a bootstraps) against serial plain execution.  Unit: jobs/s.
  ntt / ks  kernel cases for profiling (batched forward NTT; one rotation batch).

Multi-GPU: ciphertexts are independent, so each rank bootstraps its own batch
(weak scaling, no data-path collective); the step time is the max over ranks.

--impl reference: the reference has no CPU implementation of these operations,
so the CPU arm is the oracle (oracle/ckks_oracle.c, a scalar OpenMP restatement
of the reference's arithmetic) on all host cores: for boot, the C++ host library
built on the oracle runs one full bootstrap of the configured form (a shared-a
group of n, or one ordinary ciphertext), timed once and reported as one step.

The boot line also carries, after its timed region, the reference's own GPU build
(PhantomFHE + moai adapter for sm_100a, oracle/_ref/ref_golden) timed on the same
GPU on single-ciphertext calls and its per-ciphertext ct-pt loop, beside this
library's kernels on the same calls ("reference_gpu", "ours_same_calls").
"""
from __future__ import annotations

import argparse
import hashlib
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

PRIM = dict(log_n=16, bits=[60] + [50] * 23 + [60] * 8, n_special=8)
BOOT = dict(log_n=16, bits=[51] + [46] * 20 + [51] * 14 + [51] * 5, n_special=5, scale=2.0 ** 46, h=192,
            input_level=4)
# key switches of one bootstrap (counted from the pipeline: rotations in the six linear
# transforms + the conjugation, relinearisations of EvalMod on the re and im halves)
BOOT_METRIC = "bootstraps/s (S2C-first, N=2^16, 35+5 primes, dnum 7, h=192, 2^15 slots, mean err <= 2e-5)"
GELU_METRIC = "GELU ciphertexts/s (gelu_cheb degree-24 series, N=2^16, input at 12 primes)"
PRIM_METRIC = "config-1 primitive chains/s (NTT inv+fwd, HRotate, mult+relin+rescale; N=2^16, L=24, dnum=3)"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str):
    """dram bytes per unit (limb) of `kernel` recorded from an ncu capture (profiles/traffic.txt)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            return float(parts[1])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 50 ms while running."""

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.5)
        return self

    def stop(self):
        if self.p:
            self.p.send_signal(2)
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.p = None

    def summary(self):
        """Median SM clock and throttle reasons over the samples taken while the GPU was loaded."""
        self.stop()
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


def timed_steps(torch, step, steps, dist, flush):
    """Device time of exactly `steps` calls (CUDA events on the launching stream), max over ranks."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")  # lets `ncu --nvtx --nvtx-include timed/` list the timed launches only
    for i in range(steps):
        if flush is not None:
            flush.zero_()
        starts[i].record()
        step()
        ends[i].record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
    return ms / steps


def ntt_roofline(torch, ctx, L, limbs_target=4096):
    """Achieved HBM bandwidth of the batched forward NTT (fwd_col + fwd_blk), the kernel pair
    that dominates every key switch, on a batch larger than L2."""
    n = ctx.n
    rows = max(1, limbs_target // L)
    g = torch.Generator(device="cuda").manual_seed(123)
    pr = torch.tensor(ctx.primes[:L].astype(np.int64), device="cuda").view(1, L, 1)
    nt = torch.remainder(torch.randint(0, 2 ** 62, (rows, L, n), device="cuda", generator=g), pr)
    for _ in range(3):
        ctx.ntt_forward_(nt)
    torch.cuda.synchronize()
    reps = 20
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        ctx.ntt_forward_(nt)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    limbs = rows * L
    algo = limbs * n * 8 * 2  # one transform reads and writes every word of every limb once: 16N bytes per limb
    peak, kind = measured_peaks()
    achieved = algo / (ms * 1e-3) / 1e9
    tr = traffic_from_profiles("ntt_forward_pair_bytes_per_limb")
    traffic = None if tr is None else round(tr * limbs)
    return {"kernel": "ntt forward (fwd_col + fwd_blk launch pair), batched limbs", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": kind, "traffic": traffic,
            "traffic_over_algorithmic": None if traffic is None else round(traffic / algo, 3),
            "algorithmic_bytes_per_launch_pair": algo, "algorithmic_bytes_per_limb": n * 16,
            "limbs_per_launch": limbs, "launch_pair_ms": round(ms, 4)}


# ---------------------------------------------------------------------------
# the reference's own GPU build on this GPU, beside the same calls of this library

REF_GOLDEN = os.path.join(ROOT, "oracle", "_ref", "ref_golden")


def _json_doc(text: str):
    """The JSON document in a harness output (the reference prints a debug line of its own)."""
    keep = [ln for ln in text.splitlines() if ln[:1] in ("{", "}", " ") or ln == ""]
    return json.loads("\n".join(keep))


def reference_gpu_leg(ctpt_cols: int = 16):
    """Times the reference's PhantomFHE + moai adapter built for sm_100a from the reference sources
    (oracle/_ref/ref_golden, mode `time`) on this GPU with CUDA events: at the config-1 chain (N = 2^16,
    [60] + 23 x [50] + 8 x [60], dnum 3) one ciphertext's inverse + forward NTT, HRotate by one slot and
    multiply + relinearize + rescale; the same calls at the bootstrapping chain's top level (35 primes,
    dnum 7); and the per-ciphertext ct-pt loop of ct_pt_matrix_mul_wo_pre_single (Ct_pt_matrix_mul.cuh:188-303,
    one stream) for 768 inputs at 13 limbs and the first `ctpt_cols` output columns."""
    if not os.path.exists(REF_GOLDEN):
        return {"unavailable": "oracle/_ref/ref_golden was not built (no reference tree at build time)"}
    out = {"build": "reference PhantomFHE + moai adapter, nvcc -arch sm_100a -rdc (oracle/build_ref.sh)",
           "timing": "CUDA events on the reference's stream, 3 warm-up + 20 calls; ct-pt loop by wall clock "
                     "around a device synchronize"}
    for name, cols in (("prim", 0), ("boot", ctpt_cols)):
        try:
            r = subprocess.run([REF_GOLDEN, name, "time", str(cols)], capture_output=True, text=True, timeout=900)
            if r.returncode != 0:
                out[name] = {"error": "rc %d: %s | %s" % (r.returncode, r.stderr[-300:], r.stdout[-300:])}
                continue
            out[name] = _json_doc(r.stdout)["time"]
        except Exception as e:  # reported, not fatal: the leg is a side measurement
            out[name] = {"error": repr(e)[:300]}
    c = out.get("boot", {}).get("ctpt_loop")
    if c:
        c["output_cts_per_s"] = round(c["n_out"] * 1000.0 / c["ms"], 3)
    return out


def ours_per_ct_leg(dev: int, ctpt_cols: int = 16):
    """This library's kernels on the calls the reference leg times, one ciphertext per call (eager, CUDA
    events, 3 warm-up + 20 calls): inverse + forward NTT, HRotate by one slot, multiply + relinearize +
    rescale at the config-1 chain and at the bootstrapping chain's top level; and the ct-pt matmul of 768
    inputs at 13 limbs into `ctpt_cols` outputs on the INT8 tensor cores."""
    import torch

    from shmoai_b200.ckks import CKKSContext

    res = {}
    for name, P in (("prim", PRIM), ("boot", BOOT)):
        ctx = CKKSContext(P["log_n"], bits=P["bits"], n_special=P["n_special"], device=dev)
        n, L, QP, dnum = ctx.n, ctx.nq, ctx.nq + ctx.np, ctx.dnum
        g = torch.Generator(device="cuda").manual_seed(77)
        pt = torch.tensor(ctx.primes.astype(np.int64), device="cuda")

        def residues(shape, primes):
            x = torch.randint(0, 2 ** 62, shape, device="cuda", generator=g, dtype=torch.int64)
            return torch.remainder(x, primes.view(*([1] * (len(shape) - 2)), -1, 1))

        A, B = residues((2, L, n), pt[:L]), residues((2, L, n), pt[:L])
        gk, rk = residues((dnum, 2, QP, n), pt), residues((dnum, 2, QP, n), pt)
        ws = torch.empty(max(ctx.workspace_bytes("keyswitch", 1, L) // 8 + 2 * L * n,
                             ctx.workspace_bytes("rescale", 2, L) // 8), dtype=torch.int64, device="cuda")
        rot, rel = torch.empty_like(A), torch.empty_like(A)
        m = torch.empty(3, L, n, dtype=torch.int64, device="cuda")
        outr = torch.empty(2, L - 1, n, dtype=torch.int64, device="cuda")

        def ntt():
            ctx.ntt_inverse_(A)
            ctx.ntt_forward_(A)

        def mrr():
            ctx.multiply(A, B, out=m)
            ctx.relinearize(m, rk, out=rel, workspace=ws)
            ctx.rescale(rel, out=outr, workspace=ws)

        t = {"limbs": L}
        for key, fn in (("ntt_inv_fwd_ms", ntt), ("rotate1_ms", lambda: ctx.rotate(A, 1, gk, out=rot, workspace=ws)),
                        ("mul_relin_rescale_ms", mrr)):
            for _ in range(3):
                fn()
            t[key] = round(timed_steps(torch, fn, 20, None, None), 4)
        t["chain_ms"] = round(t["ntt_inv_fwd_ms"] + t["rotate1_ms"] + t["mul_relin_rescale_ms"], 4)
        if name == "boot" and ctpt_cols:
            Lc = CTPT["L"]
            X = residues((CTPT["n_in"], 2, Lc, n), pt[:Lc])
            W = torch.round(torch.randn(CTPT["n_in"], ctpt_cols, device="cuda", generator=g, dtype=torch.float64)
                            * 0.02 * 2 ** 40).to(torch.int64)
            wsm = torch.empty(ctx.workspace_bytes("ctpt", CTPT["n_in"], Lc, ctpt_cols) // 8 + 1, dtype=torch.int64,
                              device="cuda")
            Y = torch.empty(ctpt_cols, 2, Lc, n, dtype=torch.int64, device="cuda")
            mm = lambda: ctx.ctpt_matmul(X, W, out=Y, workspace=wsm)  # noqa: E731
            for _ in range(3):
                mm()
            ms = timed_steps(torch, mm, 5, None, None)
            t["ctpt"] = {"n_in": CTPT["n_in"], "n_out": ctpt_cols, "limbs": Lc, "ms": round(ms, 3),
                         "output_cts_per_s": round(ctpt_cols * 1000.0 / ms, 3)}
            del X, Y, wsm
        res[name] = t
        ctx.close()
        torch.cuda.empty_cache()
    return res


# ---------------------------------------------------------------------------
# bootstrapping workload


def setup_boot(dev, rank, shared=0, tune_batch=0, g1=0):
    """C++ host (context, secret key, relinearisation key) and bootstrapper at the
    reference parameters; with shared = n the Sh-Galois, format and backward keys of
    shared-a groups of n replace the Galois keys.  tune_batch > 0 autotunes the kernel tiles
    and the BSGS split for batches of that size first (the split decides the keys)."""
    from shmoai_b200.host import Bootstrapper, Host

    h = Host(BOOT["log_n"], bits=BOOT["bits"], n_special=BOOT["n_special"], hamming_weight=BOOT["h"],
             seed=0x5EED + rank, device=dev)
    h.gen_relin_key()
    bs = Bootstrapper(h, BOOT["scale"], BOOT["input_level"])
    bs.tuning = bs.tune(tune_batch, shared) if tune_batch else []
    if g1:  # a fixed BSGS split for every slot-transform layer (the tuned kernel tiles are kept)
        bs.split = [g1] * 6
    if shared:
        h.gen_shared_keys(shared, bs.galois_elts(), hamming_weight=BOOT["h"])
    else:
        h.gen_galois_keys(bs.galois_elts())
    return h, bs


def run_boot(args, rank, world, dist):
    import torch

    import shmoai_b200
    from shmoai_b200.ckks import CKKSContext

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = shmoai_b200.lib()
    S = args.shared
    B = args.batch
    if S and B % S:
        raise SystemExit("--batch must be a multiple of --shared")
    h, bs = setup_boot(dev, rank, S, tune_batch=0 if args.no_tune else B, g1=args.g1)
    rng = np.random.default_rng(1000 + rank)
    n = h.n // 2
    z = rng.uniform(-1, 1, (B, n)) + 1j * rng.uniform(-1, 1, (B, n))
    ct = h.encrypt(z, BOOT["scale"], BOOT["input_level"])
    holder = {}

    c2s = args.form == "c2s"
    if c2s and S:
        raise SystemExit("--form c2s is the ordinary per-ciphertext bootstrap: use --shared 0")

    def step():
        holder["out"] = bs.run_c2s_first(ct) if c2s else bs.run(ct, S)

    resident, _ = h.device_memory(reset_peak=True)  # keys, diagonals, the input batch
    clk = ClockSampler(dev).start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _, peak = h.device_memory()
    # eager: one shm_boot_run per step (every kernel launched from the host)
    eager_ms = timed_steps(torch, step, args.steps, dist, None)
    eager_out = holder.pop("out").to_host()

    if c2s:
        # the original C2S-first form, eager (one shm_boot_run_c2s_first per step), as the plain path runs
        class _Eager:
            kernels = 0

            def __init__(self):
                self.out = None

            def launch(self):
                if self.out is not None:
                    self.out.close()
                self.out = bs.run_c2s_first(ct)

            def close(self):
                pass

        graph = _Eager()
        graph.launch()
        out = graph.out
        torch.cuda.synchronize()
        if not np.array_equal(out.to_host(), eager_out):
            raise SystemExit("repeated C2S-first bootstrap differs from the first")
        l0 = lib.shm_kernel_launches()
        ms = timed_steps(torch, graph.launch, args.steps, dist, None)
        launches = lib.shm_kernel_launches() - l0
        out = graph.out
        graph.kernels = launches // max(1, args.steps)
    else:
        # the timed path: the same bootstrap recorded once as a CUDA graph (BatchBootstrapper::capture)
        # and replayed; its output must equal the eager one bit for bit
        graph, out = bs.capture(ct, S)
        for _ in range(args.warmup):
            graph.launch()
        torch.cuda.synchronize()
        if not np.array_equal(out.to_host(), eager_out):
            raise SystemExit("graph replay differs from the eager bootstrap")
        l0 = lib.shm_kernel_launches()
        ms = timed_steps(torch, graph.launch, args.steps, dist, None)  # a batch is ~1 GB of live data > L2
        launches = lib.shm_kernel_launches() - l0
    err = np.abs(h.decrypt(out) - z)
    out_level = out.level

    # end to end through the host C ABI: pinned host input -> the graph's input batch
    # (shm_ct_write), graph replay, output -> pinned host memory (shm_ct_to_host), every step
    h_in = torch.from_numpy(ct.to_host().view(np.int64)).pin_memory()
    h_out = torch.empty((out.count, out.size, out.level, h.n), dtype=torch.int64).pin_memory()

    def e2e_step():
        ct.write_from_ptr(h_in.data_ptr())
        graph.launch()
        (graph.out if c2s else out).to_ptr(h_out.data_ptr())

    if args.no_extras:
        e2e_ms, roof = ms, None
    else:
        e2e_step()
        torch.cuda.synchronize()
        e2e_ms = timed_steps(torch, e2e_step, max(1, args.steps // 2), dist, None)
        ctx = CKKSContext(BOOT["log_n"], primes=h.primes, n_special=BOOT["n_special"], device=dev)
        roof = ntt_roofline(torch, ctx, len(BOOT["bits"]) - BOOT["n_special"])
        ctx.close()
    graph_kernels = graph.kernels
    graph.close()
    clocks = clk.summary()
    side = {}
    if not args.no_extras and world == 1:
        # after the timed region, with the bootstrapper's keys and memory pool released: the same
        # single-ciphertext calls on this library and on the reference's own GPU build, one after the
        # other on this GPU
        for obj in (out, ct, bs, h):
            obj.close()
        torch.cuda.empty_cache()
        side["ours_same_calls"] = ours_per_ct_leg(dev)
        torch.cuda.empty_cache()
        side["reference_gpu"] = reference_gpu_leg()
    return {
        "metric": BOOT_METRIC, "value": round(world * B * 1000.0 / ms, 3), "unit": "bootstraps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded uniform slot values in [-1,1]^2, symmetric encryption, random keys)",
        "config": {"workload": ("boot: shared-a S2C-first bootstrap of a batch of ciphertexts per GPU per step"
                                if S else "boot: original C2S-first bootstrap (bootstrap_3 form), eager, of a batch of "
                                "ciphertexts per GPU per step" if c2s else
                                "boot: S2C-first bootstrap of a batch of ciphertexts per GPU per step"),
                   "batch_per_gpu": B, "shared_a_group": S or None, "N": h.n, "slots": n,
                   "input_primes": BOOT["input_level"], "output_primes": out_level, "Q": "[51]+20x[46]+14x[51]",
                   "P": "5x[51]", "dnum": h.nq // h.np,
                   "path": ("C++ host library over the C ABI: shm_boot_run_c2s_first per step (eager)" if c2s else
                            "C++ host library over the C ABI: shm_boot_capture once, shm_host_graph_launch per step"),
                   "graph_kernels_per_step": int(graph_kernels),
                   "eager_ms_per_step": round(eager_ms, 3),
                   "autotune": {r["knob"]: r["candidates"][r["chosen"]] for r in bs.tuning} or None,
                   "autotune_ms": {r["knob"]: dict(zip(r["candidates"], [round(t, 3) for t in r["ms"]]))
                                   for r in bs.tuning} or None,
                   "device_gb": {"resident_keys_plan_input": round(resident / 2 ** 30, 2),
                                 "peak": round(peak / 2 ** 30, 2)},
                   "h": BOOT["h"], "evalmod": "Chebyshev deg 47, K=25, 3 double angles",
                   "err_mean": float(err.mean()), "err_max": float(err.max()),
                   "l2": "not flushed: the step's live data (~1 GB per batch of 32) exceeds the 126 MB L2",
                   "reference_published": "2.30 (ordinary) / 3.67 (n=4) / 3.97 (n=8) bootstraps/s on RTX PRO 6000"},
        "e2e": {"value": round(world * B * 1000.0 / e2e_ms, 3), "unit": "bootstraps/s",
                "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8)},
        "gpu_launches": int(launches),
        "roofline": roof,
        "clocks": clocks,
        **side,
    }


def cpu_boot_run(shared: int = 0):
    """One full S2C-first bootstrap on the host cores: the C++ host library built on the CPU oracle
    (oracle/_build/libshmoai_host_oracle.so, OpenMP over limbs) at the reference parameters, keys generated
    before the timed call.  shared = n: one shared-a group of n ciphertexts; 0: one ordinary ciphertext.
    Returns (bootstraps/s, seconds of the timed bootstrap, seconds of set-up, mean decryption error)."""
    from shmoai_b200.host import Bootstrapper, Host

    lib = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
    t0 = time.perf_counter()
    h = Host(BOOT["log_n"], bits=BOOT["bits"], n_special=BOOT["n_special"], hamming_weight=BOOT["h"], seed=0x5EED,
             lib=lib)
    h.gen_relin_key()
    bs = Bootstrapper(h, BOOT["scale"], BOOT["input_level"])
    if shared:
        h.gen_shared_keys(shared, bs.galois_elts(), hamming_weight=BOOT["h"])
    else:
        h.gen_galois_keys(bs.galois_elts())
    count = shared or 1
    rng = np.random.default_rng(3000)
    z = rng.uniform(-1, 1, (count, h.n // 2)) + 1j * rng.uniform(-1, 1, (count, h.n // 2))
    ct = h.encrypt(z, BOOT["scale"], BOOT["input_level"])
    setup = time.perf_counter() - t0
    t1 = time.perf_counter()
    out = bs.run(ct, shared)
    secs = time.perf_counter() - t1
    err = float(np.abs(h.decrypt(out) - z).mean())
    out.close()
    ct.close()
    bs.close()
    h.close()
    return count / secs, secs, setup, err


def cpu_boot_sample(shared: int = 0):
    """cpu_boot_run with the sample described for the JSON line."""
    v, secs, setup, err = cpu_boot_run(shared)
    what = (f"one full shared-a S2C-first bootstrap of a group of {shared} ciphertexts" if shared else
            "one full S2C-first bootstrap of one ordinary ciphertext")
    sample = (f"{what} at N = 2^16, 35 + 5 primes, input at 4 primes ({secs:.1f} s; mean error {err:.2e}), "
              f"through the C++ host library built on the CPU oracle (OpenMP over limbs); key generation and "
              f"set-up ({setup:.1f} s) before the timed call")
    return v, os.cpu_count(), sample, secs


# ---------------------------------------------------------------------------
# serving workload: a Poisson stream of mixed jobs through the serving loop, against
# the same jobs executed one after the other on the plain per-ciphertext path

SERVE = dict(n_jobs=200, rate=3.0, seed=5, p_rot=0.65, p_mm=0.15, members=8, boot_batch=32, mm_n=192, mm_L=13,
             rot_steps=(1, 2, 4, 8), rot_max=32, rot_levels=(4, 24), slots=3, budget_gb=72, outstanding=24)


def serve_jobs(rng):
    """(kind, count, level, step or members, arrival time) of each job, Poisson arrivals."""
    S, t, jobs = SERVE, 0.0, []
    for _ in range(S["n_jobs"]):
        t += rng.exponential(1.0 / S["rate"])
        u = rng.random()
        if u < S["p_rot"]:
            lo, hi = S["rot_levels"]
            jobs.append(("rot", int(rng.integers(1, S["rot_max"] + 1)), int(rng.integers(lo, hi + 1)),
                         int(rng.choice(S["rot_steps"])), t))
        elif u < S["p_rot"] + S["p_mm"]:
            jobs.append(("mm", S["mm_n"], S["mm_L"], 0, t))
        else:
            jobs.append(("boot", S["boot_batch"], BOOT["input_level"], S["members"], t))
    return jobs


def run_serve(args, rank, world, dist):
    import threading

    import torch

    import shmoai_b200
    from shmoai_b200.host import Bootstrapper, Host, Server

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = shmoai_b200.lib()
    S = SERVE
    h = Host(BOOT["log_n"], bits=BOOT["bits"], n_special=BOOT["n_special"], hamming_weight=BOOT["h"],
             seed=0x5EED + rank, device=dev)
    h.gen_relin_key()
    bs = Bootstrapper(h, BOOT["scale"], BOOT["input_level"])
    h.gen_galois_keys(sorted(set(bs.galois_elts()) | {h.galois_elt(s) for s in S["rot_steps"]}))
    h.gen_shared_keys(S["members"], bs.galois_elts(), hamming_weight=BOOT["h"])
    jobs = serve_jobs(np.random.default_rng(S["seed"] + rank))
    rng = np.random.default_rng(77 + rank)
    w_scale = 2.0 ** 20
    W = np.rint(rng.normal(0, 0.02, (S["mm_n"], S["mm_n"])) * w_scale).astype(np.int64)
    # one encrypted batch per (kind, level) with the largest count any job of that shape asks for;
    # a job's input is a device copy of its first `count` ciphertexts (200 distinct inputs would not
    # fit beside the keys)
    masters = {}
    for kind, count, L, _, _ in jobs:
        key = (kind, L)
        masters[key] = max(masters.get(key, 0), count)
    for key, count in list(masters.items()):
        kind, L = key
        z = rng.uniform(-1, 1, (count, h.n // 2)) + 1j * rng.uniform(-1, 1, (count, h.n // 2))
        masters[key] = (z, h.encrypt(z, BOOT["scale"] if kind != "rot" else 2.0 ** 40, L))
    inputs = []
    for kind, count, L, _, _ in jobs:
        z, master = masters[(kind, L)]
        inputs.append((z[:count], master))
    h.synchronize()

    def submit(srv, i):
        kind, count, L, arg, _ = jobs[i]
        ct = h.slice(inputs[i][1], 0, count)
        if kind == "rot":
            return srv.submit_rotate(ct, arg)
        if kind == "mm":
            return srv.submit_matmul(ct, W, w_scale)
        return srv.submit_bootstrap(ct, arg)

    def digest(arr):
        return hashlib.blake2b(np.ascontiguousarray(arr).tobytes(), digest_size=16).hexdigest()

    def ends_digest(ct):
        """Digest of a batch's first and last ciphertext, compared bit for bit between the served,
        capacity and plain runs (hashing every output of 200 jobs would hold the collector back)."""
        parts = []
        for k in (0, ct.count - 1):
            one = h.slice(ct, k, 1)
            parts.append(digest(one.to_host()))
            one.close()
        return "".join(parts)

    def run_stream(srv, t0=None):
        """Submit every job (at its Poisson arrival time when t0 is given, else at once) with at most
        `outstanding` jobs submitted and not yet collected, and collect them in order on another
        thread: each output is reduced to a digest (rotations, matmuls) or a decryption error
        (bootstraps) and released at once, so device memory holds only the outstanding jobs."""
        n = len(jobs)
        ids, ready = [None] * n, [threading.Event() for _ in range(n)]
        times, digests, errs, fail = [None] * n, [None] * n, [], []
        late = [0.0] * n  # how long after its arrival time each job was submitted
        slots = threading.Semaphore(S["outstanding"])

        def feeder():
            try:
                for i, j in enumerate(jobs):
                    if t0 is not None:
                        delay = t0 + j[4] - time.perf_counter()
                        if delay > 0:
                            time.sleep(delay)
                    slots.acquire()
                    if t0 is not None:
                        late[i] = max(0.0, time.perf_counter() - (t0 + j[4]))
                    ids[i] = submit(srv, i)
                    ready[i].set()
            except Exception as e:  # reported by the main thread
                fail.append(e)
                for ev in ready:
                    ev.set()

        def collector():
            try:
                for i in range(n):
                    ready[i].wait()
                    if fail:
                        return
                    out, t, _ = srv.wait(ids[i])
                    times[i] = t
                    if jobs[i][0] == "boot":  # the first ciphertext decrypted
                        one = h.slice(out, 0, 1)
                        errs.append(float(np.abs(h.decrypt(one) - inputs[i][0][:1]).mean()))
                        one.close()
                    else:
                        digests[i] = ends_digest(out)
                    out.close()
                    slots.release()
            except Exception as e:
                fail.append(e)

        th = [threading.Thread(target=feeder), threading.Thread(target=collector)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        if fail:
            raise fail[0]
        return times, digests, errs, late

    # warm-up: one job of each kind through a server, then the timed stream
    srv = Server(h, bs, hbm_budget=S["budget_gb"] << 30, slots=S["slots"])
    for kind in ("rot", "mm", "boot"):
        i = next((k for k, j in enumerate(jobs) if j[0] == kind), None)
        if i is not None:
            out, _, _ = srv.wait(submit(srv, i))
            out.close()
    srv.close()
    srv = Server(h, bs, hbm_budget=S["budget_gb"] << 30, slots=S["slots"])
    resident, _ = h.device_memory(reset_peak=True)
    clk = ClockSampler(dev).start()
    l0 = lib.shm_kernel_launches()
    t0 = time.perf_counter()
    times, results, boot_err, late = run_stream(srv, t0)
    launches = lib.shm_kernel_launches() - l0
    _, peak = h.device_memory()
    stats = srv.stats()
    clocks = clk.summary()
    srv.close()
    # latency from the job's arrival (its scheduled submission) to its completion: the server's own
    # submit-to-end time plus any delay of the submission past the arrival
    lat = np.array([t[2] - t[0] + d for t, d in zip(times, late)])
    span = max(t[2] for t in times) - min(t[0] for t in times)

    # capacity: the same jobs queued as fast as the outstanding limit allows (slots saturated)
    srv = Server(h, bs, hbm_budget=S["budget_gb"] << 30, slots=S["slots"])
    cap_times, cap_results, _, _ = run_stream(srv)
    cap_span = max(t[2] for t in cap_times) - min(t[0] for t in cap_times)
    cap_stats = srv.stats()
    for i in range(len(jobs)):
        if results[i] is not None and cap_results[i] != results[i]:
            raise AssertionError(f"serving job {i} differs between the two runs")
    srv.close()

    # serial plain execution on the same GPU: jobs in arrival order, one ciphertext per call,
    # ordinary bootstrapping, the CUDA-core matmul; latency from the measured service times
    service, plain = [], []
    for i, (kind, count, L, arg, _) in enumerate(jobs):
        x = h.slice(inputs[i][1], 0, count)
        torch.cuda.synchronize()
        t = time.perf_counter()
        if kind == "mm":
            outs = [h.ctpt_matmul(x, W, w_scale, tensor_cores=False)]
        else:
            outs = []
            for c in range(count):
                one = h.slice(x, c, 1)
                outs.append(h.rotate(one, arg) if kind == "rot" else bs.run(one, 0))
        h.synchronize()
        service.append(time.perf_counter() - t)
        if kind == "boot":
            plain.append(None)
        elif kind == "mm":
            plain.append(ends_digest(outs[0]))
        else:  # one output per ciphertext: the first and the last
            plain.append(digest(outs[0].to_host()) + digest(outs[-1].to_host()))
        for o in outs:
            o.close()
        x.close()
    finish, plat = 0.0, []
    for (kind, _, _, _, arr), s in zip(jobs, service):
        finish = max(finish, arr) + s
        plat.append(finish - arr)
    plat = np.array(plat)

    same = {"rot": True, "mm": True}
    for i, (kind, *_rest) in enumerate(jobs):
        if kind != "boot":
            same[kind] = same[kind] and results[i] == plain[i]
    n_cts = sum(j[1] for j in jobs)
    kinds = {k: sum(1 for j in jobs if j[0] == k) for k in ("rot", "mm", "boot")}
    ms = lambda a, q: round(float(np.percentile(a, q)) * 1000.0, 2)  # noqa: E731
    by_kind = {}
    for k in ("rot", "mm", "boot"):
        sel = [i for i, j in enumerate(jobs) if j[0] == k]
        if sel:
            by_kind[k] = {"p50_ms": ms(lat[sel], 50), "p99_ms": ms(lat[sel], 99),
                          "plain_p50_ms": ms(plat[sel], 50), "plain_p99_ms": ms(plat[sel], 99)}
    return {
        "metric": "serving throughput, jobs/s with every job queued (rotation batches, ct-pt matmuls, shared-a "
                  "bootstraps); p50/p99 latency at Poisson arrivals",
        "value": round(len(jobs) / cap_span, 3), "unit": "jobs/s", "n_gpus": world, "steps": len(jobs), "warmup": 3,
        "ms_per_step": round(cap_span * 1000.0 / len(jobs), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform slot values, random keys)",
        "config": {"workload": "serve: Poisson arrivals at N=2^16 with resident keys, HBM-budget admission",
                   "rate_jobs_per_s": S["rate"], "jobs": kinds, "ciphertexts": n_cts, "slots": S["slots"],
                   "budget_gb": S["budget_gb"], "outstanding_jobs": S["outstanding"], "rotation_batches": f"1-{S['rot_max']} cts at {S['rot_levels']} limbs",
                   "matmul": f"{S['mm_n']}x{S['mm_n']} at {S['mm_L']} limbs",
                   "bootstrap": f"{S['boot_batch']} cts, shared-a n={S['members']}"},
        "serving": {"p50_ms": ms(lat, 50), "p99_ms": ms(lat, 99), "by_kind": by_kind,
                    "admission": "head of the queue when it fits the budget, else a later job that fits until the "
                                 "head has waited 0.5 s, then the released budget is kept for the head",
                    "poisson_jobs_per_s": round(len(jobs) / span, 3),
                    "capacity_jobs_per_s": round(len(jobs) / cap_span, 3),
                    "capacity_cts_per_s": round(n_cts / cap_span, 2), "capacity_batches": cap_stats["batches"],
                    "peak_admitted_gb": round(stats["peak_admitted"] / 2**30, 2),
                    "max_inflight": stats["max_inflight"], "batches": stats["batches"], "jobs_done": stats["jobs"],
                    "device_gb_resident": round(resident / 2 ** 30, 2), "device_gb_peak": round(peak / 2 ** 30, 2)},
        "plain_serial": {"p50_ms": ms(plat, 50), "p99_ms": ms(plat, 99),
                         "jobs_per_s": round(len(jobs) / sum(service), 3),
                         "path": "one ciphertext per call, ordinary bootstrapping, CUDA-core matmul"},
        "bit_exact_vs_plain": same, "bit_exact_checked": "first and last output ciphertext of every job",
        "bootstrap_err_mean_max": max(boot_err) if boot_err else None,
        "gpu_launches": int(launches), "clocks": clocks,
    }


# ---------------------------------------------------------------------------
# primitive-chain workload


def run_prim(args, rank, world, dist):
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
    pt = torch.tensor(ctx.primes.astype(np.int64), device="cuda")

    def residues(shape, primes):
        x = torch.randint(0, 2 ** 62, shape, device="cuda", generator=g, dtype=torch.int64)
        return torch.remainder(x, primes.view(*([1] * (len(shape) - 2)), -1, 1))

    ct = residues((B, 2, L, n), pt[:L])
    ct2 = residues((B, 2, L, n), pt[:L])
    gk = residues((dnum, 2, QP, n), pt)
    rk = residues((dnum, 2, QP, n), pt)
    ws = torch.empty(max(ctx.workspace_bytes("keyswitch", B, L) // 8 + B * 2 * L * n,
                         ctx.workspace_bytes("rescale", 2 * B, L) // 8), dtype=torch.int64, device="cuda")
    work, rot, rel = ct.clone(), torch.empty_like(ct), torch.empty_like(ct)
    m = torch.empty(B, 3, L, n, dtype=torch.int64, device="cuda")
    out = torch.empty(B, 2, L - 1, n, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.int64, device="cuda")
    d_in = ct.clone()

    def chain():
        work.copy_(d_in)
        ctx.ntt_inverse_(work)
        ctx.ntt_forward_(work)
        ctx.rotate(work, 1, gk, out=rot, workspace=ws)
        ctx.multiply(rot, ct2, out=m)
        ctx.relinearize(m, rk, out=rel, workspace=ws)
        ctx.rescale(rel, out=out, workspace=ws)

    clk = ClockSampler(dev).start()
    for _ in range(args.warmup):
        chain()
    torch.cuda.synchronize()
    eager_ms = timed_steps(torch, chain, args.steps, dist, flush)  # every kernel launched from the host
    eager_out = out.clone()
    # the timed path: the chain recorded once as a CUDA graph (shm_graph_begin / _end) and replayed
    graph = ctx.capture(chain)
    for _ in range(args.warmup):
        graph.launch()
    torch.cuda.synchronize()
    if not torch.equal(out, eager_out):
        raise SystemExit("graph replay differs from the eager chain")
    l0 = lib.shm_kernel_launches()
    ms = timed_steps(torch, graph.launch, args.steps, dist, flush)
    launches = lib.shm_kernel_launches() - l0
    h_in = ct.cpu().pin_memory()
    h_out = torch.empty(out.shape, dtype=torch.int64).pin_memory()

    def e2e():
        d_in.copy_(h_in, non_blocking=True)
        graph.launch()
        h_out.copy_(out, non_blocking=True)

    e2e()
    e2e_ms = timed_steps(torch, e2e, args.steps, dist, None)
    graph_kernels = graph.kernels
    graph.close()
    roof = ntt_roofline(torch, ctx, L)
    clocks = clk.summary()
    return {
        "metric": PRIM_METRIC, "value": round(world * B * 1000.0 / ms, 3), "unit": "chains/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded uniform RNS residues; random key material)",
        "config": {"workload": "prim: config-1 chain, one ciphertext per GPU per step", "N": n, "L": L,
                   "special_primes": ctx.np, "dnum": dnum, "batch_per_gpu": B,
                   "l2": "flushed between timed steps (256 MiB write)",
                   "path": "CUDA graph of the chain (shm_graph_begin / shm_graph_end), one replay per step",
                   "graph_kernels_per_step": int(graph_kernels), "eager_ms_per_step": round(eager_ms, 4)},
        "e2e": {"value": round(world * B * 1000.0 / e2e_ms, 3), "unit": "chains/s",
                "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8)},
        "gpu_launches": int(launches), "roofline": roof, "clocks": clocks,
    }


def cpu_prim_chain():
    from oracle import oracle as O

    o = O.Oracle.from_bits(PRIM["log_n"], PRIM["bits"], PRIM["n_special"])
    n, L, QP = o.n, o.nq, o.nq + o.np
    rows = list(o.primes[:L]) * 2
    ct, ct2 = O.fill(11, (2, L, n), rows), O.fill(12, (2, L, n), rows)
    key = np.stack([O.fill(13 + d, (2, QP, n), list(o.primes) * 2) for d in range(o.dnum)])
    t0 = time.perf_counter()
    w = o.ntt(o.intt(ct))
    r = o.apply_galois_ct(w, 5, key)
    o.rescale(o.relinearize(o.tensor(r, ct2), key))
    return 1.0 / (time.perf_counter() - t0), os.cpu_count()


_GELU_CPU = {}


def cpu_gelu_sample():
    """GELU of one ciphertext at 12 primes (N = 2^16, the bootstrapping chain) through the host
    library built on the CPU oracle (OpenMP over limbs); keys made once per process."""
    from oracle import oracle as O
    from shmoai_b200.host import Host

    if "h" not in _GELU_CPU:
        lib = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
        h = Host(BOOT["log_n"], O.gen_primes(BOOT["log_n"], BOOT["bits"]), BOOT["n_special"],
                 hamming_weight=BOOT["h"], seed=0x5EED, lib=lib)
        h.gen_relin_key()
        x = np.random.default_rng(2000).uniform(GELU["lo"], GELU["hi"], (1, h.n // 2))
        _GELU_CPU.update(h=h, ct=h.encrypt(x, BOOT["scale"], GELU["L"]))
    h, ct = _GELU_CPU["h"], _GELU_CPU["ct"]
    t0 = time.perf_counter()
    h.gelu(ct)
    return 1.0 / (time.perf_counter() - t0), os.cpu_count()


# ---------------------------------------------------------------------------
# config 4: one full-width BERT-base layer (shm_boot_bert_layer)

# the reference's layer chain for the shared-a form (test_single_layer.cuh:503-530): three 46-bit
# primes where the bootstrap region starts, so every rescale after a bootstrap is by a 46-bit prime
LAYER_BITS = [51] + [46] * 23 + [51] * 11 + [51] * 5
LAYER = dict(hidden=768, heads=12, ffn=3072, num_X=256, tokens=128, input_num=128, softmax_iter=13, ln_newt=3,
             ln_gold=2, gelu_input_level=13, ffn_chunk=128, boot_batch=16, w_scale=2.0 ** 40, ln_var_scale=64.0)
LAYER_METRIC = "BERT-base layer amortized seconds per input (256 inputs x 128 tokens, hidden 768, 12 heads, FFN 3072)"


def run_layer(args, rank, world, dist):
    """One BERT-base encoder layer per step on 256 inputs x 128 tokens (the column packing fills the 2^15
    slots): attention (12 heads), SelfOutput, four bootstrap segments of 768 ciphertexts, two LayerNorms,
    Intermediate, GELU and the masked Final projection.  --shared n: shared-a bootstrap segments
    (the reference's "sham" form); --shared 0: one ordinary bootstrap per ciphertext (its "orig"
    form).  Unit: seconds per input (the step's time / 256), lower is better."""
    import torch

    import shmoai_b200
    from shmoai_b200 import plain_layer as PL
    from shmoai_b200.host import Bootstrapper, Host

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = shmoai_b200.lib()
    S = args.shared
    cfg = dict(LAYER, members=S, boot_batch=(args.batch or LAYER["boot_batch"]) if S else 1)
    t_setup = time.perf_counter()
    h = Host(16, bits=LAYER_BITS, n_special=5, hamming_weight=BOOT["h"], seed=0x5EED + rank, device=dev)
    h.gen_relin_key()
    h.gen_public_key(0xE0C0 + rank)
    bs = Bootstrapper(h, BOOT["scale"], BOOT["input_level"])
    if S:
        h.gen_shared_keys(S, bs.galois_elts(), hamming_weight=BOOT["h"])
    else:
        h.gen_galois_keys(bs.galois_elts())
    # the attention's 127 rotation keys are made inside each layer call and released after its attention
    rng = np.random.default_rng(4000 + rank)
    X = rng.normal(0.0, 1.0, (cfg["num_X"], cfg["tokens"], cfg["hidden"]))
    w = PL.random_weights(rng, cfg["hidden"], cfg["ffn"])
    mask = np.ones(h.n // 2, dtype=np.int32)
    ct = h.batch_input(X, BOOT["scale"], 23)
    setup_s = time.perf_counter() - t_setup
    resident, _ = h.device_memory()
    print("layer: %.2f GB resident before the first call (keys, input)" % (resident / 2 ** 30), file=sys.stderr)
    holder = {}

    def step():
        holder["out"], holder["times"] = bs.bert_layer(ct, w, cfg, mask)

    clk = ClockSampler(dev).start()
    for _ in range(args.warmup):
        step()
        holder["out"].close()
    torch.cuda.synchronize()
    _, _ = h.device_memory(reset_peak=True)
    l0 = lib.shm_kernel_launches()
    stage_sum = {}
    ms = timed_steps(torch, lambda: (step(), [stage_sum.__setitem__(k, stage_sum.get(k, 0.0) + v)
                                              for k, v in holder["times"].items()]), args.steps, dist, None)
    launches = lib.shm_kernel_launches() - l0
    _, peak = h.device_memory()
    out = holder["out"]
    got = h.decrypt(out).real
    # end to end: the ciphertext batch written from pinned host memory, the layer, the output read back
    h_in = torch.from_numpy(ct.to_host().view(np.int64)).pin_memory()
    h_out = torch.empty((out.count, out.size, out.level, h.n), dtype=torch.int64).pin_memory()

    def e2e_step():
        ct.write_from_ptr(h_in.data_ptr())
        step()
        holder["out"].to_ptr(h_out.data_ptr())
        holder["out"].close()

    e2e_ms = timed_steps(torch, e2e_step, 1, dist, None) if not args.no_extras else ms
    clocks = clk.summary()
    cols = PL.pack_columns(X)
    approx = PL.layer(cols, w, cfg, mask, approx=True)
    exact = PL.layer(cols, w, cfg, mask, approx=False)
    e_a, e_x = np.abs(got - approx), np.abs(got - exact)
    n_in = cfg["num_X"]
    stages = {k: round(v / args.steps, 3) for k, v in stage_sum.items()}
    ref = {"orig": 10.34, "sham": 6.85}
    return {
        "metric": LAYER_METRIC, "value": round(ms / 1000.0 / n_in, 5), "unit": "s/input", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 1), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (inputs N(0,1); weights N(0, 0.02^2), LayerNorm gamma 1 beta 0; every token valid)",
        "config": {"workload": "layer: one BERT-base encoder layer per GPU per step ("
                               + ("shared-a bootstrap segments, groups of %d" % S if S else
                                  "one ordinary bootstrap per ciphertext") + ")",
                   "form": "sham" if S else "orig", "N": h.n, "Q": "[51]+23x[46]+11x[51]", "P": "5x[51]",
                   "bootstrap_call_batch": cfg["boot_batch"],
                   "inputs": n_in, "tokens": cfg["tokens"], "hidden": cfg["hidden"], "heads": cfg["heads"],
                   "ffn": cfg["ffn"], "stage_seconds": stages, "total_seconds": round(ms / 1000.0, 2),
                   "setup_seconds": round(setup_s, 1),
                   "error_vs_fp64_same_approximations": {"mean": float(e_a.mean()), "max": float(e_a.max())},
                   "error_vs_fp64_exact_layer": {"mean": float(e_x.mean()), "max": float(e_x.max())},
                   "device_gb_peak": round(peak / 2 ** 30, 2),
                   "device_gb_resident_keys_input": round(resident / 2 ** 30, 2),
                   "stage_device_gb_peak": {k: round(v, 1) for k, v in bs.last_stage_peak_gb.items()},
                   "reference_published_s_per_input": ref["sham" if S else "orig"],
                   "l2": "not flushed: every stage's live data exceeds the 126 MB L2"},
        "e2e": {"value": round(e2e_ms / 1000.0 / n_in, 5), "unit": "s/input",
                "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8)},
        "gpu_launches": int(launches), "roofline": None, "clocks": clocks,
    }


# ---------------------------------------------------------------------------
# kernel workloads (config 2 and the profiling cases)

CTPT = dict(n_in=768, n_out=768, L=13)  # config 2: one BERT-base projection at level 12


def int8_peak_tops(torch):
    """Dense INT8 tensor throughput of this GPU, measured: torch._int_mm (a cuBLASLt int8 GEMM with
    int32 accumulation) on 8192 x 8192 x 8192, best of 10 after warm-up, CUDA events."""
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        for _ in range(3):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(10):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            torch.cuda.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b
        return round(2 * 8192 ** 3 / (best * 1e-3) / 1e12, 1), "measured: torch._int_mm int8 8192^3, best of 10"
    except Exception as ex:  # reported, the datasheet figure stands in
        return 4500.0, "datasheet dense INT8 (measurement failed: %s)" % repr(ex)[:120]


CTPT_MODULI = [251, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163, 157, 151, 149]


def ctpt_moduli_counts(ctx, W, L, chunk=131072):
    """The residue moduli each pass of columns of the tensor-core ct-pt matmul runs with, and the
    pass's column count: a limb of prime q needs the first T moduli whose product M satisfies
    log2 M >= log2((q - 1) max_o sum_i |W_io|) + 1.05, and a pass takes the largest T of its rows
    (the library's rule, restated here to count the int8 work one step does)."""
    l1 = int(W.abs().sum(0).max().item())
    bits = np.cumsum(np.log2(np.array(CTPT_MODULI, dtype=np.float64)))
    limb_t = []
    for l in range(L):
        need = math.log2(int(ctx.primes[l]) - 1) + math.log2(max(l1, 1)) + 1.05
        limb_t.append(int(np.searchsorted(bits, need) + 1))
    n, R = ctx.n, 2 * L * ctx.n
    out = []
    for r0 in range(0, R, chunk):
        cur = min(chunk, R - r0)
        rows = range(r0 // n, (r0 + cur - 1) // n + 1)
        out.append((max(limb_t[r % L] for r in rows), cur))
    return out


def run_ctpt(args, rank, world, dist):
    """Config 2: 768 ciphertexts at 13 limbs (N = 2^16) times a 768 x 768 integer weight
    matrix (N(0, 0.02^2) at scale 2^40) on the INT8 tensor cores; step = the whole projection."""
    import torch

    import shmoai_b200
    from shmoai_b200.ckks import CKKSContext

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = shmoai_b200.lib()
    ctx = CKKSContext(BOOT["log_n"], bits=BOOT["bits"], n_special=BOOT["n_special"], device=dev)
    n, L, n_in, n_out = ctx.n, CTPT["L"], CTPT["n_in"], CTPT["n_out"]
    g = torch.Generator(device="cuda").manual_seed(2 + rank)
    pr = torch.tensor(ctx.primes[:L].astype(np.int64), device="cuda").view(1, 1, L, 1)
    X = torch.remainder(torch.randint(0, 2 ** 62, (n_in, 2, L, n), device="cuda", generator=g), pr)
    W = torch.round(torch.randn(n_in, n_out, device="cuda", generator=g, dtype=torch.float64) * 0.02 * 2 ** 40
                    ).to(torch.int64)
    ws = torch.empty(ctx.workspace_bytes("ctpt", n_in, L, n_out) // 8 + 1, dtype=torch.int64, device="cuda")
    Y = torch.empty(n_out, 2, L, n, dtype=torch.int64, device="cuda")

    def step():
        ctx.ctpt_matmul(X, W, out=Y, workspace=ws)

    clk = ClockSampler(dev).start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = lib.shm_kernel_launches()
    ms = timed_steps(torch, step, args.steps, dist, None)  # X and Y (20 GB) exceed L2
    launches = lib.shm_kernel_launches() - l0
    macs = n_in * n_out * 2 * L * n
    counts = ctpt_moduli_counts(ctx, W, L)
    i8_ops = 2 * n_in * n_out * sum(t * cols for t, cols in counts)  # the int8 GEMMs one step runs
    peak_i8, peak_src = int8_peak_tops(torch)
    res = {
        "metric": "ct-pt matmul output ciphertexts/s (768 -> 768, 13 limbs, N=2^16, exact)",
        "value": round(world * n_out * 1000.0 / ms, 2), "unit": "output ciphertexts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (int8 tensor-core residues)",
        "data": "synthetic (uniform residues; W ~ N(0, 0.02^2) * 2^40)",
        "config": {"workload": "ctpt: config 2, one 768x768 projection per GPU per step", "n_in": n_in,
                   "n_out": n_out, "L": L, "N": n, "modular_macs": macs,
                   "residue_moduli_per_pass": [t for t, _ in counts], "int8_ops_per_step": i8_ops},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "whole projection", "bound": "tensor",
                     "achieved": round(i8_ops / (ms * 1e-3) / 1e12, 1), "peak": peak_i8,
                     "unit": "TOPS (the int8 residue GEMMs run: moduli per pass of columns in config)",
                     "frac": round(i8_ops / (ms * 1e-3) / 1e12 / peak_i8, 4),
                     "peak_source": peak_src, "traffic": None},
        "clocks": clk.summary(),
    }
    return res


GELU = dict(L=12, lo=-19.5, hi=12.5)  # input at 12 primes of the bootstrapping chain


def run_gelu(args, rank, world, dist):
    """The BERT layer's GELU stage: gelu_cheb's degree-24 Chebyshev series on [-19.5, 12.5]
    (6 levels) over a batch of ciphertexts at 12 primes of the bootstrapping chain (N = 2^16,
    scale 2^46), slot values uniform on the interval; step = one replay of the GELU recorded
    as a CUDA graph through the host API (the eager per-call time is reported beside it).
    e2e adds the batch's upload from pinned host memory and the result's download."""
    import torch

    import shmoai_b200
    from shmoai_b200.host import Host

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = shmoai_b200.lib()
    h = Host(BOOT["log_n"], bits=BOOT["bits"], n_special=BOOT["n_special"], hamming_weight=BOOT["h"],
             seed=0x5EED + rank, device=dev)
    h.gen_relin_key()
    B, L = args.batch, GELU["L"]
    rng = np.random.default_rng(2000 + rank)
    x = rng.uniform(GELU["lo"], GELU["hi"], (B, h.n // 2))
    ct = h.encrypt(x, BOOT["scale"], L)
    holder = {}

    def step():
        holder["out"] = h.gelu(ct)

    clk = ClockSampler(dev).start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # eager: every kernel launched from the host, one call per step
    eager_ms = timed_steps(torch, step, args.steps, dist, None)
    eager_out = holder.pop("out").to_host()
    # the timed path: the same GELU recorded once as a CUDA graph and replayed (bit-identical)
    graph, out = h.capture_chebyshev(ct)
    for _ in range(args.warmup):
        graph.launch()
    torch.cuda.synchronize()
    if not np.array_equal(out.to_host(), eager_out):
        raise SystemExit("graph replay differs from the eager GELU")
    l0 = lib.shm_kernel_launches()
    ms = timed_steps(torch, graph.launch, args.steps, dist, None)  # a batch at 12 primes is 805 MB > L2
    launches = lib.shm_kernel_launches() - l0
    y = h.decrypt(out).real
    gelu = 0.5 * x * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0)))
    err = np.abs(y - gelu)
    # end to end: pinned host batch -> device, GELU, result -> pinned host memory
    h_in = torch.from_numpy(ct.to_host().view(np.int64)).pin_memory()
    h_out = torch.empty((out.count, out.size, out.level, h.n), dtype=torch.int64).pin_memory()

    def e2e_step():
        ct.write_from_ptr(h_in.data_ptr())
        graph.launch()
        (graph.out if c2s else out).to_ptr(h_out.data_ptr())

    e2e_ms = timed_steps(torch, e2e_step, args.steps, dist, None)
    clocks = clk.summary()
    return {
        "metric": GELU_METRIC,
        "value": round(world * B * 1000.0 / ms, 2), "unit": "ciphertexts/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform slot values on [-19.5, 12.5])",
        "config": {"workload": "gelu: the BERT layer's GELU stage on a batch per GPU per step", "batch_per_gpu": B,
                   "N": h.n, "input_primes": L, "output_primes": out.level, "scale": BOOT["scale"],
                   "err_vs_gelu_mean": float(err.mean()), "err_vs_gelu_max": float(err.max()),
                   "path": "host API: one CUDA graph of the GELU (shm_host_chebyshev_capture) per step",
                   "eager_ms_per_step": round(eager_ms, 3), "graph_kernels_per_step": int(graph.kernels),
                   "reference_published": "GELU stage of one layer: 3072 ciphertexts in 30.2 s (101.7/s) on "
                                          "RTX PRO 6000 (single_layer_results.csv)"},
        "e2e": {"value": round(world * B * 1000.0 / e2e_ms, 2), "unit": "ciphertexts/s",
                "h2d_bytes_per_step": int(h_in.numel() * 8), "d2h_bytes_per_step": int(h_out.numel() * 8)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }


def run_kernel_case(args, rank, world, dist):
    """Profiling cases: 'ntt' = forward NTT of 4095 limbs (2 GB, > L2) at the bootstrap primes;
    'ks' = one hoisted-free rotation of 4 ciphertexts at 35 limbs (the C2S key switch)."""
    import torch

    from shmoai_b200.ckks import CKKSContext

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    ctx = CKKSContext(BOOT["log_n"], bits=BOOT["bits"], n_special=BOOT["n_special"], device=dev)
    n, L, QP = ctx.n, 35, 40
    g = torch.Generator(device="cuda").manual_seed(3)
    pr = torch.tensor(ctx.primes.astype(np.int64), device="cuda")
    if args.workload == "ntt":
        x = torch.remainder(torch.randint(0, 2 ** 62, (117, L, n), device="cuda", generator=g), pr[:L].view(1, L, 1))

        def step():
            ctx.ntt_forward_(x)
        unit, per = "limbs/s", 117 * L
    elif args.workload == "zoo":
        # the bootstrap's other hot kernels on a few GB: Sh-Rot of one group of 8 at 34 limbs
        # (ip_multi_kernel, the ModUp- and ModDown-fused NTTs), a multiply-plain-accumulate of 8 terms over
        # 16 ciphertexts at 33 limbs (the BSGS inner sums), a 4-term linear combination of 8 ciphertexts at
        # 28 limbs (EvalMod's leaves) and the tensor product of 8 ciphertext pairs at 30 limbs
        import ctypes

        import shmoai_b200

        lib = shmoai_b200.lib()

        def res(shape, limbs):
            return torch.remainder(torch.randint(0, 2 ** 62, shape, device="cuda", generator=g),
                                   pr[:limbs].view(*([1] * (len(shape) - 2)), limbs, 1))

        qp_rows = pr.view(1, 1, QP, 1)
        sh = res((1, 9, 34, n), 34)
        shkey = torch.remainder(torch.randint(0, 2 ** 62, (7, 9, QP, n), device="cuda", generator=g), qp_rows)
        elt = ctx.galois_elt(5)
        Xm = res((16, 2, 33, n), 33)
        Pm = [res((33, n), 33) for _ in range(8)]
        Xs = [Xm] * 8
        mp_out = torch.empty_like(Xm)
        Xl = [res((8, 2, 28, n), 28) for _ in range(4)]
        w = np.ascontiguousarray(np.random.default_rng(4).integers(0, 2 ** 40, (4, 28)).astype(np.uint64))
        w0 = np.ascontiguousarray(np.random.default_rng(5).integers(0, 2 ** 40, 28).astype(np.uint64))
        lc_out = torch.empty_like(Xl[0])
        A, B = res((8, 2, 30, n), 30), res((8, 2, 30, n), 30)
        T = torch.empty(8, 3, 30, n, dtype=torch.int64, device="cuda")
        u64p = ctypes.POINTER(ctypes.c_uint64)

        def step():
            ctx.shared_rotate_hoisted(sh, [elt], [shkey])
            xp = (ctypes.c_void_p * 8)(*[t.data_ptr() for t in Xs])
            pp = (ctypes.c_void_p * 8)(*[t.data_ptr() for t in Pm])
            assert lib.shm_multiply_plain_accumulate(ctx._h, xp, pp, 8, ctypes.c_void_p(mp_out.data_ptr()), 32, 33,
                                                     0, None) == 0
            lp = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in Xl])
            lv = (ctypes.c_uint32 * 4)(28, 28, 28, 28)
            assert lib.shm_linear_combination(ctx._h, lp, lv, w.ctypes.data_as(u64p), 4, w0.ctypes.data_as(u64p),
                                              ctypes.c_void_p(lc_out.data_ptr()), 8, 28, None) == 0
            ctx.multiply(A, B, out=T)
        unit, per = "kernel-zoo passes/s", 1
    else:
        ct = torch.remainder(torch.randint(0, 2 ** 62, (4, 2, L, n), device="cuda", generator=g),
                             pr[:L].view(1, 1, L, 1))
        key = torch.remainder(torch.randint(0, 2 ** 62, (7, 2, QP, n), device="cuda", generator=g),
                              pr.view(1, 1, QP, 1))
        ws = torch.empty(ctx.workspace_bytes("keyswitch", 4, L) // 8 + 4 * 2 * L * n, dtype=torch.int64,
                         device="cuda")
        out = torch.empty_like(ct)

        def step():
            ctx.rotate(ct, 1, key, out=out, workspace=ws)
        unit, per = "ciphertext rotations/s", 4
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ms = timed_steps(torch, step, args.steps, dist, None)
    return {"metric": f"{args.workload} kernel case", "value": round(per * 1000.0 / ms, 2), "unit": unit,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "config": {"workload": args.workload}}


# ---------------------------------------------------------------------------


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="boot", choices=["boot", "prim", "ctpt", "ntt", "ks", "zoo", "serve",
                                                            "gelu", "layer"])
    ap.add_argument("--batch", type=int, default=None)
    ap.add_argument("--shared", type=int, default=8,
                    help="boot: shared-a group size n (0 = ordinary ciphertexts)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="boot: skip the autotuner (default tiles and BSGS split)")
    ap.add_argument("--g1", type=int, default=0, help="boot: baby steps of every slot-transform layer (0 = tuned)")
    ap.add_argument("--form", default="s2c", choices=["s2c", "c2s"],
                    help="boot: S2C-first (default) or the original per-ciphertext C2S-first form (with --shared 0)")
    ap.add_argument("--no-extras", action="store_true",
                    help="time the step only (no e2e, roofline or CPU legs): used for ncu launch lists")
    ap.add_argument("--small", action="store_true",
                    help="ctpt: 768 -> 768 ciphertexts at 1 limb, one column chunk of the full projection "
                         "(about 4 GB on the device) for ncu captures")
    args = ap.parse_args()
    if args.small:
        CTPT.update(L=1)
    if args.batch is None:
        args.batch = {"boot": 32, "gelu": 64, "layer": 0}.get(args.workload, 1)  # layer: 0 = LAYER's boot_batch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload not in ("boot", "prim", "gelu"):
            print(json.dumps({"impl": "reference", "unavailable": "no CPU arm for the kernel workload "
                              + args.workload + " (timed on the GPU only)"}))
            return
        if args.workload == "boot":
            # one full bootstrap of the configured form (a shared-a group of n, or one ordinary
            # ciphertext) is minutes of CPU work: the arm runs it once and reports that one step
            shared = args.shared
            need = (7 * (shared + 1) if shared else 14) * 40 * 2 ** 16 * 8 * 42 + (24 << 30)
            try:
                import psutil

                avail = psutil.virtual_memory().available
            except Exception:
                avail = need
            note = None
            if shared and avail < need:
                note = (f"host memory {avail >> 30} GiB is below the ~{need >> 30} GiB the shared-a keys of a "
                        f"group of {shared} need on the CPU: one ordinary ciphertext was bootstrapped instead")
                shared = 0
            v, cores, sample, secs = cpu_boot_sample(shared)
            print(json.dumps({
                "impl": "reference", "metric": BOOT_METRIC, "value": round(v, 6), "unit": "bootstraps/s",
                "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": round(secs * 1000.0, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic (seeded uniform slot values in [-1,1]^2)",
                "config": {"workload": "boot (reference CPU arm: the reference has no host-side CKKS path; the host "
                                       "library on the oracle restatement, one full bootstrap)",
                           "shared_a_group": shared or None, "steps_requested": args.steps,
                           "warmup_requested": args.warmup, "note": note},
                "cpu_baseline": {"value": round(v, 6), "unit": "bootstraps/s", "cores": cores, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": round(v, 6), "unit": "bootstraps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
            }))
            return
        vals = []
        for i in range(args.warmup + args.steps):
            if args.workload == "gelu":
                v, cores = cpu_gelu_sample()
                sample = "GELU of one ciphertext at 12 primes per step (host library on the oracle)"
            else:
                v, cores = cpu_prim_chain()
                sample = "one full config-1 chain per step"
            if i >= args.warmup:
                vals.append(v)
        value = statistics.mean(vals)
        unit = {"boot": "bootstraps/s", "gelu": "ciphertexts/s"}.get(args.workload, "chains/s")
        metric = {"boot": BOOT_METRIC, "gelu": GELU_METRIC}.get(args.workload, PRIM_METRIC)
        print(json.dumps({
            "impl": "reference", "metric": metric,
            "value": round(value, 6), "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000.0 / value, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": args.workload + " (reference CPU arm: the oracle restatement)",
                       "shared_a_group": (args.shared or None) if args.workload == "boot" else None},
            "cpu_baseline": {"value": round(value, 6), "unit": unit, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    runner = {"boot": run_boot, "prim": run_prim, "ctpt": run_ctpt, "serve": run_serve, "ntt": run_kernel_case,
              "ks": run_kernel_case, "zoo": run_kernel_case, "gelu": run_gelu, "layer": run_layer}[args.workload]
    res = runner(args, rank, world, dist)
    if rank == 0:
        if not args.no_cpu_baseline and args.workload in ("boot", "prim", "gelu"):
            if args.workload == "gelu":
                v, cores = cpu_gelu_sample()
                res["cpu_baseline"] = {"value": round(v, 4), "unit": "ciphertexts/s", "cores": cores, "kind": "port",
                                       "sample": "GELU of one ciphertext at 12 primes (host library on the oracle)"}
            elif args.workload == "boot":
                # bounded: one ordinary ciphertext's full bootstrap (a shared-a group is the
                # --impl reference arm's sample)
                v, cores, sample, _ = cpu_boot_sample(0)
                res["cpu_baseline"] = {"value": round(v, 6), "unit": "bootstraps/s", "cores": cores,
                                       "kind": "port", "sample": sample}
            else:
                v, cores = cpu_prim_chain()
                res["cpu_baseline"] = {"value": round(v, 4), "unit": "chains/s", "cores": cores, "kind": "port",
                                       "sample": "one config-1 chain on the CPU oracle (OpenMP over limbs)"}
        print(json.dumps(res))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
