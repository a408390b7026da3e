"""Benchmark of the EIP-7594 hot path: FK20 cell proofs and cell recovery at
256 blobs on one B200 (per rank), through libvkzg.so.

One step = vkzg_compute_proofs_batch over 256 blobs (252 seeded uniform blobs
plus 4 adversarial ones: all-zero, all r-1, one nonzero element, alternating
0/r-1) followed by vkzg_recover_cells_batch over 256 blobs whose surviving cell
sets are seeded-uniform in 64..127 cells, plus contiguous-half and every-other
patterns.  value = blobs per second through both entry points
(256 / step time), whole job over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The line also carries the same step through the public C ABI with host
buffers (e2e), the one-call-per-blob form, a served mixed stream with latency
percentiles, the phase-A roofline, the CPU oracle's rate and the clocks.

--impl reference times the CPU restatement of the reference's algorithm on the
host cores (the reference itself is Vulkan/GLSL and has no CPU path; no Vulkan
driver or software renderer is available here).  Under torchrun (N > 1) every
rank runs an independent replica (blobs are independent; no collective on the
data path) and rank 0 prints.
--profile-case [proofs|recovery] runs a small untimed case for ncu captures.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

R_MOD = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
BLOB = 131072
EXT = 262144
PROOFS = 6144
METRIC = "proof & recovery blobs/s at 256 blobs, bit-exact; served p50/p99 latency"

# Algorithmic work per blob of the reference algorithm (frozen per-unit figures):
# 1 Fp multiply = 4*12^2 = 576 32-bit IMAD, 1 Fr multiply = 4*8^2 = 256.
IMAD_FP, IMAD_FR = 576, 256
PHASE_A_FP_MUL_PER_BLOB = 2.87e6     # ~261k madd-2007-bl (11 Fp mul) per blob
PROOF_IMAD_PER_BLOB = 3.36e9         # 5.81M Fp mul + 74k Fr mul
RECOVERY_IMAD_PER_BLOB = 118e6       # 0.46M Fr mul (4 NTT-8192 + pointwise + batch division)
NOMINAL_IMAD_TPS = 148 * 64 * 1.965e9 / 1e12
# this library's Fp product (one Karatsuba level + word-serial reduction) and square
IMAD_FP_MUL_KS, IMAD_FP_SQR_KS = 516, 426
PHASE_A_TAIL = 10  # lists of at most this many points finish in Jacobian form


def phase_a_executed_products_per_output(d):
    """Fp products and squares plan 3's phase A executes per MSM output with a
    digit table of d windows (lists of 64 d points)."""
    m = 64 * d
    adds = 0
    while m > PHASE_A_TAIL:
        adds += m // 2
        m = (m + 1) // 2
    madds = max(m - 2, 0)
    return 6 * adds + 11 * madds + 16


def phase_a_executed_imad_per_output(d):
    """Multiply instructions plan 3's phase A executes per MSM output with d
    windows: affine additions (5 products + 1 square) in tree rounds down to
    lists of PHASE_A_TAIL points, then mixed additions (7 + 4) on two chains and
    one Jacobian addition (11 + 5)."""
    m = 64 * d
    adds = 0
    while m > PHASE_A_TAIL:
        adds += m // 2
        m = (m + 1) // 2
    madds = max(m - 2, 0)
    muls = 5 * adds + 7 * madds + 11
    sqrs = adds + 4 * madds + 5
    return muls * IMAD_FP_MUL_KS + sqrs * IMAD_FP_SQR_KS


def phase_a_dram_bytes(d, n_blobs):
    """DRAM bytes of one plan-3 phase-A pass over n_blobs with a digit table of
    d windows: the per-pair ncu dram__bytes_read + dram__bytes_write of the round
    kernels in a 16-blob, 9-bit-window capture, one kernel per capture
    (profiles/phase_a_dram_traffic_16blobs.md) -- 893 B per pair in round 1,
    which gathers digit-table points, 546 B in later rounds while a round's
    input lists exceed the 126 MB L2, 500 B once they fit -- applied to the
    table's exact pair counts, plus the digit recoding and the Jacobian tail
    (0.05 GB per 256 blobs).  For 20 windows at 256 blobs: 30.0 GB."""
    lists = 128 * n_blobs
    m = 64 * d
    total, first = 0.0, True
    while m > 10:
        pairs = lists * (m // 2)
        per = 893 if first else (546 if lists * m * 96 > 126e6 else 500)
        total += pairs * per
        first = False
        m = (m + 1) // 2
    return total + 0.05e9 * n_blobs / 256


# ------------------------------------------------------------------ inputs
def make_blobs(n, seed, adversarial=True):
    """n blobs: uniform field elements below r (rejection sampled); with `adversarial`
    the last 4 are all-zero, all r-1, one nonzero element, alternating 0 / r-1."""
    rng = np.random.default_rng(seed)
    r_be = np.frombuffer(R_MOD.to_bytes(32, "big"), np.uint8)
    out = np.empty((n, 4096, 32), np.uint8)
    nrand = max(0, n - 4) if adversarial else n
    flat = out[:nrand].reshape(-1, 32)
    filled = 0
    while filled < flat.shape[0]:
        cand = rng.integers(0, 256, size=(flat.shape[0] * 2, 32), dtype=np.uint8)
        cand[:, 0] &= 0x7F
        # lexicographic compare against r, big-endian
        diff = cand.astype(np.int16) - r_be.astype(np.int16)
        first = np.argmax(diff != 0, axis=1)
        lt = diff[np.arange(len(cand)), first] < 0
        good = cand[lt]
        take = min(len(good), flat.shape[0] - filled)
        flat[filled:filled + take] = good[:take]
        filled += take
    adv = []
    rm1 = (R_MOD - 1).to_bytes(32, "big")
    zero, one = bytes(32), (1).to_bytes(32, "big")
    adv.append(zero * 4096)
    adv.append(rm1 * 4096)
    adv.append(zero * 2047 + one + zero * 2048)
    adv.append(b"".join(zero if i % 2 == 0 else rm1 for i in range(4096)))
    for k in range(n - nrand):
        out[nrand + k] = np.frombuffer(adv[k], np.uint8).reshape(4096, 32)
    return out.reshape(n, BLOB)


def make_recovery(n, seed):
    """Cells (random canonical values, as the reference's bench/bench_common.h fills them)
    and uneven presence masks: 64..127 survivors, plus contiguous-half and every-other."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(0, 256, size=(n, 8192, 32), dtype=np.uint8)
    cells[:, :, 0] &= 0x3F
    present = np.zeros((n, 128), np.uint8)
    for b in range(n):
        if b % 16 == 0:
            present[b, :64] = 1
        elif b % 16 == 1:
            present[b, ::2] = 1
        else:
            present[b, rng.choice(128, int(rng.integers(64, 128)), replace=False)] = 1
    return cells.reshape(n, EXT), present


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while active; only
    samples taken after the first one has arrived (the sampler is running by
    then) count, so that they fall inside the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t_end = time.time() + 5.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        self.first = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:] or self.lines[-1:]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU legs
def cpu_rates(n_proofs, n_recover, seed=7, threads=None):
    """Oracle (CPU restatement of the reference algorithm) on `threads` host
    threads (all of them by default)."""
    from oracle import Oracle
    o = Oracle()
    with open(os.path.join(ROOT, "vkzg_b200", "data", "trusted_setup_g1_monomial.bin"), "rb") as f:
        tables = o.tables_from_setup(f.read())
    threads = threads or os.cpu_count() or 1
    # a sample of the 256-blob workload: its random part (the 4 adversarial blobs are ~free)
    blobs = make_blobs(n_proofs, seed, adversarial=False)
    t0 = time.perf_counter()
    rc, _ = o.compute_proofs(tables, blobs, threads)
    tp = time.perf_counter() - t0
    cells, present = make_recovery(n_recover, seed)
    t0 = time.perf_counter()
    rc2, _ = o.recover_cells(cells, present, threads)
    tr = time.perf_counter() - t0
    assert rc == 0 and rc2 == 0
    rp, rr = n_proofs / tp, n_recover / tr
    return {"proof_blobs_per_s": rp, "recovery_blobs_per_s": rr, "combined": 1.0 / (1.0 / rp + 1.0 / rr),
            "threads": threads, "seconds": tp + tr}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import build
    build()
    sample = args.ref_sample
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_rates(sample, sample, seed=100 + i)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.mean(x["combined"] for x in vals)
    threads = vals[0]["threads"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "blobs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (Fp/Fr Montgomery limbs)", "data": "synthetic",
        "config": {"workload": "proofs 256 blobs + uneven recovery 256 blobs", "blobs": 256,
                   "sample_per_step": sample},
        "proof_blobs_per_s": statistics.mean(x["proof_blobs_per_s"] for x in vals),
        "recovery_blobs_per_s": statistics.mean(x["recovery_blobs_per_s"] for x in vals),
        "cpu_baseline": {"value": v, "unit": "blobs/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} proof blobs + {sample} recovery blobs per step on {threads} threads "
                                   "(the reference's Vulkan code cannot run here)"},
        "e2e": {"value": v, "unit": "blobs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def plain_rates(prover, h_blobs, h_cells, h_present, sample):
    """The plain form: one blocking C-ABI call per blob (pinned host buffers)."""
    import torch
    out_p = torch.empty(PROOFS, dtype=torch.uint8).pin_memory()
    out_c = torch.empty(EXT, dtype=torch.uint8).pin_memory()
    for k in range(2):  # warm the size-1 class
        prover.compute_proofs_raw(out_p.data_ptr(), h_blobs.data_ptr() + k * BLOB, 1)
        prover.recover_cells_raw(out_c.data_ptr(), h_cells.data_ptr() + k * EXT, h_present.data_ptr() + k * 128, 1)
    t0 = time.perf_counter()
    for k in range(sample):
        assert prover.compute_proofs_raw(out_p.data_ptr(), h_blobs.data_ptr() + k * BLOB, 1) == 0
    tp = time.perf_counter() - t0
    t0 = time.perf_counter()
    for k in range(sample):
        assert prover.recover_cells_raw(out_c.data_ptr(), h_cells.data_ptr() + k * EXT,
                                        h_present.data_ptr() + k * 128, 1) == 0
    tr = time.perf_counter() - t0
    rp, rr = sample / tp, sample / tr
    return {"value": 1.0 / (1.0 / rp + 1.0 / rr), "unit": "blobs/s", "proof_blobs_per_s": rp,
            "recovery_blobs_per_s": rr, "sample": f"{sample} proof + {sample} recovery calls of 1 blob"}


def serve_sweep(want_proofs, want_cells, h_blobs, h_cells, h_present, n_pool, capacity, fractions, seconds,
                seed=99, args_warm=0.6, batch=128, lanes=3, hbm_budget=8 << 30, table_budget=0):
    """Served mixed stream (continuous batching, vkzg_b200_server_*): Poisson arrivals,
    request sizes geometric with mean 6 in 1..64 blobs, 70% proof requests and 30%
    recovery requests (64..127 cells present).  One segment per offered load
    (fraction x capacity blobs/s), after an unreported warm-up segment; latency is
    submit-to-completion inside the server.  Outputs land in reused pinned rings, as
    a serving caller's would, not in fresh pageable arrays (whose first-touch page
    faults would be charged to the lanes).  Every served request's output is
    compared with the direct call's output for the same blobs (want_proofs /
    want_cells, one row per pool blob) as soon as it completes."""
    import queue
    import torch
    import vkzg_b200
    rng = np.random.default_rng(seed)
    results = []
    checked = [0]
    mismatches = []
    warming = True
    # the rings wrap after ~0.5 s of output at the highest load, far beyond any request's latency
    ring = {"proofs": torch.empty(64 << 20, dtype=torch.uint8).pin_memory().numpy(),
            "recovery": torch.empty(768 << 20, dtype=torch.uint8).pin_memory().numpy()}
    ring_off = {"proofs": 0, "recovery": 0}

    def ring_take(kind, size):
        off = ring_off[kind]
        if off + size > len(ring[kind]):
            off = 0
        ring_off[kind] = off + size
        return ring[kind][off:off + size]

    t_setup = time.perf_counter()
    with vkzg_b200.Server(max_blobs_per_batch=batch, lanes=lanes, hbm_budget_bytes=hbm_budget,
                          table_budget_bytes=table_budget) as srv:
        setup_s = time.perf_counter() - t_setup
        charges = srv.stats()
        # warm-up segment (not reported): the lanes capture the pipelines of the batch
        # sizes they meet, so the measured segments mostly replay captured graphs
        fractions = [args_warm] + list(fractions)
        for frac in fractions:
            offered = frac * capacity
            req_rate = offered / 6.0
            tickets = queue.Queue()
            statuses = []

            def waiter():
                while True:
                    item = tickets.get()
                    if item is None:
                        return
                    statuses.append(srv.wait(item[0]))
                    kind, first, n, out = item[1]
                    want = want_proofs if kind == "proofs" else want_cells
                    if not np.array_equal(out.reshape(n, -1), want[first:first + n]):
                        mismatches.append((kind, first, n))
                    checked[0] += 1

            th = threading.Thread(target=waiter, daemon=True)
            th.start()
            srv.stats(reset=True)
            t_start = time.perf_counter()
            t_next = t_start
            while True:
                t_next += rng.exponential(1.0 / req_rate)
                if t_next - t_start > seconds:
                    break
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                n = int(min(64, rng.geometric(1.0 / 6.0)))
                first = int(rng.integers(0, n_pool - n + 1))
                if rng.random() < 0.7:
                    out = ring_take("proofs", n * PROOFS)
                    t = srv.submit_proofs(out, h_blobs.data_ptr() + first * BLOB, n)
                    tickets.put((t, ("proofs", first, n, out)))
                else:
                    out = ring_take("recovery", n * EXT)
                    t = srv.submit_recovery(out, h_cells.data_ptr() + first * EXT,
                                            h_present.data_ptr() + first * 128, n)
                    tickets.put((t, ("recovery", first, n, out)))
            tickets.put(None)
            th.join()
            st = srv.stats()
            assert all(x == 0 for x in statuses), "served request failed"
            if len(results) == 0 and warming:
                warming = False
                results.append(None)
                continue
            results.append({"offered_blobs_per_s": round(offered, 1),
                            "served_blobs_per_s": round(st["blobs"] / st["seconds"], 1),
                            "seconds": round(st["seconds"], 1),
                            "requests": int(st["requests"]), "blobs": int(st["blobs"]),
                            "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                            "p999_ms": round(st["p999_ms"], 3), "max_ms": round(st["max_ms"], 3),
                            "admission_deferrals": int(st["deferrals"]),
                            "peak_in_flight_bytes": int(st["peak_in_flight_bytes"])})
    results = [r for r in results if r is not None]
    assert not mismatches, f"served requests differ from direct calls: {mismatches[:4]}"
    info = {"setup_s": round(setup_s, 2), "hbm_budget_bytes": hbm_budget, "lanes": lanes, "max_blobs_per_batch": batch,
            "resident_bytes": int(charges["resident_bytes"]),
            "proof_bytes_per_blob": int(charges["proof_bytes_per_blob"]),
            "recover_bytes_per_blob": int(charges["recover_bytes_per_blob"]),
            "bit_exact_checked_requests": checked[0]}
    return results, info


def run_ours(args, rank, world, local_rank):
    import tempfile
    import torch
    import vkzg_b200
    from vkzg_b200 import replicas

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.blobs
    # the autotuner's decisions are shared with the serving lanes' provers through this file
    tune_dir = tempfile.mkdtemp(prefix="vkzg_tune_")
    os.environ["VKZG_TUNE_CACHE"] = os.path.join(tune_dir, "plans.txt")
    # digit-table budget: opted in above the library's 20 GiB default, so the
    # tuner may pick tables up to 18 windows (141.7 GB of the device's 179 GiB)
    os.environ.setdefault("VKZG_COMB_BUDGET_GB", str(args.table_budget_gb))
    table_budget = int(float(os.environ["VKZG_COMB_BUDGET_GB"]) * (1 << 30))
    prover = vkzg_b200.Prover(max_batch_size=n)

    blobs_np = make_blobs(n, 1234 + rank)
    cells_np, present_np = make_recovery(n, 4321 + rank)
    d_blobs = torch.from_numpy(blobs_np).to(dev)
    d_cells = torch.from_numpy(cells_np).to(dev)
    d_present = torch.from_numpy(present_np).to(dev)
    d_proofs = torch.empty(n * PROOFS, dtype=torch.uint8, device=dev)
    d_out = torch.empty(n * EXT, dtype=torch.uint8, device=dev)
    d_err = torch.zeros(2 * n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def device_step():
        rc = prover.compute_proofs_device(d_proofs.data_ptr(), d_blobs.data_ptr(), d_err.data_ptr(), n, sp)
        rc |= prover.recover_cells_device(d_out.data_ptr(), d_cells.data_ptr(), d_present.data_ptr(),
                                          d_err.data_ptr() + 4 * n, n, sp)
        assert rc == 0

    # ---- warm-up: the autotuner times the proof plans of every size class up to n
    tuning = prover.autotune(n)
    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize()
    assert int(d_err.count_nonzero()) == 0

    # ---- device-resident arm: inputs in HBM, CUDA events on the launching stream
    step_ms, proof_ms = [], []
    replicas.barrier(dev)
    torch.cuda.synchronize()
    launches0 = vkzg_b200.kernel_launches()
    with ClockSampler(local_rank) as clocks:
        for _ in range(args.steps):
            flush.fill_(1)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            prover.compute_proofs_device(d_proofs.data_ptr(), d_blobs.data_ptr(), d_err.data_ptr(), n, sp)
            e1.record(stream)
            prover.recover_cells_device(d_out.data_ptr(), d_cells.data_ptr(), d_present.data_ptr(),
                                        d_err.data_ptr() + 4 * n, n, sp)
            e2.record(stream)
            e2.synchronize()
            step_ms.append(e0.elapsed_time(e2))
            proof_ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
    launches = vkzg_b200.kernel_launches() - launches0
    total_ms = replicas.max_over_ranks(sum(step_ms), dev)
    value = world * n * args.steps / (total_ms / 1e3)
    assert int(d_err.count_nonzero()) == 0

    # ---- the timed outputs checked: every proof against a plan-0 pass (serial
    # Jacobian buckets: an independent kernel path), a seeded sample of proofs
    # and recovered blobs against the CPU oracle
    got_proofs = d_proofs.cpu().numpy().reshape(n, PROOFS)
    got_cells = d_out.cpu().numpy().reshape(n, EXT)
    saved_plan = os.environ.get("VKZG_PLAN")
    os.environ["VKZG_PLAN"] = "0"
    with vkzg_b200.Prover(max_batch_size=n) as plain0:
        plan0 = np.zeros(n * PROOFS, np.uint8)
        assert plain0.compute_proofs_raw(plan0, blobs_np, n) == 0
    if saved_plan is None:
        del os.environ["VKZG_PLAN"]
    else:
        os.environ["VKZG_PLAN"] = saved_plan
    assert np.array_equal(plan0.reshape(n, PROOFS), got_proofs), "timed proofs differ from the plan-0 pass"
    verified = {"proofs_vs_plan0": n}
    if not args.no_cpu:
        from oracle import Oracle, build
        build()
        orc = Oracle()
        with open(os.path.join(ROOT, "vkzg_b200", "data", "trusted_setup_g1_monomial.bin"), "rb") as f:
            orc_tables = orc.tables_from_setup(f.read())
        pick = np.random.default_rng(2024 + rank).choice(n, 4, replace=False)
        pick_p = sorted(set(pick.tolist()) | {n - 4, n - 1})  # two of the adversarial blobs too
        rc, want = orc.compute_proofs(orc_tables, np.ascontiguousarray(blobs_np[pick_p]))
        assert rc == 0 and np.array_equal(want.reshape(-1, PROOFS), got_proofs[pick_p]), "proofs differ from the oracle"
        pick_r = sorted(np.random.default_rng(4048 + rank).choice(n, 8, replace=False).tolist())
        rc, want = orc.recover_cells(np.ascontiguousarray(cells_np[pick_r]), np.ascontiguousarray(present_np[pick_r]))
        assert rc == 0 and np.array_equal(want.reshape(-1, EXT), got_cells[pick_r]), "recovery differs from the oracle"
        verified.update({"proofs_vs_oracle": len(pick_p), "recovered_blobs_vs_oracle": len(pick_r)})

    # ---- recovery of 16 blobs keeping exactly 64 of 128 cells,
    # seeded uniform subsets; device-resident and through the C ABI (pinned buffers)
    c1 = None
    if n >= 16:
        rng1 = np.random.default_rng(0x7594)
        c1_present = np.zeros((16, 128), np.uint8)
        for b in range(16):
            c1_present[b, rng1.choice(128, 64, replace=False)] = 1
        c1_cells = np.ascontiguousarray(cells_np[:16])
        d_c1_cells = torch.from_numpy(c1_cells).to(dev)
        d_c1_present = torch.from_numpy(c1_present).to(dev)
        for _ in range(3):
            prover.recover_cells_device(d_out.data_ptr(), d_c1_cells.data_ptr(), d_c1_present.data_ptr(),
                                        d_err.data_ptr(), 16, sp)
        c1_ms = []
        for _ in range(20):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prover.recover_cells_device(d_out.data_ptr(), d_c1_cells.data_ptr(), d_c1_present.data_ptr(),
                                        d_err.data_ptr(), 16, sp)
            e1.record(stream)
            e1.synchronize()
            c1_ms.append(e0.elapsed_time(e1))
        h_c1_cells = torch.from_numpy(c1_cells).pin_memory()
        h_c1_present = torch.from_numpy(c1_present).pin_memory()
        h_c1_out = torch.empty(16 * EXT, dtype=torch.uint8).pin_memory()
        c1_e2e = []
        for i in range(23):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            assert prover.recover_cells_raw(h_c1_out.data_ptr(), h_c1_cells.data_ptr(), h_c1_present.data_ptr(), 16) == 0
            if i >= 3:
                c1_e2e.append(time.perf_counter() - t0)
        if not args.no_cpu:
            rc, want = orc.recover_cells(c1_cells[:4], c1_present[:4])
            assert rc == 0 and np.array_equal(want.reshape(-1), h_c1_out.numpy()[:4 * EXT]), "C1 differs from the oracle"
        c1 = {"blobs": 16, "present_per_blob": 64, "device_blobs_per_s": 16 / (statistics.median(c1_ms) / 1e3),
              "e2e_blobs_per_s": 16 / statistics.median(c1_e2e)}

    # ---- the same proof step in its persistent form ($VKZG_COOP=1: each phase's
    # grid-wide rounds in one cooperative launch with grid barriers), timed the
    # same way on its own prover (the digit table is shared)
    persistent = None
    os.environ["VKZG_COOP"] = "1"
    try:
        with vkzg_b200.Prover(max_batch_size=n) as pc:
            pc.autotune(n)
            d_proofs_c = torch.empty_like(d_proofs)
            for _ in range(args.warmup):
                pc.compute_proofs_device(d_proofs_c.data_ptr(), d_blobs.data_ptr(), d_err.data_ptr(), n, sp)
            torch.cuda.synchronize()
            l0 = vkzg_b200.kernel_launches()
            c_ms = []
            for _ in range(args.steps):
                flush.fill_(1)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                pc.compute_proofs_device(d_proofs_c.data_ptr(), d_blobs.data_ptr(), d_err.data_ptr(), n, sp)
                e1.record(stream)
                e1.synchronize()
                c_ms.append(e0.elapsed_time(e1))
            c_launches = vkzg_b200.kernel_launches() - l0
            assert int(d_err[:n].count_nonzero()) == 0
            assert torch.equal(d_proofs_c, d_proofs), "persistent form's proofs differ"
            persistent = {"proof_ms": statistics.mean(c_ms), "graph_ms": statistics.mean(proof_ms),
                          "launches_per_step": c_launches / args.steps,
                          "graph_launches_per_step": launches / args.steps - 1}
    finally:
        del os.environ["VKZG_COOP"]

    # ---- per-stage breakdown from untimed steps with stage events (the timed steps
    # above replay the captured pipeline; these launch it stage by stage)
    prover.set_stage_timing(True)
    stages_acc, phase_a_ms = {}, []
    for _ in range(2):
        flush.fill_(1)
        prover.compute_proofs_device(d_proofs.data_ptr(), d_blobs.data_ptr(), d_err.data_ptr(), n, sp)
        torch.cuda.synchronize()
        st = prover.last_stage_times(False)
        for k, v in st.items():
            stages_acc[k] = stages_acc.get(k, 0.0) + v / 2
        phase_a_ms.append(st["phase_a"])
    prover.set_stage_timing(False)

    # ---- end-to-end arm: public C ABI with pinned host buffers, copies in the timed region
    h_blobs = torch.from_numpy(blobs_np).pin_memory()
    h_cells = torch.from_numpy(cells_np).pin_memory()
    h_present = torch.from_numpy(present_np).pin_memory()
    h_proofs = torch.empty(n * PROOFS, dtype=torch.uint8).pin_memory()
    h_out = torch.empty(n * EXT, dtype=torch.uint8).pin_memory()

    def e2e_step():
        t0 = time.perf_counter()
        rc = prover.compute_proofs_raw(h_proofs.data_ptr(), h_blobs.data_ptr(), n)
        t1 = time.perf_counter()
        rc2 = prover.recover_cells_raw(h_out.data_ptr(), h_cells.data_ptr(), h_present.data_ptr(), n)
        assert rc == 0 and rc2 == 0
        return t1 - t0, time.perf_counter() - t1

    for _ in range(max(1, args.warmup)):
        e2e_step()
    replicas.barrier(dev)
    torch.cuda.synchronize()
    e2e_p, e2e_r = [], []
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        tp, tr = e2e_step()
        e2e_p.append(tp)
        e2e_r.append(tr)
    e2e_total = replicas.max_over_ranks(sum(e2e_p) + sum(e2e_r), dev)
    e2e_value = world * n * args.steps / e2e_total
    e2e_proof_rate = n * args.steps / sum(e2e_p)
    e2e_rec_rate = n * args.steps / sum(e2e_r)

    # ---- the next rows through the C ABI (host buffers, copies in the timed
    # region): cells from blobs, cells + proofs from one upload, recovered
    # cells + the proofs of the recovered blobs; median of 3 calls each
    next_rows = None
    if not args.no_next:
        h_cells_out = torch.empty(n * EXT, dtype=torch.uint8).pin_memory()
        calls = {
            "cells_blobs_per_s": lambda: prover.compute_cells_raw(h_cells_out.data_ptr(), h_blobs.data_ptr(), n),
            "cells_and_proofs_blobs_per_s": lambda: prover.compute_cells_and_proofs_raw(
                h_cells_out.data_ptr(), h_proofs.data_ptr(), h_blobs.data_ptr(), n),
            "recovered_cells_and_proofs_blobs_per_s": lambda: prover.recover_cells_and_proofs_raw(
                h_cells_out.data_ptr(), h_proofs.data_ptr(), h_cells.data_ptr(), h_present.data_ptr(), n),
        }
        next_rows = {"blobs": n, "timing": "per GPU; wall clock around each synchronous call, L2 flushed before each"}
        for key, call in calls.items():
            assert call() == 0
            ts = []
            for _ in range(3):
                flush.fill_(1)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                assert call() == 0
                ts.append(time.perf_counter() - t0)
            next_rows[key] = n / statistics.median(ts)

    # ---- the plain form (one call per blob) and the served form, one replica each
    plain = plain_rates(prover, h_blobs, h_cells, h_present, args.plain_sample) if not args.no_plain else None
    serving = None
    if args.serve_seconds > 0:
        capacity = 1.0 / (0.7 / e2e_proof_rate + 0.3 / e2e_rec_rate)
        fractions = [float(x) for x in args.serve_loads.split(",")]
        want_cells = np.frombuffer(prover.recover_cells_batch(cells_np.tobytes(), present_np.tobytes(), n),
                                   np.uint8).reshape(n, EXT)
        sweep, info = serve_sweep(got_proofs, want_cells, h_blobs, h_cells, h_present, n, capacity, fractions,
                                  args.serve_seconds, batch=args.serve_batch, lanes=args.serve_lanes,
                                  hbm_budget=64 << 30, table_budget=table_budget)
        serving = {"sweep": sweep, **info, "seconds_per_load": args.serve_seconds, "outputs": "reused pinned rings",
                   "mix": "Poisson arrivals; 1-64 blobs per request (geometric, mean 6); 70% proofs, "
                          "30% recovery with 64-127 cells present"}
        if args.c4_seconds > 0:
            # BASELINE config 4 as stated: 60 s at the top offered load with the
            # admission budget at 8 GiB of working set, which binds (3 lanes x 128
            # blobs of proof work in flight would need more)
            top = [max(fractions)]
            c4, c4_info = serve_sweep(got_proofs, want_cells, h_blobs, h_cells, h_present, n, capacity, top,
                                      args.c4_seconds, seed=4242, batch=args.serve_batch, lanes=args.serve_lanes,
                                      hbm_budget=8 << 30, table_budget=table_budget)
            serving["c4_8gib_budget"] = {**c4[0], **c4_info, "seconds_per_load": args.c4_seconds}
    replicas.barrier(dev)
    if rank != 0:
        return

    # ---- roofline of the dominant kernel (phase A), integer-multiply bound
    imad_peak = vkzg_b200.microbench(0)
    product_rate = vkzg_b200.microbench(4)  # this library's Fp product alone, G/s
    pa_ms = statistics.mean(phase_a_ms)
    reference_work = PHASE_A_FP_MUL_PER_BLOB * IMAD_FP * n / (pa_ms / 1e3) / 1e12
    digit = prover.digit_table()
    plan = tuning.get(n, (None,))[0] if n in tuning else None
    executed = products = None
    if plan == 3 and digit:
        executed = 128 * phase_a_executed_imad_per_output(digit[0]) * n / (pa_ms / 1e3) / 1e12
        products = 128 * phase_a_executed_products_per_output(digit[0]) * n / (pa_ms / 1e3) / 1e9
    stages = dict(stages_acc)
    p_ms = statistics.mean(proof_ms)
    rec_ms = statistics.mean(step_ms) - p_ms

    cpu = None
    if world == 1 and not args.no_cpu:
        from oracle import build
        build()
        c = cpu_rates(args.cpu_sample, args.cpu_sample)
        one = cpu_rates(2, 4, threads=1)
        # all host threads at batches of 1 and 16 blobs beside the main sample
        # (blobs run in parallel, one thread each, so a batch of 1 uses one)
        small = {k: cpu_rates(k, k, seed=11 + k) for k in (1, 16)}
        cpu = {"value": c["combined"], "unit": "blobs/s", "cores": c["threads"], "kind": "port",
               "sample": f"{args.cpu_sample} proof blobs + {args.cpu_sample} recovery blobs of the same workload "
                         f"on {c['threads']} host threads ({c['seconds']:.1f} s)",
               "proof_blobs_per_s": c["proof_blobs_per_s"], "recovery_blobs_per_s": c["recovery_blobs_per_s"],
               "single_core": {"proof_blobs_per_s": one["proof_blobs_per_s"],
                               "recovery_blobs_per_s": one["recovery_blobs_per_s"],
                               "sample": "2 proof blobs + 4 recovery blobs on 1 thread"},
               "all_cores_by_batch": {str(k): {"proof_blobs_per_s": r["proof_blobs_per_s"],
                                               "recovery_blobs_per_s": r["recovery_blobs_per_s"]}
                                      for k, r in [(1, small[1]), (16, small[16]), (args.cpu_sample, c)]}}

    line = {
        "metric": METRIC, "value": value, "unit": "blobs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(step_ms), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (Fp/Fr Montgomery limbs)",
        "data": "synthetic (seeded uniform Fr blobs + 4 adversarial; seeded uneven survivor sets)",
        "config": {"workload": "proofs 256 blobs + uneven recovery 256 blobs per GPU", "blobs": n,
                   "parallelism": f"replicas x{world}", "l2": "flushed between timed steps (256 MB write)",
                   "setup": "mainnet G1 monomial, FK20 tables generated on the GPU",
                   "tuned_plans": {str(k): v[0] for k, v in tuning.items()}},
        "proof_blobs_per_s": world * n / (p_ms / 1e3),
        "recovery_blobs_per_s": world * n / (rec_ms / 1e3) if rec_ms > 0 else None,
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "e2e": {"value": e2e_value, "unit": "blobs/s",
                "h2d_bytes_per_step": n * BLOB + n * EXT + n * 128,
                "d2h_bytes_per_step": n * PROOFS + n * EXT,
                "proof_blobs_per_s": world * e2e_proof_rate, "recovery_blobs_per_s": world * e2e_rec_rate},
        "next_rows": next_rows,
        "plain_per_blob": plain,
        "batched_over_plain": (e2e_value / world) / plain["value"] if plain else None,
        "serving": serving,
        "roofline": {"kernel": "phase A (plan %s: %s)" % (plan, "k_flat_* rounds over the digit table" if plan == 3
                                                            else "k_phase_a_affine + k_reduce_hier"),
                     "bound": "int", "achieved": executed, "peak": imad_peak, "unit": "TIMAD/s",
                     "frac": executed / imad_peak if executed else None,
                     "peak_source": "measured in-process (vkzg_b200_microbench(0): mad.lo.u32 issue rate; "
                                    "MEASURED_PEAKS.json has no integer figure); nominal 148 SM x 64/clk x "
                                    f"1.965 GHz = {NOMINAL_IMAD_TPS:.1f}",
                     "algorithmic": "multiply instructions phase A executes: per MSM output 64 D - 1 (D windows) "
                                    "digit-table points summed by affine additions (5 products + 1 square, "
                                    "516 / 426 multiply instructions each) down to lists of 10, then mixed "
                                    "Jacobian additions",
                     "products_g_per_s": products, "product_rate_alone_g_per_s": product_rate,
                     "frac_of_product_rate": products / product_rate if products else None,
                     "reference_algorithm_tera_imad_per_s": reference_work,
                     "work_saved": reference_work / executed if executed else None,
                     "traffic": phase_a_dram_bytes(digit[0], n) if plan == 3 and digit else None,
                     "traffic_unit": "DRAM bytes per phase-A pass over the batch (ncu dram__bytes_read + write "
                                     "per pair from a 16-blob 9-bit-window capture, one kernel each, applied "
                                     "to this table's pair counts)"},
        "digit_table": {"windows": digit[0], "window_bits": vkzg_b200.comb_windows(digit[0]),
                        "build_ms": round(digit[1], 1), "bytes": digit[2],
                        "budget_bytes": table_budget,
                        "window_trials": [{"windows": d, "bytes": b, "build_ms": round(bm, 1), "proof_ms": round(t, 3)}
                                          for d, b, bm, t in prover.window_trials(n)]} if digit else None,
        "device_bytes": prover.device_bytes(),
        "persistent_form": persistent,
        "verified": verified,
        "c1_recovery_16_blobs": c1,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--blobs", type=int, default=256)
    ap.add_argument("--cpu-sample", type=int, default=256)
    ap.add_argument("--ref-sample", type=int, default=32)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-next", action="store_true", help="skip the cells / cells+proofs / recovered+proofs rates")
    ap.add_argument("--profile-case", nargs="?", const="proofs", choices=["proofs", "recovery", "cells"],
                    help="small untimed case for ncu captures")
    ap.add_argument("--plain-sample", type=int, default=16)
    ap.add_argument("--serve-seconds", type=float, default=6.0, help="per offered load; 0 skips serving")
    ap.add_argument("--serve-loads", default="0.3,0.6,0.9", help="offered loads as fractions of batched capacity")
    ap.add_argument("--serve-batch", type=int, default=128, help="the server's max_blobs_per_batch")
    ap.add_argument("--serve-lanes", type=int, default=3, help="the server's lanes")
    ap.add_argument("--c4-seconds", type=float, default=60.0,
                    help="BASELINE config 4 at the top load with an 8 GiB budget; 0 skips it")
    ap.add_argument("--table-budget-gb", type=float, default=136.0,
                    help="digit-table budget (GiB) unless $VKZG_COMB_BUDGET_GB is set")
    args = ap.parse_args()

    if args.profile_case:
        # a small fixed case for ncu captures: --steps calls on --blobs blobs
        # (proof plan from $VKZG_PLAN), nothing timed
        import numpy as np
        import vkzg_b200
        prover = vkzg_b200.Prover(max_batch_size=args.blobs)
        if args.profile_case == "proofs":
            blobs = make_blobs(args.blobs, 5, adversarial=False)
            out = np.zeros(args.blobs * PROOFS, np.uint8)
            for _ in range(args.steps):
                assert prover.compute_proofs_raw(out, blobs, args.blobs) == 0
        elif args.profile_case == "cells":
            blobs = make_blobs(args.blobs, 5, adversarial=False)
            out = np.zeros(args.blobs * EXT, np.uint8)
            for _ in range(args.steps):
                assert prover.compute_cells_raw(out, blobs, args.blobs) == 0
        else:
            # device buffers: one launch of all the blobs (host buffers of 16
            # blobs or more would be staged in parts)
            import torch
            cells, present = make_recovery(args.blobs, 6)
            d_cells = torch.from_numpy(cells).cuda()
            d_present = torch.from_numpy(present).cuda()
            d_out = torch.empty(args.blobs * EXT, dtype=torch.uint8, device="cuda")
            d_err = torch.zeros(args.blobs, dtype=torch.int32, device="cuda")
            sp = torch.cuda.current_stream().cuda_stream
            for _ in range(args.steps):
                assert prover.recover_cells_device(d_out.data_ptr(), d_cells.data_ptr(), d_present.data_ptr(),
                                                   d_err.data_ptr(), args.blobs, sp) == 0
            torch.cuda.synchronize()
            assert int(d_err.count_nonzero()) == 0
        print(json.dumps({"profile_case": args.profile_case, "blobs": args.blobs, "steps": args.steps,
                          "launches": vkzg_b200.kernel_launches()}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
