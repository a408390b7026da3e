"""Benchmark of the EIP-7594 hot path: FK20 cell proofs and cell recovery at
256 blobs on one B200 (per rank), through libvkzg.so.

One step = vkzg_compute_proofs_batch over 256 blobs (252 seeded uniform blobs
plus 4 adversarial ones: all-zero, all r-1, one nonzero element, alternating
0/r-1) followed by vkzg_recover_cells_batch over 256 blobs whose surviving cell
sets are seeded-uniform in 64..127 cells, plus contiguous-half and every-other
patterns.  value = blobs per second through both entry points
(256 / step time), whole job over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU restatement of the reference's algorithm on the
host cores (the reference itself is Vulkan/GLSL and cannot run on this machine;
see DESIGN.md).  Under torchrun (N > 1) every rank runs an independent replica
(blobs are independent; no collective on the data path) and rank 0 prints.
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
METRIC = "proof & recovery blobs/s at 256 blobs, bit-exact"

# Algorithmic work per blob of the reference algorithm (frozen per-unit figures):
# 1 Fp multiply = 4*12^2 = 576 32-bit IMAD, 1 Fr multiply = 4*8^2 = 256.
IMAD_FP, IMAD_FR = 576, 256
PHASE_A_FP_MUL_PER_BLOB = 2.87e6     # ~261k madd-2007-bl (11 Fp mul) per blob
PROOF_IMAD_PER_BLOB = 3.36e9         # 5.81M Fp mul + 74k Fr mul
RECOVERY_IMAD_PER_BLOB = 118e6       # 0.46M Fr mul (4 NTT-8192 + pointwise + batch division)
NOMINAL_IMAD_TPS = 148 * 64 * 1.965e9 / 1e12


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
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while active."""

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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
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
        for ln in self.lines:
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
def cpu_rates(n_proofs, n_recover, seed=7):
    """Oracle (CPU restatement of the reference algorithm) on all host threads."""
    from oracle import Oracle
    o = Oracle()
    with open(os.path.join(ROOT, "vkzg_b200", "data", "trusted_setup_g1_monomial.bin"), "rb") as f:
        tables = o.tables_from_setup(f.read())
    threads = os.cpu_count() or 1
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
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import vkzg_b200

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.blobs
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

    # ---- device-resident arm: inputs in HBM, CUDA events on the launching stream
    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize()
    assert int(d_err[:n - 4].count_nonzero()) == 0
    prover.set_stage_timing(True)
    step_ms, phase_a_ms, stages_acc = [], [], {}
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
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
            st = prover.last_stage_times(False)
            for k, v in st.items():
                stages_acc[k] = stages_acc.get(k, 0.0) + v
            phase_a_ms.append(st["phase_a"])
            step_ms.append(e0.elapsed_time(e2))
        torch.cuda.synchronize()
    prover.set_stage_timing(False)
    total_ms = sum(step_ms)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * n * args.steps / (total_ms / 1e3)

    # ---- end-to-end arm: public C ABI with pinned host buffers, copies in the timed region
    h_blobs = torch.from_numpy(blobs_np).pin_memory()
    h_cells = torch.from_numpy(cells_np).pin_memory()
    h_present = torch.from_numpy(present_np).pin_memory()
    h_proofs = torch.empty(n * PROOFS, dtype=torch.uint8).pin_memory()
    h_out = torch.empty(n * EXT, dtype=torch.uint8).pin_memory()

    def e2e_step():
        rc = prover.compute_proofs_raw(h_proofs.data_ptr(), h_blobs.data_ptr(), n)
        rc2 = prover.recover_cells_raw(h_out.data_ptr(), h_cells.data_ptr(), h_present.data_ptr(), n)
        assert rc == 0 and rc2 == 0

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_s = []
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        torch.cuda.synchronize()
        e2e_s.append(time.perf_counter() - t0)
    te = torch.tensor([sum(e2e_s)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * n * args.steps / float(te.item())

    if rank != 0:
        return

    # ---- roofline of the dominant kernel (phase A), integer-multiply bound
    imad_peak = vkzg_b200.microbench(0)
    pa_ms = statistics.mean(phase_a_ms)
    achieved = PHASE_A_FP_MUL_PER_BLOB * IMAD_FP * n / (pa_ms / 1e3) / 1e12
    stages = {k: v / args.steps for k, v in stages_acc.items()}
    proof_ms = sum(stages.values())
    rec_ms = statistics.mean(step_ms) - proof_ms

    cpu = None
    if world == 1 and not args.no_cpu:
        from oracle import build
        build()
        c = cpu_rates(args.cpu_sample, args.cpu_sample)
        cpu = {"value": c["combined"], "unit": "blobs/s", "cores": c["threads"], "kind": "port",
               "sample": f"{args.cpu_sample} proof blobs + {args.cpu_sample} recovery blobs of the same workload "
                         f"on {c['threads']} host threads ({c['seconds']:.1f} s)",
               "proof_blobs_per_s": c["proof_blobs_per_s"], "recovery_blobs_per_s": c["recovery_blobs_per_s"]}

    launches_per_step = 10 * ((n + prover_cap(n) - 1) // prover_cap(n)) + 2 * ((n + prover_cap(n) - 1) // prover_cap(n))
    line = {
        "metric": METRIC, "value": value, "unit": "blobs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(step_ms), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (Fp/Fr Montgomery limbs)",
        "data": "synthetic (seeded uniform Fr blobs + 4 adversarial; seeded uneven survivor sets)",
        "config": {"workload": "proofs 256 blobs + uneven recovery 256 blobs per GPU", "blobs": n,
                   "parallelism": f"replicas x{world}", "l2": "flushed between timed steps (256 MB write)",
                   "setup": "mainnet G1 monomial, FK20 tables generated on the GPU"},
        "proof_blobs_per_s": world * n / (proof_ms / 1e3),
        "recovery_blobs_per_s": world * n / (rec_ms / 1e3) if rec_ms > 0 else None,
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "e2e": {"value": e2e_value, "unit": "blobs/s",
                "h2d_bytes_per_step": n * BLOB + n * EXT + n * 128,
                "d2h_bytes_per_step": n * PROOFS + n * EXT + 4 * n},
        "roofline": {"kernel": "k_phase_a", "bound": "int", "achieved": achieved, "peak": imad_peak,
                     "unit": "TIMAD/s", "frac": achieved / imad_peak,
                     "peak_source": "measured in-process (vkzg_b200_microbench IMAD probe); "
                                    f"nominal 148 SM x 64/clk x 1.965 GHz = {NOMINAL_IMAD_TPS:.1f}",
                     "algorithmic": f"{PHASE_A_FP_MUL_PER_BLOB:.3g} Fp mul x 576 IMAD per blob x {n} blobs",
                     "traffic": None},
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * args.steps,
    }
    print(json.dumps(line), flush=True)


def prover_cap(n):
    return n


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--blobs", type=int, default=256)
    ap.add_argument("--cpu-sample", type=int, default=32)
    ap.add_argument("--ref-sample", type=int, default=8)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()

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
