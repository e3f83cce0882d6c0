"""Benchmark: residue-form Gram accumulation at 832 bits on one B200 (per GPU).

Workload (one "step"): Q = sum_b B_b^T B_b for 400 blocks B_b of m_b x 274 (m_b ~ U[20,120], numpy
seed 0) of 832-bit MPF entries (L = 26 limbs; mantissas of NB = 830 bits, random sign, exponents
U[-8, 8]), streamed as 4 chunks of 100 blocks through sdpvibe_b200.mpf.GramAcc(274, 26) with one CRT
-- the reference's GramAcc (sdpvibe/mpf.py:536-630) on its Gram configuration.

Metric: residue-GEMM INT8 TOPS, counted the reference's way: n_mod (128 moduli at L+1 = 27 limbs)
x 4 digit products x 2 ops x N(N+1)/2 x R per step, divided by the step time.  Also reported as
mp-MAC/s.  `value` times the step with inputs resident in HBM; `e2e` times the same step through the
public API with pinned host inputs copied in and Q copied out inside the timed region.

The line also carries `sdp_solver`: the metric's other half, SDPB iterations (s/iteration) of the 768-bit
Ising-structured SDP (300 blocks, N = 1000, L = 26) on the same GPU (`--workload solver` prints it as
its own line; `--workload cholsolve` measures the batched Cholesky + solve configuration).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}] [--workload ...]
Under torchrun each rank runs one replica (the Gram step has no cross-GPU exchange in scope);
rank 0 prints one JSON line.
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

METRIC = "768-bit SDP s/iter & residue-GEMM INT8 TOPS, fused vs plain, 1 B200, bit-exact"
NBLOCKS, MLO, MHI, NCOLS, L, NCHUNK = 400, 20, 120, 274, 26, 4
N_MOD = 128                       # moduli of the accumulator context (L + 1 = 27 limbs)
# DRAM bytes (read + write) of one syrk call (the full-tile launch with the fused tail, and the corner
# launch) per chunk row, from the ncu capture of `kernel_bench --kernel syrk --N 274 --K 7000 --L 27`
# ((522.41 + 32.86) MB read + (12.97 + 0.01) MB written / 7000 rows).
SYRK_DRAM_BYTES_PER_ROW = (522.40768e6 + 32.863232e6 + 12.969984e6 + 0.006656e6) / 7000


def workload_shape(seed=0):
    rng = np.random.default_rng(seed)
    m = rng.integers(MLO, MHI + 1, size=NBLOCKS)
    per = NBLOCKS // NCHUNK
    rows = [int(m[c * per:(c + 1) * per].sum()) for c in range(NCHUNK)]
    return m, rows


def gen_chunk(rng, rows, cols, L, elo=-8, ehi=8):
    """Normalised MPF (rows, cols): |mantissa| has exactly 32L-2 bits, random sign, e ~ U[elo, ehi]."""
    n = rows * cols
    mag = rng.integers(0, 1 << 32, size=(L, n), dtype=np.uint64).astype(np.uint32)
    mag[L - 1] = (mag[L - 1] & np.uint32((1 << 29) - 1)) | np.uint32(1 << 29)
    neg = rng.random(n) < 0.5
    m = mag.copy()
    m[:, neg] = ~m[:, neg]
    carry = neg.copy()
    for k in range(L):                                    # two's-complement negation, +1 with carry
        v = m[k].astype(np.uint64) + carry
        m[k] = v.astype(np.uint32)
        carry = carry & (v > 0xffffffff)
    e = rng.integers(elo, ehi + 1, size=n).astype(np.int64)
    return m.view(np.int32).reshape(L, rows, cols), e.reshape(rows, cols)


def algorithmic_ops(R, N=NCOLS):
    return N_MOD * 4 * 2 * (N * (N + 1) // 2) * R


def mp_macs(R, N=NCOLS):
    return (N * (N + 1) // 2) * R


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs"), d.get("bf16_tflops"), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()                      # sampling live before the timed region starts
            while not self.rows and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ CPU baseline (reference's own CPU path)
def cpu_reference_sample(threads):
    """Time the reference's CPU baseline (cpu_baseline/mpf_baseline.c: GMP mpf, OpenMP) on a bounded
    sample: its 274 x 274 x 274 GEMM at 832 bits.  Returns (seconds for that GEMM, kind, sample)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "mpf_baseline")
    if not os.path.exists(exe):
        from oracle import ref_build
        ref_build.build_cpu_baseline()
    if os.path.exists(exe):
        out = subprocess.run([exe, "832", str(NCOLS), str(NCOLS), str(threads)], capture_output=True, text=True,
                             timeout=600).stdout
        for line in out.splitlines():
            if line.strip().startswith("gemm"):
                return float(line.split()[1]), "reference", (
                    f"cpu_baseline/mpf_baseline.c gemm {NCOLS}x{NCOLS}x{NCOLS} at 832 bits (GMP mpf, {threads} "
                    f"threads), scaled by mp-MACs to the Gram step's N(N+1)/2*R")
    # oracle port: the C restatement of the residue path, single thread, on 2 blocks of the workload
    import oracle as O
    from oracle import mp as OM
    rng = np.random.default_rng(1)
    rows = 140
    pm, pe = gen_chunk(rng, rows, NCOLS, L)
    t = time.perf_counter()
    acc = OM.GramAcc(NCOLS, L)
    acc.add(pm, pe)
    acc.result()
    dt = time.perf_counter() - t
    return dt * (NCOLS ** 3) / mp_macs(rows), "port", f"oracle GramAcc on {rows} rows x {NCOLS} (1 thread), scaled"


def cpu_baseline(R, threads):
    t_gemm, kind, sample = cpu_reference_sample(threads)
    t_step = t_gemm * mp_macs(R) / NCOLS ** 3
    return {"value": algorithmic_ops(R) / t_step / 1e12, "unit": "TOPS", "cores": threads if kind == "reference" else 1,
            "kind": kind, "sample": sample, "s_per_step": t_step,
            "mp_mac_per_s": mp_macs(R) / t_step}


def max_over_ranks(ms, world, device):
    """The slowest rank's time: every rank calls this with its own device time (one MAX all-reduce, taken by
    all ranks in the same order); with one rank the time itself."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation of the path, on rank 0 only."""
    if rank != 0:
        return
    m, rows = workload_shape()
    R = int(sum(rows))
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference_sample(threads)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t_gemm, kind, sample = cpu_reference_sample(threads)
        vals.append(t_gemm * mp_macs(R) / NCOLS ** 3)
    wall = time.perf_counter() - t0
    t_step = statistics.mean(vals)
    value = algorithmic_ops(R) / t_step / 1e12
    cfg = workload_config(R)
    line = {"metric": METRIC, "value": value, "unit": "TOPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mpf-832 (GMP)", "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "TOPS", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "TOPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def workload_config(R):
    return {"workload": "gram_acc: Q = sum_b B_b^T B_b, 400 blocks m_b~U[20,120] (seed 0) x 274 cols, 832-bit MPF "
                        "(L=26, accumulator L+1=27, 128 moduli), 4 chunks, one CRT",
            "blocks": NBLOCKS, "rows_total": R, "cols": NCOLS, "limbs": L, "chunks": NCHUNK,
            "exponents": "U[-8,8]", "l2": "inputs (~0.86 GB) larger than L2 (126 MB); no flush",
            "parallelism": "replicas"}


# ------------------------------------------------------------------ B200 arm
def measure_int8_library_peak(torch):
    """cuBLASLt int8 GEMM (torch._int_mm) 8192^3, best of 5 -- a library reference point only."""
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        for _ in range(2):
            torch._int_mm(a, b)
        best = 1e9
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(); torch._int_mm(a, b); e.record(); e.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from sdpvibe_b200 import mpf, _trace

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    m, rows = workload_shape()
    R = int(sum(rows))
    rng = np.random.default_rng(100 + rank)
    host = [gen_chunk(rng, r, NCOLS, L) for r in rows]
    chunks = [mpf.MPF(torch.from_numpy(hm).to(dev), torch.from_numpy(he).to(dev)) for hm, he in host]
    pinned = [(torch.from_numpy(hm).pin_memory(), torch.from_numpy(he).pin_memory()) for hm, he in host]
    h2d = sum(a.numel() * a.element_size() + b.numel() * b.element_size() for a, b in pinned)
    out_m = torch.empty((L, NCOLS, NCOLS), dtype=torch.int32).pin_memory()
    out_e = torch.empty((NCOLS, NCOLS), dtype=torch.int64).pin_memory()
    d2h = out_m.numel() * 4 + out_e.numel() * 8

    def step():
        acc = mpf.GramAcc(NCOLS, L)
        for c in chunks:
            acc.add(c)
        return acc.result()

    copy_stream = torch.cuda.Stream(device=dev)
    dbuf = [(torch.empty(hm.shape, dtype=hm.dtype, device=dev), torch.empty(he.shape, dtype=he.dtype, device=dev))
            for hm, he in pinned]

    def step_e2e():
        # host -> device copies of chunk c + 1 on a copy stream while chunk c is accumulated
        main = torch.cuda.current_stream()
        ready = []
        for (hm, he), (dm, de) in zip(pinned, dbuf):
            ev = torch.cuda.Event()
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_stream(main)             # the previous step is done with the buffers
                dm.copy_(hm, non_blocking=True)
                de.copy_(he, non_blocking=True)
                ev.record(copy_stream)
            ready.append(ev)
        acc = mpf.GramAcc(NCOLS, L)
        for (dm, de), ev in zip(dbuf, ready):
            main.wait_event(ev)
            acc.add(mpf.MPF(dm, de))
        Q = acc.result()
        out_m.copy_(Q.m, non_blocking=True)
        out_e.copy_(Q.e, non_blocking=True)
        return Q

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, k, trace=None):
        barrier()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        if trace is not None:
            with trace:
                for _ in range(k):
                    fn()
        else:
            for _ in range(k):
                fn()
        e.record()
        barrier()
        return max_over_ranks(s.elapsed_time(e), world, dev)

    for _ in range(max(args.warmup, 3)):
        step()
    # The step has no host decision (GramAcc decides its flushes on the device), so it is recorded once as a
    # CUDA graph and the timed steps replay it; a separate eager pass times every kernel for the breakdown.
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        step()
    for _ in range(2):
        graph.replay()
    with ClockSampler(local_rank) as clk:
        ms = timed(graph.replay, args.steps)
    tr = _trace.Trace(timed={"sdpv_rns_gemm", "sdpv_residues_u8", "sdpv_residues_rows", "sdpv_crt_norm", "sdpv_align",
                             "sdpv_align_t", "sdpv_align_rows", "sdpv_top_max"})
    ms_eager = timed(step, args.steps, tr)
    for _ in range(2):
        step_e2e()
    ms_e2e = timed(step_e2e, args.steps)

    t_step = ms / args.steps * 1e-3
    value = world * algorithmic_ops(R) / t_step / 1e12
    gemm_ms = tr.kernel_ms("sdpv_rns_gemm")
    res_kernel = "sdpv_residues_rows" if tr.kernel_ms("sdpv_residues_rows") else "sdpv_residues_u8"
    res_ms = tr.kernel_ms(res_kernel)
    crt_ms = tr.kernel_ms("sdpv_crt_norm")
    hbm, bf16, src = load_peaks()
    if rank != 0:
        return
    int8_lib = measure_int8_library_peak(torch)
    peak = 2 * bf16
    ops_per_launch = algorithmic_ops(R) / NCHUNK
    achieved = ops_per_launch / (statistics.mean(gemm_ms) * 1e-3) / 1e12
    # decomposition: limb bytes read (L+1 limbs after alignment) + residue bytes written, per launch (the
    # operand rows it reads are 128 bytes per entry, 4 (L+1) of them limb bytes)
    res_bytes = (R / NCHUNK) * NCOLS * (4 * (L + 1) + 2 * N_MOD)
    line = {
        "metric": METRIC, "value": value, "unit": "TOPS", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8 (exact int8 x int8 -> int32 residue products)", "data": "synthetic",
        "config": workload_config(R),
        "mp_mac_per_s": world * mp_macs(R) / t_step,
        "roofline": {"bound": "tensor", "kernel": "sdpv_rns_gemm (syrk, tcgen05 kind::i8)", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": SYRK_DRAM_BYTES_PER_ROW * (R / NCHUNK),
                     "traffic_note": "ncu dram read+write of one call (full tiles + corner) at N=274, K=7000 rows, scaled per row",
                     "peak_source": f"2 x bf16_tflops of {src} (MEASURED_PEAKS.json): B200 dense int8 = 2 x dense bf16",
                     "int8_cublaslt_measured_tops": int8_lib,
                     "launch_ms_mean": statistics.mean(gemm_ms), "launches": len(gemm_ms),
                     "ops_per_launch": ops_per_launch},
        "roofline_decomposition": {"bound": "hbm", "kernel": res_kernel, "achieved":
                                   res_bytes / (statistics.mean(res_ms) * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                                   "frac": res_bytes / (statistics.mean(res_ms) * 1e-3) / 1e9 / hbm,
                                   "launch_ms_mean": statistics.mean(res_ms), "bytes_per_launch": res_bytes},
        "crt_ms": sum(crt_ms) / args.steps,
        "kernel_ms_per_step": {k: sum(tr.kernel_ms(k)) / args.steps for k in sorted(tr.timed) if tr.kernel_ms(k)},
        "e2e": {"value": world * algorithmic_ops(R) / (ms_e2e / args.steps * 1e-3) / 1e12, "unit": "TOPS",
                "ms_per_step": ms_e2e / args.steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "ms_per_step_eager": ms_eager / args.steps,
        "gpu_launches": tr.total_launches, "gpu_launches_per_step": tr.total_launches // args.steps,
        "launches_by_entry": dict(tr.launches),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(R, os.cpu_count() or 1)
    if world == 1 and not args.no_solver:
        # the metric's other half: SDPB iterations of the 768-bit Ising-structured SDP on the same GPU
        sv = solver_measurement(local_rank)
        line["sdp_solver"] = {k: sv[k] for k in ("metric", "value", "unit", "steps", "warmup", "per_iteration_s",
                                                  "metric_over", "steady_state_s_per_iter",
                                                  "config", "kernel_s_per_iter", "gpu_launches", "clocks")}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ multiprecision GEMM workload (mp-GEMM 256^3)
G_N, G_L, G_MODS, G_E = 256, 24, 112, 216        # 768 bits: 112 moduli, 216 CRT bytes (tables of L = 24)


def gemm_ops(n=G_N):
    return G_MODS * 4 * 2 * n ** 3


def gemm_cpu_baseline(threads):
    """cpu_baseline/mpf_baseline.c's gemm line at 768 bits, n = 256 (GMP mpf, all threads): the reference's
    CPU comparison for this configuration, one full GEMM (about a second of CPU work)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "mpf_baseline")
    if not os.path.exists(exe):
        from oracle import ref_build
        ref_build.build_cpu_baseline()
    if not os.path.exists(exe):
        return None
    out = subprocess.run([exe, "768", str(G_N), str(G_N), str(threads)], capture_output=True, text=True,
                         timeout=600).stdout
    for line in out.splitlines():
        if line.strip().startswith("gemm"):
            t = float(line.split()[1])
            return {"value": gemm_ops() / t / 1e12, "unit": "TOPS", "cores": threads, "kind": "reference",
                    "sample": f"cpu_baseline/mpf_baseline.c gemm {G_N}^3 at 768 bits (GMP mpf, {threads} threads), "
                              "the whole workload", "s_per_step": t, "mp_mac_per_s": G_N ** 3 / t}
    return None


def run_gemm(args, rank, world, local_rank):
    """C = A B with A, B 256 x 256 MPF at 768 bits (L = 24; NB-bit mantissas, random sign, exponents
    U[-4, 4], numpy seed 0): sdpvibe_b200.mpf.gemm (sdpvibe/mpf.py:401-452).  Metric: residue-GEMM INT8
    TOPS counted the reference's way (112 moduli x 4 digit products x 2 M N K) per GEMM.  The inputs (2 x 6.3
    MB) fit in L2, so L2 is flushed (a 256 MB write) before every timed step, outside its CUDA events."""
    import torch
    from sdpvibe_b200 import mpf, _trace
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(0)
    am, ae = gen_chunk(rng, G_N, G_N, G_L, -4, 4)
    bm, be = gen_chunk(rng, G_N, G_N, G_L, -4, 4)
    A = mpf.MPF(torch.from_numpy(am).to(dev), torch.from_numpy(ae).to(dev))
    B = mpf.MPF(torch.from_numpy(bm).to(dev), torch.from_numpy(be).to(dev))
    pinned = [torch.from_numpy(x).pin_memory() for x in (am, ae, bm, be)]
    h2d = sum(t.numel() * t.element_size() for t in pinned)
    out_m = torch.empty((G_L, G_N, G_N), dtype=torch.int32).pin_memory()
    out_e = torch.empty((G_N, G_N), dtype=torch.int64).pin_memory()
    d2h = out_m.numel() * 4 + out_e.numel() * 8
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        return mpf.gemm(A, B)

    def step_e2e():
        dm = [t.to(dev, non_blocking=True) for t in pinned]
        C = mpf.gemm(mpf.MPF(dm[0], dm[1]), mpf.MPF(dm[2], dm[3]))
        out_m.copy_(C.m, non_blocking=True)
        out_e.copy_(C.e, non_blocking=True)

    def timed(fn, k, trace=None):
        total = 0.0
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            if trace is not None:
                with trace:
                    fn()
            else:
                fn()
            e.record()
            torch.cuda.synchronize()
            total += s.elapsed_time(e)
        return max_over_ranks(total, world, dev)

    for _ in range(max(args.warmup, 3)):
        step()
        step_e2e()
    with ClockSampler(local_rank) as clk:
        ms = timed(step, args.steps)
    tr = _trace.Trace(timed={"sdpv_rns_gemm", "sdpv_residues_u8", "sdpv_crt_norm", "sdpv_align", "sdpv_top_max"})
    ms_traced = timed(step, args.steps, tr)
    ms_e2e = timed(step_e2e, args.steps)
    if rank != 0:
        return
    hbm, bf16, src = load_peaks()
    t_step = ms / args.steps * 1e-3
    gemm_ms = statistics.mean(tr.kernel_ms("sdpv_rns_gemm"))
    res_ms = statistics.mean(tr.kernel_ms("sdpv_residues_u8"))
    crt_ms = statistics.mean(tr.kernel_ms("sdpv_crt_norm"))
    ent = G_N * G_N
    res_bytes = ent * (4 * G_L + 2 * G_MODS)                 # one operand: limb bytes in, residues out
    crt_bytes = ent * (2 * G_MODS + 4 * G_L + 8)             # residues in, MPF limbs + exponents out
    crt_ops = 2 * G_E * G_MODS * ent                         # the CRT digit product on the tensor cores
    peak = 2 * bf16
    line = {
        "metric": METRIC, "value": world * gemm_ops() / t_step / 1e12, "unit": "TOPS", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8 (exact int8 x int8 -> int32 residue products)",
        "data": "synthetic",
        "config": {"workload": "mp-GEMM: C = A B, A and B 256 x 256 MPF at 768 bits (L=24, NB-bit mantissas, random "
                               "sign, exponents U[-4,4], numpy seed 0), sdpvibe_b200.mpf.gemm, output bit-exact",
                   "l2": "flushed (256 MB write) before every timed step, outside its events",
                   "ops_per_step": gemm_ops(), "mp_mac_per_step": G_N ** 3},
        "mp_mac_per_s": world * G_N ** 3 / t_step,
        "roofline": {"bound": "tensor", "kernel": "sdpv_rns_gemm (tcgen05 kind::i8)",
                     "achieved": gemm_ops() / (gemm_ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": gemm_ops() / (gemm_ms * 1e-3) / 1e12 / peak, "traffic": None,
                     "peak_source": f"2 x bf16_tflops of {src} (MEASURED_PEAKS.json): B200 dense int8 = 2 x dense bf16",
                     "launch_ms_mean": gemm_ms, "ops_per_launch": gemm_ops()},
        "roofline_decomposition": {"bound": "hbm", "kernel": "sdpv_residues_u8", "unit": "GB/s", "peak": hbm,
                                   "achieved": res_bytes / (res_ms * 1e-3) / 1e9,
                                   "frac": res_bytes / (res_ms * 1e-3) / 1e9 / hbm, "launch_ms_mean": res_ms,
                                   "bytes_per_launch": res_bytes},
        "roofline_crt": {"bound": "hbm", "kernel": "sdpv_crt_norm (CRT digit product on tcgen05 + renormalisation)",
                         "unit": "GB/s", "peak": hbm, "achieved": crt_bytes / (crt_ms * 1e-3) / 1e9,
                         "frac": crt_bytes / (crt_ms * 1e-3) / 1e9 / hbm, "launch_ms_mean": crt_ms,
                         "bytes_per_launch": crt_bytes, "tensor_tops": crt_ops / (crt_ms * 1e-3) / 1e12,
                         "tensor_frac": crt_ops / (crt_ms * 1e-3) / 1e12 / peak},
        "kernel_ms_per_step": {k: sum(tr.kernel_ms(k)) / args.steps for k in sorted(tr.timed) if tr.kernel_ms(k)},
        "ms_per_step_traced": ms_traced / args.steps,
        "e2e": {"value": world * gemm_ops() / (ms_e2e / args.steps * 1e-3) / 1e12, "unit": "TOPS",
                "ms_per_step": ms_e2e / args.steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": tr.total_launches, "gpu_launches_per_step": tr.total_launches // args.steps,
        "launches_by_entry": dict(tr.launches), "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = gemm_cpu_baseline(os.cpu_count() or 1)
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ batched Cholesky + solve workload
CS_BLOCKS, CS_NMIN, CS_NMAX, CS_NRHS, CS_L = 600, 8, 160, 8, 26
# library entry points whose launches the per-kernel tables time
TRACE_NAMES = ("sdpv_chol_tiles", "sdpv_trinv_tiles", "sdpv_residues", "sdpv_residues_u8", "sdpv_residues_rows",
               "sdpv_rns_gemm", "sdpv_rns_gemm_grouped", "sdpv_crt_norm", "sdpv_crt_block", "sdpv_shift_round",
               "sdpv_add_same", "sdpv_bitlen", "sdpv_badd_align", "sdpv_mpf_norm", "sdpv_mpf_mul", "sdpv_mpf_add",
               "sdpv_top_max", "sdpv_align", "sdpv_align_t", "sdpv_align_rows", "sdpv_grp_copy", "sdpv_grp_finish_fixed",
               "sdpv_grp_solve_round", "sdpv_grp_merge", "sdpv_grp_tile_widen",
               "sdpv_grp_tile_narrow")


def cholsolve_macs(ns):
    ns = np.asarray(ns, dtype=np.float64)
    return float((ns ** 3 / 6).sum() + (ns ** 2 * CS_NRHS).sum())


def cholsolve_cpu_baseline(ns, threads, every=20):
    """cpu_baseline/mpf_baseline.c (GMP mpf at 832 bits, OpenMP): Cholesky + trsm with 8 right-hand
    sides per block, on every `every`-th block of the workload (trsm timed once, counted twice: lower and
    upper solve), scaled to the whole workload by mp-MACs."""
    exe = os.path.join(ROOT, "oracle", "_ref", "mpf_baseline")
    if not os.path.exists(exe):
        from oracle import ref_build
        ref_build.build_cpu_baseline()
    sample = [int(n) for n in ns[::every]]
    t = 0.0
    for n in sample:
        out = subprocess.run([exe, "832", str(n), str(CS_NRHS), str(threads)], capture_output=True, text=True,
                             timeout=600).stdout
        for line in out.splitlines():
            w = line.split()
            if w and w[0] == "cholesky":
                t += float(w[1])
            elif w and w[0] == "trsm":
                t += 2 * float(w[1])
    t_all = t * cholsolve_macs(ns) / cholsolve_macs(sample)
    return {"value": cholsolve_macs(ns) / t_all, "unit": "mp-MAC/s", "cores": threads, "kind": "reference",
            "sample": f"mpf_baseline.c chol + 2 trsm (nrhs {CS_NRHS}) on {len(sample)} of {len(ns)} blocks "
                      f"(every {every}th), scaled by mp-MACs", "s_per_step": t_all}


def run_cholsolve(args, rank, world, local_rank):
    """600 SPD blocks A = G G^T + n I (n ~ U[8,160], numpy seed 0, float64 values exact in MPF), L = 26,
    8 right-hand sides, each block padded to its own multiple of 32 (the reference's callers make one batched
    Chol + solve per padded size 32..160; here all 600 blocks are factored and solved together by the grouped
    work-list engine, with every block's result that of its own bucket's call).  Metric: mp-MAC/s over the
    unpadded work sum n^3/6 + 2 * 8 n^2 / 2."""
    import torch
    from sdpvibe_b200 import mpf, _trace
    from sdpvibe_b200.kernel_bench import cholsolve_inputs, cholsolve_buckets
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cases = cholsolve_inputs(CS_BLOCKS, CS_NMIN, CS_NMAX, CS_NRHS)
    ns = [c[0] for c in cases]
    buckets = cholsolve_buckets(cases, CS_L)
    pinned = [(A.m.cpu().pin_memory(), A.e.cpu().pin_memory(), B.m.cpu().pin_memory(), B.e.cpu().pin_memory())
              for _, _, A, B in buckets]
    outs = [(torch.empty(B.m.shape, dtype=torch.int32).pin_memory(), torch.empty(B.e.shape, dtype=torch.int64)
             .pin_memory()) for _, _, _, B in buckets]
    h2d = sum(sum(t.numel() * t.element_size() for t in p) for p in pinned)
    d2h = sum(a.numel() * 4 + b.numel() * 8 for a, b in outs)

    def step():                                  # all blocks in one grouped factorisation and solve
        mpf.chol_solve_many([(A, B) for _, _, A, B in buckets])

    def step_e2e():
        pairs = [(mpf.MPF(am.to(dev, non_blocking=True), ae.to(dev, non_blocking=True)),
                  mpf.MPF(bm.to(dev, non_blocking=True), be.to(dev, non_blocking=True))) for am, ae, bm, be in pinned]
        for X, (om, oe) in zip(mpf.chol_solve_many(pairs), outs):
            om.copy_(X.m, non_blocking=True)
            oe.copy_(X.e, non_blocking=True)

    def timed(fn, k, trace=None):
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        with (trace or _trace.Trace()):
            for _ in range(k):
                fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e)
    for _ in range(max(args.warmup, 3)):
        step()
    names = TRACE_NAMES
    tr = _trace.Trace(timed=names)
    with ClockSampler(local_rank) as clk:
        ms = timed(step, args.steps, tr)
    ms_e2e = timed(step_e2e, args.steps)
    # per-kernel device time: one eager step (graphs off), every launch bracketed by CUDA events
    from sdpvibe_b200 import graphs
    graphs.ENABLED = False
    step()                                       # eager allocations
    tr_e = _trace.Trace(timed=names)
    ms_eager = timed(step, 1, tr_e)
    graphs.ENABLED = True
    if rank != 0:
        return
    macs = cholsolve_macs(ns)
    t_step = ms / args.steps * 1e-3
    kms = {k: sum(tr_e.kernel_ms(k)) for k in names if tr_e.launches[k]}
    top = max(kms, key=kms.get)
    gms = {k: sum(tr.kernel_ms(k)) / args.steps for k in tr.events if k.startswith("graph")}
    line = {"metric": "batched Cholesky + solve, 600 SPD blocks n~U[8,160], 8 RHS, 832-bit MPF (mp-MAC/s)",
            "value": world * macs / t_step, "unit": "mp-MAC/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 wide fixed point + int8 residue GEMM",
            "data": "synthetic",
            "config": {"workload": "cholsolve: 600 SPD blocks A = G G^T + n I, n~U[8,160] (numpy seed 0), "
                                   "8 RHS U(-1,1), L=26, all blocks in one grouped Chol + solve (no buckets)",
                       "buckets": {int(b[0]): len(b[1]) for b in buckets}, "limbs": CS_LIMBS_NOTE,
                       "l2": "inputs 0.88 GB (larger than L2), no flush"},
            "kernel_ms_per_step_eager": kms, "ms_per_step_eager": ms_eager, "top_kernel": top,
            "graph_ms_per_step": gms,
            "e2e": {"value": world * macs / (ms_e2e / args.steps * 1e-3), "unit": "mp-MAC/s",
                    "ms_per_step": ms_e2e / args.steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": tr.total_launches, "gpu_launches_per_step": tr.total_launches // args.steps,
            "launches_by_entry": dict(tr.launches),
            "clocks": clk.summary()}
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cholsolve_cpu_baseline(ns, os.cpu_count() or 1)
    if args.precision_iters > 0:                 # the same systems solved at L = 50
        X26 = mpf.chol_solve_many([(A, B) for _, _, A, B in buckets])
        b50 = cholsolve_buckets(cases, 50)
        X50 = mpf.chol_solve_many([(A, B) for _, _, A, B in b50])
        errs = [_rel_mpf_error(a, b) for a, b in zip(X26, X50)]
        line["error_vs_2x_precision"] = {"L": 50, "max_rel_per_bucket": errs, "max_rel": max(errs)}
    print(json.dumps(line), flush=True)


CS_LIMBS_NOTE = "26 (832 bits); base tiles in WL = 50-word fixed point"


# ------------------------------------------------------------------ objective sensitivity at the final iterate
def run_sensitivity(args, rank, world, local_rank):
    """Objective sensitivity on the Ising-structured SDP (300 blocks, N = 1000, L = 26) after `--iters`
    solver iterations (default 20): f(B, c) = c.(x + dx(B, c)), the primal objective after a Newton step
    from the final iterate, differentiated by its adjoint (one adjoint solve with the Schur and Q factors,
    then per direction one GEMM dB [y+dy, v] and dot products), along 64 Gaussian unit directions in (B, c)
    from one numpy generator (seed 1), one direction in memory at a time (25830 x 1000 MPF entries).
    value: device ms per direction (direction resident); e2e: per direction from the host float64 arrays
    (conversion and copy inside).  The first `--fd-dirs` directions are checked against central differences
    of f at L = 50 (1536-bit class precision, h = 2^-300), and the envelope value dc.x - x^T dB y is
    reported beside each."""
    import torch
    import mpmath as mp
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    from sdpvibe_b200.adjoint import NewtonObjective, iter_directions, direction_to_mpf, widen
    from sdpvibe_b200.mpf import add
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    Ls, L2, ndir, hk = 26, 50, 64, 300
    sdp, _ = ising_like_sdp(Ls)
    sol = Solver(sdp, Ls)
    iters = args.iters
    sol.run(max_iter=iters)

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn()
        b.record()
        b.synchronize()
        return r, a.elapsed_time(b)
    fo, t_setup = timed(lambda: NewtonObjective(sol))
    f0, t_fwd = timed(fo.forward)
    _, t_adj = timed(fo._adjoint)
    times, e2e, vals, env = [], [], [], []
    h2d = 0
    for k, hd in enumerate(iter_directions(sdp, ndir, seed=1, host=True)):
        h2d = sum(dB.nbytes + dc.nbytes for dB, dc in hd)
        def through_host():
            dd = direction_to_mpf(hd, Ls)
            return dd, fo.directional([x for x, _ in dd], [y for _, y in dd])
        (d, (da, de)), te = timed(through_host)
        _, t = timed(lambda: fo.directional([x for x, _ in d], [y for _, y in d]))
        times.append(t)
        e2e.append(te)
        vals.append(da)
        env.append(de)
        del d, hd
    fd = []
    t_fd = None
    if args.fd_dirs > 0:
        t0 = time.time()
        hi = NewtonObjective(sol, L=L2)
        with mp.workprec(32 * L2 + 64):
            for k, d in enumerate(iter_directions(sdp, min(args.fd_dirs, ndir), seed=1)):   # the same directions
                wd = [(widen(dB, L2).shift(-hk), widen(dc, L2).shift(-hk)) for dB, dc in d]
                fp = hi.forward([add(g.B, dB) for g, (dB, _) in zip(hi.sdp.groups, wd)],
                                [add(g.c, dc) for g, (_, dc) in zip(hi.sdp.groups, wd)])
                fm = hi.forward([add(g.B, dB, -1) for g, (dB, _) in zip(hi.sdp.groups, wd)],
                                [add(g.c, dc, -1) for g, (_, dc) in zip(hi.sdp.groups, wd)])
                v = (fp - fm) * mp.mpf(2) ** (hk - 1)
                fd.append(float(-mp.log10(abs(vals[k] - v) / abs(v))) if vals[k] != v else 999.0)
        torch.cuda.synchronize()
        t_fd = time.time() - t0
    if rank != 0:
        return
    ms = statistics.mean(times)
    rel_env = [float(abs(a - b) / abs(b)) if b else None for a, b in zip(vals, env)]
    line = {"metric": "objective sensitivity (adjoint directional derivative) per direction at the final iterate",
            "value": ms, "unit": "ms/direction", "n_gpus": world, "steps": ndir, "warmup": 0, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "832-bit MPF (L=26)",
            "data": "synthetic",
            "config": {"workload": f"sensitivity: ising_like SDP (300 blocks, N 1000) after {iters} iterations; "
                                   f"f = c.(x + dx), {ndir} Gaussian unit directions in (B, c) (numpy seed 1)",
                       "inputs": "each direction 2.7 GB in MPF (larger than L2)"},
            "e2e": {"value": statistics.mean(e2e), "unit": "ms/direction", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 5 * len(sdp.groups) * 8 * (Ls + 2)},
            "setup_ms": t_setup, "forward_ms": t_fwd, "adjoint_solve_ms": t_adj,
            "fd_check": {"L": L2, "h": f"2^-{hk}", "directions": len(fd),
                         "min_digits": min(fd) if fd else None, "digits": fd, "seconds": t_fd},
            "envelope_rel_diff": {"min": min(r for r in rel_env if r is not None),
                                  "median": statistics.median(r for r in rel_env if r is not None),
                                  "max": max(r for r in rel_env if r is not None)},
            "objective_after_newton_step": mp.nstr(f0, 30),
            "first_values": [mp.nstr(v, 20) for v in vals[:4]],
            "first_envelope_values": [mp.nstr(v, 20) for v in env[:4]]}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ full solver iterations (SDP s/iter)
SOLVER_ITERS = 20


def run_solver(args, rank, world, local_rank):
    """SDPB iterations on the Ising-structured synthetic SDP: 300 blocks (dims 1/2/3 = 180/90/30,
    degree d ~ U[20,40], K = d+1), N = 1000, L = 26 (the 768-bit precision rule).  A step is one
    iteration; the configuration's first 20 iterations run and the metric is the mean s/iteration of
    iterations 2-20 (lower is better)."""
    line = solver_measurement(local_rank, world)
    if args.precision_iters > 0:
        line["error_vs_2x_precision"] = solver_precision_check(args.precision_iters)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_plain(args, rank, world, local_rank):
    """--impl plain: the reference's own solver and GPU kernels (Triton + its CUDA C strings, per-bucket
    Cholesky) on this GPU, on the same Ising-structured SDP as --workload solver (baseline/plain_gpu.py);
    the metric is the same mean s/iteration over iterations 2-20.  Rank 0 only."""
    if rank != 0 or args.workload != "solver":
        if rank == 0:
            print(json.dumps({"impl": "plain", "unavailable": "the plain GPU path is measured for --workload solver"}))
        return
    import torch
    torch.cuda.set_device(local_rank)
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    try:
        import plain_gpu
        with ClockSampler(local_rank) as clk:
            per_it, walls = plain_gpu.run_plain_solver(SOLVER_ITERS)
    except Exception as ex:                       # noqa: BLE001 -- reported, not raised: a baseline only
        print(json.dumps({"impl": "plain", "unavailable": f"{type(ex).__name__}: {ex}"[:400]}), flush=True)
        return
    timed = per_it[1:]
    s_it = statistics.mean(timed)
    line = {"metric": "768-bit SDP s/iter (Ising-structured synthetic SDP, 300 blocks, N=1000)", "impl": "plain",
            "value": s_it, "unit": "s/iter", "n_gpus": 1, "steps": len(timed), "warmup": 1,
            "ms_per_step": s_it * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "the reference's int8 residue GEMM (Triton) + int32 fixed point, 832-bit MPF (L=26)",
            "data": "synthetic",
            "config": {"workload": "solver: the reference SDPviBe's Solver.run (its Triton and CUDA C kernels, "
                                   "per-bucket Cholesky, unmodified; CuPy stand-in compiles its CUDA strings with "
                                   "nvcc; CRT digit-sum tl.dot given out_dtype=int32 in a wrapper) on the same "
                                   "ising_like SDP (300 blocks, N=1000, L=26)",
                       "metric_over": f"mean of iterations 2..{len(per_it)}"},
            "per_iteration_s": per_it, "wall_s_at_iteration": walls, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def _rel_mpf_error(A26, A50):
    """max |A26 - A50| / max |A50| over the entries (A26 widened exactly to A50's limbs, the difference
    formed in MPF on the device)"""
    import mpmath as mp
    from sdpvibe_b200.adjoint import widen
    from sdpvibe_b200.mpf import add, max_abs
    with mp.workprec(32 * A50.L + 64):
        d = max_abs(add(widen(A26, A50.L), A50, -1))
        ref = max_abs(A50)
        return float(d / ref) if ref else float(d)


def solver_precision_check(iters):
    """the same SDP (the 26-limb data widened exactly) run at L = 50, twice the working precision: per
    iteration the relative differences of the primal and dual objectives and the step lengths, and of y
    after the last iteration.  The step lengths come from float64 eigenvalues of matrices that differ in
    their last bits, so the iterates agree to about the float64 step-length accuracy, not to 2^-830."""
    import mpmath as mp
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    from sdpvibe_b200.adjoint import widen_sdp
    sdp, _ = ising_like_sdp(26)
    runs = {}
    for L in (26, 50):
        s = Solver(widen_sdp(sdp, L) if L != 26 else sdp, L)
        log = []
        s.run(max_iter=iters, log=log)
        runs[L] = (log, s.y)
    with mp.workprec(32 * 50 + 64):
        def rel(a, b):
            return float(abs(a - b) / max(abs(b), mp.mpf(10) ** -300))
        per_it = [{k: rel(a[k], b[k]) for k in ("pobj", "dobj", "P_step", "D_step")}
                  for a, b in zip(runs[26][0], runs[50][0])]
    return {"L": 50, "iterations": len(per_it), "max_rel": {k: max(r[k] for r in per_it) for k in per_it[0]},
            "per_iteration": per_it, "y_rel_last": _rel_mpf_error(runs[26][1], runs[50][1])}


def solver_measurement(local_rank, world=1, iters=SOLVER_ITERS):
    """The configuration's run: the first `iters` (20) iterations from the start; the metric is the mean of
    iterations 2 .. iters (the first records the CUDA graphs).  Also reported: the mean of iterations 4 ..
    iters (after the chunk streams' memory pools are filled)."""
    import torch
    import mpmath as mp
    from sdpvibe_b200 import _trace
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    Ls = 26
    t0 = time.perf_counter()
    sdp, blocks = ising_like_sdp(Ls)
    t_build = time.perf_counter() - t0
    sol = Solver(sdp, Ls, timing=True)
    marks = []

    warm = 1                                    # iteration 1 records the graphs
    steps = iters - warm
    total_it = iters

    def rec(it, s, info):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks.append((it, ev, info["row"]))
        if it == warm:                          # phase and kernel tables over iterations 2 .. iters only
            s.timer.marks.clear()
            tr.launches.clear()
            tr.events.clear()
    tr = _trace.Trace(timed=TRACE_NAMES)        # graph replays are timed whole, one entry per graph key
    with ClockSampler(local_rank) as clk, tr:
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record()
        sol.run(max_iter=total_it, record=rec)
        torch.cuda.synchronize()
    ev = [start] + [m[1] for m in marks]
    per_it = [ev[i].elapsed_time(ev[i + 1]) * 1e-3 for i in range(len(ev) - 1)]
    timed = per_it[warm:]
    s_it = statistics.mean(timed)
    steady = statistics.mean(per_it[3:]) if len(per_it) > 3 else s_it
    last = marks[-1][2]
    line = {"metric": "768-bit SDP s/iter (Ising-structured synthetic SDP, 300 blocks, N=1000)",
            "value": s_it, "unit": "s/iter", "n_gpus": world, "steps": len(timed), "warmup": warm,
            "ms_per_step": s_it * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8 residue GEMM + int32 fixed point (832-bit MPF, L=26)", "data": "synthetic",
            "config": {"workload": "solver: SDPB predictor-corrector iterations, ising_like SDP "
                                   "(300 blocks dims 1/2/3 = 180/90/30, d~U[20,40], K=d+1, damped monomial "
                                   "bases, random B/c/b; numpy seed 0), N=1000, L=26",
                       "sum_P_padded": int(sum(g.nb * g.P for g in sdp.groups)),
                       "chunks": [dict(dim=g.dim, nb=g.nb, K=g.K, h=g.h[0], P=g.P) for g in sdp.groups],
                       "l2": "working set of several GB; no flush"},
            "per_iteration_s": per_it, "build_s": t_build,
            "iterations": len(per_it), "metric_over": f"mean of iterations 2..{len(per_it)}",
            "steady_state_s_per_iter": steady, "steady_state_over": f"mean of iterations 4..{len(per_it)}",
            "last_row": {k: (mp.nstr(v, 6) if isinstance(v, mp.mpf) else v) for k, v in last.items()},
            "tables_over": f"the {steps} timed iterations (plus the residue phase of the final evaluation)",
            "phase_s_per_iter": {k: v / steps for k, v in sol.timer.totals().items()},
            "kernel_s_per_iter": {k: sum(tr.kernel_ms(k)) * 1e-3 / steps for k in sorted(tr.events)},
            "gpu_launches": tr.total_launches,
            "gpu_launches_per_step": tr.total_launches // max(1, steps), "launches_by_entry": dict(tr.launches),
            "eig_refined": sol.eig_refined, "clocks": clk.summary()}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference", "plain"), default="b200",
                    help="reference: the reference's CPU path; plain: the reference's own GPU solver (solver workload)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--iters", type=int, default=20, help="sensitivity: solver iterations before the sensitivities")
    ap.add_argument("--fd-dirs", type=int, default=8, help="sensitivity: directions checked by finite differences")
    ap.add_argument("--precision-iters", type=int, default=6,
                    help="solver / cholsolve: iterations (solver) compared with a run at twice the precision; 0 skips")
    ap.add_argument("--no-solver", action="store_true", help="gram: skip the SDP s/iteration measurement")
    ap.add_argument("--workload", choices=("gram", "gemm", "cholsolve", "solver", "sensitivity"), default="gram",
                    help="gram: the residue Gram step (default); gemm: the mp-GEMM 256^3 at 768 bits; cholsolve: "
                         "batched Cholesky + solve; solver: SDPB iterations (s/iter)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.impl == "plain":
        return run_plain(args, rank, world, local_rank)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run = {"gram": run_b200, "gemm": run_gemm, "cholsolve": run_cholsolve, "solver": run_solver,
               "sensitivity": run_sensitivity}[args.workload]
        run(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
