"""Benchmark of the blocked matrix product over Blosc2-compressed containers on B200.

Workload (one step = one iarray_opt_gemm call on resident compressed containers:
decode A, decode B, product, re-encode C):
  precision_f64: A, B 8192 x 8192 float64, entries uniform(-1,1) * 2^U{-8..8}
  (numpy default_rng(3), A then B), chunkshape 2048 x 2048, blockshape 256 x 256,
  Blosc2 LZ4 clevel 5 + SHUFFLE; output with the same partition.
The headline `value` is effective TFLOP/s (2*M*N*K per step) of the split-precision
form when the library supports it, else of the native FP64 form; both forms are timed
and their normwise errors against a double-double oracle (sampled rows) are reported.

Contract: `python bench.py --gpus N --steps K --warmup W` prints one JSON line (rank 0).
`--impl reference` times the reference algorithm on the host cores instead (the
oracle's restatement of iarray_opt_gemm's block-pair loop with OpenBLAS dgemm and
liblz4), on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "iron-array_b200"))

import numpy as np  # noqa: E402

M = N = K = 8192
CHUNK, BLOCK = (2048, 2048), (256, 256)
FLOP = 2.0 * M * N * K
METRIC = "GEMM TFLOP/s split-precision vs native FP64 at stated error; decode GB/s"


def bench_config(world):
    """The workload's config, the same dict in both arms."""
    return {"workload": "precision_f64 opt_gemm 8192^3, chunk 2048^2, block 256^2, LZ4 clevel5 + SHUFFLE",
            "M": M, "N": N, "K": K, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (compressed A + B about 1 GB), no flush needed"}


def make_inputs():
    rng = np.random.default_rng(3)
    A = rng.uniform(-1, 1, (M, K)) * np.exp2(rng.integers(-8, 9, (M, K)))
    B = rng.uniform(-1, 1, (K, N)) * np.exp2(rng.integers(-8, 9, (K, N)))
    return A, B


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.p = None
        fd, self.path = tempfile.mkstemp(prefix="iarray_b200_clocks_", suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
            return
        # nvidia-smi takes a moment to start: wait for its first sample so that the
        # timed region that follows is covered
        t0 = time.time()
        while time.time() - t0 < 10 and self.p.poll() is None:
            self.f.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.remove(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ============================================================================ reference arm
def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    if rank != 0:
        barrier(pg)
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    A, B = make_inputs()
    ga, ach = O.encode_array(A, CHUNK, BLOCK)
    gb, bch = O.encode_array(B, CHUNK, BLOCK)
    gc = O.Geom((M, N), CHUNK, BLOCK, 8)
    del A, B
    cores = os.cpu_count() or 1
    # warm-up: one output chunk per step (page-ins, thread start-up, BLAS kernels); each
    # timed step is the whole product, every one of the 16 output chunks
    for s in range(args.warmup):
        O.cpu_opt_gemm_chunk(ga, ach, gb, bch, gc, s % gc.nchunks, cores)
    times = []
    for s in range(args.steps):
        t = time.perf_counter()
        O.cpu_opt_gemm(ga, ach, gb, bch, gc, cores)
        times.append(time.perf_counter() - t)
    sec = float(np.mean(times))
    v = FLOP / sec / 1e12
    sample = (f"the whole 8192^3 opt_gemm per timed step ({gc.nchunks} output chunks, {FLOP / 1e12:.2f} TFLOP): "
              f"the reference's block-pair loop with per-pair LZ4 block decode (liblz4), single-threaded OpenBLAS "
              f"dgemm per worker thread ({cores} workers over each chunk's blocks), each block LZ4-compressed by its "
              f"worker; warm-up steps compute one output chunk each")
    line = {"metric": METRIC, "value": v, "unit": "TFLOP/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (numpy default_rng(3))",
            "config": bench_config(world),
            "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "port", "sample": sample,
                             "samples": len(times), "step_s": [round(x, 3) for x in times]},
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    barrier(pg)


# ============================================================================ roofline
L_MODULI = 14          # moduli of the split-precision product (library default)


def roofline(kprof, steps, pk, dgemm_tflops, c_cbytes, a_cb, b_cb):
    """Roofline of the kernel with the largest device time in the timed steps.
    achieved = algorithmic work of one launch / its mean CUDA-event duration, where the work of
    one launch is the kernel's algorithmic work per step x steps / its launches (a kernel that
    runs once per row band of the product launches several times a step)."""
    name, (cnt, tot) = max(kprof.items(), key=lambda kv: kv[1][1])
    avg_s = tot / cnt * 1e-3
    share = steps / cnt                          # steps per launch
    img = M * N * 8                              # bytes of one dense 8192^2 float64 matrix
    if name == "k_i8gemm_mod":
        work, unit, bound = 2.0 * M * N * K * L_MODULI * share / 1e12, "TOP/s", "tensor"
        peak, src = 2 * pk["bf16_tflops"], "2 x measured dense BF16 (sm_100 dense INT8 rate is twice BF16)"
    elif name == "k_gemm_f64":
        work, unit, bound = FLOP * share / 1e12, "TFLOP/s", "tensor"
        peak, src = dgemm_tflops, "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor roof)"
    else:
        bytes_per_step = {
            "k_lz4_encode": img + (c_cbytes or img),            # read the byte-plane image, write LZ4 streams
            "k_lz4_encode_par": img + (c_cbytes or img),
            "k_lz4_decode_cta": a_cb + b_cb + 2 * img,          # upper bound: all streams LZ4
            "k_crt": L_MODULI * M * N + img,                    # residue planes in, float64 out
            "k_crt_img": L_MODULI * M * N + img,                # the same, out as C's encoder image
            "k_residues_rows": img + L_MODULI * M * K,
            "k_residues_cols": img + L_MODULI * K * N,
            "k_scatter_fast": 4 * img, "k_scatter": 4 * img,   # both operands, read + write
            "k_gather_fast": 2 * img, "k_gather": 2 * img,
            "k_emit": 2 * (c_cbytes or img),
        }.get(name)
        if bytes_per_step is None:
            return {"bound": None, "kernel": name, "achieved": None, "peak": None, "unit": None, "frac": None,
                    "traffic": None}
        work, unit, bound = bytes_per_step * share / 1e9, "GB/s", "hbm"
        peak, src = pk["hbm_gbs"], "measured HBM copy bandwidth"
    achieved = work / avg_s
    traffic = None
    tf = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(name)
    return {"bound": bound, "kernel": name, "launches": cnt, "launches_per_step": cnt / steps, "avg_ms": tot / cnt,
            "achieved": achieved,
            "peak": peak, "peak_source": src, "unit": unit, "frac": achieved / peak if peak else None,
            "traffic": traffic,
            "traffic_source": "profiles/ncu_traffic.json: dram bytes read + written of one launch of this "
                              "kernel at this workload, from a committed counter capture (not re-measured "
                              "by this run)" if traffic is not None else None}


# ============================================================================ secondary workloads
def _timed(ctx, stream, fn, steps, warmup):
    """Device time per call (CUDA events on the context stream) and wall time per call."""
    import torch
    for _ in range(warmup):
        fn()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t = time.perf_counter()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    ctx.synchronize()
    wall = (time.perf_counter() - t) / steps
    return e0.elapsed_time(e1) / steps, wall * 1e3


def secondary_gemv(ia, ctx, stream, args, pk):
    """Plain GEMV: float32 y = A x, A 20000 x 20000 with A[i, j] = sin(0.001 i) + cos(0.002 j)
    (computed in float64, stored as float32), x uniform(-1, 1) (default_rng(2)), chunk 4000^2,
    block 500^2; standalone decode of A and the full iarray_opt_gemv call."""
    import torch
    n, ch, bl = 20000, 4000, 500
    A = np.empty((n, n), np.float32)
    cj = np.cos(0.002 * np.arange(n))
    for r0 in range(0, n, 2000):
        A[r0:r0 + 2000] = (np.sin(0.001 * np.arange(r0, r0 + 2000))[:, None] + cj[None, :]).astype(np.float32)
    x = np.random.default_rng(2).uniform(-1, 1, n).astype(np.float32)
    Ac = ia.Container.from_numpy(ctx, A, (ch, ch), (bl, bl))
    xc = ia.Container.from_numpy(ctx, x, (ch,), (bl,))
    nb, cb = Ac.info()
    ref = A.astype(np.float64) @ x.astype(np.float64)
    del A
    dense = torch.empty((n, n), dtype=torch.float32, device="cuda")
    dec_ms, _ = _timed(ctx, stream, lambda: Ac.decode_to_device(dense.data_ptr(), n), args.steps, args.warmup)
    del dense
    torch.cuda.empty_cache()
    out = []

    def step():
        out.append(ia.opt_gemv(ctx, Ac, xc, (ch,), (bl,)))
        if len(out) > 1:
            out.pop(0).free()
    gemv_ms, gemv_wall = _timed(ctx, stream, step, args.steps, args.warmup)
    y = out[-1].to_numpy().astype(np.float64)
    err = float(np.linalg.norm(y - ref) / np.linalg.norm(ref))
    for c in out + [Ac, xc]:
        c.free()
    gbs = (nb + cb) / (dec_ms * 1e-3) / 1e9
    return {"workload": "gemv f32 20000x20000 smooth, chunk 4000^2, block 500^2",
            "decode_gbs": gbs, "decode_frac_of_measured_hbm": gbs / pk["hbm_gbs"], "decode_ms": dec_ms,
            "compression_ratio": nb / cb, "opt_gemv_ms": gemv_ms, "opt_gemv_wall_ms": gemv_wall,
            "opt_gemv_gflops": 2.0 * n * n / (gemv_ms * 1e-3) / 1e9,
            "opt_gemv_gbs": (cb + 8 * n) / (gemv_ms * 1e-3) / 1e9,
            "normwise_err_vs_f64": err}


def secondary_plain_f64(ia, ctx, stream, args):
    """Plain drop-in: iarray_linalg_matmul, A, B 1000 x 1000 float64, A = uniform(-1, 1)
    (default_rng(0)), B = uniform(-1, 1) (default_rng(1)), chunk 500^2, block 100^2 for A, B and
    C; both forms, normwise error against double-double on every row."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n, ch, bl = 1000, 500, 100
    A = np.random.default_rng(0).uniform(-1, 1, (n, n))
    B = np.random.default_rng(1).uniform(-1, 1, (n, n))
    hi, lo = O.dd_rows(A, B, np.arange(n))
    out = {"workload": "plain matmul f64 1000^3, chunk 500^2, block 100^2"}
    for form_name, form in (("native", ia.FORM_NATIVE), ("split", ia.FORM_SPLIT)):
        ctx.set_form(form)
        Ac = ia.Container.from_numpy(ctx, A, (ch, ch), (bl, bl))
        Bc = ia.Container.from_numpy(ctx, B, (ch, ch), (bl, bl))
        res = []

        def step():
            res.append(ia.matmul(ctx, Ac, Bc, (ch, ch), (bl, bl)))
            if len(res) > 1:
                res.pop(0).free()
        ms, wall = _timed(ctx, stream, step, args.steps, args.warmup)
        err = O.normwise_error(res[-1].to_numpy(), hi, lo, np.arange(n))
        for c in res + [Ac, Bc]:
            c.free()
        out[form_name] = {"ms": ms, "wall_ms": wall, "tflops": 2.0 * n ** 3 / (ms * 1e-3) / 1e12,
                          "normwise_err_vs_dd": err}
    ctx.set_form(ia.FORM_NATIVE)
    return out


def secondary_f32(ia, ctx, stream, args):
    """Precision, float32: A 16384 x 4096, B 4096 x 16384, normal(0, 1) (default_rng(4)) plus
    0.1 sin(0.003 (i + j)), chunk 4096^2, block 512^2; native FFMA and 3xBF16 split forms."""
    M, K, N, ch, bl = 16384, 4096, 16384, 4096, 512
    rng = np.random.default_rng(4)
    A = rng.standard_normal((M, K))
    A += 0.1 * np.sin(0.003 * (np.arange(M)[:, None] + np.arange(K)[None, :]))
    A = A.astype(np.float32)
    B = rng.standard_normal((K, N))
    B += 0.1 * np.sin(0.003 * (np.arange(K)[:, None] + np.arange(N)[None, :]))
    B = B.astype(np.float32)
    Ac = ia.Container.from_numpy(ctx, A, (ch, ch), (bl, bl))
    Bc = ia.Container.from_numpy(ctx, B, (ch, ch), (bl, bl))
    rows = np.sort(np.random.default_rng(99).choice(M, args.err_rows, replace=False))
    exact = A[rows].astype(np.float64) @ B.astype(np.float64)
    del A, B
    flop = 2.0 * M * N * K
    res = {"workload": "precision_f32 16384x4096 @ 4096x16384, chunk 4096^2, block 512^2"}
    for name, form, prods in (("native", ia.FORM_NATIVE, 0), ("split", ia.FORM_SPLIT, 6),
                              ("split_3xbf16", ia.FORM_SPLIT, 3)):
        ctx.set_form(form)
        ctx.set_split_products_f32(prods)
        out = []

        def step():
            out.append(ia.opt_gemm(ctx, Ac, Bc, (ch, ch), (bl, bl)))
            if len(out) > 1:
                out.pop(0).free()
        steps = max(2, args.steps // 2)
        ms, _ = _timed(ctx, stream, step, steps, max(1, args.warmup - 1))
        ia.profile_kernels(True)
        step()
        ctx.synchronize()
        ia.profile_kernels(False)
        prof = ia.kernel_profile()
        prod = sum(v[1] for k, v in prof.items() if k in ("k_gemm_f32", "k_bf16s_gemm", "k_split_rows", "k_split_cols"))
        tc_ms = prof.get("k_bf16s_gemm", (0, 0.0))[1]
        c = out[-1].to_numpy()[rows].astype(np.float64)
        err = float(np.linalg.norm(c - exact) / np.linalg.norm(exact))
        for x in out:
            x.free()
        res[name] = {"ms_per_step": ms, "tflops": flop / (ms * 1e-3) / 1e12, "product_ms": prod,
                     "product_tflops": flop / (prod * 1e-3) / 1e12 if prod else None,
                     "normwise_err_vs_f64": err, "kernel_ms": {k: v[1] for k, v in sorted(prof.items())}}
        if prods and tc_ms:
            # the tensor-core kernel's BF16 work: `prods` products of 2 M N K each
            bf = prods * flop / (tc_ms * 1e-3) / 1e12
            res[name]["bf16_products"] = prods
            res[name]["tensor_tflops"] = bf
            res[name]["tensor_frac_of_measured_bf16"] = bf / peaks()["bf16_tflops"]
    ctx.set_form(ia.FORM_NATIVE)
    Ac.free()
    Bc.free()
    return res


def secondary_sparse(ia, ctx, stream, args, dense_ms):
    """Block-sparse precision_f64: the benchmark's A with 90% of its 256 x 256 blocks zero
    (default_rng(7) picks them), B unchanged.  The reference skips every block pair with a
    zero block (src/linalg/iarray_gemm.c:206-211); the GPU kernels leave out the k-tiles of
    such pairs, so the step shrinks with the work."""
    A, B = make_inputs()
    rng = np.random.default_rng(7)
    zero = rng.random((M // BLOCK[0], K // BLOCK[1])) < 0.9
    for i, j in zip(*np.nonzero(zero)):
        A[i * BLOCK[0]:(i + 1) * BLOCK[0], j * BLOCK[1]:(j + 1) * BLOCK[1]] = 0.0
    Ac = ia.Container.from_numpy(ctx, A, CHUNK, BLOCK)
    Bc = ia.Container.from_numpy(ctx, B, CHUNK, BLOCK)
    rows = np.sort(np.random.default_rng(99).choice(M, 64, replace=False))
    ref = A[rows] @ B
    res = {"workload": "precision_f64 8192^3 with 90% of A's 256^2 blocks zero",
           "zero_block_fraction": float(zero.mean())}
    for name, form in (("native", ia.FORM_NATIVE), ("split", ia.FORM_SPLIT)):
        ctx.set_form(form)
        out = []

        def step():
            out.append(ia.opt_gemm(ctx, Ac, Bc, CHUNK, BLOCK))
            if len(out) > 1:
                out.pop(0).free()
        ms, _ = _timed(ctx, stream, step, max(2, args.steps // 2), max(1, args.warmup - 1))
        c = out[-1].to_numpy()[rows]
        err = float(np.linalg.norm(c - ref) / np.linalg.norm(ref))
        for x in out:
            x.free()
        res[name] = {"ms_per_step": ms, "dense_ms_per_step": dense_ms.get(name),
                     "speedup_vs_dense": dense_ms[name] / ms if dense_ms.get(name) else None,
                     "normwise_err_vs_f64": err}
    ctx.set_form(ia.FORM_NATIVE)
    Ac.free()
    Bc.free()
    return res


def secondary_batch(ia, ctx, stream, args):
    """Batching: 512 independent float64 products, m, n, k uniform integers in [64, 2048]
    (default_rng(5)), entries uniform(-1, 1), chunk 512^2, block 128^2 (ragged edges); one
    CUDA graph per form, grouped persistent product kernel in the native form."""
    rng = np.random.default_rng(5)
    dims = rng.integers(64, 2049, (512, 3))
    As, Bs = [], []
    for m, n, k in dims:
        As.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (int(m), int(k))), (512, 512), (128, 128)))
        Bs.append(ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (int(k), int(n))), (512, 512), (128, 128)))
    flop = float(sum(2.0 * int(m) * int(n) * int(k) for m, n, k in dims))
    cs, bs = [(512, 512)] * len(dims), [(128, 128)] * len(dims)
    res = {"workload": "batching 512 float64 products, m,n,k in [64,2048], chunk 512^2, block 128^2",
           "flop": flop}
    for name, form in (("native", ia.FORM_NATIVE), ("split", ia.FORM_SPLIT)):
        ctx.set_form(form)
        t = time.perf_counter()
        batch = ia.Batch(ctx, As, Bs, cs, bs)
        build_s = time.perf_counter() - t
        info = batch.info()
        if form == ia.FORM_SPLIT:
            info["split_tuning"] = batch.split_tuning()
        dev, wall = [], []
        for s in range(max(1, args.warmup - 1) + max(2, args.steps // 2)):
            t = time.perf_counter()
            outs = batch.run()
            w = time.perf_counter() - t
            d = ctx.timings()["total"]
            for c in outs:
                c.free()
            if s >= max(1, args.warmup - 1):
                dev.append(d)
                wall.append(w * 1e3)
        batch.free()
        res[name] = {"graph_ms": float(np.mean(dev)), "tflops": flop / (np.mean(dev) * 1e-3) / 1e12,
                     "run_wall_ms": float(np.mean(wall)), "build_s": build_s, **info}
    ctx.set_form(ia.FORM_NATIVE)
    for c in As + Bs:
        c.free()
    return res


# ============================================================================ our arm
def run_ours(args):
    world, rank, local, pg = dist_setup(args)
    import torch
    torch.cuda.set_device(local)
    import iarray_b200 as ia
    ia.init()
    # the parallel-parse LZ4 encoder writes the output chunks (valid LZ4 that the reference
    # decodes bit-exactly; the liblz4-identical encoder is timed as its own form below)
    ctx = ia.Context(encoder=ia.ENCODER_PARALLEL)
    stream = torch.cuda.ExternalStream(ctx.stream())

    A, B = make_inputs()
    Ac = ia.Container.from_numpy(ctx, A, CHUNK, BLOCK)
    Bc = ia.Container.from_numpy(ctx, B, CHUNK, BLOCK)
    a_nb, a_cb = Ac.info()
    b_nb, b_cb = Bc.info()

    forms = {"native": (ia.FORM_NATIVE, ia.ENCODER_PARALLEL), "split": (ia.FORM_SPLIT, ia.ENCODER_PARALLEL),
             "split_liblz4_encoder": (ia.FORM_SPLIT, ia.ENCODER_LIBLZ4)}
    results = {}
    for name, (form, encoder) in forms.items():
        ctx.set_form(form)
        ctx.set_encoder(encoder)
        try:
            C = ia.opt_gemm(ctx, Ac, Bc, CHUNK, BLOCK)
        except ia.IArrayError as e:
            if e.name == "NOT_SUPPORTED":
                continue
            raise
        for _ in range(max(args.warmup - 1, 0)):
            C.free()
            C = ia.opt_gemm(ctx, Ac, Bc, CHUNK, BLOCK)
        C.free()
        barrier(pg)
        torch.cuda.synchronize()
        clk = Clocks(local)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        parts = np.zeros(5)
        l0 = ia.lib().iarray_b200_kernel_launches()
        ia.profile_kernels(True)            # CUDA events around every launch, on its stream
        ev0.record(stream)
        for _ in range(args.steps):
            C = ia.opt_gemm(ctx, Ac, Bc, CHUNK, BLOCK)
            t = ctx.timings()
            parts += [t["decode_a"], t["decode_b"], t["product"], t["encode"], t["total"]]
            C.free()
        ev1.record(stream)
        torch.cuda.synchronize()
        ia.profile_kernels(False)
        kprof = ia.kernel_profile()
        launches = ia.lib().iarray_b200_kernel_launches() - l0
        clocks = clk.stop()
        ms = ev0.elapsed_time(ev1) / args.steps
        ms = max_over_ranks(pg, ms)
        parts /= args.steps
        results[name] = dict(ms=ms, parts=parts, launches=launches, clocks=clocks, form=form, encoder=encoder,
                             kprof=kprof)

    # errors vs double-double on sampled rows (outside the timed region)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    if rank == 0:
        import oracle as O
        rows = np.sort(np.random.default_rng(99).choice(M, args.err_rows, replace=False))
        hi, lo = O.dd_rows(A, B, rows)
        for name, r in results.items():
            ctx.set_form(r["form"])
            ctx.set_encoder(r["encoder"])
            C = ia.opt_gemm(ctx, Ac, Bc, CHUNK, BLOCK)
            c = C.to_numpy()
            r["err"] = O.normwise_error(c, hi, lo, rows)
            _, c_cb = C.info()
            r["c_cbytes"] = c_cb
            C.free()
            del c

    # split form at each moduli count (rank 0, outside the timed region): device time of the
    # step and of its product, and the normwise error on the same sampled rows
    moduli = None
    if rank == 0 and world == 1 and not args.no_secondary and "split" in results:
        moduli = {"native_err": results.get("native", {}).get("err")}
        ctx.set_encoder(ia.ENCODER_PARALLEL)
        for L in (12, 13, 14, 15, 16):
            ctx.set_form(ia.FORM_SPLIT, L)
            out, prod = [], []

            def step():
                out.append(ia.opt_gemm(ctx, Ac, Bc, CHUNK, BLOCK))
                prod.append(ctx.timings()["product"])
                if len(out) > 1:
                    out.pop(0).free()
            ms, _ = _timed(ctx, stream, step, 3, 2)
            err = O.normwise_error(out[-1].to_numpy(), hi, lo, rows)
            out[-1].free()
            moduli[str(L)] = {"ms_per_step": ms, "product_ms": float(np.mean(prod[2:])), "normwise_err_vs_dd": err,
                              "err_vs_native": err / moduli["native_err"] if moduli["native_err"] else None}
        ctx.set_form(ia.FORM_NATIVE)

    # end-to-end through the C ABI with host frames in pinned memory: every step uploads
    # the A and B frames (iarray_from_cframe), runs the product and writes C's frame back
    # to host memory (iarray_b200_to_cframe_into)
    head = "split" if "split" in results else "native"
    ctx.set_form(results[head]["form"])
    ctx.set_encoder(results[head]["encoder"])

    def pinned(n):
        return torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy()
    fa, fb = pinned(Ac.cframe_len()), pinned(Bc.cframe_len())
    Ac.to_cframe_into(fa)
    Bc.to_cframe_into(fb)
    fc = pinned(M * N * 8 + (1 << 20))
    # (a) one call, iarray_b200_opt_gemm_cframes: uploads, kernels and downloads pipelined
    # per chunk row of C
    e2e_t, d2h = [], 0
    for s in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        _, d2h = ia.opt_gemm_cframes(ctx, fa, fb, CHUNK, BLOCK, out=fc)
        torch.cuda.synchronize()
        if s >= args.warmup:
            e2e_t.append(time.perf_counter() - t)
    e2e_ms = max_over_ranks(pg, float(np.mean(e2e_t)) * 1e3)
    tl = ctx.timings()             # iarray_b200_opt_gemm_cframes: [0] B ready, [3] the bands, [4] total
    e2e_parts = {"b_ready_ms": tl["decode_a"], "bands_ms": tl["encode"], "device_total_ms": tl["total"]}
    # (b) the reference's call sequence: iarray_from_cframe x 2, iarray_opt_gemm,
    # iarray_b200_to_cframe_into (each call synchronous)
    seq_t, d2h_seq = [], 0
    for s in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        a2 = ia.Container.from_cframe(ctx, fa)
        b2 = ia.Container.from_cframe(ctx, fb)
        C = ia.opt_gemm(ctx, a2, b2, CHUNK, BLOCK)
        d2h_seq = C.to_cframe_into(fc)
        torch.cuda.synchronize()
        if s >= args.warmup:
            seq_t.append(time.perf_counter() - t)
        for x in (a2, b2, C):
            x.free()
    seq_ms = max_over_ranks(pg, float(np.mean(seq_t)) * 1e3)

    # standalone decode of A (compressed chunks resident in HBM -> dense float64 array in
    # HBM) through iarray_b200_decode_to_device; bytes = compressed read + decoded written
    dense = torch.empty((M, K), dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        Ac.decode_to_device(dense.data_ptr(), K)
    ctx.synchronize()
    d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ia.profile_kernels(True)
    d0.record(stream)
    for _ in range(args.steps):
        Ac.decode_to_device(dense.data_ptr(), K)
    d1.record(stream)
    ctx.synchronize()
    ia.profile_kernels(False)
    dec_prof = ia.kernel_profile()
    dec_ms = max_over_ranks(pg, d0.elapsed_time(d1) / args.steps)
    del dense
    torch.cuda.empty_cache()

    # cuBLAS DGEMM on the same dense shapes: the measured FP64 tensor roof
    dgemm_tflops = None
    if rank == 0:
        x = torch.randn(M, K, dtype=torch.float64, device="cuda")
        y = torch.randn(K, N, dtype=torch.float64, device="cuda")
        for _ in range(2):
            torch.matmul(x, y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            torch.matmul(x, y)
        e1.record()
        torch.cuda.synchronize()
        dgemm_tflops = FLOP / (e0.elapsed_time(e1) / 3 * 1e-3) / 1e12
        del x, y
        torch.cuda.empty_cache()

    # CPU baseline: the reference's loop on a bounded sample (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle as O
        ga, ach = O.Geom((M, K), CHUNK, BLOCK, 8), Ac.chunks()
        gb, bch = O.Geom((K, N), CHUNK, BLOCK, 8), Bc.chunks()
        gc = O.Geom((M, N), CHUNK, BLOCK, 8)
        cores = os.cpu_count() or 1
        O.cpu_opt_gemm_chunk(ga, ach, gb, bch, gc, 0, cores)      # warm-up
        ts = []
        for s in range(args.cpu_samples):
            t = time.perf_counter()
            O.cpu_opt_gemm(ga, ach, gb, bch, gc, cores)
            ts.append(time.perf_counter() - t)
        v = FLOP / float(np.median(ts)) / 1e12
        cpu = {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "port", "samples": len(ts),
               "sample_s": [round(x, 3) for x in ts], "statistic": "median",
               "sample": "the whole 8192^3 opt_gemm (16 output chunks) per sample with the reference's block-pair "
                         "loop: per-pair LZ4 block decode, single-threaded OpenBLAS dgemm per worker thread, each "
                         "block LZ4-compressed by its worker"}
        # upper bound on the host: dense float64 product of the decoded operands with
        # torch.mm on all cores (no codec work), one warm-up and one timed call
        torch.set_num_threads(cores)
        ta, tb = torch.from_numpy(A), torch.from_numpy(B)
        torch.mm(ta[:1024], tb)
        td = []
        for _ in range(3):
            t = time.perf_counter()
            torch.mm(ta, tb)
            td.append(time.perf_counter() - t)
        cpu["dense_upper_bound"] = {"value": FLOP / float(np.median(td)) / 1e12, "unit": "TFLOP/s",
                                    "cores": cores, "samples": len(td), "statistic": "median",
                                    "what": "torch.mm float64 8192^3 on decoded operands"}
        del ta, tb

    pk = peaks()
    secondary = None
    if rank == 0 and world == 1 and not args.no_secondary:
        for c in (Ac, Bc):
            c.free()
        torch.cuda.empty_cache()
        secondary = {}
        dense_ms = {k: r["ms"] for k, r in results.items() if k in ("native", "split")}
        for key, fn in (("sparse_blocks_f64", lambda: secondary_sparse(ia, ctx, stream, args, dense_ms)),
                        ("plain_f64_1000", lambda: secondary_plain_f64(ia, ctx, stream, args)),
                        ("gemv_f32", lambda: secondary_gemv(ia, ctx, stream, args, pk)),
                        ("precision_f32", lambda: secondary_f32(ia, ctx, stream, args)),
                        ("batching_f64", lambda: secondary_batch(ia, ctx, stream, args))):
            try:
                secondary[key] = fn()
            except Exception as e:          # reported, not fatal: the headline stands alone
                secondary[key] = {"error": str(e)[:200]}
            torch.cuda.empty_cache()

    if rank != 0:
        barrier(pg)
        return
    barrier(pg)
    hr = results[head]
    value = world * FLOP / (hr["ms"] * 1e-3) / 1e12
    roof = roofline(hr["kprof"], args.steps, pk, dgemm_tflops, c_cbytes=hr.get("c_cbytes"), a_cb=a_cb, b_cb=b_cb)
    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": hr["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (numpy default_rng(3))",
        "config": bench_config(world), "form": head,
        "forms": {k: {"tflops": world * FLOP / (r["ms"] * 1e-3) / 1e12, "ms_per_step": r["ms"],
                      "encoder": "liblz4-identical" if r["encoder"] == ia.ENCODER_LIBLZ4 else "parallel-parse",
                      "ms_parts": {"decode_a": r["parts"][0], "decode_b": r["parts"][1], "product": r["parts"][2],
                                   "encode": r["parts"][3]},
                      "normwise_err_vs_dd": r.get("err"), "kernel_launches": int(r["launches"])}
                  for k, r in results.items()},
        "decode": {"gbs": (a_nb + a_cb) / (dec_ms * 1e-3) / 1e9,
                   "frac_of_measured_hbm": (a_nb + a_cb) / (dec_ms * 1e-3) / 1e9 / pk["hbm_gbs"],
                   "ms": dec_ms, "bytes": a_nb + a_cb,
                   "what": "A (8192^2 float64, 16 chunks) compressed in HBM -> dense in HBM, "
                           "bytes = compressed read + decoded written",
                   "kernel_ms": {k: v[1] / args.steps for k, v in sorted(dec_prof.items())}},
        "kernel_ms_per_step": {k: {kk: v[1] / args.steps for kk, v in sorted(r["kprof"].items())}
                               for k, r in results.items()},
        "compression": {"a_ratio": a_nb / a_cb, "b_ratio": b_nb / b_cb,
                        "c_ratio": (M * N * 8) / hr["c_cbytes"] if hr.get("c_cbytes") else None},
        "roofline": roof,
        "cublas_dgemm_tflops": dgemm_tflops,
        "cpu_baseline": cpu,
        "e2e": {"value": world * FLOP / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                "h2d_bytes_per_step": len(fa) + len(fb), "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "call": "iarray_b200_opt_gemm_cframes (pinned host frames in and out)", "parts": e2e_parts},
        "e2e_calls": {"value": world * FLOP / (seq_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                      "h2d_bytes_per_step": len(fa) + len(fb), "d2h_bytes_per_step": d2h_seq, "ms_per_step": seq_ms,
                      "call": "iarray_from_cframe x2 + iarray_opt_gemm + iarray_b200_to_cframe_into"},
        "gpu_launches": int(hr["launches"]),
        "clocks": hr["clocks"],
        "peaks_used": {"hbm_gbs": pk.get("hbm_gbs"), "bf16_tflops": pk.get("bf16_tflops")},
        "split_moduli": moduli,
        "secondary": secondary,
    }
    if "split" in results and "native" in results:
        line["split_vs_native"] = {"speedup": results["native"]["ms"] / results["split"]["ms"],
                                   "err_ratio": (results["split"].get("err") or 0) /
                                                max(results["native"].get("err") or 1e-300, 1e-300)}
    print(json.dumps(line), flush=True)


def run_kernel_case(args):
    """One small case of one kernel family, for per-kernel counter captures.
    codec: an n x n float64 container (n = --case-n, default 4096) of the product's kind of
    values (gaussian) encoded with the parallel encoder, then an A-like one
    (uniform(-1,1) x 2^U{-8..8}) decoded; three rounds each.  split: the split-precision
    float64 product n x n x n on device operands (iarray_b200_dense_gemm), two rounds.  splitc:
    the split-precision iarray_opt_gemm on compressed n x n containers (chunk n/2, block 256^2;
    the product reconstructed into C's encoder image), two rounds.  f32split: the float32 split form (six BF16 products) n x n x n, two rounds.  gemv: the
    plain GEMV workload's smooth float32 matrix at n x n (chunk 4000^2, block 500^2) decoded three
    times, then one iarray_opt_gemv.  f64native: the native FP64 product n x n x n on device
    operands, two rounds.  batch: the first n / 64 problems of the batching workload in the
    split form (creation and two graph replays).
    Inputs are larger than L2 and a few GB at most are held on the device."""
    import ctypes
    import torch
    import iarray_b200 as ia
    ia.init()
    rng = np.random.default_rng(5)
    n = args.case_n
    if args.kernel_case == "codec":
        ctx = ia.Context(encoder=ia.ENCODER_PARALLEL)
        C = rng.standard_normal((n, n)) * 600.0
        A = rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))
        for _ in range(3):
            ia.Container.from_numpy(ctx, C, (2048, 2048), (256, 256)).free()
        a = ia.Container.from_numpy(ctx, A, (2048, 2048), (256, 256))
        out = torch.empty((n, n), dtype=torch.float64, device="cuda")
        for _ in range(3):
            a.decode_to_device(out.data_ptr(), n)
        ctx.synchronize()
        assert np.array_equal(out.cpu().numpy(), A)
    elif args.kernel_case == "gemv":
        ctx = ia.Context(encoder=ia.ENCODER_PARALLEL)
        A = (np.sin(0.001 * np.arange(n))[:, None] + np.cos(0.002 * np.arange(n))[None, :]).astype(np.float32)
        a = ia.Container.from_numpy(ctx, A, (4000, 4000), (500, 500))
        out = torch.empty((n, n), dtype=torch.float32, device="cuda")
        for _ in range(3):
            a.decode_to_device(out.data_ptr(), n)
        ctx.synchronize()
        assert np.array_equal(out.cpu().numpy(), A)
        x = np.random.default_rng(2).uniform(-1, 1, n).astype(np.float32)
        xc = ia.Container.from_numpy(ctx, x, (4000,), (500,))
        y = ia.opt_gemv(ctx, a, xc, (4000,), (500,)).to_numpy().astype(np.float64)
        ref = A.astype(np.float64) @ x.astype(np.float64)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-5
    elif args.kernel_case == "batch":
        # the first n // 64 problems of the batching workload (n = --case-n, default 4096: 64
        # problems), split form at 14 moduli: creation (one eager pass) and two graph replays
        ctx = ia.Context(form=ia.FORM_SPLIT, split_terms=14, encoder=ia.ENCODER_PARALLEL)
        count = max(1, min(512, n // 64))
        dims = rng.integers(64, 2049, (512, 3))[:count]
        As = [ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (int(m), int(k))), (512, 512), (128, 128))
              for m, _, k in dims]
        Bs = [ia.Container.from_numpy(ctx, rng.uniform(-1, 1, (int(k), int(nn))), (512, 512), (128, 128))
              for _, nn, k in dims]
        batch = ia.Batch(ctx, As, Bs, [(512, 512)] * count, [(128, 128)] * count)
        for _ in range(2):
            for c in batch.run():
                c.free()
        batch.free()
    elif args.kernel_case == "f64native":
        ctx = ia.Context(form=ia.FORM_NATIVE)
        A = torch.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
        B = torch.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
        C = torch.empty((n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        for _ in range(2):
            ia.check(ia.lib().iarray_b200_dense_gemm(ctx.ptr, ia.DTYPE_DOUBLE, n, n, n, ctypes.c_void_p(A.data_ptr()), n,
                                                      ctypes.c_void_p(B.data_ptr()), n, ctypes.c_void_p(C.data_ptr()), n),
                     "dense_gemm")
        ctx.synchronize()
        ref = (A[:64] @ B).cpu().numpy()
        err = np.linalg.norm(C[:64].cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err < 1e-14, err
    elif args.kernel_case == "splitc":
        # the split-precision iarray_opt_gemm on compressed n x n containers (chunk n/2, block
        # 256): decode, product reconstructed into C's encoder image, encode; two rounds
        ctx = ia.Context(form=ia.FORM_SPLIT, encoder=ia.ENCODER_PARALLEL)
        a = rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))
        b = rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))
        ch, bl = (n // 2, n // 2), (256, 256)
        Ac, Bc = ia.Container.from_numpy(ctx, a, ch, bl), ia.Container.from_numpy(ctx, b, ch, bl)
        for _ in range(2):
            C = ia.opt_gemm(ctx, Ac, Bc, ch, bl)
            got = C.to_numpy()[:64]
            C.free()
        ref = a[:64] @ b
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err < 1e-14, err
    elif args.kernel_case == "f32split":
        ctx = ia.Context(form=ia.FORM_SPLIT)
        A = torch.from_numpy(rng.standard_normal((n, n)).astype(np.float32)).cuda()
        B = torch.from_numpy(rng.standard_normal((n, n)).astype(np.float32)).cuda()
        C = torch.empty((n, n), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        for _ in range(2):
            ia.check(ia.lib().iarray_b200_dense_gemm(ctx.ptr, ia.DTYPE_FLOAT, n, n, n, ctypes.c_void_p(A.data_ptr()), n,
                                                      ctypes.c_void_p(B.data_ptr()), n, ctypes.c_void_p(C.data_ptr()), n),
                     "dense_gemm")
        ctx.synchronize()
        ref = (A[:64].double() @ B.double()).cpu().numpy()
        err = np.linalg.norm(C[:64].cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err < 2e-6, err
    else:
        ctx = ia.Context(form=ia.FORM_SPLIT)
        A = torch.from_numpy(rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))).cuda()
        B = torch.from_numpy(rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n)))).cuda()
        C = torch.empty((n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        for _ in range(2):
            ia.check(ia.lib().iarray_b200_dense_gemm(ctx.ptr, ia.DTYPE_DOUBLE, n, n, n, ctypes.c_void_p(A.data_ptr()), n,
                                                      ctypes.c_void_p(B.data_ptr()), n, ctypes.c_void_p(C.data_ptr()), n),
                     "dense_gemm")
        ctx.synchronize()
        ref = (A[:64] @ B).cpu().numpy()
        err = np.linalg.norm(C[:64].cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err < 1e-13, err
    print(json.dumps({"kernel_case": args.kernel_case, "ok": True}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--err-rows", type=int, default=256, help="rows (default_rng(99)) for the normwise error")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-samples", type=int, default=3, help="whole-product samples of the CPU baseline")
    ap.add_argument("--no-secondary", action="store_true", help="skip the GEMV, float32 and batching workloads")
    ap.add_argument("--kernel-case", choices=["codec", "split", "splitc", "f32split", "gemv", "f64native", "batch"], default=None,
                    help="run one small case of one kernel family instead of the benchmark")
    ap.add_argument("--case-n", type=int, default=4096, help="matrix size of --kernel-case")
    args = ap.parse_args()
    if args.kernel_case:
        run_kernel_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
