"""Benchmark of the SPLA local contraction on B200.

Workload (default): complex-double pgemm_ssb, C = A^H B, m = n = 1024,
k = 250000, A and B complex Gaussian scaled by 1/sqrt(k), beta = 0, C on a
1x1 block-cyclic grid with 128x128 blocks (the ZGEMM-SSB configuration of the
headline metric). One step = one contraction of the whole problem.

  value : TFLOP/s (8 m n k flops per step) of the headline path with A, B
          already resident in HBM, through the kernel-level C ABI (splab_gemm)
          on one stream, CUDA-event timed. The headline path is the Ozaki INT8
          path when it is built and meets <= 1e-14, else FP64 DMMA.
  e2e   : the same metric through the public C ABI (spla_pzgemm_ssb) with A, B,
          C in pinned HOST memory: every step streams A and B to the GPU and
          reads C back inside the timed region.
  paths : TFLOP/s and relative Frobenius error of each contraction path on the
          whole C, against the device double-double product (splab_gemm_dd),
          which is itself checked against the CPU Dot2 oracle on three columns.
  suite : at one GPU and the default shape, the other configurations of the
          benchmark suite (real-double ssb, sbs, the 64-instance batches, the
          adjoint, ssbtr), each run afterwards by `bench.py --workload NAME`
          in a child process; the line keeps their TFLOP/s, time per step,
          path and whole-C error (--no-suite skips them).

Multi-GPU (torchrun, one rank per GPU): every rank runs its own replica of the
single-rank problem (the single-rank path has no exchange step); value is the
sum of all ranks' flops over the max-over-ranks time.

--impl reference times the reference's own CPU path (oracle/_ref, the
reference library compiled from its sources, else the oracle's C
restatement) on the host cores, rank 0 only: the same metric and workload,
one full call per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

M = N = 1024
K = 250000
SEED = 20250002  # seed = 20250000 + configuration index
FLOPS = 8.0 * M * N * K


def set_shape(m, k):
    """Smaller instances of the same workload (profiling captures)."""
    global M, N, K, FLOPS
    M = N = m
    K = k
    FLOPS = 8.0 * M * N * K
OZAKI_MODULI = 15  # default modulus count of the library (<= 1e-14 at this k)
HEADLINE_METRIC = "ZGEMM-SSB TFLOP/s: Ozaki-INT8 vs FP64-DMMA at ≤1e-14 rel err, 1 B200"


def workload_name():
    return (f"pzgemm_ssb C=A^H B complex double m=n={M} k={K}, 1x1 grid 128x128 blocks, "
            "beta=0")


def max_over_ranks(torch, ms, device):
    """The step time of the slowest rank (all ranks take part in the reduction)."""
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if torch.distributed.is_initialized() and torch.distributed.get_world_size() > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(flops_per_rank, world, ms_max):
    """Replicas: every rank did flops_per_rank in the slowest rank's time."""
    return flops_per_rank * world / (ms_max / 1e3) / 1e12


def cpu_env():
    """Thread count (the CPUs this process may run on) and an explicit OpenBLAS
    core type (must precede loading BLAS)."""
    try:
        n = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        n = os.cpu_count() or 1
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(n))
    os.environ.setdefault("OMP_NUM_THREADS", str(n))
    try:
        flags = Path("/proc/cpuinfo").read_text()
        if "avx512f" in flags and "GenuineIntel" in flags:
            os.environ.setdefault("OPENBLAS_CORETYPE", "SkylakeX")
        elif "AuthenticAMD" in flags:
            os.environ.setdefault("OPENBLAS_CORETYPE", "Zen")
        elif "avx2" in flags:
            os.environ.setdefault("OPENBLAS_CORETYPE", "Haswell")
    except OSError:
        pass
    return n


def cpu_model():
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# clocks


TIMED_WINDOWS = []  # (path, host wall-clock start, end) of every timed region


class ClockSampler:
    """nvidia-smi every 20 ms; the summary keeps the samples taken inside the
    timed regions (TIMED_WINDOWS), so idle time around them does not count."""
    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(f"/tmp/spla_b200_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, path=None):
        rows = []
        try:
            for ln in self.path.read_text().splitlines():
                p = [x.strip() for x in ln.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        except OSError:
            return None
        if not rows:
            return None
        import datetime

        def inside(r):
            try:
                t = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                return False
            return any(a <= t <= b for p, a, b in TIMED_WINDOWS if path is None or p == path)

        timed = [r for r in rows if inside(r)]
        use = timed or rows
        sm = [float(r[1]) for r in use if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in use for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(use), "samples_in_timed_regions": len(timed),
                "sampling": "nvidia-smi every 20 ms; median over the samples inside the timed "
                            "regions (all samples when none fell inside)"}


# ---------------------------------------------------------------------------
# helpers


def make_inputs(torch, device):
    g = torch.Generator(device=device)
    g.manual_seed(SEED)
    s = (1.0 / (2.0 * K)) ** 0.5
    # column-major k x m (k contiguous) == row-major (m, k)
    A = torch.randn((M, K), dtype=torch.complex128, device=device, generator=g) * s
    B = torch.randn((N, K), dtype=torch.complex128, device=device, generator=g) * s
    return A, B


def measured_peaks(torch, device):
    """FP64 and INT8 tensor roofs measured here with library GEMMs (cuBLAS via
    torch): the denominators for the DMMA and Ozaki kernels."""
    out = {}
    a = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, a)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e9
    for _ in range(5):
        e0.record()
        torch.matmul(a, a)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    out["fp64_tflops"] = 2 * 8192 ** 3 / best / 1e12
    del a
    try:
        x = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device=device)
        y = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device=device).t()
        for _ in range(3):
            torch._int_mm(x, y)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(10):
            e0.record()
            torch._int_mm(x, y)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        out["int8_tops"] = 2 * 8192 ** 3 / best / 1e12
    except Exception as ex:  # pragma: no cover - depends on the torch build
        out["int8_tops"] = None
        out["int8_error"] = str(ex)[:100]
    return out


def rel_err_sampled(dC, A, B, cols=None):
    """Relative Frobenius error of columns `cols` of C against the CPU Dot2 oracle."""
    import numpy as np
    import oracle
    cols = cols or (0, N // 2, N - 1)
    An = A.cpu().numpy().ravel()
    Bs = B[list(cols)].cpu().numpy().ravel()
    ref = np.zeros(M * len(cols), np.complex128)
    assert oracle.gemm(2, 0, M, len(cols), K, 1.0, An, K, Bs, K, 0.0, ref, M) == 0
    got = dC.reshape(N, M)[list(cols)].cpu().numpy().ravel()
    return oracle.rel_fro(got, ref)


def dd_reference(torch, spla, A, B):
    """The whole C = A^H B in double-double on the device (splab_gemm_dd, the
    device form of the compensated oracle), rounded to complex128, (N, M)."""
    R = torch.zeros((N, M), dtype=torch.complex128, device=A.device)
    rc = spla.gemm_dd(3, 2, 0, M, N, K, A, K, B, K, R, M,
                      stream=torch.cuda.current_stream(A.device).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"splab_gemm_dd: status {rc}")
    torch.cuda.synchronize()
    return R


def rel_err_full(torch, C, R):
    """||C - R||_F / ||R||_F over the whole C (device or host tensor)."""
    C = C.to(R.device).reshape(R.shape)
    return float(torch.linalg.vector_norm(C - R) / torch.linalg.vector_norm(R))


def time_device_path(torch, spla, path, A, B, steps, warmup, rank):
    """Kernel-level timing of one path, device-resident operands, one stream."""
    import ctypes as ct
    L = spla.lib()
    dC = torch.zeros(M * N, dtype=torch.complex128, device=A.device)
    ws_bytes = spla.splab_gemm_workspace_size("complex128", path, 2, 0, M, N, K)
    ws = torch.empty(max(1, ws_bytes), dtype=torch.uint8, device=A.device)
    stream = torch.cuda.Stream(device=A.device)
    nphase = 3 + 16  # slice, GEMM span, reconstruct; then one per INT8 GEMM launch
    pev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * nphase)]
    for e in pev:  # torch creates the CUDA event on first record
        e.record(stream)
    stream.synchronize()
    handles = (ct.c_void_p * (2 * nphase))(*[e.cuda_event for e in pev])

    def step():
        rc = spla.splab_gemm("complex128", path, 2, 0, M, N, K, 1.0, A, K, B, K, 0.0, dC, M,
                             workspace=ws, workspace_bytes=ws_bytes, stream=stream.cuda_stream)
        if rc != 0:
            raise RuntimeError(f"splab_gemm path {path}: {L.splab_status_string(rc).decode()}")

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            step()
        stream.synchronize()
        phase_ms = [0.0] * nphase
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if torch.distributed.is_initialized():
            torch.distributed.barrier()
        torch.cuda.synchronize()
        wall0 = time.time()
        t0.record(stream)
        for _ in range(steps):
            for e in pev:
                e.record(stream)  # phases a path does not have read as zero
            L.splab_set_phase_events(handles, nphase)
            try:
                step()
            finally:
                L.splab_set_phase_events(None, 0)
            stream.synchronize()
            for p in range(nphase):
                try:
                    phase_ms[p] += pev[2 * p].elapsed_time(pev[2 * p + 1])
                except RuntimeError:
                    pass
        t1.record(stream)
        torch.cuda.synchronize()
        TIMED_WINDOWS.append((path, wall0, time.time()))
    ms = t0.elapsed_time(t1) / steps
    return dC, ms, [x / steps for x in phase_ms]


def e2e_public_api(torch, spla, path, A, B, steps, warmup):
    """Public C ABI with pinned host operands: H2D of A, B and D2H of C per step."""
    hA = torch.empty(A.shape, dtype=A.dtype, pin_memory=True)
    hB = torch.empty(B.shape, dtype=B.dtype, pin_memory=True)
    hA.copy_(A)
    hB.copy_(B)
    hC = torch.zeros(M * N, dtype=torch.complex128).pin_memory()
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    dist = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128,
                                                             128)

    def step():
        spla.pgemm_ssb(M, N, K, spla.OP_CONJ_TRANSPOSE, 1.0, hA, K, hB, K, 0.0, hC, M, 0, 0, dist,
                       ctx)

    for _ in range(warmup):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if torch.distributed.is_initialized():
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return ms, hC, hA, hB


def gauss_host(rows, cols, seed, scale, threads):
    """Column-major complex128 rows x cols buffer, re and im N(0, scale^2),
    filled by `threads` seeded generators in parallel (one per chunk)."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    out = np.empty(rows * cols, np.complex128)
    flat = out.view(np.float64)
    nch = 4 * max(1, threads)
    bounds = np.linspace(0, flat.size, nch + 1).astype(np.int64)
    gens = [np.random.default_rng(s) for s in np.random.SeedSequence(seed).spawn(nch)]

    def fill(i):
        part = flat[bounds[i]:bounds[i + 1]]
        gens[i].standard_normal(out=part)
        part *= scale

    with ThreadPoolExecutor(max(1, threads)) as ex:
        list(ex.map(fill, range(nch)))
    return out


def host_load():
    try:
        return [float(x) for x in Path("/proc/loadavg").read_text().split()[:3]]
    except OSError:
        return None


def cpu_reference_run(steps, warmup, A=None, B=None):
    """The reference's CPU path on the whole workload: one step is one full
    pzgemm_ssb call (m = n = M, k = K, op = C, beta = 0) through the C ABI of
    the reference library built from its sources (oracle/_ref), else of the
    oracle's C restatement, with every host thread this process may run on.
    `warmup` untimed calls, then `steps` timed calls (as the reference's own
    benchmark: tests/programs/benchmark.cpp:53-66). A and B: host column-major
    K x M / K x N complex128 buffers (generated here when None).
    Returns (TFLOP/s, ms per call, info)."""
    import numpy as np
    cores = cpu_env()
    import oracle
    load_before = host_load()
    have_ref = oracle.REF_LIB.exists()
    # the compensated C port is some 30x slower than the reference's BLAS: without the
    # reference library each call contracts a k-sample of the workload instead
    kk = K if have_ref else min(K, 4096)
    ld = K  # given operands hold all K rows; the first kk of them form the sample
    if A is None:
        s = (1.0 / (2.0 * K)) ** 0.5
        A = gauss_host(kk, M, SEED, s, cores)
        B = gauss_host(kk, N, SEED + 1, s, cores)
        ld = kk
    C = np.zeros(M * N, np.complex128)
    if have_ref:
        from capi import SplaCAPI
        ref = SplaCAPI(oracle.REF_LIB)
        ctx = ref.ctx(0)
        _, dist = ref.block_cyclic(1, 1, 128, 128)

        def call():
            assert ref.pgemm_ssb(np.complex128, M, N, K, 2, 1.0, A, K, B, K, 0.0, C, M, 0, 0,
                                 dist, ctx) == 0
        kind = "reference"
    else:
        def call():
            assert oracle.pgemm_ssb(M, N, kk, 2, 1.0, A, ld, B, ld, 0.0, C, M, 0, 0) == 0
        kind = "port"
    for _ in range(max(0, warmup)):
        call()
    times = []
    t_all = time.perf_counter()
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
    ms = (time.perf_counter() - t_all) * 1e3 / len(times)
    flops = 8.0 * M * N * kk
    if kk != K:  # per call of the whole workload, at the sample's rate
        ms *= K / kk
    try:
        quota = Path("/sys/fs/cgroup/cpu.max").read_text().strip()
    except OSError:
        quota = None
    info = dict(kind=kind, cores=cores, sample=(
        (f"pzgemm_ssb m=n={M} k={K} op=C beta=0 (the whole workload each call), " if kk == K
         else f"pzgemm_ssb m=n={M} k={kk} (k sampled from {K}: no reference library, the "
              "compensated C port) op=C beta=0, time scaled to k, ") +
        f"{warmup} warm-up + {len(times)} timed calls, mean {ms:.0f} ms, "
        f"OPENBLAS_NUM_THREADS={os.environ.get('OPENBLAS_NUM_THREADS')}, "
        f"OPENBLAS_CORETYPE={os.environ.get('OPENBLAS_CORETYPE')}, cpu={cpu_model()}"),
        call_ms={"min": min(times) * 1e3, "median": statistics.median(times) * 1e3,
                 "max": max(times) * 1e3},
        host={"cpus_usable": cores, "cpus_online": os.cpu_count(), "cgroup_cpu_max": quota,
              "loadavg_before": load_before, "loadavg_after": host_load()})
    return flops / (ms / 1e3) / 1e12, ms, info


# ---------------------------------------------------------------------------


# ---------------------------------------------------------------------------
# further configurations of the benchmark suite (one JSON line each)


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def workload_sbs(torch, spla, steps, warmup, path=None):
    """pzgemm_sbs subspace rotation: A 200000 x 2048 (Gaussian/sqrt(k)), B a
    Haar-random unitary 2048 x 2048 (QR of a complex Gaussian, phases of
    diag(R) folded in), C 200000 x 2048 U[-1,1], alpha = beta = 1. The path
    is AUTO (None), FP64 DMMA (1) or Ozaki INT8 (2)."""
    mloc, n, k = 200000, 2048, 2048
    g = torch.Generator(device="cuda")
    g.manual_seed(20250003)
    s = (1.0 / (2.0 * k)) ** 0.5
    A = torch.randn((k, mloc), dtype=torch.complex128, device="cuda", generator=g) * s  # cm mloc x k
    Z = torch.randn((n, k), dtype=torch.complex128, device="cuda", generator=g)
    Q, R = torch.linalg.qr(Z.T)  # k x n
    d = torch.diagonal(R)
    Q = Q * (d / d.abs()).unsqueeze(0)
    B = Q.T.contiguous()  # column-major k x n buffer: row j of B.T... stored (n, k)
    C0 = (torch.rand((n, mloc), dtype=torch.float64, device="cuda", generator=g) * 2 - 1) + 1j * (
        torch.rand((n, mloc), dtype=torch.float64, device="cuda", generator=g) * 2 - 1)
    C = C0.clone()
    flops = 8.0 * mloc * n * k
    ctx = spla.Context(spla.PU_GPU)
    if path is not None:
        ctx.set_fp64_path(path)
    resolved = spla.lib().splab_gemm_path(3, spla.PATH_AUTO if path is None else path, 0, 0, mloc,
                                          n, k)
    dist = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128,
                                                             128)

    def step():
        C.copy_(C0)
        spla.pgemm_sbs(mloc, n, k, 1.0, A, mloc, B, k, 0, 0, dist, 1.0, C, mloc, ctx)

    for _ in range(warmup):
        step()
    e0, e1 = _events(torch)
    ms_copy = 0.0
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # subtract the C reset copy (13 GB) timed separately
    e0.record()
    for _ in range(steps):
        C.copy_(C0)
    e1.record()
    torch.cuda.synchronize()
    ms_copy = e0.elapsed_time(e1) / steps
    step()
    torch.cuda.synchronize()
    # whole C against the device double-double product A B (plus C0)
    R = torch.zeros((n, mloc), dtype=torch.complex128, device="cuda")
    assert spla.gemm_dd(3, 0, 0, mloc, n, k, A, mloc, B, k, R, mloc) == 0
    torch.cuda.synchronize()
    R += C0
    err = float(torch.linalg.vector_norm(C - R) / torch.linalg.vector_norm(R))
    del R
    t = ms - ms_copy
    name = {1: "FP64 DMMA", 2: "Ozaki INT8", 3: "3xTF32"}[resolved]
    return {"metric": f"ZGEMM-SBS TFLOP/s (pzgemm_sbs, {name})", "value": flops / (t / 1e3) / 1e12,
            "unit": "TFLOP/s", "ms_per_step": t, "rel_err_whole_c_vs_double_double": err,
            "config": {"workload": "pzgemm_sbs mLocal=200000 n=k=2048 alpha=beta=1, B unitary",
                       "path": ("auto: " if path is None else "") + name}}


def workload_dssb(torch, spla, steps, warmup, path=None):
    """pdgemm_ssb real double, C = A^T B, k = 20000, m = n = 256, A and B
    U[-1, 1], C on a 1x1 grid of 64 x 64 blocks, beta = 0 (the reference's
    CPU-runnable configuration), on the context's path (AUTO by default)."""
    m = n = 256
    k = 20000
    g = torch.Generator(device="cuda")
    g.manual_seed(20250001)
    A = torch.rand((m, k), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    B = torch.rand((n, k), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    C = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    ctx = spla.Context(spla.PU_GPU)
    if path is not None:
        ctx.set_fp64_path(path)
    resolved = spla.lib().splab_gemm_path(1, spla.PATH_AUTO if path is None else path, 1, 0, m,
                                          n, k)
    dist = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 64,
                                                             64)

    def step():
        spla.pgemm_ssb(m, n, k, spla.OP_TRANSPOSE, 1.0, A, k, B, k, 0.0, C, m, 0, 0, dist, ctx)

    for _ in range(warmup):
        step()
    e0, e1 = _events(torch)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    R = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    assert spla.gemm_dd(1, 1, 0, m, n, k, A, k, B, k, R, m) == 0
    torch.cuda.synchronize()
    err = float(torch.linalg.vector_norm(C - R) / torch.linalg.vector_norm(R))
    name = {1: "FP64 DMMA", 2: "Ozaki INT8", 3: "3xTF32"}[resolved]
    return {"metric": "DGEMM-SSB TFLOP/s (pdgemm_ssb, real double, A^T B)",
            "value": 2.0 * m * n * k / (ms / 1e3) / 1e12, "unit": "TFLOP/s", "ms_per_step": ms,
            "rel_err_whole_c_vs_double_double": err,
            "config": {"workload": "pdgemm_ssb m=n=256 k=20000 op=T, 1x1 grid 64x64 blocks, "
                                   "U[-1,1]",
                       "path": ("auto: " if path is None else "") + name,
                       "l2": "inputs (82 MB) fit in L2: a per-call figure of a small problem"}}


def workload_adjoint(torch, spla, steps, warmup, path=None):
    """Differentiable ssb -> loss: C = A^H B (complex double, k = 100000,
    m = n = 512, Gaussian/sqrt(k)), L = ||C - I||_F^2, forward and backward
    (dA = B dC^H, dB = A dC on the sbs kernels) through
    spla_b200.autograd on the context's path (AUTO by default). One step is
    one forward and one backward (three contractions of 8 m n k flops).
    Checks: the gradients against torch autograd through torch.matmul (cuBLAS
    FP64), and central differences along 4 random unit directions per operand
    with Re<grad, dX> (dX the realised step), at h = 1e-6 in the
    cancellation-free form of the quadratic loss (L(X+) - L(X-) =
    Re<C+ + C- - 2I, forward(dX)>) and at h = 1e-3 in the plain
    two-evaluation form."""
    from spla_b200.autograd import ssb, ssb_autograd
    m = n = 512
    k = 100000
    g = torch.Generator(device="cuda")
    g.manual_seed(20250005)
    s = (1.0 / (2.0 * k)) ** 0.5
    A = torch.randn((m, k), dtype=torch.complex128, device="cuda", generator=g) * s
    B = torch.randn((n, k), dtype=torch.complex128, device="cuda", generator=g) * s
    ctx = spla.Context(spla.PU_GPU)
    if path is not None:
        ctx.set_fp64_path(path)
    resolved = spla.lib().splab_gemm_path(3, spla.PATH_AUTO if path is None else path, 2, 0, m,
                                          n, k)
    eye = torch.eye(m, n, dtype=torch.complex128, device="cuda")
    Ar = A.clone().requires_grad_(True)
    Br = B.clone().requires_grad_(True)

    def step():
        Ar.grad = Br.grad = None
        C = ssb_autograd(Ar, Br, ctx)
        (C - eye).abs().pow(2).sum().backward()

    for _ in range(warmup):
        step()
    e0, e1 = _events(torch)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    gA, gB = Ar.grad.detach(), Br.grad.detach()
    At = A.clone().requires_grad_(True)
    Bt = B.clone().requires_grad_(True)
    ((At.conj() @ Bt.T - eye).abs().pow(2).sum()).backward()
    grad_err = max(float((gA - At.grad).norm() / At.grad.norm()),
                   float((gB - Bt.grad).norm() / Bt.grad.norm()))
    del At, Bt

    def loss(C):
        return float((C - eye).abs().pow(2).sum())

    gen = torch.Generator(device="cuda")
    gen.manual_seed(17)
    fd_stable = fd_plain = 0.0
    for which in ("A", "B"):
        X, grad = (A, gA) if which == "A" else (B, gB)
        fwd = (lambda Xv: ssb(Xv, B, ctx)) if which == "A" else (lambda Xv: ssb(A, Xv, ctx))
        for _ in range(4):
            V = torch.randn(X.shape, dtype=X.dtype, device="cuda", generator=gen)
            V /= V.norm()
            Xp, Xm = X + 1e-6 * V, X - 1e-6 * V
            dX = Xp - Xm
            an = float((grad.conj() * dX).sum().real)
            Cp, Cm = fwd(Xp), fwd(Xm)
            st = float(((Cp + Cm - 2 * eye).conj() * fwd(dX)).sum().real)
            fd_stable = max(fd_stable, abs(st - an) / abs(an))
            Xp, Xm = X + 1e-3 * V, X - 1e-3 * V
            dX = Xp - Xm
            an = float((grad.conj() * dX).sum().real)
            fd_plain = max(fd_plain, abs(loss(fwd(Xp)) - loss(fwd(Xm)) - an) / abs(an))
    name = {1: "FP64 DMMA", 2: "Ozaki INT8", 3: "3xTF32"}[resolved]
    return {"metric": "ssb adjoint TFLOP/s (forward + backward, complex double)",
            "value": 3 * 8.0 * m * n * k / (ms / 1e3) / 1e12, "unit": "TFLOP/s",
            "ms_per_step": ms, "grad_rel_err_vs_torch_cublas": grad_err,
            "fd_central_h1e-6_cancellation_free_max_rel": fd_stable,
            "fd_central_h1e-3_plain_max_rel": fd_plain,
            "config": {"workload": "C = A^H B k=100000 m=n=512, L = ||C - I||_F^2, dA = B dC^H, "
                                   "dB = A dC (sbs kernels) via torch.autograd.Function",
                       "path": ("auto: " if path is None else "") + name}}


# The configurations of the benchmark suite beside the headline one, each run in
# its own process (its own device memory) after the headline line's figures are
# taken: (name, what it stands for).
SUITE = [("dssb", "pdgemm_ssb real double k=20000 m=n=256 (AUTO)"),
         ("sbs", "pzgemm_sbs subspace rotation mLocal=200000 n=k=2048 (AUTO)"),
         ("batch", "64 x pzgemm_ssb, one grouped persistent DMMA launch per sub-batch, autotuned"),
         ("batch_ozaki", "the same 64 instances on the Ozaki INT8 path"),
         ("batch_c64_tf32x3", "the 64 instances in complex float on 3xTF32"),
         ("adjoint", "ssb -> loss forward + backward, complex double k=100000 m=n=512 (AUTO)"),
         ("ssbtr_float", "psgemm_ssbtr lower real float k=400000 m=n=1536 (AUTO)")]


def _sig(x, digits=4):
    """x rounded to `digits` significant digits (floats only)."""
    if not isinstance(x, float) or x == 0.0 or x != x:
        return x
    return float(f"{x:.{digits}g}")


def compact_entry(res):
    """The figures of one suite entry that the headline line carries: metric,
    value, unit, time per step (or per batch), path, every error or check
    figure, the U[-1,1] figures of ssbtr; the full line is what
    `bench.py --workload NAME` prints."""
    out = {k: res[k] for k in ("metric", "unit") if k in res}
    for k in ("value", "ms_per_step", "ms_per_batch"):
        if k in res:
            out[k] = _sig(res[k])
    if "config" in res:
        out["path"] = res["config"].get("path")
    for k, v in res.items():
        if "err" in k or k.startswith("fd_"):
            out[k] = _sig(v, 3) if isinstance(v, float) else v
    if "uniform_inputs" in res:
        u = res["uniform_inputs"]
        out["uniform_inputs"] = {"value": _sig(u["value"]),
                                 "rel_err": _sig(u["rel_err_triangle_vs_double_double"], 3)}
    return out


def run_suite(steps, warmup, timeout_s=150, budget_s=360):
    """Runs each SUITE workload as `bench.py --workload NAME` in a child process
    and returns {name: its figures (compact_entry) or the failure, wall seconds}.
    A child gets at most timeout_s seconds and the suite budget_s in all (about
    80 s are needed on a B200); entries past the budget are skipped and say so,
    so that the headline line is printed in bounded time."""
    out = {}
    start = time.time()
    for name, _what in SUITE:
        t0 = time.time()
        left = budget_s - (t0 - start)
        if left < 10:
            out[name] = {"error": f"skipped: the suite's {budget_s} s budget is spent",
                         "wall_s": 0.0}
            continue
        limit = int(min(timeout_s, left))
        try:
            p = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--workload", name,
                                "--steps", str(steps), "--warmup", str(warmup)],
                               capture_output=True, text=True, timeout=limit)
            lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
            if p.returncode == 0 and lines:
                res = compact_entry(json.loads(lines[-1]))
            else:
                res = {"error": f"exit {p.returncode}: " + (p.stderr or p.stdout)[-400:]}
        except subprocess.TimeoutExpired:
            res = {"error": f"timed out after {limit} s"}
        res["wall_s"] = round(time.time() - t0, 1)
        out[name] = res
    return out


def workload_ssbtr_float(torch, spla, steps, warmup, path=None):
    """psgemm_ssbtr lower fill, real float, k = 400000, m = n = 1536, op = T:
    the headline figure on Gaussian/sqrt(k) operands, and the same call on
    U[-1, 1] operands reported beside it (timing and error)."""
    m = n = 1536
    k = 400000
    g = torch.Generator(device="cuda")
    g.manual_seed(20250006)
    C = torch.zeros((n, m), dtype=torch.float32, device="cuda")
    ctx = spla.Context(spla.PU_GPU)
    if path is not None:
        ctx.set_fp64_path(path)
    resolved = spla.lib().splab_gemm_path(0, spla.PATH_AUTO if path is None else path, 1, 0, m,
                                          n, k)
    dist = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128,
                                                             128)
    tri_mask = torch.tril(torch.ones((m, n), dtype=torch.bool, device="cuda")).T  # row >= col

    def measure(A, B):
        def step():
            spla.pgemm_ssbtr(m, n, k, spla.OP_TRANSPOSE, 1.0, A, k, B, k, 0.0, C, m, 0, 0,
                             spla.FILL_MODE_LOWER, dist, ctx)

        for _ in range(warmup):
            step()
        e0, e1 = _events(torch)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        # the whole lower triangle against the device double-double product
        R = torch.zeros((n, m), dtype=torch.float64, device="cuda")
        assert spla.gemm_dd(0, 1, 0, m, n, k, A, k, B, k, R, m) == 0
        torch.cuda.synchronize()
        diff = (C.double() - R)[tri_mask]
        return ms, float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(R[tri_mask]))

    s = (1.0 / k) ** 0.5
    A = torch.randn((m, k), dtype=torch.float32, device="cuda", generator=g) * s
    B = torch.randn((n, k), dtype=torch.float32, device="cuda", generator=g) * s
    ms, err = measure(A, B)
    A = torch.rand((m, k), dtype=torch.float32, device="cuda", generator=g) * 2 - 1
    B = torch.rand((n, k), dtype=torch.float32, device="cuda", generator=g) * 2 - 1
    ms_u, err_u = measure(A, B)
    tri = float(k) * m * (m + 1)
    name = {1: "FP64-accumulated DMMA", 2: "Ozaki INT8", 3: "3xTF32"}[resolved]
    return {"metric": "SGEMM-SSBTR TFLOP/s (lower triangle, real float)",
            "value": tri / (ms / 1e3) / 1e12, "unit": "TFLOP/s", "ms_per_step": ms,
            "full_matrix_tflops": 2.0 * m * n * k / (ms / 1e3) / 1e12,
            "rel_err_triangle_vs_double_double": err,
            "uniform_inputs": {"value": tri / (ms_u / 1e3) / 1e12, "ms_per_step": ms_u,
                               "rel_err_triangle_vs_double_double": err_u,
                               "data": "A, B U[-1,1]"},
            "config": {"workload": "psgemm_ssbtr m=n=1536 k=400000 lower, op=T, "
                                   "Gaussian/sqrt(k)",
                       "path": ("auto: " if path is None else "") + name}}


def workload_cgemm_ssb(torch, spla, steps, warmup, path=None):
    """pcgemm_ssb complex float, A^H B, k = 250000, m = n = 1024, complex
    Gaussian/sqrt(k) (the complex-double ssb configuration in single
    precision), full C, beta = 0."""
    m = n = 1024
    k = 250000
    g = torch.Generator(device="cuda")
    g.manual_seed(20250007)
    s = (1.0 / (2 * k)) ** 0.5
    A = (torch.randn((m, k), dtype=torch.complex64, device="cuda", generator=g) * s).contiguous()
    B = (torch.randn((n, k), dtype=torch.complex64, device="cuda", generator=g) * s).contiguous()
    C = torch.zeros((n, m), dtype=torch.complex64, device="cuda")
    ctx = spla.Context(spla.PU_GPU)
    if path is not None:
        ctx.set_fp64_path(path)
    dist = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128,
                                                             128)

    def step():
        spla.pgemm_ssb(m, n, k, spla.OP_CONJ_TRANSPOSE, 1.0, A, k, B, k, 0.0, C, m, 0, 0, dist,
                       ctx)

    for _ in range(warmup):
        step()
    e0, e1 = _events(torch)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    R = torch.zeros((n, m), dtype=torch.complex128, device="cuda")
    assert spla.gemm_dd(2, 2, 0, m, n, k, A, k, B, k, R, m) == 0
    torch.cuda.synchronize()
    err = float(torch.linalg.vector_norm(C.to(torch.complex128) - R) /
                torch.linalg.vector_norm(R))
    flops = 8.0 * m * n * k
    return {"metric": "CGEMM-SSB TFLOP/s (complex float, A^H B)",
            "value": flops / (ms / 1e3) / 1e12, "unit": "TFLOP/s", "ms_per_step": ms,
            "rel_err_whole_c_vs_double_double": err,
            "config": {"workload": "pcgemm_ssb m=n=1024 k=250000 op=C",
                       "path": {None: "auto", 1: "FP64-accumulated DMMA", 2: "Ozaki INT8",
                                3: "3xTF32"}[path]}}


def workload_gemm_ops(torch, spla, steps, warmup, opA, opB, path=None):
    """Local spla_zgemm, C = op(A) op(B), complex double, m = n = 1024,
    k = 250000 (the headline's size), Gaussian/sqrt(k) operands stored as each
    op requires (op N: A is m x k, B is k x n; op T/C: A is k x m, B is n x k),
    beta = 0, on the context's path (AUTO by default); error on the whole C
    against the device double-double product."""
    m = n = 1024
    k = 250000
    g = torch.Generator(device="cuda")
    g.manual_seed(20250010 + 3 * opA + opB)
    s = (1.0 / (2.0 * k)) ** 0.5
    A = torch.randn(m * k, dtype=torch.complex128, device="cuda", generator=g) * s
    B = torch.randn(n * k, dtype=torch.complex128, device="cuda", generator=g) * s
    lda = m if opA == 0 else k
    ldb = k if opB == 0 else n
    C = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    ctx = spla.Context(spla.PU_GPU)
    if path is not None:
        ctx.set_fp64_path(path)
    resolved = spla.lib().splab_gemm_path(3, spla.PATH_AUTO if path is None else path, opA, opB,
                                          m, n, k)

    def step():
        spla.gemm(opA, opB, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, m, ctx)

    for _ in range(warmup):
        step()
    e0, e1 = _events(torch)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    R = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    assert spla.gemm_dd(3, opA, opB, m, n, k, A, lda, B, ldb, R, m) == 0
    torch.cuda.synchronize()
    err = float(torch.linalg.vector_norm(C - R) / torch.linalg.vector_norm(R))
    ops = "NTC"
    name = {1: "FP64 DMMA", 2: "Ozaki INT8", 3: "3xTF32"}[resolved]
    return {"metric": f"ZGEMM TFLOP/s (spla_zgemm op(A)={ops[opA]} op(B)={ops[opB]}, {name})",
            "value": 8.0 * m * n * k / (ms / 1e3) / 1e12, "unit": "TFLOP/s", "ms_per_step": ms,
            "rel_err_whole_c_vs_double_double": err,
            "config": {"workload": f"spla_zgemm {ops[opA]}{ops[opB]} m=n=1024 k=250000",
                       "path": ("auto: " if path is None else "") + name}}


def workload_batch(torch, spla, steps, warmup, dtype="complex128", count=64, sub=32, path=None):
    """64 ssb instances, k ~ U{120000..180000}, m = n ~ U{512, 768, 1024}
    (seeded draw order: k then m per instance), Gaussian/sqrt(k); run as
    sub-batches of `sub` instances (the complex-double operands of all 64,
    ~236 GB, exceed HBM). path None/1: each sub-batch one persistent grouped
    DMMA launch replayed from a CUDA graph with the autotuned k-chunk; path 2
    (Ozaki) / 3 (3xTF32): the instances in sequence, replayed from a graph."""
    import numpy as np
    rng = np.random.default_rng(20250004)
    shapes = []
    for _ in range(count):
        k = int(rng.integers(120000, 180001))
        m = int(rng.choice([512, 768, 1024]))
        shapes.append((m, m, k))
    tdt = getattr(torch, dtype)
    total_flops = sum(8.0 * m * n * k for (m, n, k) in shapes)
    total_ms = 0.0
    tuning = []
    for b0 in range(0, count, sub):
        part = shapes[b0:b0 + sub]
        g = torch.Generator(device="cuda")
        g.manual_seed(20250004 + b0)
        probs = []
        keep = []
        for (m, n, k) in part:
            s = (1.0 / (2.0 * k)) ** 0.5
            A = torch.randn((m, k), dtype=tdt, device="cuda", generator=g) * s
            B = torch.randn((n, k), dtype=tdt, device="cuda", generator=g) * s
            C = torch.empty((n, m), dtype=tdt, device="cuda")
            keep += [A, B, C]
            probs.append(dict(opA=2, opB=0, m=m, n=n, k=k, A=A, lda=k, B=B, ldb=k, C=C, ldc=m,
                              alpha=1.0, beta=0.0))
        batch = spla.Batch(dtype, probs, path=path)
        ws = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")
        batch.run(ws, autotune=True)
        for _ in range(max(0, warmup - 1)):
            batch.run(ws)
        torch.cuda.synchronize()
        e0, e1 = _events(torch)
        e0.record()
        for _ in range(steps):
            batch.run(ws)
        e1.record()
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1) / steps
        batch.check(ws)
        tuning.append(batch.info())
        # accuracy of one instance against torch (FP64 reference on the GPU)
        if b0 == 0:
            A, B, C = keep[0], keep[1], keep[2]
            m0, n0, k0 = part[0]
            ref = torch.zeros((n0, m0), dtype=torch.complex128, device="cuda")
            assert spla.gemm_dd(2 if dtype == "complex64" else 3, 2, 0, m0, n0, k0, A, k0, B, k0,
                                ref, m0) == 0
            torch.cuda.synchronize()
            err = float((C.to(torch.complex128) - ref).norm() / ref.norm())
        del batch, ws, keep, probs
        torch.cuda.empty_cache()
    return {"metric": f"batched grouped ZGEMM-SSB TFLOP/s ({dtype})",
            "value": total_flops / (total_ms / 1e3) / 1e12, "unit": "TFLOP/s",
            "ms_per_batch": total_ms, "instances": count, "sub_batch": sub,
            "rel_err_instance0_vs_double_double": err, "autotune": tuning,
            "config": {"workload": "64 x pgemm_ssb k~U{120000..180000} m=n~{512,768,1024}",
                       "path": {None: "DMMA grouped persistent + CUDA graph",
                                1: "DMMA grouped persistent + CUDA graph",
                                2: "Ozaki INT8, instances in sequence, CUDA graph",
                                3: "3xTF32, instances in sequence, CUDA graph"}[path]}}


def run_workload(name, steps, warmup):
    import torch
    import spla_b200 as spla
    torch.cuda.set_device(0)
    fn = {"dssb": workload_dssb,
          "adjoint": workload_adjoint,
          "sbs": workload_sbs,
          "sbs_dmma": lambda t, s, st, w: workload_sbs(t, s, st, w, 1),
          "sbs_ozaki": lambda t, s, st, w: workload_sbs(t, s, st, w, 2),
          "ssbtr_float": workload_ssbtr_float,
          "ssbtr_float_dmma": lambda t, s, st, w: workload_ssbtr_float(t, s, st, w, 1),
          "ssbtr_float_ozaki": lambda t, s, st, w: workload_ssbtr_float(t, s, st, w, 2),
          "ssbtr_float_tf32x3": lambda t, s, st, w: workload_ssbtr_float(t, s, st, w, 3),
          "cgemm_ssb_dmma": lambda t, s, st, w: workload_cgemm_ssb(t, s, st, w, 1),
          "cgemm_ssb_ozaki": lambda t, s, st, w: workload_cgemm_ssb(t, s, st, w, 2),
          "cgemm_ssb_tf32x3": lambda t, s, st, w: workload_cgemm_ssb(t, s, st, w, 3),
          "zgemm_nn": lambda t, s, st, w: workload_gemm_ops(t, s, st, w, 0, 0),
          "zgemm_nt": lambda t, s, st, w: workload_gemm_ops(t, s, st, w, 0, 1),
          "zgemm_cn": lambda t, s, st, w: workload_gemm_ops(t, s, st, w, 2, 0),
          "zgemm_cc": lambda t, s, st, w: workload_gemm_ops(t, s, st, w, 2, 2),
          "batch": workload_batch,
          "batch_c64": lambda t, s, st, w: workload_batch(t, s, st, w, "complex64", 64, 64),
          "batch_ozaki": lambda t, s, st, w: workload_batch(t, s, st, w, "complex128", 64, 32, 2),
          "batch_c64_ozaki": lambda t, s, st, w: workload_batch(t, s, st, w, "complex64", 64, 64,
                                                                2),
          "batch_c64_tf32x3": lambda t, s, st, w: workload_batch(t, s, st, w, "complex64", 64,
                                                                 64, 3)}[name]
    line = fn(torch, spla, steps, warmup)
    line.update({"n_gpus": 1, "steps": steps, "warmup": warmup, "higher_is_better": True,
                 "data": "synthetic, seeded"})
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--paths", default="dmma,ozaki")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-peaks", action="store_true")
    ap.add_argument("--no-suite", action="store_true",
                    help="skip the other configurations (run by default at one GPU)")
    ap.add_argument("--m", type=int, default=1024, help="m = n (profiling of smaller cases)")
    ap.add_argument("--k", type=int, default=250000, help="k (profiling of smaller cases)")
    ap.add_argument("--workload", default="zgemm_ssb",
                    choices=["zgemm_ssb", "dssb", "adjoint", "sbs", "sbs_dmma", "sbs_ozaki",
                             "ssbtr_float",
                             "ssbtr_float_dmma",
                             "ssbtr_float_ozaki", "ssbtr_float_tf32x3", "cgemm_ssb_dmma",
                             "cgemm_ssb_ozaki", "cgemm_ssb_tf32x3", "zgemm_nn", "zgemm_nt",
                             "zgemm_cn", "zgemm_cc", "batch", "batch_c64",
                             "batch_ozaki", "batch_c64_ozaki", "batch_c64_tf32x3"])
    args = ap.parse_args()
    if args.workload != "zgemm_ssb" and args.impl == "ours":
        return run_workload(args.workload, args.steps, max(3, args.warmup))
    set_shape(args.m, args.k)
    warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        value, ms, info = cpu_reference_run(args.steps, args.warmup)
        line = {"metric": HEADLINE_METRIC, "value": value, "unit": "TFLOP/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "impl": "reference", "dtype": "complex128 (f64)",
                "data": "synthetic: complex Gaussian / sqrt(k), seeded",
                "config": {"workload": workload_name(), "path": "reference CPU path (BLAS)",
                           "sample": info["sample"]},
                "cpu_baseline": {"value": value, "unit": "TFLOP/s", **info},
                "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}, "vs_baseline": None}
        print(json.dumps(line))
        return

    import torch
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import spla_b200 as spla
    if not spla.LIB_PATH.exists():
        from spla_b200.build import build
        build()

    A, B = make_inputs(torch, device)
    peaks = {} if args.no_peaks else measured_peaks(torch, device)
    names = {"dmma": spla.PATH_DMMA, "ozaki": spla.PATH_OZAKI}
    results = {}
    with ClockSampler(local) as clk:
        for pname in [p for p in args.paths.split(",") if p]:
            try:
                dC, ms, phases = time_device_path(torch, spla, names[pname], A, B, args.steps,
                                                  warmup, rank)
            except RuntimeError as ex:
                results[pname] = {"error": str(ex)}
                continue
            ms = max_over_ranks(torch, ms, device)
            # phases 3..14 are per-launch INT8 GEMM times (Ozaki; unused ones read
            # ~0), 15..18 the parts of the slicing phase
            parts = dict(zip(["a_copy", "norms", "residues_a", "residues_b"], phases[15:19]))
            phases = phases[:3] + [x for x in phases[3:15] if x > 0.05]
            results[pname] = {"ms_per_step": ms, "tflops": whole_job_tflops(FLOPS, world, ms),
                              "phase_ms": phases, "dC": dC}
            if pname == "ozaki":
                results[pname]["slicing_parts_ms"] = parts
    clocks_by_path = {p: clk.summary(names[p]) for p in results}
    for p in results:  # the sampling note once, in the line's own clocks
        c = clocks_by_path[p]
        results[p]["clocks"] = {k: v for k, v in c.items() if k != "sampling"} if c else c
    # accuracy on the whole C against the device double-double reference, which is
    # itself checked against the CPU Dot2 oracle on three columns
    R = dd_reference(torch, spla, A, B)
    dd_check = rel_err_sampled(R, A, B) if rank == 0 and not args.no_cpu else None
    for pname, r in results.items():
        if "dC" in r:
            r["rel_err_vs_oracle"] = rel_err_full(torch, r.pop("dC"), R)
            r["rel_err_scope"] = "whole C vs the device double-double reference (splab_gemm_dd)"

    # headline: Ozaki if it ran and met the accuracy bar (checked on rank 0 and
    # broadcast, so that every rank takes the same steps), else DMMA
    head = "dmma"
    oz = results.get("ozaki", {})
    if "tflops" in oz and oz.get("rel_err_vs_oracle") is not None and oz["rel_err_vs_oracle"] <= 1e-14:
        head = "ozaki"
    if world > 1:
        flag = torch.tensor([1 if head == "ozaki" else 0], device=device)
        torch.distributed.broadcast(flag, 0)
        head = "ozaki" if int(flag.item()) else "dmma"
    hr = results[head]
    head_path = names[head]
    clocks = clocks_by_path.get(head)

    e2e = None
    hA = hB = None
    if not args.no_e2e:
        ms_e2e, hC, hA, hB = e2e_public_api(torch, spla, head_path, A, B,
                                            max(1, min(args.steps, 3)), 1)
        ms_e2e = max_over_ranks(torch, ms_e2e, device)
        e2e = {"value": whole_job_tflops(FLOPS, world, ms_e2e), "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(16 * K * (M + N)), "d2h_bytes_per_step": int(16 * M * N),
               "ms_per_step": ms_e2e, "operands": "pinned host memory, streamed in k-chunks",
               "rel_err_vs_oracle": rel_err_full(torch, hC, R),
               "rel_err_scope": "whole C of the last timed call vs the device double-double "
                                "reference"}
    del R

    if rank != 0:
        torch.distributed.destroy_process_group() if world > 1 else None
        return

    # roofline of the dominant kernel
    if head == "dmma":
        k_ms = hr["phase_ms"][0] or hr["ms_per_step"]
        achieved = FLOPS / (k_ms / 1e3) / 1e12
        peak = peaks.get("fp64_tflops")
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None, "traffic": None,
                "kernel": "dmma_gemm_kernel (mma.sync f64)",
                "peak_source": "measured here: cuBLAS DGEMM 8192^3 via torch.matmul float64"}
        launches = 2 * args.steps
    else:
        gemm_launch_ms = hr["phase_ms"][3:]
        k_ms = sum(gemm_launch_ms) or hr["phase_ms"][1] or hr["ms_per_step"]
        nmod = OZAKI_MODULI
        # residue GEMMs: three real products of m x n x k per modulus (complex)
        int8_ops = 2.0 * nmod * 3 * M * N * K
        achieved = int8_ops / (k_ms / 1e3) / 1e12
        peak = peaks.get("int8_tops")
        # DRAM bytes of one GEMM launch: 1.286 x the algorithmic residue bytes, the ratio of
        # an ncu capture of oz_gemm_pair on the same tiling with a shorter k (m = n = 1024,
        # k = 40000: 4.745 GB for 3.692 GB of residues), scaled by the k-blocks processed
        alg_bytes = float(OZAKI_MODULI) * 3 * (M + N) * ((K + 127) // 128 * 128)
        traffic = 1.286 * alg_bytes if (M, N) == (1024, 1024) else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)",
                "frac": (achieved / peak) if peak else None, "traffic": traffic,
                "traffic_source": "ncu dram__bytes_{read,write}.sum of oz_gemm_pair on "
                                  "m=n=1024 k=40000 (same tiles, one k-chunk), 1.286 x the "
                                  "residue bytes, scaled to this launch by its k-blocks "
                                  "(profiles/oz_gemm_pair_int8_traffic_zgemm_m1024_k40000.md)",
                "algorithmic_residue_bytes": float(OZAKI_MODULI) * 3 * (M + N) * K,
                "kernel": "oz_gemm_pair (tcgen05.mma.cta_group::2.kind::i8, TMA, TMEM)",
                "peak_source": "measured here: cuBLASLt int8 GEMM 8192^3 via torch._int_mm",
                "algorithmic_ops_per_launch": int8_ops}
        groups = max(1, len(gemm_launch_ms))
        # 2 row-scale, 2 slice and 1 GEMM per modulus group, 1 reconstruct
        launches = (3 + 3 * groups) * args.steps
        roof["gemm_launches_per_step"] = groups
        roof["note"] = ("achieved = INT8 ops / summed duration of the GEMM launches; with "
                        "modulus groups those launches overlap the slicing of the next group")
        hr["phase_ms"] = hr["phase_ms"][:3] + gemm_launch_ms
        hr["phase_ms_names"] = (["scale+slice (span)", "int8 GEMM (span)", "reconstruct"] +
                                [f"int8 GEMM group {i}" for i in range(len(gemm_launch_ms))])

    cpu = None
    if not args.no_cpu and world >= 1:
        # the reference's CPU path on the same workload: 1 warm-up + 3 full calls
        # (about 10 s on 16 host cores), on the pinned host copies of A and B
        v, ms_cpu, info = cpu_reference_run(
            3, 1, None if hA is None else hA.numpy().ravel(),
            None if hB is None else hB.numpy().ravel())
        cpu = {"value": v, "unit": "TFLOP/s", "ms_per_call": ms_cpu, **info}
    if dd_check is not None:
        hr["dd_reference_vs_cpu_dot2_3cols"] = dd_check

    suite = None
    if world == 1 and not args.no_suite and (M, N, K) == (1024, 1024, 250000):
        # the other configurations, each in a child process with the device memory
        # of this one released first
        del A, B
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        suite = run_suite(min(args.steps, 5), 3)

    line = {
        "metric": HEADLINE_METRIC,
        "value": hr["tflops"], "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": warmup, "ms_per_step": hr["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
        "data": "synthetic: complex Gaussian / sqrt(k), seeded",
        "config": {"workload": workload_name(), "path": head,
                   "l2": "inputs (8.2 GB) larger than L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "paths": {k: {kk: vv for kk, vv in v.items()} for k, v in results.items()},
        "roofline": roof, "peaks_measured": peaks, "e2e": e2e, "cpu_baseline": cpu,
        "clocks": clocks, "gpu_launches": launches,
    }
    if suite is not None:
        line["suite"] = suite
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
