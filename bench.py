"""Benchmark of the sparse iterative-solver path on B200.

Headline metric: time to an FP64-checked relative residual of 1e-6 on the
512x512 log-normal diffusion set (2D 5-point, sigma 1.5, correlation length
16; held-out seeds), for the solver named in config.solver, with the plain
FP32 CG drop-in timed beside it on the same systems.  One step = one solve of
one system whose CSR is already resident in HBM; L2 is flushed between steps.

Also measured in the same run (reported, not the headline):
  * spmv: CSR SpMV GB/s on the 256^3 7-point diffusion operator (1.14 GB per
    SpMV, larger than L2) -- the HBM-bound kernel whose roofline is reported;
  * e2e: the same metric through the drop-in API with host buffers --
    spmv.csr_tensor(keys, values, ...) from pinned host COO (GPU sort) and
    cgd(b, x) with pinned host b/x, every copy inside the timed region;
  * cpu_baseline: the CPU oracle's CG on the box's host cores (bounded sample)
    and scipy.sparse.linalg.cg beside it.

  * configs: the other configurations at full size, every answer checked by
    its FP64 true residual -- C1 CG on the 256^2 Laplacian (iterations
    against the FP64 oracle, scipy cg on the host), C2 BiCGSTAB on the BCSR
    4x4 system with 65,536 block rows (BCSR SpMV GB/s, scipy bicgstab), C3
    mixed-precision CG to 1e-10 with FP32 and BF16 values and plain FP32 CG
    on the 256^3 operator, with the error against the FP64 oracle on its
    64^3 member.

`--impl reference` times the reference algorithm's CPU implementation (the
oracle port of iterative/BiCGSTAB/spmv.cpp cgd_op, FP64, every solve run to
convergence) on the host cores; it never loads this package's CUDA code.
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

METRIC = "time-to-1e-6-residual"
UNIT = "ms"
WORKLOAD = "512x512 log-normal diffusion (2D 5-pt, sigma 1.5, corr 16), held-out seeds"
TEST_SEED0 = 100_000        # held-out seeds start here (training uses 0..1999)
TOL = 1e-6
# C1 (256^2 Laplacian, n 65,536, nnz 326,656): bytes of one CG iteration in
# the reference's schedule, SpMV 3,399,684 + 36 n
C1_ITER_BYTES = 3_399_684 + 36 * 65_536
MAX_ITER = 40_000


def _workloads():
    """The seeded generators (mpsparse_b200/workloads.py, numpy only) loaded
    by file path, so the CPU arms never import the package (whose import
    loads the CUDA extension)."""
    import importlib.util
    name = "mpsparse_b200_workloads"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "mpsparse_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def host_info():
    """Host cores and thread settings the CPU numbers ran with."""
    info = {"affinity_cores": host_threads(), "cpu_count": os.cpu_count()}
    for k in ("OMP_NUM_THREADS", "MKL_NUM_THREADS", "OPENBLAS_NUM_THREADS"):
        info[k] = os.environ.get(k)
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    info["cpu_model"] = line.split(":", 1)[1].strip()
                    break
    except Exception:
        pass
    try:
        from threadpoolctl import threadpool_info
        info["blas"] = [{"lib": t.get("internal_api"), "threads": t.get("num_threads")}
                        for t in threadpool_info()]
    except Exception:
        pass
    return info


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """SM clock, max clock, power and clock-event reasons of the GPU the run
    uses, sampled every 200 ms in a background thread through NVML (queries
    of the driver that do not stall the CUDA stream the way a polling
    nvidia-smi process does); nvidia-smi is the fallback."""
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, dev: int):
        self.dev = dev
        self.rows = []
        self.stop = threading.Event()
        self.thread = None
        self.proc = None
        self.path = None

    def _bus_id(self):
        import torch
        p = torch.cuda.get_device_properties(self.dev)
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"

    def _nvml_loop(self, nv, h):
        while not self.stop.is_set():
            try:
                self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                  nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                                  nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByPciBusId(self._bus_id().encode())
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self._bus_id(), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.active", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.thread is not None:
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            for line in open(self.path):
                parts = [q.strip() for q in line.split(",")]
                try:
                    self.rows.append((float(parts[0]), float(parts[1]), int(parts[2], 16)))
                except Exception:
                    pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        mx = max(r[1] for r in self.rows)
        reasons = sorted({name for r in self.rows for name, bit in self.REASONS if r[2] & bit})
        load = [v for v in sm if v > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.rows), "source": "nvml" if self.proc is None else "nvidia-smi"}


# ------------------------------------------------------------- systems -----
def c4_system(seed):
    W = _workloads()
    coo = W.diffusion_512sq(seed).shuffled(seed + 1)
    b = W.rhs(coo.n, seed + 2)
    return coo, b


def true_residual_gpu(A_csr, b, x):
    """FP64 ||b - A x|| / ||b|| on the GPU (verification only, untimed)."""
    import torch
    rp, ci, v = A_csr
    M = torch.sparse_csr_tensor(rp.long(), ci.long(), v.double(), (b.numel(), b.numel()))
    r = b.double() - (M @ x.double().unsqueeze(1)).squeeze(1)
    return float(r.norm() / b.double().norm())


def flush_l2(buf):
    buf.add_(1.0)


# ------------------------------------------------------------- our arm -----
def run_ours(args, rank, world, dev):
    import torch
    import mpsparse_b200 as mps
    torch.cuda.set_device(dev)
    steps, warm = args.steps, args.warmup
    nsys = steps + warm
    seeds = [TEST_SEED0 + rank * 10_000 + i for i in range(nsys)]
    systems = []
    e = torch.empty(0)
    for s in seeds:
        coo, b = c4_system(s)
        A = mps.spmv.csr_tensor(torch.from_numpy(coo.keys()), torch.from_numpy(coo.vals), e, e, e,
                                coo.n, coo.n, fill_outputs=False)
        systems.append((coo, A, torch.from_numpy(b).cuda()))
    n = systems[0][0].n
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2
    stream = torch.cuda.current_stream()

    # Solution buffers are the caller's (the API solves into x in place);
    # they are allocated once per system and leg, outside the timed steps,
    # so a step times the solve, not the allocator (every solver starts from
    # x = 0 and overwrites all of x).
    xbuf = {leg: [torch.zeros(n, dtype=dt, device=dev) for _ in systems]
            for leg, dt in (("plain", torch.float32), ("jacobi", torch.float32),
                            ("jacobi_mixed", torch.float64), ("learned", torch.float64))}

    def solve_plain(i):
        coo, A, b = systems[i]
        x = xbuf["plain"][i]
        info = A.cgd(b, x, tol=TOL, max_iter=args.max_iter, host_loop=args.host_loop)
        return x, info

    def solve_jacobi(i):
        coo, A, b = systems[i]
        x = xbuf["jacobi"][i]
        info = A.cgd(b, x, tol=TOL, max_iter=args.max_iter, precond="jacobi", host_loop=args.host_loop)
        return x, info

    b64 = [s[2].double() for s in systems]

    def solve_jacobi_mixed(i):
        # Jacobi-PCG with the learned solve's precision scheme (FP64 x,
        # residual replacement, FP64-checked stop): the like-for-like baseline
        coo, A, b = systems[i]
        x = xbuf["jacobi_mixed"][i]
        info = A.cg_mixed(b64[i], x, tol=TOL, inner_tol=args.inner_tol, max_inner=args.max_iter,
                          precond="jacobi", host_loop=args.host_loop)
        return x, {"iters": info["inner_iters"], "converged": info["converged"],
                   "rel_resid": info["rel_resid"], "persistent": bool(info["persistent"])}

    def solve_learned(i):
        coo, A, b = systems[i]
        fsai.attach(A)                     # network forward -> G on this system
        x = xbuf["learned"][i]
        info = A.cg_mixed(b64[i], x, tol=TOL, inner_tol=args.inner_tol, max_inner=args.max_iter,
                          precond="fsai", host_loop=args.host_loop)
        return x, {"iters": info["inner_iters"], "outer": info["outer_iters"],
                   "converged": info["converged"], "rel_resid": info["rel_resid"],
                   "form": A.fsai_apply()["form"], "persistent": bool(info["persistent"])}

    if args.solver == "learned":
        from mpsparse_b200.fsai import LearnedFsai, DEFAULT_WEIGHTS
        fsai = LearnedFsai.load(DEFAULT_WEIGHTS)
        headline = solve_learned
        solver_name = "learned-FSAI mixed-precision PCG (FP32 inner PCG, FP64 outer IR)"
    else:
        headline = solve_plain
        solver_name = "plain FP32 CG (drop-in cgd)"

    host_ms = {}

    def timed(fn):
        times, infos, xs, hms = [], [], [], []
        for i in range(nsys):
            flush_l2(flush)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            h0 = time.perf_counter()
            ev0.record(stream)
            x, info = fn(i)
            ev1.record(stream)
            h1 = time.perf_counter()
            torch.cuda.synchronize()
            if i >= warm:
                times.append(ev0.elapsed_time(ev1))
                infos.append(info)
                xs.append(x)
                hms.append(round((h1 - h0) * 1e3, 3))
        # host time from recording the first event to recording the last: a
        # step whose device time exceeds its kernels' time by a host stall
        # (the process descheduled between launches) shows it here too
        host_ms[fn.__name__] = hms
        return times, infos, xs

    # per-handle setup (workspace, CUDA-graph capture, the FSAI pattern and
    # features) happens on a handle's first solve: do it for every system
    # before the timed region; time it on the first system
    setup_ms = None
    for i in range(nsys):
        t0 = time.perf_counter()
        headline(i)
        torch.cuda.synchronize()
        if i == 0:
            setup_ms = (time.perf_counter() - t0) * 1e3
        solve_plain(i)
        solve_jacobi(i)
        solve_jacobi_mixed(i)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        time.sleep(0.5)                       # let the sampler start before timing
        t_wall0 = time.perf_counter()
        torch.cuda.nvtx.range_push("timed")   # profilers can filter on this range
        times, infos, xs = timed(headline)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        t_wall = time.perf_counter() - t_wall0
        if world > 1:
            torch.distributed.barrier()
        # plain CG and Jacobi-PCG on the same systems (the comparison the metric names)
        ptimes, pinfos, pxs = timed(solve_plain)
        jtimes, jinfos, jxs = timed(solve_jacobi)
        jmtimes, jminfos, _ = timed(solve_jacobi_mixed)
    clocks = clk.summary()
    # verification (untimed): FP64 true residual of every timed solve
    resid = []
    for k, x in enumerate(xs):
        coo, A, b = systems[warm + k]
        resid.append(true_residual_gpu(A.csr(), b, x))
    presid = [true_residual_gpu(systems[warm + k][1].csr(), systems[warm + k][2], x)
              for k, x in enumerate(pxs)]

    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    iters = [i["iters"] for i in infos]
    if args.solver == "learned":
        # per solve: attach (network forward, value map, G^T gather, G^T G
        # values in product form, the error-word fold) + ||b||^2 + init + per iteration 2
        # kernels (product form: direction + A p, update + M r) or 3 (split:
        # A p, update + G r, G^T w) + 2 per residual replacement + the FP64
        # true residual at the end; the product form's graph runs 16
        # iterations per loop body, so after each replacement (and at the
        # stop) about 7.5 iterations' kernels return at once: 15 launches
        def per_solve(i):
            if i.get("persistent"):
                # attach (forward, value map, G^T gather, G^T G values, the
                # network's error word folded into the handle's), ||b||^2,
                # the persistent solve, the FP64 true residual
                return 5 + 1 + 1 + 1
            if i.get("form") == "product":
                rounds = max(i["outer"], 1)
                return 5 + 1 + 2 + 2 * i["iters"] + 2 * rounds + 15 * rounds + 1
            return 4 + 1 + 3 + 3 * i["iters"] + 2 * i["outer"] + 1
        launches = sum(per_solve(i) for i in infos)
    else:
        launches = sum(2 + 3 * i["iters"] for i in infos)   # init + 3 kernels/iteration + copy

    ptrue = [i.get("true_resid", -1.0) for i in pinfos]
    out = {
        "solver": solver_name,
        "ms_per_solve": total_ms / steps,
        "value": total_ms / (steps * world),
        "iters_mean": statistics.mean(iters),
        "true_resid_max": max(resid),
        "step_ms": [round(t, 3) for t in times],
        "step_host_ms": host_ms.get(headline.__name__),
        "plain_cg": {"ms_per_solve": statistics.mean(ptimes), "step_ms": [round(t, 3) for t in ptimes],
                     "iters_mean": statistics.mean(i["iters"] for i in pinfos),
                     "true_resid_max": max(presid),
                     "true_resid_max_reported": max(ptrue),
                     "stop_rule_met": sum(bool(i["stop_rule_met"]) for i in pinfos),
                     "converged_fp64": sum(bool(i["converged"]) for i in pinfos),
                     "note": "FP32 CG stops on its recurrence residual; the FP64 true residual of "
                             "the FP32 x it returns stays above 1e-6 on these systems, so its "
                             "time is a lower bound on a time to 1e-6"},
        "jacobi_pcg": {"ms_per_solve": statistics.mean(jtimes), "step_ms": [round(t, 3) for t in jtimes],
                       "iters_mean": statistics.mean(i["iters"] for i in jinfos),
                       "true_resid_max": max(i.get("true_resid", -1.0) for i in jinfos)},
        "jacobi_pcg_mixed": {"ms_per_solve": statistics.mean(jmtimes),
                             "step_ms": [round(t, 3) for t in jmtimes],
                             "iters_mean": statistics.mean(i["iters"] for i in jminfos),
                             "true_resid_max": max(i["rel_resid"] for i in jminfos),
                             "converged_fp64": sum(bool(i["converged"]) for i in jminfos),
                             "persistent": all(i["persistent"] for i in jminfos)},
        "outer_mean": statistics.mean(i.get("outer", 0) for i in infos),
        "setup_ms_first_solve": setup_ms,
        "clocks": clocks, "gpu_launches": launches, "wall_s": t_wall,
    }
    out["e2e"] = e2e_drop_in(args, systems, dev, warm, steps,
                             fsai if args.solver == "learned" else None)
    out["e2e_plain_cg"] = (e2e_drop_in(args, systems, dev, warm, steps, None)
                           if args.solver == "learned" and not args.skip_e2e_plain else None)
    single = world == 1
    out["mlp"] = mlp_leg(systems[0][1], dev) if args.solver == "learned" and single else None
    c3 = C3Context(args, dev) if single and not (args.skip_spmv and args.skip_configs) else None
    out["spmv"] = spmv_c3(args, dev, c3) if single and not args.skip_spmv else None
    out["batched"] = batched_c5(args, dev, rank, world) if not args.skip_batched else None
    out["configs"] = configs_legs(args, dev, c3) if single and not args.skip_configs else None
    return out


def learned_only(args, dev):
    """The headline solve alone (attach the learned factor, mixed-precision
    FSAI-PCG to 1e-6) on warmup + steps held-out 512^2 systems, CUDA events
    per solve: a short command for profilers."""
    import torch
    import mpsparse_b200 as mps
    from mpsparse_b200.fsai import LearnedFsai
    fsai = LearnedFsai.load()
    e = torch.empty(0)
    stream = torch.cuda.current_stream()
    out = {"ms": [], "iters": [], "persistent": []}
    for i in range(args.warmup + args.steps):
        coo, b = c4_system(TEST_SEED0 + i)
        A = mps.spmv.csr_tensor(torch.from_numpy(coo.keys()), torch.from_numpy(coo.vals), e, e, e,
                                coo.n, coo.n, fill_outputs=False)
        b64 = torch.from_numpy(b).double().to(dev)
        for rep in range(2):                 # the second solve is timed (graph / plan set-up done)
            x = torch.zeros(coo.n, dtype=torch.float64, device=dev)
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fsai.attach(A)
            info = A.cg_mixed(b64, x, tol=TOL, inner_tol=args.inner_tol, max_inner=args.max_iter,
                              precond="fsai")
            z.record(stream)
            torch.cuda.synchronize()
        if i >= args.warmup:
            out["ms"].append(a.elapsed_time(z))
            out["iters"].append(info["inner_iters"])
            out["persistent"].append(bool(info["persistent"]))
    return out


def mlp_leg(A, dev):
    """The learned factor's network on the tensor cores: forward and backward
    passes over the features of a 512^2 system's G (785,408 nonzeros = rows
    of the network), BF16 features resident on the GPU, CUDA events per
    launch.  FLOPs: 2 (16*64 + 64*64 + 64) = 10,368 per row forward; the
    backward pass (forward recomputed) counted as 3x that."""
    import torch
    from mpsparse_b200.fsai import LearnedFsai
    m = LearnedFsai.load().model
    X = A.fsai_features()[0]
    Xb = X.to(torch.bfloat16).contiguous()
    N = Xb.shape[0]
    out = torch.empty(N, device=dev)
    dout = torch.randn(N, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
    grad = torch.empty(5313, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(3):
        m.forward_bf16(Xb, out)
        m.backward_bf16(Xb, dout, grad)
    m.status()
    fwd = _event_ms(lambda: m.forward_bf16(Xb, out), stream, 20)
    bwd = _event_ms(lambda: m.backward_bf16(Xb, dout, grad), stream, 20)
    m.status()
    f_fwd, f_bwd = 10368.0 * N, 3 * 10368.0 * N
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except Exception:
        pass
    tf = lambda fl, ms: fl / (ms * 1e-3) / 1e12
    return {"rows": N, "forward_us": fwd * 1e3, "forward_tflops": tf(f_fwd, fwd),
            "backward_us": bwd * 1e3, "backward_tflops": tf(f_bwd, bwd),
            "bf16_peak_tflops": peak,
            "forward_frac_of_bf16_peak": tf(f_fwd, fwd) / peak if peak else None,
            "note": "128 GELU activations per row run on the SFU/FP32 pipes beside the MMAs"}


def e2e_drop_in(args, systems, dev, warm, steps, fsai=None):
    """csr_tensor from pinned host COO + the solve with pinned host b/x, per
    step (learned: attach the network factor, then cg_mixed in FP64; else
    the plain FP32 cgd drop-in)."""
    import torch
    import mpsparse_b200 as mps
    n = systems[0][0].n
    stream = torch.cuda.current_stream()
    times = []
    h2d = d2h = 0
    e = torch.empty(0)
    for i in range(warm + steps):
        coo = systems[i][0]
        keys = torch.from_numpy(coo.keys()).pin_memory()
        vals = torch.from_numpy(coo.vals).pin_memory()
        if fsai is not None:
            b = systems[i][2].cpu().double().pin_memory()
            x = torch.zeros(n, dtype=torch.float64).pin_memory()
        else:
            b = systems[i][2].cpu().pin_memory()
            x = torch.zeros(n).pin_memory()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        A = mps.spmv.csr_tensor(keys, vals, e, e, e, n, n, fill_outputs=False)
        if fsai is not None:
            fsai.attach(A)
            A.cg_mixed(b, x, tol=TOL, inner_tol=args.inner_tol, max_inner=args.max_iter,
                       precond="fsai")
        else:
            A.cgd(b, x, tol=TOL, max_iter=args.max_iter)
        ev1.record(stream)
        torch.cuda.synchronize()
        if i >= warm:
            times.append(ev0.elapsed_time(ev1))
            h2d = keys.numel() * 8 + vals.numel() * 4 + b.numel() * b.element_size()
            d2h = x.numel() * x.element_size()
        del A
    path = ("spmv.csr_tensor(pinned host COO) + attach_fsai + cg_mixed(pinned host b, x FP64)"
            if fsai is not None else "spmv.csr_tensor(pinned host COO) + cgd(pinned host b, x)")
    return {"value": statistics.mean(times), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "path": path,
            "step_ms": [round(t, 3) for t in times], "median": statistics.median(times)}


def batched_c5(args, dev, rank=0, world=1):
    """4096 independent SPD systems (row counts log-uniform in [1024, 65536];
    half 2D log-normal diffusion grids, sigma 1, correlation 8; half random
    graph Laplacians, mean degree 8, + 1e-2 I) in one graph-launched
    persistent kernel per GPU; learned FSAI kept per class where it beats
    Jacobi, warps per system autotuned.  With N ranks each GPU solves an
    nnz-balanced share of the systems (no collective on the data path); the
    time is the max over ranks and the per-system records are gathered.
    solves/s at 1e-6, every system's FP64 true residual checked."""
    import torch
    from mpsparse_b200 import shard
    from mpsparse_b200.batched import BatchedSolver
    from mpsparse_b200.fsai import LearnedFsai
    W = _workloads()
    n_sys = args.batch_systems
    _, _, est_nnz = W.batch_plan(n_sys, 7)
    mine = shard.partition_by_nnz(est_nnz, world)[rank] if world > 1 else np.arange(n_sys)
    keys, vals, off, kinds = W.batch_systems(n_sys, seed=7, select=mine)
    S = BatchedSolver.from_coo(keys, vals, off)
    del keys, vals
    # b ~ N(0,1) per system from the system's own seed (the same b whatever
    # the sharding)
    b = torch.from_numpy(np.concatenate([W.rhs(int(off[k + 1] - off[k]), 11_000_003 + int(s))
                                         for k, s in enumerate(mine)])).to(dev)
    S.attach_fsai(LearnedFsai.load())
    choice = S.choose_precond(b, kinds, sample=16)
    tune = S.autotune(b)
    x32 = torch.zeros(S.n, device=dev)
    x = torch.zeros(S.n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    S.solve(b, x32)
    S.solve_mixed(b, x)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()

    def timed3(fn):
        ts = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts), res
    # mixed precision (FP64 x, per-system residual replacement): every system
    # stops on its FP64 true residual -- the leg's solves/s; the FP32 solve
    # (stops on the FP32 recurrence) beside it
    ms_local, (it, cv, rr) = timed3(lambda: S.solve_mixed(b, x))
    ms32_local, (it32, cv32, _) = timed3(lambda: S.solve(b, x32))
    it, cv = it.cpu().numpy(), cv.cpu().numpy()
    # FP64 true residual of every system (verification, untimed)
    rp, ci, v = S.csr
    M = torch.sparse_csr_tensor(rp.long(), ci.long(), v.double(), (S.n, S.n))
    r = b.double() - (M @ x.double().unsqueeze(1)).squeeze(1)
    seg = torch.repeat_interleave(torch.arange(S.n_systems, device=dev),
                                  torch.from_numpy(np.diff(off)).to(dev))
    rn = torch.zeros(S.n_systems, dtype=torch.float64, device=dev).index_add_(0, seg, r * r)
    bn = torch.zeros(S.n_systems, dtype=torch.float64, device=dev).index_add_(0, seg, b.double() ** 2)
    rel = (rn / bn).sqrt().cpu().numpy()
    # the FP32 solve's answers: FP64 true residual and the FP32 attainable
    # accuracy 16 * eps32 * || |A| |x| || / ||b||
    r32 = b.double() - (M @ x32.double().unsqueeze(1)).squeeze(1)
    rn32 = torch.zeros(S.n_systems, dtype=torch.float64, device=dev).index_add_(0, seg, r32 * r32)
    rel32 = (rn32 / bn).sqrt().cpu().numpy()
    Mabs = torch.sparse_csr_tensor(rp.long(), ci.long(), v.double().abs(), (S.n, S.n))
    ax = (Mabs @ x32.double().abs().unsqueeze(1)).squeeze(1)
    fn = torch.zeros(S.n_systems, dtype=torch.float64, device=dev).index_add_(0, seg, ax * ax)
    floor = (16 * 2.0 ** -24 * fn.sqrt() / bn.sqrt()).cpu().numpy()
    it32, cv32 = it32.cpu().numpy(), cv32.cpu().numpy()
    ms, ms32, rows, nnz = ms_local, ms32_local, S.n, int(S.nnz.sum())
    if world > 1:
        ms = shard.max_over_ranks(ms_local, device=dev)
        ms32 = shard.max_over_ranks(ms32_local, device=dev)
        rel = shard.gather_records(rel, mine, n_sys, device=dev)
        rel32 = shard.gather_records(rel32, mine, n_sys, device=dev)
        floor = shard.gather_records(floor, mine, n_sys, device=dev)
        it = shard.gather_records(it, mine, n_sys, device=dev)
        cv = shard.gather_records(cv, mine, n_sys, device=dev)
        cv32 = shard.gather_records(cv32, mine, n_sys, device=dev)
        kinds = W.batch_plan(n_sys, 7)[0]
        rows = int(sum(shard.gather_records([float(S.n)], [rank], world, device=dev)))
        nnz = int(sum(shard.gather_records([float(S.nnz.sum())], [rank], world, device=dev)))
    return {"workload": f"{n_sys} SPD systems, n log-uniform [1024, 65536], half 2D "
                        "log-normal diffusion (sigma 1, corr 8), half graph Laplacians + 0.01 I",
            "rows": rows, "nnz": nnz, "ms": ms, "ms_per_rank_local": ms_local, "ranks": world,
            "sharding": "nnz-balanced LPT shares, one persistent launch per GPU" if world > 1
                        else "one GPU",
            "solver": "mixed precision: FP32 recurrences, FP64 x, per-system residual replacement",
            "solves_per_s": n_sys / (ms * 1e-3), "converged_fp64_1e-6": int((rel <= 1e-6).sum()),
            "converged_flags": int(np.sum(cv)), "true_resid_max": float(np.max(rel)),
            "iters_mean": {"grid": float(np.mean(it[kinds == 0])), "graph": float(np.mean(it[kinds == 1]))},
            "fp32_solve": {"ms": ms32, "solves_per_s": n_sys / (ms32 * 1e-3),
                           "stop_rule_met": int(np.sum(cv32)),
                           "true_resid_max": float(np.max(rel32)),
                           "converged_fp64_1e-6": int((rel32 <= 1e-6).sum()),
                           "within_1e-6_or_fp32_floor": int((rel32 <= np.maximum(2e-6, floor)).sum())},
            "precond_choice": {str(k): v["chosen"] for k, v in choice.items()},
            "warps_per_system": tune["warps_per_system"], "launches_per_solve": 1}


class C3Context:
    """The 256^3 7-point log-normal diffusion operator (C3's matrix, 1.14 GB
    per SpMV) built once on the GPU from device COO keys; shared by the SpMV
    roofline leg and the C3 solve legs."""

    def __init__(self, args, dev):
        import torch
        import mpsparse_b200 as mps
        W = _workloads()
        self.m = args.c3_grid
        coo = W.lognormal_diffusion_3d(self.m, 1.0, 8.0, 0)
        e = torch.empty(0)
        self.keys = torch.from_numpy(coo.keys()).to(dev)
        self.vals = torch.from_numpy(coo.vals).to(dev)
        self.A = mps.spmv.csr_tensor(self.keys, self.vals, e, e, e, coo.n, coo.n, fill_outputs=False)
        self.n, self.nnz = coo.n, coo.nnz
        del coo

    def drop_coo(self):
        self.keys = self.vals = None


def spmv_c3(args, dev, ctx):
    """CSR SpMV on the 256^3 7-point diffusion operator: GB/s by the byte model
    8*nnz + 4*(n+1) + 4*n_cols + 4*n_rows, CUDA events per launch."""
    import torch
    A, n, nnz = ctx.A, ctx.n, ctx.nnz
    x = torch.randn(n, device=dev)
    y = torch.empty(n, device=dev)
    stream = torch.cuda.current_stream()
    plan = A.autotune()                     # tile plan chosen on this matrix (setup, untimed)
    for _ in range(3):
        A.mv(x, y)
    reps = 20
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(reps)]
    torch.cuda.nvtx.range_push("spmv_timed")      # profilers can filter on this range
    for a, b in evs:
        a.record(stream)
        A.mv(x, y)
        b.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ms = statistics.median(a.elapsed_time(b) for a, b in evs)
    bytes_alg = 8 * nnz + 4 * (n + 1) + 4 * n + 4 * n
    gbs = bytes_alg / (ms * 1e-3) / 1e9
    out = {"workload": f"{ctx.m}^3 7-pt log-normal diffusion", "n": n, "nnz": nnz,
           "bytes_per_launch": bytes_alg, "ms": ms, "gbs": gbs, "launches": reps,
           "plan": {k: plan[k] for k in ("tile_nnz", "stages", "evict_first")}}
    if not args.only_spmv:
        out["vendor"] = vendor_baselines(A, ctx.keys, ctx.vals, x, n, nnz, bytes_alg, stream)
    return out


def _event_ms(fn, stream, reps, flush=None):
    import torch
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush_l2(flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def vendor_baselines(A, keys, vals, x, n, nnz, bytes_alg, stream):
    """Library kernels on the same B200 and matrix: cuSPARSE SpMV (through
    torch's CSR addmv) and CUB's radix sort of the packed keys (torch.sort),
    beside this library's SpMV and COO -> CSR (sort + row_ptr + tile plan)."""
    import torch
    import mpsparse_b200 as mps
    rp, ci, v = A.csr()
    M = torch.sparse_csr_tensor(rp, ci, v, (n, n))
    for _ in range(3):
        torch.mv(M, x)
    sp_ms = _event_ms(lambda: torch.mv(M, x), stream, 20)
    del M
    sort_ms = _event_ms(lambda: torch.sort(keys), stream, 3)
    e = torch.empty(0)
    ours_ms = _event_ms(lambda: mps.spmv.csr_tensor(keys, vals, e, e, e, n, n, fill_outputs=False),
                        stream, 3)
    return {"cusparse_spmv_ms": sp_ms, "cusparse_spmv_gbs": bytes_alg / (sp_ms * 1e-3) / 1e9,
            "cub_sort_keys_ms": sort_ms, "ours_coo_to_csr_ms": ours_ms,
            "ours_coo_to_csr_gbs_onepass_model": (20 * nnz + 4 * (n + 1)) / (ours_ms * 1e-3) / 1e9,
            # the reference's own byte model (spmv_kernel/spmv/benchmark.py:63-68)
            "ours_coo_to_csr_gbs_ref_model": (16 * nnz + 4 * n) / (ours_ms * 1e-3) / 1e9}


# ------------------------------------------------- the other configurations --
def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def scipy_solve(method, coo, b, tol, max_iter, budget_s=None):
    """scipy.sparse.linalg cg / bicgstab on the host cores (FP64, x0 = 0),
    the CPU path the reference benchmarks against; time, iterations, FP64
    true residual.  budget_s: a bounded run (stopped by maxiter), flagged."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    rp, ci, v = coo.to_csr()
    A = sp.csr_matrix((v.astype(np.float64), ci, rp), shape=(coo.n, coo.n))
    bb = np.asarray(b, np.float64)
    fn = spla.cg if method == "cg" else spla.bicgstab
    cap = max_iter
    if budget_s is not None:
        t0 = time.perf_counter()
        fn(A, bb, rtol=1e-300, atol=0.0, maxiter=20)
        per_it = (time.perf_counter() - t0) / 20
        cap = max(20, min(max_iter, int(budget_s / per_it)))
    it = [0]
    t0 = time.perf_counter()
    x, flag = fn(A, bb, rtol=tol, atol=0.0, maxiter=cap, callback=lambda xk: it.__setitem__(0, it[0] + 1))
    dt = time.perf_counter() - t0
    res = float(np.linalg.norm(bb - A @ x) / np.linalg.norm(bb))
    return {"ms": dt * 1e3, "iters": it[0], "converged": flag == 0, "true_resid": res,
            "capped_by_budget": bool(flag != 0 and cap < max_iter)}


def c1_leg(dev, flush):
    """C1: plain FP32 CG (the drop-in cgd) on the 256x256 5-point Laplacian,
    seed-shuffled COO built on the GPU, tol 1e-6, max 2000 iterations."""
    import torch
    import mpsparse_b200 as mps
    from oracle import oracle as O
    W = _workloads()
    coo = W.laplacian_256().shuffled(1)
    b = W.rhs(coo.n, 0)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(coo.keys()).to(dev), torch.from_numpy(coo.vals).to(dev),
                            e, e, e, coo.n, coo.n, fill_outputs=False)
    bt = torch.from_numpy(b).to(dev)
    x = torch.zeros(coo.n, device=dev)
    last = {}

    def solve():
        x.zero_()
        last["info"] = A.cgd(bt, x, tol=1e-6, max_iter=2000)
    solve()
    ms = _event_ms(solve, torch.cuda.current_stream(), 10, flush)
    info = last["info"]
    Ao = O.Csr(*coo.to_csr(), coo.n)
    xo, io = O.cg(Ao, b.astype(np.float64), tol=1e-6, max_iter=2000, threads=host_threads())
    x20 = torch.zeros(coo.n, device=dev)
    A.cgd(bt, x20, tol=1e-300, max_iter=20)
    xo20, _ = O.cg(Ao, b.astype(np.float64), tol=0.0, max_iter=20)
    # the FP32 x of cgd cannot reach an FP64 true residual of 1e-6 here (its
    # rounding floor is above it): mixed-precision CG (FP64 x) to 1e-6 beside
    b64t = bt.double()
    x64 = torch.zeros(coo.n, dtype=torch.float64, device=dev)
    last_mp = {}

    def solve_mp():
        x64.zero_()
        last_mp["info"] = A.cg_mixed(b64t, x64, tol=1e-6, inner_tol=1e-3, max_inner=2000)
    solve_mp()
    ms_mp = _event_ms(solve_mp, torch.cuda.current_stream(), 10, flush)
    imp = last_mp["info"]
    xc = torch.zeros(coo.n, device=dev)
    ic = A.cgd(bt, xc, reference_compat=True)
    xoc, ioc = O.cg(Ao, b.astype(np.float64), compat=True)
    sc = scipy_solve("cg", coo, b, 1e-6, 2000)
    return {"workload": "256x256 5-pt Laplacian (Dirichlet), n 65,536, nnz 326,656, shuffled COO",
            "solver": "cgd (plain FP32 CG), tol 1e-6, max 2000", "ms": ms, "iters": info["iters"],
            "oracle_fp64_iters": io["iters"], "true_resid": info["true_resid"],
            "converged_fp64": bool(info["converged"]),
            "persistent": bool(info["persistent"]),
            # algorithmic bytes of one iteration of the reference's 3-kernel
            # schedule: SpMV (8 nnz + 4 (n+1) + 8 n) + 9 vector passes (36 n)
            "cg_iteration_bytes_model": C1_ITER_BYTES,
            "gbs_model": C1_ITER_BYTES * info["iters"] / (ms * 1e-3) / 1e9,
            "iterate20_rel_diff_vs_oracle": _rel(x20.cpu().numpy(), xo20),
            "mixed_precision_cg": {"ms": ms_mp, "iters": imp["inner_iters"],
                                   "replacements": imp["outer_iters"],
                                   "true_resid": imp["rel_resid"],
                                   "converged_fp64": bool(imp["converged"]),
                                   "persistent": bool(imp["persistent"])},
            "reference_compat": {"iters": ic["iters"], "oracle_iters": ioc["iters"],
                                 "true_resid": ic["true_resid"],
                                 "rel_diff_vs_oracle": _rel(xc.cpu().numpy(), xoc)},
            "scipy_cg_host": sc}


def c2_leg(dev, flush):
    """C2: plain FP32 BiCGSTAB on the BCSR 4x4 system with 65,536 block rows
    (8 off-diagonal blocks per row, diagonally dominant, nonsymmetric), BCSR
    built on the GPU from seed-shuffled COO keys; BCSR SpMV GB/s with L2
    flushed before each launch."""
    import torch
    import mpsparse_b200 as mps
    from oracle import oracle as O
    W = _workloads()
    bm = W.block_dominant_65536(0)
    coo = bm.to_coo(drop_zeros=True).shuffled(2)
    n = coo.n
    b = W.rhs(n, 3)
    ei = torch.empty(0, dtype=torch.int32)
    A = mps.bcsr.bcsr_tensor(torch.from_numpy(coo.keys()).to(dev), torch.from_numpy(coo.vals).to(dev),
                             ei, ei, n, n, 4)
    bt = torch.from_numpy(b).to(dev)
    x = torch.zeros(n, device=dev)
    last = {}

    def solve():
        x.zero_()
        last["info"] = A.bicgstab(bt, x, tol=1e-6, max_iter=2000)
    solve()
    stream = torch.cuda.current_stream()
    ms = _event_ms(solve, stream, 10, flush)
    info = last["info"]
    nb = int(bm.col_ind.shape[0])
    nbr = n // 4
    bytes_alg = 68 * nb + 4 * (nbr + 1) + 8 * n
    xs, ys = torch.randn(n, device=dev), torch.empty(n, device=dev)
    for _ in range(3):
        A.mv(xs, ys)
    mv_cold = _event_ms(lambda: A.mv(xs, ys), stream, 20, flush)
    mv_warm = _event_ms(lambda: A.mv(xs, ys), stream, 20)
    yo = O.spmv(O.Csr(bm.row_ptr, bm.col_ind, bm.vals, n, 4), xs.cpu().numpy().astype(np.float64))
    Ao = O.Csr(*coo.to_csr(), n)
    _, io = O.bicgstab(Ao, b.astype(np.float64), tol=1e-6, max_iter=2000, threads=host_threads())
    sc = scipy_solve("bicgstab", coo, b, 1e-6, 2000)
    return {"workload": "BCSR 4x4, 65,536 block rows, 589,824 blocks (n 262,144), shuffled COO",
            "solver": "bicgstab (plain FP32), tol 1e-6", "ms": ms, "iters": info["iters"],
            "oracle_fp64_iters": io["iters"], "true_resid": info["true_resid"],
            "converged_fp64": bool(info["converged"]),
            # one BiCGSTAB iteration: 2 BCSR SpMVs + 17 vector passes (68 n)
            "bicgstab_iteration_bytes_model": 2 * bytes_alg + 68 * n,
            "gbs_model": (2 * bytes_alg + 68 * n) * info["iters"] / (ms * 1e-3) / 1e9,
            "bcsr_spmv": {"bytes_per_launch": bytes_alg, "ms_l2_flushed": mv_cold,
                          "gbs_l2_flushed": bytes_alg / (mv_cold * 1e-3) / 1e9,
                          "ms_l2_resident": mv_warm,
                          "effective_gbs_l2_resident": bytes_alg / (mv_warm * 1e-3) / 1e9,
                          "rel_err_vs_oracle": _rel(ys.cpu().numpy(), yo)},
            "scipy_bicgstab_host": sc}


def c3_leg(args, dev, ctx):
    """C3: mixed-precision CG with FP64 refinement to 1e-10 (FP32 values,
    reliable updates; BF16 values, restarted refinement) and plain FP32 CG to
    1e-6 on the 256^3 operator, each checked by its FP64 true residual; the
    error against the FP64 oracle's solution on the 64^3 member of the same
    family (sigma 1, correlation 8), where the oracle runs in seconds."""
    import torch
    import mpsparse_b200 as mps
    from oracle import oracle as O
    W = _workloads()
    stream = torch.cuda.current_stream()

    def run(A, n, b32):
        b64 = b32.double()
        out = {}
        for name, kw in (("mp_fp32_values", dict(value_bits=32)),
                         ("mp_bf16_values", dict(value_bits=16, max_inner=20000, max_outer=200))):
            x = torch.zeros(n, dtype=torch.float64, device=dev)
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            info = A.cg_mixed(b64, x, tol=1e-10, **kw)
            e.record(stream)
            torch.cuda.synchronize()
            out[name] = ({"ms": a.elapsed_time(e), "inner_iters": info["inner_iters"],
                          "outer_iters": info["outer_iters"], "true_resid": info["rel_resid"],
                          "converged_fp64": bool(info["converged"])}, x)
        x = torch.zeros(n, device=dev)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        info = A.cgd(b32, x, tol=1e-6, max_iter=40000)
        e.record(stream)
        torch.cuda.synchronize()
        out["plain_fp32_cg_1e-6"] = ({"ms": a.elapsed_time(e), "iters": info["iters"],
                                      "true_resid": info["true_resid"],
                                      "converged_fp64": bool(info["converged"])}, x)
        return out

    big = run(ctx.A, ctx.n, torch.from_numpy(W.rhs(ctx.n, 3)).to(dev))
    # 64^3 member: errors against the FP64 oracle solution
    c64 = W.lognormal_diffusion_3d(64, 1.0, 8.0, 0)
    e0 = torch.empty(0)
    A64 = mps.spmv.csr_tensor(torch.from_numpy(c64.keys()).to(dev), torch.from_numpy(c64.vals).to(dev),
                              e0, e0, e0, c64.n, c64.n, fill_outputs=False)
    b64h = W.rhs(c64.n, 3)
    small = run(A64, c64.n, torch.from_numpy(b64h).to(dev))
    Ao = O.Csr(*c64.to_csr(), c64.n)
    xref, iref = O.cg(Ao, b64h.astype(np.float64), tol=1e-14, max_iter=100000, threads=host_threads())
    errs = {k: {**v[0], "err_vs_fp64_oracle": _rel(v[1].cpu().numpy(), xref)} for k, v in small.items()}
    return {"workload": f"{ctx.m}^3 7-pt log-normal diffusion (sigma 1, corr 8), n {ctx.n}, nnz {ctx.nnz}",
            "solves": {k: v[0] for k, v in big.items()},
            "member_64cubed": {"oracle": {"solver": "FP64 CG to 1e-14", "iters": iref["iters"],
                                          "true_resid": O.true_residual(Ao, b64h.astype(np.float64), xref)},
                               "solves": errs}}


def reference_sizes_leg(dev):
    """The reference's own CSR solver benchmarks, re-run here on B200: CG on
    2D 5-point Laplacians with n = 1,024 ... 20,449 (iterative/cgd/
    comp_bench.py) and BiCGSTAB with n = 1,024 ... 16,384
    (iterative/BiCGSTAB/benchmark.py), each from x = 0 to a relative
    residual of 1e-6, device time per solve (median of 5 after a warm-up),
    the persistent form (the default) beside the graph form.  The
    reference's published times are Metal timings on an Apple GPU, so no
    ratio is formed."""
    import torch
    import mpsparse_b200 as mps
    W = _workloads()
    stream = torch.cuda.current_stream()
    e = torch.empty(0)

    def time_solve(fn, n):
        times, info = [], None
        for rep in range(6):
            x = torch.zeros(n, device=dev)
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            info = fn(x)
            z.record(stream)
            torch.cuda.synchronize()
            if rep:
                times.append(a.elapsed_time(z))
        return {"ms": statistics.median(times), "iters": info["iters"], "true_resid": info["true_resid"],
                "persistent": bool(info["persistent"])}

    out = {}
    for name, grids in (("cg", (32, 71, 84, 101, 123, 143)), ("bicgstab", (32, 64, 100, 128))):
        rows = []
        for g in grids:
            c = W.laplacian_2d(g)
            A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e,
                                    c.n, c.n, fill_outputs=False)
            b = torch.from_numpy(W.rhs(c.n, 1)).to(dev)
            solve = (lambda x: A.cgd(b, x, tol=1e-6, max_iter=20000)) if name == "cg" else \
                (lambda x: A.bicgstab(b, x, tol=1e-6, max_iter=20000))
            row = {"n": c.n}
            for pers in (True, False):
                A.set_persistent(pers)
                row["persistent_form" if pers else "graph_form"] = time_solve(solve, c.n)
            rows.append(row)
        out[name] = rows
    return out


def persistent_forms_leg(dev):
    """The persistent forms against the graph form of the same solve, device
    time per solve (median of 5 after a warm-up) on 2D 5-point systems from
    512^2 to 1024^2: learned-FSAI mixed-precision PCG to an FP64 1e-6 on
    log-normal diffusion systems (sigma 1.5, correlation 16, seed 5), plain
    CG on the Laplacian and BiCGSTAB on the Laplacian with each east
    coupling halved, both to the 1e-6 recurrence target.  512^2 runs in the
    window form (and, for comparison, in each form: all three fit there);
    700^2 and up, whose rows of A and GᵀG no longer fit shared memory, in the
    stream form (rows read from L2 in every step); plain CG and BiCGSTAB on a
    random graph Laplacian (60,000 rows, mean degree 6, + 0.05 I) in the
    gather form; Richardson (2,000 iterations) on that graph and on the
    1024^2 Laplacian."""
    import torch
    import mpsparse_b200 as mps
    from mpsparse_b200.fsai import LearnedFsai
    W = _workloads()
    stream = torch.cuda.current_stream()
    e = torch.empty(0)

    def time_solve(fn, x):
        times, info = [], None
        for rep in range(6):
            x.zero_()
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            info = fn(x)
            z.record(stream)
            torch.cuda.synchronize()
            if rep:
                times.append(a.elapsed_time(z))
        it = info.get("inner_iters", info.get("iters"))
        ms = statistics.median(times)
        return {"ms": ms, "iters": it, "us_per_iter": 1e3 * ms / max(1, it),
                "form": info["persistent_form"],
                "resid": info.get("true_resid", info.get("rel_resid"))}

    def both(A, fn, x):
        row = {}
        for pers in (True, False):
            A.set_persistent(pers)
            row["persistent" if pers else "graph"] = time_solve(fn, x)
        row["speedup"] = row["graph"]["ms"] / row["persistent"]["ms"]
        return row

    out = []
    for nx in (512, 700, 800, 1024):
        c = W.lognormal_diffusion_2d(nx, nx, 1.5, 16.0, 5)
        A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e,
                                c.n, c.n, fill_outputs=False)
        LearnedFsai.load().attach(A)
        A.set_fsai_apply("product")
        b = torch.from_numpy(W.rhs(c.n, 8).astype(np.float64)).to(dev)
        x = torch.zeros(c.n, dtype=torch.float64, device=dev)
        row = {"solve": "learned FSAI MP-PCG", "grid": nx,
               **both(A, lambda x: A.cg_mixed(b, x, tol=1e-6, precond="fsai"), x)}
        if nx == 512:   # every form fits here: the same solve in each
            row["by_form"] = {}
            for form in ("window", "gather", "stream"):
                A.set_persistent(True, form=form)
                row["by_form"][form] = time_solve(lambda x: A.cg_mixed(b, x, tol=1e-6, precond="fsai"), x)
            A.set_persistent(True)
        out.append(row)
        del A
    c = W.laplacian_2d(1024)
    x = torch.zeros(c.n, device=dev)
    b = torch.from_numpy(W.rhs(c.n, 1)).to(dev)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e,
                            c.n, c.n, fill_outputs=False)
    out.append({"solve": "cgd", "grid": 1024, **both(A, lambda x: A.cgd(b, x, tol=1e-6, max_iter=40000), x)})
    vals = c.vals.copy()
    vals[c.cols == c.rows + 1] *= 0.5
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(vals.astype(np.float32)), e, e, e,
                            c.n, c.n, fill_outputs=False)
    out.append({"solve": "bicgstab", "grid": 1024,
                **both(A, lambda x: A.bicgstab(b, x, tol=1e-6, max_iter=40000), x)})
    # an unstructured matrix: windows span the matrix, so the gather form
    c = W.graph_laplacian(60000, 6.0, 3, shift=0.05)
    x = torch.zeros(c.n, device=dev)
    b = torch.from_numpy(W.rhs(c.n, 7)).to(dev)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e,
                            c.n, c.n, fill_outputs=False)
    for solve in ("cgd", "bicgstab"):
        out.append({"solve": solve, "grid": "random graph, 60,000 rows, mean degree 6",
                    **both(A, lambda x: getattr(A, solve)(b, x, tol=1e-6, max_iter=40000), x)})
    # Richardson, 2,000 iterations at omega 0.02 (below 2 / lambda_max)
    out.append({"solve": "richardson", "grid": "random graph, 60,000 rows, mean degree 6",
                **both(A, lambda x: A.richardson(b, x, omega=0.02, iters=2000), x)})
    c = W.laplacian_2d(1024)
    x = torch.zeros(c.n, device=dev)
    b = torch.from_numpy(W.rhs(c.n, 1)).to(dev)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e,
                            c.n, c.n, fill_outputs=False)
    out.append({"solve": "richardson", "grid": 1024,
                **both(A, lambda x: A.richardson(b, x, omega=0.2, iters=2000), x)})
    return out


def configs_legs(args, dev, c3):
    import torch
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2
    out = {"C1": c1_leg(dev, flush), "C2": c2_leg(dev, flush)}
    del flush
    out["reference_benchmark_sizes"] = reference_sizes_leg(dev)
    if c3 is not None:
        c3.drop_coo()
        out["C3"] = c3_leg(args, dev, c3)
    return out


# --------------------------------------------------------- CPU baselines ---
def cpu_oracle_cg(seed, threads, max_iter=200_000):
    """The oracle's CG (FP64, OpenMP SpMV and fused vector passes) on one
    system, run to its own convergence at relative residual 1e-6."""
    from oracle import oracle as O
    coo, b = c4_system(seed)
    A = O.Csr(*coo.to_csr(), coo.n)
    b = b.astype(np.float64)
    t0 = time.perf_counter()
    x, info = O.cg(A, b, tol=TOL, max_iter=max_iter, threads=threads)
    dt = time.perf_counter() - t0
    return {"ms": dt * 1e3, "iters": info["iters"], "converged": bool(info["converged"]),
            "true_resid": O.true_residual(A, b, x)}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------- reference arm ---
def run_reference(args):
    """Rank 0 only: the oracle port of the reference's cgd_op (FP64, all host
    threads) on the same held-out systems as the timed steps of our arm, each
    solved to its own convergence at 1e-6 (no iteration budget).  Warm-up
    steps are short bounded runs (thread pool and caches), untimed."""
    threads = host_threads()
    for i in range(args.warmup):
        from oracle import oracle as O
        coo, b = c4_system(TEST_SEED0 + i)
        O.cg(O.Csr(*coo.to_csr(), coo.n), b.astype(np.float64), tol=TOL, max_iter=100, threads=threads)
    runs = [cpu_oracle_cg(TEST_SEED0 + args.warmup + i, threads) for i in range(args.steps)]
    v = statistics.mean(r["ms"] for r in runs)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": "plain CG (oracle port of cgd_op), FP64",
                       "tol": TOL},
            "step_ms": [round(r["ms"], 1) for r in runs],
            "iters": [r["iters"] for r in runs],
            "converged": sum(r["converged"] for r in runs),
            "true_resid_max": max(r["true_resid"] for r in runs),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} held-out systems (the timed systems of the GPU "
                                       "arm), each FP64 CG solve run to its own convergence at 1e-6",
                             "host": host_info()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _relaunch_distributed(args):
    """`bench.py --gpus N` started as one process: start N ranks under
    torch.distributed.run (127.0.0.1 rendezvous) and return their status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


# ------------------------------------------------------------------ main ---
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--c3-grid", type=int, default=256)
    ap.add_argument("--skip-spmv", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--skip-configs", action="store_true",
                    help="leave out the C1/C2/C3 legs")
    ap.add_argument("--skip-e2e-plain", action="store_true")
    ap.add_argument("--batch-systems", type=int, default=4096)
    ap.add_argument("--only-spmv", action="store_true",
                    help="only the 256^3 (or --c3-grid) SpMV measurement; for ncu captures")
    ap.add_argument("--only-learned", action="store_true",
                    help="only the learned solve on warmup + steps systems (for profilers)")
    ap.add_argument("--only-persistent-forms", action="store_true",
                    help="only the persistent forms against the graph form, 512^2 to 1024^2")
    ap.add_argument("--only-mlp", action="store_true",
                    help="only the network forward/backward timing on one 512^2 system's factor")
    ap.add_argument("--solver", default="learned", choices=["learned", "plain"],
                    help="headline solver (plain: the FP32 CG drop-in)")
    ap.add_argument("--inner-tol", type=float, default=1e-4,
                    help="relative residual reduction of each inner FP32 PCG sweep")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive iterations from the host (kernels visible to ncu launch lists)")
    ap.add_argument("--max-iter", type=int, default=MAX_ITER,
                    help="iteration cap of the solves (shortened runs for ncu launch lists)")
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds for scipy's CG beside the converged oracle run")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(_relaunch_distributed(args))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    if args.only_spmv:
        ctx = C3Context(args, local)
        print(json.dumps({"spmv": spmv_c3(args, local, ctx)}))
        return
    if args.only_learned:
        print(json.dumps({"learned": learned_only(args, local)}))
        return
    if args.only_persistent_forms:
        print(json.dumps({"persistent_forms": persistent_forms_leg(local)}))
        return
    if args.only_mlp:
        import mpsparse_b200 as mps
        coo, _ = c4_system(TEST_SEED0)
        e = torch.empty(0)
        A = mps.spmv.csr_tensor(torch.from_numpy(coo.keys()), torch.from_numpy(coo.vals), e, e, e,
                                coo.n, coo.n, fill_outputs=False)
        print(json.dumps({"mlp": mlp_leg(A, local)}))
        return
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    res = run_ours(args, rank, world, local)
    hbm, peak_kind = peaks()
    spmv = res["spmv"]
    roof = None
    if spmv:
        traffic = None
        tp = os.path.join(ROOT, "profiles", "spmv_c3_traffic.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get("dram_bytes_per_launch")
        roof = {"bound": "hbm", "achieved": spmv["gbs"], "peak": hbm, "unit": "GB/s",
                "frac": spmv["gbs"] / hbm, "traffic": traffic,
                "kernel": "spmv_stream<EpiStore> (TMA-staged CSR) on " + spmv["workload"],
                "peak_kind": peak_kind, "frac_of_8tbs_spec": spmv["gbs"] / 8000.0}
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = host_threads()
        seed = TEST_SEED0 + args.warmup          # the first timed system
        o = cpu_oracle_cg(seed, threads)
        coo, b = c4_system(seed)
        s = scipy_solve("cg", coo, b, TOL, 200_000, budget_s=args.cpu_budget)
        if not s["converged"] and s["iters"]:
            # a bounded run: scaled to the FP64 CG iteration count of the same
            # system (the oracle's converged run above), flagged
            s["ms_scaled_to_oracle_iters"] = s["ms"] * o["iters"] / s["iters"]
        cpu = {"value": o["ms"], "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"1 system (seed {seed}, the first timed system), oracle FP64 CG run to "
                         f"its own convergence: {o['iters']} iterations, true residual "
                         f"{o['true_resid']:.2e}",
               "host": host_info(), "scipy_cg": s}
    if rank == 0:
        line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_solve"],
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64" if args.solver == "learned" else "f32",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "solver": res["solver"], "tol": TOL,
                           "l2": "flushed between steps (256 MB write)",
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
                "step_ms": res["step_ms"], "ms_median": statistics.median(res["step_ms"]),
                "step_host_ms": res["step_host_ms"],
                "iters_mean": res["iters_mean"], "outer_mean": res["outer_mean"],
                "true_resid_max": res["true_resid_max"],
                "setup_ms_first_solve": res["setup_ms_first_solve"],
                "plain_cg": res["plain_cg"], "jacobi_pcg": res["jacobi_pcg"],
                "jacobi_pcg_mixed": res["jacobi_pcg_mixed"],
                "speedup_vs_jacobi_pcg_mixed": res["jacobi_pcg_mixed"]["ms_per_solve"] / res["ms_per_solve"],
                "speedup_vs_plain_cg": res["plain_cg"]["ms_per_solve"] / res["ms_per_solve"],
                "spmv": spmv, "batched": res["batched"], "configs": res["configs"], "mlp": res["mlp"],
                "roofline": roof, "cpu_baseline": cpu,
                "e2e": res["e2e"], "e2e_plain_cg": res["e2e_plain_cg"],
                "clocks": res["clocks"], "gpu_launches": res["gpu_launches"]}
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
