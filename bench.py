#!/usr/bin/env python3
"""SP2 benchmark: dense mixed-precision SP2 solves/s on B200 (and the FP64 SP2 beside it).

Workload (default): the two-band 1D model Hamiltonian at N=8192 (seeded), solved by the
alg2 branch rule with FP16 hi+lo split products on the tcgen05 tensor cores, FP32
accumulation, FP64 traces and one final McWeeny step whose X^2 is exact (nine INT8
residue products on the tensor cores, CRT in FP64).  A "step" is one complete
solve H -> D.  Inputs (8192^2 FP64 = 512 MiB) are larger than L2 (126 MB), so no L2
flush is needed between steps.

  value   solves/s with H resident in HBM (device pointers through the C ABI)
  e2e     solves/s through the C ABI with host buffers: H2D of H (its upper triangle,
          the library's contract for symmetric H) and D2H of D inside every step
  fp64    the same solve in FP64 (the parity form) for the mixed/FP64 ratio

Multi-GPU (torchrun): independent replicas, one Hamiltonian per rank ("replicas only":
a dense solve does not shard); value = total solves/s, timed as the max over ranks.

--impl reference times the CPU restatement of the reference's FP64 dense alg2
(oracle/sp2_oracle.py, numpy with the host BLAS, all host cores) on a bounded sample
of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "qmd-progress_b200"))


def _tuning():
    """The launch configurations the library measured in this run: key -> [choice, ms...]."""
    import sp2b
    out = {}
    for k in sp2b.tune_keys():
        got = sp2b.tune_get(k)
        if got:
            out[k] = [got[0]] + [round(m, 4) for m in got[1]]
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--precision", default="mixed_fp16",
                    choices=["mixed_fp16", "mixed_bf16", "exact_int8", "fp64"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="two_band",
                    choices=["two_band", "subgraph", "cubic_dense", "adjoint"],
                    help="two_band: dense config (default); subgraph: 32^3 lattice, 256 parts; "
                         "cubic_dense: the 32^3 lattice solved densely (N=32768); adjoint: the "
                         "differentiable SP2's forward and backward at N=2048")
    ap.add_argument("--L", type=int, default=32, help="subgraph: lattice edge")
    ap.add_argument("--parts", type=int, default=256, help="subgraph: number of parts")
    ap.add_argument("--subgraph-precision", default="exact_int8",
                    choices=["mixed_fp16", "mixed_bf16", "exact_int8", "fp64"],
                    help="precision of the sub-graph solve nested in the default line")
    ap.add_argument("--no-subgraph", action="store_true",
                    help="default workload: leave out the nested sub-graph measurement")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="default workload: leave out the nested adjoint (config 3) measurement")
    return ap.parse_args()


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of the bench's GPU, read through NVML
    every 5 ms on a host thread (queries only; no setting is touched).  The bench marks
    its timed regions with begin()/end(); summary() reports the samples taken inside
    them, so even a timed region of a few tens of milliseconds gets several samples.
    Falls back to nvidia-smi at 100 ms when NVML is not available."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.samples = []          # (t, sm_mhz, max_mhz, reasons set)
        self.windows = []
        self._open = None
        self._stop = threading.Event()
        self.proc = None
        self.thread = None
        self.source = None

    def _nvml_handle(self, nv):
        import torch
        try:
            u = str(torch.cuda.get_device_properties(self.index).uuid)
            return nv.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            pass
        try:
            p = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def run():
                while not self._stop.is_set():
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    except Exception:
                        break
                    self.samples.append((time.perf_counter(), sm, mx,
                                         {k for k, b in bits.items() if r & b}))
                    self._stop.wait(0.005)
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            self.source = "nvml 5 ms"
        except Exception:
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._read_smi, daemon=True)
                self.thread.start()
                self.source = "nvidia-smi 100 ms"
            except OSError:
                self.proc = None
        return self

    def _read_smi(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            if len(f) < 9:
                continue
            try:
                sm, mx = float(f[1]), float(f[2])
            except ValueError:
                continue
            self.samples.append((time.perf_counter(), sm, mx,
                                 {nm for nm, v in zip(self.NAMES, f[5:9]) if v.lower().startswith("active")}))

    def begin(self):
        self._open = time.perf_counter()

    def end(self):
        if self._open is not None:
            self.windows.append((self._open, time.perf_counter()))
            self._open = None

    def __exit__(self, *a):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        win = self.windows or ([(self.samples[0][0], self.samples[-1][0])] if self.samples else [])
        inside = [s for s in self.samples if any(a <= s[0] <= b for a, b in win)]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "source": self.source}
        reasons = set()
        for s in inside:
            reasons |= s[3]
        return {"sm_mhz": statistics.median(s[1] for s in inside), "sm_max_mhz": inside[-1][2],
                "sm_min_mhz": min(s[1] for s in inside), "reasons": sorted(reasons),
                "samples": len(inside), "timed_s": round(sum(b - a for a, b in win), 3),
                "source": self.source}


def host_info():
    """CPU model and the BLAS numpy calls, recorded beside every CPU figure."""
    import numpy as np
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    blas = None
    try:
        b = np.show_config(mode="dicts").get("Build Dependencies", {}).get("blas", {})
        blas = f"{b.get('name')} {b.get('version')}"
    except Exception:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count(), "blas": blas}


def cpu_baseline_sample(n, iters_per_solve, max_seconds=20.0):
    """Oracle FP64 alg2 loop on the host cores: time whole SP2 iterations of the N x N
    workload (bounded to ~max_seconds) and extrapolate to solves/s."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np
    import sp2_oracle as O
    from sp2b import modelham as M
    h = M.two_band_1d(n, seed=0)
    x, emin, emax = O.prg_normalize(h)
    trx = float(np.trace(x))
    occ = 0.5 * n
    t0 = time.perf_counter()
    done = 0
    while True:
        x2 = x @ x                                   # src/prg_sp2_mod.F90:308
        trx2 = float(np.trace(x2))
        limdiff = abs(trx2 - occ) - abs(2 * trx - trx2 - occ)
        if limdiff >= 0:
            x = 2.0 * x - x2
            trx = 2 * trx - trx2
        else:
            x = x2
            trx = trx2
        done += 1
        el = time.perf_counter() - t0
        if el > max_seconds or done >= iters_per_solve:
            break
    t_iter = el / done
    return {"value": 1.0 / (t_iter * iters_per_solve), "unit": "solves/s", "cores": os.cpu_count(),
            "kind": "port", "t_iter_s": t_iter, "host": host_info(),
            "sample": f"{done} FP64 SP2 iteration(s) of the N={n} two-band alg2 loop (numpy/OpenBLAS "
                      f"DGEMM, {os.cpu_count()} threads), extrapolated to {iters_per_solve} iterations per solve"}


def subgraph_cpu_sample(rp, col, val, n, hp, hidx, lls, seq, maxiter, emin, emax,
                        max_seconds=15.0):
    """The oracle's FP64 prg_sp2_submatrix per part (numpy with the host BLAS, all host
    cores), parts in order until ~max_seconds, extrapolated by the parts' n^3 to the whole
    serial part loop."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np
    import sp2_oracle as O
    pos = np.full(n, -1, dtype=np.int64)
    total = float(sum((hp[p + 1] - hp[p]) ** 3 for p in range(len(lls))))
    done_w = 0.0
    done = 0
    t0 = time.perf_counter()
    for p in range(len(lls)):
        idx = np.asarray(hidx[hp[p]:hp[p + 1]], dtype=np.int64)
        m = len(idx)
        pos[idx] = np.arange(m)
        sub = np.zeros((m, m))
        for r, i in enumerate(idx):
            c = col[rp[i]:rp[i + 1]]
            keep = pos[c] >= 0
            sub[r, pos[c[keep]]] = val[rp[i]:rp[i + 1]][keep]
        vv = np.zeros(max(maxiter, 1))
        O.sp2_submatrix(sub, seq, maxiter, vv, emin, emax, int(lls[p]))
        pos[idx] = -1
        done_w += float(m) ** 3
        done += 1
        if time.perf_counter() - t0 > max_seconds:
            break
    el = time.perf_counter() - t0
    t_solve = el * total / done_w
    return {"value": 1.0 / t_solve, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
            "host": host_info(),
            "sample": f"{done} of {len(lls)} parts (prg_sp2_submatrix, {maxiter} steps, numpy/OpenBLAS "
                      f"DGEMM, {os.cpu_count()} threads), extrapolated by n^3 to the serial part loop"}


def dense_metric(n):
    return "SP2 solves/s (dense two-band N=%d)" % n


L2_BYTES = 126e6


def dense_config(args, n, world):
    """The dense workload's config, the same on both arms (the reference arm times the
    same solve H -> D on the host cores)."""
    mib = n * n * 8 / 2 ** 20
    l2 = (f"inputs {mib:.0f} MiB > L2 (126 MB), no flush" if n * n * 8 > 2 * L2_BYTES else
          f"inputs {mib:.1f} MiB fit in L2: 256 MiB written between timed solves, each solve timed alone")
    return {"workload": f"two_band_1d_n{n}_{args.precision}_alg2_mcweeny1", "n": n,
            "bndfil": 0.5, "idemtol": 1e-10, "seed": "rank r solves seed r",
            "parallelism": f"replicas{world}", "l2": l2}


def oracle_solve(n, seed=0):
    """One complete FP64 alg2 genseq solve of the workload by the oracle (None stop rule,
    idemtol 1e-10, at most 100 iterations) on the host cores: the iteration count every CPU
    figure extrapolates by, and a check of its output (Tr D = N)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np
    import sp2_oracle as O
    from sp2b import modelham as M
    h = M.two_band_1d(n, seed=seed)
    t0 = time.perf_counter()
    r = O.sp2_alg2_genseq(h, 0.5, 0, 100, "None", 1e-10)
    el = time.perf_counter() - t0
    tr = float(np.trace(r.rho))
    if not abs(tr - n) <= 1e-6 * n:
        raise RuntimeError(f"oracle solve of the bench workload: Tr D = {tr} != {n}")
    return r.icount, el


def run_reference(args, rank, world):
    if rank != 0:
        return
    n = args.n
    iters, full_s = oracle_solve(n)   # untimed: the workload's FP64 iteration count
    vals = []
    for _ in range(args.warmup):
        cpu_baseline_sample(min(n, 2048), 1, 5.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_baseline_sample(n, iters, max_seconds=15.0)
        vals.append(r["value"])
    el = time.perf_counter() - t0
    v = statistics.median(vals)
    out = {"metric": dense_metric(n), "value": v, "unit": "solves/s",
           "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": dense_config(args, n, world),
           "cpu_baseline": {"value": v, "unit": "solves/s", "cores": r["cores"], "kind": "port",
                            "sample": r["sample"], "host": r["host"], "sp2_iters": iters,
                            "full_solve_s": full_s},
           "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def roofline_peak(peaks, clocks):
    """The bf16 denominator for a kernel timed inside this run: the burst figure unless the
    clocks of the timed region show the power cap, then the sustained one."""
    capped = "sw_power_cap" in (clocks.get("reasons") or [])
    key = "bf16_tflops_sustained" if capped and "bf16_tflops_sustained" in peaks else "bf16_tflops"
    return key, peaks[key]


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "subgraph":
        return run_subgraph(args, rank, world, local)
    if args.workload == "cubic_dense":
        return run_cubic_dense(args, rank, local)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, local)

    import numpy as np
    import torch
    from sp2b import _lib, modelham as M

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    L = _lib.lib()
    n = args.n
    prec = {"mixed_fp16": _lib.PREC_MIXED_FP16, "mixed_bf16": _lib.PREC_MIXED_BF16,
            "exact_int8": _lib.PREC_EXACT_INT8, "fp64": _lib.PREC_FP64}[args.precision]
    h_np = M.two_band_1d(n, seed=rank)
    stream = torch.cuda.current_stream()
    h_dev = torch.from_numpy(h_np).cuda()
    rho_dev = torch.empty_like(h_dev)
    pp = np.zeros(128, dtype=np.int32)
    vv = np.zeros(128)
    ic = C.c_int(0)
    # inputs that fit in L2 get it flushed between timed solves (each solve timed alone)
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device="cuda") \
        if n * n * 8 <= 2 * L2_BYTES else None

    def solve_dev(precision):
        o = _lib.make_opts(precision=precision, device_ptrs=True, stream=stream.cuda_stream)
        _lib.check(L.sp2b_sp2_alg2_genseq(h_dev.data_ptr(), rho_dev.data_ptr(), n, 0.0, 0.5, 0, 100,
                                          b"None", 1e-10, pp.ctypes.data, C.byref(ic), vv.ctypes.data, 0,
                                          C.byref(o)), "sp2_alg2_genseq")
        return ic.value

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_ms(fn, reps):
        """Device time of reps calls on the launch stream: one event pair around all of
        them, or, when L2 is flushed between calls, one pair per call (summed)."""
        if flush is None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1), out
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot, out

    clk = ClockSampler(local).__enter__()
    # ---- warm-up ----
    for _ in range(args.warmup):
        iters = solve_dev(prec)
    # ---- timed region: device-resident ----
    L.sp2b_set_step_timing(1)
    launches0 = L.sp2b_launch_count()
    barrier()
    clk.begin()
    t_ms, iters = timed_ms(lambda: solve_dev(prec), args.steps)
    clk.end()
    barrier()
    launches = L.sp2b_launch_count() - launches0
    step_ms = C.c_double(0)
    step_n = C.c_longlong(0)
    L.sp2b_step_timing(C.byref(step_ms), C.byref(step_n))
    ref_ms = (C.c_double * 4)()
    ref_n = C.c_longlong(0)
    L.sp2b_refinement_timing(ref_ms, C.byref(ref_n))
    L.sp2b_set_step_timing(0)
    t_ms = max_over_ranks(t_ms)
    value = world * args.steps / (t_ms / 1e3)

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        h_host = torch.from_numpy(h_np).pin_memory()
        rho_host = torch.empty_like(h_host).pin_memory()
        o = _lib.make_opts(precision=prec, device_ptrs=False, stream=stream.cuda_stream)

        def solve_host():
            _lib.check(L.sp2b_sp2_alg2_genseq(h_host.data_ptr(), rho_host.data_ptr(), n, 0.0, 0.5, 0, 100,
                                              b"None", 1e-10, pp.ctypes.data, C.byref(ic), vv.ctypes.data, 0,
                                              C.byref(o)), "sp2_alg2_genseq(host)")
        solve_host()
        barrier()
        clk.begin()
        te, _ = timed_ms(solve_host, args.steps)
        clk.end()
        barrier()
        te = max_over_ranks(te)
        # H crosses as its upper triangle (one 2D copy per 128-row panel, the library
        # rebuilds the rest on the device); D comes back whole, with pp and vv
        h2d = sum((n - r0) * min(128, n - r0) * 8 for r0 in range(0, n, 128))
        e2e = {"value": world * args.steps / (te / 1e3), "unit": "solves/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n * n * 8 + 2 * 128 * 8}

    # ---- FP64 (parity form) beside it ----
    fp64 = None
    it64 = iters if prec == _lib.PREC_FP64 else None
    rho_mixed = rho_dev.clone() if prec != _lib.PREC_FP64 else None
    if prec != _lib.PREC_FP64 and args.fp64_steps > 0:
        solve_dev(_lib.PREC_FP64)
        barrier()
        clk.begin()
        tf, it64 = timed_ms(lambda: solve_dev(_lib.PREC_FP64), args.fp64_steps)
        clk.end()
        barrier()
        tf = max_over_ranks(tf)
        fp64 = {"solves_per_s": world * args.fp64_steps / (tf / 1e3), "iters": it64,
                "ms_per_solve": tf / args.fp64_steps,
                "tflops": world * args.fp64_steps * 2.0 * n ** 3 * it64 / (tf / 1e3) / 1e12,
                "kernel": "k_sym_gemm_f64 (FP64 DMMA SP2 step)"}
        # accuracy of the mixed solve against the FP64 one (same H): ||dD||_F / N
        dd = float((rho_mixed - rho_dev).norm().item())
        fp64["mixed_err_fro_over_n"] = dd / n
        fp64["mixed_err_rel_fro"] = dd / float(rho_dev.norm().item())

    clk.__exit__(None, None, None)
    clocks = clk.summary()

    # ---- roofline of the dominant kernel (the SP2 step) ----
    peaks, src = load_peaks()
    step_avg_ms = step_ms.value / max(step_n.value, 1)
    flops_launch = 2.0 * n ** 3          # one N x N x N product per SP2 step (algorithmic)
    achieved = flops_launch / (step_avg_ms / 1e3) / 1e12
    npad = -(-n // 128) * 128
    nb = npad // 128
    if prec != _lib.PREC_FP64:
        peak_key, peak = roofline_peak(peaks, clocks)
        kernel = "k_tc_pair (SP2 step, CTA pairs)" if npad % 256 == 0 else "k_tc_persist (SP2 step)"
        if prec == _lib.PREC_EXACT_INT8:
            kernel = "k_oz_gemm (exact INT8 SP2 step: 9 residue products)"
    else:
        peak_key, peak = None, None
        kernel = "k_sym_gemm_f64 (FP64 DMMA SP2 step)"
    traffic = None
    tpath = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        ent = tj.get(f"sp2_step_{args.precision}_n{n}")
        if ent:
            traffic = ent.get("bytes_per_launch")
    # executed tensor work: upper 128 x 128 tiles (incl. the diagonal), three 16-bit
    # products each (hi*hi, hi*lo, lo*hi) over the padded K
    exec_flops = 3 * 2.0 * 128 * 128 * npad * (nb * (nb + 1) // 2) \
        if prec in (_lib.PREC_MIXED_FP16, _lib.PREC_MIXED_BF16) else None
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if peak else None, "traffic": traffic,
                "peak_source": f"{src} {peak_key}" if peak_key else "no bf16 denominator for FP64",
                "kernel": kernel, "avg_launch_ms": step_avg_ms, "launches_timed": step_n.value,
                "flops_per_launch": flops_launch,
                "frac_of_sustained": (achieved / peaks["bf16_tflops_sustained"])
                if peak and "bf16_tflops_sustained" in peaks else None,
                "executed_tflops": (exec_flops / (step_avg_ms / 1e3) / 1e12) if exec_flops else None,
                "executed_frac": (exec_flops / (step_avg_ms / 1e3) / 1e12 / peak) if exec_flops and peak else None}
    refinement = None
    if ref_n.value > 0:
        per = [ref_ms[i] / ref_n.value for i in range(4)]
        nbp = -(-npad // 256)
        oz_tiles = sum(nbp - bi // 2 for bi in range(nb))
        int8_ops = 9 * 2.0 * 128 * 256 * npad * oz_tiles       # executed, 9 residue products
        refinement = {"ms_per_solve": sum(per),
                      "phases_ms": {"residue_planes": per[0], "int8_products": per[1], "crt": per[2],
                                    "combine_product": per[3]},
                      "kernel": "k_oz_gemm (9 INT8 residue products, upper 128x256 tiles)",
                      "int8_tops_executed": int8_ops / (per[1] / 1e3) / 1e12,
                      "int8_peak_nominal_tops": 4500.0,
                      "int8_frac_of_nominal": int8_ops / (per[1] / 1e3) / 1e12 / 4500.0}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        if it64 is None:
            it64, _ = oracle_solve(n)
        cpu = cpu_baseline_sample(n, it64, max_seconds=20.0)
        cpu["sp2_iters"] = it64
    adj = None
    if args.workload == "two_band" and not args.no_adjoint and rank == 0 and world == 1:
        adj = measure_adjoint()
    sub = None
    if args.workload == "two_band" and not args.no_subgraph:
        del h_dev, rho_dev, rho_mixed
        torch.cuda.empty_cache()
        sub = measure_subgraph(args, rank, world, local, dist, args.subgraph_precision)
    if rank == 0:
        out = {"metric": dense_metric(n), "value": value,
               "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": {_lib.PREC_MIXED_FP16: "f16", _lib.PREC_MIXED_BF16: "bf16",
                                              _lib.PREC_EXACT_INT8: "i8"}.get(prec, "f64"),
               "data": "synthetic",
               "config": dense_config(args, n, world), "sp2_iters": iters,
               # algorithmic: 2N^3 per SP2 step + 4N^3 for the McWeeny step (mixed)
               "tflops": value * (2.0 * n ** 3 * iters + (4.0 * n ** 3 if prec != _lib.PREC_FP64 else 0.0)) / 1e12,
               "fp64": fp64, "e2e": e2e, "roofline": roofline, "refinement": refinement,
               "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
               "tuning": _tuning(), "subgraph": sub, "adjoint": adj}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_adjoint(args, rank, local):
    """bench.py --workload adjoint: the differentiable SP2's forward and backward
    (measure_adjoint) as its own line; value = gradients (forward + backward) per second.
    Under torchrun every rank runs an independent replica and rank 0 prints."""
    import torch
    torch.cuda.set_device(local)
    adj = measure_adjoint(reps=max(args.steps, 1))
    if rank == 0:
        ms = adj["forward_ms"] + adj["backward_ms"]
        print(json.dumps({"metric": "sp2_gradients_per_s", "value": 1e3 / ms, "unit": "gradients/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": 2, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f16", "data": "synthetic",
                          "config": {"workload": adj["workload"], "n": adj["n"],
                                     "sp2_steps": adj["sp2_steps"]},
                          "adjoint": adj}), flush=True)


def run_subgraph(args, rank, world, local):
    """bench.py --workload subgraph: the batched sub-graph measurement as its own line."""
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    out = measure_subgraph(args, rank, world, local, dist, args.precision)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def measure_adjoint(n=2048, reps=5):
    """Config 3: the differentiable SP2 (sp2b.autograd.SP2Density) on the two-band model,
    N = 2048, loss Tr(D A) with a random symmetric A; forward (replay of the genseq branch
    sequence, iterates kept in the FP16 hi/lo split form, one symmetric split product per
    step, X kept every 4 steps) and backward (segments recomputed from the checkpoints,
    one symmetric product over the concatenated K range [G | X][X | G]^T per reverse
    step) timed with CUDA events on the current stream.  Algorithmic flops: 2 n^3 per
    forward step; backward 2 n^3 per reverse step plus the recomputed steps."""
    import torch
    import sp2b
    from sp2b import modelham as M
    from sp2b.autograd import sequence_and_bounds, sp2_density
    h = torch.tensor(M.two_band_1d(n, seed=0), device="cuda", dtype=torch.float32)
    a = torch.tensor(M.random_symmetric(n, seed=1), device="cuda", dtype=torch.float32)
    pp, lo, hi = sequence_and_bounds(h, 0.5)
    K, ck = len(pp), 4
    stream = torch.cuda.current_stream()

    def one(graphs=True):
        hv = h.clone().requires_grad_(True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        d = sp2_density(hv, pp, lo, hi, ck, graphs)
        loss = (d * a).sum()
        e1.record(stream)
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), e1.elapsed_time(e2), hv.grad
    for _ in range(2):
        one()
    fw, bw = [], []
    for _ in range(reps):
        f, b, g = one()
        fw.append(f)
        bw.append(b)
    f, b = statistics.median(fw), statistics.median(bw)
    one(False)
    fe, be = [], []
    for _ in range(reps):
        fx, bx, _ = one(False)
        fe.append(fx)
        be.append(bx)
    nseg = (K + ck - 1) // ck
    recomputed = K - nseg                      # steps replayed from the checkpoints
    flops_f = 2.0 * n ** 3 * K
    flops_b = 2.0 * n ** 3 * (K + recomputed)
    return {"workload": f"two_band_1d_n{n}_adjoint_trDA", "n": n, "sp2_steps": K,
            "checkpoint": ck, "forward_ms": f, "backward_ms": b,
            "forward_tflops": flops_f / (f / 1e3) / 1e12,
            "backward_tflops": flops_b / (b / 1e3) / 1e12,
            "grad_finite": bool(torch.isfinite(g).all().item()),
            "eager_forward_ms": statistics.median(fe), "eager_backward_ms": statistics.median(be),
            "kernels": "k_tc_pair (split FP16 symmetric products: X^2, and {G, X} over the "
                       "concatenated K range); forward steps and backward replayed as CUDA "
                       "graphs",
            "timing": f"median of {reps}, CUDA events"}


def measure_subgraph(args, rank, world, local, dist, precision):
    """Batched graph-partitioned SP2 (prg_subgraphSP2Loop) on the L^3 cubic lattice.

    Setup (untimed), as the reference's sub-graph test does
    (tests/src/test_subgraphloop.F90:59-152): a dense genseq of the full H gives
    vv and pp, prg_homolumogap and prg_sp2sequence give the shared branch sequence;
    the graph is the pattern of |D^2| > 0.3 for the density D of that genseq (the test
    thresholds the density of a previous solve; the configuration partitions the graph
    of D^2); parts come from recursive coordinate bisection with split fractions
    U[0.4, 0.6]; halos are one jump in the graph.  A step is one whole sub-graph solve
    (one graph launch): extraction from CSR, normalisation, the SP2 steps, core-row
    scatter.
    """
    import numpy as np
    import torch
    import sp2b
    from sp2b import _lib, graph as G, modelham as M
    L = args.L
    n = L ** 3
    Lb = _lib.lib()
    # one system (the sharded solve splits its parts over the ranks)
    rp, col, val = M.cubic_3d_csr(L, seed=0, threshold=1e-5)
    # Gershgorin bounds from the CSR rows
    diag = np.zeros(n)
    rows = np.repeat(np.arange(n), np.diff(rp))
    on = rows == col
    diag[rows[on]] = val[on]
    rad = np.bincount(rows, weights=np.abs(val), minlength=n) - np.abs(diag)
    emin, emax = float(np.min(diag - rad)), float(np.max(diag + rad))
    # full-system genseq on the GPU for the gap estimate and the branch sequence, in the
    # exact INT8 form (FP64-grade, like the reference's double-precision genseq)
    t0 = time.time()
    hd = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    hd[torch.from_numpy(rows).cuda(), torch.from_numpy(col.astype(np.int64)).cuda()] = \
        torch.from_numpy(val).cuda()
    rd = torch.empty_like(hd)
    pp = np.zeros(128, dtype=np.int32)
    vv = np.zeros(128)
    ic = C.c_int(0)
    o = _lib.make_opts(precision=_lib.PREC_EXACT_INT8, device_ptrs=True,
                       stream=torch.cuda.current_stream().cuda_stream)
    _lib.check(Lb.sp2b_sp2_alg2_genseq(hd.data_ptr(), rd.data_ptr(), n, 0.0, 0.5, 0, 100, b"None",
                                       1e-10, pp.ctypes.data, C.byref(ic), vv.ctypes.data, 0,
                                       C.byref(o)), "genseq")
    del hd
    torch.cuda.empty_cache()
    # the graph of D^2 (the full system's density from the same genseq), thresholded at
    # 0.3: core+halo sizes 96..462 with 256 parts (configuration: 64..512)
    tg = time.time()
    g_csr = G.density_square_graph(rd, 0.3)
    graph_s = time.time() - tg
    del rd
    torch.cuda.empty_cache()
    full_iters = ic.value
    eh, el, egap = sp2b.homolumogap(vv[:full_iters], full_iters, pp[:full_iters], emin, emax)
    if egap > 0.0 and emin < eh < el < emax:
        seq, maxiter = sp2b.sp2sequence(emin, emax, eh, el, 1e-12)
        seq_source = "prg_sp2sequence(homolumogap)"
    else:
        # no usable gap estimate (the full-system ||X - X^2||_F never fell below the
        # prg_homolumogap threshold on this near-gapless lattice): the parts replay the
        # branch sequence the full-system genseq took
        seq, maxiter = [int(x) for x in pp[:full_iters]], full_iters
        seq_source = "full-system exact-INT8 genseq pp"

    parts = G.rcb_partition(G.lattice_coords(L), args.parts, seed=0, lo=0.4, hi=0.6)
    hp, hidx, ls, lls = sp2b.subgraph_halos(n, g_csr, parts, None, double_jump=False)
    nparts_all = len(parts)
    plan = None
    if world > 1:
        # the parts are sharded over the ranks (LPT on n^3); every solve ends with the
        # loop's two exchanges: vv all-reduced, core rows all-gathered (NCCL, device)
        from sp2b import dist as D
        plan = D.ShardPlan(hp, lls, world)
        hp, hidx, lls = plan.local_problem(hidx, rank)
        ls = np.diff(hp).astype(np.int32)
    setup_s = time.time() - t0
    # device-resident inputs
    rp_d = torch.from_numpy(rp).cuda()
    col_d = torch.from_numpy(col).cuda()
    val_d = torch.from_numpy(val).cuda()
    hp_d = torch.from_numpy(hp).cuda()
    hidx_d = torch.from_numpy(hidx).cuda()
    lls_d = torch.from_numpy(lls).cuda()
    core_d = torch.empty(int(np.sum(lls.astype(np.int64) * ls)), dtype=torch.float64, device="cuda")
    seq_a = np.ascontiguousarray(seq, dtype=np.int32)
    vvo = np.zeros(max(maxiter, 1))
    stream = torch.cuda.current_stream()

    def solve(prec, iters=None, refine_tol=None):
        oo = _lib.make_opts(precision=prec, device_ptrs=True, stream=stream.cuda_stream,
                            refine_tol=refine_tol)
        _lib.check(Lb.sp2b_subgraph_sp2_loop(n, rp_d.data_ptr(), col_d.data_ptr(), val_d.data_ptr(),
                                             len(lls), hp_d.data_ptr(), hidx_d.data_ptr(),
                                             lls_d.data_ptr(), seq_a.ctypes.data,
                                             maxiter if iters is None else iters, emin, emax,
                                             core_d.data_ptr(), None, vvo.ctypes.data, C.byref(oo)),
                   "subgraph_sp2_loop")
        if plan is not None:
            D.exchange(core_d, vvo[:max(maxiter, 1)] ** 2, plan, device=core_d.device)

    def events_ms(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device="cuda")

    def timed(prec, steps):
        """Device time of `steps` solves: the inputs (CSR H, 13 MB) fit in L2, so 256 MiB
        are written between solves and each solve is timed alone (summed)."""
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        l0 = Lb.sp2b_launch_count()
        t = 0.0
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solve(prec)
            e1.record(stream)
            torch.cuda.synchronize()
            t += e0.elapsed_time(e1)
        if dist:
            tt = torch.tensor([t], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t, Lb.sp2b_launch_count() - l0

    prec = {"mixed_fp16": _lib.PREC_MIXED_FP16, "mixed_bf16": _lib.PREC_MIXED_BF16,
            "exact_int8": _lib.PREC_EXACT_INT8, "fp64": _lib.PREC_FP64}[precision]
    clk = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        solve(prec)
    torch.cuda.synchronize()
    clk.begin()
    t_ms, launches = timed(prec, args.steps)
    clk.end()
    core_mixed = core_d.clone()
    nref = C.c_int(0)
    Lb.sp2b_last_subgraph_refined(C.byref(nref), None, 0, None, 0)
    # ---- roofline of the batched SP2 step (one launch covers every part) ----
    # average step-launch duration = (solve - the same solve with no SP2 steps) / maxIter,
    # both without the FP64 re-solve of flagged parts, CUDA events on the launch stream
    # (each form warmed up right before it is timed: the library re-captures its graph when
    # the step count or the outputs change)
    solve(prec, refine_tol=0.0)
    core_noref = core_d.clone()   # the same solve without the FP64 re-solve of flagged parts
    t_steps = events_ms(lambda: solve(prec, refine_tol=0.0), 3)
    solve(prec, iters=0, refine_tol=0.0)
    t_none = events_ms(lambda: solve(prec, iters=0, refine_tol=0.0), 3)
    step_avg_ms = max(t_steps - t_none, 1e-6) / max(maxiter, 1)
    flops_launch = 2.0 * float(np.sum(ls.astype(np.float64) ** 3))
    peaks, psrc = load_peaks()
    traffic = None
    tpath = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            ent = json.load(f).get(f"sp2_step_batched_{precision}_cubic20_64parts")
        if ent:
            # captured on the 20^3 / 64-part case; DRAM bytes scale with the tiles' work
            traffic = ent["bytes_per_launch"] * flops_launch / ent["flops_per_launch"]
    peak_key, peak = roofline_peak(peaks, clk.summary())
    if prec == _lib.PREC_EXACT_INT8:
        # the persistent INT8 kernel: 13 digit products of 128 x 64 x n64 per tile (tiles
        # on or above each part's diagonal, K to the part size rounded up to 64); int8
        # tensor rate = 2x the bf16 dense rate on B200
        ops = 0.0
        for nn in ls:
            n64 = -(-int(nn) // 64) * 64
            ntile = sum(n64 // 64 - 2 * bi for bi in range(-(-n64 // 128)))
            ops += ntile * 2.0 * 13 * 128 * 64 * n64
        achieved = ops / (step_avg_ms / 1e3) / 1e12
        peak = 2.0 * peak
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)",
                    "frac": achieved / peak, "traffic": traffic,
                    "peak_source": f"{psrc} {peak_key} x 2 (int8 : bf16 dense rate)",
                    "kernel": "k_i8_steps (persistent: every step of every part, one launch)",
                    "avg_step_ms": step_avg_ms, "int8_ops_per_step": ops,
                    "sp2_flops_per_step": flops_launch,
                    "sp2_tflops": flops_launch / (step_avg_ms / 1e3) / 1e12,
                    "timing": "(solve - solve with no steps) / maxIter, FP64 re-solve off"}
    else:
        achieved = flops_launch / (step_avg_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "frac_of_sustained": achieved / peaks.get("bf16_tflops_sustained", peak),
                    "peak_source": f"{psrc} {peak_key}",
                    "kernel": ("k_tc_persist<T,0,1> (batched SP2 step, all parts)"
                               if prec != _lib.PREC_FP64 else "batched FP64 step (all parts)"),
                    "avg_launch_ms": step_avg_ms, "flops_per_launch": flops_launch,
                    "timing": "(solve - solve with no steps) / maxIter, FP64 re-solve off"}
    roofline["ms_solve_without_fp64_resolve"] = t_steps
    roofline["ms_solve_without_steps"] = t_none

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        rp_h = torch.from_numpy(rp).pin_memory()
        col_h = torch.from_numpy(col).pin_memory()
        val_h = torch.from_numpy(val).pin_memory()
        core_h = torch.empty(core_d.numel(), dtype=torch.float64).pin_memory()
        oh = _lib.make_opts(precision=prec, device_ptrs=False, stream=stream.cuda_stream)
        hp_a = np.ascontiguousarray(hp, dtype=np.int64)
        hidx_a = np.ascontiguousarray(hidx, dtype=np.int32)
        lls_a = np.ascontiguousarray(lls, dtype=np.int32)

        gath_h = torch.empty(plan.world * plan.width if plan else 1, dtype=torch.float64).pin_memory()

        def solve_host():
            _lib.check(Lb.sp2b_subgraph_sp2_loop(n, rp_h.data_ptr(), col_h.data_ptr(), val_h.data_ptr(),
                                                 len(lls), hp_a.ctypes.data, hidx_a.ctypes.data,
                                                 lls_a.ctypes.data, seq_a.ctypes.data, maxiter, emin,
                                                 emax, core_h.data_ptr(), None, vvo.ctypes.data,
                                                 C.byref(oh)), "subgraph_sp2_loop(host)")
            if plan is not None:
                # this rank's core rows go to the device for the exchange; every rank reads
                # the gathered rows of all parts back
                g, _ = D.exchange(core_h, vvo[:max(maxiter, 1)] ** 2, plan, device=core_d.device)
                gath_h.copy_(g, non_blocking=True)
        solve_host()
        clk.begin()
        te = events_ms(solve_host, args.steps)
        clk.end()
        # H (CSR) and pp in; the core rows and vv out, every call (sharded: this rank's core
        # rows up for the exchange, every part's core rows back)
        h2d = rp.nbytes + col.nbytes + val.nbytes + seq_a.nbytes
        d2h = core_d.numel() * 8 + maxiter * 8
        if plan is not None:
            h2d += core_d.numel() * 8
            d2h += gath_h.numel() * 8
        e2e = {"value": 1.0 / (te / 1e3), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = subgraph_cpu_sample(rp, col, val, n, hp, hidx, lls, seq, maxiter, emin, emax)

    for _ in range(args.warmup):
        solve(_lib.PREC_FP64)
    clk.begin()
    t64, _ = timed(_lib.PREC_FP64, max(1, args.fp64_steps))
    clk.end()
    clk.__exit__(None, None, None)
    err_vs_fp64 = float((core_mixed - core_d).norm().item()) / n
    rel_vs_fp64 = float((core_mixed - core_d).norm().item() / core_d.norm().item())
    rel_noref = float((core_noref - core_d).norm().item() / core_d.norm().item())
    flops = 2.0 * float(np.sum(ls.astype(np.float64) ** 3)) * maxiter
    if plan is not None:
        ft = torch.tensor([flops], device="cuda", dtype=torch.float64)
        dist.all_reduce(ft)
        flops = float(ft.item())
    # one solve is the whole system (every part, on all ranks together): strong scaling
    value = args.steps / (t_ms / 1e3)
    if rank == 0:
        out = {"metric": f"sub-graph SP2 solves/s ({L}^3 lattice, {nparts_all} parts, batched)",
               "value": value,
               "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "strong",
               "vs_baseline": None, "dtype": precision, "data": "synthetic",
               "config": {"workload": f"cubic{L}_subgraph_{nparts_all}parts_{precision}",
                          "n": n, "parts": nparts_all, "lsize_min": int(ls.min()),
                          "parallelism": f"parts sharded over {world} ranks (LPT), vv all-reduce + "
                                         f"core-row all-gather per solve" if world > 1 else "1 GPU",
                          "lsize_max": int(ls.max()), "lsize_mean": float(ls.mean()),
                          "maxiter": maxiter, "full_genseq_iters": full_iters,
                          "homo": eh, "lumo": el, "sequence": seq_source,
                          "graph": "|D^2| > 0.3 (D: the full system's genseq density)", "halo": "one jump",
                          "partition": "RCB U[0.4,0.6]", "setup_s": setup_s,
                          "l2": "CSR H 13 MB fits in L2: 256 MiB written between timed solves",
                          "graph_s": graph_s,
                          "parts_resolved_fp64": nref.value},
               "tflops": value * flops / 1e12, "flops_per_solve": flops,
               "fp64": {"solves_per_s": max(1, args.fp64_steps) / (t64 / 1e3),
                        "ms_per_solve": t64 / max(1, args.fp64_steps)},
               "err_vs_fp64": {"fro_over_n": err_vs_fp64, "rel_fro": rel_vs_fp64,
                               "rel_fro_without_fp64_resolve": rel_noref},
               "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
               "clocks": clk.summary(), "gpu_launches": launches, "tuning": _tuning()}
        return out
    return None


def run_cubic_dense(args, rank, local):
    """Dense mixed SP2 of the L^3 lattice Hamiltonian (N = L^3), FP64 solve beside it."""
    import numpy as np
    import torch
    from sp2b import _lib, modelham as M
    torch.cuda.set_device(local)
    L = args.L
    n = L ** 3
    rp, col, val = M.cubic_3d_csr(L, seed=rank, threshold=1e-5)
    rows = np.repeat(np.arange(n), np.diff(rp))
    h = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    h[torch.from_numpy(rows).cuda(), torch.from_numpy(col.astype(np.int64)).cuda()] = \
        torch.from_numpy(val).cuda()
    rho = torch.empty_like(h)
    pp = np.zeros(130, dtype=np.int32)
    vv = np.zeros(130)
    ic = C.c_int(0)
    Lb = _lib.lib()
    stream = torch.cuda.current_stream()

    def solve(prec):
        o = _lib.make_opts(precision=prec, device_ptrs=True, stream=stream.cuda_stream)
        _lib.check(Lb.sp2b_sp2_alg2_genseq(h.data_ptr(), rho.data_ptr(), n, 0.0, 0.5, 0, 120, b"None",
                                           1e-10, pp.ctypes.data, C.byref(ic), vv.ctypes.data, 0,
                                           C.byref(o)), "genseq")
        return ic.value

    prec = {"mixed_fp16": _lib.PREC_MIXED_FP16, "mixed_bf16": _lib.PREC_MIXED_BF16,
            "exact_int8": _lib.PREC_EXACT_INT8, "fp64": _lib.PREC_FP64}[args.precision]
    for _ in range(args.warmup):
        solve(prec)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            iters = solve(prec)
        e1.record(stream)
        torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / args.steps
    rho_m = rho.clone()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    it64 = solve(_lib.PREC_FP64)
    f1.record(stream)
    torch.cuda.synchronize()
    t64 = f0.elapsed_time(f1)
    err = float((rho_m - rho).norm().item())
    out = {"metric": f"dense SP2 solves/s ({L}^3 lattice, N={n})", "value": 1e3 / t,
           "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": args.precision, "data": "synthetic",
           "config": {"workload": f"cubic{L}_dense_{args.precision}", "n": n, "sp2_iters": iters},
           "tflops": (2.0 * n ** 3 * iters + 4.0 * n ** 3) / (t / 1e3) / 1e12,
           "fp64": {"ms_per_solve": t64, "iters": it64, "solves_per_s": 1e3 / t64},
           "err_vs_fp64": {"fro_over_n": err / n, "rel_fro": err / float(rho.norm().item())},
           "clocks": clk.summary()}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
