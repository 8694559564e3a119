#!/usr/bin/env python
"""Benchmark: AINV preconditioner apply GB/s on one B200 (or N replicas).

Workload (one step = one apply y = Z * D^-1 * W^T * x, trans 'N', FP64):
3-D convection-diffusion -Lap(u) + b.grad(u), 200^3 unit-cube grid
(n = 8,000,000, nnz(A) = 55,760,000), central diffusion, first-order upwind
convection, b = 10*(1,1,1)/sqrt(3); AINV factors from the left-looking
biconjugation with drop tolerance 0.1 and fill cap 20 per column.  Synthetic
input x ~ U(-1,1) (splitmix64, seed 0).  L2 (126 MB) is flushed between
timed steps by writing a 256 MB buffer outside the timed events.

value = algorithmic bytes of one apply, the unfused CSR minimum of the
        reference's data structure: nnz_wt*(s_v+4) + nnz_z*(s_v+4)
        + 2*(n+1)*4 + n*8 [x] + n*s_d [D^-1] + 2*n*s_t [t write+read]
        + n*8 [y] (FP64: s_v = s_d = s_t = 8), over the device time.  The
        sliced layout moves fewer bytes than that minimum (offset-mode slices
        store no per-entry index); those layout bytes are reported next to it
        (config.layout_*), and the measured DRAM traffic in `roofline`.
e2e   = the same bytes / time of the host-array entry point
        (ainv_gpu_apply_host: H2D of x, apply, D2H of y; pinned buffers).

--impl reference times the CPU restatement of the reference apply (the
oracle; the Fortran reference cannot be built here) on the host cores.
Multi-GPU: independent replicas, one per rank ("replicas only"), no
data-path collective; value = sum of bytes over ranks / max time.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mld-ainv_b200"))

IDIM = 200
BETA = (10 / np.sqrt(3),) * 3
FILL, THRESH = 20, 0.1
WORKLOAD = "convdiff3d_200_upwind_ainv_llk_drop0.1_fill20_apply_N"
METRIC = "AINV apply GB/s (% HBM peak)"


def csr_stage_bytes(n, nnz_wt, nnz_z, sv=8, sd=8, st=8, si=4):
    """Algorithmic bytes of the two 'N' sweeps, the per-unit figures of the
    unfused CSR minimum: (W^T entries + row pointers + x + D^-1 + t write,
    Z entries + row pointers + t read + y write)."""
    s1 = nnz_wt * (sv + si) + 4 * (n + 1) + 8 * n + sd * n + st * n
    s2 = nnz_z * (sv + si) + 4 * (n + 1) + st * n + 8 * n
    return s1, s2


def csr_apply_bytes(n, nnz_wt, nnz_z, sv=8, sd=8, st=8):
    """Algorithmic bytes of one 'N' apply (reference CSR format, int32 indices)."""
    return sum(csr_stage_bytes(n, nnz_wt, nnz_z, sv, sd, st))


def layout_bytes(n, lay, vsize, tsize):
    """Algorithmic bytes of the two 'N' sweeps for the device layout:
    values (nnz * vsize) + stored index words (column offsets per slice, or
    per-entry columns) + two slice pointers, plus the vectors each sweep
    streams.  Returns (sweep1, sweep2)."""
    def mat(m):
        return m["nnz"] * vsize + 4 * m["nidx"] + 8 * (m["nslices"] + 1)
    s1 = mat(lay["wt"]) + 8 * n + vsize * n + tsize * n      # x, D^-1, t write
    s2 = mat(lay["z"]) + tsize * n + 8 * n                   # t read, y write
    return s1, s2


PEAK = [6650.0, "fallback"]  # HBM GB/s the fractions use; set from measured_peaks()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def recorded_traffic(kernel: str):
    """DRAM bytes per launch from a committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_convdiff3d_200.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """NVML sampling of SM clock and throttle reasons while the timed loop runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle"}

    def __init__(self, index: int, period_s: float = 0.005):
        self.index, self.period = index, period_s
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self.ok = False

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self._nv, self._h = pynvml, h
            self.ok = True
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self.ok = False
        return self

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


VARIANTS = {"INVK": {"SUB_FILLIN": 1, "INV_FILLIN": 1},
            "INVT": {"SUB_FILLIN": 20, "SUB_ILUTHRS": 0.05, "INV_FILLIN": 20, "INV_THRESH": 0.05}}


def build_workload(idim=IDIM, solver="AINV"):
    import ainv
    irp, ja, val = ainv.pde.gen_pde3d(idim, "convdiff", BETA)
    if solver == "AINV":
        sv = ainv.mld_d_ainv_solver_type()
        sv.csetc("AINV_ALG", "LLK")
        sv.cseti("SUB_FILLIN", FILL)
        sv.csetr("SUB_ILUTHRS", THRESH)
    else:
        sv = (ainv.mld_d_invk_solver_type() if solver == "INVK"
              else ainv.mld_d_invt_solver_type())
        for k, v in VARIANTS[solver].items():
            (sv.csetr if isinstance(v, float) else sv.cseti)(k, v)
    sv.check()
    info = sv.build(irp, ja, val)
    if info != 0:
        raise RuntimeError(f"factor build failed: {ainv.last_error()}")
    return (irp, ja, val), sv


def cpu_baseline_apply(f, n, budget_s=10.0, max_reps=200, threads=None):
    """Oracle apply ('N') on all host cores (or `threads`) for a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    of = O.Factors(O.CSR(n, f["wt_irp"], f["wt_ja"], f["wt_val"]),
                   O.CSR(n, f["z_irp"], f["z_ja"], f["z_val"]), f["d"])
    cores = threads or os.cpu_count() or 1
    O.set_threads(cores)
    x = np.ascontiguousarray(np.random.default_rng(0).uniform(-1, 1, n))
    O.ainv_apply(of, x)  # warm
    t0, reps = time.perf_counter(), 0
    while reps < max_reps and time.perf_counter() - t0 < budget_s:
        O.ainv_apply(of, x)
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    return dt, reps, O.get_threads()


def max_over_ranks(v, world, torch, dist, device):
    """The largest v over the ranks (every rank receives it)."""
    if world == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ms_local, bytes_per_step, world, allmax):
    """Replicas only: every rank applies its own copy of the factors, with no
    data-path collective.  The job's step time is the slowest rank's, and the
    job moved world x bytes_per_step in it.  Returns (ms, GB/s)."""
    ms = allmax(ms_local)
    return ms, bytes_per_step * world / (ms * 1e-3) / 1e9


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import ainv
    irp, ja, val = ainv.pde.gen_pde3d(IDIM, "convdiff", BETA)
    n = len(irp) - 1
    of = O.ainv_build(O.CSR(n, irp, ja, val), "LLK", FILL, THRESH)
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    x = O.rand_uniform(0, n)
    for _ in range(max(args.warmup, 1)):
        O.ainv_apply(of, x)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.ainv_apply(of, x)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    B = csr_apply_bytes(n, of.wt.nnz, of.z.nnz)
    gbs = B / (ms * 1e-3) / 1e9
    out = {"impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "n": n, "nnz_A": int(len(ja)),
                      "nnz_wt": of.wt.nnz, "nnz_z": of.z.nnz, "bytes_per_apply": B},
           "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": O.get_threads(),
                            "kind": "port",
                            "sample": f"{args.steps} full 200^3 applies, CPU restatement of "
                                      "the reference apply (OpenMP over rows); the Fortran "
                                      "reference cannot be built here"},
           "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip solves/s and mixed legs")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-rates", default="50,100,140,2000",
                    help="mean arrival rates (requests/s) of the serving sweep")
    ap.add_argument("--serve-slots", type=int, default=32)
    ap.add_argument("--serve-hbm-gb", type=float, default=0.0,
                    help="device memory for admitted requests (0: half of the free HBM)")
    ap.add_argument("--serve-prec", default="FP32",
                    help="factor precision of the served operators (FP32: the workload's)")
    ap.add_argument("--serve-iters", type=int, default=4)
    ap.add_argument("--leg", default="all",
                    choices=["all", "block", "solve", "serve", "apply", "served200"],
                    help="run one leg alone (profiler captures of its kernels)")
    ap.add_argument("--leg-prec", default="FP32",
                    help="factor precision of the apply / solve legs run alone")
    ap.add_argument("--leg-pattern", default="stencil", choices=["stencil", "scattered"],
                    help="apply leg: the stencil factors, or the same rows with scattered "
                         "columns (per-entry column layout)")
    ap.add_argument("--leg-reps", type=int, default=5, help="applies of the apply leg")
    ap.add_argument("--leg-solver", default="AINV", choices=["AINV", "INVK", "INVT"],
                    help="factors of the apply leg: AINV, or the INVK(1,1) / INVT(0.05,20) "
                         "variants")
    ap.add_argument("--leg-itmax", type=int, default=2000,
                    help="iteration cap of the solve / block legs run alone")
    ap.add_argument("--leg-idim", type=int, default=0,
                    help="grid side of the solve / block legs run alone (0: their default)")
    ap.add_argument("--idim", type=int, default=IDIM,
                    help="grid side (default 200; smaller sizes for profiler captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    import ainv

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(v):
        return max_over_ranks(v, world, torch, dist, "cuda")

    if args.leg != "all":
        return run_leg(ainv, torch, args)

    (irp, ja, val), sv = build_workload(args.idim)
    n = len(irp) - 1
    f = sv.factors()
    assert sv.cnv("FP64") == 0, ainv.last_error()
    df = sv.device
    nnz = (len(f["wt_ja"]), len(f["z_ja"]))
    lay = {k: df.layout_info(k) for k in ("wt", "z")}
    lb = layout_bytes(n, lay, 8, 8)
    B_lay = lb[0] + lb[1]
    sb = csr_stage_bytes(n, *nnz)
    B = sb[0] + sb[1]
    B_csr = B
    dev = torch.device("cuda", local)
    x = torch.from_numpy(ainv.pde.rand_uniform(0, n)).to(dev)
    y = torch.zeros(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        df.apply(x, y, 1.0, 0.0, "N", stream)
    torch.cuda.synchronize()

    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        for k in range(K):
            flush.zero_()
            ev[k][0].record(stream)
            df.apply(x, y, 1.0, 0.0, "N", stream)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        barrier()
    ms, value = replica_value(sum(a.elapsed_time(b) for a, b in ev) / K, B, world, allmax)

    # per-sweep timing (roofline of the dominant kernel)
    K2 = min(K, 100)
    st = {1: [], 2: []}
    for stage in (1, 2):
        for _ in range(K2):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            df.apply_stage(stage, x=x, y=y, alpha=1.0, beta=0.0, trans="N", stream=stream)
            b.record(stream)
            st[stage].append((a, b))
    torch.cuda.synchronize()
    st_ms = {s: sum(a.elapsed_time(b) for a, b in st[s]) / K2 for s in st}
    dom = max((1, 2), key=lambda s: st_ms[s])
    # FP64 sweep 1 runs the streaming kernel unless AINV_STREAM=0 forces the
    # register family (AINV_STREAM=1 streams sweep 2 as well)
    forced = os.environ.get("AINV_STREAM")
    names = {1: "k_sweep_dscale" if forced == "0" else "k_stream_dscale",
             2: "k_stream_axpby" if forced == "1" else "k_sweep_axpby"}
    dom_name = names[dom]
    peak, peak_kind = measured_peaks()
    PEAK[:] = [peak, peak_kind]
    achieved = sb[dom - 1] / (st_ms[dom] * 1e-3) / 1e9
    traffic = recorded_traffic(dom_name)

    # end to end through the host-array entry point (pinned buffers)
    xh = torch.from_numpy(ainv.pde.rand_uniform(0, n)).pin_memory()
    yh = torch.zeros(n, dtype=torch.float64).pin_memory()
    import ctypes as C
    lib = ainv.lib()
    Ke = min(K, 50)
    for _ in range(3):
        lib.ainv_gpu_apply_host(df.handle, b"N", 1.0, C.c_void_p(xh.data_ptr()), 0.0,
                                C.c_void_p(yh.data_ptr()))
    torch.cuda.synchronize()
    barrier()
    legacy = torch.cuda.default_stream()  # the entry point runs on the legacy stream
    t_e2e = []
    for _ in range(Ke):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(legacy)
        info = lib.ainv_gpu_apply_host(df.handle, b"N", 1.0, C.c_void_p(xh.data_ptr()), 0.0,
                                       C.c_void_p(yh.data_ptr()))
        b.record(legacy)
        assert info == 0, ainv.last_error()
        t_e2e.append((a, b))
    torch.cuda.synchronize()
    e2e_ms = allmax(sum(a.elapsed_time(b) for a, b in t_e2e) / Ke)
    e2e = {"value": round(B * world / (e2e_ms * 1e-3) / 1e9, 3), "unit": "GB/s",
           "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
           "ms_per_step": round(e2e_ms, 4)}

    # the extra legs (solves, variants, block CG, serving) describe one GPU;
    # replica runs (N > 1) report the apply metric only
    extras = {}
    if not args.no_extras and world == 1:
        extras = run_extras(ainv, torch, dev, irp, ja, val, f, sv, flush, stream, ms)
        extras["block_cg"] = run_block_cg(ainv, torch, dev)
        if not args.no_cpu:
            extras["cpu_solves"] = run_cpu_solves(ainv, torch, dev, irp, ja, val, f, extras)
    if not args.no_serve and world == 1:
        extras["serving"] = run_serving(ainv, torch, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        dt, reps, cores = cpu_baseline_apply(f, n)
        dt1, reps1, _ = cpu_baseline_apply(f, n, budget_s=5.0, max_reps=50, threads=1)
        cpu = {"value": round(B_csr / dt / 1e9, 3), "unit": "GB/s", "cores": cores, "kind": "port",
               "sample": f"{reps} full 200^3 applies ({dt * 1e3:.1f} ms each) of the CPU "
                         "restatement of the reference apply, OpenMP over rows",
               "nproc": os.cpu_count(),
               "one_thread": {"value": round(B_csr / dt1 / 1e9, 3), "unit": "GB/s",
                              "ms_per_apply": round(dt1 * 1e3, 2), "applies": reps1}}

    if rank == 0:
        out = {"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
               "steps": K, "warmup": args.warmup, "ms_per_step": round(ms, 5),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic",
               "config": {"workload": WORKLOAD if args.idim == IDIM else
                          WORKLOAD.replace("_200_", f"_{args.idim}_"), "n": n, "nnz_A": int(len(ja)),
                          "nnz_wt": nnz[0], "nnz_z": nnz[1], "bytes_per_apply": B,
                          "bytes_model": "unfused CSR minimum (12 B per FP64 entry)",
                          "layout_bytes_per_apply": B_lay,
                          "layout_GBps": round(B_lay * world / (ms * 1e-3) / 1e9, 1),
                          "layout": "32-row slices, shared column offsets per slice",
                          "offset_slices": [lay["wt"]["offset_slices"], lay["z"]["offset_slices"]],
                          "nslices": lay["wt"]["nslices"],
                          "l2": "flushed between steps (256 MB write)",
                          "parallelism": f"replicas{world}",
                          "pct_of_hbm_peak": round(100 * value / world / peak, 2)},
               "roofline": {"bound": "hbm", "kernel": dom_name,
                            "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                            "traffic": traffic, "algorithmic_bytes": sb[dom - 1],
                            "layout_bytes": lb[dom - 1],
                            "layout_frac": round(lb[dom - 1] / (st_ms[dom] * 1e-3) / 1e9 / peak, 4),
                            "stage_ms": {names[1]: round(st_ms[1], 5),
                                         names[2]: round(st_ms[2], 5)}},
               "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
               "gpu_launches": 2 * K}
        out.update(extras)
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_extras(ainv, torch, dev, irp, ja, val, f, sv, flush, stream, fp64_ms):
    """Mixed-precision apply GB/s, BiCGSTAB solves/s (FP64 vs FP32 factors),
    and the INVK / INVT variants."""
    n = len(irp) - 1
    nnz = (len(f["wt_ja"]), len(f["z_ja"]))
    out = {"mixed": {}, "solve": {}}
    x = torch.from_numpy(ainv.pde.rand_uniform(0, n)).to(dev)
    y = torch.zeros(n, dtype=torch.float64, device=dev)
    for prec, vs, ts in [("FP32", 4, 4), ("BF16", 2, 4), ("FP32_ACC64", 4, 8),
                         ("BF16_ACC64", 2, 8)]:
        df = ainv.DeviceFactors((f["wt_irp"], f["wt_ja"], f["wt_val"]),
                                (f["z_irp"], f["z_ja"], f["z_val"]), f["d"], prec=prec)
        for _ in range(5):
            df.apply(x, y, 1.0, 0.0, "N", stream)
        evs = []
        for _ in range(50):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            df.apply(x, y, 1.0, 0.0, "N", stream)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / len(evs)
        Bl = sum(layout_bytes(n, {k: df.layout_info(k) for k in ("wt", "z")}, vs, ts))
        Bm = csr_apply_bytes(n, nnz[0], nnz[1], sv=vs, sd=vs, st=ts)
        out["mixed"][prec] = {"ms": round(ms, 5), "GB/s": round(Bm / (ms * 1e-3) / 1e9, 2),
                              "bytes": Bm, "layout_bytes": Bl,
                              "layout_GBps": round(Bl / (ms * 1e-3) / 1e9, 2),
                              "layout_frac": round(Bl / (ms * 1e-3) / 1e9 / PEAK[0], 4),
                              "speedup_vs_fp64": round(fp64_ms / ms, 3)}
        df.close()
    # the transposed apply y = W D^-1 Z^T x (trans 'T'), FP64 factors: same
    # algorithmic bytes as 'N' (Z^T has nnz_Z entries, W has nnz_W)
    df = sv.device
    for _ in range(5):
        df.apply(x, y, 1.0, 0.0, "T", stream)
    evs = []
    for _ in range(50):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        df.apply(x, y, 1.0, 0.0, "T", stream)
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs) / len(evs)
    Bt = csr_apply_bytes(n, nnz[1], nnz[0], sv=8, sd=8, st=8)
    out["trans_T"] = {"ms": round(ms, 5), "GB/s": round(Bt / (ms * 1e-3) / 1e9, 2),
                      "bytes": Bt, "vs_N": round(fp64_ms / ms, 3)}
    # BiCGSTAB to 1e-9, b = A x*, x* ~ U(-1,1) seed 0
    A = ainv.DeviceOperator(irp, ja, val)
    xs = torch.from_numpy(ainv.pde.rand_uniform(0, n)).to(dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    A.spmv(xs, b, 1.0, 0.0, stream)
    bn = float(torch.linalg.vector_norm(b))
    for prec in ["FP64", "FP32", "BF16", "FP32_ACC64", "BF16_ACC64"]:
        if prec != "FP64":
            sv.cnv(prec)
        df = sv.device
        res = None
        times = []
        for rep in range(3):
            xx = torch.zeros(n, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = A.solve(b, xx, df, "BICGSTAB", 1e-9, 2000, stream)
            times.append(time.perf_counter() - t0)
        r = torch.empty_like(b)
        A.spmv(xx, r, 1.0, 0.0, stream)
        true_rel = float(torch.linalg.vector_norm(b - r)) / bn
        err_x = float((xx - xs).abs().max())
        out["solve"][prec] = {"iters": res.iter, "info": res.info, "relres": res.err,
                              "true_relres": true_rel, "max_err_vs_xstar": err_x,
                              "s_per_solve": round(min(times), 5),
                              "solves_per_s": round(1.0 / min(times), 3)}
    # iteration counts move by ~20% under rounding-level changes, so the
    # precisions are also compared over three right-hand sides (x* seeds 0-2)
    seeds = {}
    for prec in ["FP64", "FP32", "BF16", "FP32_ACC64", "BF16_ACC64"]:
        sv.cnv(prec)
        its, ts = [], []
        for seed in range(3):
            xs_k = torch.from_numpy(ainv.pde.rand_uniform(seed, n)).to(dev)
            b_k = torch.zeros(n, dtype=torch.float64, device=dev)
            A.spmv(xs_k, b_k, 1.0, 0.0, stream)
            xx = torch.zeros(n, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r_k = A.solve(b_k, xx, sv.device, "BICGSTAB", 1e-9, 2000, stream)
            ts.append(time.perf_counter() - t0)
            its.append(r_k.iter)
        seeds[prec] = {"iters": its, "s_total": round(sum(ts), 4),
                       "solves_per_s": round(3 / sum(ts), 3)}
    for prec in ("FP32", "BF16", "FP32_ACC64", "BF16_ACC64"):
        seeds[prec]["speedup_vs_fp64"] = round(seeds["FP64"]["s_total"] / seeds[prec]["s_total"], 3)
    out["solve_3rhs"] = seeds
    sv.cnv("FP64")
    out["variants"] = run_variants(ainv, torch, dev, irp, ja, val, A, b, bn, xs, x, y,
                                   flush, stream)
    A.close()
    out["general_pattern"] = run_general_pattern(ainv, torch, dev, f, x, y, flush, stream)
    served = run_served_200(ainv, torch, dev, irp, ja, val, sv)
    # the precision configuration at 200^3: plain (one solve at a time) and
    # served, each against the plain FP64 solve; residuals are FP64 b - A x
    fp64 = seeds["FP64"]["solves_per_s"]
    out["mixed_200"] = {
        "target": "mixed-precision served solve >= 1.5x the plain FP64 solve's solves/s "
                  "at FP64 relative residual 1e-9",
        "plain": {p: {"solves_per_s": seeds[p]["solves_per_s"],
                      "vs_fp64": round(seeds[p]["solves_per_s"] / fp64, 3),
                      "iters_3rhs": seeds[p]["iters"],
                      "true_relres_seed0": out["solve"][p]["true_relres"],
                      "max_err_vs_xstar_seed0": out["solve"][p]["max_err_vs_xstar"]}
                  for p in seeds},
        "served": served,
        # reduced-precision modes whose served solve meets the target: every
        # request converged, every final FP64 residual <= 1e-9, >= 1.5x
        "target_met_by": sorted(
            m for m, r in served["served"].items()
            if m != "FP64" and r["vs_plain_fp64"] is not None and r["vs_plain_fp64"] >= 1.5
            and r["converged"] == served["requests"] and r["max_final_fp64_relres"] <= 1e-9)}
    return out


def run_served_200(ainv, torch, dev, irp, ja, val, sv, requests=16, slots=16, iters=4,
                   modes=("FP32_ACC64", "BF16_ACC64", "FP32", "BF16", "FP64"), plain=True):
    """The mixed-precision, served solve on the 200^3 convection-diffusion
    case against the plain FP64 GPU solve.  `requests` right-hand sides
    b_k = A x*_k (x*_k ~ U(-1,1), seed k), BiCGSTAB to 1e-9 from x0 = 0:
      plain_fp64: ainv_gpu_solve with FP64 factors, one system after another;
      served[mode]: all requests submitted at once to a solve server holding
        the operator with factors of that precision; the server batches
        them (requests on one operator share its reads) and confirms each
        result on the FP64 true residual b - A x.
    solves/s = requests / (last completion - first submission); latency =
    submission of the host b -> solution in the host x buffer."""
    from ainv import serve
    n = len(irp) - 1
    A = ainv.DeviceOperator(irp, ja, val)
    xstar = [ainv.pde.rand_uniform(k, n) for k in range(requests)]
    bh = []
    for k in range(requests):
        bd = torch.zeros(n, dtype=torch.float64, device=dev)
        A.spmv(torch.from_numpy(xstar[k]).to(dev), bd, 1.0, 0.0)
        bh.append(bd.cpu().pin_memory())
    out = {"workload": "convdiff3d_200_upwind_bicgstab_1e-9_ainv_llk_drop0.1_fill20",
           "requests": requests, "slots": slots, "iters_per_launch": iters}
    out["served"] = {}
    plain_sps = None
    if plain:
        plain_sps, out["plain_fp64"] = plain_fp64_solves(ainv, torch, dev, A, sv, bh, requests)
    for mode in modes:
        assert sv.cnv(mode) == 0, ainv.last_error()
        xh = [torch.zeros(n, dtype=torch.float64).pin_memory() for _ in range(requests)]
        with serve.SolveServer(max_slots=slots, iters_per_launch=iters) as srv:
            op = srv.add_operator(A, sv.device)
            srv.wait(srv.submit(op, bh[0], xh[0], 1e-9, 2000))  # warm-up: graph capture
            rids = [srv.submit(op, bh[k], xh[k], 1e-9, 2000) for k in range(requests)]
            res = [srv.wait(q) for q in rids]
            st = srv.stats()
        t_first = min(q.t_submit for q in res)
        t_last = max(q.t_done for q in res)
        lat = np.array([q.latency for q in res]) * 1e3
        sps = requests / (t_last - t_first)
        out["served"][mode] = {
            "solves_per_s": round(sps, 3),
            "vs_plain_fp64": round(sps / plain_sps, 3) if plain_sps else None,
            "converged": int(sum(q.converged for q in res)),
            "max_final_fp64_relres": float(max(q.err for q in res)),
            "max_err_vs_xstar": float(max(np.abs(xh[k].numpy() - xstar[k]).max()
                                          for k in range(requests))),
            "iters_mean": round(float(np.mean([q.iter for q in res])), 2),
            "iters_max": int(max(q.iter for q in res)),
            "p50_ms": round(float(np.percentile(lat, 50)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2),
            "peak_active": st["peak_active"]}
    assert sv.cnv("FP64") == 0, ainv.last_error()
    A.close()
    return out


def plain_fp64_solves(ainv, torch, dev, A, sv, bh, requests):
    """The plain FP64 GPU solve of the same right-hand sides, one after
    another (device b and x): (solves/s, record)."""
    n = A.n
    assert sv.cnv("FP64") == 0, ainv.last_error()
    its, t_tot = [], 0.0
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    A.solve(bh[0].to(dev), x, sv.device, "BICGSTAB", 1e-9, 2000)  # warm-up
    for k in range(requests):
        b = bh[k].to(dev)
        x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = A.solve(b, x, sv.device, "BICGSTAB", 1e-9, 2000)
        torch.cuda.synchronize()
        t_tot += time.perf_counter() - t0
        its.append(r.iter)
    sps = requests / t_tot
    return sps, {"solves_per_s": round(sps, 3), "iters_mean": round(float(np.mean(its)), 2),
                 "iters": its}


def scattered_factors(f, band=40_000, seed=1):
    """General (not stencil-shaped) factors with the same rows, values and
    diagonal as f: every off-diagonal entry of row i of W^T moves to a
    column drawn uniformly from [i - band, i), and of Z from (i, i + band]
    (band 40,000 = one z-plane of the 200^3 grid, the stencil's own reach).
    The factors stay unit triangular, but no two rows share a column
    pattern, so the layout falls back to one column index per entry."""
    rng = np.random.default_rng(seed)
    n = len(f["d"])
    out = {"d": np.ascontiguousarray(f["d"])}
    for k, lower in (("wt", True), ("z", False)):
        irp, ja, val = f[k + "_irp"], f[k + "_ja"], f[k + "_val"]
        row = np.repeat(np.arange(n, dtype=np.int64), np.diff(irp))
        diag = ja == row
        reach = np.minimum(row, band) if lower else np.minimum(n - 1 - row, band)
        off = 1 + (rng.random(len(ja)) * np.maximum(reach, 1)).astype(np.int64)
        col = np.where(diag, row, row - off if lower else row + off)
        ok = diag | (reach > 0)
        row, col, v = row[ok], col[ok], val[ok]
        order = np.lexsort((col, row))
        row, col, v = row[order], col[order], v[order]
        keep = np.ones(len(col), bool)
        keep[1:] = (row[1:] != row[:-1]) | (col[1:] != col[:-1])  # drop collisions
        row, col, v = row[keep], col[keep], v[keep]
        out[k + "_irp"] = np.concatenate([[0], np.cumsum(np.bincount(row, minlength=n))]).astype(np.int32)
        out[k + "_ja"] = col.astype(np.int32)
        out[k + "_val"] = np.ascontiguousarray(v, np.float64)
    return out


def run_general_pattern(ainv, torch, dev, f, x, y, flush, stream, reps=30):
    """The apply on factors that are not stencil-shaped: the 200^3 factors
    with every off-diagonal column scattered within the stencil's reach
    (scattered_factors), FP64, L2 flushed between applies."""
    n = len(f["d"])
    g = scattered_factors(f)
    df = ainv.DeviceFactors((g["wt_irp"], g["wt_ja"], g["wt_val"]),
                            (g["z_irp"], g["z_ja"], g["z_val"]), g["d"])
    lay = {k: df.layout_info(k) for k in ("wt", "z")}
    for _ in range(3):
        df.apply(x, y, 1.0, 0.0, "N", stream)
    evs = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        df.apply(x, y, 1.0, 0.0, "N", stream)
        b.record(stream)
        evs.append((a, b))
    st = {}
    for stage in (1, 2):
        ev2 = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            df.apply_stage(stage, x=x, y=y, alpha=1.0, beta=0.0, trans="N", stream=stream)
            b.record(stream)
            ev2.append((a, b))
        torch.cuda.synchronize()
        st[stage] = sum(a.elapsed_time(b) for a, b in ev2) / reps
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs) / reps
    B = csr_apply_bytes(n, len(g["wt_ja"]), len(g["z_ja"]))
    lb = layout_bytes(n, lay, 8, 8)
    df.close()
    return {"workload": "convdiff3d_200 AINV factors, off-diagonal columns scattered "
                        "uniformly within 40,000 of the diagonal (seed 1), FP64 'N' apply",
            "offset_slices": [lay["wt"]["offset_slices"], lay["z"]["offset_slices"]],
            "nslices": lay["wt"]["nslices"], "slots": [lay["wt"]["slots"], lay["z"]["slots"]],
            "ms": round(ms, 5), "GB/s": round(B / (ms * 1e-3) / 1e9, 2), "bytes": B,
            "layout_bytes": sum(lb), "layout_GBps": round(sum(lb) / (ms * 1e-3) / 1e9, 2),
            "layout_frac": round(sum(lb) / (ms * 1e-3) / 1e9 / PEAK[0], 4),
            "stage_ms": [round(st[1], 5), round(st[2], 5)],
            "stage_layout_frac": [round(lb[i] / (st[i + 1] * 1e-3) / 1e9 / PEAK[0], 4)
                                  for i in range(2)]}


def run_variants(ainv, torch, dev, irp, ja, val, A, b, bn, xs, x, y, flush, stream):
    """The INVK (fill level 1) and INVT (threshold 0.05, fill cap 20) solvers
    on the same matrix and right-hand side: host build time, FP64 apply GB/s
    (layout bytes, L2 flushed), and BiCGSTAB to 1e-9 with FP64 and FP32
    factors."""
    n = len(irp) - 1
    out = {}
    for name, kv in VARIANTS.items():
        sv = (ainv.mld_d_invk_solver_type() if name == "INVK"
              else ainv.mld_d_invt_solver_type())
        for k, v in kv.items():
            (sv.csetr if isinstance(v, float) else sv.cseti)(k, v)
        t0 = time.perf_counter()
        info = sv.build(irp, ja, val)
        t_build = time.perf_counter() - t0
        if info != 0:
            out[name] = {"info": info, "error": ainv.last_error()}
            continue
        f = sv.factors()
        rec = {"settings": kv, "build_s": round(t_build, 2),
               "nnz_wt": int(len(f["wt_ja"])), "nnz_z": int(len(f["z_ja"]))}
        assert sv.cnv("FP64") == 0, ainv.last_error()
        df = sv.device
        for _ in range(5):
            df.apply(x, y, 1.0, 0.0, "N", stream)
        evs = []
        for _ in range(30):
            flush.zero_()
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            df.apply(x, y, 1.0, 0.0, "N", stream)
            e.record(stream)
            evs.append((a, e))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(e) for a, e in evs) / len(evs)
        Bl = sum(layout_bytes(n, {k: df.layout_info(k) for k in ("wt", "z")}, 8, 8))
        Bv = csr_apply_bytes(n, rec["nnz_wt"], rec["nnz_z"])
        rec["apply"] = {"ms": round(ms, 5), "GB/s": round(Bv / (ms * 1e-3) / 1e9, 2),
                        "bytes": Bv, "layout_bytes": Bl,
                        "layout_GBps": round(Bl / (ms * 1e-3) / 1e9, 2),
                        "layout_frac": round(Bl / (ms * 1e-3) / 1e9 / PEAK[0], 4)}
        rec["solve"] = {}
        for prec in ("FP64", "FP32"):
            if prec != "FP64":
                sv.cnv(prec)
            times, res = [], None
            for _ in range(2):
                xx = torch.zeros(n, dtype=torch.float64, device=dev)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res = A.solve(b, xx, sv.device, "BICGSTAB", 1e-9, 2000, stream)
                times.append(time.perf_counter() - t0)
            r = torch.empty_like(b)
            A.spmv(xx, r, 1.0, 0.0, stream)
            rec["solve"][prec] = {
                "iters": res.iter, "info": res.info, "relres": res.err,
                "true_relres": float(torch.linalg.vector_norm(b - r)) / bn,
                "max_err_vs_xstar": float((xx - xs).abs().max()),
                "s_per_solve": round(min(times), 5), "solves_per_s": round(1.0 / min(times), 3)}
        sv.free()
        out[name] = rec
    return out


def run_cpu_solves(ainv, torch, dev, irp, ja, val, f, extras):
    """The CPU side of the solve workloads, on all host cores with the
    oracle's restated Krylov loop (FP64 factors: the CPU path has no other),
    next to the GPU figure of the same workload:
      poisson40_cg: 40^3 Poisson (6/-1), b = A*1, x0 = 0, AINV drop 0.1 fill 20,
                    CG to 1e-9;
      convdiff200_bicgstab: the 200^3 convection-diffusion system of the solve
                    leg, BiCGSTAB to 1e-9;
      poisson128_cg_per_rhs: one of the 32 right-hand sides of the block leg
                    (128^3 Poisson, CG to 1e-9); 32 sequential CPU solves are
                    32 x that time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)

    def factors(d):
        m = len(d["d"])
        return O.Factors(O.CSR(m, d["wt_irp"], d["wt_ja"], d["wt_val"]),
                         O.CSR(m, d["z_irp"], d["z_ja"], d["z_val"]), d["d"])

    def cpu(method, a_irp, a_ja, a_val, fd, b, order="device"):
        a = O.CSR(len(a_irp) - 1, a_irp, a_ja, a_val)
        t = time.perf_counter()
        _, it, err, rc = O.solve(method, a, factors(fd), b, eps=1e-9, itmax=3000, order=order)
        return {"s_per_solve": round(time.perf_counter() - t, 4), "iters": it,
                "relres": err, "info": rc}

    def build(i, j, v):
        sv = ainv.mld_d_ainv_solver_type()
        sv.cseti("SUB_FILLIN", FILL)
        sv.csetr("SUB_ILUTHRS", THRESH)
        assert sv.build(i, j, v) == 0, ainv.last_error()
        return sv.factors()

    out = {"threads": cores, "kind": "port"}
    # 40^3 Poisson, CG
    i1, j1, v1 = ainv.pde.gen_pde3d(40, "poisson")
    f1 = build(i1, j1, v1)
    n1 = len(i1) - 1
    b1 = O.spmv(O.CSR(n1, i1, j1, v1), np.ones(n1))
    A1 = ainv.DeviceOperator(i1, j1, v1)
    d1 = ainv.DeviceFactors((f1["wt_irp"], f1["wt_ja"], f1["wt_val"]),
                            (f1["z_irp"], f1["z_ja"], f1["z_val"]), f1["d"])
    bt = torch.from_numpy(b1).to(dev)
    gpu_t = []
    for _ in range(4):
        xg = torch.zeros(n1, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = A1.solve(bt, xg, d1, "CG", 1e-9, 3000)
        torch.cuda.synchronize()
        gpu_t.append(time.perf_counter() - t)
    c1 = cpu("CG", i1, j1, v1, f1, b1)
    out["poisson40_cg"] = {"cpu": c1, "gpu": {"s_per_solve": round(min(gpu_t[1:]), 5),
                                                      "iters": r.iter, "relres": r.err},
                                   "gpu_speedup": round(c1["s_per_solve"] / min(gpu_t[1:]), 2)}
    d1.close()
    A1.close()
    # 200^3 convection-diffusion, BiCGSTAB
    n = len(irp) - 1
    xs = ainv.pde.rand_uniform(0, n)
    b2 = O.spmv(O.CSR(n, irp, ja, val), xs)
    c2 = cpu("BICGSTAB", irp, ja, val, f, b2)
    g2 = extras.get("solve", {}).get("FP64", {}).get("s_per_solve")
    gi = extras.get("solve", {}).get("FP64", {}).get("iters")
    # the same solve with sequential dots (the reference BLAS ddot order):
    # the count the oracle reaches when only the summation order changes
    c2s = cpu("BICGSTAB", irp, ja, val, f, b2, order="sequential")
    out["convdiff200_bicgstab"] = {"cpu": c2, "gpu_s_per_solve": g2,
                                   "gpu_speedup": round(c2["s_per_solve"] / g2, 2)
                                   if g2 else None,
                                   "iterations": {"gpu": gi, "oracle_device_order": c2["iters"],
                                                  "oracle_sequential_dots": c2s["iters"],
                                                  "gpu_equals_oracle": gi == c2["iters"]}}
    # 128^3 Poisson, one of the block leg's right-hand sides
    i4, j4, v4 = ainv.pde.gen_pde3d(128, "poisson")
    f4 = build(i4, j4, v4)
    b4 = ainv.pde.rand_normal(0, len(i4) - 1)
    c4 = cpu("CG", i4, j4, v4, f4, b4)
    gb = extras.get("block_cg", {}).get("s_per_block_solve")
    out["poisson128_cg_per_rhs"] = {
        "cpu": c4, "cpu_32_sequential_s": round(32 * c4["s_per_solve"], 2),
        "gpu_block_s": gb,
        "gpu_speedup": round(32 * c4["s_per_solve"] / gb, 2) if gb else None}
    return out


def run_block_cg(ainv, torch, dev, idim=128, m=32, itmax=2000, reps=3, single=True):
    """Multi-right-hand-side CG: 3-D Poisson on a 128^3 grid, 32 right-hand
    sides N(0,1) (seed k for column k), AINV drop 0.1 fill 20 with FP32
    factors, FP64 A, CG to 1e-9 per column.  One block solve (SpMM products)
    against the same 32 systems solved one after another."""
    irp, ja, val = ainv.pde.gen_pde3d(idim, "poisson")
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", FILL)
    sv.csetr("SUB_ILUTHRS", THRESH)
    assert sv.build(irp, ja, val) == 0, ainv.last_error()
    assert sv.cnv("FP32") == 0, ainv.last_error()
    A = ainv.DeviceOperator(irp, ja, val)
    Bh = np.stack([ainv.pde.rand_normal(k, n) for k in range(m)], axis=1)
    B = torch.from_numpy(Bh).to(dev)
    X = torch.zeros_like(B)
    A.block_solve(B, X, sv.device, 1e-9, itmax)  # warm-up (workspace, graph)
    times = []
    for _ in range(reps):
        X.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = A.block_solve(B, X, sv.device, 1e-9, itmax)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    R = B.clone()
    for l in range(m):
        r = torch.empty(n, dtype=torch.float64, device=dev)
        A.spmv(X[:, l].contiguous(), r, 1.0, 0.0)
        R[:, l] -= r
    rel = (torch.linalg.vector_norm(R, dim=0) / torch.linalg.vector_norm(B, dim=0)).max()
    # the same systems one at a time through the single-vector loop
    t_single, it_single = 0.0, []
    for l in range(m if single else 0):
        b = B[:, l].contiguous()
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        if l == 0:
            A.solve(b, x, sv.device, "CG", 1e-9, 2000)
            x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r1 = A.solve(b, x, sv.device, "CG", 1e-9, 2000)
        torch.cuda.synchronize()
        t_single += time.perf_counter() - t0
        it_single.append(r1.iter)
    tb = min(times)
    out = {"workload": f"poisson3d_{idim}_ainv_drop0.1_fill20_fp32_cg_{m}rhs", "n": n,
           "rhs": m, "converged": bool(res.converged), "max_true_relres": float(rel),
           "iters_mean": round(float(np.mean(res.iters)), 2), "iters_max": int(max(res.iters)),
           "s_per_block_solve": round(tb, 4), "rhs_solves_per_s": round(m / tb, 2),
           "single_rhs_s_total": round(t_single, 4) if single else None,
           "single_rhs_solves_per_s": round(m / t_single, 2) if single else None,
           "single_iters_mean": round(float(np.mean(it_single)), 2) if single else None,
           "speedup_vs_single": round(t_single / tb, 3) if single else None}
    A.close()
    sv.free()
    return out


def run_leg(ainv, torch, args):
    """One leg alone, e.g. under a profiler: `block` (multi-RHS CG),
    `solve` (one BiCGSTAB solve of the convection-diffusion workload with
    `--leg-prec` factors), `apply` (applies of those factors), `served200`
    (`--leg-reps` such solves served together) or `serve` (the serving
    stream)."""
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    if args.leg == "block":
        out = run_block_cg(ainv, torch, dev, idim=args.leg_idim or 128, itmax=args.leg_itmax,
                           reps=1, single=False)
    elif args.leg == "served200":
        # `--leg-reps` requests of the 200^3 (or --leg-idim) solve served
        # together with `--leg-prec` factors, no plain comparison
        (irp, ja, val), sv = build_workload(args.leg_idim or IDIM)
        out = run_served_200(ainv, torch, dev, irp, ja, val, sv, requests=args.leg_reps,
                             slots=args.leg_reps, modes=(args.leg_prec,), plain=False)
    elif args.leg == "apply":
        # `--leg-reps` applies ('N') of the convection-diffusion factors in
        # `--leg-prec`, each after an L2 flush
        (irp, ja, val), sv = build_workload(args.leg_idim or IDIM, args.leg_solver)
        n = len(irp) - 1
        f = sv.factors()
        if args.leg_pattern == "scattered":
            f = scattered_factors(f)
        df = ainv.DeviceFactors((f["wt_irp"], f["wt_ja"], f["wt_val"]),
                                (f["z_irp"], f["z_ja"], f["z_val"]), f["d"], prec=args.leg_prec)
        x = torch.from_numpy(ainv.pde.rand_uniform(0, n)).to(dev)
        y = torch.zeros(n, dtype=torch.float64, device=dev)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        evs = []
        for _ in range(args.leg_reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            df.apply(x, y, 1.0, 0.0, "N")
            b.record()
            evs.append((a, b))
        torch.cuda.synchronize()
        out = {"n": n, "prec": args.leg_prec, "pattern": args.leg_pattern,
               "ms": [round(a.elapsed_time(b), 4) for a, b in evs],
               "layout": {k: df.layout_info(k) for k in ("wt", "z")}}
        df.close()
    elif args.leg == "serve":
        out = run_serving(ainv, torch, args)
    else:
        (irp, ja, val), sv = build_workload(args.leg_idim or IDIM)
        n = len(irp) - 1
        assert sv.cnv(args.leg_prec) == 0, ainv.last_error()
        A = ainv.DeviceOperator(irp, ja, val)
        xs = torch.from_numpy(ainv.pde.rand_uniform(0, n)).to(dev)
        b = torch.zeros(n, dtype=torch.float64, device=dev)
        A.spmv(xs, b, 1.0, 0.0)
        x = torch.zeros_like(b)
        A.solve(b, x, sv.device, "BICGSTAB", 1e-9, args.leg_itmax)
        x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = A.solve(b, x, sv.device, "BICGSTAB", 1e-9, args.leg_itmax)
        torch.cuda.synchronize()
        out = {"n": n, "iters": res.iter, "info": res.info, "relres": res.err,
               "s": round(time.perf_counter() - t0, 5)}
        A.close()
    print(json.dumps({"leg": args.leg, **out}), flush=True)
    return 0


def run_serving(ainv, torch, args):
    """Serving: a stream of BiCGSTAB requests (tol 1e-8, FP32 factors, x0 = 0)
    with Poisson arrivals against 16 resident operators (3-D Poisson and
    convection-diffusion, n^3 grids with n log-uniform in [24, 128], AINV
    drop 0.1 fill 20), N(0,1) right-hand sides seeded by the request id.
    Latency = submit (host b) -> solution in the host x buffer."""
    from ainv import serve, workload
    specs = workload.serving_operators()
    t0 = time.perf_counter()
    ops, host = [], []
    for sp in specs:
        irp, ja, val = ainv.pde.gen_pde3d(sp.idim, sp.kind, sp.beta)
        sv = ainv.mld_d_ainv_solver_type()
        sv.cseti("SUB_FILLIN", FILL)
        sv.csetr("SUB_ILUTHRS", THRESH)
        assert sv.build(irp, ja, val) == 0, ainv.last_error()
        f = sv.factors()
        ops.append((ainv.DeviceOperator(irp, ja, val),
                    ainv.DeviceFactors((f["wt_irp"], f["wt_ja"], f["wt_val"]),
                                       (f["z_irp"], f["z_ja"], f["z_val"]), f["d"],
                                       prec=args.serve_prec), sp.n))
        host.append((irp, ja, val, f))
    t_build = time.perf_counter() - t0
    nreq = args.serve_requests
    opsel = workload.request_ops(nreq, len(ops))
    rhs = [torch.from_numpy(workload.request_rhs(r, ops[opsel[r]][2])).pin_memory()
           for r in range(nreq)]
    xs = [torch.zeros(ops[opsel[r]][2], dtype=torch.float64).pin_memory() for r in range(nreq)]

    def stream(rate, count, slots):
        arr = workload.poisson_arrivals(rate, count)
        with serve.SolveServer(max_slots=slots, iters_per_launch=args.serve_iters,
                               hbm_bytes=int(args.serve_hbm_gb * 2**30)) as srv:
            ids = [srv.add_operator(a, f) for a, f, _ in ops]
            srv.wait(srv.submit(ids[0], rhs[0], xs[0]))  # warm-up
            start = time.perf_counter()
            rids = []
            for r in range(count):
                dt = arr[r] - (time.perf_counter() - start)
                if dt > 0:
                    time.sleep(dt)
                rids.append(srv.submit(ids[opsel[r]], rhs[r], xs[r], 1e-8, 2000))
            res = [srv.wait(q) for q in rids]
            st = srv.stats()
        t_first = min(q.t_submit for q in res)
        t_last = max(q.t_done for q in res)
        lat = np.array([q.latency for q in res]) * 1e3
        wait = np.array([q.t_admit - q.t_submit for q in res]) * 1e3
        return {"rate": rate, "requests": count, "converged": int(sum(q.converged for q in res)),
                "max_relres": float(max(q.err for q in res)),
                "solves_per_s": round(count / (t_last - t_first), 2),
                "p50_ms": round(float(np.percentile(lat, 50)), 3),
                "p90_ms": round(float(np.percentile(lat, 90)), 3),
                "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "mean_queue_ms": round(float(wait.mean()), 3),
                "iters_mean": round(float(np.mean([q.iter for q in res])), 2),
                "peak_active": st["peak_active"], "graph_launches": st["graph_launches"],
                "kernel_launches": st["kernel_launches"],
                "arena_peak_bytes": st["arena_peak"], "arena_bytes": st["arena_bytes"]}

    sweep = [stream(float(r), nreq, args.serve_slots) for r in args.serve_rates.split(",")]
    # the same kernels with one slot: requests served one after another
    unbatched = stream(float(args.serve_rates.split(",")[-1]), min(nreq, 300), 1)
    for a, f, _ in ops:
        f.close()
        a.close()
    cpu = None
    if not args.no_cpu:
        # the same requests solved one after another on the host cores (the
        # oracle's restated BiCGSTAB, FP64 factors), for up to 15 s
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        O.set_threads(os.cpu_count() or 1)
        t, done = time.perf_counter(), 0
        while done < nreq and time.perf_counter() - t < 15.0:
            hi, hj, hv, hf = host[opsel[done]]
            m = len(hi) - 1
            O.solve("BICGSTAB", O.CSR(m, hi, hj, hv),
                    O.Factors(O.CSR(m, hf["wt_irp"], hf["wt_ja"], hf["wt_val"]),
                              O.CSR(m, hf["z_irp"], hf["z_ja"], hf["z_val"]), hf["d"]),
                    rhs[done].numpy(), eps=1e-8, itmax=2000)
            done += 1
        cpu = {"requests": done, "solves_per_s": round(done / (time.perf_counter() - t), 2),
               "threads": os.cpu_count() or 1, "kind": "port",
               "sample": "the first requests of the stream, solved one after another"}
    return {"cpu_sequential": cpu, "operators": [{"idim": sp.idim, "kind": sp.kind,
                           "beta": [round(b, 3) for b in sp.beta]} for sp in specs],
            "factors": f"AINV LLK drop 0.1 fill 20, {args.serve_prec}", "tol": 1e-8,
            "slots": args.serve_slots, "iters_per_launch": args.serve_iters,
            "build_s": round(t_build, 1), "sweep": sweep, "unbatched_one_slot": unbatched}


if __name__ == "__main__":
    sys.exit(main())
