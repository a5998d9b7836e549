"""Benchmark of the SIMPLE outer iteration (Ixchel2D hot path) on B200.

Workload: the heated lid-driven cavity in mixed convection, Re=100, Ri=1,
Pr=0.71, on a 701x301 staggered mesh (mi=701, nj=301: 702x302 = 212,004
p-cells) with tanh wall clustering (parameter 1.2), synthetic inputs built
in code (no dataset involved).  A step is ITERS outer SIMPLE iterations (one
inner pass of each equation, as conv_u/p/t are set so each inner loop exits
after its first pass).  Metric: Mcell-iter/s (p-cells x outer iterations per
second), whole job over all ranks, of the FP32+FP64-refined form
(IXB_PREC_FP32_REFINED: binary32 line solves, binary64 defect correction);
the plain binary64 form is timed beside it on the same box.  Both forms are
also run to a converged answer on the benchmark case itself, from rest until
the heated (bottom) wall's Nusselt number changes by less than 1e-8 over 1000
outer iterations (the on-device monitor of ixb_simple_converge), where their
Nusselt numbers, fields and wall times are compared; and to mass residual
< 1e-8 on the 64x64 natural-convection cavity.

The working set (~45 MB) fits the 126 MB L2, so L2 is flushed (a 256 MiB
write) before every timed step and every timed kernel launch.

--impl reference times the CPU restatement of the reference (oracle/, the
reference itself is Fortran + OpenACC and cannot be built here) on all host
cores for the same workload and metric.

Multi-GPU: one instance does not shard (every sweep spans the whole domain),
so N ranks run N independent replicas (weak scaling, no collective on the
data path); value = cells x iterations of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ITERS = 20                 # outer iterations per step
# converged leg at the benchmark size: Nusselt monitor interval, tolerance and iteration cap
CONV_EVERY, CONV_TOL_DNU, CONV_CAP = 1000, 1e-8, 400000
FLUSH_BYTES = 256 << 20    # > 126 MB L2
MI, NJ = 701, 301
# algorithmic bytes per p-cell of each phase (each array streamed once)
PHASES = ["u-y sweep", "u-x sweep", "v-y sweep", "v-x sweep", "p'-y sweep", "p'-x sweep", "p/u/v correction",
          "T-y sweep", "T-x sweep", "u residual"]
BYTES_PER_CELL = [48, 56, 48, 64, 48, 64, 72, 40, 48, 48]
SWEEPS = ["u-y", "u-x", "v-y", "v-x", "p'-y", "p'-x", "T-y", "T-x"]
# per outer iteration: 8 sweeps, correction and residual (loop tests ride on
# the kernels that finish their norms; the pressure loop's first pass reads
# p' as zero, so no reset pass)
METRIC = "Mcell-iter/s (SIMPLE outer iteration, p-cells): FP32+FP64-refined vs FP64"


def workload_config(world: int = 1):
    """The `config` object of both arms (identical keys and values)."""
    return {"workload": f"lid_driven_mixed_{MI}x{NJ}_Re100_Ri1_Pr0.71_tanh1.2", "mi": MI, "nj": NJ,
            "p_cells": (MI + 1) * (NJ + 1), "outer_iters_per_step": ITERS, "inner_passes": 1,
            "l2": "flushed (256 MiB write) before every timed step and kernel launch",
            "parallelism": f"replicas{world}"}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def make_case():
    from ixchel2d_b200 import cases
    return cases.lid_driven_mixed(MI, NJ, Re=100.0, Ri=1.0, Pr=0.71, beta=1.2)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    every 10 ms (reads only), or nvidia-smi every 200 ms where NVML cannot be
    used."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.gpu)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except pynvml.NVMLError:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.stop_ev = threading.Event()

            def run():
                while not self.stop_ev.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((sm, smax, {n for n, b in bits.items() if r & b}))
                    except nv.NVMLError:
                        pass
                    self.stop_ev.wait(0.01)

            self.t = threading.Thread(target=run, daemon=True)
            self.nvml = nv
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.stop_ev.set()
            self.t.join(timeout=5)
            sm = [x[0] for x in self.samples]
            smax = [x[1] for x in self.samples]
            reasons = set().union(*[x[2] for x in self.samples]) if self.samples else set()
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 10 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(self.NAMES, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def cpu_oracle_rate(case, budget_s: float = 12.0, chunk: int = 5):
    """Oracle (C++ restatement, OpenMP over grid lines) on all host cores."""
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    o = O.OracleCase(case, conv_u=1e30, conv_p=1e30, conv_t=1e30)
    o.iterations(2)  # warm
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < budget_s:
        o.iterations(chunk)
        n += chunk
    dt = time.perf_counter() - t0
    return case.cells * n / dt / 1e6, n, O.max_threads(), dt


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    case = make_case()  # built without mapping libixb.so (cases.py loads no library for this case)
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    o = O.OracleCase(case, conv_u=1e30, conv_p=1e30, conv_t=1e30)
    # each step is the same workload as the GPU arm's step: ITERS outer iterations of the full case
    o.iterations(2)
    for _ in range(args.warmup):
        o.iterations(ITERS)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.iterations(ITERS)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = case.cells * ITERS * args.steps / tot / 1e6
    loaded = sorted({ln.split()[-1] for ln in Path("/proc/self/maps").read_text().splitlines()
                     if ln.endswith(".so") and ("oracle" in ln or "ixchel2d_b200" in ln)})
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "Mcell-iter/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": workload_config(world),
        "cpu_baseline": {"value": value, "unit": "Mcell-iter/s", "cores": O.max_threads(), "cpu_model": cpu_model(),
                         "kind": "port",
                         "sample": f"{ITERS} outer iterations of the full {MI}x{NJ} case per step, "
                                   f"{args.steps} steps after {args.warmup} warm-up steps"},
        "e2e": {"value": value, "unit": "Mcell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "libraries_mapped": loaded,
        "note": "reference is Fortran+OpenACC (nvfortran-only build); its C++ restatement (oracle/) is timed",
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def time_steps(sim, stream, flush, steps, warmup):
    """Device time (ms, CUDA events on the library's stream) of `steps` steps
    of ITERS outer iterations, L2 flushed before each step; last report."""
    import torch
    for _ in range(warmup):
        sim.iterations(ITERS)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    rep = None
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            ev[k][0].record(stream)
        rep = sim.iterations(ITERS)
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev), rep


def converge(sim, stream, chunk=200, cap=40000, tol=1e-8):
    """Iterate until the mass residual maxbo < tol; device time in ms."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
    it, rep = 0, None
    while it < cap:
        rep = sim.iterations(chunk)
        it += chunk
        if rep["maxbo"] < tol:
            break
    with torch.cuda.stream(stream):
        e1.record(stream)
    torch.cuda.synchronize()
    return it, e0.elapsed_time(e1), rep


def adi_microbench(stream, n=4096, nsys=4096, reps=5):
    """Batched line-solve microbenchmark: nsys independent tridiagonal systems
    of n unknowns, a,c ~ U(-1,0), b = |a|+|c|+U(0.1,1), rhs ~ U(-1,1) (Philox,
    seed 1234), contiguous (x-sweep) and interleaved (y-sweep) layouts, binary64
    and binary32, through ixb_tridiag_f64/_f32: the hybrid solver (Thomas-PCR
    over many threads per system) and, beside it, Thomas per thread
    (IXB_SOLVER_EXACT: one thread walks each system, from shared memory in
    the contiguous layout, straight from global memory with coalesced rows in
    the interleaved one).  Algorithmic bytes: a, b, c, d read and x written
    once (40 B per unknown binary64, 20 B binary32).  Error: max |x - x_ref| /
    max |x_ref| against the sequential binary64 Thomas on the same inputs."""
    import torch
    from ixchel2d_b200 import _ffi as F
    gen = torch.Generator(device="cuda").manual_seed(1234)
    u = lambda lo, hi: torch.rand((nsys, n), generator=gen, device="cuda", dtype=torch.float64) * (hi - lo) + lo
    a, c = u(-1.0, 0.0), u(-1.0, 0.0)
    b = a.abs() + c.abs() + u(0.1, 1.0)
    d = u(-1.0, 1.0)
    peak, peak_kind = peaks()
    out = {"systems": nsys, "unknowns": n, "peak_gbs": peak, "peak_kind": peak_kind}
    sh = stream.cuda_stream
    for layout, lname in ((0, "contiguous"), (1, "strided")):
        lay = (lambda t: t.contiguous()) if layout == 0 else (lambda t: t.t().contiguous())
        A, B, C, D = map(lay, (a, b, c, d))
        ref = torch.empty_like(D)
        with torch.cuda.stream(stream):
            F.check(F.lib.ixb_tridiag_f64(A.data_ptr(), B.data_ptr(), C.data_ptr(), D.data_ptr(), ref.data_ptr(),
                                          n, nsys, layout, F.SOLVER_EXACT, sh), "ixb_tridiag_f64")
        for dt, fn, eb in ((torch.float64, F.lib.ixb_tridiag_f64, 8), (torch.float32, F.lib.ixb_tridiag_f32, 4)):
            Ai, Bi, Ci, Di = (t.to(dt) for t in (A, B, C, D))
            X = torch.empty_like(Di)
            for solver, sname in ((F.SOLVER_HYBRID, ""), (F.SOLVER_EXACT, "_thomas_per_thread")):
                args = (Ai.data_ptr(), Bi.data_ptr(), Ci.data_ptr(), Di.data_ptr(), X.data_ptr(), n, nsys, layout,
                        solver, sh)
                torch.cuda.synchronize()
                with torch.cuda.stream(stream):
                    for _ in range(2):
                        F.check(fn(*args), "ixb_tridiag")
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(reps):  # inputs (5 x n x nsys) exceed L2: no flush needed
                        F.check(fn(*args), "ixb_tridiag")
                    e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                gbs = 5 * eb * n * nsys / (ms / 1e3) / 1e9
                err = float((X.double() - ref).abs().max() / ref.abs().max())
                out[f"{lname}_{'f64' if eb == 8 else 'f32'}{sname}"] = {"ms": ms, "gbs": gbs, "frac": gbs / peak,
                                                                        "max_err_vs_f64_thomas": err}
            del Ai, Bi, Ci, Di, X
        del A, B, C, D, ref
    torch.cuda.empty_cache()
    return out


def batched_bench(stream, n_inst=256, iters=30, n_conv=16, conv_cap=20000):
    """Batched cavities (ixb_batch_*): natural-convection cavities, square
    side uniform in {64..512} and Ra log-uniform in [1e3, 1e6] (Pr 0.71,
    seed 1234).  Throughput: `iters` outer iterations of all n_inst
    instances (every instance kept active), batched in both precision
    forms, against the single-instance binary64 path looped over the first
    16 instances.  Convergence: n_conv smaller cavities (side 64..128, Ra
    1e3..1e5) each iterated to maxbo < 1e-8 (cap conv_cap iterations),
    batched refined vs the single-instance binary64 path one after the
    other; instances per second of each."""
    import torch
    from ixchel2d_b200 import Batch, Simple2D, cases
    from ixchel2d_b200 import _ffi as F
    rng = np.random.default_rng(1234)
    sides = rng.integers(64, 513, n_inst)
    ras = 10.0 ** rng.uniform(3.0, 6.0, n_inst)
    cs = [cases.natural_cavity(int(a), int(a), Ra=float(r), T0=0.5) for a, r in zip(sides, ras)]
    cells = sum(c.cells for c in cs)
    out = {"instances": n_inst, "cells": cells, "iters": iters}

    def timed(fn):  # host wall time of calls that synchronise before returning
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    for name, prec in (("refined", F.PREC_FP32_REFINED), ("fp64", F.PREC_FP64)):
        bt = Batch.from_cases(cs, prec=prec, conv_paso=0.0)
        bt.autotune(reps=2)
        bt.iterate(3)
        dt = timed(lambda: bt.iterate(iters))
        out[f"batched_{name}"] = {"ms_per_iter": dt / iters * 1e3, "mcell_iter_s": cells * iters / dt / 1e6}
        bt.close()
    sims = [Simple2D.from_case(c) for c in cs[:16]]
    for sm in sims:
        sm.iterations(3)
    dt = timed(lambda: [sm.iterations(iters) for sm in sims])
    c16 = sum(c.cells for c in cs[:16])
    out["looped_single_fp64"] = {"instances": 16, "mcell_iter_s": c16 * iters / dt / 1e6,
                                 "ms_per_instance_iter": dt / 16 / iters * 1e3}
    for sm in sims:
        sm.close()
    out["batched_refined_over_looped_fp64"] = (out["batched_refined"]["mcell_iter_s"] /
                                               out["looped_single_fp64"]["mcell_iter_s"])
    # convergence of smaller cavities
    sides = rng.integers(64, 129, n_conv)
    ras = 10.0 ** rng.uniform(3.0, 5.0, n_conv)
    cc = [cases.natural_cavity(int(a), int(a), Ra=float(r), T0=0.5) for a, r in zip(sides, ras)]
    bt = Batch.from_cases(cc, prec=F.PREC_FP32_REFINED, conv_paso=1e-8, conv_resi=1e30)
    bt.autotune(reps=2)
    bt.restart()
    left = [n_conv]
    dt_b = timed(lambda: left.__setitem__(0, bt.iterate(conv_cap)))
    reps = [bt.report(i) for i in range(n_conv)]
    bt.close()
    conv_b = sum(1 for r in reps if r["exit_code"] == 1)

    def single_all():
        n = 0
        for c in cc:
            sm = Simple2D.from_case(c, conv_paso=1e-8, conv_resi=1e30)
            it = 0
            while it < conv_cap:
                r = sm.iterations(500)
                it += 500
                if r["maxbo"] < 1e-8:
                    n += 1
                    break
            sm.close()
        return n
    conv_s = [0]
    dt_s = timed(lambda: conv_s.__setitem__(0, single_all()))
    out["converge_small"] = {
        "instances": n_conv, "criterion": "maxbo < 1e-8", "cap_iters": conv_cap,
        "batched_refined": {"converged": conv_b, "seconds": dt_b, "instances_per_s": conv_b / dt_b,
                            "iters": [r["n_simple"] for r in reps]},
        "looped_single_fp64": {"converged": conv_s[0], "seconds": dt_s, "instances_per_s": conv_s[0] / dt_s},
    }
    return out


def adjoint_bench(n=256, Ra=1e5, nodes=128, K=500, warm=500, fd_nodes=8):
    """Energy-equation adjoint with the flow held fixed: natural-convection
    cavity n x n, Ra, after `warm` SIMPLE iterations; hot-wall profile of
    `nodes` piecewise-linear nodes, value 1 + U(-0.05, 0.05) (seed 1234);
    objective the hot-wall Nusselt number after K passes of the T sweeps.
    Gradient by the adjoint against central differences of the same GPU
    forward on fd_nodes of the nodes, with h = 1e-6 and with h = 1e-2: with
    the flow held fixed the objective is affine in the nodes, so central
    differences are exact for any step and the small step only adds the
    forward's rounding divided by h.  A linearity check compares
    J(theta + d) - J(theta) with the adjoint's g . d.  The same central
    differences on two nodes of the CPU oracle's forward (oracle_fd)."""
    from ixchel2d_b200 import Simple2D, cases
    from ixchel2d_b200.adjoint import HotWallNusselt
    case = cases.natural_cavity(n, n, Ra=Ra, T0=0.5)
    sim = Simple2D.from_case(case)
    sim.iterations(warm)
    state = sim.download()
    J = HotWallNusselt(sim, state, case.yp, nodes, K, 2, n - 2)
    rng = np.random.default_rng(1234)
    theta = 1.0 + rng.uniform(-0.05, 0.05, nodes)
    J.gradient(theta)  # warm
    t0 = time.perf_counter()
    g = J.gradient(theta)
    t_adj = time.perf_counter() - t0
    t0 = time.perf_counter()
    nu = J.value(theta)
    t_fwd = time.perf_counter() - t0
    pick = np.linspace(0, nodes - 1, fd_nodes).astype(int)
    fds = {}
    for h in (1e-6, 1e-2):
        fd = np.zeros(fd_nodes)
        for q, k in enumerate(pick):
            e = np.zeros(nodes)
            e[k] = h
            fd[q] = (J.value(theta + e) - J.value(theta - e)) / (2 * h)
        fds[h] = fd
    d = rng.uniform(-0.01, 0.01, nodes)
    dj = J.value(theta + d) - nu
    sim.close()
    fd = fds[1e-6]

    # central differences of the CPU oracle (the restatement of the reference's CPU path) on two nodes
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)

    def J_oracle(th):
        o = O.OracleCase(case)
        o.set_state(state)
        o.set_bc_values(2, 0, J.P @ th)
        o.energy_passes(K)
        v = o.nusselt_x(2, n - 2)[0]
        o.close()
        return v
    oracle_fd = oracle_central_differences(J_oracle, g, theta, nodes)
    return {"case": f"natural_cavity_{n}x{n}_Ra{Ra:g}", "flow": f"held fixed after {warm} SIMPLE iterations",
            "nodes": nodes, "K": K, "nu_hot_wall": nu,
            "adjoint_s": t_adj, "forward_s": t_fwd, "fd_all_nodes_s_estimate": 2 * nodes * t_fwd,
            "fd_nodes_checked": fd_nodes,
            "max_rel_err_vs_fd": float(np.max(np.abs(g[pick] - fd) / np.maximum(np.abs(fd), 1e-300))),
            "normwise_rel_err_vs_fd": float(np.linalg.norm(g[pick] - fd) / np.linalg.norm(fd)),
            "max_rel_err_vs_fd_h1e-2": float(np.max(np.abs(g[pick] - fds[1e-2]) /
                                                 np.maximum(np.abs(fds[1e-2]), 1e-300))),
            "linearity_rel_err": float(abs(dj - g @ d) / abs(dj)),
            "oracle_fd": oracle_fd}


def oracle_central_differences(J_oracle, g, theta, nodes, picks=2):
    """Central differences of an objective evaluated on the CPU oracle, on
    `picks` nodes at steps 1e-6 and 1e-2, against the adjoint gradient g."""
    pick = [nodes // 4, nodes // 2][:picks]
    out = {"nodes_checked": pick}
    t0 = time.perf_counter()
    for h in (1e-6, 1e-2):
        errs = []
        for k in pick:
            e = np.zeros(nodes)
            e[k] = h
            fd = (J_oracle(theta + e) - J_oracle(theta - e)) / (2 * h)
            errs.append(abs(g[k] - fd) / max(abs(fd), 1e-300))
        out[f"max_rel_err_h{h:g}"] = float(max(errs))
    out["oracle_s"] = time.perf_counter() - t0
    return out


def coupled_adjoint_bench(n=256, Re=100.0, nodes=128, K=500, C=50, fd_nodes=8):
    """Energy adjoint through K outer SIMPLE iterations of an evolving flow
    that does not depend on T, with checkpoints every C iterations:
    lid-driven forced convection n x n (Re, Ri = 0), from zero flow and
    T = 0.5; hot-wall profile of `nodes` piecewise-linear nodes, value
    1 + U(-0.05, 0.05) (seed 1234); objective the hot-wall Nusselt number
    after the K iterations.  The T loop runs up to 5 passes per iteration
    (conv_t = 1e-4, iter_ecuaci_max = 3).  Gradient against central
    differences of the same GPU forward on fd_nodes nodes, h = 1e-6 and
    h = 1e-2 (the objective is affine in the nodes: exact for any step), and
    of the CPU oracle's forward on two nodes (oracle_fd)."""
    from ixchel2d_b200 import Simple2D, cases
    from ixchel2d_b200.adjoint import HotWallNusseltCoupled
    case = cases.lid_driven_forced(n, n, Re=Re, conv_t=1e-4, iter_ecuaci_max=3)
    sim = Simple2D.from_case(case)
    J = HotWallNusseltCoupled(sim, case.state, case.yp, nodes, K, 2, n - 2, ckpt=C)
    rng = np.random.default_rng(1234)
    theta = 1.0 + rng.uniform(-0.05, 0.05, nodes)
    J.gradient(theta)  # warm
    t0 = time.perf_counter()
    g = J.gradient(theta)
    t_adj = time.perf_counter() - t0
    t0 = time.perf_counter()
    nu = J.value(theta)
    t_fwd = time.perf_counter() - t0
    pick = np.linspace(0, nodes - 1, fd_nodes).astype(int)
    fds = {}
    for h in (1e-6, 1e-2):
        fd = np.zeros(fd_nodes)
        for q, k in enumerate(pick):
            e = np.zeros(nodes)
            e[k] = h
            fd[q] = (J.value(theta + e) - J.value(theta - e)) / (2 * h)
        fds[h] = fd
    sim.close()
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))

    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)

    def J_oracle(th):
        o = O.OracleCase(case)
        o.set_bc_values(2, 0, J.P @ th)
        o.iterations(K)
        v = o.nusselt_x(2, n - 2)[0]
        o.close()
        return v
    oracle_fd = oracle_central_differences(J_oracle, g, theta, nodes)
    return {"case": case.name, "flow": "evolving over the K iterations from rest (Ri = Riy = 0)",
            "nodes": nodes, "K": K, "C": C, "nu_hot_wall": nu, "adjoint_s": t_adj, "forward_s": t_fwd,
            "fd_all_nodes_s_estimate": 2 * nodes * t_fwd, "fd_nodes_checked": fd_nodes,
            "max_rel_err_vs_fd": rel(g[pick], fds[1e-6]),
            "normwise_rel_err_vs_fd": float(np.linalg.norm(g[pick] - fds[1e-6]) / np.linalg.norm(fds[1e-6])),
            "max_rel_err_vs_fd_h1e-2": rel(g[pick], fds[1e-2]), "oracle_fd": oracle_fd}


def full_adjoint_bench(n=256, Ra=1e5, nodes=128, K=500, C=50, fd_nodes=6):
    """Adjoint of the full coupled SIMPLE iteration (ixb_adjoint_simple): the
    natural-convection cavity n x n at Ra (buoyancy couples the flow to the
    wall temperature), from rest and T = 0.5; hot-wall profile of `nodes`
    piecewise-linear nodes, value 1 + U(-0.05, 0.05) (seed 1234); objective
    the hot-wall Nusselt number after K outer iterations (one pass of each
    equation), checkpoints every C.  The objective is nonlinear in the
    nodes: central differences of the GPU forward on fd_nodes nodes at
    h = 1e-6 (the configured step) and h = 1e-4, and of the CPU oracle on two
    nodes (oracle_fd)."""
    from ixchel2d_b200 import Simple2D, cases
    from ixchel2d_b200.adjoint import profile_matrix
    case = cases.natural_cavity(n, n, Ra=Ra, T0=0.5)
    P = profile_matrix(case.yp, nodes)
    rng = np.random.default_rng(1234)
    theta = 1.0 + rng.uniform(-0.05, 0.05, nodes)
    sim = Simple2D.from_case(case)

    def run(th, gradient):
        sim.upload(case.state)
        sim.set_bc_values(2, 0, P @ th)
        return sim.adjoint_simple(K, C, 2, n - 2, gradient=gradient)
    run(theta, True)  # warm
    t0 = time.perf_counter()
    g_lines, nu = run(theta, True)
    t_adj = time.perf_counter() - t0
    g = P.T @ g_lines
    t0 = time.perf_counter()
    run(theta, False)
    t_fwd = time.perf_counter() - t0
    pick = np.linspace(nodes // 16, nodes - 1 - nodes // 16, fd_nodes).astype(int)  # away from the corners
    errs, norm_errs = {}, {}
    for h in (1e-6, 1e-4):
        fd = np.zeros(len(pick))
        for q, k in enumerate(pick):
            e = np.zeros(nodes)
            e[k] = h
            fd[q] = (run(theta + e, False)[1] - run(theta - e, False)[1]) / (2 * h)
        errs[h] = float(np.max(np.abs(g[pick] - fd) / np.maximum(np.abs(fd), 1e-300)))
        norm_errs[h] = float(np.linalg.norm(g[pick] - fd) / np.linalg.norm(fd))
    sim.close()

    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)

    def J_oracle(th):
        o = O.OracleCase(case)
        o.set_bc_values(2, 0, P @ th)
        o.iterations(K)
        v = o.nusselt_x(2, n - 2)[0]
        o.close()
        return v
    oracle_fd = oracle_central_differences(J_oracle, g, theta, nodes)
    return {"case": f"natural_cavity_{n}x{n}_Ra{Ra:g}",
            "flow": "buoyant, evolving over the K iterations from rest (momentum, pressure correction and "
                    "energy all reversed)",
            "nodes": nodes, "K": K, "C": C, "nu_hot_wall": nu, "adjoint_s": t_adj, "forward_s": t_fwd,
            "fd_all_nodes_s_estimate": 2 * nodes * t_fwd, "fd_nodes_checked": int(len(pick)),
            "max_rel_err_vs_fd_h1e-6": errs[1e-6], "normwise_rel_err_vs_fd_h1e-6": norm_errs[1e-6],
            "max_rel_err_vs_fd_h1e-4": errs[1e-4], "normwise_rel_err_vs_fd_h1e-4": norm_errs[1e-4],
            "oracle_fd": oracle_fd}


def make_sim(case, prec, stream, shapes):
    from ixchel2d_b200 import Simple2D
    sim = Simple2D.from_case(case, prec=prec)
    sim.set_stream(stream.cuda_stream)
    if shapes is None:
        # launch shapes of the eight sweeps picked by the library's autotuner (cold L2)
        shapes = {k: tuple(v) for k, v in sim.autotune(reps=5, flush_bytes=FLUSH_BYTES).items()}
    else:
        for k, (tl, g, *_) in shapes.items():
            sim.set_sweep_shape(int(k), tl, g)
    return sim, shapes


def run_ours(args):
    import torch
    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    from ixchel2d_b200 import Simple2D, cases, lib
    from ixchel2d_b200 import _ffi as F
    if lib.ixb_device_count() < 1:
        raise RuntimeError("no CUDA device visible")
    case = make_case()
    stream = torch.cuda.Stream()
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    loaded = json.loads(Path(args.shapes).read_text()) if args.shapes else {}
    modes = {"refined": F.PREC_FP32_REFINED, "fp64": F.PREC_FP64}

    sims, shapes = {}, {}
    for name, prec in modes.items():
        sims[name], shapes[name] = make_sim(case, prec, stream, loaded.get(name))
    # kernels per outer iteration with the chosen shapes (fused sweeps launch one kernel, others two)
    per_iter = {name: sims[name].iteration_launches() for name in modes}
    if args.save_shapes and rank == 0:
        Path(args.save_shapes).write_text(json.dumps({n: {str(k): list(v) for k, v in sh.items()}
                                                      for n, sh in shapes.items()}))

    # ---- device-resident timed regions: the refined path (headline), then binary64 ----
    sampler = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    t_wall = time.perf_counter()
    ms, reports = {}, {}
    for name in modes:
        ms[name], reports[name] = time_steps(sims[name], stream, flush, args.steps, args.warmup)
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    if pg:
        t = torch.tensor([ms["refined"], ms["fp64"]], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = {"refined": float(t[0].item()), "fp64": float(t[1].item())}
        pg.barrier()
    torch.cuda.synchronize()
    cells_iters = case.cells * ITERS * args.steps * world
    rate = {n: cells_iters / (ms[n] / 1e3) / 1e6 for n in modes}
    # the two forms after the same iterations from the same start (not converged at this size)
    nu_big = {n: sims[n].nusselt_y(2, MI - 2) for n in modes}

    # ---- end to end through the C ABI with host buffers (refined path) ----
    sim = sims["refined"]
    keys = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
    st0 = sim.download()
    host = {}
    for kk in keys:
        t = torch.empty(st0[kk].shape[::-1], dtype=torch.float64, pin_memory=True)
        a = t.numpy().T  # Fortran-ordered view of pinned memory
        a[...] = st0[kk]
        host[kk] = a
    h2d = sum(a.nbytes for a in host.values())
    e2e_ms = 0.0
    for k in range(args.warmup + args.steps):  # the first `warmup` steps are not timed
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        sim.upload(host)
        sim.iterations(ITERS)
        sim.download(out=host)  # straight into the pinned buffers the next step uploads
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_ms += e0.elapsed_time(e1)
    if pg:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = cells_iters / (e2e_ms / 1e3) / 1e6

    # ---- converged answer at the benchmark size: both forms from rest until the bottom-wall Nusselt
    #      number (the heated wall) changes by less than 1e-8 over 1000 outer iterations, monitored on
    #      the device (ixb_simple_converge), in the autotuned shapes of the timed region ----
    big = {}
    for name in modes:
        s_ = sims[name]
        s_.upload(case.state)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            e0.record(stream)
        r = s_.converge(2, MI - 2, vertical=False, wall=0, every=CONV_EVERY, tol_dnu=CONV_TOL_DNU,
                        max_iters=CONV_CAP)
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        big[name] = {"iters": r["n_simple"], "device_s": sec, "mcell_iter_s": case.cells * r["n_simple"] / sec / 1e6,
                     "nu_bottom_wall": r["nu"][0], "nu_top_wall": r["nu"][1],
                     "dnu_last_interval": r["dnu"], "maxbo": r["maxbo"], "residuo": r["residuo"],
                     "exit": {3: "dNu", 4: "maxbo", 5: "cap"}.get(r["exit_code"], str(r["exit_code"]))}
        big[name]["_state"] = s_.download()
    fields_l2 = {k: float(np.linalg.norm(big["refined"]["_state"][k] - big["fp64"]["_state"][k]) /
                          np.linalg.norm(big["fp64"]["_state"][k])) for k in ("u", "v", "p", "T")}
    for name in modes:
        del big[name]["_state"]
    converged_big = {"case": workload_config()["workload"],
                     "criterion": f"|dNu| of the bottom (heated) wall < {CONV_TOL_DNU:g} over {CONV_EVERY} outer "
                                  f"iterations, cap {CONV_CAP}; monitored on the device",
                     **big,
                     "dnu_refined_vs_fp64": abs(big["refined"]["nu_bottom_wall"] - big["fp64"]["nu_bottom_wall"]),
                     "fields_rel_l2_refined_vs_fp64": fields_l2,
                     "wall_speedup": big["fp64"]["device_s"] / big["refined"]["device_s"]}

    # ---- converged answer: the plain 64x64 configuration to maxbo < 1e-8, both forms ----
    small = cases.natural_cavity(64, 64, Ra=1e4, T0=0.5)
    conv = {}
    for name, prec in modes.items():
        s2 = Simple2D.from_case(small, prec=prec)
        s2.set_stream(stream.cuda_stream)
        s2.iterations(10)
        s2.upload(small.state)
        it, cms, rep = converge(s2, stream)
        conv[name] = {"iters": it, "ms": cms, "maxbo": rep["maxbo"], "nu_hot_wall": s2.nusselt_x(2, 62)[0]}
        s2.close()

    # ---- per-phase times of the refined path on a scratch handle: warm (the state of the timed
    #      region, whose 45 MB working set stays in L2 between the per-step flushes) and cold ----
    scratch, _ = make_sim(case, F.PREC_FP32_REFINED, stream, shapes["refined"])
    scratch.iterations(3)
    phase_ms_warm = scratch.time_phases(reps=20, flush_bytes=0)
    phase_ms = scratch.time_phases(reps=10, flush_bytes=FLUSH_BYTES)
    scratch.close()
    # ---- batched line-solve microbenchmark (4096 systems x 4096 unknowns) ----
    adi = adi_microbench(stream)
    # ---- batched cavities ----
    batched = batched_bench(stream)
    # ---- energy adjoint (flow held fixed) ----
    adjoint = adjoint_bench()
    adjoint_coupled = coupled_adjoint_bench()
    adjoint_full = full_adjoint_bench()

    cells = case.cells
    dom = int(np.argmax(phase_ms_warm))  # the phase with the largest share of the timed step
    peak, peak_kind = peaks()
    alg_bytes = BYTES_PER_CELL[dom] * cells
    achieved = alg_bytes / (phase_ms_warm[dom] / 1e3) / 1e9
    achieved_cold = alg_bytes / (phase_ms[dom] / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(PHASES[dom])

    if rank == 0:
        cpu_val, cpu_iters, cpu_cores, cpu_s = cpu_oracle_rate(case) if world == 1 else (None, 0, 0, 0)
        iter_bytes = sum(BYTES_PER_CELL) * cells
        line = {
            "metric": METRIC, "value": rate["refined"], "unit": "Mcell-iter/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["refined"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": workload_config(world),
            "fp64": {"value": rate["fp64"], "unit": "Mcell-iter/s", "ms_per_step": ms["fp64"] / args.steps,
                     "dtype": "f64"},
            "refined_over_fp64": rate["refined"] / rate["fp64"],
            "dnu_bottom_wall_after_timed_iters": abs(nu_big["refined"][0] - nu_big["fp64"][0]),
            "converged_701x301": converged_big,
            "converged": {"case": "natural_cavity_64x64_Ra1e4_Pr0.71", "criterion": "maxbo < 1e-8", **conv,
                          "dnu": abs(conv["refined"]["nu_hot_wall"] - conv["fp64"]["nu_hot_wall"]),
                          "wall_speedup": conv["fp64"]["ms"] / conv["refined"]["ms"]},
            "e2e": {"value": e2e_value, "unit": "Mcell-iter/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": h2d,
                    "note": "refined path; per step: 7 state arrays host->device, ITERS outer iterations, "
                            "7 arrays device->host"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": PHASES[dom],
                         "peak_kind": f"{peak_kind} (copy bandwidth)",
                         "alg_bytes_per_launch": alg_bytes, "launch_ms": phase_ms_warm[dom],
                         "timing": "warm L2, as in the timed region (CUDA events around each of 20 launches "
                                   "on the library's stream); traffic: cold DRAM bytes of one ncu capture",
                         "cold_l2": {"launch_ms": phase_ms[dom], "achieved": achieved_cold,
                                     "frac": achieved_cold / peak}},
            "phases_ms_warm_l2": dict(zip(PHASES, phase_ms_warm)),
            "phases_ms_cold_l2": dict(zip(PHASES, phase_ms)),
            "adi_line_solve": adi,
            "batched_cavities": batched,
            "energy_adjoint": adjoint,
            "energy_adjoint_coupled": adjoint_coupled,
            "simple_adjoint_buoyant": adjoint_full,
            "sweep_shapes": {n: {SWEEPS[int(k)]: list(v[:2]) for k, v in sh.items()} for n, sh in shapes.items()},
            "iteration_alg_bytes": iter_bytes,
            "cpu_baseline": None if cpu_val is None else {
                "value": cpu_val, "unit": "Mcell-iter/s", "cores": cpu_cores, "cpu_model": cpu_model(), "kind": "port",
                "sample": f"{cpu_iters} outer iterations of the same 701x301 case ({cpu_s:.1f} s)"},
            "gpu_launches": sum((per_iter[n] * ITERS + 1) * args.steps for n in modes),
            "kernels_per_outer_iteration": per_iter,
            "clocks": clocks,
            "last_report": {k: reports["refined"][k] for k in ("maxbo", "residuo", "n_simple", "n_momen")},
            "wall_s_timed_region": wall,
        }
        print(json.dumps(line), flush=True)
    for s_ in sims.values():
        s_.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_profile_phases(prec, shapes_file=None):
    """Profiling driver (no timing, no JSON): the benchmark case, three outer
    iterations, then one launch of each of the ten phases in order
    (u-y, u-x, v-y, v-x, p'-y, p'-x, correction, T-y, T-x, residual), in the
    launch shapes of `shapes_file` (from --save-shapes) when given."""
    from ixchel2d_b200 import Simple2D
    sim = Simple2D.from_case(make_case(), prec=prec)
    if shapes_file:
        name = "refined" if prec == 1 else "fp64"
        for k, (tl, g, *_) in json.loads(Path(shapes_file).read_text())[name].items():
            sim.set_sweep_shape(int(k), tl, g)
    sim.iterations(3)
    for k in range(10):
        sim.phase(k)
    sim.close()


def run_profile_adi():
    """Profiling driver: one launch of each batched line solve of the
    microbenchmark (contiguous f64, contiguous f32, interleaved f64,
    interleaved f32; 4096 systems x 4096 unknowns)."""
    import torch
    from ixchel2d_b200 import _ffi as F
    n = nsys = 4096
    gen = torch.Generator(device="cuda").manual_seed(1234)
    for layout in (0, 1):
        for dt, fn in ((torch.float64, F.lib.ixb_tridiag_f64), (torch.float32, F.lib.ixb_tridiag_f32)):
            a = -torch.rand((nsys, n), generator=gen, device="cuda", dtype=dt)
            c = -torch.rand((nsys, n), generator=gen, device="cuda", dtype=dt)
            b = a.abs() + c.abs() + 0.1 + 0.9 * torch.rand((nsys, n), generator=gen, device="cuda", dtype=dt)
            d = 2 * torch.rand((nsys, n), generator=gen, device="cuda", dtype=dt) - 1
            x = torch.empty_like(d)
            F.check(fn(a.data_ptr(), b.data_ptr(), c.data_ptr(), d.data_ptr(), x.data_ptr(), n, nsys, layout,
                       F.SOLVER_HYBRID, torch.cuda.current_stream().cuda_stream), "ixb_tridiag")
            torch.cuda.synchronize()
            del a, b, c, d, x


def run_profile_batch():
    """Profiling driver: 64 natural-convection cavities (side 64..512, Ra
    1e3..1e6, seed 1234), refined form, two batched outer iterations (run
    with IXB_NO_GRAPH=1 so that ncu sees the kernels).  Shapes: y-sweeps
    2 x 64 (two kernels), x-sweeps 1 x 128 (fused), the batch autotuner's
    usual choices for the x-sweeps."""
    from ixchel2d_b200 import Batch, cases
    rng = np.random.default_rng(1234)
    sides = rng.integers(64, 513, 64)
    ras = 10.0 ** rng.uniform(3.0, 6.0, 64)
    bt = Batch.from_cases([cases.natural_cavity(int(a), int(a), Ra=float(r), T0=0.5) for a, r in zip(sides, ras)],
                          conv_paso=0.0)
    for k in range(8):
        bt.set_sweep_shape(k, 1 if k % 2 else 2, 128 if k % 2 else 64)
    bt.iterate(2)
    bt.close()


def run_batch_converge(cap):
    """Batched configuration at full size, run to convergence: the 256
    natural-convection cavities of batched_bench (side uniform in 64..512, Ra
    log-uniform in [1e3, 1e6], Pr 0.71, seed 1234) in the refined form, each
    iterated until maxbo < 1e-8 or `cap` outer iterations, in one batched
    loop.  Prints one JSON line: instances converged, device wall seconds,
    converged instances per second, and the iterations each instance took."""
    import torch
    from ixchel2d_b200 import Batch, cases
    from ixchel2d_b200 import _ffi as F
    rng = np.random.default_rng(1234)
    n_inst = 256
    sides = rng.integers(64, 513, n_inst)
    ras = 10.0 ** rng.uniform(3.0, 6.0, n_inst)
    cs = [cases.natural_cavity(int(a), int(a), Ra=float(r), T0=0.5) for a, r in zip(sides, ras)]
    bt = Batch.from_cases(cs, prec=F.PREC_FP32_REFINED, conv_paso=1e-8, conv_resi=1e30)
    bt.autotune(reps=2)
    bt.restart()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bt.iterate(cap)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    reps = [bt.report(i) for i in range(n_inst)]
    bt.close()
    conv = [i for i, r in enumerate(reps) if r["exit_code"] == 1]
    print(json.dumps({"batched_converge": {
        "instances": n_inst, "criterion": "maxbo < 1e-8", "cap_iters": cap, "form": "refined",
        "converged": len(conv), "seconds": dt, "converged_per_s": len(conv) / dt,
        "iters": [int(r["n_simple"]) for r in reps], "sides": [int(a) for a in sides],
        "ra": [float(r) for r in ras]}}))


def run_profile_adjoint():
    """Profiling driver: the energy adjoint on the 256 x 256 cavity (Ra 1e5)
    after 50 SIMPLE iterations, 128 hot-wall nodes, K = 2 passes (one launch
    of each adjoint kernel per sweep)."""
    from ixchel2d_b200 import Simple2D, cases
    from ixchel2d_b200.adjoint import HotWallNusselt
    case = cases.natural_cavity(256, 256, Ra=1e5, T0=0.5)
    sim = Simple2D.from_case(case)
    sim.iterations(50)
    J = HotWallNusselt(sim, sim.download(), case.yp, 128, 2, 2, 254)
    J.gradient(np.ones(128))
    sim.close()


def run_profile_simple_adjoint():
    """Profiling driver: the full coupled adjoint on the 256 x 256 natural-
    convection cavity (Ra 1e5) from rest, K = 2 outer iterations in one
    checkpoint segment (each reverse kernel launched once per sweep and
    iteration)."""
    from ixchel2d_b200 import Simple2D, cases
    case = cases.natural_cavity(256, 256, Ra=1e5, T0=0.5)
    sim = Simple2D.from_case(case)
    sim.adjoint_simple(2, 2, 2, 254)
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile-phases", action="store_true",
                    help="run the profiling driver instead of the benchmark")
    ap.add_argument("--prec", type=int, default=1, help="precision mode of --profile-phases (0 fp64, 1 refined)")
    ap.add_argument("--shapes", help="JSON of sweep launch shapes (from --save-shapes) instead of autotuning")
    ap.add_argument("--save-shapes", help="write the autotuned sweep launch shapes to this JSON file")
    ap.add_argument("--profile-adi", action="store_true", help="run the line-solve profiling driver")
    ap.add_argument("--profile-batch", action="store_true", help="run the batched-cavities profiling driver")
    ap.add_argument("--profile-adjoint", action="store_true", help="run the energy-adjoint profiling driver")
    ap.add_argument("--batch-converge", type=int, default=0, metavar="CAP",
                    help="run the 256 batched cavities to maxbo < 1e-8 (at most CAP outer iterations) and exit")
    ap.add_argument("--profile-simple-adjoint", action="store_true",
                    help="run the profiling driver of the full coupled adjoint")
    args = ap.parse_args()
    if args.profile_phases:
        run_profile_phases(args.prec, args.shapes)
        return
    if args.profile_adi:
        run_profile_adi()
        return
    if args.batch_converge:
        run_batch_converge(args.batch_converge)
        return
    if args.profile_batch:
        run_profile_batch()
        return
    if args.profile_simple_adjoint:
        run_profile_simple_adjoint()
        return
    if args.profile_adjoint:
        run_profile_adjoint()
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
