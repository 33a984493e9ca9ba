#!/usr/bin/env python
"""DGSEM RHS benchmark: FP64 DOF-updates/s per RHS on one B200 (or N replicas).

Workload (default): 3D Euler Taylor-Green vortex,
periodic 16^3 elements on [0, 2pi]^3, N = 3 (4^3 LGL nodes), Mach 0.1,
Kennedy-Gruber split-form volume flux, LLF surface flux, SSPRK3 with the
reference TGV time step rule.  A "step" is one SSPRK3 step = 3 fused stage
kernels = 3 RHS evaluations; DOF-updates/s = elements * n^3 * 3 / step time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dgsem_b200|reference]
                  [--workload tgv16|tgv32|tgv64|kh64|kh1024|dmr|batched|adjoint]

Without --steps, each workload times a number of steps that stays inside
the physical run it models (DEFAULT_STEPS): the Kelvin-Helmholtz roll-up of
the unlimited split-form scheme ends in a non-finite state after a few time
units, so kh64 does not run the 20000 steps of the Taylor-Green vortex.

The device arm times every step with CUDA events on the solver's stream and
flushes L2 (a 256 MiB write) before every step outside the timed events.
`e2e` repeats the step through the host-buffer C-ABI entry point
(dgsem_ssprk3_steps_host: pinned host state -> device, step, -> host).
`roofline` uses the fused stage kernel's per-launch event times and its
algorithmic bytes (state reads + writes, 8*NVARS*8/3 B per DOF per stage).
`--impl reference` times the reference solver's own CPU code (compiled with
the project's Kokkos shim and OpenMP, oracle/_ref) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (ndims, polydeg, cells, left, right, volume flux, surface flux, ic, vi, bcs)
    "tgv16": (3, 3, (16, 16, 16), (0.0,) * 3, (2 * math.pi,) * 3, "kennedy_gruber", "llf",
              "tgv3d", "split", "periodic"),
    "tgv32": (3, 3, (32, 32, 32), (0.0,) * 3, (2 * math.pi,) * 3, "kennedy_gruber", "llf",
              "tgv3d", "split", "periodic"),
    "tgv64": (3, 3, (64, 64, 64), (0.0,) * 3, (2 * math.pi,) * 3, "kennedy_gruber", "llf",
              "tgv3d", "split", "periodic"),
    "kh64": (2, 3, (64, 64), (-1.0, -1.0), (1.0, 1.0), "ranocha", "llf", "kh", "split",
             "periodic"),
    "kh1024": (2, 3, (1024, 1024), (-1.0, -1.0), (1.0, 1.0), "ranocha", "llf", "kh", "split",
               "periodic"),
    "dmr": (2, 3, (240, 60), (0.0, 0.0), (4.0, 1.0), "chandrashekar", "hllc", "dmr", "hg",
            "dmr"),
}
# timed steps when --steps is not given (simulated time reached in brackets)
DEFAULT_STEPS = {
    "tgv16": 20000,   # t ~ 19
    "tgv32": 2000,    # t ~ 0.9
    "tgv64": 300,     # t ~ 0.07
    "kh64": 500,      # t ~ 0.6 (before the roll-up)
    "kh1024": 200,    # t ~ 0.015
    "dmr": 1000,      # t ~ 0.08 (the reference runs to 0.2)
    "batched": 200,
    "adjoint": 5,
}
VF_CODE = {"chandrashekar": 0, "ranocha": 1, "kennedy_gruber": 2}
SF_CODE = {"llf": 0, "hllc": 1}


def time_step_size(name: str) -> float:
    nd, N, cells, left, right = WORKLOADS[name][:5]
    if name.startswith("tgv"):
        # examples/Euler3D/inviscid_tgv/inviscid_tgv.cpp:111-117 with order 3
        dx = min((right[a] - left[a]) / cells[a] for a in range(3))
        return 0.1 * dx / 2.0 / (3.0 * (2 * 3 + 1))
    if name == "dmr":
        # CFL 0.4, lambda_max = 12 (double_mach_reflection_structured.cpp:141-148)
        return 0.4 * min(4.0 / cells[0], 1.0 / cells[1]) / ((2.0 * (N + 1) - 1.0) * 12.0)
    # KH: CFL 0.5 with lambda_max from the initial state (|v| + c <= 1.84)
    dx = min((right[a] - left[a]) / cells[a] for a in range(nd))
    return 0.5 * dx / ((2.0 * (N + 1) - 1.0) * 1.84)


def bytes_per_dof_stage(nvars: int) -> float:
    # stage 1 reads 1 state and writes 1; stages 2, 3 read 2 and write 1
    return 8.0 * nvars * 8.0 / 3.0


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# stage kernel launched by each launch shape (dgsem_autotune / --variant)
VARIANT_KERNELS = {
    0: "stage_kernel", 1: "stage_kernel", 2: "stage_kernel",
    3: "stage_node_kernel", 4: "stage_node_kernel", 5: "stage_pipe_kernel",
    6: "stage_node2_kernel",
}
KERNEL_DESCRIPTIONS = {
    "stage_kernel": "stage_kernel (line-parallel fused RHS + SSPRK3 stage)",
    "stage_node_kernel": "stage_node_kernel (node-parallel fused RHS + SSPRK3 stage)",
    "stage_pipe_kernel": "stage_pipe_kernel (persistent node-parallel, TMA tile streaming)",
    "stage_node2_kernel": "stage_node2_kernel (node-parallel, two nodes per thread)",
}


def profile_value(workload: str, kernel: str, key: str):
    """A figure of the stage kernel's committed ncu summary (profiles/), e.g.
    traffic_bytes_per_launch (DRAM read + write bytes of one launch) or
    fp64_flops_per_dof (FP64 add + mul + 2 x fma thread operations per DOF
    and stage)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return float(line.split(":", 1)[1].strip())
    except (OSError, ValueError):
        pass
    return None


def profile_traffic(workload: str, kernel: str = "stage_kernel"):
    return profile_value(workload, kernel, "traffic_bytes_per_launch")


def fp64_peak(stream) -> dict:
    """FP64 FMA throughput of this GPU measured live (dgsem_fp64_fma_peak:
    CUDA-event-timed independent FMA chains on every SM, 2 FLOP per FMA)."""
    import ctypes

    from dgsem_b200 import _capi as C
    fl, ms = ctypes.c_double(), ctypes.c_double()
    C.check(C.lib().dgsem_fp64_fma_peak(ctypes.c_void_p(stream.cuda_stream), 4000,
                                        ctypes.byref(fl), ctypes.byref(ms)), "fp64 peak")
    return {"tflops": fl.value / 1e12, "ms": ms.value}


class ClockSampler:
    """SM clock, power and clock-event reasons sampled through NVML (read
    only) every ~1 ms on a background thread while the timed region runs, so
    that even a timed region of a few milliseconds gets samples; nvidia-smi
    -lms 200 is the fallback when NVML cannot be loaded."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40,
               "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, period_s: float = 0.001):
        self.dev = device_index
        self.period = period_s
        self.samples = []
        self.smax = None
        self._thread = None
        self._stop = None
        self._nvml = None
        self.proc = None

    def _poll(self, h):
        import time as _t
        nv = self._nvml
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((sm, mask))
            except Exception:
                pass
            _t.sleep(self.period)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.dev)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._nvml = nv
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._poll, args=(h,), daemon=True)
            self._thread.start()
            return
        except Exception:
            self._nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self._nvml is not None:
            self._stop.set()
            self._thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = {nm for nm, bit in self.REASONS.items()
                       for _, mask in self.samples if mask & bit}
            return {"sm_mhz": statistics.median(float(sm) for sm, _ in self.samples),
                    "sm_max_mhz": self.smax, "reasons": sorted(reasons),
                    "samples": len(self.samples), "source": "NVML, ~1 ms polling"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi -lms 200"}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# reference arm / CPU baseline
# ---------------------------------------------------------------------------
# One CPU sample policy for the reference arm and the device arm's
# cpu_baseline leg: W untimed warm-up steps, then max(K, enough steps for
# CPU_MIN_SAMPLE_S) timed steps, capped at CPU_MAX_SAMPLE_S of CPU time.
CPU_MIN_SAMPLE_S = 5.0
CPU_MAX_SAMPLE_S = 30.0


def reference_case(workload: str):
    """The reference solver (oracle/_ref) and the initial state of a workload."""
    from oracle import dgsem_oracle as do
    from oracle import ref_binding as rb
    nd, N, cells, left, right, vf, sf, ic, vi, bcs = WORKLOADS[workload]
    if nd == 3:
        kind = rb.EULER3D_PERIODIC_SPLIT
    elif bcs == "dmr":
        kind = rb.EULER2D_DMR_HG
    else:
        kind = rb.EULER2D_PERIODIC_SPLIT
    rc = rb.RefCase(kind, N, cells, left, right, volume_flux=VF_CODE[vf],
                    surface_flux=SF_CODE[sf])
    s = do.Scheme(ndims=nd, polydeg=N, cells=cells, left=left, right=right,
                  periodic=(bcs == "periodic"), bc=bcs if bcs == "dmr" else "periodic")
    return rc, do.initial_state(s, ic)


def reference_rate(workload: str, warmup: int, steps: int):
    """Times the reference solver's CPU code (oracle/_ref) on the workload:
    (DOF-updates/s, timed steps, seconds, threads, warm-up steps)."""
    from oracle import ref_binding as rb
    nd, N, cells = WORKLOADS[workload][:3]
    rc, u = reference_case(workload)
    dt = time_step_size(workload)
    t0 = time.perf_counter()
    u = rc.ssprk3(u, 0.0, dt, 1)
    one = time.perf_counter() - t0
    nwarm = max(1, min(warmup, int(0.5 * CPU_MAX_SAMPLE_S / max(one, 1e-6))))
    if nwarm > 1:
        u = rc.ssprk3(u, dt, dt, nwarm - 1)
    t0 = time.perf_counter()
    u = rc.ssprk3(u, nwarm * dt, dt, 1)
    one = time.perf_counter() - t0
    n = max(steps, math.ceil(CPU_MIN_SAMPLE_S / max(one, 1e-6)))
    n = max(1, min(n, int(CPU_MAX_SAMPLE_S / max(one, 1e-6))))
    t = (nwarm + 1) * dt
    t0 = time.perf_counter()
    u = rc.ssprk3(u, t, dt, n)
    el = time.perf_counter() - t0
    # top up to the minimum sample when the first estimate was pessimistic
    while el < CPU_MIN_SAMPLE_S and el < CPU_MAX_SAMPLE_S:
        more = max(1, math.ceil((CPU_MIN_SAMPLE_S - el) / (el / n)))
        t1 = time.perf_counter()
        u = rc.ssprk3(u, t + n * dt, dt, more)
        el += time.perf_counter() - t1
        n += more
    dofs = math.prod(cells) * (N + 1) ** nd
    threads = rb.lib().dgsem_ref_omp_threads()
    return dofs * 3 * n / el, n, el, threads, nwarm


def reference_rate_batched(warmup: int, steps: int):
    """The reference's own path for the batched workload: one solver per mesh,
    advanced mesh after mesh (the reference has no batched mode), on a bounded
    sample of the 256 meshes (every 16th, 16 meshes over all degrees), each
    with its own vortex and time step.  Returns (DOF-updates/s, sampled
    meshes, timed steps per mesh, seconds, threads)."""
    from oracle import dgsem_oracle as do
    from oracle import ref_binding as rb
    specs = batched_meshes()[::16]
    left, right = (-5.0, -5.0), (5.0, 5.0)
    cases = []
    for cells, N, beta, centre in specs:
        rc = rb.RefCase(rb.EULER2D_PERIODIC_SPLIT, N, cells, left, right,
                        volume_flux=VF_CODE["chandrashekar"], surface_flux=SF_CODE["llf"])
        s = do.Scheme(ndims=2, polydeg=N, cells=cells, left=left, right=right)
        u = do.initial_state(s, "vortex", beta=beta, center=centre)
        dt = 0.5 * (10.0 / cells[0]) / ((2.0 * (N + 1) - 1.0) * 4.0)
        cases.append([rc, u, dt, cells[0] * cells[1] * (N + 1) ** 2])
    for c in cases:  # warm-up
        c[1] = c[0].ssprk3(c[1], 0.0, c[2], max(1, min(warmup, 2)))
    # steps per mesh so that the sample takes CPU_MIN_SAMPLE_S .. CPU_MAX_SAMPLE_S
    t0 = time.perf_counter()
    for c in cases:
        c[1] = c[0].ssprk3(c[1], 0.0, c[2], 1)
    one = time.perf_counter() - t0
    n = max(steps, math.ceil(CPU_MIN_SAMPLE_S / max(one, 1e-6)))
    n = max(1, min(n, int(CPU_MAX_SAMPLE_S / max(one, 1e-6))))
    t0 = time.perf_counter()
    for c in cases:
        c[1] = c[0].ssprk3(c[1], 0.0, c[2], n)
    el = time.perf_counter() - t0
    dofs = sum(c[3] for c in cases)
    return dofs * 3 * n / el, len(cases), n, el, rb.lib().dgsem_ref_omp_threads()


def cpu_sample_text(workload: str, n: int, el: float, nwarm: int) -> str:
    return (f"{nwarm} warm-up + {n} timed SSPRK3 steps of the full {workload} mesh "
            f"({el:.1f} s; at least {CPU_MIN_SAMPLE_S:.0f} s, at most {CPU_MAX_SAMPLE_S:.0f} s "
            f"of timed CPU work); reference src/ compiled with the project's Kokkos shim, "
            f"OpenMP on all host threads; CPU: {cpu_model()}")


def run_reference_batched(args):
    """Reference arm of the batched workload (reference_rate_batched)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    try:
        rate, nmesh, n, el, threads = reference_rate_batched(args.warmup, args.steps)
    except Exception as exc:  # reference library missing on this machine
        print(json.dumps({"impl": "reference", "unavailable": f"{type(exc).__name__}: {exc}"}))
        return 0
    sample = (f"{nmesh} of the 256 meshes (every 16th, degrees 2-7), one reference solver "
              f"each, {n} timed SSPRK3 steps per mesh after warm-up ({el:.1f} s); the "
              f"reference has no batched mode, so its path is mesh after mesh; reference "
              f"src/ compiled with the project's Kokkos shim, OpenMP on all host threads; "
              f"CPU: {cpu_model()}")
    line = {
        "metric": "FP64 DOF-updates/s per RHS (batched)", "value": rate,
        "unit": "DOF-updates/s", "impl": "reference", "n_gpus": args.gpus, "steps": n,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded isentropic vortices)",
        "config": batched_config(),
        "cpu_baseline": {"value": rate, "unit": "DOF-updates/s", "cores": threads,
                         "kind": "reference", "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": rate, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        rate, n, el, threads, nwarm = reference_rate(args.workload, args.warmup, args.steps)
    except Exception as exc:  # reference library missing on this machine
        print(json.dumps({"impl": "reference", "unavailable": f"{type(exc).__name__}: {exc}"}))
        return 0
    line = {
        "metric": "FP64 DOF-updates/s per RHS", "value": rate, "unit": "DOF-updates/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": n, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload),
        "cpu_baseline": {"value": rate, "unit": "DOF-updates/s", "cores": threads,
                         "kind": "reference", "cpu_model": cpu_model(),
                         "sample": cpu_sample_text(args.workload, n, el, nwarm)},
        "e2e": {"value": rate, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def dmr_flag_check(solver, u, t, dt, dev, nsteps: int = 20):
    """Troubled-cell flags of the GPU indicator against the reference's
    HGIndicator (oracle/_ref, CPU) on the GPU's own stage inputs, over
    `nsteps` further SSPRK3 steps of the double Mach reflection: per-stage
    flagged counts, mismatches (must be 0) and the smallest distance of the
    unclipped logistic alpha to the alpha_min decision (indicator.hpp:409-416;
    flag = alpha > atol, volume_flux.hpp:772-773)."""
    import ctypes

    import torch

    from dgsem_b200 import _capi as C
    from oracle import dgsem_oracle as do
    nd, N, cells, left, right = WORKLOADS["dmr"][:5]
    rc, _ = reference_case("dmr")
    s = do.Scheme(ndims=nd, polydeg=N, cells=cells, left=left, right=right, periodic=False,
                  bc="dmr", shock_capturing=True, surface_flux="hllc")
    atol = do.hg_atol()
    L = C.lib()
    ud = u.clone()
    t1, t2 = torch.empty_like(ud), torch.empty_like(ud)

    def p(x):
        return ctypes.c_void_p(x.data_ptr()) if x is not None else None

    def to_ref(x):
        nx, ny = cells
        return x.cpu().numpy().reshape(ny, nx, 4, -1).transpose(1, 0, 3, 2).copy()

    flagged, mismatches, margin = [], 0, math.inf
    for _ in range(nsteps):
        for stage, (u_n, u_in, u_out) in enumerate(((None, ud, t1), (ud, t1, t2),
                                                    (ud, t2, ud)), start=1):
            _, flags = solver.indicator(u_in)
            torch.cuda.synchronize()
            uh = to_ref(u_in)
            a_r = rc.alpha(uh).T.reshape(-1)
            f_r = a_r > atol
            f_d = flags.cpu().numpy().astype(bool)
            mismatches += int((f_d != f_r).sum())
            flagged.append(int(f_d.sum()))
            raw = do.hg_alpha(s, uh, raw=True)
            margin = min(margin, float(abs(raw - s.alpha_min).min()))
            C.check(L.dgsem_ssprk3_stage(solver.handle, stage, p(u_n), p(u_in), p(u_out), t, dt),
                    "stage")
        t += dt
    return {"stages_checked": len(flagged), "flagged_per_stage_min": min(flagged),
            "flagged_per_stage_max": max(flagged), "flagged_per_stage": flagged,
            "elements": math.prod(cells), "flag_mismatches": mismatches,
            "min_abs_alpha_raw_minus_alpha_min": margin,
            "checked_against": "reference HGIndicator (oracle/_ref) on the GPU stage inputs"}


def max_over_ranks(local_ms: float, world: int, device) -> float:
    """The timed total of the slowest rank (replicas: no data-path collective)."""
    if world <= 1:
        return local_ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([local_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, dofs: int, steps: int, total_ms: float) -> float:
    """Whole-job DOF-updates/s: every rank advanced its own replica by `steps`
    SSPRK3 steps (3 RHS each) within the slowest rank's time."""
    return world * dofs * 3 * steps / (total_ms * 1e-3)


def workload_config(name: str) -> dict:
    nd, N, cells, left, right, vf, sf, ic, vi, bcs = WORKLOADS[name]
    return {"workload": name, "equation": "euler3d" if nd == 3 else "euler2d",
            "mesh": list(cells), "polydeg": N, "dofs": math.prod(cells) * (N + 1) ** nd,
            "volume_flux": vf, "surface_flux": sf,
            "volume_integral": "shock_capturing_hg" if vi == "hg" else "split_form",
            "boundaries": bcs, "initial_condition": ic, "dt": time_step_size(name),
            "l2": "flushed (256 MiB write) before every timed step, outside the step events"}


# ---------------------------------------------------------------------------
# device arm
# ---------------------------------------------------------------------------
def build_solver(name: str, dev):
    import dgsem_b200 as D
    nd, N, cells, left, right, vf, sf, ic, vi, bcs = WORKLOADS[name]
    mesh = D.StructuredMesh(left, right, cells)
    eq = D.CompressibleEuler3D(1.4) if nd == 3 else D.CompressibleEuler2D(1.4)
    flux = {"chandrashekar": D.ChandrashekarFlux, "ranocha": D.RanochaFlux,
            "kennedy_gruber": D.KennedyGruberFlux}[vf]
    vint = D.VolumeIntegralShockCapturingHG(flux) if vi == "hg" else D.VolumeIntegralSplitForm(flux)
    sflux = D.HLLCFlux() if sf == "hllc" else D.LaxFriedrichsFlux()
    if bcs == "dmr":
        bset = D.BoundarySet(D.DirichletBC("double_mach"), D.OutflowBC(),
                             D.MixedDirichletSlipWallBC("double_mach"),
                             D.DirichletBC("double_mach"))
    else:
        bset = D.BoundarySet(*[D.PeriodicBC() for _ in range(2 * nd)])
    solver = D.StructuredSolver(eq, D.LobattoLegendreBasis(N), vint, sflux, mesh, bset)
    if vi == "hg":
        solver.set_indicator_parameters(0.5, 0.001, False)
    sol = D.Solution(mesh, D.LobattoLegendreBasis(N), eq, device=dev)
    init = {"tgv3d": D.InviscidTaylorGreenVortex(), "kh": D.KelvinHelmholtzInitial(),
            "dmr": D.DoubleMachReflectionInitial(1.4)}[ic]
    solver.initialize(init, sol)
    return solver, sol


def run_device_arm(args):
    import ctypes

    import torch
    import torch.distributed as dist

    import dgsem_b200 as D
    from dgsem_b200 import _capi as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", torch.cuda.current_device())
    name = args.workload
    nd, N, cells = WORKLOADS[name][:3]
    nvars = nd + 2
    dofs = math.prod(cells) * (N + 1) ** nd
    dt = time_step_size(name)
    solver, sol = build_solver(name, dev)
    integ = D.SSPRK3(sol, solver.mesh, 0.0)
    if args.variant == "auto":
        variant, variant_ms = solver.autotune(sol.u, retime=True)
    else:
        variant, variant_ms = int(args.variant), None
        solver.set_launch_variant(variant)
    stream = solver.stream
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    L = C.lib()
    h = solver.handle
    up, t1p, t2p = (ctypes.c_void_p(x.data_ptr()) for x in (sol.u, integ.tmp1.u, integ.tmp2.u))

    def step(t, evs=None, per_stage=False):
        # timed steps record events only around the step: an event between two
        # stage kernels would serialise the launches that the library lets
        # overlap (programmatic dependent launch)
        if evs:
            evs[0].record(stream)
        C.check(L.dgsem_ssprk3_stage(h, 1, None, up, t1p, t, dt), "stage 1")
        if per_stage:
            evs[1].record(stream)
        C.check(L.dgsem_ssprk3_stage(h, 2, up, t1p, t2p, t, dt), "stage 2")
        if per_stage:
            evs[2].record(stream)
        C.check(L.dgsem_ssprk3_stage(h, 3, up, t2p, up, t, dt), "stage 3")
        if evs:
            evs[3].record(stream)

    t = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(t)
            t += dt
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
               for _ in range(args.steps)]
        sampler = ClockSampler(dev.index)
        sampler.start()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = solver.launch_count()
        wall0 = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            step(t, evs[k])
            t += dt
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        if world > 1:
            dist.barrier()
        launches = solver.launch_count() - launches0
        clocks = sampler.stop()
        # per-stage split of the step (details only; untimed, same flush)
        sevs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
                for _ in range(min(args.steps, 20))]
        for k, e in enumerate(sevs):
            flush.fill_(k & 0xFF)
            step(t, e, per_stage=True)
            t += dt
        torch.cuda.synchronize()
        solver.check_finite()
    step_ms = [e[0].elapsed_time(e[3]) for e in evs]
    stage_ms = [[e[s].elapsed_time(e[s + 1]) for e in sevs] for s in range(3)]
    total_ms = max_over_ranks(sum(step_ms), world, dev)
    value = aggregate_rate(world, dofs, args.steps, total_ms)
    # roofline of the fused stage kernel
    bpd = bytes_per_dof_stage(nvars)
    # average launch duration of the stage kernel over the timed steps
    mean_stage_s = sum(step_ms) / (3 * args.steps) * 1e-3
    achieved = dofs * bpd / mean_stage_s / 1e9
    peak, peak_kind = measured_peak()
    kernel = VARIANT_KERNELS.get(variant, "stage_kernel")
    traffic = profile_traffic(name, kernel)
    # FP64 bound: FP64 operations per launch (ncu op counters of the committed
    # summary, per DOF) over the same average launch time, against the FP64
    # FMA peak measured live on this GPU
    fpeak = fp64_peak(stream)
    fpd = profile_value(name, kernel, "fp64_flops_per_dof")
    fp64 = {"bound": "fp64", "peak": fpeak["tflops"], "unit": "TFLOP/s",
            "peak_source": "measured live: dgsem_fp64_fma_peak (FMA chains, CUDA events)",
            "flops_per_dof": fpd}
    if fpd:
        fp64["achieved"] = dofs * fpd / mean_stage_s / 1e12
        fp64["frac"] = fp64["achieved"] / fpeak["tflops"]

    # e2e through the host-buffer C-ABI entry point (pinned host state)
    n_e2e = max(3, min(args.steps, 200))
    host = sol.u.detach().to("cpu").pin_memory()
    hp = ctypes.c_void_p(host.data_ptr())
    C.check(L.dgsem_ssprk3_steps_host(h, hp, t, dt, 1), "e2e warm-up")
    e2e_ms = []
    for k in range(n_e2e):
        t0 = time.perf_counter()
        C.check(L.dgsem_ssprk3_steps_host(h, hp, t, dt, 1), "e2e step")
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        t += dt
    e2e_value = world * dofs * 3 / (statistics.mean(e2e_ms) * 1e-3)
    state_bytes = dofs * nvars * 8

    # graph-replayed steps (one graph launch = one step), same flush discipline
    g = ctypes.c_void_p()
    C.check(L.dgsem_graph_create(h, up, dt, 1, ctypes.byref(g)), "graph create")
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(min(args.steps, 2000))]
    with torch.cuda.stream(stream):
        for k, (a, b) in enumerate(gev):
            flush.fill_(k & 0xFF)
            a.record(stream)
            C.check(L.dgsem_graph_launch(g, t), "graph launch")
            b.record(stream)
            t += dt
        torch.cuda.synchronize()
    graph_ms = statistics.mean(a.elapsed_time(b) for a, b in gev)
    L.dgsem_graph_destroy(g)

    # the same steps with the fused diagnostics (volume integrals of kinetic
    # energy and entropy in the stage-3 epilogue), same flush discipline
    C.check(L.dgsem_set_diagnostics(h, 1), "diagnostics on")
    dev_ = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
            for _ in range(min(args.steps, 2000))]
    with torch.cuda.stream(stream):
        for k, e in enumerate(dev_):
            flush.fill_(k & 0xFF)
            step(t, e)
            t += dt
        torch.cuda.synchronize()
    diag_ms = statistics.mean(e[0].elapsed_time(e[3]) for e in dev_)
    dvol, dke, dent = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    C.check(L.dgsem_diagnostics(h, ctypes.byref(dvol), ctypes.byref(dke), ctypes.byref(dent)),
            "diagnostics")
    C.check(L.dgsem_set_diagnostics(h, 0), "diagnostics off")

    line = {
        "metric": "FP64 DOF-updates/s per RHS", "value": value, "unit": "DOF-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic initial condition of the workload)",
        "config": workload_config(name),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs"
                     if peak_kind == "measured" else "fallback 6650 GB/s",
                     "kernel": KERNEL_DESCRIPTIONS[kernel],
                     "algorithmic_bytes_per_launch": dofs * bpd, "fp64": fp64},
        "e2e": {"value": e2e_value, "unit": "DOF-updates/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes, "steps": n_e2e,
                "ms_per_step": statistics.mean(e2e_ms)},
        "gpu_launches": launches,
        "clocks": clocks,
        "details": {"parallelism": "replicas" if world > 1 else "single",
                    "launch_variant": variant, "variant_ms": variant_ms,
                    "stage_ms_mean": [statistics.mean(x) for x in stage_ms],
                    "step_ms_median": statistics.median(step_ms),
                    "graph_step_ms_mean": graph_ms, "wall_s_timed_loop": wall,
                    "fused_diagnostics": {
                        "step_ms_mean": diag_ms,
                        "vs_plain_step": diag_ms / statistics.mean(step_ms),
                        "mean_kinetic_energy": dke.value, "mean_entropy": dent.value}},
    }
    if rank == 0 and world == 1 and name == "tgv16" and not args.no_side_workloads:
        line["details"]["side_workloads"] = side_workloads(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, n, el, threads, nwarm = reference_rate(name, args.warmup, args.steps)
            line["cpu_baseline"] = {
                "value": rate, "unit": "DOF-updates/s", "cores": threads, "kind": "reference",
                "cpu_model": cpu_model(), "sample": cpu_sample_text(name, n, el, nwarm)}
            if name == "dmr":
                line["details"]["troubled_cells"] = dmr_flag_check(solver, sol.u, t, dt, dev)
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unavailable": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batched_meshes(seed: int = 20260512, count: int = 256):
    """256 periodic [-5,5]^2 meshes with side s ~ U{16..128},
    degree N ~ U{2..7}, vortex strength ~ U[2,6], centre ~ U[-2,2]^2."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        s = int(rng.integers(16, 129))
        N = int(rng.integers(2, 8))
        beta = float(rng.uniform(2.0, 6.0))
        cx, cy = (float(v) for v in rng.uniform(-2.0, 2.0, size=2))
        out.append(((s, s), N, beta, (cx, cy)))
    return out


def batched_config() -> dict:
    """The batched workload's config, identical in both arms."""
    specs = batched_meshes()
    dofs = sum(cells[0] * cells[1] * (N + 1) ** 2 for cells, N, _, _ in specs)
    return {"workload": "batched", "meshes": len(specs), "dofs": dofs,
            "degrees": sorted({N for _, N, _, _ in specs}),
            "volume_flux": "chandrashekar", "surface_flux": "llf",
            "l2": "inputs larger than L2 (state %.2f GB)" % (dofs * 32 / 1e9),
            "graph": "one SSPRK3 step per graph replay (per-degree launches as parallel "
                     "branches, or one persistent launch per stage)"}


def run_batched(args):
    """Batched multi-mesh throughput and speedup over the per-instance path.
    With N ranks (one per GPU, no data-path collective: meshes never
    exchange data): by default every rank advances its own 256-mesh batch
    (seed + rank; weak scaling); with --shard-meshes the one 256-mesh batch
    is split over the ranks by cost (dgsem_b200.sharding; strong scaling)."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    line = measure_batched(args, rank, world)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def measure_batched(args, rank: int = 0, world: int = 1):
    """The batched line (see run_batched)."""
    import ctypes

    import torch

    import dgsem_b200 as D
    from dgsem_b200 import _capi as C
    from dgsem_b200 import sharding

    dev = torch.device("cuda", torch.cuda.current_device())
    shard = world > 1 and getattr(args, "shard_meshes", False)
    if shard:
        job = batched_meshes()
        specs = [s for _, s in sharding.local_meshes(job, rank, world)]
        job_dofs = sum(cells[0] * cells[1] * (N + 1) ** 2 for cells, N, _, _ in job)
    else:
        specs = batched_meshes(seed=20260512 + rank)
        job_dofs = None
    eq = D.CompressibleEuler2D(1.4)
    meshes = [(D.StructuredMesh((-5.0, -5.0), (5.0, 5.0), cells), N) for cells, N, _, _ in specs]
    # dt = CFL 0.5 * dx / ((2n - 1) * lambda_max), lambda_max <= 4 for these vortices
    dts = [0.5 * (10.0 / cells[0]) / ((2.0 * (N + 1) - 1.0) * 4.0) for cells, N, _, _ in specs]
    dofs = sum(cells[0] * cells[1] * (N + 1) ** 2 for cells, N, _, _ in specs)
    batch = D.BatchSolver(eq, meshes, D.ChandrashekarFlux, D.LaxFriedrichsFlux)
    batch.initialize(C.IC_ISENTROPIC_VORTEX, [(b, c[0], c[1]) for _, _, b, c in specs])
    stream = batch.stream
    if args.variant == "auto":
        variants = batch.autotune(dts)
    else:
        batch.set_launch_variant(int(args.variant))
        variants = [int(args.variant)] * len({N for _, N, _, _ in specs})

    def timed_graph(persistent: bool):
        """Graph-replayed steps in one launch mode: (step times, launches, clocks)."""
        batch.set_persistent(persistent)
        g = batch.graph(dts, 1)
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                g.launch()
            torch.cuda.synchronize()
            sampler = ClockSampler(dev.index)
            sampler.start()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            launches0 = batch.launch_count()
            for a, b in evs:
                a.record(stream)
                g.launch()
                b.record(stream)
            torch.cuda.synchronize()
            launches = batch.launch_count() - launches0
            clocks = sampler.stop()
        batch.check_finite()
        return [a.elapsed_time(b) for a, b in evs], launches, clocks, g

    # per-degree launches (degrees as parallel graph branches), then one
    # persistent launch per stage over all degrees; the line reports the faster
    modes = {"per_degree": timed_graph(False), "persistent": timed_graph(True)}
    mode_ms = {k: sum(v[0]) / args.steps for k, v in modes.items()}
    mode = min(mode_ms, key=mode_ms.get)
    step_ms, launches, clocks, g = modes[mode]
    batch.set_persistent(mode == "persistent")
    # the job's time is the slowest rank's (max over ranks)
    total_ms = max_over_ranks(sum(step_ms), world, dev)
    if shard:
        value = job_dofs * 3 * args.steps / (total_ms * 1e-3)
    else:
        value = aggregate_rate(world, dofs, args.steps, total_ms)
    # per-instance plain path: one solver per mesh, 3 stage launches per step
    per_ms = []
    for k, (cells, N, beta, c) in enumerate(specs):
        mesh, _ = meshes[k]
        basis = D.LobattoLegendreBasis(N)
        solver = D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                                    D.LaxFriedrichsFlux(), mesh,
                                    D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]),
                                    stream=stream)
        sol = D.Solution(mesh, basis, eq, device=dev)
        solver.initialize(D.IsentropicVortex(beta, c), sol)
        if args.variant == "auto":
            solver.autotune(sol.u)
        integ = D.SSPRK3(sol, mesh, 0.0)
        with torch.cuda.stream(stream):
            integ.solve_steps(solver, sol, dts[k], 2)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            integ.solve_steps(solver, sol, dts[k], 3)
            b.record(stream)
            torch.cuda.synchronize()
        per_ms.append(a.elapsed_time(b) / 3.0)
        del solver, sol, integ
    plain_ms = max_over_ranks(sum(per_ms), world, dev)
    batched_ms = total_ms / args.steps
    # e2e: pinned host state in, one batched step, state out
    host = batch.u.detach().to("cpu").pin_memory()
    e2e = []
    for _ in range(max(3, min(args.steps, 20))):
        t0 = time.perf_counter()
        batch.u.copy_(host, non_blocking=True)
        g.launch()
        host.copy_(batch.u, non_blocking=True)
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(statistics.mean(e2e), world, dev)
    e2e_dofs = job_dofs if shard else world * dofs
    # per GPU: this rank's bytes in the job's (slowest rank's) stage time
    bytes_stage = dofs * bytes_per_dof_stage(4)
    achieved = bytes_stage / (batched_ms / 3.0 * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    line = {
        "metric": "FP64 DOF-updates/s per RHS (batched)", "value": value,
        "unit": "DOF-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": batched_ms, "higher_is_better": True,
        "scaling": "strong" if shard else "weak",
        "parallelism": (f"the 256 meshes split over {world} ranks by cost (no collective)"
                        if shard else f"{world} ranks, each its own 256-mesh batch"
                        if world > 1 else "single"),
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded isentropic vortices)",
        "config": batched_config(),
        "launch_variants": variants,
        "speedup_vs_per_instance": plain_ms / batched_ms,
        "launch_mode": mode,
        "ms_per_step_by_mode": mode_ms,
        "per_instance_ms_per_step_sum": plain_ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": profile_value("batched", "stage_node_kernel",
                                              "traffic_bytes_per_stage"),
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs"},
        "e2e": {"value": e2e_dofs * 3 / (e2e_ms * 1e-3), "unit": "DOF-updates/s",
                "h2d_bytes_per_step": dofs * 32, "d2h_bytes_per_step": dofs * 32},
        "gpu_launches": launches, "clocks": clocks,
    }
    return line


def run_adjoint(args):
    print(json.dumps(measure_adjoint(args)))
    return 0


def measure_adjoint(args):
    """Adjoint workload: gradient of the final mean kinetic energy of a 2D
    Navier-Stokes Taylor-Green vortex (32 x 32 elements, N = 4, Re = 1000,
    Pr = 0.72, 1e-3 seeded momentum noise) after 200 SSPRK3 steps of
    dt = 1e-3, with respect to the initial state; checkpoints every 20 steps.
    Reports the cost of the gradient relative to the forward run."""
    import ctypes

    import torch

    import dgsem_b200 as D
    from dgsem_b200 import _capi as C

    dev = torch.device("cuda", torch.cuda.current_device())
    nsteps, every, dt, cells, N = 200, 20, 1.0e-3, (32, 32), 4
    mesh = D.StructuredMesh((0.0, 0.0), (2 * math.pi, 2 * math.pi), cells)
    basis = D.LobattoLegendreBasis(N)
    eq = D.CompressibleNavierStokes2D(1.4, 1.0e-3, 0.72)
    solver = D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    sol = D.Solution(mesh, basis, eq, device=dev)
    solver.initialize(D.TaylorGreenVortex2D(), sol)
    gen = torch.Generator(device=dev).manual_seed(0)
    sol.u[:, 1:3, :] += 1.0e-3 * torch.randn(sol.u[:, 1:3, :].shape, generator=gen,
                                             device=dev, dtype=torch.float64)
    u0 = sol.u.clone()
    dofs = math.prod(cells) * (N + 1) ** 2
    # launch shape of the forward stage kernels (line- or node-parallel)
    variant = solver.autotune(u0)[0] if args.variant == "auto" else int(args.variant)
    solver.set_launch_variant(variant)
    adj = D.Adjoint(solver, nsteps, every)
    stream = solver.stream
    L = C.lib()
    work = u0.clone()

    def forward():
        work.copy_(u0)
        C.check(L.dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(work.data_ptr()), 0.0, dt,
                                     nsteps), "dgsem_ssprk3_steps")

    reps = max(1, min(args.steps, 5))
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            forward()
            adj.gradient(u0, 0.0, dt)
        torch.cuda.synchronize()
        sampler = ClockSampler(dev.index)
        sampler.start()
        fwd, grad_ms = [], []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            forward()
            b.record(stream)
            torch.cuda.synchronize()
            fwd.append(a.elapsed_time(b))
        launches0 = solver.launch_count()
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            J, g = adj.gradient(u0, 0.0, dt)
            b.record(stream)
            torch.cuda.synchronize()
            grad_ms.append(a.elapsed_time(b))
        launches = (solver.launch_count() - launches0) // reps
        clocks = sampler.stop()
        # e2e: initial state from pinned host memory, gradient back to host
        host_u0 = u0.detach().to("cpu").pin_memory()
        host_g = torch.empty_like(host_u0).pin_memory()
        dev_u0 = torch.empty_like(u0)
        e2e = []
        for _ in range(reps):
            t0 = time.perf_counter()
            dev_u0.copy_(host_u0, non_blocking=True)
            _, gg = adj.gradient(dev_u0, 0.0, dt)
            host_g.copy_(gg, non_blocking=True)
            torch.cuda.synchronize()
            e2e.append((time.perf_counter() - t0) * 1e3)
        # one seeded central-difference check of the gradient
        d = torch.zeros_like(u0)
        d[:, 1:3, :] = torch.randn(d[:, 1:3, :].shape, generator=gen, device=dev,
                                   dtype=torch.float64)
        eps = 1.0e-6

        def J_of(v):
            w = v.clone()
            C.check(L.dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(w.data_ptr()), 0.0, dt,
                                         nsteps), "dgsem_ssprk3_steps")
            return adj.kinetic_energy(w)

        fd = (J_of(u0 + eps * d) - J_of(u0 - eps * d)) / (2 * eps)
        ad = float(torch.sum(g * d))
    fwd_ms, adj_ms = statistics.median(fwd), statistics.median(grad_ms)
    line = {
        "metric": "adjoint gradient cost / forward cost", "value": adj_ms / fwd_ms,
        "unit": "x forward", "n_gpus": 1, "steps": reps, "warmup": args.warmup,
        "ms_per_step": adj_ms / nsteps, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Taylor-Green vortex + seeded Gaussian momentum noise)",
        "config": {"workload": "adjoint", "equation": "navier_stokes2d", "mesh": list(cells),
                   "polydeg": N, "dofs": dofs, "mu": 1.0e-3, "prandtl": 0.72,
                   "ssprk3_steps": nsteps, "dt": dt, "checkpoint_every": every,
                   "objective": "mean kinetic energy of the final state",
                   "volume_flux": "chandrashekar", "surface_flux": "llf",
                   "l2": "state 0.8 MB is L2-resident (launch-latency bound workload)"},
        "forward_ms": fwd_ms, "adjoint_gradient_ms": adj_ms, "forward_launch_variant": variant,
        "reverse_only_ratio": (adj_ms - fwd_ms) / fwd_ms,
        "objective": J,
        "fd_check": {"eps": eps, "fd": fd, "adjoint": ad, "rel": abs(fd - ad) / abs(ad)},
        "e2e": {"value": statistics.median(e2e) / fwd_ms, "unit": "x forward",
                "ms": statistics.median(e2e), "h2d_bytes_per_step": u0.numel() * 8,
                "d2h_bytes_per_step": u0.numel() * 8},
        "gpu_launches": launches, "clocks": clocks,
    }
    return line


def side_workloads(args) -> dict:
    """Short runs of the batched and adjoint workloads recorded in the
    default line's details (their own lines: --workload batched / adjoint)."""
    out = {}
    for name, fn, steps in (("batched", measure_batched, 10), ("adjoint", measure_adjoint, 3)):
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = steps, 3
        try:
            t0 = time.perf_counter()
            line = fn(sub)
            keep = ("value", "unit", "ms_per_step", "speedup_vs_per_instance", "launch_mode",
                    "ms_per_step_by_mode",
                    "per_instance_ms_per_step_sum", "roofline", "forward_ms",
                    "adjoint_gradient_ms", "fd_check", "forward_launch_variant", "steps")
            out[name] = {k: line[k] for k in keep if k in line}
            out[name]["wall_s"] = time.perf_counter() - t0
        except Exception as exc:  # a side measurement never voids the headline
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: DEFAULT_STEPS of the workload)")
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="dgsem_b200", choices=["dgsem_b200", "reference"])
    ap.add_argument("--workload", default="tgv16",
                    choices=list(WORKLOADS) + ["batched", "adjoint"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard-meshes", action="store_true",
                    help="batched workload on N GPUs: split the one 256-mesh batch over the "
                         "ranks by cost (strong scaling) instead of a batch per rank")
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="skip the short batched / adjoint runs recorded in details")
    ap.add_argument("--variant", default="auto", choices=["auto", "0", "1", "2", "3", "4", "5", "6"],
                    help="launch shape of the stage kernel (auto = autotuned)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps is None:
        args.steps = DEFAULT_STEPS[args.workload]
    if args.workload == "batched":
        if args.impl == "reference":
            return run_reference_batched(args)
        return run_batched(args)
    if args.workload == "adjoint":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no adjoint"}))
            return 0
        return run_adjoint(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_device_arm(args)


if __name__ == "__main__":
    sys.exit(main())
