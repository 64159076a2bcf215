#!/usr/bin/env python
"""Benchmark of OLAM's scalar_transport_rk hot path on B200.

Workload (the batched-tracer configuration): global icosahedral hexagonal
grid NXP=200 (400,002 columns), 60 levels (mza = 61), 128 FP32 tracers with
seeded lognormal mixing ratios clipped to [1e-12, 1e-6] (10 % of them zero
above 15 km), winds and density of a balanced 35 m/s mid-latitude jet, 120 s
long step, RK2 (OLAM's default scalar_timestep_level), second-order
horizontal / third-order vertical reconstruction.  Data are synthetic: seeded
fields with the shapes and value ranges of that configuration.

One step = one scalar_transport_rk(rho_old) call (CFL check, RK densities,
implicit factorisation, both RK stages for every tracer).  Metric: tracer
cell-updates/s = tracers x prognostic (k, iw) cells / step time.

  value  device-resident: inputs already in HBM, CUDA events on the
         library stream around K steps (inputs, 12.5 GB of tracers, exceed L2)
  e2e    through the C-ABI with OLAM-style host arrays: every step uploads
         tracers, tendencies, winds and densities and downloads the tracers
  plain  the one-kernel-per-pass-per-tracer GPU form on the same data
  long_step  one long step of the dynamical core (olamgpu_timestep) on the
         same grid and tracers, unrecorded and replayed as a CUDA graph
  adjoint  device time of one adjoint call (scalar_transport_rk_adjoint:
         per-step records, layout transposes, reverse stages) over the
         forward step's, the adjoint/forward time ratio of the metric
  cpu_baseline  the C++ oracle (restatement of the reference loops), OpenMP on
         all host cores, on a bounded sample of the same workload

--impl reference runs the CPU restatement as the reference arm (the
reference itself is Fortran and cannot be built here).
"""
from __future__ import annotations

import argparse
import atexit
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nxp", type=int, default=200)
    p.add_argument("--nlev", type=int, default=60)
    p.add_argument("--ntr", type=int, default=128)
    p.add_argument("--dt", type=float, default=120.0)
    p.add_argument("--nrk", type=int, default=2)
    p.add_argument("--order", type=int, default=2)
    p.add_argument("--monot", type=int, default=0)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-column", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-long-step", action="store_true")
    p.add_argument("--terrain", type=int, default=0,
                   help="a step-topography mountain raising lpw by up to this many levels (0: flat)")
    p.add_argument("--long-step-only", action="store_true",
                   help="time only the long step (olamgpu_timestep) and print its object")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--numbering", default="local", choices=["local", "generation", "random"],
                   help="W-point numbering of the grid (the library orders its tiles itself)")
    p.add_argument("--no-window", action="store_true")
    p.add_argument("--window-only", action="store_true",
                   help="time only the checkpointed window adjoint and print its object")
    p.add_argument("--win-nxp", type=int, default=100)
    p.add_argument("--win-ntr", type=int, default=32)
    p.add_argument("--win-steps", type=int, default=24)
    p.add_argument("--win-chk", type=int, default=6)
    p.add_argument("--win-monot", type=int, default=0)
    p.add_argument("--win-fd", type=int, default=0,
                   help="window: check the gradient against central differences of the device forward "
                        "along this many seeded directions of the initial tracers and the emission")
    p.add_argument("--large", action="store_true",
                   help="only the large combined run (NXP=400, 80 levels, 32 tracers, 24 long steps of 60 s)")
    p.add_argument("--large-nxp", type=int, default=400)
    p.add_argument("--large-chk", type=int, default=8,
                   help="large run: a checkpoint every this many steps (kept in page-locked host memory)")
    p.add_argument("--large-seg", type=int, default=4,
                   help="large run: the adjoint holds this many steps' transport inputs at once")
    p.add_argument("--tile-shape", default="",
                   help="T,G,KS: force this shape of the tiled stage kernel (default: the autotuner's)")
    p.add_argument("--shape-sweep", action="store_true",
                   help="time every tile shape in steady state (forced, after warm steps) and print them")
    return p.parse_args()


class Clocks:
    """nvidia-smi sampling during the timed region: the sampler starts before
    the warm-up (its first sample can take a second to come) and begin()
    marks the start of the timed region; stop() keeps the samples that
    arrived after the mark."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.t0 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            atexit.register(self._end)        # also when the run fails between start and stop
        except OSError:
            self.proc = None

    def _end(self):
        if self.proc is not None and self.proc.poll() is None:
            self.proc.kill()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def begin(self, wait_s=5.0):
        """Mark the start of the timed region, once the sampler runs."""
        end = time.monotonic() + wait_s
        while self.proc is not None and not self.lines and time.monotonic() < end:
            time.sleep(0.01)
        self.t0 = time.monotonic()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t_end = time.monotonic()
        # one more sample after the region ends, so that a short region has one
        while len([1 for t, _ in self.lines if t >= (self.t0 or 0.0)]) == 0 and time.monotonic() < t_end + 0.5:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, ln in list(self.lines):
            if self.t0 is not None and t < self.t0:
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_case(a):
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import fast_lognormal_tracers, transport_state
    g = build_grid(a.nxp, stretched_levels(a.nlev, 100.0, 30000.0), seed=2, numbering=a.numbering)
    st = transport_state(g, a.dt, 0, seed=2)
    if a.terrain > 0:
        from olam_b200.synth.grid import with_terrain
        g = with_terrain(g, a.terrain)
    tr = fast_lognormal_tracers(g, a.ntr, seed=2024, as_list=True)
    return g, st, tr


def acoustic_bytes(g):
    """Bytes each acoustic-step launch must move at least (every array
    element it reads or writes once; stage-averaged for wrt_begs over the 3
    RK stages), per kernel scope."""
    cw = prognostic_cells(g)                                            # above-ground W and V cells
    cv = int((g.mza + 1 - g.lpv[1:].astype(np.int64)).sum())
    return {
        "setup_w": 76 * cw, "setup_v": 16 * cv, "vmca": 20 * cv, "upw4": 36 * cw,
        "grad_upv4": 16 * cw + 20 * cv, "wrt_begs": (136 + 16 / 3) * cw + 24 * cv, "prog_v": 24 * cv + 28 * cw,
        "vel_t3d": 16 * cw + 4 * cv,
    }


def prognostic_cells(g):
    """Cells the step updates: levels lpw..mza of every W column."""
    return int((g.mza + 1 - g.lpw[1:].astype(np.int64)).sum())


def cell_updates(g, ntr):
    return ntr * prognostic_cells(g)


def bytes_per_launch(g, ntr, stage):
    """Algorithmic HBM bytes of one fused stage launch: per tracer and cell
    12 B on stage 1 (read scp0 and sct, write) and 16 B on later stages (read
    scp, scp0, sct, write), plus 32 B per cell of shared winds, densities and
    volumes (vmasc 3 faces x 4, wmasc 4, rho 8, rho_old 4, volti 4)."""
    cells = prognostic_cells(g)
    per_tr = 12 if stage == 1 else 16
    return cells * (ntr * per_tr + 32)


def oracle_module():
    """The CPU oracle (the checker and the CPU baseline), its -march=native
    build made on this machine when the compiler allows."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    oracle_lib.use_native()
    return oracle_lib


def cpu_sample(g, st, tr, a, target_s, ntr_fixed=None, keep=False):
    """Time the oracle on a bounded tracer sample of the same workload.

    The sample is the first n tracers of ``tr`` (at most len(tr)) for one
    long step, n chosen from a one-tracer calibration so the timed run takes
    about ``target_s``.  With ``keep`` the result holds the oracle's output
    (n, mwa, mza) under "out" (not printed)."""
    oracle_lib = oracle_module()
    from olam_b200 import abi
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(a.dt, nrk_scal=a.nrk, scal_order=a.order, iscal_monot=a.monot)

    class S:
        pass
    s = S()
    s.__dict__.update(st.__dict__)
    res = {}

    def run(n):
        sct = [np.zeros_like(tr[0]) for _ in range(n)]
        t0 = time.perf_counter()
        out = oracle_lib.scalar_transport(fg, opts, tr[:n], sct, s)
        dt = time.perf_counter() - t0
        if keep:
            res["out"] = out
        return dt

    if ntr_fixed is None:
        t1 = run(1)
        n = int(max(1, min(len(tr), round(target_s / max(t1, 1e-3)))))
        t = run(n) if n > 1 else t1
    else:
        n = min(ntr_fixed, len(tr))
        t = run(n)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    res.update({"value": cell_updates(g, n) / t, "unit": "cell-updates/s", "cores": cores,
                "kind": "port", "seconds": t, "ntr": n, "library": oracle_lib._NAME,
                "sample": f"{n} of {a.ntr} tracers, one long step, NXP={a.nxp}, {a.nlev} levels"})
    return res


def prognostic_mask(g):
    """(mwa, mza) bool: the cells a step updates (levels lpw..mza of every
    column but the dummy point)."""
    k = np.arange(g.mza)[None, :]
    m = k >= (g.lpw.astype(np.int64)[:, None] - 1)
    m[0] = False
    return m


def field_errors(out, ref, mask):
    """Normwise max relative error max|a - b| / max|b| and RMS relative
    error sqrt(sum (a - b)^2 / sum b^2) over the masked cells."""
    a = np.asarray(out, np.float64)[mask]
    b = np.asarray(ref, np.float64)[mask]
    d = a - b
    den_max, den_rms = np.abs(b).max(), np.sqrt((b * b).sum())
    return (float(np.abs(d).max() / den_max) if den_max > 0 else float(np.abs(d).max()),
            float(np.sqrt((d * d).sum()) / den_rms) if den_rms > 0 else float(np.sqrt((d * d).sum())))


def tracer_masses(g, rho, tracers):
    """sum over the prognostic cells of rho * volt * scp per tracer, in
    float64 on the GPU (before a step with rho_old, after it with rho)."""
    import torch
    w = np.where(prognostic_mask(g), np.asarray(rho, np.float64) * g.volt, 0.0)
    wd = torch.from_numpy(w).cuda()
    out = []
    for t in tracers:
        out.append(float((torch.from_numpy(t).cuda().double() * wd).sum().item()))
    del wd
    return np.array(out)


def error_report(g, a, gpu_first, init_sample, st, cpu, mass_before, mass_after):
    """The GPU's first step against the oracle on the sampled tracers (the
    FP32 run of the CPU baseline, and an FP64 run on up to 4 of them), and
    the global tracer mass drift of the GPU step for every tracer."""
    oracle_lib = oracle_module()
    from olam_b200 import abi
    mask = prognostic_mask(g)
    n32 = cpu["ntr"]
    n64 = min(n32, 4)
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(a.dt, nrk_scal=a.nrk, scal_order=a.order, iscal_monot=a.monot)
    ref64 = oracle_lib.scalar_transport(fg, opts, init_sample[:n64], [np.zeros_like(init_sample[0])] * n64,
                                        st, fp64=True)
    e32 = [field_errors(gpu_first[i], cpu["out"][i], mask) for i in range(n32)]
    e64 = [field_errors(gpu_first[i], ref64[i], mask) for i in range(n64)]
    s64 = [field_errors(cpu["out"][i], ref64[i], mask) for i in range(n64)]
    w = np.where(mask, np.asarray(st.rho, np.float64) * g.volt, 0.0)
    m64 = np.array([(ref64[i] * w).sum() for i in range(n64)])
    live = mass_before > 0
    drift = np.abs(mass_after[live] - mass_before[live]) / mass_before[live]
    d64 = np.abs(m64 - mass_before[:n64]) / mass_before[:n64]
    agg = lambda e: {"max_rel": max(x[0] for x in e), "rms_rel": max(x[1] for x in e)}  # noqa: E731
    return {
        "fields": "tracer scp after one step (prognostic cells), worst tracer of the sample",
        "tracers_vs_fp32_oracle": dict(agg(e32), ntr=n32),
        "tracers_vs_fp64_oracle": dict(agg(e64), ntr=n64),
        "fp32_oracle_vs_fp64_oracle": dict(agg(s64), ntr=n64),
        "mass_drift": {"definition": "|sum rho volt scp after - sum rho_old volt scp before| / before, "
                                     "per tracer, over all tracers with mass",
                       "gpu_max": float(drift.max()) if drift.size else None,
                       "gpu_median": float(np.median(drift)) if drift.size else None,
                       "fp64_oracle_max": float(d64.max()) if d64.size else None,
                       "ntr": int(live.sum())},
        "tolerance": 1e-5,
    }


def dist_init(a):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        return ws, rank, local, dist
    return 1, 0, 0, None


def workload_name(g, a):
    """The workload both arms report (the same string in both lines)."""
    return (f"scalar_transport_rk NXP={a.nxp} ({g.mwa - 1} columns), {a.nlev} levels, {a.ntr} tracers, "
            f"RK{a.nrk}, horiz order {a.order}, iscal_monot {a.monot}, dt {a.dt} s"
            + (f", terrain up to {a.terrain} levels" if a.terrain > 0 else ""))


def run_reference(a):
    ws, rank, local, dist = 1, int(os.environ.get("RANK", "0")), 0, None
    if rank != 0:
        return 0
    g, st, tr = make_case(a)
    # one whole step of every tracer (the per-step work shared by the tracers
    # -- check_cfls, the densities, the implicit factors -- amortised as in
    # the model), then the timed steps as bounded samples of it so the whole
    # run stays within a few minutes
    full = cpu_sample(g, st, tr, a, 0.0, ntr_fixed=a.ntr)
    per_step = max(2.0, min(a.cpu_seconds, 120.0 / max(1, a.warmup + a.steps)))
    res = cpu_sample(g, st, tr, a, per_step)
    times = []
    for i in range(a.warmup + a.steps):
        r = cpu_sample(g, st, tr, a, per_step, ntr_fixed=res["ntr"])
        if i >= a.warmup:
            times.append(r["value"])
    sample_v = float(np.median(times)) if times else res["value"]
    v = full["value"]
    line = {"metric": "tracer cell-updates/s", "value": v, "unit": "cell-updates/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "impl": "reference",
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(g, a), "form": "the reference's loops (C++ restatement)",
                       "parallelism": "host threads of one node"},
            "cpu_baseline": {"kind": res["kind"], "cores": res["cores"],
                             "sample": f"value: one whole step of all {a.ntr} tracers ({full['seconds']:.1f} s); "
                                       f"timed steps: {res['sample']}",
                             "value": v, "unit": "cell-updates/s", "library": full["library"],
                             "whole_step_seconds": full["seconds"], "sample_steps_value": sample_v},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def bench_long_step(g, tr, a, max_over_ranks):
    """One long step of the dynamical core on the device through
    olamgpu_timestep (tend0, 4 acoustic RK3 steps, timeavg_momsc, the tracer
    step, set_scalars_bottom), on the same grid and tracers with a balanced
    jet: device time per long step unrecorded and replayed as a CUDA graph,
    and the host time per call of each."""
    import torch
    from olam_b200 import abi
    from olam_b200.lib import HostState, OlamGpu
    from olam_b200.synth.state import dynamics_state

    ds = dynamics_state(g, seed=4)
    wz = lambda: np.zeros((g.mwa, g.mza), np.float32)   # noqa: E731
    arrays = dict(rho=ds.rho, press=ds.press, thil=ds.thil, wc=ds.wc, wmc=ds.wmc, vxe=ds.vxe,
                  vye=ds.vye, vze=ds.vze, vmc=ds.vmc, vc=ds.vc,
                  vmasc=np.zeros((g.mva, g.mza), np.float32), wmasc=wz(),
                  alpha_press=ds.alpha_press, pwfac=ds.pwfac, pvfac=ds.pvfac, thilt=wz(),
                  vmxet=wz(), vmyet=wz(), vmzet=wz(), vmt=np.zeros((g.mva, g.mza), np.float32))
    from olam_b200.abi import FortranGrid
    fg = FortranGrid(g)
    opts = abi.make_opts(a.dt, nacoust=4, nrk_scal=a.nrk, scal_order=a.order, iscal_monot=a.monot)
    hs = HostState(**arrays)
    dev = OlamGpu(fg, opts, hs)
    var_t = [np.zeros_like(tr[0]) for _ in range(len(tr))]
    dev.register_scalars(tr, var_t)
    dev.set_coherence(abi.RESIDENT)
    stream = torch.cuda.ExternalStream(dev.stream())
    out = {"workload": f"olamgpu_timestep: NXP={a.nxp}, {a.nlev} levels, {len(tr)} tracers, "
                       f"dt {a.dt} s, nacoust 4, acoustic RK3, tracer RK{a.nrk}"}
    k = max(2, min(a.steps, 5))
    for mode, flags in (("eager", 0), ("graph", abi.TS_GRAPH)):
        for _ in range(4):                     # first step, then one recording per rotation
            dev.timestep(flags)
        torch.cuda.synchronize()
        dev.launch_count(reset=True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        for _ in range(k):
            dev.timestep(flags)
        host_s = time.perf_counter() - t0
        e1.record(stream)
        torch.cuda.synchronize()
        out[f"{mode}_ms_per_step"] = max_over_ranks(e0.elapsed_time(e1) / k)
        out[f"{mode}_host_ms_per_call"] = host_s * 1e3 / k
        out["launches_per_step"] = dev.launch_count() // k
    # per-kernel device time of the acoustic step (CUDA events around each
    # launch, unrecorded steps) against its algorithmic bytes
    dev.profile(True, reset=True)
    for _ in range(2):
        dev.timestep(0)
    prof = dev.profile_read()
    dev.profile(False, reset=True)
    dev.close()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs") or 6650.0)
    algo = acoustic_bytes(g)
    kern = {}
    for name, b in algo.items():
        if name in prof and prof[name][1]:
            ms = prof[name][0] / prof[name][1]
            kern[name] = {"ms_per_launch": ms, "algorithmic_gb": b / 1e9,
                          "achieved_gbs": b / (ms * 1e-3) / 1e9, "frac": b / (ms * 1e-3) / 1e9 / peak}
    out["acoustic_kernels"] = kern
    if "prog_wrtv_rk" in prof:
        out["prog_wrtv_rk_ms"] = prof["prog_wrtv_rk"][0] / prof["prog_wrtv_rk"][1]
    return out


def shape_sweep(g, st, tr, a):
    """Every shape of the tiled stage kernel forced in turn on the workload,
    timed in steady state: two warm steps, then the stage launches of
    a.steps steps (CUDA events around each launch)."""
    import torch
    from olam_b200 import abi
    from olam_b200.lib import HostState, OlamGpu
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(a.dt, nrk_scal=a.nrk, scal_order=a.order, iscal_monot=a.monot)
    dev = OlamGpu(fg, opts, HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc))
    out = []
    try:
        dev.register_scalars(tr, [np.zeros_like(t) for t in tr])
        dev.set_coherence(abi.RESIDENT)
        dev.sync_to_device(abi.F_ALL)
        dev.scalar_transport_rk(st.rho_old)
        for ordr in (0, 1):
          for T, G, KS, pk in ((32, 64, 1, 0), (32, 32, 1, 0), (32, 128, 1, 0), (16, 64, 1, 0), (16, 128, 1, 0),
                               (16, 128, 2, 0), (16, 128, 1, 2), (8, 128, 1, 0)):
            try:
                dev.set_tile_shape(T, G, KS, ordr | pk)
            except Exception as e:   # a shape this grid cannot run
                out.append({"T": T, "G": G, "KS": KS, "order": ordr | pk, "error": str(e)})
                continue
            for _ in range(2):
                dev.scalar_transport_rk(None)
            torch.cuda.synchronize()
            dev.profile(True, reset=True)
            for _ in range(a.steps):
                dev.scalar_transport_rk(None)
            prof = dev.profile_read()
            dev.profile(False, reset=True)
            ms = [prof[k][0] / prof[k][1] for k in ("tile_stage1", "tile_stage") if k in prof]
            out.append({"T": T, "G": G, "KS": KS, "order": ordr | pk, "ms_per_stage": ms})
        used, tlog = dev.tile_shape()
    finally:
        dev.close()
    return out


def window_differences(a, g, dev, var_p, tr, emis, lam, g0, gs, h=0.5):
    """Central differences of the loss along a.win_fd seeded directions
    (dx: standard normal times each tracer, de: standard normal times each
    emission): the window's long steps run again on the device from its
    start (olamgpu_window_rewind: the same dynamics, so the same winds) at
    x0 +- h dx, E +- h de, and (J+ - J-) / 2h is set against
    <dJ/dx0, dx> + <dJ/dE, de> from the adjoint.  The unlimited step is
    linear in (x0, E) for the fixed winds, so the difference has no
    truncation error: what remains is FP32 rounding of the two runs."""
    from olam_b200 import abi
    rng = np.random.default_rng(47)
    lpw0 = g.lpw - 1
    cols = np.arange(g.mwa)

    def loss(x, e):
        dev.window_rewind()
        for t, v in zip(var_p, x):
            t[...] = v
        dev.sync_to_device(abi.F_SCALARS)
        dev.set_surface_emission(e)
        for _ in range(a.win_steps):
            dev.timestep(abi.TS_GRAPH)
        dev.sync_to_host(abi.F_SCALARS)
        return sum(float((lam[n].astype(np.float64) * var_p[n]).sum()) for n in range(len(var_p)))

    errs = []
    for _ in range(a.win_fd):
        dx = [(rng.standard_normal(t.shape) * t).astype(np.float32) for t in tr]
        de = [(rng.standard_normal(e.shape) * e).astype(np.float32) for e in emis]
        for d in dx:
            d[0] = 0.0
        jp = loss([t + h * d for t, d in zip(tr, dx)], [e + h * d for e, d in zip(emis, de)])
        jm = loss([t - h * d for t, d in zip(tr, dx)], [e - h * d for e, d in zip(emis, de)])
        fd = (jp - jm) / (2 * h)
        dot = sum(float((g0[n].astype(np.float64) * dx[n]).sum())
                  + float((gs[n][cols, lpw0].astype(np.float64) * de[n]).sum()) for n in range(len(tr)))
        errs.append(abs(fd - dot) / abs(fd) if fd else abs(dot))
    dev.set_surface_emission(emis)
    return {"directions": a.win_fd, "h": h, "max_relerr": max(errs), "median_relerr": float(np.median(errs)),
            "forward": "the device's FP32 long steps (the same winds every run: the tracers are passive)"}


def bench_window(a, max_over_ranks):
    """The adjoint of tracer transport over a window of long steps: NXP=100
    (100,002 columns), 60 levels, 32 FP32 tracers with a seeded surface
    emission each, 24 long steps of 120 s of the whole core (balanced jet,
    4 acoustic RK3 steps) with checkpoints every 6 steps; the loss is a
    seeded weighted sum of the tracers after the window at 200 receptor
    cells in the lowest 3 levels.  Device time of olamgpu_window_forward
    (the 24 steps and their checkpoints) and of olamgpu_window_adjoint
    (per segment: the checkpoint restored, the dynamics run again, the
    one-step adjoints in reverse), the second call on the same window (the
    first also allocates the adjoint's buffers; its time is reported too).  The unlimited step is linear in the
    tracers and emissions for fixed winds, so J = <dJ/dx0, x0> + <dJ/dE, E>
    exactly: a size-independent check of the gradient at full size."""
    import torch
    from olam_b200 import abi
    from olam_b200.lib import HostState, OlamGpu
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import dynamics_state, fast_lognormal_tracers
    g = build_grid(a.win_nxp, stretched_levels(a.nlev, 100.0, 30000.0), seed=4)
    ds = dynamics_state(g, seed=4)
    tr = fast_lognormal_tracers(g, a.win_ntr, seed=31, as_list=True)
    rng = np.random.default_rng(41)
    emis = [(1e-13 * rng.random(g.mwa)).astype(np.float32) for _ in range(a.win_ntr)]
    for e in emis:
        e[0] = 0.0
    wz = lambda: np.zeros((g.mwa, g.mza), np.float32)   # noqa: E731
    hs = HostState(rho=ds.rho, press=ds.press, thil=ds.thil, wc=ds.wc, wmc=ds.wmc, vxe=ds.vxe, vye=ds.vye,
                   vze=ds.vze, vmc=ds.vmc, vc=ds.vc, vmasc=np.zeros((g.mva, g.mza), np.float32), wmasc=wz(),
                   alpha_press=ds.alpha_press, pwfac=ds.pwfac, pvfac=ds.pvfac, thilt=wz(), vmxet=wz(),
                   vmyet=wz(), vmzet=wz(), vmt=np.zeros((g.mva, g.mza), np.float32))
    opts = abi.make_opts(120.0, nacoust=4, nrk_scal=3, iscal_monot=a.win_monot)
    dev = OlamGpu(abi.FortranGrid(g), opts, hs)
    out = {"workload": f"window adjoint: NXP={a.win_nxp} ({g.mwa - 1} columns), {a.nlev} levels, "
                       f"{a.win_ntr} tracers with surface emission, {a.win_steps} long steps of 120 s "
                       f"(nacoust 4, acoustic RK3, tracer RK3, iscal_monot {a.win_monot}), "
                       f"checkpoints every {a.win_chk} steps; loss: 200 receptor cells in the lowest 3 levels"}
    try:
        var_p = [t.copy() for t in tr]
        var_t = [np.zeros_like(t) for t in tr]
        dev.register_scalars(var_p, var_t)
        dev.set_surface_emission(emis)
        dev.set_coherence(abi.RESIDENT)
        dev.timestep(abi.TS_GRAPH)           # buffers, tile shape, graphs: then back to the start
        dev.sync_to_device(abi.F_ALL)
        for t, t0 in zip(var_p, tr):
            t[...] = t0
        dev.sync_to_device(abi.F_SCALARS)
        torch.cuda.synchronize()

        def used_gb():
            free, total = torch.cuda.mem_get_info()
            return (total - free) / 1e9

        mem = {"after_first_step": used_gb()}
        stream = torch.cuda.ExternalStream(dev.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dev.window_forward(a.win_steps, a.win_chk, abi.TS_GRAPH)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd_ms = max_over_ranks(e0.elapsed_time(e1))
        dev.sync_to_host(abi.F_SCALARS)
        # receptors: 200 cells in the lowest three levels, a seeded weight per tracer
        rr = np.random.default_rng(43)
        iw = rr.integers(1, g.mwa, 200)
        kk = g.lpw[iw] - 1 + rr.integers(0, 3, 200)
        w = rr.standard_normal((a.win_ntr, 200))
        lam = [np.zeros((g.mwa, g.mza), np.float32) for _ in range(a.win_ntr)]
        J = 0.0
        for n in range(a.win_ntr):
            np.add.at(lam[n], (iw, kk), w[n].astype(np.float32))
            J += float((lam[n].astype(np.float64) * var_p[n]).sum())
        mem["after_forward"] = used_gb()
        # the first adjoint call also allocates its buffers; the second, of
        # the same window, is the steady state an inversion's iterations see
        dev.profile(True, reset=True)
        dev.window_adjoint(lam)
        first_ms = max_over_ranks(dev.profile_read()["window_adjoint"][0])
        dev.profile(True, reset=True)
        g0, gs = dev.window_adjoint(lam)
        mem["after_adjoint"] = used_gb()
        prof = dev.profile_read()
        dev.profile(False, reset=True)
        adj_ms = max_over_ranks(prof["window_adjoint"][0])
        lin = 0.0
        lpw0 = g.lpw - 1
        for n in range(a.win_ntr):
            lin += float((g0[n].astype(np.float64) * np.asarray(tr[n], np.float64)).sum())
            lin += float((gs[n][np.arange(g.mwa), lpw0].astype(np.float64) * emis[n]).sum())
        if a.win_fd > 0 and a.win_monot == 0:
            out["central_differences"] = window_differences(a, g, dev, var_p, tr, emis, lam, g0, gs)
        out.update({
            "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
            "adjoint_first_call_ms": first_ms,
            "recompute_ms": prof.get("window_recompute", (0.0, 0))[0],
            "adjoint_steps_ms": prof.get("adj_stage", (0.0, 0))[0] + prof.get("adj_records", (0.0, 0))[0]
            + prof.get("adj_implicit", (0.0, 0))[0],
            "loss": J, "loss_from_gradient": lin,
            "euler_relerr": abs(lin - J) / abs(J) if J else None,
            "device_gb_in_use": mem,
            "check": "J(x0, E) = <dJ/dx0, x0> + <dJ/dE, E> for the unlimited (linear) step"
                     if a.win_monot == 0 else "limited step: no linear identity",
        })
    finally:
        dev.close()
    return out


def recomputed_steps(nsteps, nchk, part):
    """Long steps the window adjoint runs again: each part [a, b) of a
    segment [s0, s1) (parts of `part` steps from s0, reversed from the last;
    part 0 or above nchk: the whole segment) runs the steps s0 .. b-1 from
    the segment's checkpoint."""
    part = nchk if part <= 0 else min(part, nchk)
    n = 0
    for s0 in range(0, nsteps, nchk):
        s1 = min(nsteps, s0 + nchk)
        b = s1
        while b > s0:
            n += b - s0
            b = s0 + (b - 1 - s0) // part * part
    return n


def bench_large(a):
    """The large combined run: NXP=400 (1,600,002 columns), 80 levels to
    40 km, the balanced jet, 32 FP32 tracers with a surface emission each,
    through the whole device long step (4 acoustic RK3 steps, RK3 tracer
    transport, damping) for 24 steps of 60 s, replayed as a CUDA graph
    (device time of the 24 steps); then the window adjoint over the same 24
    steps with a checkpoint every a.large_chk steps kept in page-locked host
    memory, the adjoint reversing a.large_seg steps at a time (an allocation
    failure is reported, not hidden).  Throughput: tracer cell-updates/s,
    forward and backward; the HBM fraction counts the bytes of the kernels
    with an algorithmic byte count (acoustic kernels, the tracer stages and
    records, the reverse stages) over the device time.  Device memory in use
    is sampled during the window's two halves (the peak of the samples)."""
    import torch
    from olam_b200 import abi
    from olam_b200.lib import HostState, OlamGpu
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import dynamics_state, fast_lognormal_tracers
    nxp, nlev, ntr, nsteps, dt = a.large_nxp, 80, 32, 24, 60.0
    g = build_grid(nxp, stretched_levels(nlev, 100.0, 40000.0), seed=4)
    ds = dynamics_state(g, seed=4)
    tr = fast_lognormal_tracers(g, ntr, seed=31, as_list=True)
    rng = np.random.default_rng(41)
    emis = [(1e-13 * rng.random(g.mwa)).astype(np.float32) for _ in range(ntr)]
    for e in emis:
        e[0] = 0.0
    wz = lambda: np.zeros((g.mwa, g.mza), np.float32)   # noqa: E731
    hs = HostState(rho=ds.rho, press=ds.press, thil=ds.thil, wc=ds.wc, wmc=ds.wmc, vxe=ds.vxe, vye=ds.vye,
                   vze=ds.vze, vmc=ds.vmc, vc=ds.vc, vmasc=np.zeros((g.mva, g.mza), np.float32), wmasc=wz(),
                   alpha_press=ds.alpha_press, pwfac=ds.pwfac, pvfac=ds.pvfac, thilt=wz(), vmxet=wz(),
                   vmyet=wz(), vmzet=wz(), vmt=np.zeros((g.mva, g.mza), np.float32))
    opts = abi.make_opts(dt, nacoust=4, nrk_scal=3)
    cells = prognostic_cells(g)
    out = {"workload": f"NXP={nxp} ({g.mwa - 1} columns), {nlev} levels to 40 km, balanced jet, {ntr} tracers "
                       f"with surface emission, {nsteps} long steps of {dt:.0f} s (nacoust 4, acoustic RK3, "
                       f"tracer RK3, damping), the long step replayed as a CUDA graph"}
    dev = OlamGpu(abi.FortranGrid(g), opts, hs)

    def used_gb():
        free, total = torch.cuda.mem_get_info()
        return (total - free) / 1e9

    class PeakSampler:
        """Device memory in use, sampled every 20 ms while a call runs."""
        def __enter__(self):
            self.peak, self.stop = used_gb(), threading.Event()

            def run():
                while not self.stop.wait(0.02):
                    self.peak = max(self.peak, used_gb())
            self.th = threading.Thread(target=run, daemon=True)
            self.th.start()
            return self

        def __exit__(self, *exc):
            self.stop.set()
            self.th.join()
            self.peak = max(self.peak, used_gb())

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs") or 6650.0)
    try:
        # the tracers as registered are the start of both runs (the device
        # steps never write the host arrays back)
        var_p = tr
        var_t = [np.zeros_like(t) for t in tr]
        dev.register_scalars(var_p, var_t)
        dev.set_surface_emission(emis)
        dev.set_coherence(abi.RESIDENT)
        dev.timestep(abi.TS_GRAPH)            # buffers, tile shape, graph: then back to the start
        dev.sync_to_device(abi.F_ALL)
        torch.cuda.synchronize()
        mem = {"after_first_step": used_gb()}
        stream = torch.cuda.ExternalStream(dev.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nsteps):
            dev.timestep(abi.TS_GRAPH)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd_ms = e0.elapsed_time(e1)
        mem["after_forward"] = used_gb()
        # per-kernel launches and times of the step: two steps issued one
        # launch at a time (a replayed graph records no per-kernel events)
        nprof = 2
        dev.profile(True, reset=True)
        for _ in range(nprof):
            dev.timestep(0)
        prof = dev.profile_read()
        dev.profile(False, reset=True)
        # algorithmic bytes of one long step: the acoustic kernels, the tracer
        # stages (12 | 16 B per tracer-cell + 32 B per cell) and the step records
        per_launch = acoustic_bytes(g)
        per_launch["tile_stage1"] = (ntr * 12 + 32) * cells
        per_launch["tile_stage"] = (ntr * 16 + 32) * cells
        per_launch["tile_weights"] = 128 * cells

        def counted(pr, n):
            b, ms = 0.0, 0.0
            for name, x in per_launch.items():
                if name in pr and pr[name][1]:
                    b += x * pr[name][1] / n
                    ms += pr[name][0] / n
            return b, ms
        step_bytes, counted_ms = counted(prof, nprof)
        ms_step = fwd_ms / nsteps
        out["forward"] = {
            "ms_per_step": ms_step, "cell_updates_per_s": ntr * cells / (ms_step * 1e-3),
            "algorithmic_gb_per_step": step_bytes / 1e9,
            "hbm_frac": step_bytes / (ms_step * 1e-3) / 1e9 / peak,
            "hbm_frac_of_counted_kernels": step_bytes / (counted_ms * 1e-3) / 1e9 / peak if counted_ms else None,
            "counted_ms_per_step": counted_ms,
            "tile_stage_ms": (prof["tile_stage"][0] / prof["tile_stage"][1]) if "tile_stage" in prof else None,
            "kernels_ms_per_step": {k: v[0] / nprof for k, v in prof.items()},
            "peak_gbs": peak,
        }
        out["device_gb_in_use"] = mem
        # the window and its adjoint from the same start
        dev.sync_to_device(abi.F_ALL)
        torch.cuda.synchronize()
        wa = {"checkpoint_every": a.large_chk, "steps_reversed_at_once": a.large_seg,
              "checkpoints": "page-locked host memory"}
        try:
            t0 = time.perf_counter()
            dev.window_memory(True, a.large_seg, nsteps, a.large_chk)
            wa["host_page_lock_s"] = time.perf_counter() - t0
            with PeakSampler() as ps:
                e0.record(stream)
                dev.window_forward(nsteps, a.large_chk, abi.TS_GRAPH)
                e1.record(stream)
                torch.cuda.synchronize()
            wf_ms = e0.elapsed_time(e1)
            mem["window_forward_peak"] = ps.peak
            # dJ/d(tracers after the window) at 200 receptor cells per tracer,
            # in the registered arrays themselves (not read again)
            lam = var_p
            rr = np.random.default_rng(43)
            for n in range(ntr):
                lam[n][...] = 0.0
                iw = rr.integers(1, g.mwa, 200)
                kk = g.lpw[iw] - 1 + rr.integers(0, 3, 200)
                np.add.at(lam[n], (iw, kk), rr.standard_normal(200).astype(np.float32))
            dev.profile(True, reset=True)
            with PeakSampler() as ps:
                e0.record(stream)
                dev.window_adjoint(lam, lam_sct=var_t, in_place=True)
                e1.record(stream)
                torch.cuda.synchronize()
            adj_ms = e0.elapsed_time(e1)
            aprof = dev.profile_read()
            dev.profile(False, reset=True)
            mem["window_adjoint_peak"] = ps.peak
            mem["after_adjoint"] = used_gb()
            # algorithmic bytes of the backward: the recomputed dynamics (the
            # acoustic kernels' counts) and the reverse stages (24 B per
            # tracer-cell: read lam, write lam_in, read-modify-write lam(scp0)
            # and lam(sct); 128 B of records per cell)
            per_launch["adj_stage"] = (ntr * 24 + 128) * cells
            bwd_bytes, bwd_counted_ms = counted(aprof, 1)
            wa.update({
                "window_forward_ms": wf_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / wf_ms,
                "forward_cell_updates_per_s": ntr * cells * nsteps / (wf_ms * 1e-3),
                "cell_updates_per_s": ntr * cells * nsteps / (adj_ms * 1e-3),
                "algorithmic_gb": bwd_bytes / 1e9,
                "hbm_frac": bwd_bytes / (adj_ms * 1e-3) / 1e9 / peak,
                "hbm_frac_of_counted_kernels": (bwd_bytes / (bwd_counted_ms * 1e-3) / 1e9 / peak
                                                if bwd_counted_ms else None),
                "recompute_ms": aprof.get("window_recompute", (None,))[0],
                "reverse_stage_ms": aprof.get("adj_stage", (None,))[0],
                "records_ms": aprof.get("adj_records", (None,))[0],
                "recomputed_steps": recomputed_steps(nsteps, a.large_chk, a.large_seg),
                "kernels_ms": {k: v[0] for k, v in aprof.items()},
            })
            out["adjoint"] = wa
        except Exception as e:   # the library's allocation failure, reported as such
            wa.update({"unavailable": str(e)[:300], "device_gb_in_use_at_failure": used_gb()})
            out["adjoint"] = wa
    finally:
        dev.close()
    return out


def run_decomposed(a, ws, rank, dist):
    """--gpus N > 1: the same global grid and tracers split over the N
    ranks by recursive coordinate bisection (olam_b200/decomp.py, in the
    manner of OLAM's para_decomp.F90); each rank steps its own columns with
    two rings of neighbours held as a halo, and after every RK stage but the
    last the border columns of all tracers move to the neighbouring ranks
    by NCCL send/receive ordered on the library's stream
    (olam_b200/nccl_halo.py; omodel/scalar_transport_rk.F90:315-322, 343,
    379).  The total work is fixed (strong scaling); value = all ranks'
    cell-updates / the slowest rank's time."""
    import torch
    from olam_b200 import abi, decomp
    from olam_b200.lib import HostState, OlamGpu
    from olam_b200.nccl_halo import nccl_exchange
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import fast_lognormal_tracers, transport_state
    g = build_grid(a.nxp, stretched_levels(a.nlev, 100.0, 30000.0), seed=2, numbering=a.numbering)
    st = transport_state(g, a.dt, 0, seed=2)
    owner = decomp.bisect(g, ws)
    loc = decomp.local_grid(g, owner, rank)
    tr = fast_lognormal_tracers(g, a.ntr, seed=2024, as_list=True, cols=loc.wmap)
    opts = abi.make_opts(a.dt, nrk_scal=a.nrk, scal_order=a.order, iscal_monot=0)
    hs = HostState(vmasc=loc.v(st.vmasc), wmasc=loc.w(st.wmasc), rho=loc.w(st.rho), wc=loc.w(st.wc))
    rho_old = loc.w(st.rho_old)
    del st
    dev = OlamGpu(abi.FortranGrid(loc.grid), opts, hs)
    var_p = tr
    var_t = [np.zeros_like(t) for t in tr]
    dev.register_scalars(var_p, var_t)
    dev.set_halo(abi.make_halo_device(loc.send, loc.recv, nccl_exchange(dist)))
    stream = torch.cuda.ExternalStream(dev.stream())
    own = loc.owned
    mine = a.ntr * int((g.mza + 1 - loc.grid.lpw[own].astype(np.int64)).sum())
    tot = torch.tensor([mine], dtype=torch.int64, device="cuda")
    dist.all_reduce(tot)
    nupd = int(tot.item())

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    dev.set_coherence(abi.RESIDENT)
    dev.sync_to_device(abi.F_ALL)
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    dev.scalar_transport_rk(rho_old)
    for _ in range(a.warmup):
        dev.scalar_transport_rk(None)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks.begin()
    dev.profile(True, reset=True)
    dev.launch_count(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        dev.scalar_transport_rk(None)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = dev.launch_count()
    prof = dev.profile_read()
    dev.profile(False, reset=True)
    clk = clocks.stop()
    dist.barrier()
    torch.cuda.synchronize()
    ms_step = max_over_ranks(ms / a.steps)
    value = nupd / (ms_step * 1e-3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs") or 6650.0)
    cells = int((g.mza + 1 - loc.grid.lpw[own].astype(np.int64)).sum())
    tot_b, tot_ms, nl = 0.0, 0.0, 0
    for name, stage in (("tile_stage1", 1), ("tile_stage", 2)):
        if name in prof:
            m, c = prof[name]
            tot_ms += m
            nl += c
            tot_b += c * cells * (a.ntr * (12 if stage == 1 else 16) + 32)
    achieved = (tot_b / nl) / ((tot_ms / nl) * 1e-3) / 1e9 if nl else None
    # end to end through the C-ABI with host arrays on every rank
    dev.sync_to_host(abi.F_SCALARS)
    dev.set_coherence(abi.SYNC_EACH_CALL)
    dev.scalar_transport_rk(rho_old)
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(a.e2e_steps):
        dev.scalar_transport_rk(rho_old)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / a.e2e_steps)
    plane = loc.grid.mwa * g.mza * 4
    h2d = a.ntr * 2 * plane + loc.grid.mva * g.mza * 4 + plane * 2 + loc.grid.mwa * g.mza * 8 + plane
    dev.close()
    if rank == 0:
        line = {
            "metric": "tracer cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(g, a),
                       "form": "fused batched, tiled, one part of the grid per rank",
                       "parallelism": f"domain decomposition x{ws} (recursive coordinate bisection; "
                                      f"border columns of all tracers over NCCL after every RK stage but the last)",
                       "l2": "inputs larger than L2"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback",
                         "kernel": "k_tile (rank 0's launches)"},
            "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
            "halo": {"columns_sent_by_rank0": {str(r): len(v) for r, v in loc.send.items()},
                     "exchange_ms_per_step_rank0": prof.get("halo_exchange", (0.0, 0))[0] / a.steps},
            "e2e": {"value": nupd / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d * ws,
                    "d2h_bytes_per_step": a.ntr * plane * ws, "seconds_per_step": e2e_s},
            "cpu_baseline": None,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    ws, rank, local, dist = dist_init(a)
    import torch
    from olam_b200 import abi
    from olam_b200.lib import HostState, OlamGpu

    torch.cuda.set_device(local)
    if ws > 1:
        return run_decomposed(a, ws, rank, dist)
    if a.large:
        print(json.dumps({"large": bench_large(a)}), flush=True)
        return 0
    g, st, tr = make_case(a)
    if a.long_step_only:
        out = bench_long_step(g, tr, a, lambda x: x)
        if rank == 0:
            print(json.dumps({"long_step": out}), flush=True)
        return 0
    if a.window_only:
        out = bench_window(a, lambda x: x)
        if rank == 0:
            print(json.dumps({"window_adjoint": out}), flush=True)
        return 0
    if a.shape_sweep:
        print(json.dumps({"shape_sweep": shape_sweep(g, st, tr, a)}), flush=True)
        return 0
    fg = abi.FortranGrid(g)
    opts = abi.make_opts(a.dt, nrk_scal=a.nrk, scal_order=a.order, iscal_monot=a.monot)
    # the first tracers' initial values (the oracle's sample) and every
    # tracer's mass, for the error report
    report = rank == 0 and not a.no_cpu
    init_sample = [t.copy() for t in tr[:min(a.ntr, 16)]] if report else []
    mass_before = tracer_masses(g, st.rho_old, tr) if report else None
    hs = HostState(vmasc=st.vmasc, wmasc=st.wmasc, rho=st.rho, wc=st.wc)
    dev = OlamGpu(fg, opts, hs)
    var_p = tr                     # separately allocated, as OLAM's var_p
    var_t = [np.zeros_like(tr[0]) for _ in range(a.ntr)]
    dev.register_scalars(var_p, var_t)
    stream = torch.cuda.ExternalStream(dev.stream())
    nupd = cell_updates(g, a.ntr)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident fused form
    dev.set_transport_form(abi.TRANSPORT_FUSED)
    if a.tile_shape:
        dev.set_tile_shape(*[int(x) for x in a.tile_shape.split(",")])
    dev.set_coherence(abi.RESIDENT)
    dev.sync_to_device(abi.F_ALL)
    dev.scalar_transport_rk(st.rho_old)          # uploads rho_old once
    gpu_first, mass_after = None, None
    if report:
        # the first step's result for the error report (outside the timed region)
        dev.sync_to_host(abi.F_SCALARS)
        gpu_first = [t.copy() for t in var_p[:len(init_sample)]]
        mass_after = tracer_masses(g, st.rho, var_p)
    clocks = Clocks(local)
    clocks.start()
    for _ in range(a.warmup):
        dev.scalar_transport_rk(None)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks.begin()
    dev.profile(True, reset=True)
    dev.launch_count(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        dev.scalar_transport_rk(None)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = dev.launch_count()
    prof = dev.profile_read()
    used, tlog = dev.tile_shape()
    tile_shape = {"T": used[0], "G": used[1], "KS": used[2], "order": used[3],
                  "candidates_ms_per_stage": [{"T": r[0], "G": r[1], "KS": r[2], "order": r[3], "ms": r[5]}
                                              for r in tlog],
                  "note": "columns per tile, tracers per block, level chunks per tile, tile order (0: the "
                          "library's curve, 1: the caller's numbering; +2: the paired kernel, a warp per "
                          "column pair reading each U row once for both); "
                          + ("forced by --tile-shape" if a.tile_shape else
                             "chosen by the library's autotuner on the first step")}
    dev.profile(False, reset=True)
    clk = clocks.stop()
    barrier()
    torch.cuda.synchronize()
    ms_step = max_over_ranks(ms / a.steps)
    value = ws * nupd / (ms_step * 1e-3)

    # roofline of the dominant kernel (fused stage launches)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = float(peak or 6650.0)
    # the stage kernel: k_tile (tiled form) or k_fused (one column per block)
    tiled = "tile_stage1" in prof
    pre = "tile_stage" if tiled else "fused_stage"
    kname = "k_tile" if tiled else "k_fused"
    tot_bytes, tot_ms, nl = 0.0, 0.0, 0
    for name, stage in ((pre + "1", 1), (pre, 2)):
        if name in prof:
            m, c = prof[name]
            tot_ms += m
            nl += c
            tot_bytes += c * bytes_per_launch(g, a.ntr, stage)
    achieved = (tot_bytes / nl) / ((tot_ms / nl) * 1e-3) / 1e9 if nl else None
    # DRAM traffic per launch: the ratio of measured (ncu, smaller grid of the
    # same kernel) to algorithmic bytes, applied to this launch's algorithmic bytes
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"{kname}_traffic.json")
    if nl and os.path.exists(tfile):
        try:
            ratio = float(json.load(open(tfile))["dram_over_algorithmic"])
            traffic = ratio * tot_bytes / nl
        except (OSError, ValueError, KeyError):
            traffic = None

    # ---- plain one-kernel-per-tracer form on the same device data
    plain, plain_passes = None, None
    if not a.no_plain:
        dev.set_transport_form(abi.TRANSPORT_PLAIN)
        dev.scalar_transport_rk(None)
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        ksteps = max(1, min(a.steps, 3))
        p0.record(stream)
        for _ in range(ksteps):
            dev.scalar_transport_rk(None)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1) / ksteps)
        plain = ws * nupd / (pms * 1e-3)
        # each pass's time (CUDA events around every launch, one more step)
        # against the bytes it moves at least: every array it reads or writes
        # once (cells: prognostic cells; faces: V-face levels)
        dev.profile(True, reset=True)
        dev.scalar_transport_rk(None)
        pprof = dev.profile_read()
        dev.profile(False, reset=True)
        cells = prognostic_cells(g)
        faces = int((g.mza + 1 - g.lpv[1:].astype(np.int64)).sum())
        i2d = 5 if a.order == 3 else 2
        pbytes = {"pass_grad": (4 + 4 * i2d) * cells,
                  "pass_vflux": (4 + 4 * i2d) * cells + 8 * faces,
                  "pass_wcol": 28 * cells + 8 * faces}
        plain_passes = {}
        for nm, b in pbytes.items():
            if nm in pprof and pprof[nm][1]:
                pm = pprof[nm][0] / pprof[nm][1]
                plain_passes[nm] = {"ms_per_launch": pm, "launches_per_step": pprof[nm][1],
                                    "bytes_per_launch": b, "achieved_gbs": b / (pm * 1e-3) / 1e9,
                                    "frac": b / (pm * 1e-3) / 1e9 / peak}
        dev.set_transport_form(abi.TRANSPORT_FUSED)

    # ---- the batched form with one column per block, for comparison
    column = None
    if not a.no_column and a.terrain == 0:   # the per-column form runs flat grids only
        dev.set_transport_form(abi.TRANSPORT_FUSED_COLUMN)
        dev.scalar_transport_rk(None)
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        ksteps = max(1, min(a.steps, 3))
        c0.record(stream)
        for _ in range(ksteps):
            dev.scalar_transport_rk(None)
        c1.record(stream)
        torch.cuda.synchronize()
        column = ws * nupd / (max_over_ranks(c0.elapsed_time(c1) / ksteps) * 1e-3)
        dev.set_transport_form(abi.TRANSPORT_FUSED)

    # ---- adjoint of the step: device time of the adjoint call (its
    # preparation, layout transposes and reverse stages; RESIDENT, so no
    # inputs are uploaded inside it) against the forward step above
    adjoint = None
    if not a.no_adjoint and a.monot == 0:
        dev.scalar_transport_rk_adjoint(var_p)          # allocates, builds records
        torch.cuda.synchronize()
        dev.profile(True, reset=True)
        kadj = max(1, min(a.steps, 2))
        for _ in range(kadj):
            dev.scalar_transport_rk_adjoint(var_p)
        aprof = dev.profile_read()
        dev.profile(False, reset=True)
        adj_ms = max_over_ranks(aprof["adjoint"][0] / aprof["adjoint"][1])
        st_ms, st_n = aprof.get("adj_stage", (0.0, 0))
        stage_bytes = (a.ntr * 24 + 128) * prognostic_cells(g)
        adjoint = {
            "ms_per_step": adj_ms, "forward_ms_per_step": ms_step,
            "adjoint_over_forward": adj_ms / ms_step,
            "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in aprof.items()},
            "stage_kernel": "k_tile_adj",
            "stage_algorithmic_bytes": stage_bytes,
            "stage_achieved_gbs": (stage_bytes / ((st_ms / st_n) * 1e-3) / 1e9) if st_n else None,
        }

    # ---- end to end through the C-ABI with host arrays
    dev.sync_to_host(abi.F_SCALARS)
    dev.set_coherence(abi.SYNC_EACH_CALL)
    dev.scalar_transport_rk(st.rho_old)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(a.e2e_steps):
        dev.scalar_transport_rk(st.rho_old)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / a.e2e_steps)
    plane = g.mwa * g.mza * 4
    h2d = a.ntr * 2 * plane + g.mva * g.mza * 4 + plane * 2 + g.mwa * g.mza * 8 + plane
    d2h = a.ntr * plane
    e2e = {"value": ws * nupd / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "seconds_per_step": e2e_s}
    dev.close()

    long_step = None
    if not a.no_long_step:
        long_step = bench_long_step(g, tr, a, max_over_ranks)

    window = None
    if not a.no_window:
        window = bench_window(a, max_over_ranks)

    cpu, errors = None, None
    if report:
        cpu = cpu_sample(g, st, init_sample, a, a.cpu_seconds, keep=True)
        errors = error_report(g, a, gpu_first, init_sample, st, cpu, mass_before, mass_after)
        cpu.pop("out")

    if rank == 0:
        line = {
            "metric": "tracer cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": ws, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(g, a),
                       "form": "fused batched, tiled" if tiled else "fused batched",
                       "parallelism": "one domain on one GPU",
                       "l2": "inputs larger than L2 (12.5 GB of tracers per array)"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "peak_source": peak_src, "kernel": f"{kname} ({pre})",
                         "kernel_ms_per_launch": (tot_ms / nl) if nl else None},
            "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
            "tile_shape": tile_shape,
            "plain_gpu_value": plain,
            "plain_passes": plain_passes,
            "fused_over_plain": (value / plain) if plain else None,
            "fused_column_value": column,
            "e2e": e2e,
            "adjoint": adjoint,
            "window_adjoint": window,
            "long_step": long_step,
            "cpu_baseline": cpu,
            "errors": errors,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
