#!/usr/bin/env python
"""Benchmark of the FOPIS electrostatic PIC timestep on B200.

Metric: particle-steps/s of RootGrid::mainLoopES (one step = push + gather +
boundaries + absorption + deposit + emission + injection + two multigrid
Poisson solves with the capacity-matrix correction + E field + periodic sort)
on the 128^3-cell workload: Dirichlet box with thermal injection through all
six faces, electrons + ions (mass ratio 100) at 32 particles/cell/species, a
16^3-cell conductor cube at the centre emitting photoelectrons from its +x
face, solver tolerance ||r||/||f|| <= 1e-8. Synthetic plasma, Philox seeded.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fopis|reference]

With torchrun and N > 1 every rank runs an independent replica (the path does
not shard: replicas only); value is the sum over ranks of particle-steps over
the max over ranks of the timed device time.
"""
from __future__ import annotations

import argparse
import json
import re
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PUSH_BYTES_PER_PARTICLE = 56.0   # 28 B split-precision state read + 28 B written (gather+push+deposit fused)
PUSH_BYTES_FP64 = 104.0          # FP64 mode: 4 B cell + 48 B offsets and velocities, read and written


def precision_of(args):
    from fopis_b200 import _abi
    return _abi.FP64 if args.precision == "fp64" else _abi.MIXED


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons sampled during the timed region: NVML read
    every 10 ms from a thread (so a timed region of ~0.1 s still gives about ten
    samples), nvidia-smi every 200 ms where NVML is unavailable. Reading only:
    no clock or other GPU setting is changed."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, period_s: float = 0.01):
        self.index = index
        self.period = period_s
        self.proc = None
        self.lines = []
        self.samples = []          # (sm_mhz, max_mhz, set of reason names)
        self.stop = threading.Event()
        self.thread = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll_nvml(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), {k for k, b in bits.items() if r & b}))
            except Exception:
                pass
            self.stop.wait(self.period)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
            self.thread.start()
            self.source = "nvml 10 ms"
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            self.source = "nvidia-smi 200 ms"
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            if len(f) < 9:
                continue
            try:
                self.samples.append((float(f[1]), float(f[2]),
                                     {nm for nm, v in zip(self.NAMES, f[5:9]) if v.lower() == "active"}))
            except ValueError:
                continue

    def __exit__(self, *a):
        self.stop.set()
        if self.thread:
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [x[0] for x in self.samples]
        mx = self.samples[-1][1] if self.samples else None
        reasons = set()
        for x in self.samples:
            reasons |= x[2]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": self.source}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return world, rank, local


def allreduce(v: float, op: str, world: int) -> float:
    """Max or sum of a scalar over the ranks (replicas only: timing and totals)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def aggregate(ms: float, psteps: float, world: int):
    """Whole-job throughput of N replicas: particle-steps summed, time = max over ranks."""
    ms_max = allreduce(ms, "max", world)
    ps = allreduce(psteps, "sum", world)
    return ms_max, ps, ps / (ms_max * 1e-3)


WORKLOADS = {
    "periodic32": ("32^3 nodes fully periodic, e+i mass ratio 100, Te = Ti, no object", 16),
    "cube64": ("64^3 cells Dirichlet + 6-face injection, e+i mass ratio 100, 8^3 conductor cube", 32),
    "cube128": ("128^3 cells Dirichlet + 6-face injection, e+i mass ratio 100, 16^3 conductor cube with "
                "+x photoemission (10x electron flux, 0.2 Te)", 32),
    "cube128_plain": ("128^3 cells Dirichlet + 6-face injection, e+i mass ratio 100, 16^3 conductor cube", 32),
    "craft256": ("256^3 cells Dirichlet + 6-face injection, e+i mass ratio 100, 32x16x16 body + 48x4x16 panel "
                 "with +x photoemission", 32),
    "em128": ("EM solver (FDTD with damping layers), 128^3 cells Dirichlet + 6-face injection, e+i mass ratio 100, "
              "Te = 5 keV, n = 1e12 m^-3, Courant 0.5, no object", 32),
}


def workload_desc(name: str, ppc) -> str:
    text, default_ppc = WORKLOADS[name]
    if name == "em128":
        return f"{name}: {text}, {ppc or default_ppc} ppc/species, one Poisson solve at start-up (MG to 1e-8)"
    solves = "1 solve/step" if name == "periodic32" else "2 solves/step"
    return f"{name}: {text}, {ppc or default_ppc} ppc/species, MG to ||r||/||f|| <= 1e-8, {solves}"


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def guess_mode(args):
    from fopis_b200 import _abi
    return _abi.GUESS_HISTORY if args.guess == "history" else _abi.GUESS_WARM


def build_sim(args, rank, local):
    from fopis_b200 import RootGrid, config
    cfg = config.workload(args.workload, ppc=args.ppc, seed=20251203 + 7919 * rank, sort_interval=args.sort_interval,
                          precision=precision_of(args))
    g = RootGrid(cfg, device=local)
    g.set_guess_mode(guess_mode(args))
    t0 = time.time()
    for o in range(len(cfg.objects)):
        g.initializeObjectsCmatrix(o)
    t_cmat = time.time() - t0
    return cfg, g, t_cmat


def total_particles(st, nsp):
    """Valid particles after the last step or sort."""
    return int(sum(st.valid_particles[s] for s in range(nsp)))


def pushed_particles(st, nsp):
    """Valid particles the last step's push moved (its particle-steps)."""
    return int(sum(st.pushed_step[s] for s in range(nsp)))


def run_gpu(args, world, rank, local):
    import torch
    from fopis_b200 import PARTICLE_DTYPE
    cfg, g, t_cmat = build_sim(args, rank, local)
    nsp = cfg.params.nspecies
    g.generate_ambient()
    g.initialize()
    for _ in range(args.warmup):
        g.mainLoopES(1)
    stream = torch.cuda.ExternalStream(g.stream_ptr(), device=torch.device("cuda", local))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = g.stats().kernel_launches
    psteps = 0
    push_ms, vcyc, pushed, phases_all, pointwise = [], [], [], [], []
    barrier(world)
    torch.cuda.synchronize(local)
    if args.profile:
        torch.cuda.profiler.start()
    step_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for t in range(args.steps):
            g.mainLoopES(1)
            step_ev[t].record(stream)
            st = g.stats()
            n = pushed_particles(st, nsp)
            psteps += n
            pushed.append(n)
            # the push phase: the fused ES push, or the EM step's move + current + deposit pass
            push_ms.append(st.ms_phase[0] + st.ms_phase[2] if args.workload == "em128" else st.ms_phase[0])
            phases_all.append([round(x, 3) for x in st.ms_phase])
            vcyc.append(st.vcycles_step)
            pointwise.append(st.residual_pointwise)
        ev1.record(stream)
        torch.cuda.synchronize(local)
    if args.profile:
        torch.cuda.profiler.stop()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    step_ms = [ev0.elapsed_time(step_ev[0])] + [step_ev[t - 1].elapsed_time(step_ev[t]) for t in range(1, args.steps)]
    launches = g.stats().kernel_launches - launches0
    ms_max, psteps_all, _ = aggregate(ms, float(psteps), world)
    st = g.stats()
    phases = list(st.ms_phase)
    result = {
        "ms": ms_max, "psteps": psteps_all, "launches": launches, "clocks": clk.summary(),
        "push_ms": float(np.mean(push_ms)), "pushed": float(np.mean(pushed)),
        "vcycles_per_step": float(np.mean(vcyc)), "phases_last": phases, "t_cmat": t_cmat,
        "pointwise_max": float(np.max(pointwise)),
        "particles": total_particles(st, nsp), "n_cmat": [len(o.nodes) for o in cfg.objects],
        "step_ms": [round(x, 3) for x in step_ms], "phases_all": phases_all,
        "solve_mode": ["host loop", "device-loop graph", "device-loop graph with programmatic dependent launch"][
            st.solve_mode],
    }
    Cm = g.get_cmatrix(0) if cfg.objects else None
    V, Q, cur = g.getObject(0) if cfg.objects else (0.0, 0.0, None)
    result["potential_V"] = cfg.norm.unpotential(V)
    # end-to-end through the reference-facing API: the particle set enters from
    # pinned host memory in the reference's 56-byte layout, every step reads the
    # diagnostics main.cpp writes (energy, object potential/charge/current).
    if args.e2e:
        recs = [g.getParticles(s) for s in range(nsp)]
        g.close()
        host = [torch.from_numpy(r.view(np.uint8)).pin_memory() for r in recs]
        from fopis_b200 import RootGrid
        g2 = RootGrid(cfg, device=local)
        g2.set_guess_mode(guess_mode(args))
        if Cm is not None:
            g2.set_cmatrix(0, Cm)
        nbytes = sum(h.numel() for h in host)
        barrier(world)
        torch.cuda.synchronize(local)
        t0 = time.perf_counter()
        stream2 = torch.cuda.ExternalStream(g2.stream_ptr(), device=torch.device("cuda", local))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream2)
        for s in range(nsp):
            n = host[s].numel() // 56
            rc = g2.lib.fopis_load_particles(g2.h, s, host[s].data_ptr(), n)
            g2._check(rc)
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream2)
        g2.initialize()
        eb.record(stream2)
        ps2 = 0
        d2h = 0
        for _ in range(args.steps):
            g2.mainLoopES(1)
            g2.getEnergy()
            if cfg.objects:
                g2.getObject(0)
            ps2 += pushed_particles(g2.stats(), nsp)
            d2h += 16 + (16 + 8 * nsp if cfg.objects else 0)
        e1.record(stream2)
        torch.cuda.synchronize(local)
        barrier(world)
        ms2, ps2, v2 = aggregate(e0.elapsed_time(e1), float(ps2), world)
        result["e2e"] = {"value": v2, "unit": "particle-steps/s",
                         "h2d_bytes_per_step": int(nbytes // max(1, args.steps)),
                         "d2h_bytes_per_step": int(d2h // max(1, args.steps)),
                         "ms_total": ms2, "ms_upload": e0.elapsed_time(ea), "ms_initialize": ea.elapsed_time(eb),
                         "ms_steps": eb.elapsed_time(e1),
                         "note": "one upload of the particle set (56-byte records) from pinned "
                                 "host memory + initialize + K steps with per-step diagnostics"}
        g2.close()
    else:
        g.close()
    result["cmatrix"] = Cm
    return result, cfg


def learned_comparison(args, rank, local, Cm):
    """V-cycles and step time of three Poisson starts at the same tolerance, on
    contexts with the same seed: `warm` continues from the current phi (the
    reference), `history` starts each solve from the per-solve history, `learned`
    adds the network's increment to the history start of the first solve. The
    learned context trains online on its own first solves for `learned_train`
    steps (all three step together), then each runs `steps` timed steps with
    training off."""
    import torch
    from fopis_b200 import RootGrid, _abi, config

    def mk():
        return config.workload(args.workload, ppc=args.ppc, seed=20251203 + 7919 * rank,
                               sort_interval=args.sort_interval)
    cfg = mk()
    names = ("warm", "history", "learned")
    gs = [RootGrid(mk(), device=local) for _ in names]
    for g in gs:
        if Cm is not None:
            g.set_cmatrix(0, Cm)
        g.generate_ambient()
        g.initialize()
    gs[1].set_guess_mode(_abi.GUESS_HISTORY)
    gs[2].set_guess_mode(_abi.GUESS_HISTORY)
    gs[2].unet_training(True, args.learned_lr)
    loss = []
    for _ in range(args.learned_train):
        for g in gs:
            g.mainLoopES(1)
        loss.append(gs[2].unet_state()[0])
    train_ms = gs[2].unet_last()[3]
    gs[2].unet_training(False)
    gs[2].set_guess_mode(_abi.GUESS_LEARNED)
    out = {}
    for name, g in zip(names, gs):
        stream = torch.cuda.ExternalStream(g.stream_ptr(), device=torch.device("cuda", local))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        cyc, first, used, ratio, fwd = [], [], [], [], []
        torch.cuda.synchronize(local)
        e0.record(stream)
        for _ in range(args.steps):
            g.mainLoopES(1)
            st = g.stats()
            cyc.append(st.vcycles_step)
            first.append(st.vcycles_step - (st.vcycles_last if cfg.objects else 0))
            used.append(st.learned_used)
            if name == "learned":
                warm, guess, msf, _ = g.unet_last()
                fwd.append(msf)
                if st.learned_used and warm > 0:
                    ratio.append(guess / warm)
        e1.record(stream)
        torch.cuda.synchronize(local)
        out[name] = dict(ms=e0.elapsed_time(e1) / args.steps, vcycles=float(np.mean(cyc)),
                         first=float(np.mean(first)), used=int(np.sum(used)), ratio=ratio, fwd=fwd,
                         V=cfg.norm.unpotential(g.getObject(0)[0]) if cfg.objects else None)
    pol = gs[2].unet_policy()
    for g in gs:
        g.close()
    w, l = out["warm"], out["learned"]
    return {"train_steps": args.learned_train, "steps": args.steps, "tolerance": 1e-8,
            "vcycles_per_step": {k: out[k]["vcycles"] for k in names},
            "first_solve_vcycles": {k: out[k]["first"] for k in names},
            "ms_per_step": {k: out[k]["ms"] for k in names},
            "vcycle_reduction_vs_warm": {k: w["vcycles"] / out[k]["vcycles"] for k in names[1:] if out[k]["vcycles"]},
            "learned_used_steps": l["used"],
            "guess_over_history_residual_median": float(np.median(l["ratio"])) if l["ratio"] else None,
            "ms_network_forward": float(np.mean(l["fwd"])) if l["fwd"] else None, "ms_network_train_step": train_ms,
            "loss_first_last": [loss[2] if len(loss) > 2 else None, loss[-1] if loss else None],
            "spacecraft_potential_V": {k: out[k]["V"] for k in names},
            "policy_history_learned_enabled": list(pol)}


def mixed_vs_fp64(args, local, Cm, steps: int = 100):
    """The mixed-precision step against the FP64 GPU mode on the same seed and
    workload: rho, phi and E after one step (max |difference| / max |FP64
    value|), and the spacecraft-potential history over `steps` steps."""
    from fopis_b200 import RootGrid, _abi, config
    gs = []
    for prec in (_abi.MIXED, _abi.FP64):
        cfg = config.workload(args.workload, ppc=args.ppc, seed=20251203, sort_interval=args.sort_interval,
                              precision=prec)
        g = RootGrid(cfg, device=local)
        g.set_guess_mode(_abi.GUESS_HISTORY)
        if Cm is not None:
            g.set_cmatrix(0, Cm)
        g.generate_ambient()
        g.initialize()
        gs.append(g)
    for g in gs:
        g.mainLoopES(1)

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    out = {"steps": steps, "rho": rel(gs[0].getRho(), gs[1].getRho()), "phi": rel(gs[0].getPhi(), gs[1].getPhi()),
           "E": max(rel(a, b) for a, b in zip(gs[0].getEref(), gs[1].getEref()))}
    if cfg.objects:
        V = [(gs[0].getObject(0)[0], gs[1].getObject(0)[0])]
        for _ in range(steps - 1):
            for g in gs:
                g.mainLoopES(1)
            V.append((gs[0].getObject(0)[0], gs[1].getObject(0)[0]))
        V = np.array(V)
        out["potential_history"] = float(np.max(np.abs(V[:, 0] - V[:, 1])) / np.max(np.abs(V[:, 1])))
        out["potential_V_last"] = [cfg.norm.unpotential(float(v)) for v in V[-1]]
    for g in gs:
        g.close()
    out["note"] = ("mixed (fp32 split-precision particles, int64 fixed-point rho) against the fp64 GPU mode, "
                   "same seed; field errors after one step as max|diff|/max|fp64|; potential over the steps")
    return out


def craft256_block(args, local, steps: int = 8, warmup: int = 2):
    """The 256^3 spacecraft workload (32x16x16 body + 48x4x16 panel, photoemission,
    ~1.07e9 particles): ms/step, particle-steps/s and the push roofline fraction,
    with the capacity-matrix build time. Timed with CUDA events on the library stream."""
    import torch
    from fopis_b200 import RootGrid, _abi, config
    cfg = config.workload("craft256", seed=20251203, sort_interval=args.sort_interval)
    g = RootGrid(cfg, device=local)
    g.set_guess_mode(_abi.GUESS_HISTORY)
    t0 = time.time()
    g.initializeObjectsCmatrix(0)
    t_cmat = time.time() - t0
    g.generate_ambient()
    g.initialize()
    for _ in range(warmup):
        g.mainLoopES(1)
    stream = torch.cuda.ExternalStream(g.stream_ptr(), device=torch.device("cuda", local))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    psteps, push, pushed = 0, [], []
    torch.cuda.synchronize(local)
    e0.record(stream)
    for _ in range(steps):
        g.mainLoopES(1)
        st = g.stats()
        n = pushed_particles(st, cfg.params.nspecies)
        psteps += n
        pushed.append(n)
        push.append(st.ms_phase[0])
    e1.record(stream)
    torch.cuda.synchronize(local)
    ms = e0.elapsed_time(e1)
    st = g.stats()
    hbm, _ = peaks()
    achieved = PUSH_BYTES_PER_PARTICLE * float(np.mean(pushed)) / (float(np.mean(push)) * 1e-3) / 1e9
    out = {"workload": workload_desc("craft256", None), "steps": steps, "warmup": warmup,
           "ms_per_step": ms / steps, "particle_steps_per_s": psteps / (ms * 1e-3),
           "particles": total_particles(st, cfg.params.nspecies), "n_cmat": len(cfg.objects[0].nodes),
           "setup_cmatrix_s": round(t_cmat, 2), "vcycles_per_step": st.vcycles_step,
           "push_roofline": {"achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm}}
    g.close()
    return out


# Algorithmic bytes of one FDTD update per interior index of the extended Yee
# grid: three edge (face) components read and written, three of the other
# field read (the neighbours come from cache).
FDTD_BYTES_PER_INDEX = 72


def em128_block(args, local, steps: int = 6, warmup: int = 2):
    """The EM solver's step (RootGrid::mainLoopEM) on the em128 workload: ms/step,
    particle-steps/s, phase times, and the HBM fractions of the FDTD updates
    (72 B per interior index of the 389^3 extended grid) and of the particle
    pass (the velocity update, the move, the current and the deposit in one
    pass when no body emits, as here: 56 B per particle, the state read and
    written). Timed with CUDA events on the library stream."""
    import torch
    from fopis_b200 import RootGrid, config
    cfg = config.workload("em128", seed=20251203, sort_interval=args.sort_interval)
    g = RootGrid(cfg, device=local)
    g.generate_ambient()
    g.initialize()
    for _ in range(warmup):
        g.mainLoopEM(1)
    stream = torch.cuda.ExternalStream(g.stream_ptr(), device=torch.device("cuda", local))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    psteps, ph = 0, np.zeros(8)
    torch.cuda.synchronize(local)
    e0.record(stream)
    for _ in range(steps):
        g.mainLoopEM(1)
        st = g.stats()
        psteps += total_particles(st, cfg.params.nspecies)
        ph += np.array(st.ms_phase[:8])
    e1.record(stream)
    torch.cuda.synchronize(local)
    ms = e0.elapsed_time(e1)
    ph /= steps
    hbm, _ = peaks()
    _, n = g.field_shape(32)                                  # ex: one shorter than the grid along x
    interior = (n[0] - 1) * (n[1] - 2) * (n[2] - 2)          # the updates' index range [lo+1, up-1)^3
    npart = psteps / steps
    gbs = lambda b, t: b / (t * 1e-3) / 1e9
    out = {"workload": workload_desc("em128", None), "steps": steps, "warmup": warmup,
           "ms_per_step": ms / steps, "particle_steps_per_s": psteps / (ms * 1e-3), "particles": int(npart),
           "yee_grid": [n[0] + 1, n[1], n[2]],
           "phases_ms": {k: round(float(v), 4) for k, v in zip(
               ["velocity", "emit", "move_current_deposit_inject", "-", "rho_tail", "efield_fdtd", "bfield_fdtd",
                "sort"], ph)},
           "roofline": {
               "efield_fdtd": {"achieved": gbs(FDTD_BYTES_PER_INDEX * interior, ph[5]), "peak": hbm, "unit": "GB/s",
                               "frac": gbs(FDTD_BYTES_PER_INDEX * interior, ph[5]) / hbm},
               "bfield_fdtd": {"achieved": gbs(FDTD_BYTES_PER_INDEX * interior, ph[6]), "peak": hbm, "unit": "GB/s",
                               "frac": gbs(FDTD_BYTES_PER_INDEX * interior, ph[6]) / hbm},
               "kick_move_current_deposit": {"achieved": gbs(56 * npart, ph[0] + ph[2]), "peak": hbm, "unit": "GB/s",
                                             "frac": gbs(56 * npart, ph[0] + ph[2]) / hbm}}}
    g.close()
    return out


def reference_cmatrix(cfg):
    """Capacity matrix for the CPU arms, as the reference's use_existing_capacity_matrix
    would load it: the exact sine-basis build of the oracle (host only, untimed)."""
    if not cfg.objects:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    return orc.dirichlet_capacity_matrix(cfg.params, cfg.objects[0].nodes)


def run_oracle(cfg, Cm, threads: int, steps: int, warmup: int = 0, budget_s: float = float("inf")):
    """The oracle (FP64 CPU restatement of the reference path, reference PSOR with
    its 1000-sweep cap) on the same workload, capacity matrix preloaded: `warmup`
    untimed steps, then up to `steps` timed steps, stopping early once the timed
    steps pass `budget_s` seconds. Returns (particle-steps/s, seconds, particles,
    PSOR sweeps of the last solve, steps timed)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    orc.lib().orc_set_threads(threads)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(0, max_post_loop=1000)
    if Cm is not None:
        o.set_cmatrix(0, Cm)
    o.generate_ambient()
    o.initialize()
    if warmup > 0:
        o.main_loop(warmup)
    n = sum(o.L.orc_num_particles(o.h, s) for s in range(cfg.params.nspecies))
    done, dt = 0, 0.0
    while done < steps and dt < budget_s:
        t0 = time.perf_counter()
        o.main_loop(1)
        dt += time.perf_counter() - t0
        done += 1
    it, _ = o.solver_stats()
    o.close()
    return n * done / dt, dt, n, it, done


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fopis", choices=["fopis", "reference"])
    ap.add_argument("--workload", default="cube128")
    ap.add_argument("--ppc", type=int, default=None, help="particles per cell per species (workload default)")
    ap.add_argument("--sort-interval", type=int, default=8)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="mixed: FP32 split-precision particles (the headline); fp64: FP64 particles and deposit")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu", dest="cpu", action="store_false")
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--ref-budget-s", type=float, default=180.0,
                    help="--impl reference: stop the timed CPU steps once they pass this many seconds")
    ap.add_argument("--profile", action="store_true", help="cudaProfilerStart/Stop around the timed steps")
    ap.add_argument("--phases", action="store_true", help="report the phase times of every timed step")
    ap.add_argument("--learned-train", type=int, default=2000,
                    help="online training steps before the learned-guess comparison (0: skip it); "
                         "2000 as in the learned-guess configuration")
    ap.add_argument("--learned-lr", type=float, default=1e-3)
    ap.add_argument("--mixed-vs-fp64", type=int, default=100,
                    help="steps of the mixed-precision run against the FP64 GPU mode on the same seed (0: skip)")
    ap.add_argument("--no-em128", dest="em128", action="store_false",
                    help="skip the EM-solver block (em128 workload)")
    ap.add_argument("--no-craft256", dest="craft256", action="store_false",
                    help="skip the 256^3 spacecraft block")
    ap.add_argument("--guess", default="history", choices=["warm", "history"],
                    help="Poisson start of the timed run: the reference's warm start or the per-solve history")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    threads = os.cpu_count() or 1
    hbm, peak_kind = peaks()
    base = {"metric": "particle-steps/s", "unit": "particle-steps/s", "n_gpus": world, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic (Philox-seeded Maxwellian plasma)",
            "dtype": ("fp32 particles, int64 fixed-point rho, fp32 smoother in fp64 refinement" if args.precision == "mixed"
                      else "fp64 particles, fp64 deposit, fp32 smoother in fp64 refinement"),
            # the same dict on both arms: what is run, not how each arm runs it
            "config": {"workload": workload_desc(args.workload, args.ppc),
                       "parallelism": f"replicas x{world}", "sort_interval": args.sort_interval}}
    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as orc
        from fopis_b200 import config
        # bodies parsed by the oracle's own .obj loader: nothing of libfopis_gpu.so
        # is loaded on this arm
        cfg = config.workload(args.workload, ppc=args.ppc, seed=20251203, obj_parser=orc.parse_obj)
        # untimed setup: the capacity matrix the reference would load from its
        # cache, computed exactly on the host (six Dirichlet faces)
        try:
            Cm = reference_cmatrix(cfg)
        except NotImplementedError as e:
            print(json.dumps({"impl": "reference", "unavailable": f"capacity matrix of this body: {e}"}))
            return
        warm = args.warmup
        v, dt, n, it, done = run_oracle(cfg, Cm, threads, args.steps, warm, args.ref_budget_s)
        line = dict(base, impl="reference", value=v, steps=done, warmup=warm, ms_per_step=dt * 1e3 / done, n_gpus=1)
        line["dtype"] = "fp64 particles and fields (CPU restatement of the reference path)"
        line["poisson_start"] = "the reference's PSOR continues from the previous phi"
        line["l2"] = "CPU run (no GPU caches involved)"
        line["cpu_baseline"] = {"value": v, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                                "sample": f"{done} full step(s) of the workload ({n} particles) after {warm} untimed, "
                                          f"reference PSOR ({it} sweeps last solve)"
                                          + ("" if done == args.steps else
                                             f"; stopped after {done} of {args.steps} steps at the "
                                             f"{args.ref_budget_s:.0f} s budget")}
        line["e2e"] = {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        print(json.dumps(line))
        return
    res, cfg = run_gpu(args, world, rank, local)
    value = res["psteps"] / (res["ms"] * 1e-3)
    push_bytes = PUSH_BYTES_PER_PARTICLE if args.precision == "mixed" else PUSH_BYTES_FP64
    em = args.workload == "em128"
    if em:
        push_bytes = 56.0 if args.precision == "mixed" else 2 * PUSH_BYTES_FP64
    achieved = push_bytes * res["pushed"] / (res["push_ms"] * 1e-3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "push_kernel_cube64.md"
    if prof.exists() and args.precision == "mixed" and not em:
        # DRAM bytes per particle of one push_brick_kernel launch, from the committed ncu summary
        m = re.search(r"\| dram_bytes_per_particle \| ([0-9.]+) \|", prof.read_text())
        if m:
            traffic = float(m.group(1)) * res["pushed"]
    line = dict(base, value=value, steps=args.steps, warmup=args.warmup, ms_per_step=res["ms"] / args.steps)
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                        "traffic": traffic,
                        "kernel": ("push_brick_kernel<3, true> + em_tail_kernel (velocity, move, current, deposit)" if em
                                   else "push_brick_kernel + tail push_kernel (all species)" if args.precision == "mixed"
                                   else "push_kernel<double> (all species)"),
                        "peak_kind": peak_kind,
                        "bytes_per_particle": push_bytes}
    line["clocks"] = res["clocks"]
    state_gb = res["particles"] * (28 if args.precision == "mixed" else 52) / 1e9
    line["l2"] = (f"inputs larger than L2: particle state {state_gb:.2f} GB, L2 126 MB" if state_gb > 0.126 else
                  f"particle state {state_gb:.3f} GB fits in L2 (126 MB)")
    line["poisson_start"] = {"warm": "previous phi (the reference's)",
                             "history": "per-solve history (first solve from the previous first solve, second from "
                                        "it + previous conductor response)"}[args.guess]
    line["gpu_launches"] = res["launches"]
    line["solve_mode"] = res["solve_mode"]
    line["vcycles_per_step"] = res["vcycles_per_step"]
    line["particles"] = res["particles"]
    names = (["velocity", "emit", "move_current_deposit_inject", "-", "rho_tail", "efield_fdtd", "bfield_fdtd", "sort"]
             if em else ["push", "emit", "inject", "absorb", "rho+solve1", "solve2", "efield", "sort"])
    line["phases_ms_last_step"] = dict(zip(names, [round(x, 4) for x in res["phases_last"]]))
    line["spacecraft_potential_V"] = res["potential_V"]
    line["step_ms"] = res["step_ms"]
    if args.phases:
        line["phases_all"] = res["phases_all"]
    line["setup_cmatrix_s"] = round(res["t_cmat"], 2)
    line["residual_pointwise_max"] = res["pointwise_max"]
    line["residual_note"] = ("solves stop at ||r||2/||f||2 <= 1e-8; residual_pointwise_max is the largest over the "
                             "timed solves of the reference's checkPhiResidual measure max|L phi + rho/eps0|/|rho/eps0|")
    if "e2e" in res:
        line["e2e"] = res["e2e"]
    if args.learned_train > 0 and world == 1:
        line["learned_guess"] = learned_comparison(args, rank, local, res["cmatrix"])
    if args.mixed_vs_fp64 > 0 and world == 1 and args.precision == "mixed":
        line["mixed_vs_fp64"] = mixed_vs_fp64(args, local, res["cmatrix"], args.mixed_vs_fp64)
    if args.craft256 and world == 1 and args.workload != "craft256":
        line["craft256"] = craft256_block(args, local)
    if args.em128 and world == 1 and args.workload != "em128":
        line["em128"] = em128_block(args, local)
    if rank == 0 and res["cmatrix"] is not None:
        try:
            Cx = reference_cmatrix(cfg)
            line["cmatrix_rel_err_vs_exact"] = float(np.abs(res["cmatrix"] - Cx).max() / np.abs(Cx).max())
        except NotImplementedError as e:      # surface too irregular for the exact pair table
            line["cmatrix_rel_err_vs_exact"] = None
            line["cmatrix_exact_unavailable"] = str(e)
    if rank == 0 and world == 1 and args.cpu:
        try:
            Cref = reference_cmatrix(cfg)
        except NotImplementedError:
            Cref = res["cmatrix"]       # irregular body: the GPU-built matrix, checked against solves in the tests
        v, dt, n, it, _ = run_oracle(cfg, Cref, os.cpu_count() or 1, args.cpu_steps)
        line["cpu_baseline"] = {"value": v, "unit": "particle-steps/s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"{args.cpu_steps} full step(s) of the same workload ({n} particles) on the "
                                          f"oracle: FP64 AoS, OpenMP, reference PSOR ({it} sweeps last solve)",
                                "seconds": dt}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
