"""Benchmark of the explicit-dynamics hot path on B200.

Workload (one "step" = one central-difference step over the whole mesh): the
neo-Hookean Tet4 shear workload, 70^3 hexes split into 2,058,000 tets (357,911
nodes), interior jitter +-0.2h, 1000 steps at dt = 0.5 x the stable step.
Synthetic seeded inputs (numpy PCG64, seed 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--decompose]

With N > 1 (under torchrun) every rank runs its own copy of the workload (replicas,
weak scaling, no collective on the data path) unless --decompose is given: then the
mesh is one 70^3-hex z-slab per rank stacked into a 1 x 1 x N box, and every step the
interface nodes' partial forces are summed across ranks with NCCL before the nodal
update (weak scaling with the exchange the reference does with MPI).

Prints one JSON line. `value` is the mixed FP32-element / FP64-state path in
Melem-steps/s (elements x steps / device seconds), with the plain FP64 path, the
mixed-vs-FP64 errors, the adjoint/forward cost ratio (Hex8 neo-Hookean 64^3,
200 steps, checkpoints every 20), the dominant kernel's roofline, an end-to-end
figure through the public API with host buffers, and the CPU oracle timed on
this host's cores.
"""
from __future__ import annotations

import argparse
import json
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

METRIC = "Melem-steps/s, mixed vs FP64 at ≤1e-5 rel force err; adjoint/forward ratio"
UNIT = "Melem-steps/s"
WORKLOAD = "tet4_nh_shear_70"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=70, help="hexes per edge of the Tet4 workload")
    ap.add_argument("--adjoint-n", type=int, default=64)
    ap.add_argument("--box-n", type=int, default=46, help="lattice cells per unit length of the 1x1x2 box workloads")
    ap.add_argument("--hex-n", type=int, default=128, help="hexes per edge of the large Hex8 workload")
    ap.add_argument("--fbar-n", type=int, default=32, help="lattice cells per unit length of the F-bar RKPM box")
    ap.add_argument("--workload", default="tet4_nh_shear",
                    choices=["tet4_nh_shear", "hex8_nh_lognormal", "hex8_le_cube", "smoothed_tet4_box", "rkpm_box",
                             "rkpm_fbar_box", "rkpm_two_pass_box", "tet4_nh_shear_renumbered"],
                    help="workload of the headline timing (the default is the headline configuration; the others "
                         "exist to profile one kernel at a time)")
    ap.add_argument("--skip-extras", action="store_true")
    ap.add_argument("--decompose", action="store_true",
                    help="N > 1: one z-slab of the Tet4 shear mesh per rank (weak scaling) with the interface "
                         "forces summed over NCCL every step, instead of N independent replicas")
    ap.add_argument("--exchange", choices=["neighbor", "allreduce"], default="neighbor",
                    help="--decompose: interface forces sent to the neighbouring slabs (overlapped with the interior "
                         "nodes' update) or summed over all ranks")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--no-patches", action="store_true", help="per-element Tet4 kernel instead of element patches")
    a = ap.parse_args()
    if a.no_patches:
        os.environ["APERI_B200_TET4_PATCHES"] = "0"
    return a


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU): timing, set-up reductions, and the
# NCCL id for --decompose (whose per-step exchange runs inside the library)
# ---------------------------------------------------------------------------
def dist_init(n_gpus):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during a region: NVML
    polled every 10 ms from a thread (read-only queries), with one sample at entry
    and one at exit so that short regions still get a record; nvidia-smi at 200 ms
    if NVML cannot be loaded."""

    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.uuid = None
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(index).uuid)
            self.uuid = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
        except Exception:
            pass
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.lines = []
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _nvml_sample(self):
        n = self.nvml
        sm = n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self.h, n.NVML_CLOCK_SM)
        try:
            r = n.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except AttributeError:
            r = n.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        self.samples.append((float(sm), float(mx), int(r)))

    def _poll(self):
        while not self.stop.wait(0.01):
            try:
                self._nvml_sample()
            except Exception:
                return

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = (pynvml.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid
                      else pynvml.nvmlDeviceGetHandleByIndex(self.index))
            self._nvml_sample()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            ident = self.uuid or str(self.index)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={ident}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self._nvml_sample()
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        for s, m, bits in self.samples:
            sm.append(s)
            smax.append(m)
            reasons.update(name for name, b in self.BITS.items() if bits & b)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_run(torch, model, prob, steps, warmup, prec, stream, dev, world, sampler_index=None):
    """Warm-up, then `steps` timed central-difference steps (device events on the
    library's stream, max over ranks): the number reported. A second, untimed-for-the-
    headline run of the same steps records CUDA events between the kernels for the
    per-kernel breakdown (those events add small gaps, so they stay out of the first)."""
    def start():
        model.set_state(None, prob.v0)
        model.init_acceleration(prec)
        model.run(warmup, prob.dt, prec)
        torch.cuda.synchronize(dev)
        barrier(world)

    start()
    n0 = model.launch_count()
    ev0, ev1 = _events(torch)
    sampler = ClockSampler(sampler_index) if sampler_index is not None else None
    if sampler:
        sampler.__enter__()
    try:
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        model.run(steps, prob.dt, prec, t0=warmup * prob.dt)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    finally:
        if sampler:
            sampler.__exit__(None, None, None)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    launches = model.launch_count() - n0
    state = model.get_state()
    start()
    model.profile(True)
    model.run(steps, prob.dt, prec, t0=warmup * prob.dt)
    kms, kn = model.profile_read()
    model.profile(False)
    return {"ms": ms, "value": world * prob.num_elems * steps / (ms * 1e-3) / 1e6, "launches": launches,
            "state": state,
            "kernels": {"element_ms": kms[0] / max(kn[0], 1), "node_ms": kms[1] / max(kn[1], 1),
                        "exchange_ms": kms[4] / max(kn[4], 1) if kn[4] else None,
                        "element_total_ms": kms[0], "node_total_ms": kms[1]},
            "clocks": sampler.summary() if sampler else None}


def algorithmic_bytes(prob, layout, slot_bytes=12):
    """Compulsory HBM bytes per launch (every array touched once, FP64 state) of the
    element and node kernels, and apart from them the bytes this implementation's
    layout adds (`*_impl`: the node-major force slots written by the element kernel and
    read back by the node kernel, 12 B mixed / 24 B FP64 per slot, plus the node
    kernel's BC word and slot range).
    Element kernels: per node X and u read (48 B) and f written (24 B); per Gauss
    element its connectivity (4 B per element node) and 8 B per modulus field; per
    cell entry its node id and gradient (4 B + three reals) and per cell its volume.
    Node kernel (the fused central-difference update): per node u, v, f read (24 B
    each), the mass (8 B), u and v written (24 B each): 128 B."""
    N = prob.num_nodes
    S = layout["used_slots"]
    r = slot_bytes // 3
    elem = 48 * N + (24 * N if any(p.kind != "cells" for p in prob.parts) else 0)
    for p in prob.parts:
        if p.kind == "cells":
            elem += (4 + 3 * r) * int(p.cell_ptr[-1]) + 8 * p.num_elems
        else:
            elem += 4 * p.conn.size
        elem += 8 * p.num_elems * ((p.mu_field is not None) + (p.kappa_field is not None))
    rk = prob.meta.get("rk")
    if rk is not None:
        # two-pass coupling: the functions read once (index + FP64 value per entry) and
        # the physical displacement written and read once per node
        elem += 12 * int(rk[0][-1]) + 48 * N
    node = 128 * N
    return {"element": elem, "node": node,
            "element_impl": elem + slot_bytes * S - 24 * N,
            "node_impl": node + slot_bytes * S + 8 * N - 24 * N}


def profiled(workload: str, role: str, prec: str, key: str):
    """A value recorded from an ncu capture in the committed summaries under profiles/
    (lines 'traffic workload=W role=R prec=P bytes=B' for DRAM bytes read + written per
    launch, 'bound workload=W role=R prec=P bound=B' for the binding resource); None when
    no capture of that kernel on that workload is recorded."""
    tag = "traffic " if key == "bytes" else "bound "
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for line in f.read_text().splitlines():
            if not line.strip().startswith(tag):
                continue
            t = dict(kv.split("=", 1) for kv in line.split()[1:] if "=" in kv)
            if t.get("workload") == workload and t.get("role") == role and t.get("prec") == prec and key in t:
                return int(t[key]) if key == "bytes" else t[key]
    return None


def algorithmic_flop(prob):
    """Element-kernel flop per launch: about 450 per neo-Hookean Tet4 (250 linear
    elastic), 6,900 per neo-Hookean Hex8 with shape-function gradients recomputed
    from X (5,300 linear elastic), and 36 per cell entry + 250 per cell for
    smoothed/RKPM cells."""
    total = 0.0
    for p in prob.parts:
        nh = p.material.kind != "linear_elastic"
        if p.kind == "tet4":
            total += p.num_elems * (450 if nh else 250)
        elif p.kind == "hex8":
            total += p.num_elems * (6900 if nh else 5300)
        else:
            total += 36 * int(p.cell_ptr[-1]) + 250 * p.num_elems
    return total


def roofline_for(kernels, alg, peak, peak_kind, workload=None, prec="mixed", flop=None, fma=None):
    """Roofline of the kernel that takes the larger share of the step. `achieved` is its
    compulsory bytes per launch over its CUDA-event launch time, against the measured
    HBM copy bandwidth; `bound` is the resource that ncu showed binding it (from the
    committed capture of that kernel on this workload: 'issue', 'fp64_pipe', 'hbm',
    'latency'), 'hbm' where none is recorded. For element kernels `compute` gives the
    algorithmic flop rate against the measured FMA peak of the precision the kernel
    computes in (FP32 for the mixed path)."""
    dominant = "node" if kernels["node_total_ms"] >= kernels["element_total_ms"] else "element"
    ms = kernels[f"{dominant}_ms"]
    achieved = alg[dominant] / (ms * 1e-3) / 1e9
    traffic = profiled(workload, dominant, prec, "bytes") if workload else None
    out = {"bound": (profiled(workload, dominant, prec, "bound") if workload else None) or "hbm",
           "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, copy)"
           if peak_kind == "measured" else peak_kind,
           "traffic": traffic,
           "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, profiles/",
           "algorithmic_bytes_per_launch": alg[dominant],
           "implementation_bytes_per_launch": alg[f"{dominant}_impl"],
           "traffic_over_algorithmic": traffic / alg[dominant] if traffic else None,
           "ms_per_launch": ms}
    if flop and dominant == "element":
        tf = flop / (ms * 1e-3) / 1e12
        c = {"algorithmic_flop_per_launch": flop, "achieved_tflops": tf}
        key = "fp64" if prec == "fp64" else "fp32"
        if fma and fma.get(key):
            c.update({"peak_tflops": fma[key], "frac": tf / fma[key],
                      "peak_source": f"{key.upper()} FMA throughput measured in this run (am_measure_fma_peak)"})
        out["compute"] = c
    return out


def fma_peaks(stream):
    """FP32 and FP64 FMA throughput of this GPU, measured once (TFLOP/s)."""
    import ctypes as C

    from aperi_mech_b200 import capi

    lib = capi.load()
    out = {}
    for key, fp64 in (("fp32", 0), ("fp64", 1)):
        v = C.c_double(0.0)
        if lib.am_measure_fma_peak(fp64, stream.cuda_stream, C.byref(v)) == capi.AM_OK:
            out[key] = v.value / 1e12
    return out


def mixed_errors(prob, steps_total, s64, sm, f64=None, fm=None):
    """Mixed-vs-FP64 errors: the displacement after the run (relative to the FP64 one),
    the same against the part of the displacement the internal forces produced
    (u - v0 t, v0 t being the force-free drift both paths integrate in FP64), the
    acceleration at the last step, and the internal force at the FP64 displacement."""
    u64, _, a64 = s64
    um, _, am = sm
    ukin = prob.v0 * (steps_total * prob.dt)
    out = {"rel_disp_err_l2": float(np.linalg.norm(um - u64) / np.linalg.norm(u64)),
           "rel_disp_err_l2_force_part": float(np.linalg.norm(um - u64) / max(np.linalg.norm(u64 - ukin), 1e-300)),
           "rel_accel_err_l2": float(np.linalg.norm(am - a64) / max(np.linalg.norm(a64), 1e-300))}
    if f64 is not None:
        out["rel_force_err_l2"] = float(np.linalg.norm(fm - f64) / np.linalg.norm(f64))
    return out


def measure_workload(torch, prob, steps, warmup, stream, dev, world, mass=None, precs=("fp64", "mixed"), fma=None,
                     formulation=None):
    from aperi_mech_b200.model import ExplicitDynamics

    out = {"workload": prob.name, "elements": prob.num_elems, "nodes": prob.num_nodes, "steps": steps,
           "dt": prob.dt, "config": prob.meta.get("config")}
    if formulation is not None:
        out["formulation"] = list(formulation)
    peak, kind = measured_peaks()
    with ExplicitDynamics(prob.coords, prob.parts, prob.bcs, mass=mass, stream=stream.cuda_stream,
                          rk=prob.meta.get("rk"), formulation=formulation) as m:
        layout = m.layout()
        states = {}
        for prec in precs:
            r = time_run(torch, m, prob, steps, warmup, prec, stream, dev, world)
            states[prec] = r["state"]
            out[prec] = {"value": r["value"], "ms_per_step": r["ms"] / steps, "kernels": r["kernels"]}
        if "fp64" in states and "mixed" in states:
            u64 = states["fp64"][0]
            f64 = m.internal_force(u64, "fp64")
            err = mixed_errors(prob, warmup + steps, states["fp64"], states["mixed"], f64,
                               m.internal_force(u64, "mixed"))
            out["mixed_vs_fp64"] = err
            out["mixed_rel_disp_err_l2"] = err["rel_disp_err_l2"]
            out["mixed_rel_force_err_l2"] = err["rel_force_err_l2"]
        if "mixed" in precs:
            out["roofline_mixed"] = roofline_for(out["mixed"]["kernels"], algorithmic_bytes(prob, layout), peak, kind,
                                                 prob.name, "mixed", algorithmic_flop(prob), fma)
        if "fp64" in precs:
            out["roofline_fp64"] = roofline_for(out["fp64"]["kernels"], algorithmic_bytes(prob, layout, 24), peak, kind,
                                                prob.name, "fp64", algorithmic_flop(prob), fma)
    return out


def run_adjoint(torch, pa, ckpt, stream, dev):
    from aperi_mech_b200.model import ExplicitDynamics

    with ExplicitDynamics(pa.coords, pa.parts, pa.bcs, stream=stream.cuda_stream) as ma:
        times = {}
        # rep 0 warms up (the adjoint allocates its checkpoint buffers), rep 1 is timed,
        # rep 2 records the per-kernel breakdown (its events between kernels slow it down)
        for rep in range(3):
            ma.set_state(None, pa.v0)
            torch.cuda.synchronize(dev)
            a0, a1 = _events(torch)
            a0.record(stream)
            ma.init_acceleration()
            ma.run(pa.nsteps, pa.dt)
            a1.record(stream)
            torch.cuda.synchronize(dev)
            if rep == 1:
                times["forward"] = a0.elapsed_time(a1)
            ma.set_state(None, pa.v0)
            torch.cuda.synchronize(dev)
            ma.profile(rep == 2)
            a0.record(stream)
            loss, gm, gk = ma.adjoint(pa.nsteps, pa.dt, ckpt, pa.meta["sensors"])
            a1.record(stream)
            torch.cuda.synchronize(dev)
            if rep == 1:
                times["adjoint"] = a0.elapsed_time(a1)
        pms, pn = ma.profile_read()
        ma.profile(False)
    return {"workload": pa.name, "elements": pa.num_elems, "steps": pa.nsteps, "ckpt_every": ckpt,
            "forward_ms": times["forward"], "adjoint_ms": times["adjoint"], "ratio": times["adjoint"] / times["forward"],
            "loss": loss, "grad_mu_norm": float(np.linalg.norm(gm)), "grad_kappa_norm": float(np.linalg.norm(gk)),
            "kernel_ms": {"element": pms[0], "node": pms[1], "vjp": pms[2], "adjoint_node": pms[3]},
            "kernel_launches": {"element": pn[0], "node": pn[1], "vjp": pn[2], "adjoint_node": pn[3]}}


def decomposed_setup(args, prob, rank, world, dev):
    """Global mass and stable step of the slab decomposition (interface rows of the slab
    masses summed, dt the minimum over ranks), then the exchange and its communicator."""
    import torch

    mass = prob.meta["slab_mass"].copy()
    rows = torch.from_numpy(prob.meta["iface_rows"].astype(np.int64)).to(dev)
    loc = prob.meta["iface_local"]
    if world > 1:
        import torch.distributed as dist

        buf = torch.zeros(prob.meta["num_iface"], dtype=torch.float64, device=dev)
        buf[rows] = torch.from_numpy(mass[loc]).to(dev)
        dist.all_reduce(buf)
        mass[loc] = buf[rows].cpu().numpy()
        dt = torch.tensor([prob.dt], dtype=torch.float64, device=dev)
        dist.all_reduce(dt, op=dist.ReduceOp.MIN)
        prob.dt = float(dt.item())
    return mass


def attach_interface(model, prob, rank, world, exchange="neighbor"):
    """The slab's interface: a neighbour exchange with the slabs above and below (the
    default), or the all-rank sum of every interface row."""
    from aperi_mech_b200.model import nccl_unique_id

    if exchange == "neighbor" and world > 1:
        model.set_neighbors(rank, prob.meta["neighbors"], prob.meta["shared_ptr"], prob.meta["shared_nodes"])
    else:
        model.set_interface(prob.meta["iface_local"], prob.meta["iface_rows"], prob.meta["num_iface"])
    if world > 1:
        import torch.distributed as dist

        box = [nccl_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(box, src=0)
        model.set_nccl(box[0], rank, world)


def make_problem(args, rank=0, world=1):
    from aperi_mech_b200 import problems

    if args.decompose:
        return problems.tet4_nh_shear_slab(n=args.n, rank=rank, world=world, seed=0, nsteps=args.steps)
    w = args.workload
    if w == "tet4_nh_shear":
        return problems.tet4_nh_shear(n=args.n, seed=0, nsteps=args.steps)
    if w == "hex8_nh_lognormal":
        return problems.hex8_nh_lognormal(n=args.hex_n, seed=0, nsteps=args.steps, bulk_field=True)
    if w == "hex8_le_cube":
        return problems.hex8_le_cube(n=20, seed=0, nsteps=args.steps)
    if w == "smoothed_tet4_box":
        return problems.smoothed_tet4_box(n=args.box_n, seed=0, nsteps=args.steps)
    if w == "rkpm_fbar_box":
        return problems.rkpm_fbar_box(n=args.fbar_n, seed=0, nsteps=args.steps)
    if w == "rkpm_two_pass_box":
        return problems.rkpm_two_pass_box(n=args.box_n, seed=0, nsteps=args.steps)
    if w == "tet4_nh_shear_renumbered":
        return problems.renumbered(problems.tet4_nh_shear(n=args.n, seed=0, nsteps=args.steps), seed=1)[0]
    return problems.rkpm_box(n=args.box_n, seed=0, nsteps=args.steps)


def run_ours(args, rank, world, local):
    import torch

    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    dev = torch.device("cuda", local)
    prob = make_problem(args, rank, world)
    E, N = prob.num_elems, prob.num_nodes
    stream = torch.cuda.Stream(device=dev)
    res = {}
    mass = decomposed_setup(args, prob, rank, world, dev) if args.decompose else prob.meta.get("mass")
    model = ExplicitDynamics(prob.coords, prob.parts, prob.bcs, mass=mass, stream=stream.cuda_stream,
                             rk=prob.meta.get("rk"))
    if args.decompose:
        attach_interface(model, prob, rank, world, args.exchange)
    layout = model.layout()
    hbm_peak, peak_kind = measured_peaks()
    fma = fma_peaks(stream)
    for prec in ("fp64", "mixed"):
        res[prec] = time_run(torch, model, prob, args.steps, args.warmup, prec, stream, dev, world,
                             sampler_index=local if prec == "mixed" else None)
    # accuracy of the mixed path against the FP64 path (itself 1e-12 from the oracle)
    u64 = res["fp64"]["state"][0]
    errors = mixed_errors(prob, args.warmup + args.steps, res["fp64"]["state"], res["mixed"]["state"],
                          model.internal_force(u64, "fp64"), model.internal_force(u64, "mixed"))

    # end to end through the public API: pinned host state in, K steps, host state out
    e2e = None
    if not args.skip_e2e:
        u_h = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
        v_h = torch.from_numpy(prob.v0.copy()).pin_memory()
        out_u = torch.empty((N, 3), dtype=torch.float64).pin_memory()
        out_v = torch.empty((N, 3), dtype=torch.float64).pin_memory()
        torch.cuda.synchronize(dev)
        barrier(world)
        t0 = time.perf_counter()
        ev0, ev1 = _events(torch)
        ev0.record(stream)
        model.set_state(u_h.numpy(), v_h.numpy())
        model.init_acceleration("mixed")
        model.run(args.steps, prob.dt, "mixed")
        model.lib.am_get_state(model.ctx, 0, out_u.data_ptr(), out_v.data_ptr(), None)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        ms_e2e = max_over_ranks(max(ev0.elapsed_time(ev1), wall * 1e3), world)
        e2e = {"value": world * E * args.steps / (ms_e2e * 1e-3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": 2 * N * 3 * 8 / args.steps, "d2h_bytes_per_step": 2 * N * 3 * 8 / args.steps,
               "ms": ms_e2e, "path": "ExplicitDynamics.set_state/init_acceleration/run/get_state (C ABI, host buffers)"}
    model.close()

    roofline = roofline_for(res["mixed"]["kernels"], algorithmic_bytes(prob, layout), hbm_peak, peak_kind,
                            prob.name, "mixed", algorithmic_flop(prob), fma)
    roofline["layout"] = layout
    roofline_fp64 = roofline_for(res["fp64"]["kernels"], algorithmic_bytes(prob, layout, 24), hbm_peak, peak_kind,
                                 prob.name, "fp64", algorithmic_flop(prob), fma)
    # the CPU oracle on the same mesh (rank 0 at N = 1), while the problem is at hand
    cpu = None if (args.skip_cpu or rank != 0 or world != 1) else cpu_baseline(prob)

    # the other configurations, each on its own context
    extras = {}
    if args.decompose:
        args.skip_extras = args.skip_adjoint = True  # the adjoint is single-domain
    if not args.skip_extras:
        p1 = problems.hex8_le_cube(n=20, seed=0, nsteps=100)
        extras["hex8_le_cube_20"] = measure_workload(torch, p1, 100, args.warmup, stream, dev, world, fma=fma)
        p3a = problems.smoothed_tet4_box(n=args.box_n, seed=0, nsteps=500)
        extras["smoothed_tet4_box"] = measure_workload(torch, p3a, 500, args.warmup, stream, dev, world,
                                                       mass=p3a.meta["mass"], fma=fma)
        t0 = time.perf_counter()
        p3b = problems.rkpm_box(n=args.box_n, seed=0, nsteps=500)
        setup_s = time.perf_counter() - t0
        r = measure_workload(torch, p3b, 500, args.warmup, stream, dev, world, mass=p3b.meta["mass"], fma=fma)
        r["setup_s"] = setup_s
        r["entries_per_cell"] = p3b.meta["entries_per_cell"]
        extras["rkpm_box"] = r
        t0 = time.perf_counter()
        p3c = problems.rkpm_fbar_box(n=args.fbar_n, seed=0, nsteps=200)
        setup_s = time.perf_counter() - t0
        r = measure_workload(torch, p3c, 200, args.warmup, stream, dev, world, mass=p3c.meta["mass"], fma=fma)
        r["setup_s"] = setup_s
        r["entries_per_subcell"] = p3c.meta["entries_per_cell"]
        extras["rkpm_fbar_box"] = r
        t0 = time.perf_counter()
        p3d = problems.rkpm_two_pass_box(n=args.box_n, seed=0, nsteps=500)
        setup_s = time.perf_counter() - t0
        r = measure_workload(torch, p3d, 500, args.warmup, stream, dev, world, mass=p3d.meta["mass"], fma=fma)
        r["setup_s"] = setup_s
        extras["rkpm_two_pass_box"] = r
        # The headline mesh renumbered at random (an unstructured mesh's numbering): with the
        # split-hex rings found by topology, with generic patches only, and one thread per tet.
        pr, _, _ = problems.renumbered(problems.tet4_nh_shear(n=args.n, seed=0, nsteps=args.steps), seed=1)
        for label, patches in (("split_hex", None), ("generic_patches", "1"), ("per_tet", "0")):
            old_env = os.environ.get("APERI_B200_TET4_PATCHES")
            if patches is not None:
                os.environ["APERI_B200_TET4_PATCHES"] = patches
            try:
                r = measure_workload(torch, pr, args.steps, args.warmup, stream, dev, world, fma=fma)
            finally:
                if old_env is None:
                    os.environ.pop("APERI_B200_TET4_PATCHES", None)
                else:
                    os.environ["APERI_B200_TET4_PATCHES"] = old_env
            r["kernel_path"] = label
            r["vs_structured_mixed"] = r["mixed"]["value"] / res["mixed"]["value"]
            r["vs_structured_fp64"] = r["fp64"]["value"] / res["fp64"]["value"]
            extras[f"tet4_nh_shear_renumbered_{label}"] = r
        # The updated and semi-Lagrangian formulations (FP64) on the headline mesh: the current
        # (or last reference) coordinates, the displacement increment and the element H on the
        # device, the reference update every 10 steps (semi) or every step (updated).
        pl = problems.tet4_nh_shear(n=args.n, seed=0, nsteps=200)
        for label, form in (("semi_10", ("semi", 10)), ("updated", ("updated", 1))):
            extras[f"tet4_nh_shear_{label}"] = measure_workload(torch, pl, 200, args.warmup, stream, dev, world,
                                                              precs=("fp64",), fma=fma, formulation=form)
        p5 = problems.hex8_nh_lognormal(n=args.hex_n, seed=0, nsteps=1000, bulk_field=True)
        extras["hex8_nh_lognormal_large"] = measure_workload(torch, p5, 1000, args.warmup, stream, dev, world, fma=fma)
        if not args.skip_adjoint:
            extras["hex8_nh_lognormal_large"]["adjoint"] = run_adjoint(torch, p5, 50, stream, dev)

    adj = None
    if not args.skip_adjoint:
        adj = run_adjoint(torch, problems.hex8_nh_lognormal(n=args.adjoint_n, seed=0, nsteps=200), 20, stream, dev)
    kernel_ms = {p: res[p]["kernels"] for p in ("fp64", "mixed")}
    launches = {p: res[p]["launches"] for p in ("fp64", "mixed")}
    return (prob, res, errors, e2e, adj, roofline, roofline_fp64, kernel_ms, launches,
            res["mixed"]["clocks"], extras, cpu, fma)


def workload_config(prob, world, decompose):
    """The `config` of the JSON line, the same for both arms on the same workload."""
    return {"workload": prob.name, "elements": prob.num_elems, "nodes": prob.num_nodes,
            "description": prob.meta.get("config"), "material": "neo-Hookean mu=3.85e8 kappa=8.33e8"
            if "nh" in prob.name or "box" in prob.name else "linear elastic E=1e9 nu=0.3",
            "dt": prob.dt, "seed": prob.seed,
            "l2_flush": "inputs larger than L2 (state + slots + connectivity ~ 230 MB per step)",
            "parallelism": (f"z-slab domain decomposition x{world}, interface forces summed over NCCL "
                            f"({prob.meta['num_iface']} interface nodes)" if decompose else
                            f"replicas x{world}" if world > 1 else "single GPU")}


def cpu_baseline(prob, target_s=10.0):
    """The oracle (C++ FP64 restatement, all host threads) on the benchmark's own mesh:
    central-difference steps from the same initial state, as many as take about
    target_s seconds (a two-step probe sizes the sample)."""
    from oracle import oracle

    op = oracle.OracleProblem.from_problem(prob)
    u = np.zeros_like(prob.coords)
    a = op.init_acceleration(u)
    t0 = time.perf_counter()
    op.steps(u, prob.v0, a, np.full(2, prob.dt))
    t1 = (time.perf_counter() - t0) / 2
    steps = max(2, int(target_s / max(t1, 1e-6)))
    t0 = time.perf_counter()
    op.steps(u, prob.v0, a, np.full(steps, prob.dt))
    dt = time.perf_counter() - t0
    return {"value": prob.num_elems * steps / dt / 1e6, "unit": UNIT, "cores": oracle.get_threads(), "kind": "port",
            "sample": f"{prob.name} ({prob.num_elems} tets, the benchmark mesh), {steps} of its central-difference "
                      f"steps, FP64, {oracle.get_threads()} OpenMP threads; the reference CPU build is unavailable "
                      f"(Kokkos/Trilinos/Eigen/MPI missing), so the oracle restatement stands in for it"}


def run_reference(args, rank, world):
    """Reference arm: the reference's CPU implementation cannot be built here (Kokkos,
    Trilinos/STK, Eigen, yaml-cpp, MPI absent), so its CPU restatement (the oracle, FP64,
    all host threads) runs the benchmark's own workload: the same seeded mesh, initial
    state and dt, `warmup` untimed and `steps` timed central-difference steps. The
    problem is built without the CUDA library (the oracle completes the material
    properties), so this process loads only the oracle."""
    if rank != 0:
        return
    from aperi_mech_b200 import problems
    from oracle import oracle

    p = problems.tet4_nh_shear(n=args.n, seed=0, nsteps=args.steps, complete=oracle.complete_properties)
    op = oracle.OracleProblem.from_problem(p)
    u = np.zeros_like(p.coords)
    a = op.init_acceleration(u)
    u, v, a = op.steps(u, p.v0, a, np.full(args.warmup, p.dt))
    t0 = time.perf_counter()
    op.steps(u, v, a, np.full(args.steps, p.dt), t0=args.warmup * p.dt)
    dt = time.perf_counter() - t0
    value = p.num_elems * args.steps / dt / 1e6
    sample = (f"{p.name} ({p.num_elems} tets, the benchmark workload itself), {args.steps} timed FP64 "
              f"central-difference steps after {args.warmup} untimed; oracle restatement of the reference's CPU "
              f"path (reference CPU build unavailable: missing Kokkos/Trilinos/Eigen/MPI)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(p, world, False),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": oracle.get_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_init(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    (prob, res, errors, e2e, adj, roofline, roofline_fp64, kernel_ms, launches, clocks,
     extras, cpu, fma) = run_ours(args, rank, world, local)
    if rank != 0:
        return
    ms_step = res["mixed"]["ms"] / args.steps
    line = {
        "metric": METRIC, "value": res["mixed"]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": workload_config(prob, world, args.decompose),
        "value_fp64": res["fp64"]["value"],
        "fp64": {"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms"] / args.steps,
                 "note": "the plain FP64 path, the reference's precision"},
        "mixed_vs_fp64": dict(errors, speedup=res["mixed"]["value"] / res["fp64"]["value"]),
        "fma_peak_tflops": fma,
        "adjoint": adj,
        "roofline": roofline,
        "roofline_fp64": roofline_fp64,
        "kernels_ms_per_launch": kernel_ms,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches["mixed"],
        "clocks": clocks,
        "other_workloads": extras,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
