"""Benchmark: RBE + LJ/Coulomb atom-steps/s on the 200k-atom LJ electrolyte.

A step is one NVE velocity-Verlet MD step (NVEensemble::Solve): half kick,
drift with periodic wrap and skin check, neighbor rebuild when needed, the RBL
real-space force (hashed shell batch, r_core 2.5, cut_off 5, skin 0.3), RBE
k-space with P = 100 Philox-sampled k-vectors, and the second half kick.

value      mixed form (fixed-point positions, FP32 SFU phases, FP64 reductions
           and integrator), state resident on the GPU; each step is one launch
           of the engine's CUDA graph (rebuild under a conditional node).
fp64_plain the plain FP64 form of the same step on the same GPU.
phase_ms   from separate profiled runs (launch by launch, events between
           phases), so they sum to slightly more than ms_per_step.
e2e        mixed form through rbx_engine_step_host: host x, v in (pinned), one
           step, x, v, F out, every step.
roofline   the fused RBL filter + pair-force kernel against measured HBM
           bandwidth; its algorithmic bytes per launch are the candidate
           indices read (4 B each) plus 44 B of per-atom traffic (count,
           atom record, type, two hash keys, force out).  roofline.issue: the
           same launch against the SM issue limit (warp instructions per launch
           from an ncu count per candidate), the bound that holds it.
cpu_baseline  the FP64 host oracle (same step, OpenMP over all host cores).
parity_vs_oracle  both forms against the FP64 oracle at the same size: force,
           pair and k-space force errors, k-space energy and virial, pair
           energies and virial, RBL pair sets (one force evaluation each).
configs    (one GPU) the 200k electrolyte at P = 400 and the 4,000-atom
           electrolyte for 1,000 steps, both forms.
reference_gpu  (one GPU) RBMD's own kernels compiled for sm_100a (FP32 as
           shipped, and FP64) against this library's force path, N = 200,192.

--impl reference runs the reference path on the host: RBMD's hot-path kernels
exist only as CUDA, so the reference arm is the FP64 host restatement of the
same RBE + RBL step (the oracle), timed on this box's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RBE+LJ atom-steps/s @200k atoms: mixed vs FP64 plain at <=1e-5 rel force err"
UNIT = "atom-steps/s"
# DRAM bytes (read + written) per atom of one mixed k_rbl_fused launch, from an ncu
# capture of the same workload at N = 100,000 (215.1 MB per launch: the split candidate
# rows streamed once, plus neighbour-record and key gathers that miss L2).  Rows and
# gathers grow with N, so the traffic is scaled by N.
RBL_TRAFFIC_BYTES_PER_ATOM = 2151.0
# Warp instructions per 32 candidates of the same launch (186.7 M for 47.9 M candidates in
# the N = 100,000 capture), and the SM issue limit they are compared with: one warp
# instruction per cycle per SM sub-partition, four per SM.
RBL_WARP_INSTR_PER_32_CAND = 124.7
ISSUE_SLOTS_PER_SM_CYCLE = 4


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    every 2 ms (read-only queries), else nvidia-smi every 200 ms."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, cuda_device=0):
        self.dev = cuda_device
        self.sm, self.sm_max, self.reasons = [], [], set()
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _nvml_handle(self):
        import pynvml as N
        import torch

        N.nvmlInit()
        pr = torch.cuda.get_device_properties(self.dev)
        try:
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return N, N.nvmlDeviceGetHandleByPciBusId_v2(bus)
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.dev)

    def _run(self):
        try:
            N, h = self._nvml_handle()
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            while not self._stop.is_set():
                self.sm.append(float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)))
                self.sm_max.append(float(mx))
                bits = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, attr in self.REASONS:
                    if bits & getattr(N, attr):
                        self.reasons.add(name)
                self._stop.wait(0.002)
            return
        except Exception:
            pass
        while not self._stop.is_set():  # fallback: nvidia-smi
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.dev}",
                                      f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                r = [c.strip() for c in out.split(",")]
                if len(r) >= 9:
                    self.sm.append(float(r[1]))
                    self.sm_max.append(float(r[2]))
                    for k, (name, _) in enumerate(self.REASONS):
                        if r[5 + k].lower() == "active":
                            self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": max(self.sm_max),
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return ws, rank


def _init_pg(ws, backend):
    import datetime

    import torch.distributed as dist

    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return dist


def max_over_ranks(value, ws, device):
    """The largest of every rank's `value` (each rank passes its own), through
    an all-reduce on `device` ("cuda" with NCCL, "cpu" with gloo)."""
    if ws <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(ws, n, steps, ms):
    """Whole-job atom-steps/s: every rank advances its own n-atom replica
    `steps` times; `ms` is the slowest rank's device time."""
    return ws * n * steps / (ms / 1e3)


def cpu_baseline(n, p, steps, warmup):
    from oracle import oracle as O
    from rbmd_b200 import systems

    s = systems.lj_electrolyte(n, seed=2024, kspace_p=p)
    eng = O.Engine(s, seed=99)
    eng.compute_forces(0)
    eng.step(warmup)
    t0 = time.perf_counter()
    eng.step(steps)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"N={n} LJ electrolyte, P={p}, {steps} velocity-Verlet steps after "
                      f"{warmup} warm-up (FP64 host restatement, OpenMP)"}


def parity_vs_oracle(s, p, local):
    """Both forms against the FP64 oracle at the bench's own size: one force
    evaluation each on the same positions, k-samples and batch epoch.  Force
    errors are relative 3-vector RMS; the k-space energy relative to its
    sampled sum before the self term (the two nearly cancel); virials relative
    to their largest component; RBL pair sets compared exactly."""
    from oracle import oracle as O
    from rbmd_b200 import rbx, systems

    m = O.rbe_sample_philox(O.Box.make(s["lo"], s["hi"]), s["params"]["alpha"], p, 5, 0)
    t0 = time.perf_counter()
    want = O.rbl_rbe_evaluation(s, m, epoch=0)
    t_oracle = time.perf_counter() - t0
    out = {"oracle_s": t_oracle}
    parts = {}
    for name, prec in (("fp64_plain", rbx.PLAIN_FP64), ("mixed", rbx.MIXED)):
        e = rbx.Engine(s, precision=prec, device=local)
        e.set_k_samples(*m)
        e.compute_forces(0)
        fp, fk = e.force_parts()
        st = e.stats()
        el, ec, vp = e.pair_energy()
        gc, gs = e.rbl_pairs()
        vk = np.asarray(st.virial_kspace[:], float)
        out[name] = {
            "force": systems.rel_rms(fp + fk, want["force"]),
            "pair": systems.rel_rms(fp, want["f_pair"]),
            "kspace": systems.rel_rms(fk, want["f_kspace"]),
            "energy_kspace": abs(st.e_kspace - want["e_kspace"]) / want["e_kspace_scale"],
            "virial_kspace": float(np.abs(vk - want["virial_kspace"]).max() /
                                   np.abs(want["virial_kspace"]).max()),
            "energy_vdwl": abs(el - want["e_vdwl"]) / abs(want["e_vdwl"]),
            "energy_coul": abs(ec - want["e_coul"]) / abs(want["e_coul"]),
            "virial_pair": float(np.abs(vp - want["virial_pair"]).max() /
                                 np.abs(want["virial_pair"]).max()),
            "rbl_pairs_equal": bool(np.array_equal(O.pair_keys(gc), want["core_keys"]) and
                                    np.array_equal(O.pair_keys(gs), want["shell_keys"])),
        }
        parts[name] = (fp + fk, fp, fk, st.e_kspace)
        e.close()
    a, b = parts["mixed"], parts["fp64_plain"]
    out["mixed_vs_fp64"] = {"force": systems.rel_rms(a[0], b[0]),
                            "pair": systems.rel_rms(a[1], b[1]),
                            "kspace": systems.rel_rms(a[2], b[2])}
    return out


def reference_gpu(local):
    """RBMD's own hot-path kernels on this GPU (the .hip.cu sources compiled in
    place for sm_100a into oracle/_ref: FP32 as shipped and FP64), timed beside
    this library at N = 200,192 (a multiple of 256: ComputeRBEForce has
    __syncthreads inside a branch on i < N).  The reference's force path with a
    reused candidate list (lj_cut_coul_kspace.cpp:494-573,
    kspace_calculator.cpp:532-588): FilterRblNeighborCandidatesOp,
    LJCutCoulRBLForceOp, FixRBLForceOp, ComputePnumberChargeStructureFactorOp,
    ComputeRBEForceOp, each the median of 20 CUDA-event timings; its host
    k-sampling and its three host reductions before FixRBLForceOp are not
    timed.  This library's force path is the real-space plus k-space phases of
    its profiled step at the same N."""
    import ctypes as C

    import torch

    from oracle import oracle as O
    from rbmd_b200 import rbx, systems

    libs = {}
    for tag, fname, real in (("f32", "libref32.so", 4), ("f64", "libref64.so", 8)):
        path = os.path.join(ROOT, "oracle", "_ref", fname)
        if not os.path.exists(path):
            return {"unavailable": f"{path} not built (oracle/ref_harness needs the RBMD sources)"}
        lib = C.CDLL(path)
        if lib.ref_real_size() != real:
            return {"unavailable": f"{fname} has the wrong real size"}
        libs[tag] = lib
    n = 200192
    s = systems.lj_electrolyte(n, seed=2024)
    box = O.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = O.cells_sort(box, 5.3, x, y, z)
    srt = dict(s, pos=s["pos"][perm], q=s["q"][perm], type=s["type"][perm], gid=s["gid"][perm])
    cnt, rows = O.full_list(box, 5.3, x[perm], y[perm], z[perm], cell, cs, ce)

    def median_ms(fn, reps=20):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            ev[0].record()
            fn()
            ev[1].record()
            torch.cuda.synchronize()
            ts.append(ev[0].elapsed_time(ev[1]))
        return float(np.median(ts))

    def ref_path(lib, real):
        dt = torch.float64 if real == 8 else torch.float32
        pk = srt["params"]["kspace_p"]
        lo = (C.c_double * 3)(*srt["lo"])
        hi = (C.c_double * 3)(*srt["hi"])

        def T(a, dtype=None):
            return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype or dt)

        def P(t):
            return C.c_void_p(t.data_ptr())

        i32 = torch.int32
        alpha, qqr2e = srt["params"]["alpha"], srt["params"]["qqr2e"]
        S = O.rbe_gauss_sum(box, alpha)
        mx, my, mz = (T(v) for v in O.rbe_sample_philox(box, alpha, pk, 5, 0))
        px, py, pz = (T(srt["pos"][:, d]) for d in range(3))
        q, typ, gid = T(srt["q"]), T(srt["type"], i32), T(srt["gid"], i32)
        sigma, eps = T(srt["sigma"]), T(srt["eps"])
        cap = rows.shape[1]
        cstart = T(np.arange(n) * cap, i32)
        cend = T(np.arange(n) * cap + cnt, i32)
        cand, capv = T(rows.reshape(-1), i32), T(np.full(n, cap), i32)
        core_end = T(np.zeros(n), i32)
        core, shell = T(np.full(n * cap, -1), i32), T(np.full(n * cap, -1), i32)
        snum, req, realloc = (T(np.zeros(k), i32) for k in (n, 1, 1))
        re, im = T(np.zeros(pk)), T(np.zeros(pk))
        fr = [T(np.zeros(n)) for _ in range(3)]
        fk = [T(np.zeros(n)) for _ in range(3)]
        freq = O.rbl_params(n, box, 2.5, 5.0, 100)[0]
        core2, force2 = 2.5 ** 2 - 1e-4, 5.0 ** 2 - 1e-4

        def filt():
            lib.ref_rbl_filter(C.c_double(core2), C.c_double(force2), n, P(gid), P(px), P(py),
                               P(pz), P(cstart), P(cend), P(cand), P(capv), P(cstart),
                               P(core_end), P(core), cap, P(shell), P(snum), P(req), lo, hi,
                               P(realloc), freq, 0)

        def pair():
            lib.ref_pair_rbl(lo, hi, C.c_double(2.5), C.c_double(5.0), n, 100, freq,
                             C.c_double(alpha), C.c_double(qqr2e), P(typ), P(sigma), P(eps),
                             P(cstart), P(core_end), P(core), P(shell), P(snum), P(q), P(px),
                             P(py), P(pz), *[P(t) for t in fr])

        def fix():
            lib.ref_fix_rbl(n, C.c_double(0.0), C.c_double(0.0), C.c_double(0.0),
                            *[P(t) for t in fr])

        def rho():
            lib.ref_rbe_rho(lo, hi, n, pk, P(q), P(mx), P(my), P(mz), P(px), P(py), P(pz),
                            P(re), P(im))

        def force():
            lib.ref_rbe_force(lo, hi, n, pk, C.c_double(alpha), C.c_double(S),
                              C.c_double(qqr2e), P(re), P(im), P(q), P(mx), P(my), P(mz),
                              P(px), P(py), P(pz), *[P(t) for t in fk])

        filt()
        torch.cuda.synchronize()
        if int(realloc.item()) != 0:
            raise RuntimeError("reference core capacity too small")
        ms = {k: median_ms(f) for k, f in (("rbl_filter", filt), ("rbl_pair_force", pair),
                                           ("fix_rbl_force", fix), ("rbe_structure_factor", rho),
                                           ("rbe_force", force))}
        ms["force_path"] = sum(ms.values())
        return ms

    out = {"n": n, "kernels": "RBMD .hip.cu sources compiled for sm_100a (oracle/ref_harness)"}
    for tag, real in (("f32", 4), ("f64", 8)):
        out[f"reference_{tag}_ms"] = ref_path(libs[tag], real)
    for name, prec in (("ours_mixed_ms", rbx.MIXED), ("ours_fp64_ms", rbx.PLAIN_FP64)):
        e = rbx.Engine(s, precision=prec, seed=5, device=local)
        e.compute_forces(0)
        e.step(5)
        e.set_profiling(True)
        e.step(30)
        ph = e.phase_ms()
        e.close()
        out[name] = {"real_space": ph[2], "kspace": ph[3], "force_path": ph[2] + ph[3]}
    out["speedup_f32_vs_mixed"] = (out["reference_f32_ms"]["force_path"] /
                                   out["ours_mixed_ms"]["force_path"])
    out["speedup_f64_vs_fp64"] = (out["reference_f64_ms"]["force_path"] /
                                  out["ours_fp64_ms"]["force_path"])
    return out


def config_runs(local):
    """The other BASELINE configurations on the same GPU, device-timed steps of
    the engine's step graph: the 200k electrolyte at P = 400 (both forms), and
    the 4,000-atom electrolyte (P = 100) for 1,000 velocity-Verlet steps."""
    import torch

    from rbmd_b200 import rbx, systems

    def run(n, p, precision, steps, warmup):
        s = systems.lj_electrolyte(n, seed=2024, kspace_p=p)
        e = rbx.Engine(s, precision=precision, seed=77, device=local)
        e.compute_forces(0)
        e.step(warmup)
        st = torch.cuda.ExternalStream(e.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(st)
        e.step(steps)
        ev1.record(st)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        e.close()
        return {"value": n * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps}

    out = {}
    for name, n, p, steps in (("p400", 200000, 400, 50), ("n4000", 4000, 100, 1000)):
        mx = run(n, p, rbx.MIXED, steps, 5)
        f64 = run(n, p, rbx.PLAIN_FP64, steps, 5)
        out[name] = {"n": n, "p": p, "mixed": mx, "fp64_plain": f64,
                     "mixed_over_fp64": mx["value"] / f64["value"]}
    return out


def run_reference(args):
    ws, rank = _dist()
    if rank != 0:
        return 0
    base = cpu_baseline(args.n, args.p, max(1, args.steps), max(1, args.warmup))
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": args.n / base["value"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"lj_electrolyte N={args.n} rho*=0.8 RBL(r_core 2.5, cut_off 5,"
                                   f" skin 0.3) + RBE(P={args.p}, alpha=0.16)",
                       "global_batch": args.n, "parallelism": "host cores"},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    from rbmd_b200 import rbx, systems

    ws, rank = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = _init_pg(ws, "nccl")
    n, p = args.n, args.p
    s = systems.lj_electrolyte(n, seed=2024 + rank, kspace_p=p)

    # ---- parity of both forms against the FP64 oracle at this size (one force
    # evaluation each, same state, k-samples and epoch; outside any timed region)
    par = parity_vs_oracle(s, p, local) if rank == 0 and not args.no_extras else None

    def timed(precision, steps, warmup, profile=False, clk=None):
        e = rbx.Engine(s, precision=precision, seed=77 + rank, device=local)
        e.compute_forces(0)
        e.step(warmup)
        if profile:
            e.set_profiling(True)
        st = torch.cuda.ExternalStream(e.stream)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if dist and ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        if clk:
            clk.__enter__()
        l0 = rbx.launch_count()
        ev0.record(st)
        e.step(steps)
        ev1.record(st)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        launches = rbx.launch_count() - l0
        ms = ev0.elapsed_time(ev1)
        ms = max_over_ranks(ms, ws, "cuda")
        phases = e.phase_ms() if profile else None
        stats = e.stats()
        return e, ms, launches, phases, stats

    # ---- plain FP64 form (step graph), then a profiled run for its phase times
    e64, ms64, _, _, _ = timed(rbx.PLAIN_FP64, args.steps, args.warmup)
    e64.close()
    e64p, _, _, ph64, _ = timed(rbx.PLAIN_FP64, args.steps, args.warmup, profile=True)
    e64p.close()
    # ---- mixed form (headline), clocks sampled during the timed region
    clk = ClockSampler(local)
    em, ms, launches, _, stats = timed(rbx.MIXED, args.steps, args.warmup, clk=clk)
    em.close()
    # per-phase device times of the mixed step (separate profiled run)
    em2, _, _, phm, stats2 = timed(rbx.MIXED, args.steps, args.warmup, profile=True)
    em2.close()

    # ---- end to end through the host-buffer C-ABI call: each step copies x, v
    # in from pinned host memory and x, v, F back; buffers alternate so the
    # outputs of one step are the inputs of the next without a host copy
    e2 = rbx.Engine(s, precision=rbx.MIXED, seed=5, device=local)
    e2.compute_forces(0)
    bufs = [[torch.empty((3, n), dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
            for _ in range(2)]  # bufs[k] = [x, v] of parity k
    fo = torch.empty((3, n), dtype=torch.float64, pin_memory=True).numpy()
    bufs[0][0][:] = s["pos"].T
    bufs[0][1][:] = s["vel"].T
    k = 0
    for _ in range(args.warmup):
        e2.step_host(bufs[k][0], bufs[k][1], bufs[1 - k][0], bufs[1 - k][1], fo)
        k = 1 - k
    st2 = torch.cuda.ExternalStream(e2.stream)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist and ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(st2)
    for _ in range(args.steps):
        e2.step_host(bufs[k][0], bufs[k][1], bufs[1 - k][0], bufs[1 - k][1], fo)
        k = 1 - k
    ev1.record(st2)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1), ws, "cuda")
    e2.close()

    if rank != 0:
        if dist and ws > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    value = job_throughput(ws, n, args.steps, ms)
    v64 = job_throughput(ws, n, args.steps, ms64)
    peaks, peak_src = _peaks()
    # roofline of the fused RBL kernel (phase 2 of the profiled mixed step)
    cand_per_atom = stats2.candidates / n
    alg_bytes = n * (4.0 * cand_per_atom + 44.0)
    t_pair = phm[2] / 1e3
    achieved = alg_bytes / t_pair / 1e9
    roof = {"kernel": "k_rbl_fused_mixed", "bound": "hbm", "achieved": achieved,
            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
            "peak_source": peak_src, "traffic": RBL_TRAFFIC_BYTES_PER_ATOM * n,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at N=100000, "
                              "scaled by N",
            "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": phm[2]}
    # the bound that holds the kernel: instruction issue (warp instructions per
    # launch from the ncu count per candidate, against the SM count x 4 issue
    # slots x the median SM clock sampled in the timed region)
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
    if sm_mhz:
        instr = RBL_WARP_INSTR_PER_32_CAND * stats2.candidates / 32.0
        issue_peak = torch.cuda.get_device_properties(0).multi_processor_count * \
            ISSUE_SLOTS_PER_SM_CYCLE * sm_mhz * 1e6
        roof["issue"] = {"achieved": instr / t_pair, "peak": issue_peak,
                         "unit": "warp instructions/s", "frac": instr / t_pair / issue_peak,
                         "warp_instructions_per_launch": instr,
                         "source": "ncu smsp__inst_executed.sum per candidate at N=100000"}
    # ten steps hold about two list rebuilds (one every ~5 steps), like the GPU average
    base = cpu_baseline(n, p, 10, 1) if not args.no_cpu_baseline else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "mixed(u32 fixed-point, f32 SFU, f64 "
                                                         "reductions/integrator)",
        "data": "synthetic",
        "config": {"workload": f"lj_electrolyte N={n} rho*=0.8 10% ions, RBL(r_core 2.5, cut_off "
                               f"5, skin 0.3, p=100, freq={stats.selection_frequency}) + RBE(P={p},"
                               " alpha=0.16), NVE dt=0.005",
                   "global_batch": ws * n, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (candidate list "
                         f"{stats.candidates * 4 / 1e6:.0f} MB)"},
        "fp64_plain": {"value": v64, "ms_per_step": ms64 / args.steps, "phase_ms": ph64},
        "mixed_over_fp64": value / v64,
        "parity_vs_oracle": par,
        "phase_ms_mixed": {"kick_drift": phm[0], "skin_rebuild": phm[1], "real_space": phm[2],
                           "kspace": phm[3]},
        "rebuilds_per_step": stats.rebuilds / max(1, stats.steps + 1),
        "e2e": {"value": job_throughput(ws, n, args.steps, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": 6 * 8 * n, "d2h_bytes_per_step": 9 * 8 * n},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks,
        "cpu_baseline": base,
    }
    if ws == 1 and not args.no_extras:  # the other configs and RBMD's kernels, one GPU
        line["configs"] = config_runs(local)
        try:
            line["reference_gpu"] = reference_gpu(local)
        except Exception as ex:  # report, never fail the headline line
            line["reference_gpu"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    print(json.dumps(line), flush=True)
    if dist and ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batched(args):
    """Batched replicas: R independent LJ electrolytes with
    log-uniform atom counts, mixed form, all advanced by one CUDA graph launch
    per step (rbx_batch) in the phase-batched design (value) and in the
    one-branch-per-replica design, against the same replicas stepped one
    engine at a time: plain FP64 launch by launch (the one-replica-per-launch
    baseline) and mixed with each engine's own step graph."""
    import torch

    from rbmd_b200 import rbx, systems

    rng = np.random.default_rng(args.batch_seed)
    if args.batch_nmin == args.batch_nmax:  # equal replicas
        sizes = np.full(args.replicas, args.batch_nmin)
    else:
        sizes = np.exp(rng.uniform(np.log(args.batch_nmin), np.log(args.batch_nmax),
                                   args.replicas)).astype(int)
    syss = [systems.lj_electrolyte(int(n), seed=1000 + r, kspace_p=args.p)
            for r, n in enumerate(sizes)]
    total = int(sizes.sum())

    def make(precision, graph):
        es = []
        for r, s in enumerate(syss):
            e = rbx.Engine(s, precision=precision, seed=77 + r)
            e.set_step_graph(graph)
            e.compute_forces(0)
            es.append(e)
        return es

    def close(es):
        for e in es:
            e.close()

    # batched, mixed: device time on the batch stream
    es = make(rbx.MIXED, True)
    b = rbx.Batch(es)
    b.step(args.warmup)
    st = torch.cuda.ExternalStream(b.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_batch():
        torch.cuda.synchronize()
        ev0.record(st)
        b.step(args.steps)
        ev1.record(st)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    def time_design(mode):
        b.set_mode(mode)
        b.step(args.warmup)  # the first step captures the graph
        return time_batch(), b.design

    # the phase-batched graph (one launch per phase over all replicas; value)
    # and the graph of one branch per replica, with the built-in launch
    # shapes, then autotuned (per-replica shapes: the phased graph then takes
    # one launch per shape and phase)
    ms_batch, design = time_design(rbx.Batch.AUTO)
    ms_branch_default, _ = time_design(rbx.Batch.BRANCHES)
    ms_phased = ms_batch if design == rbx.Batch.PHASED else None
    if ms_phased is None:  # AUTO took the branches: time the phased graph too
        try:
            ms_phased, _ = time_design(rbx.Batch.PHASED)
        except rbx.RbxError:
            ms_phased = None
    b.set_mode(rbx.Batch.AUTO)
    # autotuner: one timing per size bin, the other replicas of the bin reuse it
    t_tune = time.perf_counter()
    b.autotune()
    t_tune = time.perf_counter() - t_tune
    ms_branch, _ = time_design(rbx.Batch.BRANCHES)
    ms_tuned, _ = time_design(rbx.Batch.AUTO)
    b.close()
    close(es)

    def one_at_a_time(precision, graph, steps):
        es = make(precision, graph)
        for e in es:
            e.step(max(1, args.warmup // 2))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            for e in es:
                e.step(1)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        close(es)
        return dt

    base_steps = max(1, args.steps // 4)
    t64 = one_at_a_time(rbx.PLAIN_FP64, False, base_steps)
    tmix = one_at_a_time(rbx.MIXED, True, base_steps)
    value = total * args.steps / (ms_batch / 1e3)
    line = {
        "metric": "batched replicas: aggregate atom-steps/s, mixed, one graph launch per step",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_batch / args.steps, "higher_is_better": True, "scaling": "weak",
        "dtype": "mixed(u32 fixed-point, f32 SFU, f64 reductions/integrator)",
        "data": "synthetic",
        "config": {"workload": f"{args.replicas} LJ electrolytes rho*=0.8 10% ions, " + (
                       f"N = {args.batch_nmin} each" if args.batch_nmin == args.batch_nmax else
                       f"N log-uniform [{args.batch_nmin}, {args.batch_nmax}] "
                       f"(seed {args.batch_seed})") + f", RBL + RBE(P={args.p}), NVE dt=0.005",
                   "total_atoms": total, "replicas": args.replicas},
        "one_replica_per_launch_fp64": {"value": total * base_steps / t64, "steps": base_steps,
                                        "timing": "host wall clock around launch-by-launch steps"},
        "one_engine_at_a_time_mixed_graph": {"value": total * base_steps / tmix,
                                             "steps": base_steps,
                                             "timing": "host wall clock, one graph launch per "
                                                       "engine and step"},
        "batched_over_fp64_baseline": value / (total * base_steps / t64),
        "design": {1: "phased: one launch per phase over all replicas, a conditional rebuild "
                      "node per replica",
                   2: "branches: one graph branch per replica"}.get(design, str(design)),
        "branch_graph": {"value": total * args.steps / (ms_branch_default / 1e3),
                         "ms_per_step": ms_branch_default / args.steps,
                         "autotuned_value": total * args.steps / (ms_branch / 1e3)},
        "phased_graph": None if ms_phased is None else {
            "value": total * args.steps / (ms_phased / 1e3),
            "ms_per_step": ms_phased / args.steps},
        "autotune": {"phased_autotuned_value": total * args.steps / (ms_tuned / 1e3),
                     "tuning_seconds": t_tune,
                     "note": "value and branch_graph.value use the built-in launch shapes"},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_water(args):
    """Rigid water with the settings of the reference's water workload
    (benchmark/systems/water.json: CVFF with special_bonds [0 0 0], RBL
    cut_off 10 r_core 6.5 skin 2, RBE P = 300, SHAKE, Nose-Hoover NVT at
    298 K with 10 fs damping, dt = 0.5 fs, REAL units): 24,327 molecules /
    72,981 atoms in a 90 A box.  The lattice start is first equilibrated
    (untimed, mixed form, same settings) so
    the timed steps see liquid at ~300 K with its normal rebuild rate; both
    forms then start from that state.  Reports device time per step of each
    form, the mixed form's force error against plain FP64 on the same state
    and k-samples, and the constraint residuals after the run."""
    import torch

    from rbmd_b200 import rbx, systems

    coulomb = args.water_coulomb
    P = args.water_p if coulomb == "RBE" else -(-args.water_p // 16) * 16  # RBSOG: multiple of 16
    s = systems.water(args.water_mol, seed=7, kspace_p=P, dt=args.water_dt,
                      rbsog_level=args.rbsog_level)
    p = s["params"]
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    damp = args.water_damp
    ns, sp = rbx.special_build(s["n"], s["bonds"], s["angles"])
    tdof = 2.0 * s["n"] - 3  # 3N - 3 - N with SHAKE (Computedof)

    def make(sysd, precision, seed=77):
        e = rbx.Engine(sysd, precision=precision, seed=seed, coulomb=coulomb)
        e.set_shake(s["clusters"], systems.WATER_BOND, systems.WATER_ANGLE)
        e.set_special(ns, sp, (0.0, 0.0, 0.0))
        return e

    # untimed equilibration from the lattice
    e = make(s, rbx.MIXED, seed=5)
    e.compute_forces(0)
    e.set_nose_hoover(298.0, 298.0, damp, kb=p["kb"], mvv2e=p["mvv2e"], tdof=tdof)
    e.step(args.water_equil)
    st0 = e.get_state()
    t_equil = e.thermostat()["temperature"]
    e.close()
    s_eq = dict(s, pos=st0["pos"], vel=st0["vel"])

    # force accuracy of the mixed form, same state and k-samples
    from oracle import oracle as O

    wbox = O.Box.make(s["lo"], s["hi"])
    m = (O.rbe_sample_philox(wbox, p["alpha"], P, 5, 0) if coulomb == "RBE" else
         O.rbsog_sample_philox(args.rbsog_level, p["cut_off"], wbox, P, 5, 0))
    forces = {}
    for prec in (rbx.PLAIN_FP64, rbx.MIXED):
        e = make(s_eq, prec)
        e.set_k_samples(*m)
        e.compute_forces(0)
        forces[prec] = e.force_parts()
        e.close()
    err = {"force": systems.rel_rms(sum(forces[1]), sum(forces[0])),
           "pair": systems.rel_rms(forces[1][0], forces[0][0]),
           "kspace": systems.rel_rms(forces[1][1], forces[0][1])}

    out = {}
    for name, prec in (("mixed", rbx.MIXED), ("fp64_plain", rbx.PLAIN_FP64)):
        e = make(s_eq, prec)
        e.compute_forces(0)
        e.set_nose_hoover(298.0, 298.0, damp, kb=p["kb"], mvv2e=p["mvv2e"], tdof=tdof)
        e.step(args.warmup)
        r0 = e.stats().rebuilds
        st = torch.cuda.ExternalStream(e.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(st)
        e.step(args.steps)
        ev1.record(st)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        rebuilds = e.stats().rebuilds - r0
        e.set_profiling(True)
        e.step(args.steps)
        ph = e.phase_ms()
        stt = e.get_state()
        cl = s["clusters"]
        d = stt["pos"][cl[:, 1]] - stt["pos"][cl[:, 0]]
        d -= L * np.rint(d / L)
        out[name] = {"value": s["n"] * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "phase_ms": {"kick_drift_shake": ph[0], "skin_check_rebuild": ph[1],
                                  "real_space_special": ph[2],
                                  "kspace_kick_rattle_thermostat": ph[3]},
                     "rebuilds_in_timed_steps": rebuilds, "shake_failures": e.shake_status()[1],
                     "bond_error_max": float(np.abs(np.linalg.norm(d, axis=1) - 1.0).max()),
                     "temperature_end": e.thermostat()["temperature"]}
        e.close()
    line = {
        "metric": f"rigid water (CVFF special bonds, RBL + {coulomb}, SHAKE, NVT): atom-steps/s",
        "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": out["mixed"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak",
        "dtype": "mixed(u32 fixed-point, f32 SFU, f64 reductions/integrator)",
        "data": "synthetic",
        "config": {"workload": f"{args.water_mol} rigid 3-site waters ({s['n']} atoms), L = "
                               f"{float(L[0]):.2f} A, REAL, cut_off 10 r_core 6.5 skin 2, "
                               + (f"RBE alpha 0.09 P={P}" if coulomb == "RBE" else
                                  f"RBSOG rbsog_level {args.rbsog_level} P={P} (+6 direct "
                                  f"vectors), real-space alpha 0.09")
                               + ", special_bonds [0 0 0], SHAKE "
                               f"(1.0 A, 109.47 deg), Nose-Hoover 298 K / {damp} fs, "
                               f"dt = {args.water_dt} fs",
                   "equilibration_steps": args.water_equil, "temperature_after_equil": t_equil},
        "mixed": out["mixed"], "fp64_plain": out["fp64_plain"],
        "mixed_over_fp64": out["mixed"]["value"] / out["fp64_plain"]["value"],
        "mixed_rel_force_err": err,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_rbsog(args):
    """RBSOG: the 200k-atom LJ electrolyte with neighbor VERLET-SOG and coulomb
    RBSOG (rbsog_level 2, P = 112: 100 rounded up to 16 as the reference
    does), and RBL real space with RBSOG k-space; mixed and plain FP64, NVE,
    device time per step; the mixed form's force error against plain FP64 on
    the same state and k-samples."""
    import torch

    from oracle import oracle as O
    from rbmd_b200 import rbx, systems

    n, level, P = args.n, args.rbsog_level, 112
    s = systems.lj_electrolyte(n, seed=2024, kspace_p=P, rbsog_level=level)
    box = O.Box.make(s["lo"], s["hi"])
    m = O.rbsog_sample_philox(level, s["params"]["cut_off"], box, P, 5, 0)
    out = {}
    for nb in ("VERLET-SOG", "RBL"):
        forces = {}
        for prec in (rbx.PLAIN_FP64, rbx.MIXED):
            e = rbx.Engine(s, precision=prec, neighbor=nb, coulomb="RBSOG", seed=7)
            e.set_k_samples(*m)
            e.compute_forces(0)
            forces[prec] = e.force_parts()
            e.close()
        err = systems.rel_rms(sum(forces[1]), sum(forces[0]))
        for name, prec in (("mixed", rbx.MIXED), ("fp64_plain", rbx.PLAIN_FP64)):
            e = rbx.Engine(s, precision=prec, neighbor=nb, coulomb="RBSOG", seed=77)
            e.compute_forces(0)
            e.step(args.warmup)
            st = torch.cuda.ExternalStream(e.stream)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record(st)
            e.step(args.steps)
            ev1.record(st)
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1)
            e.set_profiling(True)
            e.step(args.steps)
            ph = e.phase_ms()
            out[f"{nb}+RBSOG {name}"] = {
                "value": n * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                "phase_ms": {"kick_drift": ph[0], "skin_rebuild": ph[1], "real_space": ph[2],
                             "kspace": ph[3]}}
            e.close()
        out[f"{nb}+RBSOG mixed_rel_force_err"] = err
    line = {
        "metric": "RBSOG (VERLET-SOG / RBL real space): atom-steps/s @200k atoms",
        "value": out["VERLET-SOG+RBSOG mixed"]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": out["VERLET-SOG+RBSOG mixed"]["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "dtype": "mixed(u32 fixed-point, f32 SFU, f64 reductions/integrator)",
        "data": "synthetic",
        "config": {"workload": f"lj_electrolyte N={n} rho*=0.8 10% ions, cut_off 5 skin 0.3, "
                               f"RBSOG rbsog_level {level} P={P} (+6 direct vectors), "
                               f"NVE dt=0.005"},
        "runs": out,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gradient(args):
    """Force-field fitting gradient (the gradient recipe): N atoms, three types,
    16 frames every 50 steps of an MD run at theta*, a fixed k-sample per frame;
    theta perturbed by seeded +-5 %; L = mean over frames and atoms of
    |F(theta) - F(theta*)|^2.  dL/dtheta and dL/dr from the adjoint, checked
    against central differences (h = 1e-6 relative) of the same FP64 force."""
    import torch

    from oracle import oracle as O
    from rbmd_b200 import rbx, systems

    n, nf = args.grad_n, 16
    s = systems.lj_electrolyte(n, seed=2024, kspace_p=args.p)
    p = s["params"]
    box = O.Box.make(s["lo"], s["hi"])
    typ = np.asarray(s["type"])
    md = rbx.Engine(s, precision=rbx.MIXED, seed=3)
    md.compute_forces(0)
    frames = []
    for _ in range(nf):
        md.step(50)
        frames.append(md.get_state()["pos"])
    md.close()
    samples = [O.rbe_sample_philox(box, p["alpha"], p["kspace_p"], 100 + f, f) for f in range(nf)]
    th0 = {"eps": np.asarray(s["eps"], float), "sigma": np.asarray(s["sigma"], float),
           "Q": np.array([0.0, 1.0, -1.0]), "alpha": float(p["alpha"])}
    rng = np.random.default_rng(7)
    th = {k: (v * (1 + rng.uniform(-0.05, 0.05, np.shape(v))) if isinstance(v, np.ndarray)
              else v * (1 + rng.uniform(-0.05, 0.05))) for k, v in th0.items()}
    engines = {"fp32": rbx.Engine(s, precision=rbx.MIXED),
               "fp64": rbx.Engine(s, precision=rbx.PLAIN_FP64)}

    def setp(e, t):
        e.set_lj_params(t["sigma"], t["eps"])
        e.set_charges(t["Q"][typ])
        e.set_alpha(t["alpha"])

    def forces(e, t, f):
        setp(e, t)
        e.set_k_samples(*samples[f])
        e.set_positions(frames[f])
        e.compute_forces(f)
        return e.get_state()["force"]

    def gradient(e):
        """Loss and adjoint gradient over the frames, timed per frame (forward
        and backward); the reference forces come from the same engine."""
        ref = [forces(e, th0, f) for f in range(nf)]
        grad = {"eps": np.zeros(3), "sigma": np.zeros(3), "Q": np.zeros(3), "alpha": 0.0}
        dr, t_fwd, t_adj, loss = [], 0.0, 0.0, 0.0
        for f in range(nf):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            F = forces(e, th, f)
            t1 = time.perf_counter()
            d = F - ref[f]
            loss += float((d ** 2).sum()) / (nf * n)
            out = e.force_vjp(2.0 * d / (nf * n))
            t2 = time.perf_counter()
            t_fwd += t1 - t0
            t_adj += t2 - t1
            grad["eps"] += out["eps"]
            grad["sigma"] += out["sigma"]
            grad["Q"] += np.bincount(typ, weights=out["charge"], minlength=3)
            grad["alpha"] += out["alpha"]
            dr.append(out["pos"])
        return grad, loss, dr, 1e3 * t_fwd / nf, 1e3 * t_adj / nf

    res = {k: gradient(e) for k, e in engines.items()}
    e = engines["fp64"]
    ref = [forces(e, th0, f) for f in range(nf)]

    def loss_at(t):
        return sum(float(((forces(e, t, f) - ref[f]) ** 2).sum()) for f in range(nf)) / (nf * n)

    fd = {}
    for key in ("eps", "sigma", "Q", "alpha"):
        for c in range(3 if key != "alpha" else 1):
            hval = 1e-6 * max(abs(th[key][c] if key != "alpha" else th[key]), 1.0)
            up = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in th.items()}
            dn = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in th.items()}
            if key == "alpha":
                up[key] += hval
                dn[key] -= hval
            else:
                up[key][c] += hval
                dn[key][c] -= hval
            fd[f"{key}[{c}]"] = (loss_at(up) - loss_at(dn)) / (2 * hval)
    for en in engines.values():
        en.close()

    def errors(grad):
        out = {}
        for name, fdv in fd.items():
            key, c = name.split("[")[0], int(name.split("[")[1][:-1])
            a = grad[key] if key == "alpha" else grad[key][c]
            out[name] = abs(a - fdv) / max(abs(fdv), 1e-300)
        return out

    g32, loss32, dr32, tf32, ta32 = res["fp32"]
    g64, loss64, dr64, tf64, ta64 = res["fp64"]
    e32, e64 = errors(g32), errors(g64)
    dr_rel = max(float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())) for a, b in zip(dr32, dr64))
    par_rel = {k: float(np.max(np.abs(np.asarray(g32[k]) - np.asarray(g64[k])) /
                               np.maximum(np.abs(np.asarray(g64[k])), 1e-300)))
               for k in g32}
    line = {
        "metric": "force-field gradient: adjoint dL/dtheta and dL/dr, 16 frames",
        "n": n, "frames": nf, "P": args.p, "loss": loss32,
        "fp32_adjoint": {
            "engine": "mixed form: FP32 pair and k-space terms (exact fixed-point phases), "
                      "FP64 sums",
            "forward_ms_per_frame": tf32, "adjoint_ms_per_frame": ta32,
            "grad": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in g32.items()},
            "max_rel_err_vs_fp64_central_differences": max(e32.values()),
            "rel_err_vs_fp64_central_differences": e32,
            "rel_err_vs_fp64_adjoint": par_rel,
            "dL_dr_rel_rms_vs_fp64_adjoint_max": dr_rel},
        "fp64_adjoint": {
            "forward_ms_per_frame": tf64, "adjoint_ms_per_frame": ta64, "loss": loss64,
            "grad": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in g64.items()},
            "max_rel_err_vs_central_differences": max(e64.values()),
            "rel_err_vs_central_differences": e64},
        "timing": "host wall clock per frame: parameter upload, list build, force (forward); "
                  "adjoint kernels and host reductions (adjoint)",
        "central_differences": "FP64 engine, h = 1e-6 relative, same frames and k-samples",
        "forward_evaluations_replaced_per_frame": 2 * 10,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=200000)
    ap.add_argument("--p", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the oracle parity, the other configs and RBMD's kernels")
    ap.add_argument("--batched", action="store_true",
                    help="batched-replica measurement instead of the headline line")
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--batch-nmin", type=int, default=953)
    ap.add_argument("--batch-nmax", type=int, default=20000)
    ap.add_argument("--batch-seed", type=int, default=4)
    ap.add_argument("--gradient", action="store_true",
                    help="force-field gradient measurement instead of the headline line")
    ap.add_argument("--grad-n", type=int, default=20000)
    ap.add_argument("--rbsog", action="store_true",
                    help="RBSOG (VERLET-SOG and RBL real space) measurement")
    ap.add_argument("--rbsog-level", type=int, default=2)
    ap.add_argument("--water", action="store_true",
                    help="rigid-water (CVFF, SHAKE, NVT) measurement instead of the headline line")
    ap.add_argument("--water-mol", type=int, default=24327)
    ap.add_argument("--water-p", type=int, default=300)
    ap.add_argument("--water-coulomb", choices=("RBE", "RBSOG"), default="RBE",
                    help="k-space of the water run; RBSOG rounds P up to a multiple of 16")
    ap.add_argument("--water-dt", type=float, default=0.5)
    ap.add_argument("--water-damp", type=float, default=10.0)
    ap.add_argument("--water-equil", type=int, default=2000)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.batched:
        return run_batched(args)
    if args.gradient:
        return run_gradient(args)
    if args.water:
        return run_water(args)
    if args.rbsog:
        return run_rbsog(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
