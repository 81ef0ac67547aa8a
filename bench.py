"""Benchmark of the dnsbox pseudospectral time step on B200.

Workload (the forced-isotropic-turbulence configuration the metric is quoted
on): N = 256^3 in a 2 pi box, seeded spectrum E(k) ~ k^4 exp(-2 k^2/k0^2) with
k0 = 3 and E = 0.5, band forcing on |k| <= 2.5 with Pin = 0.1, nu = 2e-3,
integrating-factor Heun step with CFL control at Courant 0.5.  The headline
form is the tensor-core split-precision one (FP32 state, DFT-64 stages of the
strided passes on tcgen05 with f16 hi + lo operands); the plain FP64 form and
the FP32 SIMT form are timed beside it on the same seeded field, with the
TC-split velocity error against FP64 after the timed steps, and the 512^3
legs of all three.  One "step" is one time step of the whole box.  Inputs (the
spectral velocity) are synthetic and larger than L2 (3 x 68 MB in FP32).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 (torchrun) every rank advances its own independent box (the step
does not shard: replicas only), value = steps of all ranks / max-over-ranks
time.  ``--impl reference`` times the CPU restatement of the reference step on
the host cores (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = ("steps/s @256^3 forced turbulence (IF-Heun, CFL 0.5, band forcing), tensor-core split-precision form "
          "(FP64 and FP32 forms and 512^3 beside it)")
DTYPE = {"fp64": "f64", "fp32": "f32", "tc_split": "f32 (f16 hi+lo tensor-core DFT stages, f32 accumulate)"}
UNIT = "steps/s"
WORKLOAD = dict(n=256, k0=3.0, nu=2e-3, kCutOff=2.5, Pin=0.1, courant=0.5, dt_max=1e-2, dt0=1e-3)

# Algorithmic HBM traffic per launch of each pass, in spectral-field units
# (one field = nz*ny*(nx/2+1) complex values): reads + writes, each field once.
PASS_FIELDS_HEUN = {"z_inv": [8, 8], "y_inv": [11, 11], "x_nl": [9, 9], "y_fwd": [6, 6],
                    "z_fwd": [6, 6], "z_fin": [9, 12]}


def pruned_pass_fields(n):
    """The same for the pruned passes of a cubic n^3 box: only the kept fraction
    of each axis (kx < a plus the Nyquist column; |ky|, |kz| < a plus Nyquist,
    a = ceil(n/3)) is read or written where the pass skips the 2/3-rule zeros."""
    a = -(-n // 3)
    fx = (a + 1) / (n // 2 + 1)
    fy = fz = 2 * a / n
    fxy = fx * fy
    fxyz = fxy * fz
    return {"z_inv": [3 * fxyz + 5 * fxy] * 2, "y_inv": [5 * fxy + 6 * fx] * 2, "x_nl": [9 * fx] * 2,
            "y_fwd": [3 * fx + 3 * fxy] * 2, "z_fwd": [3 * fxy + 3 * fxyz] * 2, "z_fin": [9 * fxyz, 12 * fxyz]}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and clocks-event reasons through NVML while running."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks",
               0x1: "gpu_idle", 0x10: "sync_boost", 0x100: "display_clock"}

    def __init__(self, index):
        self.samples = []
        self.reasons = 0
        self.ok = False
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # noqa: BLE001
            log("clock sampling unavailable:", e)
            self.max_mhz = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except AttributeError:
                    r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.reasons |= int(r)
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok:
            return None
        rs = sorted(v for b, v in self.REASONS.items() if self.reasons & b and b != 0x1)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": rs, "samples": len(self.samples)}


# ----------------------------------------------------------------- reference arm
def cpu_reference_rate(n, max_steps, budget_s, warmup=1):
    """Times the CPU restatement of the reference Heun step (oracle, FP64,
    scipy.fft on all host threads) on the benchmark workload."""
    from dnsbox_b200 import ic
    from oracle import dnsbox_oracle as O
    w = WORKLOAD
    p = O.Params(nx=n, ny=n, nz=n, nu=w["nu"], kCutOff=w["kCutOff"], Pin=w["Pin"], bandlim=True,
                 courant_min=w["courant"], courant_max=w["courant"], dt_max=w["dt_max"])
    g = O.Grid(p)
    uh = ic.random_field(n, seed=0, k0=w["k0"])
    dt = w["dt0"]
    u = O.state_uhat2u(g, uh)
    dt, _ = O.set_time_step(g, dt, O.io_courant(g, u, dt))
    for _ in range(warmup):
        uh = O.heun_step(g, uh, dt)
    done, t0 = 0, time.perf_counter()
    while done < max_steps:
        uh = O.heun_step(g, uh, dt)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return done / el, done, el


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import dnsbox_oracle as O
    n = args.n
    warm = min(args.warmup, 1)
    rate, done, el = cpu_reference_rate(n, args.steps, budget_s=args.ref_budget, warmup=warm)
    cores = O.WORKERS
    line = {
        # the steps and warm-up steps this arm actually ran: a 256^3 CPU step takes
        # seconds, so the run stops at its time budget (or at --steps)
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": done, "warmup": warm, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": 1e3 / rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"forced isotropic turbulence {n}^3, IF-Heun, CFL 0.5, band forcing Pin 0.1, "
                               f"nu 2e-3, k0 3 (independent box per GPU)",
                   "n": n, "precision": "fp64 (the reference's CPU arithmetic)", "parallelism": "rank 0 host cores"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{done} full Heun steps at {n}^3 ({el:.1f} s) of the NumPy/scipy.fft "
                                   f"restatement of rhs.f90 + dnsboxheun.f90 (the Fortran/MPI/p3dfft "
                                   f"reference cannot be built on this image)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- our arm
def make_box(n, precision, rank, nu=None):
    from dnsbox_b200.ops import Box
    w = WORKLOAD
    return Box(n, precision=precision, nu=w["nu"] if nu is None else nu, kCutOff=w["kCutOff"], Pin=w["Pin"],
               bandlim=True,
               courant_min=w["courant"], courant_max=w["courant"], dt_max=w["dt_max"], dt=w["dt0"],
               device=torch.cuda.current_device())


def max_over_ranks(ms, device="cuda"):
    """Slowest rank's time (all ranks take part; NCCL on GPUs, gloo on CPU)."""
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, steps, max_ms):
    """Whole-job steps/s of `world` independent boxes timed by the slowest rank."""
    return world * steps / (max_ms / 1e3)


def timed_steps(box, u, k, dist_on):
    """K steps bracketed by barrier + synchronize; CUDA events on the launch stream."""
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    if dist_on:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    box.step(u, k, diag=False)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist_on:
        torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    if dist_on:
        ms = max_over_ranks(ms)
    return ms


def measure_e2e(box, uh_np, k):
    """Per step: H2D of the state from pinned host memory (reference layout),
    one step through the C ABI, D2H of the new state and the step record."""
    host = torch.empty((3, box.nxh, box.ny, box.nz), dtype=torch.complex128, pin_memory=True)
    host_np = host.numpy()
    host_np[...] = np.transpose(uh_np, (0, 3, 2, 1))
    out = torch.empty_like(host, pin_memory=True).numpy()
    u = box.zeros()
    box.upload_state(host_np, u)
    box.step(u, 1)
    box.download_state(u, out)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        box.upload_state(host_np, u)
        box.step(u, 1, diag=True)
        box.download_state(u, host_np)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    nbytes = 3 * box.nz * box.ny * box.nxh * 16
    return k / (ms / 1e3), nbytes, nbytes + 96


def profile_passes(box, u, k):
    box.profile(True)
    box.profile_read(reset=True)
    box.step(u, k, diag=False)
    pr = box.profile_read(reset=True)
    box.profile(False)
    return pr


def dtype_of(prec, sched):
    base = prec.split("@")[0]
    if base == "tc_split" and all(v == "simt" for v in sched["tc_kernel"]) and sched["z_fwd_kernel"] == "simt":
        return "f32 (tensor-core form; its schedule keeps every strided pass on the FP32 SIMT kernel)"
    return DTYPE[base]


def force_tc(box, prec, sched):
    """`tc_split@tc`: the tensor-core form with its strided passes A, B, D held
    on a tensor-core kernel (the cp.async-fed one where the tuner chose the
    SIMT kernel), so that the tensor-core kernels' own speed is on record."""
    if not prec.endswith("@tc"):
        return sched
    tc = tuple("cp.async" if v == "simt" else v for v in sched["tc_kernel"])
    box.set_schedule(tc, sched["x_kernel"],
                     sched["z_fwd_kernel"] == "tma")
    return dict(box.schedule(), tuned=False)


def extra_sizes(args):
    """Steps/s of the same forced workload at 512^3 (nu 8e-4; FP64, FP32 and
    TC-split), seeded on the device, K/2 steps after W warm-up steps each."""
    from dnsbox_b200 import ic
    out = {}
    for prec in ("fp64", "fp32", "tc_split", "tc_split@tc"):
        box = make_box(512, prec.split("@")[0], 0, nu=8e-4)
        u = ic.random_field_gpu(box, seed=0, k0=WORKLOAD["k0"])
        box.step(u, args.warmup, diag=False)
        sched = box.autotune(u, nsteps=2) if not args.no_tune else box.schedule()
        sched = force_tc(box, prec, sched)
        k = max(2, args.steps // 2)
        ms = timed_steps(box, u, k, False)
        out[f"{prec}_512"] = {"value": k / (ms / 1e3), "ms_per_step": ms / k, "steps": k, "nu": 8e-4,
                              "schedule": sched}
        box.close()
        del u
        torch.cuda.empty_cache()
    out["tc_split_vs_fp64_512"] = out["tc_split_512"]["value"] / out["fp64_512"]["value"]
    return out


def tc_1024_rate(args):
    """Config 4's large case: 1024^3 forced turbulence in the TC-split form
    (FP32 state, nu 4e-4), seeded on the device; steps/s over K/4 steps after
    W warm-up steps, with the largest energy-budget residual
    |dE/dt - (Pin - D)| over the timed steps."""
    from dnsbox_b200 import ic
    box = make_box(1024, "tc_split", 0, nu=4e-4)
    u = ic.random_field_gpu(box, seed=0, k0=WORKLOAD["k0"])
    torch.cuda.empty_cache()
    box.step(u, args.warmup, diag=False)
    k = max(2, args.steps // 4)
    ms = timed_steps(box, u, k, False)
    e0 = box.kinetic(u)
    recs = box.step(u, 3)
    es = [e0] + [r["ekin"] for r in recs]
    resid = max(abs((es[i + 1] - es[i]) / recs[i]["dt"]
                    - (WORKLOAD["Pin"] - 0.5 * (recs[i - 1]["dissipation"] + recs[i]["dissipation"])))
                for i in range(1, len(recs)))
    box.close()
    del u
    torch.cuda.empty_cache()
    return {"value": k / (ms / 1e3), "unit": "steps/s", "ms_per_step": ms / k, "steps": k, "nu": 4e-4,
            "energy_budget_residual": resid, "memory_gb": 18 * 1024 ** 2 * 513 * 8 / 1e9}


def orbit_rate():
    """Periodic-orbit variant of the adjoint configuration: seconds per J and
    gradient of J = 1/2 <|u(T) - u(0)|^2> at 96^3, T = 5 (500 fixed steps of
    dt = 1e-2, Kolmogorov forcing, nu = 1/40, FP32 bulk, FP64 J), checkpoints
    every 32 steps."""
    from dnsbox_b200 import ic
    from dnsbox_b200.ops import Box
    n, ns = 96, 500
    box = Box(n, precision="fp32", nu=1.0 / 40.0, bandlim=False, tstep_fix=True, dt=1e-2)
    f = box.from_numpy(ic.kolmogorov_forcing(n, 1.0, 4))
    box.set_forcing(f)
    u = box.from_numpy(ic.random_field(n, seed=0, k0=4.0))
    box.step(u, ns, diag=False)
    box.orbit_residual(u, ns, every=32)   # warm-up of the same length: grows the checkpoint arena, loads the kernels
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J, _ = box.orbit_residual(u, ns, every=32)
    el = time.perf_counter() - t0
    box.close()
    return {"value": 1.0 / el, "unit": "gradients/s", "seconds_per_gradient": el, "n": n, "steps": ns,
            "checkpoint_every": 32, "J": J}


def adjoint_rate(iters=2000, t_spinup=50.0):
    """Adjoint descent on the 64^3 Kolmogorov residual (FP32 bulk, FP64 J and
    line search, nu = 1/40, F = 1, kf = 4): the initial guess is the state
    after 50 time units (CFL-controlled Heun, Courant 0.3-0.5) from the seeded
    k0 = 4 field; then 2000 descent iterations, all timed (iterations/s)."""
    from dnsbox_b200 import ic
    from dnsbox_b200.ops import Box
    box = Box(64, precision="fp32", nu=1.0 / 40.0, bandlim=False, hminone=True, courant_min=0.3,
              courant_max=0.5, dt_max=1e-2, dt=5e-3)
    f = box.from_numpy(ic.kolmogorov_forcing(64, 1.0, 4))
    box.set_forcing(f)
    u = box.from_numpy(ic.random_field(64, seed=0, k0=4.0))
    t0 = time.perf_counter()
    steps = 0
    while box.get_time() < t_spinup:
        box.step(u, 500, diag=False)
        steps += 500
    spin_s = time.perf_counter() - t0
    t_reached = box.get_time()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist, alpha = box.adjoint_descent(u, iters, alpha=1.0)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    h = hist[np.isfinite(hist)]
    box.close()
    return {"value": (len(h) - 1) / el, "unit": "iterations/s", "n": 64, "iters": int(len(h) - 1),
            "iters_requested": iters, "spinup_time_units": t_reached, "spinup_steps": steps,
            "spinup_s": spin_s, "J_first": float(h[0]), "J_last": float(h[-1])}


def ensemble_rate(steps=300, rank=0, world=1, dist_on=False):
    """Config 2: 96 independent boxes (32 each of 32^3, 64^3, 96^3), FP32 state,
    FP64 diagnostics, seeds 0..95, nu log-uniform in [5e-3, 5e-2] (seed 1000),
    k0 = 3, fixed dt = 1e-3, IF-Heun; one CUDA-graph replay advances all boxes
    of a rank.  Under torchrun the 96 boxes are split over the ranks (each
    rank a share of every size group, no collective while stepping); the time
    is the slowest rank's and the final energies of all 96 boxes are gathered
    on rank 0 (None is returned elsewhere)."""
    from dnsbox_b200.ensemble import Ensemble, config2_local, gather_to_rank0
    local = config2_local(rank, world)
    groups = [bu for _, _, bu in local]
    ens = Ensemble(groups) if groups else None
    if ens:
        ens.run(3)
    torch.cuda.synchronize()
    if dist_on:
        torch.distributed.barrier()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if ens:
        ens.run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    mx = max_over_ranks(ms) if dist_on else ms
    ekin = {}
    for _, idx, (box, _) in local:
        recs = box.diag_read(1)[0]
        recs = recs if isinstance(recs, list) else [recs]
        ekin.update({gi: float(r["ekin"]) for gi, r in zip(idx, recs)})
    allk = gather_to_rank0(ekin, world if dist_on else 1)
    if ens:
        ens.close()
    for box, _ in groups:
        box.close()
    if rank != 0:
        return None
    return {"value": 96 * steps / (mx / 1e3), "unit": "box-steps/s", "boxes": 96, "steps": steps, "n_ranks": world,
            "ms_per_ensemble_step": mx / steps,
            "finite": len(allk) == 96 and all(np.isfinite(v) for v in allk.values()),
            "scaling": "strong: the 96 boxes are split over the ranks",
            "graph": "one CUDA-graph replay per ensemble step and rank (batched size groups)"}


def slab_fft_rate(n=1024, reps=5, rank=0, world=1, dist_on=False):
    """The slab-decomposed transform (p3dfft's 1 x P grid of the reference's
    distributed runs, variables.f90:131-157): an n^3 FP32 R2C + C2R pair of a
    random field over the ranks, each rank its z-slab, the NCCL all-to-all
    between the local halves under torchrun (strong scaling: the grid is
    fixed; one rank exchanges by a copy).  Pairs per second on the slowest
    rank's CUDA-event time, and the worst rank's round-trip error."""
    from dnsbox_b200.slab import SlabFFT
    s = SlabFFT(n, n, n, precision="fp32")
    gen = torch.Generator(device="cuda").manual_seed(rank)
    phys = torch.randn(s.phys_size, generator=gen, device="cuda")
    spec = torch.empty(s.spec_size, dtype=s.cdtype, device="cuda")
    back = torch.empty_like(phys)
    s.r2c(phys, spec)
    s.c2r(spec, back)
    torch.cuda.synchronize()
    if dist_on:
        torch.distributed.barrier()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        s.r2c(phys, spec)
        s.c2r(spec, back)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    err = float((back / float(n) ** 3 - phys).norm() / phys.norm())
    if dist_on:
        ms = max_over_ranks(ms)
        err = max_over_ranks(err)
    s.close()
    del phys, spec, back
    torch.cuda.empty_cache()
    if rank != 0:
        return None
    return {"value": 1e3 / ms, "unit": "R2C+C2R pairs/s", "grid": n, "precision": "fp32", "n_ranks": world,
            "ms_per_pair": ms, "roundtrip_rel_l2": err, "scaling": "strong: the grid is split over the ranks",
            "exchange": "NCCL all-to-all (torch.distributed)" if world > 1 else "device copy (one rank)"}


def slab_heun_rate(n=512, steps=4, rank=0, world=1, dist_on=False):
    """One box split over the ranks (p3dfft's slabs): IF-Heun steps of the
    n^3 forced workload in FP32 on the rank's ky slab, the right-hand side's
    eight per-field all-to-alls and the band-energy / CFL-maxima / (E, D)
    reductions over NCCL under torchrun (strong scaling: the box is fixed;
    one rank exchanges by copies).  Fixed dt; steps per second on the slowest
    rank's CUDA-event time."""
    from dnsbox_b200 import ic
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    s = SlabFFT(n, n, n, precision="fp32")
    kw = dict(nu=8e-4, kCutOff=WORKLOAD["kCutOff"], Pin=WORKLOAD["Pin"], bandlim=True)
    s.setup_rhs(**kw)
    # every rank draws the whole field from the same seed and keeps its ky rows
    b = Box(n, precision="fp32", **kw)
    box_uh = ic.random_field_gpu(b, seed=0, k0=WORKLOAD["k0"])
    b.close()
    nyl = n // world
    u = box_uh[:, :, rank * nyl:(rank + 1) * nyl, :].contiguous()
    del box_uh
    torch.cuda.empty_cache()
    dt = 1e-3
    s.heun_step(u, dt, 1)
    torch.cuda.synchronize()
    if dist_on:
        torch.distributed.barrier()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    recs = s.heun_step(u, dt, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    if dist_on:
        ms = max_over_ranks(ms)
    s.close()
    del u
    torch.cuda.empty_cache()
    if rank != 0:
        return None
    return {"value": 1e3 / ms, "unit": "steps/s", "grid": n, "precision": "fp32", "n_ranks": world,
            "ms_per_step": ms, "dt": dt, "ekin_last": recs[-1]["ekin"],
            "scaling": "strong: one box split over the ranks (z-slabs / ky-slabs)",
            "exchange": "NCCL all-to-all and all-reduce (torch.distributed)" if world > 1 else "device copies (one rank)"}


def read_traffic(prec, n, pruned):
    """DRAM bytes per launch from a committed ncu summary, if one exists
    (columns: pass precision n pruned bytes)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        parts = line.split()
        if (len(parts) == 5 and not line.startswith("#") and parts[1] == prec and int(parts[2]) == n
                and int(parts[3]) == int(bool(pruned))):
            out[parts[0]] = float(parts[4])
    return out


def run_ours(args, rank, world, dist_on):
    from dnsbox_b200 import ic
    n = args.n
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    uh_np = ic.random_field(n, seed=rank, k0=WORKLOAD["k0"])
    results = {}
    final = {}
    for prec in args.precisions:
        box = make_box(n, prec.split("@")[0], rank)
        u = box.from_numpy(uh_np)
        box.step(u, args.warmup, diag=False)
        sched = box.autotune(u, nsteps=4) if not args.no_tune else box.schedule()
        sched = force_tc(box, prec, sched)
        torch.cuda.synchronize()
        box.profile_read(reset=True)
        sampler = ClockSampler(torch.cuda.current_device())
        with sampler:
            ms = timed_steps(box, u, args.steps, dist_on)
        launches = box.profile_read(reset=True)["total_launches"]
        pruned = box.step_pruned()
        if rank == 0:
            final[prec] = u.to(torch.complex128).cpu()   # after W + K steps from the same field
        pr = profile_passes(box, u, args.steps)
        res = {"ms": ms, "launches": launches, "profile": pr, "clocks": sampler.summary(), "pruned": pruned,
               "schedule": sched,
               "pass_fields": pruned_pass_fields(n) if pruned else PASS_FIELDS_HEUN}
        if prec == args.precisions[0] and rank == 0:
            res["e2e"] = measure_e2e(box, uh_np, max(3, min(args.steps, 20)))
        fb = box.nz * box.ny * box.nxh * (16 if prec == "fp64" else 8)
        res["field_bytes"] = fb
        results[prec] = res
        box.close()
        del u
        torch.cuda.empty_cache()
    # the ensemble shards over the ranks (every rank takes part)
    ens_sharded = ensemble_rate(rank=rank, world=world, dist_on=dist_on) if world > 1 and not args.no_extra else None
    slab_sharded = slab_fft_rate(rank=rank, world=world, dist_on=dist_on) if world > 1 and not args.no_extra else None
    slab_step = slab_heun_rate(rank=rank, world=world, dist_on=dist_on) if world > 1 and not args.no_extra else None
    if rank != 0:
        return
    main = args.precisions[0]
    r = results[main]
    steps_s = replica_rate(world, args.steps, r["ms"])
    # dominant kernel roofline
    pr = r["profile"]
    per_pass = {}
    for name, fields in r["pass_fields"].items():
        ms = pr["ms"][name]
        nl = pr["launches"][name]
        if nl == 0 or ms <= 0:
            continue
        # launches alternate between the two RHS of each step
        nbytes = sum(fields[i % len(fields)] for i in range(nl)) * r["field_bytes"]
        per_pass[name] = {"ms_total": ms, "launches": nl, "avg_us": 1e3 * ms / nl,
                          "gbs": nbytes / (ms / 1e3) / 1e9, "bytes_per_launch": nbytes / nl}
    dom = max(per_pass, key=lambda k: per_pass[k]["ms_total"])
    d = per_pass[dom]
    traffic = read_traffic(main, n, r["pruned"]).get(dom)
    gp = float(n) ** 3
    model_bytes = 72 * (8 if main == "fp64" else 4) * gp
    step_time = r["ms"] / args.steps / 1e3
    e2e = r.get("e2e")
    line = {
        "metric": METRIC, "value": steps_s, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(main, r["schedule"]),
        "data": "synthetic",
        "config": {"workload": f"forced isotropic turbulence {n}^3, IF-Heun, CFL 0.5, band forcing Pin 0.1, "
                               f"nu 2e-3, k0 3 (independent box per GPU)",
                   "n": n, "precision": main, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (3 x %.0f MB state, 12-field workspace)" % (r["field_bytes"] / 1e6),
                   "pruned_transforms": r["pruned"]},
        "grid_point_steps_per_s": steps_s * gp,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": d["gbs"], "peak": hbm_peak, "unit": "GB/s",
                     "frac": d["gbs"] / hbm_peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": d["bytes_per_launch"], "avg_launch_us": d["avg_us"],
                     "peak_source": peak_src},
        "step_roofline": {"model_bytes_per_gp_step": 72 * (8 if main == "fp64" else 4),
                          "achieved": model_bytes / step_time / 1e9, "peak": hbm_peak,
                          "frac": model_bytes / step_time / 1e9 / hbm_peak,
                          "algorithmic_fields_per_step": sum(sum(v) for v in r["pass_fields"].values()),
                          "algorithmic_achieved": sum(sum(v) for v in r["pass_fields"].values()) * r["field_bytes"]
                          / step_time / 1e9},
        "passes": {k: {kk: round(vv, 3) for kk, vv in v.items()} for k, v in per_pass.items()},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "schedule": r["schedule"],
    }
    if e2e:
        line["e2e"] = {"value": e2e[0] * world, "unit": UNIT, "h2d_bytes_per_step": e2e[1],
                       "d2h_bytes_per_step": e2e[2]}
    if "fp64" in final:
        ref = final["fp64"]
        line["accuracy_vs_fp64"] = {
            p: {"steps": args.warmup + args.steps,
                "vel_rel_l2": float((final[p] - ref).abs().norm() / ref.abs().norm())}
            for p in final if p != "fp64"}
    if "fp64" in results and main != "fp64":
        line["speedup_vs_fp64"] = results["fp64"]["ms"] / r["ms"]
    for prec in args.precisions[1:]:
        rr = results[prec]
        prr = rr["profile"]
        line.setdefault("variants", {})[prec] = {
            "value": world * args.steps / (rr["ms"] / 1e3), "ms_per_step": rr["ms"] / args.steps,
            "gpu_launches": rr["launches"], "clocks": rr["clocks"], "schedule": rr["schedule"],
            "passes": {k: {"avg_us": round(1e3 * prr["ms"][k] / prr["launches"][k], 2),
                           "gbs": round(sum(f[i % len(f)] for i in range(prr["launches"][k])) * rr["field_bytes"]
                                        / (prr["ms"][k] / 1e3) / 1e9, 1)}
                       for k, f in rr["pass_fields"].items() if prr["launches"][k]},
            "pruned": rr["pruned"]}
    if ens_sharded:
        line["extra"] = {"ensemble_96": ens_sharded, "slab_fft_1024": slab_sharded, "slab_heun_512": slab_step}
    if world == 1 and not args.no_extra:
        line["extra"] = extra_sizes(args)
        line["extra"]["tc_split_1024"] = tc_1024_rate(args)
        line["extra"]["adjoint_descent_64"] = adjoint_rate()
        line["extra"]["periodic_orbit_grad_96"] = orbit_rate()
        line["extra"]["ensemble_96"] = ensemble_rate()
        line["extra"]["slab_fft_1024"] = slab_fft_rate()
        line["extra"]["slab_heun_512"] = slab_heun_rate()
    if world == 1 and not args.no_cpu_baseline:
        from oracle import dnsbox_oracle as O
        rate, done, el = cpu_reference_rate(n, 3, budget_s=args.cpu_budget, warmup=0)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": O.WORKERS, "kind": "port",
                                "sample": f"{done} Heun step(s) of the {n}^3 workload, {el:.1f} s, NumPy/"
                                          f"scipy.fft restatement of rhs.f90 + dnsboxheun.f90"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--precisions", default="tc_split,fp64,fp32,tc_split@tc",
                    help="forms to time, the first is the headline; tc_split@tc holds passes A, B, D on "
                         "tensor-core kernels")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the 512^3 and adjoint legs")
    ap.add_argument("--no-tune", action="store_true", help="time the default kernel schedule (no autotuning)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ref-budget", type=float, default=90.0)
    args = ap.parse_args()
    args.precisions = args.precisions.split(",")
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    global torch
    import torch
    dist_on = world > 1
    if args.impl == "reference":
        # rank 0 alone times the CPU reference; the other ranks exit without work
        run_reference(args, rank, world)
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if dist_on:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    try:
        run_ours(args, rank, world, dist_on)
    finally:
        if dist_on:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
