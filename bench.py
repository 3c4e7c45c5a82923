"""Throughput of the particle-mesh step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3] [--impl ours|reference]

One step = gather-kick + drift + rebin of every particle (updateVel +
moveParticles of the reference) followed by the scalar CIC deposit of the new
positions (scalarProjectionCIC_project + _comm): one fused lf2_step call.
Metric: particle updates per second, whole job (sum over ranks).

Workloads (seeded synthetic inputs; no dataset is involved):
  c3  512^3 lattice, 134,217,728 particles, log-normal clustering
      (rho ~ exp(2 delta_G - 2), delta_G Gaussian with P(k) ~ k^-2),
      int64 fixed-point deposit  [default: the size the throughput target is
      quoted on]
  c2  256^3, 16,777,216 particles, half uniform, half in 64 Gaussian clumps
      (sigma 0.01 box), FP32 deposit
  c5  768^3, 452,984,832 particles, 90% uniform + 10% in 1,000 halos
      (sigma 0.002 box), fixed-point deposit
Velocities N(0, 0.01^2) box units per time; drift dtau = 0.1 * 64/N so the
rms displacement per step (0.064 cells) matches the 64^3 reference case; the
kick uses the central-difference gradient of a Gaussian random field.

Multi-GPU (torchrun): every rank advances its own replica of the workload
(weak scaling, no collective on the data path); time is the max over ranks.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c3": dict(n=512, npart=512 ** 3, dist="lognormal", mode="fixed"),
    "c2": dict(n=256, npart=256 ** 3, dist="clumps", mode="fp32"),
    "c5": dict(n=768, npart=768 ** 3, dist="halos", mode="fixed"),
    "c1": dict(n=64, npart=64 ** 3, dist="uniform", mode="fp32"),
    # c3 statistics at 256^3 (16.8M particles): the size used for ncu captures
    "c3s": dict(n=256, npart=256 ** 3, dist="lognormal", mode="fixed"),
}
METRIC = "particle updates/s (CIC deposit+gather+move) & adjoint/forward time"
UNIT = "particle-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-projections", action="store_true",
                    help="skip timing the full-CIC vector and VecVec projections")
    ap.add_argument("--slab", action="store_true",
                    help="also time the step through a one-rank slab domain (ghost planes, "
                         "migration, folded deposit)")
    ap.add_argument("--no-pm", action="store_true",
                    help="skip timing the PM grid operator (FFT Poisson force)")
    ap.add_argument("--no-fp32", action="store_true",
                    help="skip the FP32-mode run of the same particles (fixed-point workloads)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling during the timed region (read-only query).  The raw
    samples go to LF2_CLOCKS_DIR (default: the system temp directory); the
    JSON line carries their summary."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(os.environ.get("LF2_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"lf2_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx = float(parts[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- workloads
def make_workload(name, device):
    import torch
    import latfield2_b200.workloads as W
    w = WORKLOADS[name]
    n = (w["n"],) * 3
    npart = w["npart"]
    if w["dist"] == "lognormal":
        cell, off = W.lognormal(n, npart, seed=3, device=device)
    elif w["dist"] == "clumps":
        cell, off = W.clumps(n, npart, 64, 0.01, seed=3, device=device)
    elif w["dist"] == "halos":
        cell, off = W.halos(n, npart, 1000, 0.002, seed=3, device=device)
    else:
        cell, off = W.uniform(n, npart, seed=3, device=device)
    vel = W.velocities(npart, 0.01, seed=4, device=device)
    F = W.grf_gradient(n, seed=2, device=device, amplitude=0.01)
    torch.cuda.synchronize() if device != "cpu" else None
    return n, cell, off, vel, F


def alg_bytes_move(npart, nsites):
    # particle state (int32 cell + 3 f32 offsets + 3 f32 velocities) read and
    # written once, 3-component field read once
    return npart * 56 + nsites * 12


def alg_bytes_deposit(npart, nsites):
    # cell + offsets read once, scalar density written once
    return npart * 16 + nsites * 4


def alg_bytes_step(npart, nsites):
    return npart * 56 + nsites * 4 * (1 + 3)


def traffic_from_profiles(kernel, workload):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload, {}).get(kernel)


# ------------------------------------------------------------ CPU baseline
def cpu_baseline_port(seconds, n_sample=64, npart_sample=64 ** 3, procs=1):
    """The oracle (reference restatement, double) on a bounded sample: a 64^3
    lattice with 262,144 particles (same one-particle-per-cell density),
    deposit + comm, updateVel with the CIC gather-kick, move; repeated until
    `seconds` of CPU work; `procs` independent processes."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.starmap(_cpu_worker, [(seconds, n_sample, npart_sample, 100 + i)
                                         for i in range(procs)])
    ups = sum(r[0] for r in res)
    steps = sum(r[1] for r in res)
    return ups, steps


def _cpu_worker(seconds, n, npart, seed):
    sys.path.insert(0, ROOT)
    import numpy as np
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    nn = (n, n, n)
    res = 1.0 / n
    pos = rng.random((npart, 3))
    vel = 0.01 * rng.standard_normal((npart, 3))
    u = np.floor(pos * n).astype(np.int64)
    cell = (u[:, 0] + n * (u[:, 1] + n * u[:, 2])).astype(np.int32)
    F = O.projection_init(nn, 1, 3)
    F[1:-1, 1:-1, 1:-1] = 0.01 * rng.standard_normal((n, n, n, 3))
    O.update_halo(F, nn, 1)
    dtau = 0.1
    steps = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds or steps == 0:
        cs, order = O.lists_from_insertion(nn, cell)
        pos, vel, cell = pos[order], vel[order], cell[order]
        O.scalar_cic(nn, 1, res, cs, pos, None, 1.0 / npart)
        O.update_vel_cic(nn, 1, cs, pos, vel, F, dtau)
        cell = O.move_simple(nn, 1.0, pos, vel, dtau)
        steps += 1
    dt = time.perf_counter() - t0
    return npart * steps / dt, steps


REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "lf2_ref_driver_double")


def _ref_grid(cores):
    """Largest power-of-two process grid g0 x g1 (both >= 2) with at most
    `cores` ranks (the MPI stand-in forks up to 64)."""
    best = None
    for g0 in (2, 4, 8):
        for g1 in (2, 4, 8):
            if g0 * g1 <= min(cores, 64) and (best is None or g0 * g1 > best[0] * best[1]):
                best = (g0, g1)
    return best


def _ref_run(inp, grid, steps, timeout):
    """One run of the reference driver's timing mode; its ranks form their own
    process group, stopped as a whole on a timeout."""
    import signal
    import subprocess
    env = dict(os.environ, LF2_MINIMPI_NP=str(grid[0] * grid[1]), LF2_REF_STEPS=str(steps))
    p = subprocess.Popen([REF_DRIVER, inp, inp + ".out"], env=env, stdin=subprocess.DEVNULL,
                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, start_new_session=True)
    try:
        out, _ = p.communicate(timeout=timeout)
    except subprocess.TimeoutExpired:
        os.killpg(p.pid, signal.SIGKILL)
        p.wait()
        return None
    if p.returncode != 0:
        return None
    for line in out.decode().splitlines():
        if line.startswith("{"):
            return json.loads(line)
    return None


def cpu_baseline_reference(seconds, cores, n=64, npart=64 ** 3):
    """The reference's own particle path (its headers compiled by
    oracle/build_ref.sh, double) on a bounded sample: a 64^3 lattice with
    262,144 uniform particles, K steps of scalarProjectionCIC_project + _comm,
    updateVel with the CIC kick and moveParticles, on a g0 x g1 process grid
    of forked ranks.  K is chosen for about `seconds` of work.  Returns
    (updates/s, steps, ranks) or None when the driver or 4 cores are not
    there."""
    import tempfile
    import numpy as np
    grid = _ref_grid(cores)
    if grid is None or not os.access(REF_DRIVER, os.X_OK):
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as G
    rng = np.random.default_rng(1)
    pos = rng.random((npart, 3))
    vel = 0.01 * rng.standard_normal((npart, 3))
    F = 0.01 * rng.standard_normal((n, n, n, 3))
    ids = np.arange(npart, dtype=np.int64)
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        G.write_input(inp, n, 1, grid, 1.0 / npart, G.OP_SCALAR | G.OP_KICK | G.OP_MOVE, 0.1, 0.1,
                      ids, pos, vel, F)
        probe = _ref_run(inp, grid, 5, 300)
        if probe is None:
            return None
        steps = max(5, min(5000, int(5 * seconds / max(probe["seconds"], 1e-6))))
        r = _ref_run(inp, grid, steps, 20 * seconds + 120)
        if r is None:
            return None
    return npart * r["steps"] / r["seconds"], r["steps"], r["ranks"]


def adjoint_ratio(device, steps=8, reps=3, operator="stencil"):
    """Differentiable chain at 128^3 with 2,097,152 uniform particles and
    per-particle masses (1/Np)(1 + 0.1 U(-1,1)): 8 kick-drift steps of
    deposit -> grid operator -> CIC gather -> kick -> drift, loss =
    sum w_g rho_g(final), particle checkpoints every 2 steps.  The grid
    operator is the periodic 27-point stencil (81 seeded weights) or, with
    operator "pm", the FFT Poisson force (coupling 4 pi).  Returns device
    times of the forward alone and of forward + adjoint (CUDA events, median
    of `reps`)."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import pm_chain_loss
    n, npart = 128, 1 << 21
    g = torch.Generator(device=device).manual_seed(41)
    pos = torch.rand(npart, 3, generator=g, device=device, dtype=torch.float64)
    vel = 0.01 * torch.randn(npart, 3, generator=g, device=device, dtype=torch.float64)
    m = (1.0 + 0.1 * (2 * torch.rand(npart, generator=g, device=device, dtype=torch.float64) - 1)) / npart
    S = 0.02 * torch.randn(81, generator=g, device=device, dtype=torch.float64)
    w = torch.randn(n ** 3, generator=g, device=device, dtype=torch.float64)
    ctx = L.Context((n, n, n), box=1.0)
    dt = 0.1 * 64.0 / n

    def timed(grad):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        leaves = [t.clone().requires_grad_(grad) for t in (pos, vel, m, S, w)]
        torch.cuda.synchronize()
        e0.record()
        if operator == "pm":
            loss = pm_chain_loss(ctx, leaves[0], leaves[1], leaves[2], None, leaves[4],
                                 steps=steps, dt=dt, checkpoint_every=2, operator="pm",
                                 coupling=4 * math.pi)
        else:
            loss = pm_chain_loss(ctx, *leaves, steps=steps, dt=dt, checkpoint_every=2)
        if grad:
            loss.backward()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    timed(True)
    fwd = sorted(timed(False) for _ in range(reps))[reps // 2]
    both = sorted(timed(True) for _ in range(reps))[reps // 2]
    ctx.close()
    return {"workload": "128^3, 2,097,152 particles, 8 steps, checkpoint every 2",
            "operator": "27-point stencil" if operator == "stencil" else "PM force (FFT)",
            "forward_ms": fwd, "forward_adjoint_ms": both, "ratio": both / fwd}


def reference_arm(args, rank):
    """The reference's CPU particle path on the host cores (rank 0 only): its
    own code compiled from its headers when oracle/_ref is there, else the C
    restatement of it (oracle/, one process per core)."""
    if rank != 0:
        return
    t0 = time.perf_counter()
    cores = os.cpu_count() or 1
    ref = cpu_baseline_reference(args.cpu_seconds, cores)
    if ref is not None:
        ups, steps, used = ref
        kind = "reference"
        sample = (f"{used} ranks ({_ref_grid(cores)[0]}x{_ref_grid(cores)[1]} process grid, forked "
                  f"MPI stand-in) x 64^3 lattice, 262,144 uniform particles, {steps} steps of "
                  "scalarProjectionCIC_project+_comm, updateVel CIC kick, moveParticles "
                  "(the reference's own headers, double)")
    else:
        used = cores
        ups, steps = cpu_baseline_port(args.cpu_seconds, procs=cores)
        kind = "port"
        sample = (f"{cores} processes x 64^3 lattice, 262,144 uniform particles, {steps} steps of "
                  "deposit+comm, updateVel CIC kick, move (CPU restatement of the reference, double)")
    wall = time.perf_counter() - t0
    w = WORKLOADS[args.workload]
    line = {
        "impl": "reference", "metric": METRIC, "value": ups, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "ms_per_step": 1e3 * w["npart"] / ups, "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": args.workload, "lattice": w["n"],
                                        "particles": w["npart"]},
        "cpu_baseline": {"value": ups, "unit": UNIT, "cores": used, "kind": kind, "sample": sample},
        "e2e": {"value": ups, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- ours
def e2e_pipelined(ctx, Fh, rho, F, n, nsites, npart, dtau, steps, pg, device, barrier):
    """Particle updates/s with the force field uploaded from pinned host memory
    and the density and max |v| downloaded to pinned host memory every step.
    Three streams: host->device copies of the next step's input, the step
    (lf2_field_import from the device copy, lf2_step, lf2_field_export to a
    device buffer, lf2_last_max_velocity), device->host copies of the
    result."""
    import numpy as np
    import torch
    from latfield2_b200 import _lib
    lib = _lib.load()
    Fref = np.ascontiguousarray(F.cpu().numpy().reshape(3, n[2], n[1], n[0]).transpose(1, 2, 3, 0))
    Fpin = torch.from_numpy(Fref).reshape(-1).pin_memory()  # reference layout (z, y, x, c)
    s_cmp, s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ctx.synchronize()
    ctx.set_stream(s_cmp.cuda_stream)
    Fd = [Fh, ctx.field(3)]
    Fin = [torch.empty(3 * nsites, device=device) for _ in range(2)]
    rho_dev = [torch.empty(nsites, device=device) for _ in range(2)]
    mv_dev = [torch.empty(1, dtype=torch.float64, device=device) for _ in range(2)]
    rho_pin = [torch.empty(nsites).pin_memory() for _ in range(2)]
    mv_pin = [torch.empty(1, dtype=torch.float64).pin_memory() for _ in range(2)]
    ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("in", "used", "res", "host")}

    def upload(k):
        b = k % 2
        if k >= 2:
            s_in.wait_event(ev["used"][b])  # step k-2 has read its input buffer
        with torch.cuda.stream(s_in):
            Fin[b].copy_(Fpin, non_blocking=True)
        ev["in"][b].record(s_in)

    def run(k):
        b = k % 2
        s_cmp.wait_event(ev["in"][b])
        if k >= 2:
            s_cmp.wait_event(ev["host"][b])  # step k-2's result has left the device buffer
        _lib.check(ctx.h, lib.lf2_field_import(ctx.h, Fd[b].h, ctypes.c_void_p(Fin[b].data_ptr()), 0, 4,
                                               _lib.PTR_DEVICE), "import")
        ev["used"][b].record(s_cmp)
        ctx.step(Fd[b], dtau, dtau, rho)
        _lib.check(ctx.h, lib.lf2_field_export(ctx.h, rho.h, ctypes.c_void_p(rho_dev[b].data_ptr()), 0, 4, 0,
                                               _lib.PTR_DEVICE), "export")
        ctx.last_max_velocity(mv_dev[b])
        ev["res"][b].record(s_cmp)
        s_out.wait_event(ev["res"][b])
        with torch.cuda.stream(s_out):
            rho_pin[b].copy_(rho_dev[b], non_blocking=True)
            mv_pin[b].copy_(mv_dev[b], non_blocking=True)
        ev["host"][b].record(s_out)

    def loop(k_steps):
        upload(0)
        for k in range(k_steps):
            if k + 1 < k_steps:
                upload(k + 1)
            run(k)
        torch.cuda.synchronize()

    loop(2)  # warm-up: allocations and first copies
    barrier()
    t0 = time.perf_counter()
    loop(steps)
    t = time.perf_counter() - t0
    ctx.set_stream(None)
    assert np.isfinite(float(mv_pin[(steps - 1) % 2][0]))
    ms, value = replica_throughput(1e3 * t, npart, steps, pg, device)
    return {"value": value, "unit": UNIT, "h2d_bytes_per_step": 3 * nsites * 4,
            "d2h_bytes_per_step": nsites * 4 + 8, "ms_per_step": ms / steps, "steps": steps,
            "path": "per step: pinned host F -> device (copy stream), lf2_field_import + lf2_step + "
                    "lf2_field_export + lf2_last_max_velocity (compute stream), rho and max|v| -> "
                    "pinned host (copy stream); copies of step k+1's input and step k's result "
                    "overlap step k"}


def full_cic_projections(ctx, npart, nsites, peak, reps=5):
    """vectorProjectionCIC and VecVecProjectionCIC of the bench's particles
    (after the timed steps): mean over `reps` deposits after one warm-up call,
    tile pass and boundary fix-up timed by the library's phase events.
    Algorithmic bytes: each particle's key, offsets and velocities read once
    (28 B), the field written once (4 B per component and site); the inputs
    are larger than L2."""
    out = {}
    for name, comps in (("vector_cic", 3), ("vecvec_cic", 6)):
        f = ctx.field(comps)
        dep = getattr(ctx, "deposit_" + name)
        dep(f)
        ctx.synchronize()
        ctx.profile_read()
        ctx.profile(True)
        for _ in range(reps):
            dep(f)
        ctx.synchronize()
        ph = ctx.profile_read()
        ctx.profile(False)
        tile = ph["deposit_tile"][0] / reps
        fix = ph["deposit_fixup"][0] / reps
        ms = tile + fix
        ab = npart * 28 + nsites * 4 * comps
        out[name] = {"ms": ms, "tile_ms": tile, "fixup_ms": fix,
                     "particle_deposits_per_s": npart / (ms / 1e3), "alg_bytes": ab,
                     "achieved_gbs": ab / (ms / 1e3) / 1e9,
                     "frac_of_hbm": ab / (ms / 1e3) / 1e9 / peak}
        del f
    return out


def pm_operator(ctx, rho, n, nsites, peak, reps=5):
    """lf2_pm_force (R2C, Green's function, C2R, gradient) on the bench's own
    density, and the bare PlanFFT-style transforms, each the mean of `reps`
    calls after one warm-up, timed with CUDA events on the context's stream
    (the default stream).  Algorithmic bytes of the force: rho read once and
    the 3-component force written once (16 B per site); the FFT route itself
    moves at least 40 B per site (transform, Green's function, inverse,
    gradient)."""
    import torch
    if not (n[0] == n[1] == n[2]):
        return None
    F2 = ctx.field(3)
    k = ctx.kfield(1)
    back = ctx.field(1)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms = timed(lambda: ctx.pm_force(rho, F2, 1.0))
    fwd = timed(lambda: ctx.fft_forward(rho, k))
    bwd = timed(lambda: ctx.fft_backward(k, back))
    ctx.synchronize()
    ab = 16 * nsites
    del F2, k, back
    return {"ms": ms, "fft_forward_ms": fwd, "fft_backward_ms": bwd, "alg_bytes": ab,
            "achieved_gbs": ab / (ms / 1e3) / 1e9, "frac_of_hbm": ab / (ms / 1e3) / 1e9 / peak,
            "route_min_bytes": 40 * nsites,
            "route_frac_of_hbm": 40 * nsites / (ms / 1e3) / 1e9 / peak}


def slab_one_rank_ms(case, F, n, npart, dtau, warmup, steps, local):
    """The same particles and steps through latfield2_b200.distributed.SlabDomain
    with one rank (its neighbours are itself): kick-drift-rebin, ghost planes
    of F, migration through the periodic z face (extract/add) and the folded
    deposit.  CUDA events around `steps` steps after `warmup`."""
    import torch
    from latfield2_b200 import _lib
    from latfield2_b200.distributed import SlabDomain
    cell, off, vel = case
    d = SlabDomain(n, box=1.0, mode=_lib.DEPOSIT_FIXED64, device=local)
    d.set_particles(cell.cpu().numpy(), off.cpu().numpy(), vel.cpu().numpy(), 1.0 / npart)
    Ff = d.field(3)
    Ff[0][:, 1:n[2] + 1] = F
    rho = d.field(1)
    for _ in range(warmup):
        d.step(Ff, dtau, dtau, rho)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        d.step(Ff, dtau, dtau, rho)
    e1.record()
    torch.cuda.synchronize()
    d.engine.synchronize()
    return e0.elapsed_time(e1) / steps


def fp32_step_ms(n, case, F, npart, dtau, warmup, steps, local):
    """Device time per lf2_step of the same particles with FP32 atomic
    deposits (CUDA events on the launching stream)."""
    import torch
    import latfield2_b200 as L
    cell, off, vel = case
    ctx = L.Context(n, box=1.0, mode=L.DEPOSIT_FP32, device=local)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / npart)
    Fh, rho = ctx.field(3, F), ctx.field(1)
    for _ in range(warmup):
        ctx.step(Fh, dtau, dtau, rho)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        ctx.step(Fh, dtau, dtau, rho)
    e1.record()
    torch.cuda.synchronize()
    ctx.synchronize()
    return e0.elapsed_time(e1) / steps


def replica_throughput(ms_local, npart, steps, pg=None, device="cpu"):
    """Whole-job time and throughput of N replicas: the time is the maximum
    over the ranks (every rank takes part in the same all-reduce), the
    throughput counts the particles of all ranks.  pg is torch.distributed
    (any backend) or None for one rank."""
    import torch
    world = 1
    ms = float(ms_local)
    if pg is not None:
        world = pg.get_world_size()
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    return ms, npart * world * steps / (ms / 1e3)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return reference_arm(args, rank)

    import numpy as np
    import torch
    import latfield2_b200 as L

    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    w = WORKLOADS[args.workload]
    mode = L.DEPOSIT_FIXED64 if w["mode"] == "fixed" else L.DEPOSIT_FP32
    n, cell, off, vel, F = make_workload(args.workload, device)
    npart = int(cell.shape[0])
    nsites = n[0] * n[1] * n[2]
    ctx = L.Context(n, box=1.0, mode=mode, device=local)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / npart)
    keep_case = (mode == L.DEPOSIT_FIXED64 and not args.no_fp32) or args.slab
    fp32_case = (cell, off, vel) if keep_case else None
    del cell, off, vel
    Fh = ctx.field(3, F)
    rho = ctx.field(1)
    torch.cuda.empty_cache()
    dtau = 0.1 * 64.0 / n[0]

    ctx.deposit_scalar(rho)
    for _ in range(args.warmup):
        ctx.step(Fh, dtau, dtau, rho)
    ctx.synchronize()
    ctx.profile_read()
    ctx.profile(True)
    l0 = ctx.kernel_launches()
    rb0 = ctx.rebin_stats()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            ctx.step(Fh, dtau, dtau, rho)
        e1.record()
        torch.cuda.synchronize()
        barrier()
    launches = ctx.kernel_launches() - l0
    rb1 = ctx.rebin_stats()
    rebin = {"repacks": rb1[0] - rb0[0], "relocations": rb1[1] - rb0[1],
             "movers_last_step": rb1[2]}
    ctx.synchronize()  # raises if a kernel flagged an error
    ms = e0.elapsed_time(e1)
    phases = ctx.profile_read()
    ctx.profile(False)
    ms, value = replica_throughput(ms, npart, args.steps, pg, device)
    ms_step = ms / args.steps

    # dominant kernel and its roofline (algorithmic bytes per launch / mean launch time)
    peak, peak_kind = peaks()
    dom = max(("move", "deposit_tile"), key=lambda p: phases[p][0])
    per_launch_ms = phases[dom][0] / max(1, phases[dom][1])
    if dom == "move":
        ab = alg_bytes_move(npart, nsites)
        kname = "k_move_pipe" if ctx.last_move_kernel() == 2 else "k_move<kick,drift>"
    else:
        ab = alg_bytes_deposit(npart, nsites)
        kname = "k_deposit<scalar>"
    achieved = ab / (per_launch_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "alg_bytes_per_launch": ab, "ms_per_launch": per_launch_ms,
                "traffic": traffic_from_profiles(kname, args.workload)}
    step_ab = alg_bytes_step(npart, nsites)
    step_roofline = {"alg_bytes": step_ab, "achieved": step_ab / (ms_step / 1e3) / 1e9,
                     "frac": step_ab / (ms_step / 1e3) / 1e9 / peak}
    phase_ms = {k: v[0] / args.steps for k, v in phases.items()}

    # End to end through the C ABI with host buffers: every step the force
    # field comes from pinned host memory (the reference layout) and the
    # density and max |v| go back to pinned host memory.  The copies of step
    # k+1's input and of step k's result run on their own streams while step
    # k computes (two buffers each way).
    e2e = e2e_pipelined(ctx, Fh, rho, F, n, nsites, npart, dtau, args.e2e_steps, pg, device, barrier)

    proj = None if args.no_projections else full_cic_projections(ctx, npart, nsites, peak)
    pm = None if args.no_pm else pm_operator(ctx, rho, n, nsites, peak)

    adj = adjoint_ratio(device) if (rank == 0 and not args.no_adjoint) else None
    adj_pm = (adjoint_ratio(device, operator="pm")
              if (rank == 0 and not args.no_adjoint and not args.no_pm) else None)

    slab = None
    if args.slab and fp32_case is not None:
        sms = slab_one_rank_ms(fp32_case, F, n, npart, dtau, args.warmup, min(args.steps, 5), local)
        slab = {"ms_per_step": sms, "vs_lf2_step": sms / ms_step, "ranks": 1,
                "note": "one self-exchanging rank; the exchange calls run, no peer"}
        torch.cuda.empty_cache()

    # the same particles and steps with FP32 atomic deposits
    fixed_vs_fp32 = None
    if fp32_case is not None and not args.no_fp32 and mode == L.DEPOSIT_FIXED64:
        del ctx, Fh, rho
        torch.cuda.empty_cache()
        ms32 = fp32_step_ms(n, fp32_case, F, npart, dtau, args.warmup, args.steps, local)
        ms32, _ = replica_throughput(ms32 * args.steps, npart, args.steps, pg, device)
        ms32 /= args.steps
        fixed_vs_fp32 = {"fixed_ms_per_step": ms_step, "fp32_ms_per_step": ms32,
                         "ratio": ms_step / ms32}
    del fp32_case

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            ref = cpu_baseline_reference(args.cpu_seconds, 4)
            if ref is not None:
                ups, steps, used = ref
                cpu = {"value": ups, "unit": UNIT, "cores": used, "kind": "reference",
                       "sample": f"{used} ranks (2x2 process grid) x 64^3 lattice, 262,144 uniform "
                                 f"particles, {steps} steps of scalarProjectionCIC_project+_comm, "
                                 "updateVel CIC kick, moveParticles (the reference's own headers, "
                                 "double)"}
            else:
                ups, steps = cpu_baseline_port(args.cpu_seconds, procs=1)
                cpu = {"value": ups, "unit": UNIT, "cores": 1, "kind": "port",
                       "sample": f"64^3 lattice, 262,144 uniform particles, {steps} steps of "
                                 "deposit+comm, updateVel CIC kick, move (CPU restatement of the "
                                 "reference, double, 1 thread)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (int64 fixed-point deposit)" if mode == L.DEPOSIT_FIXED64 else "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "lattice": n[0], "particles": npart,
                       "distribution": w["dist"], "deposit": w["mode"],
                       "step": "kick+drift+rebin+scalar deposit (lf2_step)",
                       "l2": f"inputs larger than L2 ({step_ab / 1e9:.1f} GB per step)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": roofline, "step_roofline": step_roofline, "phase_ms": phase_ms,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(),
            "gpu_launches": launches,
            "adjoint_forward_ratio": adj["ratio"] if adj else None, "adjoint": adj,
            "adjoint_pm": adj_pm,
            "fixed_vs_fp32": fixed_vs_fp32, "rebin": rebin, "projections": proj,
            "pm_operator": pm, "slab_one_rank": slab,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
