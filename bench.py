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

Multi-GPU (torchrun, N > 1): the workload is split into N z slabs, one per
rank (latfield2_b200.distributed.SlabDomain: ghost planes, migration, folded
deposit over NCCL), strong scaling; time is the max over ranks.
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
    ap.add_argument("--move-kernel", type=int, default=0,
                    help="lf2_set_move_kernel for the timed steps: 0 automatic, 1 per-brick, "
                         "2 pipelined, 3 pipelined with the fused deposit")
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


def _write_reference_input(path, name, grid, ops, dtau):
    """The workload's particles and force field for the reference driver,
    generated on the host from the bench's seeds (same generators, shapes and
    statistics as the GPU arm; torch's CPU and CUDA generators draw different
    numbers) and written in chunks: header, np x {id, pos[3], vel[3]}
    (double), F[z][y][x][c] (double)."""
    import struct
    import numpy as np
    import torch
    import latfield2_b200.workloads as W
    w = WORKLOADS[name]
    nn = w["n"]
    n = (nn,) * 3
    npart = w["npart"]
    if w["dist"] == "lognormal":
        cell, off = W.lognormal(n, npart, seed=3, device="cpu")
    elif w["dist"] == "clumps":
        cell, off = W.clumps(n, npart, 64, 0.01, seed=3, device="cpu")
    elif w["dist"] == "halos":
        cell, off = W.halos(n, npart, 1000, 0.002, seed=3, device="cpu")
    else:
        cell, off = W.uniform(n, npart, seed=3, device="cpu")
    vel = W.velocities(npart, 0.01, seed=4, device="cpu")
    F = W.grf_gradient(n, seed=2, device="cpu", amplitude=0.01)
    tmp = path + ".part"
    with open(tmp, "wb") as f:
        f.write(b"LF2G")
        f.write(struct.pack("<iiiii", 1, nn, 1, grid[0], grid[1]))
        f.write(struct.pack("<ddi", 1.0, 1.0 / npart, ops))
        f.write(struct.pack("<ddq", dtau, dtau, npart))
        ch = 1 << 23
        rec = torch.empty((ch, 7), dtype=torch.float64)  # id (int64 bits), pos[3], vel[3]
        for i0 in range(0, npart, ch):
            i1 = min(npart, i0 + ch)
            r = rec[:i1 - i0]
            c = cell[i0:i1].to(torch.int64)
            xyz = torch.stack([c % nn, (c // nn) % nn, c // (nn * nn)], 1).to(torch.float64)
            r[:, 1:4] = (xyz + off[i0:i1].to(torch.float64)) / nn
            r[:, 4:7] = vel[i0:i1].to(torch.float64)
            r.view(torch.int64)[:, 0] = torch.arange(i0, i1, dtype=torch.int64)
            f.write(r.numpy().tobytes())
        Fr = F.reshape(3, nn, nn, nn)
        for z in range(nn):
            f.write(Fr[:, z].permute(1, 2, 0).to(torch.float64).contiguous().numpy().tobytes())
    os.replace(tmp, path)
    del cell, off, vel, F
    torch.set_num_threads(torch.get_num_threads())


def cpu_reference_steps(name, cores, steps, warmup, timeout=1800):
    """The reference's own particle path (its headers compiled by
    oracle/build_ref.sh, double) on the full workload `name`: the driver's
    timing mode runs `warmup` untimed and then `steps` timed steps of
    scalarProjectionCIC_project + _comm, updateVel with the CIC kick and
    moveParticles, each step between two barriers, on the largest
    power-of-two process grid (both dims >= 2, moveParticles deadlocks on a
    grid dim of 1) within `cores` forked ranks.  The input file is kept in the
    temp directory for the next run on the same host.  Returns the driver's
    JSON record plus the grid and set-up time, or None."""
    import shutil
    grid = _ref_grid(cores)
    if grid is None or not os.access(REF_DRIVER, os.X_OK):
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as G
    w = WORKLOADS[name]
    npart, nn = w["npart"], w["n"]
    size = 68 + 56 * npart + 24 * nn ** 3
    tdir = os.environ.get("LF2_REF_INPUT_DIR", tempfile.gettempdir())
    path = os.path.join(tdir, f"lf2_ref_input_{name}_{grid[0]}x{grid[1]}.bin")
    t0 = time.perf_counter()
    if not (os.path.exists(path) and os.path.getsize(path) == size):
        if shutil.disk_usage(tdir).free < size * 1.2:
            return None
        _write_reference_input(path, name, grid, G.OP_KICK | G.OP_MOVE, 0.1 * 64.0 / nn)
    setup = time.perf_counter() - t0
    import signal
    env = dict(os.environ, LF2_MINIMPI_NP=str(grid[0] * grid[1]), LF2_REF_STEPS=str(steps),
               LF2_REF_WARMUP=str(warmup))
    p = subprocess.Popen([REF_DRIVER, path, path + ".out"], env=env, stdin=subprocess.DEVNULL,
                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, start_new_session=True)
    try:
        out, _ = p.communicate(timeout=timeout)
    except subprocess.TimeoutExpired:
        os.killpg(p.pid, signal.SIGKILL)
        p.wait()
        return None
    if p.returncode != 0:
        return None
    rec = None
    for line in out.decode().splitlines():
        if line.startswith("{"):
            rec = json.loads(line)
    if rec is None:
        return None
    rec.update(grid=grid, setup_s=setup, wall_s=time.perf_counter() - t0)
    return rec


def cpu_reference_summary(name, rec):
    w = WORKLOADS[name]
    per = rec["step_seconds"]
    return {
        "value": w["npart"] * rec["steps"] / rec["seconds"], "unit": UNIT,
        "cores": rec["ranks"], "kind": "reference",
        "sample": (f"the {name} workload itself ({w['n']}^3 lattice, {w['npart']:,} {w['dist']} "
                   f"particles): {rec['warmup']} untimed + {rec['steps']} timed steps of "
                   "scalarProjectionCIC_project + _comm, updateVel with the CIC kick, "
                   f"moveParticles; the reference's own headers (double) on {rec['ranks']} forked "
                   f"ranks ({rec['grid'][0]}x{rec['grid'][1]} process grid), one per host core"),
        "ms_per_step_median": 1e3 * statistics.median(per), "ms_per_step_min": 1e3 * min(per),
    }


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
    # one more forward + adjoint, outside the figures, in a range a profiler can select
    torch.cuda.nvtx.range_push("chain_adjoint_" + operator)
    timed(True)
    torch.cuda.nvtx.range_pop()
    ctx.close()
    return {"workload": "128^3, 2,097,152 particles, 8 steps, checkpoint every 2",
            "operator": "27-point stencil" if operator == "stencil" else "PM force (FFT)",
            "forward_ms": fwd, "forward_adjoint_ms": both, "ratio": both / fwd}


def workload_config(name):
    """The `config` both arms print: what the workload is, nothing about how an
    arm runs it (the deposit mode and the parallelism are separate keys)."""
    w = WORKLOADS[name]
    nsites = w["n"] ** 3
    return {"workload": name, "lattice": w["n"], "particles": w["npart"], "distribution": w["dist"],
            "step": "gather-kick + drift + rebin + scalar CIC deposit",
            "l2": f"inputs larger than L2 ({alg_bytes_step(w['npart'], nsites) / 1e9:.1f} GB per step)"}


def reference_arm(args, rank):
    """The reference's CPU particle path on the host cores (rank 0 only), on
    the same workload and with the same steps as the GPU arm: its own code
    compiled from its headers (oracle/_ref).  Without that build, the C
    restatement of it (oracle/) on a bounded sample."""
    if rank != 0:
        return
    t0 = time.perf_counter()
    cores = os.cpu_count() or 1
    rec = cpu_reference_steps(args.workload, cores, args.steps, args.warmup)
    if rec is not None:
        cpu = cpu_reference_summary(args.workload, rec)
        ups = cpu["value"]
        ms_step = 1e3 * rec["seconds"] / rec["steps"]
        extra = {"ms_per_step_median": cpu["ms_per_step_median"],
                 "ms_per_step_min": cpu["ms_per_step_min"], "setup_s": rec["setup_s"],
                 "parallelism": f"{rec['ranks']} MPI ranks ({rec['grid'][0]}x{rec['grid'][1]}), "
                                "one per host core"}
    else:
        ups, steps = cpu_baseline_port(args.cpu_seconds, procs=cores)
        cpu = {"value": ups, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{cores} processes x 64^3 lattice, 262,144 uniform particles, {steps} "
                         "steps of deposit+comm, updateVel CIC kick, move (CPU restatement of the "
                         "reference, double): a bounded sample, not the workload itself"}
        ms_step = 1e3 * 262144 / (ups / cores)
        extra = {"parallelism": f"{cores} processes"}
    line = {
        "impl": "reference", "metric": METRIC, "value": ups, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "ms_per_step": ms_step, "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": workload_config(args.workload),
        "deposit_mode": "double accumulation (the reference's default build)",
        "cpu_baseline": cpu,
        "e2e": {"value": ups, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t0,
    }
    line.update(extra)
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


PROJECTIONS = (("scalar", "deposit_scalar", 1, 16), ("vector_cicngp", "deposit_vector", 3, 28),
               ("symtensor_cicngp", "deposit_symtensor", 6, 28),
               ("vector_cic", "deposit_vector_cic", 3, 28), ("vecvec_cic", "deposit_vecvec_cic", 6, 28))


def projection_times(ctx, npart, nsites, peak, reps=5):
    """Every projection of the bench's particles in the context's deposit
    mode (after the timed steps): mean over `reps` deposits after one warm-up
    call; tile pass(es) and fix-up timed by the library's phase events.
    Algorithmic bytes: each particle's key and offsets (16 B), plus its
    velocities for momentum and stress (28 B), read once; the field written
    once (4 B per component and site).  The inputs are larger than L2."""
    out = {}
    for name, meth, comps, pb in PROJECTIONS:
        f = ctx.field(comps)
        dep = getattr(ctx, meth)
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
        ab = npart * pb + nsites * 4 * comps
        out[name] = {"ms": ms, "tile_ms": tile, "fixup_ms": fix,
                     "particle_deposits_per_s": npart / (ms / 1e3), "alg_bytes": ab,
                     "achieved_gbs": ab / (ms / 1e3) / 1e9,
                     "frac_of_hbm": ab / (ms / 1e3) / 1e9 / peak}
        del f
    return out


def fp64_density(cell, off, n, gmass):
    """FP64 CIC density of the particles (cell, off on the device), the
    measuring stick of the precision study: the weights of
    scalarProjectionCIC_project (projections.hpp:142-179) in double, summed
    with float64 atomics (torch index_add_), m / res^3 per particle."""
    import torch
    nsites = n[0] * n[1] * n[2]
    c = cell.to(torch.int64)
    x, y, z = c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1])
    o = off.to(torch.float64)
    rho = torch.zeros(nsites, dtype=torch.float64, device=cell.device)
    scale = gmass * n[0] * n[1] * n[2]  # m / res^3 in a unit box
    for k in range(8):
        bx, by, bz = (k >> 2) & 1, (k >> 1) & 1, k & 1
        w = ((o[:, 0] if bx else 1.0 - o[:, 0]) * (o[:, 1] if by else 1.0 - o[:, 1]) *
             (o[:, 2] if bz else 1.0 - o[:, 2]))
        idx = ((x + bx) % n[0]) + n[0] * (((y + by) % n[1]) + n[1] * ((z + bz) % n[2]))
        rho.index_add_(0, idx, w * scale)
        del w, idx
    return rho


def precision_stats(got, ref, floor_frac=1e-2):
    """Error of a density against the FP64 one: per vertex relative on the
    vertices above floor_frac of the mean density, and normalised by the
    field maximum (max and rms)."""
    import torch
    d = (got.to(torch.float64) - ref).abs()
    m = ref > floor_frac * ref.mean()
    rel = d[m] / ref[m]
    mx = ref.abs().max()
    return {"cell_max": float(rel.max()), "cell_rms": float(rel.square().mean().sqrt()),
            "norm_max": float(d.max() / mx), "norm_rms": float(d.square().mean().sqrt() / mx),
            "floor_frac": floor_frac, "cells_above_floor": int(m.sum())}


def precision_study(n, case, npart, local):
    """The density of the same particles in the three deposit modes against
    the FP64 one (C3: 512^3, 134M log-normal particles)."""
    import torch
    import latfield2_b200 as L
    cell, off, vel = case
    ref = fp64_density(cell, off, n, 1.0 / npart)
    out = {}
    for name, mode in (("fixed", L.DEPOSIT_FIXED64), ("fp32", L.DEPOSIT_FP32),
                       ("fp32_plain", L.DEPOSIT_FP32_PLAIN)):
        ctx = L.Context(n, box=1.0, mode=mode, device=local)
        ctx.set_particles(cell, off, vel, global_mass=1.0 / npart)
        rho = torch.empty(n[0] * n[1] * n[2], dtype=torch.float32, device=cell.device)
        ctx.deposit_scalar(ctx.field(1, rho))
        ctx.synchronize()
        out[name] = precision_stats(rho, ref)
        ctx.close()
        del rho
    del ref
    torch.cuda.empty_cache()
    out["reference"] = "FP64 CIC density of the same particles (torch float64 on the device)"
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
    torch.cuda.nvtx.range_push("slab_one_rank")  # the range a profiler can select
    e0.record()
    for _ in range(steps):
        d.step(Ff, dtau, dtau, rho)
    e1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    d.engine.synchronize()
    return e0.elapsed_time(e1) / steps


def fp32_step_ms(n, case, F, npart, dtau, warmup, steps, local, mode, proj_peak=None):
    """Device time per lf2_step of the same particles with an FP32 deposit
    mode (CUDA events on the launching stream); with proj_peak, also the
    projection times in that mode."""
    import torch
    import latfield2_b200 as L
    cell, off, vel = case
    ctx = L.Context(n, box=1.0, mode=mode, device=local)
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
    ms = e0.elapsed_time(e1) / steps
    proj = None
    if proj_peak is not None:
        del Fh, rho
        proj = projection_times(ctx, npart, n[0] * n[1] * n[2], proj_peak)
    ctx.close()
    return ms, proj


def chain_step_times(n, case, npart, local, reps=2):
    """One step of the differentiable particle-mesh chain on the workload's
    own particles (per-particle state, in a context of the fixed-point mode:
    the chain's deposits sum integer weights): deposit, PM force (FFT
    Poisson solve, coupling 4 pi), CIC gather, kick, drift and the final
    deposit of the loss, then its hand-written adjoint (autodiff.PMChain,
    checkpoint every step).  Device times (CUDA events) of the forward alone
    and of forward + adjoint, the median of `reps` after one warm-up."""
    import torch
    import latfield2_b200 as L
    from latfield2_b200.autodiff import pm_chain_loss
    cell, off, vel = case
    nn = n[0]
    c = cell.to(torch.int64)
    pos = torch.stack([c % nn, (c // nn) % nn, c // (nn * nn)], 1).to(torch.float64)
    del c
    pos.add_(off.to(torch.float64)).div_(nn)
    v = vel.to(torch.float64)
    m = torch.full((npart,), 1.0 / npart, dtype=torch.float64, device=pos.device)
    g = torch.Generator(device=pos.device).manual_seed(7)
    w = torch.randn(nn ** 3, generator=g, device=pos.device, dtype=torch.float64)
    ctx = L.Context(n, box=1.0, mode=L.DEPOSIT_FIXED64, device=local)  # fixed-point deposits
    dt = 0.1 * 64.0 / nn

    def timed(grad):
        leaves = [t.requires_grad_(grad) for t in (pos, v, m, w)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        loss = pm_chain_loss(ctx, leaves[0], leaves[1], leaves[2], None, leaves[3], steps=1, dt=dt,
                             checkpoint_every=1, operator="pm", coupling=4 * math.pi)
        if grad:
            loss.backward()
        e1.record()
        torch.cuda.synchronize()
        for t in leaves:
            t.grad = None
            t.requires_grad_(False)
        del loss
        return e0.elapsed_time(e1)

    timed(True)
    fwd = sorted(timed(False) for _ in range(reps))[reps // 2]
    both = sorted(timed(True) for _ in range(reps))[reps // 2]
    ctx.close()
    del pos, v, m, w
    torch.cuda.empty_cache()
    return {"workload": f"{nn}^3, {npart:,} particles, 1 step, PM force (FFT), checkpoint every step",
            "forward_ms": fwd, "forward_adjoint_ms": both, "ratio": both / fwd}


def slab_scaling(args, n, cell, off, vel, F, npart, dtau, local, pg, device):
    """N > 1: the workload split into N z slabs, one per rank
    (latfield2_b200.distributed.SlabDomain): ghost planes of F, kick-drift-
    rebin, particle migration between neighbours and the folded fixed-point
    deposit every step, over NCCL.  Strong scaling: the same lattice and
    particles whatever N.  Device time per step is the maximum over ranks."""
    import torch
    from latfield2_b200 import _lib
    from latfield2_b200.distributed import SlabDomain
    d = SlabDomain(n, box=1.0, mode=_lib.DEPOSIT_FIXED64, device=local)
    d.set_particles(cell.cpu().numpy(), off.cpu().numpy(), vel.cpu().numpy(), 1.0 / npart)
    Ff = d.field(3)
    Ff[0][:, 1:d.nz + 1] = F.reshape(3, n[2], n[1], n[0])[:, d.z0:d.z0 + d.nz]
    rho = d.field(1)
    for _ in range(args.warmup):
        d.step(Ff, dtau, dtau, rho)
    torch.cuda.synchronize()
    pg.barrier()
    l0 = d.engine.ctx.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        d.step(Ff, dtau, dtau, rho)
    e1.record()
    torch.cuda.synchronize()
    launches = d.engine.ctx.kernel_launches() - l0
    pg.barrier()
    ms, value = replica_throughput(e0.elapsed_time(e1), npart, args.steps, pg, device)
    value /= pg.get_world_size()  # one set of particles for the whole job

    # end to end: every step the rank's planes of F come from pinned host
    # memory and its planes of rho go back to pinned host memory
    own_F = Ff[0][:, 1:d.nz + 1]
    F_pin = own_F.cpu().pin_memory()
    rho_pin = torch.empty(tuple(rho[0][:, 1:d.nz + 1].shape), dtype=torch.float32).pin_memory()
    k = max(1, args.e2e_steps)
    torch.cuda.synchronize()
    pg.barrier()
    t0 = time.perf_counter()
    for _ in range(k):
        own_F.copy_(F_pin, non_blocking=True)
        d.step(Ff, dtau, dtau, rho)
        rho_pin.copy_(rho[0][:, 1:d.nz + 1], non_blocking=True)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    ms_e2e, v_e2e = replica_throughput(1e3 * t, npart, k, pg, device)
    e2e = {"value": v_e2e / pg.get_world_size(), "unit": UNIT,
           "h2d_bytes_per_step": int(F_pin.numel()) * 4 * pg.get_world_size(),
           "d2h_bytes_per_step": int(rho_pin.numel()) * 4 * pg.get_world_size(),
           "ms_per_step": ms_e2e / k, "steps": k,
           "path": "per step on every rank: its planes of F from pinned host memory, "
                   "SlabDomain.step, its planes of rho to pinned host memory (one stream)"}
    return ms / args.steps, value, d.count(), launches, e2e


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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    w = WORKLOADS[args.workload]
    mode = L.DEPOSIT_FIXED64 if w["mode"] == "fixed" else L.DEPOSIT_FP32
    n, cell, off, vel, F = make_workload(args.workload, device)
    npart = int(cell.shape[0])
    nsites = n[0] * n[1] * n[2]
    if world > 1:
        # the domain decomposition over the ranks (strong scaling)
        peak, peak_kind = peaks()
        dtau = 0.1 * 64.0 / n[0]
        with ClockSampler(local) as clocks:
            ms_step, value, local_count, launches, e2e = slab_scaling(args, n, cell, off, vel, F,
                                                                      npart, dtau, local, pg, device)
        if rank == 0:
            step_ab = alg_bytes_step(npart, nsites)
            line = {
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32 (int64 fixed-point deposit)",
                "data": "synthetic (seeded)", "config": workload_config(args.workload),
                "deposit_mode": "fixed (int64 fixed point)",
                "parallelism": f"z slabs over {world} GPUs (SlabDomain: ghost planes, migration, "
                               "folded deposit; NCCL point-to-point)",
                "roofline": {"bound": "hbm", "kernel": "whole step", "unit": "GB/s",
                             "achieved": step_ab / (ms_step / 1e3) / 1e9, "peak": peak * world,
                             "frac": step_ab / (ms_step / 1e3) / 1e9 / (peak * world),
                             "peak_source": peak_kind, "traffic": None},
                "cpu_baseline": None, "e2e": e2e, "clocks": clocks.summary(),
                "gpu_launches": launches, "particles_rank0": local_count,
            }
            print(json.dumps(line), flush=True)
        pg.barrier()
        pg.destroy_process_group()
        return
    ctx = L.Context(n, box=1.0, mode=mode, device=local)
    ctx.set_particles(cell, off, vel, global_mass=1.0 / npart)
    ctx.set_move_kernel(args.move_kernel)
    keep_case = (mode == L.DEPOSIT_FIXED64 and not args.no_fp32) or args.slab or args.workload == "c5"
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

    # one event between consecutive steps (the library runs on torch's current
    # stream): the total over the K steps and each step's own time
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    e0, e1 = evs[0], evs[-1]
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        e0.record()
        for k in range(args.steps):
            ctx.step(Fh, dtau, dtau, rho)
            evs[k + 1].record()
        torch.cuda.synchronize()
        barrier()
    step_times = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
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
    mk = ctx.last_move_kernel()
    if dom == "move":
        ab = alg_bytes_move(npart, nsites)
        kname = {1: "k_move<kick,drift>", 2: "k_move_pipe"}.get(mk, "k_move_pipe<fused deposit>")
        if mk == 3:
            ab += nsites * 4  # the density is written by the same pass (rim vertices later)
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

    proj = None if args.no_projections else {w["mode"]: projection_times(ctx, npart, nsites, peak)}
    pm = None if args.no_pm else pm_operator(ctx, rho, n, nsites, peak)

    adj = adjoint_ratio(device) if (rank == 0 and not args.no_adjoint) else None
    adj_pm = (adjoint_ratio(device, operator="pm")
              if (rank == 0 and not args.no_adjoint and not args.no_pm) else None)

    slab = None
    if args.slab and fp32_case is not None:
        sms = slab_one_rank_ms(fp32_case, F, n, npart, dtau, args.warmup, min(args.steps, 10), local)
        slab = {"ms_per_step": sms, "vs_lf2_step": sms / ms_step, "ranks": 1,
                "note": "one self-exchanging rank; the exchange calls run, no peer"}
        torch.cuda.empty_cache()

    # the same particles and steps with the FP32 deposit modes: compensated
    # atomics (within 1e-6) and the plain FP32-atomic form
    fixed_vs_fp32 = None
    precision = None
    if fp32_case is not None and not args.no_fp32 and mode == L.DEPOSIT_FIXED64:
        ctx.close()
        del ctx, Fh, rho
        torch.cuda.empty_cache()
        res32 = {}
        for nm, md in (("fp32", L.DEPOSIT_FP32), ("fp32_plain", L.DEPOSIT_FP32_PLAIN)):
            ms32, p32 = fp32_step_ms(n, fp32_case, F, npart, dtau, args.warmup, args.steps, local, md,
                                     None if args.no_projections else peak)
            ms32, _ = replica_throughput(ms32 * args.steps, npart, args.steps, pg, device)
            res32[nm] = ms32 / args.steps
            if proj is not None and p32 is not None:
                proj[nm] = p32
            torch.cuda.empty_cache()
        fixed_vs_fp32 = {"fixed_ms_per_step": ms_step, "fp32_ms_per_step": res32["fp32"],
                         "fp32_plain_ms_per_step": res32["fp32_plain"],
                         "ratio": ms_step / res32["fp32"],
                         "ratio_vs_plain": ms_step / res32["fp32_plain"]}
        if args.workload in ("c3", "c3s"):
            precision = precision_study(n, fp32_case, npart, local)
    # C5: the full forward + adjoint step of the differentiable chain on the
    # same particles, beside the library's fixed-point and plain FP32 forward
    c5 = None
    if args.workload == "c5" and fp32_case is not None and not args.no_adjoint and world == 1:
        if "ctx" in locals():  # the step's store and fields make room for the chain's state
            ctx.close()
            del ctx, Fh, rho
            torch.cuda.empty_cache()
        try:
            chain = chain_step_times(n, fp32_case, npart, local)
        except torch.cuda.OutOfMemoryError as e:  # the chain keeps every field of the step
            torch.cuda.empty_cache()
            chain = {"unavailable": f"out of device memory: {str(e).splitlines()[0]}",
                     "forward_adjoint_ms": None}
        c5 = {"forward_ms": ms_step,
              "fp32_forward_ms": fixed_vs_fp32["fp32_plain_ms_per_step"] if fixed_vs_fp32 else None,
              "forward_adjoint_ms": chain["forward_adjoint_ms"], "chain": chain,
              "note": "forward_ms: lf2_step (kick, drift, rebin, fixed-point deposit); "
                      "fp32_forward_ms: the same with the plain FP32-atomic deposit; "
                      "forward_adjoint_ms: one step of the differentiable chain (fixed-point deposits) "
                      "and its adjoint (chain.forward_ms its forward alone)"}
    del fp32_case

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            # the reference on the same workload and host cores as the reference
            # arm, bounded to one untimed and two timed steps
            rec = cpu_reference_steps(args.workload, os.cpu_count() or 1, 2, 1)
            if rec is not None:
                cpu = cpu_reference_summary(args.workload, rec)
            else:
                ups, steps = cpu_baseline_port(args.cpu_seconds, procs=1)
                cpu = {"value": ups, "unit": UNIT, "cores": 1, "kind": "port",
                       "sample": f"64^3 lattice, 262,144 uniform particles, {steps} steps of "
                                 "deposit+comm, updateVel CIC kick, move (CPU restatement of the "
                                 "reference, double, 1 thread): a bounded sample, not the workload"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "ms_per_step_median": statistics.median(step_times), "ms_per_step_min": min(step_times),
            "dtype": "f32 (int64 fixed-point deposit)" if mode == L.DEPOSIT_FIXED64 else "f32",
            "data": "synthetic (seeded)",
            "config": workload_config(args.workload),
            "deposit_mode": w["mode"] + (" (int64 fixed point)" if w["mode"] == "fixed" else ""),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "roofline": roofline, "step_roofline": step_roofline, "phase_ms": phase_ms,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(),
            "gpu_launches": launches,
            "adjoint_forward_ratio": adj["ratio"] if adj else None, "adjoint": adj,
            "adjoint_pm": adj_pm,
            "fixed_vs_fp32": fixed_vs_fp32, "precision": precision, "rebin": rebin,
            "projections": proj,
            "pm_operator": pm, "slab_one_rank": slab, "c5": c5,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
