"""Generates the golden fixtures of tests/golden/ by running the reference's
own particle path (oracle/_ref/lf2_ref_driver_{double,single}, compiled from
the reference headers by oracle/build_ref.sh) on seeded inputs.

    python tests/golden/make_golden.py

Each case writes <case>_<build>.npz with the inputs (lattice, particles,
force field, time steps) and the reference's outputs:
  rho, vec, ten     deposits after *_project + *_comm, interior sites,
                    shape (n, n, n, comps) indexed [z, y, x, c]
  vcic, vv          vectorProjectionCIC and VecVecProjectionCIC, same form
                    (multi-rank cases only: their halo folds need a 2x2 grid)
  fft_k             PlanFFT<Imag>::execute(FFT_FORWARD) of F[..., 0], the
                    global k-field in the reference's storage order
                    [ky][kz][kx] (kx = 0 .. n/2), complex
  fft_back          FFT_BACKWARD of that k-field (unnormalised), [z][y][x]
  poisson           the reference's Poisson example on F[..., 0] (res = 1/n)
  F_halo            the force field after Field::updateHalo, full gross array
                    (single-rank cases only)
  maxv, kick_*      updateVel with the CIC gather-kick callback
  move_*            moveParticles(move_particles_simple)
Particles are (id, pos[3], vel[3]) sorted by id.  Multi-rank cases run the
reference under the MPI stand-in with a 2x2 process grid (moveParticles
cannot run on a 1x1 grid: it receives from itself before sending).
"""
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

OP_SCALAR, OP_VECTOR, OP_TENSOR, OP_HALO, OP_KICK, OP_MOVE = 1, 2, 4, 8, 16, 32
OP_VECCIC, OP_VECVEC, OP_FFT, OP_POISSON = 64, 128, 256, 512
# fields in the order the driver writes them: (op, key, components)
FIELD_OPS = ((OP_SCALAR, "rho", 1), (OP_VECTOR, "vec", 3), (OP_TENSOR, "ten", 6),
             (OP_VECCIC, "vcic", 3), (OP_VECVEC, "vv", 6))

CASES = [
    # name, n, halo, grid, npart, clustered, vel sigma, dtau kick, dtau move, ops
    ("uniform8", 8, 1, (1, 1), 300, False, 0.05, 0.05, 0.0,
     OP_SCALAR | OP_VECTOR | OP_TENSOR | OP_HALO | OP_KICK | OP_FFT | OP_POISSON),
    ("clustered12", 12, 2, (1, 1), 2000, True, 0.2, 0.1, 0.0,
     OP_SCALAR | OP_VECTOR | OP_TENSOR | OP_HALO | OP_KICK),
    ("ranks16", 16, 1, (2, 2), 2500, True, 0.02, 0.05, 0.6,
     OP_SCALAR | OP_VECTOR | OP_TENSOR | OP_VECCIC | OP_VECVEC | OP_KICK | OP_MOVE | OP_FFT |
     OP_POISSON),
    ("ranks20", 20, 2, (2, 2), 3000, True, 0.3, 0.0, 0.0,
     OP_SCALAR | OP_VECCIC | OP_VECVEC),
]


def make_inputs(n, npart, clustered, vel_sigma, seed):
    rng = np.random.default_rng(seed)
    if clustered:
        centre = rng.random(3)
        pos = np.mod(centre + 0.1 * rng.standard_normal((npart, 3)), 1.0)
    else:
        pos = rng.random((npart, 3))
    vel = vel_sigma * rng.standard_normal((npart, 3))
    F = rng.standard_normal((n, n, n, 3))
    ids = rng.permutation(npart).astype(np.int64) + 1000
    return ids, pos, vel, F


def write_input(path, n, halo, grid, gmass, ops, dtk, dtm, ids, pos, vel, F):
    with open(path, "wb") as f:
        f.write(b"LF2G")
        f.write(struct.pack("<iiiii", 1, n, halo, grid[0], grid[1]))
        f.write(struct.pack("<ddi", 1.0, gmass, ops))
        f.write(struct.pack("<ddq", dtk, dtm, ids.shape[0]))
        rec = np.zeros(ids.shape[0], dtype=[("id", "<i8"), ("pv", "<f8", 6)])
        rec["id"] = ids
        rec["pv"][:, :3] = pos
        rec["pv"][:, 3:] = vel
        f.write(rec.tobytes())
        if ops & (OP_HALO | OP_KICK | OP_FFT | OP_POISSON):
            f.write(np.ascontiguousarray(F, "<f8").tobytes())


def read_rank(path, n, ops, comps_of):
    data = open(path, "rb").read()
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from(fmt, data, off)
        off += struct.calcsize(fmt)
        return v

    rank, skip0, skip1, s0, s1, s2, halo = take("<7i")
    out = {"rank": rank, "skip": (skip0, skip1), "size": (s0, s1, s2), "halo": halo}
    gross = (s0 + 2 * halo) * (s1 + 2 * halo) * (s2 + 2 * halo)

    def field(comps):
        nonlocal off
        a = np.frombuffer(data, "<f8", gross * comps, off).copy()
        off += 8 * gross * comps
        return a.reshape(s2 + 2 * halo, s1 + 2 * halo, s0 + 2 * halo, comps)

    def parts():
        nonlocal off
        (m,) = take("<q")
        rec = np.frombuffer(data, dtype=[("id", "<i8"), ("pv", "<f8", 6)], count=m, offset=off)
        off += m * 56
        return rec.copy()

    for op, _, comps in FIELD_OPS + ((OP_HALO, "F_halo", 3),):
        if ops & op:
            out[op] = field(comps)
    if ops & OP_FFT:
        k0, k1, k2, ks0, ks1 = take("<5i")
        kg = k0 * k1 * k2
        a = np.frombuffer(data, "<f8", 2 * kg, off).copy()
        off += 16 * kg
        out["k_size"], out["k_skip"] = (k0, k1, k2), (ks0, ks1)
        out[OP_FFT] = (a[0::2] + 1j * a[1::2]).reshape(k2, k1, k0)
        out["fft_back"] = field(1)
    if ops & OP_POISSON:
        out[OP_POISSON] = field(1)
    if ops & OP_KICK:
        (out["maxv"],) = take("<d")
        out[OP_KICK] = parts()
    if ops & OP_MOVE:
        out[OP_MOVE] = parts()
    return out


def assemble(ranks, n, op, comps):
    g = np.full((n, n, n, comps), np.nan)
    for r in ranks:
        h = r["halo"]
        s0, s1, s2 = r["size"]
        z0, y0 = r["skip"]
        g[z0:z0 + s2, y0:y0 + s1, 0:s0, :] = r[op][h:h + s2, h:h + s1, h:h + s0, :]
    assert not np.isnan(g).any()
    return g


def sorted_parts(ranks, op):
    rec = np.concatenate([r[op] for r in ranks])
    rec = rec[np.argsort(rec["id"], kind="stable")]
    return rec["id"], rec["pv"][:, :3].copy(), rec["pv"][:, 3:].copy()


def run_case(name, n, halo, grid, npart, clustered, vsig, dtk, dtm, ops, build, seed):
    ids, pos, vel, F = make_inputs(n, npart, clustered, vsig, seed)
    gmass = 1.0 / npart
    exe = os.path.join(REF, f"lf2_ref_driver_{build}")
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        write_input(inp, n, halo, grid, gmass, ops, dtk, dtm, ids, pos, vel, F)
        env = dict(os.environ, LF2_MINIMPI_NP=str(grid[0] * grid[1]))
        # the driver's ranks form their own process group: on a timeout the
        # whole group is stopped
        p = subprocess.Popen([exe, inp, os.path.join(td, "out")], env=env,
                             stdin=subprocess.DEVNULL, stdout=subprocess.DEVNULL)
        try:
            rc = p.wait(timeout=120)
        except subprocess.TimeoutExpired:
            os.killpg(p.pid, 9)
            p.wait()
            raise RuntimeError(f"{exe} timed out on case {name}")
        if rc != 0:
            raise RuntimeError(f"{exe} failed ({rc}) on case {name}")
        ranks = [read_rank(os.path.join(td, f"out.{r}"), n, ops, None)
                 for r in range(grid[0] * grid[1])]
    res = dict(n=n, halo=halo, grid=np.array(grid), gmass=gmass, dtau_kick=dtk, dtau_move=dtm,
               ops=ops, ids=ids, pos=pos, vel=vel, F=F)
    for op, key, comps in FIELD_OPS:
        if ops & op:
            res[key] = assemble(ranks, n, op, comps)
    if ops & OP_HALO:
        assert len(ranks) == 1
        res["F_halo"] = ranks[0][OP_HALO]
    if ops & OP_FFT:
        K = np.full((n, n, n // 2 + 1), np.nan + 0j)
        for r in ranks:
            k0, k1, k2 = r["k_size"]
            s0, s1 = r["k_skip"]
            K[s0:s0 + k2, s1:s1 + k1, :k0] = r[OP_FFT]
        assert not np.isnan(K).any()
        res["fft_k"] = K
        res["fft_back"] = assemble([dict(r, back=r["fft_back"]) for r in ranks], n, "back", 1)[..., 0]
    if ops & OP_POISSON:
        res["poisson"] = assemble(ranks, n, OP_POISSON, 1)[..., 0]
    if ops & OP_KICK:
        res["maxv"] = max(r["maxv"] for r in ranks)
        res["kick_id"], res["kick_pos"], res["kick_vel"] = sorted_parts(ranks, OP_KICK)
    if ops & OP_MOVE:
        res["move_id"], res["move_pos"], res["move_vel"] = sorted_parts(ranks, OP_MOVE)
    out = os.path.join(HERE, f"{name}_{build}.npz")
    np.savez_compressed(out, **res)
    return out


def main():
    if not os.path.exists(os.path.join(REF, "lf2_ref_driver_double")):
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True)
    for i, case in enumerate(CASES):
        for build in ("double", "single"):
            p = run_case(*case, build=build, seed=1000 + i)
            print(p, os.path.getsize(p))


if __name__ == "__main__":
    sys.exit(main())
