// lf2_deposit.cu -- CIC deposits of the brick-binned particles.
//
//   kind 0  scalar CIC        scalarProjectionCIC_project/_comm
//                             (projections.hpp:75-300), FP32 or int64 fixed point
//   kind 1  vector CIC-NGP    vectorProjectionCICNGP_project/_comm (:421-681)
//   kind 2  symtensor CIC-NGP symtensorProjectionCICNGP_project/_comm (:708-976)
//
// One CTA per brick accumulates its particles into a shared-memory tile of the
// (BRICK+1)^3 vertices they touch, then writes the tile once:
//   - vertices with every coordinate in [1, e-1] receive contributions from
//     this brick only, so their final value goes straight to the field;
//   - the other tile vertices (the "shell": a coordinate equal to 0 or to the
//     brick extent e) are written to a per-brick shell store.
// k_fixup then finishes every owned vertex with a zero coordinate by summing
// the shell values of the up to 8 bricks that touch it, in a fixed order.
// The periodic upper-halo fold of the reference's *_comm functions is thus
// part of the deposit, every vertex is written exactly once, no global
// atomics are used, and the fixed-point result is bit-exact run to run.
#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>

#include "lf2_internal.h"

namespace lf2 {

namespace {

#ifndef LF2_DEP_THREADS
#define LF2_DEP_THREADS 256
#endif
constexpr int DEP_THREADS = LF2_DEP_THREADS;

template <int KIND>
struct Comps;
template <>
struct Comps<0> { static constexpr int value = 1; };
template <>
struct Comps<1> { static constexpr int value = 3; };
template <>
struct Comps<2> { static constexpr int value = 6; };

__device__ __forceinline__ float sel(int b, float up, float dn) { return b ? up : dn; }

// Fixed-point accumulation in shared memory.  Each 64-bit vertex sum is kept
// as two 32-bit partial sums, lo = sum(q & 0xffff) and hi = sum(q >> 16), so
// that every update is a native 32-bit shared-memory reduction; the sum is
// lo + (hi << 16).  With q <= 2^32 per particle and corner, neither partial
// sum can wrap while a brick holds at most 65535 particles (DEP_SPLIT_MAX);
// larger bricks fall back to 64-bit shared atomics.
constexpr int DEP_SPLIT_MAX = 65535;
constexpr int DEP_ITEMS = 4;  // particles in flight per thread

template <bool SPLIT>
__device__ __forceinline__ void add_fixed(unsigned char* smem, int t, uint64_t q)
{
  if (SPLIT) {
    uint32_t* lo = reinterpret_cast<uint32_t*>(smem);
    uint32_t* hi = lo + TILE3;
    atomicAdd(&lo[t], (uint32_t)(q & 0xffffu));
    atomicAdd(&hi[t], (uint32_t)(q >> 16));
  } else {
    atomicAdd(reinterpret_cast<unsigned long long*>(smem) + t, (unsigned long long)q);
  }
}

template <bool SPLIT>
__device__ __forceinline__ void deposit_fixed_particle(unsigned char* smem, int t0, float fx,
                                                       float fy, float fz, bool has_mass,
                                                       uint64_t mq)
{
  // 1-D weights in units of 2^-31 (lf2o_fixed_weight in the oracle).
  const uint32_t ux = __float2uint_rn(fx * 2147483648.0f);
  const uint32_t uy = __float2uint_rn(fy * 2147483648.0f);
  const uint32_t uz = __float2uint_rn(fz * 2147483648.0f);
  const uint32_t qx[2] = {(1u << 31) - ux, ux};
  const uint32_t qy[2] = {(1u << 31) - uy, uy};
  const uint32_t qz[2] = {(1u << 31) - uz, uz};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
    uint64_t q = fixed_corner(qx[cx], qy[cy], qz[cz]);
    if (has_mass) q = (q * mq + (1ull << 23)) >> 24;
    add_fixed<SPLIT>(smem, t0 + cx + cy * TILE + cz * TILE * TILE, q);
  }
}

template <int KIND, bool FIXED>
__global__ void __launch_bounds__(DEP_THREADS) k_deposit(StoreView v, DepositParams dp,
                                                         float* __restrict__ out,
                                                         uint64_t* __restrict__ spill,
                                                         uint32_t* flags)
{
  constexpr int C = Comps<KIND>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];

  const Geom& g = v.g;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
            ez = brick_extent(g.n[2], bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  const bool split = FIXED && cnt <= DEP_SPLIT_MAX;

  {
    uint32_t* z = reinterpret_cast<uint32_t*>(smem_raw);
    const int words = FIXED ? 2 * TILE3 : C * TILE3;
    for (int t = threadIdx.x; t < words; t += blockDim.x) z[t] = 0u;
  }
  __syncthreads();

  float* facc = reinterpret_cast<float*>(smem_raw);
  for (int c0 = 0; c0 < cnt; c0 += DEP_ITEMS * DEP_THREADS) {
    uint32_t key[DEP_ITEMS];
    float fx[DEP_ITEMS], fy[DEP_ITEMS], fz[DEP_ITEMS], m[DEP_ITEMS];
    float vx[DEP_ITEMS], vy[DEP_ITEMS], vz[DEP_ITEMS];
#pragma unroll
    for (int j = 0; j < DEP_ITEMS; j++) {
      const int i = c0 + j * DEP_THREADS + threadIdx.x;
      if (i < cnt) {
        const int64_t p = base + i;
        key[j] = v.a.key[p];
        fx[j] = v.a.ox[p];
        fy[j] = v.a.oy[p];
        fz[j] = v.a.oz[p];
        m[j] = dp.has_mass ? v.a.mass[p] : 0.0f;
        if (KIND != 0) {
          vx[j] = v.a.vx[p];
          vy[j] = v.a.vy[p];
          vz[j] = v.a.vz[p];
        }
      }
    }
#pragma unroll
    for (int j = 0; j < DEP_ITEMS; j++) {
      const int i = c0 + j * DEP_THREADS + threadIdx.x;
      if (i >= cnt) continue;
      int x, y, z;
      unpack_key(g, key[j], x, y, z);
      const int t0 = (x - x0) + TILE * ((y - y0) + TILE * (z - z0));
      if (KIND == 0 && FIXED) {
        uint64_t mq = 0;
        if (dp.has_mass) {
          const float mr = __fmul_rn(m[j], dp.inv_unit);
          if (!(mr >= 0.0f && mr < 64.0f)) set_flag(flags, ERR_MASS_RANGE);
          mq = (uint64_t)__float2uint_rn(fminf(fmaxf(mr, 0.0f), 63.0f) * 16777216.0f);
        }
        if (split)
          deposit_fixed_particle<true>(smem_raw, t0, fx[j], fy[j], fz[j], dp.has_mass, mq);
        else
          deposit_fixed_particle<false>(smem_raw, t0, fx[j], fy[j], fz[j], dp.has_mass, mq);
        continue;
      }
      const float gx = __fsub_rn(1.0f, fx[j]), gy = __fsub_rn(1.0f, fy[j]),
                  gz = __fsub_rn(1.0f, fz[j]);
      const float ox = fx[j], oy = fy[j], oz = fz[j];
      const float mf = dp.has_mass ? __fmul_rn(m[j], dp.inv_vol) : dp.mf;
      if (KIND == 0) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
          const float w = __fmul_rn(
              __fmul_rn(__fmul_rn(sel(cx, ox, gx), sel(cy, oy, gy)), sel(cz, oz, gz)), mf);
          atomicAdd(&facc[t0 + cx + cy * TILE + cz * TILE * TILE], w);
        }
      } else if (KIND == 1) {
        // projections.hpp:501-544: component i is NGP along i, CIC across.
        const float vxm = __fmul_rn(mf, vx[j]);
        const float vym = __fmul_rn(mf, vy[j]);
        const float vzm = __fmul_rn(mf, vz[j]);
        constexpr int TY = TILE, TZ = TILE * TILE;
        float* a0 = facc;
        float* a1 = facc + TILE3;
        float* a2 = facc + 2 * TILE3;
        atomicAdd(&a0[t0], __fmul_rn(__fmul_rn(vxm, gy), gz));
        atomicAdd(&a0[t0 + TY], __fmul_rn(__fmul_rn(vxm, oy), gz));
        atomicAdd(&a0[t0 + TZ], __fmul_rn(__fmul_rn(vxm, gy), oz));
        atomicAdd(&a0[t0 + TY + TZ], __fmul_rn(__fmul_rn(vxm, oy), oz));
        atomicAdd(&a1[t0], __fmul_rn(__fmul_rn(vym, gx), gz));
        atomicAdd(&a1[t0 + 1], __fmul_rn(__fmul_rn(vym, ox), gz));
        atomicAdd(&a1[t0 + TZ], __fmul_rn(__fmul_rn(vym, gx), oz));
        atomicAdd(&a1[t0 + 1 + TZ], __fmul_rn(__fmul_rn(vym, ox), oz));
        atomicAdd(&a2[t0], __fmul_rn(__fmul_rn(vzm, gx), gy));
        atomicAdd(&a2[t0 + 1], __fmul_rn(__fmul_rn(vzm, ox), gy));
        atomicAdd(&a2[t0 + TY], __fmul_rn(__fmul_rn(vzm, gx), oy));
        atomicAdd(&a2[t0 + 1 + TY], __fmul_rn(__fmul_rn(vzm, ox), oy));
      } else {
        // projections.hpp:786-843: T_ii at the 8 vertices, T_ij on plaquettes.
        const float vv[3] = {vx[j], vy[j], vz[j]};
        constexpr int diag[3] = {0, 3, 5};
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const float mv2 = __fmul_rn(__fmul_rn(mf, vv[d]), vv[d]);
          float* a = facc + diag[d] * TILE3;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
            const float w = __fmul_rn(
                __fmul_rn(__fmul_rn(mv2, sel(cx, ox, gx)), sel(cy, oy, gy)), sel(cz, oz, gz));
            atomicAdd(&a[t0 + cx + cy * TILE + cz * TILE * TILE], w);
          }
        }
        const float m01 = __fmul_rn(__fmul_rn(mf, vv[0]), vv[1]);
        const float m02 = __fmul_rn(__fmul_rn(mf, vv[0]), vv[2]);
        const float m12 = __fmul_rn(__fmul_rn(mf, vv[1]), vv[2]);
        atomicAdd(&facc[1 * TILE3 + t0], __fmul_rn(m01, gz));
        atomicAdd(&facc[1 * TILE3 + t0 + TILE * TILE], __fmul_rn(m01, oz));
        atomicAdd(&facc[2 * TILE3 + t0], __fmul_rn(m02, gy));
        atomicAdd(&facc[2 * TILE3 + t0 + TILE], __fmul_rn(m02, oy));
        atomicAdd(&facc[4 * TILE3 + t0], __fmul_rn(m12, gx));
        atomicAdd(&facc[4 * TILE3 + t0 + 1], __fmul_rn(m12, ox));
      }
    }
  }
  __syncthreads();

  // Flush: interior vertices to the field, shell vertices to the shell store.
  uint64_t* sp = spill + (size_t)b * C * SHELL;
  const uint32_t* lo = reinterpret_cast<const uint32_t*>(smem_raw);
  const unsigned long long* a64 = reinterpret_cast<const unsigned long long*>(smem_raw);
  for (int t = threadIdx.x; t < TILE3; t += blockDim.x) {
    const int i = t % TILE, j = (t / TILE) % TILE, k = t / (TILE * TILE);
    if (i > ex || j > ey || k > ez) continue;
    const bool shell = i == 0 || i == ex || j == 0 || j == ey || k == 0 || k == ez;
    if (FIXED) {
      const uint64_t q = split ? (uint64_t)lo[t] + ((uint64_t)lo[TILE3 + t] << 16) : a64[t];
      if (shell) {
        sp[shell_index(i == ex ? BRICK : i, j == ey ? BRICK : j, k == ez ? BRICK : k)] = q;
      } else {
        if ((long long)q < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
        out[site_index(g, x0 + i, y0 + j, z0 + k)] = __fmul_rn(__ll2float_rn((long long)q),
                                                               dp.fixed_scale);
      }
      continue;
    }
    if (shell) {
      const int si = shell_index(i == ex ? BRICK : i, j == ey ? BRICK : j, k == ez ? BRICK : k);
#pragma unroll
      for (int c = 0; c < C; c++) reinterpret_cast<float*>(sp)[c * SHELL + si] = facc[c * TILE3 + t];
    } else {
      const int64_t s = site_index(g, x0 + i, y0 + j, z0 + k);
#pragma unroll
      for (int c = 0; c < C; c++) out[c * g.nsites + s] = facc[c * TILE3 + t];
    }
  }
}

// One CTA per brick: every owned vertex with a zero coordinate sums the shell
// values of the bricks that touch it: its own tile (subset 0) and, for every
// non-empty subset S of the dims where its coordinate is 0, the lower
// neighbour brick across S at tile coordinate BRICK in those dims.
template <int C, bool FIXED>
__global__ void k_fixup(Geom g, const uint64_t* __restrict__ spill, float fixed_scale,
                        float* __restrict__ out, uint32_t* flags)
{
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
            ez = brick_extent(g.n[2], bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int bxm = bx ? bx - 1 : g.nb[0] - 1;
  const int bym = by ? by - 1 : g.nb[1] - 1;
  const int bzm = bz ? bz - 1 : g.nb[2] - 1;
  const int nface = ey * ez + (ex - 1) * ez + (ex - 1) * (ey - 1);
  for (int f = threadIdx.x; f < nface; f += blockDim.x) {
    int i, j, k;
    if (f < ey * ez) {  // x face: i = 0
      i = 0;
      j = f % ey;
      k = f / ey;
    } else if (f < ey * ez + (ex - 1) * ez) {  // y face: j = 0, i >= 1
      const int r = f - ey * ez;
      j = 0;
      i = 1 + r % (ex - 1);
      k = r / (ex - 1);
    } else {  // z face: k = 0, i, j >= 1
      const int r = f - ey * ez - (ex - 1) * ez;
      k = 0;
      i = 1 + r % (ex - 1);
      j = 1 + r / (ex - 1);
    }
    const int zmask = (i == 0 ? 1 : 0) | (j == 0 ? 2 : 0) | (k == 0 ? 4 : 0);
    uint64_t qs[C];
    float fs[C];
#pragma unroll
    for (int c = 0; c < C; c++) {
      qs[c] = 0;
      fs[c] = 0.0f;
    }
    for (int s = 0; s < 8; s++) {
      if ((s & zmask) != s) continue;
      const int nbx = (s & 1) ? bxm : bx, nby = (s & 2) ? bym : by, nbz = (s & 4) ? bzm : bz;
      const int64_t nb = (int64_t)nbx + (int64_t)g.nb[0] * ((int64_t)nby + (int64_t)g.nb[1] * nbz);
      const int si = shell_index((s & 1) ? BRICK : i, (s & 2) ? BRICK : j, (s & 4) ? BRICK : k);
      const uint64_t* sp = spill + (size_t)nb * C * SHELL;
#pragma unroll
      for (int c = 0; c < C; c++) {
        if (FIXED)
          qs[c] += sp[c * SHELL + si];
        else
          fs[c] = __fadd_rn(fs[c], reinterpret_cast<const float*>(sp)[c * SHELL + si]);
      }
    }
    const int64_t site = site_index(g, x0 + i, y0 + j, z0 + k);
#pragma unroll
    for (int c = 0; c < C; c++) {
      if (FIXED) {
        const long long q = (long long)qs[c];
        if (q < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
        out[c * g.nsites + site] = __fmul_rn(__ll2float_rn(q), fixed_scale);
      } else {
        out[c * g.nsites + site] = fs[c];
      }
    }
  }
}

template <int KIND, bool FIXED>
cudaError_t run(lf2_ctx* c, float* out, const DepositParams& dp, int stage)
{
  constexpr int C = Comps<KIND>::value;
  const unsigned nb = (unsigned)c->g.nbricks;
  if (stage == 0) {
    const size_t smem = (size_t)C * TILE3 * (FIXED ? sizeof(unsigned long long) : sizeof(float));
    cudaError_t e = cudaFuncSetAttribute(k_deposit<KIND, FIXED>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    c->launches += 1;
    k_deposit<KIND, FIXED><<<nb, DEP_THREADS, smem, c->stream>>>(view(c), dp, out, c->spill,
                                                                 c->flags);
  } else {
    c->launches += 1;
    k_fixup<C, FIXED><<<nb, 256, 0, c->stream>>>(c->g, c->spill, dp.fixed_scale, out, c->flags);
  }
  return cudaGetLastError();
}

}  // namespace

// Shell-store slots (8 bytes each) a deposit of `comps` components needs.
size_t deposit_spill_slots(const lf2_ctx* c, int comps)
{
  return (size_t)c->g.nbricks * (size_t)comps * SHELL;
}

cudaError_t launch_deposit(lf2_ctx* c, int kind, float* out, int stage)
{
  DepositParams dp;
  const double vol = c->res * c->res * c->res;
  dp.inv_vol = (float)(1.0 / vol);
  dp.mf = (float)(c->gmass / vol);
  dp.fixed_scale = (float)(std::ldexp(1.0, -32) * c->m_unit / vol);
  dp.inv_unit = (float)(1.0 / c->m_unit);
  dp.has_mass = c->has_mass ? 1 : 0;
  const bool fixed = kind == 0 && c->mode == LF2_DEPOSIT_FIXED64;
  if (kind == 0) return fixed ? run<0, true>(c, out, dp, stage) : run<0, false>(c, out, dp, stage);
  if (kind == 1) return run<1, false>(c, out, dp, stage);
  return run<2, false>(c, out, dp, stage);
}

}  // namespace lf2
