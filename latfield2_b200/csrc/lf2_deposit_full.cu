// lf2_deposit_full.cu -- the full-CIC (staggered) projections of the
// brick-binned particles.
//
//   kind 3  vector CIC   vectorProjectionCIC_project/_comm (projections.hpp:978-1349)
//   kind 4  VecVec CIC   VecVecProjectionCIC_project/_comm (:1355-1814)
//
// Component c of the vector field (m v_c / res^3) lives on the link
// x + e_c/2 and is stored at site x; T_ij (i < j) lives on the plaquette
// centre x + (e_i + e_j)/2 and T_ii on the vertex, both stored at site x.
// Along a staggered dim a particle in cell l at in-cell offset o lies between
// the links of sites l - 1 + g and l + g, g = (o >= 1/2); with s = o - 1/2 the
// lower link gets td = (g ? 1 - s : -s), the upper one tu = 1 - td.  Along a
// vertex dim the weights are the ordinary CIC ones, 1 - o at l and o at l + 1.
//
// One CTA per brick accumulates its particles (FP32 shared atomics) into a
// tile of (BRICK+2)^3 vertices per component whose origin is one site below
// the brick, so the lower staggered neighbours are inside it (three
// components per pass; VecVec takes two passes).  The flush then writes
//   - every vertex the brick owns (tile coordinates 1..e in all dims) to the
//     field: the final value for the interior, a partial sum on the brick's
//     boundary;
//   - the outer layer (a tile coordinate 0 or e+1) to a per-brick store.
// k_fixup_full adds, to every owned boundary vertex, the outer-layer values
// of the up to 26 neighbour bricks that reach it, in a fixed order.  This is
// the periodic fold of both halos that the reference's *_comm functions do;
// no global atomics are used and no field has to be cleared first.
//
// The three deposit modes of lf2_deposit.cu apply here too.  The plain FP32
// mode keeps one word per vertex and writes the brick's own boundary
// vertices to the field as partial sums, which the fix-up completes.  The
// compensated FP32 and the fixed-point modes keep two words per vertex (the
// hi/lo pair, or the split integer sum) and write every tile vertex that
// another brick can reach -- the own boundary vertices (tile coordinate 1 or
// e) and the outer layer (0 or e+1), a shell two vertices thick -- to the
// store; the fix-up then sums the own and the neighbours' values in one
// fixed order (exact integers, or a compensated FP32 sum) and writes the
// boundary vertices once.
#include <cuda_runtime.h>

#include <type_traits>

#include "lf2_deposit_common.cuh"
#include "lf2_internal.h"

namespace lf2 {

namespace {

constexpr int FT = BRICK + 2;                         // tile vertices per dim
constexpr int FT3 = FT * FT * FT;                     // 5832 for BRICK = 16
constexpr int FOUTER = FT3 - BRICK * BRICK * BRICK;   // outer layer, 1736

// The outer-layer store reuses the deposit shell store, which is sized for
// SHELL 8-byte slots per component and brick.
static_assert(FOUTER * sizeof(float) <= SHELL * sizeof(uint64_t), "outer store fits the shell store");

// Index of an outer-layer vertex (u0, u1, u2) of the canonical FT^3 tile, in
// which a tile coordinate equal to the brick extent + 1 has been mapped to
// FT - 1 (so bricks with e < BRICK use the same layout).  Slabs: the two z
// faces (2 FT^2), the two y faces without them (2 (FT-2) FT), the two x faces
// without either (2 (FT-2)^2).
__host__ __device__ inline int outer_index(int u0, int u1, int u2)
{
  if (u2 == 0 || u2 == FT - 1) return (u2 != 0) * FT * FT + u1 * FT + u0;
  if (u1 == 0 || u1 == FT - 1) return 2 * FT * FT + ((u1 != 0) * (FT - 2) + (u2 - 1)) * FT + u0;
  return 2 * FT * FT + 2 * (FT - 2) * FT + ((u0 != 0) * (FT - 2) + (u2 - 1)) * (FT - 2) + (u1 - 1);
}

static_assert(2 * FT * FT + 2 * (FT - 2) * FT + 2 * (FT - 2) * (FT - 2) == FOUTER,
              "outer slab sizes");

// The shell two vertices thick of the compensated and fixed-point modes:
// tile vertices with a coordinate in {0, 1, e, e+1}.  Canonical coordinates
// map e to FT - 2 and e + 1 to FT - 1 (so bricks with e < BRICK share one
// layout); the shell is the two z slabs pairs (4 FT^2), then the y slab pairs
// between them (4 (FT-4) FT), then the x slab pairs between those
// (4 (FT-4)^2): 3088 slots for BRICK = 16.
constexpr int FSHELL = FT3 - (FT - 4) * (FT - 4) * (FT - 4);
static_assert(4 * FT * FT + 4 * (FT - 4) * FT + 4 * (FT - 4) * (FT - 4) == FSHELL, "thick slabs");

__host__ __device__ inline int canon(int t, int e) { return t == e + 1 ? FT - 1 : (t == e ? FT - 2 : t); }
__host__ __device__ inline bool in_thick(int u) { return u < 2 || u >= FT - 2; }
__host__ __device__ inline int thick_slot(int u) { return u < 2 ? u : u - (FT - 4); }

__host__ __device__ inline int thick_index(int u0, int u1, int u2)
{
  if (in_thick(u2)) return thick_slot(u2) * FT * FT + u1 * FT + u0;
  if (in_thick(u1)) return 4 * FT * FT + (thick_slot(u1) * (FT - 4) + (u2 - 2)) * FT + u0;
  return 4 * FT * FT + 4 * (FT - 4) * FT + (thick_slot(u0) * (FT - 4) + (u2 - 2)) * (FT - 4) + (u1 - 2);
}

// Threads per CTA of a tile pass.  Measured at 512^3: 512 (more warps on the
// same tiles) gave 5.39 ms against 5.11 ms for 256; the tile passes are bound
// by the shared atomic pipe, not by occupancy.
#ifndef LF2_FULL_THREADS
#define LF2_FULL_THREADS 256
#endif
constexpr int FULL_THREADS = LF2_FULL_THREADS;

// A tile pass accumulates three components (a 70 KB tile, 3 CTAs per SM):
//   pass 0  the vector field, components 0, 1, 2 of 3;
//   pass 1  VecVec T_00, T_11, T_22 (components 0, 3, 5 of 6), vertex CIC;
//   pass 2  VecVec T_01, T_02, T_12 (components 1, 2, 4 of 6) on plaquettes.
// Two passes for VecVec rather than one 140 KB six-component tile (one CTA
// per SM): the shared atomic pipe stays busier, at the cost of reading the
// particles twice.
template <int PASS>
struct FullPass {
  static constexpr int total = PASS == 0 ? 3 : 6;  // components of the field
  __device__ static constexpr int comp(int j)
  {
    return PASS == 0 ? j : PASS == 1 ? (j == 0 ? 0 : j == 1 ? 3 : 5) : (j == 0 ? 1 : j == 1 ? 2 : 4);
  }
};

__device__ __forceinline__ int tile_at(int t0, int t1, int t2) { return t0 + FT * (t1 + FT * t2); }

template <int PASS>
__global__ void __launch_bounds__(FULL_THREADS)
    k_deposit_full(StoreView v, DepositParams dp, float* __restrict__ out,
                   float* __restrict__ outer)
{
  constexpr int CT = FullPass<PASS>::total;
  extern __shared__ __align__(16) float tile[];

  const Geom& g = v.g;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int e[3] = {brick_extent(g.n[0], bx), brick_extent(g.n[1], by),
                    brick_extent(g.n[2], bz)};
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);

  for (int t = threadIdx.x; t < 3 * FT3; t += blockDim.x) tile[t] = 0.0f;
  __syncthreads();

  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int64_t p = base + i;
    int x, y, z;
    unpack_key(g, v.a.key[p], x, y, z);
    const float o[3] = {v.a.ox[p], v.a.oy[p], v.a.oz[p]};
    const float vel[3] = {v.a.vx[p], v.a.vy[p], v.a.vz[p]};
    const float mf = dp.has_mass ? __fmul_rn(v.a.mass[p], dp.inv_vol) : dp.mf;
    const int l[3] = {x - x0, y - y0, z - z0};
    // per dim: vertex weights (sd, su) at tile coordinates ls, ls + 1 and
    // staggered weights (td, tu) at lt, lt + 1
    float sw[3][2], tw[3][2];
    int ls[3], lt[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      sw[d][1] = o[d];
      sw[d][0] = __fsub_rn(1.0f, o[d]);
      const float s = __fsub_rn(o[d], 0.5f);
      const int gd = s >= 0.0f;
      if (gd) {
        tw[d][1] = s;
        tw[d][0] = __fsub_rn(1.0f, s);
      } else {
        tw[d][0] = -s;
        tw[d][1] = __fsub_rn(1.0f, tw[d][0]);
      }
      ls[d] = l[d] + 1;
      lt[d] = l[d] + gd;
    }
    if (PASS == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float mv = __fmul_rn(mf, vel[c]);
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int b0 = (k >> 2) & 1, b1 = (k >> 1) & 1, b2 = k & 1;
          const float w0 = c == 0 ? tw[0][b0] : sw[0][b0];
          const float w1 = c == 1 ? tw[1][b1] : sw[1][b1];
          const float w2 = c == 2 ? tw[2][b2] : sw[2][b2];
          const int t0 = (c == 0 ? lt[0] : ls[0]) + b0;
          const int t1 = (c == 1 ? lt[1] : ls[1]) + b1;
          const int t2 = (c == 2 ? lt[2] : ls[2]) + b2;
          atomicAdd(&tile[c * FT3 + tile_at(t0, t1, t2)],
                    __fmul_rn(__fmul_rn(__fmul_rn(mv, w0), w1), w2));
        }
      }
    } else if (PASS == 1) {
      // T_ii at the vertices
#pragma unroll
      for (int i2 = 0; i2 < 3; i2++) {
        const float m2 = __fmul_rn(__fmul_rn(mf, vel[i2]), vel[i2]);
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int b0 = (k >> 2) & 1, b1 = (k >> 1) & 1, b2 = k & 1;
          atomicAdd(&tile[i2 * FT3 + tile_at(ls[0] + b0, ls[1] + b1, ls[2] + b2)],
                    __fmul_rn(__fmul_rn(__fmul_rn(m2, sw[0][b0]), sw[1][b1]), sw[2][b2]));
        }
      }
    } else {
      // T_ij on the plaquettes: (0,1), (0,2), (1,2)
      constexpr int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float mm = __fmul_rn(__fmul_rn(mf, vel[pa[q]]), vel[pb[q]]);
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int bb[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
          float w[3];
          int t[3];
#pragma unroll
          for (int d = 0; d < 3; d++) {
            const bool st = d == pa[q] || d == pb[q];
            w[d] = st ? tw[d][bb[d]] : sw[d][bb[d]];
            t[d] = (st ? lt[d] : ls[d]) + bb[d];
          }
          atomicAdd(&tile[q * FT3 + tile_at(t[0], t[1], t[2])],
                    __fmul_rn(__fmul_rn(__fmul_rn(mm, w[0]), w[1]), w[2]));
        }
      }
    }
  }
  __syncthreads();

  float* os = outer + (size_t)b * CT * FOUTER;
  for (int t = threadIdx.x; t < FT3; t += blockDim.x) {
    const int t0 = t % FT, t1 = (t / FT) % FT, t2 = t / (FT * FT);
    if (t0 > e[0] + 1 || t1 > e[1] + 1 || t2 > e[2] + 1) continue;
    const bool own = t0 >= 1 && t0 <= e[0] && t1 >= 1 && t1 <= e[1] && t2 >= 1 && t2 <= e[2];
    if (own) {
      const int64_t s = site_index(g, x0 + t0 - 1, y0 + t1 - 1, z0 + t2 - 1);
#pragma unroll
      for (int j = 0; j < 3; j++) out[FullPass<PASS>::comp(j) * g.nsites + s] = tile[j * FT3 + t];
    } else {
      const int oi = outer_index(t0 == e[0] + 1 ? FT - 1 : t0, t1 == e[1] + 1 ? FT - 1 : t1,
                                 t2 == e[2] + 1 ? FT - 1 : t2);
#pragma unroll
      for (int j = 0; j < 3; j++) os[FullPass<PASS>::comp(j) * FOUTER + oi] = tile[j * FT3 + t];
    }
  }
}

// One CTA per brick: every owned vertex on the brick's boundary adds the
// outer-layer values of the neighbour bricks that reach it.  Along a dim the
// neighbour offset is 0 (same coordinate), -1 (the brick's first vertex, read
// at the neighbour's tile coordinate e'+1) or +1 (its last vertex, read at
// coordinate 0); the non-zero combinations are added after the brick's own
// partial sum, z outermost, -1 before 0 before +1.  Threads take the boundary vertices only: the two
// z faces (rows along x), then the y faces between them (rows along x), then
// the x faces between those (columns along y, so the neighbours' outer-layer
// reads stay contiguous).
template <int C>
__global__ void __launch_bounds__(256, 4)
    k_fixup_full(Geom g, const float* __restrict__ outer, float* __restrict__ out)
{
  const int64_t b = blockIdx.x;
  int bc[3];
  brick_coords(g, b, bc[0], bc[1], bc[2]);
  const int e[3] = {brick_extent(g.n[0], bc[0]), brick_extent(g.n[1], bc[1]),
                    brick_extent(g.n[2], bc[2])};
  const int nzp = e[2] > 1 ? 2 : 1, nyp = e[1] > 1 ? 2 : 1, nxp = e[0] > 1 ? 2 : 1;
  const int iz = e[2] > 2 ? e[2] - 2 : 0, iy = e[1] > 2 ? e[1] - 2 : 0;
  const int nzf = nzp * e[0] * e[1];
  const int nyf = iz * nyp * e[0];
  const int total = nzf + nyf + iz * iy * nxp;
  // neighbour brick coordinates per dim: [0] = own, [1] = below, [2] = above
  int nbc[3][3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    nbc[d][0] = bc[d];
    nbc[d][1] = wrap_add(bc[d], -1, g.nb[d]);
    nbc[d][2] = wrap_add(bc[d], 1, g.nb[d]);
  }
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    int q[3];
    if (f < nzf) {
      q[0] = f % e[0];
      q[1] = (f / e[0]) % e[1];
      q[2] = f / (e[0] * e[1]) ? e[2] - 1 : 0;
    } else if (f < nzf + nyf) {
      const int r = f - nzf;
      q[0] = r % e[0];
      q[1] = (r / e[0]) % nyp ? e[1] - 1 : 0;
      q[2] = 1 + r / (e[0] * nyp);
    } else {
      const int r = f - nzf - nyf;
      q[1] = 1 + r % iy;
      q[0] = (r / iy) % nxp ? e[0] - 1 : 0;
      q[2] = 1 + r / (iy * nxp);
    }
    const bool lo[3] = {q[0] == 0, q[1] == 0, q[2] == 0};
    const bool hi[3] = {q[0] == e[0] - 1, q[1] == e[1] - 1, q[2] == e[2] - 1};
    const int64_t site = site_index(g, bc[0] * BRICK + q[0], bc[1] * BRICK + q[1],
                                    bc[2] * BRICK + q[2]);
    float acc[C];
#pragma unroll
    for (int c = 0; c < C; c++) acc[c] = out[c * g.nsites + site];
#pragma unroll
    for (int dz = -1; dz <= 1; dz++) {
      if ((dz < 0 && !lo[2]) || (dz > 0 && !hi[2])) continue;
#pragma unroll
      for (int dy = -1; dy <= 1; dy++) {
        if ((dy < 0 && !lo[1]) || (dy > 0 && !hi[1])) continue;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
          if ((dx < 0 && !lo[0]) || (dx > 0 && !hi[0]) || (dx == 0 && dy == 0 && dz == 0))
            continue;
          const int64_t nb = (int64_t)nbc[0][dx < 0 ? 1 : (dx > 0 ? 2 : 0)] +
                             (int64_t)g.nb[0] * ((int64_t)nbc[1][dy < 0 ? 1 : (dy > 0 ? 2 : 0)] +
                                                 (int64_t)g.nb[1] * nbc[2][dz < 0 ? 1 : (dz > 0 ? 2 : 0)]);
          const int oi = outer_index(dx < 0 ? FT - 1 : (dx > 0 ? 0 : q[0] + 1),
                                     dy < 0 ? FT - 1 : (dy > 0 ? 0 : q[1] + 1),
                                     dz < 0 ? FT - 1 : (dz > 0 ? 0 : q[2] + 1));
          const float* os = outer + (size_t)nb * C * FOUTER + oi;
#pragma unroll
          for (int c = 0; c < C; c++) acc[c] = __fadd_rn(acc[c], os[c * FOUTER]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < C; c++) out[c * g.nsites + site] = acc[c];
  }
}

// Compensated FP32 and fixed-point tile pass: the same weights and vertices
// as k_deposit_full, two words per vertex (140 KB for three components, one
// CTA per SM with 512 threads), and every vertex another brick can reach goes
// to the thick-shell store.
constexpr int FULL2_THREADS = 512;

template <int PASS, int ACC>
__global__ void __launch_bounds__(FULL2_THREADS)
    k_deposit_full2(StoreView v, DepositParams dp, float* __restrict__ out,
                    uint64_t* __restrict__ store, const uint32_t* __restrict__ vmax_bits,
                    uint32_t* flags)
{
  constexpr int CT = FullPass<PASS>::total;
  constexpr bool FIXED = ACC == ACC_FIXED;
  extern __shared__ __align__(16) unsigned char smem_raw[];

  const Geom& g = v.g;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int e[3] = {brick_extent(g.n[0], bx), brick_extent(g.n[1], by),
                    brick_extent(g.n[2], bz)};
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  TileRef<FT3> tr{smem_raw, FIXED && cnt <= split_max<true>(dp.has_mass != 0)};
  int vexp = 0;
  if (FIXED) vexp = vexp_of(*vmax_bits);
  const float vscale = vel_scale(vexp);
  const float conv = FIXED ? ldexpf(dp.fixed_scale, (PASS == 0 ? vexp : 2 * vexp) - 16) : 0.0f;
  if (FIXED && threadIdx.x == 0 && b == 0 && !(conv > 0.0f && conv <= 3.402823466e38f))
    set_flag(flags, ERR_FIXED_OVERFLOW);

  {
    uint32_t* zw = reinterpret_cast<uint32_t*>(smem_raw);
    for (int t = threadIdx.x; t < 3 * 2 * FT3; t += blockDim.x) zw[t] = 0u;
  }
  __syncthreads();

  constexpr int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
  // the particle loop, instantiated per CTA for the split tile (or not) and
  // for per-particle masses (or a global mass)
  auto particles = [&](auto split_c, auto hm_c) {
    constexpr bool SPLIT = decltype(split_c)::value;
    constexpr bool HM = decltype(hm_c)::value;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const uint32_t p = (uint32_t)base + (uint32_t)i;  // slots fit in 32 bits
      int x, y, z;
      unpack_key(g, v.a.key[p], x, y, z);
      const float o[3] = {v.a.ox[p], v.a.oy[p], v.a.oz[p]};
      const float vel[3] = {v.a.vx[p], v.a.vy[p], v.a.vz[p]};
      const int l[3] = {x - x0, y - y0, z - z0};
      int ls[3], lt[3], gd[3];
      float s[3];
  #pragma unroll
      for (int d = 0; d < 3; d++) {
        s[d] = __fsub_rn(o[d], 0.5f);
        gd[d] = s[d] >= 0.0f;
        ls[d] = l[d] + 1;
        lt[d] = l[d] + gd[d];
      }
      if (FIXED) {
        const uint64_t mq = HM ? mass_q(v.a.mass[p], dp.inv_unit, flags) : 0;
        // vertex weights sq and staggered weights tq in units of 2^-31
        uint32_t sq[3][2], tq[3][2], vq[3];
  #pragma unroll
        for (int d = 0; d < 3; d++) {
          const uint32_t u = weight_q(o[d]);
          sq[d][0] = (1u << 31) - u;
          sq[d][1] = u;
          const uint32_t us = weight_q(fabsf(s[d]));
          tq[d][0] = gd[d] ? (1u << 31) - us : us;
          tq[d][1] = gd[d] ? us : (1u << 31) - us;
          vq[d] = vel_q(vel[d], vscale);
        }
        if (PASS == 0) {
  #pragma unroll
          for (int c = 0; c < 3; c++) {
            const bool neg = vel[c] < 0.0f;
  #pragma unroll
            for (int k = 0; k < 8; k++) {
              const int b0 = (k >> 2) & 1, b1 = (k >> 1) & 1, b2 = k & 1;
              const uint64_t w = fixed_corner(c == 0 ? tq[0][b0] : sq[0][b0],
                                              c == 1 ? tq[1][b1] : sq[1][b1],
                                              c == 2 ? tq[2][b2] : sq[2][b2]);
              const int t = tile_at((c == 0 ? lt[0] : ls[0]) + b0, (c == 1 ? lt[1] : ls[1]) + b1,
                                    (c == 2 ? lt[2] : ls[2]) + b2);
              add_fixed48_t<SPLIT, FT3>(smem_raw, c, t, mass_sign48_t<HM>(mul_wv48(w, vq[c]), mq, neg));
            }
          }
        } else if (PASS == 1) {
          double f2[3];  // v_d^2 2^-46 (times the relative mass), FP64
  #pragma unroll
          for (int d = 0; d < 3; d++) f2[d] = stress_factor<HM>(vq[d], vq[d], 0x1p-46, mq);
  #pragma unroll
          for (int k = 0; k < 8; k++) {
            const int b0 = (k >> 2) & 1, b1 = (k >> 1) & 1, b2 = k & 1;
            const uint64_t w = fixed_corner(sq[0][b0], sq[1][b1], sq[2][b2]);
            const int t = tile_at(ls[0] + b0, ls[1] + b1, ls[2] + b2);
  #pragma unroll
            for (int d = 0; d < 3; d++) add_fixed48_t<SPLIT, FT3>(smem_raw, d, t, stress_q(w, f2[d], false));
          }
        } else {
  #pragma unroll
          for (int q = 0; q < 3; q++) {
            const double vv = stress_factor<HM>(vq[pa[q]], vq[pb[q]], 0x1p-46, mq);  // 2^-46
            const bool neg = (vel[pa[q]] < 0.0f) != (vel[pb[q]] < 0.0f);
  #pragma unroll
            for (int k = 0; k < 8; k++) {
              const int bb[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
              uint32_t w[3];
              int t[3];
  #pragma unroll
              for (int d = 0; d < 3; d++) {
                const bool st = d == pa[q] || d == pb[q];
                w[d] = st ? tq[d][bb[d]] : sq[d][bb[d]];
                t[d] = (st ? lt[d] : ls[d]) + bb[d];
              }
              add_fixed48_t<SPLIT, FT3>(smem_raw, q, tile_at(t[0], t[1], t[2]),
                                        stress_q(fixed_corner(w[0], w[1], w[2]), vv, neg));
            }
          }
        }
        continue;
      }
      // compensated FP32: the arithmetic of k_deposit_full
      const float mf = HM ? __fmul_rn(v.a.mass[p], dp.inv_vol) : dp.mf;
      float sw[3][2], tw[3][2];
  #pragma unroll
      for (int d = 0; d < 3; d++) {
        sw[d][1] = o[d];
        sw[d][0] = __fsub_rn(1.0f, o[d]);
        if (gd[d]) {
          tw[d][1] = s[d];
          tw[d][0] = __fsub_rn(1.0f, s[d]);
        } else {
          tw[d][0] = -s[d];
          tw[d][1] = __fsub_rn(1.0f, tw[d][0]);
        }
      }
      if (PASS == 0) {
  #pragma unroll
        for (int c = 0; c < 3; c++) {
          const float mv = __fmul_rn(mf, vel[c]);
  #pragma unroll
          for (int k = 0; k < 8; k++) {
            const int b0 = (k >> 2) & 1, b1 = (k >> 1) & 1, b2 = k & 1;
            const float w0 = c == 0 ? tw[0][b0] : sw[0][b0];
            const float w1 = c == 1 ? tw[1][b1] : sw[1][b1];
            const float w2 = c == 2 ? tw[2][b2] : sw[2][b2];
            const int t = tile_at((c == 0 ? lt[0] : ls[0]) + b0, (c == 1 ? lt[1] : ls[1]) + b1,
                                  (c == 2 ? lt[2] : ls[2]) + b2);
            add_float<ACC>(tr, c, t, __fmul_rn(__fmul_rn(__fmul_rn(mv, w0), w1), w2));
          }
        }
      } else if (PASS == 1) {
  #pragma unroll
        for (int i2 = 0; i2 < 3; i2++) {
          const float m2 = __fmul_rn(__fmul_rn(mf, vel[i2]), vel[i2]);
  #pragma unroll
          for (int k = 0; k < 8; k++) {
            const int b0 = (k >> 2) & 1, b1 = (k >> 1) & 1, b2 = k & 1;
            add_float<ACC>(tr, i2, tile_at(ls[0] + b0, ls[1] + b1, ls[2] + b2),
                           __fmul_rn(__fmul_rn(__fmul_rn(m2, sw[0][b0]), sw[1][b1]), sw[2][b2]));
          }
        }
      } else {
  #pragma unroll
        for (int q = 0; q < 3; q++) {
          const float mm = __fmul_rn(__fmul_rn(mf, vel[pa[q]]), vel[pb[q]]);
  #pragma unroll
          for (int k = 0; k < 8; k++) {
            const int bb[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
            float w[3];
            int t[3];
  #pragma unroll
            for (int d = 0; d < 3; d++) {
              const bool st = d == pa[q] || d == pb[q];
              w[d] = st ? tw[d][bb[d]] : sw[d][bb[d]];
              t[d] = (st ? lt[d] : ls[d]) + bb[d];
            }
            add_float<ACC>(tr, q, tile_at(t[0], t[1], t[2]),
                           __fmul_rn(__fmul_rn(__fmul_rn(mm, w[0]), w[1]), w[2]));
          }
        }
      }
    }
  };
  const bool hm_rt = dp.has_mass != 0;
  if (FIXED && tr.split) {
    if (hm_rt) particles(std::true_type{}, std::true_type{});
    else particles(std::true_type{}, std::false_type{});
  } else {
    if (hm_rt) particles(std::false_type{}, std::true_type{});
    else particles(std::false_type{}, std::false_type{});
  }
  __syncthreads();

  // Flush: private vertices (every tile coordinate in [2, e-1]) to the field,
  // the thick shell to the store.
  uint64_t* st = store + (size_t)b * CT * FSHELL;
  const float* facc = reinterpret_cast<const float*>(smem_raw);
  for (int t = threadIdx.x; t < FT3; t += blockDim.x) {
    const int t0 = t % FT, t1 = (t / FT) % FT, t2 = t / (FT * FT);
    if (t0 > e[0] + 1 || t1 > e[1] + 1 || t2 > e[2] + 1) continue;
    const bool priv = t0 >= 2 && t0 < e[0] && t1 >= 2 && t1 < e[1] && t2 >= 2 && t2 < e[2];
    const int si = priv ? 0 : thick_index(canon(t0, e[0]), canon(t1, e[1]), canon(t2, e[2]));
    const int64_t site = priv ? site_index(g, x0 + t0 - 1, y0 + t1 - 1, z0 + t2 - 1) : 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int c = FullPass<PASS>::comp(j);
      if (FIXED) {
        const long long q = tile_fixed<true>(tr, j, t);
        if (priv) out[(size_t)c * g.nsites + site] = __fmul_rn(__ll2float_rn(q), conv);
        else st[(size_t)c * FSHELL + si] = (uint64_t)q;
      } else {
        const float hi = facc[(size_t)j * 2 * FT3 + t], lo = facc[(size_t)j * 2 * FT3 + FT3 + t];
        if (priv) out[(size_t)c * g.nsites + site] = __fadd_rn(hi, lo);
        else reinterpret_cast<float2*>(st)[(size_t)c * FSHELL + si] = make_float2(hi, lo);
      }
    }
  }
}

// Fix-up of the compensated and fixed-point modes: every owned boundary
// vertex is the sum of the thick-shell values of its own brick and of the up
// to 26 neighbours that reach it, z outermost, -1 before 0 before +1 (own
// brick included at 0, 0, 0).  Same enumeration of the boundary vertices as
// k_fixup_full.
template <int C, int ACC>
__global__ void __launch_bounds__(256, 4)
    k_fixup_full2(Geom g, const uint64_t* __restrict__ store, float fixed_scale,
                  const uint32_t* __restrict__ vmax_bits, float* __restrict__ out)
{
  const int64_t b = blockIdx.x;
  int bc[3];
  brick_coords(g, b, bc[0], bc[1], bc[2]);
  const int e[3] = {brick_extent(g.n[0], bc[0]), brick_extent(g.n[1], bc[1]),
                    brick_extent(g.n[2], bc[2])};
  const int nzp = e[2] > 1 ? 2 : 1, nyp = e[1] > 1 ? 2 : 1, nxp = e[0] > 1 ? 2 : 1;
  const int iz = e[2] > 2 ? e[2] - 2 : 0, iy = e[1] > 2 ? e[1] - 2 : 0;
  const int nzf = nzp * e[0] * e[1];
  const int nyf = iz * nyp * e[0];
  const int total = nzf + nyf + iz * iy * nxp;
  int nbc[3][3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    nbc[d][0] = bc[d];
    nbc[d][1] = wrap_add(bc[d], -1, g.nb[d]);
    nbc[d][2] = wrap_add(bc[d], 1, g.nb[d]);
  }
  float conv = 0.0f;
  if (ACC == ACC_FIXED) {
    const int vexp = vexp_of(*vmax_bits);
    conv = ldexpf(fixed_scale, (C == 3 ? vexp : 2 * vexp) - 16);
  }
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    int q[3];
    if (f < nzf) {
      q[0] = f % e[0];
      q[1] = (f / e[0]) % e[1];
      q[2] = f / (e[0] * e[1]) ? e[2] - 1 : 0;
    } else if (f < nzf + nyf) {
      const int r = f - nzf;
      q[0] = r % e[0];
      q[1] = (r / e[0]) % nyp ? e[1] - 1 : 0;
      q[2] = 1 + r / (e[0] * nyp);
    } else {
      const int r = f - nzf - nyf;
      q[1] = 1 + r % iy;
      q[0] = (r / iy) % nxp ? e[0] - 1 : 0;
      q[2] = 1 + r / (iy * nxp);
    }
    const bool lo[3] = {q[0] == 0, q[1] == 0, q[2] == 0};
    const bool hi[3] = {q[0] == e[0] - 1, q[1] == e[1] - 1, q[2] == e[2] - 1};
    const int64_t site = site_index(g, bc[0] * BRICK + q[0], bc[1] * BRICK + q[1],
                                    bc[2] * BRICK + q[2]);
    long long qs[C];
    float fs[C], fc[C];
#pragma unroll
    for (int c = 0; c < C; c++) qs[c] = 0, fs[c] = 0.0f, fc[c] = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++) {
      if ((dz < 0 && !lo[2]) || (dz > 0 && !hi[2])) continue;
#pragma unroll
      for (int dy = -1; dy <= 1; dy++) {
        if ((dy < 0 && !lo[1]) || (dy > 0 && !hi[1])) continue;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
          if ((dx < 0 && !lo[0]) || (dx > 0 && !hi[0])) continue;
          const int64_t nb = (int64_t)nbc[0][dx < 0 ? 1 : (dx > 0 ? 2 : 0)] +
                             (int64_t)g.nb[0] * ((int64_t)nbc[1][dy < 0 ? 1 : (dy > 0 ? 2 : 0)] +
                                                 (int64_t)g.nb[1] * nbc[2][dz < 0 ? 1 : (dz > 0 ? 2 : 0)]);
          const int si = thick_index(dx < 0 ? FT - 1 : (dx > 0 ? 0 : canon(q[0] + 1, e[0])),
                                     dy < 0 ? FT - 1 : (dy > 0 ? 0 : canon(q[1] + 1, e[1])),
                                     dz < 0 ? FT - 1 : (dz > 0 ? 0 : canon(q[2] + 1, e[2])));
          const uint64_t* sp = store + (size_t)nb * C * FSHELL + si;
#pragma unroll
          for (int c = 0; c < C; c++) {
            if (ACC == ACC_FIXED) {
              qs[c] += (long long)sp[(size_t)c * FSHELL];
            } else {
              const float2 hl = reinterpret_cast<const float2*>(sp)[(size_t)c * FSHELL];
              comp_acc(fs[c], fc[c], hl.x, hl.y);
            }
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < C; c++)
      out[c * g.nsites + site] = ACC == ACC_FIXED ? __fmul_rn(__ll2float_rn(qs[c]), conv)
                                                  : __fadd_rn(fs[c], fc[c]);
  }
}

template <int PASS, int ACC>
cudaError_t tile_pass2(lf2_ctx* c, float* out, const DepositParams& dp)
{
  const size_t smem = (size_t)3 * 2 * FT3 * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_deposit_full2<PASS, ACC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_deposit_full2<PASS, ACC><<<(unsigned)c->g.nbricks, FULL2_THREADS, smem, c->stream>>>(
      view(c), dp, out, c->spill, c->vmax_bits, c->flags);
  return cudaGetLastError();
}

template <int ACC>
cudaError_t run2(lf2_ctx* c, int kind, float* out, const DepositParams& dp, int stage)
{
  const unsigned nb = (unsigned)c->g.nbricks;
  if (stage == 0) {
    cudaError_t e = cudaSuccess;
    if (ACC == ACC_FIXED) e = launch_vmax(c);
    if (e != cudaSuccess) return e;
    if (kind == 3) return tile_pass2<0, ACC>(c, out, dp);
    e = tile_pass2<1, ACC>(c, out, dp);
    return e != cudaSuccess ? e : tile_pass2<2, ACC>(c, out, dp);
  }
  c->launches += 1;
  if (kind == 3)
    k_fixup_full2<3, ACC><<<nb, 256, 0, c->stream>>>(c->g, c->spill, dp.fixed_scale, c->vmax_bits, out);
  else
    k_fixup_full2<6, ACC><<<nb, 256, 0, c->stream>>>(c->g, c->spill, dp.fixed_scale, c->vmax_bits, out);
  return cudaGetLastError();
}

template <int PASS>
cudaError_t tile_pass(lf2_ctx* c, float* out, const DepositParams& dp)
{
  const size_t smem = (size_t)3 * FT3 * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_deposit_full<PASS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_deposit_full<PASS><<<(unsigned)c->g.nbricks, FULL_THREADS, smem, c->stream>>>(
      view(c), dp, out, reinterpret_cast<float*>(c->spill));
  return cudaGetLastError();
}

}  // namespace

// Store slots (8 bytes each) a full-CIC deposit of `comps` components needs
// in the context's deposit mode.
size_t deposit_full_spill_slots(const lf2_ctx* c, int comps)
{
  return (size_t)c->g.nbricks * (size_t)comps * (c->mode == LF2_DEPOSIT_FP32_PLAIN ? SHELL : FSHELL);
}

cudaError_t launch_deposit_full(lf2_ctx* c, int kind, float* out, int stage)
{
  const DepositParams dp = deposit_params(c);
  if (c->mode == LF2_DEPOSIT_FIXED64) return run2<ACC_FIXED>(c, kind, out, dp, stage);
  if (c->mode == LF2_DEPOSIT_FP32) return run2<ACC_COMP>(c, kind, out, dp, stage);
  const unsigned nb = (unsigned)c->g.nbricks;
  float* outer = reinterpret_cast<float*>(c->spill);
  if (stage == 0) {
    if (kind == 3) return tile_pass<0>(c, out, dp);
    cudaError_t e = tile_pass<1>(c, out, dp);
    return e != cudaSuccess ? e : tile_pass<2>(c, out, dp);
  }
  c->launches += 1;
  if (kind == 3)
    k_fixup_full<3><<<nb, 256, 0, c->stream>>>(c->g, outer, out);
  else
    k_fixup_full<6><<<nb, 256, 0, c->stream>>>(c->g, outer, out);
  return cudaGetLastError();
}

}  // namespace lf2
