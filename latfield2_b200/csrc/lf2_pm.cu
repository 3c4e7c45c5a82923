// lf2_pm.cu -- kernels of the differentiable particle-mesh chain: CIC deposit
// and gather on particles kept in one order for a whole call (sorted by
// brick and cell when the call starts, no rebinning, so that gradients stay
// attached to their slots), the kick-drift update, a periodic 27-point
// stencil as the grid operator, the hand-written adjoints of all of them,
// and the permutations of the particle state into that order and of the
// gradients back.
//
//   deposit   rho(v)   += m_p / res^3 * W(v - x_p)            (scalarProjectionCIC)
//   gather    G_p       = sum_k W_k(x_p) F(corner_k)           (updateVel CIC kick)
//   kick      v_p      += dt * G_p
//   drift     off_p    += dt/res * v_p, carry into the cell    (move_particles_simple)
//   stencil   F_c(g)    = sum_o S[c][o] rho(g + o), o in {-1,0,1}^3
// with W = wx*wy*wz, wx = 1 - fx or fx, f the in-cell offset (cell units).
// Adjoints (gradients with respect to the inputs, given the output gradient):
//   deposit   dL/dm_p   = 1/res^3 * sum_k W_k gR(corner_k)
//             dL/df_p   = m_p/res^3 * sum_k dW_k/df gR(corner_k)
//   gather    gF(corner_k) += W_k gG_p          (a CIC deposit of gG)
//             dL/df_p  += sum_k dW_k/df (gG_p . F(corner_k))
//   stencil   gR(h)     = sum_c sum_o S[c][o] gF_c(h - o)
//             dL/dS[c][o] = sum_g gF_c(g) rho(g + o)
// dW/dfx = (bx ? 1 : -1) * wy * wz, etc.  Offsets and their gradients are in
// cell units; positions in box units are (cell + off) * res.  The force field
// F and its gradient are stored as one float4 (x, y, z, unused) per site, so
// that a corner is one 16-byte load and one vector atomic.
#include <cuda_runtime.h>

#include "lf2_deposit_common.cuh"
#include "lf2_internal.h"

namespace lf2 {

namespace {

constexpr int PM_THREADS = 256;

inline int grid_for(int64_t n, int threads)
{
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g > 0 ? g : 1);
}

struct Corners {
  int64_t site[8];
  float w[8];
  float dw[8][3];
};

__device__ __forceinline__ void corners(const Geom& g, int32_t c, const float* off3, int64_t p,
                                        Corners& k)
{
  const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
  const int xs[2] = {x, x + 1 < g.n[0] ? x + 1 : 0};
  const int ys[2] = {y, y + 1 < g.n[1] ? y + 1 : 0};
  const int zs[2] = {z, z + 1 < g.n[2] ? z + 1 : 0};
  const float f[3] = {off3[3 * p], off3[3 * p + 1], off3[3 * p + 2]};
  const float h[3] = {1.0f - f[0], 1.0f - f[1], 1.0f - f[2]};
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int bx = (q >> 2) & 1, by = (q >> 1) & 1, bz = q & 1;
    const float wx = bx ? f[0] : h[0], wy = by ? f[1] : h[1], wz = bz ? f[2] : h[2];
    k.site[q] = site_index(g, xs[bx], ys[by], zs[bz]);
    k.w[q] = wx * wy * wz;
    k.dw[q][0] = (bx ? 1.0f : -1.0f) * wy * wz;
    k.dw[q][1] = (by ? 1.0f : -1.0f) * wx * wz;
    k.dw[q][2] = (bz ? 1.0f : -1.0f) * wx * wy;
  }
}

__global__ void k_pm_deposit(Geom g, int64_t np, const int32_t* __restrict__ cell,
                             const float* __restrict__ off3, const float* __restrict__ mass,
                             float gmass, float inv_vol, float* __restrict__ rho)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    Corners k;
    corners(g, cell[p], off3, p, k);
    const float m = (mass ? mass[p] : gmass) * inv_vol;
#pragma unroll
    for (int q = 0; q < 8; q++) atomicAdd(&rho[k.site[q]], k.w[q] * m);
  }
}

// Fixed-point form of the chain's deposit (contexts in LF2_DEPOSIT_FIXED64):
// every corner's weight is the library's deterministic integer weight
// (fixed_corner, 2^-32 units), times the particle's mass relative to the
// largest mass M of the call in 2^-24 units; the integer sums (64-bit global
// atomics) do not depend on the order, and are converted once:
// rho += (float)sum * (M / res^3 * 2^-32).
__global__ void k_pm_mass_max(int64_t np, const float* __restrict__ mass, uint32_t* mmax)
{
  uint32_t m = 0u;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(fmaxf(mass[p], 0.0f)));  // non-negative floats order as integers
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(mmax, m);
}

__global__ void k_pm_deposit_fixed(Geom g, int64_t np, const int32_t* __restrict__ cell,
                                   const float* __restrict__ off3, const float* __restrict__ mass,
                                   const uint32_t* __restrict__ mmax, unsigned long long* __restrict__ acc)
{
  const float inv_m = mass ? 1.0f / __uint_as_float(*mmax) : 0.0f;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cell[p];
    const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
    const int xs[2] = {x, x + 1 < g.n[0] ? x + 1 : 0};
    const int ys[2] = {y, y + 1 < g.n[1] ? y + 1 : 0};
    const int zs[2] = {z, z + 1 < g.n[2] ? z + 1 : 0};
    const uint32_t ux = weight_q(off3[3 * p]), uy = weight_q(off3[3 * p + 1]), uz = weight_q(off3[3 * p + 2]);
    const uint32_t qx[2] = {(1u << 31) - ux, ux}, qy[2] = {(1u << 31) - uy, uy}, qz[2] = {(1u << 31) - uz, uz};
    const uint64_t mq = mass ? (uint64_t)__float2uint_rn(fminf(__fmul_rn(mass[p], inv_m), 1.0f) * 16777216.0f) : 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int bx = (q >> 2) & 1, by = (q >> 1) & 1, bz = q & 1;
      uint64_t w = fixed_corner(qx[bx], qy[by], qz[bz]);
      if (mass) w = (w * mq + (1ull << 23)) >> 24;
      atomicAdd(&acc[site_index(g, xs[bx], ys[by], zs[bz])], (unsigned long long)w);
    }
  }
}

// Brick-tiled forms of the two deposits, for particles grouped by brick
// (brick_start[b] .. brick_start[b+1] hold the particles that were in brick
// b when the chain sorted its state; a particle that has since drifted out
// of the brick goes straight to the global sums).  One CTA per brick: its
// particles add their corner weights into the brick's (BRICK+1)^3 vertex
// tile in shared memory, then the tile's non-zero sums go to the global
// field with one atomic each: 4913 global atomics per brick instead of 8 per
// particle.  The fixed-point tile keeps a low word whose carry goes to a high
// word (the order of the additions does not change the sums); the FP32 tile
// adds floats, so its roundings depend on the order, as the global atomics'
// do.
__device__ __forceinline__ bool in_brick(int x, int y, int z, int x0, int y0, int z0)
{
  return (unsigned)(x - x0) < (unsigned)BRICK && (unsigned)(y - y0) < (unsigned)BRICK &&
         (unsigned)(z - z0) < (unsigned)BRICK;
}

// The group's range of brick b, clamped to the particle arrays.
__device__ __forceinline__ void group_range(const int64_t* brick_start, int64_t b, int64_t np,
                                            int64_t& p0, int64_t& p1)
{
  p0 = min(max(brick_start[b], (int64_t)0), np);
  p1 = min(max(brick_start[b + 1], p0), np);
}

// Vertex (x0 + i, y0 + j, z0 + k) of a brick tile, wrapped periodically.
__device__ __forceinline__ int64_t tile_site(const Geom& g, int t, int x0, int y0, int z0)
{
  int x = x0 + t % TILE, y = y0 + (t / TILE) % TILE, z = z0 + t / (TILE * TILE);
  x -= x >= g.n[0] ? g.n[0] : 0;
  y -= y >= g.n[1] ? g.n[1] : 0;
  z -= z >= g.n[2] ? g.n[2] : 0;
  return site_index(g, x, y, z);
}

__global__ void __launch_bounds__(256)
    k_pm_deposit_fixed_tile(Geom g, int64_t np, const int64_t* __restrict__ brick_start,
                            const int32_t* __restrict__ cell, const float* __restrict__ off3,
                            const float* __restrict__ mass, const uint32_t* __restrict__ mmax,
                            unsigned long long* __restrict__ acc)
{
  __shared__ uint32_t lo[TILE3], hi[TILE3];
  for (int t = threadIdx.x; t < TILE3; t += blockDim.x) lo[t] = hi[t] = 0u;
  __syncthreads();
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const float inv_m = mass ? 1.0f / __uint_as_float(*mmax) : 0.0f;
  int64_t p0, p1;
  group_range(brick_start, b, np, p0, p1);
  for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    const int32_t c = cell[p];
    const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
    const uint32_t ux = weight_q(off3[3 * p]), uy = weight_q(off3[3 * p + 1]), uz = weight_q(off3[3 * p + 2]);
    const uint32_t qx[2] = {(1u << 31) - ux, ux}, qy[2] = {(1u << 31) - uy, uy}, qz[2] = {(1u << 31) - uz, uz};
    const uint64_t mq = mass ? (uint64_t)__float2uint_rn(fminf(__fmul_rn(mass[p], inv_m), 1.0f) * 16777216.0f) : 0;
    if (in_brick(x, y, z, x0, y0, z0)) {
      const int t0 = (x - x0) + TILE * ((y - y0) + TILE * (z - z0));
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int cx = (q >> 2) & 1, cy = (q >> 1) & 1, cz = q & 1;
        uint64_t w = fixed_corner(qx[cx], qy[cy], qz[cz]);
        if (mass) w = (w * mq + (1ull << 23)) >> 24;
        const int t = t0 + cx + TILE * (cy + TILE * cz);
        const uint32_t wl = (uint32_t)w;
        const uint32_t old = atomicAdd(&lo[t], wl);
        const uint32_t up = (uint32_t)(w >> 32) + ((uint32_t)(old + wl) < old ? 1u : 0u);
        if (up) atomicAdd(&hi[t], up);
      }
    } else {  // drifted out of the brick since the sort
      const int xs[2] = {x, x + 1 < g.n[0] ? x + 1 : 0};
      const int ys[2] = {y, y + 1 < g.n[1] ? y + 1 : 0};
      const int zs[2] = {z, z + 1 < g.n[2] ? z + 1 : 0};
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int cx = (q >> 2) & 1, cy = (q >> 1) & 1, cz = q & 1;
        uint64_t w = fixed_corner(qx[cx], qy[cy], qz[cz]);
        if (mass) w = (w * mq + (1ull << 23)) >> 24;
        atomicAdd(&acc[site_index(g, xs[cx], ys[cy], zs[cz])], (unsigned long long)w);
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < TILE3; t += blockDim.x) {
    const unsigned long long v = ((unsigned long long)hi[t] << 32) | lo[t];
    if (v) atomicAdd(&acc[tile_site(g, t, x0, y0, z0)], v);
  }
}

__global__ void __launch_bounds__(256)
    k_pm_deposit_tile(Geom g, int64_t np, const int64_t* __restrict__ brick_start,
                      const int32_t* __restrict__ cell, const float* __restrict__ off3,
                      const float* __restrict__ mass, float gmass, float inv_vol,
                      float* __restrict__ rho)
{
  __shared__ float tile[TILE3];
  for (int t = threadIdx.x; t < TILE3; t += blockDim.x) tile[t] = 0.0f;
  __syncthreads();
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  int64_t p0, p1;
  group_range(brick_start, b, np, p0, p1);
  for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    const int32_t c = cell[p];
    const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
    const float m = (mass ? mass[p] : gmass) * inv_vol;
    if (in_brick(x, y, z, x0, y0, z0)) {
      const float f[3] = {off3[3 * p], off3[3 * p + 1], off3[3 * p + 2]};
      const float h[3] = {1.0f - f[0], 1.0f - f[1], 1.0f - f[2]};
      const int t0 = (x - x0) + TILE * ((y - y0) + TILE * (z - z0));
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int cx = (q >> 2) & 1, cy = (q >> 1) & 1, cz = q & 1;
        const float w = (cx ? f[0] : h[0]) * (cy ? f[1] : h[1]) * (cz ? f[2] : h[2]);
        atomicAdd(&tile[t0 + cx + TILE * (cy + TILE * cz)], w * m);
      }
    } else {  // drifted out of the brick since the sort
      Corners k;
      corners(g, c, off3, p, k);
#pragma unroll
      for (int q = 0; q < 8; q++) atomicAdd(&rho[k.site[q]], k.w[q] * m);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < TILE3; t += blockDim.x) {
    const float v = tile[t];
    if (v != 0.0f) atomicAdd(&rho[tile_site(g, t, x0, y0, z0)], v);
  }
}

__global__ void k_pm_fixed_to_rho(int64_t ns, unsigned long long* __restrict__ acc, const float* mass,
                                  const uint32_t* __restrict__ mmax, float gmass, float inv_vol,
                                  float* __restrict__ rho, uint32_t* flags)
{
  const float m = mass ? __uint_as_float(*mmax) : gmass;
  const float scale = ldexpf(__fmul_rn(m, inv_vol), -32);
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ns;
       s += (int64_t)gridDim.x * blockDim.x) {
    const long long q = (long long)acc[s];
    if (q < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
    rho[s] = __fadd_rn(rho[s], __fmul_rn(__ll2float_rn(q), scale));
    acc[s] = 0ull;  // clean for the next call
  }
}

__global__ void k_pm_gather(Geom g, int64_t np, const int32_t* __restrict__ cell,
                            const float* __restrict__ off3, const float4* __restrict__ F4,
                            float* __restrict__ out3)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    Corners k;
    corners(g, cell[p], off3, p, k);
    float a[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float4 f = __ldg(F4 + k.site[q]);
      a[0] = fmaf(k.w[q], f.x, a[0]);
      a[1] = fmaf(k.w[q], f.y, a[1]);
      a[2] = fmaf(k.w[q], f.z, a[2]);
    }
    for (int c = 0; c < 3; c++) out3[3 * p + c] = a[c];
  }
}

// v += dt_kick * G; off += dtn * v with the carry into the cell (as the
// library's drift, LATfield2 move_particles_simple in cell units).
__global__ void k_pm_kick_drift(Geom g, int64_t np, int32_t* __restrict__ cell, float* __restrict__ off3,
                                float* __restrict__ vel3, const float* __restrict__ G3, float dtk,
                                float dtn, uint32_t* flags)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cell[p];
    int xyz[3] = {c % g.n[0], (c / g.n[0]) % g.n[1], c / (g.n[0] * g.n[1])};
    for (int d = 0; d < 3; d++) {
      float v = vel3[3 * p + d];
      if (G3) v = __fmaf_rn(dtk, G3[3 * p + d], v);
      vel3[3 * p + d] = v;
      float o = __fmaf_rn(dtn, v, off3[3 * p + d]);
      if (!isfinite(o)) {
        set_flag(flags, ERR_NONFINITE);
        continue;
      }
      const float fl = floorf(o);
      o = __fsub_rn(o, fl);
      int carry = (int)fl;
      if (o >= 1.0f) {
        o = 0.0f;
        carry += 1;
      }
      off3[3 * p + d] = o;
      xyz[d] = wrap_add(xyz[d], carry, g.n[d]);
    }
    cell[p] = (int32_t)site_index(g, xyz[0], xyz[1], xyz[2]);
  }
}

// The gather, the kick and the drift of one chain step in one pass, with
// the arithmetic of k_pm_gather and k_pm_kick_drift (the same results bit
// for bit) and no gathered field written in between.
__global__ void k_pm_gather_kick_drift(Geom g, int64_t np, int32_t* __restrict__ cell,
                                       float* __restrict__ off3, float* __restrict__ vel3,
                                       const float4* __restrict__ F4, float dtk, float dtn,
                                       uint32_t* flags)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cell[p];
    Corners k;
    corners(g, c, off3, p, k);
    float a[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float4 f = __ldg(F4 + k.site[q]);
      a[0] = fmaf(k.w[q], f.x, a[0]);
      a[1] = fmaf(k.w[q], f.y, a[1]);
      a[2] = fmaf(k.w[q], f.z, a[2]);
    }
    int xyz[3] = {c % g.n[0], (c / g.n[0]) % g.n[1], c / (g.n[0] * g.n[1])};
    for (int d = 0; d < 3; d++) {
      float v = __fmaf_rn(dtk, a[d], vel3[3 * p + d]);
      vel3[3 * p + d] = v;
      float o = __fmaf_rn(dtn, v, off3[3 * p + d]);
      if (!isfinite(o)) {
        set_flag(flags, ERR_NONFINITE);
        continue;
      }
      const float fl = floorf(o);
      o = __fsub_rn(o, fl);
      int carry = (int)fl;
      if (o >= 1.0f) {
        o = 0.0f;
        carry += 1;
      }
      off3[3 * p + d] = o;
      xyz[d] = wrap_add(xyz[d], carry, g.n[d]);
    }
    cell[p] = (int32_t)site_index(g, xyz[0], xyz[1], xyz[2]);
  }
}

__global__ void k_pm_deposit_adj(Geom g, int64_t np, const int32_t* __restrict__ cell,
                                 const float* __restrict__ off3, const float* __restrict__ mass,
                                 float gmass, float inv_vol, const float* __restrict__ g_rho,
                                 float* __restrict__ g_off3, float* __restrict__ g_mass)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    Corners k;
    corners(g, cell[p], off3, p, k);
    float s = 0.f, d[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float gr = __ldg(g_rho + k.site[q]);
      s = fmaf(k.w[q], gr, s);
      for (int c = 0; c < 3; c++) d[c] = fmaf(k.dw[q][c], gr, d[c]);
    }
    const float m = (mass ? mass[p] : gmass) * inv_vol;
    if (g_mass) g_mass[p] += s * inv_vol;
    if (g_off3)
      for (int c = 0; c < 3; c++) g_off3[3 * p + c] += m * d[c];
  }
}

__global__ void k_pm_gather_adj(Geom g, int64_t np, const int32_t* __restrict__ cell,
                                const float* __restrict__ off3, const float4* __restrict__ F4,
                                const float* __restrict__ gG3, float4* __restrict__ gF4,
                                float* __restrict__ g_off3)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    Corners k;
    corners(g, cell[p], off3, p, k);
    const float gg[3] = {gG3[3 * p], gG3[3 * p + 1], gG3[3 * p + 2]};
    float d[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; q++) {
      if (gF4) atomicAdd(&gF4[k.site[q]], make_float4(k.w[q] * gg[0], k.w[q] * gg[1], k.w[q] * gg[2], 0.f));
      if (g_off3) {
        const float4 f = __ldg(F4 + k.site[q]);
        const float dot = fmaf(gg[0], f.x, fmaf(gg[1], f.y, gg[2] * f.z));
        for (int c = 0; c < 3; c++) d[c] = fmaf(k.dw[q][c], dot, d[c]);
      }
    }
    if (g_off3)
      for (int c = 0; c < 3; c++) g_off3[3 * p + c] += d[c];
  }
}

// The three stencil kernels work on tiles of SX x SY x SZ sites, one CTA of
// SX x SY threads per tile; each thread walks one z-column of the tile.  The
// tile's input with a 1-site periodic halo is staged in shared memory, so
// every input value is read from global memory about 1.5 times.
constexpr int SX = 32, SY = 8, SZ = 8;
constexpr int HX = SX + 2, HY = SY + 2, HZ = SZ + 2;
constexpr int STENCIL_THREADS = SX * SY;

struct Tile {
  int x0, y0, z0, tx, ty;
};

__device__ inline Tile tile_of()
{
  return {(int)blockIdx.x * SX, (int)blockIdx.y * SY, (int)blockIdx.z * SZ, (int)threadIdx.x % SX,
          (int)threadIdx.x / SX};
}

// halo site t of the tile (t < HX*HY*HZ) -> periodic global site index
__device__ inline int64_t halo_site(const Geom& g, const Tile& T, int t)
{
  const int i = t % HX, j = (t / HX) % HY, k = t / (HX * HY);
  return site_index(g, wrap_add(T.x0, i - 1, g.n[0]), wrap_add(T.y0, j - 1, g.n[1]),
                    wrap_add(T.z0, k - 1, g.n[2]));
}

// F_c(g) = sum_o S[c][o] rho(g + o); o = (dz, dy, dx) in {-1,0,1}^3,
// S index c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1).
__global__ void __launch_bounds__(STENCIL_THREADS) k_stencil(Geom g, const float* __restrict__ rho,
                                                             const float* __restrict__ S,
                                                             float4* __restrict__ F4)
{
  __shared__ float s[81];
  __shared__ float r[HZ][HY][HX];
  const Tile T = tile_of();
  if (threadIdx.x < 81) s[threadIdx.x] = S[threadIdx.x];
  for (int t = threadIdx.x; t < HX * HY * HZ; t += STENCIL_THREADS)
    (&r[0][0][0])[t] = __ldg(rho + halo_site(g, T, t));
  __syncthreads();
  const int x = T.x0 + T.tx, y = T.y0 + T.ty;
  if (x >= g.n[0] || y >= g.n[1]) return;
  for (int kz = 0; kz < SZ && T.z0 + kz < g.n[2]; kz++) {
    float a[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const float v = r[kz + o / 9][T.ty + (o / 3) % 3][T.tx + o % 3];
#pragma unroll
      for (int c = 0; c < 3; c++) a[c] = fmaf(s[c * 27 + o], v, a[c]);
    }
    F4[site_index(g, x, y, T.z0 + kz)] = make_float4(a[0], a[1], a[2], 0.f);
  }
}

// gR(h) = sum_c sum_o S[c][o] gF_c(h - o)
__global__ void __launch_bounds__(STENCIL_THREADS) k_stencil_adj_rho(Geom g,
                                                                     const float4* __restrict__ gF4,
                                                                     const float* __restrict__ S,
                                                                     float* __restrict__ g_rho)
{
  __shared__ float s[81];
  __shared__ float f[3][HZ][HY][HX];
  const Tile T = tile_of();
  if (threadIdx.x < 81) s[threadIdx.x] = S[threadIdx.x];
  for (int t = threadIdx.x; t < HX * HY * HZ; t += STENCIL_THREADS) {
    const float4 v = __ldg(gF4 + halo_site(g, T, t));
    (&f[0][0][0][0])[t] = v.x;
    (&f[1][0][0][0])[t] = v.y;
    (&f[2][0][0][0])[t] = v.z;
  }
  __syncthreads();
  const int x = T.x0 + T.tx, y = T.y0 + T.ty;
  if (x >= g.n[0] || y >= g.n[1]) return;
  for (int kz = 0; kz < SZ && T.z0 + kz < g.n[2]; kz++) {
    float a = 0.f;
#pragma unroll
    for (int o = 0; o < 27; o++) {
      // h - o for o = (dz, dy, dx): halo offset (1 - d) per axis
      const int k = kz + 2 - o / 9, j = T.ty + 2 - (o / 3) % 3, i = T.tx + 2 - o % 3;
#pragma unroll
      for (int c = 0; c < 3; c++) a = fmaf(s[c * 27 + o], f[c][k][j][i], a);
    }
    g_rho[site_index(g, x, y, T.z0 + kz)] += a;
  }
}

// gS[c][o] = sum_g gF_c(g) rho(g + o).  Every thread keeps the 81 sums of
// its z-column in registers; the warps reduce them with shuffles, the CTA
// adds its 8 warps in order and writes one row of `partial` per tile;
// k_stencil_adj_S_sum adds the rows in a fixed order.
__global__ void __launch_bounds__(STENCIL_THREADS) k_stencil_adj_S(Geom g,
                                                                   const float4* __restrict__ gF4,
                                                                   const float* __restrict__ rho,
                                                                   float* __restrict__ partial)
{
  __shared__ float r[HZ][HY][HX];
  __shared__ float red[STENCIL_THREADS / 32][81];
  const Tile T = tile_of();
  for (int t = threadIdx.x; t < HX * HY * HZ; t += STENCIL_THREADS)
    (&r[0][0][0])[t] = __ldg(rho + halo_site(g, T, t));
  __syncthreads();
  float acc[81];
#pragma unroll
  for (int q = 0; q < 81; q++) acc[q] = 0.f;
  const int x = T.x0 + T.tx, y = T.y0 + T.ty;
  if (x < g.n[0] && y < g.n[1]) {
    for (int kz = 0; kz < SZ && T.z0 + kz < g.n[2]; kz++) {
      const float4 q = __ldg(gF4 + site_index(g, x, y, T.z0 + kz));
#pragma unroll
      for (int o = 0; o < 27; o++) {
        const float v = r[kz + o / 9][T.ty + (o / 3) % 3][T.tx + o % 3];
        acc[o] = fmaf(q.x, v, acc[o]);
        acc[27 + o] = fmaf(q.y, v, acc[27 + o]);
        acc[54 + o] = fmaf(q.z, v, acc[54 + o]);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 81; q++) {
    float v = acc[q];
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 81) {
    const int64_t tile = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
    float v = 0.f;
    for (int w = 0; w < STENCIL_THREADS / 32; w++) v += red[w][threadIdx.x];
    partial[tile * 81 + threadIdx.x] = v;
  }
}

__global__ void k_stencil_adj_S_sum(int ntiles, const float* __restrict__ partial, float* gS)
{
  __shared__ float red[4][81];
  // 4 x 81 threads: each sums a quarter of the tiles, then the quarters
  const int out = threadIdx.x % 81, q = threadIdx.x / 81;
  if (threadIdx.x < 324) {
    float v = 0.f;
    for (int t = q; t < ntiles; t += 4) v += partial[(size_t)t * 81 + out];
    red[q][out] = v;
  }
  __syncthreads();
  if (threadIdx.x < 81) gS[threadIdx.x] += (red[0][threadIdx.x] + red[1][threadIdx.x]) +
                                           (red[2][threadIdx.x] + red[3][threadIdx.x]);
}

// ------------------------------------------------------ chain state
// Cell and FP32 in-cell offset of a box-unit FP64 position: u = pos * inv_res
// (the product by the reciprocal, as a division by a scalar runs on the GPU
// in torch), floor, the offset u - floor(u) rounded to FP32 with the carry of
// an offset that rounds up to 1, then the periodic wrap.
__device__ __forceinline__ int32_t pos_state(const Geom& g, const double* p, double inv_res,
                                             float o[3])
{
  long long ci[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double u = __dmul_rn(p[d], inv_res);
    double fl = floor(u);
    float od = __double2float_rn(__dsub_rn(u, fl));
    if (od >= 1.0f) {
      od = 0.0f;
      fl = __dadd_rn(fl, 1.0);
    }
    long long c = (long long)fl % (long long)g.n[d];
    if (c < 0) c += g.n[d];
    ci[d] = c;
    o[d] = od;
  }
  return (int32_t)(ci[0] + (long long)g.n[0] * (ci[1] + (long long)g.n[1] * ci[2]));
}

// Sort key of a cell: its brick, then its place in the brick (x fastest),
// so that sorted particles come grouped by brick and by cell inside it.
__device__ __forceinline__ int32_t brick_key(const Geom& g, int32_t c)
{
  const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
  const int64_t b = brick_of(g, x, y, z);
  return (int32_t)(b * (BRICK * BRICK * BRICK) + (x % BRICK) + BRICK * ((y % BRICK) + BRICK * (z % BRICK)));
}

// Caller order, coalesced: the sort key of every particle (brick_key) and
// its 32-byte record (cell, offsets, FP32 velocity, FP32 mass), so that the
// permutation reads one full sector per particle.
__global__ void k_pm_pack(Geom g, int64_t np, const double* __restrict__ pos,
                          const double* __restrict__ vel, const double* __restrict__ mass,
                          double inv_res, int32_t* __restrict__ key, uint4* __restrict__ rec)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    float o[3];
    const int32_t c = pos_state(g, pos + 3 * i, inv_res, o);
    key[i] = brick_key(g, c);
    const float m = mass ? __double2float_rn(mass[i]) : 0.0f;
    rec[2 * i] = make_uint4((uint32_t)c, __float_as_uint(o[0]), __float_as_uint(o[1]),
                            __float_as_uint(o[2]));
    rec[2 * i + 1] = make_uint4(__float_as_uint(__double2float_rn(vel[3 * i])),
                                __float_as_uint(__double2float_rn(vel[3 * i + 1])),
                                __float_as_uint(__double2float_rn(vel[3 * i + 2])), __float_as_uint(m));
  }
}

// Slot i takes the record of particle order[i].
__global__ void k_pm_unpack(int64_t np, const int64_t* __restrict__ order, const uint4* __restrict__ rec,
                            int32_t* __restrict__ cell, float* __restrict__ off3,
                            float* __restrict__ vel3, float* __restrict__ m)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = order[i];
    const uint4 a = rec[2 * s], b = rec[2 * s + 1];
    cell[i] = (int32_t)a.x;
    off3[3 * i] = __uint_as_float(a.y), off3[3 * i + 1] = __uint_as_float(a.z);
    off3[3 * i + 2] = __uint_as_float(a.w);
    vel3[3 * i] = __uint_as_float(b.x), vel3[3 * i + 1] = __uint_as_float(b.y);
    vel3[3 * i + 2] = __uint_as_float(b.z);
    if (m) m[i] = __uint_as_float(b.w);
  }
}

// First slot of every brick among cells sorted by brick_key (bricks without
// particles start where the next one does; brick_start[nb] = np): one thread
// per brick, a binary search over the sorted slots.
__global__ void k_pm_brick_start(Geom g, int64_t np, const int32_t* __restrict__ cell,
                                 int64_t* __restrict__ brick_start)
{
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= g.nbricks;
       b += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = np;  // first slot whose brick is b or later
    while (lo < hi) {
      const int64_t mid = lo + ((hi - lo) >> 1);
      const int32_t c = cell[mid];
      const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
      if (brick_of(g, x, y, z) < b) lo = mid + 1;
      else hi = mid;
    }
    brick_start[b] = lo;
  }
}

// The gradients of slot i as the 32-byte record of particle order[i] (one
// full sector written per particle; no partial-sector writes).
__global__ void k_pm_grads_scatter(int64_t np, const int64_t* __restrict__ order,
                                   const float* __restrict__ g_off3, const float* __restrict__ g_vel3,
                                   const float* __restrict__ g_m, uint4* __restrict__ rec)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = order[i];
    rec[2 * s] = make_uint4(__float_as_uint(g_off3[3 * i]), __float_as_uint(g_off3[3 * i + 1]),
                            __float_as_uint(g_off3[3 * i + 2]), __float_as_uint(g_m[i]));
    rec[2 * s + 1] = make_uint4(__float_as_uint(g_vel3[3 * i]), __float_as_uint(g_vel3[3 * i + 1]),
                                __float_as_uint(g_vel3[3 * i + 2]), 0u);
  }
}

// Caller order, coalesced: the records into FP64 gradients (the offset
// gradient times inv_res: per box unit).
__global__ void k_pm_grads_unpack(int64_t np, const uint4* __restrict__ rec, double inv_res,
                                  double* __restrict__ g_pos, double* __restrict__ g_vel,
                                  double* __restrict__ g_mass)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint4 a = rec[2 * i], b = rec[2 * i + 1];
    g_pos[3 * i] = __dmul_rn((double)__uint_as_float(a.x), inv_res);
    g_pos[3 * i + 1] = __dmul_rn((double)__uint_as_float(a.y), inv_res);
    g_pos[3 * i + 2] = __dmul_rn((double)__uint_as_float(a.z), inv_res);
    g_mass[i] = (double)__uint_as_float(a.w);
    g_vel[3 * i] = (double)__uint_as_float(b.x);
    g_vel[3 * i + 1] = (double)__uint_as_float(b.y);
    g_vel[3 * i + 2] = (double)__uint_as_float(b.z);
  }
}

}  // namespace

inline dim3 stencil_grid(const Geom& g)
{
  return dim3((g.n[0] + SX - 1) / SX, (g.n[1] + SY - 1) / SY, (g.n[2] + SZ - 1) / SZ);
}

inline int64_t stencil_tiles(const Geom& g)
{
  const dim3 d = stencil_grid(g);
  return (int64_t)d.x * d.y * d.z;
}

// The chain's deposit into rho (+=): per particle, or brick-tiled when
// brick_start is given (particles grouped by brick, nbricks + 1 entries).
cudaError_t launch_pm_deposit(lf2_ctx* c, int64_t np, const int64_t* brick_start, const int32_t* cell,
                              const float* off3, const float* mass, float gmass, float* rho)
{
  const double vol = c->res * c->res * c->res;
  const float inv_vol = (float)(1.0 / vol);
  const Geom g = c->g;
  const unsigned nb = (unsigned)g.nbricks;
  if (c->mode == LF2_DEPOSIT_FIXED64) {
    // integer sums in the context's scratch (zero between calls)
    if (!c->pm_acc) {
      cudaError_t e = cudaMalloc(&c->pm_acc, sizeof(unsigned long long) * (size_t)g.nsites + 256);
      if (e != cudaSuccess) return e;
      e = cudaMemsetAsync(c->pm_acc, 0, sizeof(unsigned long long) * (size_t)g.nsites + 256, c->stream);
      if (e != cudaSuccess) return e;
    }
    uint32_t* mmax = reinterpret_cast<uint32_t*>(c->pm_acc + g.nsites);
    if (mass) {
      cudaError_t e = cudaMemsetAsync(mmax, 0, sizeof(uint32_t), c->stream);
      if (e != cudaSuccess) return e;
      c->launches += 1;
      k_pm_mass_max<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(np, mass, mmax);
    }
    c->launches += 2;
    if (brick_start)
      k_pm_deposit_fixed_tile<<<nb, 256, 0, c->stream>>>(g, np, brick_start, cell, off3, mass, mmax,
                                                          c->pm_acc);
    else
      k_pm_deposit_fixed<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(g, np, cell, off3,
                                                                                mass, mmax, c->pm_acc);
    k_pm_fixed_to_rho<<<grid_for(g.nsites, PM_THREADS), PM_THREADS, 0, c->stream>>>(
        g.nsites, c->pm_acc, mass, mmax, gmass, inv_vol, rho, c->flags);
    return cudaGetLastError();
  }
  c->launches += 1;
  if (brick_start)
    k_pm_deposit_tile<<<nb, 256, 0, c->stream>>>(g, np, brick_start, cell, off3, mass, gmass, inv_vol,
                                                 rho);
  else
    k_pm_deposit<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(g, np, cell, off3, mass,
                                                                          gmass, inv_vol, rho);
  return cudaGetLastError();
}

cudaError_t launch_pm(lf2_ctx* c, int op, int64_t np, const int32_t* cell, const float* off3,
                      const float* mass, float gmass, const float* in_a, const float* in_b,
                      float* out_a, float* out_b, float dta, float dtb, int32_t* cell_rw,
                      float* off_rw, float* vel_rw)
{
  const double vol = c->res * c->res * c->res;
  const float inv_vol = (float)(1.0 / vol);
  const Geom g = c->g;
  switch (op) {
    case 0:  // deposit into out_a
      return launch_pm_deposit(c, np, nullptr, cell, off3, mass, gmass, out_a);
    case 1:  // gather in_a (F4) -> out_a (np x 3)
      c->launches += 1;
      k_pm_gather<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
          g, np, cell, off3, reinterpret_cast<const float4*>(in_a), out_a);
      break;
    case 2:  // kick (in_a = G, may be NULL) + drift
      c->launches += 1;
      k_pm_kick_drift<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
          g, np, cell_rw, off_rw, vel_rw, in_a, dta, dtb, c->flags);
      break;
    case 3:  // deposit adjoint: in_a = g_rho; out_a = g_off (+=), out_b = g_mass (+=)
      c->launches += 1;
      k_pm_deposit_adj<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
          g, np, cell, off3, mass, gmass, inv_vol, in_a, out_a, out_b);
      break;
    case 4:  // gather adjoint: in_a = F4, in_b = gG; out_a = gF4 (+=), out_b = g_off (+=)
      c->launches += 1;
      k_pm_gather_adj<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
          g, np, cell, off3, reinterpret_cast<const float4*>(in_a), in_b,
          reinterpret_cast<float4*>(out_a), out_b);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_stencil(lf2_ctx* c, int op, const float* a, const float* S, float* out,
                           float* partial)
{
  const Geom g = c->g;
  const dim3 grid = stencil_grid(g);
  if (op == 0) {  // a = rho -> out = F4
    c->launches += 1;
    k_stencil<<<grid, STENCIL_THREADS, 0, c->stream>>>(g, a, S, reinterpret_cast<float4*>(out));
  } else if (op == 1) {  // a = gF4 -> out = g_rho (+=)
    c->launches += 1;
    k_stencil_adj_rho<<<grid, STENCIL_THREADS, 0, c->stream>>>(
        g, reinterpret_cast<const float4*>(a), S, out);
  } else {  // a = gF4, S = rho -> out = gS (+=)
    c->launches += 2;
    k_stencil_adj_S<<<grid, STENCIL_THREADS, 0, c->stream>>>(
        g, reinterpret_cast<const float4*>(a), S, partial);
    k_stencil_adj_S_sum<<<1, 352, 0, c->stream>>>((int)stencil_tiles(g), partial, out);
  }
  return cudaGetLastError();
}

size_t stencil_partial_floats(const lf2_ctx* c) { return (size_t)stencil_tiles(c->g) * 81; }

cudaError_t launch_pm_step(lf2_ctx* c, int64_t np, int32_t* cell, float* off3, float* vel3,
                           const float* F4, float dtk, float dtn)
{
  if (np == 0) return cudaSuccess;
  c->launches += 1;
  k_pm_gather_kick_drift<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
      c->g, np, cell, off3, vel3, reinterpret_cast<const float4*>(F4), dtk, dtn, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_pm_pack(lf2_ctx* c, int64_t np, const double* pos, const double* vel,
                           const double* mass, double inv_res, int32_t* key, void* rec)
{
  if (np == 0) return cudaSuccess;
  c->launches += 1;
  k_pm_pack<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
      c->g, np, pos, vel, mass, inv_res, key, reinterpret_cast<uint4*>(rec));
  return cudaGetLastError();
}

cudaError_t launch_pm_unpack(lf2_ctx* c, int64_t np, const int64_t* order, const void* rec,
                             int32_t* cell, float* off3, float* vel3, float* m)
{
  if (np == 0) return cudaSuccess;
  c->launches += 1;
  k_pm_unpack<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
      np, order, reinterpret_cast<const uint4*>(rec), cell, off3, vel3, m);
  return cudaGetLastError();
}

cudaError_t launch_pm_brick_start(lf2_ctx* c, int64_t np, const int32_t* cell, int64_t* brick_start)
{
  c->launches += 1;
  k_pm_brick_start<<<grid_for(c->g.nbricks + 1, PM_THREADS), PM_THREADS, 0, c->stream>>>(
      c->g, np, cell, brick_start);
  return cudaGetLastError();
}

cudaError_t launch_pm_grads_back(lf2_ctx* c, int64_t np, const int64_t* order, const float* g_off3,
                                 const float* g_vel3, const float* g_m, double inv_res, void* rec,
                                 double* g_pos, double* g_vel, double* g_mass)
{
  if (np == 0) return cudaSuccess;
  c->launches += 2;
  k_pm_grads_scatter<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
      np, order, g_off3, g_vel3, g_m, reinterpret_cast<uint4*>(rec));
  k_pm_grads_unpack<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
      np, reinterpret_cast<const uint4*>(rec), inv_res, g_pos, g_vel, g_mass);
  return cudaGetLastError();
}

}  // namespace lf2
