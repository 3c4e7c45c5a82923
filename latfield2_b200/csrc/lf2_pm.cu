// lf2_pm.cu -- kernels of the differentiable particle-mesh chain: CIC deposit
// and gather on particles kept in the caller's order (no rebinning, so that
// gradients stay attached to their particles), the kick-drift update, a
// periodic 27-point stencil as the grid operator, and the hand-written
// adjoints of all of them.
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
// cell units; positions in box units are (cell + off) * res.
#include <cuda_runtime.h>

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

__global__ void k_pm_gather(Geom g, int64_t np, const int32_t* __restrict__ cell,
                            const float* __restrict__ off3, const float* __restrict__ F,
                            float* __restrict__ out3)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    Corners k;
    corners(g, cell[p], off3, p, k);
    float a[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; q++)
#pragma unroll
      for (int c = 0; c < 3; c++) a[c] = fmaf(k.w[q], __ldg(F + c * g.nsites + k.site[q]), a[c]);
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
                                const float* __restrict__ off3, const float* __restrict__ F,
                                const float* __restrict__ gG3, float* __restrict__ gF,
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
      float dot = 0.f;
      for (int c = 0; c < 3; c++) {
        if (gF) atomicAdd(&gF[c * g.nsites + k.site[q]], k.w[q] * gg[c]);
        if (g_off3) dot = fmaf(gg[c], __ldg(F + c * g.nsites + k.site[q]), dot);
      }
      if (g_off3)
        for (int c = 0; c < 3; c++) d[c] = fmaf(k.dw[q][c], dot, d[c]);
    }
    if (g_off3)
      for (int c = 0; c < 3; c++) g_off3[3 * p + c] += d[c];
  }
}

// F_c(g) = sum_o S[c][o] rho(g + o); o = (dz, dy, dx) in {-1,0,1}^3,
// S index c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1).
__global__ void k_stencil(Geom g, const float* __restrict__ rho, const float* __restrict__ S,
                          float* __restrict__ F)
{
  __shared__ float s[81];
  if (threadIdx.x < 81) s[threadIdx.x] = S[threadIdx.x];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.nsites;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.n[0]), y = (int)((i / g.n[0]) % g.n[1]),
              z = (int)(i / ((int64_t)g.n[0] * g.n[1]));
    float a[3] = {0.f, 0.f, 0.f};
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const float r = __ldg(rho + site_index(g, wrap_add(x, dx, g.n[0]), wrap_add(y, dy, g.n[1]),
                                                 wrap_add(z, dz, g.n[2])));
          const int o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
          for (int c = 0; c < 3; c++) a[c] = fmaf(s[c * 27 + o], r, a[c]);
        }
    for (int c = 0; c < 3; c++) F[c * g.nsites + i] = a[c];
  }
}

// gR(h) = sum_c sum_o S[c][o] gF_c(h - o)
__global__ void k_stencil_adj_rho(Geom g, const float* __restrict__ gF, const float* __restrict__ S,
                                  float* __restrict__ g_rho)
{
  __shared__ float s[81];
  if (threadIdx.x < 81) s[threadIdx.x] = S[threadIdx.x];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.nsites;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.n[0]), y = (int)((i / g.n[0]) % g.n[1]),
              z = (int)(i / ((int64_t)g.n[0] * g.n[1]));
    float a = 0.f;
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int64_t src = site_index(g, wrap_add(x, -dx, g.n[0]), wrap_add(y, -dy, g.n[1]),
                                         wrap_add(z, -dz, g.n[2]));
          const int o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
          for (int c = 0; c < 3; c++) a = fmaf(s[c * 27 + o], __ldg(gF + c * g.nsites + src), a);
        }
    g_rho[i] += a;
  }
}

// Per-CTA partial sums of gS[c][o] = sum_g gF_c(g) rho(g + o); blockIdx.y is
// the component c (27 values per thread).  k_stencil_adj_S_sum adds the CTA
// partials in a fixed order.
__global__ void __launch_bounds__(PM_THREADS) k_stencil_adj_S(Geom g, const float* __restrict__ gF,
                                                              const float* __restrict__ rho,
                                                              float* __restrict__ partial)
{
  __shared__ float red[PM_THREADS / 32][27];
  const int c = blockIdx.y;
  float acc[27];
  for (int j = 0; j < 27; j++) acc[j] = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.nsites;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.n[0]), y = (int)((i / g.n[0]) % g.n[1]),
              z = (int)(i / ((int64_t)g.n[0] * g.n[1]));
    const float f = __ldg(gF + c * g.nsites + i);
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
      for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
          const float r = __ldg(rho + site_index(g, wrap_add(x, dx, g.n[0]), wrap_add(y, dy, g.n[1]),
                                                 wrap_add(z, dz, g.n[2])));
          const int o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
          acc[o] = fmaf(f, r, acc[o]);
        }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 27; j++) {
    float v = acc[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < 27) {
    float v = 0.f;
    for (int k = 0; k < PM_THREADS / 32; k++) v += red[k][threadIdx.x];
    partial[blockIdx.x * 81 + c * 27 + threadIdx.x] = v;
  }
}

__global__ void k_stencil_adj_S_sum(int nblocks, const float* __restrict__ partial, float* gS)
{
  if (threadIdx.x < 81) {
    float v = 0.f;
    for (int b = 0; b < nblocks; b++) v += partial[b * 81 + threadIdx.x];
    gS[threadIdx.x] += v;
  }
}

}  // namespace

constexpr int STENCIL_S_BLOCKS = 148 * 2;

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
      c->launches += 1;
      k_pm_deposit<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(g, np, cell, off3, mass,
                                                                            gmass, inv_vol, out_a);
      break;
    case 1:  // gather in_a (F) -> out_a (np x 3)
      c->launches += 1;
      k_pm_gather<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(g, np, cell, off3, in_a,
                                                                           out_a);
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
    case 4:  // gather adjoint: in_a = F, in_b = gG; out_a = gF (+=), out_b = g_off (+=)
      c->launches += 1;
      k_pm_gather_adj<<<grid_for(np, PM_THREADS), PM_THREADS, 0, c->stream>>>(
          g, np, cell, off3, in_a, in_b, out_a, out_b);
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
  if (op == 0) {
    c->launches += 1;
    k_stencil<<<grid_for(g.nsites, PM_THREADS), PM_THREADS, 0, c->stream>>>(g, a, S, out);
  } else if (op == 1) {  // a = gF -> out = g_rho (+=)
    c->launches += 1;
    k_stencil_adj_rho<<<grid_for(g.nsites, PM_THREADS), PM_THREADS, 0, c->stream>>>(g, a, S, out);
  } else {  // a = gF, S = rho -> out = gS (+=)
    c->launches += 2;
    k_stencil_adj_S<<<dim3(STENCIL_S_BLOCKS, 3), PM_THREADS, 0, c->stream>>>(g, a, S, partial);
    k_stencil_adj_S_sum<<<1, 128, 0, c->stream>>>(STENCIL_S_BLOCKS, partial, out);
  }
  return cudaGetLastError();
}

size_t stencil_partial_floats() { return (size_t)STENCIL_S_BLOCKS * 81; }

}  // namespace lf2
