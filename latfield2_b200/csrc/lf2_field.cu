// lf2_field.cu -- field layout conversion, periodic halo fill and the FP64
// conservation reductions.
//
// Internal field layout: FP32, component-major, no halo, periodic.  The
// reference layout (LATfield2_Field_decl.hpp:760-788, LATfield2_Lattice.hpp:
// 110-113) is halo'd with interleaved components: data[idx * C + c] with
// idx = (x+h) + G0 * ((y+h) + G1 * (z+h)), Gi = ni + 2h.
#include <cuda_runtime.h>

#include "lf2_internal.h"

namespace lf2 {

namespace {

inline int grid_for(int64_t n, int threads)
{
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 64) g = 148 * 64;
  return (int)(g > 0 ? g : 1);
}

__device__ inline int wrap_coord(int v, int n)
{
  v %= n;
  return v < 0 ? v + n : v;
}

// Every gross site of the reference layout; halo sites either copy their
// periodic image (Field::updateHalo, LATfield2_Field_decl.hpp:889-935) or are 0.
template <typename T>
__global__ void k_export(Geom g, int comps, const float* __restrict__ src, T* __restrict__ dst,
                         int halo, int fill_halo)
{
  const int64_t G0 = g.n[0] + 2 * halo, G1 = g.n[1] + 2 * halo, G2 = g.n[2] + 2 * halo;
  const int64_t total = G0 * G1 * G2;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(idx % G0) - halo;
    int y = (int)((idx / G0) % G1) - halo;
    int z = (int)(idx / (G0 * G1)) - halo;
    const bool inside = x >= 0 && x < g.n[0] && y >= 0 && y < g.n[1] && z >= 0 && z < g.n[2];
    if (!inside && !fill_halo) {
      for (int c = 0; c < comps; c++) dst[idx * comps + c] = (T)0;
      continue;
    }
    x = wrap_coord(x, g.n[0]);
    y = wrap_coord(y, g.n[1]);
    z = wrap_coord(z, g.n[2]);
    const int64_t s = site_index(g, x, y, z);
    for (int c = 0; c < comps; c++) dst[idx * comps + c] = (T)src[c * g.nsites + s];
  }
}

template <typename T>
__global__ void k_import(Geom g, int comps, float* __restrict__ dst, const T* __restrict__ src,
                         int halo)
{
  const int64_t G0 = g.n[0] + 2 * halo, G1 = g.n[1] + 2 * halo;
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < g.nsites;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(s % g.n[0]), y = (int)((s / g.n[0]) % g.n[1]),
              z = (int)(s / ((int64_t)g.n[0] * g.n[1]));
    const int64_t idx = (x + halo) + G0 * ((y + halo) + G1 * (int64_t)(z + halo));
    for (int c = 0; c < comps; c++) dst[c * g.nsites + s] = (float)src[idx * comps + c];
  }
}

// In-place halo fill of a device array in the reference layout.
template <typename T>
__global__ void k_halo_fill(Geom g, int comps, T* __restrict__ data, int halo)
{
  const int64_t G0 = g.n[0] + 2 * halo, G1 = g.n[1] + 2 * halo, G2 = g.n[2] + 2 * halo;
  const int64_t total = G0 * G1 * G2;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(idx % G0) - halo;
    const int y = (int)((idx / G0) % G1) - halo;
    const int z = (int)(idx / (G0 * G1)) - halo;
    if (x >= 0 && x < g.n[0] && y >= 0 && y < g.n[1] && z >= 0 && z < g.n[2]) continue;
    const int64_t from = (wrap_coord(x, g.n[0]) + halo) +
                         G0 * ((wrap_coord(y, g.n[1]) + halo) + G1 * (int64_t)(wrap_coord(z, g.n[2]) + halo));
    for (int c = 0; c < comps; c++) data[idx * comps + c] = data[from * comps + c];
  }
}

// FP64 sums per brick: mass, m*vx, m*vy, m*vz and max |v|^2, then a fixed-order
// reduction over bricks (one CTA) so the totals are reproducible.
// Per brick, in a fixed order: mass, momentum (3), max |v|^2, sum |v|^2,
// min |v|^2 (FP64; |v|^2 in double from the FP32 components, as the
// reference's callbacks compute it).
constexpr int NSUM = 7;

__global__ void __launch_bounds__(256) k_brick_sums(StoreView v, double gmass, double* out)
{
  __shared__ double sh[NSUM][256];
  const int64_t b = blockIdx.x;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  double s[NSUM] = {0, 0, 0, 0, 0, 0, INFINITY};
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int64_t p = base + i;
    const double m = v.a.mass ? (double)v.a.mass[p] : gmass;
    const double vx = v.a.vx[p], vy = v.a.vy[p], vz = v.a.vz[p];
    const double v2 = vx * vx + vy * vy + vz * vz;
    s[0] += m;
    s[1] += m * vx;
    s[2] += m * vy;
    s[3] += m * vz;
    s[4] = fmax(s[4], v2);
    s[5] += v2;
    s[6] = fmin(s[6], v2);
  }
  for (int k = 0; k < NSUM; k++) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
      sh[4][threadIdx.x] = fmax(sh[4][threadIdx.x], sh[4][threadIdx.x + o]);
      sh[5][threadIdx.x] += sh[5][threadIdx.x + o];
      sh[6][threadIdx.x] = fmin(sh[6][threadIdx.x], sh[6][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x < NSUM) out[b * NSUM + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(512) k_sum_bricks(int64_t nb, const double* __restrict__ in,
                                                    double* stats)
{
  __shared__ double sh[NSUM][512];
  const int t = threadIdx.x;
  const int64_t per = (nb + blockDim.x - 1) / blockDim.x;
  const int64_t lo = t * per, hi = min(nb, lo + per);
  double s[NSUM] = {0, 0, 0, 0, 0, 0, INFINITY};
  for (int64_t b = lo; b < hi; b++) {
    for (int k = 0; k < 4; k++) s[k] += in[b * NSUM + k];
    s[4] = fmax(s[4], in[b * NSUM + 4]);
    s[5] += in[b * NSUM + 5];
    s[6] = fmin(s[6], in[b * NSUM + 6]);
  }
  for (int k = 0; k < NSUM; k++) sh[k][t] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o) {
      for (int k = 0; k < 4; k++) sh[k][t] += sh[k][t + o];
      sh[4][t] = fmax(sh[4][t], sh[4][t + o]);
      sh[5][t] += sh[5][t + o];
      sh[6][t] = fmin(sh[6][t], sh[6][t + o]);
    }
    __syncthreads();
  }
  if (t < NSUM) stats[1 + t] = sh[t][0];
}

}  // namespace

cudaError_t launch_export(lf2_ctx* c, int comps, const float* src, void* dst, int halo,
                          int real_bytes, int fill_halo)
{
  c->launches += 1;
  const int64_t total =
      (int64_t)(c->g.n[0] + 2 * halo) * (c->g.n[1] + 2 * halo) * (c->g.n[2] + 2 * halo);
  if (real_bytes == 8)
    k_export<double><<<grid_for(total, 256), 256, 0, c->stream>>>(c->g, comps, src, (double*)dst,
                                                                  halo, fill_halo);
  else
    k_export<float><<<grid_for(total, 256), 256, 0, c->stream>>>(c->g, comps, src, (float*)dst,
                                                                 halo, fill_halo);
  return cudaGetLastError();
}

cudaError_t launch_import(lf2_ctx* c, int comps, float* dst, const void* src, int halo,
                          int real_bytes)
{
  c->launches += 1;
  if (real_bytes == 8)
    k_import<double><<<grid_for(c->g.nsites, 256), 256, 0, c->stream>>>(
        c->g, comps, dst, (const double*)src, halo);
  else
    k_import<float><<<grid_for(c->g.nsites, 256), 256, 0, c->stream>>>(
        c->g, comps, dst, (const float*)src, halo);
  return cudaGetLastError();
}

cudaError_t launch_halo_fill(lf2_ctx* c, void* data, int comps, int halo, int real_bytes)
{
  c->launches += 1;
  const int64_t total =
      (int64_t)(c->g.n[0] + 2 * halo) * (c->g.n[1] + 2 * halo) * (c->g.n[2] + 2 * halo);
  if (real_bytes == 8)
    k_halo_fill<double><<<grid_for(total, 256), 256, 0, c->stream>>>(c->g, comps, (double*)data,
                                                                     halo);
  else
    k_halo_fill<float><<<grid_for(total, 256), 256, 0, c->stream>>>(c->g, comps, (float*)data,
                                                                    halo);
  return cudaGetLastError();
}

cudaError_t launch_conservation(lf2_ctx* c)
{
  c->launches += 2;
  k_brick_sums<<<(unsigned)c->g.nbricks, 256, 0, c->stream>>>(view(c), c->gmass, c->brick_sums);
  k_sum_bricks<<<1, 512, 0, c->stream>>>(c->g.nbricks, c->brick_sums, c->stats);
  return cudaGetLastError();
}

}  // namespace lf2
