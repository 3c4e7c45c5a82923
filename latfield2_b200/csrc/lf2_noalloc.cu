// lf2_noalloc.cu -- scalar CIC deposit that allocates no device memory.
//
// Some callers cannot allocate device memory once they are running: a host
// application whose device memory is handed out by its own pool (a stray
// cudaMalloc would break its budget or fragment the pool), a plugin that is
// only allowed to allocate while it is being loaded, or a time-critical loop
// that cannot afford the device-wide synchronisation cudaMalloc and cudaFree
// imply.  lf2_deposit_scalar_noalloc serves them: the caller passes its own
// device inputs and output, and the only scratch the deposit needs, the
// per-brick shell store, lives in a fixed-size array in this file.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (NOALLOC_SHELL_SLOTS * 8 bytes = 16 MiB) until the process
// exits.  Host code cannot use the array's name as a device address: the
// name is a host-side stand-in, and a kernel given it would fault or, where
// the GPU can reach host memory, silently use the wrong memory.  The device
// address is therefore looked up with cudaGetSymbolAddress, with the caller's
// device current, on every call (the lookup is cheap next to two launches,
// and a cached address would go stale if the device's context were reset and
// the module reloaded), and passed to the kernels.
//
// All calls share the array and it keeps the contents of the last call.  The
// deposit writes every shell slot it later reads and clears the error word
// at the start of each call, so nothing needs to start at zero otherwise.
// Calls that overlap on the GPU (two streams, or two host threads) race on
// the array and give wrong results; serialise them.
#include <cuda_runtime.h>

#include <cmath>

#include "lf2_common.cuh"
#include "lf2gpu.h"

namespace lf2 {

namespace {

constexpr size_t NOALLOC_SHELL_SLOTS = (size_t)LF2_NOALLOC_MAX_BRICKS * SHELL;
constexpr int NA_THREADS = 256;
constexpr int NA_SPLIT_MAX = 65535;

static __device__ __align__(256) unsigned long long g_noalloc_shell[NOALLOC_SHELL_SLOTS];
static __device__ __align__(256) unsigned int g_noalloc_flags;

struct NoallocSymbols {
  unsigned long long* shell = nullptr;
  unsigned int* flags = nullptr;
};

// Device addresses of the two arrays in the current device's context.
cudaError_t noalloc_symbols(NoallocSymbols* out)
{
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_shell);
  if (e != cudaSuccess) return e;
  void* q = nullptr;
  if ((e = cudaGetSymbolAddress(&q, g_noalloc_flags)) != cudaSuccess) return e;
  out->shell = static_cast<unsigned long long*>(p);
  out->flags = static_cast<unsigned int*>(q);
  return cudaSuccess;
}

struct NaParams {
  float mf;           // FP32: particle mass / res^3
  float fixed_scale;  // fixed: 2^-32 * particle mass / res^3
};

template <bool FIXED>
__global__ void __launch_bounds__(NA_THREADS) k_deposit_noalloc(
    Geom g, NaParams pp, int64_t np, const int32_t* __restrict__ cell,
    const float* __restrict__ off3, const int64_t* __restrict__ brick_start,
    float* __restrict__ out, unsigned long long* __restrict__ shell, unsigned int* flags)
{
  extern __shared__ __align__(16) unsigned char smem[];
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
            ez = brick_extent(g.n[2], bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  // The caller's brick offsets are checked, never trusted: they must start
  // at 0, never decrease and never pass np.  A brick whose range breaks that
  // is clamped to [0, np] (so nothing outside the particle arrays is read)
  // and reported.
  int64_t base = brick_start[b], end = brick_start[b + 1];
  if ((b == 0 && base != 0) || base < 0 || end < base || end > np) {
    if (threadIdx.x == 0) atomicOr(flags, ERR_BAD_CELL);
    base = base < 0 ? 0 : (base > np ? np : base);
    end = end < base ? base : (end > np ? np : end);
  }
  const int64_t cnt = end - base;
  const bool split = FIXED && cnt <= NA_SPLIT_MAX;

  uint32_t* lo = reinterpret_cast<uint32_t*>(smem);
  uint32_t* hi = lo + TILE3;
  unsigned long long* a64 = reinterpret_cast<unsigned long long*>(smem);
  float* facc = reinterpret_cast<float*>(smem);
  for (int t = threadIdx.x; t < (FIXED ? 2 : 1) * TILE3; t += blockDim.x) lo[t] = 0u;
  __syncthreads();

  for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int64_t p = base + i;
    const int32_t c = cell[p];
    const float fx = off3[3 * p], fy = off3[3 * p + 1], fz = off3[3 * p + 2];
    bool ok = c >= 0 && (int64_t)c < g.nsites && fx >= 0.0f && fx < 1.0f && fy >= 0.0f &&
              fy < 1.0f && fz >= 0.0f && fz < 1.0f;
    int x = 0, y = 0, z = 0;
    if (ok) {
      x = c % g.n[0];
      y = (c / g.n[0]) % g.n[1];
      z = c / (g.n[0] * g.n[1]);
      ok = x >= x0 && x < x0 + ex && y >= y0 && y < y0 + ey && z >= z0 && z < z0 + ez;
    }
    if (!ok) {  // not inside this brick: reported, never indexed
      atomicOr(flags, ERR_BAD_CELL);
      continue;
    }
    const int t0 = (x - x0) + TILE * ((y - y0) + TILE * (z - z0));
    if (FIXED) {
      const uint32_t ux = __float2uint_rn(fx * 2147483648.0f);
      const uint32_t uy = __float2uint_rn(fy * 2147483648.0f);
      const uint32_t uz = __float2uint_rn(fz * 2147483648.0f);
      const uint32_t qx[2] = {(1u << 31) - ux, ux};
      const uint32_t qy[2] = {(1u << 31) - uy, uy};
      const uint32_t qz[2] = {(1u << 31) - uz, uz};
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
        const uint64_t q = fixed_corner(qx[cx], qy[cy], qz[cz]);
        const int t = t0 + cx + cy * TILE + cz * TILE * TILE;
        if (split) {
          atomicAdd(&lo[t], (uint32_t)(q & 0xffffu));
          atomicAdd(&hi[t], (uint32_t)(q >> 16));
        } else {
          atomicAdd(&a64[t], (unsigned long long)q);
        }
      }
    } else {
      const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy), gz = __fsub_rn(1.0f, fz);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
        const float w = __fmul_rn(__fmul_rn(__fmul_rn(cx ? fx : gx, cy ? fy : gy), cz ? fz : gz),
                                  pp.mf);
        atomicAdd(&facc[t0 + cx + cy * TILE + cz * TILE * TILE], w);
      }
    }
  }
  __syncthreads();

  unsigned long long* sp = shell + (size_t)b * SHELL;
  for (int t = threadIdx.x; t < TILE3; t += blockDim.x) {
    const int i = t % TILE, j = (t / TILE) % TILE, k = t / (TILE * TILE);
    if (i > ex || j > ey || k > ez) continue;
    const bool on_shell = i == 0 || i == ex || j == 0 || j == ey || k == 0 || k == ez;
    uint64_t q = 0;
    float f = 0.0f;
    if (FIXED) q = split ? (uint64_t)lo[t] + ((uint64_t)hi[t] << 16) : a64[t];
    else f = facc[t];
    if (on_shell) {
      const int si = shell_index(i == ex ? BRICK : i, j == ey ? BRICK : j, k == ez ? BRICK : k);
      if (FIXED) sp[si] = q;
      else reinterpret_cast<float*>(sp)[si] = f;
    } else {
      const int64_t s = site_index(g, x0 + i, y0 + j, z0 + k);
      if (FIXED) {
        if ((long long)q < 0) atomicOr(flags, ERR_FIXED_OVERFLOW);
        out[s] = __fmul_rn(__ll2float_rn((long long)q), pp.fixed_scale);
      } else {
        out[s] = f;
      }
    }
  }
}

// Finishes the owned vertices with a zero coordinate from the shell values of
// the up to 8 bricks that touch them (fixed order).
template <bool FIXED>
__global__ void k_fixup_noalloc(Geom g, const unsigned long long* __restrict__ shell,
                                float fixed_scale, float* __restrict__ out, unsigned int* flags)
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
    if (f < ey * ez) {
      i = 0;
      j = f % ey;
      k = f / ey;
    } else if (f < ey * ez + (ex - 1) * ez) {
      const int r = f - ey * ez;
      j = 0;
      i = 1 + r % (ex - 1);
      k = r / (ex - 1);
    } else {
      const int r = f - ey * ez - (ex - 1) * ez;
      k = 0;
      i = 1 + r % (ex - 1);
      j = 1 + r / (ex - 1);
    }
    const int zmask = (i == 0 ? 1 : 0) | (j == 0 ? 2 : 0) | (k == 0 ? 4 : 0);
    uint64_t qs = 0;
    float fs = 0.0f;
    for (int s = 0; s < 8; s++) {
      if ((s & zmask) != s) continue;
      const int nbx = (s & 1) ? bxm : bx, nby = (s & 2) ? bym : by, nbz = (s & 4) ? bzm : bz;
      const int64_t nb = (int64_t)nbx + (int64_t)g.nb[0] * ((int64_t)nby + (int64_t)g.nb[1] * nbz);
      const int si = shell_index((s & 1) ? BRICK : i, (s & 2) ? BRICK : j, (s & 4) ? BRICK : k);
      const unsigned long long* sp = shell + (size_t)nb * SHELL;
      if (FIXED) qs += sp[si];
      else fs = __fadd_rn(fs, reinterpret_cast<const float*>(sp)[si]);
    }
    const int64_t site = site_index(g, x0 + i, y0 + j, z0 + k);
    if (FIXED) {
      if ((long long)qs < 0) atomicOr(flags, ERR_FIXED_OVERFLOW);
      out[site] = __fmul_rn(__ll2float_rn((long long)qs), fixed_scale);
    } else {
      out[site] = fs;
    }
  }
}

int bits_for(int n)
{
  int b = 0;
  while ((1ll << b) < n) b++;
  return b;
}

}  // namespace
}  // namespace lf2

using namespace lf2;

extern "C" lf2_status lf2_deposit_scalar_noalloc(const int n[3], const double box[3],
                                                 int deposit_mode, double particle_mass,
                                                 int64_t np, const int32_t* cell,
                                                 const float* off3, const int64_t* brick_start,
                                                 float* rho, void* stream, uint32_t* flags)
{
  if (!n || !box || !brick_start || !rho || np < 0 || (np > 0 && (!cell || !off3)))
    return LF2_ERR_ARG;
  if (deposit_mode != LF2_DEPOSIT_FP32 && deposit_mode != LF2_DEPOSIT_FIXED64) return LF2_ERR_ARG;
  if (!(particle_mass > 0)) return LF2_ERR_ARG;
  for (int d = 0; d < 3; d++)
    if (n[d] < 1 || !(box[d] > 0)) return LF2_ERR_ARG;
  const double res = box[0] / n[0];
  if (std::fabs(box[1] / n[1] - res) > 1e-12 * res || std::fabs(box[2] / n[2] - res) > 1e-12 * res)
    return LF2_ERR_ARG;
  const int64_t nsites = (int64_t)n[0] * n[1] * n[2];
  if (nsites >= (1ll << 31) || bits_for(n[0]) + bits_for(n[1]) + bits_for(n[2]) > 32)
    return LF2_ERR_UNSUPPORTED;
  Geom g{};
  for (int d = 0; d < 3; d++) {
    g.n[d] = n[d];
    g.nb[d] = (n[d] + BRICK - 1) / BRICK;
  }
  g.nsites = nsites;
  g.nbricks = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
  if (g.nbricks > LF2_NOALLOC_MAX_BRICKS) return LF2_ERR_UNSUPPORTED;  // shell store too small

  NoallocSymbols sym;
  if (noalloc_symbols(&sym) != cudaSuccess) return LF2_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double vol = res * res * res;
  NaParams pp;
  pp.mf = (float)(particle_mass / vol);
  pp.fixed_scale = (float)(std::ldexp(1.0, -32) * particle_mass / vol);
  const bool fixed = deposit_mode == LF2_DEPOSIT_FIXED64;
  const size_t smem = (size_t)TILE3 * (fixed ? 8 : 4);
  const unsigned grid = (unsigned)g.nbricks;

  // Each launch is checked right after it.  An error left pending by an
  // earlier, unrelated runtime call is reported by the first check too, so
  // such an error fails this call (and is cleared by it).
  if (cudaMemsetAsync(sym.flags, 0, sizeof(unsigned int), st) != cudaSuccess) return LF2_ERR_CUDA;
  if (fixed)
    k_deposit_noalloc<true><<<grid, NA_THREADS, smem, st>>>(g, pp, np, cell, off3, brick_start,
                                                            rho, sym.shell, sym.flags);
  else
    k_deposit_noalloc<false><<<grid, NA_THREADS, smem, st>>>(g, pp, np, cell, off3, brick_start,
                                                             rho, sym.shell, sym.flags);
  if (cudaGetLastError() != cudaSuccess) return LF2_ERR_CUDA;
  if (fixed)
    k_fixup_noalloc<true><<<grid, 256, 0, st>>>(g, sym.shell, pp.fixed_scale, rho, sym.flags);
  else
    k_fixup_noalloc<false><<<grid, 256, 0, st>>>(g, sym.shell, pp.fixed_scale, rho, sym.flags);
  if (cudaGetLastError() != cudaSuccess) return LF2_ERR_CUDA;
  if (flags) {
    unsigned int f = 0;
    if (cudaMemcpyAsync(&f, sym.flags, sizeof f, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return LF2_ERR_CUDA;
    *flags = f;
    if (f) return LF2_ERR_STATE;
  }
  return LF2_OK;
}
