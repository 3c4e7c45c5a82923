// lf2_exchange.cu -- particle exchange kernels of the slab decomposition.
//
// A rank of a z-slab decomposition keeps one ghost cell plane below and one
// above its own planes.  After a drift the particles that entered a ghost
// plane leave the store (k_count_outside, k_extract_outside) and are sent to
// the neighbour that owns them; particles received from the neighbours enter
// the store through the mover path (k_pack_movers, then k_insert).  This
// replaces the particle migration of moveParticles
// (LATfield2_Particles.hpp:2176-2799) for a 1-D decomposition.
#include <cuda_runtime.h>

#include "lf2_internal.h"

namespace lf2 {

namespace {

constexpr int EX_THREADS = 256;

__device__ __forceinline__ int key_z(const Geom& g, uint32_t k)
{
  return (int)((k >> g.shift[2]) & g.mask[2]);
}

// Bricks whose z range lies inside [zlo, zhi] hold no particle to move.
__device__ __forceinline__ bool brick_inside(const Geom& g, int bz, int zlo, int zhi)
{
  const int z0 = bz * BRICK, z1 = z0 + brick_extent(g.n[2], bz) - 1;
  return z0 >= zlo && z1 <= zhi;
}

__global__ void __launch_bounds__(EX_THREADS)
    k_count_outside(StoreView v, int zlo, int zhi, unsigned long long* n)
{
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(v.g, b, bx, by, bz);
  if (brick_inside(v.g, bz, zlo, zhi)) return;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  int c = 0;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int z = key_z(v.g, v.a.key[base + i]);
    c += (z < zlo || z > zhi) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(n, (unsigned long long)c);
}

// One CTA per brick: particles with z outside [zlo, zhi] go to the output
// (slots from a global counter, any order) with their cell index; the others
// are compacted to the front of the brick's segment, in order.  A chunk is
// read completely before any of it is written, and the write cursor never
// passes the chunk's start, so the compaction is safe in place.
__global__ void __launch_bounds__(EX_THREADS)
    k_extract_outside(StoreView v, int zlo, int zhi, int32_t* __restrict__ cell,
                      float* __restrict__ off3, float* __restrict__ vel3,
                      float* __restrict__ mass, int64_t* __restrict__ id,
                      unsigned long long* out_count)
{
  __shared__ int warp_tot[32];
  const Geom& g = v.g;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  if (brick_inside(g, bz, zlo, zhi)) return;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  int cursor = 0;
  for (int c0 = 0; c0 < cnt; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    const bool act = i < cnt;
    uint32_t k = 0;
    float ox = 0, oy = 0, oz = 0, vx = 0, vy = 0, vz = 0, m = 0;
    int64_t pid = 0;
    if (act) {
      const int64_t p = base + i;
      k = v.a.key[p];
      ox = v.a.ox[p], oy = v.a.oy[p], oz = v.a.oz[p];
      vx = v.a.vx[p], vy = v.a.vy[p], vz = v.a.vz[p];
      if (v.a.mass) m = v.a.mass[p];
      if (v.a.id) pid = v.a.id[p];
    }
    const int z = key_z(g, k);
    const bool out = act && (z < zlo || z > zhi);
    const bool keep = act && !out;
    int total;
    const int pos = block_exclusive_scan(keep ? 1 : 0, warp_tot, &total);  // syncs the block
    if (keep) {
      const int64_t q = base + cursor + pos;
      v.a.key[q] = k;
      v.a.ox[q] = ox, v.a.oy[q] = oy, v.a.oz[q] = oz;
      v.a.vx[q] = vx, v.a.vy[q] = vy, v.a.vz[q] = vz;
      if (v.a.mass) v.a.mass[q] = m;
      if (v.a.id) v.a.id[q] = pid;
    } else if (out) {
      int x, y, zz;
      unpack_key(g, k, x, y, zz);
      const int64_t q = (int64_t)atomicAdd(out_count, 1ull);
      cell[q] = (int32_t)site_index(g, x, y, zz);
      off3[3 * q] = ox, off3[3 * q + 1] = oy, off3[3 * q + 2] = oz;
      vel3[3 * q] = vx, vel3[3 * q + 1] = vy, vel3[3 * q + 2] = vz;
      if (mass) mass[q] = m;
      if (id) id[q] = pid;
    }
    cursor += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) v.count[b] = cursor;
}

// New particles (cell index, offsets, velocities) into the mover buffer, with
// the mover count set to n, ready for k_insert.  A cell or offset out of range
// sets ERR_BAD_CELL.  With write == false the kernel only checks (the caller
// reads the flag before anything changes).
__global__ void k_pack_movers(Geom g, int64_t n, const int32_t* __restrict__ cell,
                              const float* __restrict__ off3, const float* __restrict__ vel3,
                              const float* __restrict__ mass, const int64_t* __restrict__ id,
                              PartArrays mov, unsigned long long* mov_count, uint32_t* flags,
                              bool write)
{
  if (write && blockIdx.x == 0 && threadIdx.x == 0) *mov_count = (unsigned long long)n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cell[i];
    const float ox = off3[3 * i], oy = off3[3 * i + 1], oz = off3[3 * i + 2];
    const bool ok = c >= 0 && (int64_t)c < g.nsites && ox >= 0.0f && ox < 1.0f && oy >= 0.0f &&
                    oy < 1.0f && oz >= 0.0f && oz < 1.0f;
    if (!ok) {
      set_flag(flags, ERR_BAD_CELL);
      continue;
    }
    if (!write) continue;
    const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
    mov.key[i] = pack_key(g, x, y, z);
    mov.ox[i] = ox, mov.oy[i] = oy, mov.oz[i] = oz;
    mov.vx[i] = vel3[3 * i], mov.vy[i] = vel3[3 * i + 1], mov.vz[i] = vel3[3 * i + 2];
    if (mov.mass) mov.mass[i] = mass[i];
    if (mov.id) mov.id[i] = id[i];
  }
}

inline unsigned grid_of(int64_t n)
{
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

}  // namespace

cudaError_t launch_count_outside(lf2_ctx* c, int zlo, int zhi, unsigned long long* n)
{
  c->launches += 1;
  k_count_outside<<<(unsigned)c->g.nbricks, EX_THREADS, 0, c->stream>>>(view(c), zlo, zhi, n);
  return cudaGetLastError();
}

cudaError_t launch_extract_outside(lf2_ctx* c, int zlo, int zhi, int32_t* cell, float* off3,
                                   float* vel3, float* mass, int64_t* id,
                                   unsigned long long* out_count)
{
  c->launches += 1;
  k_extract_outside<<<(unsigned)c->g.nbricks, EX_THREADS, 0, c->stream>>>(
      view(c), zlo, zhi, cell, off3, vel3, mass, id, out_count);
  return cudaGetLastError();
}

cudaError_t launch_pack_movers(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                               const float* vel3, const float* mass, const int64_t* id, bool write)
{
  c->launches += 1;
  k_pack_movers<<<grid_of(n), 256, 0, c->stream>>>(c->g, n, cell, off3, vel3, mass, id, c->mov,
                                                    c->mov_count, c->flags, write);
  return cudaGetLastError();
}

}  // namespace lf2
