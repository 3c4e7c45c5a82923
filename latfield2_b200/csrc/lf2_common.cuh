// lf2_common.cuh -- shared device-side definitions of the B200 particle-mesh
// library: lattice geometry, packed cell keys, brick (cell tile) indexing,
// error flags and small warp/block helpers.
//
// Particle representation (replaces the per-cell forward_list of part structs,
// LATfield2_Particles.hpp:97-103, :333): a structure of arrays
//   key  : uint32  packed cell coordinates x | y << bx | z << (bx + by)
//   off  : 3 x f32 in-cell offset in cell units, each in [0, 1)
//   vel  : 3 x f32 velocity in the reference's units (box length per time)
//   mass : f32 per particle (only for "individual mass" particle types)
//   id   : int64 (optional)
// binned by brick: a brick is a BRICK^3 tile of cells; the particles of brick b
// occupy slots [seg_start[b], seg_start[b] + count[b]) of the arrays, with
// cap[b] - count[b] free slots after them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#ifndef LF2_BRICK
#define LF2_BRICK 16
#endif

namespace lf2 {

constexpr int BRICK = LF2_BRICK;
constexpr int TILE = BRICK + 1;                 // vertices per dim of a brick tile
constexpr int TILE3 = TILE * TILE * TILE;       // vertices of a brick tile
// Tile vertices with a coordinate on 0 or on the brick extent: the values a
// brick shares with its neighbours (see shell_index).
constexpr int SHELL = TILE3 - (BRICK - 1) * (BRICK - 1) * (BRICK - 1);

// Error bits reported through the context's flag word.
enum : uint32_t {
  ERR_NONFINITE = 1u << 0,      // NaN/Inf in a particle offset or velocity
  ERR_BAD_CELL = 1u << 1,       // cell index or offset outside its range on load
  ERR_MASS_RANGE = 1u << 2,     // fixed-point relative mass outside [0, 64)
  ERR_REPACK = 1u << 3,         // a brick ran out of slots; store was repacked
  ERR_CAPACITY = 1u << 4,       // repack did not fit the allocation (lost state)
  ERR_FIXED_OVERFLOW = 1u << 5, // fixed-point vertex sum reached 2^63
  ERR_TIMEOUT = 1u << 6,        // a bounded wait inside a kernel gave up
};

struct Geom {
  int n[3];         // lattice sites per dim
  int nb[3];        // bricks per dim
  int shift[3];     // bit offset of each coordinate in the packed key
  uint32_t mask[3]; // bit mask of each coordinate (after shift)
  int64_t nsites;
  int64_t nbricks;
};

__host__ __device__ inline uint32_t pack_key(const Geom& g, int x, int y, int z)
{
  return (uint32_t)x | ((uint32_t)y << g.shift[1]) | ((uint32_t)z << g.shift[2]);
}

__host__ __device__ inline void unpack_key(const Geom& g, uint32_t k, int& x, int& y, int& z)
{
  x = (int)(k & g.mask[0]);
  y = (int)((k >> g.shift[1]) & g.mask[1]);
  z = (int)((k >> g.shift[2]) & g.mask[2]);
}

__host__ __device__ inline int64_t site_index(const Geom& g, int x, int y, int z)
{
  return (int64_t)x + (int64_t)g.n[0] * ((int64_t)y + (int64_t)g.n[1] * z);
}

__host__ __device__ inline int64_t brick_of(const Geom& g, int x, int y, int z)
{
  return (int64_t)(x / BRICK) +
         (int64_t)g.nb[0] * ((int64_t)(y / BRICK) + (int64_t)g.nb[1] * (z / BRICK));
}

// Brick indices fit in 32 bits (a lattice holds at most 2^31 bricks), so
// the coordinates come from 32-bit unsigned divisions.
__host__ __device__ inline void brick_coords(const Geom& g, int64_t b, int& bx, int& by, int& bz)
{
  const uint32_t u = (uint32_t)b, n0 = (uint32_t)g.nb[0], n1 = (uint32_t)g.nb[1];
  const uint32_t r = u / n0;
  bx = (int)(u - r * n0);
  bz = (int)(r / n1);
  by = (int)(r - (uint32_t)bz * n1);
}

// Cells (and owned vertices) of a brick along one dim: BRICK except for the
// last brick of a lattice whose size is not a multiple of BRICK.
__host__ __device__ inline int brick_extent(int n, int bcoord)
{
  const int e = n - bcoord * BRICK;
  return e < BRICK ? e : BRICK;
}

__host__ __device__ inline int wrap_add(int x, int d, int n)
{
  int v = x + d;
  if (v >= 0 && v < n) return v;
  v %= n;
  return v < 0 ? v + n : v;
}

// Index of tile vertex (i, j, k) in the brick's shell store.  A tile vertex is
// in the shell when one of its coordinates is 0 or equals the brick extent e
// along that dim (callers map a coordinate equal to e to BRICK first).  The
// shell is stored as three slabs: x faces (2 * TILE * TILE), y faces without
// the x edges (2 * (BRICK-1) * TILE) and z faces without x/y edges
// (2 * (BRICK-1)^2), 1538 values for BRICK = 16.
__host__ __device__ inline int shell_index(int i, int j, int k)
{
  if (i == 0 || i == BRICK) return (i == BRICK) * TILE * TILE + k * TILE + j;
  if (j == 0 || j == BRICK)
    return 2 * TILE * TILE + (j == BRICK) * (BRICK - 1) * TILE + k * (BRICK - 1) + (i - 1);
  return 2 * TILE * TILE + 2 * (BRICK - 1) * TILE + (k == BRICK) * (BRICK - 1) * (BRICK - 1) +
         (j - 1) * (BRICK - 1) + (i - 1);
}

static_assert(2 * TILE * TILE + 2 * (BRICK - 1) * TILE + 2 * (BRICK - 1) * (BRICK - 1) == SHELL,
              "shell slab sizes");

// Particles held by a brick.  count[b] can exceed cap[b] between k_insert
// and the repack; the slots beyond cap[b] belong to the next brick.
#define LF2_BRICK_COUNT(v, b) min((v).count[(b)], (v).cap[(b)])

__device__ inline void set_flag(uint32_t* flags, uint32_t bit)
{
  atomicOr(flags, bit);
}

// Fixed-point CIC weight of one corner: 1-D weights rounded to 2^-31,
// exact 96-bit product, rounded to 2^-32 of a unit mass:
//   q = (qx*qy*qz + 2^60) >> 61.
// With qx*qy = ph*2^32 + pl:  qx*qy*qz = ph*qz*2^32 + pl*qz, and because the
// rounding term 2^60 has no bits below 2^32,
//   q = (ph*qz + umulhi(pl, qz) + 2^28) >> 29
// exactly (the dropped low 32 bits of pl*qz cannot carry across 2^61).
// Same value as the oracle's 128-bit lf2o_fixed_weight.
__device__ __forceinline__ uint64_t fixed_corner(uint32_t qx, uint32_t qy, uint32_t qz)
{
  const uint64_t p = (uint64_t)qx * (uint64_t)qy;  // <= 2^62
  const uint32_t ph = (uint32_t)(p >> 32), pl = (uint32_t)p;
  const uint64_t hi = (uint64_t)ph * (uint64_t)qz + (uint64_t)__umulhi(pl, qz) + (1ull << 28);
  return hi >> 29;
}

// Block-wide exclusive scan of one int per thread (blockDim.x <= 1024,
// multiple of 32).  `warp_tot` is shared scratch of 32 ints.  Returns the
// exclusive prefix; *total receives the block total.
__device__ inline int block_exclusive_scan(int v, int* warp_tot, int* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  const int base = warp ? warp_tot[warp - 1] : 0;
  *total = warp_tot[nw - 1];
  const int r = base + x - v;
  __syncthreads();
  return r;
}

}  // namespace lf2
