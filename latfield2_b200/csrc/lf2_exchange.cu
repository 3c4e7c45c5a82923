// lf2_exchange.cu -- particle exchange kernels of the slab decomposition.
//
// A rank of a z-slab decomposition keeps one ghost cell plane below and one
// above its own planes.  After a drift the particles that entered a ghost
// plane leave the store (k_count_outside, k_extract_outside) and are sent to
// the neighbour that owns them, as separate arrays or as packed migration
// records; particles received from the neighbours enter the store through
// the mover path (k_pack_movers or k_pack_records, then k_insert).  This
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
__host__ __device__ inline bool brick_inside(const Geom& g, int bz, int zlo, int zhi)
{
  const int z0 = bz * BRICK, z1 = z0 + brick_extent(g.n[2], bz) - 1;
  return z0 >= zlo && z1 <= zhi;
}

// The bricks a z range touches outside [zlo, zhi]: a prefix [0, lo_end) and a
// suffix [hi_begin, nbricks) of the brick order (bricks are numbered x
// fastest, z slowest, so a brick layer is a contiguous range).
struct OutsideBricks {
  int64_t lo_end, hi_begin, nbricks;

  __host__ __device__ int64_t size() const { return lo_end + (nbricks - hi_begin); }
  __device__ int64_t brick(int64_t i) const { return i < lo_end ? i : hi_begin + (i - lo_end); }
};

// Bits of slot j4*4 + t (t = 0..3) set when that slot lies in [from, to) and
// its particle's cell z is below zlo (lo), above zhi (hi).  Brick segments
// start on a multiple of 4 slots and hold a multiple of 4, so the 16-byte key
// vector never leaves the segment.
__device__ __forceinline__ void leave_masks(const StoreView& v, int64_t base, int j4, int from,
                                            int to, int zlo, int zhi, unsigned& lo, unsigned& hi,
                                            unsigned& far)
{
  const uint4 k4 = *reinterpret_cast<const uint4*>(v.a.key + base + 4 * (int64_t)j4);
  const uint32_t k[4] = {k4.x, k4.y, k4.z, k4.w};
  lo = hi = far = 0;
#pragma unroll
  for (int t = 0; t < 4; t++) {
    const int i = 4 * j4 + t;
    if (i < from || i >= to) continue;
    const int z = key_z(v.g, k[t]);
    lo |= (z < zlo ? 1u : 0u) << t;
    hi |= (z > zhi ? 1u : 0u) << t;
    far |= ((z < zlo - 1 || z > zhi + 1) ? 1u : 0u) << t;
  }
}

// n[0] += particles with z < zlo, n[1] += z > zhi, n[2] += more than one
// plane outside [zlo, zhi]; with maxv2 given, n[3] = max over bricks of
// maxv2 as float bits (non-negative floats order as their bits), each CTA
// reducing a share of the bricks.
__global__ void __launch_bounds__(EX_THREADS)
    k_count_outside(StoreView v, OutsideBricks ob, int zlo, int zhi, const float* maxv2,
                    unsigned long long* n)
{
  if (maxv2) {
    const int64_t per = (v.g.nbricks + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = blockIdx.x * per, b1 = min(v.g.nbricks, b0 + per);
    float m = 0.0f;
    for (int64_t b = b0 + threadIdx.x; b < b1; b += blockDim.x) m = fmaxf(m, maxv2[b]);
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f)
      atomicMax(&n[3], (unsigned long long)__float_as_uint(m));
  }
  if ((int64_t)blockIdx.x >= ob.size()) return;
  const int64_t b = ob.brick(blockIdx.x);
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  int lo = 0, hi = 0, far = 0;
  for (int j = threadIdx.x; 4 * j < cnt; j += blockDim.x) {
    unsigned ml, mh, mf;
    leave_masks(v, base, j, 0, cnt, zlo, zhi, ml, mh, mf);
    lo += __popc(ml);
    hi += __popc(mh);
    far += __popc(mf);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo += __shfl_xor_sync(0xffffffffu, lo, o);
    hi += __shfl_xor_sync(0xffffffffu, hi, o);
    far += __shfl_xor_sync(0xffffffffu, far, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (lo) atomicAdd(&n[0], (unsigned long long)lo);
    if (hi) atomicAdd(&n[1], (unsigned long long)hi);
    if (far) atomicAdd(&n[2], (unsigned long long)far);
  }
}

// Outputs of k_extract_outside.  SoaOut: one set of arrays (cell index,
// offsets, velocities, mass, id) for all particles that leave, slots from
// ctr[0].  RecordOut: migration records of `words` 32-bit words (cell index,
// offsets and velocities as float bits, [mass], [id low, id high]), those
// below zlo to `below` and those above zhi to `above`, slots from ctr[0] and
// ctr[1]; the cell index is the particle's cell in the neighbouring slab's
// lattice (z moved by +nz below, -nz above, nz = zhi - zlo + 1).  A slot
// beyond the given count raises ERR_CAPACITY and the particle is lost.
struct SoaOut {
  int32_t* cell;
  float* off3;
  float* vel3;
  float* mass;
  int64_t* id;

  __device__ void put(const Geom& g, int zlo, int zhi, uint32_t k, const float (&o)[3],
                      const float (&vel)[3], float m, int64_t pid, unsigned long long* ctr,
                      uint32_t*) const
  {
    int x, y, z;
    unpack_key(g, k, x, y, z);
    const int64_t q = (int64_t)atomicAdd(ctr, 1ull);
    cell[q] = (int32_t)site_index(g, x, y, z);
    off3[3 * q] = o[0], off3[3 * q + 1] = o[1], off3[3 * q + 2] = o[2];
    vel3[3 * q] = vel[0], vel3[3 * q + 1] = vel[1], vel3[3 * q + 2] = vel[2];
    if (mass) mass[q] = m;
    if (id) id[q] = pid;
  }
};

struct RecordOut {
  uint32_t* below;
  uint32_t* above;
  int64_t n_below, n_above;
  int words;
  bool has_mass, has_id;

  __device__ void put(const Geom& g, int zlo, int zhi, uint32_t k, const float (&o)[3],
                      const float (&vel)[3], float m, int64_t pid, unsigned long long* ctr,
                      uint32_t* flags) const
  {
    int x, y, z;
    unpack_key(g, k, x, y, z);
    const int side = z < zlo ? 0 : 1;
    const int64_t q = (int64_t)atomicAdd(&ctr[side], 1ull);
    if (q >= (side ? n_above : n_below)) {
      set_flag(flags, ERR_CAPACITY);
      return;
    }
    const int nz = zhi - zlo + 1;
    const int64_t zn = side ? (int64_t)z - nz : (int64_t)z + nz;
    uint32_t* r = (side ? above : below) + q * words;
    r[0] = (uint32_t)(int32_t)((int64_t)x + (int64_t)g.n[0] * ((int64_t)y + (int64_t)g.n[1] * zn));
    r[1] = __float_as_uint(o[0]), r[2] = __float_as_uint(o[1]), r[3] = __float_as_uint(o[2]);
    r[4] = __float_as_uint(vel[0]), r[5] = __float_as_uint(vel[1]), r[6] = __float_as_uint(vel[2]);
    int w = 7;
    if (has_mass) r[w++] = __float_as_uint(m);
    if (has_id) {
      r[w] = (uint32_t)((uint64_t)pid & 0xffffffffu);
      r[w + 1] = (uint32_t)((uint64_t)pid >> 32);
    }
  }
};

// One CTA per brick: particles with z outside [zlo, zhi] go to the output
// (slots from a global counter, any order) with their cell index; the others
// are compacted to the front of the brick's segment, in order.  A chunk is
// read completely before any of it is written, and the write cursor never
// passes the chunk's start, so the compaction is safe in place.
// One particle's arrays at slot p.
struct Part {
  uint32_t key;
  float o[3], vel[3], m;
  int64_t id;
};

__device__ __forceinline__ Part load_part(const StoreView& v, int64_t p)
{
  Part r;
  r.key = v.a.key[p];
  r.o[0] = v.a.ox[p], r.o[1] = v.a.oy[p], r.o[2] = v.a.oz[p];
  r.vel[0] = v.a.vx[p], r.vel[1] = v.a.vy[p], r.vel[2] = v.a.vz[p];
  r.m = v.a.mass ? v.a.mass[p] : 0.0f;
  r.id = v.a.id ? v.a.id[p] : 0;
  return r;
}

__device__ __forceinline__ void store_part(const StoreView& v, int64_t q, const Part& r)
{
  v.a.key[q] = r.key;
  v.a.ox[q] = r.o[0], v.a.oy[q] = r.o[1], v.a.oz[q] = r.o[2];
  v.a.vx[q] = r.vel[0], v.a.vy[q] = r.vel[1], v.a.vz[q] = r.vel[2];
  if (v.a.mass) v.a.mass[q] = r.m;
  if (v.a.id) v.a.id[q] = r.id;
}

// Holes a CTA pairs in shared memory; a brick with more leavers is compacted
// in order instead.
constexpr int EX_HOLES = 2048;

// One CTA per brick outside [zlo, zhi]: the particles with z outside go to
// the output; the brick keeps the others in its first cnt - k slots.  The
// leavers among those slots are holes, filled by the stayers among the last
// k slots, so only the leavers and the last k slots are read in full (the
// keys of the brick are read twice, 16 bytes at a time).  A brick with more
// than EX_HOLES leavers is compacted in order (each chunk read completely
// before any of it is written, the write cursor never passing the chunk's
// start).
template <class Out>
__global__ void __launch_bounds__(EX_THREADS)
    k_extract_outside(StoreView v, OutsideBricks ob, int zlo, int zhi, Out out_to,
                      unsigned long long* ctr, uint32_t* flags)
{
  __shared__ int warp_tot[32];
  __shared__ int holes[EX_HOLES];
  const Geom& g = v.g;
  const int64_t b = ob.brick(blockIdx.x);
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  int k_own = 0;
  for (int j = threadIdx.x; 4 * j < cnt; j += blockDim.x) {
    unsigned ml, mh, mf;
    leave_masks(v, base, j, 0, cnt, zlo, zhi, ml, mh, mf);
    k_own += __popc(ml | mh);
  }
  int k;
  block_exclusive_scan(k_own, warp_tot, &k);
  if (k == 0) return;
  if (k <= EX_HOLES) {
    const int keep = cnt - k;
    int nh = 0;
    for (int c0 = 0; 4 * c0 < keep; c0 += blockDim.x) {  // head: leavers leave holes
      const int j = c0 + threadIdx.x;
      unsigned ml = 0, mh = 0, mf = 0;
      if (4 * j < keep) leave_masks(v, base, j, 0, keep, zlo, zhi, ml, mh, mf);
      unsigned m = ml | mh;
      int tot;
      int pos = nh + block_exclusive_scan(__popc(m), warp_tot, &tot);
      while (m) {
        const int i = 4 * j + __ffs(m) - 1;
        m &= m - 1;
        holes[pos++] = i;
        const Part r = load_part(v, base + i);
        out_to.put(g, zlo, zhi, r.key, r.o, r.vel, r.m, r.id, ctr, flags);
      }
      nh += tot;
    }
    __syncthreads();
    int ns = 0;
    for (int c0 = keep / 4; 4 * c0 < cnt; c0 += blockDim.x) {  // tail: stayers fill the holes
      const int j = c0 + threadIdx.x;
      unsigned ml = 0, mh = 0, mf = 0;
      if (4 * j < cnt) leave_masks(v, base, j, keep, cnt, zlo, zhi, ml, mh, mf);
      unsigned in = 0;  // slots of [keep, cnt) in this group
#pragma unroll
      for (int t = 0; t < 4; t++) in |= (4 * j + t >= keep && 4 * j + t < cnt ? 1u : 0u) << t;
      const unsigned out = ml | mh;
      unsigned stay = in & ~out;
      int tot;
      int pos = ns + block_exclusive_scan(__popc(stay), warp_tot, &tot);
      unsigned m = in;
      while (m) {
        const int t = __ffs(m) - 1;
        m &= m - 1;
        const Part r = load_part(v, base + 4 * j + t);
        if (out >> t & 1u) out_to.put(g, zlo, zhi, r.key, r.o, r.vel, r.m, r.id, ctr, flags);
        else store_part(v, base + holes[pos++], r);
      }
      ns += tot;
    }
    if (threadIdx.x == 0) v.count[b] = keep;
    return;
  }
  int cursor = 0;
  for (int c0 = 0; c0 < cnt; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    const bool act = i < cnt;
    Part r{};
    if (act) r = load_part(v, base + i);
    const int z = key_z(g, r.key);
    const bool out = act && (z < zlo || z > zhi);
    const bool keep = act && !out;
    int total;
    const int pos = block_exclusive_scan(keep ? 1 : 0, warp_tot, &total);  // syncs the block
    if (keep) store_part(v, base + cursor + pos, r);
    else if (out) out_to.put(g, zlo, zhi, r.key, r.o, r.vel, r.m, r.id, ctr, flags);
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

// Migration records of two sources (na from a, then nb from b) into the
// mover buffer, ready for k_insert.  The valid ones take consecutive mover
// slots (one atomic on mov_count per warp; the caller zeroes it); a record
// whose cell index or offsets are out of range raises ERR_BAD_CELL and is
// dropped.
__global__ void k_pack_records(Geom g, int64_t na, const uint32_t* __restrict__ a, int64_t nb,
                               const uint32_t* __restrict__ b, int words, bool has_mass,
                               bool has_id, PartArrays mov, unsigned long long* mov_count,
                               uint32_t* flags)
{
  const int64_t n = na + nb;
  const int lane = threadIdx.x & 31;
  // every lane of a warp takes the same trips (blockDim.x is a multiple of 32)
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    const uint32_t* r = nullptr;
    bool ok = false;
    int32_t c = 0;
    float o[3] = {0, 0, 0};
    if (i < n) {
      r = i < na ? a + i * words : b + (i - na) * words;
      c = (int32_t)r[0];
      o[0] = __uint_as_float(r[1]), o[1] = __uint_as_float(r[2]), o[2] = __uint_as_float(r[3]);
      ok = c >= 0 && (int64_t)c < g.nsites && o[0] >= 0.0f && o[0] < 1.0f && o[1] >= 0.0f &&
           o[1] < 1.0f && o[2] >= 0.0f && o[2] < 1.0f;
      if (!ok) set_flag(flags, ERR_BAD_CELL);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (!bal) continue;
    const int leader = __ffs(bal) - 1;
    unsigned long long first = 0;
    if (lane == leader) first = atomicAdd(mov_count, (unsigned long long)__popc(bal));
    first = __shfl_sync(0xffffffffu, first, leader);
    if (!ok) continue;
    const int64_t q = (int64_t)first + __popc(bal & ((1u << lane) - 1u));
    const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
    const float vx = __uint_as_float(r[4]), vy = __uint_as_float(r[5]), vz = __uint_as_float(r[6]);
    int w = 7;
    const float m = has_mass ? __uint_as_float(r[w++]) : 0.0f;
    const int64_t pid = has_id ? (int64_t)((uint64_t)r[w] | ((uint64_t)r[w + 1] << 32)) : 0;
    mov.key[q] = pack_key(g, x, y, z);
    mov.ox[q] = o[0], mov.oy[q] = o[1], mov.oz[q] = o[2];
    mov.vx[q] = vx, mov.vy[q] = vy, mov.vz[q] = vz;
    if (mov.mass) mov.mass[q] = m;
    if (mov.id) mov.id[q] = pid;
  }
}

// Migration records of two sources into separate arrays (cell index,
// offsets, velocities, mass, id), unchecked: the input of lf2_particles_add.
__global__ void k_unpack_records(int64_t na, const uint32_t* __restrict__ a, int64_t nb,
                                 const uint32_t* __restrict__ b, int words, bool has_mass,
                                 bool has_id, int32_t* cell, float* off3, float* vel3, float* mass,
                                 int64_t* id)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < na + nb;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t* r = i < na ? a + i * words : b + (i - na) * words;
    cell[i] = (int32_t)r[0];
    for (int k = 0; k < 3; k++) {
      off3[3 * i + k] = __uint_as_float(r[1 + k]);
      vel3[3 * i + k] = __uint_as_float(r[4 + k]);
    }
    int w = 7;
    if (has_mass) mass[i] = __uint_as_float(r[w++]);
    if (has_id) id[i] = (int64_t)((uint64_t)r[w] | ((uint64_t)r[w + 1] << 32));
  }
}

OutsideBricks outside_bricks(const lf2_ctx* c, int zlo, int zhi)
{
  const int64_t layer = (int64_t)c->g.nb[0] * c->g.nb[1];
  const int nbz = c->g.nb[2];
  int lo = 0, hi = nbz;
  while (lo < nbz && !brick_inside(c->g, lo, zlo, zhi)) lo++;
  while (hi > lo && !brick_inside(c->g, hi - 1, zlo, zhi)) hi--;
  return {lo * layer, hi * layer, c->g.nbricks};
}

inline unsigned grid_of(int64_t n)
{
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

}  // namespace

cudaError_t launch_count_outside(lf2_ctx* c, int zlo, int zhi, unsigned long long* n,
                                 bool max_v)
{
  cudaError_t e = cudaMemsetAsync(n, 0, (max_v ? 4 : 3) * sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) return e;
  const OutsideBricks ob = outside_bricks(c, zlo, zhi);
  // enough CTAs for the max |v| share as well
  const int64_t grid = max(ob.size(), max_v ? (int64_t)c->num_sms * 2 : (int64_t)1);
  c->launches += 1;
  k_count_outside<<<(unsigned)grid, EX_THREADS, 0, c->stream>>>(
      view(c), ob, zlo, zhi, max_v ? c->brick_maxv2 : nullptr, n);
  return cudaGetLastError();
}

cudaError_t launch_extract_outside(lf2_ctx* c, int zlo, int zhi, int32_t* cell, float* off3,
                                   float* vel3, float* mass, int64_t* id,
                                   unsigned long long* out_count)
{
  const OutsideBricks ob = outside_bricks(c, zlo, zhi);
  if (ob.size() == 0) return cudaSuccess;
  c->launches += 1;
  k_extract_outside<<<(unsigned)ob.size(), EX_THREADS, 0, c->stream>>>(
      view(c), ob, zlo, zhi, SoaOut{cell, off3, vel3, mass, id}, out_count, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_extract_records(lf2_ctx* c, int zlo, int zhi, int64_t n_below, uint32_t* below,
                                   int64_t n_above, uint32_t* above, unsigned long long* ctr)
{
  cudaError_t e = cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) return e;
  const OutsideBricks ob = outside_bricks(c, zlo, zhi);
  if (ob.size() == 0) return cudaSuccess;
  c->launches += 1;
  const RecordOut out{below, above, n_below, n_above, record_words(c), c->has_mass, c->has_id};
  k_extract_outside<<<(unsigned)ob.size(), EX_THREADS, 0, c->stream>>>(view(c), ob, zlo, zhi, out,
                                                                       ctr, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_pack_records(lf2_ctx* c, int64_t na, const uint32_t* a, int64_t nb,
                                const uint32_t* b)
{
  cudaError_t e = cudaMemsetAsync(c->mov_count, 0, sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_pack_records<<<grid_of(na + nb), 256, 0, c->stream>>>(c->g, na, a, nb, b, record_words(c),
                                                          c->has_mass, c->has_id, c->mov,
                                                          c->mov_count, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_unpack_records(lf2_ctx* c, int64_t na, const uint32_t* a, int64_t nb,
                                  const uint32_t* b, int32_t* cell, float* off3, float* vel3,
                                  float* mass, int64_t* id)
{
  c->launches += 1;
  k_unpack_records<<<grid_of(na + nb), 256, 0, c->stream>>>(na, a, nb, b, record_words(c),
                                                            c->has_mass, c->has_id, cell, off3,
                                                            vel3, mass, id);
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
