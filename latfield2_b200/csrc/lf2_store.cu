// lf2_store.cu -- device particle store: bulk load (counting sort into brick
// segments), download, per-cell counts and the repack that runs when a brick
// runs out of free slots.
//
// Replaces the per-cell std::forward_list storage of the reference
// (LATfield2_Particles.hpp:97-103, :333, :370-373) and addParticle_global
// (:500-540).  Loading is a counting sort over bricks: histogram, capacity
// (count + slack) and exclusive scan, then a scatter into the segments.
#include <cuda_runtime.h>

#include "lf2_internal.h"

namespace lf2 {

namespace {

constexpr int SLACK_MIN = 32;
__host__ __device__ inline int32_t slack_of(int32_t count)
{
  const int32_t s = count >> 3;
  return s > SLACK_MIN ? s : SLACK_MIN;
}

// Slots of a brick segment: the particles plus slack, rounded up to a
// multiple of 4 so that every segment starts on a 16-byte boundary.
__host__ __device__ inline int32_t cap_of(int32_t count)
{
  return (count + slack_of(count) + 3) & ~3;
}

__device__ inline bool decode_cell(const Geom& g, int32_t c, int& x, int& y, int& z)
{
  if (c < 0 || (int64_t)c >= g.nsites) return false;
  x = c % g.n[0];
  y = (c / g.n[0]) % g.n[1];
  z = c / (g.n[0] * g.n[1]);
  return true;
}

__device__ inline bool valid_off(float o) { return o >= 0.0f && o < 1.0f; }

__global__ void k_load_count(Geom g, int64_t n, const int32_t* __restrict__ cell,
                             const float* __restrict__ off3, int32_t* count, uint32_t* flags)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    const bool ok = decode_cell(g, cell[i], x, y, z) && valid_off(off3[3 * i]) &&
                    valid_off(off3[3 * i + 1]) && valid_off(off3[3 * i + 2]);
    if (!ok) {
      set_flag(flags, ERR_BAD_CELL);
      continue;
    }
    atomicAdd(&count[brick_of(g, x, y, z)], 1);
  }
}

// One CTA: cap[b] = count[b] + slack (when caps != nullptr), starts = exclusive
// scan of caps (or of counts), starts[nb] = total.
__global__ void __launch_bounds__(1024) k_caps_scan(int64_t nb, const int32_t* __restrict__ counts,
                                                    int32_t* caps, int64_t* starts)
{
  __shared__ int64_t sh[1024];
  const int t = threadIdx.x;
  const int64_t per = (nb + blockDim.x - 1) / blockDim.x;
  const int64_t lo = t * per, hi = min(nb, lo + per);
  int64_t s = 0;
  for (int64_t b = lo; b < hi; b++) {
    const int32_t v = caps ? cap_of(counts[b]) : counts[b];
    if (caps) caps[b] = v;
    s += v;
  }
  sh[t] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const int64_t add = t >= o ? sh[t - o] : 0;
    __syncthreads();
    sh[t] += add;
    __syncthreads();
  }
  int64_t run = sh[t] - s;
  for (int64_t b = lo; b < hi; b++) {
    starts[b] = run;
    run += caps ? caps[b] : counts[b];
  }
  if (t == blockDim.x - 1) starts[nb] = sh[t];
}

__global__ void k_load_scatter(Geom g, int64_t n, const int32_t* __restrict__ cell,
                               const float* __restrict__ off3, const float* __restrict__ vel3,
                               const float* __restrict__ mass, const int64_t* __restrict__ id,
                               const int64_t* __restrict__ seg_start, int32_t* fill, PartArrays a)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    const bool ok = decode_cell(g, cell[i], x, y, z) && valid_off(off3[3 * i]) &&
                    valid_off(off3[3 * i + 1]) && valid_off(off3[3 * i + 2]);
    if (!ok) continue;
    const int64_t b = brick_of(g, x, y, z);
    const int64_t p = seg_start[b] + atomicAdd(&fill[b], 1);
    a.key[p] = pack_key(g, x, y, z);
    a.ox[p] = off3[3 * i];
    a.oy[p] = off3[3 * i + 1];
    a.oz[p] = off3[3 * i + 2];
    a.vx[p] = vel3[3 * i];
    a.vy[p] = vel3[3 * i + 1];
    a.vz[p] = vel3[3 * i + 2];
    if (a.mass) a.mass[p] = mass[i];
    if (a.id) a.id[p] = id[i];
  }
}

// Position in box units -> (cell, offset): u = pos / res, cell = floor(u) mod n
// (getPartCoord, LATfield2_Particles.hpp:463-467), offset = u - floor(u) in FP32.
template <typename T>
__global__ void k_pos_to_state(Geom g, double inv_res, int64_t n, const T* __restrict__ pos3,
                               int32_t* cell, float* off3)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int c[3];
    for (int d = 0; d < 3; d++) {
      const double u = (double)pos3[3 * i + d] * inv_res;
      double fl = floor(u);
      float o = (float)(u - fl);
      if (o >= 1.0f) {
        o = 0.0f;
        fl += 1.0;
      }
      long long ci = (long long)fl % g.n[d];
      if (ci < 0) ci += g.n[d];
      c[d] = (int)ci;
      off3[3 * i + d] = isfinite(u) ? o : -1.0f;  // -1 is rejected by the load
    }
    cell[i] = (int32_t)site_index(g, c[0], c[1], c[2]);
  }
}

template <typename T>
__global__ void k_state_to_pos(Geom g, double res, int64_t n, const int32_t* __restrict__ cell,
                               const float* __restrict__ off3, T* pos3)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cell[i];
    const int x = c % g.n[0], y = (c / g.n[0]) % g.n[1], z = c / (g.n[0] * g.n[1]);
    pos3[3 * i + 0] = (T)(((double)x + (double)off3[3 * i + 0]) * res);
    pos3[3 * i + 1] = (T)(((double)y + (double)off3[3 * i + 1]) * res);
    pos3[3 * i + 2] = (T)(((double)z + (double)off3[3 * i + 2]) * res);
  }
}

// One CTA per brick: copy the brick's particles to a dense output.
__global__ void k_get(StoreView v, const int64_t* __restrict__ out_start, int32_t* cell,
                      float* off3, float* vel3, float* mass, int64_t* id)
{
  const int64_t b = blockIdx.x;
  const int64_t base = v.seg_start[b], o0 = out_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int64_t p = base + i, o = o0 + i;
    int x, y, z;
    unpack_key(v.g, v.a.key[p], x, y, z);
    if (cell) cell[o] = (int32_t)site_index(v.g, x, y, z);
    if (off3) {
      off3[3 * o] = v.a.ox[p];
      off3[3 * o + 1] = v.a.oy[p];
      off3[3 * o + 2] = v.a.oz[p];
    }
    if (vel3) {
      vel3[3 * o] = v.a.vx[p];
      vel3[3 * o + 1] = v.a.vy[p];
      vel3[3 * o + 2] = v.a.vz[p];
    }
    if (mass && v.a.mass) mass[o] = v.a.mass[p];
    if (id && v.a.id) id[o] = v.a.id[p];
  }
}

__global__ void k_cell_counts(StoreView v, int32_t* counts)
{
  const int64_t b = blockIdx.x;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    int x, y, z;
    unpack_key(v.g, v.a.key[base + i], x, y, z);
    atomicAdd(&counts[site_index(v.g, x, y, z)], 1);
  }
}

// ------------------------------------------------------------------ repack
// Runs only when k_insert found a brick without a free slot (*repack != 0);
// every kernel returns at once otherwise, so the sequence can stay in the
// step without a host round trip.

__global__ void __launch_bounds__(1024) k_repack_caps(int64_t nb, const int32_t* __restrict__ count,
                                                      int32_t* cap_alt, int64_t* start_alt,
                                                      int64_t capacity, int32_t* repack,
                                                      uint32_t* flags)
{
  if (*repack == 0) return;
  __shared__ int64_t sh[1024];
  const int t = threadIdx.x;
  const int64_t per = (nb + blockDim.x - 1) / blockDim.x;
  const int64_t lo = t * per, hi = min(nb, lo + per);
  int64_t s = 0;
  for (int64_t b = lo; b < hi; b++) {
    const int32_t c = cap_alt[b] = cap_of(count[b]);
    s += c;
  }
  sh[t] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const int64_t add = t >= o ? sh[t - o] : 0;
    __syncthreads();
    sh[t] += add;
    __syncthreads();
  }
  int64_t run = sh[t] - s;
  for (int64_t b = lo; b < hi; b++) {
    start_alt[b] = run;
    run += cap_alt[b];
  }
  if (t == blockDim.x - 1) {
    start_alt[nb] = sh[t];
    if (sh[t] > capacity) {
      set_flag(flags, ERR_CAPACITY);
      *repack = 0;  // cannot repack: leave the store as it is
    }
  }
}

// One particle's arrays, read before any is written (source and destination
// may be the same arrays, so interleaved loads and stores would wait for
// each other).
struct PartVal {
  uint32_t key;
  float ox, oy, oz, vx, vy, vz, m;
  int64_t id;
};

__device__ inline PartVal load_particle(const PartArrays& s, int64_t ps)
{
  PartVal p;
  p.key = s.key[ps];
  p.ox = s.ox[ps];
  p.oy = s.oy[ps];
  p.oz = s.oz[ps];
  p.vx = s.vx[ps];
  p.vy = s.vy[ps];
  p.vz = s.vz[ps];
  p.m = s.mass ? s.mass[ps] : 0.0f;
  p.id = s.id ? s.id[ps] : 0;
  return p;
}

__device__ inline void store_particle(const PartArrays& d, int64_t pd, const PartVal& p)
{
  d.key[pd] = p.key;
  d.ox[pd] = p.ox;
  d.oy[pd] = p.oy;
  d.oz[pd] = p.oz;
  d.vx[pd] = p.vx;
  d.vy[pd] = p.vy;
  d.vz[pd] = p.vz;
  if (d.mass) d.mass[pd] = p.m;
  if (d.id) d.id[pd] = p.id;
}

__device__ inline void copy_particle(const PartArrays& s, int64_t ps, const PartArrays& d, int64_t pd)
{
  store_particle(d, pd, load_particle(s, ps));
}

// Copies n consecutive particles, four per thread in flight.
__device__ inline void copy_run(const PartArrays& s, int64_t s0, const PartArrays& d, int64_t d0, int n)
{
  for (int i = threadIdx.x; i < n; i += 4 * blockDim.x) {
    PartVal v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = i + u * (int)blockDim.x;
      if (k < n) v[u] = load_particle(s, s0 + k);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = i + u * (int)blockDim.x;
      if (k < n) store_particle(d, d0 + k, v[u]);
    }
  }
}

// The per-brick repack kernels run on a small grid (grid-stride over bricks)
// so that returning early costs a few microseconds, not one CTA per brick.
__global__ void k_repack_copy_out(StoreView v, PartArrays alt, const int64_t* __restrict__ start_alt,
                                  int32_t* fill, const int32_t* repack)
{
  if (*repack == 0) return;
  for (int64_t b = blockIdx.x; b < v.g.nbricks; b += gridDim.x) {
    const int placed = min(v.count[b], v.cap[b]);
    const int64_t s0 = v.seg_start[b], d0 = start_alt[b];
    copy_run(v.a, s0, alt, d0, placed);
    if (threadIdx.x == 0) fill[b] = placed;
  }
}

__global__ void k_repack_movers(Geom g, PartArrays mov, const int32_t* __restrict__ placed,
                                const unsigned long long* __restrict__ mov_count, PartArrays alt,
                                const int64_t* __restrict__ start_alt, int32_t* fill,
                                const int32_t* repack)
{
  if (*repack == 0) return;
  const int64_t nm = (int64_t)*mov_count;
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nm;
       m += (int64_t)gridDim.x * blockDim.x) {
    if (placed[m]) continue;
    int x, y, z;
    unpack_key(g, mov.key[m], x, y, z);
    const int64_t b = brick_of(g, x, y, z);
    copy_particle(mov, m, alt, start_alt[b] + atomicAdd(&fill[b], 1));
  }
}

__global__ void k_repack_copy_back(StoreView v, PartArrays alt, const int64_t* __restrict__ start_alt,
                                   const int32_t* __restrict__ fill, const int32_t* repack)
{
  if (*repack == 0) return;
  for (int64_t b = blockIdx.x; b < v.g.nbricks; b += gridDim.x) {
    const int n = fill[b];
    const int64_t d0 = start_alt[b];
    copy_run(alt, d0, v.a, d0, n);
    if (threadIdx.x == 0) v.count[b] = n;
  }
}

__global__ void k_repack_finish(int64_t nb, const int64_t* __restrict__ start_alt,
                                const int32_t* __restrict__ cap_alt, int64_t* seg_start,
                                int32_t* cap, int32_t* repack, unsigned long long* heap_top)
{
  if (*repack == 0) return;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    seg_start[b] = start_alt[b];
    if (b < nb) cap[b] = cap_alt[b];
    else *heap_top = (unsigned long long)start_alt[nb];  // relocation region starts after the segments
  }
}

__global__ void k_repack_clear(int32_t* repack, uint32_t* flags, unsigned long long* diag,
                               const unsigned long long* movers)
{
  if (*repack) {
    set_flag(flags, ERR_REPACK);
    diag[0] += 1;
    *repack = 0;
  }
  diag[1] = *movers;
}

// ----------------------------------------------------------- relocation
// A brick that ran out of free slots in k_insert is moved on its own to a
// fresh, larger segment carved from the relocation region (bump allocation
// past the contiguous segments).  Its old slots are abandoned until the next
// full repack.  Only when the region is exhausted does the whole store get
// repacked (k_repack_*).

__global__ void __launch_bounds__(1024)
    k_reloc(StoreView v, int64_t* seg_start, int32_t* cap, const int32_t* __restrict__ list,
                        const int32_t* __restrict__ nlist, int32_t* state, int32_t* fill,
                        unsigned long long* heap_top, int64_t capacity, int32_t* repack,
                        unsigned long long* diag)
{
  __shared__ long long s_new;
  const int n = *nlist;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int64_t b = list[i];
    const int32_t need = v.count[b];  // stays + every arrival that tried
    const int32_t placed = min(need, cap[b]);
    const int32_t ncap = cap_of(need);
    if (threadIdx.x == 0) {
      const unsigned long long s0 = atomicAdd(heap_top, (unsigned long long)ncap);
      s_new = (s0 + (unsigned long long)ncap <= (unsigned long long)capacity) ? (long long)s0 : -1;
      if (s_new < 0) *repack = 1;  // region exhausted: repack everything
    }
    __syncthreads();
    const long long d0 = s_new;
    if (d0 >= 0) {
      const int64_t s0 = seg_start[b];
      copy_run(v.a, s0, v.a, d0, placed);
      __syncthreads();
      if (threadIdx.x == 0) {
        seg_start[b] = d0;
        cap[b] = ncap;
        fill[b] = placed;
        state[b] = 2;
        atomicAdd(&diag[2], 1ull);
      }
    }
    __syncthreads();
  }
}

__global__ void k_reloc_movers(Geom g, PartArrays mov, int32_t* placed,
                               const unsigned long long* __restrict__ mov_count, PartArrays dst,
                               const int64_t* __restrict__ seg_start, const int32_t* __restrict__ state,
                               int32_t* fill, const int32_t* __restrict__ nlist)
{
  if (*nlist == 0) return;
  const int64_t nm = (int64_t)*mov_count;
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nm;
       m += (int64_t)gridDim.x * blockDim.x) {
    if (placed[m]) continue;
    int x, y, z;
    unpack_key(g, mov.key[m], x, y, z);
    const int64_t b = brick_of(g, x, y, z);
    if (state[b] != 2) continue;  // not relocated: left to the full repack
    copy_particle(mov, m, dst, seg_start[b] + atomicAdd(&fill[b], 1));
    placed[m] = 1;
  }
}

__global__ void k_ovf_reset(int32_t* list, int32_t* nlist, int32_t* state)
{
  const int n = *nlist;
  for (int i = threadIdx.x; i < n; i += blockDim.x) state[list[i]] = 0;
  __syncthreads();
  if (threadIdx.x == 0) *nlist = 0;
}

inline int grid_for(int64_t n, int threads)
{
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g > 0 ? g : 1);
}

}  // namespace

cudaError_t launch_load_count(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3)
{
  c->launches += 1;
  k_load_count<<<grid_for(n, 256), 256, 0, c->stream>>>(c->g, n, cell, off3, c->count, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_caps_and_scan(lf2_ctx* c, const int32_t* counts, int32_t* caps, int64_t* starts,
                                 int64_t*)
{
  c->launches += 1;
  k_caps_scan<<<1, 1024, 0, c->stream>>>(c->g.nbricks, counts, caps, starts);
  return cudaGetLastError();
}

cudaError_t launch_scan_counts(lf2_ctx* c, int64_t* out_start)
{
  c->launches += 1;
  k_caps_scan<<<1, 1024, 0, c->stream>>>(c->g.nbricks, c->count, nullptr, out_start);
  return cudaGetLastError();
}

cudaError_t launch_load_scatter(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                                const float* vel3, const float* mass, const int64_t* id)
{
  c->launches += 1;
  k_load_scatter<<<grid_for(n, 256), 256, 0, c->stream>>>(c->g, n, cell, off3, vel3, mass, id,
                                                           c->seg_start, c->fill, c->cur);
  return cudaGetLastError();
}

cudaError_t launch_pos_to_state(lf2_ctx* c, int64_t n, const void* pos3, int real_bytes,
                                int32_t* cell, float* off3)
{
  c->launches += 1;
  const double inv_res = 1.0 / c->res;
  if (real_bytes == 8)
    k_pos_to_state<double><<<grid_for(n, 256), 256, 0, c->stream>>>(
        c->g, inv_res, n, (const double*)pos3, cell, off3);
  else
    k_pos_to_state<float><<<grid_for(n, 256), 256, 0, c->stream>>>(
        c->g, inv_res, n, (const float*)pos3, cell, off3);
  return cudaGetLastError();
}

cudaError_t launch_state_to_pos(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                                void* pos3, int real_bytes)
{
  c->launches += 1;
  if (real_bytes == 8)
    k_state_to_pos<double><<<grid_for(n, 256), 256, 0, c->stream>>>(c->g, c->res, n, cell, off3,
                                                                     (double*)pos3);
  else
    k_state_to_pos<float><<<grid_for(n, 256), 256, 0, c->stream>>>(c->g, c->res, n, cell, off3,
                                                                    (float*)pos3);
  return cudaGetLastError();
}

cudaError_t launch_get(lf2_ctx* c, int64_t* out_start, int32_t* cell, float* off3, float* vel3,
                       float* mass, int64_t* id)
{
  c->launches += 1;
  k_get<<<(unsigned)c->g.nbricks, 256, 0, c->stream>>>(view(c), out_start, cell, off3, vel3, mass,
                                                       id);
  return cudaGetLastError();
}

cudaError_t launch_cell_counts(lf2_ctx* c, int32_t* counts)
{
  c->launches += 1;
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int32_t) * c->g.nsites, c->stream);
  if (e != cudaSuccess) return e;
  k_cell_counts<<<(unsigned)c->g.nbricks, 256, 0, c->stream>>>(view(c), counts);
  return cudaGetLastError();
}

cudaError_t launch_heap_reset(lf2_ctx* c)
{
  return cudaMemcpyAsync(c->heap_top, c->seg_start + c->g.nbricks, sizeof(unsigned long long),
                         cudaMemcpyDeviceToDevice, c->stream);
}

cudaError_t launch_repack(lf2_ctx* c)
{
  c->launches += 9;
  const int64_t nb = c->g.nbricks;
  k_reloc<<<148, 1024, 0, c->stream>>>(view(c), c->seg_start, c->cap, c->ovf_list, c->ovf_count,
                                      c->ovf_state, c->fill, c->heap_top, c->capacity, c->repack,
                                      c->diag);
  k_reloc_movers<<<148 * 2, 256, 0, c->stream>>>(c->g, c->mov, c->mov_placed, c->mov_count, c->cur,
                                                 c->seg_start, c->ovf_state, c->fill, c->ovf_count);
  k_repack_caps<<<1, 1024, 0, c->stream>>>(nb, c->count, c->cap_alt, c->seg_start_alt, c->capacity,
                                           c->repack, c->flags);
  const unsigned small = (unsigned)(nb < 148 * 8 ? nb : 148 * 8);
  k_repack_copy_out<<<small, 256, 0, c->stream>>>(view(c), c->alt, c->seg_start_alt, c->fill,
                                                  c->repack);
  k_repack_movers<<<148 * 4, 256, 0, c->stream>>>(c->g, c->mov, c->mov_placed, c->mov_count, c->alt,
                                                  c->seg_start_alt, c->fill, c->repack);
  k_repack_copy_back<<<small, 256, 0, c->stream>>>(view(c), c->alt, c->seg_start_alt, c->fill,
                                                   c->repack);
  k_repack_finish<<<small, 256, 0, c->stream>>>(nb, c->seg_start_alt, c->cap_alt, c->seg_start,
                                                 c->cap, c->repack, c->heap_top);
  k_repack_clear<<<1, 1, 0, c->stream>>>(c->repack, c->flags, c->diag, c->mov_count);
  k_ovf_reset<<<1, 256, 0, c->stream>>>(c->ovf_list, c->ovf_count, c->ovf_state);
  return cudaGetLastError();
}

}  // namespace lf2
