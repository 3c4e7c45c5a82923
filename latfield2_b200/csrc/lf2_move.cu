// lf2_move.cu -- gather-kick, drift and rebin of the brick-binned particles.
//
// One CTA per brick.  The kick gathers the 3-component field at the 8 cell
// corners from a shared-memory copy of the brick's (BRICK+1)^3 vertex tile
// (the CIC gather the reference leaves to the updateVel callback,
// LATfield2_Particles.hpp:752-893).  The drift is move_particles_simple
// (move_function.hpp:15-32) in cell units: off += dtau/res * vel, then the
// integer part is carried into the cell coordinates with a periodic wrap
// (the wrap and rebin of moveParticles, LATfield2_Particles.hpp:2028-2056).
//
// Rebin: particles that stay in their brick are compacted in place at the
// front of the brick's segment; particles that leave are appended to a mover
// buffer and inserted into their new brick's free slots by k_insert.  A brick
// that runs out of free slots sets the repack flag (lf2_store.cu).
#include <cuda_runtime.h>

#include "lf2_internal.h"

namespace lf2 {

namespace {

// Launch shape and access pattern of k_move (chosen by measurement):
//   MOVE_THREADS  threads per CTA (one CTA per brick)
//   MOVE_ITEMS    particles per thread per chunk; with MOVE_BLOCKED a thread
//                 owns MOVE_ITEMS consecutive slots and reads them with one
//                 16-byte vector load per array (brick segments start on a
//                 multiple of 4 slots and hold a multiple of 4 slots, so the
//                 vector never leaves the segment)
//   MOVE_F4       the brick's vertex tile of F kept as float4 (x, y, z, 0):
//                 one 16-byte shared load per corner instead of three
#ifndef LF2_MOVE_THREADS
#define LF2_MOVE_THREADS 256
#endif
#ifndef LF2_MOVE_ITEMS
#define LF2_MOVE_ITEMS 4
#endif
#ifndef LF2_MOVE_BLOCKED
#define LF2_MOVE_BLOCKED 1
#endif
#ifndef LF2_MOVE_F4
#define LF2_MOVE_F4 0
#endif
constexpr int MOVE_THREADS = LF2_MOVE_THREADS;
constexpr int MOVE_ITEMS = LF2_MOVE_ITEMS;
constexpr bool MOVE_BLOCKED = LF2_MOVE_BLOCKED != 0;
constexpr bool MOVE_F4 = LF2_MOVE_F4 != 0;
static_assert(!MOVE_BLOCKED || MOVE_ITEMS == 4, "blocked access reads 4 slots per vector");

__device__ __forceinline__ float sel(int b, float up, float dn) { return b ? up : dn; }

template <typename T>
__device__ __forceinline__ void load4(const T* __restrict__ a, int64_t p, T (&r)[4])
{
  static_assert(sizeof(T) == 4, "32-bit lanes");
  const uint4 q = __ldcs(reinterpret_cast<const uint4*>(a + p));
  r[0] = __uint_as_float(q.x), r[1] = __uint_as_float(q.y);
  r[2] = __uint_as_float(q.z), r[3] = __uint_as_float(q.w);
}

__device__ __forceinline__ void load4u(const uint32_t* __restrict__ a, int64_t p, uint32_t (&r)[4])
{
  const uint4 q = __ldcs(reinterpret_cast<const uint4*>(a + p));
  r[0] = q.x, r[1] = q.y, r[2] = q.z, r[3] = q.w;
}

template <bool KICK, bool DRIFT>
__global__ void __launch_bounds__(MOVE_THREADS) k_move(StoreView v, const float* __restrict__ F,
                                                       MoveParams mp, PartArrays mov,
                                                       unsigned long long* mov_count,
                                                       float* brick_maxv2, uint32_t* flags)
{
  extern __shared__ __align__(16) float ftile[];  // KICK: [3][TILE3] or float4[TILE3]
  __shared__ int s_scan[32];
  __shared__ float s_max[MOVE_THREADS / 32];

  const Geom& g = v.g;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);

  int write = 0;
  float maxv2 = 0.0f;
  const int lane = threadIdx.x & 31;

  for (int c0 = 0; c0 < cnt; c0 += MOVE_ITEMS * MOVE_THREADS) {
    uint32_t key[MOVE_ITEMS];
    float ox[MOVE_ITEMS], oy[MOVE_ITEMS], oz[MOVE_ITEMS];
    float vx[MOVE_ITEMS], vy[MOVE_ITEMS], vz[MOVE_ITEMS], m[MOVE_ITEMS];
    int64_t id[MOVE_ITEMS];
    bool act[MOVE_ITEMS], stay[MOVE_ITEMS];
    // slot of item j: blocked = c0 + 4*tid + j, strided = c0 + j*THREADS + tid
    auto slot = [&](int j) {
      return MOVE_BLOCKED ? c0 + MOVE_ITEMS * (int)threadIdx.x + j
                          : c0 + j * MOVE_THREADS + (int)threadIdx.x;
    };
    if constexpr (MOVE_BLOCKED) {
      const int i0 = slot(0);
      if (i0 < cnt) {
        const int64_t p = base + i0;
        {
          load4u(v.a.key, p, key);
          load4(v.a.ox, p, ox);
          load4(v.a.oy, p, oy);
          load4(v.a.oz, p, oz);
          load4(v.a.vx, p, vx);
          load4(v.a.vy, p, vy);
          load4(v.a.vz, p, vz);
        }
      }
#pragma unroll
      for (int j = 0; j < MOVE_ITEMS; j++) {
        act[j] = slot(j) < cnt;
        stay[j] = true;
        m[j] = 0.0f;
        id[j] = 0;
        if (act[j]) {
          if (DRIFT && v.a.mass) m[j] = v.a.mass[base + slot(j)];
          if (DRIFT && v.a.id) id[j] = v.a.id[base + slot(j)];
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < MOVE_ITEMS; j++) {
        act[j] = slot(j) < cnt;
        stay[j] = true;
        m[j] = 0.0f;
        id[j] = 0;
        if (act[j]) {
          const int64_t p = base + slot(j);
          key[j] = v.a.key[p];
          ox[j] = v.a.ox[p];
          oy[j] = v.a.oy[p];
          oz[j] = v.a.oz[p];
          vx[j] = v.a.vx[p];
          vy[j] = v.a.vy[p];
          vz[j] = v.a.vz[p];
          if (DRIFT && v.a.mass) m[j] = v.a.mass[p];
          if (DRIFT && v.a.id) id[j] = v.a.id[p];
        }
      }
    }
    if (KICK && c0 == 0) {
      // The brick's vertex tile of F, loaded while the first chunk's particle
      // loads are in flight; empty bricks never load it.
      const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
                ez = brick_extent(g.n[2], bz);
      for (int t = threadIdx.x; t < TILE3; t += blockDim.x) {
        const int i = t % TILE, jj = (t / TILE) % TILE, k = t / (TILE * TILE);
        if (i > ex || jj > ey || k > ez) continue;
        const int gx = x0 + i < g.n[0] ? x0 + i : 0;
        const int gy = y0 + jj < g.n[1] ? y0 + jj : 0;
        const int gz = z0 + k < g.n[2] ? z0 + k : 0;
        const int64_t s = site_index(g, gx, gy, gz);
        const float f0 = __ldg(F + s), f1 = __ldg(F + g.nsites + s), f2 = __ldg(F + 2 * g.nsites + s);
        if (MOVE_F4) {
          reinterpret_cast<float4*>(ftile)[t] = make_float4(f0, f1, f2, 0.0f);
        } else {
          ftile[t] = f0;
          ftile[TILE3 + t] = f1;
          ftile[2 * TILE3 + t] = f2;
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < MOVE_ITEMS; j++) {
      if (!act[j]) continue;
      int x, y, z;
      unpack_key(g, key[j], x, y, z);
      if (KICK) {
        const int t0 = (x - x0) + TILE * ((y - y0) + TILE * (z - z0));
        const float gx = __fsub_rn(1.0f, ox[j]), gy = __fsub_rn(1.0f, oy[j]),
                    gz = __fsub_rn(1.0f, oz[j]);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
          const float w = __fmul_rn(__fmul_rn(sel(cx, ox[j], gx), sel(cy, oy[j], gy)),
                                    sel(cz, oz[j], gz));
          const int t = t0 + cx + cy * TILE + cz * TILE * TILE;
          float f0, f1, f2;
          if (MOVE_F4) {
            const float4 q = reinterpret_cast<const float4*>(ftile)[t];
            f0 = q.x, f1 = q.y, f2 = q.z;
          } else {
            f0 = ftile[t], f1 = ftile[TILE3 + t], f2 = ftile[2 * TILE3 + t];
          }
          a0 = __fmaf_rn(w, f0, a0);
          a1 = __fmaf_rn(w, f1, a1);
          a2 = __fmaf_rn(w, f2, a2);
        }
        vx[j] = __fmaf_rn(mp.dtk, a0, vx[j]);
        vy[j] = __fmaf_rn(mp.dtk, a1, vy[j]);
        vz[j] = __fmaf_rn(mp.dtk, a2, vz[j]);
      }
      maxv2 = fmaxf(maxv2, __fadd_rn(__fadd_rn(__fmul_rn(vx[j], vx[j]), __fmul_rn(vy[j], vy[j])),
                                     __fmul_rn(vz[j], vz[j])));
      if (DRIFT) {
        float o[3] = {ox[j], oy[j], oz[j]};
        const float vv[3] = {vx[j], vy[j], vz[j]};
        int xyz[3] = {x, y, z};
        bool finite = true;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          float od = __fmaf_rn(mp.dtn, vv[d], o[d]);
          if (!isfinite(od)) {
            finite = false;
            break;
          }
          const float fl = floorf(od);
          od = __fsub_rn(od, fl);
          int carry = (int)fl;
          if (od >= 1.0f) {
            od = 0.0f;
            carry += 1;
          }
          o[d] = od;
          xyz[d] = wrap_add(xyz[d], carry, g.n[d]);
        }
        if (finite) {
          ox[j] = o[0];
          oy[j] = o[1];
          oz[j] = o[2];
          key[j] = pack_key(g, xyz[0], xyz[1], xyz[2]);
          stay[j] = brick_of(g, xyz[0], xyz[1], xyz[2]) == b;
        } else {
          set_flag(flags, ERR_NONFINITE);
        }
      }
    }

    if (!DRIFT) {
      if constexpr (MOVE_BLOCKED) {
        const int i0 = slot(0);
        if (i0 < cnt) {  // the whole vector stays inside the segment
          const int64_t p = base + i0;
          *reinterpret_cast<float4*>(v.a.vx + p) = make_float4(vx[0], vx[1], vx[2], vx[3]);
          *reinterpret_cast<float4*>(v.a.vy + p) = make_float4(vy[0], vy[1], vy[2], vy[3]);
          *reinterpret_cast<float4*>(v.a.vz + p) = make_float4(vz[0], vz[1], vz[2], vz[3]);
        }
      } else {
#pragma unroll
        for (int j = 0; j < MOVE_ITEMS; j++) {
          if (!act[j]) continue;
          const int64_t p = base + slot(j);
          v.a.vx[p] = vx[j];
          v.a.vy[p] = vy[j];
          v.a.vz[p] = vz[j];
        }
      }
      continue;
    }

    // All loads of this chunk are complete before any slot is overwritten:
    // stayers of this chunk land below the start of the next chunk.
    int mine = 0;
#pragma unroll
    for (int j = 0; j < MOVE_ITEMS; j++) mine += (act[j] && stay[j]) ? 1 : 0;
    int total;
    int q0 = block_exclusive_scan(mine, s_scan, &total);
#pragma unroll
    for (int j = 0; j < MOVE_ITEMS; j++) {
      if (act[j] && stay[j]) {
        const int64_t q = base + write + q0;
        q0++;
        v.a.key[q] = key[j];
        v.a.ox[q] = ox[j];
        v.a.oy[q] = oy[j];
        v.a.oz[q] = oz[j];
        v.a.vx[q] = vx[j];
        v.a.vy[q] = vy[j];
        v.a.vz[q] = vz[j];
        if (v.a.mass) v.a.mass[q] = m[j];
        if (v.a.id) v.a.id[q] = id[j];
      }
      const bool leave = act[j] && !stay[j];
      const unsigned bal = __ballot_sync(0xffffffffu, leave);
      if (bal) {
        const int leader = __ffs(bal) - 1;
        unsigned long long s0 = 0;
        if (lane == leader) s0 = atomicAdd(mov_count, (unsigned long long)__popc(bal));
        s0 = __shfl_sync(0xffffffffu, s0, leader);
        if (leave) {
          const int64_t q = (int64_t)s0 + __popc(bal & ((1u << lane) - 1u));
          mov.key[q] = key[j];
          mov.ox[q] = ox[j];
          mov.oy[q] = oy[j];
          mov.oz[q] = oz[j];
          mov.vx[q] = vx[j];
          mov.vy[q] = vy[j];
          mov.vz[q] = vz[j];
          if (mov.mass) mov.mass[q] = m[j];
          if (mov.id) mov.id[q] = id[j];
        }
      }
    }
    write += total;
  }
  if (DRIFT && threadIdx.x == 0) v.count[b] = write;

  // max |v|^2 of the brick
  for (int o = 16; o > 0; o >>= 1) maxv2 = fmaxf(maxv2, __shfl_xor_sync(0xffffffffu, maxv2, o));
  if (lane == 0) s_max[threadIdx.x >> 5] = maxv2;
  __syncthreads();
  if (threadIdx.x == 0) {
    float mm = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) mm = fmaxf(mm, s_max[w]);
    brick_maxv2[b] = mm;
  }
}

// Movers into the free slots of their new brick.
__global__ void k_insert(StoreView v, PartArrays mov, const unsigned long long* __restrict__ mov_count,
                         int32_t* placed, int32_t* ovf_list, int32_t* ovf_count, int32_t* ovf_state,
                         uint32_t* flags)
{
  // Whole warps step through the movers together, so that the lanes heading
  // for the same brick (consecutive movers mostly come from one source brick
  // and go to a few neighbours) take their slots with one atomic per brick.
  const int64_t nm = (int64_t)*mov_count;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp0 * 32; base < nm; base += nwarps * 32) {
    const int64_t m = base + lane;
    int64_t b = -1;
    uint32_t key = 0;
    if (m < nm) {
      int x, y, z;
      key = mov.key[m];
      unpack_key(v.g, key, x, y, z);
      if (x >= v.g.n[0] || y >= v.g.n[1] || z >= v.g.n[2]) {  // only after a failed move
        set_flag(flags, ERR_BAD_CELL);
        placed[m] = 1;
      } else {
        b = brick_of(v.g, x, y, z);
      }
    }
    const unsigned grp = __match_any_sync(0xffffffffu, b);
    int slot = 0;
    if (b >= 0) {
      const int leader = __ffs(grp) - 1;
      int first = 0;
      if (lane == leader) first = atomicAdd(&v.count[b], __popc(grp));
      slot = __shfl_sync(grp, first, leader) + __popc(grp & lt);
    }
    if (b < 0) continue;
    if (slot < v.cap[b]) {
      const int64_t q = v.seg_start[b] + slot;
      // every array read before any is written (the compiler cannot tell
      // that the mover buffer and the store do not overlap)
      const float ox = mov.ox[m], oy = mov.oy[m], oz = mov.oz[m];
      const float vx = mov.vx[m], vy = mov.vy[m], vz = mov.vz[m];
      const float ms = v.a.mass ? mov.mass[m] : 0.0f;
      const int64_t id = v.a.id ? mov.id[m] : 0;
      v.a.key[q] = key;
      v.a.ox[q] = ox;
      v.a.oy[q] = oy;
      v.a.oz[q] = oz;
      v.a.vx[q] = vx;
      v.a.vy[q] = vy;
      v.a.vz[q] = vz;
      if (v.a.mass) v.a.mass[q] = ms;
      if (v.a.id) v.a.id[q] = id;
      placed[m] = 1;
    } else {
      placed[m] = 0;  // the brick is full: it gets relocated (lf2_store.cu)
      if (atomicExch(&ovf_state[b], 1) == 0) ovf_list[atomicAdd(ovf_count, 1)] = (int32_t)b;
    }
  }
}

// max over bricks of max |v|^2 -> stats[0] (one CTA, fixed order).
__global__ void __launch_bounds__(1024) k_reduce_maxv(int64_t nb, const float* __restrict__ bm,
                                                      double* stats)
{
  __shared__ float sh[1024];
  float m = 0.0f;
  for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) m = fmaxf(m, bm[b]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) stats[0] = (double)sh[0];
}

}  // namespace

// The caller zeroes c->mov_count before a drift.
cudaError_t launch_move(lf2_ctx* c, const float* F, bool kick, bool drift, MoveParams mp)
{
  c->launches += 1;
  const size_t smem = kick ? (MOVE_F4 ? sizeof(float4) : 3 * sizeof(float)) * TILE3 : 0;
  const unsigned nb = (unsigned)c->g.nbricks;
  if (kick && drift) {
    cudaFuncSetAttribute(k_move<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_move<true, true><<<nb, MOVE_THREADS, smem, c->stream>>>(view(c), F, mp, c->mov, c->mov_count,
                                                             c->brick_maxv2, c->flags);
  } else if (kick) {
    cudaFuncSetAttribute(k_move<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    k_move<true, false><<<nb, MOVE_THREADS, smem, c->stream>>>(view(c), F, mp, c->mov, c->mov_count,
                                                              c->brick_maxv2, c->flags);
  } else if (drift) {
    k_move<false, true><<<nb, MOVE_THREADS, 0, c->stream>>>(view(c), F, mp, c->mov, c->mov_count,
                                                           c->brick_maxv2, c->flags);
  } else {
    k_move<false, false><<<nb, MOVE_THREADS, 0, c->stream>>>(view(c), F, mp, c->mov, c->mov_count,
                                                            c->brick_maxv2, c->flags);
  }
  return cudaGetLastError();
}

cudaError_t launch_insert(lf2_ctx* c)
{
  c->launches += 1;
  k_insert<<<148 * 4, 256, 0, c->stream>>>(view(c), c->mov, c->mov_count, c->mov_placed,
                                           c->ovf_list, c->ovf_count, c->ovf_state, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_reduce_maxv(lf2_ctx* c)
{
  c->launches += 1;
  k_reduce_maxv<<<1, 1024, 0, c->stream>>>(c->g.nbricks, c->brick_maxv2, c->stats);
  return cudaGetLastError();
}

namespace {
__global__ void k_sqrt_to(double* dst, const double* src) { *dst = sqrt(*src); }
}  // namespace

cudaError_t launch_maxv_to_device(lf2_ctx* c, double* dst)
{
  cudaError_t e = launch_reduce_maxv(c);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_sqrt_to<<<1, 1, 0, c->stream>>>(dst, c->stats);
  return cudaGetLastError();
}

}  // namespace lf2
