// lf2_move_pipe.cu -- fused gather-kick, drift and rebin (lf2_step) as a
// persistent, warp-specialised kernel.
//
// Same arithmetic and the same rebin as k_move<kick, drift> (lf2_move.cu):
// CIC gather of the 3-component field with the fixed corner order, kick,
// drift in cell units with the periodic carry, in-place compaction of the
// particles that stay in their brick (in slot order) and the mover buffer for
// the others.  What differs is how the data reaches the SM:
//
//   * one CTA per SM; warp 16 is the producer, warps 0-15 the consumers;
//   * bricks are taken from a global counter (load balance for clustered
//     particle distributions); empty bricks cost one atomic;
//   * the producer loads each brick's (BRICK+1)^3 vertex tile of F with one
//     4-D TMA copy (cp.async.bulk.tensor, box 20 x 17 x 17 x 3, rows padded to
//     20 floats so the box width is a multiple of 16 bytes) into one of two
//     tile buffers, and each chunk of CHUNK particles with one bulk copy per
//     array (cp.async.bulk) into a ring of chunk buffers; completion is
//     signalled on mbarriers, so the next brick's tile and the next chunks
//     stream in while the consumers work on the current ones;
//   * vertices that wrap around the periodic boundary lie outside the tensor
//     and arrive as zeros; the consumers patch those planes with plain loads.
//
// Every mbarrier wait is bounded (LF2_FLAG_TIMEOUT and an early return).
// No cluster multicast is used.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "lf2_internal.h"

namespace lf2 {

namespace {

constexpr int PC_WARPS = 16;                     // consumer warps
constexpr int PC_THREADS = PC_WARPS * 32;        // consumer threads
constexpr int P_THREADS = PC_THREADS + 32;       // + one producer warp
constexpr int P_ITEMS = 2;                       // consecutive slots per consumer thread
constexpr int CHUNK = PC_THREADS * P_ITEMS;      // particles per chunk buffer
constexpr int FX = 20;                           // padded tile row (floats)
constexpr int FCOMP = FX * TILE * TILE;          // floats per component of a tile buffer
constexpr uint32_t FBYTES = 3u * FCOMP * 4u;     // bytes one tile copy delivers
constexpr int FSTRIDE = (FBYTES + 1023) & ~1023; // tile buffer stride in shared memory
constexpr int MAX_STAGES = 4;
constexpr long long WAIT_CYCLES = 4000000000LL;  // about 2 s at the boost clock

struct Job {
  long long b;     // brick, or -1: no more bricks
  long long base;  // first slot of the brick's segment
  int cnt;         // particles
};

__device__ __forceinline__ uint32_t saddr(const void* p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity; false (and the timeout flag)
// when it has not completed within WAIT_CYCLES.
__device__ __noinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* flags)
{
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > WAIT_CYCLES) {
      set_flag(flags, ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          saddr(dst)),
      "l"(src), "r"(bytes), "r"(saddr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_tile4(void* dst, const CUtensorMap* map, int x, int y, int z,
                                          int c, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(saddr(bar))
      : "memory");
}

// named barrier of the consumer warps (the producer warp never joins it)
__device__ __forceinline__ void cbar()
{
  asm volatile("bar.sync 1, %0;" ::"n"(PC_THREADS) : "memory");
}

// Exclusive scan over the consumer threads; `buf` is 32 ints of shared
// memory that alternates between consecutive calls.
__device__ __forceinline__ int cscan(int v, int* buf, int* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) buf[warp] = x;
  cbar();
  if (warp == 0) {
    int t = lane < PC_WARPS ? buf[lane] : 0;
#pragma unroll
    for (int o = 1; o < PC_WARPS; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < PC_WARPS) buf[lane] = t;
  }
  cbar();
  *total = buf[PC_WARPS - 1];
  return (warp ? buf[warp - 1] : 0) + x - v;
}

__device__ __forceinline__ float sel(int b, float up, float dn) { return b ? up : dn; }

// Chunk buffer layout: key, ox, oy, oz, vx, vy, vz [, mass] [, id], PITCH
// entries each.  A chunk arrives at entry 0 of every array; the particles
// that stay are written back to entry a + q (q their rank among the chunk's
// stayers, a the 16-byte misalignment of their destination slot), so that
// entry 4k lines up with an aligned 4-slot group of the destination.
constexpr int PITCH = CHUNK + 32;

struct ChunkView {
  uint32_t* key;
  float *ox, *oy, *oz, *vx, *vy, *vz, *m;
  int64_t* id;
};

__device__ __forceinline__ ChunkView chunk_view(unsigned char* p, bool has_m)
{
  ChunkView c;
  c.key = reinterpret_cast<uint32_t*>(p);
  c.ox = reinterpret_cast<float*>(p + 1 * PITCH * 4);
  c.oy = reinterpret_cast<float*>(p + 2 * PITCH * 4);
  c.oz = reinterpret_cast<float*>(p + 3 * PITCH * 4);
  c.vx = reinterpret_cast<float*>(p + 4 * PITCH * 4);
  c.vy = reinterpret_cast<float*>(p + 5 * PITCH * 4);
  c.vz = reinterpret_cast<float*>(p + 6 * PITCH * 4);
  c.m = reinterpret_cast<float*>(p + 7 * PITCH * 4);
  c.id = reinterpret_cast<int64_t*>(p + (has_m ? 8 : 7) * PITCH * 4);
  return c;
}

// Copy entries [a, a + total) of a staged 32-bit array to dst[d0 + a ...):
// whole aligned 4-entry groups as 16-byte vectors, the partial first and
// last groups entry by entry.  d0 is a multiple of 4 slots.
__device__ __forceinline__ void copy_out32(const uint32_t* __restrict__ src, uint32_t* dst,
                                           int64_t d0, int a, int total, int ct)
{
  const int end = a + total, ng = (end + 3) >> 2;
  for (int k = ct; k < ng; k += PC_THREADS) {
    const int e0 = 4 * k;
    if (e0 >= a && e0 + 4 <= end) {
      *reinterpret_cast<uint4*>(dst + d0 + e0) = *reinterpret_cast<const uint4*>(src + e0);
    } else {
      for (int e = max(e0, a); e < min(e0 + 4, end); e++) dst[d0 + e] = src[e];
    }
  }
}

__device__ __forceinline__ void copy_out64(const int64_t* __restrict__ src, int64_t* dst,
                                           int64_t d0, int a, int total, int ct)
{
  const int end = a + total, ng = (end + 1) >> 1;
  for (int k = ct; k < ng; k += PC_THREADS) {
    const int e0 = 2 * k;
    if (e0 >= a && e0 + 2 <= end) {
      *reinterpret_cast<longlong2*>(dst + d0 + e0) = *reinterpret_cast<const longlong2*>(src + e0);
    } else {
      for (int e = max(e0, a); e < min(e0 + 2, end); e++) dst[d0 + e] = src[e];
    }
  }
}

__global__ void __launch_bounds__(P_THREADS, 1)
    k_move_pipe(const __grid_constant__ CUtensorMap tmF, StoreView v, const float* __restrict__ F,
                MoveParams mp, PartArrays mov, unsigned long long* mov_count,
                unsigned long long* mov_real, float* __restrict__ brick_maxv2, uint32_t* flags,
                int* work, int nst, int stage_bytes)
{
  extern __shared__ unsigned char dyn[];
  __shared__ uint64_t full_f[2], empty_f[2], full_p[MAX_STAGES], empty_p[MAX_STAGES];
  __shared__ Job job[2];
  __shared__ int s_scan[2][32];
  __shared__ float s_max[PC_WARPS];
  __shared__ int s_ok_f, s_ok_p;  // outcome of thread 0's last tile / chunk wait
  // mover block of this CTA: slots [mv_base, mv_base + MOV_BLOCK) of the mover
  // buffer, mv_used of them filled; mv_next a fresh block when a chunk's
  // movers do not fit (double-buffered by chunk parity)
  __shared__ long long s_mv_base[2], s_mv_next[2];
  __shared__ int s_mv_used[2];

  unsigned char* sm = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char* pbuf = sm + 2 * FSTRIDE;

  const Geom& g = v.g;
  const bool has_m = v.a.mass != nullptr, has_id = v.a.id != nullptr;

  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; s++) mbar_init(&full_f[s], 1), mbar_init(&empty_f[s], 1);
    for (int s = 0; s < nst; s++) mbar_init(&full_p[s], 1), mbar_init(&empty_p[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x >= PC_THREADS) {
    // ------------------------------------------------------------ producer
    if (threadIdx.x != PC_THREADS) return;
    long long fk = 0, pk = 0;  // tile buffers and chunk buffers handed out so far
    for (;;) {
      const long long b = atomicAdd(work, 1);
      const int fs = (int)(fk & 1);
      if (b >= g.nbricks) {
        if (fk >= 2 && !mbar_wait(&empty_f[fs], (uint32_t)(((fk >> 1) - 1) & 1), flags)) return;
        job[fs].b = -1;
        mbar_arrive(&full_f[fs]);
        return;
      }
      const int cnt = LF2_BRICK_COUNT(v, b);
      if (cnt == 0) {
        brick_maxv2[b] = 0.0f;
        continue;
      }
      if (fk >= 2 && !mbar_wait(&empty_f[fs], (uint32_t)(((fk >> 1) - 1) & 1), flags)) return;
      const long long base = v.seg_start[b];
      job[fs].b = b;
      job[fs].base = base;
      job[fs].cnt = cnt;
      int bx, by, bz;
      brick_coords(g, b, bx, by, bz);
      mbar_arrive_tx(&full_f[fs], FBYTES);
      tma_tile4(sm + fs * FSTRIDE, &tmF, bx * BRICK, by * BRICK, bz * BRICK, 0, &full_f[fs]);
      fk++;
      for (int c0 = 0; c0 < cnt; c0 += CHUNK) {
        const int ps = (int)(pk % nst);
        const long long use = pk / nst;
        if (use > 0 && !mbar_wait(&empty_p[ps], (uint32_t)((use - 1) & 1), flags)) return;
        const int n = min(CHUNK, cnt - c0);
        const uint32_t n4 = (uint32_t)((n + 3) & ~3);  // segments hold a multiple of 4 slots
        const uint32_t bytes = n4 * 4u * (7u + (has_m ? 1u : 0u)) + (has_id ? n4 * 8u : 0u);
        const ChunkView cv = chunk_view(pbuf + (size_t)ps * stage_bytes, has_m);
        const long long p = base + c0;
        mbar_arrive_tx(&full_p[ps], bytes);
        bulk_g2s(cv.key, v.a.key + p, n4 * 4u, &full_p[ps]);
        bulk_g2s(cv.ox, v.a.ox + p, n4 * 4u, &full_p[ps]);
        bulk_g2s(cv.oy, v.a.oy + p, n4 * 4u, &full_p[ps]);
        bulk_g2s(cv.oz, v.a.oz + p, n4 * 4u, &full_p[ps]);
        bulk_g2s(cv.vx, v.a.vx + p, n4 * 4u, &full_p[ps]);
        bulk_g2s(cv.vy, v.a.vy + p, n4 * 4u, &full_p[ps]);
        bulk_g2s(cv.vz, v.a.vz + p, n4 * 4u, &full_p[ps]);
        if (has_m) bulk_g2s(cv.m, v.a.mass + p, n4 * 4u, &full_p[ps]);
        if (has_id) bulk_g2s(cv.id, v.a.id + p, n4 * 8u, &full_p[ps]);
        pk++;
      }
    }
  }

  // -------------------------------------------------------------- consumers
  // Thread 0 does the bounded mbarrier waits and hands the outcome to the
  // other consumers through the named barrier, so that on a timeout all of
  // them leave together and none is left waiting at a barrier.
  const int ct = threadIdx.x, lane = ct & 31;
  long long fk = 0, pk = 0;
  int sc = 0;             // parity of the per-chunk shared scratch
  int pending = -1;       // chunk buffer to hand back at the next barrier
  // mover block state, kept by thread 0
  long long mv_base = -1, mv_real = 0;
  int mv_used = MOV_BLOCK;
  for (;;) {
    const int fs = (int)(fk & 1);
    const uint32_t fpar = (uint32_t)((fk >> 1) & 1);
    if (ct == 0) s_ok_f = mbar_wait(&full_f[fs], fpar, flags);
    cbar();
    if (ct == 0 && pending >= 0) mbar_arrive(&empty_p[pending]);
    pending = -1;
    if (!s_ok_f) return;
    mbar_try(&full_f[fs], fpar);  // completed: acquire for this thread
    const Job jb = job[fs];
    if (jb.b < 0) {
      // Unused slots of the last mover block get an invalid offset (-1),
      // which k_insert skips.
      if (ct == 0) {
        s_mv_base[0] = mv_base;
        s_mv_used[0] = mv_used;
        if (mv_real) atomicAdd(mov_real, (unsigned long long)mv_real);
      }
      cbar();
      if (s_mv_base[0] >= 0)
        for (int i = s_mv_used[0] + ct; i < MOV_BLOCK; i += PC_THREADS) mov.ox[s_mv_base[0] + i] = -1.0f;
      return;
    }
    const int64_t b = jb.b;
    const int cnt = jb.cnt;
    float* ft = reinterpret_cast<float*>(sm + fs * FSTRIDE);
    int bx, by, bz;
    brick_coords(g, b, bx, by, bz);
    const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
    const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
              ez = brick_extent(g.n[2], bz);
    const bool wx = x0 + ex == g.n[0], wy = y0 + ey == g.n[1], wz = z0 + ez == g.n[2];
    if (wx || wy || wz) {
      // Vertex planes on the upper periodic boundary lie outside the tensor:
      // plane i = ex maps to x = 0 (likewise y, z).
      const int np_ = TILE * TILE;
      for (int t = ct; t < 3 * np_; t += PC_THREADS) {
        const int pl = t / np_, r = t % np_, u = r % TILE, w = r / TILE;
        int i, j, k;
        if (pl == 0) {
          if (!wx) continue;
          i = ex, j = u, k = w;
        } else if (pl == 1) {
          if (!wy) continue;
          i = u, j = ey, k = w;
        } else {
          if (!wz) continue;
          i = u, j = w, k = ez;
        }
        if (i > ex || j > ey || k > ez) continue;
        const int gx = x0 + i < g.n[0] ? x0 + i : 0;
        const int gy = y0 + j < g.n[1] ? y0 + j : 0;
        const int gz = z0 + k < g.n[2] ? z0 + k : 0;
        const int64_t s = site_index(g, gx, gy, gz);
        const int o = i + FX * (j + TILE * k);
        ft[o] = __ldg(F + s);
        ft[FCOMP + o] = __ldg(F + g.nsites + s);
        ft[2 * FCOMP + o] = __ldg(F + 2 * g.nsites + s);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      cbar();
    }

    int write = 0;
    float maxv2 = 0.0f;
    for (int c0 = 0; c0 < cnt; c0 += CHUNK) {
      const int ps = (int)(pk % nst);
      const uint32_t ppar = (uint32_t)((pk / nst) & 1);
      if (ct == 0) {
        s_ok_p = mbar_wait(&full_p[ps], ppar, flags);
        s_mv_base[sc] = mv_base;
        s_mv_used[sc] = mv_used;
      }
      cbar();
      if (ct == 0 && pending >= 0) mbar_arrive(&empty_p[pending]);
      pending = -1;
      if (!s_ok_p) return;
      mbar_try(&full_p[ps], ppar);
      const ChunkView cv = chunk_view(pbuf + (size_t)ps * stage_bytes, has_m);
      const int n = min(CHUNK, cnt - c0);
      const int i0 = P_ITEMS * ct;
      uint32_t key[P_ITEMS];
      float ox[P_ITEMS], oy[P_ITEMS], oz[P_ITEMS], vx[P_ITEMS], vy[P_ITEMS], vz[P_ITEMS];
      float m[P_ITEMS];
      int64_t id[P_ITEMS];
      bool act[P_ITEMS], stay[P_ITEMS];
      if (i0 < n) {
        const uint2 k2 = *reinterpret_cast<const uint2*>(cv.key + i0);
        const float2 a = *reinterpret_cast<const float2*>(cv.ox + i0);
        const float2 bb = *reinterpret_cast<const float2*>(cv.oy + i0);
        const float2 cc = *reinterpret_cast<const float2*>(cv.oz + i0);
        const float2 d = *reinterpret_cast<const float2*>(cv.vx + i0);
        const float2 e = *reinterpret_cast<const float2*>(cv.vy + i0);
        const float2 f = *reinterpret_cast<const float2*>(cv.vz + i0);
        key[0] = k2.x, key[1] = k2.y;
        ox[0] = a.x, ox[1] = a.y, oy[0] = bb.x, oy[1] = bb.y, oz[0] = cc.x, oz[1] = cc.y;
        vx[0] = d.x, vx[1] = d.y, vy[0] = e.x, vy[1] = e.y, vz[0] = f.x, vz[1] = f.y;
      }
#pragma unroll
      for (int j = 0; j < P_ITEMS; j++) {
        act[j] = i0 + j < n;
        stay[j] = true;
        m[j] = 0.0f;
        id[j] = 0;
        if (act[j]) {
          if (has_m) m[j] = cv.m[i0 + j];
          if (has_id) id[j] = cv.id[i0 + j];
        }
      }
#pragma unroll
      for (int j = 0; j < P_ITEMS; j++) {
        if (!act[j]) continue;
        int x, y, z;
        unpack_key(g, key[j], x, y, z);
        const int t0 = (x - x0) + FX * ((y - y0) + TILE * (z - z0));
        const float gx = __fsub_rn(1.0f, ox[j]), gy = __fsub_rn(1.0f, oy[j]),
                    gz = __fsub_rn(1.0f, oz[j]);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
          const float w = __fmul_rn(__fmul_rn(sel(cx, ox[j], gx), sel(cy, oy[j], gy)),
                                    sel(cz, oz[j], gz));
          const int t = t0 + cx + cy * FX + cz * FX * TILE;
          a0 = __fmaf_rn(w, ft[t], a0);
          a1 = __fmaf_rn(w, ft[FCOMP + t], a1);
          a2 = __fmaf_rn(w, ft[2 * FCOMP + t], a2);
        }
        vx[j] = __fmaf_rn(mp.dtk, a0, vx[j]);
        vy[j] = __fmaf_rn(mp.dtk, a1, vy[j]);
        vz[j] = __fmaf_rn(mp.dtk, a2, vz[j]);
        maxv2 = fmaxf(maxv2, __fadd_rn(__fadd_rn(__fmul_rn(vx[j], vx[j]), __fmul_rn(vy[j], vy[j])),
                                       __fmul_rn(vz[j], vz[j])));
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

      // One scan ranks both groups: stayers in the low 16 bits, movers in the
      // high 16 bits (at most CHUNK of each).
      int ns = 0, nm = 0;
#pragma unroll
      for (int j = 0; j < P_ITEMS; j++) {
        ns += (act[j] && stay[j]) ? 1 : 0;
        nm += (act[j] && !stay[j]) ? 1 : 0;
      }
      int tot;
      const int pre = cscan(ns | (nm << 16), s_scan[sc], &tot);
      const int total = tot & 0xffff, mtot = tot >> 16;
      int q = pre & 0xffff, mq = pre >> 16;

      // Movers: the chunk's movers take the next mtot slots of the CTA's
      // mover block, spilling into a fresh block when the block is full.
      const long long mb = s_mv_base[sc];
      const int mu = s_mv_used[sc];
      if (mtot > MOV_BLOCK - mu) {  // uniform: every consumer sees the same values
        if (ct == 0) s_mv_next[sc] = (long long)atomicAdd(mov_count, (unsigned long long)MOV_BLOCK);
        cbar();
      }
      const long long mn = mtot > MOV_BLOCK - mu ? s_mv_next[sc] : -1;

      // Stayers are staged in the chunk buffer (all of it has been read:
      // the scan's barriers are behind every consumer), movers go out now.
      const int64_t dst = jb.base + write;
      const int a = (int)(dst & 3);
#pragma unroll
      for (int j = 0; j < P_ITEMS; j++) {
        if (!act[j]) continue;
        if (stay[j]) {
          const int e = a + q++;
          cv.key[e] = key[j];
          cv.ox[e] = ox[j];
          cv.oy[e] = oy[j];
          cv.oz[e] = oz[j];
          cv.vx[e] = vx[j];
          cv.vy[e] = vy[j];
          cv.vz[e] = vz[j];
          if (has_m) cv.m[e] = m[j];
          if (has_id) cv.id[e] = id[j];
        } else {
          const int idx = mu + mq++;
          const int64_t s = idx < MOV_BLOCK ? mb + idx : mn + (idx - MOV_BLOCK);
          mov.key[s] = key[j];
          mov.ox[s] = ox[j];
          mov.oy[s] = oy[j];
          mov.oz[s] = oz[j];
          mov.vx[s] = vx[j];
          mov.vy[s] = vy[j];
          mov.vz[s] = vz[j];
          if (mov.mass) mov.mass[s] = m[j];
          if (mov.id) mov.id[s] = id[j];
        }
      }
      if (ct == 0) {
        mv_used = mu + mtot;
        if (mn >= 0) {
          mv_base = mn;
          mv_used -= MOV_BLOCK;
        }
        mv_real += mtot;
      }
      cbar();
      const int64_t d0 = dst - a;
      copy_out32(cv.key, v.a.key, d0, a, total, ct);
      copy_out32(reinterpret_cast<const uint32_t*>(cv.ox), reinterpret_cast<uint32_t*>(v.a.ox), d0, a, total, ct);
      copy_out32(reinterpret_cast<const uint32_t*>(cv.oy), reinterpret_cast<uint32_t*>(v.a.oy), d0, a, total, ct);
      copy_out32(reinterpret_cast<const uint32_t*>(cv.oz), reinterpret_cast<uint32_t*>(v.a.oz), d0, a, total, ct);
      copy_out32(reinterpret_cast<const uint32_t*>(cv.vx), reinterpret_cast<uint32_t*>(v.a.vx), d0, a, total, ct);
      copy_out32(reinterpret_cast<const uint32_t*>(cv.vy), reinterpret_cast<uint32_t*>(v.a.vy), d0, a, total, ct);
      copy_out32(reinterpret_cast<const uint32_t*>(cv.vz), reinterpret_cast<uint32_t*>(v.a.vz), d0, a, total, ct);
      if (has_m)
        copy_out32(reinterpret_cast<const uint32_t*>(cv.m), reinterpret_cast<uint32_t*>(v.a.mass), d0, a, total, ct);
      if (has_id) copy_out64(cv.id, v.a.id, d0, a, total, ct);
      // the buffer is handed back after the next barrier, when every
      // consumer has copied its part out
      pending = ps;
      pk++;
      sc ^= 1;
      write += total;
    }

    for (int o = 16; o > 0; o >>= 1) maxv2 = fmaxf(maxv2, __shfl_xor_sync(0xffffffffu, maxv2, o));
    if (lane == 0) s_max[ct >> 5] = maxv2;
    cbar();
    if (ct == 0) {
      if (pending >= 0) mbar_arrive(&empty_p[pending]);
      float mm = 0.0f;
      for (int w = 0; w < PC_WARPS; w++) mm = fmaxf(mm, s_max[w]);
      brick_maxv2[b] = mm;
      v.count[b] = write;
      mbar_arrive(&empty_f[fs]);  // all gathers of this brick are done
    }
    pending = -1;
    fk++;
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

size_t stage_bytes_for(const lf2_ctx* c)
{
  return (size_t)PITCH * (28 + (c->has_mass ? 4 : 0) + (c->has_id ? 8 : 0));
}

}  // namespace

// Whether lf2_step's fused move can take the pipelined kernel: a 4-D tensor
// map needs 16-byte aligned rows (n0 % 4 == 0) and base, and the lattice is
// at least two bricks wide in every dim.
bool move_pipe_eligible(const lf2_ctx* c, const float* F)
{
  if (!F || ((uintptr_t)F & 15) || (c->g.n[0] & 3)) return false;
  for (int d = 0; d < 3; d++)
    if (c->g.n[d] < 2 * BRICK) return false;
  return encode_fn() != nullptr;
}

cudaError_t launch_move_pipe(lf2_ctx* c, const float* F, MoveParams mp)
{
  static_assert(sizeof(CUtensorMap) <= sizeof(c->tmap_bytes), "tensor map storage");
  CUtensorMap* map = reinterpret_cast<CUtensorMap*>(c->tmap_bytes);
  if (c->tmap_src != F) {
    const cuuint64_t dims[4] = {(cuuint64_t)c->g.n[0], (cuuint64_t)c->g.n[1],
                                (cuuint64_t)c->g.n[2], 3};
    const cuuint64_t strides[3] = {(cuuint64_t)c->g.n[0] * 4,
                                   (cuuint64_t)c->g.n[0] * c->g.n[1] * 4,
                                   (cuuint64_t)c->g.nsites * 4};
    const cuuint32_t box[4] = {FX, TILE, TILE, 3};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(F),
                                   dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      c->tmap_src = nullptr;
      return cudaErrorInvalidValue;
    }
    c->tmap_src = F;
  }
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  const size_t sb = stage_bytes_for(c);
  const size_t fixed = 1024 + 2 * (size_t)FSTRIDE + 2048;  // alignment slack, tiles, static
  int nst = (int)(((size_t)optin > fixed ? (size_t)optin - fixed : 0) / sb);
  nst = nst > MAX_STAGES ? MAX_STAGES : nst;
  if (nst < 2) return cudaErrorInvalidConfiguration;
  const size_t smem = 1024 + 2 * (size_t)FSTRIDE + (size_t)nst * sb;
  cudaError_t e = cudaFuncSetAttribute(k_move_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(c->work, 0, sizeof(int), c->stream);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_move_pipe<<<c->num_sms, P_THREADS, smem, c->stream>>>(*map, view(c), F, mp, c->mov, c->mov_count,
                                                          c->mov_real, c->brick_maxv2, c->flags,
                                                          c->work, nst, (int)sb);
  return cudaGetLastError();
}

}  // namespace lf2
