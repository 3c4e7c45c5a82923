// lf2_move_pipe.cu -- fused gather-kick, drift and rebin (lf2_step) as a
// persistent, warp-specialised kernel.
//
// Same arithmetic as k_move<kick, drift> (lf2_move.cu): CIC gather of the
// 3-component field with the fixed corner order, kick, drift in cell units
// with the periodic carry; particles that stay in their brick are written
// back in place at the front of its segment, the others go to the mover
// buffer.  What differs is how the data reaches the SM and how the work is
// shared:
//
//   * one CTA per SM: consumer warps, one producer warp (a single thread)
//     and one patch warp;
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
//     and arrive as zeros; the patch warp fills those planes with plain loads
//     before it releases the tile to the consumers, off the producer's path;
//   * the producer fetches brick indices and segment bounds ahead and posts
//     a brick's tile copy as soon as a tile buffer frees up, between the
//     chunk copies of the brick before;
//   * consumer warps never wait for one another: each takes its own slice of
//     every chunk and reserves its output slots with atomics.  The order of
//     the stayers inside a brick therefore follows the warps' timing.
//
// Every mbarrier wait is bounded (LF2_FLAG_TIMEOUT, then the warp returns).
// A producer that gives up, or that has posted its last copy, first waits
// (with the full limit) for every bulk and tensor copy it has issued to land,
// so the CTA never exits with a copy still writing its shared memory.  The
// limit of the other waits is a launch parameter (lf2_set_wait_limit); for
// the tests of this path the consumers can be made to wait on a barrier that
// nothing completes.  No cluster multicast is used.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "lf2_deposit_common.cuh"
#include "lf2_internal.h"

namespace lf2 {

namespace {

// Launch shape: consumer warps x particles per lane (measured at 512^3 with
// 134M particles before the patch warp existed: 31 x 1 2.79 ms, 24 x 1 2.81,
// 16 x 2 2.84, 8 x 4 3.78; two chunk buffers instead of three cost 9%)
#ifndef LF2_PIPE_WARPS
#define LF2_PIPE_WARPS 30
#endif
#ifndef LF2_PIPE_ITEMS
#define LF2_PIPE_ITEMS 1
#endif
// The kernel is a template of its consumer warps (WARPS; each takes WSUB
// slots of every chunk, CHUNK = WARPS * WSUB) plus a producer warp and a
// patch warp.
constexpr int W_ITEMS = LF2_PIPE_ITEMS;          // consecutive slots per lane
constexpr int WSUB = 32 * W_ITEMS;               // slots per warp per chunk
constexpr int FX = 20;                           // padded tile row (floats)
constexpr int FCOMP = FX * TILE * TILE;          // floats per component of a tile buffer
constexpr uint32_t FBYTES = 3u * FCOMP * 4u;     // bytes one tile copy delivers
constexpr int FSTRIDE = (FBYTES + 1023) & ~1023; // tile buffer stride in shared memory
constexpr int FSTRIDE_DEP = (FBYTES + 127) & ~127; // the same in the fused-deposit layout
// Fused deposit (lf2_step with the fixed-point scalar deposit): one split
// fixed-point tile of the brick's (BRICK+1)^3 vertices, two 32-bit words per
// vertex, between the vertex tiles and the chunk ring.
// Rounded up to 128 bytes: the chunk ring after it is the destination of
// bulk copies, which must start on a 16-byte boundary.
constexpr int DEP_BYTES = (2 * TILE3 * 4 + 127) & ~127;
static_assert(FSTRIDE_DEP % 128 == 0 && DEP_BYTES % 128 == 0, "bulk-copy destinations stay aligned");
// Vertices of a brick's tile that movers from the neighbour bricks can reach
// (a coordinate in {0, 1, e-1, e}): they go to the per-brick rim store, the
// others (every coordinate in [2, e-2]) are final after the fused pass.
constexpr int RIM = TILE3 - (BRICK - 3) * (BRICK - 3) * (BRICK - 3);
#ifndef LF2_PIPE_FSTAGES
#define LF2_PIPE_FSTAGES 2
#endif
constexpr int NF = LF2_PIPE_FSTAGES;             // tile buffers (1 or 2)
static_assert(NF == 1 || NF == 2, "one or two tile buffers");
#ifndef LF2_PIPE_MAX_STAGES
#define LF2_PIPE_MAX_STAGES 4
#endif
constexpr int MAX_STAGES = LF2_PIPE_MAX_STAGES;  // chunk buffers (as many as fit, up to this)
constexpr long long WAIT_CYCLES = 4000000000LL;  // about 2 s at the boost clock

struct Job {
  long long b;     // brick, or -1: no more bricks
  long long base;  // first slot of the brick's segment
  int cnt;         // particles
  int bx, by, bz;  // brick coordinates
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

// non-blocking test of a phase
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait that lets the hardware suspend the thread for up to `ns`
// nanoseconds while the phase is incomplete
__device__ __forceinline__ bool mbar_try_hint(uint64_t* bar, uint32_t parity, uint32_t ns)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity; false (and the timeout flag)
// when it has not completed within `limit` cycles.  The waiting thread is
// suspended between polls (measured: 2% faster than a plain poll loop).
__device__ __noinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* flags,
                                       long long limit)
{
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  for (;;) {
    if (mbar_try_hint(bar, parity, 20000u)) return true;
    if (clock64() - t0 > limit) {
      set_flag(flags, ERR_TIMEOUT);
      return false;
    }
  }
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

__device__ __forceinline__ float sel(int b, float up, float dn) { return b ? up : dn; }

// x + carry wrapped into [0, n): two selects cover |carry| <= n, the general
// case (a particle that crosses the whole lattice in one step) is out of line.
__device__ __noinline__ int wrap_far(int x, int carry, int n) { return wrap_add(x, carry, n); }

__device__ __forceinline__ int wrap_near(int x, int carry, int n)
{
  int v = x + carry;
  v += v < 0 ? n : 0;
  v -= v >= n ? n : 0;
  if ((unsigned)v >= (unsigned)n) v = wrap_far(x, carry, n);
  return v;
}

// Chunk buffer layout: key, ox, oy, oz, vx, vy, vz [, mass] [, id], CHUNK
// entries each.
struct ChunkView {
  uint32_t* key;
  float *ox, *oy, *oz, *vx, *vy, *vz, *m;
  int64_t* id;
};

__device__ __forceinline__ ChunkView chunk_view(unsigned char* p, bool has_m, int chunk)
{
  ChunkView c;
  c.key = reinterpret_cast<uint32_t*>(p);
  c.ox = reinterpret_cast<float*>(p + 1 * chunk * 4);
  c.oy = reinterpret_cast<float*>(p + 2 * chunk * 4);
  c.oz = reinterpret_cast<float*>(p + 3 * chunk * 4);
  c.vx = reinterpret_cast<float*>(p + 4 * chunk * 4);
  c.vy = reinterpret_cast<float*>(p + 5 * chunk * 4);
  c.vz = reinterpret_cast<float*>(p + 6 * chunk * 4);
  c.m = reinterpret_cast<float*>(p + 7 * chunk * 4);
  c.id = reinterpret_cast<int64_t*>(p + (has_m ? 8 : 7) * chunk * 4);
  return c;
}

// Canonical coordinate of a tile vertex in the rim store layout: e -> BRICK,
// e - 1 -> BRICK - 1 (when >= 2), so that bricks with e < BRICK share it.
__host__ __device__ inline int rim_canon(int t, int e)
{
  return t == e ? BRICK : (t == e - 1 && t >= 2 ? BRICK - 1 : t);
}
__host__ __device__ inline bool rim_layer(int u) { return u < 2 || u >= BRICK - 1; }
__host__ __device__ inline int rim_slot(int u) { return u < 2 ? u : u - (BRICK - 3); }
// Index of a rim vertex (canonical coordinates): the two z slab pairs
// (4 TILE^2), then the y slab pairs between them (4 (BRICK-3) TILE), then the
// x slab pairs between those (4 (BRICK-3)^2): 2716 slots for BRICK = 16.
__host__ __device__ inline int rim_index(int u0, int u1, int u2)
{
  constexpr int I = BRICK - 3;
  if (rim_layer(u2)) return rim_slot(u2) * TILE * TILE + u1 * TILE + u0;
  if (rim_layer(u1)) return 4 * TILE * TILE + (rim_slot(u1) * I + (u2 - 2)) * TILE + u0;
  return 4 * TILE * TILE + 4 * I * TILE + (rim_slot(u0) * I + (u2 - 2)) * I + (u1 - 2);
}
static_assert(4 * TILE * TILE + 4 * (BRICK - 3) * TILE + 4 * (BRICK - 3) * (BRICK - 3) == RIM,
              "rim slab sizes");

// Outputs of the fused deposit.
struct DepOut {
  float* rho;        // density (private vertices written by the fused pass)
  uint64_t* rim;     // [nbricks * RIM] integer sums of the rim vertices
  float scale;       // 2^-32 * unit mass / res^3
  float inv_unit;    // 1 / unit mass (per-particle masses)
  int split_max;     // bricks up to this count accumulate in two 32-bit words
};

// Bounded wait by lane 0 of the calling warp; the outcome is broadcast so the
// warp stays together, and every lane then acquires the completed phase.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, uint32_t* flags, int lane,
                                          long long limit)
{
  int ok = 1;
  // the first poll inline; the bounded wait out of line
  if (lane == 0 && !mbar_try(bar, parity)) ok = mbar_wait(bar, parity, flags, limit);
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (ok) mbar_try(bar, parity);
  return ok != 0;
}

template <int WARPS, bool DEP, bool HM, bool HID>
__global__ void __launch_bounds__(WARPS * 32 + 64, 1)
    k_move_pipe(const __grid_constant__ CUtensorMap tmF, StoreView v, const float* __restrict__ F,
                MoveParams mp, PartArrays mov, unsigned long long* mov_count,
                float* __restrict__ brick_maxv2, uint32_t* flags, int* work, int nst,
                int stage_bytes, long long wait_limit, int stall, DepOut dep)
{
  constexpr int CHUNK = WARPS * WSUB;            // particles per chunk buffer
  constexpr int PC_WARPS = WARPS;                // consumer warps
  constexpr int FST = DEP ? FSTRIDE_DEP : FSTRIDE;
  constexpr uint32_t ALIGN = DEP ? 127 : 1023;
  extern __shared__ __align__(128) unsigned char dyn[];
  // tma_f: tile copy landed (or the end of the bricks); full_f: tile
  // patched and ready for the consumers; empty_f: all consumer warps are
  // done with the brick; full_p / empty_p: chunk ring.
  __shared__ uint64_t full_f[2], tma_f[2], empty_f[2], full_p[MAX_STAGES], empty_p[MAX_STAGES];
  __shared__ uint64_t never;  // completed by nothing: the consumers' stall of the timeout tests
  __shared__ uint64_t dep_in, dep_clean;  // fused deposit: all deposits of the brick in; tile clean
  __shared__ Job job[2];
  __shared__ int s_cursor[2];     // stayers written back so far (per tile buffer)
  __shared__ int s_done[2];       // consumer warps finished with the brick
  __shared__ unsigned s_maxv2[2]; // max |v|^2 of the brick (bits of a non-negative float)

  // Aligned base of the tile buffers, by an offset from the shared array
  // itself (not through an integer cast), so that every access below stays
  // a shared-memory access.
  const uint32_t mis = saddr(dyn) & ALIGN;
  unsigned char* sm = dyn + (mis ? ALIGN + 1 - mis : 0u);
  uint32_t* dtile = reinterpret_cast<uint32_t*>(sm + NF * FST);  // DEP: [lo | hi] x TILE3
  unsigned char* pbuf = sm + NF * FST + (DEP ? DEP_BYTES : 0);

  const Geom& g = v.g;
  // per-particle masses and IDs (the store carries them or not), fixed at
  // compile time
  constexpr bool has_m = HM, has_id = HID;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; s++) {
      mbar_init(&full_f[s], 1);
      mbar_init(&tma_f[s], 1);
      mbar_init(&empty_f[s], 1);
    }
    for (int s = 0; s < nst; s++) mbar_init(&full_p[s], 1), mbar_init(&empty_p[s], PC_WARPS);
    mbar_init(&never, 1);
    mbar_init(&dep_in, PC_WARPS);
    mbar_init(&dep_clean, PC_WARPS);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (DEP)
    for (int t = threadIdx.x; t < 2 * TILE3; t += blockDim.x) dtile[t] = 0u;
  __syncthreads();

  if (warp == PC_WARPS) {
    // ------------------------------------------------------------ producer
    // One thread.  It posts a brick (job and tile copy) as soon as a tile
    // buffer is free, polling for that while it issues the chunks of the
    // brick before; brick indices and segment bounds are fetched ahead.
    if (lane != 0) return;
    long long fk = 0;           // bricks posted so far (tile buffer fk % NF)
    int pps = 0;                // next chunk buffer
    uint32_t ppar = 0;          // parity of the current round through the ring
    bool wrapped = false;       // every buffer has been used once
    // the phase (parity) the last copy into each chunk buffer and tile buffer
    // completes, to wait for every copy in flight before the thread exits
    bool st_busy[MAX_STAGES], tl_busy[2] = {false, false};
    uint32_t st_par[MAX_STAGES], tl_par[2] = {0u, 0u};
    for (int s = 0; s < MAX_STAGES; s++) st_busy[s] = false, st_par[s] = 0u;
    auto drain = [&]() {
      for (int s = 0; s < nst; s++)
        if (st_busy[s]) mbar_wait(&full_p[s], st_par[s], flags, WAIT_CYCLES);
      for (int f = 0; f < NF; f++)
        if (tl_busy[f]) mbar_wait(&tma_f[f], tl_par[f], flags, WAIT_CYCLES);
    };
    // q0: next brick with its count and segment start loaded; q1: the index
    // after it
    long long q0 = atomicAdd(work, 1);
    int cq0 = q0 < g.nbricks ? LF2_BRICK_COUNT(v, q0) : 0;
    long long bq0 = q0 < g.nbricks ? v.seg_start[q0] : 0;
    long long q1 = q0 < g.nbricks ? atomicAdd(work, 1) : q0;
    // the next brick with particles (b = -1 after the last)
    auto next_brick = [&](long long& b, int& cnt, long long& base) {
      for (;;) {
        b = q0, cnt = cq0, base = bq0;
        q0 = q1;
        if (q0 < g.nbricks) {
          cq0 = LF2_BRICK_COUNT(v, q0);
          bq0 = v.seg_start[q0];
          q1 = atomicAdd(work, 1);
        }
        if (b >= g.nbricks) {
          b = -1;
          return;
        }
        if (cnt > 0 || DEP) return;  // the fused deposit writes empty bricks too
        brick_maxv2[b] = 0.0f;
      }
    };
    auto post = [&](long long b, int cnt, long long base) {
      const int fs = (int)(fk % NF);
      job[fs].b = b;
      tl_par[fs] = (uint32_t)((fk / NF) & 1);
      tl_busy[fs] = b >= 0;
      fk++;
      if (b < 0) {
        mbar_arrive(&tma_f[fs]);  // the patch warp passes it on to the consumers
        return;
      }
      job[fs].base = base;
      job[fs].cnt = cnt;
      brick_coords(g, b, job[fs].bx, job[fs].by, job[fs].bz);
      s_cursor[fs] = 0;
      s_done[fs] = 0;
      s_maxv2[fs] = 0u;
      if (cnt == 0) {  // an empty brick (fused deposit): no tile to load
        tl_busy[fs] = false;
        mbar_arrive(&tma_f[fs]);
        return;
      }
      mbar_arrive_tx(&tma_f[fs], FBYTES);
      tma_tile4(sm + fs * FST, &tmF, job[fs].bx * BRICK, job[fs].by * BRICK, job[fs].bz * BRICK, 0,
                &tma_f[fs]);
    };
    // tile buffer of the next post free?
    auto tile_free = [&]() {
      return fk < NF || mbar_test(&empty_f[fk % NF], (uint32_t)(((fk / NF) - 1) & 1));
    };
    long long cb, nb_;
    int ccnt, ncnt;
    long long cbase, nbase;
    next_brick(cb, ccnt, cbase);
    post(cb, ccnt, cbase);
    next_brick(nb_, ncnt, nbase);
    bool nposted = false;
    while (cb >= 0) {
      for (int c0 = 0; c0 < ccnt; c0 += CHUNK) {
        const int ps = pps;
        if (wrapped) {
          // the previous round's phase of this buffer's empty barrier; post
          // the next brick meanwhile if its tile buffer frees up
          const long long t0 = clock64();
          while (!mbar_test(&empty_p[ps], ppar ^ 1u)) {
            if (!nposted && tile_free()) {
              post(nb_, ncnt, nbase);
              nposted = true;
            }
            if (clock64() - t0 > wait_limit) {
              set_flag(flags, ERR_TIMEOUT);
              drain();
              return;
            }
            __nanosleep(64);
          }
        }
        if (!nposted && tile_free()) {
          post(nb_, ncnt, nbase);
          nposted = true;
        }
        const int n = min(CHUNK, ccnt - c0);
        const uint32_t n4 = (uint32_t)((n + 3) & ~3);  // segments hold a multiple of 4 slots
        const uint32_t bytes = n4 * 4u * (7u + (has_m ? 1u : 0u)) + (has_id ? n4 * 8u : 0u);
        const ChunkView cv = chunk_view(pbuf + (size_t)ps * stage_bytes, has_m, CHUNK);
        const long long p = cbase + c0;
        st_busy[ps] = true;
        st_par[ps] = ppar;
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
        if (++pps == nst) {
          pps = 0;
          ppar ^= 1u;
          wrapped = true;
        }
      }
      if (!nposted) {
        const int fs = (int)(fk % NF);
        if (fk >= NF && !mbar_wait(&empty_f[fs], (uint32_t)(((fk / NF) - 1) & 1), flags, wait_limit)) {
          drain();
          return;
        }
        post(nb_, ncnt, nbase);
      }
      cb = nb_, ccnt = ncnt, cbase = nbase;
      if (cb >= 0) next_brick(nb_, ncnt, nbase);
      nposted = false;
    }
    drain();
    return;
  }

  if (warp == PC_WARPS + 1) {
    // ------------------------------------------------------------ patch warp
    // Takes every landed tile, and for a brick on the upper periodic
    // boundary fills the vertex planes that lie outside the tensor (they
    // arrive as zeros): plane i = ex holds x = 0, likewise y and z.  Then it
    // releases the tile to the consumers.
    long long fk = 0;
    for (;;) {
      const int fs = (int)(fk % NF);
      if (!warp_wait(&tma_f[fs], (uint32_t)((fk / NF) & 1), flags, lane, wait_limit)) return;
      const Job jb = job[fs];
      if (jb.b < 0) {
        if (lane == 0) mbar_arrive(&full_f[fs]);
        return;
      }
      const int bx = jb.bx, by = jb.by, bz = jb.bz;
      const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
      const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
                ez = brick_extent(g.n[2], bz);
      const bool wx = x0 + ex == g.n[0], wy = y0 + ey == g.n[1], wz = z0 + ez == g.n[2];
      if (jb.cnt > 0 && (wx || wy || wz)) {
        float* ft = reinterpret_cast<float*>(sm + fs * FST);
        constexpr int NP = TILE * TILE, NT = 3 * NP, U = 7;  // U loads in flight per lane
        for (int t0 = lane; t0 < NT; t0 += 32 * U) {
          float val[U][3];
          int dst[U];
#pragma unroll
          for (int u = 0; u < U; u++) {
            dst[u] = -1;
            const int t = t0 + 32 * u;
            if (t >= NT) continue;
            const int pl = t / NP, r = t % NP, p0 = r % TILE, p1 = r / TILE;
            int i, j, k;
            bool on;
            if (pl == 0)
              i = ex, j = p0, k = p1, on = wx;
            else if (pl == 1)
              i = p0, j = ey, k = p1, on = wy;
            else
              i = p0, j = p1, k = ez, on = wz;
            if (!on || i > ex || j > ey || k > ez) continue;
            const int gx = x0 + i < g.n[0] ? x0 + i : 0;
            const int gy = y0 + j < g.n[1] ? y0 + j : 0;
            const int gz = z0 + k < g.n[2] ? z0 + k : 0;
            const int64_t s = site_index(g, gx, gy, gz);
            dst[u] = i + FX * (j + TILE * k);
            val[u][0] = __ldg(F + s);
            val[u][1] = __ldg(F + g.nsites + s);
            val[u][2] = __ldg(F + 2 * g.nsites + s);
          }
#pragma unroll
          for (int u = 0; u < U; u++) {
            if (dst[u] < 0) continue;
            ft[dst[u]] = val[u][0];
            ft[FCOMP + dst[u]] = val[u][1];
            ft[2 * FCOMP + dst[u]] = val[u][2];
          }
        }
        // the buffer is later overwritten by a tile copy (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&full_f[fs]);
      fk++;
    }
  }

  // -------------------------------------------------------------- consumers
  // lattice sizes that are powers of two wrap with the key's bit masks
  const bool pow2 = g.n[0] == (int)g.mask[0] + 1 && g.n[1] == (int)g.mask[1] + 1 &&
                    g.n[2] == (int)g.mask[2] + 1;
  // Each warp takes slots [warp * WSUB, (warp + 1) * WSUB) of every chunk of
  // the brick and works on its own: stayers are written back in place at
  // slots taken from the brick's shared cursor, movers at slots taken from
  // the global mover counter.  The last warp to finish a brick publishes its
  // count and max |v|^2 and hands the tile buffer back.  In-place writes
  // never reach a slot whose chunk has not been copied in: the cursor never
  // exceeds the number of particles of the chunks already in the ring.
  long long fk = 0;
  int cps = 0;          // chunk buffer of the next chunk
  uint32_t cpar = 0;    // parity of its full barrier's phase
  if (stall && !warp_wait(&never, 0u, flags, lane, wait_limit)) return;
  for (;;) {
    const int fs = (int)(fk % NF);
    if (!warp_wait(&full_f[fs], (uint32_t)((fk / NF) & 1), flags, lane, wait_limit)) return;
    const Job jb = job[fs];
    if (jb.b < 0) return;
    const int64_t b = jb.b;
    const int cnt = jb.cnt;
    const float* ft = reinterpret_cast<const float*>(sm + fs * FST);
    const int bx = jb.bx, by = jb.by, bz = jb.bz;
    const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
    // slot indices fit in 32 bits (the store holds fewer than 2^32 slots)
    const uint32_t base32 = (uint32_t)jb.base;
    const uint32_t key0 = pack_key(g, x0, y0, z0);  // a harmless key for empty lanes
    const bool dsplit = DEP && cnt <= dep.split_max;  // fused deposit: split 32-bit sums

    float maxv2 = 0.0f;
    for (int c0 = 0; c0 < cnt; c0 += CHUNK) {
      const int ps = cps;
      if (!warp_wait(&full_p[ps], cpar, flags, lane, wait_limit)) return;
      if (++cps == nst) {
        cps = 0;
        cpar ^= 1u;
      }
      const ChunkView cv = chunk_view(pbuf + (size_t)ps * stage_bytes, has_m, CHUNK);
      const int n = min(CHUNK, cnt - c0);
      const int i0 = warp * WSUB + W_ITEMS * lane;
      uint32_t key[W_ITEMS];
      float ox[W_ITEMS], oy[W_ITEMS], oz[W_ITEMS], vx[W_ITEMS], vy[W_ITEMS], vz[W_ITEMS];
      float m[W_ITEMS];
      int64_t id[W_ITEMS];
      bool act[W_ITEMS];
#pragma unroll
      for (int j = 0; j < W_ITEMS; j++) {
        act[j] = i0 + j < n;
        key[j] = key0;
        ox[j] = oy[j] = oz[j] = vx[j] = vy[j] = vz[j] = m[j] = 0.0f;
        id[j] = 0;
        if (act[j]) {
          key[j] = cv.key[i0 + j];
          ox[j] = cv.ox[i0 + j], oy[j] = cv.oy[i0 + j], oz[j] = cv.oz[i0 + j];
          vx[j] = cv.vx[i0 + j], vy[j] = cv.vy[i0 + j], vz[j] = cv.vz[i0 + j];
          if (has_m) m[j] = cv.m[i0 + j];
          if (has_id) id[j] = cv.id[i0 + j];
        }
      }
      // The buffer is refilled by a bulk copy (async proxy) once every warp
      // has released it: order this warp's reads (generic proxy) before that.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty_p[ps]);  // this warp's slots are read

      bool stay[W_ITEMS];
#pragma unroll
      for (int j = 0; j < W_ITEMS; j++) {
        const int x = (int)(key[j] & g.mask[0]), y = (int)((key[j] >> g.shift[1]) & g.mask[1]),
                  z = (int)((key[j] >> g.shift[2]) & g.mask[2]);
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
        const float v2 = __fadd_rn(__fadd_rn(__fmul_rn(vx[j], vx[j]), __fmul_rn(vy[j], vy[j])),
                                   __fmul_rn(vz[j], vz[j]));
        maxv2 = fmaxf(maxv2, act[j] ? v2 : 0.0f);
        // drift in cell units: o += dtn v, integer part carried into the cell
        const float px = __fmaf_rn(mp.dtn, vx[j], ox[j]), py = __fmaf_rn(mp.dtn, vy[j], oy[j]),
                    pz = __fmaf_rn(mp.dtn, vz[j], oz[j]);
        const bool finite = fabsf(px) <= 3.402823466e38f && fabsf(py) <= 3.402823466e38f &&
                            fabsf(pz) <= 3.402823466e38f;
        const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
        float rx = __fsub_rn(px, fx), ry = __fsub_rn(py, fy), rz = __fsub_rn(pz, fz);
        int kx = (int)fx, ky = (int)fy, kz = (int)fz;
        kx += rx >= 1.0f, ky += ry >= 1.0f, kz += rz >= 1.0f;
        rx = rx >= 1.0f ? 0.0f : rx, ry = ry >= 1.0f ? 0.0f : ry, rz = rz >= 1.0f ? 0.0f : rz;
        int nx, ny, nz;
        if (pow2) {  // the periodic wrap is the key's bit mask
          nx = (x + (finite ? kx : 0)) & (int)g.mask[0];
          ny = (y + (finite ? ky : 0)) & (int)g.mask[1];
          nz = (z + (finite ? kz : 0)) & (int)g.mask[2];
        } else {
          nx = wrap_near(x, finite ? kx : 0, g.n[0]);
          ny = wrap_near(y, finite ? ky : 0, g.n[1]);
          nz = wrap_near(z, finite ? kz : 0, g.n[2]);
        }
        if (finite) {
          ox[j] = rx, oy[j] = ry, oz[j] = rz;
          key[j] = pack_key(g, nx, ny, nz);
        }
        stay[j] = ((nx / BRICK) == bx) & ((ny / BRICK) == by) & ((nz / BRICK) == bz);
        if (!finite && act[j]) set_flag(flags, ERR_NONFINITE);
      }

      // stayers: lane-major order inside the warp, slots from the brick cursor
      const unsigned lt = (1u << lane) - 1u;
      unsigned sb[W_ITEMS], mb[W_ITEMS];
      int ns = 0, nmv = 0, sq = 0, mqo = 0;
#pragma unroll
      for (int j = 0; j < W_ITEMS; j++) {
        sb[j] = __ballot_sync(0xffffffffu, act[j] && stay[j]);
        mb[j] = __ballot_sync(0xffffffffu, act[j] && !stay[j]);
        ns += __popc(sb[j]);
        nmv += __popc(mb[j]);
        sq += __popc(sb[j] & lt);
        mqo += __popc(mb[j] & lt);
      }
      int sbase = 0;
      uint32_t mbase = 0;  // mover slots stay below 2^32 like the store's
      if (lane == 0) {
        if (ns) sbase = atomicAdd(&s_cursor[fs], ns);
        if (nmv) mbase = (uint32_t)atomicAdd(mov_count, (unsigned long long)nmv);
      }
      sq += __shfl_sync(0xffffffffu, sbase, 0);
      uint32_t mq = __shfl_sync(0xffffffffu, mbase, 0) + (uint32_t)mqo;
#pragma unroll
      for (int j = 0; j < W_ITEMS; j++) {
        if (!act[j]) continue;
        if (stay[j]) {
          const uint32_t q = base32 + (uint32_t)sq++;
          v.a.key[q] = key[j];
          v.a.ox[q] = ox[j];
          v.a.oy[q] = oy[j];
          v.a.oz[q] = oz[j];
          v.a.vx[q] = vx[j];
          v.a.vy[q] = vy[j];
          v.a.vz[q] = vz[j];
          if (has_m) v.a.mass[q] = m[j];
          if (has_id) v.a.id[q] = id[j];
          if constexpr (DEP) {
            // the stayer's fixed-point CIC weights at its new position into
            // the brick's tile (the arithmetic of k_deposit, order-free sums)
            int nx, ny, nz;
            unpack_key(g, key[j], nx, ny, nz);
            const int t0 = (nx - x0) + TILE * ((ny - y0) + TILE * (nz - z0));
            const uint64_t mq = has_m ? mass_q(m[j], dep.inv_unit, flags) : 0;
            const uint32_t ux = weight_q(ox[j]), uy = weight_q(oy[j]), uz = weight_q(oz[j]);
            const uint32_t qx[2] = {(1u << 31) - ux, ux};
            const uint32_t qy[2] = {(1u << 31) - uy, uy};
            const uint32_t qz[2] = {(1u << 31) - uz, uz};
#pragma unroll
            for (int k = 0; k < 8; k++) {
              const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
              uint64_t w = fixed_corner(qx[cx], qy[cy], qz[cz]);
              if (has_m) w = (w * mq + (1ull << 23)) >> 24;
              const int t = t0 + cx + cy * TILE + cz * TILE * TILE;
              if (dsplit) {
                atomicAdd(&dtile[t], (uint32_t)(w & 0xffffu));
                atomicAdd(&dtile[TILE3 + t], (uint32_t)(w >> 16));
              } else {
                atomicAdd(reinterpret_cast<unsigned long long*>(dtile) + t, (unsigned long long)w);
              }
            }
          }
        } else {
          const uint32_t q = mq++;
          mov.key[q] = key[j];
          mov.ox[q] = ox[j];
          mov.oy[q] = oy[j];
          mov.oz[q] = oz[j];
          mov.vx[q] = vx[j];
          mov.vy[q] = vy[j];
          mov.vz[q] = vz[j];
          if (has_m) mov.mass[q] = m[j];
          if (has_id) mov.id[q] = id[j];
        }
      }
    }

    for (int o = 16; o > 0; o >>= 1) maxv2 = fmaxf(maxv2, __shfl_xor_sync(0xffffffffu, maxv2, o));
    // likewise for the tile: the next tile copy into this buffer follows
    // this warp's last read of it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) {
      atomicMax(&s_maxv2[fs], __float_as_uint(maxv2));  // non-negative floats order as integers
      __threadfence_block();
      if (atomicAdd(&s_done[fs], 1) == PC_WARPS - 1) {
        __threadfence_block();
        brick_maxv2[b] = __uint_as_float(atomicAdd(&s_maxv2[fs], 0u));
        v.count[b] = atomicAdd(&s_cursor[fs], 0);
        mbar_arrive(&empty_f[fs]);  // every warp is done with this brick
      }
    }
    __syncwarp();
    if constexpr (DEP) {
      // Every consumer warp's deposits of the brick are in the tile once all
      // have arrived; then each flushes a share of the vertices (private ones
      // to the density, the rim to the rim store) and clears them, and the
      // tile is clean for the next brick once all have arrived again.  Both
      // waits are bounded like the others.
      const uint32_t par = (uint32_t)(fk & 1);
      if (lane == 0) mbar_arrive(&dep_in);
      if (!warp_wait(&dep_in, par, flags, lane, wait_limit)) return;
      const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
                ez = brick_extent(g.n[2], bz);
      uint64_t* rs = dep.rim + (size_t)b * RIM;
      unsigned long long* d64 = reinterpret_cast<unsigned long long*>(dtile);
      for (int t = warp * 32 + lane; t < TILE3; t += PC_WARPS * 32) {
        uint64_t q;
        if (dsplit) {
          q = (uint64_t)dtile[t] + ((uint64_t)dtile[TILE3 + t] << 16);
          dtile[t] = 0u;
          dtile[TILE3 + t] = 0u;
        } else {
          q = d64[t];
          d64[t] = 0ull;
        }
        const int i = t % TILE, jj = (t / TILE) % TILE, k = t / (TILE * TILE);
        if (i > ex || jj > ey || k > ez) continue;
        if (i >= 2 && i <= ex - 2 && jj >= 2 && jj <= ey - 2 && k >= 2 && k <= ez - 2) {
          if ((long long)q < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
          dep.rho[site_index(g, x0 + i, y0 + jj, z0 + k)] =
              __fmul_rn(__ll2float_rn((long long)q), dep.scale);
        } else {
          rs[rim_index(rim_canon(i, ex), rim_canon(jj, ey), rim_canon(k, ez))] = q;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&dep_clean);
      if (!warp_wait(&dep_clean, par, flags, lane, wait_limit)) return;
    }
    fk++;
  }
}

// Fused deposit, second half: the movers of the last pass (the mover buffer)
// add their fixed-point CIC weights to the rim store of the brick they moved
// into, with 64-bit atomics (integer sums, so the order does not matter).  A
// mover that moved more than one cell into its brick reaches a private
// vertex there, which the fused pass has already written: it raises `redep`,
// and the whole deposit is then redone by the tile and fix-up kernels.
__global__ void __launch_bounds__(256) k_dep_movers(Geom g, PartArrays mov,
                                                    const unsigned long long* __restrict__ mov_count,
                                                    uint64_t* __restrict__ rim, float inv_unit,
                                                    uint32_t* redep, uint32_t* flags)
{
  const int64_t nm = (int64_t)*mov_count;
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nm;
       m += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    unpack_key(g, mov.key[m], x, y, z);
    if (x >= g.n[0] || y >= g.n[1] || z >= g.n[2]) continue;  // flagged by k_insert
    const int bx = x / BRICK, by = y / BRICK, bz = z / BRICK;
    const int e[3] = {brick_extent(g.n[0], bx), brick_extent(g.n[1], by), brick_extent(g.n[2], bz)};
    const int l[3] = {x - bx * BRICK, y - by * BRICK, z - bz * BRICK};
    const int64_t b = (int64_t)bx + (int64_t)g.nb[0] * ((int64_t)by + (int64_t)g.nb[1] * bz);
    const uint64_t mq = mov.mass ? mass_q(mov.mass[m], inv_unit, flags) : 0;
    const uint32_t ux = weight_q(mov.ox[m]), uy = weight_q(mov.oy[m]), uz = weight_q(mov.oz[m]);
    const uint32_t qx[2] = {(1u << 31) - ux, ux};
    const uint32_t qy[2] = {(1u << 31) - uy, uy};
    const uint32_t qz[2] = {(1u << 31) - uz, uz};
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
      const int u0 = rim_canon(l[0] + cx, e[0]), u1 = rim_canon(l[1] + cy, e[1]),
                u2 = rim_canon(l[2] + cz, e[2]);
      if (!(rim_layer(u0) || rim_layer(u1) || rim_layer(u2))) {
        atomicOr(redep, 1u);
        continue;
      }
      uint64_t w = fixed_corner(qx[cx], qy[cy], qz[cz]);
      if (mov.mass) w = (w * mq + (1ull << 23)) >> 24;
      atomicAdd(reinterpret_cast<unsigned long long*>(rim) + (size_t)b * RIM + rim_index(u0, u1, u2),
                (unsigned long long)w);
    }
  }
}

// Fused deposit, last part: every owned vertex of a brick that movers can
// reach (a coordinate in {0, 1, e-1}) is its own rim value plus, for every
// non-empty subset S of the dims where its coordinate is 0, the rim value of
// the lower neighbour across S at coordinate e' (canonical BRICK) in those
// dims, summed in a fixed order; then converted like the tile pass.
//
// The rim-owned vertices are enumerated directly: with R(e) the coordinates
// {0, 1, e-1} of [0, e) (all of them when e <= 3) and P(e) = [2, e-2] the
// others, they are z in R (any x, y), then z in P with y in R (any x), then
// y, z in P with x in R: 3e^2 + 3e(e-3) + 3(e-3)^2 = 1899 for e = 16.
__device__ __forceinline__ int rim_coord(int r, int e) { return r < 2 ? r : e - 1; }

__global__ void __launch_bounds__(256) k_fixup_rim(Geom g, const uint64_t* __restrict__ rim,
                                                   float scale, float* __restrict__ out,
                                                   uint32_t* flags)
{
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int e[3] = {brick_extent(g.n[0], bx), brick_extent(g.n[1], by), brick_extent(g.n[2], bz)};
  const int bm[3] = {bx ? bx - 1 : g.nb[0] - 1, by ? by - 1 : g.nb[1] - 1, bz ? bz - 1 : g.nb[2] - 1};
  const int bc[3] = {bx, by, bz};
  int nr[3], np[3];
#pragma unroll
  for (int d = 0; d < 3; d++) nr[d] = min(e[d], 3), np[d] = e[d] - nr[d];
  const int n1 = nr[2] * e[1] * e[0];          // z in R
  const int n2 = n1 + np[2] * nr[1] * e[0];    // z in P, y in R
  const int n3 = n2 + np[2] * np[1] * nr[0];   // y, z in P, x in R
  for (int f = threadIdx.x; f < n3; f += blockDim.x) {
    int q[3];
    if (f < n1) {
      q[0] = f % e[0];
      q[1] = (f / e[0]) % e[1];
      q[2] = rim_coord(f / (e[0] * e[1]), e[2]);
    } else if (f < n2) {
      const int r = f - n1;
      q[0] = r % e[0];
      q[1] = rim_coord((r / e[0]) % nr[1], e[1]);
      q[2] = 2 + r / (e[0] * nr[1]);
    } else {
      const int r = f - n2;
      q[0] = rim_coord(r % nr[0], e[0]);
      q[1] = 2 + (r / nr[0]) % np[1];
      q[2] = 2 + r / (nr[0] * np[1]);
    }
    const int zmask = (q[0] == 0 ? 1 : 0) | (q[1] == 0 ? 2 : 0) | (q[2] == 0 ? 4 : 0);
    long long sum = 0;
    for (int s = 0; s < 8; s++) {
      if ((s & zmask) != s) continue;
      int nb3[3], u[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const bool lower = (s >> d) & 1;
        nb3[d] = lower ? bm[d] : bc[d];
        u[d] = lower ? BRICK : rim_canon(q[d], e[d]);
      }
      const int64_t nb = (int64_t)nb3[0] + (int64_t)g.nb[0] * ((int64_t)nb3[1] + (int64_t)g.nb[1] * nb3[2]);
      sum += (long long)rim[(size_t)nb * RIM + rim_index(u[0], u[1], u[2])];
    }
    if (sum < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
    out[site_index(g, bc[0] * BRICK + q[0], bc[1] * BRICK + q[1], bc[2] * BRICK + q[2])] =
        __fmul_rn(__ll2float_rn(sum), scale);
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

#ifndef LF2_PIPE_DEP_WARPS
#define LF2_PIPE_DEP_WARPS 20
#endif
constexpr int DEP_WARPS = LF2_PIPE_DEP_WARPS;  // consumer warps of the fused-deposit kernel
constexpr int STATIC_SMEM = 256;               // the kernel's static shared memory, rounded up

size_t stage_bytes_for(const lf2_ctx* c, int warps)
{
  return (size_t)warps * WSUB * (28 + (c->has_mass ? 4 : 0) + (c->has_id ? 8 : 0));
}

// Chunk buffers that fit beside the vertex tiles (and the deposit tile).
int stages_for(const lf2_ctx* c, bool dep)
{
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  const size_t sb = stage_bytes_for(c, dep ? DEP_WARPS : LF2_PIPE_WARPS);
  const size_t fixed = dep ? 128 + NF * (size_t)FSTRIDE_DEP + DEP_BYTES + STATIC_SMEM
                           : 1024 + NF * (size_t)FSTRIDE + 2048;
  int nst = (int)(((size_t)optin > fixed ? (size_t)optin - fixed : 0) / sb);
  return nst > MAX_STAGES ? MAX_STAGES : nst;
}

}  // namespace

size_t rim_store_slots(const lf2_ctx* c) { return (size_t)c->g.nbricks * RIM; }

// Whether lf2_step can fuse the fixed-point scalar deposit into the
// pipelined pass: the deposit tile and two chunk buffers must fit.
bool move_dep_eligible(const lf2_ctx* c, const float* F)
{
  return move_pipe_eligible(c, F) && c->mode == LF2_DEPOSIT_FIXED64 && stages_for(c, true) >= 2;
}

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

cudaError_t launch_move_pipe(lf2_ctx* c, const float* F, MoveParams mp, float* rho)
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
  const bool dep = rho != nullptr;
  const int warps = dep ? DEP_WARPS : LF2_PIPE_WARPS;
  const size_t sb = stage_bytes_for(c, warps);
  const int nst = stages_for(c, dep);
  if (nst < 2) return cudaErrorInvalidConfiguration;
  const size_t smem = dep ? 128 + NF * (size_t)FSTRIDE_DEP + DEP_BYTES + (size_t)nst * sb
                          : 1024 + NF * (size_t)FSTRIDE + (size_t)nst * sb;
  DepOut d{};
  if (dep) {
    const double vol = c->res * c->res * c->res;
    d.rho = rho;
    d.rim = c->spill;
    d.scale = (float)(std::ldexp(1.0, -32) * c->m_unit / vol);
    d.inv_unit = (float)(1.0 / c->m_unit);
    d.split_max = split_max<false>(c->has_mass);
  }
  using Kern = decltype(&k_move_pipe<LF2_PIPE_WARPS, false, false, false>);
  const Kern kerns[2][4] = {
      {k_move_pipe<LF2_PIPE_WARPS, false, false, false>, k_move_pipe<LF2_PIPE_WARPS, false, true, false>,
       k_move_pipe<LF2_PIPE_WARPS, false, false, true>, k_move_pipe<LF2_PIPE_WARPS, false, true, true>},
      {k_move_pipe<DEP_WARPS, true, false, false>, k_move_pipe<DEP_WARPS, true, true, false>,
       k_move_pipe<DEP_WARPS, true, false, true>, k_move_pipe<DEP_WARPS, true, true, true>}};
  const Kern kern = kerns[dep ? 1 : 0][(c->has_mass ? 1 : 0) + (c->has_id ? 2 : 0)];
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(c->work, 0, sizeof(int), c->stream);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  kern<<<c->num_sms, warps * 32 + 64, smem, c->stream>>>(
      *map, view(c), F, mp, c->mov, c->mov_count, c->brick_maxv2, c->flags, c->work, nst, (int)sb,
      c->wait_cycles > 0 ? (long long)c->wait_cycles : WAIT_CYCLES, c->wait_stall, d);
  return cudaGetLastError();
}

// The movers' part and the rim fix-up of the fused deposit (after the fused
// pass; `redep` cleared before it).
cudaError_t launch_dep_movers(lf2_ctx* c)
{
  c->launches += 1;
  k_dep_movers<<<c->num_sms * 4, 256, 0, c->stream>>>(c->g, c->mov, c->mov_count, c->spill,
                                                      (float)(1.0 / c->m_unit), c->redep, c->flags);
  return cudaGetLastError();
}

cudaError_t launch_fixup_rim(lf2_ctx* c, float* rho)
{
  const double vol = c->res * c->res * c->res;
  c->launches += 1;
  k_fixup_rim<<<(unsigned)c->g.nbricks, 256, 0, c->stream>>>(
      c->g, c->spill, (float)(std::ldexp(1.0, -32) * c->m_unit / vol), rho, c->flags);
  return cudaGetLastError();
}

}  // namespace lf2
