// lf2_deposit.cu -- CIC deposits of the brick-binned particles.
//
//   kind 0  scalar CIC        scalarProjectionCIC_project/_comm
//                             (projections.hpp:75-300)
//   kind 1  vector CIC-NGP    vectorProjectionCICNGP_project/_comm (:421-681)
//   kind 2  symtensor CIC-NGP symtensorProjectionCICNGP_project/_comm (:708-976)
//
// One CTA per brick accumulates its particles into a shared-memory tile of the
// (BRICK+1)^3 vertices they touch, then writes the tile once:
//   - vertices with every coordinate in [1, e-1] receive contributions from
//     this brick only, so their final value goes straight to the field;
//   - the other tile vertices (the "shell": a coordinate equal to 0 or to the
//     brick extent e) are written to a per-brick shell store.
// k_fixup then finishes every owned vertex with a zero coordinate by summing
// the shell values of the up to 8 bricks that touch it, in a fixed order.
// The periodic upper-halo fold of the reference's *_comm functions is thus
// part of the deposit, every vertex is written exactly once and no global
// atomics are used.
//
// Three accumulation modes (the context's deposit mode):
//   LF2_DEPOSIT_FP32        FP32 shared atomics with compensation: each add
//                           returns the value it replaced, the rounding error
//                           of that add is recovered exactly (TwoSum) and
//                           accumulated in a second FP32 word.  hi + lo is the
//                           sum to within the rounding of the terms (about
//                           1e-7 relative), whatever the order.
//   LF2_DEPOSIT_FIXED64     int64 fixed point: every contribution is rounded
//                           once, deterministically, to an integer quantum;
//                           the integer sums do not depend on the order, so
//                           the result is bit-exact run to run.  Scalar: 2^-32
//                           of a unit mass.  Momentum and stress are signed:
//                           2^-32 of a unit mass times V (momentum) or V^2
//                           (stress), V the smallest power of two above every
//                           |v_i| of the particles (found on the device before
//                           the deposit, k_vmax).
//   LF2_DEPOSIT_FP32_PLAIN  FP32 shared atomics without compensation: the
//                           speed reference; its sums in dense vertices carry
//                           the rounding of unordered FP32 additions.
#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>

#include "lf2_deposit_common.cuh"
#include "lf2_internal.h"

// Owned face vertices per thread and trip of the one-component fix-up.
#ifndef FIX_V
#define FIX_V 2
#endif

namespace lf2 {

namespace {

#ifndef LF2_DEP_THREADS
#define LF2_DEP_THREADS 256
#endif
constexpr int DEP_THREADS = LF2_DEP_THREADS;

// Components of the field of a kind.
template <int KIND>
struct Comps { static constexpr int value = KIND == 0 ? 1 : KIND == 1 ? 3 : 6; };

// A tile pass accumulates NC components of the field.  The plain mode keeps
// one 32-bit word per vertex and component and does every kind in one pass
// (the tensor's six components in a 118 KB tile); the compensated and the
// fixed-point modes keep two words, so the tensor takes two passes of three
// components (T_00, T_11, T_22 at the vertices, then T_01, T_02, T_12 on the
// plaquettes), each with a 118 KB tile.
template <int KIND, int PASS, int ACC>
struct Pass {
  static constexpr int NC = KIND == 0 ? 1 : KIND == 1 ? 3 : (ACC == ACC_PLAIN ? 6 : 3);
  static constexpr int WORDS = ACC == ACC_PLAIN ? 1 : 2;
  // field component of pass-local component j
  __host__ __device__ static constexpr int comp(int j)
  {
    return KIND != 2 || ACC == ACC_PLAIN ? j
           : PASS == 0                   ? (j == 0 ? 0 : j == 1 ? 3 : 5)
                                         : (j == 0 ? 1 : j == 1 ? 2 : 4);
  }
  static constexpr size_t smem() { return (size_t)NC * WORDS * TILE3 * 4; }
  // threads per CTA: a tile above 100 KB leaves room for one CTA per SM, so
  // it gets twice the warps
  static constexpr int THREADS = smem() > 100 * 1024 ? 2 * DEP_THREADS : DEP_THREADS;
};

__device__ __forceinline__ float sel(int b, float up, float dn) { return b ? up : dn; }

// ------------------------------------------------------------- tile pass
template <int KIND, int PASS, int ACC>
__global__ void __launch_bounds__(Pass<KIND, PASS, ACC>::THREADS) k_deposit(StoreView v, DepositParams dp,
                                                         float* __restrict__ out,
                                                         uint64_t* __restrict__ spill,
                                                         const uint32_t* __restrict__ vmax_bits,
                                                         uint32_t* flags, const uint32_t* gate)
{
  // gate: run only when the word is set (the redo of a fused deposit)
  if (gate && *gate == 0u) return;
  using P = Pass<KIND, PASS, ACC>;
  constexpr int NC = P::NC;
  constexpr int C = Comps<KIND>::value;
  constexpr bool FIXED = ACC == ACC_FIXED;
  constexpr bool SIGNED = KIND != 0;
  constexpr int T = P::THREADS;
  extern __shared__ __align__(16) unsigned char smem_raw[];

  const Geom& g = v.g;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
            ez = brick_extent(g.n[2], bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  TileRef<TILE3> tr{smem_raw, FIXED && cnt <= split_max<SIGNED>(dp.has_mass != 0)};
  // fixed point: velocity quantum and conversion scale for this field
  int vexp = 0;
  if (FIXED && KIND != 0) vexp = vexp_of(*vmax_bits);
  const float vscale = vel_scale(vexp);
  const float conv =
      FIXED ? ldexpf(dp.fixed_scale, (KIND == 1 ? vexp : 2 * vexp) - (KIND != 0 ? 16 : 0)) : 0.0f;
  if (FIXED && threadIdx.x == 0 && b == 0 && !(conv > 0.0f && conv <= 3.402823466e38f))
    set_flag(flags, ERR_FIXED_OVERFLOW);  // V^p / res^3 outside the FP32 range

  {
    uint32_t* z = reinterpret_cast<uint32_t*>(smem_raw);
    constexpr int words = NC * P::WORDS * TILE3;
    for (int t = threadIdx.x; t < words; t += blockDim.x) z[t] = 0u;
  }
  __syncthreads();

  // The particle loop, instantiated for the split fixed-point tile (or not)
  // and for per-particle masses (or a global mass), chosen once per CTA.
  constexpr int ITEMS = 4;  // particles in flight per thread
  auto particles = [&](auto split_c, auto hm_c) {
    constexpr bool SPLIT = decltype(split_c)::value;
    constexpr bool HM = decltype(hm_c)::value;
    for (int c0 = 0; c0 < cnt; c0 += ITEMS * T) {
      uint32_t key[ITEMS];
      float fx[ITEMS], fy[ITEMS], fz[ITEMS], m[ITEMS];
      float vx[ITEMS], vy[ITEMS], vz[ITEMS];
  #pragma unroll
      for (int j = 0; j < ITEMS; j++) {
        const int i = c0 + j * T + threadIdx.x;
        if (i < cnt) {
          const uint32_t p = (uint32_t)base + (uint32_t)i;  // slots fit in 32 bits
          key[j] = v.a.key[p];
          fx[j] = v.a.ox[p];
          fy[j] = v.a.oy[p];
          fz[j] = v.a.oz[p];
          m[j] = HM ? v.a.mass[p] : 0.0f;
          if (KIND != 0) {
            vx[j] = v.a.vx[p];
            vy[j] = v.a.vy[p];
            vz[j] = v.a.vz[p];
          }
        }
      }
  #pragma unroll
      for (int j = 0; j < ITEMS; j++) {
        const int i = c0 + j * T + threadIdx.x;
        if (i >= cnt) continue;
        int x, y, z;
        unpack_key(g, key[j], x, y, z);
        const int t0 = (x - x0) + TILE * ((y - y0) + TILE * (z - z0));
        constexpr int TY = TILE, TZ = TILE * TILE;
        if (FIXED) {
          uint64_t mq = 0;
          if (HM) mq = mass_q(m[j], dp.inv_unit, flags);
          // 1-D weights in units of 2^-31 (lf2o_fixed_weight in the oracle)
          const uint32_t ux = weight_q(fx[j]), uy = weight_q(fy[j]), uz = weight_q(fz[j]);
          const uint32_t qx[2] = {(1u << 31) - ux, ux};
          const uint32_t qy[2] = {(1u << 31) - uy, uy};
          const uint32_t qz[2] = {(1u << 31) - uz, uz};
          constexpr uint32_t ONE = 1u << 31;
          if (KIND == 0) {
            const uint64_t pxy[4] = {(uint64_t)qx[0] * qy[0], (uint64_t)qx[0] * qy[1],
                                     (uint64_t)qx[1] * qy[0], (uint64_t)qx[1] * qy[1]};
  #pragma unroll
            for (int k = 0; k < 8; k++) {
              const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
              const int t = t0 + cx + cy * TY + cz * TZ;
              if (SPLIT && !HM) {
                add_corner_split<TILE3>(reinterpret_cast<uint32_t*>(smem_raw), t, pxy[cx * 2 + cy], qz[cz]);
              } else {
                const uint64_t q = fixed_corner(qx[cx], qy[cy], qz[cz]);
                add_fixed_t<SPLIT, TILE3>(smem_raw, 0, t, mass_sign_t<HM>(q, mq, false));
              }
            }
          } else if (KIND == 1) {
            // projections.hpp:501-544: component i is NGP along i, CIC across
            const float vv[3] = {vx[j], vy[j], vz[j]};
  #pragma unroll
            for (int c = 0; c < 3; c++) {
              const uint32_t vq = vel_q(vv[c], vscale);
              const bool neg = vv[c] < 0.0f;
  #pragma unroll
              for (int k = 0; k < 4; k++) {
                const int a = (k >> 1) & 1, bb = k & 1;
                uint64_t w;
                int t;
                if (c == 0) w = fixed_corner(ONE, qy[a], qz[bb]), t = t0 + a * TY + bb * TZ;
                else if (c == 1) w = fixed_corner(qx[a], ONE, qz[bb]), t = t0 + a + bb * TZ;
                else w = fixed_corner(qx[a], qy[bb], ONE), t = t0 + a + bb * TY;
                add_fixed48_t<SPLIT, TILE3>(smem_raw, c, t, mass_sign48_t<HM>(mul_wv48(w, vq), mq, neg));
              }
            }
          } else if (PASS == 0) {
            // projections.hpp:788-807: T_ii = m v_i^2 at the 8 vertices
            const float vv[3] = {vx[j], vy[j], vz[j]};
            double f2[3];  // v_d^2 2^-46 (times the relative mass), FP64
  #pragma unroll
            for (int d = 0; d < 3; d++) {
              const uint32_t q = vel_q(vv[d], vscale);
              f2[d] = stress_factor<HM>(q, q, 0x1p-46, mq);  // 2^-46
            }
  #pragma unroll
            for (int k = 0; k < 8; k++) {
              const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
              const uint64_t w = fixed_corner(qx[cx], qy[cy], qz[cz]);
              const int t = t0 + cx + cy * TY + cz * TZ;
  #pragma unroll
              for (int d = 0; d < 3; d++) add_fixed48_t<SPLIT, TILE3>(smem_raw, d, t, stress_q(w, f2[d], false));
            }
          } else {
            // projections.hpp:809-821: T_ij on the (i,j) plaquette, CIC along
            // the third dim
            const float vv[3] = {vx[j], vy[j], vz[j]};
            const uint32_t q0 = vel_q(vv[0], vscale), q1 = vel_q(vv[1], vscale), q2 = vel_q(vv[2], vscale);
            // velocity products times 2^-45 (FP64): a 1-D weight in 2^-31
            // units times one of them is in 2^-48 V^2 units
            const double v01 = stress_factor<HM>(q0, q1, 0x1p-45, mq),
                         v02 = stress_factor<HM>(q0, q2, 0x1p-45, mq),
                         v12 = stress_factor<HM>(q1, q2, 0x1p-45, mq);
            const bool n01 = (vv[0] < 0.0f) != (vv[1] < 0.0f), n02 = (vv[0] < 0.0f) != (vv[2] < 0.0f),
                       n12 = (vv[1] < 0.0f) != (vv[2] < 0.0f);
            add_fixed48_t<SPLIT, TILE3>(smem_raw, 0, t0, stress_q(qz[0], v01, n01));
            add_fixed48_t<SPLIT, TILE3>(smem_raw, 0, t0 + TZ, stress_q(qz[1], v01, n01));
            add_fixed48_t<SPLIT, TILE3>(smem_raw, 1, t0, stress_q(qy[0], v02, n02));
            add_fixed48_t<SPLIT, TILE3>(smem_raw, 1, t0 + TY, stress_q(qy[1], v02, n02));
            add_fixed48_t<SPLIT, TILE3>(smem_raw, 2, t0, stress_q(qx[0], v12, n12));
            add_fixed48_t<SPLIT, TILE3>(smem_raw, 2, t0 + 1, stress_q(qx[1], v12, n12));
          }
          continue;
        }
        // FP32 modes: the arithmetic of the reference's projections in FP32
        const float gx = __fsub_rn(1.0f, fx[j]), gy = __fsub_rn(1.0f, fy[j]),
                    gz = __fsub_rn(1.0f, fz[j]);
        const float ox = fx[j], oy = fy[j], oz = fz[j];
        const float mf = HM ? __fmul_rn(m[j], dp.inv_vol) : dp.mf;
        if (KIND == 0) {
  #pragma unroll
          for (int k = 0; k < 8; k++) {
            const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
            const float w = __fmul_rn(
                __fmul_rn(__fmul_rn(sel(cx, ox, gx), sel(cy, oy, gy)), sel(cz, oz, gz)), mf);
            add_float<ACC>(tr, 0, t0 + cx + cy * TY + cz * TZ, w);
          }
        } else if (KIND == 1) {
          // projections.hpp:501-544: component i is NGP along i, CIC across.
          const float vxm = __fmul_rn(mf, vx[j]);
          const float vym = __fmul_rn(mf, vy[j]);
          const float vzm = __fmul_rn(mf, vz[j]);
          add_float<ACC>(tr, 0, t0, __fmul_rn(__fmul_rn(vxm, gy), gz));
          add_float<ACC>(tr, 0, t0 + TY, __fmul_rn(__fmul_rn(vxm, oy), gz));
          add_float<ACC>(tr, 0, t0 + TZ, __fmul_rn(__fmul_rn(vxm, gy), oz));
          add_float<ACC>(tr, 0, t0 + TY + TZ, __fmul_rn(__fmul_rn(vxm, oy), oz));
          add_float<ACC>(tr, 1, t0, __fmul_rn(__fmul_rn(vym, gx), gz));
          add_float<ACC>(tr, 1, t0 + 1, __fmul_rn(__fmul_rn(vym, ox), gz));
          add_float<ACC>(tr, 1, t0 + TZ, __fmul_rn(__fmul_rn(vym, gx), oz));
          add_float<ACC>(tr, 1, t0 + 1 + TZ, __fmul_rn(__fmul_rn(vym, ox), oz));
          add_float<ACC>(tr, 2, t0, __fmul_rn(__fmul_rn(vzm, gx), gy));
          add_float<ACC>(tr, 2, t0 + 1, __fmul_rn(__fmul_rn(vzm, ox), gy));
          add_float<ACC>(tr, 2, t0 + TY, __fmul_rn(__fmul_rn(vzm, gx), oy));
          add_float<ACC>(tr, 2, t0 + 1 + TY, __fmul_rn(__fmul_rn(vzm, ox), oy));
        } else {
          // projections.hpp:786-843: T_ii at the 8 vertices, T_ij on plaquettes.
          const float vv[3] = {vx[j], vy[j], vz[j]};
          constexpr bool DIAG = ACC == ACC_PLAIN || PASS == 0;
          constexpr bool OFF = ACC == ACC_PLAIN || PASS == 1;
          if (DIAG) {
  #pragma unroll
            for (int d = 0; d < 3; d++) {
              // pass-local component of T_dd: 0, 3, 5 in the six-component
              // plain tile, 0, 1, 2 in the diagonal pass
              const int jd = ACC == ACC_PLAIN ? (d == 0 ? 0 : d == 1 ? 3 : 5) : d;
              const float mv2 = __fmul_rn(__fmul_rn(mf, vv[d]), vv[d]);
  #pragma unroll
              for (int k = 0; k < 8; k++) {
                const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
                const float w = __fmul_rn(
                    __fmul_rn(__fmul_rn(mv2, sel(cx, ox, gx)), sel(cy, oy, gy)), sel(cz, oz, gz));
                add_float<ACC>(tr, jd, t0 + cx + cy * TY + cz * TZ, w);
              }
            }
          }
          if (OFF) {
            const int j01 = ACC == ACC_PLAIN ? 1 : 0, j02 = ACC == ACC_PLAIN ? 2 : 1,
                      j12 = ACC == ACC_PLAIN ? 4 : 2;
            const float m01 = __fmul_rn(__fmul_rn(mf, vv[0]), vv[1]);
            const float m02 = __fmul_rn(__fmul_rn(mf, vv[0]), vv[2]);
            const float m12 = __fmul_rn(__fmul_rn(mf, vv[1]), vv[2]);
            add_float<ACC>(tr, j01, t0, __fmul_rn(m01, gz));
            add_float<ACC>(tr, j01, t0 + TZ, __fmul_rn(m01, oz));
            add_float<ACC>(tr, j02, t0, __fmul_rn(m02, gy));
            add_float<ACC>(tr, j02, t0 + TY, __fmul_rn(m02, oy));
            add_float<ACC>(tr, j12, t0, __fmul_rn(m12, gx));
            add_float<ACC>(tr, j12, t0 + 1, __fmul_rn(m12, ox));
          }
        }
      }
    }
  };
  const bool hm_rt = dp.has_mass != 0;
  if (FIXED && tr.split) {
    if (hm_rt) particles(std::true_type{}, std::true_type{});
    else particles(std::true_type{}, std::false_type{});
  } else {
    if (hm_rt) particles(std::false_type{}, std::true_type{});
    else particles(std::false_type{}, std::false_type{});
  }
  __syncthreads();

  // Flush: interior vertices to the field, shell vertices to the shell store
  // (8-byte slots: the integer sum, hi and lo, or the plain float).  Two
  // loops with constant divisors: the interior [1, e-1]^3 (walked as 15^3,
  // skipping what lies beyond the extents), and the shell slots in their
  // storage order (shell_index), so that those writes are contiguous.
  uint64_t* sp = spill + (size_t)b * C * SHELL;
  const float* facc = reinterpret_cast<const float*>(smem_raw);
  const int64_t site0 = site_index(g, x0, y0, z0);
  const int64_t sy = g.n[0], sz = (int64_t)g.n[0] * g.n[1];
  constexpr int I = BRICK - 1;
  for (int u = threadIdx.x; u < I * I * I; u += blockDim.x) {
    const int i = 1 + u % I, jj = 1 + (u / I) % I, k = 1 + u / (I * I);
    if (i >= ex || jj >= ey || k >= ez) continue;
    const int t = i + TILE * (jj + TILE * k);
    const int64_t s = site0 + i + sy * jj + sz * k;
#pragma unroll
    for (int j = 0; j < NC; j++) {
      const int c = P::comp(j);
      if (FIXED) {
        const long long q = tile_fixed<SIGNED>(tr, j, t);
        if (!SIGNED && q < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
        out[(size_t)c * g.nsites + s] = __fmul_rn(__ll2float_rn(q), conv);
      } else if (ACC == ACC_COMP) {
        out[(size_t)c * g.nsites + s] =
            __fadd_rn(facc[(size_t)j * 2 * TILE3 + t], facc[(size_t)j * 2 * TILE3 + TILE3 + t]);
      } else {
        out[(size_t)c * g.nsites + s] = facc[(size_t)j * TILE3 + t];
      }
    }
  }
  // canonical shell coordinate (0, 1..BRICK-1 or BRICK) -> tile coordinate,
  // or -1 where the brick's extent e leaves it out
  auto tile_of = [](int cc, int e) { return cc == BRICK ? e : (cc == 0 || cc < e ? cc : -1); };
  for (int f = threadIdx.x; f < SHELL; f += blockDim.x) {
    int ci, cj, ck;
    if (f < 2 * TILE * TILE) {  // x faces: slot (i == BRICK) TILE^2 + k TILE + j
      ci = f < TILE * TILE ? 0 : BRICK;
      const int r = f % (TILE * TILE);
      ck = r / TILE, cj = r % TILE;
    } else if (f < 2 * TILE * TILE + 2 * I * TILE) {  // y faces: + (j == BRICK) I TILE + k I + i - 1
      const int r = f - 2 * TILE * TILE;
      cj = r < I * TILE ? 0 : BRICK;
      const int r2 = r % (I * TILE);
      ck = r2 / I, ci = 1 + r2 % I;
    } else {  // z faces: + (k == BRICK) I^2 + (j - 1) I + i - 1
      const int r = f - 2 * TILE * TILE - 2 * I * TILE;
      ck = r < I * I ? 0 : BRICK;
      const int r2 = r % (I * I);
      cj = 1 + r2 / I, ci = 1 + r2 % I;
    }
    const int i = tile_of(ci, ex), jj = tile_of(cj, ey), k = tile_of(ck, ez);
    if (i < 0 || jj < 0 || k < 0) continue;
    const int t = i + TILE * (jj + TILE * k);
#pragma unroll
    for (int j = 0; j < NC; j++) {
      const int c = P::comp(j);
      if (FIXED) {
        sp[(size_t)c * SHELL + f] = (uint64_t)tile_fixed<SIGNED>(tr, j, t);
      } else if (ACC == ACC_COMP) {
        reinterpret_cast<float2*>(sp)[(size_t)c * SHELL + f] =
            make_float2(facc[(size_t)j * 2 * TILE3 + t], facc[(size_t)j * 2 * TILE3 + TILE3 + t]);
      } else {
        reinterpret_cast<float*>(sp)[(size_t)c * SHELL + f] = facc[(size_t)j * TILE3 + t];
      }
    }
  }
}

// One CTA per brick: every owned vertex with a zero coordinate sums the shell
// values of the bricks that touch it: its own tile (subset 0) and, for every
// non-empty subset S of the dims where its coordinate is 0, the lower
// neighbour brick across S at tile coordinate BRICK in those dims.  The sum
// runs in that fixed order: exact integers (fixed point), a compensated FP32
// sum of the hi and lo words, or plain FP32 additions.
template <int KIND, int ACC>
__global__ void k_fixup(Geom g, const uint64_t* __restrict__ spill, float fixed_scale,
                        const uint32_t* __restrict__ vmax_bits, float* __restrict__ out,
                        uint32_t* flags, const uint32_t* gate)
{
  if (gate && *gate == 0u) return;
  constexpr int C = Comps<KIND>::value;
  constexpr bool SIGNED = KIND != 0;
  const int64_t b = blockIdx.x;
  int bx, by, bz;
  brick_coords(g, b, bx, by, bz);
  const int ex = brick_extent(g.n[0], bx), ey = brick_extent(g.n[1], by),
            ez = brick_extent(g.n[2], bz);
  const int x0 = bx * BRICK, y0 = by * BRICK, z0 = bz * BRICK;
  const int bxm = bx ? bx - 1 : g.nb[0] - 1;
  const int bym = by ? by - 1 : g.nb[1] - 1;
  const int bzm = bz ? bz - 1 : g.nb[2] - 1;
  // the brick itself (s = 0) and its lower neighbours across every subset s
  // of the dims (bit 0: x, 1: y, 2: z)
  __shared__ uint32_t nbr[8];
  if (threadIdx.x < 8) {
    const int s = threadIdx.x;
    nbr[s] = (uint32_t)((s & 1) ? bxm : bx) +
             (uint32_t)g.nb[0] * ((uint32_t)((s & 2) ? bym : by) + (uint32_t)g.nb[1] * ((s & 4) ? bzm : bz));
  }
  __syncthreads();
  float conv = 0.0f;
  if (ACC == ACC_FIXED) {
    const int vexp = KIND != 0 ? vexp_of(*vmax_bits) : 0;
    conv = ldexpf(fixed_scale, KIND == 0 ? 0 : (KIND == 1 ? vexp : 2 * vexp) - 16);
  }
  const int nface = ey * ez + (ex - 1) * ez + (ex - 1) * (ey - 1);
  // owned face vertex number f -> tile coordinates
  auto face_vertex = [&](int f, int& i, int& j, int& k) {
    if (f < ey * ez) {  // x face: i = 0
      i = 0;
      j = f % ey;
      k = f / ey;
    } else if (f < ey * ez + (ex - 1) * ez) {  // y face: j = 0, i >= 1
      const int r = f - ey * ez;
      j = 0;
      i = 1 + r % (ex - 1);
      k = r / (ex - 1);
    } else {  // z face: k = 0, i, j >= 1
      const int r = f - ey * ez - (ex - 1) * ez;
      k = 0;
      i = 1 + r % (ex - 1);
      j = 1 + r / (ex - 1);
    }
  };
  if constexpr (C == 1) {
    // One component: FIX_V vertices per thread, all their shell reads issued
    // before any is used (the pass is bound by the latency of these
    // scattered reads; at 512^3, 2 per thread: 0.261 ms, 3: 0.287 ms, 4:
    // 0.345 ms).  Subset s of a vertex's zero coordinates is read
    // when (s & zmask) == s; the sum runs over s in ascending order.
    constexpr int FV = FIX_V;
    const float* spf = reinterpret_cast<const float*>(spill);
    for (int f0 = threadIdx.x; f0 < nface; f0 += FV * blockDim.x) {
      int vi[FV], vj[FV], vk[FV], zm[FV];
      bool on[FV];
#pragma unroll
      for (int h = 0; h < FV; h++) {
        const int f = f0 + h * blockDim.x;
        on[h] = f < nface;
        vi[h] = vj[h] = vk[h] = 0;
        if (on[h]) face_vertex(f, vi[h], vj[h], vk[h]);
        zm[h] = on[h] ? (vi[h] == 0 ? 1 : 0) | (vj[h] == 0 ? 2 : 0) | (vk[h] == 0 ? 4 : 0) : 0;
      }
      long long q[FV];
      float fs[FV], fc[FV];
#pragma unroll
      for (int h = 0; h < FV; h++) q[h] = 0, fs[h] = 0.0f, fc[h] = 0.0f;
      auto read = [&](int h, int s) -> uint64_t {
        const int si = shell_index((s & 1) ? BRICK : vi[h], (s & 2) ? BRICK : vj[h], (s & 4) ? BRICK : vk[h]);
        // a brick's shell region is SHELL 8-byte slots; the plain mode
        // fills its first SHELL floats
        const size_t at = (size_t)nbr[s] * SHELL;
        return ACC == ACC_PLAIN ? (uint64_t)__float_as_uint(spf[2 * at + si]) : spill[at + si];
      };
#pragma unroll
      for (int s = 0; s < 8; s++) {
        uint64_t r[FV];
#pragma unroll
        for (int h = 0; h < FV; h++) r[h] = on[h] && (s & zm[h]) == s ? read(h, s) : 0ull;
#pragma unroll
        for (int h = 0; h < FV; h++) {
          if (!(on[h] && (s & zm[h]) == s)) continue;
          if (ACC == ACC_FIXED)
            q[h] += (long long)r[h];
          else if (ACC == ACC_COMP)
            comp_acc(fs[h], fc[h], __uint_as_float((uint32_t)r[h]), __uint_as_float((uint32_t)(r[h] >> 32)));
          else
            fs[h] = __fadd_rn(fs[h], __uint_as_float((uint32_t)r[h]));
        }
      }
#pragma unroll
      for (int h = 0; h < FV; h++) {
        if (!on[h]) continue;
        const int64_t site = site_index(g, x0 + vi[h], y0 + vj[h], z0 + vk[h]);
        if (ACC == ACC_FIXED) {
          if (!SIGNED && q[h] < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
          out[site] = __fmul_rn(__ll2float_rn(q[h]), conv);
        } else {
          out[site] = ACC == ACC_COMP ? __fadd_rn(fs[h], fc[h]) : fs[h];
        }
      }
    }
  } else {
    for (int f = threadIdx.x; f < nface; f += blockDim.x) {
      int i, j, k;
      face_vertex(f, i, j, k);
      const int zmask = (i == 0 ? 1 : 0) | (j == 0 ? 2 : 0) | (k == 0 ? 4 : 0);
      long long qs[C];
      float fs[C], fc[C];
  #pragma unroll
      for (int c = 0; c < C; c++) {
        qs[c] = 0;
        fs[c] = 0.0f;
        fc[c] = 0.0f;
      }
      // the subsets s of zmask in ascending order (s -> (s - zmask) & zmask)
      for (int s = 0;; s = (s - zmask) & zmask) {
        const uint32_t nb = nbr[s];
        const int si = shell_index((s & 1) ? BRICK : i, (s & 2) ? BRICK : j, (s & 4) ? BRICK : k);
        const uint64_t* sp = spill + (size_t)nb * (C * SHELL);
  #pragma unroll
        for (int c = 0; c < C; c++) {
          if (ACC == ACC_FIXED) {
            qs[c] += (long long)sp[c * SHELL + si];
          } else if (ACC == ACC_COMP) {
            const float2 hl = reinterpret_cast<const float2*>(sp)[c * SHELL + si];
            comp_acc(fs[c], fc[c], hl.x, hl.y);
          } else {
            fs[c] = __fadd_rn(fs[c], reinterpret_cast<const float*>(sp)[c * SHELL + si]);
          }
        }
        if (s == zmask) break;
      }
      const int64_t site = site_index(g, x0 + i, y0 + j, z0 + k);
  #pragma unroll
      for (int c = 0; c < C; c++) {
        if (ACC == ACC_FIXED) {
          if (!SIGNED && qs[c] < 0) set_flag(flags, ERR_FIXED_OVERFLOW);
          out[c * g.nsites + site] = __fmul_rn(__ll2float_rn(qs[c]), conv);
        } else if (ACC == ACC_COMP) {
          out[c * g.nsites + site] = __fadd_rn(fs[c], fc[c]);
        } else {
          out[c * g.nsites + site] = fs[c];
        }
      }
    }
  }
}

// Largest |v_i| of the stored particles, as the bits of a non-negative float
// (they order as unsigned integers); a non-finite velocity raises the flag.
__global__ void __launch_bounds__(256) k_vmax(StoreView v, uint32_t* vmax_bits, uint32_t* flags)
{
  const int64_t b = blockIdx.x;
  const int64_t base = v.seg_start[b];
  const int cnt = LF2_BRICK_COUNT(v, b);
  uint32_t m = 0u;
  bool bad = false;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int64_t p = base + i;
    const uint32_t a = __float_as_uint(v.a.vx[p]) & 0x7fffffffu;
    const uint32_t c = __float_as_uint(v.a.vy[p]) & 0x7fffffffu;
    const uint32_t d = __float_as_uint(v.a.vz[p]) & 0x7fffffffu;
    const uint32_t mm = max(a, max(c, d));
    bad |= mm >= 0x7f800000u;
    m = max(m, mm);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) set_flag(flags, ERR_NONFINITE);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(vmax_bits, m);
}

template <int KIND, int PASS, int ACC>
cudaError_t tile_pass(lf2_ctx* c, float* out, const DepositParams& dp, const uint32_t* gate)
{
  using P = Pass<KIND, PASS, ACC>;
  const size_t smem = P::smem();
  cudaError_t e = cudaFuncSetAttribute(k_deposit<KIND, PASS, ACC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_deposit<KIND, PASS, ACC><<<(unsigned)c->g.nbricks, P::THREADS, smem, c->stream>>>(
      view(c), dp, out, c->spill, c->vmax_bits, c->flags, gate);
  return cudaGetLastError();
}

template <int KIND, int ACC>
cudaError_t run(lf2_ctx* c, float* out, const DepositParams& dp, int stage, const uint32_t* gate)
{
  const unsigned nb = (unsigned)c->g.nbricks;
  if (stage == 0) {
    if (ACC == ACC_FIXED && KIND != 0) {
      cudaError_t e = launch_vmax(c);
      if (e != cudaSuccess) return e;
    }
    cudaError_t e = tile_pass<KIND, 0, ACC>(c, out, dp, gate);
    if constexpr (KIND == 2 && ACC != ACC_PLAIN) {
      if (e == cudaSuccess) e = tile_pass<KIND, 1, ACC>(c, out, dp, gate);
    }
    return e;
  }
  c->launches += 1;
  k_fixup<KIND, ACC><<<nb, 256, 0, c->stream>>>(c->g, c->spill, dp.fixed_scale, c->vmax_bits, out,
                                                c->flags, gate);
  return cudaGetLastError();
}

template <int KIND>
cudaError_t run_mode(lf2_ctx* c, float* out, const DepositParams& dp, int stage, const uint32_t* gate)
{
  if (c->mode == LF2_DEPOSIT_FIXED64) return run<KIND, ACC_FIXED>(c, out, dp, stage, gate);
  if (c->mode == LF2_DEPOSIT_FP32_PLAIN) return run<KIND, ACC_PLAIN>(c, out, dp, stage, gate);
  return run<KIND, ACC_COMP>(c, out, dp, stage, gate);
}

}  // namespace

// Shell-store slots (8 bytes each) a deposit of `comps` components needs.
size_t deposit_spill_slots(const lf2_ctx* c, int comps)
{
  return (size_t)c->g.nbricks * (size_t)comps * SHELL;
}

cudaError_t launch_vmax(lf2_ctx* c)
{
  cudaError_t e = cudaMemsetAsync(c->vmax_bits, 0, sizeof(uint32_t), c->stream);
  if (e != cudaSuccess) return e;
  c->launches += 1;
  k_vmax<<<(unsigned)c->g.nbricks, 256, 0, c->stream>>>(view(c), c->vmax_bits, c->flags);
  return cudaGetLastError();
}

DepositParams deposit_params(const lf2_ctx* c)
{
  DepositParams dp;
  const double vol = c->res * c->res * c->res;
  dp.inv_vol = (float)(1.0 / vol);
  dp.mf = (float)(c->gmass / vol);
  dp.fixed_scale = (float)(std::ldexp(1.0, -32) * c->m_unit / vol);
  dp.inv_unit = (float)(1.0 / c->m_unit);
  dp.has_mass = c->has_mass ? 1 : 0;
  return dp;
}

cudaError_t launch_deposit(lf2_ctx* c, int kind, float* out, int stage, const uint32_t* gate)
{
  const DepositParams dp = deposit_params(c);
  if (kind == 0) return run_mode<0>(c, out, dp, stage, gate);
  if (kind == 1) return run_mode<1>(c, out, dp, stage, gate);
  return run_mode<2>(c, out, dp, stage, gate);
}

}  // namespace lf2
