// lf2_deposit_common.cuh -- accumulation helpers shared by the deposit tile
// passes of lf2_deposit.cu (CIC and CIC-NGP projections) and
// lf2_deposit_full.cu (full-CIC projections): the compensated FP32 add, the
// split fixed-point accumulation and the deterministic integer weights of the
// fixed-point mode.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lf2_common.cuh"
#include "lf2gpu.h"

namespace lf2 {

enum : int {
  ACC_COMP = LF2_DEPOSIT_FP32,
  ACC_FIXED = LF2_DEPOSIT_FIXED64,
  ACC_PLAIN = LF2_DEPOSIT_FP32_PLAIN
};

// ------------------------------------------------------------ accumulation
// Fixed point: each 64-bit vertex sum is kept as two 32-bit partial sums,
// lo = sum(q & 0xffff) and hi = sum(q >> 16) (arithmetic shift), so that every
// update is a native 32-bit shared-memory reduction; the sum is
// lo + hi * 2^16, hi read as unsigned (scalar, q >= 0) or as signed (momentum
// and stress).  Neither partial sum may wrap: per particle and vertex
// |q| <= 2^32 * M with M = 1 for a global mass and M = 64 with per-particle
// masses (relative mass < 64), so the split is exact for bricks of at most
// split_max particles; larger bricks use 64-bit shared atomics.
template <bool SIGNED>
__host__ __device__ inline int split_max(bool has_mass)
{
  return SIGNED ? (has_mass ? 511 : 32767) : (has_mass ? 1023 : 65535);
}

// A tile of N vertices per component in shared memory: component j occupies
// words [2 j N, 2 (j + 1) N) (two 32-bit words per vertex), or [j N, (j+1) N)
// in the plain mode.
template <int N>
struct TileRef {
  unsigned char* smem;
  bool split;
};

template <int N>
__device__ __forceinline__ void add_fixed(TileRef<N> tr, int j, int t, long long q)
{
  if (tr.split) {
    uint32_t* w = reinterpret_cast<uint32_t*>(tr.smem) + (size_t)j * 2 * N;
    atomicAdd(&w[t], (uint32_t)((unsigned long long)q & 0xffffu));
    atomicAdd(&w[N + t], (uint32_t)(q >> 16));
  } else {
    atomicAdd(reinterpret_cast<unsigned long long*>(tr.smem) + (size_t)j * N + t,
              (unsigned long long)q);
  }
}

// The same with the split decided at compile time (the tile passes
// instantiate their particle loop once per choice, per CTA).
template <bool SPLIT, int N>
__device__ __forceinline__ void add_fixed_t(unsigned char* smem, int j, int t, long long q)
{
  if (SPLIT) {
    uint32_t* w = reinterpret_cast<uint32_t*>(smem) + (size_t)j * 2 * N;
    atomicAdd(&w[t], (uint32_t)((unsigned long long)q & 0xffffu));
    atomicAdd(&w[N + t], (uint32_t)(q >> 16));
  } else {
    atomicAdd(reinterpret_cast<unsigned long long*>(smem) + (size_t)j * N + t, (unsigned long long)q);
  }
}

// Compensated FP32 add: the atomic returns the value it replaced, so the
// rounding error of the stored sum fl(old + w) is recovered exactly by
// Knuth's TwoSum and added to the second word.
__device__ __forceinline__ void add_comp(float* hi, float* lo, float w)
{
  const float old = atomicAdd(hi, w);
  const float s = __fadd_rn(old, w);
  const float bb = __fsub_rn(s, old);
  const float err = __fadd_rn(__fsub_rn(old, __fsub_rn(s, bb)), __fsub_rn(w, bb));
  atomicAdd(lo, err);
}

// (s, c) += (h, l): TwoSum of s and h, the error and l carried in c.
__device__ __forceinline__ void comp_acc(float& s, float& c, float h, float l)
{
  const float t = __fadd_rn(s, h);
  const float bb = __fsub_rn(t, s);
  const float err = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bb)), __fsub_rn(h, bb));
  s = t;
  c = __fadd_rn(c, __fadd_rn(err, l));
}

template <int ACC, int N>
__device__ __forceinline__ void add_float(TileRef<N> tr, int j, int t, float w)
{
  float* f = reinterpret_cast<float*>(tr.smem);
  if (ACC == ACC_PLAIN) {
    atomicAdd(&f[(size_t)j * N + t], w);
  } else {
    add_comp(&f[(size_t)j * 2 * N + t], &f[(size_t)j * 2 * N + N + t], w);
  }
}

// Signed kinds (momentum and stress): contributions are in units of 2^-48
// of a unit mass times V or V^2, |q| <= 2^48 for a global mass and 2^54 with
// per-particle masses.  The split keeps lo = the low 32 bits of the sum
// (every carry out of the 32-bit add, seen in the value the atomic returns,
// goes to hi) and hi = the sum of (q >> 32) plus those carries, so the
// vertex sum is hi 2^32 + lo exactly while hi stays within int32: bricks of
// at most 32767 particles (511 with per-particle masses), split_max<true>.
template <bool SPLIT, int N>
__device__ __forceinline__ void add_fixed48_t(unsigned char* smem, int j, int t, long long q)
{
  if (SPLIT) {
    uint32_t* w = reinterpret_cast<uint32_t*>(smem) + (size_t)j * 2 * N;
    const uint32_t lo = (uint32_t)(unsigned long long)q;
    const uint32_t old = atomicAdd(&w[t], lo);
    const int carry = (uint32_t)(old + lo) < old ? 1 : 0;
    atomicAdd(reinterpret_cast<int*>(&w[N + t]), (int)(q >> 32) + carry);
  } else {
    atomicAdd(reinterpret_cast<unsigned long long*>(smem) + (size_t)j * N + t, (unsigned long long)q);
  }
}

// Integer vertex sum of component j: the scalar's split (lo + hi 2^16) or
// the signed kinds' split (hi 2^32 + lo, add_fixed48_t).
template <bool SIGNED, int N>
__device__ __forceinline__ long long tile_fixed(const TileRef<N>& tr, int j, int t)
{
  if (tr.split) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(tr.smem) + (size_t)j * 2 * N;
    if (SIGNED) return (long long)(int32_t)w[N + t] * 4294967296ll + (long long)w[t];
    return (long long)w[t] + (long long)w[N + t] * 65536ll;
  }
  return (long long)reinterpret_cast<const unsigned long long*>(tr.smem)[(size_t)j * N + t];
}

// ----------------------------------------------------- fixed-point weights
// 1-D weight in units of 2^-31 (lf2o_fixed_weight in the oracle).
__device__ __forceinline__ uint32_t weight_q(float w) { return __float2uint_rn(w * 2147483648.0f); }

// Velocity in units of 2^-31 V (V = 2^e > |v|): |v| 2^(31-e) is exact in FP32
// and below 2^31; rounded to the nearest integer.
__device__ __forceinline__ uint32_t vel_q(float v, float vscale)
{
  return __float2uint_rn(fabsf(v) * vscale);
}

// Product of two such velocities in units of 2^-31 V^2, rounded.
__device__ __forceinline__ uint64_t vel2_q(uint32_t a, uint32_t b)
{
  return ((uint64_t)a * (uint64_t)b + (1ull << 30)) >> 31;
}

// w (2^-32 units) times a factor in 2^-31 units, rounded to 2^-32 units.
__device__ __forceinline__ uint64_t mul31(uint64_t w, uint64_t f) { return (w * f + (1ull << 30)) >> 31; }

// Momentum: w (2^-32 units, <= 2^32) times a velocity (2^-31 V units,
// < 2^31), rounded to 2^-48 V units.
__device__ __forceinline__ uint64_t mul_wv48(uint64_t w, uint64_t f) { return (w * f + (1ull << 14)) >> 15; }

// round(a * b / 2^s) for a product of up to 128 bits (32 <= s < 64), from
// its two 64-bit halves.
template <int S>
__device__ __forceinline__ uint64_t mul_round(uint64_t a, uint64_t b)
{
  const uint64_t lo = a * b, hi = __umul64hi(a, b);
  return ((lo >> S) | (hi << (64 - S))) + ((lo >> (S - 1)) & 1ull);
}

// Stress: w (2^-32 units) times the exact product of two velocities (2^-62
// V^2 units, < 2^62), rounded to 2^-48 V^2 units; a 1-D weight (2^-31 units)
// times that product likewise.
__device__ __forceinline__ uint64_t mul_wvv48(uint64_t w, uint64_t vv) { return mul_round<46>(w, vv); }
__device__ __forceinline__ uint64_t mul_avv48(uint64_t a, uint64_t vv) { return mul_round<45>(a, vv); }

// Stress contributions in FP64: the weight w (an integer below 2^52, exact
// in double) times a per-particle factor f = v_a v_b 2^-s (times the
// relative mass), both products rounded by IEEE double multiplication, then
// rounded to the nearest integer (half to even): units of 2^-48 V^2.  The
// sequence is deterministic and restated in the oracle operation by
// operation.
__device__ __forceinline__ double u2d_exact(uint64_t w)  // w < 2^52
{
  return __dadd_rn(__longlong_as_double((long long)(0x4330000000000000ull | w)), -4503599627370496.0);
}
__device__ __forceinline__ uint64_t d2u_rn(double x)  // 0 <= x < 2^51
{
  const double y = __dadd_rn(x, 6755399441055744.0);  // 1.5 * 2^52: integer part in the low bits
  return ((uint64_t)__double_as_longlong(y) & 0xFFFFFFFFFFFFFull) - (1ull << 51);
}
// f = (v_a v_b) 2^-s, times m / m_unit when HM (mq: the relative mass in
// 2^-24 units)
template <bool HM>
__device__ __forceinline__ double stress_factor(uint32_t va, uint32_t vb, double scale, uint64_t mq)
{
  double f = __dmul_rn(__dmul_rn(u2d_exact(va), u2d_exact(vb)), scale);
  if (HM) f = __dmul_rn(f, __dmul_rn(u2d_exact(mq), 0x1p-24));  // 2^-24
  return f;
}
__device__ __forceinline__ long long stress_q(uint64_t w, double f, bool neg)
{
  const long long q = (long long)d2u_rn(__dmul_rn(u2d_exact(w), f));
  return neg ? -q : q;
}

// Per-particle relative mass (2^-24 units) applied to a signed-kind
// contribution (|q| <= 2^48, so the product needs 128 bits), then the sign.
template <bool HM>
__device__ __forceinline__ long long mass_sign48_t(uint64_t q, uint64_t mq, bool neg)
{
  if (HM) q = mul_round<24>(q, mq);
  return neg ? -(long long)q : (long long)q;
}

// Per-particle relative mass m / m_unit in units of 2^-24 (range-checked).
__device__ __forceinline__ uint64_t mass_q(float m, float inv_unit, uint32_t* flags)
{
  const float mr = __fmul_rn(m, inv_unit);
  if (!(mr >= 0.0f && mr < 64.0f)) set_flag(flags, ERR_MASS_RANGE);
  return (uint64_t)__float2uint_rn(fminf(fmaxf(mr, 0.0f), 63.0f) * 16777216.0f);
}

__device__ __forceinline__ long long apply_mass_sign(uint64_t q, bool has_mass, uint64_t mq, bool neg)
{
  if (has_mass) q = (q * mq + (1ull << 23)) >> 24;
  return neg ? -(long long)q : (long long)q;
}

template <bool HM>
__device__ __forceinline__ long long mass_sign_t(uint64_t q, uint64_t mq, bool neg)
{
  if (HM) q = (q * mq + (1ull << 23)) >> 24;
  return neg ? -(long long)q : (long long)q;
}

// Scalar corner weight of a global-mass particle straight into the split
// tile: q = fixed_corner(qx, qy, qz) with p = qx qy given, so that
// q & 0xffff = bits [29, 45) and q >> 16 = bits [45, 64) of
// h = ph qz + umulhi(pl, qz) + 2^28.
template <int N>
__device__ __forceinline__ void add_corner_split(uint32_t* tile, int t, uint64_t p, uint32_t qz)
{
  const uint64_t h = (uint64_t)(uint32_t)(p >> 32) * qz + __umulhi((uint32_t)p, qz) + (1ull << 28);
  const uint32_t hl = (uint32_t)h, hh = (uint32_t)(h >> 32);
  atomicAdd(&tile[t], __funnelshift_r(hl, hh, 29) & 0xffffu);
  atomicAdd(&tile[N + t], hh >> 13);
}

// Scale 2^(31-e) as an FP32 (e within [-96, 128]).
__device__ __forceinline__ float vel_scale(int e) { return ldexpf(1.0f, 31 - e); }

// Exponent e of V = 2^e, the smallest power of two above the largest |v_i|
// (bits of a non-negative float; 0 when every velocity is 0), at least
// 2^-96 so that 2^(31-e) stays a finite FP32.
__host__ __device__ inline int vexp_of(uint32_t bits)
{
  if (bits == 0u) return 0;
  const int e = (int)((bits >> 23) & 0xffu) - 126;
  return e < -96 ? -96 : e;
}

}  // namespace lf2
