/*
 * lf2_oracle.c -- CPU oracle for the LATfield2 particle-mesh path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA path, never linked into
 * the product library.  See lf2_oracle.h for the two layers.
 *
 * Must be compiled with -ffp-contract=off so that no multiply-add is fused
 * behind the back of the restated arithmetic.
 */
#include "lf2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ layer (A) */
#define R double
#define LF2O_FN(name) name##_d
#include "lf2_oracle_ref.inc"
#undef R
#undef LF2O_FN

#define R float
#define LF2O_FN(name) name##_f
#include "lf2_oracle_ref.inc"
#undef R
#undef LF2O_FN

/* addParticle_global pushes each particle onto the front of its cell's
 * forward_list (LATfield2_Particles.hpp:500-519), so a list holds its
 * particles in reverse insertion order. */
void lf2o_lists_from_insertion(int64_t ncells, int64_t np, const int32_t* cell,
                               int64_t* cs, int64_t* order)
{
  memset(cs, 0, sizeof(int64_t) * (size_t)(ncells + 1));
  for (int64_t p = 0; p < np; p++) cs[cell[p] + 1]++;
  for (int64_t c = 0; c < ncells; c++) cs[c + 1] += cs[c];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncells);
  for (int64_t c = 0; c < ncells; c++) fill[c] = cs[c + 1];
  for (int64_t p = 0; p < np; p++) order[--fill[cell[p]]] = p;
  free(fill);
}

/* ------------------------------------------------------------ layer (B) */

static inline long wrapi(long v, long n)
{
  v %= n;
  return v < 0 ? v + n : v;
}

static inline void cell_coords(const int n[3], int32_t c, long xyz[3])
{
  xyz[0] = c % n[0];
  xyz[1] = (c / n[0]) % n[1];
  xyz[2] = c / ((long)n[0] * n[1]);
}

void lf2o_state_kick(const int n[3], int64_t np, const int32_t* cell,
                     const float* off, float* vel, const float* F, float dtk)
{
  const long ns = (long)n[0] * n[1] * n[2];
  for (int64_t p = 0; p < np; p++) {
    long xyz[3];
    cell_coords(n, cell[p], xyz);
    const float fx = off[3 * p + 0], fy = off[3 * p + 1], fz = off[3 * p + 2];
    const float gx = 1.0f - fx, gy = 1.0f - fy, gz = 1.0f - fz;
    const long xs[2] = {xyz[0], wrapi(xyz[0] + 1, n[0])};
    const long ys[2] = {xyz[1], wrapi(xyz[1] + 1, n[1])};
    const long zs[2] = {xyz[2], wrapi(xyz[2] + 1, n[2])};
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int k = 0; k < 8; k++) {
      const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
      const float w = ((bx ? fx : gx) * (by ? fy : gy)) * (bz ? fz : gz);
      const long site = xs[bx] + (long)n[0] * (ys[by] + (long)n[1] * zs[bz]);
      for (int c = 0; c < 3; c++) acc[c] = fmaf(w, F[c * ns + site], acc[c]);
    }
    for (int c = 0; c < 3; c++) vel[3 * p + c] = fmaf(dtk, acc[c], vel[3 * p + c]);
  }
}

int64_t lf2o_state_drift(const int n[3], int64_t np, int32_t* cell, float* off,
                         const float* vel, float dtn)
{
  int64_t bad = 0;
  for (int64_t p = 0; p < np; p++) {
    long xyz[3];
    cell_coords(n, cell[p], xyz);
    int ok = 1;
    for (int l = 0; l < 3; l++) {
      float o = fmaf(dtn, vel[3 * p + l], off[3 * p + l]);
      if (!isfinite(o)) {
        ok = 0;
        break;
      }
      float fl = floorf(o);
      o = o - fl;
      long carry = (long)fl;
      if (o >= 1.0f) {
        o = 0.0f;
        carry += 1;
      }
      off[3 * p + l] = o;
      xyz[l] = wrapi(xyz[l] + carry, n[l]);
    }
    if (!ok) {
      bad++;
      continue;
    }
    cell[p] = (int32_t)(xyz[0] + n[0] * (xyz[1] + (long)n[1] * xyz[2]));
  }
  return bad;
}

uint64_t lf2o_fixed_weight(float wx, float wy, float wz, int bx, int by, int bz)
{
  const uint64_t one = 1ull << 31;
  const uint64_t ux = (uint64_t)lrintf(wx * 2147483648.0f);
  const uint64_t uy = (uint64_t)lrintf(wy * 2147483648.0f);
  const uint64_t uz = (uint64_t)lrintf(wz * 2147483648.0f);
  const uint64_t qx = bx ? ux : one - ux;
  const uint64_t qy = by ? uy : one - uy;
  const uint64_t qz = bz ? uz : one - uz;
  const unsigned __int128 prod = (unsigned __int128)(qx * qy) * qz;
  return (uint64_t)((prod + ((unsigned __int128)1 << 60)) >> 61);
}

void lf2o_state_deposit_fixed(const int n[3], int64_t np, const int32_t* cell,
                              const float* off, const float* mrel, int64_t* acc)
{
  for (int64_t p = 0; p < np; p++) {
    long xyz[3];
    cell_coords(n, cell[p], xyz);
    const long xs[2] = {xyz[0], wrapi(xyz[0] + 1, n[0])};
    const long ys[2] = {xyz[1], wrapi(xyz[1] + 1, n[1])};
    const long zs[2] = {xyz[2], wrapi(xyz[2] + 1, n[2])};
    uint64_t mq = 0;
    if (mrel) mq = (uint64_t)lrintf(mrel[p] * 16777216.0f);
    for (int k = 0; k < 8; k++) {
      const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
      uint64_t q = lf2o_fixed_weight(off[3 * p], off[3 * p + 1], off[3 * p + 2],
                                     bx, by, bz);
      if (mrel) q = (q * mq + (1ull << 23)) >> 24;
      const long site = xs[bx] + (long)n[0] * (ys[by] + (long)n[1] * zs[bz]);
      acc[site] += (int64_t)q;
    }
  }
}

void lf2o_state_fixed_to_f32(int64_t nsites, const int64_t* acc, float scale,
                             float* rho)
{
  for (int64_t i = 0; i < nsites; i++) rho[i] = (float)acc[i] * scale;
}

void lf2o_state_deposit_f64(const int n[3], int64_t np, const int32_t* cell,
                            const float* off, const float* mass, double gmass,
                            double res, double* rho)
{
  const double vol = res * res * res;
  for (int64_t p = 0; p < np; p++) {
    long xyz[3];
    cell_coords(n, cell[p], xyz);
    const long xs[2] = {xyz[0], wrapi(xyz[0] + 1, n[0])};
    const long ys[2] = {xyz[1], wrapi(xyz[1] + 1, n[1])};
    const long zs[2] = {xyz[2], wrapi(xyz[2] + 1, n[2])};
    const double m = (mass ? (double)mass[p] : gmass) / vol;
    const double f[3] = {off[3 * p], off[3 * p + 1], off[3 * p + 2]};
    for (int k = 0; k < 8; k++) {
      const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
      const double w = (bx ? f[0] : 1.0 - f[0]) * (by ? f[1] : 1.0 - f[1]) *
                       (bz ? f[2] : 1.0 - f[2]);
      const long site = xs[bx] + (long)n[0] * (ys[by] + (long)n[1] * zs[bz]);
      rho[site] += w * m;
    }
  }
}

/* List order after the rebin loop of moveParticles on one rank
 * (LATfield2_Particles.hpp:1960-2056): cells are visited in site order; a
 * particle whose cell changed is spliced to the front of its new cell's list
 * (splice_after(before_begin, ...), :2049) and the walk resumes after its
 * predecessor (:2052); a particle spliced into a later cell is visited again
 * there and stays.  Input lists (cs_old, order_old) and the new cell of every
 * particle; output lists in CSR form. */
void lf2o_rebin_lists(int64_t ncells, int64_t np, const int64_t* cs_old,
                      const int64_t* order_old, const int32_t* new_cell,
                      int64_t* cs_new, int64_t* order_new)
{
  int64_t* head = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncells);
  int64_t* next = (int64_t*)malloc(sizeof(int64_t) * (size_t)(np > 0 ? np : 1));
  for (int64_t c = 0; c < ncells; c++) {
    head[c] = -1;
    for (int64_t i = cs_old[c + 1] - 1; i >= cs_old[c]; i--) {
      next[order_old[i]] = head[c];
      head[c] = order_old[i];
    }
  }
  for (int64_t c = 0; c < ncells; c++) {
    int64_t prev = -1; /* -1 stands for before_begin */
    int64_t it = head[c];
    while (it >= 0) {
      const int64_t nc = new_cell[it];
      if (nc != c) {
        if (prev < 0) head[c] = next[it];
        else next[prev] = next[it];
        next[it] = head[nc];
        head[nc] = it;
        it = (prev < 0) ? head[c] : next[prev];
      } else {
        prev = it;
        it = next[it];
      }
    }
  }
  int64_t k = 0;
  for (int64_t c = 0; c < ncells; c++) {
    cs_new[c] = k;
    for (int64_t it = head[c]; it >= 0; it = next[it]) order_new[k++] = it;
  }
  cs_new[ncells] = k;
  free(head);
  free(next);
}

/* ------------------------------------------------------------------------
 * Fixed-point momentum and stress deposits (device arithmetic restated).
 * Velocities are quantised against V = 2^e, the smallest power of two above
 * every |v_i| (lf2o_vexp), to 2^-31 V.  Contributions are signed integers in
 * units of 2^-48 of a unit mass times V (momentum: the exact integer product
 * of weight and velocity, rounded once; a per-particle mass in 2^-24 units
 * rounds it once more) or V^2 (stress: stress_q, in FP64), so the sums are
 * the device's bit for bit.  The vertex placement
 * follows the projections of the reference:
 *   kind 1  vectorProjectionCICNGP (projections.hpp:501-544)
 *   kind 2  symtensorProjectionCICNGP (:786-843)
 *   kind 3  vectorProjectionCIC (:1052-1190, staggered weights via gridChoice)
 *   kind 4  VecVecProjectionCIC (:1355-1620)
 */
int lf2o_vexp(int64_t np, const float* vel)
{
  uint32_t m = 0;
  for (int64_t i = 0; i < 3 * np; i++) {
    float a = fabsf(vel[i]);
    uint32_t b;
    memcpy(&b, &a, 4);
    if (b > m) m = b;
  }
  if (m == 0) return 0;
  int e = (int)((m >> 23) & 0xffu) - 126;
  return e < -96 ? -96 : e;
}

static inline uint32_t wq(float w) { return (uint32_t)lrintf(w * 2147483648.0f); }

static inline uint64_t corner3(uint32_t a, uint32_t b, uint32_t c)
{
  const unsigned __int128 prod = (unsigned __int128)((uint64_t)a * (uint64_t)b) * c;
  return (uint64_t)((prod + ((unsigned __int128)1 << 60)) >> 61);
}

/* round(a b / 2^s), the product exact in 128 bits */
static inline uint64_t mulr(uint64_t a, uint64_t b, int s)
{
  const unsigned __int128 prod = (unsigned __int128)a * b;
  return (uint64_t)((prod + ((unsigned __int128)1 << (s - 1))) >> s);
}
/* weight (2^-32) x velocity (2^-31 V) -> 2^-48 V */
static inline uint64_t mul_wv48(uint64_t w, uint64_t f) { return mulr(w, f, 15); }

/* Stress contributions in FP64 (the device's stress_q): the weight w (an
 * integer below 2^52, exact as a double) times a per-particle factor
 * f = (v_a v_b) 2^-s [times (mq 2^-24), the relative mass], each product
 * rounded by IEEE double multiplication, then rounded to the nearest
 * integer, half to even (1.5 2^52 added and its low mantissa bits taken, as
 * the device does).  Units of 2^-48 V^2. */
static inline uint64_t mq_of(const float* mrel, int64_t p)
{
  float mr = mrel[p];
  mr = mr < 0.0f ? 0.0f : (mr > 63.0f ? 63.0f : mr);
  return (uint64_t)lrintf(mr * 16777216.0f);
}
static inline double stress_factor(uint32_t va, uint32_t vb, int s, const float* mrel, int64_t p)
{
  double f = ((double)va * (double)vb) * ldexp(1.0, -s);
  if (mrel) f = f * ((double)mq_of(mrel, p) * ldexp(1.0, -24));
  return f;
}
static inline int64_t stress_q(uint64_t w, double f, int neg)
{
  double y = (double)w * f;
  y = y + 6755399441055744.0;
  uint64_t bits;
  memcpy(&bits, &y, 8);
  const int64_t q = (int64_t)((bits & 0xFFFFFFFFFFFFFull) - (1ull << 51));
  return neg ? -q : q;
}

static inline int64_t signed_q(uint64_t q, const float* mrel, int64_t p, int neg)
{
  if (mrel) {
    float mr = mrel[p];
    mr = mr < 0.0f ? 0.0f : (mr > 63.0f ? 63.0f : mr);
    const uint64_t mq = (uint64_t)lrintf(mr * 16777216.0f);
    q = mulr(q, mq, 24);
  }
  return neg ? -(int64_t)q : (int64_t)q;
}

void lf2o_state_deposit_fixed_kind(int kind, const int n[3], int64_t np,
                                   const int32_t* cell, const float* off,
                                   const float* vel, const float* mrel, int vexp,
                                   int64_t* acc)
{
  const long ns = (long)n[0] * n[1] * n[2];
  const float vscale = ldexpf(1.0f, 31 - vexp);
  const uint32_t ONE = 1u << 31;
  for (int64_t p = 0; p < np; p++) {
    long xyz[3];
    cell_coords(n, cell[p], xyz);
    const float* o = off + 3 * p;
    const float* v = vel + 3 * p;
    uint32_t sq[3][2], tq[3][2], vq[3];
    long vs[3][2], ts[3][2]; /* vertex and staggered coordinates */
    for (int d = 0; d < 3; d++) {
      const uint32_t u = wq(o[d]);
      sq[d][0] = ONE - u;
      sq[d][1] = u;
      const float sd = o[d] - 0.5f;
      const int gd = sd >= 0.0f;
      const uint32_t us = wq(fabsf(sd));
      tq[d][0] = gd ? ONE - us : us;
      tq[d][1] = gd ? us : ONE - us;
      vq[d] = (uint32_t)lrintf(fabsf(v[d]) * vscale);
      vs[d][0] = xyz[d];
      vs[d][1] = wrapi(xyz[d] + 1, n[d]);
      ts[d][0] = wrapi(xyz[d] - 1 + gd, n[d]);
      ts[d][1] = wrapi(xyz[d] + gd, n[d]);
    }
#define SITE(a, b, c) ((a) + (long)n[0] * ((b) + (long)n[1] * (c)))
    if (kind == 1) {
      for (int c = 0; c < 3; c++) {
        const int neg = v[c] < 0.0f;
        for (int k = 0; k < 4; k++) {
          const int a = (k >> 1) & 1, b = k & 1;
          uint64_t w;
          long site;
          if (c == 0) w = corner3(ONE, sq[1][a], sq[2][b]), site = SITE(xyz[0], vs[1][a], vs[2][b]);
          else if (c == 1) w = corner3(sq[0][a], ONE, sq[2][b]), site = SITE(vs[0][a], xyz[1], vs[2][b]);
          else w = corner3(sq[0][a], sq[1][b], ONE), site = SITE(vs[0][a], vs[1][b], xyz[2]);
          acc[c * ns + site] += signed_q(mul_wv48(w, vq[c]), mrel, p, neg);
        }
      }
    } else if (kind == 2) {
      static const int diag[3] = {0, 3, 5};
      for (int k = 0; k < 8; k++) {
        const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
        const uint64_t w = corner3(sq[0][bx], sq[1][by], sq[2][bz]);
        const long site = SITE(vs[0][bx], vs[1][by], vs[2][bz]);
        for (int d = 0; d < 3; d++) {
          acc[diag[d] * ns + site] += stress_q(w, stress_factor(vq[d], vq[d], 46, mrel, p), 0);
        }
      }
      /* T_ij on the (i,j) plaquette, CIC along the third dim k */
      static const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2}, pk[3] = {2, 1, 0}, comp[3] = {1, 2, 4};
      for (int q = 0; q < 3; q++) {
        const double vv = stress_factor(vq[pa[q]], vq[pb[q]], 45, mrel, p);
        const int neg = (v[pa[q]] < 0.0f) != (v[pb[q]] < 0.0f);
        for (int b = 0; b < 2; b++) {
          long c3[3] = {xyz[0], xyz[1], xyz[2]};
          c3[pk[q]] = vs[pk[q]][b];
          acc[comp[q] * ns + SITE(c3[0], c3[1], c3[2])] += stress_q(sq[pk[q]][b], vv, neg);
        }
      }
    } else if (kind == 3) {
      for (int c = 0; c < 3; c++) {
        const int neg = v[c] < 0.0f;
        for (int k = 0; k < 8; k++) {
          const int bb[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
          uint32_t w[3];
          long cc[3];
          for (int d = 0; d < 3; d++) {
            w[d] = d == c ? tq[d][bb[d]] : sq[d][bb[d]];
            cc[d] = d == c ? ts[d][bb[d]] : vs[d][bb[d]];
          }
          acc[c * ns + SITE(cc[0], cc[1], cc[2])] +=
              signed_q(mul_wv48(corner3(w[0], w[1], w[2]), vq[c]), mrel, p, neg);
        }
      }
    } else if (kind == 4) {
      static const int diag[3] = {0, 3, 5};
      for (int k = 0; k < 8; k++) {
        const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
        const uint64_t w = corner3(sq[0][bx], sq[1][by], sq[2][bz]);
        const long site = SITE(vs[0][bx], vs[1][by], vs[2][bz]);
        for (int d = 0; d < 3; d++) {
          acc[diag[d] * ns + site] += stress_q(w, stress_factor(vq[d], vq[d], 46, mrel, p), 0);
        }
      }
      static const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2}, comp[3] = {1, 2, 4};
      for (int q = 0; q < 3; q++) {
        const double vv = stress_factor(vq[pa[q]], vq[pb[q]], 46, mrel, p);
        const int neg = (v[pa[q]] < 0.0f) != (v[pb[q]] < 0.0f);
        for (int k = 0; k < 8; k++) {
          const int bb[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
          uint32_t w[3];
          long cc[3];
          for (int d = 0; d < 3; d++) {
            const int st = d == pa[q] || d == pb[q];
            w[d] = st ? tq[d][bb[d]] : sq[d][bb[d]];
            cc[d] = st ? ts[d][bb[d]] : vs[d][bb[d]];
          }
          acc[comp[q] * ns + SITE(cc[0], cc[1], cc[2])] += stress_q(corner3(w[0], w[1], w[2]), vv, neg);
        }
      }
    }
#undef SITE
  }
}
