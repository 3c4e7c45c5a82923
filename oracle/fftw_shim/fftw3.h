/*
 * fftw3.h -- a stand-in for the part of the FFTW3 interface that the
 * reference's distributed FFT (LATfield2_PlanFFT_decl.hpp) uses, so that the
 * reference's own PlanFFT (its transposes, data layout and normalisation)
 * can be compiled and run here, where FFTW is not installed.
 * TEST INFRASTRUCTURE ONLY: it builds the reference-compiled checker under
 * oracle/_ref.
 *
 * Only what PlanFFT needs: rank-1 "many" plans (complex-to-complex,
 * real-to-complex, complex-to-real) with FFTW's meaning of howmany, stride
 * and dist, executed on the planned arrays or on new ones.  The transforms are
 * plain DFTs evaluated in long double:
 *   c2c  X_k = sum_j x_j exp(sign * 2 pi i j k / n), sign -1 forward, +1 backward
 *   r2c  X_k for k = 0 .. n/2 of a real input (forward sign)
 *   c2r  x_j = sum_k X_k exp(+2 pi i j k / n) over the Hermitian extension of
 *        X_0 .. X_n/2, with the imaginary parts of X_0 and X_n/2 (n even) not
 *        used
 * and none is normalised.  Each transform reads all its inputs before writing
 * its outputs, so in-place plans work.  The results differ from FFTW's only
 * by rounding.
 *
 * Header-only: include it in exactly one translation unit.
 */
#ifndef LF2_FFTW_SHIM_H
#define LF2_FFTW_SHIM_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

struct lf2_fftw_plan_s {
  int kind;  // 0 c2c, 1 r2c, 2 c2r
  int n, howmany, istride, idist, ostride, odist, sign;
  void* in;
  void* out;
};
typedef lf2_fftw_plan_s* fftw_plan;
typedef lf2_fftw_plan_s* fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

namespace lf2_fftw {

inline lf2_fftw_plan_s* make(int kind, int rank, const int* n, int howmany, void* in, int istride,
                             int idist, void* out, int ostride, int odist, int sign)
{
  if (rank != 1) {
    fprintf(stderr, "fftw stand-in: only rank-1 plans are provided\n");
    abort();
  }
  lf2_fftw_plan_s* p = new lf2_fftw_plan_s;
  p->kind = kind;
  p->n = n[0];
  p->howmany = howmany;
  p->in = in;
  p->out = out;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->sign = sign;
  return p;
}

// cos and sin of 2 pi m / n for m in [0, n)
inline void twiddle(long m, long n, long double& c, long double& s)
{
  const long double a = 6.283185307179586476925286766559L * (long double)(m % n) / (long double)n;
  c = cosl(a);
  s = sinl(a);
}

// T is the real type; complex arrays are T[2] per element.  Strides and
// distances count elements of the array's own type (complex or real).
template <class T>
void run(const lf2_fftw_plan_s* p, void* vin, void* vout)
{
  const long n = p->n;
  const long nk = n / 2 + 1;
  std::vector<long double> xr(n), xi(n), yr(n), yi(n);
  for (long t = 0; t < p->howmany; t++) {
    if (p->kind == 0) {
      const T* in = (const T*)vin;
      for (long j = 0; j < n; j++) {
        const size_t e = (size_t)(t * p->idist + j * p->istride);
        xr[j] = in[2 * e];
        xi[j] = in[2 * e + 1];
      }
      for (long k = 0; k < n; k++) {
        long double sr = 0, si = 0;
        for (long j = 0; j < n; j++) {
          long double c, s;
          twiddle(j * k, n, c, s);
          s *= p->sign;
          sr += xr[j] * c - xi[j] * s;
          si += xr[j] * s + xi[j] * c;
        }
        yr[k] = sr;
        yi[k] = si;
      }
      T* out = (T*)vout;
      for (long k = 0; k < n; k++) {
        const size_t e = (size_t)(t * p->odist + k * p->ostride);
        out[2 * e] = (T)yr[k];
        out[2 * e + 1] = (T)yi[k];
      }
    } else if (p->kind == 1) {
      const T* in = (const T*)vin;
      for (long j = 0; j < n; j++) xr[j] = in[(size_t)(t * p->idist + j * p->istride)];
      for (long k = 0; k < nk; k++) {
        long double sr = 0, si = 0;
        for (long j = 0; j < n; j++) {
          long double c, s;
          twiddle(j * k, n, c, s);
          sr += xr[j] * c;
          si -= xr[j] * s;
        }
        yr[k] = sr;
        yi[k] = si;
      }
      T* out = (T*)vout;
      for (long k = 0; k < nk; k++) {
        const size_t e = (size_t)(t * p->odist + k * p->ostride);
        out[2 * e] = (T)yr[k];
        out[2 * e + 1] = (T)yi[k];
      }
    } else {
      const T* in = (const T*)vin;
      for (long k = 0; k < nk; k++) {
        const size_t e = (size_t)(t * p->idist + k * p->istride);
        xr[k] = in[2 * e];
        xi[k] = in[2 * e + 1];
      }
      T* out = (T*)vout;
      for (long j = 0; j < n; j++) {
        long double sum = xr[0];
        for (long k = 1; 2 * k < n; k++) {
          long double c, s;
          twiddle(j * k, n, c, s);
          sum += 2.0L * (xr[k] * c - xi[k] * s);
        }
        if (n % 2 == 0) sum += (j % 2 ? -1.0L : 1.0L) * xr[n / 2];
        out[(size_t)(t * p->odist + j * p->ostride)] = (T)sum;
      }
    }
  }
}

}  // namespace lf2_fftw

#define LF2_FFTW_API(P, R, C)                                                                      \
  inline lf2_fftw_plan_s* P##plan_many_dft(int rank, const int* n, int howmany, C* in,            \
                                           const int*, int istride, int idist, C* out, const int*, \
                                           int ostride, int odist, int sign, unsigned)            \
  {                                                                                                \
    return lf2_fftw::make(0, rank, n, howmany, in, istride, idist, out, ostride, odist, sign);     \
  }                                                                                                \
  inline lf2_fftw_plan_s* P##plan_many_dft_r2c(int rank, const int* n, int howmany, R* in,        \
                                               const int*, int istride, int idist, C* out,        \
                                               const int*, int ostride, int odist, unsigned)      \
  {                                                                                                \
    return lf2_fftw::make(1, rank, n, howmany, in, istride, idist, out, ostride, odist, -1);       \
  }                                                                                                \
  inline lf2_fftw_plan_s* P##plan_many_dft_c2r(int rank, const int* n, int howmany, C* in,        \
                                               const int*, int istride, int idist, R* out,        \
                                               const int*, int ostride, int odist, unsigned)      \
  {                                                                                                \
    return lf2_fftw::make(2, rank, n, howmany, in, istride, idist, out, ostride, odist, +1);       \
  }                                                                                                \
  inline void P##execute(const lf2_fftw_plan_s* p) { lf2_fftw::run<R>(p, p->in, p->out); }        \
  inline void P##execute_dft(const lf2_fftw_plan_s* p, C* in, C* out)                             \
  {                                                                                                \
    lf2_fftw::run<R>(p, in, out);                                                                  \
  }                                                                                                \
  inline void P##execute_dft_r2c(const lf2_fftw_plan_s* p, R* in, C* out)                         \
  {                                                                                                \
    lf2_fftw::run<R>(p, in, out);                                                                  \
  }                                                                                                \
  inline void P##execute_dft_c2r(const lf2_fftw_plan_s* p, C* in, R* out)                         \
  {                                                                                                \
    lf2_fftw::run<R>(p, in, out);                                                                  \
  }                                                                                                \
  inline void P##destroy_plan(lf2_fftw_plan_s* p) { delete p; }                                    \
  inline void P##print_plan(const lf2_fftw_plan_s* p)                                              \
  {                                                                                                \
    printf("(dft kind %d n %d howmany %d)", p->kind, p->n, p->howmany);                           \
  }                                                                                                \
  inline void* P##malloc(size_t b) { return malloc(b); }                                           \
  inline void P##free(void* q) { free(q); }

LF2_FFTW_API(fftw_, double, fftw_complex)
LF2_FFTW_API(fftwf_, float, fftwf_complex)

#undef LF2_FFTW_API

#endif
