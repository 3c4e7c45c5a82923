// lf2_fft.cu -- the PM grid operator, on one GPU and as the pieces of its
// z-slab form.
//
//  - PlanFFT<Imag> for a real field on a cubic lattice
//    (LATfield2_PlanFFT_decl.hpp:720-1050): execute(FFT_FORWARD) and
//    execute(FFT_BACKWARD), unnormalised, through cuFFT's 3-D R2C/C2R.  The
//    reference distributes the transform over its process grid with explicit
//    transposes; on one GPU the whole cube is one cuFFT plan.
//  - k-fields: complex, kept in cuFFT's order [k_z][k_y][k_x] per component.
//    Import/export convert to the reference's Field<Imag> on the lattice of
//    Lattice::initializeRealFFT (halo 0), whose storage order is
//    [k_y][k_z][k_x] (rKSite, LATfield2_Site.hpp:319-338), components
//    interleaved.
//  - lf2_pm_force: the Poisson solve of the reference's example
//    (examples/poissonSolver.cpp: rho_k divided by the eigenvalue of the
//    7-point lattice Laplacian, the k = 0 mode set to zero), normalised, and
//    the central-difference force F_i = -(phi(x+e_i) - phi(x-e_i)) / (2 res):
//    cuFFT R2C, k_green (Green's function, in place), cuFFT C2R, k_gradient.
//    The Laplacian eigenvalue is evaluated as -4 sum_d sin^2(pi k_d / n) / res^2,
//    which equals the example's 2 (sum_d cos(2 pi k_d / n) - 3) / res^2 without
//    its cancellation at small k.
//  - lf2_pm_force4 / lf2_pm_force4_adjoint: the same operator as the grid
//    operator of the differentiable chain (float4 per site), and its adjoint:
//    the divergence of the incoming force gradient (k_divergence4) followed
//    by the same Green's-function solve, which is self-adjoint (a
//    convolution with a real kernel even in k).
//  - lf2_slab_fft_* / lf2_slab_green / lf2_pm_gradient: the pieces of the
//    operator when z is split over ranks, after the distributed PlanFFT
//    (LATfield2_PlanFFT_decl.hpp:83-230) with one split dim: batched 2-D
//    plane transforms of a rank's planes, strided 1-D line transforms along z
//    after the caller's transpose, k_green on a k_y slab, and the gradient
//    on the rank's lattice with ghost planes.
#include <cuda_runtime.h>
#include <cufft.h>

#include <new>
#include <string>

#include "lf2_internal.h"

using namespace lf2;

struct lf2_kfield_s {
  int comps = 0;
  float2* data = nullptr;  // comps x [n2][n1][n0/2+1]
};

struct lf2_slab_fft_s {
  lf2_ctx* c = nullptr;
  int n = 0, nz = 0, nky = 0, nkx = 0;
  cufftHandle r2c = 0, c2r = 0, lines = 0;
  int planned = 0;  // bit 0 r2c, bit 1 c2r, bit 2 lines
};

namespace lf2 {

namespace {

lf2_status fft_fail(lf2_ctx* c, lf2_status code, const std::string& msg)
{
  if (c) c->err = msg;
  return code;
}

#define FFT_CUDA(c, expr)                                                                   \
  do {                                                                                      \
    cudaError_t e_ = (expr);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fft_fail((c), LF2_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
  } while (0)

#define FFT_CUFFT(c, expr)                                                                  \
  do {                                                                                      \
    cufftResult r_ = (expr);                                                                \
    if (r_ != CUFFT_SUCCESS)                                                                \
      return fft_fail((c), LF2_ERR_CUDA,                                                    \
                      std::string(#expr ": cuFFT status ") + std::to_string((int)r_));      \
  } while (0)

#define FFT_TRY(expr)            \
  do {                           \
    lf2_status s_ = (expr);      \
    if (s_ != LF2_OK) return s_; \
  } while (0)

inline int64_t k_sites(const lf2_ctx* c)
{
  return (int64_t)c->g.n[2] * c->g.n[1] * (c->g.n[0] / 2 + 1);
}

inline unsigned grid_for(int64_t n, int threads)
{
  const int64_t b = (n + threads - 1) / threads;
  return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

bool field_ok(const lf2_field f, int comps) { return f && f->data && f->comps == comps; }

lf2_status need_cubic(lf2_ctx* c)
{
  if (c->g.n[0] != c->g.n[1] || c->g.n[1] != c->g.n[2])
    return fft_fail(c, LF2_ERR_ARG,
                    "the FFT works on cubic lattices only (as PlanFFT::initialize, "
                    "LATfield2_PlanFFT_decl.hpp:787-797)");
  return LF2_OK;
}

lf2_status ensure_plans(lf2_ctx* c)
{
  FFT_TRY(need_cubic(c));
  if (!c->fft_planned) {
    cufftHandle a = 0, b = 0;
    FFT_CUFFT(c, cufftPlan3d(&a, c->g.n[2], c->g.n[1], c->g.n[0], CUFFT_R2C));
    const cufftResult rb = cufftPlan3d(&b, c->g.n[2], c->g.n[1], c->g.n[0], CUFFT_C2R);
    if (rb != CUFFT_SUCCESS) {
      cufftDestroy(a);
      return fft_fail(c, LF2_ERR_CUDA, "cufftPlan3d (C2R): cuFFT status " + std::to_string((int)rb));
    }
    c->fft_r2c = a;
    c->fft_c2r = b;
    c->fft_planned = true;
  }
  FFT_CUFFT(c, cufftSetStream(c->fft_r2c, c->stream));
  FFT_CUFFT(c, cufftSetStream(c->fft_c2r, c->stream));
  return LF2_OK;
}

// One component of complex scratch (and, when asked, one of real scratch).
lf2_status ensure_scratch(lf2_ctx* c, bool real_too)
{
  if (!c->fft_k) FFT_CUDA(c, cudaMalloc(&c->fft_k, sizeof(float2) * (size_t)k_sites(c)));
  if (real_too && !c->fft_phi)
    FFT_CUDA(c, cudaMalloc(&c->fft_phi, sizeof(float) * (size_t)c->g.nsites));
  return LF2_OK;
}

// K[kz][ky][kx] *= coef / (s2(kx) + s2(ky) + s2(kz)), s2(k) = sin^2(pi k / n),
// K_0 = 0.  coef = -coupling res^2 / (4 N) turns the unnormalised transform
// of rho into the normalised potential phi_k.  The n values of s2 sit in a
// shared table (4 n bytes of dynamic shared memory).  Each thread takes two
// consecutive complex values (one 16-byte access; n^2 (n/2+1) is even for
// even n, and an odd n takes the last value alone) and GREEN_ITEMS such pairs
// at once, so several loads are in flight before the first store.
constexpr int GREEN_ITEMS = 4;

// K holds k_y in [ky0, ky0 + nky) of the k-cube: [k_z][k_y - ky0][k_x] (the
// whole cube when nky = n and ky0 = 0).
__device__ __forceinline__ float green_factor(const float* s2tab, uint32_t i, int nky, int nkx,
                                              int ky0, float coef)
{
  const uint32_t row = i / (uint32_t)nkx;
  const int kx = (int)(i - row * (uint32_t)nkx);
  const int ky = ky0 + (int)(row % (uint32_t)nky), kz = (int)(row / (uint32_t)nky);
  return (kx | ky | kz) == 0 ? 0.0f : coef / (s2tab[kx] + (s2tab[ky] + s2tab[kz]));
}

__global__ void k_green(float2* __restrict__ K, int n, int nky, int nkx, int ky0, float coef)
{
  extern __shared__ float s2tab[];
  const float inv_n = 1.0f / (float)n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float s = sinpif((float)i * inv_n);
    s2tab[i] = s * s;
  }
  __syncthreads();
  const uint32_t total = (uint32_t)n * (uint32_t)nky * (uint32_t)nkx;
  const uint32_t pairs = total / 2;
  float4* K4 = reinterpret_cast<float4*>(K);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p0 = blockIdx.x * blockDim.x + threadIdx.x; p0 < pairs;
       p0 += stride * GREEN_ITEMS) {
    float4 v[GREEN_ITEMS];
#pragma unroll
    for (int j = 0; j < GREEN_ITEMS; j++) {
      const uint32_t p = p0 + j * stride;
      if (p < pairs) v[j] = K4[p];
    }
#pragma unroll
    for (int j = 0; j < GREEN_ITEMS; j++) {
      const uint32_t p = p0 + j * stride;
      if (p >= pairs) continue;
      const float f0 = green_factor(s2tab, 2 * p, nky, nkx, ky0, coef);
      const float f1 = green_factor(s2tab, 2 * p + 1, nky, nkx, ky0, coef);
      K4[p] = make_float4(v[j].x * f0, v[j].y * f0, v[j].z * f1, v[j].w * f1);
    }
  }
  if ((total & 1u) && blockIdx.x == 0 && threadIdx.x == 0) {
    const float f = green_factor(s2tab, total - 1, nky, nkx, ky0, coef);
    const float2 v = K[total - 1];
    K[total - 1] = make_float2(v.x * f, v.y * f);
  }
}

// F_c = (phi(x - e_c) - phi(x + e_c)) * inv_2res, periodic, component-major.
// One CTA walks x-rows (z, y).  VEC: each thread takes four consecutive x
// with 16-byte loads and stores (n0 a multiple of 4); otherwise one x.
template <bool VEC>
__global__ void k_gradient(const float* __restrict__ phi, float* __restrict__ F, Geom g,
                           float inv_2res)
{
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int64_t ns = g.nsites;
  const int rows = n1 * n2;
  for (int row = blockIdx.x; row < rows; row += gridDim.x) {
    const int y = row % n1, z = row / n1;
    const int yp = y + 1 == n1 ? 0 : y + 1, ym = y == 0 ? n1 - 1 : y - 1;
    const int zp = z + 1 == n2 ? 0 : z + 1, zm = z == 0 ? n2 - 1 : z - 1;
    const float* pr = phi + (int64_t)row * n0;
    const float* pyp = phi + ((int64_t)z * n1 + yp) * n0;
    const float* pym = phi + ((int64_t)z * n1 + ym) * n0;
    const float* pzp = phi + ((int64_t)zp * n1 + y) * n0;
    const float* pzm = phi + ((int64_t)zm * n1 + y) * n0;
    float* f0 = F + (int64_t)row * n0;
    if (VEC) {
      for (int x = 4 * threadIdx.x; x < n0; x += 4 * blockDim.x) {
        const float4 c = *reinterpret_cast<const float4*>(pr + x);
        const float lft = pr[x == 0 ? n0 - 1 : x - 1];
        const float rgt = pr[x + 4 == n0 ? 0 : x + 4];
        const float4 a = *reinterpret_cast<const float4*>(pym + x);
        const float4 b = *reinterpret_cast<const float4*>(pyp + x);
        const float4 d = *reinterpret_cast<const float4*>(pzm + x);
        const float4 e = *reinterpret_cast<const float4*>(pzp + x);
        *reinterpret_cast<float4*>(f0 + x) =
            make_float4((lft - c.y) * inv_2res, (c.x - c.z) * inv_2res, (c.y - c.w) * inv_2res,
                        (c.z - rgt) * inv_2res);
        *reinterpret_cast<float4*>(f0 + ns + x) =
            make_float4((a.x - b.x) * inv_2res, (a.y - b.y) * inv_2res, (a.z - b.z) * inv_2res,
                        (a.w - b.w) * inv_2res);
        *reinterpret_cast<float4*>(f0 + 2 * ns + x) =
            make_float4((d.x - e.x) * inv_2res, (d.y - e.y) * inv_2res, (d.z - e.z) * inv_2res,
                        (d.w - e.w) * inv_2res);
      }
    } else {
      for (int x = threadIdx.x; x < n0; x += blockDim.x) {
        const int xp = x + 1 == n0 ? 0 : x + 1, xm = x == 0 ? n0 - 1 : x - 1;
        f0[x] = (pr[xm] - pr[xp]) * inv_2res;
        f0[ns + x] = (pym[x] - pyp[x]) * inv_2res;
        f0[2 * ns + x] = (pzm[x] - pzp[x]) * inv_2res;
      }
    }
  }
}

// Reference layout d = ((ky n + kz) nkx + kx) comps + c  <->  K[c][kz][ky][kx].
template <class T>
__global__ void k_kexport(const float2* __restrict__ K, int comps, int n, int nkx,
                          T* __restrict__ dst)
{
  const int64_t nk = (int64_t)n * n * nkx;
  const int64_t total = nk * comps;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(d % comps);
    const int64_t s = d / comps;
    const int kx = (int)(s % nkx);
    const int64_t r = s / nkx;
    const int kz = (int)(r % n), ky = (int)(r / n);
    const float2 v = K[c * nk + ((int64_t)kz * n + ky) * nkx + kx];
    dst[2 * d] = (T)v.x;
    dst[2 * d + 1] = (T)v.y;
  }
}

template <class T>
__global__ void k_kimport(float2* __restrict__ K, int comps, int n, int nkx,
                          const T* __restrict__ src)
{
  const int64_t nk = (int64_t)n * n * nkx;
  const int64_t total = nk * comps;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(d % comps);
    const int64_t s = d / comps;
    const int kx = (int)(s % nkx);
    const int64_t r = s / nkx;
    const int kz = (int)(r % n), ky = (int)(r / n);
    K[c * nk + ((int64_t)kz * n + ky) * nkx + kx] =
        make_float2((float)src[2 * d], (float)src[2 * d + 1]);
  }
}

// F4(x) = (F_x, F_y, F_z, 0) with F_c = (phi(x - e_c) - phi(x + e_c)) *
// inv_2res, periodic: k_gradient for the float4-per-site layout of the
// differentiable chain.
__global__ void k_gradient4(const float* __restrict__ phi, float4* __restrict__ F4, Geom g,
                            float inv_2res)
{
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int rows = n1 * n2;
  for (int row = blockIdx.x; row < rows; row += gridDim.x) {
    const int y = row % n1, z = row / n1;
    const int yp = y + 1 == n1 ? 0 : y + 1, ym = y == 0 ? n1 - 1 : y - 1;
    const int zp = z + 1 == n2 ? 0 : z + 1, zm = z == 0 ? n2 - 1 : z - 1;
    const float* pr = phi + (int64_t)row * n0;
    const float* pyp = phi + ((int64_t)z * n1 + yp) * n0;
    const float* pym = phi + ((int64_t)z * n1 + ym) * n0;
    const float* pzp = phi + ((int64_t)zp * n1 + y) * n0;
    const float* pzm = phi + ((int64_t)zm * n1 + y) * n0;
    for (int x = threadIdx.x; x < n0; x += blockDim.x) {
      const int xp = x + 1 == n0 ? 0 : x + 1, xm = x == 0 ? n0 - 1 : x - 1;
      F4[(int64_t)row * n0 + x] = make_float4((pr[xm] - pr[xp]) * inv_2res,
                                              (pym[x] - pyp[x]) * inv_2res,
                                              (pzm[x] - pzp[x]) * inv_2res, 0.0f);
    }
  }
}

// Adjoint of k_gradient4: phi enters F_c(y + e_c) with +inv_2res and
// F_c(y - e_c) with -inv_2res, so
// g_phi(y) = inv_2res sum_c (g_F_c(y + e_c) - g_F_c(y - e_c)).
// The fourth component of g_F4 is not read.
__global__ void k_divergence4(const float4* __restrict__ gF4, float* __restrict__ gphi, Geom g,
                              float inv_2res)
{
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int rows = n1 * n2;
  for (int row = blockIdx.x; row < rows; row += gridDim.x) {
    const int y = row % n1, z = row / n1;
    const int yp = y + 1 == n1 ? 0 : y + 1, ym = y == 0 ? n1 - 1 : y - 1;
    const int zp = z + 1 == n2 ? 0 : z + 1, zm = z == 0 ? n2 - 1 : z - 1;
    const float4* r = gF4 + (int64_t)row * n0;
    const float4* ryp = gF4 + ((int64_t)z * n1 + yp) * n0;
    const float4* rym = gF4 + ((int64_t)z * n1 + ym) * n0;
    const float4* rzp = gF4 + ((int64_t)zp * n1 + y) * n0;
    const float4* rzm = gF4 + ((int64_t)zm * n1 + y) * n0;
    for (int x = threadIdx.x; x < n0; x += blockDim.x) {
      const int xp = x + 1 == n0 ? 0 : x + 1, xm = x == 0 ? n0 - 1 : x - 1;
      const float d = (r[xp].x - r[xm].x) + (ryp[x].y - rym[x].y) + (rzp[x].z - rzm[x].z);
      gphi[(int64_t)row * n0 + x] = d * inv_2res;
    }
  }
}

// dst += src over n floats.
__global__ void k_accumulate(float* __restrict__ dst, const float* __restrict__ src, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Plans and scratch of the PM operator; lattices up to 1024^3 (k_green's
// 32-bit k indices).
lf2_status pm_prepare(lf2_ctx* c, const char* who, bool real_scratch)
{
  FFT_TRY(ensure_plans(c));
  if (c->g.n[0] > 1024)
    return fft_fail(c, LF2_ERR_ARG, std::string(who) + ": lattices up to 1024^3 (32-bit k indices)");
  return ensure_scratch(c, real_scratch);
}

// dst = coupling-scaled Green's-function solve of src: R2C into fft_k,
// k_green, C2R into dst.  dst may be src.
lf2_status green_solve(lf2_ctx* c, const float* src, float* dst, double coupling)
{
  const int n = c->g.n[0], nkx = n / 2 + 1;
  FFT_CUFFT(c, cufftExecR2C(c->fft_r2c, const_cast<float*>(src),
                            reinterpret_cast<cufftComplex*>(c->fft_k)));
  const float coef = (float)(-coupling * c->res * c->res / (4.0 * (double)c->g.nsites));
  const int64_t pairs = (int64_t)n * n * nkx / 2;
  c->launches += 1;
  k_green<<<grid_for((pairs + GREEN_ITEMS - 1) / GREEN_ITEMS, 256), 256, sizeof(float) * n,
            c->stream>>>(reinterpret_cast<float2*>(c->fft_k), n, n, nkx, 0, coef);
  FFT_CUDA(c, cudaGetLastError());
  FFT_CUFFT(c, cufftExecC2R(c->fft_c2r, reinterpret_cast<cufftComplex*>(c->fft_k), dst));
  return LF2_OK;
}

}  // namespace

void fft_release(lf2_ctx* c)
{
  if (c->fft_planned) {
    cufftDestroy(c->fft_r2c);
    cufftDestroy(c->fft_c2r);
    c->fft_planned = false;
  }
  cudaFree(c->fft_k);
  cudaFree(c->fft_phi);
  c->fft_k = nullptr;
  c->fft_phi = nullptr;
}

}  // namespace lf2

extern "C" {

lf2_status lf2_kfield_create(lf2_ctx* c, int comps, lf2_kfield* out)
{
  if (!c || !out || comps < 1 || comps > 64) return LF2_ERR_ARG;
  lf2_kfield k = new (std::nothrow) lf2_kfield_s();
  if (!k) return LF2_ERR_NOMEM;
  k->comps = comps;
  const size_t bytes = sizeof(float2) * (size_t)comps * (size_t)k_sites(c);
  if (cudaMalloc(&k->data, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete k;
    return fft_fail(c, LF2_ERR_NOMEM, "cannot allocate k-field");
  }
  FFT_CUDA(c, cudaMemsetAsync(k->data, 0, bytes, c->stream));
  *out = k;
  return LF2_OK;
}

lf2_status lf2_kfield_destroy(lf2_ctx* c, lf2_kfield k)
{
  if (!k) return LF2_OK;
  if (c) cudaStreamSynchronize(c->stream);
  cudaFree(k->data);
  delete k;
  return LF2_OK;
}

lf2_status lf2_kfield_export(lf2_ctx* c, lf2_kfield k, void* dst, int real_bytes, int ptr_kind)
{
  if (!c || !k || !k->data || !dst || (real_bytes != 4 && real_bytes != 8) ||
      (ptr_kind != LF2_PTR_HOST && ptr_kind != LF2_PTR_DEVICE))
    return LF2_ERR_ARG;
  const int64_t total = k_sites(c) * k->comps;
  const size_t bytes = (size_t)total * 2 * real_bytes;
  void* d = dst;
  if (ptr_kind == LF2_PTR_HOST) FFT_CUDA(c, cudaMallocAsync(&d, bytes, c->stream));
  const int n = c->g.n[0], nkx = c->g.n[0] / 2 + 1;
  c->launches += 1;
  if (real_bytes == 4)
    k_kexport<float><<<grid_for(total, 256), 256, 0, c->stream>>>(k->data, k->comps, n, nkx,
                                                                  (float*)d);
  else
    k_kexport<double><<<grid_for(total, 256), 256, 0, c->stream>>>(k->data, k->comps, n, nkx,
                                                                   (double*)d);
  cudaError_t e = cudaGetLastError();
  if (ptr_kind == LF2_PTR_HOST) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(d, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  }
  FFT_CUDA(c, e);
  return LF2_OK;
}

lf2_status lf2_kfield_import(lf2_ctx* c, lf2_kfield k, const void* src, int real_bytes,
                             int ptr_kind)
{
  if (!c || !k || !k->data || !src || (real_bytes != 4 && real_bytes != 8) ||
      (ptr_kind != LF2_PTR_HOST && ptr_kind != LF2_PTR_DEVICE))
    return LF2_ERR_ARG;
  const int64_t total = k_sites(c) * k->comps;
  const size_t bytes = (size_t)total * 2 * real_bytes;
  void* d = const_cast<void*>(src);
  if (ptr_kind == LF2_PTR_HOST) {
    FFT_CUDA(c, cudaMallocAsync(&d, bytes, c->stream));
    const cudaError_t e = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) {
      cudaFreeAsync(d, c->stream);
      FFT_CUDA(c, e);
    }
  }
  const int n = c->g.n[0], nkx = c->g.n[0] / 2 + 1;
  c->launches += 1;
  if (real_bytes == 4)
    k_kimport<float><<<grid_for(total, 256), 256, 0, c->stream>>>(k->data, k->comps, n, nkx,
                                                                  (const float*)d);
  else
    k_kimport<double><<<grid_for(total, 256), 256, 0, c->stream>>>(k->data, k->comps, n, nkx,
                                                                   (const double*)d);
  const cudaError_t e = cudaGetLastError();
  if (ptr_kind == LF2_PTR_HOST) cudaFreeAsync(d, c->stream);
  FFT_CUDA(c, e);
  return LF2_OK;
}

lf2_status lf2_fft_forward(lf2_ctx* c, lf2_field r, lf2_kfield k)
{
  if (!c || !k || !k->data || !field_ok(r, k->comps)) return LF2_ERR_ARG;
  FFT_TRY(ensure_plans(c));
  const int64_t nk = k_sites(c);
  for (int comp = 0; comp < k->comps; comp++)
    FFT_CUFFT(c, cufftExecR2C(c->fft_r2c, r->data + (size_t)comp * c->g.nsites,
                              reinterpret_cast<cufftComplex*>(k->data + (size_t)comp * nk)));
  return LF2_OK;
}

lf2_status lf2_fft_backward(lf2_ctx* c, lf2_kfield k, lf2_field r)
{
  if (!c || !k || !k->data || !field_ok(r, k->comps)) return LF2_ERR_ARG;
  FFT_TRY(ensure_plans(c));
  FFT_TRY(ensure_scratch(c, false));
  const int64_t nk = k_sites(c);
  // cuFFT's C2R overwrites its input; the reference keeps the k-field.
  for (int comp = 0; comp < k->comps; comp++) {
    FFT_CUDA(c, cudaMemcpyAsync(c->fft_k, k->data + (size_t)comp * nk, sizeof(float2) * nk,
                                cudaMemcpyDeviceToDevice, c->stream));
    FFT_CUFFT(c, cufftExecC2R(c->fft_c2r, reinterpret_cast<cufftComplex*>(c->fft_k),
                              r->data + (size_t)comp * c->g.nsites));
  }
  return LF2_OK;
}

lf2_status lf2_pm_force(lf2_ctx* c, lf2_field rho, lf2_field phi, lf2_field F, double coupling)
{
  if (!c || !field_ok(rho, 1) || !field_ok(F, 3) || (phi && !field_ok(phi, 1)))
    return LF2_ERR_ARG;
  FFT_TRY(pm_prepare(c, "lf2_pm_force", phi == nullptr));
  float* p = phi ? phi->data : c->fft_phi;
  FFT_TRY(green_solve(c, rho->data, p, coupling));
  c->launches += 1;
  const int grows = c->g.n[1] * c->g.n[2];
  const unsigned gblocks = grows < 148 * 8 ? grows : 148 * 8;
  const bool vec = c->g.n[0] % 4 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(F->data) & 15) == 0;
  const int gthreads = vec ? 128 : 256;
  if (vec)
    k_gradient<true><<<gblocks, gthreads, 0, c->stream>>>(p, F->data, c->g, (float)(0.5 / c->res));
  else
    k_gradient<false><<<gblocks, gthreads, 0, c->stream>>>(p, F->data, c->g, (float)(0.5 / c->res));
  FFT_CUDA(c, cudaGetLastError());
  return LF2_OK;
}

lf2_status lf2_pm_force4(lf2_ctx* c, const float* rho, float* F4, double coupling)
{
  if (!c || !rho || !F4 || !aligned16(F4)) return LF2_ERR_ARG;
  FFT_TRY(pm_prepare(c, "lf2_pm_force4", true));
  FFT_TRY(green_solve(c, rho, c->fft_phi, coupling));
  const int grows = c->g.n[1] * c->g.n[2];
  c->launches += 1;
  k_gradient4<<<grows < 148 * 8 ? grows : 148 * 8, 256, 0, c->stream>>>(
      c->fft_phi, reinterpret_cast<float4*>(F4), c->g, (float)(0.5 / c->res));
  FFT_CUDA(c, cudaGetLastError());
  return LF2_OK;
}

lf2_status lf2_pm_force4_adjoint(lf2_ctx* c, const float* g_F4, float* g_rho, double coupling)
{
  if (!c || !g_F4 || !g_rho || !aligned16(g_F4)) return LF2_ERR_ARG;
  FFT_TRY(pm_prepare(c, "lf2_pm_force4_adjoint", true));
  const int grows = c->g.n[1] * c->g.n[2];
  c->launches += 1;
  k_divergence4<<<grows < 148 * 8 ? grows : 148 * 8, 256, 0, c->stream>>>(
      reinterpret_cast<const float4*>(g_F4), c->fft_phi, c->g, (float)(0.5 / c->res));
  FFT_CUDA(c, cudaGetLastError());
  // The Green's-function solve is a convolution with a real, even kernel:
  // its own adjoint.  R2C reads fft_phi before C2R writes it back.
  FFT_TRY(green_solve(c, c->fft_phi, c->fft_phi, coupling));
  c->launches += 1;
  k_accumulate<<<grid_for(c->g.nsites, 256), 256, 0, c->stream>>>(g_rho, c->fft_phi,
                                                                   c->g.nsites);
  FFT_CUDA(c, cudaGetLastError());
  return LF2_OK;
}

lf2_status lf2_pm_gradient(lf2_ctx* c, lf2_field phi, lf2_field F)
{
  if (!c || !field_ok(phi, 1) || !field_ok(F, 3)) return LF2_ERR_ARG;
  c->launches += 1;
  const int grows = c->g.n[1] * c->g.n[2];
  k_gradient<false><<<grows < 148 * 8 ? grows : 148 * 8, 256, 0, c->stream>>>(
      phi->data, F->data, c->g, (float)(0.5 / c->res));
  FFT_CUDA(c, cudaGetLastError());
  return LF2_OK;
}

lf2_status lf2_slab_fft_destroy(lf2_slab_fft p)
{
  if (!p) return LF2_OK;
  if (p->c) cudaStreamSynchronize(p->c->stream);
  if (p->planned & 1) cufftDestroy(p->r2c);
  if (p->planned & 2) cufftDestroy(p->c2r);
  if (p->planned & 4) cufftDestroy(p->lines);
  delete p;
  return LF2_OK;
}

lf2_status lf2_slab_fft_create(lf2_ctx* c, int n, int nz, int nky, lf2_slab_fft* out)
{
  if (!c || !out || n < 2 || n > 1024 || nz < 1 || nz > n || nky < 1 || nky > n)
    return LF2_ERR_ARG;
  if (c->g.n[0] != n || c->g.n[1] != n)
    return fft_fail(c, LF2_ERR_ARG, "lf2_slab_fft_create: the planes must be n x n");
  lf2_slab_fft p = new (std::nothrow) lf2_slab_fft_s();
  if (!p) return LF2_ERR_NOMEM;
  p->c = c;
  p->n = n;
  p->nz = nz;
  p->nky = nky;
  p->nkx = n / 2 + 1;
  int dims[2] = {n, n};
  int line[1] = {n};
  const int S = nky * p->nkx;
  cufftResult r = cufftPlanMany(&p->r2c, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, nz);
  if (r == CUFFT_SUCCESS) {
    p->planned |= 1;
    r = cufftPlanMany(&p->c2r, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, nz);
  }
  if (r == CUFFT_SUCCESS) {
    p->planned |= 2;
    r = cufftPlanMany(&p->lines, 1, line, line, S, 1, line, S, 1, CUFFT_C2C, S);
  }
  if (r == CUFFT_SUCCESS) p->planned |= 4;
  if (r != CUFFT_SUCCESS) {
    lf2_slab_fft_destroy(p);
    return fft_fail(c, LF2_ERR_CUDA, "lf2_slab_fft_create: cuFFT status " + std::to_string((int)r));
  }
  *out = p;
  return LF2_OK;
}

lf2_status lf2_slab_fft_planes_r2c(lf2_slab_fft p, const float* planes, void* A)
{
  if (!p || !planes || !A) return LF2_ERR_ARG;
  lf2_ctx* c = p->c;
  FFT_CUFFT(c, cufftSetStream(p->r2c, c->stream));
  FFT_CUFFT(c, cufftExecR2C(p->r2c, const_cast<float*>(planes),
                            reinterpret_cast<cufftComplex*>(A)));
  return LF2_OK;
}

lf2_status lf2_slab_fft_planes_c2r(lf2_slab_fft p, void* A, float* planes)
{
  if (!p || !planes || !A) return LF2_ERR_ARG;
  lf2_ctx* c = p->c;
  FFT_CUFFT(c, cufftSetStream(p->c2r, c->stream));
  FFT_CUFFT(c, cufftExecC2R(p->c2r, reinterpret_cast<cufftComplex*>(A), planes));
  return LF2_OK;
}

lf2_status lf2_slab_fft_lines(lf2_slab_fft p, void* B, int direction)
{
  if (!p || !B || (direction != LF2_FFT_FORWARD && direction != LF2_FFT_BACKWARD))
    return LF2_ERR_ARG;
  lf2_ctx* c = p->c;
  FFT_CUFFT(c, cufftSetStream(p->lines, c->stream));
  cufftComplex* b = reinterpret_cast<cufftComplex*>(B);
  FFT_CUFFT(c, cufftExecC2C(p->lines, b, b,
                            direction == LF2_FFT_FORWARD ? CUFFT_FORWARD : CUFFT_INVERSE));
  return LF2_OK;
}

lf2_status lf2_slab_green(lf2_slab_fft p, void* B, int ky0, double coupling)
{
  if (!p || !B || ky0 < 0 || ky0 + p->nky > p->n || !aligned16(B)) return LF2_ERR_ARG;
  lf2_ctx* c = p->c;
  const int n = p->n;
  const double res = c->res;
  const float coef = (float)(-coupling * res * res / (4.0 * (double)n * n * n));
  const int64_t pairs = (int64_t)n * p->nky * p->nkx / 2;
  c->launches += 1;
  k_green<<<grid_for((pairs + GREEN_ITEMS - 1) / GREEN_ITEMS, 256), 256, sizeof(float) * n,
            c->stream>>>(reinterpret_cast<float2*>(B), n, p->nky, p->nkx, ky0, coef);
  FFT_CUDA(c, cudaGetLastError());
  return LF2_OK;
}

}  // extern "C"
