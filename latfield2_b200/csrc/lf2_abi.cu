// lf2_abi.cu -- implementation of the C ABI declared in include/lf2gpu.h.
//
// Host-side orchestration only: argument checks, device allocation owned by
// the context, host<->device staging of borrowed host arrays, and the kernel
// sequences of each call.  All kernels live in lf2_store.cu, lf2_move.cu,
// lf2_deposit.cu and lf2_field.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "lf2_internal.h"

namespace lf2 {
size_t deposit_spill_slots(const lf2_ctx* c, int comps);
}

using namespace lf2;

namespace {

lf2_status fail(lf2_ctx* c, lf2_status code, const std::string& msg)
{
  if (c) c->err = msg;
  return code;
}

#define LF2_CUDA(c, expr)                                                              \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail((c), LF2_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
  } while (0)

#define LF2_TRY(expr)                    \
  do {                                   \
    lf2_status s_ = (expr);              \
    if (s_ != LF2_OK) return s_;         \
  } while (0)

// Stream-ordered device scratch, released on the context's stream.
struct Scratch {
  lf2_ctx* c;
  void* p = nullptr;
  Scratch(lf2_ctx* ctx) : c(ctx) {}
  cudaError_t alloc(size_t bytes)
  {
    return cudaMallocAsync(&p, bytes > 0 ? bytes : 16, c->stream);
  }
  ~Scratch()
  {
    if (p) cudaFreeAsync(p, c->stream);
  }
};

// Brackets one phase of a call with CUDA events on the context's stream when
// profiling is on, and attributes the kernels launched inside it.
cudaEvent_t take_event(lf2_ctx* c)
{
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

struct PhaseScope {
  lf2_ctx* c;
  int phase;
  int64_t l0;
  cudaEvent_t e0 = nullptr;
  PhaseScope(lf2_ctx* ctx, int ph) : c(ctx), phase(ph), l0(ctx->launches)
  {
    if (c->profiling) {
      e0 = take_event(c);
      if (e0) cudaEventRecord(e0, c->stream);
    }
  }
  ~PhaseScope()
  {
    c->phase_launches[phase] += c->launches - l0;
    if (e0) {
      cudaEvent_t e1 = take_event(c);
      if (e1) {
        cudaEventRecord(e1, c->stream);
        c->pending[phase].push_back({e0, e1});
      }
    }
  }
};

enum { PH_MOVE = 0, PH_INSERT = 1, PH_DEPOSIT = 2, PH_FIXUP = 3, PH_OTHER = 4 };

int bits_for(int n)
{
  int b = 0;
  while ((1ll << b) < n) b++;
  return b;
}

void free_parts(PartArrays& a)
{
  cudaFree(a.key);
  cudaFree(a.ox);
  cudaFree(a.oy);
  cudaFree(a.oz);
  cudaFree(a.vx);
  cudaFree(a.vy);
  cudaFree(a.vz);
  cudaFree(a.mass);
  cudaFree(a.id);
  a = PartArrays();
}

cudaError_t alloc_parts(PartArrays& a, int64_t slots, bool mass, bool id)
{
  const size_t n = (size_t)(slots > 0 ? slots : 1);
  cudaError_t e;
  if ((e = cudaMalloc(&a.key, n * sizeof(uint32_t))) != cudaSuccess) return e;
  float** fs[6] = {&a.ox, &a.oy, &a.oz, &a.vx, &a.vy, &a.vz};
  for (auto f : fs)
    if ((e = cudaMalloc(f, n * sizeof(float))) != cudaSuccess) return e;
  if (mass && (e = cudaMalloc(&a.mass, n * sizeof(float))) != cudaSuccess) return e;
  if (id && (e = cudaMalloc(&a.id, n * sizeof(int64_t))) != cudaSuccess) return e;
  return cudaSuccess;
}

lf2_status check_flags(lf2_ctx* c)
{
  LF2_CUDA(c, cudaMemcpyAsync(c->h_flags, c->flags, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  const uint32_t f = *c->h_flags & ~(uint32_t)ERR_REPACK;
  if (f) {
    char buf[160];
    snprintf(buf, sizeof buf,
             "device error flags 0x%x (1 non-finite state, 2 bad cell/offset, 4 mass range, "
             "16 capacity, 32 fixed overflow)",
             f);
    return fail(c, LF2_ERR_STATE, buf);
  }
  return LF2_OK;
}

lf2_status ensure_spill(lf2_ctx* c, size_t need)
{
  if (need <= c->spill_slots) return LF2_OK;
  if (c->spill) {
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(c->spill);
    c->spill = nullptr;
    c->spill_slots = 0;
  }
  if (cudaMalloc(&c->spill, need * sizeof(uint64_t)) != cudaSuccess)
    return fail(c, LF2_ERR_NOMEM, "cannot allocate the deposit shell store");
  c->spill_slots = need;
  return LF2_OK;
}

bool valid_field(lf2_ctx* c, lf2_field f) { return c && f && f->data; }

// Common load path: inputs already on the device.
// Slots of the mover buffer for a store loaded with n particles: every
// particle may change brick in one step, and later inserts may grow the store
// to the largest size that fits_store still accepts (about 1.11 n).
static int64_t mover_slots(int64_t n, int64_t nb) { return n + (n >> 3) + 64 * nb + 1024; }

// Whether a store of `total` particles fits the current allocation without a
// reload: the mover buffer holds every particle, and a repack lays each brick
// out at cap_of(count) <= count + count/8 + 35 slots, so it always fits.
static bool fits_store(const lf2_ctx* c, int64_t total)
{
  return total <= c->mov_capacity && total + (total >> 3) + 36 * c->g.nbricks <= c->capacity;
}

lf2_status load_device(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                       const float* vel3, const float* mass, double gmass, const int64_t* id)
{
  const bool has_mass = mass != nullptr, has_id = id != nullptr;
  const int64_t nb = c->g.nbricks;
  // segments (count + slack, rounded to 4) plus a relocation region of about
  // the same size as the slack
  const int64_t need = n + (n >> 2) + 100 * nb + 1024;
  const int64_t mov_need = mover_slots(n, nb);
  // the kernels index slots with 32-bit integers
  if (need > (int64_t)UINT32_MAX)
    return fail(c, LF2_ERR_UNSUPPORTED, "the particle store is limited to 2^32 - 1 slots (" +
                                            std::to_string(n) + " particles requested)");
  if (need > c->capacity || has_mass != c->has_mass || has_id != c->has_id ||
      mov_need > c->mov_capacity) {
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
    free_parts(c->cur);
    free_parts(c->alt);
    free_parts(c->mov);
    cudaFree(c->mov_placed);
    c->mov_placed = nullptr;
    c->capacity = c->mov_capacity = 0;
    if (alloc_parts(c->cur, need, has_mass, has_id) != cudaSuccess ||
        alloc_parts(c->alt, need, has_mass, has_id) != cudaSuccess ||
        alloc_parts(c->mov, mov_need, has_mass, has_id) != cudaSuccess ||
        cudaMalloc(&c->mov_placed, sizeof(int32_t) * (size_t)mov_need) != cudaSuccess) {
      cudaGetLastError();
      return fail(c, LF2_ERR_NOMEM, "cannot allocate the particle store");
    }
    c->capacity = need;
    c->mov_capacity = mov_need;
  }
  c->has_mass = has_mass;
  c->has_id = has_id;
  c->gmass = gmass;
  LF2_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(uint32_t), c->stream));
  LF2_CUDA(c, cudaMemsetAsync(c->count, 0, sizeof(int32_t) * nb, c->stream));
  LF2_CUDA(c, cudaMemsetAsync(c->fill, 0, sizeof(int32_t) * nb, c->stream));
  LF2_CUDA(c, launch_load_count(c, n, cell, off3));
  LF2_CUDA(c, launch_caps_and_scan(c, c->count, c->cap, c->seg_start, nullptr));
  LF2_CUDA(c, launch_load_scatter(c, n, cell, off3, vel3, mass, id));
  LF2_CUDA(c, cudaMemcpyAsync(c->count, c->fill, sizeof(int32_t) * nb, cudaMemcpyDeviceToDevice,
                              c->stream));
  LF2_CUDA(c, launch_heap_reset(c));
  c->np = n;
  if (check_flags(c) != LF2_OK) {
    c->np = 0;
    LF2_CUDA(c, cudaMemsetAsync(c->count, 0, sizeof(int32_t) * nb, c->stream));
    return fail(c, LF2_ERR_ARG, "particles_set: a cell index or offset is out of range");
  }
  c->m_unit = gmass > 0 ? gmass : 1.0;
  if (has_mass) {
    LF2_CUDA(c, launch_conservation(c));
    LF2_CUDA(c, cudaMemcpyAsync(c->h_stats, c->stats, sizeof(double) * 8, cudaMemcpyDeviceToHost,
                                c->stream));
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
    c->m_unit = (n > 0 && c->h_stats[1] > 0) ? c->h_stats[1] / (double)n : 1.0;
  }
  return LF2_OK;
}

template <typename T>
lf2_status stage_in(lf2_ctx* c, Scratch& s, const T* src, size_t count, int ptr_kind, const T** out)
{
  if (!src) {
    *out = nullptr;
    return LF2_OK;
  }
  if (ptr_kind == LF2_PTR_DEVICE) {
    *out = src;
    return LF2_OK;
  }
  LF2_CUDA(c, s.alloc(count * sizeof(T)));
  LF2_CUDA(c, cudaMemcpyAsync(s.p, src, count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  *out = (const T*)s.p;
  return LF2_OK;
}

}  // namespace

extern "C" {

lf2_status lf2_create(lf2_ctx** out, int device, const int n[3], const double box[3],
                      int deposit_mode, void* stream)
{
  if (!out || !n || !box) return LF2_ERR_ARG;
  *out = nullptr;
  for (int d = 0; d < 3; d++)
    if (n[d] < 1 || !(box[d] > 0)) return LF2_ERR_ARG;
  if (deposit_mode != LF2_DEPOSIT_FP32 && deposit_mode != LF2_DEPOSIT_FIXED64 &&
      deposit_mode != LF2_DEPOSIT_FP32_PLAIN)
    return LF2_ERR_ARG;
  // get_lattice_resolution (particles_tools.hpp:6-19) demands equal
  // resolutions; equal here means to 1e-12 relative, so that box = res * n
  // computed in floating point is accepted for any n.
  const double res = box[0] / n[0];
  if (std::fabs(box[1] / n[1] - res) > 1e-12 * res || std::fabs(box[2] / n[2] - res) > 1e-12 * res)
    return LF2_ERR_ARG;
  const int bits = bits_for(n[0]) + bits_for(n[1]) + bits_for(n[2]);
  const int64_t nsites = (int64_t)n[0] * n[1] * n[2];
  if (bits > 32 || nsites >= (1ll << 31)) return LF2_ERR_UNSUPPORTED;

  lf2_ctx* c = new (std::nothrow) lf2_ctx();
  if (!c) return LF2_ERR_NOMEM;
  c->device = device;
  c->stream = (cudaStream_t)stream;
  c->mode = deposit_mode;
  c->res = res;
  for (int d = 0; d < 3; d++) c->box[d] = box[d];
  Geom& g = c->g;
  int shift = 0;
  for (int d = 0; d < 3; d++) {
    g.n[d] = n[d];
    g.nb[d] = (n[d] + BRICK - 1) / BRICK;
    g.shift[d] = shift;
    const int b = bits_for(n[d]);
    g.mask[d] = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
    shift += b;
  }
  g.nsites = nsites;
  g.nbricks = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
  const int64_t nb = g.nbricks;

  bool ok = cudaSetDevice(device) == cudaSuccess;
  ok = ok && cudaMalloc(&c->seg_start, sizeof(int64_t) * (nb + 1)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->seg_start_alt, sizeof(int64_t) * (nb + 1)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->count, sizeof(int32_t) * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->cap, sizeof(int32_t) * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->cap_alt, sizeof(int32_t) * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->fill, sizeof(int32_t) * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->brick_maxv2, sizeof(float) * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->brick_sums, sizeof(double) * 7 * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->stats, sizeof(double) * 8) == cudaSuccess;
  ok = ok && cudaMalloc(&c->mov_count, sizeof(unsigned long long)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->mig, sizeof(unsigned long long) * 4) == cudaSuccess;
  ok = ok && cudaMalloc(&c->flags, sizeof(uint32_t)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->vmax_bits, sizeof(uint32_t)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->redep, sizeof(uint32_t)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->repack, sizeof(int32_t)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->diag, sizeof(unsigned long long) * 3) == cudaSuccess;
  ok = ok && cudaMalloc(&c->heap_top, sizeof(unsigned long long)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->ovf_list, sizeof(int32_t) * nb) == cudaSuccess;
  ok = ok && cudaMalloc(&c->ovf_count, sizeof(int32_t)) == cudaSuccess;
  ok = ok && cudaMalloc(&c->ovf_state, sizeof(int32_t) * nb) == cudaSuccess;
  ok = ok && cudaMallocHost(&c->h_stats, sizeof(double) * 8) == cudaSuccess;
  ok = ok && cudaMallocHost(&c->h_flags, sizeof(uint32_t)) == cudaSuccess;
  ok = ok && cudaMallocHost(&c->h_i64, sizeof(int64_t) * 4) == cudaSuccess;
  ok = ok && cudaMalloc(&c->work, sizeof(int)) == cudaSuccess;
  ok = ok && cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess;
  if (ok) {
    ok = cudaMemsetAsync(c->count, 0, sizeof(int32_t) * nb, c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->cap, 0, sizeof(int32_t) * nb, c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->seg_start, 0, sizeof(int64_t) * (nb + 1), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->flags, 0, sizeof(uint32_t), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->repack, 0, sizeof(int32_t), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->diag, 0, 3 * sizeof(unsigned long long), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->ovf_count, 0, sizeof(int32_t), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->ovf_state, 0, sizeof(int32_t) * nb, c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->heap_top, 0, sizeof(unsigned long long), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->mov_count, 0, sizeof(unsigned long long), c->stream) == cudaSuccess &&
         cudaMemsetAsync(c->brick_maxv2, 0, sizeof(float) * nb, c->stream) == cudaSuccess &&
         cudaStreamSynchronize(c->stream) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    lf2_destroy(c);
    return LF2_ERR_CUDA;
  }
  *out = c;
  return LF2_OK;
}

lf2_status lf2_destroy(lf2_ctx* c)
{
  if (!c) return LF2_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  free_parts(c->cur);
  free_parts(c->alt);
  free_parts(c->mov);
  cudaFree(c->mov_placed);
  cudaFree(c->seg_start);
  cudaFree(c->seg_start_alt);
  cudaFree(c->count);
  cudaFree(c->cap);
  cudaFree(c->cap_alt);
  cudaFree(c->fill);
  cudaFree(c->brick_maxv2);
  cudaFree(c->brick_sums);
  cudaFree(c->stats);
  cudaFree(c->mov_count);
  cudaFree(c->mig);
  cudaFree(c->work);
  cudaFree(c->flags);
  cudaFree(c->vmax_bits);
  cudaFree(c->redep);
  cudaFree(c->repack);
  cudaFree(c->diag);
  cudaFree(c->heap_top);
  cudaFree(c->ovf_list);
  cudaFree(c->ovf_count);
  cudaFree(c->ovf_state);
  cudaFree(c->spill);
  cudaFree(c->stencil_partial);
  cudaFree(c->pm_acc);
  fft_release(c);
  cudaFreeHost(c->h_stats);
  cudaFreeHost(c->h_flags);
  cudaFreeHost(c->h_i64);
  for (auto& v : c->pending)
    for (auto& pr : v) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  delete c;
  return LF2_OK;
}

const char* lf2_last_error(const lf2_ctx* c) { return c ? c->err.c_str() : "null context"; }

lf2_status lf2_set_stream(lf2_ctx* c, void* stream)
{
  if (!c) return LF2_ERR_ARG;
  c->stream = (cudaStream_t)stream;
  return LF2_OK;
}

lf2_status lf2_synchronize(lf2_ctx* c)
{
  if (!c) return LF2_ERR_ARG;
  return check_flags(c);
}

lf2_status lf2_get_flags(lf2_ctx* c, uint32_t* flags, int clear)
{
  if (!c || !flags) return LF2_ERR_ARG;
  LF2_CUDA(c, cudaMemcpyAsync(c->h_flags, c->flags, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  *flags = *c->h_flags;
  if (clear) LF2_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(uint32_t), c->stream));
  return LF2_OK;
}

lf2_status lf2_particles_set(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                             const float* vel3, const float* mass, double global_mass,
                             const int64_t* id, int ptr_kind)
{
  if (!c || n < 0 || (n > 0 && (!cell || !off3 || !vel3))) return LF2_ERR_ARG;
  if (n >= (1ll << 31)) return fail(c, LF2_ERR_UNSUPPORTED, "more than 2^31-1 particles");
  if (!mass && !(global_mass > 0))
    return fail(c, LF2_ERR_ARG, "particles need a mass (global or per particle)");
  Scratch s1(c), s2(c), s3(c), s4(c), s5(c);
  const int32_t* dc;
  const float *doff, *dvel, *dmass;
  const int64_t* did;
  LF2_TRY(stage_in(c, s1, cell, (size_t)n, ptr_kind, &dc));
  LF2_TRY(stage_in(c, s2, off3, (size_t)n * 3, ptr_kind, &doff));
  LF2_TRY(stage_in(c, s3, vel3, (size_t)n * 3, ptr_kind, &dvel));
  LF2_TRY(stage_in(c, s4, mass, (size_t)n, ptr_kind, &dmass));
  LF2_TRY(stage_in(c, s5, id, (size_t)n, ptr_kind, &did));
  return load_device(c, n, dc, doff, dvel, dmass, global_mass, did);
}

lf2_status lf2_particles_set_pos(lf2_ctx* c, int64_t n, const void* pos3, const void* vel3,
                                 int real_bytes, const float* mass, double global_mass,
                                 const int64_t* id)
{
  if (!c || n < 0 || (n > 0 && (!pos3 || !vel3)) || (real_bytes != 4 && real_bytes != 8))
    return LF2_ERR_ARG;
  if (n >= (1ll << 31)) return fail(c, LF2_ERR_UNSUPPORTED, "more than 2^31-1 particles");
  if (!mass && !(global_mass > 0))
    return fail(c, LF2_ERR_ARG, "particles need a mass (global or per particle)");
  std::vector<float> vel((size_t)n * 3);
  for (size_t i = 0; i < vel.size(); i++)
    vel[i] = real_bytes == 8 ? (float)((const double*)vel3)[i] : ((const float*)vel3)[i];
  Scratch sp(c), sc(c), so(c), sv(c), sm(c), si(c);
  LF2_CUDA(c, sp.alloc((size_t)n * 3 * real_bytes));
  LF2_CUDA(c, sc.alloc((size_t)n * sizeof(int32_t)));
  LF2_CUDA(c, so.alloc((size_t)n * 3 * sizeof(float)));
  LF2_CUDA(c, cudaMemcpyAsync(sp.p, pos3, (size_t)n * 3 * real_bytes, cudaMemcpyHostToDevice,
                              c->stream));
  LF2_CUDA(c, launch_pos_to_state(c, n, sp.p, real_bytes, (int32_t*)sc.p, (float*)so.p));
  const float* dvel;
  const float* dmass;
  const int64_t* did;
  LF2_TRY(stage_in(c, sv, vel.data(), vel.size(), LF2_PTR_HOST, &dvel));
  LF2_TRY(stage_in(c, sm, mass, (size_t)n, LF2_PTR_HOST, &dmass));
  LF2_TRY(stage_in(c, si, id, (size_t)n, LF2_PTR_HOST, &did));
  return load_device(c, n, (const int32_t*)sc.p, (const float*)so.p, dvel, dmass, global_mass,
                     did);
}

// Whether the automatic kernel choice fuses the fixed-point deposit into the
// pipelined pass.
#ifndef LF2_FUSED_AUTO
#define LF2_FUSED_AUTO 0
#endif

static lf2_status rebin_tail(lf2_ctx* c);

lf2_status lf2_particles_extract_z(lf2_ctx* c, int z_lo, int z_hi, int64_t capacity,
                                   int32_t* cell, float* off3, float* vel3, float* mass,
                                   int64_t* id, int64_t* n_out)
{
  if (!c || !n_out || capacity < 0 || z_lo > z_hi) return LF2_ERR_ARG;
  if (capacity > 0 && (!cell || !off3 || !vel3)) return LF2_ERR_ARG;
  if (capacity > 0 && ((mass != nullptr) != c->has_mass || (id != nullptr) != c->has_id))
    return fail(c, LF2_ERR_ARG, "extract_z: give mass and id exactly when the store carries them");
  *n_out = 0;
  if (c->np == 0) return LF2_OK;
  LF2_CUDA(c, launch_count_outside(c, z_lo, z_hi, c->mig));
  LF2_CUDA(c, cudaMemcpyAsync(c->h_i64, c->mig, 2 * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  const int64_t n = c->h_i64[0] + c->h_i64[1];
  *n_out = n;
  if (n > capacity)
    return fail(c, LF2_ERR_ARG, "extract_z: " + std::to_string(n) + " particles, capacity " +
                                    std::to_string(capacity));
  if (n == 0) return LF2_OK;
  LF2_CUDA(c, cudaMemsetAsync(c->mig, 0, sizeof(unsigned long long), c->stream));
  LF2_CUDA(c, launch_extract_outside(c, z_lo, z_hi, cell, off3, vel3, mass, id, c->mig));
  c->np -= n;
  return LF2_OK;
}

lf2_status lf2_slab_record_words(lf2_ctx* c, int* words)
{
  if (!c || !words) return LF2_ERR_ARG;
  *words = record_words(c);
  return LF2_OK;
}

lf2_status lf2_slab_count(lf2_ctx* c, int z_lo, int z_hi, int64_t* counts)
{
  if (!c || !counts || z_lo > z_hi) return LF2_ERR_ARG;
  if (c->np == 0) {
    LF2_CUDA(c, cudaMemsetAsync(counts, 0, 4 * sizeof(int64_t), c->stream));
    return LF2_OK;
  }
  LF2_CUDA(c, launch_count_outside(c, z_lo, z_hi, (unsigned long long*)counts, true));
  return LF2_OK;
}

lf2_status lf2_slab_extract(lf2_ctx* c, int z_lo, int z_hi, int64_t n_below, uint32_t* below,
                            int64_t n_above, uint32_t* above)
{
  if (!c || z_lo > z_hi || n_below < 0 || n_above < 0 || (n_below > 0 && !below) ||
      (n_above > 0 && !above))
    return LF2_ERR_ARG;
  if (n_below + n_above > c->np)
    return fail(c, LF2_ERR_ARG, "slab_extract: more particles than the store holds");
  if (c->np == 0) return LF2_OK;
  // launched whatever the counts, so that a particle beyond them is reported
  LF2_CUDA(c, launch_extract_records(c, z_lo, z_hi, n_below, below, n_above, above, c->mig));
  c->np -= n_below + n_above;
  return LF2_OK;
}

lf2_status lf2_slab_insert(lf2_ctx* c, int64_t n_a, const uint32_t* a, int64_t n_b,
                           const uint32_t* b)
{
  if (!c || n_a < 0 || n_b < 0 || (n_a > 0 && !a) || (n_b > 0 && !b)) return LF2_ERR_ARG;
  if (c->capacity == 0)
    return fail(c, LF2_ERR_ARG, "slab_insert: create the store with lf2_particles_set first");
  const int64_t n = n_a + n_b;
  if (n == 0) return LF2_OK;
  if (c->np + n >= (1ll << 31)) return fail(c, LF2_ERR_UNSUPPORTED, "more than 2^31-1 particles");
  const int64_t total = c->np + n;
  if (fits_store(c, total)) {
    // through the mover path, in stream order
    LF2_CUDA(c, launch_pack_records(c, n_a, a, n_b, b));
    LF2_TRY(rebin_tail(c));
    LF2_CUDA(c, cudaMemsetAsync(c->mov_count, 0, sizeof(unsigned long long), c->stream));
    c->np = total;
    return LF2_OK;
  }
  // the store is too small: separate arrays, then the reloading add (it waits)
  Scratch sc(c), so(c), sv(c), sm(c), si(c);
  LF2_CUDA(c, sc.alloc(sizeof(int32_t) * n));
  LF2_CUDA(c, so.alloc(sizeof(float) * 3 * n));
  LF2_CUDA(c, sv.alloc(sizeof(float) * 3 * n));
  if (c->has_mass) LF2_CUDA(c, sm.alloc(sizeof(float) * n));
  if (c->has_id) LF2_CUDA(c, si.alloc(sizeof(int64_t) * n));
  LF2_CUDA(c, launch_unpack_records(c, n_a, a, n_b, b, (int32_t*)sc.p, (float*)so.p, (float*)sv.p,
                                    (float*)sm.p, (int64_t*)si.p));
  return lf2_particles_add(c, n, (const int32_t*)sc.p, (const float*)so.p, (const float*)sv.p,
                           c->has_mass ? (const float*)sm.p : nullptr,
                           c->has_id ? (const int64_t*)si.p : nullptr, LF2_PTR_DEVICE);
}

lf2_status lf2_particles_add(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                             const float* vel3, const float* mass, const int64_t* id,
                             int ptr_kind)
{
  if (!c || n < 0 || (n > 0 && (!cell || !off3 || !vel3))) return LF2_ERR_ARG;
  if (c->capacity == 0)
    return fail(c, LF2_ERR_ARG, "particles_add: create the store with lf2_particles_set first");
  if (n == 0) return LF2_OK;
  if ((mass != nullptr) != c->has_mass || (id != nullptr) != c->has_id)
    return fail(c, LF2_ERR_ARG, "particles_add: give mass and id exactly when the store carries them");
  if (c->np + n >= (1ll << 31)) return fail(c, LF2_ERR_UNSUPPORTED, "more than 2^31-1 particles");
  Scratch s1(c), s2(c), s3(c), s4(c), s5(c);
  const int32_t* dc;
  const float *doff, *dvel, *dmass;
  const int64_t* did;
  LF2_TRY(stage_in(c, s1, cell, (size_t)n, ptr_kind, &dc));
  LF2_TRY(stage_in(c, s2, off3, (size_t)n * 3, ptr_kind, &doff));
  LF2_TRY(stage_in(c, s3, vel3, (size_t)n * 3, ptr_kind, &dvel));
  LF2_TRY(stage_in(c, s4, mass, (size_t)n, ptr_kind, &dmass));
  LF2_TRY(stage_in(c, s5, id, (size_t)n, ptr_kind, &did));
  // check every input first: nothing changes when one is out of range
  LF2_CUDA(c, launch_pack_movers(c, n, dc, doff, dvel, dmass, did, false));
  if (check_flags(c) != LF2_OK) {
    LF2_CUDA(c, cudaMemsetAsync(c->flags, 0, sizeof(uint32_t), c->stream));
    return fail(c, LF2_ERR_ARG, "particles_add: a cell index or offset is out of range");
  }
  const int64_t total = c->np + n;
  if (fits_store(c, total)) {
    // through the mover path: pack, insert
    LF2_CUDA(c, launch_pack_movers(c, n, dc, doff, dvel, dmass, did, true));
    LF2_TRY(rebin_tail(c));
    LF2_CUDA(c, cudaMemsetAsync(c->mov_count, 0, sizeof(unsigned long long), c->stream));
    c->np = total;
    return LF2_OK;
  }
  // the store is too small: reload the current particles and the new ones
  Scratch tc(c), to(c), tv(c), tm(c), ti(c), st(c);
  LF2_CUDA(c, tc.alloc(sizeof(int32_t) * total));
  LF2_CUDA(c, to.alloc(sizeof(float) * 3 * total));
  LF2_CUDA(c, tv.alloc(sizeof(float) * 3 * total));
  if (c->has_mass) LF2_CUDA(c, tm.alloc(sizeof(float) * total));
  if (c->has_id) LF2_CUDA(c, ti.alloc(sizeof(int64_t) * total));
  LF2_CUDA(c, st.alloc(sizeof(int64_t) * (c->g.nbricks + 1)));
  LF2_CUDA(c, launch_scan_counts(c, (int64_t*)st.p));
  LF2_CUDA(c, launch_get(c, (int64_t*)st.p, (int32_t*)tc.p, (float*)to.p, (float*)tv.p,
                         (float*)tm.p, (int64_t*)ti.p));
  const int64_t np0 = c->np;
  const cudaMemcpyKind d2d = cudaMemcpyDeviceToDevice;
  LF2_CUDA(c, cudaMemcpyAsync((int32_t*)tc.p + np0, dc, sizeof(int32_t) * n, d2d, c->stream));
  LF2_CUDA(c, cudaMemcpyAsync((float*)to.p + 3 * np0, doff, sizeof(float) * 3 * n, d2d, c->stream));
  LF2_CUDA(c, cudaMemcpyAsync((float*)tv.p + 3 * np0, dvel, sizeof(float) * 3 * n, d2d, c->stream));
  if (c->has_mass)
    LF2_CUDA(c, cudaMemcpyAsync((float*)tm.p + np0, dmass, sizeof(float) * n, d2d, c->stream));
  if (c->has_id)
    LF2_CUDA(c, cudaMemcpyAsync((int64_t*)ti.p + np0, did, sizeof(int64_t) * n, d2d, c->stream));
  return load_device(c, total, (const int32_t*)tc.p, (const float*)to.p, (const float*)tv.p,
                     (const float*)tm.p, c->gmass, (const int64_t*)ti.p);
}

// Checkpoint file (little endian): int32 "LF2C", int32 version 1,
// int32 n[3], int32 deposit mode, int32 has_mass, int32 has_id (32 bytes),
// double box[3], double global mass, double unit mass of the fixed-point
// deposit, int64 np (80 bytes in all); then np x int32 cell, np x 3 f32
// offsets, np x 3 f32 velocities, [np x f32 mass], [np x int64 id]: the
// store in brick order.
static bool write_all(FILE* f, const void* p, size_t bytes)
{
  return bytes == 0 || fwrite(p, 1, bytes, f) == bytes;
}
static bool read_all(FILE* f, void* p, size_t bytes)
{
  return bytes == 0 || fread(p, 1, bytes, f) == bytes;
}

lf2_status lf2_checkpoint_save(lf2_ctx* c, const char* path)
{
  if (!c || !path) return LF2_ERR_ARG;
  const int64_t n = c->np;
  std::vector<int32_t> cell((size_t)n);
  std::vector<float> off((size_t)n * 3), vel((size_t)n * 3), mass(c->has_mass ? (size_t)n : 0);
  std::vector<int64_t> id(c->has_id ? (size_t)n : 0);
  LF2_TRY(lf2_particles_get(c, cell.data(), off.data(), vel.data(),
                            c->has_mass ? mass.data() : nullptr, c->has_id ? id.data() : nullptr,
                            LF2_PTR_HOST));
  FILE* f = fopen(path, "wb");
  if (!f) return fail(c, LF2_ERR_ARG, std::string("checkpoint_save: cannot open ") + path);
  const int32_t head[8] = {0x4332464c /* "LF2C" */, 1, c->g.n[0], c->g.n[1], c->g.n[2], c->mode,
                           c->has_mass ? 1 : 0, c->has_id ? 1 : 0};
  bool ok = write_all(f, head, sizeof head) && write_all(f, c->box, sizeof(double) * 3) &&
            write_all(f, &c->gmass, sizeof(double)) &&
            write_all(f, &c->m_unit, sizeof(double)) && write_all(f, &n, sizeof(int64_t)) &&
            write_all(f, cell.data(), sizeof(int32_t) * cell.size()) &&
            write_all(f, off.data(), sizeof(float) * off.size()) &&
            write_all(f, vel.data(), sizeof(float) * vel.size()) &&
            write_all(f, mass.data(), sizeof(float) * mass.size()) &&
            write_all(f, id.data(), sizeof(int64_t) * id.size());
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(c, LF2_ERR_ARG, std::string("checkpoint_save: write failed: ") + path);
  return LF2_OK;
}

lf2_status lf2_checkpoint_load(lf2_ctx* c, const char* path)
{
  if (!c || !path) return LF2_ERR_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(c, LF2_ERR_ARG, std::string("checkpoint_load: cannot open ") + path);
  int32_t head[8];
  double box[3], gmass = 0, m_unit = 1;
  int64_t n = 0;
  bool ok = read_all(f, head, sizeof head) && read_all(f, box, sizeof box) &&
            read_all(f, &gmass, sizeof gmass) &&
            read_all(f, &m_unit, sizeof m_unit) && read_all(f, &n, sizeof n);
  if (!ok || head[0] != 0x4332464c || head[1] != 1 || n < 0 || n >= (1ll << 31)) {
    fclose(f);
    return fail(c, LF2_ERR_ARG, std::string("checkpoint_load: not a checkpoint: ") + path);
  }
  if (head[2] != c->g.n[0] || head[3] != c->g.n[1] || head[4] != c->g.n[2] || box[0] != c->box[0] ||
      box[1] != c->box[1] || box[2] != c->box[2] || head[5] != c->mode) {
    fclose(f);
    return fail(c, LF2_ERR_ARG, "checkpoint_load: the checkpoint has another lattice, box or mode");
  }
  const bool has_mass = head[6] != 0, has_id = head[7] != 0;
  std::vector<int32_t> cell((size_t)n);
  std::vector<float> off((size_t)n * 3), vel((size_t)n * 3), mass(has_mass ? (size_t)n : 0);
  std::vector<int64_t> id(has_id ? (size_t)n : 0);
  ok = read_all(f, cell.data(), sizeof(int32_t) * cell.size()) &&
       read_all(f, off.data(), sizeof(float) * off.size()) &&
       read_all(f, vel.data(), sizeof(float) * vel.size()) &&
       read_all(f, mass.data(), sizeof(float) * mass.size()) &&
       read_all(f, id.data(), sizeof(int64_t) * id.size());
  fclose(f);
  if (!ok) return fail(c, LF2_ERR_ARG, std::string("checkpoint_load: truncated: ") + path);
  LF2_TRY(lf2_particles_set(c, n, cell.data(), off.data(), vel.data(),
                            has_mass ? mass.data() : nullptr, gmass, has_id ? id.data() : nullptr,
                            LF2_PTR_HOST));
  c->m_unit = m_unit;  // the fixed-point unit of the saved run, for a bit-exact restart
  return LF2_OK;
}

lf2_status lf2_particles_count(lf2_ctx* c, int64_t* n)
{
  if (!c || !n) return LF2_ERR_ARG;
  *n = c->np;
  return LF2_OK;
}

lf2_status lf2_particles_get(lf2_ctx* c, int32_t* cell, float* off3, float* vel3, float* mass,
                             int64_t* id, int ptr_kind)
{
  if (!c) return LF2_ERR_ARG;
  if ((mass && !c->has_mass) || (id && !c->has_id))
    return fail(c, LF2_ERR_ARG, "mass/id requested but not carried");
  const int64_t n = c->np;
  Scratch st(c), sc(c), so(c), sv(c), sm(c), si(c);
  LF2_CUDA(c, st.alloc(sizeof(int64_t) * (c->g.nbricks + 1)));
  LF2_CUDA(c, launch_scan_counts(c, (int64_t*)st.p));
  int32_t* dc = cell;
  float *doff = off3, *dvel = vel3, *dmass = mass;
  int64_t* did = id;
  if (ptr_kind == LF2_PTR_HOST) {
    if (cell) {
      LF2_CUDA(c, sc.alloc(sizeof(int32_t) * n));
      dc = (int32_t*)sc.p;
    }
    if (off3) {
      LF2_CUDA(c, so.alloc(sizeof(float) * 3 * n));
      doff = (float*)so.p;
    }
    if (vel3) {
      LF2_CUDA(c, sv.alloc(sizeof(float) * 3 * n));
      dvel = (float*)sv.p;
    }
    if (mass) {
      LF2_CUDA(c, sm.alloc(sizeof(float) * n));
      dmass = (float*)sm.p;
    }
    if (id) {
      LF2_CUDA(c, si.alloc(sizeof(int64_t) * n));
      did = (int64_t*)si.p;
    }
  }
  LF2_CUDA(c, launch_get(c, (int64_t*)st.p, dc, doff, dvel, dmass, did));
  if (ptr_kind == LF2_PTR_HOST) {
    const cudaMemcpyKind k = cudaMemcpyDeviceToHost;
    if (cell) LF2_CUDA(c, cudaMemcpyAsync(cell, dc, sizeof(int32_t) * n, k, c->stream));
    if (off3) LF2_CUDA(c, cudaMemcpyAsync(off3, doff, sizeof(float) * 3 * n, k, c->stream));
    if (vel3) LF2_CUDA(c, cudaMemcpyAsync(vel3, dvel, sizeof(float) * 3 * n, k, c->stream));
    if (mass) LF2_CUDA(c, cudaMemcpyAsync(mass, dmass, sizeof(float) * n, k, c->stream));
    if (id) LF2_CUDA(c, cudaMemcpyAsync(id, did, sizeof(int64_t) * n, k, c->stream));
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return LF2_OK;
}

lf2_status lf2_particles_get_pos(lf2_ctx* c, void* pos3, void* vel3, int real_bytes, int64_t* id)
{
  if (!c || (real_bytes != 4 && real_bytes != 8)) return LF2_ERR_ARG;
  if (id && !c->has_id) return fail(c, LF2_ERR_ARG, "id requested but not carried");
  const int64_t n = c->np;
  Scratch st(c), sc(c), so(c), sv(c), sp(c), si(c);
  LF2_CUDA(c, st.alloc(sizeof(int64_t) * (c->g.nbricks + 1)));
  LF2_CUDA(c, sc.alloc(sizeof(int32_t) * n));
  LF2_CUDA(c, so.alloc(sizeof(float) * 3 * n));
  LF2_CUDA(c, sv.alloc(sizeof(float) * 3 * n));
  LF2_CUDA(c, sp.alloc((size_t)real_bytes * 3 * n));
  if (id) LF2_CUDA(c, si.alloc(sizeof(int64_t) * n));
  LF2_CUDA(c, launch_scan_counts(c, (int64_t*)st.p));
  LF2_CUDA(c, launch_get(c, (int64_t*)st.p, (int32_t*)sc.p, (float*)so.p, (float*)sv.p, nullptr,
                         (int64_t*)si.p));
  LF2_CUDA(c, launch_state_to_pos(c, n, (const int32_t*)sc.p, (const float*)so.p, sp.p, real_bytes));
  std::vector<float> vel((size_t)n * 3);
  if (pos3)
    LF2_CUDA(c, cudaMemcpyAsync(pos3, sp.p, (size_t)real_bytes * 3 * n, cudaMemcpyDeviceToHost,
                                c->stream));
  LF2_CUDA(c, cudaMemcpyAsync(vel.data(), sv.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost,
                              c->stream));
  if (id) LF2_CUDA(c, cudaMemcpyAsync(id, si.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  if (vel3)
    for (size_t i = 0; i < vel.size(); i++) {
      if (real_bytes == 8) ((double*)vel3)[i] = vel[i];
      else ((float*)vel3)[i] = vel[i];
    }
  return LF2_OK;
}

lf2_status lf2_cell_counts(lf2_ctx* c, int32_t* counts, int ptr_kind)
{
  if (!c || !counts) return LF2_ERR_ARG;
  Scratch s(c);
  int32_t* d = counts;
  if (ptr_kind == LF2_PTR_HOST) {
    LF2_CUDA(c, s.alloc(sizeof(int32_t) * c->g.nsites));
    d = (int32_t*)s.p;
  }
  LF2_CUDA(c, launch_cell_counts(c, d));
  if (ptr_kind == LF2_PTR_HOST) {
    LF2_CUDA(c, cudaMemcpyAsync(counts, d, sizeof(int32_t) * c->g.nsites, cudaMemcpyDeviceToHost,
                                c->stream));
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return LF2_OK;
}

lf2_status lf2_field_create(lf2_ctx* c, int comps, lf2_field* out)
{
  if (!c || !out || comps < 1 || comps > 64) return LF2_ERR_ARG;
  *out = nullptr;
  lf2_field f = new (std::nothrow) lf2_field_s();
  if (!f) return LF2_ERR_NOMEM;
  f->comps = comps;
  if (cudaMalloc(&f->data, sizeof(float) * comps * c->g.nsites) != cudaSuccess) {
    cudaGetLastError();
    delete f;
    return fail(c, LF2_ERR_NOMEM, "cannot allocate field");
  }
  LF2_CUDA(c, cudaMemsetAsync(f->data, 0, sizeof(float) * comps * c->g.nsites, c->stream));
  *out = f;
  return LF2_OK;
}

lf2_status lf2_field_wrap(lf2_ctx* c, int comps, float* device_data, lf2_field* out)
{
  if (!c || !out || !device_data || comps < 1 || comps > 64) return LF2_ERR_ARG;
  lf2_field f = new (std::nothrow) lf2_field_s();
  if (!f) return LF2_ERR_NOMEM;
  f->comps = comps;
  f->data = device_data;
  f->owned = false;
  *out = f;
  return LF2_OK;
}

lf2_status lf2_field_destroy(lf2_ctx* c, lf2_field f)
{
  if (!f) return LF2_OK;
  if (f->owned) {
    if (c) cudaStreamSynchronize(c->stream);
    cudaFree(f->data);
  }
  delete f;
  return LF2_OK;
}

lf2_status lf2_field_device_ptr(lf2_ctx* c, lf2_field f, float** data)
{
  if (!valid_field(c, f) || !data) return LF2_ERR_ARG;
  *data = f->data;
  return LF2_OK;
}

lf2_status lf2_field_components(lf2_ctx* c, lf2_field f, int* comps)
{
  if (!valid_field(c, f) || !comps) return LF2_ERR_ARG;
  *comps = f->comps;
  return LF2_OK;
}

lf2_status lf2_field_zero(lf2_ctx* c, lf2_field f)
{
  if (!valid_field(c, f)) return LF2_ERR_ARG;
  LF2_CUDA(c, cudaMemsetAsync(f->data, 0, sizeof(float) * f->comps * c->g.nsites, c->stream));
  return LF2_OK;
}

lf2_status lf2_field_export(lf2_ctx* c, lf2_field f, void* dst, int halo, int real_bytes,
                            int fill_halo, int ptr_kind)
{
  if (!valid_field(c, f) || !dst || halo < 0 || (real_bytes != 4 && real_bytes != 8))
    return LF2_ERR_ARG;
  const size_t gross = (size_t)(c->g.n[0] + 2 * halo) * (c->g.n[1] + 2 * halo) *
                       (c->g.n[2] + 2 * halo);
  const size_t bytes = gross * f->comps * real_bytes;
  Scratch s(c);
  void* d = dst;
  if (ptr_kind == LF2_PTR_HOST) {
    LF2_CUDA(c, s.alloc(bytes));
    d = s.p;
  }
  LF2_CUDA(c, launch_export(c, f->comps, f->data, d, halo, real_bytes, fill_halo));
  if (ptr_kind == LF2_PTR_HOST) {
    LF2_CUDA(c, cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return LF2_OK;
}

lf2_status lf2_field_import(lf2_ctx* c, lf2_field f, const void* src, int halo, int real_bytes,
                            int ptr_kind)
{
  if (!valid_field(c, f) || !src || halo < 0 || (real_bytes != 4 && real_bytes != 8))
    return LF2_ERR_ARG;
  const size_t gross = (size_t)(c->g.n[0] + 2 * halo) * (c->g.n[1] + 2 * halo) *
                       (c->g.n[2] + 2 * halo);
  const size_t bytes = gross * f->comps * real_bytes;
  Scratch s(c);
  const void* d = src;
  if (ptr_kind == LF2_PTR_HOST) {
    LF2_CUDA(c, s.alloc(bytes));
    LF2_CUDA(c, cudaMemcpyAsync(s.p, src, bytes, cudaMemcpyHostToDevice, c->stream));
    d = s.p;
  }
  LF2_CUDA(c, launch_import(c, f->comps, f->data, d, halo, real_bytes));
  return LF2_OK;
}

lf2_status lf2_halo_fill(lf2_ctx* c, void* data, int comps, int halo, int real_bytes)
{
  if (!c || !data || comps < 1 || halo < 0 || (real_bytes != 4 && real_bytes != 8))
    return LF2_ERR_ARG;
  for (int d = 0; d < 3; d++)
    if (halo > c->g.n[d]) return fail(c, LF2_ERR_ARG, "halo wider than the lattice");
  LF2_CUDA(c, launch_halo_fill(c, data, comps, halo, real_bytes));
  return LF2_OK;
}

static lf2_status deposit(lf2_ctx* c, lf2_field f, int kind, int comps)
{
  if (!valid_field(c, f)) return LF2_ERR_ARG;
  if (f->comps != comps) return fail(c, LF2_ERR_ARG, "field has the wrong number of components");
  LF2_TRY(ensure_spill(c, kind >= 3 ? deposit_full_spill_slots(c, comps)
                                     : deposit_spill_slots(c, comps)));
  {
    PhaseScope ps(c, PH_DEPOSIT);
    LF2_CUDA(c, kind >= 3 ? launch_deposit_full(c, kind, f->data, 0)
                          : launch_deposit(c, kind, f->data, 0));
  }
  {
    PhaseScope ps(c, PH_FIXUP);
    LF2_CUDA(c, kind >= 3 ? launch_deposit_full(c, kind, f->data, 1)
                          : launch_deposit(c, kind, f->data, 1));
  }
  return LF2_OK;
}

lf2_status lf2_deposit_scalar(lf2_ctx* c, lf2_field rho) { return deposit(c, rho, 0, 1); }
lf2_status lf2_deposit_vector_cicngp(lf2_ctx* c, lf2_field v) { return deposit(c, v, 1, 3); }
lf2_status lf2_deposit_symtensor_cicngp(lf2_ctx* c, lf2_field t) { return deposit(c, t, 2, 6); }
lf2_status lf2_deposit_vector_cic(lf2_ctx* c, lf2_field v) { return deposit(c, v, 3, 3); }
lf2_status lf2_deposit_vecvec_cic(lf2_ctx* c, lf2_field t) { return deposit(c, t, 4, 6); }

// Whether the automatic kernel choice fuses the fixed-point deposit into the
// pipelined pass.
#ifndef LF2_FUSED_AUTO
#define LF2_FUSED_AUTO 0
#endif

static lf2_status rebin_tail(lf2_ctx* c)
{
  PhaseScope ps(c, PH_INSERT);
  LF2_CUDA(c, launch_insert(c));
  LF2_CUDA(c, launch_repack(c));
  return LF2_OK;
}

lf2_status lf2_gather_kick(lf2_ctx* c, lf2_field F, double dtau, double* max_v)
{
  if (!valid_field(c, F)) return LF2_ERR_ARG;
  if (F->comps != 3) return fail(c, LF2_ERR_ARG, "the kick field needs 3 components");
  MoveParams mp{(float)dtau, 0.0f};
  {
    PhaseScope ps(c, PH_MOVE);
    LF2_CUDA(c, launch_move(c, F->data, true, false, mp));
  }
  if (max_v) {
    LF2_CUDA(c, launch_reduce_maxv(c));
    LF2_CUDA(c, cudaMemcpyAsync(c->h_stats, c->stats, sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    LF2_CUDA(c, cudaStreamSynchronize(c->stream));
    *max_v = std::sqrt(c->h_stats[0]);
  }
  return LF2_OK;
}

lf2_status lf2_drift_rebin(lf2_ctx* c, double dtau)
{
  if (!c) return LF2_ERR_ARG;
  MoveParams mp{0.0f, (float)(dtau / c->res)};
  LF2_CUDA(c, cudaMemsetAsync(c->mov_count, 0, sizeof(unsigned long long), c->stream));
  {
    PhaseScope ps(c, PH_MOVE);
    LF2_CUDA(c, launch_move(c, nullptr, false, true, mp));
  }
  return rebin_tail(c);
}

lf2_status lf2_step(lf2_ctx* c, lf2_field F, double dtau_kick, double dtau_drift, lf2_field rho)
{
  if (!valid_field(c, F)) return LF2_ERR_ARG;
  if (F->comps != 3) return fail(c, LF2_ERR_ARG, "the kick field needs 3 components");
  MoveParams mp{(float)dtau_kick, (float)(dtau_drift / c->res)};
  LF2_CUDA(c, cudaMemsetAsync(c->mov_count, 0, sizeof(unsigned long long), c->stream));
  if ((c->move_kernel == 2 || c->move_kernel == 3) && !move_pipe_eligible(c, F->data))
    return fail(c, LF2_ERR_UNSUPPORTED, "pipelined move needs n0 % 4 == 0, n >= 32, aligned F");
  if (c->move_kernel == 3 && !move_dep_eligible(c, F->data))
    return fail(c, LF2_ERR_UNSUPPORTED, "the fused deposit needs the fixed-point mode and room "
                                        "for its tile");
  const bool pipe = c->move_kernel >= 2 || (c->move_kernel == 0 && move_pipe_eligible(c, F->data));
  // the fixed-point scalar deposit fused into the pipelined pass (automatic
  // when eligible, or kernel 3), finished by the movers' rim atomics and the
  // rim fix-up; redone by the tile pass if a mover went past the rim
  const bool fused = rho && valid_field(c, rho) && rho->comps == 1 && pipe &&
                     (c->move_kernel == 3 || (c->move_kernel == 0 && LF2_FUSED_AUTO)) &&
                     move_dep_eligible(c, F->data);
  c->last_move_kernel = fused ? 3 : (pipe ? 2 : 1);
  if (!fused) {
    {
      PhaseScope ps(c, PH_MOVE);
      LF2_CUDA(c, pipe ? launch_move_pipe(c, F->data, mp, nullptr)
                       : launch_move(c, F->data, true, true, mp));
    }
    LF2_TRY(rebin_tail(c));
    if (rho) LF2_TRY(deposit(c, rho, 0, 1));
    return LF2_OK;
  }
  LF2_TRY(ensure_spill(c, std::max(rim_store_slots(c), deposit_spill_slots(c, 1))));
  LF2_CUDA(c, cudaMemsetAsync(c->redep, 0, sizeof(uint32_t), c->stream));
  {
    PhaseScope ps(c, PH_MOVE);
    LF2_CUDA(c, launch_move_pipe(c, F->data, mp, rho->data));
  }
  {
    PhaseScope ps(c, PH_FIXUP);
    LF2_CUDA(c, launch_dep_movers(c));
    LF2_CUDA(c, launch_fixup_rim(c, rho->data));
  }
  LF2_TRY(rebin_tail(c));
  {
    PhaseScope ps(c, PH_DEPOSIT);  // runs only when redep was raised
    LF2_CUDA(c, launch_deposit(c, 0, rho->data, 0, c->redep));
    LF2_CUDA(c, launch_deposit(c, 0, rho->data, 1, c->redep));
  }
  return LF2_OK;
}

lf2_status lf2_set_global_mass(lf2_ctx* c, double mass)
{
  if (!c || !(mass > 0)) return LF2_ERR_ARG;
  if (c->has_mass) return fail(c, LF2_ERR_ARG, "set_global_mass: the particles carry individual masses");
  c->gmass = mass;
  c->m_unit = mass;
  return LF2_OK;
}

lf2_status lf2_set_wait_limit(lf2_ctx* c, int64_t cycles, int stall)
{
  if (!c || cycles < 0) return LF2_ERR_ARG;
  c->wait_cycles = cycles;
  c->wait_stall = stall ? 1 : 0;
  return LF2_OK;
}

lf2_status lf2_set_move_kernel(lf2_ctx* c, int which)
{
  if (!c || which < 0 || which > 3) return LF2_ERR_ARG;
  c->move_kernel = which;
  return LF2_OK;
}

lf2_status lf2_last_max_velocity(lf2_ctx* c, double* max_v, int ptr_kind)
{
  if (!c || !max_v || (ptr_kind != LF2_PTR_HOST && ptr_kind != LF2_PTR_DEVICE)) return LF2_ERR_ARG;
  if (ptr_kind == LF2_PTR_DEVICE) {
    LF2_CUDA(c, launch_maxv_to_device(c, max_v));
    return LF2_OK;
  }
  LF2_CUDA(c, launch_reduce_maxv(c));
  LF2_CUDA(c, cudaMemcpyAsync(c->h_stats, c->stats, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  *max_v = std::sqrt(c->h_stats[0]);
  return LF2_OK;
}

lf2_status lf2_last_move_kernel(lf2_ctx* c, int* which)
{
  if (!c || !which) return LF2_ERR_ARG;
  *which = c->last_move_kernel;
  return LF2_OK;
}

lf2_status lf2_conservation(lf2_ctx* c, double* mass, double mom[3], double* max_v)
{
  if (!c) return LF2_ERR_ARG;
  LF2_CUDA(c, launch_conservation(c));
  LF2_CUDA(c, cudaMemcpyAsync(c->h_stats, c->stats, sizeof(double) * 8, cudaMemcpyDeviceToHost,
                              c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  if (mass) *mass = c->h_stats[1];
  if (mom)
    for (int d = 0; d < 3; d++) mom[d] = c->h_stats[2 + d];
  if (max_v) *max_v = std::sqrt(c->h_stats[5]);
  return LF2_OK;
}

lf2_status lf2_velocity_reductions(lf2_ctx* c, double* sum_v2, double* min_v2, double* max_v2)
{
  if (!c) return LF2_ERR_ARG;
  LF2_CUDA(c, launch_conservation(c));
  LF2_CUDA(c, cudaMemcpyAsync(c->h_stats, c->stats, sizeof(double) * 8, cudaMemcpyDeviceToHost,
                              c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  if (sum_v2) *sum_v2 = c->h_stats[6];
  if (min_v2) *min_v2 = c->h_stats[7];
  if (max_v2) *max_v2 = c->h_stats[5];
  return LF2_OK;
}

// F4 fields hold one float4 per site and must start on a 16-byte boundary.
static bool f4_ok(const float* p) { return !p || ((uintptr_t)p & 15) == 0; }

static lf2_status pm_call(lf2_ctx* c, int op, int64_t np, const int32_t* cell, const float* off3,
                          const float* mass, double gmass, const float* in_a, const float* in_b,
                          float* out_a, float* out_b, double dta, double dtb, int32_t* cell_rw,
                          float* off_rw, float* vel_rw)
{
  if (!c || np < 0) return LF2_ERR_ARG;
  if (np == 0) return LF2_OK;
  PhaseScope ps(c, PH_OTHER);
  LF2_CUDA(c, launch_pm(c, op, np, cell, off3, mass, (float)gmass, in_a, in_b, out_a, out_b,
                        (float)dta, (float)dtb, cell_rw, off_rw, vel_rw));
  return LF2_OK;
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

lf2_status lf2_pm_state_pack(lf2_ctx* c, int64_t np, const double* pos3, const double* vel3,
                             const double* mass, double inv_res, int32_t* key, void* records)
{
  if (!c || np < 0 || !(inv_res > 0)) return LF2_ERR_ARG;
  if (np > 0 && (!pos3 || !vel3 || !key || !records || !aligned16(records))) return LF2_ERR_ARG;
  if (c->g.nbricks * 4096 > INT32_MAX)
    return fail(c, LF2_ERR_UNSUPPORTED, "pm_state_pack: sort keys need nbricks * 4096 < 2^31");
  LF2_CUDA(c, launch_pm_pack(c, np, pos3, vel3, mass, inv_res, key, records));
  return LF2_OK;
}

lf2_status lf2_pm_state_unpack(lf2_ctx* c, int64_t np, const int64_t* order, const void* records,
                               int32_t* cell, float* off3, float* vel3, float* mass)
{
  if (!c || np < 0) return LF2_ERR_ARG;
  if (np > 0 && (!order || !records || !aligned16(records) || !cell || !off3 || !vel3))
    return LF2_ERR_ARG;
  LF2_CUDA(c, launch_pm_unpack(c, np, order, records, cell, off3, vel3, mass));
  return LF2_OK;
}

lf2_status lf2_pm_brick_start(lf2_ctx* c, int64_t np, const int32_t* cell, int64_t* brick_start)
{
  if (!c || np < 0 || !brick_start || (np > 0 && !cell)) return LF2_ERR_ARG;
  LF2_CUDA(c, launch_pm_brick_start(c, np, cell, brick_start));
  return LF2_OK;
}

lf2_status lf2_pm_grads_unorder(lf2_ctx* c, int64_t np, const int64_t* order, const float* g_off3,
                                const float* g_vel3, const float* g_mass, double inv_res,
                                void* records, double* g_pos3_out, double* g_vel3_out,
                                double* g_mass_out)
{
  if (!c || np < 0) return LF2_ERR_ARG;
  if (np > 0 && (!order || !g_off3 || !g_vel3 || !g_mass || !records || !aligned16(records) ||
                 !g_pos3_out || !g_vel3_out || !g_mass_out))
    return LF2_ERR_ARG;
  LF2_CUDA(c, launch_pm_grads_back(c, np, order, g_off3, g_vel3, g_mass, inv_res, records,
                                   g_pos3_out, g_vel3_out, g_mass_out));
  return LF2_OK;
}

lf2_status lf2_pm_deposit_bricks(lf2_ctx* c, int64_t np, const int32_t* cell, const float* off3,
                                 const float* mass, double gmass, const int64_t* brick_start,
                                 float* rho)
{
  if (!c || np < 0 || !brick_start || !rho || (np > 0 && (!cell || !off3))) return LF2_ERR_ARG;
  LF2_CUDA(c, launch_pm_deposit(c, np, brick_start, cell, off3, mass, (float)gmass, rho));
  return LF2_OK;
}

lf2_status lf2_pm_deposit(lf2_ctx* c, int64_t np, const int32_t* cell, const float* off3,
                          const float* mass, double gmass, float* rho)
{
  if (!cell || !off3 || !rho) return LF2_ERR_ARG;
  return pm_call(c, 0, np, cell, off3, mass, gmass, nullptr, nullptr, rho, nullptr, 0, 0, nullptr,
                 nullptr, nullptr);
}

lf2_status lf2_pm_gather(lf2_ctx* c, int64_t np, const int32_t* cell, const float* off3,
                         const float* F4, float* out3)
{
  if (!cell || !off3 || !F4 || !out3 || !f4_ok(F4)) return LF2_ERR_ARG;
  return pm_call(c, 1, np, cell, off3, nullptr, 0, F4, nullptr, out3, nullptr, 0, 0, nullptr,
                 nullptr, nullptr);
}

lf2_status lf2_pm_kick_drift(lf2_ctx* c, int64_t np, int32_t* cell, float* off3, float* vel3,
                             const float* G3, double dt_kick, double dt_drift)
{
  if (!c || !cell || !off3 || !vel3) return LF2_ERR_ARG;
  return pm_call(c, 2, np, nullptr, nullptr, nullptr, 0, G3, nullptr, nullptr, nullptr, dt_kick,
                 dt_drift / c->res, cell, off3, vel3);
}

lf2_status lf2_pm_step(lf2_ctx* c, int64_t np, int32_t* cell, float* off3, float* vel3,
                       const float* F4, double dt_kick, double dt_drift)
{
  if (!c || np < 0 || !F4 || !f4_ok(F4) || (np > 0 && (!cell || !off3 || !vel3))) return LF2_ERR_ARG;
  if (np == 0) return LF2_OK;
  PhaseScope ps(c, PH_OTHER);
  LF2_CUDA(c, launch_pm_step(c, np, cell, off3, vel3, F4, (float)dt_kick, (float)(dt_drift / c->res)));
  return LF2_OK;
}

lf2_status lf2_pm_deposit_adjoint(lf2_ctx* c, int64_t np, const int32_t* cell, const float* off3,
                                  const float* mass, double gmass, const float* g_rho,
                                  float* g_off3, float* g_mass)
{
  if (!cell || !off3 || !g_rho) return LF2_ERR_ARG;
  return pm_call(c, 3, np, cell, off3, mass, gmass, g_rho, nullptr, g_off3, g_mass, 0, 0, nullptr,
                 nullptr, nullptr);
}

lf2_status lf2_pm_gather_adjoint(lf2_ctx* c, int64_t np, const int32_t* cell, const float* off3,
                                 const float* F4, const float* g_out3, float* g_F4, float* g_off3)
{
  if (!cell || !off3 || !g_out3 || (g_off3 && !F4) || !f4_ok(F4) || !f4_ok(g_F4))
    return LF2_ERR_ARG;
  return pm_call(c, 4, np, cell, off3, nullptr, 0, F4, g_out3, g_F4, g_off3, 0, 0, nullptr, nullptr,
                 nullptr);
}

lf2_status lf2_stencil27(lf2_ctx* c, const float* rho, const float* S81, float* F4)
{
  if (!c || !rho || !S81 || !F4 || !f4_ok(F4)) return LF2_ERR_ARG;
  PhaseScope ps(c, PH_OTHER);
  LF2_CUDA(c, launch_stencil(c, 0, rho, S81, F4, nullptr));
  return LF2_OK;
}

lf2_status lf2_stencil27_adjoint(lf2_ctx* c, const float* rho, const float* S81, const float* g_F4,
                                 float* g_rho, float* g_S81)
{
  if (!c || !g_F4 || !f4_ok(g_F4) || (g_rho && !S81) || (g_S81 && !rho)) return LF2_ERR_ARG;
  PhaseScope ps(c, PH_OTHER);
  if (g_rho) LF2_CUDA(c, launch_stencil(c, 1, g_F4, S81, g_rho, nullptr));
  if (g_S81) {
    if (!c->stencil_partial &&
        cudaMalloc(&c->stencil_partial, sizeof(float) * stencil_partial_floats(c)) != cudaSuccess)
      return fail(c, LF2_ERR_NOMEM, "cannot allocate stencil partial sums");
    LF2_CUDA(c, launch_stencil(c, 2, g_F4, rho, g_S81, c->stencil_partial));
  }
  return LF2_OK;
}

lf2_status lf2_profile_enable(lf2_ctx* c, int on)
{
  if (!c) return LF2_ERR_ARG;
  c->profiling = on != 0;
  return LF2_OK;
}

lf2_status lf2_profile_read(lf2_ctx* c, double* ms, int64_t* launches)
{
  if (!c) return LF2_ERR_ARG;
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int p = 0; p < LF2_NPHASE; p++) {
    double t = 0.0;
    for (auto& pr : c->pending[p]) {
      float x = 0.0f;
      if (cudaEventElapsedTime(&x, pr.first, pr.second) == cudaSuccess) t += x;
      c->event_pool.push_back(pr.first);
      c->event_pool.push_back(pr.second);
    }
    c->pending[p].clear();
    if (ms) ms[p] = t;
    if (launches) launches[p] = c->phase_launches[p];
    c->phase_launches[p] = 0;
  }
  return LF2_OK;
}

lf2_status lf2_rebin_stats(lf2_ctx* c, int64_t* repacks, int64_t* relocations, int64_t* movers)
{
  if (!c) return LF2_ERR_ARG;
  unsigned long long d[3] = {0, 0, 0};  // repacks, movers of the last drift, relocations
  LF2_CUDA(c, cudaMemcpyAsync(d, c->diag, sizeof d, cudaMemcpyDeviceToHost, c->stream));
  LF2_CUDA(c, cudaStreamSynchronize(c->stream));
  if (repacks) *repacks = (int64_t)d[0];
  if (movers) *movers = (int64_t)d[1];
  if (relocations) *relocations = (int64_t)d[2];
  return LF2_OK;
}

lf2_status lf2_kernel_launches(lf2_ctx* c, int64_t* n)
{
  if (!c || !n) return LF2_ERR_ARG;
  *n = c->launches;
  return LF2_OK;
}

}  // extern "C"
