// lf2_internal.h -- context layout and kernel launchers shared by the .cu
// files of liblf2gpu.so.  Not part of the public ABI (include/lf2gpu.h).
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "lf2_common.cuh"
#include "lf2gpu.h"

namespace lf2 {

// Structure-of-arrays particle store (see lf2_common.cuh).
struct PartArrays {
  uint32_t* key = nullptr;
  float* ox = nullptr;
  float* oy = nullptr;
  float* oz = nullptr;
  float* vx = nullptr;
  float* vy = nullptr;
  float* vz = nullptr;
  float* mass = nullptr;  // only with per-particle masses
  int64_t* id = nullptr;  // only when IDs are carried
};

// Arguments shared by the per-brick kernels.
struct StoreView {
  Geom g;
  PartArrays a;
  const int64_t* seg_start;  // [nbricks + 1]
  int32_t* count;            // [nbricks]
  const int32_t* cap;        // [nbricks]
};

struct DepositParams {
  float mf;          // FP32 mode: mass / res^3 for a global mass
  float inv_vol;     // 1 / res^3
  float fixed_scale; // fixed mode: 2^-32 * unit mass / res^3
  float inv_unit;    // fixed mode: 1 / unit mass (per-particle masses)
  int has_mass;
};

struct MoveParams {
  float dtk;   // kick: dtau
  float dtn;   // drift: dtau / res (cell units per velocity unit)
};

}  // namespace lf2

struct lf2_field_s {
  int comps = 0;
  float* data = nullptr;
  bool owned = true;
};

struct lf2_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  lf2::Geom g{};
  double res = 0.0;
  double box[3] = {0, 0, 0};
  int mode = LF2_DEPOSIT_FP32;
  std::string err;

  // particle store
  int64_t np = 0;
  bool has_mass = false;
  bool has_id = false;
  double gmass = 0.0;   // global particle mass (GLOBAL_MASS types)
  double m_unit = 1.0;  // unit mass of the fixed-point deposit
  int64_t capacity = 0; // slots allocated in cur/alt
  lf2::PartArrays cur, alt, mov;
  int64_t mov_capacity = 0;
  int32_t* mov_placed = nullptr;
  int64_t* seg_start = nullptr;      // [nbricks + 1]
  int64_t* seg_start_alt = nullptr;  // [nbricks + 1]
  int32_t* count = nullptr;          // [nbricks]
  int32_t* cap = nullptr;            // [nbricks]
  int32_t* cap_alt = nullptr;        // [nbricks]
  int32_t* fill = nullptr;           // [nbricks] scratch
  unsigned long long* mov_count = nullptr;
  unsigned long long* mig = nullptr;  // device [4]: slab migration counters
  uint32_t* flags = nullptr;         // device error bits
  int32_t* repack = nullptr;         // device: 1 when the whole store must be repacked
  unsigned long long* diag = nullptr; // device [3]: repacks, movers of the last drift, relocations
  unsigned long long* heap_top = nullptr;  // device: next free slot of the relocation region
  int32_t* ovf_list = nullptr;       // [nbricks] bricks that ran out of slots in the last insert
  int32_t* ovf_count = nullptr;      // device: entries of ovf_list
  int32_t* ovf_state = nullptr;      // [nbricks] 0 none, 1 listed, 2 relocated
  float* brick_maxv2 = nullptr;      // [nbricks]
  double* brick_sums = nullptr;      // [nbricks * 5]
  double* stats = nullptr;           // [8] device
  uint64_t* spill = nullptr;         // deposit shell store (8-byte slots)
  uint32_t* vmax_bits = nullptr;     // device: largest |v_i| (float bits), fixed-point deposits
  uint32_t* redep = nullptr;         // device: the fused deposit must be redone by the tile pass
  float* stencil_partial = nullptr;  // per-CTA partial sums of the stencil weight gradient
  unsigned long long* pm_acc = nullptr; // chain's fixed-point deposit: [nsites] sums + max mass word
  size_t spill_slots = 0;
  double* h_stats = nullptr;         // pinned [8]
  uint32_t* h_flags = nullptr;       // pinned
  int64_t* h_i64 = nullptr;          // pinned [4]

  // pipelined fused move (lf2_move_pipe.cu)
  int num_sms = 0;
  int move_kernel = 0;               // 0 auto, 1 per-brick k_move, 2 pipelined
  int last_move_kernel = 0;          // kernel of the last kick-drift pass (1 or 2)
  int* work = nullptr;               // device brick counter
  int64_t wait_cycles = 0;           // limit of its bounded waits (0: about 2 s)
  int wait_stall = 0;                // consumers first wait on a barrier nothing completes
  const float* tmap_src = nullptr;   // field the cached tensor map describes
  alignas(64) unsigned char tmap_bytes[128];

  // PM grid operator (lf2_fft.cu)
  int fft_r2c = 0;                   // cuFFT plan handles, valid when fft_planned
  int fft_c2r = 0;
  bool fft_planned = false;
  float2* fft_k = nullptr;           // one component of complex scratch
  float* fft_phi = nullptr;          // one component of real scratch

  // measurement (lf2_profile_*)
  int64_t launches = 0;              // kernels launched, all phases
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[LF2_NPHASE];
  std::vector<cudaEvent_t> event_pool;
  int64_t phase_launches[LF2_NPHASE] = {0, 0, 0, 0, 0};
};

// ---------------------------------------------------------------- launchers
namespace lf2 {

inline StoreView view(lf2_ctx* c)
{
  StoreView v;
  v.g = c->g;
  v.a = c->cur;
  v.seg_start = c->seg_start;
  v.count = c->count;
  v.cap = c->cap;
  return v;
}

// lf2_store.cu
cudaError_t launch_load_count(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3);
cudaError_t launch_caps_and_scan(lf2_ctx* c, const int32_t* counts, int32_t* caps, int64_t* starts,
                                 int64_t* total_dev);
cudaError_t launch_load_scatter(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                                const float* vel3, const float* mass, const int64_t* id);
cudaError_t launch_pos_to_state(lf2_ctx* c, int64_t n, const void* pos3, int real_bytes,
                                int32_t* cell, float* off3);
cudaError_t launch_get(lf2_ctx* c, int64_t* out_start, int32_t* cell, float* off3, float* vel3,
                       float* mass, int64_t* id);
cudaError_t launch_state_to_pos(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                                void* pos3, int real_bytes);
cudaError_t launch_cell_counts(lf2_ctx* c, int32_t* counts);
cudaError_t launch_scan_counts(lf2_ctx* c, int64_t* out_start);
cudaError_t launch_repack(lf2_ctx* c);
cudaError_t launch_heap_reset(lf2_ctx* c);

// lf2_move.cu
cudaError_t launch_move(lf2_ctx* c, const float* F, bool kick, bool drift, MoveParams mp);
cudaError_t launch_insert(lf2_ctx* c);
cudaError_t launch_reduce_maxv(lf2_ctx* c);
cudaError_t launch_maxv_to_device(lf2_ctx* c, double* dst);

// lf2_move_pipe.cu (rho != nullptr: the fixed-point scalar deposit fused in;
// its rim store is c->spill, rim_store_slots(c) slots)
bool move_pipe_eligible(const lf2_ctx* c, const float* F);
bool move_dep_eligible(const lf2_ctx* c, const float* F);
size_t rim_store_slots(const lf2_ctx* c);
cudaError_t launch_move_pipe(lf2_ctx* c, const float* F, MoveParams mp, float* rho);
cudaError_t launch_dep_movers(lf2_ctx* c);
cudaError_t launch_fixup_rim(lf2_ctx* c, float* rho);

// lf2_deposit.cu
// stage 0: tile pass (k_deposit), stage 1: face fix-up (k_fixup)
cudaError_t launch_deposit(lf2_ctx* c, int kind, float* out, int stage,
                           const uint32_t* gate = nullptr);
// largest |v_i| of the store into c->vmax_bits (fixed-point momentum/stress)
cudaError_t launch_vmax(lf2_ctx* c);
DepositParams deposit_params(const lf2_ctx* c);

// lf2_exchange.cu (slab decomposition): particles with cell z outside
// [zlo, zhi] counted (below, above, more than one plane outside: 3 counters)
// / moved out of the store; new particles into the mover buffer for k_insert
cudaError_t launch_count_outside(lf2_ctx* c, int zlo, int zhi, unsigned long long* n,
                                 bool max_v = false);
cudaError_t launch_extract_outside(lf2_ctx* c, int zlo, int zhi, int32_t* cell, float* off3,
                                   float* vel3, float* mass, int64_t* id,
                                   unsigned long long* out_count);
cudaError_t launch_pack_movers(lf2_ctx* c, int64_t n, const int32_t* cell, const float* off3,
                               const float* vel3, const float* mass, const int64_t* id,
                               bool write);
// migration records (lf2_slab_*): 32-bit words per particle
inline int record_words(const lf2_ctx* c) { return 7 + (c->has_mass ? 1 : 0) + (c->has_id ? 2 : 0); }
cudaError_t launch_extract_records(lf2_ctx* c, int zlo, int zhi, int64_t n_below, uint32_t* below,
                                   int64_t n_above, uint32_t* above, unsigned long long* ctr);
cudaError_t launch_pack_records(lf2_ctx* c, int64_t na, const uint32_t* a, int64_t nb,
                                const uint32_t* b);
cudaError_t launch_unpack_records(lf2_ctx* c, int64_t na, const uint32_t* a, int64_t nb,
                                  const uint32_t* b, int32_t* cell, float* off3, float* vel3,
                                  float* mass, int64_t* id);

// lf2_fft.cu: releases the cuFFT plans and scratch of the context
void fft_release(lf2_ctx* c);

// lf2_deposit_full.cu: kind 3 vector CIC, kind 4 VecVec CIC; stage 0 tile
// pass (k_deposit_full), stage 1 boundary fix-up (k_fixup_full)
cudaError_t launch_deposit_full(lf2_ctx* c, int kind, float* out, int stage);
size_t deposit_full_spill_slots(const lf2_ctx* c, int comps);
size_t deposit_spill_slots(const lf2_ctx* c, int comps);

// lf2_pm.cu (differentiable chain; op codes documented there)
cudaError_t launch_pm(lf2_ctx* c, int op, int64_t np, const int32_t* cell, const float* off3,
                      const float* mass, float gmass, const float* in_a, const float* in_b,
                      float* out_a, float* out_b, float dta, float dtb, int32_t* cell_rw,
                      float* off_rw, float* vel_rw);
// the chain's deposit, per particle or brick-tiled (brick_start given)
cudaError_t launch_pm_deposit(lf2_ctx* c, int64_t np, const int64_t* brick_start, const int32_t* cell,
                              const float* off3, const float* mass, float gmass, float* rho);
// the chain's particle state: sort keys and 32-byte records in the caller's
// order, the state in a given order, the bricks' first slots; gradients back
// to the caller's order through the same records
cudaError_t launch_pm_step(lf2_ctx* c, int64_t np, int32_t* cell, float* off3, float* vel3,
                           const float* F4, float dtk, float dtn);
cudaError_t launch_pm_pack(lf2_ctx* c, int64_t np, const double* pos, const double* vel,
                           const double* mass, double inv_res, int32_t* key, void* rec);
cudaError_t launch_pm_unpack(lf2_ctx* c, int64_t np, const int64_t* order, const void* rec,
                             int32_t* cell, float* off3, float* vel3, float* m);
cudaError_t launch_pm_brick_start(lf2_ctx* c, int64_t np, const int32_t* cell, int64_t* brick_start);
cudaError_t launch_pm_grads_back(lf2_ctx* c, int64_t np, const int64_t* order, const float* g_off3,
                                 const float* g_vel3, const float* g_m, double inv_res, void* rec,
                                 double* g_pos, double* g_vel, double* g_mass);
cudaError_t launch_stencil(lf2_ctx* c, int op, const float* a, const float* S, float* out,
                           float* partial);
size_t stencil_partial_floats(const lf2_ctx* c);

// lf2_field.cu
cudaError_t launch_export(lf2_ctx* c, int comps, const float* src, void* dst, int halo,
                          int real_bytes, int fill_halo);
cudaError_t launch_import(lf2_ctx* c, int comps, float* dst, const void* src, int halo,
                          int real_bytes);
cudaError_t launch_halo_fill(lf2_ctx* c, void* data, int comps, int halo, int real_bytes);
cudaError_t launch_conservation(lf2_ctx* c);

}  // namespace lf2
