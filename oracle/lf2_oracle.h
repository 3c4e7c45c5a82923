/*
 * lf2_oracle.h -- CPU oracle for the LATfield2 particle-mesh path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, the smoke check and the CPU-baseline leg of
 * bench.py use it, and only as the checker of the CUDA path.
 *
 * Two layers live here:
 *
 *  (A) "ref" functions restate the reference algorithm in the reference's own
 *      data layout: fields are halo'd, component-interleaved arrays
 *      (index = (x+h) + G0*((y+h) + G1*(z+h)), value = data[index*C + c],
 *      Gi = Ni + 2h, LATfield2_Field_decl.hpp:760-788, LATfield2_Lattice.hpp:110-113)
 *      and particles sit in per-cell lists walked in site order
 *      (x fastest, LATfield2_Site.hpp:55-76).  Each function is compiled twice:
 *      suffix _d with Real = double (the default reference build) and suffix
 *      _f with Real = float (the reference's -DSINGLE build).  The arithmetic,
 *      including the mixed float/double evaluation of the SINGLE build, follows
 *      the cited reference lines statement by statement.
 *
 *  (B) "state" functions restate the arithmetic of the device path of this
 *      library on its own particle representation (int32 cell + FP32 in-cell
 *      offset, FP32 velocity): the FP32 kick/drift with the same fmaf order
 *      and the int64 fixed-point deposit.  They are bit-exact checkers for the
 *      CUDA kernels.
 *
 * Build: oracle/Makefile -> oracle/liblf2oracle.so (gcc, -ffp-contract=off).
 */
#ifndef LF2_ORACLE_H
#define LF2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- (A) */

/* Particle lists are given in CSR form over the cells of the halo-0 particle
 * lattice in site order: the particles of cell c = x + n0*(y + n1*z) are
 * entries [cell_start[c], cell_start[c+1]) of pos/vel/pmass, in list order.
 * pos and vel are AoS (3 per particle) in box units, like part_simple.pos/vel
 * (LATfield2_particle_simple.hpp:40-45). pmass (optional, may be NULL) is the
 * per-particle double mass of an "individual mass" particle type. */

#define LF2O_DECL(R, S)                                                        \
  void lf2o_projection_init_##S(R* f, const int n[3], int halo, int comps);   \
  void lf2o_scalar_cic_project_##S(const int n[3], int halo, R res,            \
        const int64_t* cell_start, const R* pos, const double* pmass,          \
        double gmass, R* rho);                                                 \
  void lf2o_scalar_cic_comm_##S(R* rho, const int n[3], int halo);            \
  void lf2o_vector_cicngp_project_##S(const int n[3], int halo, R res,         \
        const int64_t* cell_start, const R* pos, const R* vel,                 \
        const double* pmass, double gmass, R* v);                              \
  void lf2o_vector_cicngp_comm_##S(R* v, const int n[3], int halo);           \
  void lf2o_symtensor_cicngp_project_##S(const int n[3], int halo, R res,      \
        const int64_t* cell_start, const R* pos, const R* vel,                 \
        const double* pmass, double gmass, R* t);                              \
  void lf2o_symtensor_cicngp_comm_##S(R* t, const int n[3], int halo);        \
  void lf2o_vector_cic_project_##S(const int n[3], int halo, R res,            \
        const int64_t* cell_start, const R* pos, const R* vel,                 \
        const double* pmass, double gmass, R* v);                              \
  void lf2o_vector_cic_comm_##S(R* v, const int n[3], int halo);              \
  void lf2o_vecvec_cic_project_##S(const int n[3], int halo, R res,            \
        const int64_t* cell_start, const R* pos, const R* vel,                 \
        const double* pmass, double gmass, R* t);                              \
  void lf2o_vecvec_cic_comm_##S(R* t, const int n[3], int halo);              \
  void lf2o_update_halo_##S(R* f, const int n[3], int halo, int comps);       \
  double lf2o_update_vel_cic_##S(const int n[3], int halo,                     \
        const int64_t* cell_start, const R* pos, R* vel, const R* F,           \
        double dtau, double* sum_v2);                                          \
  void lf2o_move_simple_##S(const int n[3], R box, int64_t np, R* pos,         \
        const R* vel, double dtau, int32_t* cell_out);

LF2O_DECL(double, d)
LF2O_DECL(float, f)

/* Per-cell linked lists with push_front semantics, used to reproduce the
 * list order that addParticle_global (LATfield2_Particles.hpp:500-519) and the
 * splice in moveParticles (:2035-2056) leave behind.  order_out receives the
 * particle indices in CSR list order; cell_start_out has ncells+1 entries. */
void lf2o_lists_from_insertion(int64_t ncells, int64_t np, const int32_t* cell,
                               int64_t* cell_start_out, int64_t* order_out);

/* List order after the rebin loop of moveParticles on one rank
 * (LATfield2_Particles.hpp:1960-2056). */
void lf2o_rebin_lists(int64_t ncells, int64_t np, const int64_t* cs_old,
                      const int64_t* order_old, const int32_t* new_cell,
                      int64_t* cs_new, int64_t* order_new);

/* ---------------------------------------------------------------- (B) */

/* FP32 CIC gather + kick of the device path: acc_c = sum_k w_k F_c(corner_k)
 * accumulated with fmaf in corner order k = 4*bx + 2*by + bz, then
 * vel_c = fmaf(dtk, acc_c, vel_c).  F is the library's internal layout:
 * component-major, no halo, periodic. */
void lf2o_state_kick(const int n[3], int64_t np, const int32_t* cell,
                     const float* off, float* vel, const float* F, float dtk);

/* FP32 drift of the device path: o = fmaf(dtn, v, o); carry = floor(o);
 * o -= carry; if (o >= 1) { o = 0; carry += 1; }; coordinate += carry
 * (periodic).  Returns the number of particles whose state was not finite. */
int64_t lf2o_state_drift(const int n[3], int64_t np, int32_t* cell, float* off,
                         const float* vel, float dtn);

/* Fixed-point weight of one corner: the three 1-D weights are rounded to
 * 2^-31, multiplied exactly (96-bit) and rounded to 2^-32 of a unit mass. */
uint64_t lf2o_fixed_weight(float wx_up, float wy_up, float wz_up, int bx,
                           int by, int bz);

/* Fixed-point scalar CIC deposit into an int64 accumulator (internal layout,
 * one component, no halo, periodic).  mrel (optional) is the per-particle
 * mass in units of the deposit unit mass. */
void lf2o_state_deposit_fixed(const int n[3], int64_t np, const int32_t* cell,
                              const float* off, const float* mrel,
                              int64_t* acc);

/* Converts the accumulator to FP32 exactly as the device does:
 * rho = (float)acc * scale. */
void lf2o_state_fixed_to_f32(int64_t nsites, const int64_t* acc, float scale,
                             float* rho);

/* FP64 CIC scalar deposit on the device representation (used to measure the
 * error of the FP32 and fixed-point modes): rho = m/res^3 * prod(w). */
void lf2o_state_deposit_f64(const int n[3], int64_t np, const int32_t* cell,
                            const float* off, const float* mass, double gmass,
                            double res, double* rho);

/* Exponent e of the fixed-point velocity unit V = 2^e: the smallest power of
 * two above every |v_i| (0 when all are 0), at least -96. */
int lf2o_vexp(int64_t np, const float* vel);

/* Fixed-point momentum / stress deposit of the device path (kinds 1 vector
 * CIC-NGP, 2 symtensor CIC-NGP, 3 vector CIC, 4 VecVec CIC) into a
 * component-major int64 accumulator (3 or 6 components, internal layout).
 * Quantum: 2^-32 of a unit mass times V (kinds 1, 3) or V^2 (2, 4). */
void lf2o_state_deposit_fixed_kind(int kind, const int n[3], int64_t np,
                                   const int32_t* cell, const float* off,
                                   const float* vel, const float* mrel, int vexp,
                                   int64_t* acc);

#ifdef __cplusplus
}
#endif
#endif
