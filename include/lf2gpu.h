/*
 * lf2gpu.h -- C ABI of the B200 particle-mesh library (liblf2gpu.so).
 *
 * This is the boundary that replaces the reference's header-only particle
 * path (particles/LATfield2_Particles.hpp, particles/projections.hpp,
 * LATfield2_Field_decl.hpp) and its real-to-complex Fourier transform
 * (LATfield2_PlanFFT_decl.hpp).  Plain C types only: pointers, sizes, status
 * codes.  The C++ compatibility layer (include/latfield2_b200.hpp) and the
 * Python package (latfield2_b200) are both written on top of these functions.
 *
 * Sections: context; particles (set, get, the slab exchange: extract_z /
 * add and the migration records of slab_count / slab_extract / slab_insert,
 * checkpoint); fields; projections (scalar CIC, vector and
 * symtensor CIC-NGP, full-CIC vector and VecVec); particle moves (kick,
 * drift and rebin, the fused step); PM grid operator (k-fields, FFT, Poisson
 * force); differentiable PM chain; the no-allocation deposit; measurement.
 *
 * Conventions
 *  - Every function returns an lf2_status: 0 on success, < 0 on failure;
 *    lf2_last_error() gives the message.  Nothing exits or throws across the
 *    boundary (the reference exit()s, throws 1 or calls MPI_Abort).
 *  - The context owns all device memory it allocates.  Host pointers passed
 *    in are only borrowed for the duration of the call.
 *  - Work is stream-ordered on the context's stream.  Calls that return a
 *    host value (counts, max |v|, conservation sums, flags) synchronise it.
 *  - ptr_kind tells whether an array argument lives on the host
 *    (LF2_PTR_HOST) or on the context's device (LF2_PTR_DEVICE).
 *  - Lattice geometry: n[3] sites per dim, periodic, lattice resolution
 *    res = box[i] / n[i] equal in every dim (particles_tools.hpp:6-19).
 *    Cell index c = x + n0*(y + n1*z) (site order, LATfield2_Site.hpp:55-76).
 *  - Particle state on the device: cell (int), in-cell offset in cell units
 *    (FP32, [0,1)), velocity in box units per time (FP32), optional FP32
 *    mass, optional int64 ID.  Positions in box units are
 *    pos = (coord + off) * res.
 *  - Fields on the device: FP32, component-major, no halo, periodic:
 *    data[c * n0*n1*n2 + cell].  lf2_field_export/import convert to and from
 *    the reference layout (halo'd, components interleaved, float or double).
 */
#ifndef LF2GPU_H
#define LF2GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lf2_ctx lf2_ctx;
typedef struct lf2_field_s* lf2_field;
typedef struct lf2_kfield_s* lf2_kfield;
typedef struct lf2_slab_fft_s* lf2_slab_fft;
typedef int lf2_status;

#define LF2_OK 0
#define LF2_ERR_ARG (-1)         /* invalid argument */
#define LF2_ERR_CUDA (-2)        /* CUDA runtime error */
#define LF2_ERR_STATE (-3)       /* a kernel raised an error flag */
#define LF2_ERR_NOMEM (-4)       /* device allocation failed */
#define LF2_ERR_UNSUPPORTED (-5) /* combination not provided */

/* Deposit modes (lf2_create).  FP32: FP32 atomics whose rounding errors are
 * recovered exactly and carried in a second FP32 word, so every vertex sum
 * is within about 1e-7 of exact whatever the order (not bit-identical run to
 * run).  FIXED64: int64 fixed point, bit-exact run to run; quantum 2^-32 of
 * a unit mass (the global particle mass, or the mean of per-particle
 * masses) for the density, 2^-48 of a unit mass times V for momentum and
 * times V^2 for stress, V the smallest power of two above every |v_i| of the
 * particles.  FP32_PLAIN: FP32 atomics without
 * compensation, the fastest FP32 form; unordered additions leave a few 1e-6
 * of error in dense vertices. */
#define LF2_DEPOSIT_FP32 0
#define LF2_DEPOSIT_FIXED64 1
#define LF2_DEPOSIT_FP32_PLAIN 2

#define LF2_PTR_HOST 0
#define LF2_PTR_DEVICE 1

/* Device error bits returned by lf2_get_flags. */
#define LF2_FLAG_NONFINITE 0x1u      /* NaN/Inf offset or velocity met */
#define LF2_FLAG_BAD_CELL 0x2u       /* cell/offset out of range on load */
#define LF2_FLAG_MASS_RANGE 0x4u     /* relative mass outside [0,64) (fixed) */
#define LF2_FLAG_REPACK 0x8u         /* informational: store was repacked */
#define LF2_FLAG_CAPACITY 0x10u      /* repack did not fit: state lost */
#define LF2_FLAG_FIXED_OVERFLOW 0x20u /* fixed-point vertex sum overflowed */
#define LF2_FLAG_TIMEOUT 0x40u       /* a bounded in-kernel wait gave up */

/* ------------------------------------------------------------------ context
 * Replaces Lattice(3, n, halo) + Particles::initialize(info, type, &lat_part,
 * boxSize) (LATfield2_Lattice.hpp:27-223, LATfield2_Particles.hpp:358-428):
 * geometry, resolution check (get_lattice_resolution, particles_tools.hpp:6-19)
 * and the deposit mode.  stream may be NULL (default stream) or a
 * cudaStream_t. */
lf2_status lf2_create(lf2_ctx** out, int device, const int n[3],
                      const double box[3], int deposit_mode, void* stream);
lf2_status lf2_destroy(lf2_ctx* ctx);
const char* lf2_last_error(const lf2_ctx* ctx);
/* Later calls run on `stream`.  Work already queued on the previous stream
 * is not waited for: order it first (lf2_synchronize, or an event). */
lf2_status lf2_set_stream(lf2_ctx* ctx, void* stream);
/* Waits for the context's stream and turns raised device flags into
 * LF2_ERR_STATE. */
lf2_status lf2_synchronize(lf2_ctx* ctx);
/* Reads (and with clear != 0, clears) the device error bits. */
lf2_status lf2_get_flags(lf2_ctx* ctx, uint32_t* flags, int clear);

/* --------------------------------------------------------------- particles
 * Replaces the addParticle_global loop (LATfield2_Particles.hpp:500-540):
 * bulk upload of n particles in any order, binned on the device.  cell[i] in
 * [0, n0*n1*n2); off3/vel3 are AoS (3 per particle).  mass may be NULL
 * (global mass `global_mass`, the part_info mass, GLOBAL_MASS) or hold one
 * FP32 mass per particle (INDIVIDUAL_MASS, :400-425).  id may be NULL (no
 * IDs carried).  The store holds at most 2^32 - 1 slots (about 1.25 n plus
 * 100 per brick): larger sets are refused with LF2_ERR_UNSUPPORTED. */
lf2_status lf2_particles_set(lf2_ctx* ctx, int64_t n, const int32_t* cell,
                             const float* off3, const float* vel3,
                             const float* mass, double global_mass,
                             const int64_t* id, int ptr_kind);
/* Same from positions in box units (part.pos, LATfield2_particle_simple.hpp:
 * 40-45), as float (real_bytes 4) or double (8); the cell is
 * floor(pos/res) mod n (getPartCoord, LATfield2_Particles.hpp:463-467).
 * Host pointers only. */
lf2_status lf2_particles_set_pos(lf2_ctx* ctx, int64_t n, const void* pos3,
                                 const void* vel3, int real_bytes,
                                 const float* mass, double global_mass,
                                 const int64_t* id);
/* The global particle mass (part_info.mass of GLOBAL_MASS types) used by
 * later deposits and conservation sums; for particles without individual
 * masses it is also the unit of the fixed-point deposit.  The projections'
 * oset / FROM_INFO argument (projections.hpp:115-126) in the C++ layer sets
 * it for one deposit.  LF2_ERR_ARG when the particles carry individual
 * masses or mass <= 0. */
lf2_status lf2_set_global_mass(lf2_ctx* ctx, double mass);
/* Slab decomposition (one rank per GPU, z split across ranks, one ghost
 * cell plane below and above the rank's own planes): the particle
 * migration of moveParticles (LATfield2_Particles.hpp:2176-2799) as two
 * local operations around the exchange.
 *   extract_z: every particle whose cell z lies outside [z_lo, z_hi] leaves
 *     the store and is written (any order) as cell index, offsets (3 per
 *     particle), velocities (3), mass and id, to DEVICE arrays of `capacity`
 *     entries.  mass / id must be given exactly when the store carries them
 *     (capacity 0: a count only, all arrays may be NULL).  *n_out receives
 *     the number of such particles; when it exceeds capacity, nothing
 *     changes and LF2_ERR_ARG is returned.
 *   add: particles in the same format (host or device arrays) join the store;
 *     a cell or offset out of range gives LF2_ERR_ARG and adds nothing.  The
 *     store must exist (lf2_particles_set, possibly with 0 particles). */
lf2_status lf2_particles_extract_z(lf2_ctx* ctx, int z_lo, int z_hi,
                                   int64_t capacity, int32_t* cell, float* off3,
                                   float* vel3, float* mass, int64_t* id,
                                   int64_t* n_out);
lf2_status lf2_particles_add(lf2_ctx* ctx, int64_t n, const int32_t* cell,
                             const float* off3, const float* vel3,
                             const float* mass, const int64_t* id, int ptr_kind);
/* The same migration in stream order, without host waits (the form a step
 * over several GPUs uses: the caller reads the counts once, together with
 * whatever else it needs, and sizes the messages from them).  A migration
 * record is record_words = 7 + has_mass + 2 has_id 32-bit words: cell index,
 * offsets (3) and velocities (3) as float bits[, mass][, id low word, id high
 * word].  All pointers are DEVICE memory.
 *   slab_count: counts[0..3] <- the particles with cell z below z_lo, above
 *     z_hi, and more than one plane outside [z_lo, z_hi] (these cannot be
 *     routed to a neighbour), and max |v|^2 after the last kick (0 before
 *     any) as the bits of a float: non-negative floats order as their bits,
 *     so an integer maximum over ranks is the float maximum.
 *   slab_extract: the particles outside [z_lo, z_hi] leave the store, those
 *     below z_lo as n_below records in `below`, those above z_hi as n_above
 *     records in `above` (any order), each with the cell index it has in the
 *     neighbouring slab's lattice: z moved by +nz (below) or -nz (above),
 *     nz = z_hi - z_lo + 1.  n_below and n_above must be the counts
 *     slab_count gave for the same store; a particle beyond them is lost and
 *     raises LF2_FLAG_CAPACITY.
 *   slab_insert: n_a records from `a` and n_b from `b` join the store through
 *     the mover path.  A record with a cell index or offset out of range is
 *     dropped and raises LF2_FLAG_BAD_CELL (the store is then not valid).
 *     When the store lacks room the records go through lf2_particles_add,
 *     which waits and refuses the whole set (LF2_ERR_ARG, nothing added)
 *     when a record is out of range.
 * Raised flags fail the context's next waiting call (lf2_synchronize) with
 * LF2_ERR_STATE. */
lf2_status lf2_slab_record_words(lf2_ctx* ctx, int* words);
lf2_status lf2_slab_count(lf2_ctx* ctx, int z_lo, int z_hi, int64_t* counts);
lf2_status lf2_slab_extract(lf2_ctx* ctx, int z_lo, int z_hi, int64_t n_below,
                            uint32_t* below, int64_t n_above, uint32_t* above);
lf2_status lf2_slab_insert(lf2_ctx* ctx, int64_t n_a, const uint32_t* a,
                           int64_t n_b, const uint32_t* b);
/* Checkpoint of the particle store for an exact restart: the library's
 * particle state (cell, offsets, velocities, mass, id) and the unit mass of
 * the fixed-point deposit, written to / read from a little-endian file: an
 * 80-byte header (int32 "LF2C", version 1, n[3], deposit mode, has_mass,
 * has_id; double box[3], global mass, unit mass; int64 count), then the
 * arrays (cell, offsets, velocities[, mass][, id]).  A run restored into a context of the same
 * lattice, box and mode continues bit for bit.  The reference's own format
 * (Particles::saveHDF5 / loadHDF5, LATfield2_Particles.hpp:2809-3045) is
 * HDF5; its records (ID, pos, vel) come from lf2_particles_get_pos. */
lf2_status lf2_checkpoint_save(lf2_ctx* ctx, const char* path);
lf2_status lf2_checkpoint_load(lf2_ctx* ctx, const char* path);
/* Particles::numParticles (LATfield2_Particles.hpp:316-320). */
lf2_status lf2_particles_count(lf2_ctx* ctx, int64_t* n);
/* Downloads the particles in storage order (brick by brick).  Any output
 * pointer may be NULL; mass and id must be NULL when not carried. */
lf2_status lf2_particles_get(lf2_ctx* ctx, int32_t* cell, float* off3,
                             float* vel3, float* mass, int64_t* id,
                             int ptr_kind);
/* Positions in box units as float or double (host pointers). */
lf2_status lf2_particles_get_pos(lf2_ctx* ctx, void* pos3, void* vel3,
                                 int real_bytes, int64_t* id);
/* Number of particles in every cell (the size of each per-cell list). */
lf2_status lf2_cell_counts(lf2_ctx* ctx, int32_t* counts, int ptr_kind);

/* ------------------------------------------------------------------ fields
 * Replaces Field<Real>(lattice, comps) / Field<Real>(lattice, 3, 3,
 * symmetric) and alloc() (LATfield2_Field_decl.hpp:620-712).  A symmetric
 * 3x3 field has 6 components in the order 00,01,02,11,12,22 (:772-788). */
lf2_status lf2_field_create(lf2_ctx* ctx, int comps, lf2_field* out);
/* A field over caller-owned device memory (comps * n0*n1*n2 FP32 values in
 * the internal layout); lf2_field_destroy then releases only the handle. */
lf2_status lf2_field_wrap(lf2_ctx* ctx, int comps, float* device_data,
                          lf2_field* out);
lf2_status lf2_field_destroy(lf2_ctx* ctx, lf2_field f);
/* Device pointer of the field data (FP32, comps * n0*n1*n2 values). */
lf2_status lf2_field_device_ptr(lf2_ctx* ctx, lf2_field f, float** data);
lf2_status lf2_field_components(lf2_ctx* ctx, lf2_field f, int* comps);
/* projection_init (projections.hpp:31-34). */
lf2_status lf2_field_zero(lf2_ctx* ctx, lf2_field f);
/* Writes the field in the reference layout: halo `halo`, components
 * interleaved, float (real_bytes 4) or double (8).  fill_halo != 0 fills the
 * halo periodically (Field::updateHalo, LATfield2_Field_decl.hpp:889-935);
 * otherwise the halo is zero. */
lf2_status lf2_field_export(lf2_ctx* ctx, lf2_field f, void* dst, int halo,
                            int real_bytes, int fill_halo, int ptr_kind);
/* Reads a field given in the reference layout (halo values are ignored). */
lf2_status lf2_field_import(lf2_ctx* ctx, lf2_field f, const void* src,
                            int halo, int real_bytes, int ptr_kind);
/* Field::updateHalo for a device array already in the reference layout. */
lf2_status lf2_halo_fill(lf2_ctx* ctx, void* data, int comps, int halo,
                         int real_bytes);

/* -------------------------------------------------------------- projections
 * Each call is projection_init + *_project + *_comm of the reference: the
 * field is overwritten with the periodic deposit of the current particles
 * (the upper-halo fold of *_comm is done inside the deposit).
 *   scalar : scalarProjectionCIC_project/_comm (projections.hpp:75-300),
 *            rho = sum m W / res^3, deposit mode of the context.
 *   vector : vectorProjectionCICNGP_project/_comm (:421-681), momentum
 *            m v / res^3, component i on the link x + e_i/2 (NGP along i,
 *            CIC across).  FP32 mode.
 *   tensor : symtensorProjectionCICNGP_project/_comm (:708-976),
 *            T_ii = m v_i^2 at vertices (CIC), T_ij = m v_i v_j on the (i,j)
 *            plaquette (CIC along the third dim).  FP32 mode.
 *   vector CIC : vectorProjectionCIC_project/_comm (:978-1349), m v / res^3,
 *            component i on the link x + e_i/2 with CIC on the staggered
 *            (link-centred) grid along i and CIC across; both halos folded.
 *            FP32 mode.
 *   VecVec CIC : VecVecProjectionCIC_project/_comm (:1355-1814), symmetric
 *            m v_i v_j / res^3 (components 00,01,02,11,12,22): T_ii CIC at the
 *            vertices, T_ij on the (i,j) plaquette centre with staggered CIC
 *            along i and j.  FP32 mode.  The reference's folds for these two
 *            need a process grid of at least 2x2; this library's fold is the
 *            periodic one those grids compute. */
lf2_status lf2_deposit_scalar(lf2_ctx* ctx, lf2_field rho);
lf2_status lf2_deposit_vector_cicngp(lf2_ctx* ctx, lf2_field v);
lf2_status lf2_deposit_symtensor_cicngp(lf2_ctx* ctx, lf2_field t);
lf2_status lf2_deposit_vector_cic(lf2_ctx* ctx, lf2_field v);
lf2_status lf2_deposit_vecvec_cic(lf2_ctx* ctx, lf2_field t);

/* ---------------------------------------------------------- particle moves
 * Particles::updateVel(cic_kick, dtau, &F, 1) (LATfield2_Particles.hpp:
 * 752-893) with the library's CIC gather-kick: vel_c += dtau * sum_k w_k
 * F_c(corner_k), F a 3-component field.  max_v (may be NULL; synchronises)
 * receives the return value of updateVel, sqrt(max |v|^2). */
lf2_status lf2_gather_kick(lf2_ctx* ctx, lf2_field F, double dtau,
                           double* max_v);
/* Particles::moveParticles(move_particles_simple, dtau)
 * (LATfield2_Particles.hpp:1810-2803, move_function.hpp:15-32): drift
 * pos += dtau * vel, periodic wrap and rebin into cells. */
lf2_status lf2_drift_rebin(lf2_ctx* ctx, double dtau);
/* One fused kick-drift-rebin pass (updateVel then moveParticles) followed,
 * when rho is not NULL, by the scalar deposit of the new positions.  In the
 * fixed-point mode, with the pipelined kernel, the deposit of the particles
 * that stay in their brick is fused into the pass (the movers' share is
 * added by a separate kernel); the density is the same bit for bit. */
lf2_status lf2_step(lf2_ctx* ctx, lf2_field F, double dtau_kick,
                    double dtau_drift, lf2_field rho);
/* Kernel of lf2_step's kick-drift-rebin pass: 0 automatic (the persistent
 * TMA-pipelined kernel where the lattice allows it, with the deposit fused
 * in for the fixed-point mode, else the per-brick kernel), 1 the per-brick
 * kernel, 2 the pipelined kernel without the fused deposit, 3 the pipelined
 * kernel with the fused deposit (pipelined kernels need n0 % 4 == 0, every
 * n >= 32 and F 16-byte aligned; the fused deposit the fixed-point mode,
 * else LF2_ERR_UNSUPPORTED).  All give the same particles (the order of the
 * particles inside a brick may differ) and the same fixed-point density; no
 * reference counterpart. */
lf2_status lf2_set_move_kernel(lf2_ctx* ctx, int which);
/* Bounded waits of the pipelined kernel (no reference counterpart): every
 * wait on a copy or on another warp gives up after `cycles` SM clock cycles
 * (0: the default, about 2 s), raises LF2_FLAG_TIMEOUT and leaves the kernel
 * after the copies already issued have landed.  With stall != 0 the consumer
 * warps first wait on a barrier that nothing completes, so that their limit
 * runs out: the way the tests drive this path (the particles of an
 * interrupted pass are not valid; load them again). */
lf2_status lf2_set_wait_limit(lf2_ctx* ctx, int64_t cycles, int stall);
/* Kernel the last lf2_step used for its kick-drift-rebin pass: 1 per-brick,
 * 2 pipelined, 3 pipelined with the fused deposit, 0 before the first step. */
lf2_status lf2_last_move_kernel(lf2_ctx* ctx, int* which);
/* max |v| after the last kick (lf2_step or lf2_gather_kick): the value
 * updateVel returns (LATfield2_Particles.hpp:870-893), from the per-brick
 * maxima the kick already computed.  ptr_kind LF2_PTR_HOST: waits and writes
 * *max_v; LF2_PTR_DEVICE: max_v is device memory, written in stream order
 * without waiting. */
lf2_status lf2_last_max_velocity(lf2_ctx* ctx, double* max_v, int ptr_kind);
/* FP64 conservation sums over all particles: total mass, momentum sum m v
 * and max |v| (cout_particle_velocity_stats, LATfield2_Particles.hpp:
 * 543-583, and the SUM/MAX outputs of updateVel).  Any pointer may be NULL. */
lf2_status lf2_conservation(lf2_ctx* ctx, double* mass, double mom[3],
                            double* max_v);
/* FP64 SUM, MIN and MAX over all particles of |v|^2 (|v|^2 in double from
 * the FP32 components): the reductions updateVel applies (reduce_type SUM,
 * MIN, MAX, LATfield2_Particles.hpp:786-893) to the output the library's
 * kick reports per particle.  MIN over no particles is +infinity.  Any
 * pointer may be NULL; synchronises. */
lf2_status lf2_velocity_reductions(lf2_ctx* ctx, double* sum_v2,
                                   double* min_v2, double* max_v2);

/* ------------------------------------------------------ PM grid operator
 * Fourier transforms of real fields on a cubic lattice, as PlanFFT<Imag>
 * (LATfield2_PlanFFT_decl.hpp:83-230, :720-1050; LF2_ERR_ARG on other
 * lattices), and a Poisson force built on them.
 * A k-field holds the transform of a `comps`-component real field: the
 * Field<Imag> of a Lattice initialised by initializeRealFFT (halo 0,
 * LATfield2_Lattice.hpp:225-258), sizes (n/2+1, n, n).
 *   kfield_export/import: the reference's storage order [k_y][k_z][k_x]
 *     (outermost first; rKSite coord(1) = k_y, coord(2) = k_z,
 *     LATfield2_Site.hpp:319-338), components interleaved, each value
 *     (re, im) of real_bytes (4 or 8).
 *   fft_forward  = execute(FFT_FORWARD):  K(k) = sum_x r(x) exp(-2 pi i k.x/n)
 *   fft_backward = execute(FFT_BACKWARD): r(x) = sum_k K(k) exp(+2 pi i k.x/n)
 *     over the Hermitian extension; neither is normalised; k is kept.
 *   pm_force: phi solves the 7-point lattice Poisson equation
 *     lap(phi) = coupling (rho - mean rho), with the Green's function of the
 *     reference's Poisson example (examples/poissonSolver.cpp) normalised by
 *     1/n^3; then F_i = -(phi(x+e_i) - phi(x-e_i)) / (2 res), periodic,
 *     ready for lf2_gather_kick.  phi (1 component) may be NULL.  Lattices up
 *     to 1024^3 (LF2_ERR_ARG beyond). */
lf2_status lf2_kfield_create(lf2_ctx* ctx, int comps, lf2_kfield* out);
lf2_status lf2_kfield_destroy(lf2_ctx* ctx, lf2_kfield k);
lf2_status lf2_kfield_export(lf2_ctx* ctx, lf2_kfield k, void* dst,
                             int real_bytes, int ptr_kind);
lf2_status lf2_kfield_import(lf2_ctx* ctx, lf2_kfield k, const void* src,
                             int real_bytes, int ptr_kind);
lf2_status lf2_fft_forward(lf2_ctx* ctx, lf2_field r, lf2_kfield k);
lf2_status lf2_fft_backward(lf2_ctx* ctx, lf2_kfield k, lf2_field r);
lf2_status lf2_pm_force(lf2_ctx* ctx, lf2_field rho, lf2_field phi,
                        lf2_field F, double coupling);

/* ------------------------------------------------ PM operator over z slabs
 * The pieces of the PM force when the lattice is split in z over R ranks
 * (the distributed PlanFFT, LATfield2_PlanFFT_decl.hpp:83-230, with a 1-D
 * split: 2-D plane transforms, a transpose, 1-D line transforms).  The
 * global lattice is n^3; a rank owns nz = n / R planes and, after the
 * transpose, nky = n / R values of k_y.  Complex arrays hold (re, im) float
 * pairs; nkx = n/2 + 1.  ctx is the rank's local context (planes n x n).
 *   slab_fft_planes_r2c: planes [nz][n][n] -> A [nz][k_y n][k_x nkx], 2-D
 *     R2C of every plane, unnormalised
 *   slab_fft_planes_c2r: the inverse, unnormalised; A is overwritten
 *   slab_fft_lines: B [z or k_z n][nky][nkx], 1-D C2C along the outer axis
 *     in place, LF2_FFT_FORWARD (exp(-i...)) or LF2_FFT_BACKWARD,
 *     unnormalised
 *   slab_green: B [k_z][k_y - ky0][k_x] *= the Green's function of
 *     lf2_pm_force (coupling, 1/n^3 included, zero mode removed); B 16-byte
 *     aligned
 *   pm_gradient: F_i = -(phi(x+e_i) - phi(x-e_i)) / (2 res) on ctx's
 *     lattice, periodic (with filled ghost planes, exact on the own planes)
 * The transforms run on ctx's stream.  A slab FFT belongs to its context:
 * destroy it before the context. */
#define LF2_FFT_FORWARD 1
#define LF2_FFT_BACKWARD (-1)
lf2_status lf2_slab_fft_create(lf2_ctx* ctx, int n, int nz, int nky,
                               lf2_slab_fft* out);
lf2_status lf2_slab_fft_destroy(lf2_slab_fft p);
lf2_status lf2_slab_fft_planes_r2c(lf2_slab_fft p, const float* planes, void* A);
lf2_status lf2_slab_fft_planes_c2r(lf2_slab_fft p, void* A, float* planes);
lf2_status lf2_slab_fft_lines(lf2_slab_fft p, void* B, int direction);
lf2_status lf2_slab_green(lf2_slab_fft p, void* B, int ky0, double coupling);
lf2_status lf2_pm_gradient(lf2_ctx* ctx, lf2_field phi, lf2_field F);

/* ------------------------------------------------- differentiable PM chain
 * Particle kernels on arrays kept in the caller's order (no rebinning, so
 * gradients stay attached to their particles), for the adjoint of a
 * multi-step particle-mesh chain.  They have no reference counterpart beyond
 * the forward operations they differentiate: the CIC deposit
 * (scalarProjectionCIC_project, projections.hpp:75-184), the CIC gather-kick
 * of updateVel (LATfield2_Particles.hpp:752-893) and the drift of
 * move_particles_simple (move_function.hpp:15-32).  All pointers are device
 * pointers; offsets and offset gradients are in cell units; outputs marked
 * (+=) are accumulated.  mass may be NULL (global mass gmass).
 * The force field F4 and its gradient g_F4 hold one float4 (x, y, z, unused)
 * per site, in site order, 16-byte aligned (LF2_ERR_ARG otherwise).
 *   deposit          rho (+=) m/res^3 W                (FP32 atomics; in a
 *                    context of the fixed-point mode: 64-bit integer sums of
 *                    the deterministic corner weights of lf2_deposit_scalar,
 *                    times m / M in 2^-24 units with M the largest mass of
 *                    the call, converted once, so independent of the order)
 *   gather           out3[p] = sum_k W_k F4(corner_k)
 *   kick_drift       vel += dt_kick * G3 (G3 may be NULL); off += dt_drift/res
 *                    * vel with the carry into cell
 *   deposit_adjoint  g_off3 (+=), g_mass (+=) from g_rho
 *   gather_adjoint   g_F4 (+=) CIC deposit of g_out3; g_off3 (+=)
 *   stencil27        F4_c(g) = sum_o S[c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1)]
 *                    rho(g + o), periodic, S81 on the device
 *   stencil27_adjoint g_rho (+=) and g_S81 (+=) from g_F4
 *   pm_force4        the PM force of lf2_pm_force as the chain's grid
 *                    operator: F4 = (F_x, F_y, F_z, 0) from rho (cubic
 *                    lattices up to 1024^3)
 *   pm_force4_adjoint g_rho (+=) from g_F4: the divergence
 *                    g_phi(y) = sum_c (g_F_c(y+e_c) - g_F_c(y-e_c)) / (2 res),
 *                    then the same Green's-function solve (self-adjoint) */
/* The chain's particle state from box-unit FP64 positions, and its
 * gradients back to the caller's order (all device pointers, no wait).  The
 * permutations move one 32-byte record per particle (`records`: 32 bytes
 * per particle, 16-byte aligned), a full sector each way:
 *   pm_state_pack    caller order: the sort key of particle i (its brick
 *                    times 4096 plus its cell's place in the brick, x
 *                    fastest; LF2_ERR_UNSUPPORTED when nbricks * 4096 does
 *                    not fit 31 bits) and its record: the cell of pos3[i]
 *                    (u = pos * inv_res per dim, floor, the offset u -
 *                    floor(u) rounded to FP32, an offset that rounds to 1
 *                    carrying into the next cell, periodic wrap), offsets,
 *                    velocity and mass rounded to FP32 (mass may be NULL: 0)
 *   pm_state_unpack  slot i <- the record of particle order[i] (mass may be
 *                    NULL: not written)
 *   pm_brick_start   brick_start[b] (nbricks + 1 entries): the first slot of
 *                    brick b among cells sorted by the pack's key
 *   pm_grads_unorder g_pos3_out[order[i]] = g_off3[i] * inv_res,
 *                    g_vel3_out[order[i]] = g_vel3[i], g_mass_out[order[i]] =
 *                    g_mass[i], in FP64, through `records` as scratch
 *   pm_deposit_bricks  pm_deposit of particles grouped by brick_start: one
 *                    CTA per brick sums in a shared vertex tile and adds the
 *                    tile to the field; a particle that has left its group's
 *                    brick since is deposited on its own.  The same sums in
 *                    the fixed-point mode; FP32 roundings in another order.
 *                    brick_start must come from cells sorted by the key. */
lf2_status lf2_pm_state_pack(lf2_ctx* ctx, int64_t np, const double* pos3,
                             const double* vel3, const double* mass,
                             double inv_res, int32_t* key, void* records);
lf2_status lf2_pm_state_unpack(lf2_ctx* ctx, int64_t np, const int64_t* order,
                               const void* records, int32_t* cell,
                               float* off3, float* vel3, float* mass);
lf2_status lf2_pm_brick_start(lf2_ctx* ctx, int64_t np, const int32_t* cell,
                              int64_t* brick_start);
lf2_status lf2_pm_grads_unorder(lf2_ctx* ctx, int64_t np,
                                const int64_t* order, const float* g_off3,
                                const float* g_vel3, const float* g_mass,
                                double inv_res, void* records,
                                double* g_pos3_out, double* g_vel3_out,
                                double* g_mass_out);
lf2_status lf2_pm_deposit_bricks(lf2_ctx* ctx, int64_t np, const int32_t* cell,
                                 const float* off3, const float* mass,
                                 double gmass, const int64_t* brick_start,
                                 float* rho);
lf2_status lf2_pm_deposit(lf2_ctx* ctx, int64_t np, const int32_t* cell,
                          const float* off3, const float* mass, double gmass,
                          float* rho);
lf2_status lf2_pm_gather(lf2_ctx* ctx, int64_t np, const int32_t* cell,
                         const float* off3, const float* F4, float* out3);
lf2_status lf2_pm_kick_drift(lf2_ctx* ctx, int64_t np, int32_t* cell,
                             float* off3, float* vel3, const float* G3,
                             double dt_kick, double dt_drift);
/* gather + kick_drift in one pass, the same results bit for bit:
 * vel += dt_kick * sum_k W_k F4(corner_k), then the drift. */
lf2_status lf2_pm_step(lf2_ctx* ctx, int64_t np, int32_t* cell, float* off3,
                       float* vel3, const float* F4, double dt_kick,
                       double dt_drift);
lf2_status lf2_pm_deposit_adjoint(lf2_ctx* ctx, int64_t np,
                                  const int32_t* cell, const float* off3,
                                  const float* mass, double gmass,
                                  const float* g_rho, float* g_off3,
                                  float* g_mass);
lf2_status lf2_pm_gather_adjoint(lf2_ctx* ctx, int64_t np,
                                 const int32_t* cell, const float* off3,
                                 const float* F4, const float* g_out3,
                                 float* g_F4, float* g_off3);
lf2_status lf2_stencil27(lf2_ctx* ctx, const float* rho, const float* S81,
                         float* F4);
lf2_status lf2_stencil27_adjoint(lf2_ctx* ctx, const float* rho,
                                 const float* S81, const float* g_F4,
                                 float* g_rho, float* g_S81);
lf2_status lf2_pm_force4(lf2_ctx* ctx, const float* rho, float* F4,
                         double coupling);
lf2_status lf2_pm_force4_adjoint(lf2_ctx* ctx, const float* g_F4,
                                 float* g_rho, double coupling);

/* ---------------------------------------------------------- no allocation
 * Scalar CIC deposit that allocates no device memory.  It has no
 * counterpart in the reference; it exists for callers that may not allocate
 * device memory while running (an application whose device memory comes
 * from its own pool, a plugin allowed to allocate only at load time, a
 * time-critical loop that cannot pay for cudaMalloc's synchronisation).
 * No context is needed: the caller passes device inputs and the output.
 *   cell[np], off3[3*np]  particles grouped by brick: brick b (BRICK^3 = 16^3
 *                         cells; bricks numbered bx + nbx*(by + nby*bz),
 *                         nbi = ceil(n[i]/16)) owns entries
 *                         [brick_start[b], brick_start[b+1]); cells and
 *                         offsets as in lf2_particles_set
 *   brick_start[nb+1]     int64, device
 *   rho[n0*n1*n2]         FP32 output, internal layout, overwritten
 * Mass is global (particle_mass); deposit_mode as for lf2_create.  The
 * scratch (the per-brick shell store) is a fixed 16 MiB device array inside
 * the library, present on every GPU that loads it until the process exits,
 * so lattices with more than LF2_NOALLOC_MAX_BRICKS bricks are rejected with
 * LF2_ERR_UNSUPPORTED.  Every call looks the array's device address up in
 * the current device's context (cudaGetSymbolAddress); make the first call
 * on a device before any stream capture.  Calls share the array: calls that
 * overlap on the GPU race and must be serialised.  The work is queued on
 * `stream` (NULL: default stream).  brick_start is checked on the device:
 * it must start at 0, never decrease and end at np or below; a brick whose
 * range breaks that is clamped to [0, np] and reported.  With flags != NULL
 * the call waits for the work and returns the device error bits
 * (LF2_FLAG_BAD_CELL for a particle outside its brick, an offset outside
 * [0,1) or a bad brick range), with LF2_ERR_STATE if any.  With flags ==
 * NULL nothing is waited for and such errors are not reported: the call
 * returns LF2_OK.  A runtime error left pending by an earlier, unrelated
 * CUDA call is picked up by the launch checks and fails the call with
 * LF2_ERR_CUDA. */
#define LF2_NOALLOC_MAX_BRICKS 1363
lf2_status lf2_deposit_scalar_noalloc(const int n[3], const double box[3],
                                      int deposit_mode, double particle_mass,
                                      int64_t np, const int32_t* cell,
                                      const float* off3,
                                      const int64_t* brick_start, float* rho,
                                      void* stream, uint32_t* flags);

/* ------------------------------------------------------------- measurement
 * Per-phase device time, measured with CUDA events recorded on the context's
 * stream around each kernel (no extra synchronisation while running).
 * Phases: 0 gather-kick/drift/rebin pass, 1 mover insertion and repack,
 * 2 deposit tile pass, 3 deposit face fix-up, 4 other kernels.  The
 * launch counter counts every kernel this library launched. */
#define LF2_NPHASE 5
lf2_status lf2_profile_enable(lf2_ctx* ctx, int on);
/* Synchronises; adds the milliseconds and launches of each phase since the
 * previous read into ms[LF2_NPHASE] / launches[LF2_NPHASE] (either may be
 * NULL) and resets the accumulators. */
lf2_status lf2_profile_read(lf2_ctx* ctx, double* ms, int64_t* launches);
/* Total kernel launches since the context was created. */
lf2_status lf2_kernel_launches(lf2_ctx* ctx, int64_t* n);
/* Rebin diagnostics (synchronises): full store repacks and single-brick
 * relocations since the context was created, and the number of particles
 * that changed brick in the last drift.  Any pointer may be NULL. */
lf2_status lf2_rebin_stats(lf2_ctx* ctx, int64_t* repacks, int64_t* relocations,
                           int64_t* movers);

#ifdef __cplusplus
}
#endif
#endif
