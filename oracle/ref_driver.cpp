// ref_driver.cpp -- runs the reference's own particle path on given inputs and
// writes its results, to pin the oracle and the golden fixtures.
// TEST INFRASTRUCTURE ONLY (built by oracle/build_ref.sh into oracle/_ref/).
//
// It includes the reference headers unmodified (LATfield2.hpp) with the
// builder-written MPI stand-in (mpi_shim/mpi.h).  Two things are added around
// them, both outside the reference sources:
//  - a partList<part_simple> specialisation that also answers `.size != 0`:
//    vectorProjectionCICNGP_project and symtensorProjectionCICNGP_project
//    test `parts->field()(xPart).size != 0` (projections.hpp:473, :761,
//    :1038, :1414), a
//    member the shipped partList no longer has (LATfield2_Particles.hpp:
//    97-103); here it means "the list is not empty", the intent of the test;
//  - the CIC gather-kick callback for updateVel (the reference ships only the
//    no-op updateVel_simple), the same arithmetic as the oracle's
//    lf2o_update_vel_cic.
//
// Input  (little endian): "LF2G", int32 version=1, int32 n, int32 halo,
//        int32 grid0, int32 grid1, double box, double gmass, int32 ops,
//        double dtau_kick, double dtau_move, int64 np,
//        np x {int64 id; double pos[3]; double vel[3]},
//        if ops & OP_KICK: n^3 x 3 doubles, the force field F[z][y][x][c].
// Output (one file per rank, <prefix>.<rank>): int32 rank, int32 coordSkip0
//        (z offset), int32 coordSkip1 (y offset), int32 sizeLocal[3], int32 halo,
//        then the local gross field (double) of each requested deposit in the
//        order scalar, vector CIC-NGP, symtensor CIC-NGP, vector CIC,
//        VecVec CIC, then the halo-filled F; for the kick: double max_v,
//        int64 nloc, nloc x {id, pos[3], vel[3]}; for the move: int64 nloc,
//        nloc x {id, pos[3], vel[3]}.  The vector-CIC and VecVec-CIC folds
//        (sendUpDown) need a process grid of at least 2x2.
//        OP_FFT (built with -DFFT3D against oracle/fftw_shim): component 0 of
//        F as a real field through PlanFFT::execute(FFT_FORWARD), written as
//        int32 kSizeLocal[3], int32 kSkip[2] (storage dims 2 and 1), then the
//        local k-field as (re, im) doubles; then FFT_BACKWARD of that k-field,
//        the local gross real field.  OP_POISSON: the reference's Poisson
//        example (examples/poissonSolver.cpp) on the same real field, res =
//        1/n: the local gross potential.
//        With LF2_REF_FIELD_WRITE=<path>, the vector CIC-NGP field is also
//        written to <path> by the reference's Field::write.
#include <cstdint>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "LATfield2.hpp"

using namespace LATfield2;

struct part_simple_dataType {};

namespace LATfield2 {
template <>
struct partList<part_simple> {
  struct NonEmpty {
    bool operator!=(int v) const
    {
      const partList* self = reinterpret_cast<const partList*>(this);
      return v == 0 ? !self->parts.empty() : true;
    }
  } size;  // first member: its address is the list's address
  std::forward_list<part_simple> parts;
  partList() : size(), parts() {}
};
}  // namespace LATfield2

enum {
  OP_SCALAR = 1,
  OP_VECTOR = 2,
  OP_TENSOR = 4,
  OP_HALO = 8,
  OP_KICK = 16,
  OP_MOVE = 32,
  OP_VECCIC = 64,
  OP_VECVEC = 128,
  OP_FFT = 256,
  OP_POISSON = 512
};

// CIC gather of the 3-component field at the cell corners and kick, in the
// callback signature of Particles::updateVel (LATfield2_Particles.hpp:753).
Real cic_kick(double dtau, double lat_resolution, part_simple* part, double* frac,
              part_simple_info info, Field<Real>** fields, Site* sites, int nfield,
              double* params, double* outputs, int noutputs)
{
  Field<Real>& F = *fields[0];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 8; k++) {
    const int b[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
    double w = 1.0;
    Site c = sites[0];
    for (int l = 0; l < 3; l++) {
      w *= b[l] ? frac[l] : 1.0 - frac[l];
      if (b[l]) c = c + l;
    }
    for (int cc = 0; cc < 3; cc++) acc[cc] += w * F(c, cc);
  }
  double v2 = 0.0;
  for (int cc = 0; cc < 3; cc++) {
    part->vel[cc] += dtau * acc[cc];
    v2 += (double)part->vel[cc] * (double)part->vel[cc];
  }
  if (noutputs > 0) outputs[0] = v2;
  return v2;
}

template <typename T>
static void rd(FILE* f, T* p, size_t n)
{
  if (fread(p, sizeof(T), n, f) != n) {
    fprintf(stderr, "ref_driver: short input\n");
    exit(2);
  }
}

template <typename T>
static void wr(FILE* f, const T* p, size_t n)
{
  fwrite(p, sizeof(T), n, f);
}

static void write_field(FILE* o, Field<Real>& f)
{
  const long gross = f.lattice().sitesLocalGross() * (long)f.components();
  std::vector<double> buf(gross);
  for (long i = 0; i < gross; i++) buf[i] = (double)f(i);
  wr(o, buf.data(), buf.size());
}

static void write_particles(FILE* o, Particles<part_simple, part_simple_info, part_simple_dataType>& parts)
{
  std::vector<double> rec;
  std::vector<int64_t> ids;
  Site x(parts.lattice());
  for (x.first(); x.test(); x.next())
    for (auto it = parts.field()(x).parts.begin(); it != parts.field()(x).parts.end(); ++it) {
      ids.push_back(it->ID);
      for (int l = 0; l < 3; l++) rec.push_back((double)it->pos[l]);
      for (int l = 0; l < 3; l++) rec.push_back((double)it->vel[l]);
    }
  const int64_t n = (int64_t)ids.size();
  wr(o, &n, 1);
  for (int64_t i = 0; i < n; i++) {
    wr(o, &ids[i], 1);
    wr(o, &rec[6 * i], 6);
  }
}

int main(int argc, char** argv)
{
  if (argc < 3) {
    fprintf(stderr, "usage: %s input.bin output_prefix\n", argv[0]);
    return 2;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) {
    perror("input");
    return 2;
  }
  char magic[4];
  rd(in, magic, 4);
  int32_t version, n, halo, g0, g1, ops;
  double box, gmass, dtk, dtm;
  int64_t np;
  rd(in, &version, 1);
  rd(in, &n, 1);
  rd(in, &halo, 1);
  rd(in, &g0, 1);
  rd(in, &g1, 1);
  rd(in, &box, 1);
  rd(in, &gmass, 1);
  rd(in, &ops, 1);
  rd(in, &dtk, 1);
  rd(in, &dtm, 1);
  rd(in, &np, 1);
  if (memcmp(magic, "LF2G", 4) != 0 || version != 1) {
    fprintf(stderr, "ref_driver: bad input header\n");
    return 2;
  }

  parallel.initialize(g0, g1);

  Lattice lat_part(3, n, 0);
  Lattice lat(3, n, halo);
  Real boxSize[3] = {(Real)box, (Real)box, (Real)box};
  part_simple_info info;
  info.mass = gmass;
  info.relativistic = 0;
  set_parts_typename(&info, "part_simple");
  part_simple_dataType dtype;
  Particles<part_simple, part_simple_info, part_simple_dataType> parts;
  parts.initialize(info, dtype, &lat_part, boxSize);

  // Every rank reads every particle (in chunks of records) and offers it to
  // addParticle_global, which keeps the ones in its local domain.
  {
    const int64_t CH = 1 << 16;
    std::vector<unsigned char> buf((size_t)CH * 56);
    for (int64_t i0 = 0; i0 < np; i0 += CH) {
      const int64_t m = np - i0 < CH ? np - i0 : CH;
      rd(in, buf.data(), (size_t)m * 56);
      for (int64_t i = 0; i < m; i++) {
        int64_t id;
        double pv[6];
        memcpy(&id, &buf[(size_t)i * 56], 8);
        memcpy(pv, &buf[(size_t)i * 56 + 8], 48);
        part_simple p;
        p.ID = id;
        for (int l = 0; l < 3; l++) {
          p.pos[l] = (Real)pv[l];
          p.vel[l] = (Real)pv[3 + l];
        }
        parts.addParticle_global(p);
      }
    }
  }

  // The force field, read one z plane at a time; each rank keeps its sites.
  Field<Real> F(lat, 3);
  if (ops & (OP_HALO | OP_KICK | OP_FFT | OP_POISSON)) {
    std::vector<double> plane((size_t)n * n * 3);
    const long z0 = lat.coordSkip()[0], z1 = z0 + lat.sizeLocal(2);
    const long y0 = lat.coordSkip()[1], y1 = y0 + lat.sizeLocal(1);
    Site x(lat);
    for (long gz = 0; gz < n; gz++) {
      rd(in, plane.data(), plane.size());
      if (gz < z0 || gz >= z1) continue;
      for (long gy = y0; gy < y1; gy++)
        for (long gx = 0; gx < n; gx++) {
          int c3[3] = {(int)gx, (int)gy, (int)gz};
          if (!x.setCoord(c3)) continue;
          for (int c = 0; c < 3; c++) F(x, c) = (Real)plane[(gy * (size_t)n + gx) * 3 + c];
        }
    }
    F.updateHalo();
  }
  fclose(in);

  // Timing mode (LF2_REF_STEPS=K, LF2_REF_WARMUP=W): W untimed steps, then K
  // particle-mesh steps of the reference as a user's loop runs them --
  // scalarProjectionCIC_project + _comm, updateVel with the CIC kick,
  // moveParticles -- each between two barriers; rank 0 prints the total and
  // the per-step wall times as one JSON line.  Nothing is written.
  if (const char* ks = getenv("LF2_REF_STEPS")) {
    const int steps = atoi(ks);
    const char* ws = getenv("LF2_REF_WARMUP");
    const int warm = ws ? atoi(ws) : 0;
    Field<Real> rho(lat, 1);
    Field<Real>* fl[1] = {&F};
    double out1[1];
    int red[1] = {SUM};
    std::vector<double> per;
    double sec = 0.0;
    for (int s = 0; s < warm + steps; s++) {
      parallel.barrier();
      const auto t0 = std::chrono::steady_clock::now();
      projection_init(&rho);
      scalarProjectionCIC_project(&parts, &rho);
      scalarProjectionCIC_comm(&rho);
      parts.updateVel(&cic_kick, dtk, fl, 1, NULL, out1, red, 1);
      parts.moveParticles(&move_particles_simple, dtm);
      parallel.barrier();
      const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (s >= warm) {
        per.push_back(dt);
        sec += dt;
      }
    }
    long nloc = 0;
    {
      Site xp(parts.lattice());
      for (xp.first(); xp.test(); xp.next())
        for (auto it = parts.field()(xp).parts.begin(); it != parts.field()(xp).parts.end(); ++it) nloc++;
    }
    parallel.sum(nloc);
    if (parallel.rank() == 0) {
      printf("{\"seconds\": %.6f, \"steps\": %d, \"warmup\": %d, \"particles\": %lld, "
             "\"particles_after\": %ld, \"ranks\": %d, \"step_seconds\": [",
             sec, steps, warm, (long long)np, nloc, g0 * g1);
      for (size_t i = 0; i < per.size(); i++) printf("%s%.6f", i ? ", " : "", per[i]);
      printf("]}\n");
    }
    return 0;
  }

  const std::string out_name = std::string(argv[2]) + "." + std::to_string(parallel.rank());
  FILE* o = fopen(out_name.c_str(), "wb");
  if (!o) {
    perror("output");
    return 3;
  }
  const int32_t rank = parallel.rank();
  const int32_t skip0 = (int32_t)lat.coordSkip()[0], skip1 = (int32_t)lat.coordSkip()[1];
  const int32_t sl[3] = {lat.sizeLocal(0), lat.sizeLocal(1), lat.sizeLocal(2)};
  wr(o, &rank, 1);
  wr(o, &skip0, 1);
  wr(o, &skip1, 1);
  wr(o, sl, 3);
  wr(o, &halo, 1);

  if (ops & OP_SCALAR) {
    Field<Real> rho(lat, 1);
    projection_init(&rho);
    scalarProjectionCIC_project(&parts, &rho);
    scalarProjectionCIC_comm(&rho);
    write_field(o, rho);
  }
  if (ops & OP_VECTOR) {
    Field<Real> B(lat, 3);
    projection_init(&B);
    vectorProjectionCICNGP_project(&parts, &B);
    vectorProjectionCICNGP_comm(&B);
    write_field(o, B);
    // the reference's own binary field file (Field::write), when asked
    if (const char* fw = getenv("LF2_REF_FIELD_WRITE")) B.write(fw);
  }
  if (ops & OP_TENSOR) {
    Field<Real> T(lat, 3, 3, symmetric);
    projection_init(&T);
    symtensorProjectionCICNGP_project(&parts, &T);
    symtensorProjectionCICNGP_comm(&T);
    write_field(o, T);
  }
  if (ops & OP_VECCIC) {
    Field<Real> V(lat, 3);
    projection_init(&V);
    vectorProjectionCIC_project(&parts, &V);
    vectorProjectionCIC_comm(&V);
    write_field(o, V);
  }
  if (ops & OP_VECVEC) {
    Field<Real> T(lat, 3, 3, symmetric);
    projection_init(&T);
    VecVecProjectionCIC_project(&parts, &T);
    VecVecProjectionCIC_comm(&T);
    write_field(o, T);
  }
  if (ops & OP_HALO) write_field(o, F);
#ifdef FFT3D
  if (ops & (OP_FFT | OP_POISSON)) {
    Lattice latK;
    latK.initializeRealFFT(lat, 0);
    Field<Real> r(lat, 1), back(lat, 1);
    Field<Imag> rK(latK, 1), backK(latK, 1);
    PlanFFT<Imag> plan(&r, &rK);
    PlanFFT<Imag> planBack(&back, &backK);
    Site x(lat);
    for (x.first(); x.test(); x.next()) r(x) = F(x, 0);
    plan.execute(FFT_FORWARD);
    if (ops & OP_FFT) {
      const int32_t ks[5] = {latK.sizeLocal(0), latK.sizeLocal(1), latK.sizeLocal(2),
                             (int32_t)latK.coordSkip()[0], (int32_t)latK.coordSkip()[1]};
      wr(o, ks, 5);
      const long kg = latK.sitesLocalGross();
      std::vector<double> buf(2 * kg);
      for (long i = 0; i < kg; i++) {
        buf[2 * i] = (double)rK(i).real();
        buf[2 * i + 1] = (double)rK(i).imag();
      }
      wr(o, buf.data(), buf.size());
      for (long i = 0; i < kg; i++) backK(i) = rK(i);
      planBack.execute(FFT_BACKWARD);
      write_field(o, back);
    }
    if (ops & OP_POISSON) {
      // examples/poissonSolver.cpp, with the lattice of this run and res = 1/n
      const double res = 1.0 / n, res2 = res * res;
      rKSite k(latK);
      k.first();
      if (parallel.isRoot()) {
        backK(k) = 0.0;
        k.next();
      }
      for (; k.test(); k.next())
        backK(k) = rK(k) / (2.0 * (cos(2.0 * M_PI * k.coord(0) / n) + cos(2.0 * M_PI * k.coord(1) / n) +
                                   cos(2.0 * M_PI * k.coord(2) / n) - 3.0) / res2);
      planBack.execute(FFT_BACKWARD);
      write_field(o, back);
    }
  }
#endif
  if (ops & OP_KICK) {
    Field<Real>* fl[1] = {&F};
    double out1[1];
    int red[1] = {SUM};
    const double maxv = parts.updateVel(&cic_kick, dtk, fl, 1, NULL, out1, red, 1);
    wr(o, &maxv, 1);
    write_particles(o, parts);
  }
  if (ops & OP_MOVE) {
    parts.moveParticles(&move_particles_simple, dtm);
    write_particles(o, parts);
  }
  fclose(o);
  return 0;
}
