// The parts of the reference's particle interface around the kick and the
// projections that a user program may lean on, run through
// include/latfield2_b200.hpp:
//   - updateVel's outputs: the kick reports |v|^2 per particle; output[i]
//     is reduced with reduce_type[i] (SUM, MIN, MAX);
//   - the mappingClass overload of updateVel (LATfield2_Particles.hpp:191-200);
//   - the projections' oset / flag_where (projections.hpp:115-126): the mass
//     read at a byte offset of part_info, or the particle type's own members;
//     an offset the GPU store does not hold is refused.
//
//   outputs_demo N NPART OUT
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "latfield2_b200.hpp"

using namespace LATfield2;

struct Mapping {
  int unused = 0;
};

static uint64_t rng_state = 0x2545F4914F6CDD1Dull;
static double uniform()
{
  rng_state = rng_state * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(rng_state >> 11) * (1.0 / 9007199254740992.0);
}

static std::vector<double> interior(Field<Real>& f)
{
  std::vector<double> out;
  Site x(f.lattice());
  for (x.first(); x.test(); x.next())
    for (int c = 0; c < f.components(); c++) out.push_back((double)f(x, c));
  return out;
}

static void put(FILE* fp, const std::vector<double>& v)
{
  const int64_t n = (int64_t)v.size();
  fwrite(&n, sizeof n, 1, fp);
  fwrite(v.data(), sizeof(double), v.size(), fp);
}

int main(int argc, char** argv)
{
  if (argc != 4) {
    fprintf(stderr, "usage: outputs_demo N NPART OUT\n");
    return 2;
  }
  const int N = atoi(argv[1]);
  const long npart = atol(argv[2]);
  Real boxSize[3] = {1, 1, 1};
  const double dtau = 0.1;
  Lattice lat(3, N, 1), lat_part(3, N, 0);
  Field<Real> rho(lat, 1), rho2(lat, 1), F(lat, 3), B(lat, 3);

  part_simple_info info;
  info.mass = 1.0 / npart;
  info.relativistic = 0;
  part_simple_dataType type;
  Particles<part_simple, part_simple_info, part_simple_dataType> parts;
  parts.initialize(info, type, &lat_part, boxSize);
  std::vector<double> pos0, vel0, id0;
  part_simple p;
  for (long i = 0; i < npart; i++) {
    p.ID = i;
    for (int d = 0; d < 3; d++) p.pos[d] = (Real)uniform();
    for (int d = 0; d < 3; d++) p.vel[d] = (Real)(0.02 * (uniform() - 0.5));
    parts.addParticle_global(p);
    id0.push_back((double)p.ID);
    for (int d = 0; d < 3; d++) pos0.push_back((double)p.pos[d]), vel0.push_back((double)p.vel[d]);
  }
  Site x(lat);
  for (x.first(); x.test(); x.next())
    for (int c = 0; c < 3; c++)
      F(x, c) = (Real)(0.01 * std::cos(2 * M_PI * (x.coord((c + 2) % 3) + 0.25 * c) / N));
  F.updateHalo();
  std::vector<double> Fv = interior(F);
  Field<Real>* Fp = &F;

  // updateVel with three outputs reduced as SUM, MIN, MAX
  double out3[3];
  int red3[3] = {SUM, MIN, MAX};
  const double maxv1 = parts.updateVel(cic_gather_kick, dtau, &Fp, 1, NULL, out3, red3, 3);
  // the same kick through the mappingClass overload, outputs MAX and SUM
  Mapping map;
  double out2[2];
  int red2[2] = {MAX, SUM};
  const double maxv2 = parts.updateVel(cic_gather_kick_mapped<part_simple, part_simple_info, Mapping>,
                                       dtau, &Fp, 1, &map, NULL, out2, red2, 2);

  // projections: default members, oset naming the same members, and the
  // part_info mass at its offset after the user doubled it
  size_t oset[2] = {offsetof(part_simple_info, mass), offsetof(part_simple, vel)};
  projection_init(&rho);
  scalarProjectionCIC_project(&parts, &rho);
  scalarProjectionCIC_comm(&rho);
  vectorProjectionCICNGP_project(&parts, &B, oset, FROM_INFO);
  vectorProjectionCICNGP_comm(&B);
  parts.parts_info()->mass *= 2;
  projection_init(&rho2);
  scalarProjectionCIC_project(&parts, &rho2, oset, FROM_INFO);
  scalarProjectionCIC_comm(&rho2);
  parts.parts_info()->mass /= 2;
  // an offset the GPU store does not hold (the particle ID) is refused
  int refused = 0;
  try {
    size_t bad[2] = {offsetof(part_simple_info, mass), offsetof(part_simple, ID)};
    vectorProjectionCICNGP_project(&parts, &B, bad, FROM_INFO);
  } catch (const std::invalid_argument&) {
    refused = 1;
  }
  try {
    size_t bad = offsetof(part_simple, ID);
    scalarProjectionCIC_project(&parts, &rho, &bad, FROM_PART);
  } catch (const std::invalid_argument&) {
    refused += 1;
  }

  FILE* fp = fopen(argv[3], "wb");
  if (!fp) return 1;
  put(fp, {(double)N, (double)npart, dtau, maxv1, maxv2, out3[0], out3[1], out3[2], out2[0], out2[1],
           (double)refused});
  for (auto* v : {&id0, &pos0, &vel0, &Fv}) put(fp, *v);
  put(fp, interior(rho));
  put(fp, interior(rho2));
  put(fp, interior(B));
  fclose(fp);
  printf("ok refused %d\n", refused);
  return 0;
}
