// A particle-mesh loop written against LATfield2's particle interface, built
// against include/latfield2_b200.hpp (the GPU path) instead of LATfield2.hpp.
//
//   compat_demo N NPART OUT
//
// Seeded particles in a unit box; one scalar projection, the CIC kick with a
// force field set on the host, the drift, then the scalar, vector CIC-NGP,
// symtensor CIC-NGP, vector CIC and VecVec CIC projections.
// Everything the checks need goes to OUT as raw arrays (see write_all).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "latfield2_b200.hpp"

using namespace LATfield2;

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static double uniform()
{
  rng_state = rng_state * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(rng_state >> 11) * (1.0 / 9007199254740992.0);
}

// interior values of a field, [z][y][x][c], as double
static std::vector<double> interior(Field<Real>& f)
{
  Lattice& lat = f.lattice();
  std::vector<double> out;
  Site x(lat);
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
    fprintf(stderr, "usage: compat_demo N NPART OUT\n");
    return 2;
  }
  const int N = atoi(argv[1]);
  const long npart = atol(argv[2]);
  Real boxSize[3] = {1, 1, 1};
  const double dtau = 0.1;

  Lattice lat(3, N, 1), lat_part(3, N, 0);
  Field<Real> rho(lat, 1), F(lat, 3), B(lat, 3), Tij(lat, 3, 3, symmetric);
  Field<Real> V(lat, 3), VV(lat, 3, 3, symmetric);

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
    if (!parts.addParticle_global(p)) continue;
    id0.push_back((double)p.ID);
    for (int d = 0; d < 3; d++) pos0.push_back((double)p.pos[d]), vel0.push_back((double)p.vel[d]);
  }

  projection_init(&rho);
  scalarProjectionCIC_project(&parts, &rho);
  scalarProjectionCIC_comm(&rho);
  std::vector<double> rho0 = interior(rho);

  // a smooth periodic force set on the host
  Site x(lat);
  for (x.first(); x.test(); x.next())
    for (int c = 0; c < 3; c++)
      F(x, c) = (Real)(0.01 * std::sin(2 * M_PI * (x.coord(c) + 0.5 * c) / N) *
                       std::cos(2 * M_PI * x.coord((c + 1) % 3) / N));
  F.updateHalo();
  std::vector<double> Fv = interior(F);
  Field<Real>* Fp = &F;
  const double maxv = parts.updateVel(cic_gather_kick, dtau, &Fp, 1);
  parts.moveParticles(move_particles_simple, dtau);

  projection_init(&rho);
  scalarProjectionCIC_project(&parts, &rho);
  scalarProjectionCIC_comm(&rho);
  vectorProjectionCICNGP_project(&parts, &B);
  vectorProjectionCICNGP_comm(&B);
  symtensorProjectionCICNGP_project(&parts, &Tij);
  symtensorProjectionCICNGP_comm(&Tij);
  vectorProjectionCIC_project(&parts, &V);
  vectorProjectionCIC_comm(&V);
  VecVecProjectionCIC_project(&parts, &VV);
  VecVecProjectionCIC_comm(&VV);

  std::vector<part_simple> out;
  parts.getParticles(out);
  std::vector<double> pos1(3 * out.size()), vel1(3 * out.size()), id1(out.size());
  for (size_t i = 0; i < out.size(); i++) {
    id1[i] = (double)out[i].ID;
    for (int d = 0; d < 3; d++) pos1[3 * i + d] = out[i].pos[d], vel1[3 * i + d] = out[i].vel[d];
  }

  FILE* fp = fopen(argv[3], "wb");
  if (!fp) return 1;
  const double header[4] = {(double)N, (double)parts.numParticles(), dtau, maxv};
  put(fp, std::vector<double>(header, header + 4));
  for (auto* v : {&id0, &pos0, &vel0, &rho0, &Fv, &id1, &pos1, &vel1})
    put(fp, *v);
  put(fp, interior(rho));
  put(fp, interior(B));
  put(fp, interior(Tij));
  put(fp, interior(V));
  put(fp, interior(VV));
  fclose(fp);
  printf("ok %ld particles, max|v| %.6e, sizeof(Real) %zu\n", parts.numParticles(), maxv, sizeof(Real));
  return 0;
}
