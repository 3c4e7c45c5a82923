// A restart through Particles::saveHDF5 / loadHDF5 of
// include/latfield2_b200.hpp:
//
//   restart_demo N NPART DIR
//
// Seeded particles take two kick-drift steps and are saved; a second particle
// set loads the file; both take two more steps.  Prints "ok" when the two
// sets then hold the same particles (ID, position, velocity) bit for bit and
// their scalar projections are equal.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "latfield2_b200.hpp"

using namespace LATfield2;

typedef Particles<part_simple, part_simple_info, part_simple_dataType> PS;

static uint64_t rng_state = 0x2545F4914F6CDD1Dull;
static double uniform()
{
  rng_state = rng_state * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(rng_state >> 11) * (1.0 / 9007199254740992.0);
}

static void steps(PS& parts, Field<Real>& F, int k)
{
  Field<Real>* Fp = &F;
  for (int s = 0; s < k; s++) {
    parts.updateVel(cic_gather_kick, 0.1, &Fp, 1);
    parts.moveParticles(move_particles_simple, 0.1);
  }
}

static std::vector<part_simple> sorted(PS& parts)
{
  std::vector<part_simple> out;
  parts.getParticles(out);
  std::sort(out.begin(), out.end(),
            [](const part_simple& a, const part_simple& b) { return a.ID < b.ID; });
  return out;
}

int main(int argc, char** argv)
{
  if (argc != 4) {
    std::fprintf(stderr, "usage: restart_demo N NPART DIR\n");
    return 2;
  }
  const int N = std::atoi(argv[1]);
  const long npart = std::atol(argv[2]);
  const std::string base = std::string(argv[3]) + "/run";
  Real boxSize[3] = {1, 1, 1};
  Lattice lat(3, N, 1), lat_part(3, N, 0);
  Field<Real> F(lat, 3), rho_a(lat, 1), rho_b(lat, 1);
  Site x(lat);
  for (x.first(); x.test(); x.next())
    for (int c = 0; c < 3; c++)
      F(x, c) = (Real)(0.02 * std::cos(2 * M_PI * (x.coord((c + 2) % 3) + c) / N));
  F.updateHalo();

  part_simple_info info;
  info.mass = 1.0 / npart;
  info.relativistic = 0;
  part_simple_dataType type;
  PS a, b;
  a.initialize(info, type, &lat_part, boxSize);
  b.initialize(info, type, &lat_part, boxSize);
  part_simple p;
  for (long i = 0; i < npart; i++) {
    p.ID = i;
    for (int d = 0; d < 3; d++) p.pos[d] = (Real)uniform();
    for (int d = 0; d < 3; d++) p.vel[d] = (Real)(0.05 * (uniform() - 0.5));
    a.addParticle_global(p);
  }
  steps(a, F, 2);
  a.saveHDF5(base, 1);
  b.loadHDF5(base, 1);
  if (b.numParticles() != a.numParticles()) {
    std::printf("count %ld != %ld\n", b.numParticles(), a.numParticles());
    return 1;
  }
  steps(a, F, 2);
  steps(b, F, 2);
  const std::vector<part_simple> pa = sorted(a), pb = sorted(b);
  for (size_t i = 0; i < pa.size(); i++) {
    bool same = pa[i].ID == pb[i].ID;
    for (int d = 0; d < 3; d++)
      same = same && pa[i].pos[d] == pb[i].pos[d] && pa[i].vel[d] == pb[i].vel[d];
    if (!same) {
      std::printf("particle %zu differs\n", i);
      return 1;
    }
  }
  scalarProjectionCIC_project(&a, &rho_a);
  scalarProjectionCIC_comm(&rho_a);
  scalarProjectionCIC_project(&b, &rho_b);
  scalarProjectionCIC_comm(&rho_b);
  for (x.first(); x.test(); x.next())
    if (rho_a(x) != rho_b(x)) {
      std::printf("density differs at %ld\n", x.index());
      return 1;
    }
  std::printf("ok %ld particles\n", a.numParticles());
  return 0;
}
