// User physics on the GPU through include/latfield2_b200.hpp: a kick and a
// drift written as functors with __device__ operator() and the reference's
// callback arguments, passed to updateVel and moveParticles (built with
// nvcc).  The kick is the CIC gather-kick and the drift pos += dtau vel,
// written the way a user of the reference writes callbacks, so the results
// can be checked against the library's own kick and drift.
//
//   device_physics_demo N NPART OUT
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "latfield2_b200.hpp"

using namespace LATfield2;

struct UserKick {
  template <class part, class info_t, class F, class S>
  __device__ Real operator()(double dtau, double, part* p, double* frac, info_t, F** fields, S* sites,
                             int, double* params, double* outputs, int noutputs) const
  {
    const double g = params ? params[0] : 1.0;
    double a[3] = {0, 0, 0};
    for (int k = 0; k < 8; k++) {
      const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
      S s = sites[0];
      if (cx) s = s + 0;
      if (cy) s = s + 1;
      if (cz) s = s + 2;
      const double w = (cx ? frac[0] : 1 - frac[0]) * (cy ? frac[1] : 1 - frac[1]) *
                       (cz ? frac[2] : 1 - frac[2]);
      for (int c = 0; c < 3; c++) a[c] += w * (*fields[0])(s, c);
    }
    double v2 = 0;
    for (int c = 0; c < 3; c++) {
      p->vel[c] += (Real)(g * dtau * a[c]);
      v2 += (double)p->vel[c] * p->vel[c];
    }
    // |v|^2 into every output slot; updateVel reduces slot i with reduce_type[i]
    for (int i = 0; i < noutputs; i++) outputs[i] = v2;
    return (Real)v2;
  }
};

struct UserDrift {
  template <class part, class info_t, class F, class S>
  __device__ void operator()(double dtau, double, part* p, double*, info_t, F**, S*, int, double*,
                             double*, int) const
  {
    for (int l = 0; l < 3; l++) p->pos[l] += (Real)(dtau * p->vel[l]);
  }
};

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static double uniform()
{
  rng_state = rng_state * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(rng_state >> 11) * (1.0 / 9007199254740992.0);
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
    fprintf(stderr, "usage: device_physics_demo N NPART OUT\n");
    return 2;
  }
  const int N = atoi(argv[1]);
  const long npart = atol(argv[2]);
  Real boxSize[3] = {1, 1, 1};
  const double dtau = 0.1;
  Lattice lat(3, N, 1), lat_part(3, N, 0);
  Field<Real> F(lat, 3);
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
  std::vector<double> Fv;
  for (x.first(); x.test(); x.next())
    for (int c = 0; c < 3; c++) {
      F(x, c) = (Real)(0.01 * std::sin(2 * M_PI * (x.coord(c) + 0.5 * c) / N));
      Fv.push_back((double)F(x, c));
    }
  F.updateHalo();
  Field<Real>* Fp = &F;
  double* g = nullptr;  // the coupling, in memory the GPU can read
  cudaMallocManaged(&g, sizeof(double));
  *g = 1.0;
  double out[2];
  int red[2] = {SUM, MAX};
  const double maxv = parts.updateVel(UserKick(), dtau, &Fp, 1, g, out, red, 2);
  parts.moveParticles(UserDrift(), dtau);
  std::vector<part_simple> got;
  parts.getParticles(got);
  std::vector<double> id1, pos1, vel1;
  for (auto& q : got) {
    id1.push_back((double)q.ID);
    for (int d = 0; d < 3; d++) pos1.push_back((double)q.pos[d]), vel1.push_back((double)q.vel[d]);
  }
  cudaFree(g);
  FILE* fp = fopen(argv[3], "wb");
  if (!fp) return 1;
  put(fp, {(double)N, (double)parts.numParticles(), dtau, maxv, out[0], out[1]});
  for (auto* v : {&id0, &pos0, &vel0, &Fv, &id1, &pos1, &vel1}) put(fp, *v);
  fclose(fp);
  printf("ok %ld particles\n", parts.numParticles());
  return 0;
}
