// A Poisson solve written against LATfield2's Fourier interface
// (Lattice::initializeRealFFT, rKSite, Field<Imag>, PlanFFT<Imag>), built
// against include/latfield2_b200.hpp (the GPU path) instead of LATfield2.hpp.
//
//   poisson_demo N OUT [KHALO]
//
// rho is a smooth periodic density (two Gaussian bumps on a constant); phi_k
// is rho_k divided by the eigenvalue of the 7-point lattice Laplacian, the
// zero mode removed; after the backward transform (not normalised) the
// 7-point Laplacian of phi / N^3 must give back rho minus its mean.  Writes
// rho, rho_k (re, im pairs in the Fourier lattice's site order) and phi to
// OUT and prints the largest error of that check relative to max |rho - mean|.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "latfield2_b200.hpp"

using namespace LATfield2;

static void put(FILE* fp, const std::vector<double>& v)
{
  const int64_t n = (int64_t)v.size();
  fwrite(&n, sizeof n, 1, fp);
  fwrite(v.data(), sizeof(double), v.size(), fp);
}

int main(int argc, char** argv)
{
  if (argc != 3 && argc != 4) {
    fprintf(stderr, "usage: poisson_demo N OUT [KHALO]\n");
    return 2;
  }
  const int N = atoi(argv[1]);
  const int khalo = argc == 4 ? atoi(argv[3]) : 0;  // halo of the Fourier lattice
  const double res = 1.0 / N;
  parallel.initialize(1, 1);

  Lattice lat(3, N, 1);
  Lattice latK;
  latK.initializeRealFFT(lat, khalo);
  Field<Real> rho(lat, 1), phi(lat, 1);
  Field<Imag> rhoK(latK, 1), phiK(latK, 1);
  PlanFFT<Imag> planRho(&rho, &rhoK);
  PlanFFT<Imag> planPhi(&phi, &phiK);

  Site x(lat);
  double mean = 0.0;
  for (x.first(); x.test(); x.next()) {
    double v = 0.3;
    for (int b = 0; b < 2; b++) {
      double r2 = 0.0;
      for (int d = 0; d < 3; d++) {
        double u = (x.coord(d) + 0.5) * res - (b ? 0.3 : 0.7);
        u -= std::floor(u + 0.5);  // periodic distance
        r2 += u * u;
      }
      v += (b ? 2.0 : 1.0) * std::exp(-r2 / 0.01);
    }
    rho(x) = (Real)v;
    mean += rho(x);
  }
  parallel.sum(mean);
  mean /= (double)lat.sites();

  planRho.execute(FFT_FORWARD);
  rKSite k(latK);
  for (k.first(); k.test(); k.next()) {
    if (k.coord(0) == 0 && k.coord(1) == 0 && k.coord(2) == 0) {
      phiK(k) = 0.0;
      continue;
    }
    const double lam = 2.0 * (std::cos(2 * M_PI * k.coord(0) / N) + std::cos(2 * M_PI * k.coord(1) / N) +
                              std::cos(2 * M_PI * k.coord(2) / N) - 3.0) / (res * res);
    phiK(k) = rhoK(k) / lam;
  }
  planPhi.execute(FFT_BACKWARD);
  phi.updateHalo();

  double err = 0.0, scale = 0.0;
  std::vector<double> vr, vk, vp;
  for (x.first(); x.test(); x.next()) {
    double lap = 0.0;
    for (int d = 0; d < 3; d++) lap += (phi(x + d) - 2.0 * phi(x) + phi(x - d)) / (res * res);
    err = std::fmax(err, std::fabs(lap / lat.sites() - (rho(x) - mean)));
    scale = std::fmax(scale, std::fabs(rho(x) - mean));
    vr.push_back(rho(x));
    vp.push_back(phi(x));
  }
  for (k.first(); k.test(); k.next()) {
    vk.push_back(rhoK(k).real());
    vk.push_back(rhoK(k).imag());
  }
  FILE* fp = fopen(argv[2], "wb");
  if (!fp) return 1;
  put(fp, std::vector<double>{(double)N});
  put(fp, vr);
  put(fp, vk);
  put(fp, vp);
  fclose(fp);
  printf("ok laplacian check %.3e sizeof(Real) %zu\n", err / scale, sizeof(Real));
  return 0;
}
