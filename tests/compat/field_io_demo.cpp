// Field::write / read / saveHDF5 / loadHDF5 of include/latfield2_b200.hpp on
// the host (no GPU call): a 3-component Field<Real> written the way a
// reference program writes it, read back into a second field, and written
// again.  Usage: field_io_demo <dir>; writes <dir>/field.bin (Field::write)
// and <dir>/outBIN (saveHDF5 without HDF5), prints "ok" when the fields read
// back equal the originals, halos included.
#include <cstdio>
#include <string>

#include "latfield2_b200.hpp"

using namespace LATfield2;

int main(int argc, char** argv)
{
  if (argc != 2) {
    std::fprintf(stderr, "usage: %s dir\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const int n[3] = {6, 5, 4};
  Lattice lat(3, n, 1);
  Field<Real> B(lat, 3), C(lat, 3), D(lat, 3);
  Site x(lat);
  for (x.first(); x.test(); x.next())
    for (int c = 0; c < 3; c++)
      B(x, c) = (Real)(x.coord(0) + 10 * x.coord(1) + 100 * x.coord(2)) + (Real)c / 4;
  B.updateHalo();
  B.write(dir + "/field.bin");
  C.read(dir + "/field.bin");
  C.saveHDF5(dir + "/out");
  D.loadHDF5(dir + "/out");
  for (long i = 0; i < lat.sitesGross(); i++)
    for (int c = 0; c < 3; c++)
      if (C(i, c) != B(i, c) || D(i, c) != B(i, c)) {
        std::printf("mismatch at %ld/%d\n", i, c);
        return 1;
      }
  std::printf("ok\n");
  return 0;
}
