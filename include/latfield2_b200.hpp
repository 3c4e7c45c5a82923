/* latfield2_b200.hpp -- header-only C++ layer with the names and signatures
 * of LATfield2's particle path, over the C ABI of lf2gpu.h.
 *
 * Code written against the reference's particle interface compiles against
 * this header instead of LATfield2.hpp for that path:
 *
 *   Lattice lat(3, N, 1), lat_part(3, N, 0);             LATfield2_Lattice_decl.hpp:17-57
 *   Field<Real> rho(lat, 1), F(lat, 3);                  LATfield2_Field_decl.hpp:75-98
 *   Particles<part_simple, part_simple_info, part_simple_dataType> parts;
 *   parts.initialize(info, type, &lat_part, boxSize);    LATfield2_Particles.hpp:358-428
 *   parts.addParticle_global(p);                         :500-540
 *   projection_init(&rho);                               projections.hpp:31-34
 *   scalarProjectionCIC_project(&parts, &rho);           :75-184
 *   scalarProjectionCIC_comm(&rho);                      :194-300
 *   F(x, c) = ...;  F.updateHalo();                      LATfield2_Field_decl.hpp:889-935
 *   parts.updateVel(cic_gather_kick, dtau, &Fp, 1);      LATfield2_Particles.hpp:752-893
 *   parts.moveParticles(move_particles_simple, dtau);    :1810-2803, move_function.hpp:15-32
 *   latK.initializeRealFFT(lat, 0); rKSite k(latK);      LATfield2_Lattice.hpp:225-258
 *   PlanFFT<Imag> plan(&rho, &rhoK);                      LATfield2_PlanFFT_decl.hpp:83-230
 *   plan.execute(FFT_FORWARD); plan.execute(FFT_BACKWARD); :720-1050
 *
 * Where the data live:
 *   - Particles live on the GPU.  addParticle_global stages them on the host;
 *     they are uploaded before the next GPU operation.
 *   - A Field keeps a host array in the reference layout (halo, components
 *     interleaved, Real) and, once a particle operation has used it, a device
 *     copy in the Particles' context.
 *   - The two sides are brought together at the reference's own
 *     synchronisation points:
 *     - updateHalo() fills the host halo and marks the host values as the
 *       current ones, so the next particle operation uploads them;
 *     - the *_comm functions bring a projection back to the host array.
 *
 * Only the library's kernels run on the GPU: updateVel accepts
 * cic_gather_kick and moveParticles accepts move_particles_simple (matched
 * by function identity).  Any other callback raises std::invalid_argument;
 * the reference runs such callbacks on the host per particle, and this layer
 * has no host path.
 *
 * Errors of the C ABI are raised as std::runtime_error carrying
 * lf2_last_error(); the reference exits or throws in the same places.
 * One GPU, one process: the MPI process grid of the reference is 1 x 1
 * (`parallel` is a one-process stand-in).
 */
#ifndef LATFIELD2_B200_HPP
#define LATFIELD2_B200_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "lf2gpu.h"
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace LATfield2 {

#ifdef SINGLE
typedef float Real;
#else
typedef double Real;
#endif

// LATfield2_Particles.hpp:76-86, projections.hpp:38-39, LATfield2_Field.hpp:16-17
#ifndef GLOBAL_MASS
#define GLOBAL_MASS 0
#define INDIVIDUAL_MASS 1
#define NO_MASS 2
#endif
static int const FROM_PART = INDIVIDUAL_MASS;
static int const FROM_INFO = GLOBAL_MASS;
// reduction types of updateVel / moveParticles outputs (LATfield2_Particles.hpp:81-86)
#ifndef SUM
#define SUM 1
#define MIN 2
#define MAX 4
#define SUM_LOCAL 8
#define MIN_LOCAL 16
#define MAX_LOCAL 32
#endif
static int const symmetric = 1;
static int const unsymmetric = 0;

namespace lf2detail {

inline void check(const lf2_ctx* ctx, lf2_status s, const char* what)
{
  if (s == LF2_OK) return;
  std::string msg = std::string(what) + ": status " + std::to_string(s);
  if (ctx) msg += std::string(": ") + lf2_last_error(ctx);
  throw std::runtime_error(msg);
}

// A particle type with a `mass` member carries individual masses
// (INDIVIDUAL_MASS, LATfield2_Particles.hpp:400-425).
template <class T, class = void>
struct has_mass : std::false_type {};
template <class T>
struct has_mass<T, decltype((void)std::declval<T&>().mass, void())> : std::true_type {};

template <class T>
float mass_of(const T& p, std::true_type)
{
  return (float)p.mass;
}
template <class T>
float mass_of(const T&, std::false_type)
{
  return 0.0f;
}

// A projection's global mass (oset / FROM_INFO) for the duration of one
// deposit, when it differs from the particles' part_info mass.
struct MassScope {
  lf2_ctx* ctx;
  double restore;
  bool set = false;
  MassScope(lf2_ctx* c, double mass, double current) : ctx(c), restore(current)
  {
    if (mass >= 0.0 && mass != current) {
      check(ctx, lf2_set_global_mass(ctx, mass), "lf2_set_global_mass");
      set = true;
    }
  }
  ~MassScope()
  {
    if (set) lf2_set_global_mass(ctx, restore);
  }
  MassScope(const MassScope&) = delete;
  MassScope& operator=(const MassScope&) = delete;
};

}  // namespace lf2detail

// --------------------------------------------------------------------- Imag
// Complex number of two Reals with the reference's operators (Imag.hpp:
// 17-113).  As there, `Real - Imag` keeps the imaginary part's sign
// (Imag.hpp:66) and `Imag / Imag` divides by the squared norm.
class Imag {
 public:
  Imag() : data{0, 0} {}
  Imag(Real a, Real b) : data{a, b} {}
  Imag operator-() const { return Imag(-data[0], -data[1]); }
  Imag operator+(Imag z) const { return Imag(data[0] + z.data[0], data[1] + z.data[1]); }
  Imag operator-(Imag z) const { return Imag(data[0] - z.data[0], data[1] - z.data[1]); }
  Imag operator*(Imag z) const
  {
    return Imag(data[0] * z.data[0] - data[1] * z.data[1], data[0] * z.data[1] + data[1] * z.data[0]);
  }
  Imag operator/(Imag z) const
  {
    const Real q = z.norm();
    return Imag((data[0] * z.data[0] + data[1] * z.data[1]) / q,
                (data[1] * z.data[0] - data[0] * z.data[1]) / q);
  }
  void operator=(Real r) { data[0] = r, data[1] = 0; }
  friend Imag operator+(Imag z, Real a) { return Imag(z.data[0] + a, z.data[1]); }
  friend Imag operator+(Real a, Imag z) { return Imag(z.data[0] + a, z.data[1]); }
  friend Imag operator-(Imag z, Real a) { return Imag(z.data[0] - a, z.data[1]); }
  friend Imag operator-(Real a, Imag z) { return Imag(a - z.data[0], z.data[1]); }
  friend Imag operator*(Imag z, Real a) { return Imag(z.data[0] * a, z.data[1] * a); }
  friend Imag operator*(Real a, Imag z) { return Imag(z.data[0] * a, z.data[1] * a); }
  friend Imag operator/(Imag z, Real a) { return Imag(z.data[0] / a, z.data[1] / a); }
  void operator+=(Imag z) { data[0] += z.data[0], data[1] += z.data[1]; }
  void operator-=(Imag z) { data[0] -= z.data[0], data[1] -= z.data[1]; }
  void operator*=(Imag z) { *this = *this * z; }
  void operator+=(Real a) { data[0] += a; }
  void operator-=(Real a) { data[0] -= a; }
  void operator*=(Real a) { data[0] *= a, data[1] *= a; }
  void operator/=(Real a) { data[0] /= a, data[1] /= a; }
  Real& real() { return data[0]; }
  Real& imag() { return data[1]; }
  Real real() const { return data[0]; }
  Real imag() const { return data[1]; }
  Real norm() const { return data[0] * data[0] + data[1] * data[1]; }
  Imag conj() const { return Imag(data[0], -data[1]); }
  Real phase() const
  {
    return std::acos(data[0] / std::sqrt(norm())) * (data[1] < 0 ? -1 : 1);
  }
  friend Imag expi(Real x) { return Imag(std::cos(x), std::sin(x)); }
  friend std::ostream& operator<<(std::ostream& os, const Imag& z)
  {
    return os << z.data[0] << " + i" << z.data[1];
  }

 private:
  Real data[2];
};

// ----------------------------------------------------------------- parallel
// The reference's process grid (LATfield2_parallel2d_decl.hpp) reduced to one
// process: the whole lattice is local, reductions over processes are the
// identity.  initialize(n, m) accepts only a 1 x 1 grid.
class Parallel2d {
 public:
  void initialize(int proc0, int proc1)
  {
    if (proc0 * proc1 != 1)
      throw std::invalid_argument("parallel.initialize: one GPU runs a 1 x 1 process grid");
  }
  bool isRoot() const { return true; }
  int rank() const { return 0; }
  int size() const { return 1; }
  int root() const { return 0; }
  void barrier() const {}
  template <class T>
  void sum(T&) const {}
  template <class T>
  void max(T&) const {}
  template <class T>
  void min(T&) const {}
};
inline Parallel2d parallel;  // C++17 inline variable: one object per program

// ------------------------------------------------------------------ Lattice
// 3-D periodic lattice of size[0] x size[1] x size[2] sites with a halo of
// `halo` sites (LATfield2_Lattice_decl.hpp:17-135).  One process: the local
// sublattice is the whole lattice.
class Lattice {
 public:
  Lattice() {}
  Lattice(int dim, const int* size, int halo) { initialize(dim, size, halo); }
  Lattice(int dim, const int size, int halo) { initialize(dim, size, halo); }
  void initialize(int dim, const int* size, int halo)
  {
    if (dim != 3) throw std::invalid_argument("Lattice: only 3 dimensions are provided");
    for (int d = 0; d < 3; d++) size_[d] = size[d];
    halo_ = halo;
  }
  void initialize(int dim, const int size, int halo)
  {
    const int s[3] = {size, size, size};
    initialize(dim, s, halo);
  }
  // The lattice of the Fourier transform of a real field on the cubic
  // lattice `lat_real`: sizes (n/2+1, n, n) (Lattice::initializeRealFFT,
  // LATfield2_Lattice.hpp:225-258).
  void initializeRealFFT(Lattice& lat_real, int halo)
  {
    const int n = lat_real.size(0);
    if (lat_real.size(1) != n || lat_real.size(2) != n)
      throw std::invalid_argument("Lattice::initializeRealFFT: the real lattice is not cubic");
    const int s[3] = {n / 2 + 1, n, n};
    initialize(3, s, halo);
  }
  int dim() { return 3; }
  int halo() { return halo_; }
  int* size() { return size_; }
  int size(int direction) { return size_[direction]; }
  int* sizeLocal() { return size_; }
  int sizeLocal(int direction) { return size_[direction]; }
  long sites() { return (long)size_[0] * size_[1] * size_[2]; }
  long sitesGross() { return (long)gross(0) * gross(1) * gross(2); }
  long sitesLocal() { return sites(); }
  long sitesLocalGross() { return sitesGross(); }
  // index step of one site in a direction of the halo'd lattice
  long jump(int direction) { return direction == 0 ? 1 : direction == 1 ? gross(0) : (long)gross(0) * gross(1); }
  int gross(int d) const { return size_[d] + 2 * halo_; }

 private:
  int size_[3] = {0, 0, 0};
  int halo_ = 0;
};

// --------------------------------------------------------------------- Site
// A site of a lattice, walked with first()/test()/next() over the local
// sites (LATfield2_Site_decl.hpp:19-195); index() addresses the halo'd
// arrays of the fields on that lattice.
class Site {
 public:
  Site() {}
  explicit Site(Lattice& lattice) { initialize(lattice); }
  Site(Lattice& lattice, long index) { initialize(lattice, index); }
  void initialize(Lattice& lattice) { lat_ = &lattice; first(); }
  void initialize(Lattice& lattice, long index)
  {
    lat_ = &lattice;
    setIndex(index);
  }
  void first()
  {
    c_[0] = c_[1] = c_[2] = 0;
    reindex();
  }
  bool test() { return c_[2] < lat_->size(2); }
  void next()
  {
    if (++c_[0] < lat_->size(0)) {
      index_ += 1;
      return;
    }
    c_[0] = 0;
    if (++c_[1] >= lat_->size(1)) {
      c_[1] = 0;
      ++c_[2];
    }
    reindex();
  }
  int coord(int direction) const { return c_[direction]; }
  long index() const { return index_; }
  void setIndex(long index)
  {
    index_ = index;
    long r = index;
    for (int d = 0; d < 3; d++) {
      c_[d] = (int)(r % lat_->gross(d)) - lat_->halo();
      r /= lat_->gross(d);
    }
  }
  bool setCoord(int x, int y, int z)
  {
    c_[0] = x, c_[1] = y, c_[2] = z;
    reindex();
    return true;
  }
  // neighbour in +direction / -direction (may be a halo site)
  Site operator+(int direction) const
  {
    Site s(*this);
    s.c_[direction] += 1;
    s.index_ += lat_->jump(direction);
    return s;
  }
  Site operator-(int direction) const
  {
    Site s(*this);
    s.c_[direction] -= 1;
    s.index_ -= lat_->jump(direction);
    return s;
  }
  Lattice& lattice() const { return *lat_; }

 protected:
  void reindex()
  {
    const int h = lat_->halo();
    index_ = (long)(c_[0] + h) + (long)lat_->gross(0) * ((c_[1] + h) + (long)lat_->gross(1) * (c_[2] + h));
  }
  Lattice* lat_ = nullptr;
  long index_ = 0;
  int c_[3] = {0, 0, 0};
};

// ------------------------------------------------------------------- rKSite
// A site of the Fourier lattice of initializeRealFFT.  Its storage dims are
// (k_x, k_z, k_y); coord(1) returns k_y and coord(2) returns k_z, and
// operator+/- and setCoord take directions in the same (x, y, z) sense
// (LATfield2_Site.hpp:319-416).
class rKSite : public Site {
 public:
  rKSite() {}
  explicit rKSite(Lattice& lattice) : Site(lattice) {}
  rKSite(Lattice& lattice, long index) : Site(lattice, index) {}
  int coord(int direction) const { return Site::coord(storage_dim(direction)); }
  rKSite operator+(int direction) const { return rKSite(Site::operator+(storage_dim(direction))); }
  rKSite operator-(int direction) const { return rKSite(Site::operator-(storage_dim(direction))); }
  bool setCoord(int x, int y, int z) { return Site::setCoord(x, z, y); }

 private:
  explicit rKSite(const Site& s) : Site(s) {}
  static int storage_dim(int direction) { return direction == 0 ? 0 : 3 - direction; }
};

// -------------------------------------------------------------------- Field
// A field of Real on a lattice: `components` values per site, or a rows x
// cols matrix (symmetric: rows*(rows+1)/2 values, order 00,01,02,11,12,22
// for 3x3; LATfield2_Field_decl.hpp:75-208, :772-788).  The host array is
// laid out like the reference's: halo'd sites, components interleaved.
template <class FieldType>
class Field {
  static_assert(std::is_same<FieldType, Real>::value || std::is_same<FieldType, Imag>::value,
                "the GPU path provides Field<Real> and Field<Imag> (Fourier space)");

 public:
  Field() {}
  Field(Lattice& lattice, int components = 1) { initialize(lattice, components); }
  Field(Lattice& lattice, int rows, int cols, int symmetry = unsymmetric)
  {
    initialize(lattice, rows, cols, symmetry);
  }
  ~Field() { release_device(); }
  Field(const Field&) = delete;
  Field& operator=(const Field&) = delete;

  void initialize(Lattice& lattice, int components = 1)
  {
    lat_ = &lattice;
    rows_ = components, cols_ = 1, symmetry_ = unsymmetric;
    components_ = components;
    alloc();
  }
  void initialize(Lattice& lattice, int rows, int cols, int symmetry = unsymmetric)
  {
    lat_ = &lattice;
    rows_ = rows, cols_ = cols, symmetry_ = symmetry;
    components_ = symmetry == symmetric ? rows * (rows + 1) / 2 : rows * cols;
    alloc();
  }
  void alloc()
  {
    if ((long)data_.size() != lat_->sitesGross() * components_)
      data_.assign((size_t)(lat_->sitesGross() * components_), FieldType());
  }
  void dealloc()
  {
    release_device();
    std::vector<FieldType>().swap(data_);
  }

  FieldType& operator()(long index) { return data_[(size_t)(index * components_)]; }
  FieldType& operator()(long index, int component)
  {
    return data_[(size_t)(index * components_ + component)];
  }
  FieldType& operator()(long index, int i, int j) { return (*this)(index, matrix_index(i, j)); }
  FieldType& operator()(const Site& site) { return (*this)(site.index()); }
  FieldType& operator()(const Site& site, int component) { return (*this)(site.index(), component); }
  FieldType& operator()(const Site& site, int i, int j) { return (*this)(site.index(), i, j); }

  // Periodic halo on the host; the host values become the current ones
  // (uploaded before the next particle operation that reads this field).
  void updateHalo()
  {
    if (device_newer_) pull();
    const int h = lat_->halo();
    if (h > 0) fill_halo();
    device_newer_ = false;
    host_newer_ = true;
  }

  // Field::write (LATfield2_Field_decl.hpp:1179-1239): the lattice without
  // halo, x fastest, components interleaved, raw FieldType values, no header
  // (the file the reference's ranks write together; here one process holds
  // the whole lattice).
  void write(const std::string& filename)
  {
    if (device_newer_) pull();
    std::FILE* f = std::fopen(filename.c_str(), "wb");
    if (!f) throw std::runtime_error("Field::write: cannot open " + filename);
    bool ok = true;
    for (int z = 0; z < lat_->size(2) && ok; z++)
      for (int y = 0; y < lat_->size(1) && ok; y++)
        ok = std::fwrite(row(y, z), sizeof(FieldType), row_values(), f) == row_values();
    if (std::fclose(f) != 0 || !ok) throw std::runtime_error("Field::write: cannot write " + filename);
  }
  // Field::read (LATfield2_Field_decl.hpp:1286-1345): a file of write's
  // layout, then updateHalo.
  void read(const std::string& filename)
  {
    std::FILE* f = std::fopen(filename.c_str(), "rb");
    if (!f) throw std::runtime_error("Field::read: cannot open " + filename);
    bool ok = true;
    for (int z = 0; z < lat_->size(2) && ok; z++)
      for (int y = 0; y < lat_->size(1) && ok; y++)
        ok = std::fread(row(y, z), sizeof(FieldType), row_values(), f) == row_values();
    std::fclose(f);
    if (!ok) throw std::runtime_error("Field::read: short file " + filename);
    device_newer_ = false;
    host_newer_ = true;
    updateHalo();
  }
  // Field::saveHDF5 / loadHDF5 of a build without HDF5
  // (LATfield2_Field_decl.hpp:1532-1555): the binary file filename + "BIN".
  void saveHDF5(const std::string& filename, const std::string& = "data") { write(filename + "BIN"); }
  void loadHDF5(const std::string& filename, const std::string& = "data") { read(filename + "BIN"); }

  int components() const { return components_; }
  int rows() const { return rows_; }
  int cols() const { return cols_; }
  int symmetry() const { return symmetry_; }
  Lattice& lattice() { return *lat_; }
  FieldType* data() { return data_.data(); }

  // ---- GPU side (not in the reference) ----
  // The field's device copy in the given context, with the host values
  // uploaded first when they are the current ones.
  // The field holds a reference to the context, so that the context outlives
  // the field's device copy whatever the order of destruction.
  lf2_field lf2_handle(const std::shared_ptr<lf2_ctx>& owner, bool upload = true)
  {
    static_assert(std::is_same<FieldType, Real>::value, "device copies exist for Field<Real>");
    lf2_ctx* ctx = owner.get();
    if (ctx_ != ctx) {
      if (ctx_ && device_newer_) pull();
      release_device();
      lf2detail::check(ctx, lf2_field_create(ctx, components_, &dev_), "lf2_field_create");
      owner_ = owner;
      ctx_ = ctx;
      host_newer_ = true;
    }
    if (upload && host_newer_) {
      lf2detail::check(ctx_, lf2_field_import(ctx_, dev_, data_.data(), lat_->halo(), sizeof(FieldType),
                                              LF2_PTR_HOST),
                       "lf2_field_import");
      host_newer_ = false;
    }
    return dev_;
  }
  // a particle operation has written the device copy
  void mark_device_written()
  {
    device_newer_ = true;
    host_newer_ = false;
  }
  // the context of the field's device copy (empty before the first GPU use)
  const std::shared_ptr<lf2_ctx>& lf2_context_owner() const { return owner_; }
  // device copy -> host array (halo filled periodically)
  void pull()
  {
    if (!ctx_) return;
    lf2detail::check(ctx_, lf2_field_export(ctx_, dev_, data_.data(), lat_->halo(), sizeof(FieldType), 1,
                                            LF2_PTR_HOST),
                     "lf2_field_export");
    device_newer_ = false;
  }

 private:
  int matrix_index(int i, int j) const
  {
    if (symmetry_ == symmetric) {
      const int a = i < j ? i : j, b = i < j ? j : i;
      return (b - a) + a * rows_ - a * (a - 1) / 2;
    }
    return j * rows_ + i;
  }
  // first value of the x-row (y, z) of the interior, and the values in it
  FieldType* row(int y, int z)
  {
    const int h = lat_->halo();
    const long i = h + (long)lat_->gross(0) * ((y + h) + (long)lat_->gross(1) * (z + h));
    return &data_[(size_t)(i * components_)];
  }
  size_t row_values() const { return (size_t)lat_->size(0) * components_; }
  void fill_halo()
  {
    const int h = lat_->halo();
    const int g[3] = {lat_->gross(0), lat_->gross(1), lat_->gross(2)};
    const int n[3] = {lat_->size(0), lat_->size(1), lat_->size(2)};
    for (int z = 0; z < g[2]; z++)
      for (int y = 0; y < g[1]; y++)
        for (int x = 0; x < g[0]; x++) {
          if (x >= h && x < h + n[0] && y >= h && y < h + n[1] && z >= h && z < h + n[2]) continue;
          const int sx = ((x - h) % n[0] + n[0]) % n[0] + h;
          const int sy = ((y - h) % n[1] + n[1]) % n[1] + h;
          const int sz = ((z - h) % n[2] + n[2]) % n[2] + h;
          const long dst = x + (long)g[0] * (y + (long)g[1] * z);
          const long src = sx + (long)g[0] * (sy + (long)g[1] * sz);
          for (int c = 0; c < components_; c++)
            data_[(size_t)(dst * components_ + c)] = data_[(size_t)(src * components_ + c)];
        }
  }
  void release_device()
  {
    if (ctx_ && dev_) lf2_field_destroy(ctx_, dev_);
    ctx_ = nullptr;
    dev_ = nullptr;
    owner_.reset();
  }

  Lattice* lat_ = nullptr;
  int components_ = 0, rows_ = 0, cols_ = 1, symmetry_ = unsymmetric;
  std::vector<FieldType> data_;
  std::shared_ptr<lf2_ctx> owner_;
  lf2_ctx* ctx_ = nullptr;
  lf2_field dev_ = nullptr;
  bool host_newer_ = true;
  bool device_newer_ = false;
};

// ------------------------------------------------------------------ PlanFFT
// LATfield2_PlanFFT.hpp:14-17
const int FFT_FORWARD = 1;
const int FFT_BACKWARD = -1;
const int FFT_IN_PLACE = 16;
const int FFT_OUT_OF_PLACE = -16;

// Real-to-complex transforms between a Field<Real> on a cubic lattice and a
// Field<Imag> on the lattice of initializeRealFFT (LATfield2_PlanFFT_decl.hpp:
// 83-230, :720-1050), with the reference's storage order and normalisation
// (neither direction normalised).  execute() runs on the GPU (lf2_fft_forward,
// lf2_fft_backward) and leaves its result in the output field's host array, as
// the reference does.  The plan uses the real field's GPU context when it
// already has one (a field used by particle operations), otherwise a context
// of its own.  FFT_IN_PLACE (one array shared by both fields in the reference)
// gives the same values; the two fields keep separate arrays here.
template <class compType>
class PlanFFT {
  static_assert(std::is_same<compType, Imag>::value, "PlanFFT<Imag> is provided");

 public:
  PlanFFT() {}
  PlanFFT(Field<Real>* rfield, Field<Imag>* kfield, const int mem_type = FFT_OUT_OF_PLACE)
  {
    initialize(rfield, kfield, mem_type);
  }
  ~PlanFFT() { release(); }
  PlanFFT(const PlanFFT&) = delete;
  PlanFFT& operator=(const PlanFFT&) = delete;

  void initialize(Field<Real>* rfield, Field<Imag>* kfield, const int mem_type = FFT_OUT_OF_PLACE)
  {
    (void)mem_type;
    Lattice& lr = rfield->lattice();
    Lattice& lk = kfield->lattice();
    const int n = lr.size(0);
    if (lr.size(1) != n || lr.size(2) != n)
      throw std::invalid_argument("PlanFFT::initialize: the real lattice is not cubic");
    if (lk.size(0) != n / 2 + 1 || lk.size(1) != n || lk.size(2) != n)
      throw std::invalid_argument("PlanFFT::initialize: the Fourier lattice is not initializeRealFFT's");
    if (rfield->components() != kfield->components())
      throw std::invalid_argument("PlanFFT::initialize: the fields have different numbers of components");
    release();
    r_ = rfield;
    k_ = kfield;
  }

  void execute(int fft_type)
  {
    if (!r_) throw std::logic_error("PlanFFT::execute: plan not initialised");
    if (fft_type != FFT_FORWARD && fft_type != FFT_BACKWARD)
      throw std::invalid_argument("PlanFFT::execute: FFT_FORWARD or FFT_BACKWARD");
    bind();
    lf2_ctx* ctx = owner_.get();
    lf2_field rd = r_->lf2_handle(owner_, fft_type == FFT_FORWARD);
    if (fft_type == FFT_FORWARD) {
      lf2detail::check(ctx, lf2_fft_forward(ctx, rd, kdev_), "lf2_fft_forward");
      k_to_host();
    } else {
      k_to_device();
      lf2detail::check(ctx, lf2_fft_backward(ctx, kdev_, rd), "lf2_fft_backward");
      r_->mark_device_written();
      r_->pull();
    }
  }

 private:
  void bind()
  {
    if (!owner_) {
      owner_ = r_->lf2_context_owner();
      if (!owner_) {
        const int n = r_->lattice().size(0);
        const int ns[3] = {n, n, n};
        const double box[3] = {1.0, 1.0, 1.0};
        lf2_ctx* c = nullptr;
        lf2detail::check(nullptr, lf2_create(&c, 0, ns, box, LF2_DEPOSIT_FP32, nullptr), "lf2_create");
        owner_.reset(c, [](lf2_ctx* p) { lf2_destroy(p); });
      }
    }
    if (!kdev_)
      lf2detail::check(owner_.get(), lf2_kfield_create(owner_.get(), k_->components(), &kdev_),
                       "lf2_kfield_create");
  }
  // the k-field without halo, in the reference's order, <-> the host array
  // of k_ (which may have a halo)
  void k_to_host()
  {
    lf2_ctx* ctx = owner_.get();
    Lattice& lk = k_->lattice();
    if (lk.halo() == 0) {
      lf2detail::check(ctx, lf2_kfield_export(ctx, kdev_, k_->data(), sizeof(Real), LF2_PTR_HOST),
                       "lf2_kfield_export");
      return;
    }
    std::vector<Imag> tmp((size_t)lk.sites() * k_->components());
    lf2detail::check(ctx, lf2_kfield_export(ctx, kdev_, tmp.data(), sizeof(Real), LF2_PTR_HOST),
                     "lf2_kfield_export");
    copy_halo(tmp, true);
  }
  void k_to_device()
  {
    lf2_ctx* ctx = owner_.get();
    Lattice& lk = k_->lattice();
    if (lk.halo() == 0) {
      lf2detail::check(ctx, lf2_kfield_import(ctx, kdev_, k_->data(), sizeof(Real), LF2_PTR_HOST),
                       "lf2_kfield_import");
      return;
    }
    std::vector<Imag> tmp((size_t)lk.sites() * k_->components());
    copy_halo(tmp, false);
    lf2detail::check(ctx, lf2_kfield_import(ctx, kdev_, tmp.data(), sizeof(Real), LF2_PTR_HOST),
                     "lf2_kfield_import");
  }
  void copy_halo(std::vector<Imag>& flat, bool to_field)
  {
    Lattice& lk = k_->lattice();
    const int comps = k_->components();
    Site s(lk);
    long i = 0;
    for (s.first(); s.test(); s.next(), i++)
      for (int c = 0; c < comps; c++) {
        Imag& f = (*k_)(s, c);
        Imag& t = flat[(size_t)(i * comps + c)];
        if (to_field) f = t;
        else t = f;
      }
  }
  void release()
  {
    if (kdev_ && owner_) lf2_kfield_destroy(owner_.get(), kdev_);
    kdev_ = nullptr;
    owner_.reset();
  }

  Field<Real>* r_ = nullptr;
  Field<Imag>* k_ = nullptr;
  std::shared_ptr<lf2_ctx> owner_;
  lf2_kfield kdev_ = nullptr;
};

// ---------------------------------------------------------- particle types
// LATfield2_particle_simple.hpp:40-82 (the HDF5 datatype structure is empty
// here: no HDF5 on this path).
struct part_simple {
  long ID;
  Real pos[3];
  Real vel[3];
};
inline std::ostream& operator<<(std::ostream& os, const part_simple& p)
{
  os << "ID: " << p.ID << " , Pos: (" << p.pos[0] << "," << p.pos[1] << "," << p.pos[2]
     << ") , Vel: (" << p.vel[0] << "," << p.vel[1] << "," << p.vel[2] << ")";
  return os;
}
struct part_simple_info {
  double mass;
  int relativistic;
  int type_name_size;
  char type_name[64];
};
struct part_simple_dataType {};

// ------------------------------------------------------------ callbacks
// move_particles_simple (move_function.hpp:15-32): pos += dtau * vel.  The
// GPU runs it inside moveParticles; a direct call updates one particle.
template <class part, class part_info>
void move_particles_simple_t(double dtau, double, part* p, double*, part_info, Field<Real>**, Site*, int,
                             double*, double*, int)
{
  for (int l = 0; l < 3; l++) p->pos[l] += dtau * p->vel[l];
}

// The CIC gather-kick: vel_c += dtau * sum over the 8 cell corners of
// w * F_c(corner), w the product of the 1-D CIC weights (frac or 1 - frac),
// F = fields[0] with 3 components, sites[0] the particle's cell in F's
// lattice.  Returns |v|^2 (the quantity updateVel maximises).  The GPU runs
// it inside updateVel; a direct call kicks one particle on the host arrays.
template <class part, class part_info>
Real cic_gather_kick_t(double dtau, double, part* p, double* frac, part_info, Field<Real>** fields,
                       Site* sites, int, double*, double* outputs, int noutputs)
{
  Field<Real>& F = *fields[0];
  Real a[3] = {0, 0, 0};
  for (int k = 0; k < 8; k++) {
    const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
    Site s = sites[0];
    if (cx) s = s + 0;
    if (cy) s = s + 1;
    if (cz) s = s + 2;
    const Real w = (Real)((cx ? frac[0] : 1 - frac[0]) * (cy ? frac[1] : 1 - frac[1]) *
                          (cz ? frac[2] : 1 - frac[2]));
    for (int c = 0; c < 3; c++) a[c] += w * F(s, c);
  }
  Real v2 = 0;
  double v2d = 0.0;
  for (int c = 0; c < 3; c++) {
    p->vel[c] += dtau * a[c];
    v2 += p->vel[c] * p->vel[c];
    v2d += (double)p->vel[c] * (double)p->vel[c];
  }
  // the per-particle outputs updateVel reduces: |v|^2 in every slot, each
  // slot reduced with its own reduce_type
  for (int i = 0; i < noutputs; i++) outputs[i] = v2d;
  return v2;
}

// The same kick in the signature of updateVel's mappingClass overload
// (LATfield2_Particles.hpp:191-200): the mapping object is not used.
template <class part, class part_info, class mappingClass>
Real cic_gather_kick_mapped(double dtau, double res, part* p, double* frac, part_info info,
                            Field<Real>** fields, Site* sites, mappingClass*, int nfield,
                            double* params, double* outputs, int noutputs)
{
  return cic_gather_kick_t<part, part_info>(dtau, res, p, frac, info, fields, sites, nfield, params,
                                            outputs, noutputs);
}

inline void move_particles_simple(double dtau, double res, part_simple* p, double* frac,
                                  part_simple_info info, Field<Real>** fields, Site* sites, int nfield,
                                  double* params, double* outputs, int noutputs)
{
  move_particles_simple_t<part_simple, part_simple_info>(dtau, res, p, frac, info, fields, sites, nfield,
                                                         params, outputs, noutputs);
}

inline Real cic_gather_kick(double dtau, double res, part_simple* p, double* frac, part_simple_info info,
                            Field<Real>** fields, Site* sites, int nfield, double* params,
                            double* outputs, int noutputs)
{
  return cic_gather_kick_t<part_simple, part_simple_info>(dtau, res, p, frac, info, fields, sites, nfield,
                                                          params, outputs, noutputs);
}

namespace lf2detail {
typedef Real (*kick_simple_fn)(double, double, part_simple*, double*, part_simple_info, Field<Real>**,
                               Site*, int, double*, double*, int);
typedef void (*move_simple_fn)(double, double, part_simple*, double*, part_simple_info, Field<Real>**,
                               Site*, int, double*, double*, int);
inline bool is_simple_kick(kick_simple_fn f) { return f == &cic_gather_kick; }
template <class F>
bool is_simple_kick(F)
{
  return false;
}
inline bool is_simple_move(move_simple_fn f) { return f == &move_particles_simple; }
template <class F>
bool is_simple_move(F)
{
  return false;
}
}  // namespace lf2detail

#ifdef __CUDACC__
// ------------------------------------------------------- user physics on the GPU
// updateVel and moveParticles also take a functor whose operator() is a
// __device__ function with the reference's callback arguments
// (LATfield2_Particles.hpp:752-893, :1810-2803):
//   Real operator()(double dtau, double res, part* p, double* frac, part_info info,
//                   F** fields, S* sites, int nfields, double* params,
//                   double* outputs, int noutputs) const      (kick; returns |v|^2)
//   void operator()(... same ...) const                       (move)
// F and S are lf2dev::Field and lf2dev::Site: (*fields[i])(sites[i] + dir, c),
// sites[i] - dir, sites[i].coord(d) work as on the reference's Field and Site
// (periodic; the GPU field, FP32).  The particle is a copy of `part` filled
// from the GPU store (ID, pos in box units, vel, mass for types with one);
// a kick may change vel, a move pos (any distance: the particles are rebinned
// afterwards).  params must be memory the GPU can read (device, managed or
// mapped pinned memory).  Per-particle outputs are reduced with reduce_type
// (SUM, MIN, MAX) into output.  Compile the user's file with nvcc.
namespace lf2dev {
struct Site {
  int x[3];
  int n[3];
  __host__ __device__ Site operator+(int d) const
  {
    Site s = *this;
    s.x[d] = x[d] + 1 == n[d] ? 0 : x[d] + 1;
    return s;
  }
  __host__ __device__ Site operator-(int d) const
  {
    Site s = *this;
    s.x[d] = x[d] == 0 ? n[d] - 1 : x[d] - 1;
    return s;
  }
  __host__ __device__ int coord(int d) const { return x[d]; }
  __host__ __device__ long index() const { return x[0] + (long)n[0] * (x[1] + (long)n[1] * x[2]); }
};
struct Field {
  float* data;
  int comps;
  long nsites;
  __device__ float& operator()(const Site& s, int c = 0) const { return data[c * nsites + s.index()]; }
  __host__ __device__ int components() const { return comps; }
};
constexpr int MAX_FIELDS = 8;
constexpr int MAX_OUTPUTS = 8;

__device__ inline void reduce_out(double* dst, int type, double v)
{
  if (type & (SUM | SUM_LOCAL)) {
    atomicAdd(dst, v);
    return;
  }
  const bool mn = (type & (MIN | MIN_LOCAL)) != 0;
  if (!mn && !(type & (MAX | MAX_LOCAL))) return;
  unsigned long long* a = reinterpret_cast<unsigned long long*>(dst);
  unsigned long long old = *a;
  for (;;) {  // compare-and-swap: every failed attempt means another thread progressed
    const double cur = __longlong_as_double((long long)old);
    if (mn ? !(v < cur) : !(v > cur)) return;
    const unsigned long long got = atomicCAS(a, old, (unsigned long long)__double_as_longlong(v));
    if (got == old) return;
    old = got;
  }
}

template <class T>
__device__ inline void set_mass(T& p, float m, std::true_type)
{
  p.mass = m;
}
template <class T>
__device__ inline void set_mass(T&, float, std::false_type)
{
}

template <class Fn, class part, class part_info, bool MOVE>
__global__ void k_user(Fn fn, int64_t np, int32_t* cell, float* off3, float* vel3, const float* mass,
                       const int64_t* id, part_info info, double dtau, double res, int n0, int n1,
                       int n2, const Field* fields, int nfields, double* params, int noutput,
                       const int* red, double* red_out, unsigned long long* maxv2)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int c = cell[p];
    const int xyz[3] = {c % n0, (c / n0) % n1, c / (n0 * n1)};
    part q{};
    q.ID = (long)id[p];
    double frac[3];
    for (int d = 0; d < 3; d++) {
      frac[d] = (double)off3[3 * p + d];
      q.pos[d] = (Real)(((double)xyz[d] + frac[d]) * res);
      q.vel[d] = (Real)vel3[3 * p + d];
    }
    set_mass(q, mass ? mass[p] : 0.0f, lf2detail::has_mass<part>());
    Site s[MAX_FIELDS];
    Field* fp[MAX_FIELDS];
    for (int f = 0; f < nfields; f++) {
      s[f] = Site{{xyz[0], xyz[1], xyz[2]}, {n0, n1, n2}};
      fp[f] = const_cast<Field*>(&fields[f]);
    }
    double outs[MAX_OUTPUTS];
    for (int i = 0; i < noutput; i++) outs[i] = 0.0;
    if constexpr (MOVE) {
      fn(dtau, res, &q, frac, info, fp, s, nfields, params, outs, noutput);
      // the new position back into cell + in-cell offset
      const int nn[3] = {n0, n1, n2};
      int k[3];
      for (int d = 0; d < 3; d++) {
        const double u = (double)q.pos[d] / res;
        double fl = floor(u);
        float o = (float)(u - fl);
        if (o >= 1.0f) o = 0.0f, fl += 1.0;
        long kk = (long)fl % nn[d];
        k[d] = (int)(kk < 0 ? kk + nn[d] : kk);
        off3[3 * p + d] = o;
      }
      cell[p] = k[0] + n0 * (k[1] + n1 * k[2]);
    } else {
      const double v2 = (double)fn(dtau, res, &q, frac, info, fp, s, nfields, params, outs, noutput);
      atomicMax(maxv2, (unsigned long long)__double_as_longlong(v2 > 0 ? v2 : 0.0));
    }
    for (int d = 0; d < 3; d++) vel3[3 * p + d] = (float)q.vel[d];
    for (int i = 0; i < noutput; i++) reduce_out(&red_out[i], red[i], outs[i]);
  }
}
}  // namespace lf2dev
#endif

// ---------------------------------------------------------------- Particles
// LATfield2_Particles.hpp:131-344 for particles that live on the GPU.
template <class part, class part_info, class part_dataType>
class Particles {
 public:
  typedef Real (*kick_fn)(double, double, part*, double*, part_info, Field<Real>**, Site*, int, double*,
                          double*, int);
  typedef void (*move_fn)(double, double, part*, double*, part_info, Field<Real>**, Site*, int, double*,
                          double*, int);

  Particles() {}
  Particles(const Particles&) = delete;
  Particles& operator=(const Particles&) = delete;

  // The deposit mode is the int64 fixed point (bit-exact and independent of
  // particle order); define LF2_COMPAT_FP32_DEPOSIT for FP32 atomics.
  void initialize(part_info info, part_dataType, Lattice* lat_part, Real boxSize[3], int device = 0)
  {
    info_ = info;
    lat_ = lat_part;
    for (int d = 0; d < 3; d++) box_[d] = boxSize[d];
    res_ = (Real)(boxSize[0] / lat_part->size(0));
#ifdef LF2_COMPAT_FP32_DEPOSIT
    const int mode = LF2_DEPOSIT_FP32;
#else
    const int mode = LF2_DEPOSIT_FIXED64;
#endif
    lf2_ctx* c = nullptr;
    lf2detail::check(nullptr, lf2_create(&c, device, lat_part->size(), box_, mode, nullptr), "lf2_create");
    owner_.reset(c, [](lf2_ctx* p) { lf2_destroy(p); });
    ctx_ = c;
    on_device_ = 0;
  }

  bool addParticle_global(part newPart) { return addParticle_global(newPart, false); }
  bool addParticle_global(part newPart, bool assignID)
  {
    if (assignID) newPart.ID = (long)(on_device_ + ids_.size());
    for (int d = 0; d < 3; d++) {
      Real x = newPart.pos[d];
      if (x < 0 || x >= box_[d]) return false;  // outside the box (the reference drops it too)
      pos_.push_back((double)x);
      vel_.push_back((double)newPart.vel[d]);
    }
    ids_.push_back((int64_t)newPart.ID);
    mass_.push_back(lf2detail::mass_of(newPart, lf2detail::has_mass<part>()));
    return true;
  }

  long numParticles()
  {
    sync();
    int64_t n = 0;
    lf2detail::check(ctx_, lf2_particles_count(ctx_, &n), "lf2_particles_count");
    return (long)n;
  }

  // updateVel with the CIC gather-kick: fields[0] is the 3-component force.
  // Returns sqrt(max |v|^2) like the reference.  The kick reports |v|^2 as
  // each of its per-particle outputs; output[i] receives its SUM, MIN or MAX
  // over the particles (FP64 on the GPU) as reduce_type[i] says.  With no
  // particles every output keeps the reduction's starting value (0,
  // 9223372036854775807, -9223372036854775807), as in the reference.
  Real updateVel(kick_fn updateVel_funct, double dtau, Field<Real>** fields = NULL, int nfields = 0,
                 double* params = NULL, double* output = NULL, int* reduce_type = NULL, int noutput = 0)
  {
    (void)params;
    if (!(updateVel_funct == &cic_gather_kick_t<part, part_info> ||
          lf2detail::is_simple_kick(updateVel_funct)))
      throw std::invalid_argument("updateVel: only cic_gather_kick runs on the GPU");
    return gpu_kick(dtau, fields, nfields, output, reduce_type, noutput);
  }

  // The mappingClass overload (LATfield2_Particles.hpp:191-200, :609-750):
  // the callback takes the mapping object after the sites.
  template <typename mappingClass>
  Real updateVel(Real (*updateVel_funct)(double, double, part*, double*, part_info, Field<Real>**, Site*,
                                         mappingClass*, int, double*, double*, int),
                 double dtau, Field<Real>** fields = NULL, int nfields = 0, mappingClass* mc = NULL,
                 double* params = NULL, double* output = NULL, int* reduce_type = NULL, int noutput = 0)
  {
    (void)mc, (void)params;
    if (updateVel_funct != &cic_gather_kick_mapped<part, part_info, mappingClass>)
      throw std::invalid_argument("updateVel: only cic_gather_kick_mapped runs on the GPU");
    return gpu_kick(dtau, fields, nfields, output, reduce_type, noutput);
  }

  // The global mass a projection deposits with, after checking oset and
  // flag_where (projections.hpp:115-126, :458-459, :746-747) against what
  // the GPU store holds: positions, velocities (`vel`) and the mass member
  // of particle types that have one.  oset NULL: the particle type's own
  // mass.  FROM_INFO: the double at byte oset[0] of part_info, for particles
  // without individual masses.  FROM_PART: oset[0] must be the mass member.
  // oset[1] (momentum and stress) must be `vel`.  Returns a negative value
  // for individual masses.
  double projection_mass(const size_t* oset, int flag_where, bool reads_vel, const char* what)
  {
    const bool individual = lf2detail::has_mass<part>::value;
    if (!oset) return individual ? -1.0 : (double)info_.mass;
    if (reads_vel && oset[1] != offsetof(part, vel))
      throw std::invalid_argument(std::string(what) +
                                  ": oset[1] must be the vel member: the GPU store holds only vel");
    if (flag_where == FROM_INFO) {
      if (individual)
        throw std::invalid_argument(std::string(what) +
                                    ": FROM_INFO for particles with individual masses is not provided");
      return *reinterpret_cast<const double*>(reinterpret_cast<const char*>(&info_) + oset[0]);
    }
    if (flag_where == FROM_PART) {
      if (!individual || oset[0] != mass_offset())
        throw std::invalid_argument(std::string(what) +
                                    ": FROM_PART must name the particle type's mass member");
      return -1.0;
    }
    throw std::invalid_argument(std::string(what) + ": flag_where is FROM_INFO or FROM_PART");
  }
  // the global mass the GPU store was loaded with
  double global_mass() const { return gmass_dev_; }

  // LATfield2_Particles.hpp:400-425: how the projections find the mass.
  int mass_type() const { return lf2detail::has_mass<part>::value ? INDIVIDUAL_MASS : GLOBAL_MASS; }
  size_t mass_offset() const { return mass_offset_of(lf2detail::has_mass<part>()); }

#ifdef __CUDACC__
  // user physics on the GPU (a functor with a __device__ operator(); see
  // lf2dev above)
  template <class Kick, typename std::enable_if<!std::is_convertible<Kick, kick_fn>::value, int>::type = 0>
  Real updateVel(Kick kick, double dtau, Field<Real>** fields = NULL, int nfields = 0,
                 double* params = NULL, double* output = NULL, int* reduce_type = NULL, int noutput = 0)
  {
    return (Real)run_user<Kick, false>(kick, dtau, fields, nfields, params, output, reduce_type,
                                       noutput);
  }
  template <class Move, typename std::enable_if<!std::is_convertible<Move, move_fn>::value, int>::type = 0>
  void moveParticles(Move move, double dtau, Field<Real>** fields = NULL, int nfields = 0,
                     double* params = NULL, double* output = NULL, int* reduce_type = NULL,
                     int noutput = 0)
  {
    run_user<Move, true>(move, dtau, fields, nfields, params, output, reduce_type, noutput);
  }

  template <class Fn, bool MOVE>
  double run_user(Fn fn, double dtau, Field<Real>** fields, int nfields, double* params,
                  double* output, int* reduce_type, int noutput)
  {
    if (nfields < 0 || nfields > lf2dev::MAX_FIELDS || noutput < 0 || noutput > lf2dev::MAX_OUTPUTS)
      throw std::invalid_argument("user physics: at most 8 fields and 8 outputs");
    if (noutput > 0 && (!output || !reduce_type))
      throw std::invalid_argument("user physics: outputs need output and reduce_type arrays");
    for (int f = 0; f < nfields; f++) check_field(fields[f], "user physics");
    sync();
    const int64_t np = numParticles();
    const bool hm = lf2detail::has_mass<part>::value;
    std::vector<lf2dev::Field> fv((size_t)nfields);
    for (int f = 0; f < nfields; f++) {
      float* data = nullptr;
      lf2detail::check(ctx_, lf2_field_device_ptr(ctx_, fields[f]->lf2_handle(owner_), &data),
                       "lf2_field_device_ptr");
      fv[(size_t)f] = lf2dev::Field{data, fields[f]->components(),
                                    (long)lat_->size(0) * lat_->size(1) * lat_->size(2)};
    }
    std::vector<double> red0((size_t)noutput);
    for (int i = 0; i < noutput; i++)
      red0[(size_t)i] = (reduce_type[i] & (MIN | MIN_LOCAL))   ? 9223372036854775807.0
                        : (reduce_type[i] & (MAX | MAX_LOCAL)) ? -9223372036854775807.0
                                                               : 0.0;
    // scratch for the particles in storage order and the call's arguments
    const size_t n = (size_t)(np > 0 ? np : 1);
    const size_t bytes = n * (4 + 12 + 12 + 8 + (hm ? 4 : 0)) + sizeof(lf2dev::Field) * 8 +
                         (sizeof(int) + sizeof(double)) * 8 + 8 + 256 * 8;
    char* buf = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) throw std::runtime_error("user physics: cudaMalloc");
    std::unique_ptr<char, void (*)(char*)> guard(buf, [](char* q) { cudaFree(q); });
    char* at = buf;
    auto take = [&](size_t b) {
      char* r = at;
      at += (b + 255) & ~(size_t)255;
      return r;
    };
    int32_t* d_cell = (int32_t*)take(n * 4);
    float* d_off = (float*)take(n * 12);
    float* d_vel = (float*)take(n * 12);
    int64_t* d_id = (int64_t*)take(n * 8);
    float* d_mass = hm ? (float*)take(n * 4) : nullptr;
    lf2dev::Field* d_f = (lf2dev::Field*)take(sizeof(lf2dev::Field) * 8);
    int* d_red = (int*)take(sizeof(int) * 8);
    double* d_out = (double*)take(sizeof(double) * 8);
    unsigned long long* d_max = (unsigned long long*)take(8);
    if (np > 0) {
      lf2detail::check(ctx_, lf2_particles_get(ctx_, d_cell, d_off, d_vel, d_mass, d_id, LF2_PTR_DEVICE),
                       "lf2_particles_get");
      lf2detail::check(ctx_, lf2_synchronize(ctx_), "lf2_synchronize");
      bool ok = true;
      if (nfields) ok &= cudaMemcpy(d_f, fv.data(), sizeof(lf2dev::Field) * nfields, cudaMemcpyHostToDevice) == cudaSuccess;
      if (noutput) {
        ok &= cudaMemcpy(d_red, reduce_type, sizeof(int) * noutput, cudaMemcpyHostToDevice) == cudaSuccess;
        ok &= cudaMemcpy(d_out, red0.data(), sizeof(double) * noutput, cudaMemcpyHostToDevice) == cudaSuccess;
      }
      ok &= cudaMemset(d_max, 0, 8) == cudaSuccess;
      if (!ok) throw std::runtime_error("user physics: copies to the GPU failed");
      const int grid = (int)std::min<int64_t>((np + 255) / 256, 148 * 16);
      lf2dev::k_user<Fn, part, part_info, MOVE><<<grid, 256>>>(
          fn, np, d_cell, d_off, d_vel, d_mass, d_id, info_, dtau, (double)res_, lat_->size(0),
          lat_->size(1), lat_->size(2), d_f, nfields, params, noutput, d_red, d_out, d_max);
      if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        throw std::runtime_error("user physics: the kernel failed");
      lf2detail::check(ctx_, lf2_particles_set(ctx_, np, d_cell, d_off, d_vel, d_mass, gmass_dev_, d_id,
                                               LF2_PTR_DEVICE),
                       "lf2_particles_set");
    }
    unsigned long long mx = 0;
    if (noutput && np > 0) cudaMemcpy(output, d_out, sizeof(double) * noutput, cudaMemcpyDeviceToHost);
    else
      for (int i = 0; i < noutput; i++) output[i] = red0[(size_t)i];
    if (np > 0) cudaMemcpy(&mx, d_max, 8, cudaMemcpyDeviceToHost);
    double mx2 = 0.0;
    std::memcpy(&mx2, &mx, sizeof mx2);
    return std::sqrt(mx2);
  }
#endif

  // The part of updateVel the GPU does: the CIC kick, then the output
  // reductions.
  Real gpu_kick(double dtau, Field<Real>** fields, int nfields, double* output, int* reduce_type,
                int noutput)
  {
    if (nfields < 1 || !fields || fields[0]->components() != 3)
      throw std::invalid_argument("updateVel: cic_gather_kick takes one 3-component field");
    if (noutput > 0 && (!output || !reduce_type))
      throw std::invalid_argument("updateVel: outputs need output and reduce_type arrays");
    check_field(fields[0], "updateVel");
    sync();
    double maxv = 0.0;
    lf2_field F = fields[0]->lf2_handle(owner_);
    lf2detail::check(ctx_, lf2_gather_kick(ctx_, F, dtau, &maxv), "lf2_gather_kick");
    if (noutput > 0) {
      double s = 0.0, mn = 0.0, mx = 0.0;
      lf2detail::check(ctx_, lf2_velocity_reductions(ctx_, &s, &mn, &mx), "lf2_velocity_reductions");
      const bool any = numParticles() > 0;
      for (int i = 0; i < noutput; i++) {
        if (reduce_type[i] & (SUM | SUM_LOCAL))
          output[i] = any ? s : 0.0;
        else if (reduce_type[i] & (MIN | MIN_LOCAL))
          output[i] = any ? std::min(mn, 9223372036854775807.0) : 9223372036854775807.0;
        else if (reduce_type[i] & (MAX | MAX_LOCAL))
          output[i] = any ? mx : -9223372036854775807.0;
      }
    }
    return (Real)maxv;
  }

  void moveParticles(move_fn move_funct, double dtau, Field<Real>** fields = NULL, int nfields = 0,
                     double* params = NULL, double* output = NULL, int* reduce_type = NULL,
                     int noutput = 0)
  {
    (void)fields, (void)nfields, (void)params, (void)output, (void)reduce_type, (void)noutput;
    if (!(move_funct == &move_particles_simple_t<part, part_info> ||
          lf2detail::is_simple_move(move_funct)))
      throw std::invalid_argument("moveParticles: only move_particles_simple runs on the GPU");
    sync();
    lf2detail::check(ctx_, lf2_drift_rebin(ctx_, dtau), "lf2_drift_rebin");
  }

  // Particles::saveHDF5 / loadHDF5 (LATfield2_Particles.hpp:2808-3045) for a
  // restart.  HDF5 is not available to this layer: the particles go to
  // filename_base + ".lf2c" in lf2_checkpoint_save's format (the library's
  // state; a restored run continues bit for bit).  fileNumber must be 1 (one
  // process).  loadHDF5 replaces the particles, as a restart into an empty
  // set does in the reference (which adds the file's particles to the set).
  // latfield2_b200.snapshot writes the reference's HDF5 datasets themselves.
  void saveHDF5(const std::string& filename_base, int fileNumber)
  {
    one_file(fileNumber, "saveHDF5");
    sync();
    lf2detail::check(ctx_, lf2_checkpoint_save(ctx_, (filename_base + ".lf2c").c_str()),
                     "lf2_checkpoint_save");
  }
  void loadHDF5(const std::string& filename_base, int fileNumber)
  {
    one_file(fileNumber, "loadHDF5");
    if (!ctx_) throw std::logic_error("Particles: initialize() first");
    pos_.clear(), vel_.clear(), ids_.clear(), mass_.clear();
    lf2detail::check(ctx_, lf2_checkpoint_load(ctx_, (filename_base + ".lf2c").c_str()),
                     "lf2_checkpoint_load");
    int64_t n = 0;
    lf2detail::check(ctx_, lf2_particles_count(ctx_, &n), "lf2_particles_count");
    on_device_ = n;
  }

  Lattice& lattice() { return *lat_; }
  Real res() { return res_; }
  // a field used with these particles covers the same sites
  void check_field(Field<Real>* f, const char* what)
  {
    for (int d = 0; d < 3; d++)
      if (f->lattice().size(d) != lat_->size(d))
        throw std::invalid_argument(std::string(what) + ": field and particle lattices differ in size");
  }
  part_info* parts_info() { return &info_; }

  // ---- GPU side (not in the reference) ----
  lf2_ctx* lf2_context()
  {
    sync();
    return ctx_;
  }
  const std::shared_ptr<lf2_ctx>& lf2_context_owner()
  {
    sync();
    return owner_;
  }
  // All particles (ID, position in box units, velocity), in storage order.
  void getParticles(std::vector<part>& out)
  {
    sync();
    const long n = numParticles();
    std::vector<Real> pos((size_t)(3 * n)), vel((size_t)(3 * n));
    std::vector<int64_t> id((size_t)n);
    lf2detail::check(ctx_, lf2_particles_get_pos(ctx_, pos.data(), vel.data(), sizeof(Real), id.data()),
                     "lf2_particles_get_pos");
    out.assign((size_t)n, part());
    for (long i = 0; i < n; i++) {
      out[(size_t)i].ID = (long)id[(size_t)i];
      for (int d = 0; d < 3; d++) {
        out[(size_t)i].pos[d] = pos[(size_t)(3 * i + d)];
        out[(size_t)i].vel[d] = vel[(size_t)(3 * i + d)];
      }
    }
  }
  // Uploads the particles staged by addParticle_global (with those already
  // on the GPU when there are some).
  void sync()
  {
    if (!ctx_) throw std::logic_error("Particles: initialize() first");
    if (ids_.empty()) return;
    if (on_device_ > 0 && lf2detail::has_mass<part>::value)
      // the GPU does not hand individual masses back with the positions
      throw std::logic_error("Particles: adding particles with individual masses after the upload");
    if (on_device_ > 0) {
      const size_t old = (size_t)on_device_;
      std::vector<double> p(3 * old), v(3 * old);
      std::vector<int64_t> id(old);
      lf2detail::check(ctx_, lf2_particles_get_pos(ctx_, p.data(), v.data(), 8, id.data()),
                       "lf2_particles_get_pos");
      pos_.insert(pos_.begin(), p.begin(), p.end());
      vel_.insert(vel_.begin(), v.begin(), v.end());
      ids_.insert(ids_.begin(), id.begin(), id.end());
    }
    const bool individual = lf2detail::has_mass<part>::value;
    lf2detail::check(ctx_,
                     lf2_particles_set_pos(ctx_, (int64_t)ids_.size(), pos_.data(), vel_.data(), 8,
                                           individual ? mass_.data() : nullptr,
                                           individual ? 0.0 : info_.mass, ids_.data()),
                     "lf2_particles_set_pos");
    gmass_dev_ = individual ? 0.0 : (double)info_.mass;
    on_device_ = (int64_t)ids_.size();
    pos_.clear(), vel_.clear(), ids_.clear(), mass_.clear();
  }

 private:
  template <class P = part>
  static size_t mass_offset_of(std::true_type)
  {
    return offsetof(P, mass);
  }
  static size_t mass_offset_of(std::false_type) { return offsetof(part_info, mass); }

  static void one_file(int fileNumber, const char* what)
  {
    if (fileNumber != 1)
      throw std::invalid_argument(std::string("Particles::") + what + ": one file (one process)");
  }

  std::shared_ptr<lf2_ctx> owner_;  // released by the last of the particles and their fields
  lf2_ctx* ctx_ = nullptr;
  Lattice* lat_ = nullptr;
  part_info info_{};
  double box_[3] = {1, 1, 1};
  Real res_ = 1;
  int64_t on_device_ = 0;
  double gmass_dev_ = 0.0;
  std::vector<double> pos_, vel_;
  std::vector<int64_t> ids_;
  std::vector<float> mass_;
};

// -------------------------------------------------------------- projections
// projection_init (projections.hpp:31-34): the GPU deposits overwrite the
// field, so nothing is needed here.
inline void projection_init(Field<Real>*) {}

template <class part, class part_info, class part_dataType>
void scalarProjectionCIC_project(Particles<part, part_info, part_dataType>* parts, Field<Real>* rho,
                                 size_t* oset = NULL, int flag_where = FROM_INFO)
{
  parts->check_field(rho, "scalarProjectionCIC_project");
  const std::shared_ptr<lf2_ctx>& owner = parts->lf2_context_owner();
  lf2_ctx* ctx = owner.get();
  lf2detail::MassScope ms(ctx, parts->projection_mass(oset, flag_where, false,
                                                      "scalarProjectionCIC_project"),
                          parts->global_mass());
  lf2detail::check(ctx, lf2_deposit_scalar(ctx, rho->lf2_handle(owner, false)), "lf2_deposit_scalar");
  rho->mark_device_written();
}

template <class part, class part_info, class part_dataType>
void vectorProjectionCICNGP_project(Particles<part, part_info, part_dataType>* parts, Field<Real>* vel,
                                    size_t* oset = NULL, int flag_where = FROM_INFO)
{
  parts->check_field(vel, "vectorProjectionCICNGP_project");
  const std::shared_ptr<lf2_ctx>& owner = parts->lf2_context_owner();
  lf2_ctx* ctx = owner.get();
  lf2detail::MassScope ms(ctx, parts->projection_mass(oset, flag_where, true, "vectorProjectionCICNGP_project"),
                          parts->global_mass());
  lf2detail::check(ctx, lf2_deposit_vector_cicngp(ctx, vel->lf2_handle(owner, false)),
                   "lf2_deposit_vector_cicngp");
  vel->mark_device_written();
}

template <class part, class part_info, class part_dataType>
void symtensorProjectionCICNGP_project(Particles<part, part_info, part_dataType>* parts, Field<Real>* Tij,
                                       size_t* oset = NULL, int flag_where = FROM_INFO)
{
  parts->check_field(Tij, "symtensorProjectionCICNGP_project");
  const std::shared_ptr<lf2_ctx>& owner = parts->lf2_context_owner();
  lf2_ctx* ctx = owner.get();
  lf2detail::MassScope ms(ctx, parts->projection_mass(oset, flag_where, true, "symtensorProjectionCICNGP_project"),
                          parts->global_mass());
  lf2detail::check(ctx, lf2_deposit_symtensor_cicngp(ctx, Tij->lf2_handle(owner, false)),
                   "lf2_deposit_symtensor_cicngp");
  Tij->mark_device_written();
}

// vectorProjectionCIC_project (projections.hpp:978-1190): m v / res^3 on
// the links, CIC on the staggered grid along each component's own dim.
template <class part, class part_info, class part_dataType>
void vectorProjectionCIC_project(Particles<part, part_info, part_dataType>* parts, Field<Real>* vel,
                                 size_t* oset = NULL, int flag_where = FROM_INFO)
{
  parts->check_field(vel, "vectorProjectionCIC_project");
  const std::shared_ptr<lf2_ctx>& owner = parts->lf2_context_owner();
  lf2_ctx* ctx = owner.get();
  lf2detail::MassScope ms(ctx, parts->projection_mass(oset, flag_where, true, "vectorProjectionCIC_project"),
                          parts->global_mass());
  lf2detail::check(ctx, lf2_deposit_vector_cic(ctx, vel->lf2_handle(owner, false)),
                   "lf2_deposit_vector_cic");
  vel->mark_device_written();
}

// VecVecProjectionCIC_project (projections.hpp:1355-1620): symmetric
// m v_i v_j / res^3, T_ii on the vertices and T_ij on the (i,j) plaquettes.
template <class part, class part_info, class part_dataType>
void VecVecProjectionCIC_project(Particles<part, part_info, part_dataType>* parts, Field<Real>* Tij,
                                 size_t* oset = NULL, int flag_where = FROM_INFO)
{
  parts->check_field(Tij, "VecVecProjectionCIC_project");
  const std::shared_ptr<lf2_ctx>& owner = parts->lf2_context_owner();
  lf2_ctx* ctx = owner.get();
  lf2detail::MassScope ms(ctx, parts->projection_mass(oset, flag_where, true, "VecVecProjectionCIC_project"),
                          parts->global_mass());
  lf2detail::check(ctx, lf2_deposit_vecvec_cic(ctx, Tij->lf2_handle(owner, false)),
                   "lf2_deposit_vecvec_cic");
  Tij->mark_device_written();
}

// The *_comm functions (projections.hpp:194-300, :558-681, :856-976,
// :1192-1349, :1624-1814): the periodic fold of both halos is part of the
// GPU deposit; here the result comes back to the host array (with its halo
// filled).  The reference's vectorProjectionCIC_comm and
// VecVecProjectionCIC_comm need a process grid of at least 2x2 ranks; on
// this one-GPU layer they give the periodic fold such grids compute.
inline void scalarProjectionCIC_comm(Field<Real>* rho) { rho->pull(); }
inline void vectorProjectionCICNGP_comm(Field<Real>* vel) { vel->pull(); }
inline void symtensorProjectionCICNGP_comm(Field<Real>* Tij) { Tij->pull(); }
inline void vectorProjectionCIC_comm(Field<Real>* vel) { vel->pull(); }
inline void VecVecProjectionCIC_comm(Field<Real>* Tij) { Tij->pull(); }

}  // namespace LATfield2

#endif  // LATFIELD2_B200_HPP
