// glamer_b200.hpp -- C++ mirror of GLAMER/SLsimLib's ray-shooting interface
// over the C ABI of libglamer_b200.so (glamer_b200.h).
//
// Header-only.  The classes carry the reference's names, constructor
// arguments and method signatures for the ray-shooting path, so that code
// written against the reference's Lens / LensHalo* / TreeQuadParticles /
// GridMap compiles against this header with the namespace changed:
//   TreeQuadParticles      include/quadTree.h:49-60, 932
//   LensHalo::force_halo   include/lens_halos.h:182-190
//   LensHaloParticles      include/particle_halo.h:58-93
//   LensHaloNFW            include/lens_halos.h:749-757
//   LensHaloRealNSIE       include/lens_halos.h:1027-1028
//   LensPlaneTree          include/planes.h:35-63
//   Lens                   include/lens.h:73-75, 150-185, 330-349, 458
//   GridMap                include/gridmap.h:35, 80-83
// Point and RAY types are taken as template parameters with the reference's
// member names (Point: x[2], image->x, A.a[4], dt, in_image; RAY: x, y,
// A.a[4], dt, z), so the reference's own structs can be passed unchanged.
//
// Errors: where the reference throws std::invalid_argument the mirror does
// too; every other failure (CUDA, out of memory, a feature outside the
// library) is a std::runtime_error carrying glb_last_error().
#ifndef GLAMER_B200_HPP
#define GLAMER_B200_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "glamer_b200.h"

namespace glamer_b200 {

typedef double PosType;    // include/standard.h:105-128
typedef double KappaType;

// Precision of the tree walk (GLB_PREC_*).  FP64 is the reference's arithmetic.
enum class Precision { FP64 = GLB_PREC_FP64, SPLIT = GLB_PREC_SPLIT, FP32 = GLB_PREC_FP32 };

// Boo of include/point.h:30 (a Point with in_image == MAYBE is not shot,
// include/lens.h:959).
enum { kBooNO = 0, kBooYES = 1, kBooMAYBE = 2 };

// A Point-like type has an `image` member (point.h:428); a RAY has none.
template <class T, class = void>
struct has_image : std::false_type {};
template <class T>
struct has_image<T, decltype((void)std::declval<T &>().image)> : std::true_type {};

inline void check(int rc) {
  if (rc == GLB_OK) return;
  const std::string msg = glb_last_error();
  if (rc == GLB_ERR_ARG || rc == GLB_ERR_SAME_PLACE) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

// Flat Lambda-CDM cosmology (the only one the library implements): the
// stand-in for CosmoLib's COSMOLOGY in the constructors below.
class COSMOLOGY {
 public:
  explicit COSMOLOGY(double omega_matter = 0.3, double omega_lambda = 0.7, double hubble = 0.7)
      : om_(omega_matter), ol_(omega_lambda), h_(hubble) {}
  double getOmega_matter() const { return om_; }
  double getOmega_lambda() const { return ol_; }
  double gethubble() const { return h_; }

 private:
  double om_, ol_, h_;
};

// ParticleType<float> (include/particle_types.h:46-58) or any record with
// x[0..1], Mass and Size, repacked into the library's 24-byte record.
template <class PType>
std::vector<glb_particle> pack_particles(const PType *p, size_t n) {
  std::vector<glb_particle> out(n);
  for (size_t i = 0; i < n; ++i) {
    out[i].x[0] = (float)p[i].x[0];
    out[i].x[1] = (float)p[i].x[1];
    out[i].x[2] = 0.f;
    out[i].Mass = (float)p[i].Mass;
    out[i].Size = (float)p[i].Size;
    out[i].type = 0;
  }
  return out;
}

// ------------------------------------------------------------- the tree
class TreeQuadParticles {
 public:
  template <class PType>
  TreeQuadParticles(PType *xp, size_t Npoints, float mass_fixed = -1, float size_fixed = -1, PosType my_inv_area = 0,
                    int bucket = 5, PosType theta_force = 0.1, bool periodic_buffer = false,
                    PosType my_inv_screening_scale = 0, PosType maximum_range = -1) {
    const std::vector<glb_particle> p = pack_particles(xp, Npoints);
    glb_tree *t = nullptr;
    check(glb_tree_create(p.data(), Npoints, mass_fixed, size_fixed, my_inv_area, bucket, theta_force,
                          periodic_buffer ? 1 : 0, my_inv_screening_scale, maximum_range, &t));
    t_.reset(t);
  }
  // force2D_recur (quadTree.h:932): one ray, outputs overwritten.
  void force2D_recur(const PosType *ray, PosType *alpha, KappaType *kappa, KappaType *gamma, KappaType *phi) {
    check(glb_tree_force2D_recur(t_.get(), 1, ray, alpha, kappa, gamma, phi));
  }
  // The same for n rays (2n positions; alpha 2n, kappa n, gamma 3n, phi n).
  void force2D_recur(size_t n, const PosType *rays, PosType *alpha, KappaType *kappa, KappaType *gamma,
                     KappaType *phi) {
    check(glb_tree_force2D_recur(t_.get(), n, rays, alpha, kappa, gamma, phi));
  }
  glb_tree *handle() const { return t_.get(); }

 private:
  struct Del {
    void operator()(glb_tree *t) const { glb_tree_destroy(t); }
  };
  std::unique_ptr<glb_tree, Del> t_;
};

// ------------------------------------------------------------- the halos
class LensHalo {
 public:
  virtual ~LensHalo() = default;
  void setTheta(PosType PosX, PosType PosY) {
    th_[0] = PosX;
    th_[1] = PosY;
    if (h_) check(glb_halo_set_theta(h_.get(), PosX, PosY));
  }
  void setTheta(const PosType *PosXY) { setTheta(PosXY[0], PosXY[1]); }
  void getTheta(PosType *MyPosHalo) const {
    MyPosHalo[0] = th_[0];
    MyPosHalo[1] = th_[1];
  }
  float get_mass() const { return param(0); }
  float getRsize() const { return param(1); }
  float get_Rmax() const { return param(2); }
  PosType getZlens() const { return z_; }

  // LensHalo::force_halo (lens_halos.h:182-190).  Analytic haloes add to
  // alpha, kappa, gamma and phi; particle haloes overwrite them and return
  // alpha pointing toward the mass (particle_halo.h:426-434).  subtract_point
  // and screening as LensHalo::force_point / force_halo_sym
  // (lens_halos.cpp:1528-1640; glb_halo_force_ex).
  virtual void force_halo(PosType *alpha, KappaType *kappa, KappaType *gamma, KappaType *phi, PosType const *xcm,
                          bool subtract_point = false, PosType screening = 1.0) {
    PosType a[2];
    KappaType k, g[3], p;
    check(glb_halo_force_ex(h_.get(), 1, xcm, a, &k, g, &p, subtract_point ? 1 : 0, screening));
    if (overwrites()) {
      alpha[0] = a[0];
      alpha[1] = a[1];
      *kappa = k;
      gamma[0] = g[0];
      gamma[1] = g[1];
      gamma[2] = g[2];
      *phi = p;
    } else {
      alpha[0] += a[0];
      alpha[1] += a[1];
      *kappa += k;
      gamma[0] += g[0];
      gamma[1] += g[1];
      gamma[2] += g[2];
      *phi += p;
    }
  }

  // Library handle, released to a Lens by Lens::moveinMainHalo; a copy is
  // made from the construction arguments for Lens::insertMainHalo.
  glb_halo *release() { return h_.release(); }
  virtual glb_halo *make_copy() const = 0;

 protected:
  virtual bool overwrites() const { return false; }
  void adopt(glb_halo *h, PosType z) {
    h_.reset(h);
    z_ = z;
  }
  glb_halo *with_theta(glb_halo *h) const {
    if (th_[0] != 0 || th_[1] != 0) check(glb_halo_set_theta(h, th_[0], th_[1]));
    return h;
  }

 private:
  float param(int i) const {
    if (!h_) throw std::runtime_error("LensHalo: halo has been moved into a Lens");
    float v[3];
    check(glb_halo_params(h_.get(), &v[0], &v[1], &v[2]));
    return v[i];
  }
  struct Del {
    void operator()(glb_halo *h) const { glb_halo_destroy(h); }
  };
  std::unique_ptr<glb_halo, Del> h_;
  PosType th_[2] = {0, 0};
  PosType z_ = 0;
};

class LensHaloParticles : public LensHalo {
 public:
  // particle_halo.h:58-75: takes possession of the particles and leaves the
  // vector empty.  theta_rotate must be (0, 0), recenter false and MinPSize
  // 0 (the library's scope); max_range reaches the tree as its
  // inv_screening_scale, as in the reference (particle_halo.h:416).
  // theta_rotate: a Point_2d or anything indexable by [0], [1].
  template <class PType, class Rot>
  LensHaloParticles(std::vector<PType> &pvector, float redshift, const COSMOLOGY &cosmo, const Rot &theta_rotate,
                    bool recenter, double my_inv_area, float MinPSize = 0, double max_range = -1,
                    bool verbose = false)
      : LensHaloParticles(pvector.data(), pvector.size(), redshift, cosmo, theta_rotate, recenter, my_inv_area,
                          MinPSize, max_range, verbose) {
    std::vector<PType>().swap(pvector);
  }
  // particle_halo.h:77-93: does not take possession.
  template <class PType, class Rot>
  LensHaloParticles(PType *begin, size_t n, float redshift, const COSMOLOGY &, const Rot &theta_rotate,
                    bool recenter, double my_inv_area, float MinPSize = 0, double max_range = -1, bool = false)
      : parts_(pack_particles(begin, n)), inv_area_(my_inv_area), max_range_(max_range) {
    if (theta_rotate[0] != 0 || theta_rotate[1] != 0 || recenter || MinPSize > 0)
      throw std::runtime_error("LensHaloParticles: rotation, recentring and MinPSize are not supported");
    glb_halo *h = nullptr;
    check(glb_halo_particles(parts_.data(), parts_.size(), redshift, inv_area_, max_range_, &h));
    adopt(h, redshift);
  }
  glb_halo *make_copy() const override {
    glb_halo *h = nullptr;
    check(glb_halo_particles(parts_.data(), parts_.size(), getZlens(), inv_area_, max_range_, &h));
    return with_theta(h);
  }

  // particle_halo.h:159-162 (def :683-730), on the GPU: pp[i].Size for
  // i < Npoints becomes the distance to the (Nsmooth+1)-th nearest of the
  // Npoints particles (itself counted), TreeSimple::NNDistance's value.
  // Throws std::invalid_argument where the reference exits (Nsmooth < 1,
  // Npoints <= Nsmooth+1).
  // particle_halo.h:734-762: "# nparticles N", "# nsmooth NS", one Size per
  // line as std::ostream prints a float.
  template <class PType>
  static void writeSizes(const std::string &filename, int Nsmooth, const PType *pp, size_t Npoints) {
    std::ofstream f(filename);
    if (!f.is_open()) throw std::runtime_error("file writing error");
    f << "# nparticles " << Npoints << std::endl;
    f << "# nsmooth " << Nsmooth << std::endl;
    for (size_t i = 0; i < Npoints; ++i) {
      f << pp[i].Size << std::endl;
      if (!f) throw std::runtime_error("file writing error");
    }
  }
  // particle_halo.h:557-632: false when the file is missing or was made with
  // another Nsmooth; sizes below min_size are raised to it.
  template <class PType>
  static bool readSizesFile(const std::string &filename, PType *pp, size_t Npoints, int Nsmooth, double min_size) {
    std::ifstream f(filename);
    if (!f.is_open()) return false;
    std::string str, label;
    int count = 0;
    while (std::getline(f, str)) {
      std::stringstream ss(str);
      ss >> label;
      if (label == "#") {
        ss >> label;
        if (label == "nparticles") {
          size_t n = 0;
          ss >> n;
          if (n != Npoints) throw std::runtime_error("file reading error");
          ++count;
        }
        if (label == "nsmooth") {
          int ns = 0;
          ss >> ns;
          if (ns != Nsmooth) return false;
          ++count;
        }
      } else {
        break;
      }
      if (count == 2) break;
    }
    if (count != 2) throw std::runtime_error("file reading error");
    size_t row = 0;
    while (std::getline(f, str)) {
      if (str[0] == '#') continue;
      if (row >= Npoints) throw std::runtime_error("file reading error");
      std::stringstream ss(str);
      ss >> pp[row].Size;
      if (min_size > pp[row].Size) pp[row].Size = (float)min_size;
      ++row;
    }
    if (row != Npoints) throw std::runtime_error("file reading error");
    return true;
  }

  template <class PType>
  static void calculate_smoothing(int Nsmooth, PType *pp, size_t Npoints, bool /*verbose*/ = false) {
    std::vector<glb_particle> v(Npoints);
    for (size_t i = 0; i < Npoints; ++i) {
      for (int k = 0; k < 3; ++k) v[i].x[k] = (float)pp[i].x[k];
      v[i].Mass = (float)pp[i].Mass;
      v[i].Size = (float)pp[i].Size;
      v[i].type = 0;
    }
    check(glb_particles_smoothing(v.data(), Npoints, Nsmooth));
    for (size_t i = 0; i < Npoints; ++i) pp[i].Size = v[i].Size;
  }

 protected:
  bool overwrites() const override { return true; }

 private:
  std::vector<glb_particle> parts_;
  double inv_area_, max_range_;
};

// MakeParticleLenses (particle_halo.h:975-1073, particle_lens.cpp:22-341) for
// glmb and csv3 / csv4 / csv5 files; the smoothing runs on the GPU.  Records are
// glb_particle, the layout of ParticleType<float>.
enum class SimFileFormat { csv3, csv4, csv5, csv6, gadget2, ascii, glmb };

class MakeParticleLenses {
 public:
  std::vector<glb_particle> data;
  std::vector<LensHaloParticles *> halos;

  // particle_lens.cpp:22-107: glmb reads the file; csvN reads
  // <filename>_S<Nsmooth>.glmb when it exists, else the csv file, and writes
  // that glmb file.  csv6 and the other formats throw std::invalid_argument
  // (the reference's switch falls through to its error branch for csv6).
  MakeParticleLenses(const std::string &filename, SimFileFormat format, int Nsmooth, bool recenter)
      : filename_(filename), Nsmooth_(Nsmooth) {
    if (format == SimFileFormat::glmb) {
      if (!readSizesB(filename, data, Nsmooth_, nparticles_, z_original_))
        throw std::invalid_argument("Can't find file.");
    } else {
      const std::string sizefile = filename + "_S" + std::to_string(Nsmooth) + ".glmb";
      std::ifstream probe(sizefile);
      if (probe.good()) {
        readSizesB(sizefile, data, Nsmooth_, nparticles_, z_original_);
      } else {
        if (format == SimFileFormat::csv3) readCSV(3);
        else if (format == SimFileFormat::csv4) readCSV(4);
        else if (format == SimFileFormat::csv5) readCSV(5);
        else throw std::invalid_argument("missing format");
        writeSizesB(sizefile, data, Nsmooth_, nparticles_, z_original_);
      }
    }
    moments(false);
    if (recenter) shift(cm_);
  }
  // particle_lens.cpp:109-137 (its bounding box starts at the origin)
  MakeParticleLenses(const std::string &filename, bool recenter) : filename_(filename), Nsmooth_(0) {
    readSizesB(filename, data, Nsmooth_, nparticles_, z_original_);
    moments(true);
    if (recenter) Recenter(cm_);
  }
  ~MakeParticleLenses() {
    for (auto *h : halos) delete h;
  }
  MakeParticleLenses(const MakeParticleLenses &) = delete;
  MakeParticleLenses &operator=(const MakeParticleLenses &) = delete;

  std::vector<size_t> getnp() const { return nparticles_; }
  std::array<double, 3> getCenterOfMass() const { return cm_; }
  void getBoundingBox(std::array<double, 3> &Xmin, std::array<double, 3> &Xmax) const {
    Xmin = ll_;
    Xmax = ur_;
  }
  double getZoriginal() const { return z_original_; }

  // particle_lens.cpp:139-151
  void Recenter(std::array<double, 3> x) {
    shift(x);
    for (auto *h : halos) delete h;
    halos.clear();
  }

  // particle_lens.cpp:447-478: drops the particles farther than radius from
  // center (each swapped with the last kept one); re-sorted by type when more
  // than one type remains (stable here)
  void radialCut(std::array<double, 3> center, double radius) {
    cut([&](const glb_particle &p) {
      const double a = p.x[0] - center[0], b = p.x[1] - center[1], c = p.x[2] - center[2];
      return a * a + b * b + c * c;
    }, radius);
  }
  // particle_lens.cpp:497-520: the same with the distance in x, y
  void cylindricalCut(std::array<double, 2> center, double radius) {
    cut([&](const glb_particle &p) {
      const double a = p.x[0] - center[0], b = p.x[1] - center[1];
      return a * a + b * b;
    }, radius);
  }
  // particle_lens.cpp:480-495: position of the largest Mass/Size^3 (float)
  std::array<double, 3> densest_particle() const {
    double dmax = -1;
    std::array<double, 3> x{0, 0, 0};
    for (const auto &p : data) {
      const double d = p.Mass / p.Size / p.Size / p.Size;
      if (d > dmax) {
        dmax = d;
        x = {p.x[0], p.x[1], p.x[2]};
      }
    }
    return x;
  }

  // particle_lens.cpp:153-209: records to comoving Mpc / Msun (divided by h),
  // one LensHaloParticles per particle type present
  void CreateHalos(const COSMOLOGY &cosmo, double redshift, double inv_area) {
    const float h = (float)cosmo.gethubble();
    const double unit = 1.0 / h;
    for (auto &p : data) {
      for (int k = 0; k < 3; ++k) p.x[k] = (float)(p.x[k] * unit);
      p.Size = (float)(p.Size * unit);
      p.Mass = (float)(p.Mass * unit);
    }
    for (auto *hh : halos) delete hh;
    halos.clear();
    size_t skip = 0;
    struct Zero {
      double operator[](int) const { return 0.0; }
    };
    for (int i = 0; i < 6; ++i) {
      if (nparticles_[i] > 0)
        halos.push_back(new LensHaloParticles(data.data() + skip, nparticles_[i], (float)redshift, cosmo, Zero(),
                                              false, inv_area));
      skip += nparticles_[i];
    }
  }

  // particle_halo.h:1036-1053
  static void writeSizesB(const std::string &filename, const std::vector<glb_particle> &pv, int Nsmooth,
                          const std::vector<size_t> &numbytype, double redshift) {
    if (numbytype.size() != 6) throw std::invalid_argument("numbytype must have 6 entries");
    std::ofstream f(filename, std::ios::out | std::ios::binary);
    if (!f.write((const char *)&Nsmooth, sizeof(int))) throw std::runtime_error("file writing error");
    const size_t ntot = pv.size();
    f.write((const char *)&ntot, sizeof(size_t));
    f.write((const char *)numbytype.data(), sizeof(size_t) * 6);
    f.write((const char *)&redshift, sizeof(double));
    f.write((const char *)pv.data(), sizeof(glb_particle) * ntot);
  }
  // particle_halo.h:1056-1073
  static bool readSizesB(const std::string &filename, std::vector<glb_particle> &pv, int &Nsmooth,
                         std::vector<size_t> &numbytype, double &redshift) {
    numbytype.assign(6, 0);
    std::ifstream f(filename, std::ios::in | std::ios::binary);
    if (!f.read((char *)&Nsmooth, sizeof(int))) return false;
    size_t ntot = 0;
    f.read((char *)&ntot, sizeof(size_t));
    f.read((char *)numbytype.data(), sizeof(size_t) * 6);
    f.read((char *)&redshift, sizeof(double));
    pv.assign(ntot, glb_particle{});
    f.read((char *)pv.data(), sizeof(glb_particle) * ntot);
    return true;
  }

 private:
  std::string filename_;
  int Nsmooth_;
  std::vector<size_t> nparticles_ = std::vector<size_t>(6, 0);
  double z_original_ = -1;
  std::array<double, 3> cm_{}, ll_{}, ur_{};

  // particle_lens.cpp:211-341 for 3, 4 and 5 columns
  void readCSV(int columns_used) {
    std::ifstream file(filename_);
    std::string line;
    while (std::getline(file, line) && line[0] == '#') {
    }
    auto split = [](const std::string &l) {
      std::vector<std::string> v;
      std::stringstream ss(l);
      std::string c;
      while (std::getline(ss, c, ',')) v.push_back(c);
      return v;
    };
    if ((int)split(line).size() < columns_used) throw std::invalid_argument("bad file");
    data.clear();
    do {
      const std::vector<std::string> v = split(line);
      glb_particle p{};
      p.x[0] = std::stof(v[0]);
      p.x[1] = std::stof(v[1]);
      p.x[2] = std::stof(v[2]);
      p.Mass = columns_used == 3 ? 1.0f : std::stof(v[3]);
      if (columns_used == 5) p.Size = std::stof(v[4]);
      data.push_back(p);
    } while (std::getline(file, line));
    nparticles_ = {data.size(), 0, 0, 0, 0, 0};
    if (columns_used < 5) LensHaloParticles::calculate_smoothing(Nsmooth_, data.data(), data.size());
  }
  void moments(bool from_origin) {
    double m = 0;
    cm_ = {0, 0, 0};
    for (int k = 0; k < 3; ++k) ll_[k] = ur_[k] = (from_origin || data.empty()) ? 0.0 : data[0].x[k];
    for (const auto &p : data) {
      for (int k = 0; k < 3; ++k) {
        cm_[k] += p.x[k] * p.Mass;
        if (ll_[k] > p.x[k]) ll_[k] = p.x[k];
        if (ur_[k] < p.x[k]) ur_[k] = p.x[k];
      }
      m += p.Mass;
    }
    for (int k = 0; k < 3; ++k) cm_[k] /= m;
  }
  template <class R2>
  void cut(R2 r2of, double radius) {
    const double radius2 = radius * radius;
    size_t end = data.size(), i = 0;
    while (i < end) {
      if (r2of(data[i]) > radius2) {
        --nparticles_[data[i].type];
        --end;
        std::swap(data[i], data[end]);
      } else {
        ++i;
      }
    }
    data.resize(end);
    int ntypes = 0;
    for (size_t k : nparticles_) ntypes += k > 0;
    if (ntypes > 1)
      std::stable_sort(data.begin(), data.end(),
                       [](const glb_particle &a, const glb_particle &b) { return a.type < b.type; });
  }
  void shift(std::array<double, 3> x) {
    for (auto &p : data)
      for (int k = 0; k < 3; ++k) p.x[k] = (float)(p.x[k] - x[k]);
    for (int k = 0; k < 3; ++k) {
      ll_[k] -= x[k];
      ur_[k] -= x[k];
      cm_[k] -= x[k];
    }
  }
};

class LensHaloNFW : public LensHalo {
 public:
  // lens_halos.h:749-757 (fratio must be 1: the library's NFW is spherical)
  LensHaloNFW(float my_mass, float my_Rsize, PosType my_zlens, float my_concentration, float my_fratio, float my_pa,
              const COSMOLOGY &)
      : m_(my_mass), r_(my_Rsize), c_(my_concentration), f_(my_fratio), pa_(my_pa) {
    glb_halo *h = nullptr;
    check(glb_halo_nfw(m_, r_, my_zlens, c_, f_, pa_, &h));
    adopt(h, my_zlens);
  }
  glb_halo *make_copy() const override {
    glb_halo *h = nullptr;
    check(glb_halo_nfw(m_, r_, getZlens(), c_, f_, pa_, &h));
    return with_theta(h);
  }

 private:
  float m_, r_, c_, f_, pa_;
};

class LensHaloRealNSIE : public LensHalo {
 public:
  // lens_halos.h:1027-1028
  LensHaloRealNSIE(float my_mass, PosType my_zlens, float my_sigma, float my_rcore, float my_fratio, float my_pa,
                   const COSMOLOGY &)
      : m_(my_mass), s_(my_sigma), rc_(my_rcore), f_(my_fratio), pa_(my_pa) {
    glb_halo *h = nullptr;
    check(glb_halo_nsie(m_, my_zlens, s_, rc_, f_, pa_, &h));
    adopt(h, my_zlens);
  }
  glb_halo *make_copy() const override {
    glb_halo *h = nullptr;
    check(glb_halo_nsie(m_, getZlens(), s_, rc_, f_, pa_, &h));
    return with_theta(h);
  }

 private:
  float m_, s_, rc_, f_, pa_;
};

// LensPlaneTree(z, halos, Nhalos, sigma_background, inv_screening_scale)
// (include/planes.h:35-63, MultiPlane/planes.cpp:13-18): a plane of NFW /
// NSIE field haloes walked as TreeQuadHalos.  The plane holds its own copies
// of the haloes (moved to redshift z), so the caller's objects stay usable.
class LensPlaneTree {
 public:
  LensPlaneTree(float z, LensHalo **my_halos, size_t Nhalos, PosType my_sigma_background,
                PosType my_inv_screening_scale = 0) {
    std::vector<glb_halo *> members;
    try {
      for (size_t i = 0; i < Nhalos; ++i) members.push_back(my_halos[i]->make_copy());
    } catch (...) {
      for (glb_halo *m : members) glb_halo_destroy(m);
      throw;
    }
    glb_halo *h = nullptr;
    const int rc = glb_halo_field_plane(members.data(), (int)members.size(), z, my_sigma_background,
                                        my_inv_screening_scale, &h);
    if (rc != GLB_OK) {
      for (glb_halo *m : members) glb_halo_destroy(m);
      check(rc);
    }
    h_.reset(h);
  }
  // LensPlaneTree::force (planes.cpp:65-68): outputs overwritten.
  void force(PosType *alpha, KappaType *kappa, KappaType *gamma, KappaType *phi, PosType *xx) {
    if (!h_) throw std::runtime_error("LensPlaneTree: plane has been moved into a Lens");
    check(glb_halo_force(h_.get(), 1, xx, alpha, kappa, gamma, phi));
  }
  glb_halo *release() { return h_.release(); }

 private:
  struct Del {
    void operator()(glb_halo *h) const { glb_halo_destroy(h); }
  };
  std::unique_ptr<glb_halo, Del> h_;
};

// ------------------------------------------------------------- the lens
class Lens {
 public:
  // lens.h:75 (the seed drives only the reference's field-halo generation,
  // which is outside this library)
  Lens(long *, PosType z_source, const COSMOLOGY &cosmo, bool = false) {
    glb_lens *l = nullptr;
    check(glb_lens_create(z_source, cosmo.getOmega_matter(), cosmo.getOmega_lambda(), cosmo.gethubble(), &l));
    l_.reset(l);
  }
  // lens.h:150-170: the lens keeps its own copy of the halo.
  template <class T>
  void insertMainHalo(const T &halo_in, bool addplanes, bool = false) {
    check(glb_lens_insert_halo(l_.get(), halo_in.make_copy(), addplanes ? 1 : 0));
  }
  // lens.h:173-185: the lens takes the halo; halo_in is left empty.
  template <class T>
  void moveinMainHalo(T &halo_in, bool addplanes, bool = false) {
    glb_halo *h = halo_in.release();
    if (!h) throw std::invalid_argument("moveinMainHalo: halo already moved");
    check(glb_lens_insert_halo(l_.get(), h, addplanes ? 1 : 0));
  }
  // A field plane among the lens planes, as Lens::createFieldPlanes adds each
  // LensPlaneTree (lens.cpp:443-452); the lens takes the plane.
  void insertFieldPlane(LensPlaneTree &plane) {
    glb_halo *h = plane.release();
    if (!h) throw std::invalid_argument("insertFieldPlane: plane already moved");
    check(glb_lens_insert_field_plane(l_.get(), h));
  }
  int getNplanes() const {
    int n = 0;
    check(glb_lens_nplanes(l_.get(), &n));
    return n;
  }
  PosType getSourceZ() const {
    const int n = getNplanes();
    std::vector<double> z(n + 1);
    check(glb_lens_planes(l_.get(), z.data(), nullptr, nullptr));
    return z[n];
  }
  // lens.h:458
  short ResetSourcePlane(PosType z, bool nearest = false, bool = false) {
    int j = 0;
    check(glb_lens_reset_source(l_.get(), z, nearest ? 1 : 0, &j));
    return (short)j;
  }

  // rayshooterInternal(Npoints, Point*) (lens.h:330-333): i_points[].x in
  // radians in; image->x (source position), A on both points and dt = 0 out.
  // Points with in_image == MAYBE are left untouched.
  template <class PointT, typename std::enable_if<has_image<PointT>::value, int>::type = 0>
  void rayshooterInternal(unsigned long Npoints, PointT *i_points, bool = false) {
    shoot_points(Npoints, i_points, nullptr);
  }
  // rayshooterInternal(Npoints, LinkedPoint*, source_zs) (lens.h:340-344)
  template <class PointT>
  void rayshooterInternal(unsigned long Npoints, PointT *i_points, std::vector<double> &source_zs, bool = false) {
    if (source_zs.size() != Npoints)
      throw std::invalid_argument("number of source redshifts and rays do not match");
    shoot_points(Npoints, i_points, &source_zs);
  }
  // rayshooterInternal(Npoints, RAY*) (lens.h:346): x in, y, A and dt out,
  // per-ray source redshift z (z <= 0: the lens's source plane).
  template <class RayT, typename std::enable_if<!has_image<RayT>::value, int>::type = 0>
  void rayshooterInternal(unsigned long Npoints, RayT *rays) {
    std::vector<double> x(2 * Npoints), zs(Npoints), y(2 * Npoints), A(4 * Npoints);
    bool any_z = false;
    const double zsrc = getSourceZ();
    for (unsigned long i = 0; i < Npoints; ++i) {
      x[2 * i] = rays[i].x[0];
      x[2 * i + 1] = rays[i].x[1];
      zs[i] = rays[i].z > 0 ? (double)rays[i].z : zsrc;
      any_z = any_z || rays[i].z > 0;
    }
    check(glb_lens_rayshoot(l_.get(), Npoints, x.data(), any_z ? zs.data() : nullptr, y.data(), A.data(),
                            (int)precision));
    for (unsigned long i = 0; i < Npoints; ++i) {
      rays[i].y[0] = y[2 * i];
      rays[i].y[1] = y[2 * i + 1];
      for (int c = 0; c < 4; ++c) rays[i].A.a[c] = A[4 * i + c];
      rays[i].dt = 0;
    }
  }
  // rayshooterInternal(RAY&) (lens.h:349)
  template <class RayT, typename std::enable_if<!has_image<RayT>::value, int>::type = 0>
  void rayshooterInternal(RayT &ray) {
    rayshooterInternal(1ul, &ray);
  }

  // Precision of the walk for this lens's calls (default: the reference's FP64).
  Precision precision = Precision::FP64;
  glb_lens *handle() const { return l_.get(); }

 private:
  template <class PointT>
  void shoot_points(unsigned long Npoints, PointT *p, const std::vector<double> *zs) {
    std::vector<unsigned long> idx;
    idx.reserve(Npoints);
    for (unsigned long i = 0; i < Npoints; ++i)
      if ((int)p[i].in_image != kBooMAYBE) idx.push_back(i);
    const size_t n = idx.size();
    std::vector<double> x(2 * n), z(zs ? n : 0), y(2 * n), A(4 * n);
    for (size_t k = 0; k < n; ++k) {
      x[2 * k] = p[idx[k]].x[0];
      x[2 * k + 1] = p[idx[k]].x[1];
      if (zs) z[k] = (*zs)[idx[k]];
    }
    check(glb_lens_rayshoot(l_.get(), n, x.data(), zs ? z.data() : nullptr, y.data(), A.data(), (int)precision));
    for (size_t k = 0; k < n; ++k) {
      PointT &q = p[idx[k]];
      q.image->x[0] = y[2 * k];
      q.image->x[1] = y[2 * k + 1];
      for (int c = 0; c < 4; ++c) q.A.a[c] = q.image->A.a[c] = A[4 * k + c];
      q.dt = q.image->dt = 0;
    }
  }
  struct Del {
    void operator()(glb_lens *l) const { glb_lens_destroy(l); }
  };
  std::unique_ptr<glb_lens, Del> l_;
};

// ------------------------------------------------------------- sources
// The analytic sources of GridMap::RefreshSurfaceBrightnesses that the library
// evaluates on the GPU (glb_gridmap_surface_brightness).  Constructors take
// the reference's arguments (AnalyticNSIE/source.cpp, Source/sersic.cpp);
// Point_2d-like positions are anything indexable by [0], [1].
class Source {
 public:
  virtual ~Source() = default;
  void setTheta(PosType x, PosType y) {
    prm_[0] = x;
    prm_[1] = y;
  }
  int kind() const { return kind_; }
  const std::vector<double> &params() const { return prm_; }

 protected:
  int kind_ = 0;
  std::vector<double> prm_;
};

class SourceUniform : public Source {
 public:
  template <class P2>
  SourceUniform(const P2 &position, PosType /*z*/, PosType radius_in_radians) {
    kind_ = 0;
    prm_ = {position[0], position[1], radius_in_radians};
  }
};

class SourceGaussian : public Source {
 public:
  template <class P2>
  SourceGaussian(const P2 &position, double r_size, double /*z*/, double /*SBlimit*/, double /*zero_point*/) {
    kind_ = 1;
    prm_ = {position[0], position[1], r_size};
  }
};

class SourceSersic : public Source {
 public:
  // SourceSersic(mag, Reff [arcsec], PA, index, q, z, zeropoint, band): the total
  // flux is mag_to_flux(mag, zeropoint) = 10^(-0.4 (mag - zeropoint))
  // (include/source.h:31-34); the source sits at (0, 0) until setTheta.
  template <class BandT>
  SourceSersic(double my_mag, double my_Reff, double my_PA, double my_index, double my_q, double /*my_z*/,
               double my_zeropoint, BandT /*band*/) {
    kind_ = 2;
    const double flux = my_mag == 100 ? 0.0 : std::pow(10, -0.4 * (my_mag - my_zeropoint));
    prm_ = {0.0, 0.0, flux, my_Reff, my_PA, my_index, my_q, -1.0};
  }
};

// LensingVariable (include/standard.h:89-102)
enum class LensingVariable { DELAYT, ALPHA, ALPHA1, ALPHA2, KAPPA, GAMMA, GAMMA1, GAMMA2, GAMMA3, INVMAG, PHI,
                             SurfBrightness };

// ------------------------------------------------------------- GridMap
// GridMap(LensHndl, N1d, center, range) (gridmap.h:35, gridmap.cpp:93-120):
// the grid is generated and shot on the GPU; y and A are kept per point in
// GridMap order (x fastest).
class GridMap {
 public:
  GridMap(Lens *lens, unsigned long N1d, const double center[2], double range,
          Precision prec = Precision::FP64)
      : n_(N1d), range_(range), y_(2 * N1d * N1d), A_(4 * N1d * N1d) {
    center_[0] = center[0];
    center_[1] = center[1];
    check(glb_gridmap(lens->handle(), N1d, center, range, y_.data(), A_.data(), (int)prec));
  }
  size_t getNumberOfPoints() const { return n_ * n_; }
  int getInitNgrid() const { return (int)n_; }
  double getInitRange() const { return range_; }
  void getInitCenter(double *c) const {
    c[0] = center_[0];
    c[1] = center_[1];
  }
  // image position of point i (PositionFromIndex, utilities.cpp:149-158)
  void image(size_t i, double *x) const {
    if (n_ == 1) {
      x[0] = center_[0];
      x[1] = center_[1];
      return;
    }
    x[0] = center_[0] + range_ * (1.0 * (double)(i % n_) / (double)(n_ - 1) - 0.5);
    x[1] = center_[1] + range_ * (1.0 * (double)(i / n_) / (double)(n_ - 1) - 0.5);
  }
  const double *source(size_t i) const { return &y_[2 * i]; }
  const double *A(size_t i) const { return &A_[4 * i]; }
  // the derived quantities of Point (point.h:377-381, 446-448)
  double kappa(size_t i) const { return 1 - 0.5 * (A_[4 * i] + A_[4 * i + 3]); }
  double gamma1(size_t i) const { return 0.5 * (A_[4 * i] - A_[4 * i + 3]); }
  double gamma2(size_t i) const { return 0.5 * (A_[4 * i + 1] + A_[4 * i + 2]); }
  double gamma3(size_t i) const { return 0.5 * (A_[4 * i + 2] - A_[4 * i + 1]); }
  double invmag(size_t i) const { return A_[4 * i] * A_[4 * i + 3] - A_[4 * i + 1] * A_[4 * i + 2]; }

  // GridMap::writePixelMap (gridmap.h:529-598) as a plain array in grid
  // order (x fastest) from this GridMap's points.
  std::vector<double> writePixelMap(LensingVariable lensvar) const {
    const size_t n = getNumberOfPoints();
    std::vector<double> m(n, 0.0);
    for (size_t i = 0; i < n; ++i) {
      double x[2];
      image(i, x);
      const double d0 = x[0] - y_[2 * i], d1 = x[1] - y_[2 * i + 1];
      switch (lensvar) {
        case LensingVariable::DELAYT: m[i] = 0; break;
        case LensingVariable::ALPHA: m[i] = std::sqrt(d0 * d0 + d1 * d1); break;
        case LensingVariable::ALPHA1: m[i] = d0; break;
        case LensingVariable::ALPHA2: m[i] = d1; break;
        case LensingVariable::KAPPA: m[i] = kappa(i); break;
        case LensingVariable::GAMMA: m[i] = std::sqrt(gamma1(i) * gamma1(i) + gamma2(i) * gamma2(i)); break;
        case LensingVariable::GAMMA1: m[i] = gamma1(i); break;
        case LensingVariable::GAMMA2: m[i] = gamma2(i); break;
        case LensingVariable::GAMMA3: m[i] = gamma3(i); break;
        case LensingVariable::INVMAG: m[i] = invmag(i); break;
        default:
          throw std::runtime_error("GridMap::writePixelMap() does not work for the input LensingVariable");
      }
    }
    return m;
  }
  // GridMap::RefreshSurfaceBrightnesses (gridmap.cpp:174-187) on the GPU for
  // this grid's lens: per-point surface brightness into `sb` (optional) and
  // the reference's total (sum of sb x resolution^2 in point order).
  static double RefreshSurfaceBrightnesses(Lens *lens, unsigned long N1d, const double center[2], double range,
                                           const Source &source, std::vector<double> *sb = nullptr,
                                           Precision prec = Precision::FP64) {
    std::vector<double> tmp(N1d * N1d);
    double total = 0;
    check(glb_gridmap_surface_brightness(lens->handle(), N1d, center, range, source.kind(), source.params().data(),
                                         tmp.data(), &total, (int)prec));
    if (sb) sb->swap(tmp);
    return total;
  }
  // GridMap::AdaptiveRefreshSurfaceBrightnesses (gridmap.cpp:189-258): the
  // refinement sub-rays batched on the GPU (glb_gridmap_adaptive_surface_brightness).
  static double AdaptiveRefreshSurfaceBrightnesses(Lens *lens, unsigned long N1d, const double center[2],
                                                   double range, const Source &source,
                                                   std::vector<double> *sb = nullptr,
                                                   Precision prec = Precision::FP64) {
    std::vector<double> tmp(N1d * N1d);
    double total = 0;
    check(glb_gridmap_adaptive_surface_brightness(lens->handle(), N1d, center, range, source.kind(),
                                                  source.params().data(), tmp.data(), &total, (int)prec));
    if (sb) sb->swap(tmp);
    return total;
  }
  // The same map computed on the GPU from a fresh grid (no per-point arrays
  // on the host): glb_gridmap_pixelmap.
  static std::vector<double> writePixelMapOnDevice(Lens *lens, unsigned long N1d, const double center[2],
                                                   double range, LensingVariable lensvar,
                                                   Precision prec = Precision::FP64) {
    std::vector<double> m(N1d * N1d);
    check(glb_gridmap_pixelmap(lens->handle(), N1d, center, range, (int)lensvar, m.data(), (int)prec));
    return m;
  }

 private:
  size_t n_;
  double range_, center_[2];
  std::vector<double> y_, A_;
};

}  // namespace glamer_b200

#endif
