// Drives the C++ mirror (include/glamer_b200.hpp) with structs shaped like
// the reference's own (ParticleType<float>, Point with image / A / dt /
// in_image, RAY with x, y, A, dt, z, Point_2d with operator[]), checks the
// mirror's semantics against direct C-ABI calls, and writes its inputs and
// GridMap results for tests/test_cpp_mirror.py to compare with the oracle.
//
//   mirror_test <output directory>      exit 0 and "OK" on success
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "glamer_b200.hpp"

namespace ref {  // the reference's shapes (point.h, particle_types.h)
typedef enum { NO, YES, MAYBE } Boo;
struct ParticleType {
  float x[3];
  float Mass;
  float Size;
  int type;
};
struct Matrix2x2 {
  double a[4];
};
struct Point_2d {
  double x[2];
  double &operator[](size_t i) { return x[i]; }
  const double &operator[](size_t i) const { return x[i]; }
};
struct Point {
  double x[2];
  Point *image = nullptr;
  Boo in_image = NO;
  double dt = -1;
  Matrix2x2 A;
};
struct RAY {
  Point_2d x, y;
  Matrix2x2 A;
  double dt = -1;
  double z = -1;
};
}  // namespace ref

namespace g = glamer_b200;

static unsigned long long rng_state = 88172645463325252ull;
static double urand() {  // xorshift64*, uniform in [0, 1)
  rng_state ^= rng_state >> 12;
  rng_state ^= rng_state << 25;
  rng_state ^= rng_state >> 27;
  return (double)((rng_state * 2685821657736338717ull) >> 11) * (1.0 / 9007199254740992.0);
}
static double grand() { return std::sqrt(-2 * std::log(1 - urand())) * std::cos(2 * M_PI * urand()); }

static std::vector<ref::ParticleType> blob(size_t n, double sigma, double cx, double cy, float mass, float size) {
  std::vector<ref::ParticleType> p(n);
  for (auto &q : p) {
    q.x[0] = (float)(cx + sigma * grand());
    q.x[1] = (float)(cy + sigma * grand());
    q.x[2] = 0;
    q.Mass = mass;
    q.Size = size;
    q.type = 0;
  }
  return p;
}

#define REQUIRE(c)                                                         \
  do {                                                                     \
    if (!(c)) {                                                            \
      std::fprintf(stderr, "FAILED %s at line %d\n", #c, __LINE__);        \
      std::exit(1);                                                        \
    }                                                                      \
  } while (0)

static void write(const std::string &path, const void *p, size_t bytes) {
  FILE *f = std::fopen(path.c_str(), "wb");
  REQUIRE(f);
  REQUIRE(std::fwrite(p, 1, bytes, f) == bytes);
  std::fclose(f);
}

int main(int argc, char **argv) {
  const std::string out = argc > 1 ? argv[1] : ".";
  const double arcsec = 4.848136811e-6;
  g::COSMOLOGY cosmo(0.3, 0.7, 0.7);
  long seed = -1;

  // two particle planes + NFW + NSIE, inserted the reference's ways
  std::vector<ref::ParticleType> p1 = blob(20000, 0.02, 0.0, 0.0, 2e9f, 1e-3f);
  std::vector<ref::ParticleType> p2 = blob(15000, 0.03, 0.01, -0.005, 2e9f, 1e-3f);
  write(out + "/plane1.bin", p1.data(), p1.size() * sizeof(ref::ParticleType));
  write(out + "/plane2.bin", p2.data(), p2.size() * sizeof(ref::ParticleType));
  const double zsrc = 2.0;
  ref::Point_2d norot{{0, 0}};

  g::Lens lens(&seed, zsrc, cosmo);
  g::Lens lens_copy(&seed, zsrc, cosmo);
  {
    std::vector<ref::ParticleType> v1 = p1;
    g::LensHaloParticles h1(v1, 0.3f, cosmo, norot, false, 0.0);
    REQUIRE(v1.empty());  // the vector constructor takes possession
    g::LensHaloParticles h2(p2.data(), p2.size(), 0.6f, cosmo, norot, false, 0.0);
    g::LensHaloNFW nfw(5e13f, 0.5f, 0.45, 6.0f, 1.0f, 0.0f, cosmo);
    nfw.setTheta(3 * arcsec, -2 * arcsec);
    g::LensHaloRealNSIE nsie(1e13f, 0.3, 220.0f, 3e-4f, 0.75f, 0.4f, cosmo);
    lens_copy.insertMainHalo(h1, true);
    lens_copy.insertMainHalo(h2, true);
    lens_copy.insertMainHalo(nfw, true);
    lens_copy.insertMainHalo(nsie, true);
    REQUIRE(nfw.get_mass() > 0);  // insertMainHalo leaves the halo usable
    lens.moveinMainHalo(h1, true);
    lens.moveinMainHalo(h2, true);
    lens.moveinMainHalo(nfw, true);
    lens.moveinMainHalo(nsie, true);
    bool threw = false;
    try {
      lens.moveinMainHalo(nfw, true);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    REQUIRE(threw);
  }
  // particle haloes keep their redshift as a float (0.3f), which puts the
  // NSIE at z = 0.3 on a plane of its own: 0.3f, 0.3, 0.45, 0.6
  REQUIRE(lens.getNplanes() == 4);
  REQUIRE(std::fabs(lens.getSourceZ() - zsrc) < 1e-12);

  // GridMap, copy- and move-built lenses agree bit for bit
  const double center[2] = {0, 0};
  const unsigned long n1d = 24;
  const double range = 40 * arcsec;
  g::GridMap gm(&lens, n1d, center, range);
  g::GridMap gm2(&lens_copy, n1d, center, range);
  REQUIRE(gm.getNumberOfPoints() == n1d * n1d && gm.getInitNgrid() == (int)n1d);
  std::vector<double> gy(2 * n1d * n1d), gA(4 * n1d * n1d);
  for (size_t i = 0; i < n1d * n1d; ++i) {
    for (int c = 0; c < 2; ++c) REQUIRE(gm.source(i)[c] == gm2.source(i)[c]);
    for (int c = 0; c < 4; ++c) REQUIRE(gm.A(i)[c] == gm2.A(i)[c]);
    std::memcpy(&gy[2 * i], gm.source(i), 2 * sizeof(double));
    std::memcpy(&gA[4 * i], gm.A(i), 4 * sizeof(double));
  }
  for (g::LensingVariable v : {g::LensingVariable::ALPHA, g::LensingVariable::KAPPA, g::LensingVariable::GAMMA,
                               g::LensingVariable::INVMAG, g::LensingVariable::GAMMA3}) {
    const std::vector<double> host = gm.writePixelMap(v);
    const std::vector<double> dev = g::GridMap::writePixelMapOnDevice(&lens, n1d, center, range, v);
    for (size_t i = 0; i < host.size(); ++i)
      REQUIRE(std::fabs(host[i] - dev[i]) <= 1e-12 * std::fabs(host[i]) + 1e-300);
  }
  {  // surface brightness of a Sersic source placed where the lens maps the grid centre
    g::SourceSersic src(22.0, 0.5, 0.3, 2.0, 0.8, 2.0, 0.0, 0);
    const size_t mid = n1d * n1d / 2;
    src.setTheta(gm.source(mid)[0], gm.source(mid)[1]);
    std::vector<double> sb;
    const double total = g::GridMap::RefreshSurfaceBrightnesses(&lens, n1d, center, range, src, &sb);
    const double res2 = std::pow(range / (n1d - 1), 2);
    double expect = 0;
    for (double v : sb) expect += v * res2;
    REQUIRE(sb.size() == n1d * n1d && sb[mid] > 0 && total == expect);
    std::vector<double> sba;
    const double ta = g::GridMap::AdaptiveRefreshSurfaceBrightnesses(&lens, n1d, center, range, src, &sba);
    REQUIRE(sba.size() == n1d * n1d && ta > 0);
  }
  write(out + "/grid_y.bin", gy.data(), gy.size() * sizeof(double));
  write(out + "/grid_A.bin", gA.data(), gA.size() * sizeof(double));

  // Point* overload: image points linked to source points; MAYBE left alone
  const size_t np = 300;
  std::vector<ref::Point> img(np), src(np);
  std::vector<double> x(2 * np);
  for (size_t i = 0; i < np; ++i) {
    img[i].x[0] = x[2 * i] = (urand() - 0.5) * 30 * arcsec;
    img[i].x[1] = x[2 * i + 1] = (urand() - 0.5) * 30 * arcsec;
    img[i].image = &src[i];
    src[i].image = &img[i];
    if (i % 7 == 3) img[i].in_image = ref::MAYBE;
  }
  lens.rayshooterInternal(np, img.data());
  std::vector<double> y(2 * np), A(4 * np);
  g::check(glb_lens_rayshoot(lens.handle(), np, x.data(), nullptr, y.data(), A.data(), GLB_PREC_FP64));
  for (size_t i = 0; i < np; ++i) {
    if (i % 7 == 3) {
      REQUIRE(img[i].dt == -1 && src[i].dt == -1);  // untouched
      continue;
    }
    REQUIRE(src[i].x[0] == y[2 * i] && src[i].x[1] == y[2 * i + 1]);
    for (int c = 0; c < 4; ++c) REQUIRE(img[i].A.a[c] == A[4 * i + c] && src[i].A.a[c] == A[4 * i + c]);
    REQUIRE(img[i].dt == 0 && src[i].dt == 0);
  }

  // LinkedPoint + source_zs overload and RAY* overload agree; z <= 0 means
  // the lens's source plane
  std::vector<double> zs(np);
  std::vector<ref::RAY> rays(np);
  for (size_t i = 0; i < np; ++i) {
    img[i].in_image = ref::NO;
    zs[i] = i % 5 == 0 ? zsrc : 0.5 + 2.5 * urand();
    rays[i].x[0] = x[2 * i];
    rays[i].x[1] = x[2 * i + 1];
    rays[i].z = i % 5 == 0 ? -1 : zs[i];
  }
  lens.rayshooterInternal(np, img.data(), zs);
  lens.rayshooterInternal(np, rays.data());
  for (size_t i = 0; i < np; ++i) {
    REQUIRE(rays[i].y[0] == src[i].x[0] && rays[i].y[1] == src[i].x[1]);
    for (int c = 0; c < 4; ++c) REQUIRE(rays[i].A.a[c] == img[i].A.a[c]);
    REQUIRE(rays[i].dt == 0);
  }
  ref::RAY one = rays[7];
  lens.rayshooterInternal(one);
  REQUIRE(one.y[0] == rays[7].y[0] && one.y[1] == rays[7].y[1]);
  {
    bool threw = false;
    std::vector<double> short_zs(np - 1, 1.0);
    try {
      lens.rayshooterInternal(np, img.data(), short_zs);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    REQUIRE(threw);
  }

  // force_halo: analytic haloes accumulate, particle haloes overwrite
  {
    g::LensHaloNFW nfw(5e13f, 0.5f, 0.45, 6.0f, 1.0f, 0.0f, cosmo);
    g::LensHaloParticles hp(p1.data(), p1.size(), 0.3f, cosmo, norot, false, 0.0);
    const double xcm[2] = {0.01, -0.004};
    double a[2] = {0, 0}, k = 0, gm3[3] = {0, 0, 0}, ph = 0;
    nfw.force_halo(a, &k, gm3, &ph, xcm);
    const double a1 = a[0], k1 = k;
    nfw.force_halo(a, &k, gm3, &ph, xcm);
    REQUIRE(a[0] == 2 * a1 && k == 2 * k1 && k1 > 0);
    hp.force_halo(a, &k, gm3, &ph, xcm);
    const double ap = a[0];
    hp.force_halo(a, &k, gm3, &ph, xcm);
    REQUIRE(a[0] == ap);
    // subtract_point with screening (LensHalo::force_point / force_halo_sym):
    // inside Rmax the screened and the unscreened point mass are both added
    double as[2] = {0, 0}, ks = 0, gs[3] = {0, 0, 0}, phs = 0;
    nfw.force_halo(as, &ks, gs, &phs, xcm, true, 0.5);
    const double r2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
    const double point = (double)5e13f / r2 / 3.141592653589793;  // the float mass member
    REQUIRE(std::fabs(as[0] - (a1 + 1.5 * point * xcm[0])) <= 1e-9 * std::fabs(as[0]) && ks == k1);
  }

  // TreeQuadParticles: one ray at a time equals the batched call
  {
    g::TreeQuadParticles tree(p1.data(), p1.size(), -1, -1, 0.0, 20, 0.1);
    const double rr[4] = {0.003, -0.002, 0.05, 0.01};
    double a[4], k[2], gg[6], ph[2];
    tree.force2D_recur(2, rr, a, k, gg, ph);
    double a1[2], k1, g1[3], ph1;
    tree.force2D_recur(rr + 2, a1, &k1, g1, &ph1);
    REQUIRE(a1[0] == a[2] && a1[1] == a[3] && k1 == k[1] && g1[0] == gg[3]);
  }

  // a field plane: its force through the mirror equals the C ABI's, and the
  // lens gains one plane
  {
    g::LensHaloNFW f1(2e12f, 0.15f, 0.2, 7.0f, 1.0f, 0.0f, cosmo);
    f1.setTheta(5 * arcsec, 1 * arcsec);
    g::LensHaloNFW f2(8e11f, 0.1f, 0.2, 8.0f, 1.0f, 0.0f, cosmo);
    f2.setTheta(-4 * arcsec, 6 * arcsec);
    g::LensHaloRealNSIE f3(3e12f, 0.2, 180.0f, 1e-4f, 0.8f, 0.2f, cosmo);
    f3.setTheta(-8 * arcsec, -3 * arcsec);
    g::LensHalo *members[3] = {&f1, &f2, &f3};
    g::LensPlaneTree plane(0.2f, members, 3, 0.0);
    double xx[2] = {0.004, -0.003}, a[2], k, gg[3], ph;
    plane.force(a, &k, gg, &ph, xx);
    glb_halo *hs[3] = {f1.make_copy(), f2.make_copy(), f3.make_copy()}, *hp = nullptr;
    g::check(glb_halo_field_plane(hs, 3, (double)0.2f, 0.0, 0.0, &hp));
    double a2[2], k2, g2[3], ph2;
    g::check(glb_halo_force(hp, 1, xx, a2, &k2, g2, &ph2));
    glb_halo_destroy(hp);
    REQUIRE(a[0] == a2[0] && a[1] == a2[1] && k == k2 && gg[0] == g2[0] && ph == ph2 && k > 0);
    const int before = lens_copy.getNplanes();
    lens_copy.insertFieldPlane(plane);
    REQUIRE(lens_copy.getNplanes() == before + 1);
    bool threw = false;
    try {
      plane.force(a, &k, gg, &ph, xx);
    } catch (const std::runtime_error &) {
      threw = true;
    }
    REQUIRE(threw);
  }

  // the SPLIT precision through the mirror stays within the deflection bound
  {
    lens.precision = g::Precision::SPLIT;
    std::vector<ref::RAY> r2 = rays;
    lens.rayshooterInternal(np, r2.data());
    for (size_t i = 0; i < np; ++i) {
      const double ax = rays[i].x[0] - rays[i].y[0], ay = rays[i].x[1] - rays[i].y[1];
      const double dx = r2[i].y[0] - rays[i].y[0], dy = r2[i].y[1] - rays[i].y[1];
      REQUIRE(std::hypot(dx, dy) <= 1e-4 * std::hypot(ax, ay) + 1e-300);
    }
  }
  // adaptive kNN smoothing: the static helper on the reference's particle
  // struct writes Size only; the sizes go to the oracle comparison
  {
    std::vector<ref::ParticleType> sp(3000);
    for (auto &q : sp) {
      for (int k = 0; k < 3; ++k) q.x[k] = (float)(0.1 * grand());
      q.Mass = 1.0f;
      q.Size = -1.0f;
      q.type = 7;
    }
    const std::vector<ref::ParticleType> before = sp;
    g::LensHaloParticles::calculate_smoothing(16, sp.data(), sp.size());
    for (size_t i = 0; i < sp.size(); ++i) {
      REQUIRE(sp[i].Size > 0 && sp[i].type == 7 && sp[i].x[2] == before[i].x[2]);
    }
    write(out + "/smooth_in.bin", before.data(), before.size() * sizeof(ref::ParticleType));
    write(out + "/smooth_out.bin", sp.data(), sp.size() * sizeof(ref::ParticleType));
    bool threw = false;
    try {
      g::LensHaloParticles::calculate_smoothing(16, sp.data(), 17);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    REQUIRE(threw);
  }
  std::printf("OK\n");
  return 0;
}
