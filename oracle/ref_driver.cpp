/*
 * ORACLE -- test infrastructure only.
 *
 * Driver for the reference itself: this file is compiled together with the
 * reference's own sources (left in place; see oracle/Makefile) into
 * oracle/_ref/glamer_ref.  It reads one command per line on stdin, runs the
 * reference code path named by the command and writes raw little-endian
 * float64 arrays.  Used by tests/ to pin the C restatement (oracle.c) and by
 * bench.py's reference arm as the CPU baseline.
 *
 * Commands (files are raw arrays; particles are 24-byte ParticleType<float>):
 *   tree PFILE N BUCKET THETA INV_AREA MAX_RANGE PERIODIC INV_SCREEN RFILE NR OUT [EXPORT]
 *        TreeQuadParticles ctor + force2D_recur at NR rays -> OUT: per ray
 *        alpha[2] kappa gamma[3] phi.  EXPORT: 16 doubles per branch (preorder).
 *   nfw MASS RSIZE Z CONC FRATIO PA XFILE N OUT [SCREEN]   LensHaloNFW::force_halo
 *   nsie MASS Z SIGMA RCORE FRATIO PA XFILE N OUT [SCREEN] LensHaloRealNSIE::force_halo
 *        (SCREEN given: force_halo(..., subtract_point = true, SCREEN))
 *   lens ZSOURCE                                     new Lens (replaces previous)
 *   particles PFILE N Z INV_AREA MAX_RANGE TX TY     moveinMainHalo(LensHaloParticles, true)
 *   addnfw MASS RSIZE Z CONC TX TY                   insertMainHalo(LensHaloNFW, true)
 *   addnsie MASS Z SIGMA RCORE FRATIO PA TX TY       insertMainHalo(LensHaloRealNSIE, true)
 *   haloforce I XFILE N OUT                          force_halo of the lens's i-th main halo
 *   threads OUT                                      Utilities::GetNThreads()
 *   planes OUT                                       z, Dl, dDl of every plane (+ source)
 *   grid N CX CY RANGE OUT TIMEFILE                  GridMap ctor -> per ray y[2] A[4];
 *                                                    TIMEFILE gets the ctor wall seconds
 *   rays XFILE N ZFILE OUT TIMEFILE                  rayshooterInternal(N, RAY*) with per-ray z
 *   points XFILE N OUT TIMEFILE                      rayshooterInternal(N, Point*)
 *   lpoints XFILE N ZFILE OUT                        rayshooterInternal(N, LinkedPoint*, source_zs)
 *   rayshooter XFILE N OUT                           rayshooter(RAY&) per ray
 *   sourcesb KIND A B C D E F G YFILE N OUT
 *        Source::SurfaceBrightness at N source-plane positions -> OUT: N values
 *        and the source's total flux.  KIND 0 SourceUniform(Point_2d(A,B), 1, C);
 *        1 SourceGaussian(Point_2d(A,B), C, 1, -1, 0); 2 SourceSersic(mag C,
 *        Reff D arcsec, PA E, index F, q G, z 1, zeropoint 0) at (A, B).
 *   adaptive N CX CY RANGE KIND A B C D E F G OUT
 *        GridMap ctor + AdaptiveRefreshSurfaceBrightnesses(lens, source) with
 *        the source of sourcesb -> OUT: the returned total flux.
 *   fieldplane HFILE NH Z SIGMA_BACK INV_SCREEN XFILE N OUT
 *        LensPlaneTree(Z, haloes, NH, SIGMA_BACK, INV_SCREEN)::force at N plane
 *        positions -> per position alpha[2] kappa gamma[3] phi.  HFILE: 8
 *        doubles per halo {kind, mass, a, b, c, d, tx, ty}: kind 0 = LensHaloNFW
 *        (a = Rsize, b = concentration), 1 = LensHaloRealNSIE (a = sigma,
 *        b = rcore, c = fratio, d = pa); each halo moved to Z with
 *        setZlensDist, as Lens::createFieldPlanes does.
 *   makeparticles FILE FMT NSMOOTH RECENTER OUT [CUT CX CY CZ RADIUS]
 *        MakeParticleLenses from a glmb file (FMT 0) or a csv file (FMT 3-6,
 *        SimFileFormat::csvFMT; writes FILE_S<NSMOOTH>.glmb beside it), then
 *        radialCut (CUT 1) or cylindricalCut (CUT 2) -> OUT: the particle
 *        records; OUT.meta: {1, cm[3], bbox_ll[3], bbox_ur[3], z_original,
 *        nparticles[6], densest_particle[3]}, or {0} when the constructor throws.
 *   particlefile FILE Z NSMOOTH MULTIMASS INV_AREA MINPSIZE MASSSCALING RECENTER TX TY XFILE N OUT
 *        LensHaloParticles from an ascii position file (reads or writes
 *        FILE.<NSMOOTH>sizes) -> force_halo at N physical positions.
 *   writesizes PFILE N NSMOOTH OUT     LensHaloParticles::writeSizes
 *   readsizes FILE N NSMOOTH MIN_SIZE OUT
 *        LensHaloParticles::readSizesFile -> OUT: {found, sizes[N]}, or {-1}
 *        when it throws.
 *   smooth PFILE N NSMOOTH OUT TIMEFILE
 *        LensHaloParticles<ParticleType<float>>::calculate_smoothing -> OUT: the
 *        N particle sizes; TIMEFILE gets the wall seconds.
 * Refinement clients of rayshooterInternal (the reference's own code, run
 * through whichever rayshooter the binary was linked with):
 *   findcritmap N CX CY RANGE OUT
 *        GridMap ctor + ImageFinding::find_crit(lens, gridmap, curves)
 *        (TreeCode_link/find_crit.cpp:1036-1090) -> OUT: curves (see dump_curves).
 *   magcontour N CX CY RANGE INVMAG OUT
 *        GridMap ctor + ImageFinding::find_magnification_contour -> OUT:
 *        {ncontours, per contour: n, hits_boundary, per point x[2] y[2] A[4]}.
 *   gridrefine N CX CY RANGE STRIDE OUT
 *        Grid ctor, then Grid::RefineLeaves on every STRIDE-th image point
 *        (TreeCode_link/grid_maintenance.cpp:543-600) -> OUT: {npoints, per
 *        point (point-list order) x[2] image->x[2] A[4]}.
 *   gridcrit N CX CY RANGE RES OUT
 *        Grid ctor + ImageFinding::find_crit(lens, grid, curves, &n, RES)
 *        (kist refinement rounds, TreeCode_link/find_crit.cpp:37-) -> OUT: curves.
 *   dropin PREC   the GPU drop-in's precision (binaries linked with it only)
 *   uniform N CX CY RANGE MCX MCY NX NY VAR OUT
 *        GridMap ctor + writePixelMapUniform<double>({MCX, MCY}, NX, NY,
 *        LensingVariable VAR) (include/gridmap.h:506-690) -> OUT: NX*NY values.
 */
#include "slsimlib.h"
#include "particle_halo.h"
#include "sersic_source.h"
#include "gridmap.h"
#include "grid_maintenance.h"
#include "oracle.h"
#ifdef GLAMER_B200_DROPIN
#include "glamer_b200_dropin.hpp"
#endif

#include <chrono>
#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

/* The flat LambdaCDM distances of the oracle, shared with the restatement. */
double COSMOLOGY::coorDist(double z) const { return orc_coordist(z); }
double COSMOLOGY::invCoorDist(double d) const { return orc_invcoordist(d); }

typedef ParticleType<float> PT;

template <typename T>
static std::vector<T> read_arr(const std::string &f, size_t n) {
  std::vector<T> v(n);
  if (n == 0) return v;
  FILE *fp = fopen(f.c_str(), "rb");
  if (!fp || fread(v.data(), sizeof(T), n, fp) != n) {
    fprintf(stderr, "glamer_ref: cannot read %s\n", f.c_str());
    exit(2);
  }
  fclose(fp);
  return v;
}
static void write_arr(const std::string &f, const std::vector<double> &v) {
  FILE *fp = fopen(f.c_str(), "wb");
  if (!fp) { fprintf(stderr, "glamer_ref: cannot write %s\n", f.c_str()); exit(2); }
  fwrite(v.data(), sizeof(double), v.size(), fp);
  fclose(fp);
}
static void write_time(const std::string &f, double s) {
  if (f == "-") return;
  write_arr(f, std::vector<double>(1, s));
}

/* Exposes the protected tree for the branch export. */
struct ExportTree : public TreeQuadParticles<PT> {
  using TreeQuadParticles<PT>::TreeQuadParticles;
  void export_branches(std::vector<double> &out) {
    out.clear();
    QBranchNB *b = tree->top;
    while (b) {
      bool leaf = !b->child0 && !b->child1 && !b->child2 && !b->child3;
      double w = b->boundary_p2[0] - b->boundary_p1[0];
      double v[16] = {(double)b->level, b->boundary_p1[0], b->boundary_p1[1], b->boundary_p2[0],
                      b->boundary_p2[1], (double)b->nparticles, (double)b->Nbig_particles, b->mass,
                      b->center[0], b->center[1], b->quad[0], b->quad[1], b->quad[2],
                      b->r2crit_angle, (double)leaf, w * w};
      out.insert(out.end(), v, v + 16);
      b = b->child0 ? b->child0 : b->brother;
    }
  }
};

/* The LensHaloRealNSIE constructor resets the mass of a cored halo by 1D
 * integration (MultiPlane/lens_halos.cpp:1073-1075) before it assigns `units`
 * (:1077), so that integral reads an indeterminate value.  Repeat the
 * integration once `units` is set, which is the mass the constructor intends. */
static void fix_cored_nsie_mass(LensHaloRealNSIE &h, float nominal_mass) {
  if (h.get_rcore() > 0.0) {
    h.setMass(nominal_mass);
    h.setMass(h.MassBy1DIntegation(h.getRsize()));
  }
}

/* {ncurves, per curve: type, touches_edge, npoints, critical_area,
 * critical_center[2], caustic_area, caustic_center[2], then per point of
 * critcurve x[2] y[2] A[4]} */
static void dump_curves(const std::string &out, const std::vector<ImageFinding::CriticalCurve> &c) {
  std::vector<double> o{(double)c.size()};
  for (const auto &k : c) {
    double h[9] = {(double)(int)k.type, (double)k.touches_edge, (double)k.critcurve.size(), k.critical_area,
                   k.critical_center[0], k.critical_center[1], k.caustic_area, k.caustic_center[0],
                   k.caustic_center[1]};
    o.insert(o.end(), h, h + 9);
    for (const RAY &r : k.critcurve) {
      double v[8] = {r.x[0], r.x[1], r.y[0], r.y[1], r.A.a[0], r.A.a[1], r.A.a[2], r.A.a[3]};
      o.insert(o.end(), v, v + 8);
    }
  }
  write_arr(out, o);
}

int main() {
  COSMOLOGY cosmo;
  long seed = 1;
  std::unique_ptr<Lens> lens;
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream in(line);
    std::string cmd;
    if (!(in >> cmd)) continue;
    if (cmd == "tree") {
      std::string pf, rf, out, exp;
      size_t n, nr;
      int bucket, periodic;
      double theta, inv_area, max_range, inv_screen;
      in >> pf >> n >> bucket >> theta >> inv_area >> max_range >> periodic >> inv_screen >> rf >> nr >> out >> exp;
      std::vector<PT> p = read_arr<PT>(pf, n);
      std::vector<double> r = read_arr<double>(rf, 2 * nr);
      ExportTree t(p.data(), n, -1, -1, inv_area, bucket, theta, periodic != 0, inv_screen, max_range);
      std::vector<double> o(7 * nr);
      for (size_t i = 0; i < nr; ++i) {
        double a[2], k, g[3], ph;
        t.force2D_recur(&r[2 * i], a, &k, g, &ph);
        double v[7] = {a[0], a[1], k, g[0], g[1], g[2], ph};
        std::copy(v, v + 7, &o[7 * i]);
      }
      write_arr(out, o);
      if (!exp.empty()) {
        std::vector<double> e;
        t.export_branches(e);
        write_arr(exp, e);
      }
    } else if (cmd == "nfw" || cmd == "nsie") {
      std::unique_ptr<LensHalo> h;
      std::string xf, out;
      size_t n;
      if (cmd == "nfw") {
        float mass, rsize, conc, fratio, pa;
        double z;
        in >> mass >> rsize >> z >> conc >> fratio >> pa >> xf >> n >> out;
        h.reset(new LensHaloNFW(mass, rsize, z, conc, fratio, pa, cosmo));
      } else {
        float mass, sigma, rcore, fratio, pa;
        double z;
        in >> mass >> z >> sigma >> rcore >> fratio >> pa >> xf >> n >> out;
        LensHaloRealNSIE *nh = new LensHaloRealNSIE(mass, z, sigma, rcore, fratio, pa, cosmo);
        fix_cored_nsie_mass(*nh, mass);
        h.reset(nh);
      }
      double screen = 1.0;
      const bool sub = static_cast<bool>(in >> screen);
      std::vector<double> x = read_arr<double>(xf, 2 * n), o(7 * n + 3);
      for (size_t i = 0; i < n; ++i) {
        double a[2] = {0, 0}, k = 0, g[3] = {0, 0, 0}, ph = 0;
        if (sub) h->force_halo(a, &k, g, &ph, &x[2 * i], true, screen);
        else h->force_halo(a, &k, g, &ph, &x[2 * i]);
        double v[7] = {a[0], a[1], k, g[0], g[1], g[2], ph};
        std::copy(v, v + 7, &o[7 * i]);
      }
      o[7 * n] = h->get_mass();
      o[7 * n + 1] = h->getRsize();
      o[7 * n + 2] = h->get_Rmax();
      write_arr(out, o);
    } else if (cmd == "lens") {
      double zs;
      in >> zs;
      lens.reset(new Lens(&seed, zs, cosmo));
    } else if (cmd == "particles") {
      std::string pf;
      size_t n;
      double z, inv_area, max_range, tx, ty;
      in >> pf >> n >> z >> inv_area >> max_range >> tx >> ty;
      std::vector<PT> p = read_arr<PT>(pf, n);
      LensHaloParticles<PT> h(p, (float)z, cosmo, Point_2d(0, 0), false, inv_area, 0, max_range);
      h.setTheta(tx, ty);
      lens->moveinMainHalo(h, true);
    } else if (cmd == "addnfw") {
      float mass, rsize, conc;
      double z, tx, ty;
      in >> mass >> rsize >> z >> conc >> tx >> ty;
      LensHaloNFW h(mass, rsize, z, conc, 1.0f, 0.0f, cosmo);
      h.setTheta(tx, ty);
      lens->insertMainHalo(h, true);
    } else if (cmd == "addnsie") {
      float mass, sigma, rcore, fratio, pa;
      double z, tx, ty;
      in >> mass >> z >> sigma >> rcore >> fratio >> pa >> tx >> ty;
      LensHaloRealNSIE h(mass, z, sigma, rcore, fratio, pa, cosmo);
      fix_cored_nsie_mass(h, mass);
      h.setTheta(tx, ty);
      lens->insertMainHalo(h, true);
    } else if (cmd == "haloforce") {
      /* force_halo of the lens's i-th main halo at physical positions */
      std::string xf, out;
      size_t i, n;
      in >> i >> xf >> n >> out;
      std::vector<double> x = read_arr<double>(xf, 2 * n), o(7 * n);
      LensHalo *h = lens->getMainHalo(i);
      for (size_t k = 0; k < n; ++k) {
        double a[2] = {0, 0}, kk = 0, g[3] = {0, 0, 0}, ph = 0;
        h->force_halo(a, &kk, g, &ph, &x[2 * k]);
        double v[7] = {a[0], a[1], kk, g[0], g[1], g[2], ph};
        std::copy(v, v + 7, &o[7 * k]);
      }
      write_arr(out, o);
    } else if (cmd == "threads") {
      /* the thread count Lens::rayshooterInternal uses (utilities.cpp:553) */
      std::string out;
      in >> out;
      write_arr(out, std::vector<double>(1, (double)Utilities::GetNThreads()));
    } else if (cmd == "planes") {
      std::string out;
      in >> out;
      std::vector<double> o;
      /* z, Dl and dDl are protected; rebuild them from the public accessors */
      int np = lens->getNplanes();
      std::vector<PosType> zz = lens->get_plane_redshifts();
      o.push_back(np);
      for (auto z : zz) o.push_back(z);
      write_arr(out, o);
    } else if (cmd == "grid") {
      size_t N;
      double c[2], range;
      std::string out, tf;
      in >> N >> c[0] >> c[1] >> range >> out >> tf;
      auto t0 = std::chrono::steady_clock::now();
      GridMap gm(lens.get(), N, c, range);
      double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      std::vector<double> o(6 * N * N);
      for (size_t i = 0; i < N * N; ++i) {
        RAY r = gm.ray(i);
        double v[6] = {r.y[0], r.y[1], r.A.a[0], r.A.a[1], r.A.a[2], r.A.a[3]};
        std::copy(v, v + 6, &o[6 * i]);
      }
      write_arr(out, o);
      write_time(tf, secs);
    } else if (cmd == "rays" || cmd == "points") {
      std::string xf, zf, out, tf;
      size_t n;
      if (cmd == "rays") in >> xf >> n >> zf >> out >> tf;
      else in >> xf >> n >> out >> tf;
      std::vector<double> x = read_arr<double>(xf, 2 * n), o(6 * n);
      double secs;
      if (cmd == "rays") {
        std::vector<double> z = read_arr<double>(zf, n);
        std::vector<RAY> rays(n);
        for (size_t i = 0; i < n; ++i) { rays[i].x[0] = x[2 * i]; rays[i].x[1] = x[2 * i + 1]; rays[i].z = z[i]; }
        auto t0 = std::chrono::steady_clock::now();
        lens->rayshooterInternal(n, rays.data());
        secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (size_t i = 0; i < n; ++i) {
          double v[6] = {rays[i].y[0], rays[i].y[1], rays[i].A.a[0], rays[i].A.a[1], rays[i].A.a[2], rays[i].A.a[3]};
          std::copy(v, v + 6, &o[6 * i]);
        }
      } else {
        std::vector<Point> ip(n), sp(n);
        for (size_t i = 0; i < n; ++i) {
          ip[i].x[0] = x[2 * i]; ip[i].x[1] = x[2 * i + 1];
          ip[i].image = &sp[i]; sp[i].image = &ip[i];
        }
        auto t0 = std::chrono::steady_clock::now();
        lens->rayshooterInternal(n, ip.data());
        secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (size_t i = 0; i < n; ++i) {
          double v[6] = {sp[i].x[0], sp[i].x[1], ip[i].A.a[0], ip[i].A.a[1], ip[i].A.a[2], ip[i].A.a[3]};
          std::copy(v, v + 6, &o[6 * i]);
        }
      }
      write_arr(out, o);
      write_time(tf, secs);
    } else if (cmd == "lpoints" || cmd == "rayshooter") {
      std::string xf, zf, out;
      size_t n;
      in >> xf >> n;
      if (cmd == "lpoints") in >> zf;
      in >> out;
      std::vector<double> x = read_arr<double>(xf, 2 * n), o(6 * n);
      if (cmd == "lpoints") {
        std::vector<double> z = read_arr<double>(zf, n);
        std::vector<LinkedPoint> p(n);
        for (size_t i = 0; i < n; ++i) { p[i].x[0] = x[2 * i]; p[i].x[1] = x[2 * i + 1]; }
        lens->rayshooterInternal(n, p.data(), z);
        for (size_t i = 0; i < n; ++i) {
          double v[6] = {p[i].image->x[0], p[i].image->x[1], p[i].A.a[0], p[i].A.a[1], p[i].A.a[2], p[i].A.a[3]};
          std::copy(v, v + 6, &o[6 * i]);
        }
      } else {
        for (size_t i = 0; i < n; ++i) {
          RAY r;
          r.x[0] = x[2 * i];
          r.x[1] = x[2 * i + 1];
          lens->rayshooter(r);
          double v[6] = {r.y[0], r.y[1], r.A.a[0], r.A.a[1], r.A.a[2], r.A.a[3]};
          std::copy(v, v + 6, &o[6 * i]);
        }
      }
      write_arr(out, o);
    } else if (cmd == "sourcesb") {
      int kind;
      double p[7];
      std::string yf, out;
      size_t n;
      in >> kind >> p[0] >> p[1] >> p[2] >> p[3] >> p[4] >> p[5] >> p[6] >> yf >> n >> out;
      std::unique_ptr<Source> src;
      if (kind == 0) {
        src.reset(new SourceUniform(Point_2d(p[0], p[1]), 1.0, p[2]));
      } else if (kind == 1) {
        src.reset(new SourceGaussian(Point_2d(p[0], p[1]), p[2], 1.0, -1, 0));
      } else {
        SourceSersic *ss = new SourceSersic(p[2], p[3], p[4], p[5], p[6], 1.0, 0.0, Band::NoBand);
        ss->setTheta(p[0], p[1]);
        src.reset(ss);
      }
      std::vector<double> y = read_arr<double>(yf, 2 * n), o(n + 1);
      for (size_t i = 0; i < n; ++i) o[i] = src->SurfaceBrightness(&y[2 * i]);
      o[n] = src->getTotalFlux();
      write_arr(out, o);
    } else if (cmd == "adaptive") {
      size_t N;
      double c[2], range, p[7];
      int kind;
      std::string out;
      in >> N >> c[0] >> c[1] >> range >> kind >> p[0] >> p[1] >> p[2] >> p[3] >> p[4] >> p[5] >> p[6] >> out;
      std::unique_ptr<Source> src;
      if (kind == 0) {
        src.reset(new SourceUniform(Point_2d(p[0], p[1]), 1.0, p[2]));
      } else if (kind == 1) {
        src.reset(new SourceGaussian(Point_2d(p[0], p[1]), p[2], 1.0, -1, 0));
      } else {
        SourceSersic *ss = new SourceSersic(p[2], p[3], p[4], p[5], p[6], 1.0, 0.0, Band::NoBand);
        ss->setTheta(p[0], p[1]);
        src.reset(ss);
      }
      GridMap gm(lens.get(), N, c, range);
      double total = gm.AdaptiveRefreshSurfaceBrightnesses(*lens, *src);
      write_arr(out, std::vector<double>(1, total));
    } else if (cmd == "fieldplane") {
      std::string hf, xf, out;
      size_t nh, n;
      double z, sb, iscr;
      in >> hf >> nh >> z >> sb >> iscr >> xf >> n >> out;
      std::vector<double> hd = read_arr<double>(hf, 8 * nh);
      std::vector<std::unique_ptr<LensHalo>> hs;
      std::vector<LensHalo *> hp;
      for (size_t i = 0; i < nh; ++i) {
        const double *d = &hd[8 * i];
        LensHalo *h;
        if (d[0] == 0) {
          h = new LensHaloNFW((float)d[1], (float)d[2], z, (float)d[3], 1.0f, 0.0f, cosmo);
        } else {
          LensHaloRealNSIE *nh2 = new LensHaloRealNSIE((float)d[1], z, (float)d[2], (float)d[3], (float)d[4],
                                                       (float)d[5], cosmo);
          fix_cored_nsie_mass(*nh2, (float)d[1]);
          h = nh2;
        }
        h->setTheta(d[6], d[7]);
        h->setZlensDist(z, cosmo);
        hs.emplace_back(h);
        hp.push_back(h);
      }
      LensPlaneTree plane((float)z, hp.data(), nh, sb, iscr);
      std::vector<double> x = read_arr<double>(xf, 2 * n), o(7 * n);
      for (size_t k = 0; k < n; ++k) {
        double a[2] = {0, 0}, kk = 0, g[3] = {0, 0, 0}, ph = 0;
        plane.force(a, &kk, g, &ph, &x[2 * k]);
        double v[7] = {a[0], a[1], kk, g[0], g[1], g[2], ph};
        std::copy(v, v + 7, &o[7 * k]);
      }
      write_arr(out, o);
    } else if (cmd == "findcritmap" || cmd == "magcontour") {
      size_t N;
      double c[2], range, invmag = 0;
      std::string out;
      in >> N >> c[0] >> c[1] >> range;
      if (cmd == "magcontour") in >> invmag;
      in >> out;
      GridMap gm(lens.get(), N, c, range);
      if (cmd == "findcritmap") {
        std::vector<ImageFinding::CriticalCurve> crits;
        ImageFinding::find_crit(*lens, gm, crits);
        dump_curves(out, crits);
      } else {
        std::vector<std::vector<RAY>> contour;
        std::vector<bool> hits;
        ImageFinding::find_magnification_contour(*lens, gm, invmag, contour, hits);
        std::vector<double> o{(double)contour.size()};
        for (size_t i = 0; i < contour.size(); ++i) {
          o.push_back((double)contour[i].size());
          o.push_back((double)hits[i]);
          for (const RAY &r : contour[i]) {
            double v[8] = {r.x[0], r.x[1], r.y[0], r.y[1], r.A.a[0], r.A.a[1], r.A.a[2], r.A.a[3]};
            o.insert(o.end(), v, v + 8);
          }
        }
        write_arr(out, o);
      }
    } else if (cmd == "gridrefine" || cmd == "gridcrit") {
      size_t N;
      double c[2], range, arg;
      std::string out;
      in >> N >> c[0] >> c[1] >> range >> arg >> out;
      Grid grid(lens.get(), N, c, range);
      if (cmd == "gridrefine") {
        std::vector<Point *> pts;
        PointList::iterator it;
        it.current = grid.i_tree->pointlist.Top();
        const size_t stride = (size_t)arg;
        for (size_t i = 0; i < grid.i_tree->pointlist.size(); ++i, --it)
          if (i % stride == 0) pts.push_back(*it);
        grid.RefineLeaves(lens.get(), pts);
        std::vector<double> o{(double)grid.i_tree->pointlist.size()};
        it.current = grid.i_tree->pointlist.Top();
        for (size_t i = 0; i < grid.i_tree->pointlist.size(); ++i, --it) {
          const Point *p = *it;
          double v[8] = {p->x[0], p->x[1], p->image->x[0], p->image->x[1], p->A.a[0], p->A.a[1], p->A.a[2],
                         p->A.a[3]};
          o.insert(o.end(), v, v + 8);
        }
        write_arr(out, o);
      } else {
        std::vector<ImageFinding::CriticalCurve> crits;
        int ncrit = 0;
        ImageFinding::find_crit(lens.get(), &grid, crits, &ncrit, arg, 0.0, false);
        crits.resize(ncrit);
        dump_curves(out, crits);
      }
    } else if (cmd == "uniform") {
      size_t N, nx, ny;
      double c[2], mc[2], range;
      int var;
      std::string out;
      in >> N >> c[0] >> c[1] >> range >> mc[0] >> mc[1] >> nx >> ny >> var >> out;
      GridMap gm(lens.get(), N, c, range);
      PixelMap<double> map = gm.writePixelMapUniform<double>(mc, nx, ny, (LensingVariable)var);
      std::vector<double> o(nx * ny);
      for (size_t i = 0; i < nx * ny; ++i) o[i] = map[i];
      write_arr(out, o);
    } else if (cmd == "dropin") {
      int prec;
      in >> prec;
#ifdef GLAMER_B200_DROPIN
      glamer_b200_dropin::set_precision(prec);
#else
      (void)prec;
#endif
    } else if (cmd == "smooth") {
      std::string pf, out, tf;
      size_t n;
      int nsmooth;
      in >> pf >> n >> nsmooth >> out >> tf;
      std::vector<PT> p = read_arr<PT>(pf, n);
      auto t0 = std::chrono::steady_clock::now();
      LensHaloParticles<PT>::calculate_smoothing(nsmooth, p.data(), n);
      auto t1 = std::chrono::steady_clock::now();
      std::vector<double> o(n);
      for (size_t i = 0; i < n; ++i) o[i] = p[i].Size;
      write_arr(out, o);
      write_time(tf, std::chrono::duration<double>(t1 - t0).count());
    } else if (cmd == "makeparticles") {
      std::string file, out;
      int fmt, nsmooth, recenter, cut = 0;
      double ccx = 0, ccy = 0, ccz = 0, crad = 0;
      in >> file >> fmt >> nsmooth >> recenter >> out;
      in >> cut >> ccx >> ccy >> ccz >> crad;
      const SimFileFormat f = fmt == 0 ? SimFileFormat::glmb
                              : fmt == 3 ? SimFileFormat::csv3
                              : fmt == 4 ? SimFileFormat::csv4
                              : fmt == 5 ? SimFileFormat::csv5 : SimFileFormat::csv6;
      std::vector<double> meta;
      try {
        std::unique_ptr<MakeParticleLenses> m(fmt == 0 ? new MakeParticleLenses(file, recenter != 0)
                                                       : new MakeParticleLenses(file, f, nsmooth, recenter != 0));
        if (cut == 1) m->radialCut(Point_3d<>(ccx, ccy, ccz), crad);
        if (cut == 2) m->cylindricalCut(Point_2d(ccx, ccy), crad);
        FILE *fp = fopen(out.c_str(), "wb");
        fwrite(m->data.data(), sizeof(PT), m->data.size(), fp);
        fclose(fp);
        Point_3d<> cm = m->getCenterOfMass(), lo, hi;
        m->getBoundingBox(lo, hi);
        meta = {1.0, cm[0], cm[1], cm[2], lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], m->getZoriginal()};
        for (size_t k : m->getnp()) meta.push_back((double)k);
        Point_3d<> dp = m->densest_particle();
        meta.push_back(dp[0]);
        meta.push_back(dp[1]);
        meta.push_back(dp[2]);
      } catch (const std::exception &e) {
        meta = {0.0};
      }
      write_arr(out + ".meta", meta);
    } else if (cmd == "particlefile") {
      /* LensHaloParticles(file, ascii, z, Nsmooth, cosmo, (tx, ty), recenter,
       * multimass, inv_area, MinPSize, massscaling) -> force_halo at N
       * physical positions (7 doubles each) */
      std::string file, xf, out;
      double z, inv_area, minp, mscale, tx, ty;
      int nsmooth, multimass, recenter;
      size_t n;
      in >> file >> z >> nsmooth >> multimass >> inv_area >> minp >> mscale >> recenter >> tx >> ty >> xf >> n >> out;
      Point_2d rot(tx, ty);
      LensHaloParticles<PT> h(file, SimFileFormat::ascii, z, nsmooth, cosmo, rot, recenter != 0, multimass != 0,
                              inv_area, minp, mscale, false);
      std::vector<double> x = read_arr<double>(xf, 2 * n), o(7 * n);
      for (size_t k = 0; k < n; ++k) {
        double a[2] = {0, 0}, kk = 0, g[3] = {0, 0, 0}, ph = 0;
        h.force_halo(a, &kk, g, &ph, &x[2 * k]);
        double v[7] = {a[0], a[1], kk, g[0], g[1], g[2], ph};
        std::copy(v, v + 7, &o[7 * k]);
      }
      write_arr(out, o);
    } else if (cmd == "writesizes") {
      std::string pf, out;
      size_t n;
      int nsmooth;
      in >> pf >> n >> nsmooth >> out;
      std::vector<PT> p = read_arr<PT>(pf, n);
      LensHaloParticles<PT>::writeSizes(out, nsmooth, p.data(), n);
    } else if (cmd == "readsizes") {
      std::string file, out;
      size_t n;
      int nsmooth;
      double min_size;
      in >> file >> n >> nsmooth >> min_size >> out;
      std::vector<PT> p(n);
      std::vector<double> o;
      try {
        const bool ok = LensHaloParticles<PT>::readSizesFile(file, p.data(), n, nsmooth, min_size);
        o.push_back(ok ? 1.0 : 0.0);
        for (auto &q : p) o.push_back(q.Size);
      } catch (const std::exception &e) {
        o = {-1.0};
      }
      write_arr(out, o);
    } else {
      fprintf(stderr, "glamer_ref: unknown command %s\n", cmd.c_str());
      return 2;
    }
    printf("ok\n");
    fflush(stdout);
  }
  return 0;
}
