// Drives the C++ mirror's particle files (include/glamer_b200.hpp:
// MakeParticleLenses, LensHaloParticles::writeSizes / readSizesFile) on a csv
// file given on the command line; no GPU needed for csv5 and glmb.
//
//   particle_io_test <csv5 file> <Nsmooth> <recenter 0|1> <output prefix>
// writes <prefix>.bin (records), <prefix>.meta (cm[3], bbox_ll[3],
// bbox_ur[3], z_original, nparticles[6] as doubles) and <prefix>.sizes.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "glamer_b200.hpp"

namespace g = glamer_b200;

int main(int argc, char **argv) {
  if (argc != 5) return 2;
  const std::string prefix = argv[4];
  g::MakeParticleLenses m(argv[1], g::SimFileFormat::csv5, std::atoi(argv[2]), std::atoi(argv[3]) != 0);
  FILE *f = std::fopen((prefix + ".bin").c_str(), "wb");
  std::fwrite(m.data.data(), sizeof(glb_particle), m.data.size(), f);
  std::fclose(f);
  std::array<double, 3> lo, hi, cm = m.getCenterOfMass();
  m.getBoundingBox(lo, hi);
  std::vector<double> meta(cm.begin(), cm.end());
  meta.insert(meta.end(), lo.begin(), lo.end());
  meta.insert(meta.end(), hi.begin(), hi.end());
  meta.push_back(m.getZoriginal());
  for (size_t k : m.getnp()) meta.push_back((double)k);
  const std::array<double, 3> dp = m.densest_particle();
  meta.insert(meta.end(), dp.begin(), dp.end());
  f = std::fopen((prefix + ".meta").c_str(), "wb");
  std::fwrite(meta.data(), sizeof(double), meta.size(), f);
  std::fclose(f);
  g::LensHaloParticles::writeSizes(prefix + ".sizes", 64, m.data.data(), m.data.size());
  std::vector<glb_particle> back(m.data.size());
  if (!g::LensHaloParticles::readSizesFile(prefix + ".sizes", back.data(), back.size(), 64, 0.0)) return 3;
  if (g::LensHaloParticles::readSizesFile(prefix + ".sizes", back.data(), back.size(), 32, 0.0)) return 4;
  // cuts: the records kept after radialCut around the centre of the box
  {
    std::array<double, 3> c = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
    g::MakeParticleLenses m2(argv[1], g::SimFileFormat::csv5, std::atoi(argv[2]), false);
    m2.radialCut(c, 0.25 * (hi[0] - lo[0]));
    f = std::fopen((prefix + ".cut.bin").c_str(), "wb");
    std::fwrite(m2.data.data(), sizeof(glb_particle), m2.data.size(), f);
    std::fclose(f);
    std::vector<double> cm2 = {c[0], c[1], c[2], 0.25 * (hi[0] - lo[0])};
    f = std::fopen((prefix + ".cut.meta").c_str(), "wb");
    std::fwrite(cm2.data(), sizeof(double), cm2.size(), f);
    std::fclose(f);
  }
  std::printf("OK\n");
  return 0;
}
