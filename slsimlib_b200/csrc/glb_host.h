// Host-side objects behind the C ABI (include/glamer_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "glb_internal.h"

struct glb_particle_rec {
  float x[3];
  float Mass;
  float Size;
  int type;
};
static_assert(sizeof(glb_particle_rec) == 24, "ParticleType<float> is 24 bytes");

namespace glb {

// Error status carried through the C ABI.
struct Status {
  int code = 0;
  std::string msg;
  static Status ok() { return Status(); }
  static Status err(int c, const std::string &m) {
    Status s;
    s.code = c;
    s.msg = m;
    return s;
  }
  bool good() const { return code == 0; }
};

// Device memory owned by RAII.
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    return cudaMalloc((void **)&p, count * sizeof(T));
  }
};

// TreeQuadParticles built on the device.
struct Tree {
  TreeDev dev{};
  DBuf<GNode> nodes;
  DBuf<GNodeS> snodes;
  DBuf<float4> parts;
  DBuf<float4> prel;
  DBuf<float4> bigs;
  int nnodes = 0;
  size_t nparticles = 0;
  size_t nbranches = 0;            // including empty children (reference count)
  double theta = 0.1;              // opening angle the tree was built with
  std::vector<double> export_rows; // 16 doubles per branch when requested
  float build_ms = 0;
};

struct TreeParams {
  float mass_fixed = -1, size_fixed = -1;
  double inv_area = 0;
  int bucket = 5;
  double theta = 0.1;
  int periodic = 0;
  double inv_screening = 0;
  double max_range = -1;
};

// Builds a tree from host particle records (ParticleType<float>).
Status build_tree(const glb_particle_rec *host_particles, size_t n, const TreeParams &prm,
                  bool want_export, cudaStream_t stream, std::unique_ptr<Tree> &out);

// TreeQuadHalos (include/quadTreeHalos.h:129-515) built on the host: branch
// arrays in preorder, ready for upload.  xp: 2n halo positions (physical
// Mpc), rmax / mass: the haloes' float members.  Returns false with `err` set
// when the positions span no area ("particles in same place.").
struct HaloTreeHost {
  std::vector<HNode> nodes;
  std::vector<int> bigs;
  double period_x = 0, period_y = 0;
};
bool build_halo_tree(const std::vector<double> &xp, const std::vector<float> &rmax, const std::vector<float> &mass,
                     int bucket, double theta, double max_range, HaloTreeHost &out, std::string &err);

// LensHaloParticles::calculate_smoothing on the device: Size of every record
// of d_p (device, n records) written to d_size (device, n floats) as the
// distance to the (nsmooth+1)-th nearest particle, the particle itself
// counted.  ms_out (nullable): [0] sort and bucket boxes, [1] search, in ms.
Status smooth_particles_device(const glb_particle_rec *d_p, size_t n, int nsmooth, float *d_size,
                               cudaStream_t stream, float *ms_out);

// Global options.
extern int g_keep_tree_export;

}  // namespace glb
