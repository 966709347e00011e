// Drop-in update methods for rezucch1/nbody-FMM backed by libfmmgpu.so.
//
// Include this header in the reference's own build (its src/ directory on
// the include path) and link libfmmgpu.so:
//
//   GpuFMM            replaces FMM           (src/system_updaters/FMM.cpp:9-12)
//   GpuNaiveUpdate    replaces NaiveUpdate   (src/system_updaters/naive_update.cpp:9-35)
//   GpuFrameExporter  replaces HDF5Exporter  (src/io/hdf5_exporter.cpp:10-128)
//
// Both derive from the reference's SystemUpdateMethod
// (system_update_method.hpp:24-31), so QuadratureMethod::integrate and the
// existing integrators call them unchanged.  The force pass runs with G = 1
// and each particle then receives its gradient through
// Particle::compute_new_accelaration (particle.cpp:16-21), which applies the
// reference's GRAV_CONST exactly as FMM::update does.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "fmm_gpu.h"
#include "particle.hpp"
#include "system_updaters/system_update_method.hpp"

namespace fmm_b200 {

inline void check(int rc, const char *what) {
  if (rc != FMM_OK) throw std::runtime_error(std::string(what) + ": " + fmm_strerror(rc));
}

// Packs the particles into row-major position and mass arrays.
inline int pack(const std::vector<Particle> &ps, std::vector<double> &pos, std::vector<double> &mass) {
  const int dim = ps.empty() ? 3 : (int)ps.front().get_position().dim;
  pos.resize(ps.size() * dim);
  mass.resize(ps.size());
  for (size_t i = 0; i < ps.size(); ++i) {
    const Tensor &x = ps[i].get_position();
    for (int d = 0; d < dim; ++d) pos[i * dim + d] = x[d];
    mass[i] = ps[i].get_weight();
  }
  return dim;
}

// Hands each particle its gradient, as Leaf::compute_acceleration does
// (leaf.cpp:206): acceleration = GRAV_CONST * grad.
inline void deliver(const std::vector<Particle> &ps, const std::vector<double> &grad, int dim) {
  for (size_t i = 0; i < ps.size(); ++i) {
    Tensor g(dim);
    for (int d = 0; d < dim; ++d) g[d] = grad[i * dim + d];
    ps[i].compute_new_accelaration(g);
  }
}

// One GPU context per dimension, created on first use.
class ContextCache {
 public:
  explicit ContextCache(fmm_config base) : base_(base) {}
  ~ContextCache() {
    for (auto *c : ctx_)
      if (c) fmm_destroy(c);
  }
  ContextCache(const ContextCache &) = delete;
  ContextCache &operator=(const ContextCache &) = delete;
  fmm_ctx *get(int dim) {
    fmm_ctx *&c = ctx_[dim == 2 ? 0 : 1];
    if (!c) {
      fmm_config cfg = base_;
      cfg.dim = dim;
      cfg.G = 1.0;
      check(fmm_create(&cfg, &c), "fmm_create");
    }
    return c;
  }

 private:
  fmm_config base_;
  fmm_ctx *ctx_[2] = {nullptr, nullptr};
};

inline fmm_config default_config(int p, int leaf_cap) {
  fmm_config c;
  fmm_config_default(&c);
  c.p = p;
  c.leaf_cap = leaf_cap;
  return c;
}

}  // namespace fmm_b200

// FMM force pass on the GPU.  p and leaf_cap default to the reference's
// hard-coded L = 2 (tree.cpp:94) and threshold = 20 (tree.cpp:32);
// direct_max = 0 evaluates every interaction-list pair by M2L as the
// reference does (-1 lets the library sum small pairs directly).
class GpuFMM : public SystemUpdateMethod {
 public:
  explicit GpuFMM(int p = 2, int leaf_cap = 20, int direct_max = 0) : cache_(cfg(p, leaf_cap, direct_max)) {}
  void update(const std::vector<Particle> &particles) override {
    if (particles.empty()) return;
    const int dim = fmm_b200::pack(particles, pos_, mass_);
    grad_.assign(particles.size() * dim, 0.0);
    fmm_b200::check(fmm_evaluate(cache_.get(dim), (int64_t)particles.size(), pos_.data(), mass_.data(),
                                 grad_.data(), nullptr),
                    "fmm_evaluate");
    fmm_b200::deliver(particles, grad_, dim);
  }

 private:
  static fmm_config cfg(int p, int leaf_cap, int direct_max) {
    fmm_config c = fmm_b200::default_config(p, leaf_cap);
    c.direct_max = direct_max;
    return c;
  }
  fmm_b200::ContextCache cache_;
  std::vector<double> pos_, mass_, grad_;
};

// FP64 O(N^2) direct sum on the GPU with NaiveUpdate's softening.
class GpuNaiveUpdate : public SystemUpdateMethod {
 public:
  GpuNaiveUpdate() : cache_(fmm_b200::default_config(2, 20)) {}
  void update(const std::vector<Particle> &particles) override {
    if (particles.empty()) return;
    const int dim = fmm_b200::pack(particles, pos_, mass_);
    grad_.assign(particles.size() * dim, 0.0);
    fmm_b200::check(fmm_direct(cache_.get(dim), (int64_t)particles.size(), pos_.data(), mass_.data(), 0, nullptr,
                               FMM_SOFT_NAIVE_REF, grad_.data(), nullptr),
                    "fmm_direct");
    fmm_b200::deliver(particles, grad_, dim);
  }

 private:
  fmm_b200::ContextCache cache_;
  std::vector<double> pos_, mass_, grad_;
};

// Frame output with HDF5Exporter's interface (hdf5_exporter.hpp:20-49): the
// same datasets per step and the same XDMF time series, the datasets stored
// as raw FP64 in one .bin per step (fmm_frames_*: no libhdf5).  The writer
// opens at the first frame, which fixes the dimension.
class GpuFrameExporter {
 public:
  explicit GpuFrameExporter(const std::string &dir = "output", const std::string &base = "particles")
      : dir_(dir), base_(base) {}
  GpuFrameExporter(const GpuFrameExporter &) = delete;
  GpuFrameExporter &operator=(const GpuFrameExporter &) = delete;
  ~GpuFrameExporter() {
    if (f_) fmm_frames_close(f_);
  }
  void write_frame(const std::vector<Particle> &particles, int step, double time) {
    if (particles.empty()) return;  // hdf5_exporter.cpp:22
    const int dim = fmm_b200::pack(particles, pos_, mass_);
    if (!f_) fmm_b200::check(fmm_frames_open(dir_.c_str(), base_.c_str(), dim, &f_), "fmm_frames_open");
    vel_.resize(pos_.size());
    acc_.resize(pos_.size());
    for (size_t i = 0; i < particles.size(); ++i) {
      const Tensor &v = particles[i].get_velocity(), &a = particles[i].get_acceleration();
      for (int d = 0; d < dim; ++d) {
        vel_[i * dim + d] = v[d];
        acc_[i * dim + d] = a[d];
      }
    }
    fmm_b200::check(fmm_frames_write(f_, (int64_t)particles.size(), pos_.data(), vel_.data(), acc_.data(),
                                     mass_.data(), step, time),
                    "fmm_frames_write");
  }

 private:
  std::string dir_, base_;
  fmm_frames *f_ = nullptr;
  std::vector<double> pos_, vel_, acc_, mass_;
};
