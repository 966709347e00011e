// Runs the reference's own test scenarios with the GPU update methods of
// nbody-fmm_b200/cpp/gpu_fmm.hpp plugged into the reference's classes
// (Particle, SystemUpdateMethod, SyplecticEuler, NaiveUpdate), compiled
// against the reference's headers and objects.  TEST INFRASTRUCTURE: built
// by oracle/Makefile into _ref/adapter_check, run by tests/test_gpu_adapter.py
// (GPU checks) and tests/test_frames.py (`adapter_check frames <dir>`: the
// frame exporter alone, no GPU).  Exit status 0 = every check passed.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gpu_fmm.hpp"
#include "quadratures/symplectic_euler.hpp"
#include "system_updaters/naive_update.hpp"

static int failures = 0;
#define CHECK(c, ...)                    \
  do {                                   \
    if (!(c)) {                          \
      ++failures;                        \
      std::fprintf(stderr, __VA_ARGS__); \
      std::fprintf(stderr, "\n");        \
    }                                    \
  } while (0)

// tests/test_naive_update.cpp:13-55 with GpuFMM as the update method.
static void two_bodies() {
  std::vector<Particle> ps = {Particle(1.0e9, {-10.0, 0.0, 0.0}, {0.0, 0.0, 0.0}),
                              Particle(1.0e9, {10.0, 0.0, 0.0}, {0.0, 0.0, 0.0})};
  GpuFMM fmm(4, 20, 0);
  SyplecticEuler se;
  double prev = 20.0;
  for (int s = 0; s < 20; ++s) {
    se.integrate(&fmm, ps, 0.5);
    double d = (ps[1].get_position() - ps[0].get_position()).norm();
    CHECK(d < prev, "two bodies: distance did not decrease at step %d", s);
    prev = d;
  }
}

// tests/test_fmm_vs_naive_3d.cpp:17-208 and test_fmm_vs_naive_2d... setting:
// glibc srand(42), positions in [-50,50]^3, mass 1e9.
static std::vector<Particle> make3d(int n) {
  srand(42);
  std::vector<Particle> ps;
  for (int i = 0; i < n; ++i) {
    double x = (rand() * 2.0 * 50.0) / RAND_MAX - 50.0, y = (rand() * 2.0 * 50.0) / RAND_MAX - 50.0,
           z = (rand() * 2.0 * 50.0) / RAND_MAX - 50.0;
    double vx = (rand() * 2.0) / RAND_MAX - 1.0, vy = (rand() * 2.0) / RAND_MAX - 1.0,
           vz = (rand() * 2.0) / RAND_MAX - 1.0;
    ps.push_back(Particle(1.0e9, {x, y, z}, {vx, vy, vz}));
  }
  return ps;
}

static void fmm_vs_naive_3d() {
  std::vector<Particle> a = make3d(100), b = a, c = a;
  NaiveUpdate naive;
  naive.update(a);
  GpuFMM fmm(2, 20, 0);
  fmm.update(b);
  GpuNaiveUpdate gnaive;
  gnaive.update(c);
  double worst = 0, num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i)
    for (int d = 0; d < 3; ++d) {
      worst = std::fmax(worst, std::fabs(b[i].get_acceleration()[d] - a[i].get_acceleration()[d]));
      double e = c[i].get_acceleration()[d] - a[i].get_acceleration()[d];
      num += e * e;
      den += a[i].get_acceleration()[d] * a[i].get_acceleration()[d];
    }
  // the reference's own tolerance (test_fmm_vs_naive_3d.cpp:198-203)
  CHECK(worst < 1e-2, "GpuFMM vs NaiveUpdate: max abs %.3e", worst);
  CHECK(std::sqrt(num / den) < 1e-12, "GpuNaiveUpdate vs NaiveUpdate: rel L2 %.3e", std::sqrt(num / den));
}

// The reference driver's frame loop (main.cpp:85-91) with GpuFrameExporter
// in place of HDF5Exporter: three frames of 3D particles whose velocities
// and accelerations are set; each .bin holds position, velocity,
// acceleration (n x 3) and weight (n) as the particles have them.
static void frames(const char *dir) {
  std::vector<Particle> ps = make3d(50);
  {
    GpuFrameExporter ex(dir, "particles");
    for (int step = 0; step < 3; ++step) {
      for (size_t i = 0; i < ps.size(); ++i) {
        Tensor g(3);
        for (int d = 0; d < 3; ++d) g[d] = 0.01 * (double)(i + d + step);
        ps[i].compute_new_accelaration(g);
      }
      ex.write_frame(ps, step, 0.5 * step);
      const std::string path = std::string(dir) + "/particles_0000" + std::to_string(step) + ".bin";
      std::FILE *fp = std::fopen(path.c_str(), "rb");
      CHECK(fp != nullptr, "frames: %s missing", path.c_str());
      if (!fp) continue;
      const size_t n = ps.size();
      std::vector<double> buf(10 * n);
      CHECK(std::fread(buf.data(), sizeof(double), buf.size(), fp) == buf.size(), "frames: %s short", path.c_str());
      std::fclose(fp);
      for (size_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
          CHECK(buf[3 * i + d] == ps[i].get_position()[d], "frames: position %zu %d", i, d);
          CHECK(buf[3 * n + 3 * i + d] == ps[i].get_velocity()[d], "frames: velocity %zu %d", i, d);
          CHECK(buf[6 * n + 3 * i + d] == ps[i].get_acceleration()[d], "frames: acceleration %zu %d", i, d);
        }
      for (size_t i = 0; i < n; ++i) CHECK(buf[9 * n + i] == ps[i].get_weight(), "frames: weight %zu", i);
    }
  }
}

int main(int argc, char **argv) {
  if (argc == 3 && std::string(argv[1]) == "frames") {
    frames(argv[2]);
    std::fprintf(stderr, "%d failure(s)\n", failures);
    return failures ? 1 : 0;
  }
  two_bodies();
  fmm_vs_naive_3d();
  std::fprintf(stderr, "%d failure(s)\n", failures);
  return failures ? 1 : 0;
}
