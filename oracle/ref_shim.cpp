// extern "C" shim over the reference implementation (rezucch1/nbody-FMM),
// compiled against the reference's own headers and sources by oracle/Makefile
// into oracle/_ref/libref.so.  TEST INFRASTRUCTURE ONLY: it is the checker
// that pins the CPU restatement (oracle/fmm_oracle.c) and the CPU baseline arm
// of bench.py; nothing in the product loads it.
//
// Each entry point drives the reference's public classes exactly as its
// callers do:
//   ref_fmm          FMM::update                    src/system_updaters/FMM.cpp:9-12
//   ref_naive        NaiveUpdate::update            src/system_updaters/naive_update.cpp:9-35
//   ref_se_steps     SyplecticEuler::integrate      src/quadratures/symplectic_euler.cpp:8-15
//   ref_tree_*       Tree::init_tree leaf membership and interaction lists
//                                                   tree_components/tree.cpp:15-91, node_i.cpp:23-99
//   ref_p2m_3d       Leaf::compute_multipoles (P2M) leaf.cpp:15-35, multipole_set3D.cpp:31-43
//   ref_regular_3d   PowerSet<3>                    power_set3D.cpp:10-48
//   ref_irregular_3d Irregular                      irregular.cpp:10-57
// The expansion order L and leaf threshold are globals read by the build-dir
// copy of tree.cpp (the reference hard-codes them at tree.cpp:32 and :94).
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>
#include <algorithm>

#include "particle.hpp"
#include "system_updaters/FMM.hpp"
#include "system_updaters/naive_update.hpp"
#include "quadratures/symplectic_euler.hpp"
#include "system_updaters/tree_components/tree.hpp"
#include "system_updaters/tree_components/leaf.hpp"
#include "system_updaters/multipole_utils/multipole_set.hpp"
#include "system_updaters/multipole_utils/power_set3D.hpp"
#include "system_updaters/multipole_utils/irregular.hpp"

unsigned int g_ref_threshold = 20;  // tree.cpp:32 default
unsigned int g_ref_L = 2;           // tree.cpp:94 default

namespace {
std::vector<Particle> make_particles(int dim, int64_t n, const double *pos, const double *vel, const double *mass) {
  std::vector<Particle> ps;
  ps.reserve(n);
  for (int64_t i = 0; i < n; ++i) {
    Tensor x(dim), v(dim);
    for (int d = 0; d < dim; ++d) {
      x[d] = pos[i * dim + d];
      v[d] = vel ? vel[i * dim + d] : 0.0;
    }
    ps.emplace_back(mass[i], std::move(x), std::move(v));
  }
  return ps;
}

// Exposes the protected tree state the same way tests/test_tree.cpp:14-40 does.
class TreeX : public Tree {
 public:
  template <class It>
  TreeX(It b, It e) : Tree(b, e) {}
  unsigned depth() const { return nodes_vector.size() - 1; }
  const std::unordered_map<u_int64_t, std::unique_ptr<NodeI>> &level(unsigned d) const { return nodes_vector[d]; }
};
struct LeafX : public Leaf {
  const std::vector<const Particle *> &parts() const { return particles; }
};
struct NodeX : public NodeI {
  uint64_t key() const { return id_child; }
  const std::vector<NodeI *> &nbrs() const { return neighbours_list; }
  const std::vector<NodeI *> &ilist() const { return interaction_list; }
};

std::unique_ptr<TreeX> g_tree;
std::vector<Particle> g_tree_particles;
}  // namespace

extern "C" {

void ref_set_params(unsigned L, unsigned threshold) {
  g_ref_L = L;
  g_ref_threshold = threshold;
}

double ref_grav_const() { return GRAV_CONST; }

// acc_out[n*dim] = the reference's acceleration (G * grad).
int ref_fmm(int dim, int64_t n, const double *pos, const double *mass, double *acc_out) {
  auto ps = make_particles(dim, n, pos, nullptr, mass);
  FMM f;
  f.update(ps);
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) acc_out[i * dim + d] = ps[i].get_acceleration()[d];
  return 0;
}

int ref_naive(int dim, int64_t n, const double *pos, const double *mass, double *acc_out) {
  auto ps = make_particles(dim, n, pos, nullptr, mass);
  NaiveUpdate f;
  f.update(ps);
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) acc_out[i * dim + d] = ps[i].get_acceleration()[d];
  return 0;
}

// Runs `steps` SyplecticEuler steps with FMM (use_fmm=1) or NaiveUpdate (0);
// pos/vel are updated in place.
int ref_se_steps(int dim, int64_t n, double *pos, double *vel, const double *mass, double dt, int steps, int use_fmm) {
  auto ps = make_particles(dim, n, pos, vel, mass);
  FMM f;
  NaiveUpdate nv;
  SyplecticEuler se;
  for (int s = 0; s < steps; ++s) se.integrate(use_fmm ? (SystemUpdateMethod *)&f : (SystemUpdateMethod *)&nv, ps, dt);
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) {
      pos[i * dim + d] = ps[i].get_position()[d];
      vel[i * dim + d] = ps[i].get_velocity()[d];
    }
  return 0;
}

// Builds the reference Tree and keeps it for the accessors below.
// Returns the leaf depth.
int ref_tree_build(int dim, int64_t n, const double *pos, const double *mass) {
  g_tree.reset();
  g_tree_particles = make_particles(dim, n, pos, nullptr, mass);
  g_tree = std::make_unique<TreeX>(g_tree_particles.begin(), g_tree_particles.end());
  return (int)g_tree->depth();
}

int64_t ref_tree_level_size(int d) { return (int64_t)g_tree->level(d).size(); }

// Leaves sorted by key: keys[nleaves], start[nleaves+1], perm[n] holds the
// particle indices of each leaf in the order the reference stores them.
int64_t ref_tree_leaves(uint64_t *keys, int64_t *start, int64_t *perm) {
  const auto &lv = g_tree->level(g_tree->depth());
  std::vector<uint64_t> ks;
  for (auto &kv : lv) ks.push_back(kv.first);
  std::sort(ks.begin(), ks.end());
  const Particle *base = g_tree_particles.data();
  int64_t pos = 0;
  for (size_t i = 0; i < ks.size(); ++i) {
    keys[i] = ks[i];
    start[i] = pos;
    const auto *leaf = (const LeafX *)lv.at(ks[i]).get();
    for (const Particle *p : leaf->parts()) perm[pos++] = p - base;
  }
  start[ks.size()] = pos;
  return (int64_t)ks.size();
}

// Sorted keys of all cells at level d.
int64_t ref_tree_level_keys(int d, uint64_t *keys) {
  const auto &lv = g_tree->level(d);
  int64_t i = 0;
  for (auto &kv : lv) keys[i++] = kv.first;
  std::sort(keys, keys + i);
  return i;
}

// Number of (target, source) pairs in neighbour (kind=0) or interaction (kind=1) lists at level d.
int64_t ref_tree_npairs(int d, int kind) {
  int64_t c = 0;
  for (auto &kv : g_tree->level(d)) {
    const auto *nx = (const NodeX *)kv.second.get();
    c += kind ? nx->ilist().size() : nx->nbrs().size();
  }
  return c;
}

int64_t ref_tree_pairs(int d, int kind, uint64_t *tkey, uint64_t *skey) {
  int64_t c = 0;
  for (auto &kv : g_tree->level(d)) {
    const auto *nx = (const NodeX *)kv.second.get();
    for (NodeI *s : (kind ? nx->ilist() : nx->nbrs())) {
      tkey[c] = kv.first;
      skey[c] = ((const NodeX *)s)->key();
      ++c;
    }
  }
  return c;
}

void ref_tree_free() {
  g_tree.reset();
  g_tree_particles.clear();
}

// P2M of n particles about `centre` at order L; out holds the reference's
// MultipoleSet<3> element vector (2L^2+4L+1 doubles).
int ref_p2m_3d(unsigned L, int64_t n, const double *pos, const double *mass, const double *centre, double *out) {
  MultipoleSet<3> m(L);
  m = 0;
  for (int64_t i = 0; i < n; ++i) {
    Tensor r(3);
    for (int d = 0; d < 3; ++d) r[d] = pos[i * 3 + d] - centre[d];
    PowerSet<3> z(L, r);
    z *= mass[i];
    m += z;
  }
  const auto &e = m.get_elements();
  std::memcpy(out, e.data(), e.size() * sizeof(double));
  return (int)e.size();
}

int ref_regular_3d(unsigned L, const double *r3, double *out) {
  Tensor r(3);
  for (int d = 0; d < 3; ++d) r[d] = r3[d];
  PowerSet<3> z(L, r);
  const auto &e = z.get_elements();
  std::memcpy(out, e.data(), e.size() * sizeof(double));
  return (int)e.size();
}

int ref_irregular_3d(unsigned L, const double *r3, double *out) {
  Tensor r(3);
  for (int d = 0; d < 3; ++d) r[d] = r3[d];
  Irregular z(L, r);
  const auto &e = z.get_elements();
  std::memcpy(out, e.data(), e.size() * sizeof(double));
  return (int)e.size();
}

}  // extern "C"
