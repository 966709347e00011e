/* CPU restatement of the rezucch1/nbody-FMM force pass — TEST INFRASTRUCTURE.
 *
 * Only tests, the smoke entry and bench.py's CPU-baseline leg load this
 * library; the product never does.  Parity is pinned by tests/test_oracle*.py
 * against the reference's own test_tree golden membership and against the
 * reference compiled from source (oracle/_ref).
 *
 * Every routine cites the reference file:line it restates (paths are inside
 * the reference project).  Deliberate differences, each stated where it
 * occurs:
 *  - keys are 64-bit throughout; the reference truncates interaction-list
 *    keys to 32 bits (node_i.cpp:31,63) and shifts a 32-bit value by up to
 *    63 bits in Morton::encode (morton_code.cpp:15), so its keys are only
 *    well defined for depth <= 10 (3D) / 16 (2D);
 *  - 3D translation operators are the correct solid-harmonic addition
 *    theorems, because the reference's M2M/M2L/L2L (multipole_set3D.cpp:45-118,
 *    local_set3D.cpp:51-81) do not converge and its L2P z-component has the
 *    wrong sign (local_set3D.cpp:206);
 *  - 2D binomials are computed in FP64, where the reference's unsigned ints
 *    overflow above p ~ 15 (multipole_set2D.cpp:77-83).
 */
#include "fmm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ------------------------------------------------------------------ Morton */
/* morton_code.cpp:9-22: bit b of coordinate i is placed at bit i + b*dim. */
uint64_t orc_morton_encode(const uint32_t *c, int dim) {
  uint64_t code = 0;
  for (int i = 0; i < dim; ++i)
    for (int b = 0; b < 32 && i + b * dim < 64; ++b)
      if ((c[i] >> b) & 1u) code |= (uint64_t)1 << (i + b * dim);
  return code;
}

/* morton_code.cpp:24-36 */
void orc_morton_decode(uint64_t code, int dim, uint32_t *c) {
  for (int i = 0; i < dim; ++i) c[i] = 0;
  for (int bit = 0; bit < 64; ++bit)
    if ((code >> bit) & 1u) c[bit % dim] |= 1u << (bit / dim);
}

/* double -> unsigned int exactly as the reference's x86-64 build converts
 * `n_coor[i] = p_pos[i] / leaf_size[i]` (tree.cpp:58): a truncating 64-bit
 * conversion whose low 32 bits are kept; NaN (a zero-extent axis, 0/0) gives 0. */
static uint32_t to_u32_like_ref(double v) {
  if (isnan(v) || v >= 9.2e18 || v <= -9.2e18) return 0u;
  return (uint32_t)(uint64_t)(int64_t)v;
}

static int bit_width_u64(uint64_t v) {
  int w = 0;
  while (v) { ++w; v >>= 1; }
  return w;
}

typedef struct { uint64_t key; int64_t idx; } kv_t;
static int cmp_kv(const void *a, const void *b) {
  const kv_t *x = (const kv_t *)a, *y = (const kv_t *)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return (x->idx > y->idx) - (x->idx < y->idx);
}

struct orc_tree {
  int dim, depth;
  int64_t n;
  double lo[3], hi[3];
  int64_t *ncell;      /* [depth+1] */
  uint64_t **keys;     /* [depth+1][ncell] sorted */
  int64_t **cbeg;      /* [depth][ncell]: first child index in level d+1 */
  int64_t **cend;
  int64_t *leaf_start; /* [nleaves+1] */
  int64_t *perm;       /* [n] */
  int64_t **nb_off, **nb_idx, **il_off, **il_idx; /* CSR lists per level */
};

static int64_t find_key(const uint64_t *keys, int64_t n, uint64_t k) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (keys[mid] < k) lo = mid + 1; else hi = mid;
  }
  return (lo < n && keys[lo] == k) ? lo : -1;
}

/* Leaf coordinates at `depth` (tree.cpp:47-61). */
static void bin_keys(int dim, int64_t n, const double *pos, const double *a, const double *b, int depth, kv_t *kv) {
  uint64_t nld = (uint64_t)1 << depth;
  double leaf_size[3];
  for (int d = 0; d < dim; ++d) leaf_size[d] = (b[d] - a[d]) / (double)nld;
  for (int64_t i = 0; i < n; ++i) {
    uint32_t c[3];
    for (int d = 0; d < dim; ++d) {
      double pp = pos[i * dim + d] - a[d];
      c[d] = to_u32_like_ref(pp / leaf_size[d]);
      if ((uint64_t)c[d] >= nld) c[d] = (uint32_t)(nld - 1);
    }
    kv[i].key = orc_morton_encode(c, dim);
    kv[i].idx = i;
  }
}

/* Tree::init_tree, tree.cpp:15-91. */
orc_tree *orc_tree_build(int dim, int64_t n, const double *pos, unsigned threshold) {
  if (n <= 0 || (dim != 2 && dim != 3) || threshold == 0) return NULL;
  orc_tree *t = (orc_tree *)calloc(1, sizeof(orc_tree));
  t->dim = dim;
  t->n = n;
  /* AABB, tree.cpp:20-30 (note the else-if) */
  for (int d = 0; d < dim; ++d) t->lo[d] = t->hi[d] = pos[d];
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) {
      double x = pos[i * dim + d];
      if (x < t->lo[d]) t->lo[d] = x;
      else if (x > t->hi[d]) t->hi[d] = x;
    }
  /* depth loop, tree.cpp:32-69 */
  unsigned max_n = (unsigned)n;
  unsigned depth = 0;
  unsigned max_depth = ((64u / dim) >> dim) << dim;
  kv_t *kv = (kv_t *)malloc(sizeof(kv_t) * n);
  do {
    uint64_t n_leafs = (uint64_t)(max_n - 1) / threshold + 1;
    depth += bit_width_u64(n_leafs) / dim + 1;
    if (depth > max_depth) depth = max_depth;
    bin_keys(dim, n, pos, t->lo, t->hi, (int)depth, kv);
    qsort(kv, n, sizeof(kv_t), cmp_kv);
    max_n = 0;
    for (int64_t i = 0, run = 0; i < n; ++i) {
      run = (i > 0 && kv[i].key == kv[i - 1].key) ? run + 1 : 1;
      if ((unsigned)run > max_n) max_n = (unsigned)run;
    }
  } while (depth < max_depth && max_n > threshold);
  t->depth = (int)depth;
  int D = t->depth;
  /* leaves keep input order inside each leaf (tree.cpp:62-66): kv is sorted by (key, idx) */
  t->ncell = (int64_t *)calloc(D + 1, sizeof(int64_t));
  t->keys = (uint64_t **)calloc(D + 1, sizeof(uint64_t *));
  t->cbeg = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  t->cend = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  t->perm = (int64_t *)malloc(sizeof(int64_t) * n);
  int64_t nl = 0;
  for (int64_t i = 0; i < n; ++i) {
    t->perm[i] = kv[i].idx;
    if (i == 0 || kv[i].key != kv[i - 1].key) ++nl;
  }
  t->ncell[D] = nl;
  t->keys[D] = (uint64_t *)malloc(sizeof(uint64_t) * nl);
  t->leaf_start = (int64_t *)malloc(sizeof(int64_t) * (nl + 1));
  for (int64_t i = 0, j = -1; i < n; ++i)
    if (i == 0 || kv[i].key != kv[i - 1].key) {
      ++j;
      t->keys[D][j] = kv[i].key;
      t->leaf_start[j] = i;
    }
  t->leaf_start[nl] = n;
  free(kv);
  /* ancestors, tree.cpp:76-83: parent key = key >> dim */
  for (int d = D - 1; d >= 0; --d) {
    int64_t m = t->ncell[d + 1], c = 0;
    uint64_t *k = (uint64_t *)malloc(sizeof(uint64_t) * m);
    for (int64_t i = 0; i < m; ++i) {
      uint64_t pk = t->keys[d + 1][i] >> dim;
      if (c == 0 || k[c - 1] != pk) k[c++] = pk;
    }
    t->keys[d] = k;
    t->ncell[d] = c;
    t->cbeg[d] = (int64_t *)malloc(sizeof(int64_t) * c);
    t->cend[d] = (int64_t *)malloc(sizeof(int64_t) * c);
    for (int64_t i = 0, j = 0; i < c; ++i) {
      t->cbeg[d][i] = j;
      while (j < m && (t->keys[d + 1][j] >> dim) == k[i]) ++j;
      t->cend[d][i] = j;
    }
  }
  /* lists, node_i.cpp:23-99 */
  t->nb_off = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  t->nb_idx = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  t->il_off = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  t->il_idx = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  for (int d = 0; d <= D; ++d) {
    int64_t m = t->ncell[d];
    int64_t *nbo = (int64_t *)malloc(sizeof(int64_t) * (m + 1));
    int64_t *ilo = (int64_t *)malloc(sizeof(int64_t) * (m + 1));
    int64_t cap_nb = m * 26 + 1, cap_il = m * (dim == 3 ? 189 : 27) + 1;
    int64_t *nbi = (int64_t *)malloc(sizeof(int64_t) * cap_nb);
    int64_t *ili = (int64_t *)malloc(sizeof(int64_t) * cap_il);
    int64_t cnb = 0, cil = 0;
    for (int64_t i = 0; i < m; ++i) {
      nbo[i] = cnb;
      ilo[i] = cil;
      uint32_t c[3] = {0, 0, 0};
      orc_morton_decode(t->keys[d][i], dim, c);
      int st[3], en[3], dir[3];
      for (int a = 0; a < dim; ++a) {
        st[a] = -(int)(c[a] % 2) - 2;
        en[a] = 3 - (int)(c[a] % 2);
        dir[a] = st[a];
      }
      for (;;) {
        int out = 0, nbr = 1;
        uint32_t nc[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) {
          int64_t v = (int64_t)c[a] + dir[a];
          if (v < 0) out = 1;
          nc[a] = (uint32_t)v;
          if (dir[a] < -1 || dir[a] > 1) nbr = 0;
        }
        if (!out) {
          int64_t j = find_key(t->keys[d], m, orc_morton_encode(nc, dim));
          if (j >= 0) {
            if (nbr) { if (j != i) nbi[cnb++] = j; }
            else ili[cil++] = j;
          }
        }
        int a = 0;
        for (; a < dim; ++a) {
          if (dir[a] == en[a]) dir[a] = st[a];
          else { ++dir[a]; break; }
        }
        if (a == dim) break;
      }
    }
    nbo[m] = cnb;
    ilo[m] = cil;
    t->nb_off[d] = nbo; t->nb_idx[d] = nbi; t->il_off[d] = ilo; t->il_idx[d] = ili;
  }
  return t;
}

void orc_tree_free(orc_tree *t) {
  if (!t) return;
  for (int d = 0; d <= t->depth; ++d) {
    free(t->keys[d]); free(t->cbeg[d]); free(t->cend[d]);
    free(t->nb_off[d]); free(t->nb_idx[d]); free(t->il_off[d]); free(t->il_idx[d]);
  }
  free(t->keys); free(t->cbeg); free(t->cend); free(t->ncell);
  free(t->nb_off); free(t->nb_idx); free(t->il_off); free(t->il_idx);
  free(t->leaf_start); free(t->perm); free(t);
}

int orc_tree_depth(const orc_tree *t) { return t->depth; }
void orc_tree_box(const orc_tree *t, double *lo, double *hi) {
  for (int d = 0; d < t->dim; ++d) { lo[d] = t->lo[d]; hi[d] = t->hi[d]; }
}
int64_t orc_tree_level_size(const orc_tree *t, int d) { return t->ncell[d]; }
int64_t orc_tree_level_keys(const orc_tree *t, int d, uint64_t *keys) {
  memcpy(keys, t->keys[d], sizeof(uint64_t) * t->ncell[d]);
  return t->ncell[d];
}
int64_t orc_tree_leaves(const orc_tree *t, uint64_t *keys, int64_t *start, int64_t *perm) {
  int64_t nl = t->ncell[t->depth];
  memcpy(keys, t->keys[t->depth], sizeof(uint64_t) * nl);
  memcpy(start, t->leaf_start, sizeof(int64_t) * (nl + 1));
  memcpy(perm, t->perm, sizeof(int64_t) * t->n);
  return nl;
}
int64_t orc_tree_npairs(const orc_tree *t, int d, int kind) {
  return kind ? t->il_off[d][t->ncell[d]] : t->nb_off[d][t->ncell[d]];
}
int64_t orc_tree_pairs(const orc_tree *t, int d, int kind, uint64_t *tkey, uint64_t *skey) {
  const int64_t *off = kind ? t->il_off[d] : t->nb_off[d];
  const int64_t *idx = kind ? t->il_idx[d] : t->nb_idx[d];
  int64_t c = 0;
  for (int64_t i = 0; i < t->ncell[d]; ++i)
    for (int64_t k = off[i]; k < off[i + 1]; ++k) {
      tkey[c] = t->keys[d][i];
      skey[c] = t->keys[d][idx[k]];
      ++c;
    }
  return c;
}

/* -------------------------------------------------------------- direct sum */
void orc_direct(int dim, int64_t n, const double *pos, const double *mass, double eps2,
                int64_t ntargets, const int64_t *targets, double *grad, double *pot) {
  if (!targets) ntargets = n;
  for (int64_t t = 0; t < ntargets; ++t) {
    int64_t i = targets ? targets[t] : t;
    double g[3] = {0, 0, 0}, ph = 0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double dd[3] = {0, 0, 0}, r2 = eps2;
      for (int a = 0; a < dim; ++a) { dd[a] = pos[i * dim + a] - pos[j * dim + a]; r2 += dd[a] * dd[a]; }
      if (dim == 3) {
        double ir = 1.0 / sqrt(r2), ir3 = ir * ir * ir;
        for (int a = 0; a < 3; ++a) g[a] -= mass[j] * dd[a] * ir3;
        ph += mass[j] * ir;
      } else {
        for (int a = 0; a < 2; ++a) g[a] -= mass[j] * dd[a] / r2;
        ph -= 0.5 * mass[j] * log(r2);
      }
    }
    for (int a = 0; a < dim; ++a) grad[t * dim + a] = g[a];
    if (pot) pot[t] = ph;
  }
}

/* naive_update.cpp:9-35 */
void orc_naive_ref(int dim, int64_t n, const double *pos, const double *mass, double *grad) {
  for (int64_t i = 0; i < n; ++i) {
    double g[3] = {0, 0, 0};
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double dd[3] = {0, 0, 0}, r2 = 0;
      for (int a = 0; a < dim; ++a) { dd[a] = pos[i * dim + a] - pos[j * dim + a]; r2 += dd[a] * dd[a]; }
      double f = (dim == 2) ? mass[j] / (r2 + 1.0e-4) : mass[j] / ((r2 + 1.0e-4) * sqrt(r2));
      for (int a = 0; a < dim; ++a) g[a] -= f * dd[a];
    }
    for (int a = 0; a < dim; ++a) grad[i * dim + a] = g[a];
  }
}

/* -------------------------------------------------------------- harmonics */
static inline int hidx(int n, int m) { return n * (n + 1) / 2 + m; }

/* Scaled regular harmonics Rs_n^m (m >= 0), from the Racah recurrences of
 * power_set3D.cpp:22-47 divided through by sqrt((n-m)!(n+m)!):
 *   Rs_l^l = -(x+iy) Rs_{l-1}^{l-1} / (2l)
 *   Rs_l^m = ((2l-1) z Rs_{l-1}^m - r^2 Rs_{l-2}^m) / (l^2 - m^2),  m < l. */
static void regular_s(int p, const double *r, cplx *R) {
  double x = r[0], y = r[1], z = r[2], r2 = x * x + y * y + z * z;
  cplx xy = x + I * y;
  R[0] = 1.0;
  for (int l = 1; l <= p; ++l) {
    R[hidx(l, l)] = -xy * R[hidx(l - 1, l - 1)] / (2.0 * l);
    for (int m = 0; m < l; ++m) {
      cplx v = (2.0 * l - 1.0) * z * R[hidx(l - 1, m)];
      if (m <= l - 2) v -= r2 * R[hidx(l - 2, m)];
      R[hidx(l, m)] = v / (double)(l * l - m * m);
    }
  }
}

/* Scaled irregular harmonics Is_n^m = I_n^m sqrt((n-m)!(n+m)!) (m >= 0), from
 * irregular.cpp:10-57 multiplied through:
 *   Is_0^0 = 1/r,  Is_l^l = -(2l-1)(x+iy) Is_{l-1}^{l-1} / r^2
 *   Is_l^m = ((2l-1) z Is_{l-1}^m - (l-1-m)(l-1+m) Is_{l-2}^m) / r^2. */
static void irregular_s(int p, const double *r, cplx *S) {
  double x = r[0], y = r[1], z = r[2], r2 = x * x + y * y + z * z, ir2 = 1.0 / r2;
  cplx xy = x + I * y;
  S[0] = 1.0 / sqrt(r2);
  for (int l = 1; l <= p; ++l) {
    S[hidx(l, l)] = -(2.0 * l - 1.0) * xy * S[hidx(l - 1, l - 1)] * ir2;
    for (int m = 0; m < l; ++m) {
      cplx v = (2.0 * l - 1.0) * z * S[hidx(l - 1, m)];
      if (m <= l - 2) v -= (double)((l - 1 - m) * (l - 1 + m)) * S[hidx(l - 2, m)];
      S[hidx(l, m)] = v * ir2;
    }
  }
}

/* X_n^m for any m from m >= 0 storage: X_n^{-m} = (-1)^m conj(X_n^m). */
static inline cplx hget(const cplx *X, int n, int m) {
  if (m >= 0) return X[hidx(n, m)];
  cplx v = conj(X[hidx(n, -m)]);
  return (m & 1) ? -v : v;
}

static double fact(int k) {
  double f = 1;
  for (int i = 2; i <= k; ++i) f *= i;
  return f;
}

void orc_regular_scaled(unsigned p, const double *r, double *out) {
  int K = (p + 1) * (p + 2) / 2;
  cplx *R = (cplx *)malloc(sizeof(cplx) * K);
  regular_s((int)p, r, R);
  for (int i = 0; i < K; ++i) { out[2 * i] = creal(R[i]); out[2 * i + 1] = cimag(R[i]); }
  free(R);
}

void orc_irregular_scaled(unsigned p, const double *r, double *out) {
  int K = (p + 1) * (p + 2) / 2;
  cplx *S = (cplx *)malloc(sizeof(cplx) * K);
  irregular_s((int)p, r, S);
  for (int i = 0; i < K; ++i) { out[2 * i] = creal(S[i]); out[2 * i + 1] = cimag(S[i]); }
  free(S);
}

/* The reference's element layout for PowerSet<3>/Irregular: index l*l for
 * m = 0, then (re, im) pairs at l*l + 2m - 1 (power_set3D.cpp:50-63). */
static void to_racah_layout(int p, const cplx *X, double *out, int irregular) {
  for (int l = 0; l <= p; ++l)
    for (int m = 0; m <= l; ++m) {
      double f = sqrt(fact(l - m) * fact(l + m));
      cplx v = irregular ? X[hidx(l, m)] / f : X[hidx(l, m)] * f;
      if (m == 0) out[l * l] = creal(v);
      else { out[l * l + 2 * m - 1] = creal(v); out[l * l + 2 * m] = cimag(v); }
    }
}

void orc_regular_racah(unsigned p, const double *r, double *out) {
  cplx *R = (cplx *)malloc(sizeof(cplx) * (p + 1) * (p + 2) / 2);
  regular_s((int)p, r, R);
  to_racah_layout((int)p, R, out, 0);
  free(R);
}

void orc_irregular_racah(unsigned p, const double *r, double *out) {
  cplx *S = (cplx *)malloc(sizeof(cplx) * (p + 1) * (p + 2) / 2);
  irregular_s((int)p, r, S);
  to_racah_layout((int)p, S, out, 1);
  free(S);
}

void orc_p2m_3d(unsigned p, int64_t n, const double *pos, const double *mass, const double *c, double *out) {
  int K = (p + 1) * (p + 2) / 2;
  cplx *R = (cplx *)malloc(sizeof(cplx) * K);
  cplx *M = (cplx *)calloc(K, sizeof(cplx));
  for (int64_t i = 0; i < n; ++i) {
    double d[3] = {pos[3 * i] - c[0], pos[3 * i + 1] - c[1], pos[3 * i + 2] - c[2]};
    regular_s((int)p, d, R);
    for (int k = 0; k < K; ++k) M[k] += mass[i] * conj(R[k]);
  }
  for (int k = 0; k < K; ++k) { out[2 * k] = creal(M[k]); out[2 * k + 1] = cimag(M[k]); }
  free(R);
  free(M);
}

/* ------------------------------------------------------------------ FMM 3D */
/* Operators (all verified against direct summation in the tests):
 *   P2M  M_n^m  = sum_i q_i conj(Rs_n^m(x_i - c))
 *   M2M  M'_n^m = sum_{k,l} conj(Rs_k^l(t)) M_{n-k}^{m-l},      t = c_child - c_parent
 *   M2L  L_k^l  = (-1)^{k+l} sum_{n,m} M_n^m Is_{n+k}^{m-l}(r), r = c_target - c_source
 *   L2L  L'_k^l = sum_{n,m} L_n^m Rs_{n-k}^{m-l}(t),            t = c_child - c_parent
 *   L2P  phi = sum_{n,m} L_n^m Rs_n^m(x - c), with
 *        d/dz Rs_n^m = Rs_{n-1}^m, d/dx = (Rs_{n-1}^{m+1} - Rs_{n-1}^{m-1})/2,
 *        d/dy = -i (Rs_{n-1}^{m-1} + Rs_{n-1}^{m+1})/2. */
static void m2m_3d(int p, const cplx *Mc, const double *t, cplx *Mp, cplx *R) {
  regular_s(p, t, R);
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      cplx s = 0;
      for (int k = 0; k <= n; ++k)
        for (int l = -k; l <= k; ++l) {
          int mm = m - l;
          if (mm < -(n - k) || mm > (n - k)) continue;
          s += conj(hget(R, k, l)) * hget(Mc, n - k, mm);
        }
      Mp[hidx(n, m)] += s;
    }
}

static void m2l_3d(int p, const cplx *M, const double *r, cplx *L, cplx *S) {
  irregular_s(2 * p, r, S);
  for (int k = 0; k <= p; ++k)
    for (int l = 0; l <= k; ++l) {
      cplx s = 0;
      for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) s += hget(M, n, m) * hget(S, n + k, m - l);
      L[hidx(k, l)] += ((k + l) & 1) ? -s : s;
    }
}

static void l2l_3d(int p, const cplx *Lp, const double *t, cplx *Lc, cplx *R) {
  regular_s(p, t, R);
  for (int k = 0; k <= p; ++k)
    for (int l = 0; l <= k; ++l) {
      cplx s = 0;
      for (int n = k; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
          int dm = m - l;
          if (dm < -(n - k) || dm > (n - k)) continue;
          s += hget(Lp, n, m) * hget(R, n - k, dm);
        }
      Lc[hidx(k, l)] += s;
    }
}

static void l2p_3d(int p, const cplx *L, const double *u, double *g, double *phi, cplx *R) {
  regular_s(p, u, R);
  double gx = 0, gy = 0, gz = 0, ph = 0;
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      cplx Lv = hget(L, n, m);
      ph += creal(Lv * hget(R, n, m));
      if (n == 0) continue;
      cplx rp = (m + 1 <= n - 1) ? hget(R, n - 1, m + 1) : 0;
      cplx rm = (m - 1 >= -(n - 1)) ? hget(R, n - 1, m - 1) : 0;
      cplx r0 = (m >= -(n - 1) && m <= n - 1) ? hget(R, n - 1, m) : 0;
      gx += creal(Lv * (rp - rm) * 0.5);
      gy += creal(Lv * (-I) * (rm + rp) * 0.5);
      gz += creal(Lv * r0);
    }
  g[0] += gx; g[1] += gy; g[2] += gz;
  *phi += ph;
}

/* ------------------------------------------------------------------ FMM 2D */
/* multipole_set2D.cpp / local_set2D.cpp / power_set2D.cpp:
 *   P2M a_k = sum q (z - c)^k
 *   M2M a'_l = sum_{k<=l} C(l,k) d^k a_{l-k}                (d = child - parent)
 *   M2L b_0 = a_0 log z - sum_k a_k/(k z^k)
 *       b_n = (-1)^{n+1} [a_0/(n z^n) + sum_k C(n+k-1,k-1) a_k/(k z^{n+k})]
 *   L2L b'_k = sum_{n>=k} C(n,k) b_n z^{n-k}                (z = child - parent)
 *   L2P grad = (-Re, +Im)(sum n b_n u^{n-1}),  phi = -Re(sum b_n u^n). */
static double binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  double b = 1;
  for (int i = 1; i <= k; ++i) b = b * (n - k + i) / i;
  return b;
}

static void m2m_2d(int p, const cplx *a, cplx d, cplx *out) {
  for (int l = 0; l <= p; ++l) {
    cplx s = 0, dk = 1;
    for (int k = 0; k <= l; ++k) {
      s += binom(l, k) * dk * a[l - k];
      dk *= d;
    }
    out[l] += s;
  }
}

static void m2l_2d(int p, const cplx *a, cplx z, cplx *b) {
  cplx b0 = a[0] * clog(z), zk = 1;
  for (int k = 1; k <= p; ++k) { zk *= z; b0 -= a[k] / ((double)k * zk); }
  b[0] += b0;
  cplx zn = 1;
  for (int n = 1; n <= p; ++n) {
    zn *= z;
    double sign = (n & 1) ? 1.0 : -1.0;
    cplx s = a[0] / ((double)n * zn), zkn = zn;
    for (int k = 1; k <= p; ++k) {
      zkn *= z;
      s += binom(n + k - 1, k - 1) * a[k] / ((double)k * zkn);
    }
    b[n] += sign * s;
  }
}

static void l2l_2d(int p, const cplx *b, cplx z, cplx *out) {
  for (int k = 0; k <= p; ++k) {
    cplx s = 0, zp = 1;
    for (int n = k; n <= p; ++n) {
      s += binom(n, k) * b[n] * zp;
      zp *= z;
    }
    out[k] += s;
  }
}

static void l2p_2d(int p, const cplx *b, cplx u, double *g, double *phi) {
  cplx dphi = 0, up = 1, phic = b[0];
  for (int q = 1; q <= p; ++q) {
    dphi += (double)q * b[q] * up;
    up *= u;
    phic += b[q] * up;
  }
  g[0] -= creal(dphi);
  g[1] += cimag(dphi);
  *phi -= creal(phic);
}

/* M2P: the outer expansion w(z) = a_0 log z - sum_k a_k/(k z^k) at z = x - c,
 * w'(z) = a_0/z + sum_k a_k/z^{k+1}; grad and phi as in L2P. */
static void m2p_2d(int p, const cplx *a, cplx z, double *g, double *phi) {
  const cplx iz = 1.0 / z;
  cplx w = a[0] * clog(z), dw = a[0] * iz, izk = 1;
  for (int k = 1; k <= p; ++k) {
    izk *= iz;
    w -= a[k] * izk / (double)k;
    dw += a[k] * izk * iz;
  }
  g[0] -= creal(dw);
  g[1] += cimag(dw);
  *phi -= creal(w);
}

/* ------------------------------------------------------------ FMM driver */
/* Tree::compute_accelerations, tree.cpp:93-111: P2M/M2M bottom-up, M2L over
 * every interaction list, L2L top-down, then per leaf L2P + P2P over the leaf
 * itself (j != i) and its neighbour leaves (leaf.cpp:55-148). */
static void pair_kernel(int dim, const double *xi, const double *xj, double mj, double eps2, double *g, double *ph) {
  double dd[3] = {0, 0, 0}, r2 = eps2;
  for (int a = 0; a < dim; ++a) { dd[a] = xi[a] - xj[a]; r2 += dd[a] * dd[a]; }
  if (dim == 3) {
    double ir = 1.0 / sqrt(r2);
    for (int a = 0; a < 3; ++a) g[a] -= mj * dd[a] * ir * ir * ir;
    *ph += mj * ir;
  } else {
    for (int a = 0; a < 2; ++a) g[a] -= mj * dd[a] / r2;
    *ph -= 0.5 * mj * log(r2);
  }
}

int orc_fmm(int dim, int64_t n, const double *pos, const double *mass, unsigned p_, unsigned threshold,
            int centre_mode, double *grad, double *pot) {
  return orc_fmm_ex(dim, n, pos, mass, p_, threshold, centre_mode, 0.0, 0, grad, pot);
}

/* With geometric centres, an interaction-list pair whose cells are not well
 * separated for the box's aspect ratio -- the sum of the two cells' radii
 * over the distance of their centres above FMM_RHO_MAX -- is summed directly,
 * as on the GPU.  The lists (node_i.cpp:39-43) count offsets in cells of the
 * rectangular bounding box (tree.cpp:20-30), so along a short axis a pair two
 * cells apart can have a divergent expansion. */
#define ORC_RHO_MAX 0.9
static int orc_not_well_separated(int dim, uint64_t kt, uint64_t ks, const double *ext) {
  uint32_t qt[3] = {0, 0, 0}, qs[3] = {0, 0, 0};
  orc_morton_decode(kt, dim, qt);
  orc_morton_decode(ks, dim, qs);
  double diag = 0.0, dist = 0.0;
  for (int a = 0; a < dim; ++a) {
    const double dd = ((double)qs[a] - (double)qt[a]) * ext[a];
    diag += ext[a] * ext[a];
    dist += dd * dd;
  }
  return dist <= 0.0 || sqrt(diag) > ORC_RHO_MAX * sqrt(dist);
}

int orc_fmm_ex(int dim, int64_t n, const double *pos, const double *mass, unsigned p_, unsigned threshold,
               int centre_mode, double eps2, int64_t direct_max, double *grad, double *pot) {
  orc_tree *t = orc_tree_build(dim, n, pos, threshold);
  if (!t) return -1;
  int p = (int)p_, D = t->depth;
  int K = (dim == 3) ? (p + 1) * (p + 2) / 2 : p + 1;
  int KW = (dim == 3) ? (2 * p + 1) * (2 * p + 2) / 2 : 1;
  cplx *work = (cplx *)malloc(sizeof(cplx) * KW);
  double **cen = (double **)calloc(D + 1, sizeof(double *));
  cplx **M = (cplx **)calloc(D + 1, sizeof(cplx *));
  cplx **Lx = (cplx **)calloc(D + 1, sizeof(cplx *));
  for (int d = 0; d <= D; ++d) {
    cen[d] = (double *)calloc(t->ncell[d] * 3, sizeof(double));
    M[d] = (cplx *)calloc(t->ncell[d] * K, sizeof(cplx));
    Lx[d] = (cplx *)calloc(t->ncell[d] * K, sizeof(cplx));
  }
  double ext[3];
  for (int a = 0; a < dim; ++a) ext[a] = t->hi[a] - t->lo[a];
  /* particle range [pb, pe) of every cell in leaf order */
  int64_t **pb = (int64_t **)calloc(D + 1, sizeof(int64_t *)), **pe = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  for (int d = D; d >= 0; --d) {
    pb[d] = (int64_t *)malloc(sizeof(int64_t) * t->ncell[d]);
    pe[d] = (int64_t *)malloc(sizeof(int64_t) * t->ncell[d]);
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      if (d == D) { pb[d][i] = t->leaf_start[i]; pe[d][i] = t->leaf_start[i + 1]; }
      else { pb[d][i] = pb[d + 1][t->cbeg[d][i]]; pe[d][i] = pe[d + 1][t->cend[d][i] - 1]; }
    }
  }
  double *fd = (double *)calloc((size_t)n * 4, sizeof(double)); /* direct far field: grad xyz + phi per input index */
  /* centres */
  for (int d = D; d >= 0; --d)
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      double *c = cen[d] + 3 * i;
      if (centre_mode == 0) {
        uint32_t q[3] = {0, 0, 0};
        orc_morton_decode(t->keys[d][i], dim, q);
        for (int a = 0; a < dim; ++a) c[a] = t->lo[a] + (q[a] + 0.5) * (ext[a] / (double)((uint64_t)1 << d));
      } else if (d == D) {
        double tm = 0;
        for (int64_t k = t->leaf_start[i]; k < t->leaf_start[i + 1]; ++k) {
          int64_t j = t->perm[k];
          tm += mass[j];
          for (int a = 0; a < dim; ++a) c[a] += mass[j] * pos[j * dim + a];
        }
        for (int a = 0; a < dim; ++a) c[a] /= tm;
      } else {
        double tm = 0;
        for (int64_t ch = t->cbeg[d][i]; ch < t->cend[d][i]; ++ch) {
          double cm = creal(M[d + 1][ch * K]);
          tm += cm;
          for (int a = 0; a < dim; ++a) c[a] += cm * cen[d + 1][3 * ch + a];
        }
        for (int a = 0; a < dim; ++a) c[a] /= tm;
      }
      /* P2M / M2M right after the centre is known (the reference interleaves
       * calculateMC and compute_multipoles the same way, node.cpp:14-24) */
      cplx *Mi = M[d] + (int64_t)K * i;
      if (d == D) {
        for (int64_t k = t->leaf_start[i]; k < t->leaf_start[i + 1]; ++k) {
          int64_t j = t->perm[k];
          if (dim == 3) {
            double r[3] = {pos[3 * j] - c[0], pos[3 * j + 1] - c[1], pos[3 * j + 2] - c[2]};
            regular_s(p, r, work);
            for (int q = 0; q < K; ++q) Mi[q] += mass[j] * conj(work[q]);
          } else {
            cplx zz = (pos[2 * j] - c[0]) + I * (pos[2 * j + 1] - c[1]), zp = 1;
            for (int q = 0; q <= p; ++q) { Mi[q] += mass[j] * zp; zp *= zz; }
          }
        }
      } else {
        for (int64_t ch = t->cbeg[d][i]; ch < t->cend[d][i]; ++ch) {
          double tv[3] = {0, 0, 0};
          for (int a = 0; a < dim; ++a) tv[a] = cen[d + 1][3 * ch + a] - c[a];
          if (dim == 3) m2m_3d(p, M[d + 1] + (int64_t)K * ch, tv, Mi, work);
          else m2m_2d(p, M[d + 1] + (int64_t)K * ch, tv[0] + I * tv[1], Mi);
        }
      }
    }
  /* M2L (or the direct far field for small pairs) */
  for (int d = 0; d <= D; ++d)
    for (int64_t i = 0; i < t->ncell[d]; ++i)
      for (int64_t k = t->il_off[d][i]; k < t->il_off[d][i + 1]; ++k) {
        int64_t s = t->il_idx[d][k];
        if ((direct_max > 0 && (pe[d][i] - pb[d][i]) * (pe[d][s] - pb[d][s]) <= direct_max) ||
            (centre_mode == 0 && orc_not_well_separated(dim, t->keys[d][i], t->keys[d][s], ext))) {
          for (int64_t a = pb[d][i]; a < pe[d][i]; ++a) {
            int64_t pi = t->perm[a];
            for (int64_t b = pb[d][s]; b < pe[d][s]; ++b) {
              int64_t pj = t->perm[b];
              pair_kernel(dim, pos + pi * dim, pos + pj * dim, mass[pj], eps2, fd + 4 * pi, fd + 4 * pi + 3);
            }
          }
          continue;
        }
        double r[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) r[a] = cen[d][3 * i + a] - cen[d][3 * s + a];
        if (dim == 3) m2l_3d(p, M[d] + (int64_t)K * s, r, Lx[d] + (int64_t)K * i, work);
        else m2l_2d(p, M[d] + (int64_t)K * s, r[0] + I * r[1], Lx[d] + (int64_t)K * i);
      }
  /* L2L */
  for (int d = 0; d < D; ++d)
    for (int64_t i = 0; i < t->ncell[d]; ++i)
      for (int64_t ch = t->cbeg[d][i]; ch < t->cend[d][i]; ++ch) {
        double tv[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) tv[a] = cen[d + 1][3 * ch + a] - cen[d][3 * i + a];
        if (dim == 3) l2l_3d(p, Lx[d] + (int64_t)K * i, tv, Lx[d + 1] + (int64_t)K * ch, work);
        else l2l_2d(p, Lx[d] + (int64_t)K * i, tv[0] + I * tv[1], Lx[d + 1] + (int64_t)K * ch);
      }
  /* L2P + P2P */
  for (int64_t i = 0; i < t->ncell[D]; ++i) {
    const double *c = cen[D] + 3 * i;
    const cplx *Li = Lx[D] + (int64_t)K * i;
    for (int64_t k = t->leaf_start[i]; k < t->leaf_start[i + 1]; ++k) {
      int64_t pi = t->perm[k];
      double g[3] = {0, 0, 0}, ph = 0;
      if (dim == 3) {
        double u[3] = {pos[3 * pi] - c[0], pos[3 * pi + 1] - c[1], pos[3 * pi + 2] - c[2]};
        l2p_3d(p, Li, u, g, &ph, work);
      } else {
        l2p_2d(p, Li, (pos[2 * pi] - c[0]) + I * (pos[2 * pi + 1] - c[1]), g, &ph);
      }
      /* near field: the leaf itself then its neighbours */
      for (int64_t nb = -1; nb < t->nb_off[D][i + 1] - t->nb_off[D][i]; ++nb) {
        int64_t src = nb < 0 ? i : t->nb_idx[D][t->nb_off[D][i] + nb];
        for (int64_t kk = t->leaf_start[src]; kk < t->leaf_start[src + 1]; ++kk) {
          int64_t pj = t->perm[kk];
          if (pj == pi) continue;
          pair_kernel(dim, pos + pi * dim, pos + pj * dim, mass[pj], eps2, g, &ph);
        }
      }
      for (int a = 0; a < dim; ++a) grad[pi * dim + a] = g[a] + fd[4 * pi + a];
      if (pot) pot[pi] = ph + fd[4 * pi + 3];
    }
  }
  for (int d = 0; d <= D; ++d) { free(cen[d]); free(M[d]); free(Lx[d]); free(pb[d]); free(pe[d]); }
  free(cen); free(M); free(Lx); free(work); free(pb); free(pe); free(fd);
  orc_tree_free(t);
  return 0;
}

/* ------------------------------------------------------- adaptive targets */
/* M2P: the multipole M (centre c) evaluated at a point r = x - c, through
 * the order-0 and order-1 local coefficients at x (M2L to the point, then
 * L2P at offset zero); g and phi accumulate. */
static void m2p_3d(int p, const cplx *M, const double *r, double *g, double *phi, cplx *S, cplx *Lw, cplx *R) {
  irregular_s(p + 1, r, S);
  for (int q = 0; q < 3; ++q) Lw[q] = 0;
  for (int k = 0; k <= 1; ++k)
    for (int l = 0; l <= k; ++l) {
      cplx s = 0;
      for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) s += hget(M, n, m) * hget(S, n + k, m - l);
      Lw[hidx(k, l)] = ((k + l) & 1) ? -s : s;
    }
  const double zero[3] = {0, 0, 0};
  l2p_3d(1, Lw, zero, g, phi, R);
}

/* Particle range [pb, pe) in leaf order and parent index of every cell
 * (the root's parent is -1); arrays of t->ncell[d] entries per level. */
static void cell_ranges(const orc_tree *t, int64_t **pb, int64_t **pe, int64_t **par) {
  const int D = t->depth;
  for (int d = D; d >= 0; --d)
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      if (d == D) { pb[d][i] = t->leaf_start[i]; pe[d][i] = t->leaf_start[i + 1]; }
      else {
        pb[d][i] = pb[d + 1][t->cbeg[d][i]];
        pe[d][i] = pe[d + 1][t->cend[d][i] - 1];
        for (int64_t ch = t->cbeg[d][i]; ch < t->cend[d][i]; ++ch) par[d + 1][ch] = i;
      }
    }
  par[0][0] = -1;
}

/* Active target cells and adaptive leaves, top down: the root is active; a
 * cell is active if its parent is active and not an adaptive leaf; an active
 * cell with at most `aleaf` particles, or at depth D, is an adaptive leaf. */
static void adaptive_flags(const orc_tree *t, int64_t **pb, int64_t **pe, int64_t **par, unsigned aleaf, char **act,
                           char **leaf) {
  const int D = t->depth;
  for (int d = 0; d <= D; ++d)
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      const int64_t cnt = pe[d][i] - pb[d][i];
      act[d][i] = d == 0 ? 1 : (act[d - 1][par[d][i]] && !leaf[d - 1][par[d][i]]);
      leaf[d][i] = act[d][i] && (cnt <= (int64_t)aleaf || d == D);
    }
}

/* An FMM whose targets stop descending at small cells, the adaptive form
 * of the uniform-depth tree of orc_tree_build (3D and 2D, geometric centres).
 *
 * Every cell of the uniform tree stays a source.  A target cell is active
 * if it is the root or its parent is active and holds more than `aleaf`
 * particles; an active cell with at most `aleaf` particles, or at depth D,
 * is an adaptive leaf.  A particle of an adaptive leaf B at level d gets the
 * interaction lists of B and of its ancestors (M2L into active cells, L2L
 * down active cells, L2P from B) and, directly, the particles of B's
 * colleagues at level d.  Those pairs, at all deeper levels and in the leaf
 * level's near field, are exactly what the uniform FMM sums below level d.
 * A colleague cell C is summed particle by particle when
 * n_B n_C <= w_direct_max or C is at depth D; otherwise its children are
 * taken in its place: a child too close to B (touching it, or its radius
 * over its distance from B's box above 0.75) again as a colleague, a child
 * farther away through its multipole evaluated at B's particles (M2P; the
 * W list of the adaptive FMM), or directly when n_B n_child <= w_direct_max.
 * Interaction-list pairs follow orc_fmm_ex's rules (direct_max, separation).
 */
int orc_fmm_adaptive(int dim, int64_t n, const double *pos, const double *mass, unsigned p_, unsigned threshold,
                     unsigned aleaf, double eps2, int64_t direct_max, int64_t w_direct_max, double *grad,
                     double *pot) {
  if (dim != 2 && dim != 3) return -2;
  orc_tree *t = orc_tree_build(dim, n, pos, threshold);
  if (!t) return -1;
  const int p = (int)p_, D = t->depth;
  const int K = dim == 3 ? (p + 1) * (p + 2) / 2 : p + 1, KW = (2 * p + 2) * (2 * p + 3) / 2;
  cplx *work = (cplx *)malloc(sizeof(cplx) * KW), *work2 = (cplx *)malloc(sizeof(cplx) * KW);
  cplx Lw[3];
  double ext[3] = {0, 0, 0};
  for (int a = 0; a < dim; ++a) ext[a] = t->hi[a] - t->lo[a];
  double **cen = (double **)calloc(D + 1, sizeof(double *));
  cplx **M = (cplx **)calloc(D + 1, sizeof(cplx *)), **Lx = (cplx **)calloc(D + 1, sizeof(cplx *));
  int64_t **pb = (int64_t **)calloc(D + 1, sizeof(int64_t *)), **pe = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  int64_t **par = (int64_t **)calloc(D + 1, sizeof(int64_t *));
  char **act = (char **)calloc(D + 1, sizeof(char *)), **leaf = (char **)calloc(D + 1, sizeof(char *));
  for (int d = 0; d <= D; ++d) {
    const int64_t m = t->ncell[d];
    cen[d] = (double *)calloc(m * 3, sizeof(double));
    M[d] = (cplx *)calloc(m * K, sizeof(cplx));
    Lx[d] = (cplx *)calloc(m * K, sizeof(cplx));
    pb[d] = (int64_t *)malloc(sizeof(int64_t) * m);
    pe[d] = (int64_t *)malloc(sizeof(int64_t) * m);
    par[d] = (int64_t *)malloc(sizeof(int64_t) * m);
    act[d] = (char *)calloc(m, 1);
    leaf[d] = (char *)calloc(m, 1);
  }
  cell_ranges(t, pb, pe, par);
  /* geometric centres, P2M at depth D, M2M up */
  for (int d = D; d >= 0; --d)
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      double *c = cen[d] + 3 * i;
      uint32_t q[3] = {0, 0, 0};
      orc_morton_decode(t->keys[d][i], dim, q);
      for (int a = 0; a < dim; ++a) c[a] = t->lo[a] + (q[a] + 0.5) * (ext[a] / (double)((uint64_t)1 << d));
      cplx *Mi = M[d] + (int64_t)K * i;
      if (d == D) {
        for (int64_t k = pb[d][i]; k < pe[d][i]; ++k) {
          const int64_t j = t->perm[k];
          if (dim == 3) {
            double r[3] = {pos[3 * j] - c[0], pos[3 * j + 1] - c[1], pos[3 * j + 2] - c[2]};
            regular_s(p, r, work);
            for (int qq = 0; qq < K; ++qq) Mi[qq] += mass[j] * conj(work[qq]);
          } else {
            cplx zz = (pos[2 * j] - c[0]) + I * (pos[2 * j + 1] - c[1]), zp = 1;
            for (int qq = 0; qq <= p; ++qq) { Mi[qq] += mass[j] * zp; zp *= zz; }
          }
        }
      } else {
        for (int64_t ch = t->cbeg[d][i]; ch < t->cend[d][i]; ++ch) {
          double tv[3] = {0, 0, 0};
          for (int a = 0; a < dim; ++a) tv[a] = cen[d + 1][3 * ch + a] - c[a];
          if (dim == 3) m2m_3d(p, M[d + 1] + (int64_t)K * ch, tv, Mi, work);
          else m2m_2d(p, M[d + 1] + (int64_t)K * ch, tv[0] + I * tv[1], Mi);
        }
      }
    }
  adaptive_flags(t, pb, pe, par, aleaf, act, leaf);
  double *fd = (double *)calloc((size_t)n * 4, sizeof(double));
  /* interaction lists of the active targets: M2L, or direct (orc_fmm_ex's rules) */
  for (int d = 0; d <= D; ++d)
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      if (!act[d][i]) continue;
      for (int64_t k = t->il_off[d][i]; k < t->il_off[d][i + 1]; ++k) {
        const int64_t s = t->il_idx[d][k];
        if ((direct_max > 0 && (pe[d][i] - pb[d][i]) * (pe[d][s] - pb[d][s]) <= direct_max) ||
            orc_not_well_separated(dim, t->keys[d][i], t->keys[d][s], ext)) {
          for (int64_t a = pb[d][i]; a < pe[d][i]; ++a) {
            const int64_t pi = t->perm[a];
            for (int64_t b = pb[d][s]; b < pe[d][s]; ++b) {
              const int64_t pj = t->perm[b];
              pair_kernel(dim, pos + pi * dim, pos + pj * dim, mass[pj], eps2, fd + 4 * pi, fd + 4 * pi + 3);
            }
          }
          continue;
        }
        double r[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) r[a] = cen[d][3 * i + a] - cen[d][3 * s + a];
        if (dim == 3) m2l_3d(p, M[d] + (int64_t)K * s, r, Lx[d] + (int64_t)K * i, work);
        else m2l_2d(p, M[d] + (int64_t)K * s, r[0] + I * r[1], Lx[d] + (int64_t)K * i);
      }
    }
  /* L2L down the active cells */
  for (int d = 0; d < D; ++d)
    for (int64_t i = 0; i < t->ncell[d]; ++i) {
      if (!act[d][i] || leaf[d][i]) continue;
      for (int64_t ch = t->cbeg[d][i]; ch < t->cend[d][i]; ++ch) {
        double tv[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) tv[a] = cen[d + 1][3 * ch + a] - cen[d][3 * i + a];
        if (dim == 3) l2l_3d(p, Lx[d] + (int64_t)K * i, tv, Lx[d + 1] + (int64_t)K * ch, work);
        else l2l_2d(p, Lx[d] + (int64_t)K * i, tv[0] + I * tv[1], Lx[d + 1] + (int64_t)K * ch);
      }
    }
  /* adaptive leaves: L2P, then the colleagues' particles (with the W list) */
  int64_t cap = 1024, top = 0;
  int64_t *stk = (int64_t *)malloc(sizeof(int64_t) * 2 * cap);
  for (int d = 0; d <= D; ++d)
    for (int64_t b = 0; b < t->ncell[d]; ++b) {
      if (!leaf[d][b]) continue;
      const int64_t nB = pe[d][b] - pb[d][b];
      const double *cb = cen[d] + 3 * b;
      double hb[3] = {0, 0, 0};
      for (int a = 0; a < dim; ++a) hb[a] = 0.5 * ext[a] / (double)((uint64_t)1 << d);
      for (int64_t k = pb[d][b]; k < pe[d][b]; ++k) {
        const int64_t pi = t->perm[k];
        double *g = fd + 4 * pi;
        if (dim == 3) {
          double u[3] = {pos[3 * pi] - cb[0], pos[3 * pi + 1] - cb[1], pos[3 * pi + 2] - cb[2]};
          l2p_3d(p, Lx[d] + (int64_t)K * b, u, g, g + 3, work);
        } else {
          l2p_2d(p, Lx[d] + (int64_t)K * b, (pos[2 * pi] - cb[0]) + I * (pos[2 * pi + 1] - cb[1]), g, g + 3);
        }
        for (int64_t kk = pb[d][b]; kk < pe[d][b]; ++kk) {  /* the leaf itself */
          const int64_t pj = t->perm[kk];
          if (pj != pi) pair_kernel(dim, pos + pi * dim, pos + pj * dim, mass[pj], eps2, g, g + 3);
        }
      }
      top = 0;
      for (int64_t k = t->nb_off[d][b]; k < t->nb_off[d][b + 1]; ++k) {
        stk[2 * top] = d;
        stk[2 * top + 1] = t->nb_idx[d][k];
        ++top;
      }
      while (top > 0) {
        --top;
        const int e = (int)stk[2 * top];
        const int64_t C = stk[2 * top + 1];
        const int64_t nC = pe[e][C] - pb[e][C];
        if (e == D || nB * nC <= w_direct_max) {
          for (int64_t k = pb[d][b]; k < pe[d][b]; ++k) {
            const int64_t pi = t->perm[k];
            for (int64_t kk = pb[e][C]; kk < pe[e][C]; ++kk) {
              const int64_t pj = t->perm[kk];
              pair_kernel(dim, pos + pi * dim, pos + pj * dim, mass[pj], eps2, fd + 4 * pi, fd + 4 * pi + 3);
            }
          }
          continue;
        }
        for (int64_t ch = t->cbeg[e][C]; ch < t->cend[e][C]; ++ch) {
          const double *cc = cen[e + 1] + 3 * ch;
          double dist2 = 0.0, rad2 = 0.0;
          for (int a = 0; a < dim; ++a) {
            const double hc = 0.5 * ext[a] / (double)((uint64_t)1 << (e + 1));
            const double gap = fabs(cc[a] - cb[a]) - hb[a];
            if (gap > 0) dist2 += gap * gap;
            rad2 += hc * hc;
          }
          const int64_t nc = pe[e + 1][ch] - pb[e + 1][ch];
          if (dist2 <= 0.0 || rad2 > 0.75 * 0.75 * dist2) {  /* too close: a colleague again */
            if (top + 1 > cap) {
              cap *= 2;
              stk = (int64_t *)realloc(stk, sizeof(int64_t) * 2 * cap);
            }
            stk[2 * top] = e + 1;
            stk[2 * top + 1] = ch;
            ++top;
          } else if (nB * nc <= w_direct_max) {
            for (int64_t k = pb[d][b]; k < pe[d][b]; ++k) {
              const int64_t pi = t->perm[k];
              for (int64_t kk = pb[e + 1][ch]; kk < pe[e + 1][ch]; ++kk) {
                const int64_t pj = t->perm[kk];
                pair_kernel(dim, pos + pi * dim, pos + pj * dim, mass[pj], eps2, fd + 4 * pi, fd + 4 * pi + 3);
              }
            }
          } else {
            for (int64_t k = pb[d][b]; k < pe[d][b]; ++k) {
              const int64_t pi = t->perm[k];
              double *g = fd + 4 * pi;
              if (dim == 3) {
                double r[3] = {pos[3 * pi] - cc[0], pos[3 * pi + 1] - cc[1], pos[3 * pi + 2] - cc[2]};
                m2p_3d(p, M[e + 1] + (int64_t)K * ch, r, g, g + 3, work, Lw, work2);
              } else {
                m2p_2d(p, M[e + 1] + (int64_t)K * ch, (pos[2 * pi] - cc[0]) + I * (pos[2 * pi + 1] - cc[1]), g,
                       g + 3);
              }
            }
          }
        }
      }
    }
  for (int64_t i = 0; i < n; ++i) {
    for (int a = 0; a < dim; ++a) grad[dim * i + a] = fd[4 * i + a];
    if (pot) pot[i] = fd[4 * i + 3];
  }
  free(stk);
  for (int d = 0; d <= D; ++d) {
    free(cen[d]); free(M[d]); free(Lx[d]); free(pb[d]); free(pe[d]); free(par[d]); free(act[d]); free(leaf[d]);
  }
  free(cen); free(M); free(Lx); free(pb); free(pe); free(par); free(act); free(leaf); free(work); free(work2); free(fd);
  orc_tree_free(t);
  return 0;
}

/* The flags of orc_fmm_adaptive for every cell, level by level in the order
 * of orc_tree_level_keys: bit 0 active target, bit 1 adaptive leaf.  Returns
 * the number of cells (writing nothing when it exceeds cap), or -1. */
int64_t orc_adaptive_flags(int dim, int64_t n, const double *pos, unsigned threshold, unsigned aleaf, int64_t cap,
                           uint8_t *flags) {
  orc_tree *t = orc_tree_build(dim, n, pos, threshold);
  if (!t) return -1;
  const int D = t->depth;
  int64_t total = 0;
  for (int d = 0; d <= D; ++d) total += t->ncell[d];
  if (total <= cap && flags) {
    const size_t nlev = (size_t)(D < 0 ? 0 : D) + 1;
    int64_t **pb = (int64_t **)calloc(nlev, sizeof(int64_t *)), **pe = (int64_t **)calloc(nlev, sizeof(int64_t *));
    int64_t **par = (int64_t **)calloc(nlev, sizeof(int64_t *));
    char **act = (char **)calloc(nlev, sizeof(char *)), **leaf = (char **)calloc(nlev, sizeof(char *));
    for (int d = 0; d <= D; ++d) {
      const int64_t m = t->ncell[d];
      pb[d] = (int64_t *)malloc(sizeof(int64_t) * m);
      pe[d] = (int64_t *)malloc(sizeof(int64_t) * m);
      par[d] = (int64_t *)malloc(sizeof(int64_t) * m);
      act[d] = (char *)calloc(m, 1);
      leaf[d] = (char *)calloc(m, 1);
    }
    cell_ranges(t, pb, pe, par);
    adaptive_flags(t, pb, pe, par, aleaf, act, leaf);
    int64_t o = 0;
    for (int d = 0; d <= D; ++d)
      for (int64_t i = 0; i < t->ncell[d]; ++i, ++o) flags[o] = (uint8_t)((act[d][i] ? 1 : 0) | (leaf[d][i] ? 2 : 0));
    for (int d = 0; d <= D; ++d) { free(pb[d]); free(pe[d]); free(par[d]); free(act[d]); free(leaf[d]); }
    free(pb); free(pe); free(par); free(act); free(leaf);
  }
  orc_tree_free(t);
  return total;
}
