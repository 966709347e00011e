// FP64 construction of the translation operators (M2L, M2M, L2L) as real
// matrices, stored FP32 for the contraction kernels.
//
// 3D uses scaled solid harmonics Rs_n^m = R_n^m / sqrt((n-m)!(n+m)!) and
// Is_n^m = I_n^m sqrt((n-m)!(n+m)!), where R and I are the Racah-normalised
// regular/irregular harmonics of the reference (power_set3D.cpp:10-48,
// irregular.cpp:10-57).  With geometric cell centres and coefficients scaled
// by the cell size s_d (M~_n = M_n / s^n, L^_n = s^(n+1) L_n):
//   M2M  M~'_n^m = sum conj(Rs_k^l(t)) 2^-(n-k) M~_{n-k}^{m-l},  t = (c_child - c_parent)/s_parent
//   M2L  L^_k^l  = (-1)^(k+l) sum M~_n^m Is_{n+k}^{m-l}(rho),   rho = (c_t - c_s)/s
//   L2L  L^'_k^l = sum L^_n^m Rs_{n-k}^{m-l}(t) 2^-(k+1)
// so every operator depends only on the relative offset and the box aspect
// ratio, never on the level.  (The reference's own 3D M2M/M2L/L2L,
// multipole_set3D.cpp:45-118 and local_set3D.cpp:51-81, do not converge.)
//
// 2D follows the reference's complex-log expansions (multipole_set2D.cpp,
// local_set2D.cpp) with a_k scaled by s^-k and b_n by s^n.
#include <cmath>
#include <vector>

#include "expansions.cuh"

namespace fmm {

struct cd {
  double re, im;
};
__device__ inline cd cmul(cd a, cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ inline cd cadd(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
__device__ inline cd csub(cd a, cd b) { return {a.re - b.re, a.im - b.im}; }
__device__ inline cd cscale(cd a, double s) { return {a.re * s, a.im * s}; }
__device__ inline cd cconj(cd a) { return {a.re, -a.im}; }
__device__ inline int hid(int n, int m) { return n * (n + 1) / 2 + m; }

// X_n^m for any m from m >= 0 storage (X_n^-m = (-1)^m conj(X_n^m)); 0 outside |m| <= n.
__device__ inline cd hget(const cd *X, int n, int m) {
  if (n < 0 || m > n || m < -n) return {0.0, 0.0};
  if (m >= 0) return X[hid(n, m)];
  cd v = cconj(X[hid(n, -m)]);
  return (m & 1) ? cd{-v.re, -v.im} : v;
}

__device__ void regular_s(int p, const double *r, cd *R) {
  double x = r[0], y = r[1], z = r[2], r2 = x * x + y * y + z * z;
  R[0] = {1.0, 0.0};
  for (int l = 1; l <= p; ++l) {
    cd d = R[hid(l - 1, l - 1)];
    cd v = cmul({-x, -y}, d);
    R[hid(l, l)] = cscale(v, 1.0 / (2.0 * l));
    for (int m = 0; m < l; ++m) {
      cd a = cscale(R[hid(l - 1, m)], (2.0 * l - 1.0) * z);
      if (m <= l - 2) a = csub(a, cscale(R[hid(l - 2, m)], r2));
      R[hid(l, m)] = cscale(a, 1.0 / (double)(l * l - m * m));
    }
  }
}

__device__ void irregular_s(int p, const double *r, cd *S) {
  double x = r[0], y = r[1], z = r[2], r2 = x * x + y * y + z * z, ir2 = 1.0 / r2;
  S[0] = {1.0 / sqrt(r2), 0.0};
  for (int l = 1; l <= p; ++l) {
    cd d = S[hid(l - 1, l - 1)];
    S[hid(l, l)] = cscale(cmul({x, y}, d), -(2.0 * l - 1.0) * ir2);
    for (int m = 0; m < l; ++m) {
      cd a = cscale(S[hid(l - 1, m)], (2.0 * l - 1.0) * z);
      if (m <= l - 2) a = csub(a, cscale(S[hid(l - 2, m)], (double)((l - 1 - m) * (l - 1 + m))));
      S[hid(l, m)] = cscale(a, ir2);
    }
  }
}

// Real index -> (n, m, imaginary part?)
__device__ inline void dec_idx(int i, int &n, int &m, int &im) {
  n = (int)sqrt((double)i);
  while ((n + 1) * (n + 1) <= i) ++n;
  while (n * n > i) --n;
  int r = i - n * n;
  if (r == 0) {
    m = 0;
    im = 0;
  } else {
    m = (r + 1) / 2;
    im = (r & 1) ? 0 : 1;
  }
}

// Complex coefficient C(out=(k,l), in=(n,m')) of each operator kind.
// kind 0: M2L, 1: M2M, 2: L2L.
__device__ inline cd op_coef(int kind, const cd *H, int k, int l, int n, int mp) {
  if (kind == 0) {
    cd v = hget(H, n + k, mp - l);
    return ((k + l) & 1) ? cd{-v.re, -v.im} : v;
  } else if (kind == 1) {  // out (k,l) = parent (n,m); in (n,mp) = child
    if (n > k) return {0.0, 0.0};
    cd v = cconj(hget(H, k - n, l - mp));
    return cscale(v, ldexp(1.0, -n));
  } else {
    if (n < k) return {0.0, 0.0};
    cd v = hget(H, n - k, mp - l);
    return cscale(v, ldexp(1.0, -(k + 1)));
  }
}

// One block per slot.  Builds K x KP (input-major) FP32 matrix.
__global__ void k_build_ops3d(float *tab, double *tab64, int p, int K, int KP, int n_m2l, double ax, double ay,
                              double az) {
  extern __shared__ cd H[];
  const int slot = blockIdx.x;
  int kind;
  double r[3];
  bool zero = false;
  if (slot < n_m2l) {
    kind = 0;
    // slot offset = source cell - target cell; M2L translates by
    // rho = (c_target - c_source) / s
    int dx = slot % 7 - 3, dy = (slot / 7) % 7 - 3, dz = slot / 49 - 3;
    r[0] = -dx * ax;
    r[1] = -dy * ay;
    r[2] = -dz * az;
    if ((dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) ||
        r[0] * r[0] + r[1] * r[1] + r[2] * r[2] == 0.0)
      zero = true;
  } else {
    int s = slot - n_m2l;
    kind = s < 8 ? 1 : 2;
    int c = s & 7;
    r[0] = (2 * (c & 1) - 1) * ax * 0.25;
    r[1] = (2 * ((c >> 1) & 1) - 1) * ay * 0.25;
    r[2] = (2 * ((c >> 2) & 1) - 1) * az * 0.25;
  }
  if (threadIdx.x == 0 && !zero) {
    if (kind == 0) irregular_s(2 * p, r, H);
    else regular_s(p, r, H);
  }
  __syncthreads();
  float *T = tab + (size_t)slot * K * KP;
  for (int e = threadIdx.x; e < K * KP; e += blockDim.x) {
    int in = e / KP, out = e % KP;
    double val = 0.0;
    if (!zero && out < K) {
      int k, l, po, n, mp, pi;
      dec_idx(out, k, l, po);
      dec_idx(in, n, mp, pi);
      if (mp == 0) {
        cd A = op_coef(kind, H, k, l, n, 0);
        val = po ? A.im : A.re;
      } else {
        cd A = op_coef(kind, H, k, l, n, mp);
        cd B = op_coef(kind, H, k, l, n, -mp);
        if (mp & 1) B = {-B.re, -B.im};
        cd S = cadd(A, B), Dd = csub(A, B);
        if (pi == 0) val = po ? S.im : S.re;
        else val = po ? Dd.re : -Dd.im;
      }
    }
    T[e] = (float)val;
    if (tab64 && slot < n_m2l) tab64[(size_t)slot * K * KP + e] = val;
  }
}

// ------------------------------------------------------------------- 2D
// Expansion of order p: a_0 real then (Re a_k, Im a_k) for k = 1..p
// (K = 2p+1).  Local: (Re b_0) then (Re b_n, Im b_n).  The M2L matrix of
// offset rho is built for a unit cell size; the level-dependent a_0 log(s)
// term of b_0 only affects the potential and is added in the L2P pass.
__device__ inline double binom_d(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double b = 1.0;
  for (int i = 1; i <= k; ++i) b = b * (n - k + i) / i;
  return b;
}

__device__ inline void dec2(int i, int &k, int &im) {
  if (i == 0) {
    k = 0;
    im = 0;
  } else {
    k = (i + 1) / 2;
    im = (i & 1) ? 0 : 1;
  }
}

__device__ inline cd cpow_i(cd z, int k) {
  cd r = {1.0, 0.0};
  for (int i = 0; i < k; ++i) r = cmul(r, z);
  return r;
}

__device__ inline cd cinv(cd z) {
  double d = z.re * z.re + z.im * z.im;
  return {z.re / d, -z.im / d};
}

// Complex coefficient C(out n, in k) such that out_n = sum_k C x_k, with x
// complex (a_k, b_k) and out complex; kinds as in 3D.
__device__ inline cd op2_coef(int kind, cd z, int n, int k) {
  if (kind == 0) {  // M2L, multipole_set2D.cpp:53-88; z = rho
    cd iz = cinv(z);
    if (n == 0) {
      if (k == 0) {
        // a_0 log z: real part log|z| (imag part irrelevant to grad/phi)
        return {0.5 * log(z.re * z.re + z.im * z.im), atan2(z.im, z.re)};
      }
      cd v = cscale(cpow_i(iz, k), -1.0 / k);
      return v;
    }
    double sign = (n & 1) ? 1.0 : -1.0;
    if (k == 0) return cscale(cpow_i(iz, n), sign / n);
    return cscale(cpow_i(iz, n + k), sign * binom_d(n + k - 1, k - 1) / k);
  } else if (kind == 1) {  // M2M, multipole_set2D.cpp:20-51: a'_n = sum C(n,j) d^(n-j) a_j 2^-j
    if (k > n) return {0.0, 0.0};
    return cscale(cpow_i(z, n - k), binom_d(n, k) * ldexp(1.0, -k));
  } else {  // L2L, local_set2D.cpp:42-58: b'_n = sum_{j>=n} C(j,n) t^(j-n) b_j 2^-n
    if (k < n) return {0.0, 0.0};
    return cscale(cpow_i(z, k - n), binom_d(k, n) * ldexp(1.0, -n));
  }
}

// 2D M2L tables are per level: the physical offset is s_d * rho, and
// a_0 log(s_d rho) adds a_0 log(s_d) to b_0 (log_s0 = log s_0, s_d = s_0 2^-d).
__global__ void k_build_ops2d(float *tab, int p, int K, int KP, int n_m2l, double ax, double ay, double log_s0) {
  const int slot = blockIdx.x;
  int kind;
  cd z;
  bool zero = false;
  double log_s = 0.0;
  if (slot < n_m2l) {
    kind = 0;
    const int lev = slot / 49, off = slot % 49;
    log_s = log_s0 - lev * 0.69314718055994530942;
    int dx = off % 7 - 3, dy = off / 7 - 3;  // source - target
    z = {-dx * ax, -dy * ay};
    if ((dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1) || (z.re == 0.0 && z.im == 0.0)) zero = true;
  } else {
    int s = slot - n_m2l;
    kind = s < 4 ? 1 : 2;
    int c = s & 3;
    z = {(2 * (c & 1) - 1) * ax * 0.25, (2 * ((c >> 1) & 1) - 1) * ay * 0.25};
  }
  float *T = tab + (size_t)slot * K * KP;
  for (int e = threadIdx.x; e < K * KP; e += blockDim.x) {
    int in = e / KP, out = e % KP;
    double val = 0.0;
    if (!zero && out < K) {
      int n, po, k, pi;
      dec2(out, n, po);
      dec2(in, k, pi);
      cd C = op2_coef(kind, z, n, k);
      if (kind == 0 && n == 0 && k == 0) C.re += log_s;
      // x_k = a + i b: out += C a  (pi = 0),  out += C i b (pi = 1)
      if (pi == 0) val = po ? C.im : C.re;
      else val = po ? C.re : -C.im;
    }
    T[e] = (float)val;
  }
}

int build_op_tables(OpTables &ops, int dim, int p, int depth, const PassGeom &g, cudaStream_t st, int64_t &launches,
                    bool want64) {
  int K = dim == 3 ? (p + 1) * (p + 1) : 2 * p + 1;
  int KP = 32 * ((K + 31) / 32);
  int KS = (K + 3) & ~3;
  ops.dim = dim;
  ops.p = p;
  ops.K = K;
  ops.KP = KP;
  ops.KS = KS;
  ops.n_m2l = dim == 3 ? 343 : 49 * (depth + 1);
  ops.off_m2m = ops.n_m2l;
  ops.off_l2l = ops.n_m2l + (1 << dim);
  ops.n_slots = ops.n_m2l + 2 * (1 << dim);
  if (!ops.tab.reserve((size_t)ops.n_slots * K * KP)) return FMM_ERR_OUT_OF_MEMORY;
  double emax = g.emax > 0 ? g.emax : 1.0;
  double a[3] = {g.ext[0] / emax, g.ext[1] / emax, dim == 3 ? g.ext[2] / emax : 0.0};
  if (dim == 3) {
    size_t sh = sizeof(double) * 2 * (size_t)(2 * p + 1) * (2 * p + 2) / 2;
    double *t64 = nullptr;
    if (want64) {
      if (!ops.tab64.reserve((size_t)ops.n_m2l * K * KP)) return FMM_ERR_OUT_OF_MEMORY;
      t64 = ops.tab64.ptr;
    }
    k_build_ops3d<<<ops.n_slots, 256, sh, st>>>(ops.tab.ptr, t64, p, K, KP, ops.n_m2l, a[0], a[1], a[2]);
  } else {
    k_build_ops2d<<<ops.n_slots, 256, 0, st>>>(ops.tab.ptr, p, K, KP, ops.n_m2l, a[0], a[1], std::log(emax));
  }
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

}  // namespace fmm
