// Learned expansion order of the M2L tiles: cell and tile features, the FP64
// error probe that labels training tiles, the MLP (forward, backward, Adam)
// and the hot-path inference that sets each M2L tile's order.
//
// MLP: 32 inputs -> 64 -> 64 -> 9, ReLU, weights and activations rounded to
// BF16 (round to nearest) before every product, FP32 accumulation, FP32
// biases; the FP32 master weights take the gradients (straight-through).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "order.cuh"

namespace fmm {

__device__ inline float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// ---------------------------------------------------------------- features
// Cell features, ORD_CF values per cell stored as BF16 (32 bytes: one memory
// sector, so the per-pair gathers of the tile features read one sector per
// cell; the MLP rounds its inputs to BF16 in any case).
__global__ void k_cell_features(const float *M, const int *pbeg, const int *pend, int first, int count, int cell0,
                                int p, int KS, const uint8_t *mode, uint16_t *cf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int c = first + i;
  if (mode && !mode[c - cell0]) return;
  const float *m = M + (size_t)(c - cell0) * KS;
  float o[ORD_CF];
  const float m0 = fabsf(m[0]);
  o[0] = log2f(1.f + (float)(pend[c] - pbeg[c]));
  for (int n = 1; n <= 12; ++n) {
    float v = -30.f;
    if (n <= p && m0 > 0.f) {
      float s = m[re_idx(n, 0)] * m[re_idx(n, 0)];
      for (int k = 1; k <= n; ++k) s += 2.f * (m[re_idx(n, k)] * m[re_idx(n, k)] + m[im_idx(n, k)] * m[im_idx(n, k)]);
      v = s > 0.f ? fmaxf(log10f(sqrtf(s) / m0), -30.f) : -30.f;
    }
    o[n] = v;
  }
  o[13] = m0 > 0.f ? log10f(m0) : -30.f;
  o[14] = o[15] = 0.f;
  uint32_t w[ORD_CF / 2];
#pragma unroll
  for (int k = 0; k < ORD_CF / 2; ++k) {
    const __nv_bfloat162 t = __floats2bfloat162_rn(o[2 * k], o[2 * k + 1]);
    w[k] = *reinterpret_cast<const uint32_t *>(&t);
  }
  uint4 *dst = reinterpret_cast<uint4 *>(cf + (size_t)(c - cell0) * ORD_CF);
  dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
  dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// The 16 BF16 features of a cell, as floats.
__device__ inline void load_cf(const uint16_t *cf, float *f) {
  const uint4 *src = reinterpret_cast<const uint4 *>(cf);
  const uint4 a = src[0], b = src[1];
  const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    f[2 * k] = __uint_as_float(w[k] << 16);
    f[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
  }
}

__global__ void k_mass_total(const float4 *part, int64_t n, double *mtot) {
  __shared__ double s[8];
  double v = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v += (double)part[i].w;
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    atomicAdd(mtot, t);
  }
}

__device__ inline unsigned long long splitmix(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Warp-wide maximum of a non-NaN float in one redux.sync: the float's bits
// mapped to an int of the same order (negative values have their magnitude
// bits flipped).
__device__ inline float warp_max(float v) {
  const int i = __float_as_int(v);
  const int m = __reduce_max_sync(0xffffffffu, i >= 0 ? i : i ^ 0x7fffffff);
  return __int_as_float(m >= 0 ? m : m ^ 0x7fffffff);
}

// Features of tile (batch b, present slot i), computed by one warp (lanes
// over the 128 rows); every lane returns all of them.  Also returns the
// offset slot and the level.
__device__ void tile_features(const TileArgs &a, int b, int i, int lane, float *f, int &off, int &level) {
  const int4 bt = a.batches[b];
  const size_t base = (size_t)b * 189;
  const int sl = a.slot_list[base + i];
  off = a.tslot_list[base + i];
  level = bt.z;
  float mT = 0.f, mS = 0.f, sp1 = -30.f, sp2 = -30.f, mA[13];
#pragma unroll
  for (int n = 0; n < 13; ++n) mA[n] = -60.f;
  int cnt = 0;
  for (int r = lane; r < bt.y; r += 32) {
    const int S = a.src_tab[(base + sl) * 128 + r];
    if (S < 0) continue;
    const int T = a.tlist[bt.x + r];
    float cT[ORD_CF], cS[ORD_CF];
    load_cf(a.cf + (size_t)(T - a.cell0) * ORD_CF, cT);
    load_cf(a.cf + (size_t)(S - a.cell0) * ORD_CF, cS);
    mT = fmaxf(mT, cT[0]);
    mS = fmaxf(mS, cS[0]);
    sp1 = fmaxf(sp1, cT[1]);
    sp2 = fmaxf(sp2, cT[2]);
    const float l0 = cS[13];
    mA[0] = fmaxf(mA[0], l0);
#pragma unroll
    for (int n = 1; n < 13; ++n) mA[n] = fmaxf(mA[n], l0 + cS[n]);
    ++cnt;
  }
  mT = warp_max(mT);
  mS = warp_max(mS);
  sp1 = warp_max(sp1);
  sp2 = warp_max(sp2);
#pragma unroll
  for (int n = 0; n < 13; ++n) mA[n] = warp_max(mA[n]);
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  const float lmt = log10f((float)fmax(*a.mtot, 1e-300));
  f[0] = level * (1.f / 16.f);
  f[1] = mT * 0.125f;
  f[2] = mS * 0.125f;
#pragma unroll
  for (int n = 0; n < 13; ++n) f[3 + n] = fmaxf(mA[n] - lmt, -40.f) * 0.25f;
  f[16] = sp1 * 0.25f;
  f[17] = sp2 * 0.25f;
  f[18] = cnt * (1.f / 128.f);
  const int dx = off % 7 - 3, dy = (off / 7) % 7 - 3, dz = off / 49 - 3;
  float e0 = fabsf((float)dx) * a.ax, e1 = fabsf((float)dy) * a.ay, e2 = fabsf((float)dz) * a.az;
  const float R = sqrtf(e0 * e0 + e1 * e1 + e2 * e2);
  f[19] = R * 0.25f;
  if (e0 < e1) { const float t = e0; e0 = e1; e1 = t; }
  if (e1 < e2) { const float t = e1; e1 = e2; e2 = t; }
  if (e0 < e1) { const float t = e0; e0 = e1; e1 = t; }
  f[20] = e0 * (1.f / 3.f);
  f[21] = e1 * (1.f / 3.f);
  f[22] = e2 * (1.f / 3.f);
  const float diag = sqrtf(a.ax * a.ax + a.ay * a.ay + a.az * a.az);
  f[23] = R > 0.f ? log10f(diag / R) : 0.f;
#pragma unroll
  for (int k = 24; k < ORD_NF; ++k) f[k] = 0.f;
  if (cnt == 0) {
#pragma unroll
    for (int k = 0; k < ORD_NF; ++k) f[k] = 0.f;
  }
}

// One warp per sampled tile.
__global__ void k_order_sample_tiles(TileArgs a, int nbm, int n, unsigned long long seed, int2 *tiles, float *feat,
                                     int4 *pairs) {
  const int lane = threadIdx.x & 31;
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= n) return;
  const unsigned long long h = splitmix(seed * 0x100000001B3ull + (unsigned long long)k);
  const int b = (int)(h % (unsigned long long)nbm);
  const int ns = a.nslots[b];
  int4 *pr = pairs + (size_t)k * 128;
  if (ns == 0) {
    if (lane == 0) tiles[k] = make_int2(-1, -1);
    for (int r = lane; r < 128; r += 32) pr[r] = make_int4(-1, -1, -1, -1);
    for (int q = lane; q < ORD_NF; q += 32) feat[(size_t)k * ORD_NF + q] = 0.f;
    return;
  }
  const int i = (int)((h >> 20) % (unsigned long long)ns);
  float f[ORD_NF];
  int off, level;
  tile_features(a, b, i, lane, f, off, level);
  if (lane == 0) tiles[k] = make_int2(b, i);
  for (int q = 0; q < ORD_NF; ++q)
    if (lane == q) feat[(size_t)k * ORD_NF + q] = f[q];
  const int4 bt = a.batches[b];
  const size_t base = (size_t)b * 189;
  const int sl = a.slot_list[base + i];
  for (int r = lane; r < 128; r += 32) {
    int4 v = make_int4(-1, -1, -1, -1);
    if (r < bt.y) {
      const int S = a.src_tab[(base + sl) * 128 + r];
      if (S >= 0) v = make_int4(a.tlist[bt.x + r], S, off, level);
    }
    pr[r] = v;
  }
}

__global__ void k_tile_labels(const float *pl, int n, const double *mtot, float *labels, float *feat) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float lmt = log10f((float)fmax(*mtot, 1e-300));
  float mx[ORD_NQ];
  bool any = false;
  for (int q = 0; q < ORD_NQ; ++q) mx[q] = -1e30f;
  for (int r = 0; r < 128; ++r) {
    const float *l = pl + ((size_t)k * 128 + r) * ORD_NQ;
    if (l[0] < -1e29f) continue;
    any = true;
    for (int q = 0; q < ORD_NQ; ++q) mx[q] = fmaxf(mx[q], l[q]);
  }
  for (int q = 0; q < ORD_NQ; ++q) labels[(size_t)k * ORD_NQ + q] = any ? mx[q] - lmt : 0.f;
  if (!any)
    for (int q = 0; q < ORD_NF; ++q) feat[(size_t)k * ORD_NF + q] = 0.f;
}

// ---------------------------------------------------------------- FP64 probe
__device__ inline void lget_d(const double *L, int n, int m, double &re, double &im) {
  if (m > n) {
    re = im = 0.0;
  } else if (m >= 0) {
    re = L[re_idx(n, m)];
    im = m ? L[im_idx(n, m)] : 0.0;
  } else {  // L_n^-1 = -conj(L_n^1)
    re = -L[re_idx(n, 1)];
    im = L[im_idx(n, 1)];
  }
}

// Gradient of the order-q local expansion L^ (scaled units) at x: the same
// recurrences of the scaled regular harmonics as the FP32 L2P, in FP64.
__device__ void l2p_grad_d(const double *L, int q, double x, double y, double z, double &gx, double &gy,
                           double &gz) {
  const double r2 = x * x + y * y + z * z;
  double dre = 1.0, dim = 0.0;
  gx = gy = gz = 0.0;
  for (int m = 0; m <= q; ++m) {
    if (m > 0) {
      const double h = -0.5 / m;
      const double nre = h * (x * dre - y * dim), nim = h * (x * dim + y * dre);
      dre = nre;
      dim = nim;
    }
    const double wm = m ? 2.0 : 1.0;
    double p1re = dre, p1im = dim, p2re = 0.0, p2im = 0.0;
    for (int l = m; l < q; ++l) {
      double cre, cim;
      if (l == m) {
        cre = dre;
        cim = dim;
      } else {
        const double den = (double)(l * l - m * m);
        const double a1 = (2.0 * l - 1.0) * z / den, a2 = r2 / den;
        cre = a1 * p1re - a2 * p2re;
        cim = a1 * p1im - a2 * p2im;
        p2re = p1re;
        p2im = p1im;
        p1re = cre;
        p1im = cim;
      }
      double Ar, Ai, Mr, Mi, Pr, Pi;
      lget_d(L, l + 1, m, Ar, Ai);
      lget_d(L, l + 1, m - 1, Mr, Mi);
      lget_d(L, l + 1, m + 1, Pr, Pi);
      gz += wm * (Ar * cre - Ai * cim);
      gx += wm * (0.5 * (Mr - Pr) * cre - 0.5 * (Mi - Pi) * cim);
      gy += wm * 0.5 * ((Pr + Mr) * cim + (Pi + Mi) * cre);
    }
  }
}

static constexpr int PROBE_T = 256;
static constexpr int PROBE_MAX_NT = 256;

__global__ void __launch_bounds__(PROBE_T) k_probe(ProbeArgs a) {
  extern __shared__ double sh[];
  const int K = a.K;
  double *Ms = sh;                              // [K]
  double *Lq = Ms + K;                          // [ORD_NQ][K]
  double *Fx = Lq + ORD_NQ * K;                 // [PROBE_MAX_NT][3]
  double *e2 = Fx + 3 * PROBE_MAX_NT;           // [ORD_NQ]
  double *wpart = e2 + ORD_NQ;                  // [8][K] per-warp P2M partials
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int4 pr = reinterpret_cast<const int4 *>(a.pairs)[blockIdx.x];
  float *lab = a.labels + (size_t)blockIdx.x * ORD_NQ;
  if (pr.x < 0) {
    if (tid < ORD_NQ) lab[tid] = -1e30f;
    return;
  }
  const int T = pr.x, S = pr.y, d = pr.w;
  const int tb = a.pbeg[T], nt = a.pend[T] - tb, sb = a.pbeg[S], nsrc = a.pend[S] - sb;
  double cT[3], cS[3];
  {
    uint32_t q[3], r[3];
    morton_decode(3, a.ckey[T], q[0], q[1], q[2]);
    morton_decode(3, a.ckey[S], r[0], r[1], r[2]);
    for (int k = 0; k < 3; ++k) {
      const double sk = a.g.ext[k] * ldexp(1.0, -d);
      cT[k] = a.g.lo[k] + (q[k] + 0.5) * sk;
      cS[k] = a.g.lo[k] + (r[k] + 0.5) * sk;
    }
  }
  const double s = a.g.emax * ldexp(1.0, -d), inv_s = 1.0 / s;
  for (int i = tid; i < 8 * K; i += PROBE_T) wpart[i] = 0.0;
  for (int i = tid; i < ORD_NQ; i += PROBE_T) e2[i] = 0.0;
  __syncthreads();
  // P2M in FP64 about c_S: M~_l^m = sum w conj(Rs_l^m((x - c_S) / s)), per-warp sums
  for (int j0 = warp * 32; j0 < nsrc; j0 += PROBE_T) {
    const int j = j0 + lane;
    double x = 0.0, y = 0.0, z = 0.0, w = 0.0;
    if (j < nsrc) {
      const uint32_t o = a.perm[sb + j];
      x = (a.pos[3 * (size_t)o] - cS[0]) * inv_s;
      y = (a.pos[3 * (size_t)o + 1] - cS[1]) * inv_s;
      z = (a.pos[3 * (size_t)o + 2] - cS[2]) * inv_s;
      w = a.mass[o];
    }
    const double r2 = x * x + y * y + z * z;
    double dre = 1.0, dim = 0.0;
    for (int m = 0; m <= a.p; ++m) {
      if (m > 0) {
        const double h = -0.5 / m;
        const double nre = h * (x * dre - y * dim), nim = h * (x * dim + y * dre);
        dre = nre;
        dim = nim;
      }
      double p1re = dre, p1im = dim, p2re = 0.0, p2im = 0.0;
      for (int l = m; l <= a.p; ++l) {
        double cre, cim;
        if (l == m) {
          cre = dre;
          cim = dim;
        } else {
          const double den = (double)(l * l - m * m);
          const double a1 = (2.0 * l - 1.0) * z / den, a2 = r2 / den;
          cre = a1 * p1re - a2 * p2re;
          cim = a1 * p1im - a2 * p2im;
          p2re = p1re;
          p2im = p1im;
          p1re = cre;
          p1im = cim;
        }
        double vr = w * cre, vi = -w * cim;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          vr += __shfl_xor_sync(0xffffffffu, vr, o);
          vi += __shfl_xor_sync(0xffffffffu, vi, o);
        }
        if (lane == 0) {
          wpart[warp * K + re_idx(l, m)] += vr;
          if (m) wpart[warp * K + im_idx(l, m)] += vi;
        }
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < K; i += PROBE_T) {
    double v = 0.0;
    for (int w = 0; w < 8; ++w) v += wpart[w * K + i];
    Ms[i] = v;
  }
  __syncthreads();
  // M2L at every order q: cumulative sums over the input degrees
  const double *Tm = a.tab64 + (size_t)pr.z * K * a.KP;
  for (int k = tid; k < K; k += PROBE_T) {
    int dk = 0;
    while ((dk + 1) * (dk + 1) <= k) ++dk;
    double acc = 0.0;
    for (int dn = 0; dn <= a.p; ++dn) {
      for (int ni = dn * dn; ni < (dn + 1) * (dn + 1); ++ni) acc += Tm[(size_t)ni * a.KP + k] * Ms[ni];
      if (dn >= ORD_QMIN && dn <= ORD_QMAX) Lq[(dn - ORD_QMIN) * K + k] = dk <= dn ? acc : 0.0;
    }
  }
  // exact far field of S on the target particles (FP64)
  const int ntc = min(nt, PROBE_MAX_NT);
  for (int i = tid; i < ntc; i += PROBE_T) {
    const uint32_t o = a.perm[tb + i];
    const double xi = a.pos[3 * (size_t)o], yi = a.pos[3 * (size_t)o + 1], zi = a.pos[3 * (size_t)o + 2];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int j = 0; j < nsrc; ++j) {
      const uint32_t u = a.perm[sb + j];
      const double rx = xi - a.pos[3 * (size_t)u], ry = yi - a.pos[3 * (size_t)u + 1], rz = zi - a.pos[3 * (size_t)u + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      const double inv = 1.0 / sqrt(r2);
      const double w3 = a.mass[u] * inv * inv * inv;
      fx -= rx * w3;
      fy -= ry * w3;
      fz -= rz * w3;
    }
    Fx[3 * i] = fx;
    Fx[3 * i + 1] = fy;
    Fx[3 * i + 2] = fz;
  }
  __syncthreads();
  // truncated field at every order; squared error summed over the targets
  const int qhi = min(a.p, ORD_QMAX);
  const int nq = qhi - ORD_QMIN + 1;
  for (int e = tid; e < ntc * nq; e += PROBE_T) {
    const int i = e / nq, qi = e % nq;
    const uint32_t o = a.perm[tb + i];
    const double x = (a.pos[3 * (size_t)o] - cT[0]) * inv_s, y = (a.pos[3 * (size_t)o + 1] - cT[1]) * inv_s,
                 z = (a.pos[3 * (size_t)o + 2] - cT[2]) * inv_s;
    double gx, gy, gz;
    l2p_grad_d(Lq + qi * K, ORD_QMIN + qi, x, y, z, gx, gy, gz);
    const double s2 = inv_s * inv_s;
    const double ex = gx * s2 - Fx[3 * i], ey = gy * s2 - Fx[3 * i + 1], ez = gz * s2 - Fx[3 * i + 2];
    atomicAdd(&e2[qi], ex * ex + ey * ey + ez * ez);
  }
  __syncthreads();
  if (tid < ORD_NQ) {
    float v = 0.f;
    if (tid < nq) {
      double R2 = 0.0;
      for (int k = 0; k < 3; ++k) R2 += (cS[k] - cT[k]) * (cS[k] - cT[k]);
      v = (float)log10(sqrt(e2[tid] / (double)ntc) * R2 + 1e-300);
    }
    lab[tid] = v;
  }
}

// ---------------------------------------------------------------- MLP
// Forward pass of one row with parameters in shared memory (weights already
// rounded to BF16).  h1, h2: BF16-rounded activations.
__device__ inline void mlp_forward(const float *w, const float *x, float *h1, float *h2, float *y) {
#pragma unroll 4
  for (int j = 0; j < ORD_NH; ++j) {
    float acc = w[ORD_B1 + j];
#pragma unroll
    for (int i = 0; i < ORD_NF; ++i) acc = fmaf(w[ORD_W1 + j * ORD_NF + i], x[i], acc);
    h1[j] = bf16r(fmaxf(acc, 0.f));
  }
#pragma unroll 2
  for (int j = 0; j < ORD_NH; ++j) {
    float acc = w[ORD_B2 + j];
#pragma unroll
    for (int i = 0; i < ORD_NH; ++i) acc = fmaf(w[ORD_W2 + j * ORD_NH + i], h1[i], acc);
    h2[j] = bf16r(fmaxf(acc, 0.f));
  }
#pragma unroll
  for (int o = 0; o < ORD_NQ; ++o) {
    float acc = w[ORD_B3 + o];
#pragma unroll
    for (int i = 0; i < ORD_NH; ++i) acc = fmaf(w[ORD_W3 + o * ORD_NH + i], h2[i], acc);
    y[o] = acc;
  }
}

// parameters into shared memory, weights rounded to BF16, biases FP32
__device__ inline void load_params(const float *params, float *w) {
  for (int i = threadIdx.x; i < ORD_NPARAM; i += blockDim.x) {
    const bool bias = (i >= ORD_B1 && i < ORD_W2) || (i >= ORD_B2 && i < ORD_W3) || i >= ORD_B3;
    w[i] = bias ? params[i] : bf16r(params[i]);
  }
}

static constexpr int MLP_ROWS = 128;  // rows per training block

// Forward + backward of MLP_ROWS rows per block; gradients of the mean
// squared error (over rows_total rows and the ORD_NQ outputs) added into
// grad, loss sum into *loss.  Rows at or beyond n are ignored.
__global__ void __launch_bounds__(MLP_ROWS) k_mlp_grad(const float *feat, const float *labels, int n, int row0,
                                                       int rows_total, const float *params, float *grad, float *loss,
                                                       float *pred) {
  extern __shared__ float shm[];
  float *w = shm;                               // ORD_NPARAM
  float *X = w + ORD_NPARAM;                    // [ROWS][NF]
  float *H1 = X + MLP_ROWS * ORD_NF;            // [ROWS][NH]
  float *H2 = H1 + MLP_ROWS * ORD_NH;           // [ROWS][NH]
  float *D2 = H2 + MLP_ROWS * ORD_NH;           // [ROWS][NH] dL/d(pre-activation 2)
  float *D1 = D2 + MLP_ROWS * ORD_NH;           // [ROWS][NH] dL/d(pre-activation 1)
  float *DY = D1 + MLP_ROWS * ORD_NH;           // [ROWS][16]
  const int t = threadIdx.x;
  load_params(params, w);
  __syncthreads();
  const int r = row0 + blockIdx.x * MLP_ROWS + t;
  const bool valid = r < n && r < row0 + rows_total;
  float x[ORD_NF], h1[ORD_NH], h2[ORD_NH], y[ORD_NQ];
  for (int i = 0; i < ORD_NF; ++i) x[i] = valid ? bf16r(feat[(size_t)r * ORD_NF + i]) : 0.f;
  mlp_forward(w, x, h1, h2, y);
  const float inv = 1.f / ((float)rows_total * ORD_NQ);
  float l = 0.f;
  for (int o = 0; o < 16; ++o) {
    float dy = 0.f;
    if (o < ORD_NQ && valid) {
      const float lab = fmaxf(labels[(size_t)r * ORD_NQ + o], -16.f);
      const float e = y[o] - lab;
      l += e * e;
      dy = 2.f * e * inv;
      if (pred) pred[(size_t)r * ORD_NQ + o] = y[o];
    }
    DY[t * 16 + o] = dy;
  }
  if (valid) atomicAdd(loss, l * inv);
  for (int i = 0; i < ORD_NF; ++i) X[t * ORD_NF + i] = x[i];
  for (int i = 0; i < ORD_NH; ++i) {
    H1[t * ORD_NH + i] = h1[i];
    H2[t * ORD_NH + i] = h2[i];
  }
  // back through layer 3 and the second ReLU
  for (int i = 0; i < ORD_NH; ++i) {
    float g = 0.f;
    for (int o = 0; o < ORD_NQ; ++o) g = fmaf(w[ORD_W3 + o * ORD_NH + i], DY[t * 16 + o], g);
    D2[t * ORD_NH + i] = h2[i] > 0.f ? g : 0.f;
  }
  // back through layer 2 and the first ReLU
  for (int i = 0; i < ORD_NH; ++i) {
    float g = 0.f;
    for (int j = 0; j < ORD_NH; ++j) g = fmaf(w[ORD_W2 + j * ORD_NH + i], D2[t * ORD_NH + j], g);
    D1[t * ORD_NH + i] = h1[i] > 0.f ? g : 0.f;
  }
  __syncthreads();
  // parameter gradients: sums over the block's rows
  for (int e = t; e < ORD_NPARAM; e += MLP_ROWS) {
    float g = 0.f;
    if (e < ORD_B1) {
      const int j = e / ORD_NF, i = e % ORD_NF;
      for (int k = 0; k < MLP_ROWS; ++k) g = fmaf(D1[k * ORD_NH + j], X[k * ORD_NF + i], g);
    } else if (e < ORD_W2) {
      const int j = e - ORD_B1;
      for (int k = 0; k < MLP_ROWS; ++k) g += D1[k * ORD_NH + j];
    } else if (e < ORD_B2) {
      const int j = (e - ORD_W2) / ORD_NH, i = (e - ORD_W2) % ORD_NH;
      for (int k = 0; k < MLP_ROWS; ++k) g = fmaf(D2[k * ORD_NH + j], H1[k * ORD_NH + i], g);
    } else if (e < ORD_W3) {
      const int j = e - ORD_B2;
      for (int k = 0; k < MLP_ROWS; ++k) g += D2[k * ORD_NH + j];
    } else if (e < ORD_B3) {
      const int o = (e - ORD_W3) / ORD_NH, i = (e - ORD_W3) % ORD_NH;
      if (o < ORD_NQ)
        for (int k = 0; k < MLP_ROWS; ++k) g = fmaf(DY[k * 16 + o], H2[k * ORD_NH + i], g);
    } else {
      const int o = e - ORD_B3;
      if (o < ORD_NQ)
        for (int k = 0; k < MLP_ROWS; ++k) g += DY[k * 16 + o];
    }
    if (g != 0.f) atomicAdd(&grad[e], g);
  }
}

__global__ void k_adam(float *params, float *grad, float *m, float *v, int step, float lr, float b1, float b2,
                       float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ORD_NPARAM) return;
  const bool pad = (i >= ORD_W3 + ORD_NQ * ORD_NH && i < ORD_B3) || i >= ORD_B3 + ORD_NQ;
  const float g = pad ? 0.f : grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g, vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.f - powf(b1, (float)step)), vh = vi / (1.f - powf(b2, (float)step));
  if (!pad) params[i] -= lr * mh / (sqrtf(vh) + eps);
  grad[i] = 0.f;
}

static size_t mlp_grad_smem() {
  return sizeof(float) * ((size_t)ORD_NPARAM + MLP_ROWS * ORD_NF + 4 * MLP_ROWS * ORD_NH + MLP_ROWS * 16);
}

// ---------------------------------------------------------------- inference
// Persistent blocks, each loading the weights into shared memory once (as
// BF16): a block takes M2L batches in turn and each warp takes groups of 16
// of the batch's present slots (tiles).  The warp computes the features of
// its 16 tiles (lanes over each tile's rows), then runs the MLP on all 16 at
// once with warp-level BF16 tensor-core products (mma.sync m16n8k16, FP32
// accumulation; rows = tiles, the layer outputs of one product are the
// inputs of the next in registers), then sets each tile's order: the lowest
// within the budget of its offset.
static constexpr int INF_WARPS = 8;
static constexpr int INF_T = 16;  // tiles per warp group (the product's M)

__device__ inline uint32_t bf2(float lo, float hi) {
  const __nv_bfloat162 t = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&t);
}

__device__ inline void mma16816(float *c, const uint32_t *a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One dense layer of the 16-tile group: out[16 x 8 NT] = in[16 x 16 KT] W^T
// + bias, ReLU (relu) and rounding to BF16 for the next layer's A fragments.
// W is [out][in] BF16 in shared memory with row stride ws (in 16-bit
// units); A fragments of k-step k are afrag[k][4].
template <int KT, int NT>
__device__ inline void mlp_layer(const uint32_t (*afrag)[4], const uint16_t *W, int ws, const float *bias, int lane,
                                 float (*c)[4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const float b0 = bias[nt * 8 + t4 * 2], b1 = bias[nt * 8 + t4 * 2 + 1];
    c[nt][0] = b0;
    c[nt][1] = b1;
    c[nt][2] = b0;
    c[nt][3] = b1;
    const uint16_t *wr = W + (size_t)(nt * 8 + g) * ws + t4 * 2;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const uint32_t w0 = *reinterpret_cast<const uint32_t *>(wr + kt * 16);
      const uint32_t w1 = *reinterpret_cast<const uint32_t *>(wr + kt * 16 + 8);
      mma16816(c[nt], afrag[kt], w0, w1);
    }
  }
}

// C fragments of n-tiles 2k and 2k+1 (ReLU, BF16) are the A fragment of k-step k.
template <int NT>
__device__ inline void relu_to_a(const float (*c)[4], uint32_t (*afrag)[4]) {
#pragma unroll
  for (int k = 0; k < NT / 2; ++k) {
    afrag[k][0] = bf2(fmaxf(c[2 * k][0], 0.f), fmaxf(c[2 * k][1], 0.f));
    afrag[k][1] = bf2(fmaxf(c[2 * k][2], 0.f), fmaxf(c[2 * k][3], 0.f));
    afrag[k][2] = bf2(fmaxf(c[2 * k + 1][0], 0.f), fmaxf(c[2 * k + 1][1], 0.f));
    afrag[k][3] = bf2(fmaxf(c[2 * k + 1][2], 0.f), fmaxf(c[2 * k + 1][3], 0.f));
  }
}

static constexpr int INF_W1S = ORD_NF + 8, INF_W2S = ORD_NH + 8;  // padded row strides (16-bit units)

__global__ void __launch_bounds__(32 * INF_WARPS) k_order_infer(InferArgs a, int nbm) {
  __shared__ __align__(16) uint16_t w1s[ORD_NH * INF_W1S], w2s[ORD_NH * INF_W2S], w3s[16 * INF_W2S];
  __shared__ float bias[2 * ORD_NH + 16];
  __shared__ __align__(16) uint16_t xs[INF_WARPS][INF_T][ORD_NF + 8];  // features, BF16, one row per tile
  __shared__ float ys[INF_WARPS][INF_T][17];                          // outputs
  __shared__ float thr_s[INF_WARPS][INF_T];
  __shared__ uint8_t empty_s[INF_WARPS][INF_T];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < ORD_NH * ORD_NF; e += blockDim.x)
    w1s[(e / ORD_NF) * INF_W1S + e % ORD_NF] = __bfloat16_as_ushort(__float2bfloat16_rn(a.params[ORD_W1 + e]));
  for (int e = tid; e < ORD_NH * ORD_NH; e += blockDim.x)
    w2s[(e / ORD_NH) * INF_W2S + e % ORD_NH] = __bfloat16_as_ushort(__float2bfloat16_rn(a.params[ORD_W2 + e]));
  for (int e = tid; e < 16 * ORD_NH; e += blockDim.x)
    w3s[(e / ORD_NH) * INF_W2S + e % ORD_NH] = __bfloat16_as_ushort(__float2bfloat16_rn(a.params[ORD_W3 + e]));
  for (int e = tid; e < ORD_NH; e += blockDim.x) {
    bias[e] = a.params[ORD_B1 + e];
    bias[ORD_NH + e] = a.params[ORD_B2 + e];
  }
  if (tid < 16) bias[2 * ORD_NH + tid] = a.params[ORD_B3 + tid];
  __syncthreads();
  const double frms = *a.frms;
  const double pbar = a.n > 0 ? (double)(*a.nt_sum) / (double)a.n : 1.0;
  const float lmt = log10f((float)fmax(*a.t.mtot, 1e-300));
  const int g = lane >> 2, t4 = lane & 3;
  for (int b = blockIdx.x; b < nbm; b += gridDim.x) {
    const int ns = a.t.nslots[b];
    const size_t base = (size_t)b * 189;
    const float sd = (float)(a.emax * ldexp(1.0, -a.t.batches[b].z));
    for (int i0 = warp * INF_T; i0 < ns; i0 += INF_WARPS * INF_T) {
      const int nt = min(INF_T, ns - i0);
      if (frms <= 0.0) {  // no budget yet (the system's first evaluation): every tile at p
        if (lane < nt) {
          const int K = (a.p + 1) * (a.p + 1);
          a.slot_p16[base + i0 + lane] = (uint8_t)((K + 15) & ~15);
        }
        continue;
      }
      // features of the group's tiles, one row each (zero rows past the end)
      for (int tt = 0; tt < INF_T; ++tt) {
        float f[ORD_NF];
        int off = 0, level = 0;
        if (tt < nt) {
          tile_features(a.t, b, i0 + tt, lane, f, off, level);
        } else {
#pragma unroll
          for (int k = 0; k < ORD_NF; ++k) f[k] = 0.f;
        }
        if (lane == 0) {
#pragma unroll
          for (int k = 0; k < ORD_NF; k += 2)
            *reinterpret_cast<uint32_t *>(&xs[warp][tt][k]) = bf2(f[k], f[k + 1]);
          const int dx = off % 7 - 3, dy = (off / 7) % 7 - 3, dz = off / 49 - 3;
          const float ex = dx * a.t.ax * sd, ey = dy * a.t.ay * sd, ez = dz * a.t.az * sd;
          const float R2 = ex * ex + ey * ey + ez * ez;
          thr_s[warp][tt] = log10f(a.tol * (float)frms * R2 / (float)sqrt(pbar)) - lmt;
          empty_s[warp][tt] = f[18] == 0.f;
        }
      }
      __syncwarp();
      // the MLP on the 16 tiles
      uint32_t a1[2][4];
#pragma unroll
      for (int kt = 0; kt < 2; ++kt) {
        a1[kt][0] = *reinterpret_cast<const uint32_t *>(&xs[warp][g][kt * 16 + t4 * 2]);
        a1[kt][1] = *reinterpret_cast<const uint32_t *>(&xs[warp][g + 8][kt * 16 + t4 * 2]);
        a1[kt][2] = *reinterpret_cast<const uint32_t *>(&xs[warp][g][kt * 16 + t4 * 2 + 8]);
        a1[kt][3] = *reinterpret_cast<const uint32_t *>(&xs[warp][g + 8][kt * 16 + t4 * 2 + 8]);
      }
      float c1[8][4];
      mlp_layer<2, 8>(a1, w1s, INF_W1S, bias, lane, c1);
      uint32_t a2[4][4];
      relu_to_a<8>(c1, a2);
      float c2[8][4];
      mlp_layer<4, 8>(a2, w2s, INF_W2S, bias + ORD_NH, lane, c2);
      uint32_t a3[4][4];
      relu_to_a<8>(c2, a3);
      float c3[2][4];
      mlp_layer<4, 2>(a3, w3s, INF_W2S, bias + 2 * ORD_NH, lane, c3);
#pragma unroll
      for (int nt2 = 0; nt2 < 2; ++nt2) {
        ys[warp][g][nt2 * 8 + t4 * 2] = c3[nt2][0];
        ys[warp][g][nt2 * 8 + t4 * 2 + 1] = c3[nt2][1];
        ys[warp][g + 8][nt2 * 8 + t4 * 2] = c3[nt2][2];
        ys[warp][g + 8][nt2 * 8 + t4 * 2 + 1] = c3[nt2][3];
      }
      __syncwarp();
      // each tile's order: the lowest q in 4..p-1 whose predicted error is within its budget, else p
      if (lane < nt) {
        int q = a.p;
        for (int k = 0; k < ORD_NQ; ++k)
          if (ORD_QMIN + k < a.p && ys[warp][lane][k] <= thr_s[warp][lane]) {
            q = ORD_QMIN + k;
            break;
          }
        if (empty_s[warp][lane]) q = ORD_QMIN;  // no pair in the tile
        const int K = (q + 1) * (q + 1);
        a.slot_p16[base + i0 + lane] = (uint8_t)((K + 15) & ~15);
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------- F_rms
__global__ void k_force_sq(const double *acc, int64_t n, int dim, double invG2, double *out) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int d = 0; d < dim; ++d) v += acc[dim * i + d] * acc[dim * i + d];
    s += v;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s * invG2);
}

__global__ void k_force_rms_final(const double *sum, int64_t n, double *frms) {
  *frms = n > 0 ? sqrt(*sum / (double)n) : 0.0;
}

__global__ void k_judge_compare(const double *acc, const double *ref, const int64_t *targets, int64_t nt, int dim,
                                double *out) {
  double e = 0.0, r = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = targets[k];
    for (int d = 0; d < dim; ++d) {
      const double a = acc[dim * i + d], b = ref[dim * k + d];
      e += (a - b) * (a - b);
      r += b * b;
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], e);
    atomicAdd(&out[1], r);
  }
}

// ---------------------------------------------------------------- host
int order_judge_compare(const double *acc, const double *ref, const int64_t *targets, int64_t nt, int dim, double *out,
                        cudaStream_t st, int64_t &launches) {
  CUDA_TRY(cudaMemsetAsync(out, 0, 2 * sizeof(double), st));
  k_judge_compare<<<std::max(1, std::min(cdiv(nt, 256), 148)), 256, 0, st>>>(acc, ref, targets, nt, dim, out);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_cell_features(const float *M, const int *pbeg, const int *pend, int first, int count, int cell0, int p,
                        int KS, const uint8_t *mode, uint16_t *cf, const float4 *part, int64_t n, double *mtot,
                        cudaStream_t st, int64_t &launches) {
  CUDA_TRY(cudaMemsetAsync(mtot, 0, sizeof(double), st));
  if (n > 0) {
    k_mass_total<<<std::max(1, std::min(cdiv(n, 256), 148 * 2)), 256, 0, st>>>(part, n, mtot);
    launches += 1;
  }
  if (count <= 0) return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
  k_cell_features<<<cdiv(count, 256), 256, 0, st>>>(M, pbeg, pend, first, count, cell0, p, KS, mode, cf);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_sample_tiles(const TileArgs &a, int nbm, int n, unsigned long long seed, int *tiles, float *feat,
                       int *pairs, cudaStream_t st, int64_t &launches) {
  if (n <= 0 || nbm <= 0) return FMM_OK;
  k_order_sample_tiles<<<cdiv((int64_t)n * 32, 256), 256, 0, st>>>(a, nbm, n, seed, reinterpret_cast<int2 *>(tiles),
                                                                   feat, reinterpret_cast<int4 *>(pairs));
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_tile_labels(const float *pair_labels, int n, const double *mtot, float *labels, float *feat,
                      cudaStream_t st, int64_t &launches) {
  if (n <= 0) return FMM_OK;
  k_tile_labels<<<cdiv(n, 128), 128, 0, st>>>(pair_labels, n, mtot, labels, feat);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_probe_errors(const ProbeArgs &a, cudaStream_t st, int64_t &launches) {
  if (a.n <= 0) return FMM_OK;
  const size_t sh = sizeof(double) * ((size_t)a.K + ORD_NQ * (size_t)a.K + 3 * PROBE_MAX_NT + ORD_NQ + 8 * (size_t)a.K);
  if (sh > 227 * 1024) return FMM_ERR_UNSUPPORTED;
  if (cudaFuncSetAttribute(k_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
    return FMM_ERR_CUDA;
  k_probe<<<a.n, PROBE_T, sh, st>>>(a);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_infer(const InferArgs &a, int nbm, cudaStream_t st, int64_t &launches) {
  if (nbm <= 0) return FMM_OK;
  // persistent blocks: the weights are staged once per block
  k_order_infer<<<std::min(nbm, 148 * 4), 32 * INF_WARPS, 0, st>>>(a, nbm);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_forward_grad(const float *feat, const float *labels, int n, const float *params, float *pred, float *grad,
                       float *loss, cudaStream_t st, int64_t &launches) {
  if (n <= 0) return FMM_OK;
  const size_t sh = mlp_grad_smem();
  if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
    return FMM_ERR_CUDA;
  if (cudaMemsetAsync(grad, 0, sizeof(float) * ORD_NPARAM, st) != cudaSuccess ||
      cudaMemsetAsync(loss, 0, sizeof(float), st) != cudaSuccess)
    return FMM_ERR_CUDA;
  k_mlp_grad<<<cdiv(n, MLP_ROWS), MLP_ROWS, sh, st>>>(feat, labels, n, 0, n, params, grad, loss, pred);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int order_train(const float *feat, const float *labels, int n, int epochs, int batch, float lr, float *params,
                float *loss_out, cudaStream_t st, int64_t &launches) {
  if (n <= 0 || epochs <= 0) return FMM_OK;
  batch = std::max(MLP_ROWS, (batch / MLP_ROWS) * MLP_ROWS);
  const size_t sh = mlp_grad_smem();
  if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
    return FMM_ERR_CUDA;
  DevBuf<float> gbuf, mbuf, vbuf, lbuf;
  if (!gbuf.reserve(ORD_NPARAM) || !mbuf.reserve(ORD_NPARAM) || !vbuf.reserve(ORD_NPARAM) || !lbuf.reserve(epochs))
    return FMM_ERR_OUT_OF_MEMORY;
  CUDA_TRY(cudaMemsetAsync(gbuf.ptr, 0, sizeof(float) * ORD_NPARAM, st));
  CUDA_TRY(cudaMemsetAsync(mbuf.ptr, 0, sizeof(float) * ORD_NPARAM, st));
  CUDA_TRY(cudaMemsetAsync(vbuf.ptr, 0, sizeof(float) * ORD_NPARAM, st));
  CUDA_TRY(cudaMemsetAsync(lbuf.ptr, 0, sizeof(float) * epochs, st));
  int step = 0;
  const int steps_per_epoch = (n + batch - 1) / batch;
  for (int e = 0; e < epochs; ++e) {
    for (int s = 0; s < steps_per_epoch; ++s) {
      const int row0 = s * batch, rows = std::min(batch, n - row0);
      k_mlp_grad<<<cdiv(rows, MLP_ROWS), MLP_ROWS, sh, st>>>(feat, labels, n, row0, rows, params, gbuf.ptr,
                                                              lbuf.ptr + e, nullptr);
      k_adam<<<cdiv(ORD_NPARAM, 256), 256, 0, st>>>(params, gbuf.ptr, mbuf.ptr, vbuf.ptr, ++step, lr, 0.9f, 0.999f,
                                                   1e-8f);
      launches += 2;
    }
  }
  CUDA_TRY(cudaGetLastError());
  std::vector<float> hl(epochs);
  CUDA_TRY(cudaMemcpyAsync(hl.data(), lbuf.ptr, sizeof(float) * epochs, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  for (int e = 0; e < epochs; ++e) loss_out[e] = hl[e] / (float)steps_per_epoch;
  return FMM_OK;
}

int order_force_rms(const double *acc, int64_t n, int dim, double G, double *scratch, double *frms, cudaStream_t st,
                    int64_t &launches) {
  CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(double), st));
  const double invG2 = G != 0.0 ? 1.0 / (G * G) : 1.0;
  k_force_sq<<<std::min(cdiv(n, 256), 148 * 8), 256, 0, st>>>(acc, n, dim, invG2, scratch);
  k_force_rms_final<<<1, 1, 0, st>>>(scratch, n, frms);
  launches += 2;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

}  // namespace fmm
