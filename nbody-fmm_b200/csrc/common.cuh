// Shared device/host helpers for the B200 FMM library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fmm_gpu.h"

#define FMM_MAX_P 16           // largest expansion order the kernels accept
#define FMM_MAX_DEPTH 32       // 2D max depth (tree.cpp:38 gives 16 in 3D, 32 in 2D)

// Device error word bits (ORed by kernels, read back after a pass).
#define FMM_DEV_ERR_NONFINITE_INPUT 1u
#define FMM_DEV_ERR_NONFINITE_OUTPUT 2u
#define FMM_DEV_ERR_LIST_OVERFLOW 4u
#define FMM_DEV_ERR_TIMEOUT 8u

namespace fmm {

// Real layout of an expansion of order p: for degree n the entries
// [Re(n,0), Re(n,1), Im(n,1), ..., Re(n,n), Im(n,n)] start at n*n, so an
// expansion holds (p+1)^2 floats (the same indexing as the reference's
// PowerSet<3>, power_set3D.cpp:50-63).
// Interaction-list pairs whose cells are not well separated for the box's
// aspect ratio (sum of the cells' radii over the distance of their centres
// above this) are summed directly instead of by M2L.
static constexpr double FMM_RHO_MAX = 0.9;

__host__ __device__ inline int re_idx(int n, int m) { return n * n + (m ? 2 * m - 1 : 0); }
__host__ __device__ inline int im_idx(int n, int m) { return n * n + 2 * m; }

// Order-preserving map from double to uint64 (for atomic min/max).
__device__ inline unsigned long long dbl_to_ordered(double v) {
  unsigned long long u = __double_as_longlong(v);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ inline double ordered_to_dbl(unsigned long long u) {
  u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double(u);
}

// Bit spreading for Morton codes: bit b of x goes to bit b*3 (3D) / b*2 (2D).
__host__ __device__ inline uint64_t spread3(uint64_t x) {
  x &= 0x1fffff;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}
__host__ __device__ inline uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
  x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
  x = (x ^ (x >> 8)) & 0x1f0000ff0000ffull;
  x = (x ^ (x >> 16)) & 0x1f00000000ffffull;
  x = (x ^ (x >> 32)) & 0x1fffffull;
  return (uint32_t)x;
}
__host__ __device__ inline uint64_t spread2(uint64_t x) {
  x &= 0xffffffffull;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}
__host__ __device__ inline uint32_t compact2(uint64_t x) {
  x &= 0x5555555555555555ull;
  x = (x | (x >> 1)) & 0x3333333333333333ull;
  x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x >> 4)) & 0x00ff00ff00ff00ffull;
  x = (x | (x >> 8)) & 0x0000ffff0000ffffull;
  x = (x | (x >> 16)) & 0x00000000ffffffffull;
  return (uint32_t)x;
}
// Morton::encode (morton_code.cpp:9-22): coordinate i's bit b at i + b*dim.
__host__ __device__ inline uint64_t morton_encode(int dim, uint32_t x, uint32_t y, uint32_t z) {
  return dim == 3 ? (spread3(x) | (spread3(y) << 1) | (spread3(z) << 2)) : (spread2(x) | (spread2(y) << 1));
}
__host__ __device__ inline void morton_decode(int dim, uint64_t k, uint32_t &x, uint32_t &y, uint32_t &z) {
  if (dim == 3) {
    x = compact3(k);
    y = compact3(k >> 1);
    z = compact3(k >> 2);
  } else {
    x = compact2(k);
    y = compact2(k >> 1);
    z = 0;
  }
}

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace fmm
