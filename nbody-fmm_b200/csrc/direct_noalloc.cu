// FP64 direct sum that allocates nothing (fmm_direct_noalloc).
//
// Some callers cannot allocate device memory at the moment they need forces:
// codes that hand all device memory to their own pool at start-up, callers
// running under a fixed memory budget, and host threads that must not
// synchronise the device (cudaMalloc and cudaFree can).  For them this entry
// point needs no context and no allocation: the caller passes its own device
// buffers for inputs and outputs, and the only scratch is the fixed array
// below, which every GPU that loads this library holds until the process
// exits.
//
// The sum is the same as fmm_direct_device's: targets are spread over
// blocks and sources over a second grid dimension, but instead of adding the
// partial sums of each source chunk into the output with atomics, each block
// writes them to the scratch array and a second kernel adds the chunks of
// every target in a fixed order (so the result is also deterministic).
#include <mutex>

#include "direct.cuh"

namespace fmm {

static constexpr int NA_THREADS = 256;
static constexpr int FMM_NOALLOC_MAX_DEVICES = 64;

// Partial sums (ax, ay, az, phi) of one (target, source chunk); a call uses
// ntargets * nchunks of them and writes every one it reads, so nothing needs
// clearing between calls (the array keeps the last call's contents).
static __device__ __align__(256) double4 g_noalloc_partials[FMM_NOALLOC_MAX_TARGETS];

static std::mutex g_noalloc_mutex;
static double4 *g_noalloc_ptr[FMM_NOALLOC_MAX_DEVICES] = {};
static int g_noalloc_sms[FMM_NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device, and that
// device's SM count (which sizes the source chunks).  In host code the
// array's name is only a stand-in, so the address must come from
// cudaGetSymbolAddress, once per device, with that device current.
static int noalloc_scratch(double4 **out, int *sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FMM_ERR_NO_DEVICE;
  if (dev < 0 || dev >= FMM_NOALLOC_MAX_DEVICES) return FMM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
      set_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_partials)", __FILE__, __LINE__);
      return FMM_ERR_CUDA;
    }
    int nsm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || nsm <= 0) {
      set_cuda_error(e, "cudaDeviceGetAttribute(cudaDevAttrMultiProcessorCount)", __FILE__, __LINE__);
      return FMM_ERR_CUDA;
    }
    g_noalloc_sms[dev] = nsm;
    g_noalloc_ptr[dev] = (double4 *)p;
  }
  *out = g_noalloc_ptr[dev];
  *sms = g_noalloc_sms[dev];
  return FMM_OK;
}

__global__ void k_direct_partials(const double *pos, const double *mass, int64_t n, const int64_t *targets, int64_t nt,
                                  int dim, double eps2, int soft_mode, int64_t chunk, double4 *partials) {
  __shared__ double4 sp[NA_THREADS];
  const int64_t ti = (int64_t)blockIdx.x * NA_THREADS + threadIdx.x;
  const bool act = ti < nt;
  const int64_t i = act ? (targets ? targets[ti] : ti) : 0;
  double xi = 0, yi = 0, zi = 0;
  if (act) {
    xi = pos[i * dim];
    yi = pos[i * dim + 1];
    zi = dim == 3 ? pos[i * dim + 2] : 0.0;
  }
  double ax = 0, ay = 0, az = 0, ph = 0;
  const int64_t j0 = (int64_t)blockIdx.y * chunk, j1 = min(n, j0 + chunk);
  for (int64_t jb = j0; jb < j1; jb += NA_THREADS) {
    const int64_t j = jb + threadIdx.x;
    sp[threadIdx.x] = j < j1 ? make_double4(pos[j * dim], pos[j * dim + 1], dim == 3 ? pos[j * dim + 2] : 0.0, mass[j])
                             : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = (int)min((int64_t)NA_THREADS, j1 - jb);
    if (act) {
      for (int k = 0; k < cnt; ++k) {
        if (jb + k == i) continue;
        const double4 q = sp[k];
        const double dx = xi - q.x, dy = yi - q.y, dz = zi - q.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        double f, pw;
        if (dim == 3) {
          if (soft_mode == FMM_SOFT_NAIVE_REF) {
            const double r = sqrt(r2);
            f = q.w / ((r2 + 1.0e-4) * r);
            pw = q.w / r;
          } else {
            const double ir = rsqrt(r2 + eps2);
            pw = q.w * ir;
            f = pw * ir * ir;
          }
        } else {
          const double rr = soft_mode == FMM_SOFT_NAIVE_REF ? r2 + 1.0e-4 : r2 + eps2;
          f = q.w / rr;
          pw = -0.5 * q.w * log(rr);
        }
        ax -= f * dx;
        ay -= f * dy;
        az -= f * dz;
        ph += pw;
      }
    }
    __syncthreads();
  }
  if (act) partials[(int64_t)blockIdx.y * nt + ti] = make_double4(ax, ay, az, ph);
}

__global__ void k_direct_reduce(const double4 *partials, int64_t nt, int nchunks, int dim, double G, double *acc,
                                double *pot) {
  const int64_t ti = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= nt) return;
  double4 s = make_double4(0, 0, 0, 0);
  for (int c = 0; c < nchunks; ++c) {
    const double4 v = partials[(int64_t)c * nt + ti];
    s.x += v.x;
    s.y += v.y;
    s.z += v.z;
    s.w += v.w;
  }
  acc[ti * dim] = G * s.x;
  acc[ti * dim + 1] = G * s.y;
  if (dim == 3) acc[ti * dim + 2] = G * s.z;
  if (pot) pot[ti] = G * s.w;
}

}  // namespace fmm

using namespace fmm;

extern "C" int fmm_direct_noalloc(int32_t dim, int64_t n, const double *d_pos, const double *d_mass, int64_t ntargets,
                                  const int64_t *d_targets, int32_t soft_mode, double eps2, double G, double *d_acc,
                                  double *d_pot, void *stream) {
  if ((dim != 2 && dim != 3) || n < 0 || ntargets < 0 || !(eps2 >= 0.0)) return FMM_ERR_INVALID_ARGUMENT;
  if (soft_mode != FMM_SOFT_PLUMMER && soft_mode != FMM_SOFT_NAIVE_REF) return FMM_ERR_INVALID_ARGUMENT;
  const int64_t nt = d_targets ? ntargets : n;
  if (nt > FMM_NOALLOC_MAX_TARGETS) return FMM_ERR_TOO_LARGE;
  if (nt == 0) return FMM_OK;
  if (n == 0) return FMM_ERR_INVALID_ARGUMENT;  // targets given but no particles
  if (!d_pos || !d_mass || !d_acc) return FMM_ERR_INVALID_ARGUMENT;
  double4 *scratch = nullptr;
  int sms = 0;
  int rc = noalloc_scratch(&scratch, &sms);
  if (rc) return rc;
  const int bx = (int)((nt + NA_THREADS - 1) / NA_THREADS);
  // about four blocks per SM, without exceeding the scratch or 4096 sources per chunk
  int64_t by = std::max<int64_t>(1, std::min<int64_t>(((int64_t)sms * 4 + bx - 1) / bx, (n + 4095) / 4096));
  by = std::min<int64_t>(by, FMM_NOALLOC_MAX_TARGETS / nt);
  const int64_t chunk = (n + by - 1) / by;
  cudaStream_t st = (cudaStream_t)stream;
  k_direct_partials<<<dim3(bx, (unsigned)by), NA_THREADS, 0, st>>>(d_pos, d_mass, n, d_targets, nt, dim, eps2,
                                                                   soft_mode, chunk, scratch);
  k_direct_reduce<<<bx, NA_THREADS, 0, st>>>(scratch, nt, (int)by, dim, G, d_acc, d_pot);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "fmm_direct_noalloc launch", __FILE__, __LINE__);
    return FMM_ERR_CUDA;
  }
  return FMM_OK;
}
