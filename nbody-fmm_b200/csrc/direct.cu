// FP64 O(N^2) direct summation on the GPU, the judge of every FMM result
// and the drop-in for NaiveUpdate::update (naive_update.cpp:9-35).
// Targets are split over blocks and sources over a second grid dimension;
// partial sums meet through FP64 atomics.
#include "direct.cuh"

namespace fmm {

static constexpr int DS_THREADS = 256;

__global__ void k_direct(const double *pos, const double *mass, int64_t n, const int64_t *targets, int64_t nt,
                         int dim, double eps2, int soft_mode, int64_t chunk, double G, double *acc, double *pot) {
  __shared__ double4 sp[DS_THREADS];
  const int64_t ti = (int64_t)blockIdx.x * DS_THREADS + threadIdx.x;
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
  for (int64_t jb = j0; jb < j1; jb += DS_THREADS) {
    int64_t j = jb + threadIdx.x;
    if (j < j1) {
      sp[threadIdx.x] = make_double4(pos[j * dim], pos[j * dim + 1], dim == 3 ? pos[j * dim + 2] : 0.0, mass[j]);
    } else {
      sp[threadIdx.x] = make_double4(0, 0, 0, 0);
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)DS_THREADS, j1 - jb);
    if (act) {
      for (int k = 0; k < cnt; ++k) {
        if (jb + k == i) continue;
        double4 q = sp[k];
        double dx = xi - q.x, dy = yi - q.y, dz = zi - q.z;
        double r2 = dx * dx + dy * dy + dz * dz;
        double f, pw;
        if (dim == 3) {
          if (soft_mode == FMM_SOFT_NAIVE_REF) {
            double r = sqrt(r2);
            f = q.w / ((r2 + 1.0e-4) * r);
            pw = q.w / r;
          } else {
            double ir = rsqrt(r2 + eps2);
            pw = q.w * ir;
            f = pw * ir * ir;
          }
        } else {
          double rr = soft_mode == FMM_SOFT_NAIVE_REF ? r2 + 1.0e-4 : r2 + eps2;
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
  if (act) {
    if (gridDim.y == 1) {
      acc[ti * dim] = G * ax;
      acc[ti * dim + 1] = G * ay;
      if (dim == 3) acc[ti * dim + 2] = G * az;
      if (pot) pot[ti] = G * ph;
    } else {
      atomicAdd(&acc[ti * dim], G * ax);
      atomicAdd(&acc[ti * dim + 1], G * ay);
      if (dim == 3) atomicAdd(&acc[ti * dim + 2], G * az);
      if (pot) atomicAdd(&pot[ti], G * ph);
    }
  }
}

int direct_sum(const double *d_pos, const double *d_mass, int64_t n, const int64_t *d_targets, int64_t nt, int dim,
               double eps2, int soft_mode, double G, double *d_acc, double *d_pot, cudaStream_t st, int64_t &launches) {
  if (nt <= 0 || n <= 0) return FMM_OK;
  int bx = (int)((nt + DS_THREADS - 1) / DS_THREADS);
  // enough source chunks to give ~4 blocks per SM
  int by = (int)std::max<int64_t>(1, std::min<int64_t>((148 * 4 + bx - 1) / bx, (n + 4095) / 4096));
  int64_t chunk = (n + by - 1) / by;
  if (by > 1) {
    cudaMemsetAsync(d_acc, 0, sizeof(double) * nt * dim, st);
    if (d_pot) cudaMemsetAsync(d_pot, 0, sizeof(double) * nt, st);
  }
  dim3 grid(bx, by);
  k_direct<<<grid, DS_THREADS, 0, st>>>(d_pos, d_mass, n, d_targets, nt, dim, eps2, soft_mode, chunk, G, d_acc, d_pot);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

// ---------------------------------------------------------- integrators
// SyplecticEuler::integrate (symplectic_euler.cpp:10-14): v += dt a; x += dt v.
__global__ void k_se_update(double *x, double *v, const double *a, int64_t nd, double dt) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  double vv = v[i] + dt * a[i];
  v[i] = vv;
  x[i] += dt * vv;
}

// Classical RK4 for x' = v, v' = a(x).  From stage s (position x_s,
// velocity v_s, acceleration a_s = a(x_s); x_1 = x0, v_1 = v0):
//   v_{s+1} = v0 + c_s dt a_s,   x_{s+1} = x0 + c_s dt v_s,   c = 1/2, 1/2, 1
// and finally
//   v += dt/6 (a1 + 2a2 + 2a3 + a4),  x += dt/6 (v1 + 2v2 + 2v3 + v4),
// which is what runge_kutta_4.cpp:10-93 sets out to compute.  `cdt` is
// c_s * dt and `wprev` the weight of stage s in the final sums.
__global__ void k_rk4_stage(const double *x0, const double *v0, const double *a_prev, double *xs, double *vs,
                            double *asum, double *vsum, int64_t nd, double cdt, double wprev, int first) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  double vprev = first ? v0[i] : vs[i];
  double as = first ? 0.0 : asum[i], vsm = first ? 0.0 : vsum[i];
  asum[i] = as + wprev * a_prev[i];
  vsum[i] = vsm + wprev * vprev;
  vs[i] = v0[i] + cdt * a_prev[i];
  xs[i] = x0[i] + cdt * vprev;
}

__global__ void k_rk4_final(double *x, double *v, const double *a4, const double *v4, const double *asum,
                            const double *vsum, int64_t nd, double dt) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  double as = asum[i] + a4[i], vsm = vsum[i] + v4[i];
  v[i] += dt / 6.0 * as;
  x[i] += dt / 6.0 * vsm;
}

void se_update(double *x, double *v, const double *a, int64_t nd, double dt, cudaStream_t st, int64_t &launches) {
  k_se_update<<<(int)((nd + 255) / 256), 256, 0, st>>>(x, v, a, nd, dt);
  launches += 1;
}

void rk4_stage(const double *x0, const double *v0, const double *a_prev, double *xs, double *vs, double *asum,
               double *vsum, int64_t nd, double c, double wprev, int first, cudaStream_t st, int64_t &launches) {
  k_rk4_stage<<<(int)((nd + 255) / 256), 256, 0, st>>>(x0, v0, a_prev, xs, vs, asum, vsum, nd, c, wprev, first);
  launches += 1;
}

void rk4_final(double *x, double *v, const double *a4, const double *v4, const double *asum, const double *vsum,
               int64_t nd, double dt, cudaStream_t st, int64_t &launches) {
  k_rk4_final<<<(int)((nd + 255) / 256), 256, 0, st>>>(x, v, a4, v4, asum, vsum, nd, dt);
  launches += 1;
}

}  // namespace fmm
