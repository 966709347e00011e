#pragma once
#include <algorithm>

#include "tree.cuh"

namespace fmm {
int direct_sum(const double *d_pos, const double *d_mass, int64_t n, const int64_t *d_targets, int64_t nt, int dim,
               double eps2, int soft_mode, double G, double *d_acc, double *d_pot, cudaStream_t st, int64_t &launches);
void se_update(double *x, double *v, const double *a, int64_t nd, double dt, cudaStream_t st, int64_t &launches);
void rk4_stage(const double *x0, const double *v0, const double *a_prev, double *xs, double *vs, double *asum,
               double *vsum, int64_t nd, double cdt, double wprev, int first, cudaStream_t st, int64_t &launches);
void rk4_final(double *x, double *v, const double *a4, const double *v4, const double *asum, const double *vsum,
               int64_t nd, double dt, cudaStream_t st, int64_t &launches);
}  // namespace fmm
