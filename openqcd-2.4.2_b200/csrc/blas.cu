// Layout-agnostic BLAS-1 on spinor arrays of n sites in the reference's
// array-of-structures order (24 reals per site), for the drop-in entry points
// of modules/linalg/salg.c and salg_dble.c and for the generic fgcr().
//
// Products accumulate in double per thread and in double-double across the
// CTA partials (the reference's qflt sums, modules/utils/qsum.c:265-359),
// deterministically: fixed grid, fixed tree, fixed final order.
#include "lib.h"

namespace qcd {

static const int FB = 1184;   // reduction CTAs (8 per SM)
static const int FT = 256;

__device__ __forceinline__ double fwarp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NC>
__device__ __forceinline__ void fblock_store(double v[NC], double *out) {
  __shared__ double sh[NC][FT / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    double t = fwarp_sum(v[k]);
    if (lane == 0) sh[k][w] = t;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < NC; k++) {
      double t = threadIdx.x < FT / 32 ? sh[k][threadIdx.x] : 0.0;
      t = fwarp_sum(t);
      if (threadIdx.x == 0) out[(size_t)NC * blockIdx.x + k] = t;
    }
  }
}

// out[2k], out[2k+1]: double-double (hi, lo) sum over the nb partials of component k
template <int NC>
__global__ void k_fsum_dd(const double *__restrict__ part, int nb, double *out) {
  __shared__ double hi[NC][32], lo[NC][32];
  int t = threadIdx.x;
  for (int k = 0; k < NC; k++) {
    double h = 0.0, l = 0.0;
    for (int b = t; b < nb; b += 32) {
      double x = part[(size_t)NC * b + k];
      double s = h + x, bb = s - h;
      l += (h - (s - bb)) + (x - bb);
      h = s;
    }
    hi[k][t] = h;
    lo[k][t] = l;
  }
  __syncwarp();
  if (t < NC) {
    double h = 0.0, l = 0.0;
    for (int j = 0; j < 32; j++) {
      double x = hi[t][j];
      double s = h + x, bb = s - h;
      l += (h - (s - bb)) + (x - bb) + lo[t][j];
      h = s;
    }
    double s = h + l;
    out[2 * t] = s;
    out[2 * t + 1] = l - (s - h);
  }
}

// (x, y) = sum conj(x) y over n complex numbers; MODE 0: complex, 1: |x|^2
template <typename R, int MODE>
__global__ void k_fdot(const R *__restrict__ x, const R *__restrict__ y, size_t n, double *part) {
  double v[2] = {0.0, 0.0};
  for (size_t i = blockIdx.x * (size_t)FT + threadIdx.x; i < n; i += (size_t)gridDim.x * FT) {
    double ar = x[2 * i], ai = x[2 * i + 1];
    if (MODE == 1) {
      v[0] += ar * ar + ai * ai;
    } else {
      double br = y[2 * i], bi = y[2 * i + 1];
      v[0] += ar * br + ai * bi;
      v[1] += ar * bi - ai * br;
    }
  }
  if (MODE == 1) {
    double w[1] = {v[0]};
    fblock_store<1>(w, part);
  } else {
    fblock_store<2>(v, part);
  }
}

// max over sites of |x(site)|^2, 12 complex per site
template <typename R>
__global__ void k_fumax(const R *__restrict__ x, size_t nsite, double *part) {
  double m = 0.0;
  for (size_t i = blockIdx.x * (size_t)FT + threadIdx.x; i < nsite; i += (size_t)gridDim.x * FT) {
    double s = 0.0;
    for (int k = 0; k < 24; k++) s += (double)x[24 * i + k] * x[24 * i + k];
    m = fmax(m, s);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double sh[FT / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < FT / 32; w++) t = fmax(t, sh[w]);
    part[blockIdx.x] = t;
  }
}

__global__ void k_fmax_finish(const double *__restrict__ part, int nb, double *out) {
  double m = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) m = fmax(m, part[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if (threadIdx.x == 0) { out[0] = m; out[1] = 0.0; }
}

// y += (ar + i ai) x ; y = a*y (real) ; y = x - y ; y = T(x)
template <typename R>
__global__ void k_faxpy(R *y, const R *__restrict__ x, size_t n, R ar, R ai) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < n) {
    R xr = x[2 * i], xi = x[2 * i + 1];
    y[2 * i] += ar * xr - ai * xi;
    y[2 * i + 1] += ar * xi + ai * xr;
  }
}
template <typename R>
__global__ void k_fscale(R *y, size_t n, R a) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < n) y[i] *= a;
}
template <typename A, typename B>
__global__ void k_fconv(const A *__restrict__ x, B *y, size_t n) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < n) y[i] = (B)x[i];
}
__global__ void k_fadd_s2sd(const float *__restrict__ s, double *sd, size_t n) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < n) sd[i] += (double)s[i];
}
__global__ void k_fdiff_sd2s(const double *__restrict__ a, const double *__restrict__ b, float *r, size_t n) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < n) r[i] = (float)(a[i] - b[i]);
}
template <typename R>
__global__ void k_fdiff(const R *__restrict__ x, R *y, size_t n) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < n) y[i] = x[i] - y[i];
}

static unsigned g256(size_t n) { return (unsigned)((n + 255) / 256); }

static int nblocks(size_t n) {
  size_t b = (n + FT - 1) / FT;
  return (int)(b < (size_t)FB ? (b ? b : 1) : FB);
}

// ------------------------------------------------------------- host wrappers
// All pointers here are device-accessible; res_dd receives (hi, lo) pairs.
int flat_dot(Ctx &c, int prec, const void *x, const void *y, size_t nsite, double *res_dd, double *scratch,
             double *out_dev) {
  size_t n = nsite * 12;
  int nb = nblocks(n);
  if (prec == 64) k_fdot<double, 0><<<nb, FT, 0, c.stream>>>((const double *)x, (const double *)y, n, scratch);
  else k_fdot<float, 0><<<nb, FT, 0, c.stream>>>((const float *)x, (const float *)y, n, scratch);
  k_fsum_dd<2><<<1, 32, 0, c.stream>>>(scratch, nb, out_dev);
  if (!res_dd) return 0;
  cudaMemcpyAsync(c.h_red, out_dev, 4 * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("reduction: CUDA error");
  for (int k = 0; k < 4; k++) res_dd[k] = c.h_red[k];
  return 0;
}

int flat_norm2(Ctx &c, int prec, const void *x, size_t nsite, double *res_dd, double *scratch, double *out_dev) {
  size_t n = nsite * 12;
  int nb = nblocks(n);
  if (prec == 64) k_fdot<double, 1><<<nb, FT, 0, c.stream>>>((const double *)x, nullptr, n, scratch);
  else k_fdot<float, 1><<<nb, FT, 0, c.stream>>>((const float *)x, nullptr, n, scratch);
  k_fsum_dd<1><<<1, 32, 0, c.stream>>>(scratch, nb, out_dev);
  cudaMemcpyAsync(c.h_red, out_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("reduction: CUDA error");
  res_dd[0] = c.h_red[0];
  res_dd[1] = c.h_red[1];
  return 0;
}

int flat_umax(Ctx &c, int prec, const void *x, size_t nsite, double *res, double *scratch, double *out_dev) {
  int nb = nblocks(nsite);
  if (prec == 64) k_fumax<double><<<nb, FT, 0, c.stream>>>((const double *)x, nsite, scratch);
  else k_fumax<float><<<nb, FT, 0, c.stream>>>((const float *)x, nsite, scratch);
  k_fmax_finish<<<1, 32, 0, c.stream>>>(scratch, nb, out_dev);
  cudaMemcpyAsync(c.h_red, out_dev, sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("reduction: CUDA error");
  *res = c.h_red[0];
  return 0;
}

void flat_axpy(Ctx &c, int prec, void *y, const void *x, size_t nsite, double ar, double ai) {
  size_t n = nsite * 12;
  if (prec == 64) k_faxpy<double><<<g256(n), 256, 0, c.stream>>>((double *)y, (const double *)x, n, ar, ai);
  else k_faxpy<float><<<g256(n), 256, 0, c.stream>>>((float *)y, (const float *)x, n, (float)ar, (float)ai);
}
void flat_scale(Ctx &c, int prec, void *y, size_t nsite, double a) {
  size_t n = nsite * 24;
  if (prec == 64) k_fscale<double><<<g256(n), 256, 0, c.stream>>>((double *)y, n, a);
  else k_fscale<float><<<g256(n), 256, 0, c.stream>>>((float *)y, n, (float)a);
}
void flat_zero(Ctx &c, int prec, void *y, size_t nsite) {
  cudaMemsetAsync(y, 0, nsite * 24 * (prec == 64 ? 8 : 4), c.stream);
}
void flat_copy(Ctx &c, int pin, const void *x, int pout, void *y, size_t nsite) {
  size_t n = nsite * 24;
  if (pin == pout) cudaMemcpyAsync(y, x, n * (pin == 64 ? 8 : 4), cudaMemcpyDeviceToDevice, c.stream);
  else if (pin == 64) k_fconv<double, float><<<g256(n), 256, 0, c.stream>>>((const double *)x, (float *)y, n);
  else k_fconv<float, double><<<g256(n), 256, 0, c.stream>>>((const float *)x, (double *)y, n);
}
void flat_add_s2sd(Ctx &c, const void *s, void *sd, size_t nsite) {
  size_t n = nsite * 24;
  k_fadd_s2sd<<<g256(n), 256, 0, c.stream>>>((const float *)s, (double *)sd, n);
}
void flat_diff_sd2s(Ctx &c, const void *a, const void *b, void *r, size_t nsite) {
  size_t n = nsite * 24;
  k_fdiff_sd2s<<<g256(n), 256, 0, c.stream>>>((const double *)a, (const double *)b, (float *)r, n);
}
void flat_diff(Ctx &c, int prec, const void *x, void *y, size_t nsite) {
  size_t n = nsite * 24;
  if (prec == 64) k_fdiff<double><<<g256(n), 256, 0, c.stream>>>((const double *)x, (double *)y, n);
  else k_fdiff<float><<<g256(n), 256, 0, c.stream>>>((const float *)x, (float *)y, n);
}

// FP64 complex arrays of n entries (little vectors)
int flat_cdot(Ctx &c, const double2 *x, const double2 *y, size_t n, double *res_dd, double *scratch, double *out_dev) {
  int nb = nblocks(n);
  k_fdot<double, 0><<<nb, FT, 0, c.stream>>>((const double *)x, (const double *)y, n, scratch);
  k_fsum_dd<2><<<1, 32, 0, c.stream>>>(scratch, nb, out_dev);
  cudaMemcpyAsync(c.h_red, out_dev, 4 * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("reduction: CUDA error");
  for (int k = 0; k < 4; k++) res_dd[k] = c.h_red[k];
  return 0;
}
void flat_caxpy(Ctx &c, double2 *y, const double2 *x, size_t n, double ar, double ai) {
  k_faxpy<double><<<g256(n), 256, 0, c.stream>>>((double *)y, (const double *)x, n, ar, ai);
}
void flat_cscale(Ctx &c, double2 *y, size_t n, double a) {
  k_fscale<double><<<g256(2 * n), 256, 0, c.stream>>>((double *)y, 2 * n, a);
}

int flat_scratch(Ctx &c, double **scratch, double **out) {
  if (!c.red) {
    if (cudaMalloc(&c.red, (size_t)FB * 4 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c.red_out, 8 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&c.h_red, 8 * sizeof(double)) != cudaSuccess)
      return fail("out of memory (reduction buffers)");
  }
  *scratch = c.red;
  *out = c.red_out;
  return 0;
}

}  // namespace qcd
