// BLAS-1 on spinor fields in the device layout, with the reference's
// precision rules: products of FP32 fields accumulate in double
// (modules/linalg/salg.c:1050-1078; here after summing the four products of
// a float4 in FP32), products of FP64 fields accumulate in double-double
// (modules/linalg/salg_dble.c:2319-2357 with utils/qsum.c).
//
// A parity half of a field is a contiguous range (even chunks come first), so
// everything here works on flat arrays: FP64 fields as double2 (one complex
// component), FP32 fields as float4 (two complex components).
//
// Reductions are two deterministic passes: a fixed grid of RB blocks sums in
// double (per thread, then a fixed tree in the block), then one block adds
// the RB partials in double-double (Knuth's TwoSum), so results are
// bit-identical from run to run.
#include <cstring>
#include "lib.h"

namespace qcd {

static const int RB = 1184;   // 8 blocks per SM on 148 SMs
static const int RT = 256;

struct Range { size_t beg, n; };

static Range range(const Ctx &c, int prec, int par) {
  size_t per_site = prec == 64 ? 12 : 6;       // double2 or float4 elements per site
  size_t half = (size_t)c.g.volh * per_site;
  if (par == PAR_ALL) return {0, 2 * half};
  return {par == PAR_ODD ? half : 0, half};
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block sum of NC values into out[NC*blockIdx.x + k]
template <int NC>
__device__ __forceinline__ void block_store(double v[NC], double *out) {
  __shared__ double sh[NC][RT / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    double t = warp_sum(v[k]);
    if (lane == 0) sh[k][w] = t;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < NC; k++) {
      double t = threadIdx.x < RT / 32 ? sh[k][threadIdx.x] : 0.0;
      t = warp_sum(t);
      if (threadIdx.x == 0) out[(size_t)NC * blockIdx.x + k] = t;
    }
  }
}

// final pass: out[2k], out[2k+1] = double-double sum of part[NC*b + k]
template <int NC>
__global__ void k_finish(const double *__restrict__ part, int nb, double *out) {
  __shared__ double hi[NC][32], lo[NC][32];
  int t = threadIdx.x;   // 32 threads
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

// FP32 fields: the products of one float4 (two complex components) are
// summed in FP32 and that sum is added in double (per-product FP64
// arithmetic made these reductions FP64-throughput bound on B200, at about
// half their bandwidth-bound speed)
template <typename R>
__global__ void k_norm2(const void *__restrict__ x, Range r, double *part) {
  double v[1] = {0.0};
  for (size_t i = blockIdx.x * (size_t)RT + threadIdx.x; i < r.n; i += (size_t)RB * RT) {
    if (sizeof(R) == 8) {
      double2 a = __ldg((const double2 *)x + r.beg + i);
      v[0] += a.x * a.x + a.y * a.y;
    } else {
      float4 a = __ldg((const float4 *)x + r.beg + i);
      v[0] += (double)(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w);
    }
  }
  block_store<1>(v, part);
}

template <typename R>
__global__ void k_dot(const void *__restrict__ x, const void *__restrict__ y, Range r, double *part) {
  double v[2] = {0.0, 0.0};
  for (size_t i = blockIdx.x * (size_t)RT + threadIdx.x; i < r.n; i += (size_t)RB * RT) {
    if (sizeof(R) == 8) {
      double2 a = __ldg((const double2 *)x + r.beg + i), b = __ldg((const double2 *)y + r.beg + i);
      v[0] += a.x * b.x + a.y * b.y;
      v[1] += a.x * b.y - a.y * b.x;
    } else {
      float4 a = __ldg((const float4 *)x + r.beg + i), b = __ldg((const float4 *)y + r.beg + i);
      v[0] += (double)(a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w);
      v[1] += (double)(a.x * b.y - a.y * b.x + a.z * b.w - a.w * b.z);
    }
  }
  block_store<2>(v, part);
}

// uniform norm: max over sites of the spinor norm (sflds/unorm.c)
template <typename R>
__global__ void k_unorm(Geom g, const void *__restrict__ x, int c0, int nch, double *part) {
  double m = 0.0;
  size_t nsite = (size_t)nch * g.vbh;
  for (size_t i = blockIdx.x * (size_t)RT + threadIdx.x; i < nsite; i += (size_t)RB * RT) {
    int chunk = c0 + (int)(i / g.vbh), s = (int)(i % g.vbh);
    spinor<R> v = Store<R>::load_spinor(x, chunk, s, g.vbh);
    double n2 = 0.0;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int k = 0; k < 3; k++) n2 += (double)v.c[a].c[k].re * v.c[a].c[k].re + (double)v.c[a].c[k].im * v.c[a].c[k].im;
    m = fmax(m, n2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double sh[RT / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < RT / 32; w++) t = fmax(t, sh[w]);
    part[blockIdx.x] = t;
  }
}

__global__ void k_max_finish(const double *__restrict__ part, int nb, double *out) {
  double m = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) m = fmax(m, part[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if (threadIdx.x == 0) { out[0] = sqrt(m); out[1] = 0.0; }
}

static int ensure_red(Ctx &c) {
  if (c.red) return 0;
  if (cudaMalloc(&c.red, (size_t)RB * 4 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c.red_out, 8 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&c.h_red, 8 * sizeof(double)) != cudaSuccess)
    return fail("out of memory (reduction buffers)");
  c.red_blocks = RB;
  return 0;
}

// the nc (hi, lo) results of this rank, then (domain decomposition) their
// sum or maximum over the ranks, the same on every rank
static int finish(Ctx &c, int nc, double *res, bool is_max = false) {
  cudaMemcpyAsync(c.h_red, c.red_out, 2 * nc * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("reduction: CUDA error");
  for (int k = 0; k < 2 * nc; k++) res[k] = c.h_red[k];
  return dd_on(c) ? dd_global(c, res, nc, is_max) : 0;
}

int la_norm2(Ctx &c, int prec, const void *x, int par, double *res) {
  if (ensure_red(c)) return -1;
  Range r = range(c, prec, par);
  if (prec == 64) k_norm2<double><<<RB, RT, 0, c.stream>>>(x, r, c.red);
  else k_norm2<float><<<RB, RT, 0, c.stream>>>(x, r, c.red);
  k_finish<1><<<1, 32, 0, c.stream>>>(c.red, RB, c.red_out);
  return finish(c, 1, res);
}

int la_dot(Ctx &c, int prec, const void *x, const void *y, int par, double *res) {
  if (ensure_red(c)) return -1;
  Range r = range(c, prec, par);
  if (prec == 64) k_dot<double><<<RB, RT, 0, c.stream>>>(x, y, r, c.red);
  else k_dot<float><<<RB, RT, 0, c.stream>>>(x, y, r, c.red);
  k_finish<2><<<1, 32, 0, c.stream>>>(c.red, RB, c.red_out);
  return finish(c, 2, res);
}

// x += a p ; r -= a ap ; then |r|^2 -- the FP64 CG update of the
// multi-shift solver (modules/linsolv/mscg.c:242-275, cg_step2 with the norm
// of cg_step3) in one pass
__global__ void k_xr_norm2(Range rg, double2 *__restrict__ x, double2 *__restrict__ r,
                           const double2 *__restrict__ p, const double2 *__restrict__ ap, double a,
                           double *part) {
  double v[1] = {0.0};
  for (size_t i = blockIdx.x * (size_t)RT + threadIdx.x; i < rg.n; i += (size_t)RB * RT) {
    const size_t j = rg.beg + i;
    const double2 pp = __ldg(p + j), aa = __ldg(ap + j);
    double2 xx = x[j], rr = r[j];
    xx.x += a * pp.x;
    xx.y += a * pp.y;
    rr.x -= a * aa.x;
    rr.y -= a * aa.y;
    x[j] = xx;
    r[j] = rr;
    v[0] += rr.x * rr.x + rr.y * rr.y;
  }
  block_store<1>(v, part);
}

int la_xr_norm2(Ctx &c, void *x, void *r, const void *p, const void *ap, double a, int par, double *res) {
  if (ensure_red(c)) return -1;
  Range rg = range(c, 64, par);
  k_xr_norm2<<<RB, RT, 0, c.stream>>>(rg, (double2 *)x, (double2 *)r, (const double2 *)p, (const double2 *)ap, a,
                                      c.red);
  k_finish<1><<<1, 32, 0, c.stream>>>(c.red, RB, c.red_out);
  return finish(c, 1, res);
}

// x -> gamma5 x on a parity range of an FP64 field (spin components 2, 3 of
// every site change sign: double2 planes 6..11 of a chunk), then |x|^2
__global__ void k_mulg5_norm2(Range rg, double2 *__restrict__ x, int vbh, double *part) {
  double v[1] = {0.0};
  const size_t per = (size_t)12 * vbh;
  for (size_t i = blockIdx.x * (size_t)RT + threadIdx.x; i < rg.n; i += (size_t)RB * RT) {
    const size_t j = rg.beg + i;
    double2 xx = x[j];
    if ((j % per) / vbh >= 6) {
      xx.x = -xx.x;
      xx.y = -xx.y;
      x[j] = xx;
    }
    v[0] += xx.x * xx.x + xx.y * xx.y;
  }
  block_store<1>(v, part);
}

int la_mulg5_norm2(Ctx &c, void *x, int par, double *res) {
  if (ensure_red(c)) return -1;
  Range rg = range(c, 64, par);
  k_mulg5_norm2<<<RB, RT, 0, c.stream>>>(rg, (double2 *)x, c.g.vbh, c.red);
  k_finish<1><<<1, 32, 0, c.stream>>>(c.red, RB, c.red_out);
  return finish(c, 1, res);
}

int la_unorm(Ctx &c, int prec, const void *x, int par, double *res) {
  if (ensure_red(c)) return -1;
  int c0 = par == PAR_ODD ? c.g.nbl : 0;
  int nch = par == PAR_ALL ? 2 * c.g.nbl : c.g.nbl;
  if (prec == 64) k_unorm<double><<<RB, RT, 0, c.stream>>>(c.g, x, c0, nch, c.red);
  else k_unorm<float><<<RB, RT, 0, c.stream>>>(c.g, x, c0, nch, c.red);
  k_max_finish<<<1, 32, 0, c.stream>>>(c.red, RB, c.red_out);
  return finish(c, 1, res, true);
}

// ------------------------------------------------------------- elementwise
static unsigned nblk(size_t n) { return (unsigned)((n + 255) / 256); }

__global__ void k_copy_dd(Range r, const double2 *x, double2 *y) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) y[r.beg + i] = x[r.beg + i];
}
__global__ void k_copy_ff(Range r, const float4 *x, float4 *y) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) y[r.beg + i] = x[r.beg + i];
}
// Precision conversion works per site: plane j (float4) of an FP32 chunk
// holds components 2j, 2j+1, while an FP64 chunk has one double2 plane per
// component, so the two layouts do not line up element by element.
template <typename A, typename B>
__global__ void k_convert(Geom g, int c0, int nch, const void *x, void *y) {
  size_t i = blockIdx.x * (size_t)128 + threadIdx.x;
  if (i >= (size_t)nch * g.vbh) return;
  int chunk = c0 + (int)(i / g.vbh), s = (int)(i % g.vbh);
  spinor<A> a = Store<A>::load_spinor_rw(x, chunk, s, g.vbh);
  spinor<B> b;
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int j = 0; j < 3; j++) b.c[k].c[j] = mk<B>((B)a.c[k].c[j].re, (B)a.c[k].c[j].im);
  Store<B>::store_spinor(y, chunk, s, g.vbh, b);
}

void la_copy(const Ctx &c, int pin, const void *x, int pout, void *y, int par, cudaStream_t st) {
  if (pin == pout) {
    Range r = range(c, pin, par);
    if (pin == 64) k_copy_dd<<<nblk(r.n), 256, 0, st>>>(r, (const double2 *)x, (double2 *)y);
    else k_copy_ff<<<nblk(r.n), 256, 0, st>>>(r, (const float4 *)x, (float4 *)y);
    return;
  }
  int c0 = par == PAR_ODD ? c.g.nbl : 0;
  int nch = par == PAR_ALL ? 2 * c.g.nbl : c.g.nbl;
  size_t n = (size_t)nch * c.g.vbh;
  unsigned nb = (unsigned)((n + 127) / 128);
  if (pin == 64) k_convert<double, float><<<nb, 128, 0, st>>>(c.g, c0, nch, x, y);
  else k_convert<float, double><<<nb, 128, 0, st>>>(c.g, c0, nch, x, y);
}

void la_zero(const Ctx &c, int prec, void *x, int par, cudaStream_t st) {
  Range r = range(c, prec, par);
  size_t es = prec == 64 ? sizeof(double2) : sizeof(float4);
  cudaMemsetAsync((char *)x + r.beg * es, 0, r.n * es, st);
}

__global__ void k_scale_d(Range r, double2 *x, double a) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) { double2 v = x[r.beg + i]; x[r.beg + i] = make_double2(a * v.x, a * v.y); }
}
__global__ void k_scale_f(Range r, float4 *x, float a) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) { float4 v = x[r.beg + i]; x[r.beg + i] = make_float4(a * v.x, a * v.y, a * v.z, a * v.w); }
}
void la_scale(const Ctx &c, int prec, void *x, double a, int par, cudaStream_t st) {
  Range r = range(c, prec, par);
  if (prec == 64) k_scale_d<<<nblk(r.n), 256, 0, st>>>(r, (double2 *)x, a);
  else k_scale_f<<<nblk(r.n), 256, 0, st>>>(r, (float4 *)x, (float)a);
}

// y += a x  (mulc_spinor_add, salg.c:1319 / salg_dble.c)
__global__ void k_axpy_d(Range r, double2 *y, double ar, double ai, const double2 *x) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) {
    double2 a = x[r.beg + i], b = y[r.beg + i];
    b.x += ar * a.x - ai * a.y;
    b.y += ar * a.y + ai * a.x;
    y[r.beg + i] = b;
  }
}
__global__ void k_axpy_f(Range r, float4 *y, float ar, float ai, const float4 *x) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) {
    float4 a = x[r.beg + i], b = y[r.beg + i];
    b.x += ar * a.x - ai * a.y;
    b.y += ar * a.y + ai * a.x;
    b.z += ar * a.z - ai * a.w;
    b.w += ar * a.w + ai * a.z;
    y[r.beg + i] = b;
  }
}
void la_axpy(const Ctx &c, int prec, void *y, double ar, double ai, const void *x, int par, cudaStream_t st) {
  Range r = range(c, prec, par);
  if (prec == 64) k_axpy_d<<<nblk(r.n), 256, 0, st>>>(r, (double2 *)y, ar, ai, (const double2 *)x);
  else k_axpy_f<<<nblk(r.n), 256, 0, st>>>(r, (float4 *)y, (float)ar, (float)ai, (const float4 *)x);
}

// y (+)= sum of c_l x_l over up to 16 terms, applied in the given order with
// the arithmetic of k_axpy_f: the solution update of fgcr (update_psi,
// fgcr.c:181) in one pass over the fields instead of one axpy per term
struct LcTerms {
  const float4 *x[16];
  float2 c[16];
};
__global__ void k_lincomb_f(Range r, float4 *y, int nt, int acc, LcTerms t) {
  const size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i >= r.n) return;
  float4 b = acc ? y[r.beg + i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int l = 0; l < nt; l++) {
    const float4 a = t.x[l][r.beg + i];
    const float ar = t.c[l].x, ai = t.c[l].y;
    b.x += ar * a.x - ai * a.y;
    b.y += ar * a.y + ai * a.x;
    b.z += ar * a.z - ai * a.w;
    b.w += ar * a.w + ai * a.z;
  }
  y[r.beg + i] = b;
}
void la_lincomb32(const Ctx &c, void *y, int n, const float *cre, const float *cim, void *const *x,
                  cudaStream_t st) {
  const Range r = range(c, 32, PAR_ALL);
  if (n <= 0) {
    la_zero(c, 32, y, PAR_ALL, st);
    return;
  }
  for (int l0 = 0; l0 < n; l0 += 16) {
    LcTerms t;
    std::memset(&t, 0, sizeof(t));
    const int nt = n - l0 < 16 ? n - l0 : 16;
    for (int l = 0; l < nt; l++) {
      t.x[l] = (const float4 *)x[l0 + l];
      t.c[l] = make_float2(cre[l0 + l], cim[l0 + l]);
    }
    k_lincomb_f<<<nblk(r.n), 256, 0, st>>>(r, (float4 *)y, nt, l0 > 0, t);
  }
}

// y = x - y
__global__ void k_diff_f(Range r, const float4 *x, float4 *y) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) {
    float4 a = x[r.beg + i], b = y[r.beg + i];
    y[r.beg + i] = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
  }
}
__global__ void k_diff_d(Range r, const double2 *x, double2 *y) {
  size_t i = blockIdx.x * (size_t)256 + threadIdx.x;
  if (i < r.n) {
    double2 a = x[r.beg + i], b = y[r.beg + i];
    y[r.beg + i] = make_double2(a.x - b.x, a.y - b.y);
  }
}
void la_diff(const Ctx &c, int prec, const void *x, void *y, int par, cudaStream_t st) {
  Range r = range(c, prec, par);
  if (prec == 64) k_diff_d<<<nblk(r.n), 256, 0, st>>>(r, (const double2 *)x, (double2 *)y);
  else k_diff_f<<<nblk(r.n), 256, 0, st>>>(r, (const float4 *)x, (float4 *)y);
}

// sd += s (add_s2sd, sflds.c:1356) and r = a - b rounded to FP32 (diff_sd2s, sflds.c:1390)
template <int MODE>
__global__ void k_mixed(Geom g, int c0, int nch, const void *a, const void *b, void *out) {
  size_t i = blockIdx.x * (size_t)128 + threadIdx.x;
  if (i >= (size_t)nch * g.vbh) return;
  int chunk = c0 + (int)(i / g.vbh), s = (int)(i % g.vbh);
  if (MODE == 0) {   // out(FP64) += a(FP32)
    spinor<float> x = Store<float>::load_spinor_rw(a, chunk, s, g.vbh);
    spinor<double> y = Store<double>::load_spinor_rw(out, chunk, s, g.vbh);
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int j = 0; j < 3; j++) { y.c[k].c[j].re += x.c[k].c[j].re; y.c[k].c[j].im += x.c[k].c[j].im; }
    Store<double>::store_spinor(out, chunk, s, g.vbh, y);
  } else {           // out(FP32) = a(FP64) - b(FP64)
    spinor<double> x = Store<double>::load_spinor_rw(a, chunk, s, g.vbh);
    spinor<double> y = Store<double>::load_spinor_rw(b, chunk, s, g.vbh);
    spinor<float> z;
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int j = 0; j < 3; j++)
        z.c[k].c[j] = mk<float>((float)(x.c[k].c[j].re - y.c[k].c[j].re), (float)(x.c[k].c[j].im - y.c[k].c[j].im));
    Store<float>::store_spinor(out, chunk, s, g.vbh, z);
  }
}

void la_add_s2sd(const Ctx &c, const void *s32, void *sd, int par, cudaStream_t st) {
  int c0 = par == PAR_ODD ? c.g.nbl : 0, nch = par == PAR_ALL ? 2 * c.g.nbl : c.g.nbl;
  size_t n = (size_t)nch * c.g.vbh;
  k_mixed<0><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(c.g, c0, nch, s32, nullptr, sd);
}

void la_diff_sd2s(const Ctx &c, const void *ad, const void *bd, void *r32, int par, cudaStream_t st) {
  int c0 = par == PAR_ODD ? c.g.nbl : 0, nch = par == PAR_ALL ? 2 * c.g.nbl : c.g.nbl;
  size_t n = (size_t)nch * c.g.vbh;
  k_mixed<1><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(c.g, c0, nch, ad, bd, r32);
}

}  // namespace qcd
