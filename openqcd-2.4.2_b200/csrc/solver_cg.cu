// Conjugate-gradient solver of the normal equations on device fields:
// the reference's cgne (modules/linsolv/cgne.c:377-560: single-precision CG
// iterations, double-precision solution and residual recomputation at every
// reset, reset after 100 steps or when the residual reaches
// PRECISION_LIMIT = 512 FLT_EPSILON times the solution norm) and its
// twisted-mass drivers tmcg / tmcgeo (modules/forces/tmcg.c:118-260), which
// solve (Dw^dag Dw) psi = eta with Dop = gamma5 Dw(mu) applied with
// alternating sign of mu, or the even-odd preconditioned Dwhat on the even
// sites.
#include "lib.h"
#include <cfloat>
#include <cmath>
#include <functional>

namespace qcd {

// gamma5 on a parity range: the lower two spin components change sign.
// FP64 fields: double2 planes k = 6..11 of a chunk; FP32: float4 planes 3..5.
__global__ void k_mulg5_d(size_t beg, size_t n, double2 *x, int vbh) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t j = beg + i;
  const int k = (int)((j % ((size_t)12 * vbh)) / vbh);
  if (k >= 6) {
    const double2 v = x[j];
    x[j] = make_double2(-v.x, -v.y);
  }
}
__global__ void k_mulg5_f(size_t beg, size_t n, float4 *x, int vbh) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t j = beg + i;
  const int k = (int)((j % ((size_t)6 * vbh)) / vbh);
  if (k >= 3) {
    const float4 v = x[j];
    x[j] = make_float4(-v.x, -v.y, -v.z, -v.w);
  }
}

static void mulg5(const Ctx &c, int prec, void *x, int par, cudaStream_t st) {
  const size_t per = prec == 64 ? 12 : 6, half = (size_t)c.g.volh * per;
  const size_t beg = par == PAR_ODD ? half : 0, n = par == PAR_ALL ? 2 * half : half;
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (prec == 64) k_mulg5_d<<<nb, 256, 0, st>>>(beg, n, (double2 *)x, c.g.vbh);
  else k_mulg5_f<<<nb, 256, 0, st>>>(beg, n, (float4 *)x, c.g.vbh);
}

// x += a p ; p = b p + r  (cgne.c update_xp), FP32 on a parity range
__global__ void k_update_xp(size_t beg, size_t n, float4 *x, float4 *p, const float4 *__restrict__ r, float a, float b) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t j = beg + i;
  float4 xx = x[j], pp = p[j];
  const float4 rr = r[j];
  xx.x += a * pp.x; xx.y += a * pp.y; xx.z += a * pp.z; xx.w += a * pp.w;
  pp.x = b * pp.x + rr.x; pp.y = b * pp.y + rr.y; pp.z = b * pp.z + rr.z; pp.w = b * pp.w + rr.w;
  x[j] = xx;
  p[j] = pp;
}

static float norm_sq32(Ctx &c, const void *x, int par) {
  double r[2];
  la_norm2(c, 32, x, par, r);
  return (float)(r[0] + r[1]);
}

static cplxf dot32(Ctx &c, const void *x, const void *y, int par) {
  double r[4];
  la_dot(c, 32, x, y, par, r);
  return cplxf{(float)(r[0] + r[1]), (float)(r[2] + r[3])};
}

static double unorm32(Ctx &c, const void *x, int par) {
  double r[2];
  la_unorm(c, 32, x, par, r);
  return (double)(float)r[0];
}

using CgOp = std::function<void(const void *, void *)>;

// cgne (cgne.c:452) on the sites of parity range par; Dop / Dop_dble apply
// D and D^dag alternately.  Returns the residual norm; status[0] = CG
// iterations or -1.
static double cgne_core(Ctx &c, int par, const CgOp &Dop, const CgOp &Dop_dble, int nmx, int istop, double res,
                        const void *eta, void *psi, int *status) {
  cudaStream_t st = c.stream;
  void *x = c.ws32[0], *r = c.ws32[1], *p = c.ws32[2], *ap = c.ws32[3], *w = c.ws32[4];
  void *wd = c.ws64[0], *vd = c.ws64[1];
  const double PRECISION_LIMIT = (double)(512.0f * FLT_EPSILON);
  const size_t half = (size_t)c.g.volh * 6;
  const size_t beg = par == PAR_ODD ? half : 0, n = par == PAR_ALL ? 2 * half : half;
  const unsigned nbk = (unsigned)((n + 255) / 256);
  // cg_init
  la_zero(c, 32, x, par, st);
  la_copy(c, 64, eta, 32, r, par, st);
  la_copy(c, 32, r, 32, p, par, st);
  la_zero(c, 64, psi, par, st);
  float rsq = norm_sq32(c, r, par);
  double xn = 0.0, rn = istop ? unorm32(c, r, par) : std::sqrt((double)rsq);
  const double tol = res * rn;
  status[0] = 0;
  while (rn > tol) {
    int ncg = 0;
    for (;;) {
      // cg_step
      Dop(p, w);
      Dop(w, ap);
      const float ai = rsq / norm_sq32(c, w, par);
      la_axpy(c, 32, r, -ai, 0.0, ap, par, st);
      const float rsq_old = rsq;
      rsq = norm_sq32(c, r, par);
      const float bi = rsq / rsq_old;
      k_update_xp<<<nbk, 256, 0, st>>>(beg, n, (float4 *)x, (float4 *)p, (const float4 *)r, ai, bi);
      ncg += 1;
      status[0] += 1;
      if (istop) {
        xn = unorm32(c, x, par);
        rn = unorm32(c, r, par);
      } else {
        xn = std::sqrt((double)norm_sq32(c, x, par));
        rn = std::sqrt((double)rsq);
      }
      if (rn <= tol || rn <= PRECISION_LIMIT * xn || ncg >= 100 || status[0] >= nmx) break;
    }
    la_add_s2sd(c, x, psi, par, st);
    // cg_reset
    Dop_dble(psi, wd);
    Dop_dble(wd, vd);
    la_diff_sd2s(c, eta, vd, r, par, st);
    rsq = norm_sq32(c, r, par);
    la_copy(c, 32, p, 32, w, par, st);
    la_copy(c, 32, r, 32, p, par, st);
    cplxf z = dot32(c, r, w, par);
    z.re = -z.re / rsq;
    z.im = -z.im / rsq;
    la_axpy(c, 32, w, z.re, z.im, r, par, st);
    Dop(w, x);
    Dop(x, ap);
    const float rr = norm_sq32(c, x, par);
    z = dot32(c, ap, r, par);
    if ((z.re * z.re + z.im * z.im) < (2.0f * rr * rr)) {
      z.re = -z.re / rr;
      z.im = -z.im / rr;
      la_axpy(c, 32, p, z.re, z.im, w, par, st);
    }
    la_zero(c, 32, x, par, st);
    rn = istop ? unorm32(c, r, par) : std::sqrt((double)rsq);
    if (status[0] >= nmx && rn > tol) {
      status[0] = -1;
      return rn;
    }
  }
  return rn;
}

static int cg_reserve(Ctx &c) {
  while (c.ws32.size() < 5) {
    void *q = nullptr;
    if (cudaMalloc(&q, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory (workspace)");
    c.ws32.push_back(q);
  }
  while (c.ws64.size() < 3) {
    void *q = nullptr;
    if (cudaMalloc(&q, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory (workspace)");
    c.ws64.push_back(q);
  }
  if (!c.tmp32 && cudaMalloc(&c.tmp32, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory");
  if (!c.tmp64 && cudaMalloc(&c.tmp64, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory");
  return 0;
}

// tmcg (eo = 0, tmcg.c:118) and tmcgeo (eo = 1, tmcg.c:206) on device
// fields; with eo = 1 only the even sites of eta and psi are used.
double tmcg_dev(Ctx &c, int eo, int nmx, int istop, double res, double mu, const void *eta, void *psi, int *ifail,
                int *status) {
  ifail[0] = 0;
  status[0] = 0;
  if (!c.have_ud || !c.have_sw) { fail("tmcg: gauge or SW field missing on the device"); return -1.0; }
  if (nmx < 1 || res <= DBL_EPSILON || istop < 0 || istop > 1) { fail("cgne: parameters are out of range"); return -1.0; }
  if (cg_reserve(c)) return -1.0;
  const int par = eo ? PAR_EVEN : PAR_ALL;
  cudaStream_t st = c.stream;
  // the twisted-mass eo flag is switched off for tmcg (tmcg.c:128-131)
  const int eo_save = c.eoflg;
  if (!eo) c.eoflg = 0;
  double rho;
  {
    double r[2];
    if (istop) {
      la_unorm(c, 64, eta, par, r);
      rho = r[0];
    } else {
      la_norm2(c, 64, eta, par, r);
      rho = std::sqrt(r[0]);
    }
  }
  if (eo && (c.sw_inv_fail & 2)) {
    ifail[0] = -3;   // unsafe inversion of the odd SW term (tmcg.c:233)
  } else if (rho != 0.0) {
    void *rsd = c.ws64[2];
    la_copy(c, 64, eta, 64, rsd, par, st);
    la_scale(c, 64, rsd, 1.0 / rho, par, st);
    float mus = (float)mu;
    double mud = mu;
    CgOp Dop = [&](const void *s, void *r) {
      dirac_op<float>(c, eo ? 5 : 0, mus, s, r, c.tmp32, st);
      mulg5(c, 32, r, par, st);
      mus = -mus;
    };
    CgOp Dop_dble = [&](const void *s, void *r) {
      dirac_op<double>(c, eo ? 5 : 0, mud, s, r, c.tmp64, st);
      mulg5(c, 64, r, par, st);
      mud = -mud;
    };
    const double rn = cgne_core(c, par, Dop, Dop_dble, nmx, istop, res, rsd, psi, status);
    la_scale(c, 64, psi, rho, par, st);
    rho = rn * rho;
    if (status[0] < 0) {
      ifail[0] = -1;
      status[0] = nmx;
    }
  } else {
    la_zero(c, 64, psi, par, st);
  }
  if (ifail[0] == -3 && psi != eta) la_zero(c, 64, psi, par, st);
  c.eoflg = eo_save;
  cudaStreamSynchronize(st);
  return rho;
}

}  // namespace qcd
