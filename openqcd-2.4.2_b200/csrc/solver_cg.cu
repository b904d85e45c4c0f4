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

// ------------------------------------------------------------ multi-shift CG
// Multi-shift CG of modules/linsolv/mscg.c:387-560 on the even sites, with
// the operator pair of tmcgm (modules/forces/tmcgm.c:83-92): Op = gamma5
// Dwhat(mu), Op^dag = gamma5 Dwhat(-mu), so that Op^dag Op = Dwhat^dag Dwhat
// + mu^2.  All vectors are FP64, as in the reference.  The base system is the
// shift of smallest |mu|; every other shift k keeps its solution xh and
// direction ph and the scalars of mscg.c:81-88.

constexpr int MS_G = 12;   // shifted systems updated per launch

struct ShiftGroup {
  double2 *xh[MS_G];
  double2 *ph[MS_G];
  double ah[MS_G], bh[MS_G], gh[MS_G];
  int n;
};

// p = b p + r and, for each shifted system j of the group,
//   xh_j += ah_j ph_j ;  ph_j = bh_j ph_j + gh_j r
// (cg_step2 of the shifted solutions, mscg.c:249-253, and cg_step4,
// mscg.c:285-296: the solution update reads ph before its own update, so
// both happen while ph is in registers and r is read once for all shifts).
// Even sites only: the range is [0, n) of every field.
__global__ void k_mscg_p(size_t n, double2 *__restrict__ p, const double2 *__restrict__ r, double b, int upd_p,
                         ShiftGroup g) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 rr = r[i];
  if (upd_p) {
    double2 pp = p[i];
    pp.x = b * pp.x + rr.x;
    pp.y = b * pp.y + rr.y;
    p[i] = pp;
  }
  for (int j = 0; j < g.n; j++) {
    double2 ph = g.ph[j][i], xh = g.xh[j][i];
    xh.x += g.ah[j] * ph.x;
    xh.y += g.ah[j] * ph.y;
    ph.x = g.bh[j] * ph.x + g.gh[j] * rr.x;
    ph.y = g.bh[j] * ph.y + g.gh[j] * rr.y;
    g.xh[j][i] = xh;
    g.ph[j][i] = ph;
  }
}

namespace {

struct MsShift {
  int stop;
  double s, tol, ah, bh, gh, rh;
  void *xh, *ph;
};

struct MsWork {
  void *r, *p, *ap, *w, *x;
};

}  // namespace

static double ms_norm(double *dd) { return dd[0] + dd[1]; }

// Op^dag Op s -> ap with the intermediate Op s in w; |Op s|^2 when wn2
static int ms_op2(Ctx &c, double mu, const void *s, void *w, void *ap, double *wn2) {
  cudaStream_t st = c.stream;
  dirac_op<double>(c, 5, mu, s, w, c.tmp64, st);
  if (wn2) {
    double dd[2];
    if (la_mulg5_norm2(c, w, PAR_EVEN, dd)) return -1;
    *wn2 = ms_norm(dd);
  } else {
    mulg5(c, 64, w, PAR_EVEN, st);
  }
  dirac_op<double>(c, 5, -mu, w, ap, c.tmp64, st);
  mulg5(c, 64, ap, PAR_EVEN, st);
  return 0;
}

static double ms_rn(Ctx &c, const void *r, int istop, double rnsq) {
  if (!istop) return std::sqrt(rnsq);
  double u[2];
  la_unorm(c, 64, r, PAR_EVEN, u);
  return u[0];
}

// check_res (mscg.c:318-384): residual of psi recomputed in FP64 and, if it
// is above res*rn0, plain CG on the correction while iterations are left
static int ms_check_res(Ctx &c, const MsWork &ws, double mu, int nmx, int istop, double tol, const void *eta,
                        void *psi, int *ncg) {
  cudaStream_t st = c.stream;
  const size_t n = (size_t)c.g.volh * 12;
  const unsigned nbk = (unsigned)((n + 255) / 256);
  ShiftGroup none{};
  if (ms_op2(c, mu, psi, ws.w, ws.r, nullptr)) return -1;
  la_axpy(c, 64, ws.r, -1.0, 0.0, eta, PAR_EVEN, st);
  double dd[2];
  if (la_norm2(c, 64, ws.r, PAR_EVEN, dd)) return -1;
  double rnsq = ms_norm(dd);
  double rn = ms_rn(c, ws.r, istop, rnsq);
  if (rn <= tol) return 0;
  if (ncg[0] >= nmx) return 1;
  la_zero(c, 64, ws.x, PAR_EVEN, st);
  la_copy(c, 64, ws.r, 64, ws.p, PAR_EVEN, st);
  while (rn > tol && ncg[0] < nmx) {
    double wn2;
    if (ms_op2(c, mu, ws.p, ws.w, ws.ap, &wn2)) return -1;
    const double a = rnsq / wn2;
    if (la_xr_norm2(c, ws.x, ws.r, ws.p, ws.ap, a, PAR_EVEN, dd)) return -1;
    const double b = ms_norm(dd) / rnsq;
    rnsq = ms_norm(dd);
    rn = ms_rn(c, ws.r, istop, rnsq);
    k_mscg_p<<<nbk, 256, 0, st>>>(n, (double2 *)ws.p, (const double2 *)ws.r, b, 1, none);
    ncg[0] += 1;
  }
  la_axpy(c, 64, psi, -1.0, 0.0, ws.x, PAR_EVEN, st);
  return rn <= tol ? 0 : 1;
}

// mscg (mscg.c:387) on the even sites; status[0] = total CG iterations or -1
static int mscg_dev(Ctx &c, const MsWork &ws, int nmu, const double *mu, const double *res, int nmx, int istop,
                    const void *eta, void *const *psi, std::vector<void *> &ph, int *status) {
  cudaStream_t st = c.stream;
  const size_t n = (size_t)c.g.volh * 12;
  const unsigned nbk = (unsigned)((n + 255) / 256);
  // alloc_cgs (mscg.c:115-184): base system = smallest |mu|
  int k0 = 0;
  for (int k = 1; k < nmu; k++)
    if (std::fabs(mu[k]) < std::fabs(mu[k0])) k0 = k;
  int cstop = 0;
  const double cmu = mu[k0];
  double ca = 1.0, cb = 0.0, ctol = res[k0], rn0, rn, rnsq;
  void *x = psi[k0];
  std::vector<MsShift> sh;
  for (int k = 0; k < nmu; k++) {
    if (k == k0) continue;
    MsShift s;
    s.stop = 0;
    s.s = mu[k] * mu[k] - mu[k0] * mu[k0];
    s.tol = res[k];
    s.ah = 1.0;
    s.bh = 0.0;
    s.gh = 1.0;
    s.rh = 1.0;
    s.xh = psi[k];
    s.ph = ph[sh.size()];
    sh.push_back(s);
  }
  // cg_init (mscg.c:187-213)
  la_zero(c, 64, x, PAR_EVEN, st);
  la_copy(c, 64, eta, 64, ws.r, PAR_EVEN, st);
  la_copy(c, 64, eta, 64, ws.p, PAR_EVEN, st);
  double dd[2];
  if (la_norm2(c, 64, eta, PAR_EVEN, dd)) return -1;
  rnsq = ms_norm(dd);
  rn = ms_rn(c, eta, istop, rnsq);
  rn0 = rn;
  ctol *= rn0;
  for (auto &s : sh) {
    la_zero(c, 64, s.xh, PAR_EVEN, st);
    la_copy(c, 64, eta, 64, s.ph, PAR_EVEN, st);
    s.tol *= rn0;
  }
  // set_stop_flag (mscg.c:299-315)
  auto set_stop = [&]() {
    cstop |= (rn < 0.99 * ctol);
    int ns = cstop;
    for (auto &s : sh) {
      s.stop |= ((s.gh * rn) < (0.99 * s.tol));
      ns += s.stop;
    }
    return ns;
  };
  int nstop = set_stop(), ncg = 0;
  while (ncg < nmx && nstop < nmu) {
    // cg_step1
    double wn2;
    if (ms_op2(c, cmu, ws.p, ws.w, ws.ap, &wn2)) return -1;
    double om = cb / ca;
    ca = rnsq / wn2;
    om *= ca;
    for (auto &s : sh)
      if (!s.stop) {
        s.rh = 1.0 / (1.0 + s.s * ca + (1.0 - s.rh) * om);
        s.ah = s.rh * ca;
      }
    // cg_step2 (base system) and cg_step3
    if (la_xr_norm2(c, x, ws.r, ws.p, ws.ap, ca, PAR_EVEN, dd)) return -1;
    const double rn2 = ms_norm(dd);
    cb = rn2 / rnsq;
    rnsq = rn2;
    rn = ms_rn(c, ws.r, istop, rnsq);
    for (auto &s : sh)
      if (!s.stop) {
        s.bh = s.rh * s.rh * cb;
        s.gh *= s.rh;
      }
    // cg_step2 (shifted solutions) and cg_step4, fused
    ShiftGroup g{};
    int upd_p = 1;
    size_t j = 0;
    do {
      g.n = 0;
      for (; j < sh.size() && g.n < MS_G; j++) {
        if (sh[j].stop) continue;
        g.xh[g.n] = (double2 *)sh[j].xh;
        g.ph[g.n] = (double2 *)sh[j].ph;
        g.ah[g.n] = sh[j].ah;
        g.bh[g.n] = sh[j].bh;
        g.gh[g.n] = sh[j].gh;
        g.n++;
      }
      k_mscg_p<<<nbk, 256, 0, st>>>(n, (double2 *)ws.p, (const double2 *)ws.r, cb, upd_p, g);
      upd_p = 0;
    } while (j < sh.size());
    ncg += 1;
    nstop = set_stop();
  }
  if (ncg == nmx && nstop < nmu) {
    status[0] = -1;
    return 0;
  }
  int ie = ms_check_res(c, ws, mu[k0], nmx, istop, res[k0] * rn0, eta, psi[k0], &ncg);
  if (ie < 0) return -1;
  for (int k = 0; k < nmu; k++) {
    if (k == k0) continue;
    const int ic = ms_check_res(c, ws, mu[k], nmx, istop, res[k] * rn0, eta, psi[k], &ncg);
    if (ic < 0) return -1;
    ie |= ic;
  }
  status[0] = ie ? -1 : ncg;
  return 0;
}

// tmcgm (modules/forces/tmcgm.c:100-150) on device fields: even sites of eta
// and of the nmu solutions psi[k]; returns 0, or -1 on an error
int tmcgm_dev(Ctx &c, int nmx, int istop, const double *res, int nmu, const double *mu, const void *eta,
              void *const *psi, int *ifail, int *status) {
  ifail[0] = 0;
  status[0] = 0;
  if (!c.have_ud || !c.have_sw) return fail("tmcgm: gauge or SW field missing on the device");
  if (nmu < 0) return fail("mscg: parameters are out of range");
  if (cg_reserve(c)) return -1;
  while (c.ws64.size() < 6) {
    void *q = nullptr;
    if (cudaMalloc(&q, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory (workspace)");
    c.ws64.push_back(q);
  }
  cudaStream_t st = c.stream;
  double u[2];
  if (la_unorm(c, 64, eta, PAR_EVEN, u)) return -1;
  const double rho0 = u[0];
  int rc = 0;
  if (c.sw_inv_fail & 2) {
    ifail[0] = -3;   // unsafe inversion of the odd SW term (tmcgm.c:110-115)
    for (int k = 0; k < nmu; k++) la_zero(c, 64, psi[k], PAR_EVEN, st);
  } else if (rho0 != 0.0) {
    // the checks of mscg.c:394-450
    if (nmu < 1 || nmx < 1 || istop < 0 || istop > 1) return fail("mscg: parameters are out of range");
    for (int k = 0; k < nmu; k++)
      if (res[k] <= DBL_EPSILON) return fail("mscg: improper choice of residues");
    MsWork ws{c.ws64[0], c.ws64[1], c.ws64[2], c.ws64[3], c.ws64[5]};
    void *e = c.ws64[4];
    la_copy(c, 64, eta, 64, e, PAR_EVEN, st);
    la_scale(c, 64, e, 1.0 / rho0, PAR_EVEN, st);
    // the shifted directions live on the even sites only: half fields
    std::vector<void *> ph;
    for (int k = 1; k < nmu; k++) {
      void *q = nullptr;
      if (cudaMalloc(&q, spinor_bytes(c, 64) / 2) != cudaSuccess) {
        for (void *f : ph) cudaFree(f);
        return fail("out of device memory (multi-shift directions)");
      }
      ph.push_back(q);
    }
    rc = mscg_dev(c, ws, nmu, mu, res, nmx, istop, e, psi, ph, status);
    cudaStreamSynchronize(st);
    for (void *f : ph) cudaFree(f);
    if (rc == 0) {
      for (int k = 0; k < nmu; k++) la_scale(c, 64, psi[k], rho0, PAR_EVEN, st);
      if (status[0] < 0) {
        ifail[0] = -1;
        status[0] = nmx;
      }
    }
  } else {
    for (int k = 0; k < nmu; k++) la_zero(c, 64, psi[k], PAR_EVEN, st);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("tmcgm: CUDA error");
  return rc;
}

}  // namespace qcd
