// Flexible GCR and the SAP+GCR solver on device-resident fields.
//
// fgcr_dev restates the reference's fgcr (modules/linsolv/fgcr.c:215-299,
// gcr_step :157, update_psi :181, get_res :128): Krylov vectors in FP32,
// Gram-Schmidt products accumulated in double, the small scalar arrays a, b,
// c in single precision on the host, the true residual recomputed in FP64 at
// every restart, and the restart rule rn < PRECISION_LIMIT * rn_old with
// PRECISION_LIMIT = 100 * FLT_EPSILON.  sap_gcr_dev restates
// modules/sap/sap_gcr.c:140-250 with Mop = ncy SAP cycles (sap_gcr.c:126).
#include "lib.h"
#include <cfloat>
#include <cmath>
#include <functional>

namespace qcd {

size_t spinor_bytes(const Ctx &c, int prec) { return (size_t)c.g.vol * 12 * (prec == 64 ? 16 : 8); }

static int reserve(Ctx &c, std::vector<void *> &ws, size_t n, int prec) {
  while (ws.size() < n) {
    void *p = nullptr;
    if (cudaMalloc(&p, spinor_bytes(c, prec)) != cudaSuccess) return fail("out of device memory (workspace)");
    ws.push_back(p);
  }
  return 0;
}

using DopFn = std::function<void(const void *s64, void *r64)>;
using MopFn = std::function<void(int k, const void *rho32, void *phi32, void *chi32)>;

double fgcr_core(const KrylovOps &o, int nkv, int nmx, int istop, double res, const void *eta, void *psi,
                 int *status, const DopFn &Dop, const MopFn &Mop, const std::vector<void *> &phi,
                 const std::vector<void *> &chi, void *rho, void *wrk) {
  if (nkv < 1 || nmx < 1 || res <= DBL_EPSILON || istop < 0 || istop > 1) {
    fail("fgcr: parameters are out of range");
    return -1.0;
  }
  std::vector<cplxf> a((size_t)nkv * nkv), cc(nkv);
  std::vector<float> b(nkv);
  const double PRECISION_LIMIT = (double)(100.0f * FLT_EPSILON);

  o.zero64(psi);
  o.copy64to32(eta, rho);
  double rn = o.res32(rho, istop);
  double tol = res * rn;
  status[0] = 0;

  while (rn > tol) {
    double rn_old = rn;
    int k;
    for (k = 0;; k++) {
      // gcr_step (fgcr.c:157)
      Mop(k, rho, phi[k], chi[k]);
      for (int l = 0; l < k; l++) {
        cplxf z = o.dot32(chi[l], chi[k]);
        a[(size_t)nkv * l + k] = z;
        o.axpy32(chi[k], -z.re, -z.im, chi[l]);
      }
      b[k] = o.normalize32(chi[k]);
      cc[k] = o.dot32(chi[k], rho);
      o.axpy32(rho, -cc[k].re, -cc[k].im, chi[k]);
      rn = o.res32(rho, istop);
      status[0] += 1;
      if (rn <= tol || rn < PRECISION_LIMIT * rn_old || k == nkv - 1 || status[0] >= nmx) break;
    }
    // update_psi (fgcr.c:181)
    for (int l = k; l >= 0; l--) {
      cplxf z = cc[l];
      for (int i = l + 1; i <= k; i++) {
        cplxf al = a[(size_t)l * nkv + i];
        z.re -= al.re * cc[i].re - al.im * cc[i].im;
        z.im -= al.re * cc[i].im + al.im * cc[i].re;
      }
      float r = 1.0f / b[l];
      cc[l].re = z.re * r;
      cc[l].im = z.im * r;
    }
    if (o.lincomb32) {
      std::vector<cplxf> cl;
      std::vector<void *> xl;
      for (int l = k; l >= 0; l--) {
        cl.push_back(cc[l]);
        xl.push_back(phi[l]);
      }
      o.lincomb32(rho, k + 1, cl.data(), xl.data());
    } else {
      o.zero32(rho);
      for (int l = k; l >= 0; l--) o.axpy32(rho, cc[l].re, cc[l].im, phi[l]);
    }
    o.add32to64(rho, psi);
    Dop(psi, wrk);
    o.diff64to32(eta, wrk, rho);
    rn = o.res32(rho, istop);
    if (status[0] >= nmx && rn > tol) {
      status[0] = -1;
      return rn;
    }
  }
  return rn;
}

// Vector operations on fields in the device layout (la_* of linalg.cu).
KrylovOps dev_krylov_ops(Ctx &c) {
  KrylovOps o;
  cudaStream_t st = c.stream;
  o.res32 = [&c](const void *x, int istop) {
    double r[4];
    if (istop) {
      la_unorm(c, 32, x, PAR_ALL, r);
      return (double)(float)r[0];
    }
    la_norm2(c, 32, x, PAR_ALL, r);
    return sqrt((double)(float)(r[0] + r[1]));
  };
  o.dot32 = [&c](const void *x, const void *y) {
    double r[4];
    la_dot(c, 32, x, y, PAR_ALL, r);
    return cplxf{(float)(r[0] + r[1]), (float)(r[2] + r[3])};
  };
  o.normalize32 = [&c, st](void *x) {
    double r[2];
    la_norm2(c, 32, x, PAR_ALL, r);
    float n = (float)sqrt((double)(float)(r[0] + r[1]));
    if (n != 0.0f) la_scale(c, 32, x, 1.0f / n, PAR_ALL, st);
    return n;
  };
  o.axpy32 = [&c, st](void *y, float ar, float ai, const void *x) { la_axpy(c, 32, y, ar, ai, x, PAR_ALL, st); };
  o.zero32 = [&c, st](void *x) { la_zero(c, 32, x, PAR_ALL, st); };
  o.lincomb32 = [&c, st](void *y, int n, const cplxf *cl, void *const *x) {
    std::vector<float> re(n), im(n);
    for (int l = 0; l < n; l++) {
      re[l] = cl[l].re;
      im[l] = cl[l].im;
    }
    la_lincomb32(c, y, n, re.data(), im.data(), x, st);
  };
  o.zero64 = [&c, st](void *x) { la_zero(c, 64, x, PAR_ALL, st); };
  o.copy64to32 = [&c, st](const void *x, void *y) { la_copy(c, 64, x, 32, y, PAR_ALL, st); };
  o.add32to64 = [&c, st](const void *s, void *d) { la_add_s2sd(c, s, d, PAR_ALL, st); };
  o.diff64to32 = [&c, st](const void *a, const void *b, void *r) { la_diff_sd2s(c, a, b, r, PAR_ALL, st); };
  return o;
}

double fgcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, const void *eta, void *psi, int *status,
                const DopFn &Dop, const MopFn &Mop) {
  if (reserve(c, c.ws32, 2 * nkv + 1, 32) || reserve(c, c.ws64, 2, 64)) return -1.0;
  std::vector<void *> phi(c.ws32.begin(), c.ws32.begin() + nkv),
      chi(c.ws32.begin() + nkv + 1, c.ws32.begin() + 2 * nkv + 1);
  return fgcr_core(dev_krylov_ops(c), nkv, nmx, istop, res, eta, psi, status, Dop, Mop, phi, chi, c.ws32[nkv], c.ws64[0]);
}

// Device twin of sap_gcr(): eta, psi FP64 device fields (psi may equal eta).
double sap_gcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                   int *ifail, int *status) {
  ifail[0] = 0;
  status[0] = 0;
  if (!c.sap_set) { fail("sap_gcr: SAP parameters are not set"); return -1.0; }
  if (!c.have_ud || !c.have_sw) { fail("sap_gcr: gauge or SW field missing on the device"); return -1.0; }
  if (sap_prepare(c, c.stream)) return -1.0;
  double rho = 0.0;
  if (c.isolv == 1 && (c.sw_inv_fail & 2)) {
    ifail[0] = -3;
  } else {
    double u[2];
    la_unorm(c, 64, eta, PAR_ALL, u);
    double rho0 = u[0];
    if (rho0 != 0.0) {
      if (reserve(c, c.ws64, 3, 64) || reserve(c, c.ws32, 2 * nkv + 2, 32)) return -1.0;
      void *rsd = c.ws64[1];
      void *phib = c.ws32[2 * nkv + 1];
      la_copy(c, 64, eta, 64, rsd, PAR_ALL, c.stream);
      la_scale(c, 64, rsd, 1.0 / rho0, PAR_ALL, c.stream);
      const float muf = (float)mu;
      const int isolv = c.isolv, nmr = c.nmr, ncy = c.ncy;
      DopFn Dop = [&](const void *s, void *r) { dirac_op<double>(c, 0, mu, s, r, c.tmp64, c.stream); };
      const int kind = c.precond;
      const bool net = kind == 1 || kind == 2 || kind == 4;
      if (net) {
        if (!c.net.ready) { fail("sap_gcr: the network preconditioner has no weights"); return -1.0; }
        if (reserve(c, c.ws32, 2 * nkv + 4, 32)) return -1.0;
      }
      void *ws2 = net ? c.ws32[2 * nkv + 2] : nullptr;
      void *ws3 = kind == 4 ? c.ws32[2 * nkv + 3] : nullptr;
      bool fallback = false;
      double rn_prev = -1.0;
      auto sap_mop = [&](const void *rh, void *ph, void *ch) {
        qcd::sap_mop(c, muf, isolv, nmr, ncy, rh, ph, ch, phib, c.stream);
      };
      MopFn Mop = [&](int, const void *rh, void *ph, void *ch) {
        if (kind == 0) {
          sap_mop(rh, ph, ch);
        } else if (kind == 4) {
          // SAP plus the network's estimate of the error SAP leaves (a
          // network trained on (residual, SAP-error) pairs):
          // ph = M_sap rh + N rh, ch = D ph; the network part is dropped
          // once a step reduces the residual by less than 10 %
          double r2[2];
          la_norm2(c, 32, rh, PAR_ALL, r2);
          const double rn = sqrt(r2[0] + r2[1]);
          if (rn_prev > 0.0 && rn > 0.9 * rn_prev) fallback = true;
          rn_prev = rn;
          sap_mop(rh, ph, ch);
          if (!fallback) {
            net_apply(c, rh, ws2, true, c.stream);
            dirac_op<float>(c, 0, muf, ws2, ws3, c.tmp32, c.stream);
            la_axpy(c, 32, ph, 1.0, 0.0, ws2, PAR_ALL, c.stream);
            la_axpy(c, 32, ch, 1.0, 0.0, ws3, PAR_ALL, c.stream);
          }
        } else if (kind == 3) {
          la_copy(c, 32, rh, 32, ph, PAR_ALL, c.stream);
          dirac_op<float>(c, 0, muf, ph, ch, c.tmp32, c.stream);
        } else if (kind == 1) {
          // the network, until a step reduces the residual by less than
          // 10 %; SAP from then on
          double r2[2];
          la_norm2(c, 32, rh, PAR_ALL, r2);
          const double rn = sqrt(r2[0] + r2[1]);
          if (rn_prev > 0.0 && rn > 0.9 * rn_prev) fallback = true;
          rn_prev = rn;
          if (fallback) {
            sap_mop(rh, ph, ch);
          } else {
            net_apply(c, rh, ph, true, c.stream);
            dirac_op<float>(c, 0, muf, ph, ch, c.tmp32, c.stream);
          }
        } else {
          // the network, then SAP on what it leaves: ph = M rh + SAP(rh - D M rh)
          net_apply(c, rh, ws2, true, c.stream);
          dirac_op<float>(c, 0, muf, ws2, ch, c.tmp32, c.stream);
          la_diff(c, 32, rh, ch, PAR_ALL, c.stream);            // ch = rh - D M rh
          la_zero(c, 32, ph, PAR_ALL, c.stream);
          sap_cycles(c, muf, isolv, nmr, ncy, ph, ch, phib, c.stream);
          la_diff(c, 32, rh, ch, PAR_ALL, c.stream);            // ch = rh - final residual = D ph_total
          la_axpy(c, 32, ph, 1.0, 0.0, ws2, PAR_ALL, c.stream);
        }
      };
      // psi may alias eta: fgcr only reads rsd from here on
      rho = fgcr_dev(c, nkv, nmx, istop, res, rsd, psi, status, Dop, Mop);
      la_scale(c, 64, psi, rho0, PAR_ALL, c.stream);
      rho *= rho0;
      if (status[0] < 0) {
        ifail[0] = -1;
        status[0] = nmx;
      }
    } else {
      la_zero(c, 64, psi, PAR_ALL, c.stream);
    }
  }
  if (ifail[0] <= -2) {
    if (psi != eta) la_zero(c, 64, psi, PAR_ALL, c.stream);
    double r[2];
    if (istop) { la_unorm(c, 64, eta, PAR_ALL, r); rho = r[0]; }
    else { la_norm2(c, 64, eta, PAR_ALL, r); rho = sqrt(r[0]); }
  }
  cudaStreamSynchronize(c.stream);
  return rho;
}

}  // namespace qcd
