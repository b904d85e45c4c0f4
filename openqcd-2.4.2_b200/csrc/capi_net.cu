// C entry points of the learned preconditioner (net.cu; no reference
// counterpart).  Fields are FP32 device fields in the library's layout.
#include "lib.h"
#include "../../include/openqcd_b200.h"
#include <vector>

namespace qcd {
double sap_gcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                   int *ifail, int *status);
}

using qcd::Ctx;
using qcd::ctx;
using qcd::fail;

extern "C" {

int b200_net_nweights(void) { return qcd::net_nweights(); }

int b200_net_init(unsigned long long seed, float scale) {
  if (qcd::dd_unsupported(ctx(), "the learned preconditioner")) return -1;
  return qcd::net_init(ctx(), seed, scale);
}

int b200_net_set_weights(const float *w) {
  if (qcd::dd_unsupported(ctx(), "the learned preconditioner")) return -1;
  return qcd::net_set_weights(ctx(), w);
}

int b200_net_get_weights(float *w) { return qcd::net_get_weights(ctx(), w); }

int b200_net_apply(const void *in, void *out, int half) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (qcd::net_apply(c, in, out, half != 0, c.stream)) return -1;
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("network: CUDA error");
}

int b200_net_grad(const void *r, const void *e, double *loss, float *grad) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  return qcd::net_grad(c, r, e, loss, grad);
}

int b200_net_train(int npairs, void *const *r, void *const *e, int steps, int batch, float lr,
                   unsigned long long seed, float *loss_hist) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  return qcd::net_train(c, npairs, (const void *const *)r, (const void *const *)e, steps, batch, lr, seed, loss_hist);
}

int b200_net_batch_grad(int npairs, void *const *r, void *const *e, double *loss, float *grad) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  return qcd::net_batch_grad(c, npairs, (const void *const *)r, (const void *const *)e, loss, grad);
}

int b200_net_adam_step(const float *grad, float lr) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  return qcd::net_adam(c, grad, lr);
}

// Training pairs from the plain solver: r[k] a Gaussian source (FP32 copy),
// e[k] = Dw(mu)^-1 r[k] from sap_gcr to relative residual res (FP32 copy).
int b200_net_make_pairs(int npairs, void *const *r, void *const *e, double mu, double res,
                        unsigned long long seed) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (!c.sap_set) return fail("net_make_pairs: SAP parameters are not set");
  void *eta = nullptr, *psi = nullptr;
  if (cudaMalloc(&eta, qcd::spinor_bytes(c, 64)) != cudaSuccess ||
      cudaMalloc(&psi, qcd::spinor_bytes(c, 64)) != cudaSuccess)
    return fail("out of device memory");
  const int keep = c.precond;
  c.precond = 0;
  int rc = 0;
  for (int k = 0; k < npairs && rc == 0; k++) {
    if (qcd::gen_spinor(c, 64, eta, 1.0, seed * 7919ull + (uint64_t)k, c.stream)) { rc = -1; break; }
    int ifail = 0, status = 0;
    if (qcd::sap_gcr_dev(c, 16, 1024, 0, res, mu, eta, psi, &ifail, &status) < 0 || ifail) {
      rc = fail("net_make_pairs: the solver failed");
      break;
    }
    qcd::la_copy(c, 64, eta, 32, r[k], qcd::PAR_ALL, c.stream);
    qcd::la_copy(c, 64, psi, 32, e[k], qcd::PAR_ALL, c.stream);
  }
  c.precond = keep;
  cudaStreamSynchronize(c.stream);
  cudaFree(eta);
  cudaFree(psi);
  return rc;
}

// Training pairs for a network that corrects SAP: r[k] a Gaussian residual
// (FP32 copy), e[k] = Dw(mu)^-1 r[k] - M_sap r[k], the error the SAP
// preconditioner (ncy cycles from zero with the current SAP parameters)
// leaves, with Dw^-1 r from sap_gcr to relative residual res.
int b200_net_make_sap_pairs(int npairs, void *const *r, void *const *e, double mu, double res,
                            unsigned long long seed) {
  Ctx &c = ctx();
  if (b200_net_make_pairs(npairs, r, e, mu, res, seed)) return -1;
  void *psi = nullptr, *rho = nullptr, *phi = nullptr;
  const size_t nb = qcd::spinor_bytes(c, 32);
  if (cudaMalloc(&psi, nb) != cudaSuccess || cudaMalloc(&rho, nb) != cudaSuccess ||
      cudaMalloc(&phi, nb) != cudaSuccess) {
    cudaFree(psi);
    cudaFree(rho);
    return fail("out of device memory");
  }
  int rc = 0;
  for (int k = 0; k < npairs && rc == 0; k++) {
    qcd::la_zero(c, 32, psi, qcd::PAR_ALL, c.stream);
    qcd::la_copy(c, 32, r[k], 32, rho, qcd::PAR_ALL, c.stream);
    if (qcd::sap_cycles(c, (float)mu, c.isolv, c.nmr, c.ncy, psi, rho, phi, c.stream)) rc = -1;
    else qcd::la_axpy(c, 32, e[k], -1.0, 0.0, psi, qcd::PAR_ALL, c.stream);   // e = Dw^-1 r - M_sap r
  }
  cudaStreamSynchronize(c.stream);
  cudaFree(psi);
  cudaFree(rho);
  cudaFree(phi);
  return rc;
}

int b200_set_precond(int kind) {
  if (kind < 0 || kind > 4)
    return fail("set_precond: kind must be 0 (SAP), 1 (network), 2 (network + SAP), 3 (none), 4 (SAP + network)");
  ctx().precond = kind;
  return 0;
}

}  // extern "C"
