// Block-shape autotuner (b200_tune_block_shape, no reference counterpart).
//
// The SAP block is also the tile of the device layout and the deflation
// block, so its shape decides both the cost of a SAP cycle (sites per CTA,
// shared memory, the boundary share) and how much of the operator the
// block solves capture (the convergence of the Krylov solver).  The tuner
// measures the product directly: for every candidate shape it lays the
// resident gauge and SW fields out again, runs a fixed number of steps of
// the SAP-preconditioned GCR (the library's sap_gcr, with the current SAP
// parameters) on a Gaussian source, and scores the shape by the residual
// reduction per second, ln(|eta| / |r|) / t.  With deflation (Ns > 0) the
// shape is also the DFL block, which decides how much of the low modes the
// subspace holds: each candidate then gets its own subspace (dfl_modes with
// the current generation parameters, not timed) and the steps timed are
// those of the deflated solver.  The fastest-converging shape stays in
// force.
#include "lib.h"
#include "../../include/openqcd_b200.h"
#include <chrono>
#include <cmath>
#include <vector>

namespace qcd {

double sap_gcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                   int *ifail, int *status);

// a shape the geometry and the SAP kernels accept (geometry_init, sap_prepare)
static bool shape_ok(const int L[4], const int bs[4]) {
  int vb = 1;
  for (int mu = 0; mu < 4; mu++) {
    if (bs[mu] < 2 || bs[mu] % 2 || bs[mu] > 255 || L[mu] % bs[mu] || (L[mu] / bs[mu]) % 2) return false;
    vb *= bs[mu];
  }
  return vb <= 1536;
}

}  // namespace qcd

extern "C" int b200_tune_block_shape(const int *cand, int ncand, int nsteps, double mu, int Ns, float *score) {
  qcd::Ctx &c = qcd::ctx();
  if (!c.ready || !c.have_ud || !c.have_sw) return qcd::fail("tune_block_shape: geometry and fields must be set");
  if (!c.have_ipt) return qcd::fail("tune_block_shape: needs the reference site order (ipt[] at the geometry call)");
  if (!c.sap_set) return qcd::fail("tune_block_shape: SAP parameters are not set");
  if (qcd::dd_unsupported(c, "tune_block_shape")) return -1;
  if (ncand < 1 || nsteps < 1 || Ns < 0) return qcd::fail("tune_block_shape: no candidates or steps");
  if (Ns > 0 && !c.dfl.gen_set) return qcd::fail("tune_block_shape: deflation generation parameters are not set");
  const int L[4] = {c.g.L[0], c.g.L[1], c.g.L[2], c.g.L[3]};
  const int bs0[4] = {c.g.bs[0], c.g.bs[1], c.g.bs[2], c.g.bs[3]};
  const int isolv = c.isolv, nmr = c.nmr, ncy = c.ncy;
  const std::vector<int> ipt = c.h_ipt;
  const size_t V = (size_t)c.g.vol;
  std::vector<double> ud(V * 4 * 18), sw(V * 2 * 36);
  if (b200_download_ud((su3_dble *)ud.data()) || b200_download_swd((pauli_dble *)sw.data(), 0)) return -1;
  // lay the fields out with block shape bs and set SAP up for it
  auto load = [&](const int *bs) {
    if (b200_geometry(L, bs, ipt.data()) || b200_upload_ud((const su3_dble *)ud.data())) return -1;
    if (b200_upload_swd((const pauli_dble *)sw.data()) < 0) return -1;
    return b200_set_sap_parms(bs, isolv, nmr, ncy);
  };
  int best = -1;
  double best_score = 0.0;
  for (int i = 0; i < ncand; i++) {
    const int *bs = cand + 4 * i;
    if (score) score[i] = -1.0f;
    if (!qcd::shape_ok(L, bs)) continue;
    if (load(bs)) return -1;
    void *eta = nullptr, *psi = nullptr;
    const size_t nb = qcd::spinor_bytes(c, 64);
    if (cudaMalloc(&eta, nb) != cudaSuccess || cudaMalloc(&psi, nb) != cudaSuccess) {
      cudaFree(eta);
      return qcd::fail("tune_block_shape: out of device memory");
    }
    qcd::gen_spinor(c, 64, eta, 1.0, 31337, c.stream);
    double n2[2];
    qcd::la_norm2(c, 64, eta, qcd::PAR_ALL, n2);
    int ifail = 0, status[3] = {0, 0, 0};
    if (Ns > 0) {
      int fl = 0, st[2] = {0, 0};
      if (qcd::dfl_set_parms(c, bs, Ns) < 0 || qcd::dfl_modes_dev(c, 1, &fl, st) < 0 || fl) {
        cudaFree(eta);
        cudaFree(psi);
        continue;
      }
    }
    auto solve = [&](int n) {
      return Ns > 0 ? qcd::dfl_sap_gcr_dev(c, 16, n, 0, 1e-12, mu, eta, psi, &ifail, status)
                    : qcd::sap_gcr_dev(c, 16, n, 0, 1e-12, mu, eta, psi, &ifail, status);
    };
    // warm-up: the SAP kernel's own launch tuning and the graphs
    solve(2);
    cudaStreamSynchronize(c.stream);
    const auto t0 = std::chrono::steady_clock::now();
    const double rn = solve(nsteps);
    cudaStreamSynchronize(c.stream);
    const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    cudaFree(eta);
    cudaFree(psi);
    if (rn <= 0.0 || t <= 0.0) continue;
    const double s = std::log(std::sqrt(n2[0] + n2[1]) / rn) / t;
    if (score) score[i] = (float)s;
    if (best < 0 || s > best_score) {
      best = i;
      best_score = s;
    }
  }
  if (load(best >= 0 ? cand + 4 * best : bs0)) return -1;
  return best >= 0 ? best : qcd::fail("tune_block_shape: no candidate shape fits the lattice");
}
