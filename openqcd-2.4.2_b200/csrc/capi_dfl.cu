// C entry points of the deflation part: the reference's names from
// include/dfl.h and include/little.h, plus the b200_* parameter setters and
// device-layout variants.  Little vectors (Ns complex_dble per DFL block, in
// the reference's block order) and spinor fields (reference layout) may be
// in host or device memory.
#include "lib.h"
#include "../../include/openqcd_b200.h"
#include <cfloat>
#include <cmath>
#include <vector>

namespace qcd {

static int dfl_ready(Ctx &c) {
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (!c.dfl.ready) return fail("deflation parameters are not set (b200_set_dfl_parms)");
  return 0;
}

static int fields_ready(Ctx &c) {
  if (!c.have_ud || !c.have_sw) return fail("gauge or SW field missing on the device");
  if (!c.tmp32 && cudaMalloc(&c.tmp32, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory");
  if (!c.tmp64 && cudaMalloc(&c.tmp64, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory");
  return 0;
}

// little-vector staging: two device buffers of nv complex doubles
static double2 *lbuf(Ctx &c, int k) {
  DflState &d = c.dfl;
  while ((int)d.lvd.size() < 4) {
    double2 *p = nullptr;
    if (cudaMalloc(&p, (size_t)d.nv * sizeof(double2)) != cudaSuccess) { fail("out of device memory"); return nullptr; }
    d.lvd.push_back(p);
  }
  return d.lvd[k];
}

static void *spinor_stage(Ctx &c, int prec, int k) {
  std::vector<void *> &v = prec == 64 ? c.ws64 : c.ws32;
  while ((int)v.size() <= k) {
    void *p = nullptr;
    if (cudaMalloc(&p, spinor_bytes(c, prec)) != cudaSuccess) { fail("out of device memory"); return nullptr; }
    v.push_back(p);
  }
  return v[k];
}

static int stage_bytes_ok(Ctx &c, size_t n) {
  if (c.stage_bytes >= n) return 0;
  cudaFree(c.stage);
  c.stage = nullptr;
  c.stage_bytes = 0;
  if (cudaMalloc(&c.stage, n) != cudaSuccess) return fail("out of device memory (staging)");
  c.stage_bytes = n;
  return 0;
}

// reference-layout FP32 field (host or device) -> device-layout field
static int ref32_in(Ctx &c, const void *q, void *dev) {
  size_t nb = spinor_bytes(c, 32);
  if (stage_bytes_ok(c, nb)) return -1;
  cudaMemcpyAsync(c.stage, q, nb, cudaMemcpyDefault, c.stream);
  return spinor_from_ref(c, 32, c.stage, dev, c.stream);
}

static int ref32_out(Ctx &c, const void *dev, void *q) {
  size_t nb = spinor_bytes(c, 32);
  if (stage_bytes_ok(c, nb)) return -1;
  if (spinor_to_ref(c, 32, dev, c.stage, c.stream)) return -1;
  cudaMemcpyAsync(q, c.stage, nb, cudaMemcpyDefault, c.stream);
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("CUDA error");
}

}  // namespace qcd

using qcd::Ctx;
using qcd::ctx;
using qcd::fail;

extern "C" {

int b200_set_dfl_parms(const int bs[4], int Ns) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (qcd::dd_unsupported(c, "deflation")) return -1;
  return qcd::dfl_set_parms(c, bs, Ns);
}

int b200_set_dfl_pro_parms(int nkv, int nmx, double res, int nmx_gcr, double res_gcr) {
  // modules/flags/dfl_parms.c:300-302
  if (nkv < 2 || nmx < 1 || res <= DBL_EPSILON || nmx_gcr < 2 || res_gcr <= FLT_EPSILON)
    return fail("set_dfl_pro_parms: improper parameter values");
  qcd::DflState &d = ctx().dfl;
  d.nkv = nkv; d.nmx = nmx; d.res = res; d.nmx_gcr = nmx_gcr; d.res_gcr = res_gcr;
  return 0;
}

int b200_set_dfl_gen_parms(double kappa, double mu, int ninv, int nmr, int ncy) {
  // modules/flags/dfl_parms.c:379-380
  if (ninv < 4 || nmr < 1 || ncy < 1 || kappa < 0.0) return fail("set_dfl_gen_parms: parameters are out of range");
  qcd::DflState &d = ctx().dfl;
  d.gen_kappa = kappa; d.gen_mu = mu; d.gen_ninv = ninv; d.gen_nmr = nmr; d.gen_ncy = ncy;
  d.gen_set = true;
  return 0;
}

int b200_dfl_profile(int on, double *out) {
  qcd::DflState &d = ctx().dfl;
  if (out)
    for (int k = 0; k < 6; k++) out[k] = d.prof[k];
  if (on && !d.profile)
    for (int k = 0; k < 6; k++) d.prof[k] = 0.0;
  d.profile = on != 0;
  d.prof_t0 = 0.0;
  return 0;
}

// Device timing of the deflation kernels (no reference counterpart): what =
// 0 restriction of an FP32 field, 1 prolongation, 2 Awhat_dble, 3 Aw_dble,
// 4 ltl_gcr on a random little vector (status[0] of the last solve in *its),
// 5, 6, 7 the batched restriction, prolongation and little solver on four
// right-hand sides, 8 the batched Awhat, 9 the batched little solver on one
// right-hand side, 10 the block orthonormalisation of the subspace (in
// place), 11 the little-operator set-up (set_Awhat), 12 ltl_gcr with the
// reference's algorithm (fgcr4vd + gcr4v + global-mode deflation).
int b200_dfl_time(int what, int n, float *ms, int *its) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return -1;
  qcd::DflState &d = c.dfl;
  if (!d.have_basis) return fail("dfl_time: no deflation subspace");
  if ((what == 2 || what == 3 || what == 4 || what == 12) &&
      qcd::dfl_set_Awhat(c, d.aw_valid ? d.aw_mu : 0.0, c.stream) < 0)
    return -1;
  void *f = qcd::spinor_stage(c, 32, 0);
  double2 *a = qcd::lbuf(c, 0), *b = qcd::lbuf(c, 1), *t = qcd::lbuf(c, 2);
  if (!f || !a || !b || !t) return -1;
  qcd::gen_uniform_spinor32(c, f, 11, c.stream);
  qcd::dfl_restrict(c, 32, f, a, c.stream);
  // four fields and little vectors for the batched kernels (what >= 5)
  const void *fs[4];
  double2 *vs[4];
  if (what >= 5) {
    if (qcd::dfl_batch_alloc(c) || qcd::ensure_lvd_n(c, 8)) return -1;
    for (int i = 0; i < 4; i++) {
      void *fi = qcd::spinor_stage(c, 32, 1 + i);
      if (!fi) return -1;
      qcd::gen_uniform_spinor32(c, fi, 20 + i, c.stream);
      fs[i] = fi;
      vs[i] = d.lvd[4 + i];
      cudaMemcpyAsync(vs[i], a, (size_t)d.nv * sizeof(double2), cudaMemcpyDeviceToDevice, c.stream);
    }
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c.stream);
  int st[2] = {0, 0}, fl = 0;
  for (int i = 0; i < n; i++) {
    if (what == 0) qcd::dfl_restrict(c, 32, f, b, c.stream);
    else if (what == 1) qcd::dfl_prolong(c, a, f, c.stream);
    else if (what == 2) qcd::dfl_Awhat(c, a, b, t, c.stream);
    else if (what == 3) qcd::dfl_Aw(c, a, b, c.stream);
    else if (what == 4) qcd::dfl_ltl_gcr(c, d.aw_mu, a, b, &fl, st, c.stream);
    else if (what == 12) qcd::ltl_gcr_ref(c, d.aw_mu, a, b, &fl, st, c.stream);
    else if (what == 5) qcd::dfl_restrict_b(c, 4, fs, vs, c.stream);
    else if (what == 6) qcd::dfl_prolong_b(c, 4, (const double2 *const *)vs, (void *const *)fs, c.stream);
    else if (what == 7 || what == 9) {
      int f4[4], s4[4];
      const int nr = what == 7 ? 4 : 1;
      qcd::ltl_gcr_b(c, d.aw_mu, nr, (const double2 *const *)vs, vs + 4 - nr, f4, s4, c.stream);
      st[0] = s4[0];
    } else if (what == 10) {
      qcd::dfl_subspace_dev(c, d.basis, c.stream);   // re-orthonormalise the basis in place
    } else if (what == 11) {
      d.awhat_valid = d.aw_valid = false;
      qcd::dfl_set_Awhat(c, d.aw_mu, c.stream);
    } else {
      qcd::dfl_Awhat_b(c, 4, (const double2 *const *)vs, vs + 0, vs + 0, c.stream);
    }
  }
  cudaEventRecord(e1, c.stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (its) *its = st[0];
  if (cudaGetLastError() != cudaSuccess) return fail("dfl_time: CUDA error");
  return qcd::dfl_batch_check(c);
}

// Several systems at once (solver_batch.cu); device fields in the library's
// layout.  status needs 2*nrhs entries when dfl != 0.
int b200_dev_gcr_batch(int nrhs, int dfl, int nkv, int nmx, int istop, double res, const double *mu,
                       void *const *eta, void *const *psi, double *rho, int *ifail, int *status) {
  Ctx &c = ctx();
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (qcd::fields_ready(c) || qcd::dd_unsupported(c, "batched solves")) return -1;
  return qcd::gcr_batch(c, nrhs, dfl, nkv, nmx, istop, res, mu, (const void *const *)eta, psi, rho, ifail, status);
}

// Free the solvers' work fields (they are kept between calls otherwise).
int b200_release_workspace(void) {
  Ctx &c = ctx();
  qcd::gcr_batch_release();
  for (void *p : c.ws32) cudaFree(p);
  for (void *p : c.ws64) cudaFree(p);
  c.ws32.clear();
  c.ws64.clear();
  // the SAP graphs address the library-owned SAP fields: both go together
  qcd::graphs_release();
  for (int k = 0; k < 3; k++) {
    cudaFree(c.sap_fld[k]);
    c.sap_fld[k] = nullptr;
    cudaFree(c.sap_mfld[k]);
    c.sap_mfld[k] = nullptr;
  }
  c.sap_mfld_n = 0;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : fail("CUDA error");
}

int b200_dfl_nv(void) { return ctx().dfl.ready ? ctx().dfl.nv : 0; }

// Load basis vector l of every block from a global field in the reference
// layout (host or device).  The blocks' vectors are used as given.
int b200_dfl_set_basis(int l, const spinor *field) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return -1;
  if (l < 0 || l >= c.dfl.Ns) return fail("dfl_set_basis: index out of range");
  if (qcd::ref32_in(c, field, c.dfl.basis[l])) return -1;
  c.dfl.have_basis = true;
  c.dfl.aw_valid = c.dfl.awhat_valid = false;
  qcd::ltl_forget_lmodes(c);   // they belong to the previous basis
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("CUDA error");
}

int b200_dfl_get_basis(int l, spinor *field) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return -1;
  if (l < 0 || l >= c.dfl.Ns) return fail("dfl_get_basis: index out of range");
  return qcd::ref32_out(c, c.dfl.basis[l], field);
}

// dfl_subspace.c:171: the basis from Ns global fields (reference layout)
void dfl_subspace(spinor **mds) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return;
  std::vector<void *> modes;
  for (int l = 0; l < c.dfl.Ns; l++) {
    void *f = qcd::spinor_stage(c, 32, l);
    if (!f || qcd::ref32_in(c, mds[l], f)) return;
    modes.push_back(f);
  }
  qcd::dfl_subspace_dev(c, modes, c.stream, true);
}

void dfl_s2vd(spinor *s, complex_dble *vd) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || !c.dfl.have_basis) { if (c.dfl.ready) fail("dfl_s2vd: no deflation subspace"); return; }
  void *f = qcd::spinor_stage(c, 32, 0);
  double2 *v = qcd::lbuf(c, 0);
  if (!f || !v || qcd::ref32_in(c, s, f)) return;
  qcd::dfl_restrict(c, 32, f, v, c.stream);
  cudaMemcpyAsync(vd, v, (size_t)c.dfl.nv * sizeof(double2), cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

void dfl_vd2s(complex_dble *vd, spinor *s) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || !c.dfl.have_basis) { if (c.dfl.ready) fail("dfl_vd2s: no deflation subspace"); return; }
  void *f = qcd::spinor_stage(c, 32, 0);
  double2 *v = qcd::lbuf(c, 0);
  if (!f || !v) return;
  cudaMemcpyAsync(v, vd, (size_t)c.dfl.nv * sizeof(double2), cudaMemcpyDefault, c.stream);
  qcd::dfl_prolong(c, v, f, c.stream);
  qcd::ref32_out(c, f, s);
}

// dfl_s2vd / dfl_vd2s of nr fields at once through the batched kernels
// (four fields per pass on the tensor cores, the rest on the CUDA cores)
int b200_dfl_s2vd_multi(int nr, spinor *const *s, complex_dble *const *vd) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || !c.dfl.have_basis) return c.dfl.ready ? fail("dfl_s2vd_multi: no deflation subspace") : -1;
  if (nr < 1 || nr > 16) return fail("dfl_s2vd_multi: nr must be in [1, 16]");
  if (qcd::dfl_batch_alloc(c) || qcd::ensure_lvd_n(c, nr)) return -1;
  std::vector<const void *> f(nr);
  for (int r = 0; r < nr; r++) {
    void *p = qcd::spinor_stage(c, 32, r);
    if (!p || qcd::ref32_in(c, s[r], p)) return -1;
    f[r] = p;
  }
  qcd::dfl_restrict_b(c, nr, f.data(), c.dfl.lvd.data(), c.stream);
  for (int r = 0; r < nr; r++)
    cudaMemcpyAsync(vd[r], c.dfl.lvd[r], (size_t)c.dfl.nv * sizeof(double2), cudaMemcpyDefault, c.stream);
  if (b200_sync()) return -1;
  return qcd::dfl_batch_check(c);
}

int b200_dfl_vd2s_multi(int nr, complex_dble *const *vd, spinor *const *s) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || !c.dfl.have_basis) return c.dfl.ready ? fail("dfl_vd2s_multi: no deflation subspace") : -1;
  if (nr < 1 || nr > 16) return fail("dfl_vd2s_multi: nr must be in [1, 16]");
  if (qcd::dfl_batch_alloc(c) || qcd::ensure_lvd_n(c, nr)) return -1;
  std::vector<void *> f(nr);
  for (int r = 0; r < nr; r++) {
    f[r] = qcd::spinor_stage(c, 32, r);
    if (!f[r]) return -1;
    cudaMemcpyAsync(c.dfl.lvd[r], vd[r], (size_t)c.dfl.nv * sizeof(double2), cudaMemcpyDefault, c.stream);
  }
  qcd::dfl_prolong_b(c, nr, (const double2 *const *)c.dfl.lvd.data(), f.data(), c.stream);
  for (int r = 0; r < nr; r++)
    if (qcd::ref32_out(c, f[r], s[r])) return -1;
  return qcd::dfl_batch_check(c);
}

void set_Aw(double mu) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return;
  qcd::dfl_set_Aw(c, mu, c.stream);
}

int set_Awhat(double mu) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return -1;
  return qcd::dfl_set_Awhat(c, mu, c.stream);
}

static void little_apply(int which, complex_dble *v, complex_dble *w) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return;
  qcd::DflState &d = c.dfl;
  // Aw, Awoe, Aweo need the little operator, Awhat, Aweeinv, Awooinv the
  // even-odd preconditioned one (Aw.c:44-48)
  const bool hat = which >= 1 && which <= 3;
  if (!d.aw_valid || (hat && !d.awhat_valid)) { fail("Aw: the little operator is not set (set_Aw / set_Awhat)"); return; }
  double2 *a = qcd::lbuf(c, 0), *b = qcd::lbuf(c, 1), *t = qcd::lbuf(c, 2);
  if (!a || !b || !t) return;
  size_t nb = (size_t)d.nv * sizeof(double2);
  cudaMemcpyAsync(a, v, nb, cudaMemcpyDefault, c.stream);
  cudaMemcpyAsync(b, w, nb, cudaMemcpyDefault, c.stream);
  if (which == 0) qcd::dfl_Aw(c, a, b, c.stream);
  else qcd::dfl_Awhat(c, a, b, t, c.stream);
  cudaMemcpyAsync(w, b, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

void Aw_dble(complex_dble *v, complex_dble *w) { little_apply(0, v, w); }

// Awhat_dble of nr little vectors at once (the batched path: four vectors
// per pass on the tensor cores with FP32 matrices, the rest in FP64)
int b200_Awhat_dble_multi(int nr, complex_dble *const *v, complex_dble *const *w) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return -1;
  qcd::DflState &d = c.dfl;
  if (!d.aw_valid || !d.awhat_valid) return fail("Awhat_dble_multi: the little operator is not set (set_Awhat)");
  if (nr < 1 || nr > 16) return fail("Awhat_dble_multi: nr must be in [1, 16]");
  if (qcd::ensure_lvd_n(c, 3 * nr)) return -1;
  const size_t nb = (size_t)d.nv * sizeof(double2);
  std::vector<double2 *> a(nr), b(nr), t(nr);
  for (int r = 0; r < nr; r++) {
    a[r] = d.lvd[r];
    b[r] = d.lvd[nr + r];
    t[r] = d.lvd[2 * nr + r];
    cudaMemcpyAsync(a[r], v[r], nb, cudaMemcpyDefault, c.stream);
    cudaMemcpyAsync(b[r], w[r], nb, cudaMemcpyDefault, c.stream);
  }
  qcd::dfl_Awhat_b(c, nr, (const double2 *const *)a.data(), b.data(), t.data(), c.stream);
  for (int r = 0; r < nr; r++) cudaMemcpyAsync(w[r], b[r], nb, cudaMemcpyDefault, c.stream);
  return b200_sync();
}
void Awhat_dble(complex_dble *v, complex_dble *w) { little_apply(1, v, w); }

double ltl_gcr(double mu, complex_dble *eta, complex_dble *psi, int *ifail, int *status) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return -1.0;
  qcd::DflState &d = c.dfl;
  double2 *a = qcd::lbuf(c, 2), *b = qcd::lbuf(c, 3);
  if (!a || !b) return -1.0;
  size_t nb = (size_t)d.nv * sizeof(double2);
  cudaMemcpyAsync(a, eta, nb, cudaMemcpyDefault, c.stream);
  double rho;
  if (d.ltl_kind == 1) {
    rho = qcd::ltl_gcr_ref(c, mu, a, b, ifail, status, c.stream);
  } else {
    rho = qcd::dfl_ltl_gcr(c, mu, a, b, ifail, status, c.stream);
    status[1] = 0;
  }
  cudaMemcpyAsync(psi, b, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
  return rho;
}

// RHS tiles (fields per pass) the autotuner chose for the streamed
// restriction (tile[0]) and prolongation (tile[1]), 0 if not tuned yet, and
// the times of four fields with tiles 1, 2, 4 (ms[0..2] restriction,
// ms[3..5] prolongation)
int b200_rhs_tiles(int *tile, int *tc, float *ms) { return qcd::rhs_tiles(ctx(), tile, tc, ms); }
int b200_set_rhs_tiles(const int *tile, const int *tc) { return qcd::set_rhs_tiles(ctx(), tile, tc); }

int b200_set_ltl_solver(int kind) {
  Ctx &c = ctx();
  if (kind < 0 || kind > 1) return fail("set_ltl_solver: kind must be 0 or 1");
  const int prev = c.dfl.ltl_kind;
  c.dfl.ltl_kind = kind;
  return prev;
}

// ---- the eo pieces and the FP32 little operator (Aw_dble.c, Aw.c)
static void little_eo(int which, complex_dble *v, complex_dble *w) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return;
  qcd::DflState &d = c.dfl;
  if (!d.awhat_valid) { fail("Aw: the even-odd preconditioned little operator is not set (set_Awhat)"); return; }
  double2 *a = qcd::lbuf(c, 0), *b = qcd::lbuf(c, 1);
  if (!a || !b) return;
  const size_t nb = (size_t)d.nv * sizeof(double2);
  cudaMemcpyAsync(a, v, nb, cudaMemcpyDefault, c.stream);
  cudaMemcpyAsync(b, w, nb, cudaMemcpyDefault, c.stream);
  if (which == 0) qcd::dfl_Aweeinv(c, a, b, c.stream);
  else if (which == 1) qcd::dfl_Awooinv(c, a, b, c.stream);
  else if (which == 2) qcd::dfl_Awoe(c, a, b, c.stream);
  else qcd::dfl_Aweo(c, a, b, c.stream);
  cudaMemcpyAsync(w, b, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

void Aweeinv_dble(complex_dble *v, complex_dble *w) { little_eo(0, v, w); }
void Awooinv_dble(complex_dble *v, complex_dble *w) { little_eo(1, v, w); }
void Awoe_dble(complex_dble *v, complex_dble *w) { little_eo(2, v, w); }
void Aweo_dble(complex_dble *v, complex_dble *w) { little_eo(3, v, w); }

static void little_f32(int which, complex *v, complex *w) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return;
  qcd::DflState &d = c.dfl;
  if (!d.aw_valid || (which == 1 && !d.awhat_valid)) { fail("Aw: the little operator is not set (set_Aw / set_Awhat)"); return; }
  double2 *a = qcd::lbuf(c, 0), *b = qcd::lbuf(c, 1);   // used as float2 buffers
  if (!a || !b) return;
  const size_t nb = (size_t)d.nv * sizeof(float2);
  cudaMemcpyAsync(a, v, nb, cudaMemcpyDefault, c.stream);
  cudaMemcpyAsync(b, w, nb, cudaMemcpyDefault, c.stream);
  qcd::little32_apply(c, which, (const float2 *)a, (float2 *)b);
  cudaMemcpyAsync(w, b, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

void Aw(complex *v, complex *w) { little_f32(0, v, w); }
void Awhat(complex *v, complex *w) { little_f32(1, v, w); }
void Aweeinv(complex *v, complex *w) { little_f32(2, v, w); }
void Awooinv(complex *v, complex *w) { little_f32(3, v, w); }
void Awoe(complex *v, complex *w) { little_f32(4, v, w); }
void Aweo(complex *v, complex *w) { little_f32(5, v, w); }

// ---- global-mode deflation (ltl_modes.c)
int set_ltl_modes(void) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return -1;
  if (!c.dfl.awhat_valid) return fail("set_ltl_modes: the even-odd preconditioned little operator is not set");
  return qcd::ltl_set_modes(c);
}

complex_dble *ltl_matrix(void) {
  const double *m = qcd::ltl_matrix_host(ctx());
  return (complex_dble *)m;
}

static int ltl_ready(Ctx &c) {
  if (qcd::dfl_ready(c)) return -1;
  if (!qcd::ltl_matrix_host(c)) return fail("little modes are not set (set_ltl_modes)");
  return 0;
}

void dfl_Lvd(complex_dble *vd) {
  Ctx &c = ctx();
  if (ltl_ready(c)) return;
  double2 *a = qcd::lbuf(c, 0);
  const size_t nb = (size_t)c.dfl.nv * sizeof(double2);
  cudaMemcpyAsync(a, vd, nb, cudaMemcpyDefault, c.stream);
  qcd::dfl_Lvd_dev(c, a);
  cudaMemcpyAsync(vd, a, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

static void ltl_pair(int which, complex_dble *vd, complex_dble *wd) {
  Ctx &c = ctx();
  if (ltl_ready(c)) return;
  double2 *a = qcd::lbuf(c, 0), *b = qcd::lbuf(c, 1);
  const size_t nb = (size_t)c.dfl.nv * sizeof(double2);
  cudaMemcpyAsync(a, vd, nb, cudaMemcpyDefault, c.stream);
  cudaMemcpyAsync(b, wd, nb, cudaMemcpyDefault, c.stream);
  if (which == 0) qcd::dfl_LRvd_dev(c, a, b);
  else qcd::dfl_RLvd_dev(c, a, b);
  cudaMemcpyAsync(vd, a, nb, cudaMemcpyDefault, c.stream);
  cudaMemcpyAsync(wd, b, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

void dfl_LRvd(complex_dble *vd, complex_dble *wd) { ltl_pair(0, vd, wd); }
void dfl_RLvd(complex_dble *vd, complex_dble *wd) { ltl_pair(1, vd, wd); }

void dfl_Lv(complex *v) {
  Ctx &c = ctx();
  if (ltl_ready(c)) return;
  double2 *a = qcd::lbuf(c, 0);
  const size_t nb = (size_t)c.dfl.nv * sizeof(float2);
  cudaMemcpyAsync(a, v, nb, cudaMemcpyDefault, c.stream);
  qcd::dfl_Lv_dev(c, (float2 *)a);
  cudaMemcpyAsync(v, a, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
}

// little mode l (the mode's coefficients in the block basis, complex
// floats, nv of them): load, for a subspace that was uploaded as a basis
int b200_dfl_set_lmode(int l, const complex *v) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return -1;
  return qcd::ltl_lmode_set(c, l, v);
}

int b200_dev_dfl_modes(unsigned long long seed, int *ifail, int *status) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return -1;
  return qcd::dfl_modes_dev(c, seed, ifail, status);
}

// Start fields of the next dfl_modes call: Ns FP32 fields in the reference's
// storage order, one after another (host or device memory).
int b200_dfl_set_start_fields(const spinor *fields) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c)) return -1;
  qcd::DflState &d = c.dfl;
  while ((int)d.start.size() < d.Ns) {
    void *p = nullptr;
    if (cudaMalloc(&p, qcd::spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory");
    d.start.push_back(p);
  }
  for (int l = 0; l < d.Ns; l++)
    if (qcd::ref32_in(c, fields + (size_t)l * c.g.vol, d.start[l])) return -1;
  d.use_start = true;
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("CUDA error");
}

// dfl_modes.c:423 with the library's generator seeded by 1
void dfl_modes(int *ifail, int *status) {
  if (b200_dev_dfl_modes(1ull, ifail, status) < 0 && ifail[0] == 0) ifail[0] = -2;
}

double b200_dev_dfl_sap_gcr(int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                            int *ifail, int *status) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return -1.0;
  return qcd::dfl_sap_gcr_dev(c, nkv, nmx, istop, res, mu, eta, psi, ifail, status);
}

// dfl_sap_gcr.c:353 on reference-layout FP64 fields (host or device)
double dfl_sap_gcr(int nkv, int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi,
                   int *ifail, int *status) {
  Ctx &c = ctx();
  if (qcd::dfl_ready(c) || qcd::fields_ready(c)) return -1.0;
  size_t nb = qcd::spinor_bytes(c, 64);
  void *fe = nullptr, *fp = nullptr;
  if (cudaMalloc(&fe, nb) != cudaSuccess || cudaMalloc(&fp, nb) != cudaSuccess) { fail("out of device memory"); return -1.0; }
  if (qcd::stage_bytes_ok(c, nb)) return -1.0;
  cudaMemcpyAsync(c.stage, eta, nb, cudaMemcpyDefault, c.stream);
  qcd::spinor_from_ref(c, 64, c.stage, fe, c.stream);
  double rho = qcd::dfl_sap_gcr_dev(c, nkv, nmx, istop, res, mu, fe, fp, ifail, status);
  qcd::spinor_to_ref(c, 64, fp, c.stage, c.stream);
  cudaMemcpyAsync(psi, c.stage, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
  cudaFree(fe);
  cudaFree(fp);
  return rho;
}

// dfl_sap_gcr.c:383: retry once with a regenerated subspace if the first
// solve fails with ifail -1 or -2
double dfl_sap_gcr2(int nkv, int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi,
                    int *ifail, int *status) {
  ifail[1] = 0;
  for (int l = 0; l < 6; l++) status[l] = 0;
  double rho = dfl_sap_gcr(nkv, nmx, istop, res, mu, eta, psi, ifail, status);
  if (ifail[0] == -1 || ifail[0] == -2) {
    int st2[2] = {0, 0};
    b200_dev_dfl_modes(2ull, ifail + 1, st2);
    status[4] = st2[0];
    status[5] = st2[1];
    if (ifail[1] == 0) rho = dfl_sap_gcr(nkv, nmx, istop, res, mu, eta, psi, ifail + 1, status + 3);
  }
  return rho;
}

}  // extern "C"
