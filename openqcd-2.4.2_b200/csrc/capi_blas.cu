// Drop-in BLAS-1 (modules/linalg/salg.c, salg_dble.c) and the generic
// flexible GCR solver (modules/linsolv/fgcr.c) on caller arrays in the
// reference's storage order.
//
// Argument meaning follows the reference: vol sites, and with icom & 0x2 the
// reference's fields span vol sites per OpenMP thread, NTHREAD threads
// (sflds/README.icom), so the library covers vol * nthread sites with
// nthread set by b200_set_nthread() (default 1).  icom & 0x1 (sum over MPI
// processes) sums over the ranks of the domain decomposition (b200_dd_setup)
// in rank order in double-double, and is a no-op on one rank.  Arrays may be in
// device memory (used in place) or in host memory (staged through device
// buffers, written back when the call modifies them).
#include "lib.h"
#include "../../include/openqcd_b200.h"
#include <cfloat>
#include <cmath>
#include <vector>

namespace qcd {

static int ensure_stream(Ctx &c) {
  if (!c.stream && cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail("no CUDA device available");
  return 0;
}

static bool on_device(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// A device view of a caller array; slot selects one of three staging buffers.
struct View {
  Ctx &c;
  void *user;
  void *dev;
  size_t bytes;
  bool staged = false, write;
  View(Ctx &cc, const void *p, size_t n, int slot, bool w) : c(cc), user((void *)p), dev((void *)p), bytes(n), write(w) {
    if (on_device(p)) return;
    if (c.fstage_bytes[slot] < n) {
      cudaFree(c.fstage[slot]);
      c.fstage[slot] = nullptr;
      c.fstage_bytes[slot] = 0;
      if (cudaMalloc(&c.fstage[slot], n) != cudaSuccess) { fail("out of device memory (staging)"); dev = nullptr; return; }
      c.fstage_bytes[slot] = n;
    }
    dev = c.fstage[slot];
    staged = true;
    cudaMemcpyAsync(dev, p, n, cudaMemcpyHostToDevice, c.stream);
  }
  ~View() {
    if (staged && write && dev) {
      cudaMemcpyAsync(user, dev, bytes, cudaMemcpyDeviceToHost, c.stream);
      cudaStreamSynchronize(c.stream);
    }
  }
};

static size_t nsites(const Ctx &c, int vol, int icom) { return (size_t)vol * ((icom & 2) ? c.nthread : 1); }

static int dd_dot(int prec, int vol, int icom, const void *s, const void *r, double *out4) {
  Ctx &c = ctx();
  if (ensure_stream(c)) return -1;
  size_t n = nsites(c, vol, icom), b = n * 24 * (prec == 64 ? 8 : 4);
  double *scr, *od;
  if (flat_scratch(c, &scr, &od)) return -1;
  View vs(c, s, b, 0, false), vr(c, r, b, 1, false);
  if (!vs.dev || !vr.dev) return -1;
  if (flat_dot(c, prec, vs.dev, vr.dev, n, out4, scr, od)) return -1;
  // icom & 0x1: the sum over the ranks (domain decomposition)
  return ((icom & 1) && dd_on(c)) ? dd_global(c, out4, 2, false) : 0;
}

static int dd_norm(int prec, int vol, int icom, const void *s, double *out2) {
  Ctx &c = ctx();
  if (ensure_stream(c)) return -1;
  size_t n = nsites(c, vol, icom), b = n * 24 * (prec == 64 ? 8 : 4);
  double *scr, *od;
  if (flat_scratch(c, &scr, &od)) return -1;
  View vs(c, s, b, 0, false);
  if (!vs.dev) return -1;
  if (flat_norm2(c, prec, vs.dev, n, out2, scr, od)) return -1;
  return ((icom & 1) && dd_on(c)) ? dd_global(c, out2, 1, false) : 0;
}

static void axpy(int prec, int vol, int icom, void *s, const void *r, double ar, double ai) {
  Ctx &c = ctx();
  if (ensure_stream(c)) return;
  size_t n = nsites(c, vol, icom), b = n * 24 * (prec == 64 ? 8 : 4);
  View vs(c, s, b, 0, true), vr(c, r, b, 1, false);
  if (!vs.dev || !vr.dev) return;
  flat_axpy(c, prec, vs.dev, vr.dev, n, ar, ai);
  if (!vs.staged) cudaStreamSynchronize(c.stream);
}

static void scal(int prec, int vol, int icom, double a, void *s) {
  Ctx &c = ctx();
  if (ensure_stream(c)) return;
  size_t n = nsites(c, vol, icom), b = n * 24 * (prec == 64 ? 8 : 4);
  View vs(c, s, b, 0, true);
  if (!vs.dev) return;
  flat_scale(c, prec, vs.dev, n, a);
  if (!vs.staged) cudaStreamSynchronize(c.stream);
}

}  // namespace qcd

using qcd::ctx;

extern "C" {

int b200_set_nthread(int n) {
  if (n < 1) return qcd::fail("set_nthread: n must be positive");
  ctx().nthread = n;
  return 0;
}

// ------------------------------------------------------ salg_dble.c drop-ins
complex_qflt spinor_prod_dble(int vol, int icom, spinor_dble *s, spinor_dble *r) {
  double o[4] = {0, 0, 0, 0};
  qcd::dd_dot(64, vol, icom, s, r, o);
  complex_qflt z;
  z.re.q[0] = o[0]; z.re.q[1] = o[1];
  z.im.q[0] = o[2]; z.im.q[1] = o[3];
  return z;
}

qflt spinor_prod_re_dble(int vol, int icom, spinor_dble *s, spinor_dble *r) {
  complex_qflt z = spinor_prod_dble(vol, icom, s, r);
  return z.re;
}

qflt norm_square_dble(int vol, int icom, spinor_dble *s) {
  double o[2] = {0, 0};
  qcd::dd_norm(64, vol, icom, s, o);
  qflt q;
  q.q[0] = o[0];
  q.q[1] = o[1];
  return q;
}

void mulc_spinor_add_dble(int vol, int icom, spinor_dble *s, spinor_dble *r, complex_dble z) {
  qcd::axpy(64, vol, icom, s, r, z.re, z.im);
}

void mulr_spinor_add_dble(int vol, int icom, spinor_dble *s, spinor_dble *r, double c) {
  qcd::axpy(64, vol, icom, s, r, c, 0.0);
}

void scale_dble(int vol, int icom, double c, spinor_dble *s) { qcd::scal(64, vol, icom, c, s); }

double normalize_dble(int vol, int icom, spinor_dble *s) {
  qflt q = norm_square_dble(vol, icom, s);
  double r = sqrt(q.q[0]);
  if (r != 0.0) scale_dble(vol, icom, 1.0 / r, s);
  else if (icom != 0) qcd::fail("normalize_dble: vector has vanishing norm");
  return r;
}

// ----------------------------------------------------------- salg.c drop-ins
complex spinor_prod(int vol, int icom, spinor *s, spinor *r) {
  double o[4] = {0, 0, 0, 0};
  qcd::dd_dot(32, vol, icom, s, r, o);
  complex z;
  z.re = (float)(o[0] + o[1]);
  z.im = (float)(o[2] + o[3]);
  return z;
}

float spinor_prod_re(int vol, int icom, spinor *s, spinor *r) { return spinor_prod(vol, icom, s, r).re; }

float norm_square(int vol, int icom, spinor *s) {
  double o[2] = {0, 0};
  qcd::dd_norm(32, vol, icom, s, o);
  return (float)(o[0] + o[1]);
}

void mulc_spinor_add(int vol, int icom, spinor *s, spinor *r, complex z) { qcd::axpy(32, vol, icom, s, r, z.re, z.im); }
void mulr_spinor_add(int vol, int icom, spinor *s, spinor *r, float c) { qcd::axpy(32, vol, icom, s, r, c, 0.0); }
void scale(int vol, int icom, float c, spinor *s) { qcd::scal(32, vol, icom, c, s); }

float normalize(int vol, int icom, spinor *s) {
  float r = norm_square(vol, icom, s);
  r = (float)sqrt((double)r);
  if (r != 0.0f) scale(vol, icom, 1.0f / r, s);
  else if (icom != 0) qcd::fail("normalize: vector has vanishing norm");
  return r;
}

// ----------------------------------------------------------- fgcr drop-in
double fgcr(int vol, void (*Dop)(spinor_dble *s, spinor_dble *r), void (*Mop)(int k, spinor *rho, spinor *phi, spinor *chi),
            spinor **ws, spinor_dble **wsd, int nkv, int nmx, int istop, double res, spinor_dble *eta,
            spinor_dble *psi, int *status) {
  using qcd::Ctx;
  using qcd::View;
  using qcd::KrylovOps;
  using qcd::cplxf;
  using qcd::fail;
  Ctx &c = ctx();
  if (qcd::ensure_stream(c)) return -1.0;
  if (vol <= 0) { fail("fgcr: parameters are out of range"); return -1.0; }
  // the reference calls its BLAS with icom = 3 inside fgcr
  const size_t n = qcd::nsites(c, vol, 3);
  const size_t b32 = n * 96, b64 = n * 192;
  double *scr, *od;
  if (qcd::flat_scratch(c, &scr, &od)) return -1.0;
  KrylovOps o;
  o.res32 = [&](const void *x, int is) {
    if (is) {
      double m;
      View v(c, x, b32, 0, false);
      qcd::flat_umax(c, 32, v.dev, n, &m, scr, od);
      if (qcd::dd_on(c)) {
        double mm[2] = {m, 0.0};
        qcd::dd_global(c, mm, 1, true);
        m = mm[0];
      }
      return (double)(float)sqrt(m);
    }
    double d[2];
    View v(c, x, b32, 0, false);
    qcd::flat_norm2(c, 32, v.dev, n, d, scr, od);
    if (qcd::dd_on(c)) qcd::dd_global(c, d, 1, false);
    return sqrt((double)(float)(d[0] + d[1]));
  };
  o.dot32 = [&](const void *x, const void *y) {
    double d[4];
    View vx(c, x, b32, 0, false), vy(c, y, b32, 1, false);
    qcd::flat_dot(c, 32, vx.dev, vy.dev, n, d, scr, od);
    if (qcd::dd_on(c)) qcd::dd_global(c, d, 2, false);
    return cplxf{(float)(d[0] + d[1]), (float)(d[2] + d[3])};
  };
  o.normalize32 = [&](void *x) { return normalize((int)n, 0, (spinor *)x); };
  o.axpy32 = [&](void *y, float ar, float ai, const void *x) { qcd::axpy(32, (int)n, 0, y, x, ar, ai); };
  o.zero32 = [&](void *x) { View v(c, x, b32, 0, true); qcd::flat_zero(c, 32, v.dev, n); };
  o.zero64 = [&](void *x) { View v(c, x, b64, 0, true); qcd::flat_zero(c, 64, v.dev, n); };
  o.copy64to32 = [&](const void *x, void *y) {
    View vx(c, x, b64, 0, false), vy(c, y, b32, 1, true);
    qcd::flat_copy(c, 64, vx.dev, 32, vy.dev, n);
  };
  o.add32to64 = [&](const void *s, void *d) {
    View vs(c, s, b32, 0, false), vd(c, d, b64, 1, true);
    qcd::flat_add_s2sd(c, vs.dev, vd.dev, n);
  };
  o.diff64to32 = [&](const void *a, const void *bb, void *r) {
    View va(c, a, b64, 0, false), vb(c, bb, b64, 1, false), vr(c, r, b32, 2, true);
    qcd::flat_diff_sd2s(c, va.dev, vb.dev, vr.dev, n);
  };
  auto sync_all = [&]() { cudaStreamSynchronize(c.stream); };
  std::function<void(const void *, void *)> D = [&](const void *s, void *r) {
    sync_all();
    Dop((spinor_dble *)s, (spinor_dble *)r);
  };
  std::function<void(int, const void *, void *, void *)> M = [&](int k, const void *rh, void *ph, void *ch) {
    sync_all();
    Mop(k, (spinor *)rh, (spinor *)ph, (spinor *)ch);
  };
  std::vector<void *> phi(ws, ws + nkv), chi(ws + nkv + 1, ws + 2 * nkv + 1);
  double rn = qcd::fgcr_core(o, nkv, nmx, istop, res, eta, psi, status, D, M, phi, chi, ws[nkv], wsd[0]);
  sync_all();
  return rn;
}

}  // extern "C"
