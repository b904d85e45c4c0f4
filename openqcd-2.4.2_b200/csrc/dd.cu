// Domain decomposition along x0: several ranks (processes, one GPU each)
// hold consecutive x0-slabs of the lattice, as openQCD's process grid with
// NPROC0 > 1 does (include/global.h:18-36, main/README.global:60-127).
//
// What crosses a rank boundary, and how (the reference's counterparts):
//
// - Dirac operator: one half-spinor face per direction and application.
//   Rank r sends to r-1 the projections h = (s1 + s3, s2 + s4) of its first
//   plane (the forward hop of r-1's last plane multiplies them by its own
//   link), and to r+1 the products c = U(x,0)^dag (s1 - s3, s2 - s4) of its
//   last plane (the backward hop of r+1's first plane needs the link r
//   holds).  This is the split of modules/sflds/sdcom.c (cpsd_int_bnd,
//   cpsd_ext_bnd, :414, :509): 96 bytes per face site in FP64, 48 in FP32.
// - SAP: the same face of the block solutions after each colour
//   (modules/sap/sap_com.c:465), so the block-boundary update of the other
//   colour sees the neighbour rank's blocks.
// - Global sums: every reduction's double-double (hi, lo) pair is gathered
//   from all ranks and added in rank order with TwoSum, so every rank gets
//   the same, reproducible sum (modules/utils/qsum.c:389 global_qsum).
// - Gauge field in openQCD's storage order: the forward time links of the
//   last plane's even sites live at the next rank (as backward links of its
//   first plane's odd sites); they cross once per upload or download.
//
// The transport is the caller's: an exchange callback moves the two send
// buffers to the neighbours (NCCL on device buffers, CUDA-aware MPI, or a
// host copy), an all-gather callback moves the reduction partials.  No
// kernel waits on another rank.
#include "lib.h"
#include <algorithm>
#include <string>
#include <vector>

namespace qcd {

// ---------------------------------------------------------------- packing
// thread i < F: face index i of the first plane (to the rank below),
// F <= i < 2F: face index i - F of the last plane (to the rank above)
template <typename R, int L12>
__global__ void k_dd_pack(Geom g, DDGeom dg, const void *__restrict__ t, const void *__restrict__ u, void *dn,
                          void *up) {
  const int F = face_sites(g);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * F) return;
  const int side = i >= F, f = i - side * F;
  int chunk, s, n[4], y[4];
  face_site(g, side, f, chunk, s, n, y);
  const spinor<R> v = Store<R>::load_spinor(t, chunk, s, g.vbh);
  vec3<R> a, b;
  if (side == 0) {
    dd_proj_fwd<R>(v, a, b);
    Half<R>::store(dn, F, f, a, b);
  } else {
    su3<R> uu;
    if constexpr (L12 != 0) uu = load_link12(u, chunk, 0, s, g.vbh, dg.x0off + g.L[0] - 1 == dg.N0 - 1);
    else uu = Store<R>::load_link(u, chunk, 0, s, g.vbh);
    dd_proj_bwd<R>(uu, v, a, b);
    Half<R>::store(up, F, f, a, b);
  }
}

int dd_exchange(Ctx &c, size_t bytes, cudaStream_t st) {
  DDState &d = c.dd;
  if (bytes > d.bytes) return fail("domain decomposition: face larger than the exchange buffers");
  const int rc = d.xchg(d.buf[0], d.buf[1], d.buf[2], d.buf[3], bytes, (void *)st, d.user);
  d.nxchg++;
  return rc == 0 ? 0 : fail("domain decomposition: the exchange callback failed");
}

int dd_faces(Ctx &c, int prec, const void *t, const void *u, int l12, cudaStream_t st, DDGeom &dg) {
  const int F = c.g.L[1] * c.g.L[2] * c.g.L[3];
  const int th = 128;
  const unsigned nb = (unsigned)((2 * F + th - 1) / th);
  DDState &d = c.dd;
  if (prec == 64)
    k_dd_pack<double, 0><<<nb, th, 0, st>>>(c.g, c.ddg, t, u, d.buf[0], d.buf[1]);
  else if (l12)
    k_dd_pack<float, 1><<<nb, th, 0, st>>>(c.g, c.ddg, t, u, d.buf[0], d.buf[1]);
  else
    k_dd_pack<float, 0><<<nb, th, 0, st>>>(c.g, c.ddg, t, u, d.buf[0], d.buf[1]);
  if (cudaGetLastError() != cudaSuccess) return fail("domain decomposition: pack launch failed");
  if (dd_exchange(c, (size_t)F * (prec == 64 ? 96 : 48), st)) return -1;
  dg = c.ddg;
  dg.hup = d.buf[2];
  dg.hdn = d.buf[3];
  return 0;
}

// ------------------------------------------------ gauge field at the faces
// The reference's storage order keeps U(x-0,0) at the odd sites x of the
// first plane (slot 8(ix - V/2) + 1); on the device it is the forward link
// of an even site of the rank below's last plane.
__global__ void k_dd_links_ref_to_face(Geom g, const int *__restrict__ d2q, const double *__restrict__ q,
                                       double *dn) {
  const int F = face_sites(g);
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  int chunk, s, n[4], y[4];
  face_site(g, 0, f, chunk, s, n, y);
  if (chunk < g.nbl) return;                        // even site: no backward links stored there
  const int ix = __ldg(d2q + (size_t)chunk * g.vbh + s);
  const double *src = q + ((size_t)8 * (ix - g.volh) + 1) * 18;
  for (int k = 0; k < 18; k++) dn[(size_t)f * 18 + k] = src[k];
}
__global__ void k_dd_face_to_links_dev(Geom g, const double *__restrict__ up, double2 *ud) {
  const int F = face_sites(g);
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  int chunk, s, n[4], y[4];
  face_site(g, 1, f, chunk, s, n, y);
  if (chunk >= g.nbl) return;                       // odd site: its forward link came with the local array
  double2 *dst = ud + (size_t)chunk * 36 * g.vbh + s;   // mu = 0
  for (int k = 0; k < 9; k++) dst[(size_t)k * g.vbh] = make_double2(up[(size_t)f * 18 + 2 * k], up[(size_t)f * 18 + 2 * k + 1]);
}
__global__ void k_dd_links_dev_to_face(Geom g, const double2 *__restrict__ ud, double *upb) {
  const int F = face_sites(g);
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  int chunk, s, n[4], y[4];
  face_site(g, 1, f, chunk, s, n, y);
  if (chunk >= g.nbl) return;
  const double2 *src = ud + (size_t)chunk * 36 * g.vbh + s;
  for (int k = 0; k < 9; k++) {
    const double2 v = src[(size_t)k * g.vbh];
    upb[(size_t)f * 18 + 2 * k] = v.x;
    upb[(size_t)f * 18 + 2 * k + 1] = v.y;
  }
}
__global__ void k_dd_face_to_links_ref(Geom g, const int *__restrict__ d2q, const double *__restrict__ rdn, double *q) {
  const int F = face_sites(g);
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  int chunk, s, n[4], y[4];
  face_site(g, 0, f, chunk, s, n, y);
  if (chunk < g.nbl) return;
  const int ix = __ldg(d2q + (size_t)chunk * g.vbh + s);
  double *dst = q + ((size_t)8 * (ix - g.volh) + 1) * 18;
  for (int k = 0; k < 18; k++) dst[k] = rdn[(size_t)f * 18 + k];
}

int dd_links_after_upload(Ctx &c, const void *qud, cudaStream_t st) {
  const int F = c.g.L[1] * c.g.L[2] * c.g.L[3], th = 128;
  const unsigned nb = (unsigned)((F + th - 1) / th);
  DDState &d = c.dd;
  k_dd_links_ref_to_face<<<nb, th, 0, st>>>(c.g, c.d_dev2q, (const double *)qud, (double *)d.buf[0]);
  if (dd_exchange(c, (size_t)F * 144, st)) return -1;
  k_dd_face_to_links_dev<<<nb, th, 0, st>>>(c.g, (const double *)d.buf[2], c.ud);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("domain decomposition: link face launch failed");
}

int dd_links_after_download(Ctx &c, void *qud, cudaStream_t st) {
  const int F = c.g.L[1] * c.g.L[2] * c.g.L[3], th = 128;
  const unsigned nb = (unsigned)((F + th - 1) / th);
  DDState &d = c.dd;
  k_dd_links_dev_to_face<<<nb, th, 0, st>>>(c.g, c.ud, (double *)d.buf[1]);
  if (dd_exchange(c, (size_t)F * 144, st)) return -1;
  k_dd_face_to_links_ref<<<nb, th, 0, st>>>(c.g, c.d_dev2q, (const double *)d.buf[3], (double *)qud);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("domain decomposition: link face launch failed");
}

// ------------------------------------------------------------ global sums
static void two_sum(double &h, double &l, double x) {
  const double s = h + x, bb = s - h;
  l += (h - (s - bb)) + (x - bb);
  h = s;
}

int dd_global(Ctx &c, double *res, int n, bool is_max) {
  DDState &d = c.dd;
  if (d.np <= 1) return 0;
  std::vector<double> all((size_t)d.np * 2 * n);
  if (d.gather(res, all.data(), 2 * n, d.user) != 0) return fail("domain decomposition: the all-gather callback failed");
  for (int k = 0; k < n; k++) {
    if (is_max) {
      double m = 0.0;
      for (int r = 0; r < d.np; r++) m = std::max(m, all[(size_t)r * 2 * n + 2 * k]);
      res[2 * k] = m;
      res[2 * k + 1] = 0.0;
    } else {
      double h = 0.0, l = 0.0;
      for (int r = 0; r < d.np; r++) {
        two_sum(h, l, all[(size_t)r * 2 * n + 2 * k]);
        two_sum(h, l, all[(size_t)r * 2 * n + 2 * k + 1]);
      }
      const double s = h + l;
      res[2 * k] = s;
      res[2 * k + 1] = l - (s - h);
    }
  }
  return 0;
}

int dd_all(Ctx &c, int flag) {
  DDState &d = c.dd;
  if (d.np <= 1) return flag;
  double v[2] = {(double)flag, 0.0};
  std::vector<double> all((size_t)d.np * 2);
  if (d.gather(v, all.data(), 2, d.user) != 0) {
    fail("domain decomposition: the all-gather callback failed");
    return 0;
  }
  for (int r = 0; r < d.np; r++)
    if (all[2 * r] == 0.0) return 0;
  return 1;
}

int dd_rank0(Ctx &c, int value) {
  DDState &d = c.dd;
  if (d.np <= 1) return value;
  double v[2] = {(double)value, 0.0};
  std::vector<double> all((size_t)d.np * 2);
  if (d.gather(v, all.data(), 2, d.user) != 0) {
    fail("domain decomposition: the all-gather callback failed");
    return value;
  }
  return (int)all[0];
}

int dd_buffers(Ctx &c) {
  DDState &d = c.dd;
  for (void *&p : d.buf) {
    cudaFree(p);
    p = nullptr;
  }
  d.bytes = 0;
  if (d.np <= 1) return 0;
  const size_t F = (size_t)c.g.L[1] * c.g.L[2] * c.g.L[3];
  const size_t bytes = F * 576;     // the largest face: four FP64 links per site (the SW term's)
  for (void *&p : d.buf)
    if (cudaMalloc(&p, bytes) != cudaSuccess) return fail("domain decomposition: out of device memory (faces)");
  d.bytes = bytes;
  return 0;
}

int dd_unsupported(const Ctx &c, const char *what) {
  if (c.dd.np <= 1) return 0;
  return fail(std::string(what) + ": not available with domain decomposition (ranks along x0)");
}

}  // namespace qcd

extern "C" {

int b200_dd_setup(int nproc0, int cpr0, b200_dd_exchange_fn xchg, b200_dd_allgather_fn gather, void *user) {
  qcd::Ctx &c = qcd::ctx();
  if (nproc0 < 1 || cpr0 < 0 || cpr0 >= nproc0) return qcd::fail("dd_setup: need 0 <= cpr0 < nproc0");
  if (nproc0 > 1 && (!xchg || !gather)) return qcd::fail("dd_setup: exchange and all-gather callbacks are required");
  c.dd.np = nproc0;
  c.dd.rank = cpr0;
  c.dd.xchg = xchg;
  c.dd.gather = gather;
  c.dd.user = user;
  return 0;
}

int b200_dd_global_sum(const double *in, double *out, int n) {
  qcd::Ctx &c = qcd::ctx();
  if (n < 0) return qcd::fail("dd_global_sum: n must be >= 0");
  for (int k = 0; k < 2 * n; k++) out[k] = in[k];
  return qcd::dd_global(c, out, n, false);
}

int b200_dd_info(void **bufs, size_t *bytes, long long *nexchange) {
  qcd::Ctx &c = qcd::ctx();
  if (bufs)
    for (int k = 0; k < 4; k++) bufs[k] = c.dd.buf[k];
  if (bytes) *bytes = c.dd.bytes;
  if (nexchange) *nexchange = c.dd.nxchg;
  return c.dd.np;
}

}  // extern "C"
