// The C ABI: library context, error handling, and every extern "C" entry
// point declared in include/openqcd_b200.h.
#include "lib.h"
#include <cuda_profiler_api.h>
#include "../../include/openqcd_b200.h"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>

namespace qcd {

double sap_gcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                   int *ifail, int *status);

static Ctx g_ctx;
static thread_local std::string g_err;
static bool g_fatal = true;

Ctx &ctx() { return g_ctx; }
void set_error(const std::string &m) { g_err = m; }

int fail(const std::string &msg) {
  g_err = msg;
  if (g_fatal) {
    fprintf(stderr, "\nError in openqcd_b200: %s\nProgram aborted\n", msg.c_str());
    fflush(stderr);
    exit(1);
  }
  return -1;
}

static int need(bool ok, const char *what) { return ok ? 0 : fail(what); }

static int ensure_stage(Ctx &c, size_t bytes) {
  if (c.stage_bytes >= bytes) return 0;
  cudaFree(c.stage);
  c.stage = nullptr;
  c.stage_bytes = 0;
  if (cudaMalloc(&c.stage, bytes) != cudaSuccess) return fail("out of device memory (staging buffer)");
  c.stage_bytes = bytes;
  return 0;
}

static int ensure_tmp(Ctx &c) {
  if (!c.tmp64 && cudaMalloc(&c.tmp64, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory");
  if (!c.tmp32 && cudaMalloc(&c.tmp32, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory");
  return 0;
}

static int check_ready(const Ctx &c) { return need(c.ready, "geometry not set (call b200_geometry first)"); }
static int check_fields(const Ctx &c) {
  if (check_ready(c)) return -1;
  if (!c.have_ud) return fail("no gauge field on the device (b200_upload_ud or b200_random_ud)");
  if (!c.have_sw) return fail("no SW field on the device (b200_upload_swd or b200_sw_term)");
  return 0;
}

// Run a device-layout operator on reference-layout arrays (host or device):
// copy in, convert, apply, convert back, copy out.  The output array is read
// first because the even/odd pieces leave one parity of r unchanged.
static bool pinned_host(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Dw on page-locked host arrays, pipelined: the input pieces are copied
// back to back on one stream in the order np-1, 0, 1, ..., np-2 and each is
// converted to the device layout on a second; the operator runs on a block
// row (a slab) on the library stream as soon as the pieces holding its
// planes and the two neighbouring planes are in; its result is converted
// back there, and every piece whose rows are all done is copied out on a
// third stream (adjacent ranges in one copy), so that the two transfer
// directions overlap.  The output
// of a piece is written only after its own input was copied, so s and r may
// be the same array.
// The two parity ranges of a piece (or of the pieces a row completes), at
// offsets o[0] < o[1] of both arrays, as one copy of two rows (pitch o[1] -
// o[0]) when they are equally long; otherwise, or if the pitch is refused,
// as two copies.
static void copy_pair(char *dst, const char *src, const size_t o[2], const size_t n[2], cudaMemcpyKind kind,
                      cudaStream_t st) {
  if (n[0] == n[1] && n[0] > 0 && o[1] >= o[0] + n[0] &&
      cudaMemcpy2DAsync(dst + o[0], o[1] - o[0], src + o[0], o[1] - o[0], n[0], 2, kind, st) == cudaSuccess)
    return;
  cudaGetLastError();
  for (int p = 0; p < 2; p++)
    if (n[p]) cudaMemcpyAsync(dst + o[p], src + o[p], n[p], kind, st);
}

template <typename R>
static int dw_pipelined(Ctx &c, R mu, const void *s, void *r, void *fs, void *fr, char *st_in, char *st_out) {
  const int prec = sizeof(R) == 8 ? 64 : 32;
  const size_t site = 24 * sizeof(R);
  const int np = (int)c.piece.size(), nr = (int)c.slab.size(), L0 = c.g.L[0];
  if ((!c.st_in && cudaStreamCreateWithFlags(&c.st_in, cudaStreamNonBlocking) != cudaSuccess) ||
      (!c.st_out && cudaStreamCreateWithFlags(&c.st_out, cudaStreamNonBlocking) != cudaSuccess) ||
      (!c.st_cv && cudaStreamCreateWithFlags(&c.st_cv, cudaStreamNonBlocking) != cudaSuccess))
    return fail("no CUDA stream for the pipelined transfers");
  while ((int)c.slab_ev.size() < 2 * np + nr + 1) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail("no CUDA event");
    c.slab_ev.push_back(e);
  }
  cudaEvent_t *ev_cp = c.slab_ev.data(), *ev_in = ev_cp + np, *ev_out = ev_in + np, ev0 = ev_out[nr];
  // the transfer position of each piece; a row can run once the last of
  // the pieces holding its planes and its two neighbouring planes is in
  const int P = c.piece[0].t1 - c.piece[0].t0;
  auto pos = [&](int i) { return i == np - 1 ? 0 : i + 1; };
  std::vector<int> need(nr, 0), rows_left(np, 0);
  for (int k = 0; k < nr; k++) {
    const Slab &sb = c.slab[k];
    for (int t = sb.t0 - 1; t <= sb.t1; t++) need[k] = std::max(need[k], pos(((t + L0) % L0) / P));
    for (int i = sb.t0 / P; i <= (sb.t1 - 1) / P; i++) rows_left[i]++;
  }
  cudaEventRecord(ev0, c.stream);
  cudaStreamWaitEvent(c.st_in, ev0, 0);
  cudaStreamWaitEvent(c.st_cv, ev0, 0);
  cudaStreamWaitEvent(c.st_out, ev0, 0);
  auto h2d = [&](int i) {
    const Piece &pc = c.piece[i];
    const size_t o[2] = {(size_t)pc.q0[0] * site, (size_t)pc.q0[1] * site};
    const size_t n[2] = {(size_t)(pc.q1[0] - pc.q0[0]) * site, (size_t)(pc.q1[1] - pc.q0[1]) * site};
    copy_pair(st_in, (const char *)s, o, n, cudaMemcpyHostToDevice, c.st_in);
    cudaEventRecord(ev_cp[i], c.st_in);
    cudaStreamWaitEvent(c.st_cv, ev_cp[i], 0);
    spinor_from_ref_piece(c, prec, st_in, fs, pc, c.st_cv);
    cudaEventRecord(ev_in[i], c.st_cv);
  };
  // the pieces a row completes go out together: per parity half, their
  // storage ranges sorted and the adjacent ones joined into one copy
  auto d2h = [&](const std::vector<int> &done) {
    std::vector<std::pair<int, int>> rg[2];
    for (int p = 0; p < 2; p++) {
      std::vector<std::pair<int, int>> in;
      for (int i : done) in.push_back({c.piece[i].q0[p], c.piece[i].q1[p]});
      std::sort(in.begin(), in.end());
      for (size_t a = 0; a < in.size();) {
        size_t b = a + 1;
        int q1 = in[a].second;
        while (b < in.size() && in[b].first == q1) q1 = in[b++].second;
        rg[p].push_back({in[a].first, q1});
        a = b;
      }
    }
    if (rg[0].size() == 1 && rg[1].size() == 1) {
      const size_t o[2] = {(size_t)rg[0][0].first * site, (size_t)rg[1][0].first * site};
      const size_t n[2] = {(size_t)(rg[0][0].second - rg[0][0].first) * site,
                           (size_t)(rg[1][0].second - rg[1][0].first) * site};
      copy_pair((char *)r, st_out, o, n, cudaMemcpyDeviceToHost, c.st_out);
      return;
    }
    for (int p = 0; p < 2; p++)
      for (const auto &q : rg[p]) {
        const size_t o = (size_t)q.first * site, n = (size_t)(q.second - q.first) * site;
        cudaMemcpyAsync((char *)r + o, st_out + o, n, cudaMemcpyDeviceToHost, c.st_out);
      }
  };
  // row k after the conversion of piece `after` (the conversions run in
  // order on one stream, so the earlier ones are done too)
  auto comp = [&](int k, int after) {
    const Slab &sb = c.slab[k];
    cudaStreamWaitEvent(c.stream, ev_in[after], 0);
    qcd::dirac_dw_blocks<R>(c, mu, fs, fr, c.d_ident + sb.b0, sb.b1 - sb.b0, c.stream);
    for (int p = 0; p < 2; p++) {
      const int d0 = (p * c.g.nbl + sb.b0) * c.g.vbh, nd = (sb.b1 - sb.b0) * c.g.vbh;
      spinor_to_ref_range(c, prec, fr, st_out, d0, nd, c.stream);
    }
    cudaEventRecord(ev_out[k], c.stream);
    std::vector<int> done;
    for (int i = sb.t0 / P; i <= (sb.t1 - 1) / P; i++)
      if (--rows_left[i] == 0) done.push_back(i);
    if (!done.empty()) {
      cudaStreamWaitEvent(c.st_out, ev_out[k], 0);
      d2h(done);
    }
  };
  for (int j = 0; j < np; j++) {
    const int i = j == 0 ? np - 1 : j - 1;
    h2d(i);
    for (int k = 0; k < nr; k++)
      if (need[k] == j) comp(k, i);
  }
  const cudaError_t e1 = cudaStreamSynchronize(c.st_out), e2 = cudaStreamSynchronize(c.stream),
                    e3 = cudaStreamSynchronize(c.st_in), e4 = cudaStreamSynchronize(c.st_cv);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess)
    return fail(std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
  return 0;
}

template <typename R>
static void ref_layout_op(int op, R mu, const void *s, void *r) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return;
  const int prec = sizeof(R) == 8 ? 64 : 32;
  const size_t nb = spinor_bytes(c, prec);
  if (ensure_stage(c, 2 * nb)) return;
  while (c.ws64.size() < 2 || c.ws32.size() < 2) {
    void *p;
    bool d = c.ws64.size() < 2;
    if (cudaMalloc(&p, spinor_bytes(c, d ? 64 : 32)) != cudaSuccess) { fail("out of device memory"); return; }
    (d ? c.ws64 : c.ws32).push_back(p);
  }
  void *fs = prec == 64 ? c.ws64[0] : c.ws32[0];
  void *fr = prec == 64 ? c.ws64[1] : c.ws32[1];
  char *st_in = (char *)c.stage, *st_out = (char *)c.stage + nb;
  cudaStream_t st = c.stream;
  if (op == 0 && c.pipeline && !qcd::dd_on(c) && c.slab.size() >= 3 && c.piece.size() >= 3 && pinned_host(s) &&
      pinned_host(r)) {
    c.pipeline_used = 1;
    dw_pipelined<R>(c, mu, s, r, fs, fr, st_in, st_out);
    return;
  }
  if (op == 0) c.pipeline_used = 0;
  cudaMemcpyAsync(st_in, s, nb, cudaMemcpyDefault, st);
  spinor_from_ref(c, prec, st_in, fs, st);
  if (op != 0) {
    cudaMemcpyAsync(st_out, r, nb, cudaMemcpyDefault, st);
    spinor_from_ref(c, prec, st_out, fr, st);
  }
  dirac_op<R>(c, op, mu, fs, fr, prec == 64 ? c.tmp64 : c.tmp32, st);
  spinor_to_ref(c, prec, fr, st_out, st);
  cudaMemcpyAsync(r, st_out, nb, cudaMemcpyDefault, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) fail(std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
}

}  // namespace qcd

using qcd::Ctx;
using qcd::ctx;
using qcd::fail;
using qcd::g_err;
using qcd::g_fatal;
using qcd::check_ready;
using qcd::check_fields;
using qcd::ensure_stage;
using qcd::ensure_tmp;
using qcd::need;
using qcd::ref_layout_op;
using qcd::spinor_bytes;
using qcd::spinor_from_ref;
using qcd::spinor_to_ref;
using qcd::dirac_op;
using qcd::sap_prepare;
using qcd::sap_cycle;
using qcd::sap_gcr_dev;
using qcd::la_norm2;
using qcd::PAR_ALL;
using qcd::apply_sw_ref_layout;
using qcd::apply_swinv_ref_layout;

extern "C" {

const char *b200_last_error(void) { return g_err.c_str(); }
void b200_clear_error(void) { g_err.clear(); }

void *b200_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) { fail("page-locked host allocation failed"); return nullptr; }
  return p;
}
void b200_host_free(void *p) { cudaFreeHost(p); }

void *b200_dev_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) { fail("device allocation failed"); return nullptr; }
  return p;
}

// Ordered on the library's stream and complete on return (a plain
// cudaMemcpy from pageable host memory may return before its DMA reaches
// device memory, and the library's stream does not wait for the legacy
// default stream).
int b200_memcpy(void *dst, const void *src, size_t bytes) {
  cudaStream_t st = ctx().stream;
  if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st) != cudaSuccess) return fail("memcpy failed");
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : fail("memcpy failed");
}
void b200_set_fatal(int on) { g_fatal = on != 0; }
int b200_sync(void) {
  Ctx &c = ctx();
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("CUDA error");
  if (c.h_kerr && *(volatile int *)c.h_kerr) {
    *(volatile int *)c.h_kerr = 0;
    return fail("a kernel gave up waiting for its bulk copies (results invalid)");
  }
  return 0;
}
int b200_volume(void) { return ctx().ready ? ctx().g.vol : 0; }

int b200_set_device(int dev) {
  Ctx &c = ctx();
  if (c.stream) return fail("set_device: must be called before the first geometry call");
  if (cudaSetDevice(dev) != cudaSuccess) return fail("set_device: no such CUDA device");
  c.dev = dev;
  return 0;
}

int b200_geometry(const int L[4], const int bs[4], const int *ipt) {
  Ctx &c = ctx();
  if (!c.stream && cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail("no CUDA device available");
  if (!c.h_kerr) {
    if (cudaHostAlloc((void **)&c.h_kerr, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&c.d_kerr, c.h_kerr, 0) != cudaSuccess)
      return fail("no page-locked memory for the kernel error flag");
    *(volatile int *)c.h_kerr = 0;
  }
  // a new geometry invalidates every resident field
  void *bufs[] = {c.ud, c.u32, c.swd, c.swd_inv, c.sw32, c.sw32_inv, c.tmp64, c.tmp32, c.stage,
                  c.u16, c.sw16, c.sw16_inv, c.u12, c.sap_fld[0], c.sap_fld[1], c.sap_fld[2],
                  c.sap_mfld[0], c.sap_mfld[1], c.sap_mfld[2]};
  for (void *p : bufs) cudaFree(p);
  for (void *p : c.ws32) cudaFree(p);
  for (void *p : c.ws64) cudaFree(p);
  c.ws32.clear(); c.ws64.clear();
  c.ud = nullptr; c.u32 = nullptr; c.swd = c.swd_inv = nullptr; c.sw32 = c.sw32_inv = nullptr;
  c.tmp64 = c.tmp32 = c.stage = nullptr; c.stage_bytes = 0;
  c.u16 = c.sw16 = c.sw16_inv = nullptr; c.h16_valid = false;
  c.sap_tuned_vbh[0] = c.sap_tuned_vbh[1] = c.sap_tuned_vbh[2] = 0;
  c.u12 = nullptr; c.u12_valid = c.u12_ok = false;
  c.sap_fld[0] = c.sap_fld[1] = c.sap_fld[2] = nullptr;
  c.sap_mfld[0] = c.sap_mfld[1] = c.sap_mfld[2] = nullptr;
  c.sap_mfld_n = 0;
  c.have_ud = c.have_sw = false;
  qcd::dfl_release(c);
  qcd::net_fields_release(c);
  qcd::graphs_release();
  c.ready = false;
  if (geometry_init(c, L, bs, ipt) || qcd::dd_buffers(c)) return -1;
  c.ready = true;
  return 0;
}

int b200_set_lat_parms(double csw) { ctx().csw = csw; ctx().have_sw = false; return 0; }
int b200_set_sw_type(int isw) {
  if (isw < 0 || isw > 1) return fail("set_lat_parms: the SW type isw must be either 0 or 1");
  ctx().isw = isw;
  ctx().have_sw = false;
  return 0;
}
int b200_set_bc_parms(int type) {
  if (type != 3) return fail("set_bc_parms: only boundary condition type 3 is supported");
  ctx().bc = type;
  return 0;
}
int b200_set_bc_theta(const double theta[3]) {
  Ctx &c = ctx();
  for (int k = 0; k < 3; k++) c.theta[k] = theta ? theta[k] : 0.0;
  return 0;
}
int b200_set_sw_parms(double m0) { ctx().m0 = m0; ctx().have_sw = false; return 0; }
int b200_set_tm_parms(int eoflg) { ctx().eoflg = eoflg != 0; return 0; }

int b200_set_sap_parms(const int bs[4], int isolv, int nmr, int ncy) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  for (int mu = 0; mu < 4; mu++)
    if (bs[mu] != c.g.bs[mu]) return fail("set_sap_parms: the SAP block size must equal the geometry block size");
  if (isolv < 0 || isolv > 1 || nmr < 1 || ncy < 1) return fail("set_sap_parms: parameters are out of range");
  c.isolv = isolv; c.nmr = nmr; c.ncy = ncy;
  c.sap_set = true;
  return 0;
}

// Start (on != 0) or stop the CUDA profiler's collection, for profiles of a
// chosen region (ncu --profile-from-start off).
int b200_profiler(int on) {
  cudaDeviceSynchronize();
  return (on ? cudaProfilerStart() : cudaProfilerStop()) == cudaSuccess ? 0 : fail("profiler start/stop failed");
}

int b200_dev_dirac_multi(int n, float mu, void *const *s, void *const *r, void *const *sub) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1;
  if (n < 1) return fail("dirac_multi: no fields");
  if (qcd::dirac_multi32(c, n, mu, s, r, sub, c.stream)) return fail("dirac_multi: launch failed");
  return b200_sync();
}

// ------------------------------------------------------- CG normal equations
// tmcg.c:118 / :206 on reference-layout FP64 fields (host or device)
static double tmcg_ref_layout(int eo, int nmx, int istop, double res, double mu, spinor_dble *eta,
                              spinor_dble *psi, int *ifail, int *status) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1.0;
  const size_t nb = spinor_bytes(c, 64);
  if (ensure_stage(c, nb)) return -1.0;
  void *fe = nullptr, *fp = nullptr;
  if (cudaMalloc(&fe, nb) != cudaSuccess || cudaMalloc(&fp, nb) != cudaSuccess) {
    fail("out of device memory");
    return -1.0;
  }
  cudaMemcpyAsync(c.stage, eta, nb, cudaMemcpyDefault, c.stream);
  spinor_from_ref(c, 64, c.stage, fe, c.stream);
  cudaMemcpyAsync(c.stage, psi, nb, cudaMemcpyDefault, c.stream);   // odd sites of psi kept with eo = 1
  spinor_from_ref(c, 64, c.stage, fp, c.stream);
  const double rho = qcd::tmcg_dev(c, eo, nmx, istop, res, mu, fe, fp, ifail, status);
  spinor_to_ref(c, 64, fp, c.stage, c.stream);
  cudaMemcpyAsync(psi, c.stage, nb, cudaMemcpyDefault, c.stream);
  cudaStreamSynchronize(c.stream);
  cudaFree(fe);
  cudaFree(fp);
  return rho;
}

double tmcg(int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi, int *ifail,
            int *status) {
  return tmcg_ref_layout(0, nmx, istop, res, mu, eta, psi, ifail, status);
}

double tmcgeo(int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi, int *ifail,
              int *status) {
  return tmcg_ref_layout(1, nmx, istop, res, mu, eta, psi, ifail, status);
}

double b200_dev_tmcg(int eo, int nmx, int istop, double res, double mu, const void *eta, void *psi, int *ifail,
                     int *status) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1.0;
  return qcd::tmcg_dev(c, eo, nmx, istop, res, mu, eta, psi, ifail, status);
}

// tmcgm.c:100 on reference-layout FP64 fields (host or device): the even
// sites of eta and of the nmu solutions psi[k]
void tmcgm(int nmx, int istop, double *res, int nmu, double *mu, spinor_dble *eta, spinor_dble **psi, int *ifail,
           int *status) {
  Ctx &c = ctx();
  ifail[0] = 0;
  status[0] = 0;
  if (check_fields(c)) return;
  if (nmu < 0) {
    fail("mscg: parameters are out of range");
    return;
  }
  const size_t nb = spinor_bytes(c, 64);
  if (ensure_stage(c, nb)) return;
  std::vector<void *> f(nmu + 1, nullptr);
  for (auto &q : f)
    if (cudaMalloc(&q, nb) != cudaSuccess) {
      for (void *p : f) cudaFree(p);
      fail("out of device memory");
      return;
    }
  cudaMemcpyAsync(c.stage, eta, nb, cudaMemcpyDefault, c.stream);
  spinor_from_ref(c, 64, c.stage, f[0], c.stream);
  for (int k = 0; k < nmu; k++) {   // odd sites of psi[k] are kept
    cudaMemcpyAsync(c.stage, psi[k], nb, cudaMemcpyDefault, c.stream);
    spinor_from_ref(c, 64, c.stage, f[k + 1], c.stream);
  }
  const int rc = qcd::tmcgm_dev(c, nmx, istop, res, nmu, mu, f[0], f.data() + 1, ifail, status);
  if (rc == 0)
    for (int k = 0; k < nmu; k++) {
      spinor_to_ref(c, 64, f[k + 1], c.stage, c.stream);
      cudaMemcpyAsync(psi[k], c.stage, nb, cudaMemcpyDefault, c.stream);
    }
  cudaStreamSynchronize(c.stream);
  for (void *p : f) cudaFree(p);
}

int b200_dev_tmcgm(int nmx, int istop, const double *res, int nmu, const double *mu, const void *eta,
                   void *const *psi, int *ifail, int *status) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1;
  return qcd::tmcgm_dev(c, nmx, istop, res, nmu, mu, eta, psi, ifail, status);
}

// ------------------------------------------------------------ archives
// archive.c:804, :878 and sarchive.c:424, :522; files in the universal format
void export_cnfg(char *out) { qcd::export_cnfg(ctx(), out); }
void import_cnfg(char *in, int mask) { qcd::import_cnfg(ctx(), in, mask); }
void export_sfld(char *out, int eo, spinor_dble *sd) { qcd::export_sfld(ctx(), out, eo, sd); }
void import_sfld(char *in, int eo, spinor_dble *sd) { qcd::import_sfld(ctx(), in, eo, sd); }

// plaq_sum_dble(1) (modules/uflds/plaq_sum.c:161) of the device gauge field
double b200_plaq_sum(void) {
  double s = 0.0;
  if (qcd::plaq_sum(ctx(), &s)) return -1.0e300;
  return s;
}

int b200_set_sap_prec(int bits) {
  if (bits != 16 && bits != 32) return fail("set_sap_prec: the storage precision must be 16 or 32");
  ctx().sap_prec = bits;
  return 0;
}

int b200_set_sap_link12(int on) {
  ctx().sap_link12 = on != 0;
  return 0;
}

int b200_set_cuda_graphs(int on) {
  Ctx &c = ctx();
  const int prev = c.use_graphs;
  c.use_graphs = on != 0;
  if (!c.use_graphs) qcd::graphs_release();
  return prev;
}

int b200_graphs_cached(void) { return (int)qcd::graphs_cached(); }

// 1 (default): Dw_dble / Dw on page-locked host arrays overlap their
// transfers over x0-slabs when the storage order allows; 0: whole-field copies
int b200_set_pipeline(int on) {
  Ctx &c = ctx();
  const int prev = c.pipeline;
  c.pipeline = on != 0;
  return prev;
}

int b200_pipeline_slabs(void) { return (int)ctx().slab.size(); }
int b200_pipeline_pieces(void) { return (int)ctx().piece.size(); }
int b200_pipeline_used(void) { return ctx().pipeline_used; }

int b200_pipeline_plan(const int L[4], const int bs[4], const int *ipt, int *npieces, int *nslabs) {
  if (!L || !bs || !ipt || !npieces || !nslabs) return fail("pipeline_plan: null argument");
  for (int mu = 0; mu < 4; mu++)
    if (L[mu] < 2 || bs[mu] < 2 || L[mu] % bs[mu] || L[mu] > 4096)
      return fail("pipeline_plan: block sizes must divide the lattice sizes");
  std::vector<qcd::Piece> pc;
  std::vector<qcd::Slab> sl;
  qcd::pipeline_plan(L, bs, ipt, pc, sl);
  *npieces = (int)pc.size();
  *nslabs = (int)sl.size();
  return 0;
}

int b200_set_dw_staged(int mode) {
  Ctx &c = ctx();
  const int prev = c.dw_staged;
  c.dw_staged = mode != 0;
  return prev;
}

int b200_set_sap_variant(int variant) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1;
  return qcd::sap_set_variant(c, variant);
}

int b200_set_block_order(int kind) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  const int prev = c.block_order;
  if (qcd::set_block_order(c, kind)) return -1;
  return prev;
}

int b200_tune_block_order(float *ms) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return -1;
  const size_t nb = qcd::spinor_bytes(c, 64);
  void *s = nullptr, *r = nullptr;
  if (cudaMalloc(&s, nb) != cudaSuccess || cudaMalloc(&r, nb) != cudaSuccess) {
    cudaFree(s);
    return fail("tune_block_order: out of device memory");
  }
  qcd::gen_spinor(c, 64, s, 1.0, 4711, c.stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = -1;
  float tbest = 0.0f;
  for (int kind = 0; kind < qcd::kBlockOrders; kind++) {
    if (qcd::set_block_order(c, kind)) { best = -2; break; }
    for (int i = 0; i < 2; i++) dirac_op<double>(c, 0, 0.0, s, r, c.tmp64, c.stream);
    cudaEventRecord(e0, c.stream);
    for (int i = 0; i < 10; i++) dirac_op<double>(c, 0, 0.0, s, r, c.tmp64, c.stream);
    cudaEventRecord(e1, c.stream);
    cudaEventSynchronize(e1);
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) ms[kind] = t / 10.0f;
    if (best < 0 || t < tbest) { best = kind; tbest = t; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(s);
  cudaFree(r);
  if (best < 0) return -1;
  if (qcd::set_block_order(c, best)) return -1;
  return b200_sync() ? -1 : best;
}

int b200_links12_active(void) {
  Ctx &c = ctx();
  if (check_ready(c) || need(c.have_ud, "no gauge field on the device")) return -1;
  return qcd::links12(c, c.stream) != nullptr;
}

int b200_sap_tuning(int prec, int *variant, int *threads, float *ms) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  const int slot = prec == 16 ? 1 : (prec == 12 ? 2 : 0);
  if (c.sap_tuned_vbh[slot] != c.g.vbh) return fail("sap_tuning: the SAP kernel is not tuned for this geometry yet");
  *variant = c.sap_variant[slot];
  *threads = qcd::sap_variant_threads(c, slot);
  *ms = c.sap_tuned_ms[slot];
  return 0;
}

int b200_upload_ud(const su3_dble *ud) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  size_t n = (size_t)c.g.vol * 36 * sizeof(double2);
  if (!c.ud && cudaMalloc(&c.ud, n) != cudaSuccess) return fail("out of device memory (gauge field)");
  if (ensure_stage(c, n)) return -1;
  cudaMemcpyAsync(c.stage, ud, 4 * (size_t)c.g.vol * sizeof(su3_dble), cudaMemcpyDefault, c.stream);
  if (links_from_ref(c, c.stage, c.stream)) return -1;
  // the forward time links of the last plane's even sites are at the rank above
  if (qcd::dd_on(c) && qcd::dd_links_after_upload(c, c.stage, c.stream)) return -1;
  c.have_ud = true;
  if (links_refresh_f32(c, c.stream)) return -1;
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("upload_ud: CUDA error");
}

int b200_download_ud(su3_dble *ud) {
  Ctx &c = ctx();
  if (check_ready(c) || need(c.have_ud, "no gauge field on the device")) return -1;
  size_t n = 4 * (size_t)c.g.vol * sizeof(su3_dble);
  if (ensure_stage(c, n)) return -1;
  if (links_to_ref(c, c.stage, c.stream)) return -1;
  if (qcd::dd_on(c) && qcd::dd_links_after_download(c, c.stage, c.stream)) return -1;
  cudaMemcpyAsync(ud, c.stage, n, cudaMemcpyDefault, c.stream);
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("download_ud: CUDA error");
}

int b200_upload_swd(const pauli_dble *swd) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  size_t n = 2 * (size_t)c.g.vol * sizeof(pauli_dble);
  if (!c.swd && cudaMalloc(&c.swd, n) != cudaSuccess) return fail("out of device memory (SW field)");
  if (ensure_stage(c, n)) return -1;
  cudaMemcpyAsync(c.stage, swd, n, cudaMemcpyDefault, c.stream);
  if (pauli_from_ref(c, c.stage, c.stream)) return -1;
  if (sw_refresh_derived(c, c.stream)) return -1;
  return c.sw_inv_fail;
}

int b200_download_swd(pauli_dble *swd, int which) {
  Ctx &c = ctx();
  if (check_ready(c) || need(c.have_sw, "no SW field on the device")) return -1;
  size_t n = 2 * (size_t)c.g.vol * sizeof(pauli_dble);
  if (ensure_stage(c, n)) return -1;
  if (pauli_to_ref(c, which, c.stage, c.stream)) return -1;
  cudaMemcpyAsync(swd, c.stage, n, cudaMemcpyDefault, c.stream);
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("download_swd: CUDA error");
}

int b200_sw_term(void) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  if (sw_compute(c, c.stream)) return -1;
  return c.sw_inv_fail;
}

int b200_random_ud(double eps, unsigned long long seed) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  if (gen_links(c, eps, seed, c.stream)) return -1;
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : fail("random_ud: CUDA error");
}

// ------------------------------------------------------- drop-in operators
void Dw_dble(double mu, spinor_dble *s, spinor_dble *r) { ref_layout_op<double>(0, mu, s, r); }
void Dwee_dble(double mu, spinor_dble *s, spinor_dble *r) { ref_layout_op<double>(1, mu, s, r); }
void Dwoo_dble(double mu, spinor_dble *s, spinor_dble *r) { ref_layout_op<double>(2, mu, s, r); }
void Dwoe_dble(spinor_dble *s, spinor_dble *r) { ref_layout_op<double>(3, 0.0, s, r); }
void Dweo_dble(spinor_dble *s, spinor_dble *r) { ref_layout_op<double>(4, 0.0, s, r); }
void Dwhat_dble(double mu, spinor_dble *s, spinor_dble *r) { ref_layout_op<double>(5, mu, s, r); }
void Dw(float mu, spinor *s, spinor *r) { ref_layout_op<float>(0, mu, s, r); }
void Dwee(float mu, spinor *s, spinor *r) { ref_layout_op<float>(1, mu, s, r); }
void Dwoo(float mu, spinor *s, spinor *r) { ref_layout_op<float>(2, mu, s, r); }
void Dwoe(spinor *s, spinor *r) { ref_layout_op<float>(3, 0.0f, s, r); }
void Dweo(spinor *s, spinor *r) { ref_layout_op<float>(4, 0.0f, s, r); }
void Dwhat(float mu, spinor *s, spinor *r) { ref_layout_op<float>(5, mu, s, r); }

// Site-local SW term on arbitrary arrays of vol sites.
static void sw_local(int prec, int vol, double mu, const void *m, const void *s, void *r, bool inverse, int *ifail) {
  Ctx &c = ctx();
  if (!c.stream && cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
    fail("no CUDA device available");
    return;
  }
  if (vol <= 0) return;
  size_t es = prec == 64 ? 8 : 4;
  size_t nm = (size_t)vol * 72 * es, ns = (size_t)vol * 24 * es;
  if (ensure_stage(c, nm + 2 * ns + 64)) return;
  char *dm = (char *)c.stage, *ds = dm + nm, *dr = ds + ns;
  int *df = (int *)(dr + ns);
  cudaStream_t st = c.stream;
  cudaMemcpyAsync(dm, m, nm, cudaMemcpyDefault, st);
  cudaMemcpyAsync(ds, s, ns, cudaMemcpyDefault, st);
  if (inverse) {
    cudaMemsetAsync(df, 0, sizeof(int), st);
    apply_swinv_ref_layout(vol, mu, dm, ds, dr, df, st);
  } else {
    apply_sw_ref_layout(prec, vol, mu, dm, ds, dr, st);
  }
  cudaMemcpyAsync(r, dr, ns, cudaMemcpyDefault, st);
  int hf = 0;
  if (inverse) cudaMemcpyAsync(&hf, df, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) fail("apply_sw: CUDA error");
  if (ifail) *ifail = hf;
}

void apply_sw_dble(int vol, double mu, pauli_dble *m, spinor_dble *s, spinor_dble *r) {
  sw_local(64, vol, mu, m, s, r, false, nullptr);
}
void apply_sw(int vol, float mu, pauli *m, spinor *s, spinor *r) { sw_local(32, vol, mu, m, s, r, false, nullptr); }
int apply_swinv_dble(int vol, double mu, pauli_dble *m, spinor_dble *s, pauli_wsp_t *pwsp, spinor_dble *r) {
  (void)pwsp;
  int f = 0;
  sw_local(64, vol, mu, m, s, r, true, &f);
  return f;
}

// ---------------------------------------------------------- drop-in solvers
void sap(float mu, int isolv, int nmr, spinor *psi, spinor *rho) {
  Ctx &c = ctx();
  if (check_fields(c)) return;
  if (isolv == 1 && (c.sw_inv_fail & 2)) { fail("sap: the SW term on the odd sites is not safely invertible"); return; }
  if (sap_prepare(c, c.stream)) return;
  size_t nb = spinor_bytes(c, 32);
  if (ensure_stage(c, 2 * nb)) return;
  void *fp = b200_dev_alloc_spinor(32), *fr = b200_dev_alloc_spinor(32), *fb = b200_dev_alloc_spinor(32);
  if (!fp || !fr || !fb) return;
  char *s0 = (char *)c.stage, *s1 = s0 + nb;
  cudaStream_t st = c.stream;
  cudaMemcpyAsync(s0, psi, nb, cudaMemcpyDefault, st);
  cudaMemcpyAsync(s1, rho, nb, cudaMemcpyDefault, st);
  spinor_from_ref(c, 32, s0, fp, st);
  spinor_from_ref(c, 32, s1, fr, st);
  sap_cycle(c, mu, isolv, nmr, fp, fr, fb, st);
  spinor_to_ref(c, 32, fp, s0, st);
  spinor_to_ref(c, 32, fr, s1, st);
  cudaMemcpyAsync(psi, s0, nb, cudaMemcpyDefault, st);
  cudaMemcpyAsync(rho, s1, nb, cudaMemcpyDefault, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) fail("sap: CUDA error");
  cudaFree(fp); cudaFree(fr); cudaFree(fb);
}

double sap_gcr(int nkv, int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi, int *ifail,
               int *status) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1.0;
  size_t nb = spinor_bytes(c, 64);
  if (ensure_stage(c, nb)) return -1.0;
  void *fe = b200_dev_alloc_spinor(64), *fp = b200_dev_alloc_spinor(64);
  if (!fe || !fp) return -1.0;
  cudaStream_t st = c.stream;
  cudaMemcpyAsync(c.stage, eta, nb, cudaMemcpyDefault, st);
  spinor_from_ref(c, 64, c.stage, fe, st);
  double rho = sap_gcr_dev(c, nkv, nmx, istop, res, mu, fe, fp, ifail, status);
  spinor_to_ref(c, 64, fp, c.stage, st);
  cudaMemcpyAsync(psi, c.stage, nb, cudaMemcpyDefault, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) fail("sap_gcr: CUDA error");
  cudaFree(fe); cudaFree(fp);
  return rho;
}

// ------------------------------------------------------- device-resident API
void *b200_dev_alloc_spinor(int prec) {
  Ctx &c = ctx();
  if (check_ready(c)) return nullptr;
  void *p = nullptr;
  if (cudaMalloc(&p, spinor_bytes(c, prec)) != cudaSuccess) { fail("out of device memory"); return nullptr; }
  cudaMemset(p, 0, spinor_bytes(c, prec));
  return p;
}
void b200_dev_free(void *p) { cudaFree(p); }

// Point source: f = 0 except component (spin, colour) = 1 at the site with
// coordinates x[0..3] (x0 = time).
int b200_dev_point_source(int prec, void *f, const int x[4], int spin, int colour) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  if (spin < 0 || spin > 3 || colour < 0 || colour > 2) return fail("point_source: spin or colour out of range");
  int n[4], y[4];
  for (int mu = 0; mu < 4; mu++) {
    if (x[mu] < 0 || x[mu] >= c.g.L[mu]) return fail("point_source: site out of range");
    n[mu] = x[mu] / c.g.bs[mu];
    y[mu] = x[mu] % c.g.bs[mu];
  }
  const int blk = ((n[0] * c.g.nb[1] + n[1]) * c.g.nb[2] + n[2]) * c.g.nb[3] + n[3];
  const int l = ((y[0] * c.g.bs[1] + y[1]) * c.g.bs[2] + y[2]) * c.g.bs[3] + y[3];
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1, sidx = l >> 1, chunk = p * c.g.nbl + blk;
  const int k = 3 * spin + colour;
  cudaMemsetAsync(f, 0, spinor_bytes(c, prec), c.stream);
  if (prec == 64) {
    const double2 one = make_double2(1.0, 0.0);
    cudaMemcpyAsync((double2 *)f + ((size_t)chunk * 12 + k) * c.g.vbh + sidx, &one, sizeof(one),
                    cudaMemcpyHostToDevice, c.stream);
  } else {
    const float one = 1.0f;
    // FP32 plane j = k/2 holds components 2j and 2j+1 as (re, im, re, im)
    cudaMemcpyAsync((float *)((float4 *)f + ((size_t)chunk * 6 + k / 2) * c.g.vbh + sidx) + 2 * (k & 1), &one,
                    sizeof(one), cudaMemcpyHostToDevice, c.stream);
  }
  return b200_sync();
}

int b200_dev_random_spinor(int prec, void *f, double sigma, unsigned long long seed) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  if (gen_spinor(c, prec, f, sigma, seed, c.stream)) return -1;
  return b200_sync();
}

int b200_dev_from_ref(int prec, const void *q, void *f) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  size_t nb = spinor_bytes(c, prec);
  if (ensure_stage(c, nb)) return -1;
  cudaMemcpyAsync(c.stage, q, nb, cudaMemcpyDefault, c.stream);
  if (spinor_from_ref(c, prec, c.stage, f, c.stream)) return -1;
  return b200_sync();
}

int b200_dev_to_ref(int prec, const void *f, void *q) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1;
  size_t nb = spinor_bytes(c, prec);
  if (ensure_stage(c, nb)) return -1;
  if (spinor_to_ref(c, prec, f, c.stage, c.stream)) return -1;
  cudaMemcpyAsync(q, c.stage, nb, cudaMemcpyDefault, c.stream);
  return b200_sync();
}

int b200_dev_dirac(int prec, int op, double mu, const void *s, void *r) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return -1;
  int rc = prec == 64 ? dirac_op<double>(c, op, mu, s, r, c.tmp64, c.stream)
                      : dirac_op<float>(c, op, (float)mu, s, r, c.tmp32, c.stream);
  if (rc) return fail("dirac: bad operator code or launch failure");
  return b200_sync();
}

int b200_dev_sap(float mu, int isolv, int nmr, int ncy, void *psi, void *rho) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return -1;
  if (isolv == 1 && (c.sw_inv_fail & 2)) return fail("sap: the SW term on the odd sites is not safely invertible");
  if (sap_prepare(c, c.stream)) return -1;
  if (sap_cycles(c, mu, isolv, nmr, ncy, psi, rho, c.tmp32, c.stream)) return -1;
  return b200_sync();
}

double b200_dev_sap_gcr(int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi, int *ifail,
                        int *status) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return -1.0;
  return sap_gcr_dev(c, nkv, nmx, istop, res, mu, eta, psi, ifail, status);
}

double b200_dev_norm2(int prec, const void *f) {
  Ctx &c = ctx();
  if (check_ready(c)) return -1.0;
  double r[2];
  if (la_norm2(c, prec, f, PAR_ALL, r)) return -1.0;
  return r[0] + r[1];
}

int b200_dev_time_dirac(int prec, int op, double mu, const void *s, void *r, int n, float *ms) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaStreamSynchronize(c.stream);
  cudaEventRecord(e0, c.stream);
  for (int i = 0; i < n; i++) {
    if (prec == 64) dirac_op<double>(c, op, mu, s, r, c.tmp64, c.stream);
    else dirac_op<float>(c, op, (float)mu, s, r, c.tmp32, c.stream);
  }
  cudaEventRecord(e1, c.stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("time_dirac: CUDA error");
}

int b200_dev_time_sap(float mu, int isolv, int nmr, int ncy, void *psi, void *rho, int n, float *ms) {
  Ctx &c = ctx();
  if (check_fields(c) || ensure_tmp(c)) return -1;
  if (sap_prepare(c, c.stream)) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaStreamSynchronize(c.stream);
  cudaEventRecord(e0, c.stream);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < ncy; k++) sap_cycle(c, mu, isolv, nmr, psi, rho, c.tmp32, c.stream);
  cudaEventRecord(e1, c.stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("time_sap: CUDA error");
}

int b200_time_Dw_dble_host(double mu, spinor_dble *s, spinor_dble *r, int n, float *ms) {
  Ctx &c = ctx();
  if (check_fields(c)) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaStreamSynchronize(c.stream);
  cudaEventRecord(e0, c.stream);
  for (int i = 0; i < n; i++) Dw_dble(mu, s, r);
  cudaEventRecord(e1, c.stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("time_Dw_dble_host: CUDA error");
}

}  // extern "C"
