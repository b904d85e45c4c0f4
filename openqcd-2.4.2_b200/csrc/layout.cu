// Geometry tables and conversion between the reference's storage order and
// the device layout of qcd.cuh.
//
// The reference labels sites by ix = ipt[x3 + L3*x2 + L2*L3*x1 + L1*L2*L3*x0]
// with the even sites first (main/README.global:128-160).  Its spinor fields
// are arrays of 24 doubles (spinor_dble) or 24 floats (spinor) in that order,
// its gauge field stores 8 links per odd site, U(x,mu) at ud[8*(ix-V/2)+2mu]
// and U(x-mu,mu) at ud[8*(ix-V/2)+2mu+1] (main/README.global:229-262), and its
// SW field stores the upper/lower Pauli matrix of site ix at swd[2ix] and
// swd[2ix+1] (modules/sw_term/sw_term.c:42-44).  The tables built here map
// every device site to those positions; the conversion kernels are plain
// gathers.
#include "lib.h"
#include <algorithm>
#include <cstring>
#include <utility>

namespace qcd {

// the pieces of the host pipeline hold at least this many sites (or a
// sixteenth of the lattice, if less): 25 MB of FP64 spinors.  At 32^3x64
// (lexicographic order, pieces of 1, 2 or 4 planes) a Dw_dble call took
// 11.0, 10.5-10.8 and 10.2-10.3 ms on one box, 16.4, 15.5 and 15.2 ms on
// another, and on a third 11.2 and 10.4 ms for 1 and 2 planes against
// 10.9 ms with the earlier pipeline of block rows
#ifndef PIPE_PIECE_SITES
#define PIPE_PIECE_SITES 131072
#endif
static const size_t kPieceSites = PIPE_PIECE_SITES;

static int pack4(const int a[4]) { return a[0] | (a[1] << 8) | (a[2] << 16) | (a[3] << 24); }

static uint64_t interleave(const int *n, int dims, int first) {
  uint64_t k = 0;
  for (int bit = 0; bit < 8; bit++)
    for (int d = 0; d < dims; d++) k |= (uint64_t)((n[first + d] >> bit) & 1) << (dims * bit + dims - 1 - d);
  return k;
}

// Traversal order of the blocks in the full-lattice operator kernels (the
// sched table).  The order decides how long the face data of a block (the
// neighbour spinors and backward links its neighbours read) waits in L2
// between its uses.  Kinds:
//   0  Morton order of the four block coordinates (bits interleaved)
//   1  lexicographic, n0 slowest (neighbours along x0 nb1*nb2*nb3 blocks apart)
//   2  lexicographic with n0 fastest (neighbours along x3 nb0 blocks apart ...)
//   3  columns along x0 (n0 fastest) in Morton order of (n1, n2, n3)
//   4  slabs of two block rows along x0, Morton order of (n1, n2, n3) inside
//      each slab, the two rows of a column together
int set_block_order(Ctx &c, int kind) {
  const Geom &g = c.g;
  if (kind < 0 || kind >= kBlockOrders) return fail("block order: unknown kind");
  std::vector<std::pair<uint64_t, int>> key(g.nbl);
  for (int b = 0; b < g.nbl; b++) {
    int n[4], r = b;
    for (int mu = 3; mu >= 0; mu--) { n[mu] = r % g.nb[mu]; r /= g.nb[mu]; }
    uint64_t k = 0;
    switch (kind) {
      case 0: k = interleave(n, 4, 0); break;
      case 1: k = (uint64_t)b; break;
      case 2: k = ((uint64_t)((n[1] * g.nb[2] + n[2]) * g.nb[3] + n[3])) * g.nb[0] + n[0]; break;
      case 3: k = interleave(n, 3, 1) * g.nb[0] + n[0]; break;
      default: k = ((uint64_t)(n[0] / 2) << 40) | (interleave(n, 3, 1) << 1) | (uint64_t)(n[0] & 1); break;
    }
    key[b] = {k, b};
  }
  std::sort(key.begin(), key.end());
  std::vector<int> sch(g.nbl);
  for (int b = 0; b < g.nbl; b++) sch[b] = key[b].second;
  if (!c.sched && cudaMalloc(&c.sched, g.nbl * sizeof(int)) != cudaSuccess)
    return fail("block order: device allocation failed");
  cudaMemcpy(c.sched, sch.data(), g.nbl * sizeof(int), cudaMemcpyHostToDevice);
  c.block_order = kind;
  return 0;
}

// Plans of the host pipeline (Dw / Dw_dble on page-locked host arrays):
// the slabs are the block rows along x0 (at least three); the pieces are
// the thinnest x0-slabs of at least kPieceSites sites (or a sixteenth of
// the lattice; at least three pieces) whose sites are a contiguous range of
// each parity half of the storage order.  Lexicographic orders with x0
// slowest qualify plane by plane; openQCD's ipt orders the sites by the
// thread-local sub-lattices with x0 slowest (modules/lattice/
// geometry.c:200-240), so pieces of L0_TRD planes qualify.  Host code only
// (the values of ipt are compared, never used as addresses).
void pipeline_plan(const int L[4], const int bs[4], const int *ipt, std::vector<Piece> &piece,
                   std::vector<Slab> &slab) {
  slab.clear();
  piece.clear();
  const int nb0 = L[0] / bs[0], bstr0 = (L[1] / bs[1]) * (L[2] / bs[2]) * (L[3] / bs[3]);
  const int vol = L[0] * L[1] * L[2] * L[3];
  if (!ipt || nb0 < 3) return;
  const int L0 = L[0], ps = vol / L0;
  std::vector<int> lo(2 * L0, vol), hi(2 * L0, -1);
  int x[4];
  for (x[0] = 0; x[0] < L0; x[0]++)
    for (x[1] = 0; x[1] < L[1]; x[1]++)
      for (x[2] = 0; x[2] < L[2]; x[2]++)
        for (x[3] = 0; x[3] < L[3]; x[3]++) {
          const int q = ipt[x[3] + L[3] * (x[2] + L[2] * (x[1] + L[1] * x[0]))];
          const int k = 2 * x[0] + ((x[0] + x[1] + x[2] + x[3]) & 1);
          lo[k] = std::min(lo[k], q);
          hi[k] = std::max(hi[k], q);
        }
  for (int P = 1; P <= L0 / 3 && piece.empty(); P++) {
    if (L0 % P || (size_t)P * ps < std::min(kPieceSites, (size_t)vol / 16)) continue;
    std::vector<Piece> pcs(L0 / P);
    bool ok = true;
    for (int i = 0; i < L0 / P && ok; i++) {
      Piece &pc = pcs[i];
      pc.t0 = i * P;
      pc.t1 = (i + 1) * P;
      for (int p = 0; p < 2 && ok; p++) {
        int a = vol, b = -1;
        for (int t = pc.t0; t < pc.t1; t++) {
          a = std::min(a, lo[2 * t + p]);
          b = std::max(b, hi[2 * t + p]);
        }
        ok = b - a + 1 == P * ps / 2;   // a plane holds ps/2 sites of each parity
        pc.q0[p] = a;
        pc.q1[p] = b + 1;
      }
    }
    if (ok) piece = pcs;
  }
  if (!piece.empty())
    for (int k = 0; k < nb0; k++) slab.push_back(Slab{k * bstr0, (k + 1) * bstr0, k * bs[0], (k + 1) * bs[0]});
}

int geometry_init(Ctx &c, const int L[4], const int bs[4], const int *ipt) {
  Geom &g = c.g;
  for (int mu = 0; mu < 4; mu++) {
    if (L[mu] < 2 || bs[mu] < 2 || (bs[mu] % 2) || (L[mu] % bs[mu]))
      return fail("geometry: block sizes must be even and divide the lattice sizes");
    if ((L[mu] / bs[mu]) % 2) return fail("geometry: the number of blocks along every axis must be even");
    if (L[mu] > 4096 || bs[mu] > 255 || L[mu] / bs[mu] > 255) return fail("geometry: sizes out of range");
    g.L[mu] = L[mu]; g.bs[mu] = bs[mu]; g.nb[mu] = L[mu] / bs[mu];
  }
  g.vol = L[0] * L[1] * L[2] * L[3];
  g.volh = g.vol / 2;
  g.nbl = g.nb[0] * g.nb[1] * g.nb[2] * g.nb[3];
  g.vb = bs[0] * bs[1] * bs[2] * bs[3];
  g.vbh = g.vb / 2;
  g.lstr[3] = 1; g.lstr[2] = bs[3]; g.lstr[1] = bs[3] * bs[2]; g.lstr[0] = bs[3] * bs[2] * bs[1];
  // domain decomposition along x0: this rank's slab of the global lattice
  c.ddg.x0off = c.dd.rank * L[0];
  c.ddg.N0 = c.dd.np * L[0];
  c.ddg.hup = c.ddg.hdn = nullptr;
  g.bstr[3] = 1; g.bstr[2] = g.nb[3]; g.bstr[1] = g.nb[3] * g.nb[2]; g.bstr[0] = g.nb[3] * g.nb[2] * g.nb[1];

  std::vector<int> bco(g.nbl), lco(g.vb);
  for (int b = 0; b < g.nbl; b++) {
    int n[4], r = b;
    for (int mu = 3; mu >= 0; mu--) { n[mu] = r % g.nb[mu]; r /= g.nb[mu]; }
    bco[b] = pack4(n);
  }
  for (int l = 0; l < g.vb; l++) {
    int y[4], r = l;
    for (int mu = 3; mu >= 0; mu--) { y[mu] = r % bs[mu]; r /= bs[mu]; }
    int p = (y[0] + y[1] + y[2] + y[3]) & 1;
    lco[p * g.vbh + l / 2] = pack4(y);
  }
  cudaFree(c.d_bcoord); cudaFree(c.d_lcoord); cudaFree(c.sched);
  c.sched = nullptr;
  if (cudaMalloc(&c.d_bcoord, g.nbl * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c.d_lcoord, g.vb * sizeof(int)) != cudaSuccess)
    return fail("geometry: device allocation failed");
  cudaMemcpy(c.d_bcoord, bco.data(), g.nbl * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(c.d_lcoord, lco.data(), g.vb * sizeof(int), cudaMemcpyHostToDevice);
  if (set_block_order(c, c.block_order)) return -1;
  g.bcoord = c.d_bcoord;
  g.lcoord = c.d_lcoord;

  cudaFree(c.d_dev2q); cudaFree(c.d_link2q); cudaFree(c.d_q2dev);
  c.d_dev2q = c.d_link2q = c.d_q2dev = nullptr;
  c.have_ipt = false;
  if (ipt) {
    std::vector<int> d2q(g.vol), l2q(4 * (size_t)g.vol), seen(g.vol, 0);
    auto lex = [&](const int x[4]) { return x[3] + L[3] * (x[2] + L[2] * (x[1] + L[1] * x[0])); };
    for (int p = 0; p < 2; p++)
      for (int b = 0; b < g.nbl; b++)
        for (int s = 0; s < g.vbh; s++) {
          int n[4], y[4], x[4];
          for (int mu = 0; mu < 4; mu++) {
            n[mu] = (bco[b] >> (8 * mu)) & 255;
            y[mu] = (lco[p * g.vbh + s] >> (8 * mu)) & 255;
            x[mu] = n[mu] * bs[mu] + y[mu];
          }
          size_t d = (size_t)(p * g.nbl + b) * g.vbh + s;
          int ix = ipt[lex(x)];
          if (ix < 0 || ix >= g.vol || seen[ix] || ((ix >= g.volh) != (p == 1)))
            return fail("geometry: ipt[] is not an even-first permutation of the lattice sites");
          seen[ix] = 1;
          d2q[d] = ix;
          for (int mu = 0; mu < 4; mu++) {
            if (p == 1) {
              l2q[4 * d + mu] = 8 * (ix - g.volh) + 2 * mu;
            } else {
              int xu[4] = {x[0], x[1], x[2], x[3]};
              xu[mu] = (xu[mu] + 1) % L[mu];
              int iy = ipt[lex(xu)];
              l2q[4 * d + mu] = 8 * (iy - g.volh) + 2 * mu + 1;
            }
          }
        }
    if (cudaMalloc(&c.d_dev2q, g.vol * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c.d_link2q, 4 * (size_t)g.vol * sizeof(int)) != cudaSuccess)
      return fail("geometry: device allocation failed");
    cudaMemcpy(c.d_dev2q, d2q.data(), g.vol * sizeof(int), cudaMemcpyHostToDevice);
    {
      std::vector<int> q2d(g.vol);
      for (int d = 0; d < g.vol; d++) q2d[d2q[d]] = d;
      if (cudaMalloc(&c.d_q2dev, g.vol * sizeof(int)) != cudaSuccess) return fail("geometry: device allocation failed");
      cudaMemcpy(c.d_q2dev, q2d.data(), g.vol * sizeof(int), cudaMemcpyHostToDevice);
    }
    cudaMemcpy(c.d_link2q, l2q.data(), 4 * (size_t)g.vol * sizeof(int), cudaMemcpyHostToDevice);
    c.h_dev2q = d2q;
    c.h_ipt.assign(ipt, ipt + g.vol);
    c.have_ipt = true;
  }
  pipeline_plan(L, bs, ipt, c.piece, c.slab);
  cudaFree(c.d_ident);
  c.d_ident = nullptr;
  {
    std::vector<int> id(g.nbl);
    for (int b = 0; b < g.nbl; b++) id[b] = b;
    if (cudaMalloc(&c.d_ident, g.nbl * sizeof(int)) != cudaSuccess) return fail("geometry: device allocation failed");
    cudaMemcpy(c.d_ident, id.data(), g.nbl * sizeof(int), cudaMemcpyHostToDevice);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : fail("geometry: CUDA error");
}

// ------------------------------------------------------------------ spinors
template <typename R>
__global__ void k_spinor_from_ref(Geom g, const int *__restrict__ d2q, const R *__restrict__ q, void *dev, int d0,
                                  int nd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  const int d = d0 + i;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  const R *src = q + (size_t)__ldg(d2q + d) * 24;
  spinor<R> v;
#pragma unroll
  for (int k = 0; k < 12; k++) v.c[k / 3].c[k % 3] = mk<R>(src[2 * k], src[2 * k + 1]);
  Store<R>::store_spinor(dev, chunk, s, g.vbh, v);
}

template <typename R>
__global__ void k_spinor_to_ref(Geom g, const int *__restrict__ d2q, const void *dev, R *q, int d0, int nd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) return;
  const int d = d0 + i;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  R *dst = q + (size_t)__ldg(d2q + d) * 24;
  spinor<R> v = Store<R>::load_spinor_rw(dev, chunk, s, g.vbh);
#pragma unroll
  for (int k = 0; k < 12; k++) { dst[2 * k] = v.c[k / 3].c[k % 3].re; dst[2 * k + 1] = v.c[k / 3].c[k % 3].im; }
}

// the sites of a piece, both parity halves in one launch: thread i takes
// storage index q0[0] + i or q0[1] + (i - n0), reads it (contiguous) and
// stores it at its device site
template <typename R>
__global__ void k_spinor_from_ref_piece(Geom g, const int *__restrict__ q2d, const R *__restrict__ q, void *dev,
                                        int qa, int na, int qb, int nb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na + nb) return;
  const int iq = i < na ? qa + i : qb + (i - na);
  const int d = __ldg(q2d + iq);
  const int chunk = d / g.vbh, s = d - chunk * g.vbh;
  const R *src = q + (size_t)iq * 24;
  spinor<R> v;
#pragma unroll
  for (int k = 0; k < 12; k++) v.c[k / 3].c[k % 3] = mk<R>(src[2 * k], src[2 * k + 1]);
  Store<R>::store_spinor(dev, chunk, s, g.vbh, v);
}

int spinor_from_ref_piece(const Ctx &c, int prec, const void *q, void *dev, const Piece &pc, cudaStream_t st) {
  if (!c.d_q2dev) return fail("no reference site order: pass ipt[] to the geometry call");
  const int t = 128, na = pc.q1[0] - pc.q0[0], nb = pc.q1[1] - pc.q0[1];
  const unsigned grid = (unsigned)((na + nb + t - 1) / t);
  if (prec == 64)
    k_spinor_from_ref_piece<double><<<grid, t, 0, st>>>(c.g, c.d_q2dev, (const double *)q, dev, pc.q0[0], na,
                                                        pc.q0[1], nb);
  else
    k_spinor_from_ref_piece<float><<<grid, t, 0, st>>>(c.g, c.d_q2dev, (const float *)q, dev, pc.q0[0], na,
                                                       pc.q0[1], nb);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("spinor_from_ref: launch failed");
}

int spinor_from_ref_range(const Ctx &c, int prec, const void *q, void *dev, int d0, int n, cudaStream_t st) {
  if (!c.have_ipt) return fail("no reference site order: pass ipt[] to the geometry call");
  const int t = 128;
  if (n <= 0) return 0;
  if (prec == 64)
    k_spinor_from_ref<double><<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_dev2q, (const double *)q, dev, d0, n);
  else
    k_spinor_from_ref<float><<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_dev2q, (const float *)q, dev, d0, n);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("spinor_from_ref: launch failed");
}

int spinor_to_ref_range(const Ctx &c, int prec, const void *dev, void *q, int d0, int n, cudaStream_t st) {
  if (!c.have_ipt) return fail("no reference site order: pass ipt[] to the geometry call");
  const int t = 128;
  if (n <= 0) return 0;
  if (prec == 64) k_spinor_to_ref<double><<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_dev2q, dev, (double *)q, d0, n);
  else k_spinor_to_ref<float><<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_dev2q, dev, (float *)q, d0, n);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("spinor_to_ref: launch failed");
}

int spinor_from_ref(const Ctx &c, int prec, const void *q, void *dev, cudaStream_t st) {
  return spinor_from_ref_range(c, prec, q, dev, 0, c.g.vol, st);
}

int spinor_to_ref(const Ctx &c, int prec, const void *dev, void *q, cudaStream_t st) {
  return spinor_to_ref_range(c, prec, dev, q, 0, c.g.vol, st);
}

// -------------------------------------------------------------------- links
__global__ void k_links_from_ref(Geom g, const int *__restrict__ l2q, const double *__restrict__ q, double2 *ud) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * g.vol) return;
  int d = i >> 2, mu = i & 3;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  const double *src = q + (size_t)__ldg(l2q + i) * 18;
  double2 *dst = ud + ((size_t)chunk * 4 + mu) * 9 * g.vbh + s;
#pragma unroll
  for (int k = 0; k < 9; k++) dst[(size_t)k * g.vbh] = make_double2(src[2 * k], src[2 * k + 1]);
}

__global__ void k_links_to_ref(Geom g, const int *__restrict__ l2q, const double2 *__restrict__ ud, double *q) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * g.vol) return;
  int d = i >> 2, mu = i & 3;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  double *dst = q + (size_t)__ldg(l2q + i) * 18;
  const double2 *src = ud + ((size_t)chunk * 4 + mu) * 9 * g.vbh + s;
#pragma unroll
  for (int k = 0; k < 9; k++) { double2 v = src[(size_t)k * g.vbh]; dst[2 * k] = v.x; dst[2 * k + 1] = v.y; }
}

int links_from_ref(Ctx &c, const void *qud, cudaStream_t st) {
  if (!c.have_ipt) return fail("no reference site order: pass ipt[] to the geometry call");
  int n = 4 * c.g.vol, t = 128;
  k_links_from_ref<<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_link2q, (const double *)qud, c.ud);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("links_from_ref: launch failed");
}

int links_to_ref(const Ctx &c, void *qud, cudaStream_t st) {
  if (!c.have_ipt) return fail("no reference site order: pass ipt[] to the geometry call");
  int n = 4 * c.g.vol, t = 128;
  k_links_to_ref<<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_link2q, c.ud, (double *)qud);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("links_to_ref: launch failed");
}

// -------------------------------------------------------------------- pauli
__global__ void k_pauli_from_ref(Geom g, const int *__restrict__ d2q, const double *__restrict__ q, double2 *sw) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  const double *src = q + (size_t)__ldg(d2q + d) * 72;
  double2 *dst = sw + (size_t)chunk * 36 * g.vbh + s;
#pragma unroll 4
  for (int k = 0; k < 36; k++) dst[(size_t)k * g.vbh] = make_double2(src[2 * k], src[2 * k + 1]);
}

__global__ void k_pauli_to_ref(Geom g, const int *__restrict__ d2q, const double2 *__restrict__ sw, double *q) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  double *dst = q + (size_t)__ldg(d2q + d) * 72;
  const double2 *src = sw + (size_t)chunk * 36 * g.vbh + s;
#pragma unroll 4
  for (int k = 0; k < 36; k++) { double2 v = src[(size_t)k * g.vbh]; dst[2 * k] = v.x; dst[2 * k + 1] = v.y; }
}

int pauli_from_ref(Ctx &c, const void *qsw, cudaStream_t st) {
  if (!c.have_ipt) return fail("no reference site order: pass ipt[] to the geometry call");
  int n = c.g.vol, t = 128;
  k_pauli_from_ref<<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_dev2q, (const double *)qsw, c.swd);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("pauli_from_ref: launch failed");
}

int pauli_to_ref(const Ctx &c, int which, void *qsw, cudaStream_t st) {
  if (!c.have_ipt) return fail("no reference site order: pass ipt[] to the geometry call");
  int n = c.g.vol, t = 128;
  k_pauli_to_ref<<<(n + t - 1) / t, t, 0, st>>>(c.g, c.d_dev2q, which ? c.swd_inv : c.swd, (double *)qsw);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("pauli_to_ref: launch failed");
}

}  // namespace qcd
