// SW (clover) term on the device: construction from the gauge field, 6x6
// inversion with the reference's safety criterion, FP32 copies, and the
// site-local apply_sw/apply_swinv on arrays in the reference's storage order.
#include "lib.h"
#include <cfloat>
#include <cmath>

namespace qcd {

// ------------------------------------------------------------ 6x6 inversion
// Inverse of the complex 6x6 matrix m + i mu (m Hermitian in the packed
// format of mul_pauli), by Gauss-Jordan elimination with partial pivoting.
// Returns the Hermitian part of the inverse in packed format, and the
// reference's safety flag (modules/sw_term/pauli_dble.c:1718-1759): the
// inversion is unsafe if a pivot is below eps = 1e-4 |m+i mu|_F^2 or if
// eps |(m+i mu)^-1|_F^2 > 1, i.e. the Frobenius condition number exceeds 100.
__device__ int inv_pauli(double mu, const double u[36], double out[36]) {
  double ar[36], ai[36], br[36], bi[36];
  double fn = 0.0;
#pragma unroll
  for (int i = 0; i < 36; i++) { ar[i] = ai[i] = br[i] = bi[i] = 0.0; }
  int k = 6;
  for (int i = 0; i < 6; i++) {
    ar[7 * i] = u[i];
    ai[7 * i] = mu;
    br[7 * i] = 1.0;
    fn += u[i] * u[i] + mu * mu;
    for (int j = i + 1; j < 6; j++) {
      ar[6 * i + j] = u[k]; ai[6 * i + j] = u[k + 1];
      ar[6 * j + i] = u[k]; ai[6 * j + i] = -u[k + 1];
      fn += 2.0 * (u[k] * u[k] + u[k + 1] * u[k + 1]);
      k += 2;
    }
  }
  const double eps = 1.0e-4 * fn;
  int ifail = 0;
  for (int c = 0; c < 6; c++) {
    int piv = c;
    double best = ar[6 * c + c] * ar[6 * c + c] + ai[6 * c + c] * ai[6 * c + c];
    for (int r = c + 1; r < 6; r++) {
      double v = ar[6 * r + c] * ar[6 * r + c] + ai[6 * r + c] * ai[6 * r + c];
      if (v > best) { best = v; piv = r; }
    }
    if (best == 0.0) ifail = 1;
    if (piv != c) {
      for (int j = 0; j < 6; j++) {
        double t;
        t = ar[6 * c + j]; ar[6 * c + j] = ar[6 * piv + j]; ar[6 * piv + j] = t;
        t = ai[6 * c + j]; ai[6 * c + j] = ai[6 * piv + j]; ai[6 * piv + j] = t;
        t = br[6 * c + j]; br[6 * c + j] = br[6 * piv + j]; br[6 * piv + j] = t;
        t = bi[6 * c + j]; bi[6 * c + j] = bi[6 * piv + j]; bi[6 * piv + j] = t;
      }
    }
    // 1 / pivot
    double pr = ar[6 * c + c], pi = ai[6 * c + c];
    double d = pr * pr + pi * pi;
    if (d == 0.0) d = 1.0;
    double qr = pr / d, qi = -pi / d;
    for (int j = 0; j < 6; j++) {
      double xr = ar[6 * c + j], xi = ai[6 * c + j];
      ar[6 * c + j] = xr * qr - xi * qi; ai[6 * c + j] = xr * qi + xi * qr;
      xr = br[6 * c + j]; xi = bi[6 * c + j];
      br[6 * c + j] = xr * qr - xi * qi; bi[6 * c + j] = xr * qi + xi * qr;
    }
    for (int r = 0; r < 6; r++) {
      if (r == c) continue;
      double fr = ar[6 * r + c], fi = ai[6 * r + c];
      for (int j = 0; j < 6; j++) {
        ar[6 * r + j] -= fr * ar[6 * c + j] - fi * ai[6 * c + j];
        ai[6 * r + j] -= fr * ai[6 * c + j] + fi * ar[6 * c + j];
        br[6 * r + j] -= fr * br[6 * c + j] - fi * bi[6 * c + j];
        bi[6 * r + j] -= fr * bi[6 * c + j] + fi * br[6 * c + j];
      }
    }
  }
  double sm = 0.0;
  for (int i = 0; i < 36; i++) sm += br[i] * br[i] + bi[i] * bi[i];
  if (eps * sm > 1.0) ifail = 1;
  k = 6;
  for (int i = 0; i < 6; i++) {
    out[i] = br[7 * i];
    for (int j = i + 1; j < 6; j++) {
      out[k] = 0.5 * (br[6 * i + j] + br[6 * j + i]);
      out[k + 1] = 0.5 * (bi[6 * i + j] - bi[6 * j + i]);
      k += 2;
    }
  }
  return ifail;
}

// swd -> swd_inv (all sites, mu = 0), sw32, sw32_inv
// INV = false: swd_inv already holds the inverses (exponential SW term),
// only the FP32 copies are made
template <bool INV>
__global__ void k_sw_derive(Geom g, const double2 *__restrict__ swd, double2 *swd_inv, float4 *sw32,
                            float4 *sw32_inv, int *fail) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  int bad = 0;
  for (int half = 0; half < 2; half++) {
    double u[36], v[36];
    const double2 *src = swd + ((size_t)chunk * 36 + 18 * half) * g.vbh + s;
    for (int k = 0; k < 18; k++) { double2 x = src[(size_t)k * g.vbh]; u[2 * k] = x.x; u[2 * k + 1] = x.y; }
    double2 *dst = swd_inv + ((size_t)chunk * 36 + 18 * half) * g.vbh + s;
    if (INV) {
      bad |= inv_pauli(0.0, u, v);
      for (int k = 0; k < 18; k++) dst[(size_t)k * g.vbh] = make_double2(v[2 * k], v[2 * k + 1]);
    } else {
      for (int k = 0; k < 18; k++) {
        const double2 x = dst[(size_t)k * g.vbh];
        v[2 * k] = x.x;
        v[2 * k + 1] = x.y;
      }
    }
    float4 *d32 = sw32 + ((size_t)chunk * 18 + 9 * half) * g.vbh + s;
    float4 *i32 = sw32_inv + ((size_t)chunk * 18 + 9 * half) * g.vbh + s;
    for (int j = 0; j < 9; j++) {
      d32[(size_t)j * g.vbh] = make_float4((float)u[4 * j], (float)u[4 * j + 1], (float)u[4 * j + 2], (float)u[4 * j + 3]);
      i32[(size_t)j * g.vbh] = make_float4((float)v[4 * j], (float)v[4 * j + 1], (float)v[4 * j + 2], (float)v[4 * j + 3]);
    }
  }
  if (bad) atomicOr(fail, 1 << (chunk >= g.nbl ? 1 : 0));
}

static int alloc_sw(Ctx &c) {
  size_t n64 = (size_t)c.g.vol * 36 * sizeof(double2);
  size_t n32 = (size_t)c.g.vol * 18 * sizeof(float4);
  if (!c.swd && cudaMalloc(&c.swd, n64) != cudaSuccess) return fail("out of device memory (SW field)");
  if (!c.swd_inv && cudaMalloc(&c.swd_inv, n64) != cudaSuccess) return fail("out of device memory (SW field)");
  if (!c.sw32 && cudaMalloc(&c.sw32, n32) != cudaSuccess) return fail("out of device memory (SW field)");
  if (!c.sw32_inv && cudaMalloc(&c.sw32_inv, n32) != cudaSuccess) return fail("out of device memory (SW field)");
  return 0;
}

int sw_refresh_derived(Ctx &c, cudaStream_t st, bool inv_given) {
  if (alloc_sw(c)) return -1;
  int *dfail;
  if (cudaMallocAsync(&dfail, sizeof(int), st) != cudaSuccess) return fail("allocation failed");
  cudaMemsetAsync(dfail, 0, sizeof(int), st);
  int t = 128;
  if (inv_given)
    k_sw_derive<false><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, c.swd, c.swd_inv, c.sw32, c.sw32_inv, dfail);
  else
    k_sw_derive<true><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, c.swd, c.swd_inv, c.sw32, c.sw32_inv, dfail);
  int hf = 0;
  cudaMemcpyAsync(&hf, dfail, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dfail, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("sw_refresh_derived: CUDA error");
  c.sw_inv_fail = hf;   // bit 0: even sites unsafe, bit 1: odd sites unsafe
  c.h16_valid = false;
  c.sw_inv_ok = (hf == 0);
  c.have_sw = true;
  return 0;
}

// ------------------------------------------------------------ SW from links
__device__ __forceinline__ void dev_index(const Geom &g, const int x[4], int &chunk, int &s) {
  int blk = 0, l = 0, p = 0;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    int xm = x[mu];
    int n = xm / g.bs[mu];
    int y = xm - n * g.bs[mu];
    blk += n * g.bstr[mu];
    l += y * g.lstr[mu];
    p += xm;
  }
  chunk = (p & 1) * g.nbl + blk;
  s = l >> 1;
}

__device__ __forceinline__ su3<double> link_at(const Geom &g, const double2 *ud, const int x[4], int mu) {
  int chunk, s;
  dev_index(g, x, chunk, s);
  return Store<double>::load_link(ud, chunk, mu, s, g.vbh);
}

// With domain decomposition x[0] runs from -1 to L0: the planes x0 = -1 and
// x0 = L0 are the neighbour ranks' last and first planes, whose four links
// per site arrived in the faces dg.hdn, dg.hup (18 doubles per link, four
// links per face site).
__device__ __forceinline__ su3<double> link_dd(const Geom &g, const DDGeom &dg, const double2 *ud, const int x[4],
                                               int mu) {
  if (x[0] >= 0 && x[0] < g.L[0]) return link_at(g, ud, x, mu);
  int n[4], y[4];
  for (int k = 1; k < 4; k++) {
    n[k] = x[k] / g.bs[k];
    y[k] = x[k] - n[k] * g.bs[k];
  }
  n[0] = y[0] = 0;
  const double *p = (const double *)(x[0] < 0 ? dg.hdn : dg.hup) + ((size_t)face_index_of(g, n, y) * 4 + mu) * 18;
  su3<double> u;
  for (int k = 0; k < 9; k++) u.e[k] = mk<double>(p[2 * k], p[2 * k + 1]);
  return u;
}

__device__ __forceinline__ su3<double> mm(const su3<double> &a, const su3<double> &b) {
  su3<double> r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        re += a.e[3 * i + k].re * b.e[3 * k + j].re - a.e[3 * i + k].im * b.e[3 * k + j].im;
        im += a.e[3 * i + k].re * b.e[3 * k + j].im + a.e[3 * i + k].im * b.e[3 * k + j].re;
      }
      r.e[3 * i + j] = mk<double>(re, im);
    }
  return r;
}
__device__ __forceinline__ su3<double> dag(const su3<double> &a) {
  su3<double> r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) r.e[3 * i + j] = mk<double>(a.e[3 * j + i].re, -a.e[3 * j + i].im);
  return r;
}
// X += (M - M^dag)/8 in the 9-real U(3) algebra convention of the reference
// (modules/su3fcts/su3prod.c:56-63): X_kk = i c_k, X_01 = c4 + i c5,
// X_02 = c6 + i c7, X_12 = c8 + i c9.
__device__ __forceinline__ void add_antiherm(const su3<double> &m, double X[9]) {
  const double r = 0.125;
  X[0] += r * 2.0 * m.e[0].im;
  X[1] += r * 2.0 * m.e[4].im;
  X[2] += r * 2.0 * m.e[8].im;
  X[3] += r * (m.e[1].re - m.e[3].re);
  X[4] += r * (m.e[1].im + m.e[3].im);
  X[5] += r * (m.e[2].re - m.e[6].re);
  X[6] += r * (m.e[2].im + m.e[6].im);
  X[7] += r * (m.e[5].re - m.e[7].re);
  X[8] += r * (m.e[5].im + m.e[7].im);
}

// Clover field tensor F_{mu nu}(x) = (1/8) sum over the four plaquettes with a
// corner at x of (P - P^dag), each plaquette read in the orientation the
// reference uses (modules/tcharge/ftensor.c:141-192, periodic case).
template <int DD>
__device__ void ftensor_site(const Geom &g, const DDGeom &dg, const double2 *ud, const int x[4], int mu, int nu,
                             double X[9]) {
  for (int k = 0; k < 9; k++) X[k] = 0.0;
  int c[4], a[4], b[4], ab[4];
  // periodic shifts; with domain decomposition x0 is not wrapped (the
  // planes -1 and L0 come from the neighbour ranks)
  auto sh = [&](const int *in, int *o, int dm, int sm, int dn, int sn) {
    for (int k = 0; k < 4; k++) o[k] = in[k];
    if (sm) o[dm] = (DD && dm == 0) ? o[dm] + sm : (o[dm] + sm + g.L[dm]) % g.L[dm];
    if (sn) o[dn] = (DD && dn == 0) ? o[dn] + sn : (o[dn] + sn + g.L[dn]) % g.L[dn];
  };
  auto link_at = [&](const Geom &gg, const double2 *u, const int *xx, int m) {
    if constexpr (DD != 0) return link_dd(gg, dg, u, xx, m);
    else return qcd::link_at(gg, u, xx, m);
  };
  // corner c = x : leaf = w1 w2,  w1 = U(c,mu)U(c+mu,nu), w2 = U(c+nu,mu)^dag U(c,nu)^dag
  sh(x, c, mu, 0, nu, 0);
  sh(c, a, mu, 1, nu, 0);
  sh(c, b, mu, 0, nu, 1);
  {
    su3<double> w1 = mm(link_at(g, ud, c, mu), link_at(g, ud, a, nu));
    su3<double> w2 = mm(dag(link_at(g, ud, b, mu)), dag(link_at(g, ud, c, nu)));
    add_antiherm(mm(w1, w2), X);
  }
  // corner c = x - mu - nu : leaf = w2 w1
  sh(x, c, mu, -1, nu, -1);
  sh(c, a, mu, 1, nu, 0);
  sh(c, b, mu, 0, nu, 1);
  {
    su3<double> w1 = mm(link_at(g, ud, c, mu), link_at(g, ud, a, nu));
    su3<double> w2 = mm(dag(link_at(g, ud, b, mu)), dag(link_at(g, ud, c, nu)));
    add_antiherm(mm(w2, w1), X);
  }
  // corner c = x - nu : leaf = w1' w2', w1' = U(c,nu)^dag U(c,mu), w2' = U(c+mu,nu) U(c+nu,mu)^dag
  sh(x, c, mu, 0, nu, -1);
  sh(c, a, mu, 1, nu, 0);
  sh(c, b, mu, 0, nu, 1);
  {
    su3<double> w1 = mm(dag(link_at(g, ud, c, nu)), link_at(g, ud, c, mu));
    su3<double> w2 = mm(link_at(g, ud, a, nu), dag(link_at(g, ud, b, mu)));
    add_antiherm(mm(w1, w2), X);
  }
  // corner c = x - mu : leaf = w2' w1'
  sh(x, c, mu, -1, nu, 0);
  sh(c, a, mu, 1, nu, 0);
  sh(c, b, mu, 0, nu, 1);
  {
    su3<double> w1 = mm(dag(link_at(g, ud, c, nu)), link_at(g, ud, c, mu));
    su3<double> w2 = mm(link_at(g, ud, a, nu), dag(link_at(g, ud, b, mu)));
    add_antiherm(mm(w2, w1), X);
  }
}

// The linear map from a U(3) algebra element X (9 reals) to the entries of a
// packed Pauli matrix, one map per spatial pairing of field-tensor
// components.  Restated from u3_alg2pauli1/2/3 of the reference
// (modules/sw_term/sw_term.c:145-219); entry = (target, source, sign), with
// mode 0 = assign, 1 = add.
struct PMap { signed char t, src, sgn, add; };
__constant__ PMap pmap1[15] = {
    {10, 0, -1, 0}, {12, 4, -1, 0}, {13, 3, 1, 0}, {14, 6, -1, 0}, {15, 5, 1, 0},
    {18, 4, -1, 0}, {19, 3, -1, 0}, {20, 1, -1, 0}, {22, 8, -1, 0}, {23, 7, 1, 0},
    {24, 6, -1, 0}, {25, 5, -1, 0}, {26, 8, -1, 0}, {27, 7, -1, 0}, {28, 2, -1, 0}};
__constant__ PMap pmap2[17] = {
    {11, 0, 1, 0}, {12, 3, 1, 1}, {13, 4, 1, 1}, {14, 5, 1, 1}, {15, 6, 1, 1}, {18, 3, -1, 1},
    {19, 4, 1, 1}, {21, 1, 1, 0}, {22, 7, 1, 1}, {23, 8, 1, 1}, {24, 5, -1, 1}, {25, 6, 1, 1},
    {26, 7, -1, 1}, {27, 8, 1, 1}, {29, 2, 1, 0}, {0, 0, 0, 2}, {0, 0, 0, 2}};
__constant__ PMap pmap3[18] = {
    {0, 0, -1, 0}, {1, 1, -1, 0}, {2, 2, -1, 0}, {3, 0, 1, 0}, {4, 1, 1, 0}, {5, 2, 1, 0},
    {6, 4, -1, 0}, {7, 3, 1, 0}, {8, 6, -1, 0}, {9, 5, 1, 0}, {16, 8, -1, 0}, {17, 7, 1, 0},
    {30, 4, 1, 0}, {31, 3, -1, 0}, {32, 6, 1, 0}, {33, 5, -1, 0}, {34, 8, 1, 0}, {35, 7, -1, 0}};

__device__ __forceinline__ void apply_pmap(const PMap *m, int n, const double X[9], double u[36]) {
  for (int i = 0; i < n; i++) {
    PMap e = m[i];
    if (e.add == 2) continue;
    double v = e.sgn * X[e.src];
    if (e.add) u[e.t] += v;
    else u[e.t] = v;
  }
}

// SW term per site (modules/sw_term/sw_term.c:225-243 pauli_term and
// :247-345 set_swd, periodic case): with c2 = -csw/2,
//   upper = c2*(F23-F01, F31-F02, F12-F03) mapped by pmap1/2/3, + (4+m0) on the diagonal
//   lower = c2*(F23+F01, F31+F02, F12+F03) likewise.
// ------------------------------------------------ exponential SW term
// isw = 1 (modules/sw_term/sw_term.c:46-49, swexp.c): the SW matrices are
// c exp(A) with A = c2/c * (clover term) traceless Hermitian, and their
// inverses (1/c) exp(-A).  exp(A) is its Taylor series to order n (the order
// of sw_order(), sw_term.c:95) reduced to a polynomial of degree 5 in A by
// the characteristic polynomial A^6 = -(p4 A^4 + p3 A^3 + p2 A^2 + p1 A + p0)
// (Cayley-Hamilton; A traceless, so no A^5 term), the p_k from the power
// sums s_k = tr A^k by Newton's identities; the series is folded in from its
// highest term down (Horner).
struct ExpCoef {
  int n;
  double c[100];   // 1/k!, k = 0..n
};

typedef double2 cmat6[6][6];

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ void cmat_mul(const cmat6 a, const cmat6 b, cmat6 out) {
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double2 z = make_double2(0.0, 0.0);
      for (int k = 0; k < 6; k++) {
        const double2 t = cmul(a[i][k], b[k][j]);
        z.x += t.x;
        z.y += t.y;
      }
      out[i][j] = z;
    }
}

// r * sum_k q_k A^k from A, A^2, A^3: (q0 + q1 A + q2 A^2) + (q3 + q4 A + q5 A^2) A^3,
// packed as a Pauli matrix (the result is Hermitian)
__device__ void exp_pack(const cmat6 A, const cmat6 A2, const cmat6 A3, const double q[6], double r, double out[36]) {
  cmat6 M;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      const double d = i == j ? q[3] : 0.0;
      M[i][j] = make_double2(d + q[4] * A[i][j].x + q[5] * A2[i][j].x, q[4] * A[i][j].y + q[5] * A2[i][j].y);
    }
  int k = 6;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++) {
      double2 z = make_double2((i == j ? q[0] : 0.0) + q[1] * A[i][j].x + q[2] * A2[i][j].x,
                               q[1] * A[i][j].y + q[2] * A2[i][j].y);
      for (int l = 0; l < 6; l++) {
        const double2 t = cmul(M[i][l], A3[l][j]);
        z.x += t.x;
        z.y += t.y;
      }
      if (i == j) {
        out[i] = r * z.x;
      } else {
        out[k] = r * z.x;
        out[k + 1] = r * z.y;
        k += 2;
      }
    }
}

// Taylor coefficients (sign = -1: of exp(-A)) folded to degree 5
__device__ void exp_fold(const ExpCoef &ec, double sign, const double p[5], double q[6]) {
  const int n = ec.n;
  auto cs = [&](int k) { return (sign < 0.0 && (k & 1)) ? -ec.c[k] : ec.c[k]; };
  if (n > 5) {
    for (int j = 0; j < 6; j++) q[j] = cs(n - 5 + j);
    for (int k = n - 6; k >= 0; k--) {
      const double q5 = q[5];
      q[5] = q[4];
      q[4] = q[3] - q5 * p[4];
      q[3] = q[2] - q5 * p[3];
      q[2] = q[1] - q5 * p[2];
      q[1] = q[0] - q5 * p[1];
      q[0] = cs(k) - q5 * p[0];
    }
  } else {
    for (int j = 0; j < 6; j++) q[j] = j <= n ? cs(j) : 0.0;
  }
}

// u: the Pauli matrix of A; B = r exp(A), Binv = (1/r) exp(-A)
__device__ void sw_exp_site(const double u[36], const ExpCoef &ec, double r, double B[36], double Binv[36]) {
  cmat6 A, A2, A3;
  int k = 6;
  for (int i = 0; i < 6; i++) {
    A[i][i] = make_double2(u[i], 0.0);
    for (int j = i + 1; j < 6; j++) {
      A[i][j] = make_double2(u[k], u[k + 1]);
      A[j][i] = make_double2(u[k], -u[k + 1]);
      k += 2;
    }
  }
  cmat_mul(A, A, A2);
  cmat_mul(A2, A, A3);
  double s2 = 0.0, s3 = 0.0, s4 = 0.0, s5 = 0.0, s6 = 0.0;
  for (int i = 0; i < 6; i++) {
    s2 += A2[i][i].x;
    s3 += A3[i][i].x;
    for (int j = 0; j < 6; j++) {
      s4 += A2[i][j].x * A2[i][j].x + A2[i][j].y * A2[i][j].y;   // tr A^4 = sum |(A^2)_ij|^2
      s6 += A3[i][j].x * A3[i][j].x + A3[i][j].y * A3[i][j].y;   // tr A^6
      s5 += cmul(A2[i][j], A3[j][i]).x;                          // tr A^5
    }
  }
  double p[5];
  p[4] = -0.5 * s2;
  p[3] = -s3 / 3.0;
  p[2] = (s2 * s2 - 2.0 * s4) / 8.0;
  p[1] = (5.0 * s2 * s3 - 6.0 * s5) / 30.0;
  p[0] = (8.0 * s3 * s3 - 24.0 * s6 + s2 * (18.0 * s4 - 3.0 * s2 * s2)) / 144.0;
  double q[6];
  exp_fold(ec, 1.0, p, q);
  exp_pack(A, A2, A3, q, r, B);
  exp_fold(ec, -1.0, p, q);
  exp_pack(A, A2, A3, q, 1.0 / r, Binv);
}

// sw_order (sw_term.c:95-121): the Taylor order that reaches machine
// precision for matrices with |A| <= 3 csw/(4+m0); -1 if none below 100
static int sw_exp_order(double csw, double m0) {
  const double c = 3.0 * std::fabs(csw / (4.0 + m0));
  double a = c * std::exp(c), b = DBL_EPSILON;
  for (int n = 1; n < 100; n++) {
    a *= c;
    b *= (double)(n + 1);
    if (a < b) return n;
  }
  return -1;
}

template <bool ISW, int DD>
__global__ void k_sw_term(Geom g, DDGeom dg, const double2 *__restrict__ ud, double2 *swd, double2 *swd_inv,
                          double c1, double c2, ExpCoef ec) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  int p = chunk >= g.nbl;
  int blk = chunk - p * g.nbl;
  Site xs;
  site_decode(g, p, blk, s, xs);
  int x[4];
  for (int mu = 0; mu < 4; mu++) x[mu] = xs.n[mu] * g.bs[mu] + xs.y[mu];
  const int planes[6][2] = {{0, 1}, {0, 2}, {0, 3}, {2, 3}, {3, 1}, {1, 2}};
  double F[6][9];
  for (int n = 0; n < 6; n++) ftensor_site<DD>(g, dg, ud, x, planes[n][0], planes[n][1], F[n]);
  for (int half = 0; half < 2; half++) {
    double u[36], X[9];
    const double sg = half == 0 ? -1.0 : 1.0;
    for (int k = 0; k < 9; k++) X[k] = c2 * (F[3][k] + sg * F[0][k]);
    apply_pmap(pmap1, 15, X, u);
    for (int k = 0; k < 9; k++) X[k] = c2 * (F[4][k] + sg * F[1][k]);
    apply_pmap(pmap2, 17, X, u);
    for (int k = 0; k < 9; k++) X[k] = c2 * (F[5][k] + sg * F[2][k]);
    apply_pmap(pmap3, 18, X, u);
    double2 *dst = swd + ((size_t)chunk * 36 + 18 * half) * g.vbh + s;
    if (ISW) {
      double B[36], Bi[36];
      sw_exp_site(u, ec, c1, B, Bi);
      double2 *dsti = swd_inv + ((size_t)chunk * 36 + 18 * half) * g.vbh + s;
      for (int k = 0; k < 18; k++) {
        dst[(size_t)k * g.vbh] = make_double2(B[2 * k], B[2 * k + 1]);
        dsti[(size_t)k * g.vbh] = make_double2(Bi[2 * k], Bi[2 * k + 1]);
      }
    } else {
      for (int k = 0; k < 6; k++) u[k] += c1;
      for (int k = 0; k < 18; k++) dst[(size_t)k * g.vbh] = make_double2(u[2 * k], u[2 * k + 1]);
    }
  }
}

// the four links of each site of the first (side 0) and last (side 1)
// local planes, for the neighbour ranks' clover leaves
__global__ void k_sw_dd_pack(Geom g, const double2 *__restrict__ ud, double *dn, double *up) {
  const int F = face_sites(g);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * F) return;
  const int side = i >= F, f = i - side * F;
  int chunk, s, n[4], y[4];
  face_site(g, side, f, chunk, s, n, y);
  double *dst = (side ? up : dn) + (size_t)f * 72;
  for (int mu = 0; mu < 4; mu++) {
    const su3<double> u = Store<double>::load_link(ud, chunk, mu, s, g.vbh);
    for (int k = 0; k < 9; k++) {
      dst[mu * 18 + 2 * k] = u.e[k].re;
      dst[mu * 18 + 2 * k + 1] = u.e[k].im;
    }
  }
}

int sw_compute(Ctx &c, cudaStream_t st) {
  if (!c.have_ud) return fail("sw_term: no gauge field on the device");
  if (c.bc != 3) return fail("sw_term: only periodic boundary conditions (type 3) are supported");
  if (alloc_sw(c)) return -1;
  int t = 64;
  DDGeom dg = c.ddg;
  const bool dd = dd_on(c);
  if (dd) {
    // the neighbours' link planes: x0 = -1 (from below) and x0 = L0 (from above)
    const int F = c.g.L[1] * c.g.L[2] * c.g.L[3];
    k_sw_dd_pack<<<(unsigned)((2 * F + 127) / 128), 128, 0, st>>>(c.g, c.ud, (double *)c.dd.buf[0],
                                                                   (double *)c.dd.buf[1]);
    if (dd_exchange(c, (size_t)F * 576, st)) return -1;
    dg.hup = c.dd.buf[2];
    dg.hdn = c.dd.buf[3];
  }
  const double c1 = 4.0 + c.m0;
  ExpCoef ec{};
  if (c.isw) {
    ec.n = sw_exp_order(c.csw, c.m0);
    if (ec.n < 0) return fail("sw_order: SW parameters are out of range");
    ec.c[0] = 1.0;
    for (int k = 1; k <= ec.n; k++) ec.c[k] = ec.c[k - 1] / (double)k;
    if (dd) k_sw_term<true, 1><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, dg, c.ud, c.swd, c.swd_inv, c1, -0.5 * c.csw / c1, ec);
    else k_sw_term<true, 0><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, dg, c.ud, c.swd, c.swd_inv, c1, -0.5 * c.csw / c1, ec);
  } else {
    if (dd) k_sw_term<false, 1><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, dg, c.ud, c.swd, c.swd_inv, c1, -0.5 * c.csw, ec);
    else k_sw_term<false, 0><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, dg, c.ud, c.swd, c.swd_inv, c1, -0.5 * c.csw, ec);
  }
  if (cudaGetLastError() != cudaSuccess) return fail("sw_term: launch failed");
  // the exponential form brings its exact inverse (1/c) exp(-A): no
  // numerical inversion, no failure (sw_term.c:312-320)
  return sw_refresh_derived(c, st, c.isw != 0);
}

// Add dm to the diagonal of every Pauli matrix (a change of the bare mass
// m0 in the SW term, whose diagonal is 4 + m0 + clover part), then refresh
// the inverses and FP32 copies.
__global__ void k_sw_shift(Geom g, double2 *swd, double dm) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  for (int half = 0; half < 2; half++) {
    double2 *p = swd + ((size_t)chunk * 36 + 18 * half) * g.vbh + s;
    for (int k = 0; k < 3; k++) {   // u[0..5] are the real parts of planes 0..2
      double2 v = p[(size_t)k * g.vbh];
      v.x += dm;
      v.y += dm;
      p[(size_t)k * g.vbh] = v;
    }
  }
}

int sw_shift_mass(Ctx &c, double dm, cudaStream_t st) {
  if (!c.have_sw) return fail("no SW field on the device");
  if (c.isw) {
    // exponential form: the mass enters the exponent, so recompute from the
    // links (as the reference's sw_term does after set_sw_parms)
    const double m0 = c.m0;
    c.m0 = m0 + dm;
    const int rc = sw_compute(c, st);
    c.m0 = m0;
    return rc;
  }
  int t = 128;
  k_sw_shift<<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, c.swd, dm);
  return sw_refresh_derived(c, st);
}

// ------------------------------------------------------------ FP32 links
__global__ void k_links_f32(size_t n, const double2 *__restrict__ a, float2 *b) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) { double2 v = a[i]; b[i] = make_float2((float)v.x, (float)v.y); }
}

int links_refresh_f32(Ctx &c, cudaStream_t st) {
  size_t n = (size_t)c.g.vol * 36;
  if (!c.u32 && cudaMalloc(&c.u32, n * sizeof(float2)) != cudaSuccess) return fail("out of device memory (links)");
  k_links_f32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, c.ud, c.u32);
  c.h16_valid = false;
  c.u12_valid = false;
  return cudaGetLastError() == cudaSuccess ? 0 : fail("links_refresh_f32: launch failed");
}

// ------------------------------------------- site-local SW on reference arrays
// apply_sw_dble(vol,mu,m,s,r) / apply_sw(vol,mu,m,s,r): r = (m + i mu gamma5) s
// on the first vol sites, m[2*vol] packed Pauli matrices, s and r spinors in
// the reference's array-of-structures order (pauli_dble.c:1840, pauli.c:1107).
template <typename R>
__global__ void k_apply_sw_aos(int vol, R mu, const R *__restrict__ m, const R *__restrict__ s, R *r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= vol) return;
  for (int half = 0; half < 2; half++) {
    R u[36];
    cpx<R> w[6], o[6];
    const R *mp = m + ((size_t)2 * i + half) * 36;
    for (int k = 0; k < 36; k++) u[k] = mp[k];
    const R *sp = s + (size_t)i * 24 + 12 * half;
    for (int k = 0; k < 6; k++) w[k] = mk<R>(sp[2 * k], sp[2 * k + 1]);
    mul_pauli<R>(half == 0 ? mu : -mu, u, w, o);
    R *rp = r + (size_t)i * 24 + 12 * half;
    for (int k = 0; k < 6; k++) { rp[2 * k] = o[k].re; rp[2 * k + 1] = o[k].im; }
  }
}

int apply_sw_ref_layout(int prec, int vol, double mu, const void *m, const void *s, void *r, cudaStream_t st) {
  int t = 128;
  if (prec == 64)
    k_apply_sw_aos<double><<<(vol + t - 1) / t, t, 0, st>>>(vol, mu, (const double *)m, (const double *)s, (double *)r);
  else
    k_apply_sw_aos<float><<<(vol + t - 1) / t, t, 0, st>>>(vol, (float)mu, (const float *)m, (const float *)s, (float *)r);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("apply_sw: launch failed");
}

// apply_swinv_dble (pauli_dble.c:1860): r = (m + i mu gamma5)^-1 s with the
// matrices inverted on the fly; the full (not Hermitian-part) inverse is
// applied, as the reference's apply_aa does.
__device__ int inv_apply(double mu, const double u[36], const cpx<double> w[6], cpx<double> o[6]) {
  // Solve (m + i mu) o = w by Gaussian elimination with partial pivoting.
  double ar[36], ai[36], xr[6], xi[6], fn = 0.0;
  int k = 6;
  for (int i = 0; i < 6; i++) {
    ar[7 * i] = u[i]; ai[7 * i] = mu;
    fn += u[i] * u[i] + mu * mu;
    for (int j = i + 1; j < 6; j++) {
      ar[6 * i + j] = u[k]; ai[6 * i + j] = u[k + 1];
      ar[6 * j + i] = u[k]; ai[6 * j + i] = -u[k + 1];
      fn += 2.0 * (u[k] * u[k] + u[k + 1] * u[k + 1]);
      k += 2;
    }
    xr[i] = w[i].re; xi[i] = w[i].im;
  }
  double out[36];
  int ifail = inv_pauli(mu, u, out);   // safety flag by the same criterion
  for (int c = 0; c < 6; c++) {
    int piv = c;
    double best = ar[7 * c] * ar[7 * c] + ai[7 * c] * ai[7 * c];
    for (int r = c + 1; r < 6; r++) {
      double v = ar[6 * r + c] * ar[6 * r + c] + ai[6 * r + c] * ai[6 * r + c];
      if (v > best) { best = v; piv = r; }
    }
    if (piv != c) {
      for (int j = 0; j < 6; j++) {
        double t = ar[6 * c + j]; ar[6 * c + j] = ar[6 * piv + j]; ar[6 * piv + j] = t;
        t = ai[6 * c + j]; ai[6 * c + j] = ai[6 * piv + j]; ai[6 * piv + j] = t;
      }
      double t = xr[c]; xr[c] = xr[piv]; xr[piv] = t;
      t = xi[c]; xi[c] = xi[piv]; xi[piv] = t;
    }
    double pr = ar[7 * c], pi = ai[7 * c], d = pr * pr + pi * pi;
    if (d == 0.0) d = 1.0;
    double qr = pr / d, qi = -pi / d;
    for (int r = c + 1; r < 6; r++) {
      double fr0 = ar[6 * r + c], fi0 = ai[6 * r + c];
      double fr = fr0 * qr - fi0 * qi, fi = fr0 * qi + fi0 * qr;
      for (int j = c; j < 6; j++) {
        ar[6 * r + j] -= fr * ar[6 * c + j] - fi * ai[6 * c + j];
        ai[6 * r + j] -= fr * ai[6 * c + j] + fi * ar[6 * c + j];
      }
      xr[r] -= fr * xr[c] - fi * xi[c];
      xi[r] -= fr * xi[c] + fi * xr[c];
    }
  }
  for (int c = 5; c >= 0; c--) {
    double sr = xr[c], si = xi[c];
    for (int j = c + 1; j < 6; j++) {
      sr -= ar[6 * c + j] * xr[j] - ai[6 * c + j] * xi[j];
      si -= ar[6 * c + j] * xi[j] + ai[6 * c + j] * xr[j];
    }
    double pr = ar[7 * c], pi = ai[7 * c], d = pr * pr + pi * pi;
    if (d == 0.0) d = 1.0;
    xr[c] = (sr * pr + si * pi) / d;
    xi[c] = (si * pr - sr * pi) / d;
  }
  for (int i = 0; i < 6; i++) o[i] = mk<double>(xr[i], xi[i]);
  return ifail;
}

__global__ void k_apply_swinv_aos(int vol, double mu, const double *__restrict__ m, const double *__restrict__ s,
                                  double *r, int *fail) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= vol) return;
  int bad = 0;
  for (int half = 0; half < 2; half++) {
    double u[36];
    cpx<double> w[6], o[6];
    const double *mp = m + ((size_t)2 * i + half) * 36;
    for (int k = 0; k < 36; k++) u[k] = mp[k];
    const double *sp = s + (size_t)i * 24 + 12 * half;
    for (int k = 0; k < 6; k++) w[k] = mk<double>(sp[2 * k], sp[2 * k + 1]);
    bad |= inv_apply(half == 0 ? mu : -mu, u, w, o);
    double *rp = r + (size_t)i * 24 + 12 * half;
    for (int k = 0; k < 6; k++) { rp[2 * k] = o[k].re; rp[2 * k + 1] = o[k].im; }
  }
  if (bad) atomicOr(fail, 1);
}

int apply_swinv_ref_layout(int vol, double mu, const void *m, const void *s, void *r, int *d_fail,
                           cudaStream_t st) {
  int t = 64;
  k_apply_swinv_aos<<<(vol + t - 1) / t, t, 0, st>>>(vol, mu, (const double *)m, (const double *)s, (double *)r,
                                                    d_fail);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("apply_swinv_dble: launch failed");
}

}  // namespace qcd
