// Synthetic field generation on the device: gauge links U = exp(eps X) and
// Gaussian spinor sources, from a counter-based generator so every element
// depends only on (seed, element index) and the result does not depend on the
// launch shape.
//
// Generator: Philox-4x32 with 10 rounds (J. Salmon et al., "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), written from the published round
// function and constants.
#include "lib.h"

namespace qcd {

struct P4 { uint32_t x, y, z, w; };

__device__ __forceinline__ P4 philox(P4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    P4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// uniform in (0,1] with 53 random bits
__device__ __forceinline__ double u01(uint32_t a, uint32_t b) {
  uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)b;
  v &= ((1ull << 53) - 1);
  return ((double)v + 1.0) * (1.0 / 9007199254740992.0);
}

// Two normal deviates with variance 1/2 each (Box-Muller without the factor 2,
// the normalisation of the reference's gauss_dble, modules/random/gauss.c).
__device__ __forceinline__ void gauss2(P4 r, double &g0, double &g1) {
  double a = u01(r.x, r.y), b = u01(r.z, r.w);
  double rho = sqrt(-log(a));
  double sn, cs;
  sincospi(2.0 * b - 1.0, &sn, &cs);
  g0 = rho * sn;
  g1 = rho * cs;
}

// 3x3 complex matrices as 18 doubles, row major
__device__ void m3mul(const double *a, const double *b, double *c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; k++) {
        re += a[2 * (3 * i + k)] * b[2 * (3 * k + j)] - a[2 * (3 * i + k) + 1] * b[2 * (3 * k + j) + 1];
        im += a[2 * (3 * i + k)] * b[2 * (3 * k + j) + 1] + a[2 * (3 * i + k) + 1] * b[2 * (3 * k + j)];
      }
      c[2 * (3 * i + j)] = re;
      c[2 * (3 * i + j) + 1] = im;
    }
}

// exp(M) for an anti-Hermitian traceless M by scaling and squaring of the
// Taylor series, followed by projection onto SU(3) (row Gram-Schmidt, third
// row = conj(row1 x row2)).
__device__ void su3_exp(const double *M, double *U) {
  double nrm = 0;
  for (int i = 0; i < 18; i++) nrm += M[i] * M[i];
  nrm = sqrt(nrm);
  int k = 0;
  double sc = 1.0;
  while (nrm * sc > 0.25 && k < 30) { sc *= 0.5; k++; }
  double A[18], T[18], E[18], W[18];
  for (int i = 0; i < 18; i++) { A[i] = M[i] * sc; E[i] = 0; T[i] = 0; }
  for (int i = 0; i < 3; i++) { E[8 * i] = 1.0; T[8 * i] = 1.0; }
  for (int n = 1; n <= 12; n++) {
    m3mul(T, A, W);
    for (int i = 0; i < 18; i++) { T[i] = W[i] / n; E[i] += T[i]; }
  }
  for (int s = 0; s < k; s++) {
    m3mul(E, E, W);
    for (int i = 0; i < 18; i++) E[i] = W[i];
  }
  // project: normalise row 0, orthogonalise row 1, row 2 = conj(r0 x r1)
  double *r0 = E, *r1 = E + 6;
  double n0 = 0;
  for (int i = 0; i < 6; i++) n0 += r0[i] * r0[i];
  n0 = 1.0 / sqrt(n0);
  for (int i = 0; i < 6; i++) r0[i] *= n0;
  double pr = 0, pi = 0;   // (r0, r1) = sum conj(r0) r1
  for (int j = 0; j < 3; j++) {
    pr += r0[2 * j] * r1[2 * j] + r0[2 * j + 1] * r1[2 * j + 1];
    pi += r0[2 * j] * r1[2 * j + 1] - r0[2 * j + 1] * r1[2 * j];
  }
  for (int j = 0; j < 3; j++) {
    r1[2 * j] -= pr * r0[2 * j] - pi * r0[2 * j + 1];
    r1[2 * j + 1] -= pr * r0[2 * j + 1] + pi * r0[2 * j];
  }
  double n1 = 0;
  for (int i = 0; i < 6; i++) n1 += r1[i] * r1[i];
  n1 = 1.0 / sqrt(n1);
  for (int i = 0; i < 6; i++) r1[i] *= n1;
  for (int j = 0; j < 3; j++) {
    int a = (j + 1) % 3, b = (j + 2) % 3;
    // (r0 x r1)_j = r0_a r1_b - r0_b r1_a ; row2_j = conj of that
    double xr = r0[2 * a] * r1[2 * b] - r0[2 * a + 1] * r1[2 * b + 1] - (r0[2 * b] * r1[2 * a] - r0[2 * b + 1] * r1[2 * a + 1]);
    double xi = r0[2 * a] * r1[2 * b + 1] + r0[2 * a + 1] * r1[2 * b] - (r0[2 * b] * r1[2 * a + 1] + r0[2 * b + 1] * r1[2 * a]);
    E[12 + 2 * j] = xr;
    E[12 + 2 * j + 1] = -xi;
  }
  for (int i = 0; i < 18; i++) U[i] = E[i];
}

// One link per thread.  X is drawn with the distribution of the reference's
// random_alg (modules/linalg/liealg.c:41-65): with g_k normal of variance 1/2,
//   x1 = a g0 + b g1, x2 = a g1 + b g0, x3..x8 = g_k / sqrt(2),
//   a = (sqrt3+1)/6, b = (sqrt3-1)/6,
// and X_11 = i(x1+x2), X_22 = i(x2-2x1), X_33 = i(x1-2x2), X_12 = x3+i x4,
// X_13 = x5+i x6, X_23 = x7+i x8 (anti-Hermitian).  U = exp(eps X).  With
// antiperiodic fermion boundary conditions (type 3) the time links at
// x0 = L0-1 get the factor -1, as the reference's set_ud_phase does
// (modules/uflds/uflds.c:307-335), and with phase angles theta the spatial
// links U(x,k) get the factor exp(i theta[k-1]/N[k]) (uflds.c:249-300).
struct LinkPhase {
  double re[3], im[3];
  int on;
};

bool spatial_phases(const Ctx &c, double pr[3], double pi[3]) {
  bool on = false;
  for (int k = 0; k < 3; k++) {
    const double p = c.theta[k] / (double)c.g.L[k + 1];
    pr[k] = cos(p);
    pi[k] = sin(p);
    on |= p != 0.0;
  }
  return on;
}

__global__ void k_gen_links(Geom g, DDGeom dg, double2 *ud, double eps, uint32_t k0, uint32_t k1,
                            int antiperiodic, LinkPhase ph) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * g.vol) return;
  int d = i >> 2, mu = i & 3;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
  Site xs;
  site_decode(g, p, blk, s, xs);
  int x0 = dg.x0off + xs.n[0] * g.bs[0] + xs.y[0];     // global time coordinate
  // global counter: lexicographic index of the site in the global lattice,
  // so the field depends neither on the block size nor on the ranks
  uint32_t lex = (uint32_t)x0;
  for (int m = 1; m < 4; m++) lex = lex * g.L[m] + (xs.n[m] * g.bs[m] + xs.y[m]);
  double gg[8];
  for (int r = 0; r < 2; r++) {
    P4 c = {lex, (uint32_t)mu, (uint32_t)r, 0x4c494e4bu};
    P4 o = philox(c, k0, k1);
    gauss2(o, gg[4 * r], gg[4 * r + 1]);
    P4 o2 = philox({lex, (uint32_t)mu, (uint32_t)r, 0x4c494e4cu}, k0, k1);
    gauss2(o2, gg[4 * r + 2], gg[4 * r + 3]);
  }
  const double a = (sqrt(3.0) + 1.0) / 6.0, b = (sqrt(3.0) - 1.0) / 6.0, c = 0.5 * sqrt(2.0);
  double x1 = a * gg[0] + b * gg[1], x2 = a * gg[1] + b * gg[0];
  double x3 = c * gg[2], x4 = c * gg[3], x5 = c * gg[4], x6 = c * gg[5], x7 = c * gg[6], x8 = c * gg[7];
  double M[18] = {0};
  M[1] = eps * (x1 + x2);
  M[9] = eps * (x2 - 2 * x1);
  M[17] = eps * (x1 - 2 * x2);
  M[2] = eps * x3; M[3] = eps * x4;     // X_12
  M[4] = eps * x5; M[5] = eps * x6;     // X_13
  M[10] = eps * x7; M[11] = eps * x8;   // X_23
  M[6] = -M[2]; M[7] = M[3];            // X_21 = -conj(X_12)
  M[12] = -M[4]; M[13] = M[5];          // X_31
  M[14] = -M[10]; M[15] = M[11];        // X_32
  double U[18];
  su3_exp(M, U);
  double sg = (antiperiodic && mu == 0 && x0 == dg.N0 - 1) ? -1.0 : 1.0;
  double2 *dst = ud + ((size_t)chunk * 4 + mu) * 9 * g.vbh + s;
  if (ph.on && mu > 0) {
    const double pr = ph.re[mu - 1], pi = ph.im[mu - 1];
    for (int k = 0; k < 9; k++)
      dst[(size_t)k * g.vbh] = make_double2(U[2 * k] * pr - U[2 * k + 1] * pi, U[2 * k] * pi + U[2 * k + 1] * pr);
  } else {
    for (int k = 0; k < 9; k++) dst[(size_t)k * g.vbh] = make_double2(sg * U[2 * k], sg * U[2 * k + 1]);
  }
}

int gen_links(Ctx &c, double eps, uint64_t seed, cudaStream_t st) {
  size_t n = (size_t)c.g.vol * 36 * sizeof(double2);
  if (!c.ud && cudaMalloc(&c.ud, n) != cudaSuccess) return fail("out of device memory (gauge field)");
  int t = 128, m = 4 * c.g.vol;
  LinkPhase ph;
  ph.on = spatial_phases(c, ph.re, ph.im);
  k_gen_links<<<(m + t - 1) / t, t, 0, st>>>(c.g, c.ddg, c.ud, eps, (uint32_t)seed, (uint32_t)(seed >> 32), c.bc == 3,
                                              ph);
  if (cudaGetLastError() != cudaSuccess) return fail("gen_links: launch failed");
  c.have_ud = true;
  return links_refresh_f32(c, st);
}

// Gaussian spinor field: every real component normal with variance sigma^2/2.
template <typename R>
__global__ void k_gen_spinor(Geom g, DDGeom dg, void *dst, double sigma, uint32_t k0, uint32_t k1) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
  Site xs;
  site_decode(g, p, blk, s, xs);
  uint32_t lex = (uint32_t)(dg.x0off + xs.n[0] * g.bs[0] + xs.y[0]);
  for (int m = 1; m < 4; m++) lex = lex * g.L[m] + (xs.n[m] * g.bs[m] + xs.y[m]);
  spinor<R> v;
  for (int k = 0; k < 6; k++) {
    P4 o = philox({lex, (uint32_t)k, 0x53504e52u, 0u}, k0, k1);
    double a, b, c2, d2;
    gauss2(o, a, b);
    P4 o2 = philox({lex, (uint32_t)k, 0x53504e53u, 0u}, k0, k1);
    gauss2(o2, c2, d2);
    int q = 2 * k;
    v.c[q / 3].c[q % 3] = mk<R>((R)(sigma * a), (R)(sigma * b));
    v.c[(q + 1) / 3].c[(q + 1) % 3] = mk<R>((R)(sigma * c2), (R)(sigma * d2));
  }
  Store<R>::store_spinor(dst, chunk, s, g.vbh, v);
}

int gen_spinor(const Ctx &c, int prec, void *dev, double sigma, uint64_t seed, cudaStream_t st) {
  int t = 128;
  if (prec == 64)
    k_gen_spinor<double><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, c.ddg, dev, sigma, (uint32_t)seed, (uint32_t)(seed >> 32));
  else
    k_gen_spinor<float><<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, c.ddg, dev, sigma, (uint32_t)seed, (uint32_t)(seed >> 32));
  return cudaGetLastError() == cudaSuccess ? 0 : fail("gen_spinor: launch failed");
}

// Uniform random FP32 spinor field, every real component in [-0.5, 0.5)
// (the distribution of dfl_modes.c random_fields, :248-274).
__global__ void k_uniform_spinor(Geom g, float4 *dst, uint32_t k0, uint32_t k1) {
  int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= g.vol) return;
  int chunk = d / g.vbh, s = d - chunk * g.vbh;
  int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
  Site xs;
  site_decode(g, p, blk, s, xs);
  uint32_t lex = 0;
  for (int m = 0; m < 4; m++) lex = lex * g.L[m] + (xs.n[m] * g.bs[m] + xs.y[m]);
  spinor<float> v;
  for (int k = 0; k < 6; k++) {
    P4 o = philox({lex, (uint32_t)k, 0x554e4946u, 0u}, k0, k1);
    const float sc = 1.0f / 4294967296.0f;
    int q = 2 * k;
    v.c[q / 3].c[q % 3] = mk<float>(o.x * sc - 0.5f, o.y * sc - 0.5f);
    v.c[(q + 1) / 3].c[(q + 1) % 3] = mk<float>(o.z * sc - 0.5f, o.w * sc - 0.5f);
  }
  Store<float>::store_spinor(dst, chunk, s, g.vbh, v);
}

int gen_uniform_spinor32(const Ctx &c, void *dev, uint64_t seed, cudaStream_t st) {
  int t = 128;
  k_uniform_spinor<<<(c.g.vol + t - 1) / t, t, 0, st>>>(c.g, (float4 *)dev, (uint32_t)seed, (uint32_t)(seed >> 32));
  return cudaGetLastError() == cudaSuccess ? 0 : fail("uniform spinor: launch failed");
}

}  // namespace qcd
