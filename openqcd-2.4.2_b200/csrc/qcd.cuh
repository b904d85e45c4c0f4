// Device-side types, field layout and lattice arithmetic shared by all kernels.
//
// Field layout in HBM ("block-major, parity-split, structure of arrays"):
//   The lattice L0 x L1 x L2 x L3 (x0 = time, x3 fastest, as the reference's
//   ipt[] convention in main/README.global) is tiled by blocks b0 x b1 x b2 x b3,
//   the SAP block size.  A "chunk" is one parity half of one block; chunks are
//   numbered  chunk = p * nbl + blk  with p the site parity (0 even) and blk
//   the lexicographic block index (n3 fastest).  Inside a chunk the vbh = vb/2
//   sites of that parity are numbered s = l/2, l the lexicographic position
//   in the block.  Every field stores its components as separate planes of
//   vbh consecutive sites inside each chunk, so a warp reading one component
//   of 32 consecutive sites issues one 512-byte (FP64) or 256-byte (FP32)
//   coalesced request, and each chunk of a field is one contiguous byte range.
//
//   spinor FP64 : 12 complex  -> double2 plane k   at ((chunk*12+k)*vbh + s)
//   spinor FP32 : 12 complex  -> float4  plane j   at ((chunk*6 +j)*vbh + s)
//   link   FP64 : U(x,mu)     -> double2 plane k   at (((chunk*4+mu)*9+k)*vbh + s)
//   link   FP32 : U(x,mu)     -> float2  plane k   at (((chunk*4+mu)*9+k)*vbh + s)
//   pauli  FP64 : 2 x 36 real -> double2 plane k   at ((chunk*36+k)*vbh + s)
//   pauli  FP32 : 2 x 36 real -> float4  plane j   at ((chunk*18+j)*vbh + s)
//
// Only forward links U(x,mu) are stored, at the site x; the backward link of x
// in direction mu is the forward link of x - mu.  This turns the reference's
// scatter over even sites (modules/dirac/Dw_dble.c:1244 deo) into a pure
// gather, so no kernel needs atomics.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qcd {

template <typename R> struct cpx { R re, im; };
template <typename R> struct vec3 { cpx<R> c[3]; };
template <typename R> struct spinor { vec3<R> c[4]; };   // c[0..3] = c1..c4
template <typename R> struct su3 { cpx<R> e[9]; };      // row major c11..c33

struct Geom {
  int L[4], bs[4], nb[4];
  int vol, volh, nbl, vb, vbh;
  int lstr[4], bstr[4];
  const int *bcoord;   // [nbl]    packed n0 | n1<<8 | n2<<16 | n3<<24
  const int *lcoord;   // [2*vbh]  packed y0 | y1<<8 | y2<<16 | y3<<24 for (p, s)
};

// Domain decomposition along x0 (dd.cu): the local lattice starts at global
// time x0off of a global extent N0 (x0off = 0, N0 = L[0] on one rank).  The
// kernels built for it hop across the local x0-faces with the half-spinor
// faces hup (neighbour at x0 + 1, for the forward hop at the last local
// plane) and hdn (neighbour at x0 - 1, for the backward hop at the first
// plane) instead of wrapping around.  Kept apart from Geom, which every
// kernel takes: a larger Geom made the compiler spill in the FP32 operator.
struct DDGeom {
  int x0off, N0;
  const void *hup, *hdn;
};

// Sites of one x0-face: F = L1 L2 L3.  Face index of a site (its spatial
// coordinates): parity q of y1 + y2 + y3, then the block (n1, n2, n3)
// lexicographically, then half the in-block spatial index
// (y1 bs2 + y2) bs3 + y3, so that consecutive sites of a chunk on the face
// have consecutive face indices.
__device__ __forceinline__ int face_sites(const Geom &g) { return g.L[1] * g.L[2] * g.L[3]; }
__device__ __forceinline__ int face_index_of(const Geom &g, const int n[4], const int y[4]) {
  const int vb3h = g.bs[1] * g.bs[2] * g.bs[3] / 2;
  const int q = (y[1] + y[2] + y[3]) & 1;
  const int b3 = (n[1] * g.nb[2] + n[2]) * g.nb[3] + n[3];
  const int l3 = (y[1] * g.bs[2] + y[2]) * g.bs[3] + y[3];
  return (q * (g.nb[1] * g.nb[2] * g.nb[3]) + b3) * vb3h + (l3 >> 1);
}
// the site of face index f on the local plane x0 = 0 (side 0) or
// x0 = L0 - 1 (side 1): chunk and in-chunk index
__device__ __forceinline__ void face_site(const Geom &g, int side, int f, int &chunk, int &s, int n[4], int y[4]) {
  const int vb3h = g.bs[1] * g.bs[2] * g.bs[3] / 2;
  const int nb3 = g.nb[1] * g.nb[2] * g.nb[3];
  const int s3 = f % vb3h, qb = f / vb3h;
  const int q = qb / nb3, b3 = qb - q * nb3;
  n[3] = b3 % g.nb[3];
  n[2] = (b3 / g.nb[3]) % g.nb[2];
  n[1] = b3 / (g.nb[3] * g.nb[2]);
  n[0] = side ? g.nb[0] - 1 : 0;
  const int hb3 = g.bs[3] / 2;
  const int t = s3 / hb3;
  y[2] = t % g.bs[2];
  y[1] = t / g.bs[2];
  y[3] = 2 * (s3 - t * hb3) + ((q + y[1] + y[2]) & 1);
  y[0] = side ? g.bs[0] - 1 : 0;
  const int blk = ((n[0] * g.nb[1] + n[1]) * g.nb[2] + n[2]) * g.nb[3] + n[3];
  const int l = y[0] * g.lstr[0] + y[1] * g.lstr[1] + y[2] * g.lstr[2] + y[3];
  const int p = (y[0] + y[1] + y[2] + y[3]) & 1;
  chunk = p * g.nbl + blk;
  s = l >> 1;
}

__device__ __forceinline__ void unpack4(int v, int a[4]) {
  a[0] = v & 255; a[1] = (v >> 8) & 255; a[2] = (v >> 16) & 255; a[3] = (v >> 24) & 255;
}

// Position of a site: chunk and in-chunk index, plus what the neighbour
// arithmetic needs.
struct Site {
  int p, blk, s, l, lb;
  int y[4], n[4];
};

__device__ __forceinline__ void site_decode(const Geom &g, int p, int blk, int s, Site &x) {
  x.p = p; x.blk = blk; x.s = s;
  unpack4(__ldg(g.lcoord + p * g.vbh + s), x.y);
  unpack4(__ldg(g.bcoord + blk), x.n);
  x.l = x.y[0] * g.lstr[0] + x.y[1] * g.lstr[1] + x.y[2] * g.lstr[2] + x.y[3] * g.lstr[3];
  x.lb = blk;
}

// chunk and in-chunk index of x + dir*mu (dir = +1 or -1), periodic.
__device__ __forceinline__ void site_nbr(const Geom &g, const Site &x, int mu, int dir,
                                         int &chunk, int &s) {
  int l = x.l, blk = x.blk;
  if (dir > 0) {
    if (x.y[mu] + 1 < g.bs[mu]) l += g.lstr[mu];
    else {
      l -= (g.bs[mu] - 1) * g.lstr[mu];
      blk += (x.n[mu] + 1 < g.nb[mu]) ? g.bstr[mu] : -(g.nb[mu] - 1) * g.bstr[mu];
    }
  } else {
    if (x.y[mu] > 0) l -= g.lstr[mu];
    else {
      l += (g.bs[mu] - 1) * g.lstr[mu];
      blk += (x.n[mu] > 0) ? -g.bstr[mu] : (g.nb[mu] - 1) * g.bstr[mu];
    }
  }
  chunk = (1 - x.p) * g.nbl + blk;
  s = l >> 1;
}

// True if x + dir*mu lies outside the block of x.
__device__ __forceinline__ bool crosses_block(const Geom &g, const Site &x, int mu, int dir) {
  return dir > 0 ? (x.y[mu] + 1 == g.bs[mu]) : (x.y[mu] == 0);
}

// ---------------------------------------------------------------- complex ops
template <typename R> __device__ __forceinline__ cpx<R> mk(R a, R b) { cpx<R> z; z.re = a; z.im = b; return z; }

template <typename R> __device__ __forceinline__ void vzero(vec3<R> &v) {
#pragma unroll
  for (int i = 0; i < 3; i++) v.c[i] = mk<R>(0, 0);
}
template <typename R> __device__ __forceinline__ void szero(spinor<R> &v) {
#pragma unroll
  for (int a = 0; a < 4; a++) vzero(v.c[a]);
}

// r = a + b, a - b, a + i b, a - i b
template <typename R> __device__ __forceinline__ vec3<R> vadd(const vec3<R> &a, const vec3<R> &b) {
  vec3<R> r;
#pragma unroll
  for (int i = 0; i < 3; i++) r.c[i] = mk<R>(a.c[i].re + b.c[i].re, a.c[i].im + b.c[i].im);
  return r;
}
template <typename R> __device__ __forceinline__ vec3<R> vsub(const vec3<R> &a, const vec3<R> &b) {
  vec3<R> r;
#pragma unroll
  for (int i = 0; i < 3; i++) r.c[i] = mk<R>(a.c[i].re - b.c[i].re, a.c[i].im - b.c[i].im);
  return r;
}
template <typename R> __device__ __forceinline__ vec3<R> viadd(const vec3<R> &a, const vec3<R> &b) {
  vec3<R> r;
#pragma unroll
  for (int i = 0; i < 3; i++) r.c[i] = mk<R>(a.c[i].re - b.c[i].im, a.c[i].im + b.c[i].re);
  return r;
}
template <typename R> __device__ __forceinline__ vec3<R> visub(const vec3<R> &a, const vec3<R> &b) {
  vec3<R> r;
#pragma unroll
  for (int i = 0; i < 3; i++) r.c[i] = mk<R>(a.c[i].re + b.c[i].im, a.c[i].im - b.c[i].re);
  return r;
}
// r += a, r -= a, r += i a, r -= i a
template <typename R> __device__ __forceinline__ void vacc(vec3<R> &r, const vec3<R> &a) {
#pragma unroll
  for (int i = 0; i < 3; i++) { r.c[i].re += a.c[i].re; r.c[i].im += a.c[i].im; }
}
template <typename R> __device__ __forceinline__ void vdec(vec3<R> &r, const vec3<R> &a) {
#pragma unroll
  for (int i = 0; i < 3; i++) { r.c[i].re -= a.c[i].re; r.c[i].im -= a.c[i].im; }
}
template <typename R> __device__ __forceinline__ void viacc(vec3<R> &r, const vec3<R> &a) {
#pragma unroll
  for (int i = 0; i < 3; i++) { r.c[i].re -= a.c[i].im; r.c[i].im += a.c[i].re; }
}
template <typename R> __device__ __forceinline__ void videc(vec3<R> &r, const vec3<R> &a) {
#pragma unroll
  for (int i = 0; i < 3; i++) { r.c[i].re += a.c[i].im; r.c[i].im -= a.c[i].re; }
}

// U * v and U^dag * v
template <typename R> __device__ __forceinline__ vec3<R> umul(const su3<R> &u, const vec3<R> &v) {
  vec3<R> r;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    R re = 0, im = 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const cpx<R> a = u.e[3 * i + j];
      re += a.re * v.c[j].re - a.im * v.c[j].im;
      im += a.re * v.c[j].im + a.im * v.c[j].re;
    }
    r.c[i] = mk<R>(re, im);
  }
  return r;
}
template <typename R> __device__ __forceinline__ vec3<R> udagmul(const su3<R> &u, const vec3<R> &v) {
  vec3<R> r;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    R re = 0, im = 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const cpx<R> a = u.e[3 * j + i];
      re += a.re * v.c[j].re + a.im * v.c[j].im;
      im += a.re * v.c[j].im - a.im * v.c[j].re;
    }
    r.c[i] = mk<R>(re, im);
  }
  return r;
}

// ------------------------------------------------------------ field accessors
template <typename R> struct Store;

template <> struct Store<double> {
  __device__ __forceinline__ static spinor<double> load_spinor(const void *base, int chunk, int s, int vbh) {
    const double2 *p = (const double2 *)base + (size_t)chunk * 12 * vbh + s;
    spinor<double> r;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 v = __ldg(p + (size_t)k * vbh);
      r.c[k / 3].c[k % 3] = mk<double>(v.x, v.y);
    }
    return r;
  }
  __device__ __forceinline__ static void store_spinor(void *base, int chunk, int s, int vbh, const spinor<double> &r) {
    double2 *p = (double2 *)base + (size_t)chunk * 12 * vbh + s;
#pragma unroll
    for (int k = 0; k < 12; k++) p[(size_t)k * vbh] = make_double2(r.c[k / 3].c[k % 3].re, r.c[k / 3].c[k % 3].im);
  }
  // plain (non-__ldg) load for fields written by the same kernel launch
  __device__ __forceinline__ static spinor<double> load_spinor_rw(const void *base, int chunk, int s, int vbh) {
    const double2 *p = (const double2 *)base + (size_t)chunk * 12 * vbh + s;
    spinor<double> r;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 v = p[(size_t)k * vbh];
      r.c[k / 3].c[k % 3] = mk<double>(v.x, v.y);
    }
    return r;
  }
  __device__ __forceinline__ static su3<double> load_link(const void *base, int chunk, int mu, int s, int vbh) {
    const double2 *p = (const double2 *)base + ((size_t)chunk * 4 + mu) * 9 * vbh + s;
    su3<double> u;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 v = __ldg(p + (size_t)k * vbh);
      u.e[k] = mk<double>(v.x, v.y);
    }
    return u;
  }
  // half = 0 upper, 1 lower: 36 reals
  __device__ __forceinline__ static void load_pauli(const void *base, int chunk, int half, int s, int vbh, double u[36]) {
    const double2 *p = (const double2 *)base + ((size_t)chunk * 36 + 18 * half) * vbh + s;
#pragma unroll
    for (int k = 0; k < 18; k++) {
      double2 v = __ldg(p + (size_t)k * vbh);
      u[2 * k] = v.x; u[2 * k + 1] = v.y;
    }
  }
};

template <> struct Store<float> {
  __device__ __forceinline__ static spinor<float> load_spinor(const void *base, int chunk, int s, int vbh) {
    const float4 *p = (const float4 *)base + (size_t)chunk * 6 * vbh + s;
    spinor<float> r;
#pragma unroll
    for (int j = 0; j < 6; j++) {
      float4 v = __ldg(p + (size_t)j * vbh);
      int k = 2 * j;
      r.c[k / 3].c[k % 3] = mk<float>(v.x, v.y);
      r.c[(k + 1) / 3].c[(k + 1) % 3] = mk<float>(v.z, v.w);
    }
    return r;
  }
  __device__ __forceinline__ static spinor<float> load_spinor_rw(const void *base, int chunk, int s, int vbh) {
    const float4 *p = (const float4 *)base + (size_t)chunk * 6 * vbh + s;
    spinor<float> r;
#pragma unroll
    for (int j = 0; j < 6; j++) {
      float4 v = p[(size_t)j * vbh];
      int k = 2 * j;
      r.c[k / 3].c[k % 3] = mk<float>(v.x, v.y);
      r.c[(k + 1) / 3].c[(k + 1) % 3] = mk<float>(v.z, v.w);
    }
    return r;
  }
  __device__ __forceinline__ static void store_spinor(void *base, int chunk, int s, int vbh, const spinor<float> &r) {
    float4 *p = (float4 *)base + (size_t)chunk * 6 * vbh + s;
#pragma unroll
    for (int j = 0; j < 6; j++) {
      int k = 2 * j;
      p[(size_t)j * vbh] = make_float4(r.c[k / 3].c[k % 3].re, r.c[k / 3].c[k % 3].im,
                                       r.c[(k + 1) / 3].c[(k + 1) % 3].re, r.c[(k + 1) / 3].c[(k + 1) % 3].im);
    }
  }
  __device__ __forceinline__ static su3<float> load_link(const void *base, int chunk, int mu, int s, int vbh) {
    const float2 *p = (const float2 *)base + ((size_t)chunk * 4 + mu) * 9 * vbh + s;
    su3<float> u;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float2 v = __ldg(p + (size_t)k * vbh);
      u.e[k] = mk<float>(v.x, v.y);
    }
    return u;
  }
  __device__ __forceinline__ static void load_pauli(const void *base, int chunk, int half, int s, int vbh, float u[36]) {
    const float4 *p = (const float4 *)base + ((size_t)chunk * 18 + 9 * half) * vbh + s;
#pragma unroll
    for (int j = 0; j < 9; j++) {
      float4 v = __ldg(p + (size_t)j * vbh);
      u[4 * j] = v.x; u[4 * j + 1] = v.y; u[4 * j + 2] = v.z; u[4 * j + 3] = v.w;
    }
  }
};

// FP32 link stored as its first two rows (12 reals, planes
// ((chunk*4 + mu)*6 + k)*vbh + s); the third row is rebuilt as the complex
// conjugate of the cross product of the first two, exact for SU(3), and
// negated for a link that carries the antiperiodic time-boundary sign
// (neg).  The library checks every link for this relation, with the sign
// its position implies, before it reads 12-real links.
__device__ __forceinline__ su3<float> load_link12(const void *base, int chunk, int mu, int s, int vbh, bool neg) {
  const float2 *p = (const float2 *)base + ((size_t)chunk * 4 + mu) * 6 * vbh + s;
  su3<float> r;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const float2 v = __ldg(p + (size_t)k * vbh);
    r.e[k] = mk<float>(v.x, v.y);
  }
  const float sg = neg ? -1.0f : 1.0f;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int a = (j + 1) % 3, b = (j + 2) % 3;
    const cpx<float> x1 = r.e[a], y2 = r.e[3 + b], x2 = r.e[b], y1 = r.e[3 + a];
    const float re = x1.re * y2.re - x1.im * y2.im - (x2.re * y1.re - x2.im * y1.im);
    const float im = x1.re * y2.im + x1.im * y2.re - (x2.re * y1.im + x2.im * y1.re);
    r.e[6 + j] = mk<float>(sg * re, -sg * im);
  }
  return r;
}

// ---------------------------------------------------------------- Pauli 6x6
// The Hermitian 6x6 matrix is packed as in the reference
// (modules/sw_term/pauli_dble.c:1336-1442 and set_aa :1644-1675): u[0..5] the
// real diagonal, u[6..35] the 15 complex entries above the diagonal row by
// row, (0,1),(0,2),..,(0,5),(1,2),..,(4,5).  r = (A + i mu) w.
template <typename R>
__device__ __forceinline__ void mul_pauli(R mu, const R u[36], const cpx<R> w[6], cpx<R> r[6]) {
#pragma unroll
  for (int i = 0; i < 6; i++) r[i] = mk<R>(u[i] * w[i].re - mu * w[i].im, u[i] * w[i].im + mu * w[i].re);
  int k = 6;
#pragma unroll
  for (int i = 0; i < 6; i++) {
#pragma unroll
    for (int j = i + 1; j < 6; j++) {
      const R are = u[k], aim = u[k + 1];
      k += 2;
      r[i].re += are * w[j].re - aim * w[j].im;
      r[i].im += are * w[j].im + aim * w[j].re;
      r[j].re += are * w[i].re + aim * w[i].im;
      r[j].im += are * w[i].im - aim * w[i].re;
    }
  }
}

// Weyl halves of a spinor as 6 complex numbers: upper (c1,c2), lower (c3,c4)
template <typename R> __device__ __forceinline__ void weyl_get(const spinor<R> &s, int half, cpx<R> w[6]) {
#pragma unroll
  for (int i = 0; i < 3; i++) { w[i] = s.c[2 * half].c[i]; w[3 + i] = s.c[2 * half + 1].c[i]; }
}
template <typename R> __device__ __forceinline__ void weyl_put(spinor<R> &s, int half, const cpx<R> w[6]) {
#pragma unroll
  for (int i = 0; i < 3; i++) { s.c[2 * half].c[i] = w[i]; s.c[2 * half + 1].c[i] = w[3 + i]; }
}

// r = (A_upper + i mu) s_upper  (+)  (A_lower - i mu) s_lower, the site-local
// SW term with twisted mass i mu gamma5 (pauli_dble.c:1840 apply_sw_dble).
template <typename R>
__device__ __forceinline__ spinor<R> apply_sw_site(const void *sw, int chunk, int s, int vbh, R mu,
                                                   const spinor<R> &in) {
  spinor<R> out;
  R u[36];
  cpx<R> w[6], r[6];
#pragma unroll
  for (int half = 0; half < 2; half++) {
    Store<R>::load_pauli(sw, chunk, half, s, vbh, u);
    weyl_get(in, half, w);
    mul_pauli<R>(half == 0 ? mu : -mu, u, w, r);
    weyl_put(out, half, r);
  }
  return out;
}

// ----------------------------------------------------------- hopping term
// Contribution of one direction to H s(x) = sum_mu [ U(x,mu)(1-g_mu) s(x+mu)
// + U(x-mu,mu)^dag (1+g_mu) s(x-mu) ], restated from the projector structure of
// the reference's doe() (modules/dirac/Dw_dble.c:1114-1242) in the chiral
// basis.  The caller multiplies the sum by the coefficient (-1/2).
template <typename R>
__device__ __forceinline__ void hop_fwd(int mu, const su3<R> &u, const spinor<R> &sp, spinor<R> &acc) {
  vec3<R> h, c;
  switch (mu) {
    case 0:
      h = vadd(sp.c[0], sp.c[2]); c = umul(u, h); vacc(acc.c[0], c); vacc(acc.c[2], c);
      h = vadd(sp.c[1], sp.c[3]); c = umul(u, h); vacc(acc.c[1], c); vacc(acc.c[3], c);
      break;
    case 1:
      h = viadd(sp.c[0], sp.c[3]); c = umul(u, h); vacc(acc.c[0], c); videc(acc.c[3], c);
      h = viadd(sp.c[1], sp.c[2]); c = umul(u, h); vacc(acc.c[1], c); videc(acc.c[2], c);
      break;
    case 2:
      h = vadd(sp.c[0], sp.c[3]); c = umul(u, h); vacc(acc.c[0], c); vacc(acc.c[3], c);
      h = vsub(sp.c[1], sp.c[2]); c = umul(u, h); vacc(acc.c[1], c); vdec(acc.c[2], c);
      break;
    default:
      h = viadd(sp.c[0], sp.c[2]); c = umul(u, h); vacc(acc.c[0], c); videc(acc.c[2], c);
      h = visub(sp.c[1], sp.c[3]); c = umul(u, h); vacc(acc.c[1], c); viacc(acc.c[3], c);
      break;
  }
}

template <typename R>
__device__ __forceinline__ void hop_bwd(int mu, const su3<R> &u, const spinor<R> &sm, spinor<R> &acc) {
  vec3<R> h, c;
  switch (mu) {
    case 0:
      h = vsub(sm.c[0], sm.c[2]); c = udagmul(u, h); vacc(acc.c[0], c); vdec(acc.c[2], c);
      h = vsub(sm.c[1], sm.c[3]); c = udagmul(u, h); vacc(acc.c[1], c); vdec(acc.c[3], c);
      break;
    case 1:
      h = visub(sm.c[0], sm.c[3]); c = udagmul(u, h); vacc(acc.c[0], c); viacc(acc.c[3], c);
      h = visub(sm.c[1], sm.c[2]); c = udagmul(u, h); vacc(acc.c[1], c); viacc(acc.c[2], c);
      break;
    case 2:
      h = vsub(sm.c[0], sm.c[3]); c = udagmul(u, h); vacc(acc.c[0], c); vdec(acc.c[3], c);
      h = vadd(sm.c[1], sm.c[2]); c = udagmul(u, h); vacc(acc.c[1], c); vacc(acc.c[2], c);
      break;
    default:
      h = visub(sm.c[0], sm.c[2]); c = udagmul(u, h); vacc(acc.c[0], c); viacc(acc.c[2], c);
      h = viadd(sm.c[1], sm.c[3]); c = udagmul(u, h); vacc(acc.c[1], c); videc(acc.c[3], c);
      break;
  }
}

// ------------------------------------------------- half-spinor x0-faces
// Planes of F face sites: FP64 as 6 double2 planes, FP32 as 3 float4 planes
// (two complex components each); h0 = components 0..2, h1 = 3..5.
template <typename R> struct Half;
template <> struct Half<double> {
  __device__ __forceinline__ static void load(const void *b, int F, int f, vec3<double> &h0, vec3<double> &h1) {
    const double2 *p = (const double2 *)b + f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double2 a = __ldg(p + (size_t)k * F), c = __ldg(p + (size_t)(k + 3) * F);
      h0.c[k] = mk<double>(a.x, a.y);
      h1.c[k] = mk<double>(c.x, c.y);
    }
  }
  __device__ __forceinline__ static void store(void *b, int F, int f, const vec3<double> &h0, const vec3<double> &h1) {
    double2 *p = (double2 *)b + f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      p[(size_t)k * F] = make_double2(h0.c[k].re, h0.c[k].im);
      p[(size_t)(k + 3) * F] = make_double2(h1.c[k].re, h1.c[k].im);
    }
  }
};
template <> struct Half<float> {
  __device__ __forceinline__ static void load(const void *b, int F, int f, vec3<float> &h0, vec3<float> &h1) {
    const float4 *p = (const float4 *)b + f;
    const float4 a = __ldg(p), c = __ldg(p + F), d = __ldg(p + 2 * (size_t)F);
    h0.c[0] = mk<float>(a.x, a.y); h0.c[1] = mk<float>(a.z, a.w); h0.c[2] = mk<float>(c.x, c.y);
    h1.c[0] = mk<float>(c.z, c.w); h1.c[1] = mk<float>(d.x, d.y); h1.c[2] = mk<float>(d.z, d.w);
  }
  __device__ __forceinline__ static void store(void *b, int F, int f, const vec3<float> &h0, const vec3<float> &h1) {
    float4 *p = (float4 *)b + f;
    p[0] = make_float4(h0.c[0].re, h0.c[0].im, h0.c[1].re, h0.c[1].im);
    p[F] = make_float4(h0.c[2].re, h0.c[2].im, h1.c[0].re, h1.c[0].im);
    p[2 * (size_t)F] = make_float4(h1.c[1].re, h1.c[1].im, h1.c[2].re, h1.c[2].im);
  }
};

// The x0 hops across a rank boundary, split where the two ranks meet.  The
// forward hop U(x,0)(1 - g0) s(x+0) needs the neighbour's projection
// h = (s1 + s3, s2 + s4) (the same sums hop_fwd forms); the backward hop
// U(x-0,0)^dag (1 + g0) s(x-0) needs c = U^dag (s1 - s3, s2 - s4), which the
// rank holding the link forms.  Same operations in the same order as
// hop_fwd / hop_bwd with mu = 0, so the results are bit-identical.
template <typename R>
__device__ __forceinline__ void dd_proj_fwd(const spinor<R> &s, vec3<R> &h0, vec3<R> &h1) {
  h0 = vadd(s.c[0], s.c[2]);
  h1 = vadd(s.c[1], s.c[3]);
}
template <typename R>
__device__ __forceinline__ void dd_proj_bwd(const su3<R> &u, const spinor<R> &s, vec3<R> &c0, vec3<R> &c1) {
  c0 = udagmul(u, vsub(s.c[0], s.c[2]));
  c1 = udagmul(u, vsub(s.c[1], s.c[3]));
}
template <typename R>
__device__ __forceinline__ void dd_hop_fwd(const su3<R> &u, const vec3<R> &h0, const vec3<R> &h1, spinor<R> &acc) {
  vec3<R> c = umul(u, h0);
  vacc(acc.c[0], c); vacc(acc.c[2], c);
  c = umul(u, h1);
  vacc(acc.c[1], c); vacc(acc.c[3], c);
}
template <typename R>
__device__ __forceinline__ void dd_hop_bwd(const vec3<R> &c0, const vec3<R> &c1, spinor<R> &acc) {
  vacc(acc.c[0], c0); vdec(acc.c[2], c0);
  vacc(acc.c[1], c1); vdec(acc.c[3], c1);
}

template <typename R> __device__ __forceinline__ void sscale(spinor<R> &s, R c) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int i = 0; i < 3; i++) { s.c[a].c[i].re *= c; s.c[a].c[i].im *= c; }
}
template <typename R> __device__ __forceinline__ void sadd(spinor<R> &r, const spinor<R> &a) {
#pragma unroll
  for (int k = 0; k < 4; k++) vacc(r.c[k], a.c[k]);
}
template <typename R> __device__ __forceinline__ void ssub(spinor<R> &r, const spinor<R> &a) {
#pragma unroll
  for (int k = 0; k < 4; k++) vdec(r.c[k], a.c[k]);
}

}  // namespace qcd
