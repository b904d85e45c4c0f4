// The reference's little solver, restated on the device: the flexible FP64
// GCR of modules/linsolv/fgcr4vd.c:339 on the even-odd preconditioned
// little system, preconditioned by the single-pass FP32 GCR of
// modules/linsolv/gcr4v.c:302, with the global-mode ("little-little")
// deflation of modules/little/ltl_modes.c and the driver of
// modules/dfl/ltl_gcr.c:155.  The scalar recursions run on the host as in
// the reference; every vector operation is a device kernel on little
// vectors (nv = Ns * nblocks complex numbers, even blocks first).
//
// The little modes are the modes of the last subspace expressed in the
// block basis: for block n, entries (n*Ns + j) = R_jl of the block QR
// factorisation V = Q R (dfl_subspace.c:171-240 stores the Gram-Schmidt
// coefficients); they are the restriction of mode l onto the basis, rounded
// to FP32 like the reference's single-precision vector fields.
//
// Products of little vectors accumulate in double (vprod, vprod_dble), FP32
// vectors are updated in FP32 (mulc_vadd), FP64 vectors in FP64.
#include "lib.h"
#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstring>

namespace qcd {

constexpr int VT = 64;           // vectors per pointer table
constexpr int DG = 296, DT = 256;  // multi-dot grid

struct VTab {
  const void *p[VT];
};
struct ZTab {
  double2 z[VT];
};

__device__ __forceinline__ double2 ldv(const double2 *p, size_t i) { return p[i]; }
__device__ __forceinline__ double2 ldv(const float2 *p, size_t i) {
  const float2 v = p[i];
  return make_double2(v.x, v.y);
}

// part[b*32 + j] = block partial of (Q_{j0+j}, y), j < k <= 32
template <typename V>
__global__ void __launch_bounds__(DT) k_vdot(VTab Q, int j0, int k, const V *__restrict__ y, int n, double2 *part) {
  __shared__ double2 red[DT / 32][32];
  double ar[32], ai[32];
#pragma unroll
  for (int j = 0; j < 32; j++) ar[j] = ai[j] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 yy = ldv(y, i);
#pragma unroll
    for (int j = 0; j < 32; j++)
      if (j < k) {
        const double2 q = ldv((const V *)Q.p[j0 + j], i);
        ar[j] += q.x * yy.x + q.y * yy.y;
        ai[j] += q.x * yy.y - q.y * yy.x;
      }
  }
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 32; j++)
    if (j < k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ar[j] += __shfl_down_sync(0xffffffffu, ar[j], o);
        ai[j] += __shfl_down_sync(0xffffffffu, ai[j], o);
      }
      if (lane == 0) red[wp][j] = make_double2(ar[j], ai[j]);
    }
  __syncthreads();
  if (threadIdx.x < k) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < DT / 32; w++) {
      re += red[w][threadIdx.x].x;
      im += red[w][threadIdx.x].y;
    }
    part[blockIdx.x * 32 + threadIdx.x] = make_double2(re, im);
  }
}

__global__ void k_vdot_fin(const double2 *__restrict__ part, int k, double2 *out) {
  const int j = threadIdx.x;
  if (j >= k) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < DG; b++) {
    re += part[b * 32 + j].x;
    im += part[b * 32 + j].y;
  }
  out[j] = make_double2(re, im);
}

// y += sum_j Z_j X_j in the precision of the vectors, terms in order j
template <typename V>
__global__ void k_vaxpy(V *y, VTab X, ZTab Z, int k, int n);
template <>
__global__ void k_vaxpy<double2>(double2 *y, VTab X, ZTab Z, int k, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 a = y[i];
    for (int j = 0; j < k; j++) {
      const double2 x = ((const double2 *)X.p[j])[i], z = Z.z[j];
      a.x += z.x * x.x - z.y * x.y;
      a.y += z.x * x.y + z.y * x.x;
    }
    y[i] = a;
  }
}
template <>
__global__ void k_vaxpy<float2>(float2 *y, VTab X, ZTab Z, int k, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 a = y[i];
    for (int j = 0; j < k; j++) {
      const float2 x = ((const float2 *)X.p[j])[i];
      const float zr = (float)Z.z[j].x, zi = (float)Z.z[j].y;
      a.x += zr * x.x - zi * x.y;
      a.y += zr * x.y + zi * x.x;
    }
    y[i] = a;
  }
}

template <typename V>
__global__ void k_vscale(V *y, double r, int n);
template <>
__global__ void k_vscale<double2>(double2 *y, double r, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 a = y[i];
    y[i] = make_double2(r * a.x, r * a.y);
  }
}
template <>
__global__ void k_vscale<float2>(float2 *y, double r, int n) {
  const float f = (float)r;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 a = y[i];
    y[i] = make_float2(f * a.x, f * a.y);
  }
}

__global__ void k_v64to32(const double2 *__restrict__ a, float2 *b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 x = a[i];
    b[i] = make_float2((float)x.x, (float)x.y);
  }
}
__global__ void k_v32to64(const float2 *__restrict__ a, double2 *b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 x = a[i];
    b[i] = make_double2(x.x, x.y);
  }
}
// b = a - b (FP64)
__global__ void k_vdiff(const double2 *__restrict__ a, double2 *b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 x = a[i], y = b[i];
    b[i] = make_double2(x.x - y.x, x.y - y.y);
  }
}
// little mode l from the restriction of mode l: entries j > l of every
// block are zero (the triangular factor), all rounded to FP32
__global__ void k_lmode_fix(double2 *v, int Ns, int l, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 x = v[i];
    v[i] = (i % Ns) > l ? make_double2(0.0, 0.0) : make_double2((double)(float)x.x, (double)(float)x.y);
  }
}

// FP32 little operator (modules/little/Aw.c:122, :361): one thread per row
// k of block n, FP32 arithmetic on FP32-rounded matrices M (double2: the
// FP64 matrices rounded on load; float2: FP32 copies).  Modes as in
// k_little_w: 0 A v + sum H v[nbr] (all blocks), 1 sum H v[nbr], 2 v - sum
// H u[nbr], 3 A v.  Matrices are column-major.
template <typename M>
__device__ __forceinline__ float2 ldm(const M *p, size_t i);
template <>
__device__ __forceinline__ float2 ldm<double2>(const double2 *p, size_t i) {
  const double2 a = __ldg(p + i);
  return make_float2((float)a.x, (float)a.y);
}
template <>
__device__ __forceinline__ float2 ldm<float2>(const float2 *p, size_t i) {
  return __ldg(p + i);
}

template <typename M>
__global__ void k_lw32(int mode, int Ns, int b0, const M *__restrict__ A, const M *__restrict__ H,
                       const int *__restrict__ nbr, const float2 *__restrict__ v, const float2 *__restrict__ u,
                       float2 *w) {
  const int n = b0 + blockIdx.x, k = threadIdx.x;
  if (k >= Ns) return;
  float re = 0.f, im = 0.f;
  const size_t nn = (size_t)Ns * Ns;
  if (mode == 0 || mode == 3) {
    const M *a = A + (size_t)n * nn;
    const float2 *x = v + (size_t)n * Ns;
    for (int l = 0; l < Ns; l++) {
      const float2 m = ldm<M>(a, (size_t)l * Ns + k), xv = x[l];
      re += m.x * xv.x - m.y * xv.y;
      im += m.x * xv.y + m.y * xv.x;
    }
  }
  if (mode != 3)
    for (int ifc = 0; ifc < 8; ifc++) {
      const M *a = H + ((size_t)8 * n + ifc) * nn;
      const float2 *x = (mode == 2 ? u : v) + (size_t)__ldg(nbr + 8 * n + ifc) * Ns;
      for (int l = 0; l < Ns; l++) {
        const float2 m = ldm<M>(a, (size_t)l * Ns + k), xv = x[l];
        re += m.x * xv.x - m.y * xv.y;
        im += m.x * xv.y + m.y * xv.x;
      }
    }
  const size_t o = (size_t)n * Ns + k;
  if (mode == 2) w[o] = make_float2(v[o].x - re, v[o].y - im);
  else w[o] = make_float2(re, im);
}

__global__ void k_m64to32(const double2 *__restrict__ a, float2 *b, size_t n) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = make_float2((float)a[i].x, (float)a[i].y);
}

// ------------------------------------------------------------------ state
struct LtlRef {
  int Ns = 0, nv = 0, nvh = 0;
  std::vector<double2 *> lmode;   // little modes (FP32-rounded), nv each
  bool lmode_valid = false;
  std::vector<double2 *> vds;     // [Ns] FP64: even half v_l, odd half (Awhat v_l) even part
  std::vector<float2 *> vs;       // [Ns] FP32 copies of vds
  std::vector<double> Ads;        // Ns x Ns row-major inverse of (v_l, Awhat v_j)
  bool modes_set = false;
  int modes_ver = -1;   // awhat_ver the little-little operator was built for
  float2 *Mhop32 = nullptr;       // FP32 copy of the preconditioned hop matrices
  bool mhop32_valid = false;
  std::vector<double2 *> wvd;     // FP64 work vectors (nv)
  std::vector<float2 *> wvs;      // FP32 work vectors (nv)
  double2 *part = nullptr, *dots = nullptr, *h_dots = nullptr;
  double2 *t64 = nullptr;          // odd scratch of Awhat_dble
  float2 *t32 = nullptr;           // odd scratch of Awhat
  // recursion state of the two solvers
  double tol = 0.0, res_gcr = 0.0;
  int nmx_gcr = 0, *stat_gcr = nullptr;
};

static LtlRef *lr(Ctx &c) {
  if (!c.dfl.ltlref) c.dfl.ltlref = new LtlRef();
  return c.dfl.ltlref;
}

void ltl_ref_release(Ctx &c) {
  LtlRef *r = c.dfl.ltlref;
  if (!r) return;
  for (auto p : r->lmode) cudaFree(p);
  for (auto p : r->vds) cudaFree(p);
  for (auto p : r->vs) cudaFree(p);
  for (auto p : r->wvd) cudaFree(p);
  for (auto p : r->wvs) cudaFree(p);
  cudaFree(r->Mhop32);
  cudaFree(r->part);
  cudaFree(r->dots);
  cudaFree(r->t64);
  cudaFree(r->t32);
  if (r->h_dots) cudaFreeHost(r->h_dots);
  delete r;
  c.dfl.ltlref = nullptr;
}

static int ensure_base(Ctx &c) {
  DflState &d = c.dfl;
  LtlRef &r = *lr(c);
  if (r.Ns != d.Ns || r.nv != d.nv) {
    ltl_ref_release(c);
    LtlRef &q = *lr(c);
    q.Ns = d.Ns;
    q.nv = d.nv;
    q.nvh = d.nv / 2;
  }
  LtlRef &q = *lr(c);
  if (!q.part) {
    if (cudaMalloc(&q.part, (size_t)DG * 32 * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&q.dots, VT * sizeof(double2)) != cudaSuccess ||
        cudaMallocHost(&q.h_dots, VT * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&q.t64, (size_t)q.nv * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&q.t32, (size_t)q.nv * sizeof(float2)) != cudaSuccess)
      return fail("out of device memory (little solver)");
  }
  return 0;
}

template <typename T>
static int grow(std::vector<T *> &v, size_t n, size_t len) {
  while (v.size() < n) {
    T *p = nullptr;
    if (cudaMalloc(&p, len * sizeof(T)) != cudaSuccess) return fail("out of device memory (little vectors)");
    cudaMemset(p, 0, len * sizeof(T));
    v.push_back(p);
  }
  return 0;
}

static unsigned vgrid(int n) { return (unsigned)std::min((n + 255) / 256, 4 * 148); }

// (Q_j, y) for j < k on the host
template <typename V>
static void vdots(Ctx &c, const V *const *Q, int k, const V *y, int n, double2 *out) {
  LtlRef &r = *lr(c);
  cudaStream_t st = c.stream;
  for (int j0 = 0; j0 < k; j0 += 32) {
    const int kk = std::min(32, k - j0);
    VTab t;
    std::memset(&t, 0, sizeof(t));
    for (int j = 0; j < kk; j++) t.p[j] = Q[j0 + j];
    k_vdot<V><<<DG, DT, 0, st>>>(t, 0, kk, y, n, r.part);
    k_vdot_fin<<<1, 32, 0, st>>>(r.part, kk, r.dots + j0);
  }
  cudaMemcpyAsync(r.h_dots, r.dots, k * sizeof(double2), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  for (int j = 0; j < k; j++) out[j] = r.h_dots[j];
}

template <typename V>
static double vnorm2(Ctx &c, const V *y, int n) {
  double2 z;
  const V *q[1] = {y};
  vdots<V>(c, q, 1, y, n, &z);
  return z.x;
}

// y += sum_j z_j X_j
template <typename V>
static void vaxpy(Ctx &c, V *y, const V *const *X, const double2 *z, int k, int n) {
  for (int j0 = 0; j0 < k; j0 += VT) {
    const int kk = std::min(VT, k - j0);
    VTab t;
    ZTab zz;
    std::memset(&t, 0, sizeof(t));
    std::memset(&zz, 0, sizeof(zz));
    for (int j = 0; j < kk; j++) {
      t.p[j] = X[j0 + j];
      zz.z[j] = z[j0 + j];
    }
    k_vaxpy<V><<<vgrid(n), 256, 0, c.stream>>>(y, t, zz, kk, n);
  }
}

template <typename V>
static void vscale(Ctx &c, V *y, double r, int n) {
  k_vscale<V><<<vgrid(n), 256, 0, c.stream>>>(y, r, n);
}

static void vcopy64(Ctx &c, double2 *dst, const double2 *src, int n) {
  cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, c.stream);
}

// little operators on little vectors (even half written)
static void awhat64(Ctx &c, const double2 *v, double2 *w) { dfl_Awhat(c, v, w, lr(c)->t64, c.stream); }

static void little32(int mode, Ctx &c, int b0, int nblk, const void *A, const void *H, bool h32, const float2 *v,
                     const float2 *u, float2 *w) {
  DflState &d = c.dfl;
  const int t = (d.Ns + 31) / 32 * 32;
  if (h32)
    k_lw32<float2><<<nblk, t, 0, c.stream>>>(mode, d.Ns, b0, (const float2 *)A, (const float2 *)H, d.nbr, v, u, w);
  else
    k_lw32<double2><<<nblk, t, 0, c.stream>>>(mode, d.Ns, b0, (const double2 *)A, (const double2 *)H, d.nbr, v, u,
                                             w);
}

static int mhop32(Ctx &c) {
  DflState &d = c.dfl;
  LtlRef &r = *lr(c);
  const size_t n = (size_t)8 * d.nb * d.Ns * d.Ns;
  if (!r.Mhop32 && cudaMalloc(&r.Mhop32, n * sizeof(float2)) != cudaSuccess)
    return fail("out of device memory (FP32 little operator)");
  if (!r.mhop32_valid) {
    k_m64to32<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(d.Mhop, r.Mhop32, n);
    r.mhop32_valid = true;
  }
  return 0;
}

// Awhat (FP32): w_e = v_e - H_eo H_oe v_e with the FP32 preconditioned hops
static void awhat32(Ctx &c, const float2 *v, float2 *w) {
  DflState &d = c.dfl;
  LtlRef &r = *lr(c);
  const int nbh = d.nb / 2;
  little32(1, c, nbh, nbh, nullptr, r.Mhop32, true, v, nullptr, r.t32);
  little32(2, c, 0, nbh, nullptr, r.Mhop32, true, v, r.t32, w);
}

// ------------------------------------------------------------ little modes
// Little modes from the Ns global mode fields (FP32) of the subspace just
// built: the restriction of every mode, made triangular and FP32-rounded.
int ltl_lmodes_from_fields(Ctx &c, const std::vector<void *> &modes, cudaStream_t st) {
  DflState &d = c.dfl;
  if (ensure_base(c)) return -1;
  LtlRef &r = *lr(c);
  if (grow(r.lmode, d.Ns, d.nv) || dfl_batch_alloc(c)) return -1;
  for (int l0 = 0; l0 < d.Ns; l0 += 4) {
    const int na = std::min(4, d.Ns - l0);
    const void *f[4];
    double2 *v[4];
    for (int i = 0; i < na; i++) {
      f[i] = modes[l0 + i];
      v[i] = r.lmode[l0 + i];
    }
    dfl_restrict_b(c, na, f, v, st);
  }
  for (int l = 0; l < d.Ns; l++) k_lmode_fix<<<vgrid(d.nv), 256, 0, st>>>(r.lmode[l], d.Ns, l, d.nv);
  r.lmode_valid = true;
  r.modes_set = false;
  return 0;
}

// little mode l from a host/device array (complex floats, nv of them)
int ltl_lmode_set(Ctx &c, int l, const void *v32) {
  DflState &d = c.dfl;
  if (ensure_base(c)) return -1;
  LtlRef &r = *lr(c);
  if (l < 0 || l >= d.Ns) return fail("little mode index out of range");
  if (grow(r.lmode, d.Ns, d.nv) || grow(r.wvs, 1, d.nv)) return -1;
  cudaMemcpyAsync(r.wvs[0], v32, (size_t)d.nv * sizeof(float2), cudaMemcpyDefault, c.stream);
  k_v32to64<<<vgrid(d.nv), 256, 0, c.stream>>>(r.wvs[0], r.lmode[l], d.nv);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("CUDA error");
  if (l == d.Ns - 1) r.lmode_valid = true;
  r.modes_set = false;
  return 0;
}

void ltl_forget_lmodes(Ctx &c) {
  if (c.dfl.ltlref) {
    c.dfl.ltlref->lmode_valid = false;
    c.dfl.ltlref->modes_set = false;
  }
}

void ltl_invalidate(Ctx &c) {
  if (c.dfl.ltlref) {
    c.dfl.ltlref->modes_set = false;
    c.dfl.ltlref->mhop32_valid = false;
  }
}

// inverse of an n x n complex matrix (row-major) by Gauss-Jordan with
// partial pivoting; Frobenius condition number in *k; 1 if singular
static int cmat_inv(int n, std::vector<double> a, std::vector<double> &b, double *k) {
  // a, b: 2*n*n reals (re, im interleaved)
  b.assign(2 * (size_t)n * n, 0.0);
  double fa = 0.0;
  for (int i = 0; i < n * n; i++) fa += a[2 * i] * a[2 * i] + a[2 * i + 1] * a[2 * i + 1];
  for (int i = 0; i < n; i++) b[2 * (i * n + i)] = 1.0;
  for (int col = 0; col < n; col++) {
    int piv = col;
    double best = -1.0;
    for (int i = col; i < n; i++) {
      const double m = std::hypot(a[2 * (i * n + col)], a[2 * (i * n + col) + 1]);
      if (m > best) {
        best = m;
        piv = i;
      }
    }
    if (!(best > 0.0)) return 1;
    if (piv != col)
      for (int j = 0; j < n; j++)
        for (int q = 0; q < 2; q++) {
          std::swap(a[2 * (piv * n + j) + q], a[2 * (col * n + j) + q]);
          std::swap(b[2 * (piv * n + j) + q], b[2 * (col * n + j) + q]);
        }
    const double pr = a[2 * (col * n + col)], pi = a[2 * (col * n + col) + 1];
    const double den = pr * pr + pi * pi, ir = pr / den, ii = -pi / den;
    for (int j = 0; j < n; j++) {
      double xr = a[2 * (col * n + j)], xi = a[2 * (col * n + j) + 1];
      a[2 * (col * n + j)] = xr * ir - xi * ii;
      a[2 * (col * n + j) + 1] = xr * ii + xi * ir;
      xr = b[2 * (col * n + j)];
      xi = b[2 * (col * n + j) + 1];
      b[2 * (col * n + j)] = xr * ir - xi * ii;
      b[2 * (col * n + j) + 1] = xr * ii + xi * ir;
    }
    for (int i = 0; i < n; i++) {
      if (i == col) continue;
      const double fr = a[2 * (i * n + col)], fi = a[2 * (i * n + col) + 1];
      if (fr == 0.0 && fi == 0.0) continue;
      for (int j = 0; j < n; j++) {
        a[2 * (i * n + j)] -= fr * a[2 * (col * n + j)] - fi * a[2 * (col * n + j) + 1];
        a[2 * (i * n + j) + 1] -= fr * a[2 * (col * n + j) + 1] + fi * a[2 * (col * n + j)];
        b[2 * (i * n + j)] -= fr * b[2 * (col * n + j)] - fi * b[2 * (col * n + j) + 1];
        b[2 * (i * n + j) + 1] -= fr * b[2 * (col * n + j) + 1] + fi * b[2 * (col * n + j)];
      }
    }
  }
  double fb = 0.0;
  for (int i = 0; i < n * n; i++) fb += b[2 * i] * b[2 * i] + b[2 * i + 1] * b[2 * i + 1];
  *k = std::sqrt(fa * fb);
  return 0;
}

// set_ltl_modes (ltl_modes.c:286): needs Awhat up to date; 1 if the
// little-little operator is not safely invertible (Frobenius condition
// number 10^6 or more), -1 on an error
int ltl_set_modes(Ctx &c) {
  DflState &d = c.dfl;
  if (ensure_base(c)) return -1;
  LtlRef &r = *lr(c);
  if (!r.lmode_valid) return fail("ltl_gcr: no little modes (the subspace was not built from modes)");
  const int Ns = d.Ns, nvh = r.nvh;
  if (grow(r.vds, Ns, d.nv) || grow(r.vs, Ns, d.nv)) return -1;
  // vs2vds: the even halves, orthonormalised in the reference's order
  for (int l = 0; l < Ns; l++) vcopy64(c, r.vds[l], r.lmode[l], nvh);
  double rr = vnorm2<double2>(c, r.vds[0], nvh);
  int ifail = 0;
  double s = std::sqrt(rr);
  if (s == 0.0) ifail = 1;
  else s = 1.0 / s;
  std::vector<double2> B(Ns);
  for (int l = 1; l < Ns; l++) {
    vscale<double2>(c, r.vds[l - 1], s, nvh);
    vdots<double2>(c, r.vds.data(), l, r.vds[l], nvh, B.data());
    for (int j = 0; j < l; j++) B[j] = make_double2(-B[j].x, -B[j].y);
    vaxpy<double2>(c, r.vds[l], r.vds.data(), B.data(), l, nvh);
    rr = vnorm2<double2>(c, r.vds[l], nvh);
    s = std::sqrt(rr);
    if (s == 0.0) ifail = 1;
    else s = 1.0 / s;
  }
  vscale<double2>(c, r.vds[Ns - 1], s, nvh);
  if (ifail) return fail("set_ltl_modes: degenerate basis vector fields");
  // vds2Avds: odd halves = Awhat v_l (even part); FP32 copies of both halves
  for (int l = 0; l < Ns; l++) {
    awhat64(c, r.vds[l], r.t64);
    vcopy64(c, r.vds[l] + nvh, r.t64, nvh);
    k_v64to32<<<vgrid(d.nv), 256, 0, c.stream>>>(r.vds[l], r.vs[l], d.nv);
  }
  // set_Ads: C_lj = (v_l, Awhat v_j), Ads = C^-1
  std::vector<double> C(2 * (size_t)Ns * Ns), Ai;
  std::vector<const double2 *> odd(Ns);
  for (int j = 0; j < Ns; j++) odd[j] = r.vds[j] + nvh;
  for (int l = 0; l < Ns; l++) {
    // (v_l, A v_j) = conj((A v_j, v_l))
    vdots<double2>(c, odd.data(), Ns, r.vds[l], nvh, B.data());
    for (int j = 0; j < Ns; j++) {
      C[2 * (l * Ns + j)] = B[j].x;
      C[2 * (l * Ns + j) + 1] = -B[j].y;
    }
  }
  double cn = 0.0;
  int ie = cmat_inv(Ns, C, Ai, &cn);
  ie |= (cn > 1.0e6);
  r.Ads = Ai;
  r.modes_set = true;
  r.modes_ver = d.awhat_ver;
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return fail("set_ltl_modes: CUDA error");
  return ie ? 1 : 0;
}

// y = Ads x (Ns)
static void ads_vec(const LtlRef &r, const double2 *x, double2 *y) {
  const int n = r.Ns;
  for (int i = 0; i < n; i++) {
    double re = 0.0, im = 0.0;
    for (int j = 0; j < n; j++) {
      const double ar = r.Ads[2 * (i * n + j)], ai = r.Ads[2 * (i * n + j) + 1];
      re += ar * x[j].x - ai * x[j].y;
      im += ar * x[j].y + ai * x[j].x;
    }
    y[i] = make_double2(re, im);
  }
}

// the projections of ltl_modes.c:336-446 (even halves)
void dfl_Lvd_dev(Ctx &c, double2 *vd) {
  LtlRef &r = *lr(c);
  const int Ns = r.Ns, nvh = r.nvh;
  std::vector<double2> B(Ns), Cc(Ns);
  vdots<double2>(c, r.vds.data(), Ns, vd, nvh, B.data());
  for (int l = 0; l < Ns; l++) Cc[l] = make_double2(-B[l].x, -B[l].y);
  ads_vec(r, Cc.data(), B.data());
  std::vector<const double2 *> odd(Ns);
  for (int l = 0; l < Ns; l++) odd[l] = r.vds[l] + nvh;
  vaxpy<double2>(c, vd, odd.data(), B.data(), Ns, nvh);
}

void dfl_LRvd_dev(Ctx &c, double2 *vd, double2 *wd) {
  LtlRef &r = *lr(c);
  const int Ns = r.Ns, nvh = r.nvh;
  std::vector<double2> B(Ns), Cc(Ns), mB(Ns);
  vdots<double2>(c, r.vds.data(), Ns, vd, nvh, Cc.data());
  ads_vec(r, Cc.data(), B.data());
  cudaMemsetAsync(wd, 0, (size_t)nvh * sizeof(double2), c.stream);
  std::vector<const double2 *> odd(Ns);
  for (int l = 0; l < Ns; l++) {
    odd[l] = r.vds[l] + nvh;
    mB[l] = make_double2(-B[l].x, -B[l].y);
  }
  vaxpy<double2>(c, wd, r.vds.data(), B.data(), Ns, nvh);
  vaxpy<double2>(c, vd, odd.data(), mB.data(), Ns, nvh);
}

void dfl_RLvd_dev(Ctx &c, double2 *vd, double2 *wd) {
  LtlRef &r = *lr(c);
  const int Ns = r.Ns, nvh = r.nvh;
  std::vector<double2> B(Ns), Cc(Ns);
  vdots<double2>(c, r.vds.data(), Ns, wd, nvh, B.data());
  for (int l = 0; l < Ns; l++) Cc[l] = make_double2(-B[l].x, -B[l].y);
  ads_vec(r, Cc.data(), B.data());
  std::vector<const double2 *> odd(Ns);
  for (int l = 0; l < Ns; l++) odd[l] = r.vds[l] + nvh;
  vaxpy<double2>(c, wd, odd.data(), B.data(), Ns, nvh);
  vaxpy<double2>(c, vd, r.vds.data(), B.data(), Ns, nvh);
}

void dfl_Lv_dev(Ctx &c, float2 *v) {
  LtlRef &r = *lr(c);
  const int Ns = r.Ns, nvh = r.nvh;
  std::vector<double2> B(Ns), Cc(Ns);
  vdots<float2>(c, r.vs.data(), Ns, v, nvh, Cc.data());
  ads_vec(r, Cc.data(), B.data());
  std::vector<const float2 *> odd(Ns);
  for (int l = 0; l < Ns; l++) {
    odd[l] = r.vs[l] + nvh;
    B[l] = make_double2(-(double)(float)B[l].x, -(double)(float)B[l].y);
  }
  vaxpy<float2>(c, v, odd.data(), B.data(), Ns, nvh);
}

// ------------------------------------------------------------------ gcr4v
// gcr4v.c:302 on the even halves: Dop = Awhat (FP32) then dfl_Lv
static float gcr4v_dev(Ctx &c, int nmx, float res, const float2 *eta, float2 *psi, int *status) {
  LtlRef &r = *lr(c);
  const int n = r.nvh;
  float2 *rho = r.wvs[2];
  float2 **phi = &r.wvs[3], **chi = &r.wvs[3 + nmx];
  const float PRECISION_LIMIT = (float)(100.0 * FLT_EPSILON);
  std::vector<double2> a((size_t)nmx * nmx), cc(nmx), dd(std::max(nmx, 2));
  std::vector<double> b(nmx);
  // gcr_init
  cudaMemsetAsync(psi, 0, (size_t)n * sizeof(float2), c.stream);
  cudaMemcpyAsync(rho, eta, (size_t)n * sizeof(float2), cudaMemcpyDeviceToDevice, c.stream);
  float rn = (float)std::sqrt(vnorm2<float2>(c, eta, n));
  const float tol = res * rn;
  int nst = 0, is = 0;
  if (rn != 0.0f) {
    while (nst < nmx) {
      const float rn_old = rn;
      const int m = nst;
      // gcr_step
      awhat32(c, rho, chi[m]);
      dfl_Lv_dev(c, chi[m]);
      if (m > 0) {
        vdots<float2>(c, chi, m, chi[m], n, dd.data());
        for (int l = 0; l < m; l++) a[(size_t)nmx * l + m] = dd[l];
        std::vector<double2> z(m);
        for (int l = 0; l < m; l++) z[l] = make_double2(-(double)(float)dd[l].x, -(double)(float)dd[l].y);
        vaxpy<float2>(c, chi[m], chi, z.data(), m, n);
      }
      cudaMemcpyAsync(phi[m], rho, (size_t)n * sizeof(float2), cudaMemcpyDeviceToDevice, c.stream);
      double2 c0;
      {
        const float2 *q[1] = {chi[m]};
        vdots<float2>(c, q, 1, rho, n, &c0);
      }
      const double c1 = vnorm2<float2>(c, chi[m], n);
      b[m] = std::sqrt(c1);
      nst++;
      if (b[m] != 0.0) {
        const double rb = 1.0 / b[m];
        cc[m] = make_double2(rb * c0.x, rb * c0.y);
        vscale<float2>(c, chi[m], rb, n);
        const double2 z = make_double2(-(double)(float)cc[m].x, -(double)(float)cc[m].y);
        const float2 *q[1] = {chi[m]};
        vaxpy<float2>(c, rho, q, &z, 1, n);
        rn = (float)std::sqrt(vnorm2<float2>(c, rho, n));
        is = 0;
      } else {
        is = 1;
      }
      if (rn <= tol || rn <= PRECISION_LIMIT * rn_old || is == 1) break;
    }
    // set_psi
    int m = nst - 1;
    if (b[m] == 0.0) m -= 1;
    for (int l = m; l >= 0; l--) {
      double2 w = cc[l];
      for (int j = l + 1; j <= m; j++) {
        const double2 al = a[(size_t)l * nmx + j];
        w.x -= al.x * cc[j].x - al.y * cc[j].y;
        w.y -= al.x * cc[j].y + al.y * cc[j].x;
      }
      const double rb = 1.0 / b[l];
      cc[l] = make_double2(w.x * rb, w.y * rb);
    }
    for (int l = m; l >= 0; l--) {
      const double2 z = make_double2((double)(float)cc[l].x, (double)(float)cc[l].y);
      const float2 *q[1] = {phi[l]};
      vaxpy<float2>(c, psi, q, &z, 1, n);
    }
  }
  status[0] = rn <= tol ? nst : -1;
  return rn;
}

// --------------------------------------------------------------- fgcr4vd
// Mop of ltl_gcr.c:119-146: FP32 gcr4v solve, then w, z = (P_L Awhat) w
static void ltl_mop(Ctx &c, const double2 *vd, double2 *wd, double2 *zd) {
  LtlRef &r = *lr(c);
  const int n = r.nvh;
  k_v64to32<<<vgrid(n), 256, 0, c.stream>>>(vd, r.wvs[0], n);
  const double rn = std::sqrt(vnorm2<float2>(c, r.wvs[0], n));
  float res;
  if (rn * r.res_gcr < r.tol) res = (float)(r.tol / rn);
  else res = (float)r.res_gcr;
  int status = 0;
  (void)gcr4v_dev(c, r.nmx_gcr, res, r.wvs[0], r.wvs[1], &status);
  *r.stat_gcr += status < 0 ? r.nmx_gcr : status;
  k_v32to64<<<vgrid(n), 256, 0, c.stream>>>(r.wvs[1], wd, n);
  awhat64(c, wd, zd);
  dfl_RLvd_dev(c, wd, zd);
}

static void ltl_dop(Ctx &c, const double2 *v, double2 *w) {
  awhat64(c, v, w);
  dfl_Lvd_dev(c, w);
}

// fgcr4vd.c:339 with the Dop and Mop above; vectors of nvh entries
static double fgcr4vd_dev(Ctx &c, int nkv, int nmx, double res, const double2 *eta, double2 *psi, int *status) {
  LtlRef &r = *lr(c);
  const int n = r.nvh;
  double2 *rho = r.wvd[2];
  double2 **phi = &r.wvd[3], **chi = &r.wvd[3 + nkv];
  const double PRECISION_LIMIT = 100.0 * DBL_EPSILON;
  std::vector<double2> a((size_t)nkv * nkv), cc(nkv), dd(nkv);
  std::vector<double> b(nkv);
  cudaMemsetAsync(psi, 0, (size_t)n * sizeof(double2), c.stream);
  vcopy64(c, rho, eta, n);
  double rn = std::sqrt(vnorm2<double2>(c, eta, n));
  const double tol = res * rn;
  int nst = 0, is = 0;
  if (rn != 0.0) {
    while (nst < nmx) {
      const double rn_old = rn;
      int m = 0;
      is = 0;
      while (m < nkv && nst < nmx) {
        // gcr_step
        ltl_mop(c, rho, phi[m], chi[m]);
        if (m > 0) {
          vdots<double2>(c, chi, m, chi[m], n, dd.data());
          for (int l = 0; l < m; l++) a[(size_t)nkv * l + m] = dd[l];
          std::vector<double2> z(m);
          for (int l = 0; l < m; l++) z[l] = make_double2(-dd[l].x, -dd[l].y);
          vaxpy<double2>(c, chi[m], chi, z.data(), m, n);
        }
        double2 c0;
        {
          const double2 *q[1] = {chi[m]};
          vdots<double2>(c, q, 1, rho, n, &c0);
        }
        b[m] = std::sqrt(vnorm2<double2>(c, chi[m], n));
        if (b[m] != 0.0) {
          const double rb = 1.0 / b[m];
          cc[m] = make_double2(rb * c0.x, rb * c0.y);
          vscale<double2>(c, chi[m], rb, n);
          const double2 z = make_double2(-cc[m].x, -cc[m].y);
          const double2 *q[1] = {chi[m]};
          vaxpy<double2>(c, rho, q, &z, 1, n);
          rn = std::sqrt(vnorm2<double2>(c, rho, n));
          is = 0;
        } else {
          is = 1;
        }
        m++;
        nst++;
        if (rn <= tol || rn <= PRECISION_LIMIT * rn_old || is == 1) break;
      }
      // update_psi
      int mm = m - 1;
      const bool irho = (rn > tol) && (nst < nmx) && (is == 0);
      if (b[mm] == 0.0) mm -= 1;
      for (int l = mm; l >= 0; l--) {
        double2 z = cc[l];
        for (int j = l + 1; j <= mm; j++) {
          const double2 al = a[(size_t)l * nkv + j];
          z.x -= al.x * cc[j].x - al.y * cc[j].y;
          z.y -= al.x * cc[j].y + al.y * cc[j].x;
        }
        const double rb = 1.0 / b[l];
        cc[l] = make_double2(z.x * rb, z.y * rb);
      }
      for (int l = mm; l >= 0; l--) {
        const double2 *q[1] = {phi[l]};
        vaxpy<double2>(c, psi, q, &cc[l], 1, n);
      }
      if (irho) {
        ltl_dop(c, psi, rho);
        k_vdiff<<<vgrid(n), 256, 0, c.stream>>>(eta, rho, n);
        rn = std::sqrt(vnorm2<double2>(c, rho, n));
      }
      if (rn <= tol || is == 1) break;
    }
  }
  status[0] = rn <= tol ? nst : -1;
  return rn;
}

// ----------------------------------------------------------------- ltl_gcr
// ltl_gcr.c:155 on device little vectors eta, psi (nv each, may be equal)
double ltl_gcr_ref(Ctx &c, double mu, const double2 *eta, double2 *psi, int *ifail, int *status, cudaStream_t st) {
  DflState &d = c.dfl;
  (void)st;
  ifail[0] = 0;
  status[0] = status[1] = 0;
  if (ensure_base(c)) return -1.0;
  LtlRef &r = *lr(c);
  const int nv = d.nv, nvh = r.nvh, nbh = d.nb / 2;
  if (d.nkv < 2 || d.nmx < 1 || d.res <= DBL_EPSILON) {
    fail("fgcr4vd: improper choice of vol, nkv, nmx or res");
    return -1.0;
  }
  if (d.nmx_gcr < 2 || d.nmx_gcr > VT) {
    fail("gcr4v: nmx must be in [2, 64]");
    return -1.0;
  }
  const int aw = dfl_set_Awhat(c, mu, c.stream);
  if (aw < 0) return -1.0;
  if (aw) {
    ifail[0] = -2;
    if (psi != eta) cudaMemsetAsync(psi, 0, (size_t)nv * sizeof(double2), c.stream);
    return std::sqrt(vnorm2<double2>(c, eta, nv));
  }
  if (!r.modes_set || r.modes_ver != d.awhat_ver) {
    r.mhop32_valid = false;
    const int lm = ltl_set_modes(c);
    if (lm < 0) return -1.0;
    if (lm) {
      // the reference stops when set_ltl_modes fails (Aw_ops.c set_Awhat)
      fail("set_Awhat: unsafe inversion of the little-little Dirac operator");
      return -1.0;
    }
  }
  if (mhop32(c)) return -1.0;
  if (grow(r.wvd, 2 * d.nkv + 3, nv) || grow(r.wvs, 2 * d.nmx_gcr + 3, nv)) return -1.0;
  double2 *w0 = r.wvd[0], *w1 = r.wvd[1];
  // wvd1 = eta; odd: Aoo^-1 eta_o; even: eta_e - Aeo (.); w0_e = Aee^-1 (.)
  vcopy64(c, w1, eta, nv);
  dfl_Awooinv(c, eta, w1, c.stream);
  dfl_Aweo(c, w1, w1, c.stream);
  dfl_Aweeinv(c, w1, w0, c.stream);
  const double rho0 = std::sqrt(vnorm2<double2>(c, w0, nvh));
  dfl_LRvd_dev(c, w0, w0 + nvh);
  const double rho1 = std::sqrt(vnorm2<double2>(c, w0, nvh));
  double rho;
  if (rho1 != 0.0) {
    r.nmx_gcr = d.nmx_gcr;
    r.stat_gcr = status + 1;
    double fact = std::sqrt((double)nvh) / rho1;
    vscale<double2>(c, w0, fact, nvh);
    const double res = (rho0 / rho1) * d.res;
    r.res_gcr = (rho0 / rho1) * d.res_gcr;
    r.tol = fact * rho1 * res;
    rho = fgcr4vd_dev(c, d.nkv, d.nmx, (rho0 / rho1) * d.res, w0, w1, status);
    fact = 1.0 / fact;
    vscale<double2>(c, w1, fact, nvh);
    {
      const double2 *q[1] = {w0 + nvh};
      const double2 one = make_double2(1.0, 0.0);
      vaxpy<double2>(c, w1, q, &one, 1, nvh);
    }
    rho *= fact;
    if (status[0] < 0) {
      ifail[0] = -1;
      status[0] = d.nmx;
    }
  } else {
    rho = 0.0;
    vcopy64(c, w1, w0 + nvh, nvh);
  }
  // psi_e = x_e ; psi_o = Aoo^-1 (eta_o - Aoe x_e).  Only the even half of
  // psi is written before eta_o is read (psi may be eta).
  dfl_Awoe(c, w1, w1, c.stream);
  vcopy64(c, psi, w1, nvh);
  k_vdiff<<<vgrid(nvh), 256, 0, c.stream>>>(eta + nvh, w1 + nvh, nvh);
  dfl_Awooinv(c, w1, psi, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) {
    fail("ltl_gcr: CUDA error");
    return -1.0;
  }
  return rho;
}

// the inverse little-little matrix (ltl_matrix, ltl_modes.c:325), host copy
const double *ltl_matrix_host(Ctx &c) {
  LtlRef *r = c.dfl.ltlref;
  return (r && r->modes_set) ? r->Ads.data() : nullptr;
}

// FP32 little operators on device little vectors (complex floats): Aw
// (Aw.c:122, all blocks), Awhat (Aw.c:361, even blocks) and the even-odd
// pieces of Aw.c:202-359 -- 2 Aweeinv (w_e = Aee^-1 v_e), 3 Awooinv
// (w_o = Aoo^-1 v_o), 4 Awoe (w_o = Aoe v_e), 5 Aweo (w_e -= Aeo v_o)
int little32_apply(Ctx &c, int which, const float2 *v, float2 *w) {
  DflState &d = c.dfl;
  if (ensure_base(c)) return -1;
  LtlRef &r = *lr(c);
  const int nbh = d.nb / 2;
  if (which == 0) {
    little32(0, c, 0, d.nb, d.Ablk, d.Ahop, false, v, nullptr, w);
  } else if (which == 1) {
    little32(1, c, nbh, nbh, nullptr, d.Mhop, false, v, nullptr, r.t32);
    little32(2, c, 0, nbh, nullptr, d.Mhop, false, v, r.t32, w);
  } else if (which == 2) {
    little32(3, c, 0, nbh, d.Ainv, nullptr, false, v, nullptr, w);
  } else if (which == 3) {
    little32(3, c, nbh, nbh, d.Ainv, nullptr, false, v, nullptr, w);
  } else if (which == 4) {
    little32(1, c, nbh, nbh, nullptr, d.Ahop, false, v, nullptr, w);
  } else {
    little32(2, c, 0, nbh, nullptr, d.Ahop, false, w, v, w);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : fail("little operator: launch failed");
}

}  // namespace qcd
