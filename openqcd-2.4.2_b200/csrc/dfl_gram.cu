// Orthonormalisation of deflation modes by Cholesky QR, applied twice.
//
// The reference orthonormalises the Ns modes block by block with
// Gram-Schmidt in double precision (modules/dfl/dfl_subspace.c:171-240) and
// renormalises the global modes between inverse iterations the same way
// (dfl_subspace.c:243-259).  Both compute Q of the QR factorisation V = QR
// with a positive real diagonal of R, which is unique, so here it is formed
// as Q = V R^-1 from the Cholesky factor of the Gram matrix G = V^H V = R^H R.
// A second pass on Q removes the loss of orthogonality of the first
// (cond(V)^2 eps), which makes the result as orthonormal as Gram-Schmidt's.
//
// Gram-Schmidt goes over every block's vectors about Ns/2 times per vector
// (0.37 s per subspace at 48^3x96 with Ns = 28); here each pass reads the
// vectors twice: once for the Gram matrices and once for the transform.
//
//   k_blk_gram   per block: G = V^H V, FP64 sums of exact products of the
//                FP32 components (a product of two FP32 numbers is exact in
//                FP64), the block's sites streamed through shared memory
//   k_gram_sum   G of the whole lattice = sum of the block matrices
//   k_chol_inv   per matrix: Cholesky G = R^H R (one warp), T = R^-1
//   k_blk_apply  per block: Q_l = sum_{k<=l} V_k T_kl in FP64, stored FP32
#include "lib.h"
#include <algorithm>

namespace qcd {

// shared-memory tile of S sites of all Ns vectors: row k holds the 12
// complex components of each site at a site stride of 13 float2 (the pad
// spreads the sites of a warp over the banks), rows padded by one float2
constexpr int GSS = 13;

__device__ __forceinline__ void load_tile(const Geom &g, int blk, const float4 *const *v, int Ns, int S, int s0,
                                          float2 *tile, int ld) {
  const int nsite = 2 * g.vbh;
  for (int idx = threadIdx.x; idx < Ns * S * 6; idx += blockDim.x) {
    const int s = idx % S, j = (idx / S) % 6, k = idx / (6 * S);
    const int t = s0 + s;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t < nsite) {
      const int p = t >= g.vbh, si = t - p * g.vbh, chunk = p * g.nbl + blk;
      x = __ldg(v[k] + ((size_t)chunk * 6 + j) * g.vbh + si);
    }
    float2 *row = tile + (size_t)k * ld + s * GSS + 2 * j;
    row[0] = make_float2(x.x, x.y);
    row[1] = make_float2(x.z, x.w);
  }
}

// G[n] = V_n^H V_n (full Hermitian Ns x Ns, row-major) for block n.  Each
// thread owns a 4x4 tile (ti, tj), ti <= tj, of the upper triangle and one
// of KS slices of the site components (split-K); the slices are summed at
// the end.  Rows Ns..4*nt-1 of the shared tile stay zero.
__global__ void __launch_bounds__(256) k_blk_gram(Geom g, const int *__restrict__ vd2lex,
                                                  const float4 *const *__restrict__ v, int Ns, int S, double2 *G) {
  extern __shared__ float2 gtile[];
  const int n = blockIdx.x, blk = __ldg(vd2lex + n);
  const int ld = S * GSS + 1, nt = (Ns + 3) / 4, nr = 4 * nt;
  const int U = nt * (nt + 1) / 2, KS = max(1, (int)blockDim.x / U);
  const int t = threadIdx.x, u = t % U, ks = t / U;
  const bool busy = t < U * KS;
  int ti = 0, tj = 0;
  {
    int r = u;
    while (r >= nt - ti) {
      r -= nt - ti;
      ti++;
    }
    tj = ti + r;
  }
  for (int e = threadIdx.x; e < (nr - Ns) * ld; e += blockDim.x) gtile[(size_t)Ns * ld + e] = make_float2(0.f, 0.f);
  double2 acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = make_double2(0.0, 0.0);
  const int nel = S * 12;
  for (int s0 = 0; s0 < 2 * g.vbh; s0 += S) {
    __syncthreads();
    load_tile(g, blk, v, Ns, S, s0, gtile, ld);
    __syncthreads();
    if (!busy) continue;
    for (int i = ks; i < nel; i += KS) {
      const int off = (i / 12) * GSS + i % 12;
      double xr[4], xi[4], yr[4], yi[4];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const float2 x = gtile[(size_t)(4 * ti + a) * ld + off];
        const float2 y = gtile[(size_t)(4 * tj + a) * ld + off];
        xr[a] = x.x;
        xi[a] = x.y;
        yr[a] = y.x;
        yi[a] = y.y;
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {   // conj(x_a) y_b
          acc[a][b].x += xr[a] * yr[b] + xi[a] * yi[b];
          acc[a][b].y += xr[a] * yi[b] - xi[a] * yr[b];
        }
    }
  }
  // sum the KS slices through shared memory (the tile is free now)
  __syncthreads();
  double2 *part = (double2 *)gtile;   // [KS][U][16]
  if (busy)
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) part[((size_t)ks * U + u) * 16 + 4 * a + b] = acc[a][b];
  __syncthreads();
  double2 *gn = G + (size_t)n * Ns * Ns;
  for (int e = threadIdx.x; e < U * 16; e += blockDim.x) {
    const int uu = e / 16, ab = e % 16;
    double2 z = make_double2(0.0, 0.0);
    for (int q = 0; q < KS; q++) {
      const double2 y = part[((size_t)q * U + uu) * 16 + ab];
      z.x += y.x;
      z.y += y.y;
    }
    int a0 = 0, r = uu;
    while (r >= nt - a0) {
      r -= nt - a0;
      a0++;
    }
    const int k = 4 * a0 + ab / 4, l = 4 * (a0 + r) + ab % 4;
    if (k < Ns && l < Ns && k <= l) {
      gn[k * Ns + l] = z;
      gn[l * Ns + k] = make_double2(z.x, -z.y);
    }
  }
}

// G_tot = sum over nb block matrices
__global__ void k_gram_sum(int nb, int nn, const double2 *__restrict__ G, double2 *out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nn) return;
  double re = 0.0, im = 0.0;
  for (int n = 0; n < nb; n++) {
    const double2 x = G[(size_t)n * nn + e];
    re += x.x;
    im += x.y;
  }
  out[e] = make_double2(re, im);
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zcmul(double2 a, double2 b) {   // conj(a) b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// one warp per matrix: Cholesky G = R^H R (R upper, real positive diagonal)
// in shared memory, then T = R^-1 (upper triangular, lower part zero)
__global__ void k_chol_inv(int Ns, const double2 *__restrict__ G, double2 *T, int *fail) {
  extern __shared__ double2 cA[];
  const int lane = threadIdx.x;
  const double2 *gm = G + (size_t)blockIdx.x * Ns * Ns;
  double2 *tm = T + (size_t)blockIdx.x * Ns * Ns;
  for (int e = lane; e < Ns * Ns; e += 32) cA[e] = gm[e];
  __syncwarp();
  bool bad = false;
  for (int j = 0; j < Ns; j++) {
    double d = cA[j * Ns + j].x;
    for (int k = 0; k < j; k++) {
      const double2 r = cA[k * Ns + j];
      d -= r.x * r.x + r.y * r.y;
    }
    bad |= !(d > 0.0);
    const double rjj = d > 0.0 ? sqrt(d) : 1.0;
    __syncwarp();
    for (int i = j + 1 + lane; i < Ns; i += 32) {
      double2 z = cA[j * Ns + i];
      for (int k = 0; k < j; k++) {
        const double2 t = zcmul(cA[k * Ns + j], cA[k * Ns + i]);
        z.x -= t.x;
        z.y -= t.y;
      }
      cA[j * Ns + i] = make_double2(z.x / rjj, z.y / rjj);
    }
    __syncwarp();
    if (lane == 0) cA[j * Ns + j] = make_double2(rjj, 0.0);
    __syncwarp();
  }
  if (bad && lane == 0) atomicOr(fail, 1);
  // back substitution, one column of T per lane: R T = 1
  for (int j = lane; j < Ns; j += 32) {
    for (int i = Ns - 1; i > j; i--) tm[i * Ns + j] = make_double2(0.0, 0.0);
    for (int i = j; i >= 0; i--) {
      const double rii = cA[i * Ns + i].x;
      if (i == j) {
        tm[i * Ns + j] = make_double2(1.0 / rii, 0.0);
        continue;
      }
      double2 s = make_double2(0.0, 0.0);
      for (int k = i + 1; k <= j; k++) {
        const double2 t = zmul(cA[i * Ns + k], tm[k * Ns + j]);
        s.x += t.x;
        s.y += t.y;
      }
      tm[i * Ns + j] = make_double2(-s.x / rii, -s.y / rii);
    }
  }
}

// block n: w_l = sum_{k<=l} v_k T_kl, T = T0 + n * tstride (tstride 0: the
// same matrix for every block); w may be v (the tile is read before the
// writes of its sites).  A thread forms four outputs l = 4q..4q+3 of one
// site and one float4 plane, so the tile values it loads serve four T
// entries (broadcast across the warp, whose lanes share q).
__global__ void __launch_bounds__(256) k_blk_apply(Geom g, const int *__restrict__ vd2lex, const float4 *const *v,
                                                   float4 *const *w, int Ns, int S, const double2 *__restrict__ T0,
                                                   size_t tstride) {
  extern __shared__ float2 atile[];
  const int ld = S * GSS + 1;
  double2 *Ts = (double2 *)(atile + (((size_t)Ns * ld + 1) & ~(size_t)1));
  const int n = blockIdx.x, blk = __ldg(vd2lex + n);
  const double2 *T = T0 + (size_t)n * tstride;
  for (int e = threadIdx.x; e < Ns * Ns; e += blockDim.x) Ts[e] = T[e];
  const int nsite = 2 * g.vbh, nq = (Ns + 3) / 4;
  for (int s0 = 0; s0 < nsite; s0 += S) {
    __syncthreads();
    load_tile(g, blk, v, Ns, S, s0, atile, ld);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nq * S * 6; idx += blockDim.x) {
      const int s = idx % S, j = (idx / S) % 6, q = idx / (6 * S);
      const int t = s0 + s;
      if (t >= nsite) continue;
      double2 z0[4], z1[4];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        z0[c] = make_double2(0.0, 0.0);
        z1[c] = make_double2(0.0, 0.0);
      }
      const int lmax = min(4 * q + 3, Ns - 1);
      for (int k = 0; k <= lmax; k++) {
        const float2 *row = atile + (size_t)k * ld + s * GSS + 2 * j;
        const float2 fa = row[0], fb = row[1];
        const double ar = fa.x, ai = fa.y, br = fb.x, bi = fb.y;
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int l = 4 * q + c;
          if (l >= Ns || k > l) continue;
          const double2 tk = Ts[k * Ns + l];
          z0[c].x += ar * tk.x - ai * tk.y;
          z0[c].y += ar * tk.y + ai * tk.x;
          z1[c].x += br * tk.x - bi * tk.y;
          z1[c].y += br * tk.y + bi * tk.x;
        }
      }
      const int p = t >= g.vbh, si = t - p * g.vbh, chunk = p * g.nbl + blk;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int l = 4 * q + c;
        if (l < Ns)
          w[l][((size_t)chunk * 6 + j) * g.vbh + si] =
              make_float4((float)z0[c].x, (float)z0[c].y, (float)z1[c].x, (float)z1[c].y);
      }
    }
  }
}

// ------------------------------------------------------------------ host
// sites per shared-memory tile: 16 lets three CTAs share an SM for Ns = 28
// (180 -> 161 ms per two-pass subspace at 48^3x96 against 32-site tiles)
static int gram_tile_sites(int Ns) { return Ns <= 32 ? 16 : 8; }

// shared memory of the Gram kernel: the tile with its rows padded to a
// multiple of four, or the split-K partial sums, whichever is larger
static size_t gram_smem(int Ns, int S) {
  const int nt = (Ns + 3) / 4, U = nt * (nt + 1) / 2, KS = std::max(1, 256 / U);
  const size_t tile = (size_t)4 * nt * (S * GSS + 1) * sizeof(float2);
  const size_t part = (size_t)KS * U * 16 * sizeof(double2);
  return std::max(tile, part);
}

static int gram_alloc(Ctx &c) {
  DflState &d = c.dfl;
  const size_t nn = (size_t)d.Ns * d.Ns;
  if (!d.gram && cudaMalloc(&d.gram, (size_t)(d.nb + 1) * nn * sizeof(double2)) != cudaSuccess)
    return fail("out of device memory (Gram matrices)");
  if (!d.tri && cudaMalloc(&d.tri, (size_t)d.nb * nn * sizeof(double2)) != cudaSuccess)
    return fail("out of device memory (Gram matrices)");
  if (!d.gfail && cudaMalloc(&d.gfail, sizeof(int)) != cudaSuccess) return fail("out of device memory");
  return 0;
}

bool gram_supported(const Ctx &c) { return c.dfl.Ns <= 64; }   // 136 4x4 tiles at most: one per thread

// one Cholesky-QR pass: w = orthonormalised v, per block (global = false)
// or over the whole lattice (global = true); returns 1 if a Gram matrix was
// not positive definite
static int cholqr_pass(Ctx &c, const float4 *const *dv, float4 *const *dw, bool global, cudaStream_t st) {
  DflState &d = c.dfl;
  const int Ns = d.Ns, S = gram_tile_sites(Ns);
  const size_t nn = (size_t)Ns * Ns;
  const size_t tile_bytes = (size_t)Ns * (S * GSS + 1) * sizeof(float2);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_blk_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_blk_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr = true;
  }
  k_blk_gram<<<d.nb, 256, gram_smem(Ns, S), st>>>(c.g, d.vd2lex, dv, Ns, S, d.gram);
  cudaMemsetAsync(d.gfail, 0, sizeof(int), st);
  const size_t csm = nn * sizeof(double2);
  if (global) {
    double2 *gt = d.gram + (size_t)d.nb * nn;
    k_gram_sum<<<(unsigned)((nn + 127) / 128), 128, 0, st>>>(d.nb, (int)nn, d.gram, gt);
    k_chol_inv<<<1, 32, csm, st>>>(Ns, gt, d.tri, d.gfail);
  } else {
    k_chol_inv<<<d.nb, 32, csm, st>>>(Ns, d.gram, d.tri, d.gfail);
  }
  const size_t asm_bytes = ((tile_bytes + 15) & ~(size_t)15) + csm;
  k_blk_apply<<<d.nb, 256, asm_bytes, st>>>(c.g, d.vd2lex, dv, dw, Ns, S, d.tri, global ? 0 : nn);
  int hf = 0;
  cudaMemcpyAsync(&hf, d.gfail, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("Cholesky QR: CUDA error");
  return hf ? 1 : 0;
}

// v -> w orthonormalised (two passes), per block or over the lattice;
// v and w are device tables of Ns FP32 fields (w may equal v).  Returns 0,
// 1 if the vectors are linearly dependent, -1 on an error.
int dfl_cholqr(Ctx &c, const float4 *const *dv, float4 *const *dw, bool global, cudaStream_t st) {
  if (gram_alloc(c)) return -1;
  int rc = cholqr_pass(c, dv, dw, global, st);
  if (rc) return rc;
  return cholqr_pass(c, dw, dw, global, st);
}

}  // namespace qcd
