// Deflation for several right-hand sides at once: restriction,
// prolongation, the little Dirac operator and the little solver applied to
// NR fields / little vectors in one pass over the block basis and the
// little-operator matrices, which dominate the memory traffic of these
// steps (Ns FP32 basis fields, 8 nb Ns^2 FP64 matrix entries).  Each system
// keeps its own arithmetic: the results equal those of the single-system
// routines of dfl.cu up to the summation order.
#include "lib.h"
#include "tma.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace qcd {

constexpr int BT = 4;            // right-hand sides per pass over the basis / matrices

// the fields or vectors of one pass, passed to the kernels by value
template <int N> struct Ptrs {
  void *p[N];
};
constexpr int BSPLIT_T = 352;    // threads of a restriction/prolongation CTA

// sites of one parity chunk are split over nsplit CTAs of at most BSPLIT_T
// threads, one site per thread
static int chunk_split(int vbh) { return (vbh + BSPLIT_T - 1) / BSPLIT_T; }

// ------------------------------------------------------------- restriction
// part[(n, y, r, l)] = (basis_l, x_r) over the sites of CTA y of block n
template <int NRT>
__global__ void __launch_bounds__(BSPLIT_T) k_restrict_b(Geom g, const int *__restrict__ vd2lex,
                                                         const float4 *const *__restrict__ basis, int Ns,
                                                         Ptrs<NRT> x, int nsplit, double2 *part) {
  extern __shared__ double2 red[];   // [Ns][NRT][nw]
  const int n = blockIdx.x, y = blockIdx.y, p = y / nsplit, h = y - p * nsplit;
  const int blk = __ldg(vd2lex + n), chunk = p * g.nbl + blk;
  const int per = (g.vbh + nsplit - 1) / nsplit, si = h * per + threadIdx.x;
  const bool ok = (int)threadIdx.x < per && si < g.vbh;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  spinor<float> xs[NRT];
#pragma unroll
  for (int r = 0; r < NRT; r++) {
    szero(xs[r]);
    if (ok) xs[r] = Store<float>::load_spinor(x.p[r], chunk, si, g.vbh);
  }
  for (int l = 0; l < Ns; l++) {
    spinor<float> b;
    szero(b);
    if (ok) b = Store<float>::load_spinor(basis[l], chunk, si, g.vbh);
#pragma unroll
    for (int r = 0; r < NRT; r++) {
      float sr = 0.0f, sim = 0.0f;
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const cpx<float> bb = b.c[a].c[k], xx = xs[r].c[a].c[k];
          sr += bb.re * xx.re + bb.im * xx.im;
          sim += bb.re * xx.im - bb.im * xx.re;
        }
      double re = sr, im = sim;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
      }
      if (lane == 0) red[((size_t)l * NRT + r) * nw + wp] = make_double2(re, im);
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < Ns * NRT; q += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < nw; w++) {
      re += red[(size_t)q * nw + w].x;
      im += red[(size_t)q * nw + w].y;
    }
    const int l = q / NRT, r = q - l * NRT;
    part[(((size_t)n * gridDim.y + y) * NRT + r) * Ns + l] = make_double2(re, im);
  }
}

// vd_r[n*Ns + l] = sum_y part[(n, y, r, l)], rounded to float
template <int NRT>
__global__ void k_restrict_b_fin(const double2 *__restrict__ part, int Ns, int nb, int ny, Ptrs<NRT> vd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (i >= nb * Ns) return;
  const int n = i / Ns, l = i - n * Ns;
  double re = 0.0, im = 0.0;
  for (int y = 0; y < ny; y++) {
    const double2 a = part[(((size_t)n * ny + y) * NRT + r) * Ns + l];
    re += a.x;
    im += a.y;
  }
  ((double2 *)vd.p[r])[i] = make_double2((double)(float)re, (double)(float)im);
}

// ------------------------------------------------------------ prolongation
// s_r = sum_l vd_r[n, l] basis_l on every block n, float coefficients
template <int NRT>
__global__ void __launch_bounds__(BSPLIT_T) k_prolong_b(Geom g, const int *__restrict__ vd2lex,
                                                        const float4 *const *__restrict__ basis, int Ns,
                                                        Ptrs<NRT> vd, int nsplit, Ptrs<NRT> s) {
  __shared__ float2 z[NRT][64];
  const int n = blockIdx.x, y = blockIdx.y, p = y / nsplit, h = y - p * nsplit;
  const int blk = __ldg(vd2lex + n), chunk = p * g.nbl + blk;
  for (int q = threadIdx.x; q < NRT * Ns; q += blockDim.x) {
    const int r = q / Ns, l = q - r * Ns;
    const double2 v = ((const double2 *)vd.p[r])[(size_t)n * Ns + l];
    z[r][l] = make_float2((float)v.x, (float)v.y);
  }
  __syncthreads();
  const int per = (g.vbh + nsplit - 1) / nsplit, si = h * per + threadIdx.x;
  if ((int)threadIdx.x >= per || si >= g.vbh) return;
  spinor<float> acc[NRT];
#pragma unroll
  for (int r = 0; r < NRT; r++) szero(acc[r]);
  for (int l = 0; l < Ns; l++) {
    const spinor<float> b = Store<float>::load_spinor(basis[l], chunk, si, g.vbh);
#pragma unroll
    for (int r = 0; r < NRT; r++) {
      const float zr = z[r][l].x, zi = z[r][l].y;
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
          acc[r].c[a].c[k].re += zr * b.c[a].c[k].re - zi * b.c[a].c[k].im;
          acc[r].c[a].c[k].im += zr * b.c[a].c[k].im + zi * b.c[a].c[k].re;
        }
    }
  }
#pragma unroll
  for (int r = 0; r < NRT; r++) Store<float>::store_spinor(s.p[r], chunk, si, g.vbh, acc[r]);
}

// -------------------------------------------------- little operator, NR vectors
// The modes of k_little_w (dfl.cu) applied to NRT vectors v_r, u_r -> w_r:
// every matrix entry is loaded once for all of them.
template <int NRT>
__global__ void __launch_bounds__(288) k_little_b(int mode, int Ns, int b0, const double2 *__restrict__ Ablk,
                                                  const double2 *__restrict__ H, const int *__restrict__ nbr,
                                                  Ptrs<NRT> v, Ptrs<NRT> u, Ptrs<NRT> w) {
  __shared__ double2 part[9][64][NRT];
  const int n = b0 + blockIdx.x, wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const bool diag = mode == 3 || wp == 8;
  const double2 *a = diag ? Ablk + (size_t)n * Ns * Ns : H + ((size_t)8 * n + wp) * Ns * Ns;
  const size_t xoff = diag ? (size_t)n * Ns : (size_t)__ldg(nbr + 8 * n + wp) * Ns;
  const Ptrs<NRT> &src = (!diag && mode == 2) ? u : v;
#pragma unroll
  for (int hh = 0; hh < 2; hh++) {
    const int k = lane + 32 * hh;
    if (k < Ns) {
      double re[NRT], im[NRT];
#pragma unroll
      for (int r = 0; r < NRT; r++) re[r] = im[r] = 0.0;
      for (int l = 0; l < Ns; l++) {
        const double2 aa = __ldg(a + (size_t)l * Ns + k);
#pragma unroll
        for (int r = 0; r < NRT; r++) {
          const double2 xx = __ldg((const double2 *)src.p[r] + xoff + l);
          re[r] += aa.x * xx.x - aa.y * xx.y;
          im[r] += aa.x * xx.y + aa.y * xx.x;
        }
      }
#pragma unroll
      for (int r = 0; r < NRT; r++) part[wp][k][r] = make_double2(re[r], im[r]);
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < Ns * NRT; q += blockDim.x) {
    const int k = q / NRT, r = q - k * NRT;
    double re = 0.0, im = 0.0;
    for (int j = 0; j < nw; j++) {
      re += part[j][k][r].x;
      im += part[j][k][r].y;
    }
    if (mode == 2) {
      const double2 vv = ((const double2 *)v.p[r])[(size_t)n * Ns + k];
      ((double2 *)w.p[r])[(size_t)n * Ns + k] = make_double2(vv.x - re, vv.y - im);
    } else {
      ((double2 *)w.p[r])[(size_t)n * Ns + k] = make_double2(re, im);
    }
  }
}

// ----------------------------------------------- TMA-staged variants
constexpr int NSTAGE = 3;        // depth of the shared-memory copy ring
// The same restriction and prolongation with the basis planes of the
// CTA's sites streamed into shared memory by bulk asynchronous copies
// (cp.async.bulk, one per plane and basis vector, issued by one thread),
// in a ring of NSTAGE buffers so that the copies of basis vectors l+1 ..
// l+NSTAGE-1 overlap the arithmetic on vector l.  A plane segment is cnt consecutive float4 at
// ((chunk*6 + j)*vbh + s0): 16-byte aligned, cnt*16 bytes.
template <int NRT, bool RESTRICT>
__global__ void __launch_bounds__(BSPLIT_T) k_dfl_stream(Geom g, const int *__restrict__ vd2lex,
                                                         const float4 *const *__restrict__ basis, int Ns,
                                                         Ptrs<NRT> fld, Ptrs<NRT> vd, int nsplit, double2 *part,
                                                         int *err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar[NSTAGE];
  __shared__ float2 z[RESTRICT ? 1 : NRT][64];
  const int n = blockIdx.x, y = blockIdx.y, p = y / nsplit, h = y - p * nsplit;
  const int blk = __ldg(vd2lex + n), chunk = p * g.nbl + blk;
  const int per = (g.vbh + nsplit - 1) / nsplit, s0 = h * per, cnt = min(per, g.vbh - s0);
  const int si = s0 + threadIdx.x;
  const bool ok = (int)threadIdx.x < cnt;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float4 *buf = (float4 *)smraw;                                  // [NSTAGE][6][per]
  double2 *red = (double2 *)(buf + (size_t)NSTAGE * 6 * per);     // [Ns][NRT][nw]
  const unsigned bytes = (unsigned)cnt * 16u;
  if (threadIdx.x == 0) {
    for (int k = 0; k < NSTAGE; k++) mbar_init(&bar[k], 1);
    mbar_fence_init();
  }
  if (!RESTRICT)
    for (int q = threadIdx.x; q < NRT * Ns; q += blockDim.x) {
      const int r = q / Ns, l = q - r * Ns;
      const double2 v = ((const double2 *)vd.p[r])[(size_t)n * Ns + l];
      z[r][l] = make_float2((float)v.x, (float)v.y);
    }
  __syncthreads();
  auto issue = [&](int l, int stg) {
    mbar_expect_tx(&bar[stg], 6u * bytes);
    const float4 *src = basis[l] + (size_t)chunk * 6 * g.vbh + s0;
#pragma unroll
    for (int j = 0; j < 6; j++) bulk_g2s(buf + ((size_t)stg * 6 + j) * per, src + (size_t)j * g.vbh, bytes, &bar[stg]);
  };
  spinor<float> xs[NRT];
#pragma unroll
  for (int r = 0; r < NRT; r++) {
    szero(xs[r]);
    if (RESTRICT && ok) xs[r] = Store<float>::load_spinor(fld.p[r], chunk, si, g.vbh);
  }
  if (threadIdx.x == 0)
    for (int l = 0; l < NSTAGE - 1 && l < Ns; l++) issue(l, l);
  for (int l = 0; l < Ns; l++) {
    const int stg = l % NSTAGE;
    // the buffer of vector l-1 was released by the barrier that ended step l-1
    if (threadIdx.x == 0 && l + NSTAGE - 1 < Ns) issue(l + NSTAGE - 1, (l + NSTAGE - 1) % NSTAGE);
    mbar_wait(&bar[stg], (unsigned)(l / NSTAGE) & 1u, err);
    spinor<float> b;
    szero(b);
    if (ok)
#pragma unroll
      for (int j = 0; j < 6; j++) {
        const float4 v = buf[((size_t)stg * 6 + j) * per + threadIdx.x];
        const int k = 2 * j;
        b.c[k / 3].c[k % 3] = mk<float>(v.x, v.y);
        b.c[(k + 1) / 3].c[(k + 1) % 3] = mk<float>(v.z, v.w);
      }
    if constexpr (RESTRICT && NRT == 4) {
      // the 8 sums of a warp (4 fields x re, im) by a reduce-scatter
      // butterfly: 9 shuffles instead of 40; lane L ends with the sum of
      // value (L>>4 & 1)*4 + (L>>3 & 1)*2 + (L>>2 & 1)
      float v[8];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        float sr = 0.0f, sim = 0.0f;
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int k = 0; k < 3; k++) {
            const cpx<float> bb = b.c[a].c[k], xx = xs[r].c[a].c[k];
            sr += bb.re * xx.re + bb.im * xx.im;
            sim += bb.re * xx.im - bb.im * xx.re;
          }
        v[2 * r] = sr;
        v[2 * r + 1] = sim;
      }
      const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const float snd = h16 ? v[i] : v[i + 4], keep = h16 ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, snd, 16);
      }
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const float snd = h8 ? v[i] : v[i + 2], keep = h8 ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, snd, 8);
      }
      {
        const float snd = h4 ? v[0] : v[1], keep = h4 ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, snd, 4);
      }
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
      if ((lane & 3) == 0) {
        const int idx = (h16 ? 4 : 0) + (h8 ? 2 : 0) + (h4 ? 1 : 0), r = idx >> 1;
        double2 *dst = &red[((size_t)l * NRT + r) * nw + wp];
        if (idx & 1) dst->y = v[0];
        else dst->x = v[0];
      }
    } else
#pragma unroll
    for (int r = 0; r < NRT; r++) {
      if (RESTRICT) {
        float sr = 0.0f, sim = 0.0f;
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int k = 0; k < 3; k++) {
            const cpx<float> bb = b.c[a].c[k], xx = xs[r].c[a].c[k];
            sr += bb.re * xx.re + bb.im * xx.im;
            sim += bb.re * xx.im - bb.im * xx.re;
          }
        // a warp's 32 site products are summed in FP32 (the result is
        // rounded to FP32), the warps' sums in double
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          sr += __shfl_down_sync(0xffffffffu, sr, o);
          sim += __shfl_down_sync(0xffffffffu, sim, o);
        }
        if (lane == 0) red[((size_t)l * NRT + r) * nw + wp] = make_double2(sr, sim);
      } else {
        const float zr = z[r][l].x, zi = z[r][l].y;
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int k = 0; k < 3; k++) {
            xs[r].c[a].c[k].re += zr * b.c[a].c[k].re - zi * b.c[a].c[k].im;
            xs[r].c[a].c[k].im += zr * b.c[a].c[k].im + zi * b.c[a].c[k].re;
          }
      }
    }
    __syncthreads();   // buffer stg is refilled by the copy issued in step l + 1
  }
  if (RESTRICT) {
    for (int q = threadIdx.x; q < Ns * NRT; q += blockDim.x) {
      double re = 0.0, im = 0.0;
      for (int w = 0; w < nw; w++) {
        re += red[(size_t)q * nw + w].x;
        im += red[(size_t)q * nw + w].y;
      }
      const int l = q / NRT, r = q - l * NRT;
      part[(((size_t)n * gridDim.y + y) * NRT + r) * Ns + l] = make_double2(re, im);
    }
  } else if (ok) {
#pragma unroll
    for (int r = 0; r < NRT; r++) Store<float>::store_spinor(fld.p[r], chunk, si, g.vbh, xs[r]);
  }
}

// ------------------------------------------------------------ host wrappers
template <int N> static Ptrs<N> ptrs(const void *const *a) {
  Ptrs<N> q;
  for (int i = 0; i < N; i++) q.p[i] = a ? const_cast<void *>(a[i]) : nullptr;
  return q;
}

int dfl_batch_alloc(Ctx &c) {
  DflState &d = c.dfl;
  if (d.bpart) return 0;
  const int ns = chunk_split(c.g.vbh);
  if (cudaMalloc(&d.bpart, (size_t)d.nb * 2 * ns * BT * d.Ns * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&d.kerr, sizeof(int)) != cudaSuccess)
    return fail("out of device memory (batched deflation)");
  cudaMemset(d.kerr, 0, sizeof(int));
  return 0;
}

// 0, or -1 with an error message if a kernel's bounded wait gave up
int dfl_batch_check(Ctx &c) {
  DflState &d = c.dfl;
  if (!d.kerr) return 0;
  int h = 0;
  cudaMemcpy(&h, d.kerr, sizeof(int), cudaMemcpyDeviceToHost);
  if (h) {
    cudaMemset(d.kerr, 0, sizeof(int));
    return fail("deflation: a bulk copy did not complete in time");
  }
  return 0;
}

template <int NRT>
static void restrict_pass(Ctx &c, const void *const *x, double2 *const *vd, cudaStream_t st) {
  DflState &d = c.dfl;
  const int ns = chunk_split(c.g.vbh), per = (c.g.vbh + ns - 1) / ns, t = (per + 31) / 32 * 32;
  const size_t shm = (size_t)NSTAGE * 6 * per * sizeof(float4) + (size_t)d.Ns * NRT * (t / 32) * sizeof(double2);
  cudaFuncSetAttribute(k_dfl_stream<NRT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  k_dfl_stream<NRT, true><<<dim3(d.nb, 2 * ns), t, shm, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis,
                                                               d.Ns, ptrs<NRT>(x), ptrs<NRT>(nullptr), ns, d.bpart,
                                                               d.kerr);
  const int nn = d.nb * d.Ns;
  k_restrict_b_fin<NRT><<<dim3((nn + 255) / 256, NRT), 256, 0, st>>>(d.bpart, d.Ns, d.nb, 2 * ns,
                                                                      ptrs<NRT>((const void *const *)vd));
}

// RHS tile autotuner: the number of fields per pass of the streamed
// restriction and prolongation (1, 2 or 4), timed once per geometry on the
// first call with four or more fields (on the caller's own data: every tile
// computes the same result) and kept.
namespace {
struct TileTune {
  int vbh = 0, nb = 0, Ns = 0;
  int tile[2] = {BT, BT};            // restriction, prolongation
  float ms[2][3] = {{0, 0, 0}, {0, 0, 0}};
  bool done[2] = {false, false};
};
TileTune g_tile;
}  // namespace

static bool tile_key_changed(const Ctx &c) {
  const DflState &d = c.dfl;
  if (g_tile.vbh == c.g.vbh && g_tile.nb == d.nb && g_tile.Ns == d.Ns) return false;
  g_tile = TileTune();
  g_tile.vbh = c.g.vbh;
  g_tile.nb = d.nb;
  g_tile.Ns = d.Ns;
  return true;
}

template <class F>
static float time_on(cudaStream_t st, F f) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  f();   // warm-up (attributes, caches)
  cudaEventRecord(e0, st);
  f();
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

static void restrict_tiled(Ctx &c, int tile, int nr, const void *const *x, double2 *const *vd, cudaStream_t st) {
  int r = 0;
  if (tile >= 4)
    for (; r + 4 <= nr; r += 4) restrict_pass<4>(c, x + r, vd + r, st);
  if (tile >= 2)
    for (; r + 2 <= nr; r += 2) restrict_pass<2>(c, x + r, vd + r, st);
  for (; r < nr; r++) restrict_pass<1>(c, x + r, vd + r, st);
}

template <int NRT>
static void prolong_pass(Ctx &c, const double2 *const *vd, void *const *s, cudaStream_t st);

static void prolong_tiled(Ctx &c, int tile, int nr, const double2 *const *vd, void *const *s, cudaStream_t st) {
  int r = 0;
  if (tile >= 4)
    for (; r + 4 <= nr; r += 4) prolong_pass<4>(c, vd + r, s + r, st);
  if (tile >= 2)
    for (; r + 2 <= nr; r += 2) prolong_pass<2>(c, vd + r, s + r, st);
  for (; r < nr; r++) prolong_pass<1>(c, vd + r, s + r, st);
}

// vd[r] = restriction of the FP32 fields x[r], r < nr
void dfl_restrict_b(Ctx &c, int nr, const void *const *x, double2 *const *vd, cudaStream_t st) {
  tile_key_changed(c);
  if (nr >= 4 && !g_tile.done[0]) {
    const int tiles[3] = {1, 2, 4};
    int best = 2;
    for (int i = 0; i < 3; i++) {
      g_tile.ms[0][i] = time_on(st, [&]() { restrict_tiled(c, tiles[i], 4, x, vd, st); });
      if (g_tile.ms[0][i] < g_tile.ms[0][best]) best = i;
    }
    g_tile.tile[0] = tiles[best];
    g_tile.done[0] = true;
  }
  restrict_tiled(c, g_tile.tile[0], nr, x, vd, st);
}

int rhs_tiles(const Ctx &c, int *tile, float *ms) {
  (void)c;
  for (int k = 0; k < 2; k++) {
    tile[k] = g_tile.done[k] ? g_tile.tile[k] : 0;
    for (int i = 0; i < 3; i++) ms[3 * k + i] = g_tile.ms[k][i];
  }
  return 0;
}

template <int NRT>
static void prolong_pass(Ctx &c, const double2 *const *vd, void *const *s, cudaStream_t st) {
  DflState &d = c.dfl;
  const int ns = chunk_split(c.g.vbh), per = (c.g.vbh + ns - 1) / ns, t = (per + 31) / 32 * 32;
  const size_t shm = (size_t)NSTAGE * 6 * per * sizeof(float4);
  cudaFuncSetAttribute(k_dfl_stream<NRT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  k_dfl_stream<NRT, false><<<dim3(d.nb, 2 * ns), t, shm, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis,
                                                                d.Ns, ptrs<NRT>((const void *const *)s),
                                                                ptrs<NRT>((const void *const *)vd), ns, nullptr,
                                                                d.kerr);
}

// s[r] = prolongation of the little vectors vd[r], r < nr
void dfl_prolong_b(Ctx &c, int nr, const double2 *const *vd, void *const *s, cudaStream_t st) {
  tile_key_changed(c);
  if (nr >= 4 && !g_tile.done[1]) {
    const int tiles[3] = {1, 2, 4};
    int best = 2;
    for (int i = 0; i < 3; i++) {
      g_tile.ms[1][i] = time_on(st, [&]() { prolong_tiled(c, tiles[i], 4, vd, s, st); });
      if (g_tile.ms[1][i] < g_tile.ms[1][best]) best = i;
    }
    g_tile.tile[1] = tiles[best];
    g_tile.done[1] = true;
  }
  prolong_tiled(c, g_tile.tile[1], nr, vd, s, st);
}

template <int NRT>
static void little_pass(Ctx &c, int mode, int b0, int nblk, const double2 *A, const double2 *H,
                        const double2 *const *v, const double2 *const *u, double2 *const *w, cudaStream_t st) {
  DflState &d = c.dfl;
  const int nw = mode == 3 ? 1 : (mode == 0 ? 9 : 8);
  k_little_b<NRT><<<nblk, 32 * nw, 0, st>>>(mode, d.Ns, b0, A, H, d.nbr, ptrs<NRT>((const void *const *)v),
                                            ptrs<NRT>((const void *const *)u), ptrs<NRT>((const void *const *)w));
}

void little_b(Ctx &c, int nr, int mode, int b0, int nblk, const double2 *A, const double2 *H,
              const double2 *const *v, const double2 *const *u, double2 *const *w, cudaStream_t st) {
  int r = 0;
  for (; r + BT <= nr; r += BT) little_pass<BT>(c, mode, b0, nblk, A, H, v + r, u ? u + r : nullptr, w + r, st);
  for (; r < nr; r++) little_pass<1>(c, mode, b0, nblk, A, H, v + r, u ? u + r : nullptr, w + r, st);
}

// w_r = Awhat v_r (even halves), t_r odd intermediates
void dfl_Awhat_b(Ctx &c, int nr, const double2 *const *v, double2 *const *w, double2 *const *t, cudaStream_t st) {
  DflState &d = c.dfl;
  const int nbh = d.nb / 2;
  little_b(c, nr, 1, nbh, nbh, nullptr, d.Mhop, v, nullptr, t, st);
  little_b(c, nr, 2, 0, nbh, nullptr, d.Mhop, v, (const double2 *const *)t, w, st);
}

void dfl_Aw_b(Ctx &c, int nr, const double2 *const *v, double2 *const *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_b(c, nr, 0, 0, d.nb, d.Ablk, d.Ahop, v, nullptr, w, st);
}

}  // namespace qcd
