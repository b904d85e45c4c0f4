// Deflation for several right-hand sides at once: restriction,
// prolongation, the little Dirac operator and the little solver applied to
// NR fields / little vectors in one pass over the block basis and the
// little-operator matrices, which dominate the memory traffic of these
// steps (Ns FP32 basis fields, 8 nb Ns^2 FP64 matrix entries).  Each system
// keeps its own arithmetic: the results equal those of the single-system
// routines of dfl.cu up to the summation order.
#include "lib.h"
#include "mma.cuh"
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
// Restriction and prolongation of NRT fields on the CUDA cores, one site
// per thread, with the basis planes of the CTA's sites streamed into shared memory by bulk asynchronous copies
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

// ------------------------------------- tensor-core restriction / prolongation
// Four fields at a time as real matrix products on the tensor cores
// (mma.sync m16n8k8, TF32 head/tail operands; mma.cuh).  Each lane copies
// the operand values it will use (the basis, and for the restriction the
// fields) from global memory into its own slots of a
// per-warp shared-memory ring with cp.async, RD - 1 stages ahead of the
// arithmetic: no registers are tied up by loads in flight and no barrier is
// needed, since every lane reads only what it copied itself.
constexpr int TC_W = 4;          // warps of a CTA; one CTA per (DFL block, parity)

__device__ __forceinline__ float f4c(const float4 &v, int q) {
  return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w;
}
__device__ __forceinline__ void *pick4(const Ptrs<4> &a, int i) {
  return i == 0 ? a.p[0] : i == 1 ? a.p[1] : i == 2 ? a.p[2] : a.p[3];
}

// Restriction: C[l][2r] = Re (b_l, x_r), C[l][2r+1] = Im (b_l, x_r) with
//   Re = sum_k B_l[k] X_r[k],  Im = sum_k B_l[k] Xh_r[k],
// k over the 24 reals of each site (re, im interleaved) and Xh = (x_im,
// -x_re) per complex component.  M = 16 basis vectors (MT tiles cover Ns),
// N = 4 fields x (re, im), K = one real component at 8 sites (K row t <->
// site 8 gi + t, row t+4 <-> site 8 gi + t + 4).  A stage of the ring is
// one plane (4 real components) of one group of 8 sites: NV float4 per lane.
// The sums of a warp over a group are added into FP64, the warps' sums in
// FP64; part[(n, p, r, l)] as the CUDA-core kernel writes it (two parities).
template <int MT> struct RestrictTc {
  static constexpr int NV = 2 + 4 * MT;
  static constexpr int RD = MT <= 2 ? 4 : 3;
  static constexpr size_t smem = (size_t)TC_W * RD * NV * 32 * sizeof(float4);
};

template <int MT>
__global__ void __launch_bounds__(32 * TC_W) k_restrict_tc(Geom g, const int *__restrict__ vd2lex,
                                                          const float4 *const *__restrict__ basis, int Ns,
                                                          Ptrs<4> fld, double2 *part) {
  constexpr int NV = RestrictTc<MT>::NV, RD = RestrictTc<MT>::RD;
  extern __shared__ float4 ring[];
  __shared__ double2 red[TC_W][16 * MT][4];
  const int n = blockIdx.x, p = blockIdx.y, chunk = p * g.nbl + __ldg(vd2lex + n);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, gq = lane >> 2, tq = lane & 3;
  const bool imc = gq & 1;
  const size_t off = (size_t)chunk * 6 * g.vbh;
  const float4 *xf = (const float4 *)pick4(fld, gq >> 1) + off;
  const float4 *bp[MT][2];
#pragma unroll
  for (int mt = 0; mt < MT; mt++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int l = 16 * mt + gq + 8 * h;
      bp[mt][h] = l < Ns ? basis[l] + off : nullptr;
    }
  float4 *my = ring + (size_t)w * RD * NV * 32 + lane;
  const int ngrp = (g.vbh + 7) >> 3;
  const int T = w < ngrp ? 6 * ((ngrp - 1 - w) / TC_W + 1) : 0;   // stages of this warp
  auto issue = [&](int t) {
    if (t < T) {
      const int gq6 = t / 6, j = t - 6 * gq6, gi = w + TC_W * gq6;
      const int s0 = 8 * gi + tq, s1 = s0 + 4;
      const bool ok0 = s0 < g.vbh, ok1 = s1 < g.vbh;
      const size_t pj = (size_t)j * g.vbh;
      float4 *dst = my + (size_t)(t % RD) * NV * 32;
      cp_async16(dst, ok0 ? xf + pj + s0 : xf, ok0);
      cp_async16(dst + 32, ok1 ? xf + pj + s1 : xf, ok1);
#pragma unroll
      for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const float4 *b = bp[mt][h];
          // slots 2 + 4 mt + k: k = 0 (row g, K row t), 1 (row g+8, t), 2 (g, t+4), 3 (g+8, t+4)
          cp_async16(dst + (2 + 4 * mt + h) * 32, (b && ok0) ? b + pj + s0 : xf, b && ok0);
          cp_async16(dst + (4 + 4 * mt + h) * 32, (b && ok1) ? b + pj + s1 : xf, b && ok1);
        }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int t = 0; t < RD - 1; t++) issue(t);
  double dacc[MT][4];
  float acc[MT][4];
#pragma unroll
  for (int mt = 0; mt < MT; mt++)
#pragma unroll
    for (int i = 0; i < 4; i++) {
      dacc[mt][i] = 0.0;
      acc[mt][i] = 0.0f;
    }
  for (int t = 0; t < T; t++) {
    issue(t + RD - 1);
    cp_async_wait<RD - 1>();
    const float4 *src = my + (size_t)(t % RD) * NV * 32;
    const float4 x0 = src[0], x1 = src[32];
    const float4 y0 = imc ? make_float4(x0.y, -x0.x, x0.w, -x0.z) : x0;
    const float4 y1 = imc ? make_float4(x1.y, -x1.x, x1.w, -x1.z) : x1;
    float4 a[MT][4];
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
      for (int k = 0; k < 4; k++) a[mt][k] = src[(2 + 4 * mt + k) * 32];
    // the 4 components of the plane (12 products) summed on the tensor
    // cores, then added to acc with round-to-nearest
    float d[MT][4];
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
      for (int i = 0; i < 4; i++) d[mt][i] = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const Tf32x2 bs[2] = {tf32_split(f4c(y0, q)), tf32_split(f4c(y1, q))};
#pragma unroll
      for (int mt = 0; mt < MT; mt++) {
        const Tf32x2 as[4] = {tf32_split(f4c(a[mt][0], q)), tf32_split(f4c(a[mt][1], q)),
                              tf32_split(f4c(a[mt][2], q)), tf32_split(f4c(a[mt][3], q))};
        mma_tf32x3(d[mt], as, bs);
      }
    }
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
      for (int i = 0; i < 4; i++) acc[mt][i] += d[mt][i];
    if (t % 6 == 5) {   // end of a group of 8 sites
#pragma unroll
      for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int i = 0; i < 4; i++) {
          dacc[mt][i] += (double)acc[mt][i];
          acc[mt][i] = 0.0f;
        }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int mt = 0; mt < MT; mt++) {
    red[w][16 * mt + gq][tq] = make_double2(dacc[mt][0], dacc[mt][1]);
    red[w][16 * mt + gq + 8][tq] = make_double2(dacc[mt][2], dacc[mt][3]);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 4 * Ns; q += blockDim.x) {
    const int r = q / Ns, l = q - r * Ns;
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int v = 0; v < TC_W; v++) {
      re += red[v][l][r].x;
      im += red[v][l][r].y;
    }
    part[(((size_t)n * 2 + p) * 4 + r) * Ns + l] = make_double2(re, im);
  }
}

// Prolongation: s_r = sum_l z_{r,l} b_l with z the FP32-rounded little
// vectors.  M = 16 complex components of 8 sites x one plane j (row g <->
// site 8 gi + g, component 2 j; row g+8 <-> the same site, component 2 j +
// 1), N = 4 fields x (re, im), K = 4 basis vectors x (re, im) (K row t <->
// (l = 4 ks + t, re), row t+4 <-> (l, im)):
//   B[(l, re)][(r, re)] = Re z,  B[(l, im)][(r, re)] = -Im z,
//   B[(l, re)][(r, im)] = Im z,  B[(l, im)][(r, im)] = Re z.
// The A fragment of a lane is one float4 of basis vector l at its site
// (a0, a2, a1, a3), its C fragment one float4 of field t there.  The B
// fragments depend only on the block: they are split once per CTA into
// shared memory.  A stage of the ring is one tile with all its k-steps: KS
// float4 per lane.  KS >= (Ns + 3) / 4.
template <int KS> struct ProlongTc {
  static constexpr int RD = 3;
  static constexpr size_t smem = (size_t)TC_W * RD * KS * 32 * sizeof(float4);
};

template <int KS>
__global__ void __launch_bounds__(32 * TC_W) k_prolong_tc(Geom g, const int *__restrict__ vd2lex,
                                                         const float4 *const *__restrict__ basis, int Ns,
                                                         Ptrs<4> vd, Ptrs<4> s) {
  constexpr int RD = ProlongTc<KS>::RD;
  extern __shared__ float4 pring[];
  __shared__ uint4 zf[KS][32];
  __shared__ const float4 *bq[4 * KS];
  const int n = blockIdx.x, p = blockIdx.y, chunk = p * g.nbl + __ldg(vd2lex + n);
  const size_t off = (size_t)chunk * 6 * g.vbh;
  for (int i = threadIdx.x; i < 32 * KS; i += blockDim.x) {
    const int ks = i >> 5, ln = i & 31, gg = ln >> 2, l = 4 * ks + (ln & 3);
    float zr = 0.0f, zi = 0.0f;
    if (l < Ns) {
      const double2 v = ((const double2 *)pick4(vd, gg >> 1))[(size_t)n * Ns + l];
      zr = (float)v.x;
      zi = (float)v.y;
    }
    const Tf32x2 b0 = tf32_split((gg & 1) ? zi : zr), b1 = tf32_split((gg & 1) ? zr : -zi);
    zf[ks][ln] = make_uint4(b0.hi, b0.lo, b1.hi, b1.lo);
  }
  for (int i = threadIdx.x; i < 4 * KS; i += blockDim.x) bq[i] = i < Ns ? basis[i] + off : nullptr;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, gq = lane >> 2, tq = lane & 3;
  float4 *out = (float4 *)pick4(s, tq) + off;
  float4 *my = pring + (size_t)w * RD * KS * 32 + lane;
  const int ntile = ((g.vbh + 7) >> 3) * 6, nks = (Ns + 3) >> 2;
  const int T = w < ntile ? (ntile - 1 - w) / TC_W + 1 : 0;   // tiles of this warp
  const float4 *dummy = bq[0];
  Tf32x2 bs[KS][2];   // this lane's B fragments, the same for every tile
#pragma unroll
  for (int ks = 0; ks < KS; ks++) {
    const uint4 z = zf[ks][lane];
    bs[ks][0] = {z.x, z.y};
    bs[ks][1] = {z.z, z.w};
  }
  auto issue = [&](int t) {
    if (t < T) {
      const int ti = w + TC_W * t, gi = ti / 6, j = ti - 6 * gi, si = 8 * gi + gq;
      const bool ok = si < g.vbh;
      const size_t ia = (size_t)j * g.vbh + si;
      float4 *dst = my + (size_t)(t % RD) * KS * 32;
      for (int ks = 0; ks < nks; ks++) {
        const float4 *b = bq[4 * ks + tq];
        cp_async16(dst + ks * 32, (b && ok) ? b + ia : dummy, b && ok);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int t = 0; t < RD - 1; t++) issue(t);
  for (int t = 0; t < T; t++) {
    issue(t + RD - 1);
    cp_async_wait<RD - 1>();
    const float4 *src = my + (size_t)(t % RD) * KS * 32;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int ks = 0; ks < KS; ks++)
      if (ks < nks) {
        const float4 v = src[ks * 32];
        const Tf32x2 as[4] = {tf32_split(v.x), tf32_split(v.z), tf32_split(v.y), tf32_split(v.w)};
        mma_tf32x3_add(acc, as, bs[ks]);
      }
    const int ti = w + TC_W * t, gi = ti / 6, j = ti - 6 * gi, si = 8 * gi + gq;
    if (si < g.vbh) out[(size_t)j * g.vbh + si] = make_float4(acc[0], acc[1], acc[2], acc[3]);
  }
  cp_async_wait<0>();
}

// ----------------------------- preconditioned little hops on the tensor cores
// The hop part of Awhat (modes 1 and 2 of k_little_b) for four vectors
// with the FP32 copy of the matrices H = Ablk^-1 Ahop (Mhop32) on the
// tensor cores (mma.sync m16n8k8, TF32 head/tail operands, FP32 sums per
// matrix, FP64 across the 8 matrices of a block).  One warp per matrix; for
// matrix A and the vectors x_r (rounded to FP32)
//   W[k][(r, re)] = sum_l Re A[k][l] Re x_r[l] - Im A[k][l] Im x_r[l]
//   W[k][(r, im)] = sum_l Re A[k][l] Im x_r[l] + Im A[k][l] Re x_r[l]
// is a real product with M = 16 rows k per tile (MT tiles), N = 4 vectors
// x (re, im), K = 4 columns l x (re, im): K row t <-> (l = 4 ks + t, re),
// row t+4 <-> (l, im), A[k][(l, re)] = Re A, A[k][(l, im)] = -Im A,
// B[(l, re)][(r, re)] = Re x, B[(l, im)][(r, re)] = Im x,
// B[(l, re)][(r, im)] = Im x, B[(l, im)][(r, im)] = -Re x.
template <int MT>
__global__ void __launch_bounds__(256) k_little_hop_tc(int mode, int Ns, int b0, const float2 *__restrict__ H,
                                                       const int *__restrict__ nbr, Ptrs<4> v, Ptrs<4> u,
                                                       Ptrs<4> w) {
  __shared__ double2 part[8][16 * MT][4];
  const int n = b0 + blockIdx.x, wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float2 *a = H + ((size_t)8 * n + wp) * Ns * Ns;
  const size_t xoff = (size_t)__ldg(nbr + 8 * n + wp) * Ns;
  const Ptrs<4> &src = mode == 2 ? u : v;
  const int gq = lane >> 2, tq = lane & 3;
  const bool imcol = gq & 1;
  const double2 *x = (const double2 *)pick4(src, gq >> 1) + xoff;
  float acc[MT][4];
#pragma unroll
  for (int mt = 0; mt < MT; mt++)
#pragma unroll
    for (int i = 0; i < 4; i++) acc[mt][i] = 0.0f;
  const int nks = (Ns + 3) >> 2;
#pragma unroll 2
  for (int ks = 0; ks < nks; ks++) {
    const int l = 4 * ks + tq;
    const bool lok = l < Ns;
    const double2 xv = lok ? __ldg(x + l) : make_double2(0.0, 0.0);
    const float xr = (float)xv.x, xi = (float)xv.y;
    const Tf32x2 bs[2] = {tf32_split(imcol ? xi : xr), tf32_split(imcol ? -xr : xi)};
    const float2 *al = a + (size_t)l * Ns;
#pragma unroll
    for (int mt = 0; mt < MT; mt++) {
      const int k = 16 * mt + gq;
      const float2 m0 = (lok && k < Ns) ? __ldg(al + k) : make_float2(0.0f, 0.0f);
      const float2 m1 = (lok && k + 8 < Ns) ? __ldg(al + k + 8) : make_float2(0.0f, 0.0f);
      const Tf32x2 as[4] = {tf32_split(m0.x), tf32_split(m1.x), tf32_split(-m0.y), tf32_split(-m1.y)};
      mma_tf32x3_add(acc[mt], as, bs);
    }
  }
#pragma unroll
  for (int mt = 0; mt < MT; mt++) {
    part[wp][16 * mt + gq][tq] = make_double2(acc[mt][0], acc[mt][1]);
    part[wp][16 * mt + gq + 8][tq] = make_double2(acc[mt][2], acc[mt][3]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Ns * 4; i += blockDim.x) {
    const int k = i >> 2, r = i & 3;
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      re += part[j][k][r].x;
      im += part[j][k][r].y;
    }
    double2 *wr = (double2 *)pick4(w, r) + (size_t)n * Ns + k;
    if (mode == 2) {
      const double2 vv = ((const double2 *)pick4(v, r))[(size_t)n * Ns + k];
      *wr = make_double2(vv.x - re, vv.y - im);
    } else {
      *wr = make_double2(re, im);
    }
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

template <int MT>
static void restrict_tc(Ctx &c, const void *const *x, cudaStream_t st) {
  DflState &d = c.dfl;
  const size_t shm = RestrictTc<MT>::smem;
  cudaFuncSetAttribute(k_restrict_tc<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  k_restrict_tc<MT><<<dim3(d.nb, 2), 32 * TC_W, shm, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis, d.Ns,
                                                            ptrs<4>(x), d.bpart);
}

// four fields (TC) or NRT fields on the CUDA cores
template <int NRT>
static void restrict_pass(Ctx &c, const void *const *x, double2 *const *vd, bool tc, cudaStream_t st) {
  DflState &d = c.dfl;
  const int nn = d.nb * d.Ns;
  if (NRT == 4 && tc) {
    const int mt = (d.Ns + 15) / 16;
    if (mt == 1) restrict_tc<1>(c, x, st);
    else if (mt == 2) restrict_tc<2>(c, x, st);
    else if (mt == 3) restrict_tc<3>(c, x, st);
    else restrict_tc<4>(c, x, st);
    k_restrict_b_fin<4><<<dim3((nn + 255) / 256, 4), 256, 0, st>>>(d.bpart, d.Ns, d.nb, 2,
                                                                    ptrs<4>((const void *const *)vd));
    return;
  }
  const int ns = chunk_split(c.g.vbh), per = (c.g.vbh + ns - 1) / ns, t = (per + 31) / 32 * 32;
  const size_t shm = (size_t)NSTAGE * 6 * per * sizeof(float4) + (size_t)d.Ns * NRT * (t / 32) * sizeof(double2);
  cudaFuncSetAttribute(k_dfl_stream<NRT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  k_dfl_stream<NRT, true><<<dim3(d.nb, 2 * ns), t, shm, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis,
                                                               d.Ns, ptrs<NRT>(x), ptrs<NRT>(nullptr), ns, d.bpart,
                                                               d.kerr);
  k_restrict_b_fin<NRT><<<dim3((nn + 255) / 256, NRT), 256, 0, st>>>(d.bpart, d.Ns, d.nb, 2 * ns,
                                                                      ptrs<NRT>((const void *const *)vd));
}

template <int KS>
static void prolong_tc(Ctx &c, const double2 *const *vd, void *const *s, cudaStream_t st) {
  DflState &d = c.dfl;
  const size_t shm = ProlongTc<KS>::smem;
  cudaFuncSetAttribute(k_prolong_tc<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  k_prolong_tc<KS><<<dim3(d.nb, 2), 32 * TC_W, shm, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis, d.Ns,
                                                           ptrs<4>((const void *const *)vd),
                                                           ptrs<4>((const void *const *)s));
}

template <int NRT>
static void prolong_pass(Ctx &c, const double2 *const *vd, void *const *s, bool tc, cudaStream_t st) {
  DflState &d = c.dfl;
  if (NRT == 4 && tc) {
    const int ks = (d.Ns + 3) / 4;
    if (ks <= 4) prolong_tc<4>(c, vd, s, st);
    else if (ks <= 8) prolong_tc<8>(c, vd, s, st);
    else if (ks <= 12) prolong_tc<12>(c, vd, s, st);
    else prolong_tc<16>(c, vd, s, st);
    return;
  }
  const int ns = chunk_split(c.g.vbh), per = (c.g.vbh + ns - 1) / ns, t = (per + 31) / 32 * 32;
  const size_t shm = (size_t)NSTAGE * 6 * per * sizeof(float4);
  cudaFuncSetAttribute(k_dfl_stream<NRT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  k_dfl_stream<NRT, false><<<dim3(d.nb, 2 * ns), t, shm, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis,
                                                                d.Ns, ptrs<NRT>((const void *const *)s),
                                                                ptrs<NRT>((const void *const *)vd), ns, nullptr,
                                                                d.kerr);
}

// RHS tile autotuner of the restriction and the prolongation (k = 0, 1):
// one, two or four fields per pass on the CUDA cores, or four on the tensor
// cores (kinds 0..3), timed once per geometry and deflation set-up on the
// first call with four or more fields (on the caller's own data: every kind
// computes the same result up to rounding) and kept.
namespace {
constexpr int NKIND = 4;
constexpr int kKindTile[NKIND] = {1, 2, 4, 4};
constexpr bool kKindTc[NKIND] = {false, false, false, true};
struct TileTune {
  int vbh = 0, nb = 0, Ns = 0;
  int kind[2] = {3, 3};
  float ms[2][NKIND] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
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

static void restrict_kind(Ctx &c, int kind, int nr, const void *const *x, double2 *const *vd, cudaStream_t st) {
  const int tile = kKindTile[kind];
  const bool tc = kKindTc[kind];
  int r = 0;
  if (tile >= 4)
    for (; r + 4 <= nr; r += 4) restrict_pass<4>(c, x + r, vd + r, tc, st);
  if (tile >= 2)
    for (; r + 2 <= nr; r += 2) restrict_pass<2>(c, x + r, vd + r, false, st);
  for (; r < nr; r++) restrict_pass<1>(c, x + r, vd + r, false, st);
}

static void prolong_kind(Ctx &c, int kind, int nr, const double2 *const *vd, void *const *s, cudaStream_t st) {
  const int tile = kKindTile[kind];
  const bool tc = kKindTc[kind];
  int r = 0;
  if (tile >= 4)
    for (; r + 4 <= nr; r += 4) prolong_pass<4>(c, vd + r, s + r, tc, st);
  if (tile >= 2)
    for (; r + 2 <= nr; r += 2) prolong_pass<2>(c, vd + r, s + r, false, st);
  for (; r < nr; r++) prolong_pass<1>(c, vd + r, s + r, false, st);
}

template <class F>
static void tune_kind(int k, cudaStream_t st, F run) {
  for (int i = 0; i < NKIND; i++) g_tile.ms[k][i] = time_on(st, [&]() { run(i); });
  int best = NKIND - 1;
  for (int i = 0; i < NKIND; i++)
    if (g_tile.ms[k][i] < g_tile.ms[k][best]) best = i;
  g_tile.kind[k] = best;
  g_tile.done[k] = true;
}

// vd[r] = restriction of the FP32 fields x[r], r < nr
void dfl_restrict_b(Ctx &c, int nr, const void *const *x, double2 *const *vd, cudaStream_t st) {
  tile_key_changed(c);
  if (nr >= 4 && !g_tile.done[0]) tune_kind(0, st, [&](int i) { restrict_kind(c, i, 4, x, vd, st); });
  restrict_kind(c, g_tile.kind[0], nr, x, vd, st);
}

// s[r] = prolongation of the little vectors vd[r], r < nr
void dfl_prolong_b(Ctx &c, int nr, const double2 *const *vd, void *const *s, cudaStream_t st) {
  tile_key_changed(c);
  if (nr >= 4 && !g_tile.done[1]) tune_kind(1, st, [&](int i) { prolong_kind(c, i, 4, vd, s, st); });
  prolong_kind(c, g_tile.kind[1], nr, vd, s, st);
}

// fixes the tiles of the current geometry and deflation set-up (tile 1, 2
// or 4, tc for four fields on the tensor cores; tile 0 hands the choice back
// to the autotuner)
int set_rhs_tiles(Ctx &c, const int *tile, const int *tc) {
  for (int k = 0; k < 2; k++)
    if (tile[k] != 0 && tile[k] != 1 && tile[k] != 2 && tile[k] != 4)
      return fail("set_rhs_tiles: tiles must be 0, 1, 2 or 4");
  tile_key_changed(c);
  for (int k = 0; k < 2; k++) {
    g_tile.done[k] = tile[k] != 0;
    g_tile.kind[k] = tile[k] == 1 ? 0 : tile[k] == 2 ? 1 : (tile[k] == 4 && !tc[k]) ? 2 : 3;
  }
  return 0;
}

int rhs_tiles(const Ctx &c, int *tile, int *tc, float *ms) {
  (void)c;
  for (int k = 0; k < 2; k++) {
    tile[k] = g_tile.done[k] ? kKindTile[g_tile.kind[k]] : 0;
    tc[k] = g_tile.done[k] && kKindTc[g_tile.kind[k]];
    for (int i = 0; i < NKIND; i++) ms[NKIND * k + i] = g_tile.ms[k][i];
  }
  return 0;
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

template <int MT>
static void hop_tc(Ctx &c, int mode, int b0, int nblk, const double2 *const *v, const double2 *const *u,
                   double2 *const *w, cudaStream_t st) {
  DflState &d = c.dfl;
  k_little_hop_tc<MT><<<nblk, 256, 0, st>>>(mode, d.Ns, b0, d.Mhop32, d.nbr, ptrs<4>((const void *const *)v),
                                            ptrs<4>((const void *const *)u), ptrs<4>((const void *const *)w));
}

// modes 1 and 2 with H = Mhop: four vectors at a time on the tensor cores
// (FP32 matrices), the rest on the CUDA cores (FP64 matrices)
static void awhat_hops(Ctx &c, int nr, int mode, int b0, int nblk, const double2 *const *v,
                       const double2 *const *u, double2 *const *w, cudaStream_t st) {
  DflState &d = c.dfl;
  const int mt = (d.Ns + 15) / 16;
  int r = 0;
  for (; r + 4 <= nr; r += 4) {
    const double2 *const *ur = u ? u + r : nullptr;
    if (mt == 1) hop_tc<1>(c, mode, b0, nblk, v + r, ur, w + r, st);
    else if (mt == 2) hop_tc<2>(c, mode, b0, nblk, v + r, ur, w + r, st);
    else if (mt == 3) hop_tc<3>(c, mode, b0, nblk, v + r, ur, w + r, st);
    else hop_tc<4>(c, mode, b0, nblk, v + r, ur, w + r, st);
  }
  for (; r < nr; r++) little_pass<1>(c, mode, b0, nblk, nullptr, d.Mhop, v + r, u ? u + r : nullptr, w + r, st);
}

// w_r = Awhat v_r (even halves), t_r odd intermediates
void dfl_Awhat_b(Ctx &c, int nr, const double2 *const *v, double2 *const *w, double2 *const *t, cudaStream_t st) {
  DflState &d = c.dfl;
  const int nbh = d.nb / 2;
  awhat_hops(c, nr, 1, nbh, nbh, v, nullptr, t, st);
  awhat_hops(c, nr, 2, 0, nbh, v, (const double2 *const *)t, w, st);
}

void dfl_Aw_b(Ctx &c, int nr, const double2 *const *v, double2 *const *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_b(c, nr, 0, 0, d.nb, d.Ablk, d.Ahop, v, nullptr, w, st);
}

}  // namespace qcd
