// Schwarz alternating procedure (SAP) on the device, FP32.
//
// One cycle of the reference's sap() (modules/sap/sap.c:720) visits the
// blocks of colour 0 and then those of colour 1.  For every block of the
// current colour it solves the block Dirac equation with Dirichlet (zero)
// exterior by nmr minimal-residual steps, adds the block solution phi to psi,
// replaces rho on the block by the block residual, and then subtracts the hop
// of phi out of the block from rho on the neighbouring blocks
// (Dw_bnd + sap_com, modules/dirac/Dw_bnd.c:801, modules/sap/sap_com.c:465).
// Blocks of one colour never touch each other, so they run as independent
// CTAs; the exterior update is a separate gather kernel over the sites of the
// other colour.
//
// k_sap_blocks_eo restates the even-odd preconditioned block solve of the
// reference (isolv=1: Dwoo_blk, Dweo_blk, blk_eo_mres, Dwoe_blk, Dwoo_blk,
// update_flds1/2; sap.c:740-767, blk_solv.c:1153, sap.c:618-716);
// k_sap_blocks_plain the plain one (isolv=0: blk_mres, update_flds0;
// blk_solv.c:1117, sap.c:592).  One CTA owns one block: the fields that
// neighbouring sites read (the current even residual, the odd intermediate,
// the even solution) live in shared memory as 24 planes of vbh floats, the
// Dhat image of the residual stays in registers, links and SW matrices come
// through the L1 cache.  Fields that only their own site reads (the odd
// start vector of the eo solve, the solution of the plain solve) are kept in
// the phi output field, so that blocks of up to 768 sites per parity (6^4
// blocks among them) fit into shared memory.
#include "lib.h"
#include <cstring>
#include <cuda_fp16.h>

namespace qcd {

// nsys systems (SAP_MS at most) per launch, with their own fields psi,
// rho, phi and twisted masses; the CTAs of one block are adjacent (CTA x:
// block x / nsys, system x % nsys), so the block's links and SW matrices
// are read by all systems while they are in L2.
struct SapArgs {
  Geom g;
  int colour;
  float mu;             // system 0
  int nmr;
  int eoflg;
  float4 *psi[SAP_MS], *rho[SAP_MS], *phi[SAP_MS];
  const void *u;        // links as the block solver's policy reads them
  const void *ub;       // links for the block-boundary hops (as u, but 18-real FP32 in the FP32 mode)
  const void *sw, *swinv;
  int nsys;
  float mus[SAP_MS];
};

// the fields and twisted mass of system r of a launch
struct SapSys {
  float4 *psi, *rho, *phi;
  float mu;
};
__device__ __forceinline__ SapSys sap_sys(const SapArgs &a, int r) {
  // selected without indexing the parameter arrays by a variable (which
  // would copy them to local memory)
  SapSys y;
  y.psi = a.psi[0];
  y.rho = a.rho[0];
  y.phi = a.phi[0];
  y.mu = a.mus[0];
#pragma unroll
  for (int q = 1; q < SAP_MS; q++)
    if (r == q) {
      y.psi = a.psi[q];
      y.rho = a.rho[q];
      y.phi = a.phi[q];
      y.mu = a.mus[q];
    }
  return y;
}

// block of the given colour with in-colour index h (block lex index of the
// pair 2h, 2h+1 that has the requested parity of sum(n))
__device__ __forceinline__ int block_of_colour(const Geom &g, int h, int colour) {
  int q = 2 * h;
  int n[4];
  unpack4(__ldg(g.bcoord + q), n);
  return q + (((n[0] + n[1] + n[2] + n[3]) & 1) != colour);
}

// Storage policies of the block solver.  All keep the block work vectors
// in shared memory as 6 float4 planes (plane j at sm[4*(j*ld + s)], the
// complex components 2j and 2j+1 of site s: one 16-byte access per pair);
// SapF32
// reads the FP32 links and Pauli matrices, SapF16 FP16 copies of them (links
// as __half2 planes, Pauli matrices as uint2 planes of four halves), with
// all arithmetic in FP32.  (FP16 work vectors were tried: their rounding,
// relative to each cycle's input residual, is of the size of the residual
// reduction of five cycles and cost half as many GCR iterations again.)
struct SapF32 {
  using T = float;
  static constexpr int NP = 24;
  __device__ __forceinline__ static spinor<float> sm_load(const float *sm, int ld, int s) {
    const float4 *p = reinterpret_cast<const float4 *>(sm);
    spinor<float> r;
#pragma unroll
    for (int j = 0; j < 6; j++) {
      const float4 v = p[j * ld + s];
      const int k = 2 * j;
      r.c[k / 3].c[k % 3] = mk<float>(v.x, v.y);
      r.c[(k + 1) / 3].c[(k + 1) % 3] = mk<float>(v.z, v.w);
    }
    return r;
  }
  __device__ __forceinline__ static void sm_store(float *sm, int ld, int s, const spinor<float> &v) {
    float4 *p = reinterpret_cast<float4 *>(sm);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      const int k = 2 * j;
      const cpx<float> a = v.c[k / 3].c[k % 3], b = v.c[(k + 1) / 3].c[(k + 1) % 3];
      p[j * ld + s] = make_float4(a.re, a.im, b.re, b.im);
    }
  }
  __device__ __forceinline__ static su3<float> link(const void *u, int chunk, int mu, int s, int vbh) {
    return Store<float>::load_link(u, chunk, mu, s, vbh);
  }
  // a link of the block-boundary hops (18 reals: the time-boundary sign is stored)
  __device__ __forceinline__ static su3<float> blink(const void *u, int chunk, int mu, int s, int vbh, bool) {
    return link(u, chunk, mu, s, vbh);
  }
  __device__ __forceinline__ static spinor<float> sw(const void *m, int chunk, int s, int vbh, float mu,
                                                     const spinor<float> &in) {
    return apply_sw_site<float>(m, chunk, s, vbh, mu, in);
  }
};

struct SapF16 {
  using T = float;
  static constexpr int NP = 24;
  __device__ __forceinline__ static spinor<float> sm_load(const float *sm, int ld, int s) {
    return SapF32::sm_load(sm, ld, s);
  }
  __device__ __forceinline__ static void sm_store(float *sm, int ld, int s, const spinor<float> &v) {
    SapF32::sm_store(sm, ld, s, v);
  }
  __device__ __forceinline__ static su3<float> link(const void *u, int chunk, int mu, int s, int vbh) {
    const __half2 *p = (const __half2 *)u + ((size_t)chunk * 4 + mu) * 9 * vbh + s;
    su3<float> r;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float2 f = __half22float2(__ldg(p + (size_t)k * vbh));
      r.e[k] = mk<float>(f.x, f.y);
    }
    return r;
  }
  __device__ __forceinline__ static su3<float> blink(const void *u, int chunk, int mu, int s, int vbh, bool) {
    return link(u, chunk, mu, s, vbh);
  }
  __device__ __forceinline__ static spinor<float> sw(const void *m, int chunk, int s, int vbh, float mu,
                                                     const spinor<float> &in) {
    spinor<float> out;
    float u[36];
    cpx<float> w[6], r[6];
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const uint2 *p = (const uint2 *)m + ((size_t)chunk * 18 + 9 * half) * vbh + s;
#pragma unroll
      for (int j = 0; j < 9; j++) {
        uint2 v = __ldg(p + (size_t)j * vbh);
        const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&v.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&v.y));
        u[4 * j] = a.x; u[4 * j + 1] = a.y; u[4 * j + 2] = b.x; u[4 * j + 3] = b.y;
      }
      weyl_get(in, half, w);
      mul_pauli<float>(half == 0 ? mu : -mu, u, w, r);
      weyl_put(out, half, r);
    }
    return out;
  }
};

// FP32 with the links stored as their first two rows (12 reals, planes
// ((chunk*4 + mu)*6 + k)*vbh + s) and the third row rebuilt as the complex
// conjugate of the cross product of the first two, exact for SU(3).  The
// hops inside a block never use the time-boundary links that carry the
// antiperiodic sign (a block does not wrap); the block-boundary hops give
// the sign by position (load_link12).  The library checks every link for
// the relation, with that sign, before it selects this policy.
struct SapF32R {
  using T = float;
  static constexpr int NP = 24;
  __device__ __forceinline__ static spinor<float> sm_load(const float *sm, int ld, int s) {
    return SapF32::sm_load(sm, ld, s);
  }
  __device__ __forceinline__ static void sm_store(float *sm, int ld, int s, const spinor<float> &v) {
    SapF32::sm_store(sm, ld, s, v);
  }
  __device__ __forceinline__ static su3<float> link(const void *u, int chunk, int mu, int s, int vbh) {
    return load_link12(u, chunk, mu, s, vbh, false);
  }
  // a link of the block-boundary hops, which may carry the time-boundary sign
  __device__ __forceinline__ static su3<float> blink(const void *u, int chunk, int mu, int s, int vbh, bool neg) {
    return load_link12(u, chunk, mu, s, vbh, neg);
  }
  __device__ __forceinline__ static spinor<float> sw(const void *m, int chunk, int s, int vbh, float mu,
                                                     const spinor<float> &in) {
    return apply_sw_site<float>(m, chunk, s, vbh, mu, in);
  }
};

// h += H restricted to the block (Dirichlet exterior): hop terms of the
// field in shared memory (parity 1-p) around site (p, s) of block blk.
template <class P>
__device__ __forceinline__ void block_hop_acc(const SapArgs &a, int p, int blk, int s, const typename P::T *src,
                                              int ld, spinor<float> &h) {
  const Geom &g = a.g;
  int y[4];
  unpack4(__ldg(g.lcoord + p * g.vbh + s), y);
  int l = y[0] * g.lstr[0] + y[1] * g.lstr[1] + y[2] * g.lstr[2] + y[3] * g.lstr[3];
  const int chunk = p * g.nbl + blk, ochunk = (1 - p) * g.nbl + blk;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    if (y[mu] + 1 < g.bs[mu]) {
      int s2 = (l + g.lstr[mu]) >> 1;
      spinor<float> sp = P::sm_load(src, ld, s2);
      su3<float> uu = P::link(a.u, chunk, mu, s, g.vbh);
      hop_fwd<float>(mu, uu, sp, h);
    }
    if (y[mu] > 0) {
      int s2 = (l - g.lstr[mu]) >> 1;
      spinor<float> sm = P::sm_load(src, ld, s2);
      su3<float> uu = P::link(a.u, ochunk, mu, s2, g.vbh);
      hop_bwd<float>(mu, uu, sm, h);
    }
  }
}

// -1/2 * H restricted to the block
template <class P>
__device__ __forceinline__ spinor<float> block_hop(const SapArgs &a, int p, int blk, int s,
                                                   const typename P::T *src, int ld) {
  spinor<float> h;
  szero(h);
  block_hop_acc<P>(a, p, blk, s, src, ld, h);
  sscale<float>(h, -0.5f);
  return h;
}

// v = the block's sums of v, the same in every thread (the warps' partial
// sums added in warp order by each thread), with one barrier.  The callers
// separate two reductions by other barriers, so red is never overwritten
// while a thread still reads it.
template <int NC>
__device__ __forceinline__ void block_allreduce(double v[NC], double *red) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NC; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  }
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NC; k++) red[k * 32 + w] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NC; k++) {
    double t = 0.0;
    for (int j = 0; j < nw; j++) t += red[k * 32 + j];
    v[k] = t;
  }
}

// The kernel runs as one loop over phases so that each heavy routine (the
// odd-site hop, the even-site hop, the two SW products) has a single call
// site; with separate set-up, MR and reconstruction code the kernel
// overflowed the instruction cache.
//   step 0         : V = W = A_o^-1 rho_o ;  S1 = rho_e - D_eo W ; S0 = 0
//                    (V is kept in phi_o until the last step)
//   step 1..nmr    : W = A_o^-1 D_oe S1 ;  s2 = (A_e + i mu g5) S1 - D_eo W ;
//                    z = (s2,S1)/|s2|^2 ; S0 += z S1 ; S1 -= z s2
//   step nmr+1     : phi_o = V - A_o^-1 D_oe S0 ; phi_e = S0 ; psi += phi ;
//                    rho_e = S1 ; rho_o = -i mu g5 phi_o (0 with the eo flag)
template <int NS, class P, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_sap_blocks_eo(SapArgs a) {
  using T = typename P::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  const Geom &g = a.g;
  const int ld = g.vbh;
  T *S1 = smem, *W = smem + P::NP * ld, *S0 = smem + 2 * P::NP * ld;
  __shared__ double red[3 * 32];
  const SapSys y = sap_sys(a, blockIdx.x % a.nsys);
  const int blk = block_of_colour(g, blockIdx.x / a.nsys, a.colour);
  const int ce = blk, co = g.nbl + blk;
  const int T_ = blockDim.x;
  const int nmr = a.nmr;
  for (int step = 0; step <= nmr + 1; step++) {
    const bool last = step == nmr + 1;
    // ---- odd sites
#pragma unroll
    for (int k = 0; k < NS; k++) {
      int s = threadIdx.x + k * T_;
      if (s < g.vbh) {
        spinor<float> h;
        if (step == 0) {
          h = Store<float>::load_spinor_rw(y.rho, co, s, g.vbh);
        } else {
          h = block_hop<P>(a, 1, blk, s, last ? S0 : S1, ld);
        }
        spinor<float> t = P::sw(a.swinv, co, s, g.vbh, 0.0f, h);
        if (step == 0) {
          Store<float>::store_spinor(y.phi, co, s, g.vbh, t);
          P::sm_store(W, ld, s, t);
        } else if (!last) {
          P::sm_store(W, ld, s, t);
        } else {
          // one field at a time, so that few spinors are live at once
          spinor<float> ph = Store<float>::load_spinor_rw(y.phi, co, s, g.vbh);
          ssub(ph, t);
          Store<float>::store_spinor(y.phi, co, s, g.vbh, ph);
          {
            spinor<float> ps = Store<float>::load_spinor_rw(y.psi, co, s, g.vbh);
            sadd(ps, ph);
            Store<float>::store_spinor(y.psi, co, s, g.vbh, ps);
          }
          spinor<float> ro;
          if (a.eoflg) {
            szero(ro);
          } else {
#pragma unroll
            for (int c = 0; c < 4; c++) {
              const float m = c < 2 ? -y.mu : y.mu;   // rho_o = i m phi_o
#pragma unroll
              for (int j = 0; j < 3; j++) ro.c[c].c[j] = mk<float>(-m * ph.c[c].c[j].im, m * ph.c[c].c[j].re);
            }
          }
          Store<float>::store_spinor(y.rho, co, s, g.vbh, ro);
        }
      }
    }
    __syncthreads();
    // ---- even sites
    if (last) {
#pragma unroll
      for (int k = 0; k < NS; k++) {
        int s = threadIdx.x + k * T_;
        if (s < g.vbh) {
          const spinor<float> s0 = P::sm_load(S0, ld, s);
          Store<float>::store_spinor(y.phi, ce, s, g.vbh, s0);
          {
            spinor<float> ps = Store<float>::load_spinor_rw(y.psi, ce, s, g.vbh);
            sadd(ps, s0);
            Store<float>::store_spinor(y.psi, ce, s, g.vbh, ps);
          }
          Store<float>::store_spinor(y.rho, ce, s, g.vbh, P::sm_load(S1, ld, s));
        }
      }
      break;
    }
    spinor<float> s2[NS];
    double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < NS; k++) {
      int s = threadIdx.x + k * T_;
      if (s < g.vbh) {
        // base - (-1/2) H W as (2 base + H W) / 2 (exact scalings), with
        // base = rho_e (step 0) or (A_e + i mu g5) S1: the hop accumulates
        // straight into it, so no second spinor is live across the hop
        spinor<float> b2;
        if (step == 0) b2 = Store<float>::load_spinor_rw(y.rho, ce, s, g.vbh);
        else b2 = P::sw(a.sw, ce, s, g.vbh, y.mu, P::sm_load(S1, ld, s));
        sscale<float>(b2, 2.0f);
        block_hop_acc<P>(a, 0, blk, s, W, ld, b2);
        sscale<float>(b2, 0.5f);
        if (step == 0) {
          P::sm_store(S1, ld, s, b2);
          spinor<float> z;
          szero(z);
          P::sm_store(S0, ld, s, z);
        } else {
          const spinor<float> s1 = P::sm_load(S1, ld, s);
          s2[k] = b2;
#pragma unroll
          for (int c = 0; c < 4; c++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
              const cpx<float> x2 = s2[k].c[c].c[j], x1 = s1.c[c].c[j];
              v[0] += (double)x2.re * x2.re + (double)x2.im * x2.im;
              v[1] += (double)x2.re * x1.re + (double)x2.im * x1.im;
              v[2] += (double)x2.re * x1.im - (double)x2.im * x1.re;
            }
        }
      }
    }
    if (step == 0) {
      __syncthreads();
      continue;
    }
    // MR coefficient (blk_solv.c:1153-1188): stop if |s2|^2 < 2 FLT_MIN;
    // every thread has the same sums and computes the same coefficient
    block_allreduce<3>(v, red);
    const float rr = (float)v[0];
    if (rr < 2.0f * 1.17549435e-38f) {
      step = nmr;   // go to the reconstruction step
      continue;
    }
    const float ri = 1.0f / rr, zr = (float)v[1] * ri, zi = (float)v[2] * ri;
#pragma unroll
    for (int k = 0; k < NS; k++) {
      int s = threadIdx.x + k * T_;
      if (s < g.vbh) {
        // plane by plane (two complex components), so that only s2 stays
        // live across the update
        float4 *v1 = reinterpret_cast<float4 *>(S1), *v0 = reinterpret_cast<float4 *>(S0);
#pragma unroll
        for (int jp = 0; jp < 6; jp++) {
          float4 a1 = v1[jp * ld + s], a0 = v0[jp * ld + s];
          const cpx<float> x2 = s2[k].c[(2 * jp) / 3].c[(2 * jp) % 3];
          const cpx<float> y2 = s2[k].c[(2 * jp + 1) / 3].c[(2 * jp + 1) % 3];
          a0.x += zr * a1.x - zi * a1.y;
          a0.y += zr * a1.y + zi * a1.x;
          a0.z += zr * a1.z - zi * a1.w;
          a0.w += zr * a1.w + zi * a1.z;
          a1.x -= zr * x2.re - zi * x2.im;
          a1.y -= zr * x2.im + zi * x2.re;
          a1.z -= zr * y2.re - zi * y2.im;
          a1.w -= zr * y2.im + zi * y2.re;
          v0[jp * ld + s] = a0;
          v1[jp * ld + s] = a1;
        }
      }
    }
    __syncthreads();
  }
}

// Plain MR on the block Dirac operator Dw_blk + i mu g5 (twisted mass off on
// odd sites with the eo flag): all sites, s0/s1 in shared memory, Dw s1 in
// registers.  Sites are handled as (parity, s) pairs.
template <int NS>
__global__ void __launch_bounds__(256) k_sap_blocks_plain(SapArgs a) {
  using P = SapF32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *smem = reinterpret_cast<float *>(smem_raw);
  const Geom &g = a.g;
  const int ld = g.vbh;
  // planes: S1 even, S1 odd; the solution S0 accumulates in phi
  float *S1[2] = {smem, smem + 24 * ld};
  __shared__ double red[3 * 32];
  const SapSys y = sap_sys(a, blockIdx.x % a.nsys);
  const int blk = block_of_colour(g, blockIdx.x / a.nsys, a.colour);
  const int T = blockDim.x;
  const float muo = a.eoflg ? 0.0f : y.mu;

  for (int p = 0; p < 2; p++)
#pragma unroll
    for (int k = 0; k < NS; k++) {
      int s = threadIdx.x + k * T;
      if (s < g.vbh) {
        P::sm_store(S1[p], ld, s, Store<float>::load_spinor_rw(y.rho, p * g.nbl + blk, s, g.vbh));
        spinor<float> z;
        szero(z);
        Store<float>::store_spinor(y.phi, p * g.nbl + blk, s, g.vbh, z);
      }
    }
  __syncthreads();

  for (int imr = 0; imr < a.nmr; imr++) {
    spinor<float> s2[2][NS];
    double v[3] = {0.0, 0.0, 0.0};
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int k = 0; k < NS; k++) {
        int s = threadIdx.x + k * T;
        if (s < g.vbh) {
          spinor<float> s1 = P::sm_load(S1[p], ld, s);
          s2[p][k] = apply_sw_site<float>(a.sw, p * g.nbl + blk, s, g.vbh, p ? muo : y.mu, s1);
          sadd(s2[p][k], block_hop<P>(a, p, blk, s, S1[1 - p], ld));
#pragma unroll
          for (int c = 0; c < 4; c++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
              const cpx<float> x2 = s2[p][k].c[c].c[j], x1 = s1.c[c].c[j];
              v[0] += (double)x2.re * x2.re + (double)x2.im * x2.im;
              v[1] += (double)x2.re * x1.re + (double)x2.im * x1.im;
              v[2] += (double)x2.re * x1.im - (double)x2.im * x1.re;
            }
        }
      }
    block_allreduce<3>(v, red);
    const float rr = (float)v[0];
    if (rr < 2.0f * 1.17549435e-38f) break;
    const float ri = 1.0f / rr, zr = (float)v[1] * ri, zi = (float)v[2] * ri;
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int k = 0; k < NS; k++) {
        int s = threadIdx.x + k * T;
        if (s < g.vbh) {
          const int ch = p * g.nbl + blk;
          spinor<float> s1 = P::sm_load(S1[p], ld, s), s0 = Store<float>::load_spinor_rw(y.phi, ch, s, g.vbh);
#pragma unroll
          for (int c = 0; c < 4; c++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
              cpx<float> x1 = s1.c[c].c[j], x2 = s2[p][k].c[c].c[j];
              s0.c[c].c[j].re += zr * x1.re - zi * x1.im;
              s0.c[c].c[j].im += zr * x1.im + zi * x1.re;
              s1.c[c].c[j].re -= zr * x2.re - zi * x2.im;
              s1.c[c].c[j].im -= zr * x2.im + zi * x2.re;
            }
          Store<float>::store_spinor(y.phi, ch, s, g.vbh, s0);
          P::sm_store(S1[p], ld, s, s1);
        }
      }
    __syncthreads();
  }
  for (int p = 0; p < 2; p++)
#pragma unroll
    for (int k = 0; k < NS; k++) {
      int s = threadIdx.x + k * T;
      if (s < g.vbh) {
        int ch = p * g.nbl + blk;
        spinor<float> s0 = Store<float>::load_spinor_rw(y.phi, ch, s, g.vbh);
        spinor<float> ps = Store<float>::load_spinor_rw(y.psi, ch, s, g.vbh);
        sadd(ps, s0);
        Store<float>::store_spinor(y.psi, ch, s, g.vbh, ps);
        Store<float>::store_spinor(y.rho, ch, s, g.vbh, P::sm_load(S1[p], ld, s));
      }
    }
}

// rho(y) -= D_{y,x} phi(x) for every site y of a block of colour 1-c and every
// neighbour x of y in a (colour c) block: the block-boundary hop of the
// reference's Dw_bnd/sap_com, as a gather.
// 8 resident CTAs per SM (64 registers): two SAP cycles at 48^3x96 with 6^4
// blocks 17.86 ms against 17.99 ms with the compiler's choice (80-87
// registers, 6 CTAs); 12 CTAs (40 registers) spilled
#ifndef SAP_BND_MINB
#define SAP_BND_MINB 8
#endif
template <class P, int DD>
__device__ __forceinline__ void sap_bnd_body(const SapArgs &a, const DDGeom &dg) {
  const Geom &g = a.g;
  const SapSys y = sap_sys(a, blockIdx.x % a.nsys);
  size_t i = (blockIdx.x / a.nsys) * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)(g.nbl / 2) * g.vb) return;
  int h = (int)(i / g.vb), r = (int)(i % g.vb);
  int p = r >= g.vbh, s = r - p * g.vbh;
  int blk = block_of_colour(g, h, 1 - a.colour);
  Site x;
  site_decode(g, p, blk, s, x);
  const int chunk = p * g.nbl + blk;
  // global time coordinate: the time links at x0 = N0-1 carry the boundary sign
  const int x0 = (DD ? dg.x0off : 0) + x.n[0] * g.bs[0] + x.y[0];
  const int xlast = (DD ? dg.N0 : g.L[0]) - 1;
  // DD: the x0-neighbour blocks across the rank boundary are on the other
  // ranks; their hops come from the exchanged faces of phi
  const bool dd_up = DD && x.n[0] + 1 == g.nb[0] && x.y[0] + 1 == g.bs[0];
  const bool dd_dn = DD && x.n[0] == 0 && x.y[0] == 0;
  spinor<float> hsum;
  szero(hsum);
  bool any = false;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    if (crosses_block(g, x, mu, +1)) {
      su3<float> uu = P::blink(a.ub, chunk, mu, s, g.vbh, mu == 0 && x0 == xlast);
      if (mu == 0 && dd_up) {
        vec3<float> h0, h1;
        Half<float>::load(dg.hup, face_sites(g), face_index_of(g, x.n, x.y), h0, h1);
        dd_hop_fwd<float>(uu, h0, h1, hsum);
      } else {
        int c2, s2;
        site_nbr(g, x, mu, +1, c2, s2);
        spinor<float> sp = Store<float>::load_spinor(y.phi, c2, s2, g.vbh);
        hop_fwd<float>(mu, uu, sp, hsum);
      }
      any = true;
    }
    if (crosses_block(g, x, mu, -1)) {
      if (mu == 0 && dd_dn) {
        vec3<float> c0, c1;
        Half<float>::load(dg.hdn, face_sites(g), face_index_of(g, x.n, x.y), c0, c1);
        dd_hop_bwd<float>(c0, c1, hsum);
      } else {
        int c2, s2;
        site_nbr(g, x, mu, -1, c2, s2);
        spinor<float> sm = Store<float>::load_spinor(y.phi, c2, s2, g.vbh);
        su3<float> uu = P::blink(a.ub, c2, mu, s2, g.vbh, mu == 0 && x0 == 0);
        hop_bwd<float>(mu, uu, sm, hsum);
      }
      any = true;
    }
  }
  if (!any) return;
  sscale<float>(hsum, 0.5f);   // rho -= (-1/2) H phi
  spinor<float> rr = Store<float>::load_spinor_rw(y.rho, chunk, s, g.vbh);
  sadd(rr, hsum);
  Store<float>::store_spinor(y.rho, chunk, s, g.vbh, rr);
}

// the single-GPU kernel keeps its parameter list; the DD twin takes the
// slab's geometry with the received faces
template <class P>
__global__ void __launch_bounds__(128, SAP_BND_MINB) k_sap_bnd(SapArgs a) {
  sap_bnd_body<P, 0>(a, DDGeom{0, 0, nullptr, nullptr});
}
template <class P>
__global__ void __launch_bounds__(128, SAP_BND_MINB) k_sap_bnd_dd(SapArgs a, DDGeom dg) {
  sap_bnd_body<P, 1>(a, dg);
}

// DD: the x0-faces of the block solutions phi (FP32 half spinors, as
// k_dd_pack in dd.cu, with the links as the boundary hops read them)
template <class P>
__global__ void k_sap_dd_pack(SapArgs a, DDGeom dg, void *dn, void *up) {
  const Geom &g = a.g;
  const int F = face_sites(g);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * F) return;
  const int side = i >= F, f = i - side * F;
  int chunk, s, n[4], y[4];
  face_site(g, side, f, chunk, s, n, y);
  const spinor<float> v = Store<float>::load_spinor(a.phi[0], chunk, s, g.vbh);
  vec3<float> h0, h1;
  if (side == 0) {
    dd_proj_fwd<float>(v, h0, h1);
    Half<float>::store(dn, F, f, h0, h1);
  } else {
    const su3<float> uu = P::blink(a.ub, chunk, 0, s, g.vbh, dg.x0off + g.L[0] - 1 == dg.N0 - 1);
    dd_proj_bwd<float>(uu, v, h0, h1);
    Half<float>::store(up, F, f, h0, h1);
  }
}

template <class P>
static void sap_bnd_launch(Ctx &c, SapArgs a, cudaStream_t st) {
  const size_t nb_sites = (size_t)(c.g.nbl / 2) * c.g.vb;
  const unsigned nbnd = (unsigned)((nb_sites + 127) / 128);
  DDGeom dg = c.ddg;
  if (!dd_on(c)) {
    k_sap_bnd<P><<<nbnd * a.nsys, 128, 0, st>>>(a);
    return;
  }
  const int F = c.g.L[1] * c.g.L[2] * c.g.L[3];
  k_sap_dd_pack<P><<<(unsigned)((2 * F + 127) / 128), 128, 0, st>>>(a, dg, c.dd.buf[0], c.dd.buf[1]);
  if (dd_exchange(c, (size_t)F * 48, st)) return;
  dg.hup = c.dd.buf[2];
  dg.hdn = c.dd.buf[3];
  k_sap_bnd_dd<P><<<nbnd, 128, 0, st>>>(a, dg);
}

// dynamic shared memory a block kernel may use (of 227 KB per CTA)
static const int SAP_SMEM_MAX = 224 * 1024;

// Threads of the plain block kernel: up to three sites per thread.
static int pick_threads(int vbh, int &ns) {
  for (ns = 1; ns <= 3; ns++) {
    int t = ((vbh + ns - 1) / ns + 31) / 32 * 32;
    if (t <= 256) return t;
  }
  ns = 0;
  return 0;
}

// FP16 copies of the FP32 links and Pauli matrices, same plane indexing
__global__ void k_to_half2(size_t n, const float2 *__restrict__ a, __half2 *b) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float22half2_rn(__ldg(a + i));
}
__global__ void k_to_half4(size_t n, const float4 *__restrict__ a, uint2 *b) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) {
    const float4 v = __ldg(a + i);
    __half2 x = __floats2half2_rn(v.x, v.y), y = __floats2half2_rn(v.z, v.w);
    b[i] = make_uint2(*reinterpret_cast<unsigned *>(&x), *reinterpret_cast<unsigned *>(&y));
  }
}

static int sap_half_fields(Ctx &c, cudaStream_t st) {
  if (c.h16_valid) return 0;
  const size_t nl = (size_t)c.g.vol * 36, np = (size_t)c.g.vol * 18;
  if (!c.u16 && cudaMalloc(&c.u16, nl * sizeof(__half2)) != cudaSuccess) return fail("out of device memory (FP16 links)");
  if (!c.sw16 && cudaMalloc(&c.sw16, np * sizeof(uint2)) != cudaSuccess) return fail("out of device memory (FP16 SW)");
  if (!c.sw16_inv && cudaMalloc(&c.sw16_inv, np * sizeof(uint2)) != cudaSuccess)
    return fail("out of device memory (FP16 SW)");
  k_to_half2<<<(unsigned)((nl + 255) / 256), 256, 0, st>>>(nl, c.u32, (__half2 *)c.u16);
  k_to_half4<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(np, c.sw32, (uint2 *)c.sw16);
  k_to_half4<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(np, c.sw32_inv, (uint2 *)c.sw16_inv);
  if (cudaGetLastError() != cudaSuccess) return fail("sap: FP16 conversion failed");
  c.h16_valid = true;
  return 0;
}

// 12-real copies of the FP32 links (first two rows) and a check that every
// link satisfies row3 = conj(row1 x row2) to FP32 accuracy, with the sign
// flipped on the time links at x0 = N0-1 (the antiperiodic boundary phase
// of bc type 3); bad[0] counts links that do not.
__global__ void k_links12(Geom g, DDGeom dg, size_t nlink, const float2 *__restrict__ u32, float2 *u12, int *bad) {
  const int vbh = g.vbh;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= nlink) return;
  const size_t cm = i / vbh, s = i - cm * vbh;   // cm = chunk*4 + mu
  const int chunk = (int)(cm >> 2), mu = (int)(cm & 3);
  const int par = chunk >= g.nbl;
  Site x;
  site_decode(g, par, chunk - par * g.nbl, (int)s, x);
  const bool neg = mu == 0 && dg.x0off + x.n[0] * g.bs[0] + x.y[0] == dg.N0 - 1;
  const float2 *p = u32 + cm * 9 * vbh + s;
  float2 e[9];
#pragma unroll
  for (int k = 0; k < 9; k++) e[k] = p[(size_t)k * vbh];
  float2 *q = u12 + cm * 6 * vbh + s;
#pragma unroll
  for (int k = 0; k < 6; k++) q[(size_t)k * vbh] = e[k];
  float dp = 0.0f, dm = 0.0f;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int a = (j + 1) % 3, b = (j + 2) % 3;
    const float re = e[a].x * e[3 + b].x - e[a].y * e[3 + b].y - (e[b].x * e[3 + a].x - e[b].y * e[3 + a].y);
    const float im = -(e[a].x * e[3 + b].y + e[a].y * e[3 + b].x - (e[b].x * e[3 + a].y + e[b].y * e[3 + a].x));
    dp = fmaxf(dp, fabsf(re - e[6 + j].x) + fabsf(im - e[6 + j].y));
    dm = fmaxf(dm, fabsf(re + e[6 + j].x) + fabsf(im + e[6 + j].y));
  }
  if ((neg ? dm : dp) > 1e-5f) atomicAdd(bad, 1);
}

static int sap_link12_fields(Ctx &c, cudaStream_t st) {
  if (c.u12_valid) return 0;
  const size_t nlink = (size_t)c.g.vol * 4;
  if (!c.u12 && cudaMalloc(&c.u12, nlink * 6 * sizeof(float2)) != cudaSuccess)
    return fail("out of device memory (12-real links)");
  int *bad = nullptr;
  if (cudaMallocAsync(&bad, sizeof(int), st) != cudaSuccess) return fail("out of device memory");
  cudaMemsetAsync(bad, 0, sizeof(int), st);
  k_links12<<<(unsigned)((nlink + 255) / 256), 256, 0, st>>>(c.g, c.ddg, nlink, c.u32, (float2 *)c.u12, bad);
  int h = 0;
  cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(bad, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("sap: 12-real link conversion failed");
  c.u12_ok = dd_all(c, h == 0) != 0;   // the same choice on every rank
  c.u12_valid = true;
  return 0;
}

// The 12-real FP32 links when they may be read (on, and every link passed
// the check), else null: the FP32 Dirac operators read them too.
const void *links12(Ctx &c, cudaStream_t st) {
  if (!c.sap_link12 || !c.u32) return nullptr;
  if (sap_link12_fields(c, st)) return nullptr;
  return c.u12_ok ? c.u12 : nullptr;
}

// storage mode of the even-odd block solver: 0 FP32, 1 FP16, 2 FP32 with
// 12-real links (the FP32 default when all links pass the SU(3) check)
static int sap_mode(Ctx &c, int isolv, cudaStream_t st) {
  if (!isolv) return 0;
  if (c.sap_prec == 16) return 1;
  if (!c.sap_link12) return 0;
  if (sap_link12_fields(c, st)) return -1;
  return c.u12_ok ? 2 : 0;
}

// Launch variants of the even-odd block kernel: sites per thread, the
// launch bound and the register budget it implies.  The autotuner below
// times every variant that fits the block on the resident fields and keeps
// the fastest per block size and storage mode.
struct EoVariant {
  int ns, maxt;
  void (*k[3])(SapArgs);   // per storage mode
};
static const EoVariant kEo[] = {
    {1, 256, {k_sap_blocks_eo<1, SapF32, 256, 2>, k_sap_blocks_eo<1, SapF16, 256, 2>, k_sap_blocks_eo<1, SapF32R, 256, 2>}},
    {1, 672, {k_sap_blocks_eo<1, SapF32, 672, 1>, k_sap_blocks_eo<1, SapF16, 672, 1>, k_sap_blocks_eo<1, SapF32R, 672, 1>}},
    {2, 384, {k_sap_blocks_eo<2, SapF32, 384, 1>, k_sap_blocks_eo<2, SapF16, 384, 1>, k_sap_blocks_eo<2, SapF32R, 384, 1>}},
    {3, 256, {k_sap_blocks_eo<3, SapF32, 256, 1>, k_sap_blocks_eo<3, SapF16, 256, 1>, k_sap_blocks_eo<3, SapF32R, 256, 1>}},
};
static const int kNEo = sizeof(kEo) / sizeof(kEo[0]);

static int eo_threads(const EoVariant &v, int vbh) {
  int t = ((vbh + v.ns - 1) / v.ns + 31) / 32 * 32;
  return t > v.maxt ? 0 : t;
}

static size_t eo_smem(int vbh) { return (size_t)vbh * 72 * sizeof(float); }

static void launch_blocks(Ctx &c, const SapArgs &a, int isolv, int mode, cudaStream_t st) {
  const int nbh = c.g.nbl / 2;
  if (isolv) {
    const EoVariant &v = kEo[c.sap_variant[mode]];
    const int t = eo_threads(v, c.g.vbh);
    v.k[mode]<<<nbh * a.nsys, t, eo_smem(c.g.vbh), st>>>(a);
  } else {
    int ns;
    int t = pick_threads(c.g.vbh, ns);
    const size_t shm = (size_t)48 * c.g.vbh * sizeof(float);
    if (ns == 1) k_sap_blocks_plain<1><<<nbh * a.nsys, t, shm, st>>>(a);
    else if (ns == 2) k_sap_blocks_plain<2><<<nbh * a.nsys, t, shm, st>>>(a);
    else k_sap_blocks_plain<3><<<nbh * a.nsys, t, shm, st>>>(a);
  }
}

static SapArgs sap_args(Ctx &c, float mu, int nmr, int mode, void *psi, void *rho, void *phi) {
  SapArgs a;
  std::memset(&a, 0, sizeof(a));   // the bytes are also a CUDA-graph key
  const bool half = mode == 1;
  a.g = c.g;
  a.colour = 0;
  a.mu = mu;
  a.nmr = nmr;
  a.eoflg = c.eoflg;
  a.psi[0] = (float4 *)psi;
  a.rho[0] = (float4 *)rho;
  a.phi[0] = (float4 *)phi;
  a.nsys = 1;
  a.mus[0] = mu;
  a.u = half ? (const void *)c.u16 : (mode == 2 ? (const void *)c.u12 : (const void *)c.u32);
  a.ub = half ? (const void *)c.u16 : (mode == 2 ? (const void *)c.u12 : (const void *)c.u32);
  a.sw = half ? (const void *)c.sw16 : (const void *)c.sw32;
  a.swinv = half ? (const void *)c.sw16_inv : (const void *)c.sw32_inv;
  return a;
}

// Time every fitting variant of the even-odd block kernel (both colours, 4
// MR steps, on a random residual) and keep the fastest.
static int sap_autotune(Ctx &c, int mode, cudaStream_t st) {
  if (c.sap_tuned_vbh[mode] == c.g.vbh) return 0;
  for (int i = 0; i < kNEo; i++)
    for (int m = 0; m < 3; m++)
      cudaFuncSetAttribute(kEo[i].k[m], cudaFuncAttributeMaxDynamicSharedMemorySize, SAP_SMEM_MAX);
  if (eo_smem(c.g.vbh) > (size_t)SAP_SMEM_MAX) return fail("sap: block too large for shared memory");
  const size_t nb = spinor_bytes(c, 32);
  void *psi = nullptr, *rho = nullptr, *phi = nullptr;
  if (cudaMallocAsync(&psi, nb, st) != cudaSuccess || cudaMallocAsync(&rho, nb, st) != cudaSuccess ||
      cudaMallocAsync(&phi, nb, st) != cudaSuccess)
    return fail("sap: out of device memory (autotuning)");
  cudaMemsetAsync(psi, 0, nb, st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = -1;
  float best_ms = 0.0f;
  for (int i = 0; i < kNEo; i++) {
    if (!eo_threads(kEo[i], c.g.vbh)) continue;
    c.sap_variant[mode] = i;
    SapArgs a = sap_args(c, 0.0f, 4, mode, psi, rho, phi);
    float tot = 0.0f;
    for (int rep = 0; rep < 4; rep++) {
      gen_uniform_spinor32(c, rho, 977ull + rep, st);
      cudaEventRecord(e0, st);
      for (int ic = 0; ic < 2; ic++) {
        a.colour = ic;
        launch_blocks(c, a, 1, mode, st);
      }
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) tot += ms;   // the first run warms up
    }
    if (cudaGetLastError() != cudaSuccess) continue;   // a variant that cannot launch is skipped
    if (best < 0 || tot < best_ms) {
      best = i;
      best_ms = tot;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(psi, st);
  cudaFreeAsync(rho, st);
  cudaFreeAsync(phi, st);
  if (best < 0) return fail("sap: no block-kernel variant fits this block size");
  best = dd_rank0(c, best);   // every rank runs rank 0's choice (the same arithmetic everywhere)
  c.sap_variant[mode] = best;
  c.sap_tuned_vbh[mode] = c.g.vbh;
  c.sap_tuned_ms[mode] = best_ms / 3.0f;
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : fail("sap: CUDA error while autotuning");
}

int sap_variant_threads(const Ctx &c, int slot) { return eo_threads(kEo[c.sap_variant[slot]], c.g.vbh); }

// Fix the launch variant of the even-odd block kernel for the current block
// size and storage mode (-1: tune again on the next use).
int sap_set_variant(Ctx &c, int v) {
  const int mode = sap_mode(c, 1, c.stream);
  if (mode < 0) return -1;
  if (v < 0) {
    c.sap_tuned_vbh[mode] = 0;
    return 0;
  }
  if (v >= kNEo || !eo_threads(kEo[v], c.g.vbh)) return fail("sap: this launch variant does not fit the block size");
  for (int m = 0; m < 3; m++)
    cudaFuncSetAttribute(kEo[v].k[m], cudaFuncAttributeMaxDynamicSharedMemorySize, SAP_SMEM_MAX);
  c.sap_variant[mode] = v;
  c.sap_tuned_vbh[mode] = c.g.vbh;
  c.sap_tuned_ms[mode] = 0.0f;
  return 0;
}

int sap_prepare(Ctx &c, cudaStream_t st) {
  int ns;
  if (!pick_threads(c.g.vbh, ns)) return fail("sap: block volume too large (at most 1536 sites)");
  static bool attrs = false;
  if (!attrs) {
    cudaFuncSetAttribute(k_sap_blocks_plain<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, SAP_SMEM_MAX);
    cudaFuncSetAttribute(k_sap_blocks_plain<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SAP_SMEM_MAX);
    cudaFuncSetAttribute(k_sap_blocks_plain<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, SAP_SMEM_MAX);
    attrs = true;
  }
  if (c.sap_prec == 16 && sap_half_fields(c, st)) return -1;
  const int mode = sap_mode(c, 1, st);
  if (mode < 0) return -1;
  return sap_autotune(c, mode, st);
}

// storage mode in use (for reports): 0 FP32, 1 FP16, 2 FP32 with 12-real links
int sap_storage_mode(Ctx &c) { return sap_mode(c, 1, c.stream); }

// Everything a SAP cycle needs before its launches (storage mode, derived
// link/SW copies, autotuned variant), done outside any stream capture.
// Returns the storage mode or -1.
static int sap_ready(Ctx &c, int isolv, cudaStream_t st) {
  const int mode = sap_mode(c, isolv, st);
  if (mode < 0) return -1;
  if (isolv && c.sap_tuned_vbh[mode] != c.g.vbh && sap_prepare(c, st)) return -1;
  if (mode == 1 && !c.h16_valid && sap_half_fields(c, st)) return -1;
  int ns;
  if (!pick_threads(c.g.vbh, ns) || (!isolv && (size_t)48 * c.g.vbh * sizeof(float) > (size_t)SAP_SMEM_MAX))
    return fail("sap: block too large");
  return mode;
}

// the launches of one cycle: block solves and boundary updates, colour 0
// then colour 1 (sap.c:720)
static void sap_cycle_launch(Ctx &c, SapArgs a, int isolv, int mode, cudaStream_t st) {
  for (int ic = 0; ic < 2; ic++) {
    a.colour = ic;
    launch_blocks(c, a, isolv, mode, st);
    if (mode == 1) sap_bnd_launch<SapF16>(c, a, st);
    else if (mode == 2) sap_bnd_launch<SapF32R>(c, a, st);
    else sap_bnd_launch<SapF32>(c, a, st);
  }
}

namespace {
struct SapKey {
  int tag, isolv, mode, variant, ncy, pad;
  SapArgs a;
};
}  // namespace

// ph = sap psi (+ add), ch = base - sap rho: the output step of the
// preconditioner (base = rh, or the residual the caller's preconditioner
// started from; add = the part of the solution applied before SAP)
__global__ void k_sap_out(size_t n, const float4 *__restrict__ spsi, const float4 *__restrict__ srho,
                          const float4 *base, const float4 *__restrict__ add, float4 *ph, float4 *ch) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = base[i], b = srho[i];
  float4 p = spsi[i];
  if (add) {
    const float4 q = add[i];
    p = make_float4(p.x + q.x, p.y + q.y, p.z + q.z, p.w + q.w);
  }
  ph[i] = p;
  ch[i] = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

int sap_cycles(Ctx &c, float mu, int isolv, int nmr, int ncy, void *psi, void *rho, void *phi_blk,
               cudaStream_t st) {
  const int mode = sap_ready(c, isolv, st);
  if (mode < 0) return -1;
  const SapArgs a = sap_args(c, mu, nmr, mode, psi, rho, phi_blk);
  for (int n = 0; n < ncy; n++) sap_cycle_launch(c, a, isolv, mode, st);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
}

// ncy cycles for n systems with the same twisted mass on their own fields
// (psi[r], rho[r] in and out, phi_blk[r] scratch), up to SAP_MS systems per
// launch; with domain decomposition one system after the other
int sap_cycles_multi(Ctx &c, int n, float mu, int isolv, int nmr, int ncy, void *const *psi, void *const *rho,
                     void *const *phi_blk, cudaStream_t st) {
  if (dd_on(c)) {
    for (int r = 0; r < n; r++)
      if (sap_cycles(c, mu, isolv, nmr, ncy, psi[r], rho[r], phi_blk[r], st)) return -1;
    return 0;
  }
  const int mode = sap_ready(c, isolv, st);
  if (mode < 0) return -1;
  for (int r0 = 0; r0 < n; r0 += SAP_MS) {
    const int m = n - r0 < SAP_MS ? n - r0 : SAP_MS;
    SapArgs a = sap_args(c, mu, nmr, mode, psi[r0], rho[r0], phi_blk[r0]);
    a.nsys = m;
    for (int r = 0; r < m; r++) {
      a.psi[r] = (float4 *)psi[r0 + r];
      a.rho[r] = (float4 *)rho[r0 + r];
      a.phi[r] = (float4 *)phi_blk[r0 + r];
      a.mus[r] = mu;
    }
    for (int k = 0; k < ncy; k++) sap_cycle_launch(c, a, isolv, mode, st);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
}

// The preconditioner of sap_gcr (sap_gcr.c:126-134): psi = ncy SAP cycles
// from psi = 0 on rho = rh, then rho = rh - rho (= D psi); with base given,
// rho = base - (final residual), and psi += add (the deflated
// preconditioner of dfl_sap_gcr.c:212-241, where SAP runs on what the
// deflation part left and base is the residual it started from).  With CUDA graphs
// on, the cycles run on three library-owned fields (solution, residual,
// block scratch) whose addresses never change, so the captured sequence
// (zero the solution, ncy x [block solves, boundary updates] per colour) is
// one graph per parameter set, replayed at every GCR step: rh is copied in
// before the replay and the results copied out after it.
// The field the captured SAP sequence reads its input from (null when CUDA
// graphs are off): a caller that computes rh can write it there directly
// and pass it as rh, which saves sap_mop the copy.
void *sap_input_field(Ctx &c) {
  if (!c.use_graphs || dd_on(c)) return nullptr;
  if (!c.sap_fld[1] && cudaMalloc(&c.sap_fld[1], spinor_bytes(c, 32)) != cudaSuccess) return nullptr;
  return c.sap_fld[1];
}

int sap_mop(Ctx &c, float mu, int isolv, int nmr, int ncy, const void *rh, void *psi, void *rho, void *phi_blk,
            cudaStream_t st, const void *base, const void *add) {
  if (!base) base = rh;
  // with domain decomposition the cycles call the exchange between their
  // launches, so they are not captured
  if (!c.use_graphs || dd_on(c)) {
    la_zero(c, 32, psi, PAR_ALL, st);
    if (rho != rh) la_copy(c, 32, rh, 32, rho, PAR_ALL, st);
    if (sap_cycles(c, mu, isolv, nmr, ncy, psi, rho, phi_blk, st)) return -1;
    la_diff(c, 32, base, rho, PAR_ALL, st);
    if (add) la_axpy(c, 32, psi, 1.0, 0.0, add, PAR_ALL, st);
    return 0;
  }
  for (int k = 0; k < 3; k++)
    if (!c.sap_fld[k] && cudaMalloc(&c.sap_fld[k], spinor_bytes(c, 32)) != cudaSuccess)
      return fail("out of device memory (SAP graph fields)");
  const int mode = sap_ready(c, isolv, st);
  if (mode < 0) return -1;
  void *spsi = c.sap_fld[0], *srho = c.sap_fld[1], *sphi = c.sap_fld[2];
  SapKey key;
  std::memset(&key, 0, sizeof(key));
  key.tag = 0x5a9;
  key.isolv = isolv;
  key.mode = mode;
  key.variant = c.sap_variant[mode];
  key.ncy = ncy;
  key.a = sap_args(c, mu, nmr, mode, spsi, srho, sphi);
  if (base == srho) return fail("sap_mop: an input in the SAP input field needs a separate base");
  if (rh != srho) la_copy(c, 32, rh, 32, srho, PAR_ALL, st);
  const int rc = graph_run(c, &key, sizeof(key), st, [&]() {
    la_zero(c, 32, spsi, PAR_ALL, st);
    for (int n = 0; n < ncy; n++) sap_cycle_launch(c, key.a, isolv, mode, st);
    return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
  });
  if (rc) return -1;
  const size_t n = (size_t)c.g.vol * 6;
  k_sap_out<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, (const float4 *)spsi, (const float4 *)srho,
                                                           (const float4 *)base, (const float4 *)add,
                                                           (float4 *)psi, (float4 *)rho);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
}

// the fields of sap_mop_multi for n systems; false (and nothing held) when
// the device has no room for them, in which case the systems run one at a
// time
static bool sap_multi_fields(Ctx &c, int n) {
  if (c.sap_mfld_n >= n) return true;
  for (int k = 0; k < 3; k++) {
    cudaFree(c.sap_mfld[k]);
    c.sap_mfld[k] = nullptr;
  }
  c.sap_mfld_n = 0;
  for (int k = 0; k < 3; k++)
    if (cudaMalloc(&c.sap_mfld[k], (size_t)n * spinor_bytes(c, 32)) != cudaSuccess) {
      cudaGetLastError();
      for (int j = 0; j < 3; j++) {
        cudaFree(c.sap_mfld[j]);
        c.sap_mfld[j] = nullptr;
      }
      return false;
    }
  c.sap_mfld_n = n;
  return true;
}

void *sap_input_field_multi(Ctx &c, int r, int n) {
  if (!c.use_graphs || dd_on(c) || r < 0 || r >= n || n > SAP_MS || !sap_multi_fields(c, n)) return nullptr;
  return (char *)c.sap_mfld[1] + (size_t)r * spinor_bytes(c, 32);
}

// Several systems: the SAP sequence of sap_mop captured once for up to
// SAP_MS systems on library-owned fields, every block-solver and boundary
// launch covering all of them.  Without graphs, or with domain
// decomposition, the systems run one after the other through sap_mop.
int sap_mop_multi(Ctx &c, int ns, const float *mu, int isolv, int nmr, int ncy, const void *const *rh,
                  void *const *psi, void *const *rho, void *phi_blk, cudaStream_t st, const void *const *base,
                  const void *const *add) {
  if (!c.use_graphs || dd_on(c) || ns == 1 || !sap_multi_fields(c, ns < SAP_MS ? ns : SAP_MS)) {
    for (int r = 0; r < ns; r++)
      if (sap_mop(c, mu[r], isolv, nmr, ncy, rh[r], psi[r], rho[r], phi_blk, st, base ? base[r] : nullptr,
                  add ? add[r] : nullptr))
        return -1;
    return 0;
  }
  const size_t fb = spinor_bytes(c, 32);
  const int mode = sap_ready(c, isolv, st);
  if (mode < 0) return -1;
  const size_t n = (size_t)c.g.vol * 6;   // float4 of a field
  for (int r0 = 0; r0 < ns; r0 += SAP_MS) {
    const int m = ns - r0 < SAP_MS ? ns - r0 : SAP_MS;
    SapKey key;
    std::memset(&key, 0, sizeof(key));
    key.tag = 0x5aa;
    key.isolv = isolv;
    key.mode = mode;
    key.variant = c.sap_variant[mode];
    key.ncy = ncy;
    key.a = sap_args(c, mu[r0], nmr, mode, c.sap_mfld[0], c.sap_mfld[1], c.sap_mfld[2]);
    key.a.nsys = m;
    for (int r = 0; r < m; r++) {
      key.a.psi[r] = (float4 *)c.sap_mfld[0] + (size_t)r * n;
      key.a.rho[r] = (float4 *)c.sap_mfld[1] + (size_t)r * n;
      key.a.phi[r] = (float4 *)c.sap_mfld[2] + (size_t)r * n;
      key.a.mus[r] = mu[r0 + r];
    }
    for (int r = 0; r < m; r++) {
      void *in = (char *)c.sap_mfld[1] + (size_t)r * fb;
      const void *b = base && base[r0 + r] ? base[r0 + r] : rh[r0 + r];
      if (b == in) return fail("sap_mop_multi: an input in the SAP input field needs a separate base");
      if (rh[r0 + r] != in) la_copy(c, 32, rh[r0 + r], 32, in, PAR_ALL, st);
    }
    const int rc = graph_run(c, &key, sizeof(key), st, [&]() {
      cudaMemsetAsync(c.sap_mfld[0], 0, (size_t)m * fb, st);
      for (int k = 0; k < ncy; k++) sap_cycle_launch(c, key.a, isolv, mode, st);
      return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
    });
    if (rc) return -1;
    for (int r = 0; r < m; r++) {
      const float4 *spsi = (const float4 *)((char *)c.sap_mfld[0] + (size_t)r * fb);
      const float4 *srho = (const float4 *)((char *)c.sap_mfld[1] + (size_t)r * fb);
      const void *b = base && base[r0 + r] ? base[r0 + r] : rh[r0 + r];
      k_sap_out<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, spsi, srho, (const float4 *)b,
                                                               (const float4 *)(add ? add[r0 + r] : nullptr),
                                                               (float4 *)psi[r0 + r], (float4 *)rho[r0 + r]);
    }
  }
  (void)phi_blk;
  return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
}

// One SAP cycle sap(mu, isolv, nmr, psi, rho) on FP32 device fields.
// phi_blk is a scratch FP32 field.  The even-odd block solver (isolv = 1)
// reads the links and SW matrices in the storage mode of sap_mode(); the
// plain solver (isolv = 0) always in FP32.
int sap_cycle(Ctx &c, float mu, int isolv, int nmr, void *psi, void *rho, void *phi_blk, cudaStream_t st) {
  const int mode = sap_ready(c, isolv, st);
  if (mode < 0) return -1;
  sap_cycle_launch(c, sap_args(c, mu, nmr, mode, psi, rho, phi_blk), isolv, mode, st);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("sap: launch failed");
}

}  // namespace qcd
