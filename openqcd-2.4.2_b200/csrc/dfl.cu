// Local deflation on the device: block basis, restriction/prolongation, the
// little Dirac operator, its even-odd preconditioned form and solver, the
// subspace generation, and the deflated SAP+GCR solver.
//
// Reference: modules/dfl/dfl_subspace.c (dfl_s2vd :83, dfl_vd2s :126,
// dfl_subspace :171), modules/little/Aw_ops.c (set_Aw :186, set_Awhat :223),
// Aw_dble.c (Aw_dble :122, Awhat_dble :361), modules/dfl/ltl_gcr.c (:155),
// modules/dfl/dfl_modes.c (:423), modules/dfl/dfl_sap_gcr.c (:212-381).
//
// The DFL blocks are the tiles of the device layout (the same block size as
// the SAP blocks), so the sites of one DFL block are two contiguous chunks.
// Little vectors hold Ns complex numbers per block in the reference's block
// order: the nb/2 blocks of colour 0 first, each colour in lexicographic
// order of the block coordinates (modules/block/blk_grid.c:20-32).  Little
// matrices are stored column-major (entry (k,l) at [l*Ns + k]) so that the
// threads of a block, one per row k, read consecutive words.
#include "lib.h"
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <chrono>
#include <functional>

namespace qcd {

// ---------------------------------------------------------------- timers
static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
// with profiling on: wait for the stream and charge the time since the
// previous mark to phase k
void dfl_mark(Ctx &c, int k) {
  DflState &d = c.dfl;
  if (!d.profile) return;
  cudaStreamSynchronize(c.stream);
  const double t = now_s();
  if (k >= 0 && d.prof_t0 > 0.0) d.prof[k] += t - d.prof_t0;
  d.prof_t0 = t;
}

// ------------------------------------------------------------- block maps
static int lex_of_vd(const Geom &g, const std::vector<int> &bco, int n) {
  const int nbh = g.nbl / 2;
  const int colour = n >= nbh, h = n - colour * nbh;
  const int q = 2 * h;
  int s = 0;
  for (int mu = 0; mu < 4; mu++) s += (bco[q] >> (8 * mu)) & 255;
  return q + ((s & 1) != colour);
}

static int dfl_alloc(Ctx &c) {
  DflState &d = c.dfl;
  const int Ns = d.Ns, nb = c.g.nbl;
  d.nb = nb;
  d.nv = Ns * nb;
  // block tables
  std::vector<int> bco(nb), v2l(nb), l2v(nb), nbr(8 * nb);
  cudaMemcpy(bco.data(), c.d_bcoord, nb * sizeof(int), cudaMemcpyDeviceToHost);
  for (int n = 0; n < nb; n++) {
    v2l[n] = lex_of_vd(c.g, bco, n);
    l2v[v2l[n]] = n;
  }
  for (int n = 0; n < nb; n++) {
    int b = v2l[n], x[4];
    for (int mu = 0; mu < 4; mu++) x[mu] = (bco[b] >> (8 * mu)) & 255;
    for (int ifc = 0; ifc < 8; ifc++) {
      int mu = ifc >> 1, dir = (ifc & 1) ? 1 : -1;
      int y[4] = {x[0], x[1], x[2], x[3]};
      y[mu] = (y[mu] + dir + c.g.nb[mu]) % c.g.nb[mu];
      int lb = ((y[0] * c.g.nb[1] + y[1]) * c.g.nb[2] + y[2]) * c.g.nb[3] + y[3];
      nbr[8 * n + ifc] = l2v[lb];
    }
  }
  auto up = [](int *&p, const std::vector<int> &v) {
    cudaFree(p);
    cudaMalloc(&p, v.size() * sizeof(int));
    cudaMemcpy(p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice);
  };
  up(d.vd2lex, v2l);
  up(d.nbr, nbr);
  // sites (p << 16 | s) of a block on each of its 8 faces, block-local
  {
    const int *bs = c.g.bs;
    int fmax = 0;
    for (int mu = 0; mu < 4; mu++) fmax = std::max(fmax, c.g.vb / bs[mu]);
    std::vector<int> fs(8 * fmax, 0), nf(8, 0);
    for (int y0 = 0; y0 < bs[0]; y0++)
      for (int y1 = 0; y1 < bs[1]; y1++)
        for (int y2 = 0; y2 < bs[2]; y2++)
          for (int y3 = 0; y3 < bs[3]; y3++) {
            const int y[4] = {y0, y1, y2, y3};
            const int l = ((y0 * bs[1] + y1) * bs[2] + y2) * bs[3] + y3;
            const int p = (y0 + y1 + y2 + y3) & 1;
            for (int ifc = 0; ifc < 8; ifc++) {
              const int mu = ifc >> 1;
              if (y[mu] == ((ifc & 1) ? bs[mu] - 1 : 0)) fs[ifc * fmax + nf[ifc]++] = (p << 16) | (l >> 1);
            }
          }
    up(d.faces, fs);
    up(d.nfc, nf);
    d.fmax = fmax;
  }
  // basis and matrices
  while ((int)d.basis.size() < Ns) {
    void *p = nullptr;
    if (cudaMalloc(&p, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory (deflation basis)");
    cudaMemset(p, 0, spinor_bytes(c, 32));
    d.basis.push_back(p);
  }
  cudaFree(d.d_basis);
  cudaMalloc(&d.d_basis, Ns * sizeof(void *));
  cudaMemcpy(d.d_basis, d.basis.data(), Ns * sizeof(void *), cudaMemcpyHostToDevice);
  cudaFree(d.rpart);
  if (cudaMalloc(&d.rpart, (size_t)nb * 2 * Ns * sizeof(double2)) != cudaSuccess)
    return fail("out of device memory (deflation)");
  size_t m = (size_t)nb * Ns * Ns * sizeof(double2);
  double2 **mats[] = {&d.Ablk, &d.Ainv, &d.Ahop, &d.Mhop};
  size_t sz[] = {m, m, 8 * m, 8 * m};
  for (int i = 0; i < 4; i++) {
    cudaFree(*mats[i]);
    if (cudaMalloc(mats[i], sz[i]) != cudaSuccess) return fail("out of device memory (little operator)");
  }
  cudaFree(d.Mhop32);
  if (cudaMalloc(&d.Mhop32, 4 * m) != cudaSuccess) return fail("out of device memory (little operator)");
  // the further masses' arrays have the old sizes
  for (auto &x : d.xsets)
    for (void *p : x) cudaFree(p);
  d.xsets.clear();
  d.aw_valid = d.awhat_valid = false;
  d.have_basis = false;
  d.ready = true;
  return cudaGetLastError() == cudaSuccess ? 0 : fail("deflation: CUDA error in set-up");
}

// ------------------------------------------------ restriction / prolongation
// vd[n*Ns + l] = (basis_l, s) on block n; FP32 products accumulated in double
// and rounded to float, as spinor_prod returns them (dfl_subspace.c:83-123).
// Restriction by parity chunks: CTA (n, p) owns the vbh sites of parity p
// of block n, one site per thread (the site's field values stay in
// registers while the Ns basis vectors stream past); the 12 products of a
// site are summed in the field's precision, everything after in double
// (FP64 arithmetic per product halved the kernel's speed); per-warp partial sums
// go to shared memory without a barrier per l, and the two parities are
// added by k_dfl_restrict_fin in a fixed order.
constexpr int RESTRICT_T = 704;

template <typename R>
__global__ void __launch_bounds__(RESTRICT_T) k_dfl_restrict2(Geom g, const int *__restrict__ vd2lex,
                                                              const float4 *const *__restrict__ basis, int Ns,
                                                              const void *__restrict__ s, double2 *part) {
  __shared__ double2 red[64][RESTRICT_T / 32 + 1];
  const int n = blockIdx.x, p = blockIdx.y, blk = __ldg(vd2lex + n), chunk = p * g.nbl + blk;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool one = g.vbh <= (int)blockDim.x;
  spinor<R> x;
  szero(x);
  if (one && (int)threadIdx.x < g.vbh) x = Store<R>::load_spinor(s, chunk, threadIdx.x, g.vbh);
  for (int l = 0; l < Ns; l++) {
    double re = 0.0, im = 0.0;
    const float4 *bl = basis[l];
    for (int si = threadIdx.x; si < g.vbh; si += blockDim.x) {
      const spinor<R> xx = one ? x : Store<R>::load_spinor(s, chunk, si, g.vbh);
      const spinor<float> b = Store<float>::load_spinor(bl, chunk, si, g.vbh);
      // the 12 products of a site in R, the sums over sites in double
      R sr = 0, sim = 0;
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const R br = b.c[a].c[k].re, bi = b.c[a].c[k].im, xr = xx.c[a].c[k].re, xi = xx.c[a].c[k].im;
          sr += br * xr + bi * xi;
          sim += br * xi - bi * xr;
        }
      re += (double)sr;
      im += (double)sim;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_down_sync(0xffffffffu, re, o);
      im += __shfl_down_sync(0xffffffffu, im, o);
    }
    if (lane == 0) red[l][wp] = make_double2(re, im);
  }
  __syncthreads();
  for (int l = threadIdx.x; l < Ns; l += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < nw; w++) {
      re += red[l][w].x;
      im += red[l][w].y;
    }
    part[((size_t)n * 2 + p) * Ns + l] = make_double2(re, im);
  }
}

__global__ void k_dfl_restrict_fin(const double2 *__restrict__ part, int Ns, int nb, double2 *vd, int round_float) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb * Ns) return;
  const int n = i / Ns, l = i - n * Ns;
  const double2 a = part[((size_t)n * 2) * Ns + l], b = part[((size_t)n * 2 + 1) * Ns + l];
  double re = a.x + b.x, im = a.y + b.y;
  if (round_float) {
    re = (double)(float)re;
    im = (double)(float)im;
  }
  vd[i] = make_double2(re, im);
}

// s = sum_l vd[n,l] basis_l on every block n, with float coefficients and
// float accumulation (dfl_vd2s, dfl_subspace.c:126-167).
__global__ void k_dfl_prolong(Geom g, const int *__restrict__ vd2lex, const float4 *const *__restrict__ basis,
                              int Ns, const double2 *__restrict__ vd, float4 *s) {
  const int n = blockIdx.x, blk = __ldg(vd2lex + n);
  const int nsite = 2 * g.vbh;
  for (int t = threadIdx.x; t < nsite; t += blockDim.x) {
    const int p = t >= g.vbh, si = t - p * g.vbh, chunk = p * g.nbl + blk;
    spinor<float> acc;
    szero(acc);
    for (int l = 0; l < Ns; l++) {
      const double2 z = vd[(size_t)n * Ns + l];
      const float zr = (float)z.x, zi = (float)z.y;
      spinor<float> b = Store<float>::load_spinor(basis[l], chunk, si, g.vbh);
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
          acc.c[a].c[k].re += zr * b.c[a].c[k].re - zi * b.c[a].c[k].im;
          acc.c[a].c[k].im += zr * b.c[a].c[k].im + zi * b.c[a].c[k].re;
        }
    }
    Store<float>::store_spinor(s, chunk, si, g.vbh, acc);
  }
}

// ------------------------------------------------------ block Gram-Schmidt
// basis_l(block) = orthonormalised mode_l(block) against basis_0..l-1 of the
// same block, in double precision (dfl_subspace.c:171-240).  One CTA per
// block; the vector being orthonormalised is held in the FP64 work field,
// each site read and written only by the thread that owns it.
__global__ void k_dfl_gs(Geom g, const int *__restrict__ vd2lex, float4 *const *basis,
                         const float4 *const *__restrict__ modes, int Ns, double2 *work, int *fail) {
  const int n = blockIdx.x, blk = __ldg(vd2lex + n);
  const int nsite = 2 * g.vbh;
  __shared__ double red[2][32];
  __shared__ double zsh[2];
  for (int l = 0; l < Ns; l++) {
    for (int t = threadIdx.x; t < nsite; t += blockDim.x) {
      const int p = t >= g.vbh, si = t - p * g.vbh, chunk = p * g.nbl + blk;
      spinor<float> m = Store<float>::load_spinor(modes[l], chunk, si, g.vbh);
      spinor<double> md;
#pragma unroll
      for (int k = 0; k < 12; k++) md.c[k / 3].c[k % 3] = mk<double>(m.c[k / 3].c[k % 3].re, m.c[k / 3].c[k % 3].im);
      Store<double>::store_spinor(work, chunk, si, g.vbh, md);
    }
    for (int j = 0; j <= l; j++) {
      // j < l: z = (basis_j, v), v -= z basis_j ; j == l: normalise
      double re = 0.0, im = 0.0;
      for (int t = threadIdx.x; t < nsite; t += blockDim.x) {
        const int p = t >= g.vbh, si = t - p * g.vbh, chunk = p * g.nbl + blk;
        spinor<double> x = Store<double>::load_spinor_rw(work, chunk, si, g.vbh);
        if (j < l) {
          spinor<float> b = Store<float>::load_spinor(basis[j], chunk, si, g.vbh);
#pragma unroll
          for (int k = 0; k < 12; k++) {
            const double br = b.c[k / 3].c[k % 3].re, bi = b.c[k / 3].c[k % 3].im;
            const double xr = x.c[k / 3].c[k % 3].re, xi = x.c[k / 3].c[k % 3].im;
            re += br * xr + bi * xi;
            im += br * xi - bi * xr;
          }
        } else {
#pragma unroll
          for (int k = 0; k < 12; k++)
            re += x.c[k / 3].c[k % 3].re * x.c[k / 3].c[k % 3].re + x.c[k / 3].c[k % 3].im * x.c[k / 3].c[k % 3].im;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
      }
      if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = re; red[1][threadIdx.x >> 5] = im; }
      __syncthreads();
      if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a += red[0][w]; b += red[1][w]; }
        zsh[0] = a;
        zsh[1] = b;
      }
      __syncthreads();
      const double zr = zsh[0], zi = zsh[1];
      const double nrm = sqrt(zr);
      if (j == l && nrm == 0.0 && threadIdx.x == 0) atomicOr(fail, 1);
      const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
      for (int t = threadIdx.x; t < nsite; t += blockDim.x) {
        const int p = t >= g.vbh, si = t - p * g.vbh, chunk = p * g.nbl + blk;
        spinor<double> x = Store<double>::load_spinor_rw(work, chunk, si, g.vbh);
        if (j < l) {
          spinor<float> b = Store<float>::load_spinor(basis[j], chunk, si, g.vbh);
#pragma unroll
          for (int k = 0; k < 12; k++) {
            const double br = b.c[k / 3].c[k % 3].re, bi = b.c[k / 3].c[k % 3].im;
            x.c[k / 3].c[k % 3].re -= zr * br - zi * bi;
            x.c[k / 3].c[k % 3].im -= zr * bi + zi * br;
          }
          Store<double>::store_spinor(work, chunk, si, g.vbh, x);
        } else {
          spinor<float> o;
#pragma unroll
          for (int k = 0; k < 12; k++)
            o.c[k / 3].c[k % 3] = mk<float>((float)(x.c[k / 3].c[k % 3].re * inv), (float)(x.c[k / 3].c[k % 3].im * inv));
          Store<float>::store_spinor(basis[l], chunk, si, g.vbh, o);
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------ little operator set-up
// t = D_blk w (in-block hops only, Dirichlet exterior) + SW term with twisted
// mass, or t = the hop of w across face ifc only; FP64 output from an FP32
// input field.
__global__ void k_dfl_dapply(Geom g, const float4 *__restrict__ w, double2 *t, const double2 *__restrict__ ud,
                             const double2 *__restrict__ swd, double mu_e, double mu_o, int ifc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.vol) return;
  const int chunk = i / g.vbh, si = i - chunk * g.vbh;
  const int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
  Site x;
  site_decode(g, p, blk, si, x);
  spinor<double> acc, h;
  szero(acc);
  szero(h);
  if (ifc < 0) {
    spinor<float> in = Store<float>::load_spinor(w, chunk, si, g.vbh);
    spinor<double> ind;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int k = 0; k < 3; k++) ind.c[a].c[k] = mk<double>(in.c[a].c[k].re, in.c[a].c[k].im);
    acc = apply_sw_site<double>(swd, chunk, si, g.vbh, p ? mu_o : mu_e, ind);
  }
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
#pragma unroll
    for (int dd = 0; dd < 2; dd++) {
      const int dir = dd ? 1 : -1;
      const bool cross = crosses_block(g, x, mu, dir);
      const bool take = (ifc < 0) ? !cross : (cross && ifc == 2 * mu + dd);
      if (!take) continue;
      int c2, s2;
      site_nbr(g, x, mu, dir, c2, s2);
      spinor<float> nf = Store<float>::load_spinor(w, c2, s2, g.vbh);
      spinor<double> nd;
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int k = 0; k < 3; k++) nd.c[a].c[k] = mk<double>(nf.c[a].c[k].re, nf.c[a].c[k].im);
      if (dir > 0) hop_fwd<double>(mu, Store<double>::load_link(ud, chunk, mu, si, g.vbh), nd, h);
      else hop_bwd<double>(mu, Store<double>::load_link(ud, c2, mu, s2, g.vbh), nd, h);
    }
  }
  sscale<double>(h, -0.5);
  sadd(acc, h);
  Store<double>::store_spinor(t, chunk, si, g.vbh, acc);
}

// Little operator by block-local products (Aw_blk.c:242 set_Awblk and
// Aw_hop.c:279 set_Awhop restated as small dense products).  CTA (n, 0)
// computes Ablk[n](k,l) = (b_k, D_blk b_l) over the sites of block n, with
// D_blk the SW term plus the hops inside the block; CTA (n, 1+ifc) computes
// Ahop[n][ifc](k,l) = (b_k, H_ifc b_l) over the sites of block n on face
// ifc, H_ifc the hop from the neighbouring block across that face.  The
// sites are taken TS at a time: D b_l on the tile for all l goes to shared
// memory in FP64 (Y), the basis on the tile in FP32 (B), and every thread
// accumulates a 2x2 tile of (k,l) pairs in FP64.  Rows are stored in pairs
// (l even, l odd interleaved) and padded to an odd length so that the
// 16-byte loads of B by consecutive k are free of bank conflicts.
template <int TS, int MAXT>
__global__ void __launch_bounds__(256) k_aw_tiles(Geom g, const int *__restrict__ vd2lex,
                                                  const float4 *const *__restrict__ basis, int Ns,
                                                  const double2 *__restrict__ ud, const double2 *__restrict__ swd,
                                                  double mu_e, double mu_o, const int *__restrict__ faces,
                                                  const int *__restrict__ nfc, int fmax, double2 *Ablk,
                                                  double2 *Ahop) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int LD = TS * 12 + 1;
  const int NT = Ns / 2;
  double2 *Y = (double2 *)smraw;                         // [NT][LD][2]
  float4 *B = (float4 *)(Y + (size_t)NT * LD * 2);       // [NT][LD]
  const int n = blockIdx.x, blk = __ldg(vd2lex + n);
  const int ifc = (int)blockIdx.y - 1;
  const int nsites = ifc < 0 ? 2 * g.vbh : __ldg(nfc + ifc);
  const int ntile = NT * NT;
  double acc[MAXT][4][2];
#pragma unroll
  for (int j = 0; j < MAXT; j++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[j][q][0] = acc[j][q][1] = 0.0;

  for (int t0 = 0; t0 < nsites; t0 += TS) {
    // D b_l and b_l on the tile sites
    for (int it = threadIdx.x; it < TS * Ns; it += blockDim.x) {
      const int i = it % TS, l = it / TS, t = t0 + i;
      spinor<double> y;
      spinor<float> b;
      szero(y);
      szero(b);
      if (t < nsites) {
        int p, s;
        if (ifc < 0) {
          p = t >= g.vbh;
          s = t - p * g.vbh;
        } else {
          const int f = __ldg(faces + ifc * fmax + t);
          p = f >> 16;
          s = f & 0xffff;
        }
        const int chunk = p * g.nbl + blk;
        Site x;
        site_decode(g, p, blk, s, x);
        const float4 *bl = basis[l];
        b = Store<float>::load_spinor(bl, chunk, s, g.vbh);
        spinor<double> h;
        szero(h);
        if (ifc < 0) {
          spinor<double> bd;
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int k = 0; k < 3; k++) bd.c[a].c[k] = mk<double>(b.c[a].c[k].re, b.c[a].c[k].im);
          y = apply_sw_site<double>(swd, chunk, s, g.vbh, p ? mu_o : mu_e, bd);
#pragma unroll
          for (int mu = 0; mu < 4; mu++)
#pragma unroll
            for (int dd = 0; dd < 2; dd++) {
              const int dir = dd ? 1 : -1;
              if (crosses_block(g, x, mu, dir)) continue;
              int c2, s2;
              site_nbr(g, x, mu, dir, c2, s2);
              const spinor<float> nf = Store<float>::load_spinor(bl, c2, s2, g.vbh);
              spinor<double> nd;
#pragma unroll
              for (int a = 0; a < 4; a++)
#pragma unroll
                for (int k = 0; k < 3; k++) nd.c[a].c[k] = mk<double>(nf.c[a].c[k].re, nf.c[a].c[k].im);
              if (dir > 0) hop_fwd<double>(mu, Store<double>::load_link(ud, chunk, mu, s, g.vbh), nd, h);
              else hop_bwd<double>(mu, Store<double>::load_link(ud, c2, mu, s2, g.vbh), nd, h);
            }
        } else {
          const int mu = ifc >> 1, dir = (ifc & 1) ? 1 : -1;
          int c2, s2;
          site_nbr(g, x, mu, dir, c2, s2);
          const spinor<float> nf = Store<float>::load_spinor(bl, c2, s2, g.vbh);
          spinor<double> nd;
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int k = 0; k < 3; k++) nd.c[a].c[k] = mk<double>(nf.c[a].c[k].re, nf.c[a].c[k].im);
          if (dir > 0) hop_fwd<double>(mu, Store<double>::load_link(ud, chunk, mu, s, g.vbh), nd, h);
          else hop_bwd<double>(mu, Store<double>::load_link(ud, c2, mu, s2, g.vbh), nd, h);
        }
        sscale<double>(h, -0.5);
        sadd(y, h);
      }
      double2 *yd = Y + ((size_t)(l >> 1) * LD + i * 12) * 2 + (l & 1);
      float2 *bd = (float2 *)(B + (size_t)(l >> 1) * LD + i * 12) + (l & 1);
#pragma unroll
      for (int k = 0; k < 12; k++) {
        yd[2 * k] = make_double2(y.c[k / 3].c[k % 3].re, y.c[k / 3].c[k % 3].im);
        bd[2 * k] = make_float2(b.c[k / 3].c[k % 3].re, b.c[k / 3].c[k % 3].im);
      }
    }
    __syncthreads();
    // (k,l) pairs: thread tile (kt, lt) holds k = 2kt, 2kt+1 and l = 2lt, 2lt+1
#pragma unroll
    for (int j = 0; j < MAXT; j++) {
      const int q = threadIdx.x + j * blockDim.x;
      if (q < ntile) {
        const int kt = q % NT, lt = q / NT;
        const float4 *bp = B + (size_t)kt * LD;
        const double2 *yp = Y + (size_t)lt * LD * 2;
        for (int e = 0; e < TS * 12; e++) {
          const float4 bb = bp[e];
          const double2 y0 = yp[2 * e], y1 = yp[2 * e + 1];
          const double b0r = bb.x, b0i = bb.y, b1r = bb.z, b1i = bb.w;
          acc[j][0][0] += b0r * y0.x + b0i * y0.y;  acc[j][0][1] += b0r * y0.y - b0i * y0.x;
          acc[j][1][0] += b0r * y1.x + b0i * y1.y;  acc[j][1][1] += b0r * y1.y - b0i * y1.x;
          acc[j][2][0] += b1r * y0.x + b1i * y0.y;  acc[j][2][1] += b1r * y0.y - b1i * y0.x;
          acc[j][3][0] += b1r * y1.x + b1i * y1.y;  acc[j][3][1] += b1r * y1.y - b1i * y1.x;
        }
      }
    }
    __syncthreads();
  }
  const size_t npair = (size_t)Ns * Ns;
  double2 *dst = ifc < 0 ? Ablk + n * npair : Ahop + ((size_t)8 * n + ifc) * npair;
#pragma unroll
  for (int j = 0; j < MAXT; j++) {
    const int q = threadIdx.x + j * blockDim.x;
    if (q < ntile) {
      const int kt = q % NT, lt = q / NT, k = 2 * kt, l = 2 * lt;
      dst[(size_t)l * Ns + k] = make_double2(acc[j][0][0], acc[j][0][1]);
      dst[(size_t)(l + 1) * Ns + k] = make_double2(acc[j][1][0], acc[j][1][1]);
      dst[(size_t)l * Ns + k + 1] = make_double2(acc[j][2][0], acc[j][2][1]);
      dst[(size_t)(l + 1) * Ns + k + 1] = make_double2(acc[j][3][0], acc[j][3][1]);
    }
  }
}

// M[n][col l] (entries k) = (basis_k, t) on block n, FP64 field t
__global__ void k_dfl_project(Geom g, const int *__restrict__ vd2lex, const float4 *const *__restrict__ basis,
                              int Ns, const double2 *__restrict__ t, double2 *M, size_t mstride, int l) {
  const int n = blockIdx.x, blk = __ldg(vd2lex + n);
  __shared__ double red[2][32];
  const int nsite = 2 * g.vbh;
  for (int k = 0; k < Ns; k++) {
    double re = 0.0, im = 0.0;
    for (int tt = threadIdx.x; tt < nsite; tt += blockDim.x) {
      const int p = tt >= g.vbh, si = tt - p * g.vbh, chunk = p * g.nbl + blk;
      spinor<float> b = Store<float>::load_spinor(basis[k], chunk, si, g.vbh);
      spinor<double> x = Store<double>::load_spinor(t, chunk, si, g.vbh);
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const double br = b.c[a].c[c].re, bi = b.c[a].c[c].im, xr = x.c[a].c[c].re, xi = x.c[a].c[c].im;
          re += br * xr + bi * xi;
          im += br * xi - bi * xr;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_down_sync(0xffffffffu, re, o);
      im += __shfl_down_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = re; red[1][threadIdx.x >> 5] = im; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a += red[0][w]; b += red[1][w]; }
      M[n * mstride + (size_t)l * Ns + k] = make_double2(a, b);
    }
    __syncthreads();
  }
}

// Batched inverse of Ns x Ns complex matrices (column-major) by Gauss-Jordan
// elimination with partial pivoting, one CTA per matrix; flags matrices whose
// Frobenius condition number exceeds 1e6 (modules/little/Aw_ops.c:35-40).
__global__ void k_cinv(int Ns, const double2 *__restrict__ A, double2 *B, int *fail) {
  extern __shared__ double2 sm[];   // a[Ns*Ns], b[Ns*Ns] row-major
  double2 *a = sm, *b = sm + Ns * Ns;
  __shared__ int piv;
  __shared__ double fn[2];
  __shared__ double2 fcol[64];
  const size_t off = (size_t)blockIdx.x * Ns * Ns;
  for (int e = threadIdx.x; e < Ns * Ns; e += blockDim.x) {
    const int r = e / Ns, cc = e % Ns;
    a[e] = A[off + (size_t)cc * Ns + r];
    b[e] = make_double2(r == cc ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int e = 0; e < Ns * Ns; e++) s += a[e].x * a[e].x + a[e].y * a[e].y;
    fn[0] = s;
  }
  for (int c = 0; c < Ns; c++) {
    if (threadIdx.x == 0) {
      int p = c;
      double best = -1.0;
      for (int r = c; r < Ns; r++) {
        double v = a[r * Ns + c].x * a[r * Ns + c].x + a[r * Ns + c].y * a[r * Ns + c].y;
        if (v > best) { best = v; p = r; }
      }
      piv = p;
      if (best == 0.0) atomicOr(fail, 1);
    }
    __syncthreads();
    const int p = piv;
    if (p != c)
      for (int j = threadIdx.x; j < Ns; j += blockDim.x) {
        double2 t = a[c * Ns + j]; a[c * Ns + j] = a[p * Ns + j]; a[p * Ns + j] = t;
        t = b[c * Ns + j]; b[c * Ns + j] = b[p * Ns + j]; b[p * Ns + j] = t;
      }
    __syncthreads();
    double2 pv = a[c * Ns + c];
    double d = pv.x * pv.x + pv.y * pv.y;
    if (d == 0.0) d = 1.0;
    const double qr = pv.x / d, qi = -pv.y / d;
    __syncthreads();
    for (int j = threadIdx.x; j < Ns; j += blockDim.x) {
      double2 x = a[c * Ns + j];
      a[c * Ns + j] = make_double2(x.x * qr - x.y * qi, x.x * qi + x.y * qr);
      x = b[c * Ns + j];
      b[c * Ns + j] = make_double2(x.x * qr - x.y * qi, x.x * qi + x.y * qr);
    }
    // the multipliers (column c) are read by every element of their row,
    // so they are saved before the elimination overwrites them
    for (int r = threadIdx.x; r < Ns; r += blockDim.x) fcol[r] = a[r * Ns + c];
    __syncthreads();
    for (int e = threadIdx.x; e < Ns * Ns; e += blockDim.x) {
      const int r = e / Ns, j = e % Ns;
      if (r == c) continue;
      const double2 f = fcol[r];
      const double2 ac = a[c * Ns + j], bc = b[c * Ns + j];
      a[e] = make_double2(a[e].x - (f.x * ac.x - f.y * ac.y), a[e].y - (f.x * ac.y + f.y * ac.x));
      b[e] = make_double2(b[e].x - (f.x * bc.x - f.y * bc.y), b[e].y - (f.x * bc.y + f.y * bc.x));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < Ns * Ns; e += blockDim.x) {
    const int r = e / Ns, cc = e % Ns;
    B[off + (size_t)cc * Ns + r] = b[e];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int e = 0; e < Ns * Ns; e++) s += b[e].x * b[e].x + b[e].y * b[e].y;
    if (fn[0] * s > 1.0e12) atomicOr(fail, 1);
  }
}

// b = a rounded to FP32
static __global__ void k_round32(const double2 *__restrict__ a, float2 *b, size_t n) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = make_float2((float)a[i].x, (float)a[i].y);
}

// M[n][ifc] = Ainv[n] * Ahop[n][ifc]  (column-major products)
__global__ void k_cmatmul8(int Ns, const double2 *__restrict__ Ainv, const double2 *__restrict__ Ahop, double2 *M) {
  const int n = blockIdx.x >> 3, ifc = blockIdx.x & 7;
  const double2 *a = Ainv + (size_t)n * Ns * Ns;
  const double2 *h = Ahop + ((size_t)8 * n + ifc) * Ns * Ns;
  double2 *m = M + ((size_t)8 * n + ifc) * Ns * Ns;
  for (int e = threadIdx.x; e < Ns * Ns; e += blockDim.x) {
    const int k = e % Ns, l = e / Ns;
    double re = 0.0, im = 0.0;
    for (int j = 0; j < Ns; j++) {
      const double2 x = a[(size_t)j * Ns + k], y = h[(size_t)l * Ns + j];
      re += x.x * y.x - x.y * y.y;
      im += x.x * y.y + x.y * y.x;
    }
    m[(size_t)l * Ns + k] = make_double2(re, im);
  }
}

// ----------------------------------------------------- little operator apply
// mode 0: w[n] = Ablk[n] v[n] + sum_ifc Ahop[n][ifc] v[nbr]        all blocks
// mode 1: w[n] = sum_ifc H[n][ifc] v[nbr]   for blocks in [b0, b0+cnt)
// mode 2: w[n] = v[n] - sum_ifc H[n][ifc] u[nbr]
// mode 3: w[n] = Ablk[n] v[n] (Ablk holding an inverse)
// One warp per matrix: warps 0..7 take the
// eight face matrices, warp 8 (mode 0) or warp 0 (mode 3) the diagonal one;
// lanes hold rows k and k+32, the column loop is unrolled four times so that
// every lane keeps four independent 16-byte loads in flight; the warps'
// partial rows are summed in shared memory.
__global__ void __launch_bounds__(288) k_little_w(int mode, int Ns, int b0, const double2 *__restrict__ Ablk,
                                                  const double2 *__restrict__ H, const int *__restrict__ nbr,
                                                  const double2 *__restrict__ v, const double2 *__restrict__ u,
                                                  double2 *w) {
  __shared__ double2 part[9][64];
  const int n = b0 + blockIdx.x, wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const double2 *a, *x;
  if (mode == 3 || wp == 8) {
    a = Ablk + (size_t)n * Ns * Ns;
    x = v + (size_t)n * Ns;
  } else {
    a = H + ((size_t)8 * n + wp) * Ns * Ns;
    x = (mode == 2 ? u : v) + (size_t)__ldg(nbr + 8 * n + wp) * Ns;
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int k = lane + 32 * h;
    if (k < Ns) {
      double r0 = 0.0, i0 = 0.0, r1 = 0.0, i1 = 0.0;
      int l = 0;
      for (; l + 4 <= Ns; l += 4) {
        const double2 a0 = __ldg(a + (size_t)l * Ns + k), a1 = __ldg(a + (size_t)(l + 1) * Ns + k);
        const double2 a2 = __ldg(a + (size_t)(l + 2) * Ns + k), a3 = __ldg(a + (size_t)(l + 3) * Ns + k);
        const double2 x0 = __ldg(x + l), x1 = __ldg(x + l + 1), x2 = __ldg(x + l + 2), x3 = __ldg(x + l + 3);
        r0 += a0.x * x0.x - a0.y * x0.y; i0 += a0.x * x0.y + a0.y * x0.x;
        r1 += a1.x * x1.x - a1.y * x1.y; i1 += a1.x * x1.y + a1.y * x1.x;
        r0 += a2.x * x2.x - a2.y * x2.y; i0 += a2.x * x2.y + a2.y * x2.x;
        r1 += a3.x * x3.x - a3.y * x3.y; i1 += a3.x * x3.y + a3.y * x3.x;
      }
      for (; l < Ns; l++) {
        const double2 a0 = __ldg(a + (size_t)l * Ns + k), x0 = __ldg(x + l);
        r0 += a0.x * x0.x - a0.y * x0.y; i0 += a0.x * x0.y + a0.y * x0.x;
      }
      part[wp][k] = make_double2(r0 + r1, i0 + i1);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < Ns; k += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int j = 0; j < nw; j++) {
      re += part[j][k].x;
      im += part[j][k].y;
    }
    if (mode == 2) {
      const double2 vv = v[(size_t)n * Ns + k];
      w[(size_t)n * Ns + k] = make_double2(vv.x - re, vv.y - im);
    } else {
      w[(size_t)n * Ns + k] = make_double2(re, im);
    }
  }
}

static void little_launch(int mode, int Ns, int b0, int nblk, const double2 *Ablk, const double2 *H, const int *nbr,
                          const double2 *v, const double2 *u, double2 *w, cudaStream_t st) {
  const int nw = mode == 3 ? 1 : (mode == 0 ? 9 : 8);
  k_little_w<<<nblk, 32 * nw, 0, st>>>(mode, Ns, b0, Ablk, H, nbr, v, u, w);
}

// ------------------------------------------------ little-vector GCR kernels
// Dots (Q_j, y) = sum_i conj(Q_j[i]) y[i] for j < k (k <= LMAXK) in one pass
// over y, per-CTA partial sums, then a fixed-order final sum: deterministic.
constexpr int LMAXK = 32, LGRID = 296;

__global__ void __launch_bounds__(256) k_mdot(const double2 *const *__restrict__ Q, int k,
                                              const double2 *__restrict__ y, int n, double2 *part) {
  __shared__ double2 red[8][LMAXK];
  double ar[LMAXK], ai[LMAXK];
#pragma unroll
  for (int j = 0; j < LMAXK; j++) ar[j] = ai[j] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 yy = y[i];
#pragma unroll
    for (int j = 0; j < LMAXK; j++)
      if (j < k) {
        const double2 q = Q[j][i];
        ar[j] += q.x * yy.x + q.y * yy.y;
        ai[j] += q.x * yy.y - q.y * yy.x;
      }
  }
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < LMAXK; j++)
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
    for (int w = 0; w < 8; w++) {
      re += red[w][threadIdx.x].x;
      im += red[w][threadIdx.x].y;
    }
    part[blockIdx.x * LMAXK + threadIdx.x] = make_double2(re, im);
  }
}

__global__ void k_mdot_fin(const double2 *__restrict__ part, int k, double2 *dots) {
  const int j = threadIdx.x;
  if (j >= k) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < LGRID; b++) {
    re += part[b * LMAXK + j].x;
    im += part[b * LMAXK + j].y;
  }
  dots[j] = make_double2(re, im);
}

// qk -= sum_j dots[j] Q_j ; pk -= sum_j dots[j] P_j
__global__ void k_gs_sub(const double2 *const *__restrict__ Q, const double2 *const *__restrict__ P, int k,
                         const double2 *__restrict__ dots, double2 *qk, double2 *pk, int n) {
  __shared__ double2 c[LMAXK];
  if (threadIdx.x < k) c[threadIdx.x] = dots[threadIdx.x];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 q = qk[i], p = pk[i];
    for (int j = 0; j < k; j++) {
      const double2 a = Q[j][i], b = P[j][i], z = c[j];
      q.x -= z.x * a.x - z.y * a.y; q.y -= z.x * a.y + z.y * a.x;
      p.x -= z.x * b.x - z.y * b.y; p.y -= z.x * b.y + z.y * b.x;
    }
    qk[i] = q;
    pk[i] = p;
  }
}

// qk, pk /= |qk| (nrm2 = |qk|^2, left unchanged when zero)
__global__ void k_norm_scale(double2 *qk, double2 *pk, const double2 *__restrict__ nrm2, int n) {
  const double s2 = nrm2[0].x;
  if (!(s2 > 0.0)) return;
  const double f = 1.0 / sqrt(s2);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 q = qk[i], p = pk[i];
    qk[i] = make_double2(q.x * f, q.y * f);
    pk[i] = make_double2(p.x * f, p.y * f);
  }
}

// x += c pk ; r -= c qk with c = (qk, r)
__global__ void k_xr_update(double2 *x, double2 *r, const double2 *__restrict__ pk, const double2 *__restrict__ qk,
                            const double2 *__restrict__ cc, int n) {
  const double2 z = cc[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 p = pk[i], q = qk[i];
    double2 xx = x[i], rr = r[i];
    xx.x += z.x * p.x - z.y * p.y; xx.y += z.x * p.y + z.y * p.x;
    rr.x -= z.x * q.x - z.y * q.y; rr.y -= z.x * q.y + z.y * q.x;
    x[i] = xx;
    r[i] = rr;
  }
}

// ----------------------------------------------------------- host routines

void dfl_release(Ctx &c) {
  DflState &d = c.dfl;
  for (void *p : d.basis) cudaFree(p);
  for (void *p : d.modes) cudaFree(p);
  for (void *p : d.start) cudaFree(p);
  for (auto &x : d.xsets)
    for (void *p : x) cudaFree(p);
  for (double2 *p : d.lv) cudaFree(p);
  for (double2 *p : d.lvd) cudaFree(p);
  void *bufs[] = {d.vd2lex, d.nbr, d.faces, d.nfc, d.d_basis, d.Ablk, d.Ainv, d.Ahop, d.Mhop, d.Mhop32,
                  d.lvtab, d.ldots, d.lpart, d.rpart, d.bpart, d.kerr, d.gram, d.tri, d.gfail};
  if (d.h_ldots) cudaFreeHost(d.h_ldots);
  for (void *p : bufs) cudaFree(p);
  ltl_ref_release(c);
  DflState fresh;
  // the solver and generation parameters outlive a change of geometry
  fresh.gen_set = d.gen_set;
  fresh.nkv = d.nkv; fresh.nmx = d.nmx; fresh.nmx_gcr = d.nmx_gcr;
  fresh.res = d.res; fresh.res_gcr = d.res_gcr;
  fresh.gen_kappa = d.gen_kappa; fresh.gen_mu = d.gen_mu;
  fresh.gen_ninv = d.gen_ninv; fresh.gen_nmr = d.gen_nmr; fresh.gen_ncy = d.gen_ncy;
  fresh.ltl_kind = d.ltl_kind;
  d = fresh;
}

int dfl_set_parms(Ctx &c, const int bs[4], int Ns) {
  for (int mu = 0; mu < 4; mu++)
    if (bs[mu] != c.g.bs[mu]) return fail("set_dfl_parms: the DFL block size must equal the geometry block size");
  // check_block_size (modules/flags/dfl_parms.c:175-205) without the
  // per-thread rule, and the once-only rule of set_dfl_parms (:228)
  for (int mu = 0; mu < 4; mu++) {
    if (bs[mu] < 4 || bs[mu] > c.g.L[mu]) return fail("set_dfl_parms: block sizes are out of range");
    if (bs[mu] & 1) return fail("set_dfl_parms: block sizes must be even");
    if (c.g.nb[mu] & 1) return fail("set_dfl_parms: there must be an even number of blocks in each direction");
  }
  if (Ns < 2 || (Ns & 1) || Ns > 64) return fail("set_dfl_parms: Ns must be even and in [2, 64]");
  if (c.dfl.ready && Ns != c.dfl.Ns) return fail("set_dfl_parms: bs[4] and Ns may be set only once");
  if (c.dfl.ready) return 0;
  c.dfl.Ns = Ns;
  return dfl_alloc(c);
}

void dfl_restrict(Ctx &c, int prec, const void *s, double2 *vd, cudaStream_t st) {
  DflState &d = c.dfl;
  const dim3 grid(d.nb, 2);
  const int t = std::min(RESTRICT_T, (c.g.vbh + 31) / 32 * 32);
  const float4 *const *bas = (const float4 *const *)d.d_basis;
  if (prec == 32) k_dfl_restrict2<float><<<grid, t, 0, st>>>(c.g, d.vd2lex, bas, d.Ns, s, d.rpart);
  else k_dfl_restrict2<double><<<grid, t, 0, st>>>(c.g, d.vd2lex, bas, d.Ns, s, d.rpart);
  const int nn = d.nb * d.Ns;
  k_dfl_restrict_fin<<<(nn + 255) / 256, 256, 0, st>>>(d.rpart, d.Ns, d.nb, vd, prec == 32);
}

void dfl_prolong(Ctx &c, const double2 *vd, void *s, cudaStream_t st) {
  DflState &d = c.dfl;
  k_dfl_prolong<<<d.nb, 256, 0, st>>>(c.g, d.vd2lex, (const float4 *const *)d.d_basis, d.Ns, vd, (float4 *)s);
}

// basis from Ns global mode fields (FP32, device layout)
int dfl_subspace_dev(Ctx &c, const std::vector<void *> &modes, cudaStream_t st, bool lmodes) {
  DflState &d = c.dfl;
  if (lmodes) {
    const int rc = dfl_subspace_dev(c, modes, st, false);
    if (rc) return rc;
    // the modes in the new basis, for the little solver's global-mode
    // deflation (dfl_subspace.c stores them as Gram-Schmidt coefficients)
    return ltl_lmodes_from_fields(c, modes, st);
  }
  ltl_invalidate(c);
  if (gram_supported(c)) {
    // block-wise Cholesky QR (the Q of the block Gram-Schmidt of
    // dfl_subspace.c:171-240, to rounding): modes -> basis
    float4 **dm = nullptr;
    if (cudaMalloc(&dm, d.Ns * sizeof(void *)) != cudaSuccess) return fail("out of device memory");
    cudaMemcpy(dm, modes.data(), d.Ns * sizeof(void *), cudaMemcpyHostToDevice);
    const int rc = dfl_cholqr(c, (const float4 *const *)dm, (float4 *const *)d.d_basis, false, st);
    cudaFree(dm);
    if (rc < 0) return -1;
    if (rc) return fail("dfl_subspace: degenerate block modes");
    d.have_basis = true;
    d.aw_valid = d.awhat_valid = false;
    return 0;
  }
  float4 **dm = nullptr;
  int *dfail = nullptr;
  cudaMallocAsync(&dm, d.Ns * sizeof(void *), st);
  cudaMallocAsync(&dfail, sizeof(int), st);
  cudaMemcpyAsync(dm, modes.data(), d.Ns * sizeof(void *), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(dfail, 0, sizeof(int), st);
  if (!c.tmp64 && cudaMalloc(&c.tmp64, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory");
  k_dfl_gs<<<d.nb, 256, 0, st>>>(c.g, d.vd2lex, (float4 *const *)d.d_basis, (const float4 *const *)dm, d.Ns,
                                 (double2 *)c.tmp64, dfail);
  int hf = 0;
  cudaMemcpyAsync(&hf, dfail, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dm, st);
  cudaFreeAsync(dfail, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("dfl_subspace: CUDA error");
  if (hf) return fail("dfl_subspace: degenerate block modes");
  d.have_basis = true;
  d.aw_valid = d.awhat_valid = false;
  return 0;
}

// Little operator for twisted mass mu (set_Aw); returns 0
// diag_only: the diagonal blocks alone (the twisted mass enters only
// there; the hop matrices d.Ahop are those of any mass)
int dfl_set_Aw(Ctx &c, double mu, cudaStream_t st, bool diag_only) {
  DflState &d = c.dfl;
  if (!d.have_basis) return fail("set_Aw: the deflation subspace is not set");
  if (!diag_only && d.aw_valid && d.aw_mu == mu && d.aw_eo == c.eoflg) return 0;
  const double muo = c.eoflg ? 0.0 : mu;
  constexpr int TS = 8, LD = TS * 12 + 1;
  const int NT = d.Ns / 2, ntile = NT * NT;
  const size_t shm = (size_t)NT * LD * (2 * sizeof(double2) + sizeof(float4));
  const dim3 grid(d.nb, diag_only ? 1 : 9);
  const float4 *const *bas = (const float4 *const *)d.d_basis;
  if (ntile <= 256) {
    cudaFuncSetAttribute(k_aw_tiles<TS, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    k_aw_tiles<TS, 1><<<grid, 256, shm, st>>>(c.g, d.vd2lex, bas, d.Ns, c.ud, c.swd, mu, muo, d.faces, d.nfc,
                                              d.fmax, d.Ablk, d.Ahop);
  } else {
    cudaFuncSetAttribute(k_aw_tiles<TS, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    k_aw_tiles<TS, 4><<<grid, 256, shm, st>>>(c.g, d.vd2lex, bas, d.Ns, c.ud, c.swd, mu, muo, d.faces, d.nfc,
                                              d.fmax, d.Ablk, d.Ahop);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("set_Aw: CUDA error");
  d.aw_valid = true;
  d.aw_mu = mu;
  d.aw_eo = c.eoflg;
  d.awhat_valid = false;
  return 0;
}

// Even-odd preconditioned little operator (set_Awhat): inverses of the
// diagonal blocks and H = Ablk^-1 Ahop.  Returns 1 if an inversion was unsafe.
int dfl_set_Awhat(Ctx &c, double mu, cudaStream_t st, bool diag_only) {
  DflState &d = c.dfl;
  if (dfl_set_Aw(c, mu, st, diag_only)) return -1;
  if (d.awhat_valid && !diag_only) return d.awhat_fail;
  int *dfail = nullptr;
  cudaMallocAsync(&dfail, sizeof(int), st);
  cudaMemsetAsync(dfail, 0, sizeof(int), st);
  size_t shm = (size_t)2 * d.Ns * d.Ns * sizeof(double2);
  cudaFuncSetAttribute(k_cinv, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  k_cinv<<<d.nb, 256, shm, st>>>(d.Ns, d.Ablk, d.Ainv, dfail);
  k_cmatmul8<<<8 * d.nb, 256, 0, st>>>(d.Ns, d.Ainv, d.Ahop, d.Mhop);
  const size_t nm = (size_t)8 * d.nb * d.Ns * d.Ns;
  k_round32<<<(unsigned)((nm + 255) / 256), 256, 0, st>>>(d.Mhop, d.Mhop32, nm);
  int hf = 0;
  cudaMemcpyAsync(&hf, dfail, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dfail, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("set_Awhat: CUDA error");
  d.awhat_valid = true;
  d.awhat_ver++;
  d.awhat_fail = hf ? 1 : 0;
  return d.awhat_fail;
}

// w = Aw v (Aw_dble) on all blocks
void dfl_Aw(Ctx &c, const double2 *v, double2 *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_launch(0, d.Ns, 0, d.nb, d.Ablk, d.Ahop, d.nbr, v, nullptr, w, st);
}

// Aw_dble.c:202-359, on all little vectors of nv entries (even blocks
// first): w_e = Aee^-1 v_e, w_o = Aoo^-1 v_o, w_o = Aoe v_e, w_e -= Aeo v_o;
// the other half of w is unchanged
void dfl_Aweeinv(Ctx &c, const double2 *v, double2 *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_launch(3, d.Ns, 0, d.nb / 2, d.Ainv, nullptr, d.nbr, v, nullptr, w, st);
}
void dfl_Awooinv(Ctx &c, const double2 *v, double2 *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_launch(3, d.Ns, d.nb / 2, d.nb / 2, d.Ainv, nullptr, d.nbr, v, nullptr, w, st);
}
void dfl_Awoe(Ctx &c, const double2 *v, double2 *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_launch(1, d.Ns, d.nb / 2, d.nb / 2, nullptr, d.Ahop, d.nbr, v, nullptr, w, st);
}
void dfl_Aweo(Ctx &c, const double2 *v, double2 *w, cudaStream_t st) {
  DflState &d = c.dfl;
  little_launch(2, d.Ns, 0, d.nb / 2, nullptr, d.Ahop, d.nbr, w, v, w, st);
}

// w_e = v_e - H_eo H_oe v_e (Awhat_dble): t holds the odd intermediate
void dfl_Awhat(Ctx &c, const double2 *v, double2 *w, double2 *t, cudaStream_t st) {
  DflState &d = c.dfl;
  const int nbh = d.nb / 2;
  little_launch(1, d.Ns, nbh, nbh, nullptr, d.Mhop, d.nbr, v, nullptr, t, st);
  little_launch(2, d.Ns, 0, nbh, nullptr, d.Mhop, d.nbr, v, t, w, st);
}

// ------------------------------------------------------------ little solver
// Little-vector BLAS on nv complex numbers (FP64)
static double lv_dot_re(Ctx &c, const double2 *x, const double2 *y, size_t n, double *im) {
  double *scr, *od, r[4];
  flat_scratch(c, &scr, &od);
  flat_cdot(c, x, y, n, r, scr, od);
  if (im) *im = r[2] + r[3];
  return r[0] + r[1];
}

// Little-vector workspace of ltl_gcr: 2 nkv + 6 vectors of nv complex
// doubles, a device table of the Krylov vectors' addresses (p_0..p_nkv-1,
// q_0..q_nkv-1, r) for the multi-vector kernels, the dot buffers.
static int ltl_ensure(Ctx &c) {
  DflState &d = c.dfl;
  const size_t nv = (size_t)d.nv;
  const int nkv = d.nkv;
  if (nkv > LMAXK) return fail("ltl_gcr: nkv must not exceed 32");
  bool grown = false;
  while ((int)d.lv.size() < 2 * nkv + 6) {
    double2 *p = nullptr;
    if (cudaMalloc(&p, nv * sizeof(double2)) != cudaSuccess) return fail("out of device memory (little vectors)");
    d.lv.push_back(p);
    grown = true;
  }
  if (!d.lvtab) {
    if (cudaMalloc(&d.lvtab, (2 * LMAXK + 8) * sizeof(double2 *)) != cudaSuccess ||
        cudaMalloc(&d.ldots, 64 * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&d.lpart, (size_t)LGRID * LMAXK * sizeof(double2)) != cudaSuccess ||
        cudaMallocHost(&d.h_ldots, 4 * sizeof(double2)) != cudaSuccess)
      return fail("out of device memory (little solver)");
    grown = true;
  }
  if (grown || d.lvtab_nkv != nkv) {
    std::vector<double2 *> tab(2 * nkv + 1);
    for (int k = 0; k < nkv; k++) {
      tab[k] = d.lv[6 + k];
      tab[nkv + k] = d.lv[6 + nkv + k];
    }
    tab[2 * nkv] = d.lv[1];
    cudaMemcpy(d.lvtab, tab.data(), tab.size() * sizeof(double2 *), cudaMemcpyHostToDevice);
    d.lvtab_nkv = nkv;
  }
  return 0;
}

static void ldot(Ctx &c, double2 *const *Q, int k, const double2 *y, int n, double2 *out, cudaStream_t st) {
  DflState &d = c.dfl;
  k_mdot<<<LGRID, 256, 0, st>>>((const double2 *const *)Q, k, y, n, d.lpart);
  k_mdot_fin<<<1, 32, 0, st>>>(d.lpart, k, out);
}

// ltl_gcr (modules/dfl/ltl_gcr.c:155): even-odd reduction of the little
// system, GCR on Awhat for the even blocks to relative residue res (at most
// nmx Krylov vectors, restart after nkv), back-substitution for the odd
// blocks.  The reference additionally preconditions with a single-precision
// GCR and deflates the little-little modes; this solver runs plain
// double-precision GCR with the same stopping rule.  The Krylov step runs on
// the device: the Gram-Schmidt coefficients (classical Gram-Schmidt, applied
// twice), the normalisation and the update coefficient never leave the GPU,
// and the host reads two numbers per step (|q_k|^2 and |r|^2) for the
// stopping test.  Returns the norm of the residue of the even-odd
// preconditioned system; ifail 0, -1 (no convergence) or -2 (unsafe
// inversion).
double dfl_ltl_gcr(Ctx &c, double mu, const double2 *eta, double2 *psi, int *ifail, int *status,
                   cudaStream_t st) {
  DflState &d = c.dfl;
  ifail[0] = 0;
  status[0] = 0;
  const size_t nv = (size_t)d.nv, nvh = nv / 2;
  const int nbh = d.nb / 2, n = (int)nvh;
  if (dfl_set_Awhat(c, mu, st)) {
    ifail[0] = -2;
    cudaMemsetAsync(psi, 0, nv * sizeof(double2), st);
    return sqrt(lv_dot_re(c, eta, eta, nv, nullptr));
  }
  if (ltl_ensure(c)) return -1.0;
  const int nkv = d.nkv;
  double2 *x = d.lv[0], *r = d.lv[1], *t = d.lv[2], *eh = d.lv[3], *w = d.lv[4], *y = d.lv[5];
  double2 **p = &d.lv[6], **q = &d.lv[6 + nkv];
  double2 *const *Ptab = d.lvtab, *const *Qtab = d.lvtab + nkv, *const *Rtab = d.lvtab + 2 * nkv;
  double2 *dots = d.ldots;
  const unsigned gv = (unsigned)std::min<size_t>((nvh + 255) / 256, 4 * 148);
  auto read3 = [&](double *nq2, double *rr) {
    cudaMemcpyAsync(d.h_ldots, dots + 32, 3 * sizeof(double2), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    *nq2 = d.h_ldots[0].x;
    *rr = d.h_ldots[2].x;
  };
  // eh_e = Aee^-1 (eta_e - Aeo Aoo^-1 eta_o)   [even half of eh]
  cudaMemcpyAsync(w, eta, nv * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  little_launch(3, d.Ns, nbh, nbh, d.Ainv, nullptr, d.nbr, eta, nullptr, w, st);    // w_o = Aoo^-1 eta_o
  little_launch(2, d.Ns, 0, nbh, nullptr, d.Ahop, d.nbr, eta, w, t, st);            // t_e = eta_e - Aeo w_o
  little_launch(3, d.Ns, 0, nbh, d.Ainv, nullptr, d.nbr, t, nullptr, eh, st);       // eh_e = Aee^-1 t_e
  // GCR on Awhat x = eh (even half)
  cudaMemsetAsync(x, 0, nvh * sizeof(double2), st);
  cudaMemcpyAsync(r, eh, nvh * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  double nq2 = 0.0, rr = 0.0;
  ldot(c, Rtab, 1, r, n, dots + 34, st);
  read3(&nq2, &rr);
  const double rn0 = sqrt(rr);
  double rn = rn0;
  const double tol = d.res * rn0;
  int it = 0;
  while (rn > tol && it < d.nmx) {
    for (int k = 0; k < nkv && it < d.nmx && rn > tol; k++) {
      cudaMemcpyAsync(p[k], r, nvh * sizeof(double2), cudaMemcpyDeviceToDevice, st);
      dfl_Awhat(c, p[k], q[k], y, st);
      if (k > 0)
        for (int pass = 0; pass < 2; pass++) {
          ldot(c, Qtab, k, q[k], n, dots, st);
          k_gs_sub<<<gv, 256, 0, st>>>(Qtab, Ptab, k, dots, q[k], p[k], n);
        }
      ldot(c, Qtab + k, 1, q[k], n, dots + 32, st);
      k_norm_scale<<<gv, 256, 0, st>>>(q[k], p[k], dots + 32, n);
      ldot(c, Qtab + k, 1, r, n, dots + 33, st);
      k_xr_update<<<gv, 256, 0, st>>>(x, r, p[k], q[k], dots + 33, n);
      ldot(c, Rtab, 1, r, n, dots + 34, st);
      read3(&nq2, &rr);
      if (nq2 == 0.0) break;
      it++;
      rn = sqrt(rr);
    }
    // restart from the true residual
    dfl_Awhat(c, x, w, y, st);
    cudaMemcpyAsync(r, eh, nvh * sizeof(double2), cudaMemcpyDeviceToDevice, st);
    flat_caxpy(c, r, w, nvh, -1.0, 0.0);
    ldot(c, Rtab, 1, r, n, dots + 34, st);
    read3(&nq2, &rr);
    rn = sqrt(rr);
    if (nq2 == 0.0 && rn > tol) break;   // the Krylov space collapsed
  }
  status[0] = it;
  if (rn > tol) ifail[0] = -1;
  // psi_e = x_e ; psi_o = Aoo^-1 (eta_o - Aoe x_e)
  cudaMemcpyAsync(psi, x, nvh * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  little_launch(2, d.Ns, nbh, nbh, nullptr, d.Ahop, d.nbr, eta, x, t, st);          // t_o = eta_o - Aoe x_e
  little_launch(3, d.Ns, nbh, nbh, d.Ainv, nullptr, d.nbr, t, nullptr, psi, st);     // psi_o
  return rn;
}

// ------------------------------------------------------ deflated SAP+GCR
static int reserve32(Ctx &c, std::vector<void *> &v, size_t n) {
  while (v.size() < n) {
    void *p = nullptr;
    if (cudaMalloc(&p, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory (workspace)");
    v.push_back(p);
  }
  return 0;
}

// Mop of dfl_sap_gcr (modules/dfl/dfl_sap_gcr.c:212-241): little solve of the
// restricted residue, prolongation, SAP on the remainder.
static void dfl_mop(Ctx &c, double mu, const void *rho, void *phi, void *chi, void *ws0, void *phib, int *lstat) {
  DflState &d = c.dfl;
  cudaStream_t st = c.stream;
  double2 *vd = d.lvd[0];
  int ifail, status[2] = {0, 0};
  dfl_mark(c, 5);
  dfl_restrict(c, 32, rho, vd, st);
  if (d.ltl_kind == 1) ltl_gcr_ref(c, mu, vd, vd, &ifail, status, st);
  else dfl_ltl_gcr(c, mu, vd, vd, &ifail, status, st);
  dfl_prolong(c, vd, ws0, st);
  dfl_mark(c, 3);
  // rho - D ws0, written where the SAP sequence reads its input
  void *in = sap_input_field(c);
  if (!in) in = chi;
  void *const sv[1] = {ws0}, *const rv[1] = {in}, *const bv[1] = {(void *)rho};
  dirac_multi32(c, 1, (float)mu, sv, rv, bv, st);
  dfl_mark(c, 5);
  // SAP on it, then chi = rho - (final residual), phi = SAP solution + ws0
  sap_mop(c, (float)mu, c.isolv, c.nmr, c.ncy, in, phi, chi, phib, st, rho, ws0);
  dfl_mark(c, 4);
  lstat[0] += status[0];
  lstat[1] += status[1];
}

int ensure_lvd_n(Ctx &c, int n) {
  DflState &d = c.dfl;
  while ((int)d.lvd.size() < n) {
    double2 *p = nullptr;
    if (cudaMalloc(&p, (size_t)d.nv * sizeof(double2)) != cudaSuccess) return fail("out of device memory");
    d.lvd.push_back(p);
  }
  return 0;
}

static int ensure_lvd(Ctx &c) {
  DflState &d = c.dfl;
  while (d.lvd.size() < 2) {
    double2 *p = nullptr;
    if (cudaMalloc(&p, (size_t)d.nv * sizeof(double2)) != cudaSuccess) return fail("out of device memory");
    d.lvd.push_back(p);
  }
  return 0;
}

// dfl_sap_gcr on device fields (FP64 eta, psi; psi may equal eta)
double dfl_sap_gcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                       int *ifail, int *status) {
  DflState &d = c.dfl;
  ifail[0] = 0;
  status[0] = status[1] = status[2] = 0;
  if (!c.sap_set) { fail("dfl_sap_gcr: SAP parameters are not set"); return -1.0; }
  if (!d.ready || !d.have_basis) { fail("dfl_sap_gcr: the deflation subspace is not set"); return -1.0; }
  if (sap_prepare(c, c.stream) || ensure_lvd(c)) return -1.0;
  cudaStream_t st = c.stream;
  double rho;
  {
    double r[2];
    if (istop) { la_unorm(c, 64, eta, PAR_ALL, r); rho = r[0]; }
    else { la_norm2(c, 64, eta, PAR_ALL, r); rho = sqrt(r[0]); }
  }
  if (c.isolv == 1 && (c.sw_inv_fail & 2)) {
    ifail[0] = -3;
  } else if ((dfl_mark(c, 5), dfl_set_Awhat(c, mu, st))) {
    ifail[0] = -2;
  } else if ((dfl_mark(c, 2), rho != 0.0)) {
    if (reserve32(c, c.ws32, 2 * nkv + 3)) return -1.0;
    while (c.ws64.size() < 3) {
      void *p = nullptr;
      if (cudaMalloc(&p, spinor_bytes(c, 64)) != cudaSuccess) { fail("out of device memory"); return -1.0; }
      c.ws64.push_back(p);
    }
    void *rsd = c.ws64[1];
    void *phib = c.ws32[2 * nkv + 1], *ws0 = c.ws32[2 * nkv + 2];
    const double rho0 = rho;
    la_copy(c, 64, eta, 64, rsd, PAR_ALL, st);
    la_scale(c, 64, rsd, 1.0 / rho0, PAR_ALL, st);
    int lstat[2] = {0, 0};
    std::function<void(const void *, void *)> Dop = [&](const void *s, void *r) {
      dirac_op<double>(c, 0, mu, s, r, c.tmp64, st);
    };
    std::function<void(int, const void *, void *, void *)> Mop = [&](int, const void *rh, void *ph, void *ch) {
      dfl_mop(c, mu, rh, ph, ch, ws0, phib, lstat);
    };
    std::vector<void *> phi(c.ws32.begin(), c.ws32.begin() + nkv),
        chi(c.ws32.begin() + nkv + 1, c.ws32.begin() + 2 * nkv + 1);
    rho = fgcr_core(dev_krylov_ops(c), nkv, nmx, istop, res, rsd, psi, status, Dop, Mop, phi, chi, c.ws32[nkv],
                    c.ws64[0]);
    la_scale(c, 64, psi, rho0, PAR_ALL, st);
    rho *= rho0;
    if (status[0] < 0) {
      ifail[0] = -1;
      status[0] = nmx;
    }
    if (status[0] > 0) {
      status[1] = (lstat[0] + status[0] / 2) / status[0];
      status[2] = (lstat[1] + status[0] / 2) / status[0];
    }
  } else {
    la_zero(c, 64, psi, PAR_ALL, st);
  }
  if (ifail[0] <= -2 && psi != eta) la_zero(c, 64, psi, PAR_ALL, st);
  cudaStreamSynchronize(st);
  return rho;
}

// ---------------------------------------------------- subspace generation
// dfl_modes (modules/dfl/dfl_modes.c:423-502): Ns random fields smoothed by
// 1, 2 and 3 SAP cycles, block-orthonormalised, then ninv-3 steps of
// deflated inverse iteration (little solve of the restricted mode, SAP on
// the remainder), global renormalisation and block orthonormalisation.
// The iteration uses the generation mass m0 = 1/(2 kappa) - 4, twisted mass
// mu_gen and the twisted-mass eo flag set, as the reference does.
int dfl_modes_dev(Ctx &c, uint64_t seed, int *ifail, int *status) {
  DflState &d = c.dfl;
  ifail[0] = 0;
  status[0] = status[1] = 0;
  if (!d.ready) return fail("dfl_modes: deflation parameters are not set");
  if (!d.gen_set) return fail("dfl_modes: subspace generation parameters are not set");
  if (d.gen_kappa == 0.0) return fail("dfl_modes: kappa = 0 (infinite generation mass) is not supported");
  if (!c.sap_set) return fail("dfl_modes: SAP parameters are not set");
  cudaStream_t st = c.stream;
  if (sap_prepare(c, st) || ensure_lvd(c) || reserve32(c, d.modes, d.Ns) || reserve32(c, c.ws32, 9 + 2 * SAP_MS) ||
      dfl_batch_alloc(c) || ensure_lvd_n(c, 4))
    return -1;
  // device table of the mode fields (for the Cholesky QR kernels)
  float4 **dmodes = nullptr;
  if (cudaMalloc(&dmodes, d.Ns * sizeof(void *)) != cudaSuccess) return fail("out of device memory");
  cudaMemcpy(dmodes, d.modes.data(), d.Ns * sizeof(void *), cudaMemcpyHostToDevice);
  struct FreeTab {
    float4 **p;
    ~FreeTab() { cudaFree(p); }
  } free_tab{dmodes};
  // generation mass and eo flag
  const double m0_save = c.m0;
  const int eo_save = c.eoflg;
  const double m0g = 1.0 / (2.0 * d.gen_kappa) - 4.0;
  if (m0g != c.m0) {
    if (sw_shift_mass(c, m0g - c.m0, st)) return -1;
    c.m0 = m0g;
  }
  c.eoflg = 1;
  if (c.sw_inv_fail & 2) ifail[0] = -3;
  // SAP runs on up to SAP_MS modes per launch: ws32[9 ..] holds their
  // residuals in the smoothing rounds, ws32[9 + SAP_MS ..] their block
  // scratch
  void *const *rs = c.ws32.data() + 9, *const *phib = c.ws32.data() + 9 + SAP_MS;
  const float mug = (float)d.gen_mu;
  if (d.use_start) {
    // the caller's start fields (e.g. the reference's ranlxs fields)
    for (int l = 0; l < d.Ns; l++) la_copy(c, 32, d.start[l], 32, d.modes[l], PAR_ALL, st);
    d.use_start = false;
  } else {
    for (int l = 0; l < d.Ns; l++) gen_uniform_spinor32(c, d.modes[l], seed * 1000003ull + l, st);
  }
  dfl_mark(c, -1);
  if (ifail[0] == 0) {
    int n;
    for (n = 0; n < 3; n++) {
      for (int l0 = 0; l0 < d.Ns; l0 += SAP_MS) {
        const int m = std::min(SAP_MS, d.Ns - l0);
        for (int i = 0; i < m; i++) {
          la_copy(c, 32, d.modes[l0 + i], 32, rs[i], PAR_ALL, st);
          la_zero(c, 32, d.modes[l0 + i], PAR_ALL, st);
        }
        if (sap_cycles_multi(c, m, mug, 1, d.gen_nmr, n + 1, d.modes.data() + l0, rs, phib, st)) return -1;
      }
    }
    dfl_mark(c, 0);
    if (dfl_subspace_dev(c, d.modes, st)) return -1;
    dfl_mark(c, 1);
    for (; n < d.gen_ninv && ifail[0] == 0; n++) {
      if (dfl_set_Awhat(c, d.gen_mu, st)) {
        ifail[0] = -2;
        break;
      }
      dfl_mark(c, 2);
      // one step of the deflated inverse iteration per mode
      // (dfl_modes.c:354-380: restriction, little solve, prolongation,
      // residual, SAP on it), the deflation part for four modes at a time
      // with the multi-right-hand-side kernels
      for (int l0 = 0; l0 < d.Ns; l0 += 4) {
        const int na = std::min(4, d.Ns - l0);
        const void *rh[4];
        double2 *vd[4];
        void *w1[4], *w0[4], *md[4];
        int lf[4], ls[4];
        for (int i = 0; i < na; i++) {
          rh[i] = d.modes[l0 + i];
          md[i] = d.modes[l0 + i];
          vd[i] = d.lvd[i];
          w0[i] = c.ws32[i];
          w1[i] = c.ws32[4 + i];
        }
        dfl_restrict_b(c, na, rh, vd, st);
        if (ltl_gcr_b(c, d.gen_mu, na, (const double2 *const *)vd, vd, lf, ls, st)) return -1;
        dfl_prolong_b(c, na, (const double2 *const *)vd, w1, st);
        dfl_mark(c, 3);
        dirac_multi32(c, na, mug, w1, w0, md, st);          // w0 = mode - D w1
        dfl_mark(c, 5);
        for (int i = 0; i < na; i++) la_zero(c, 32, d.modes[l0 + i], PAR_ALL, st);
        if (sap_cycles_multi(c, na, mug, 1, d.gen_nmr, d.gen_ncy, d.modes.data() + l0, w0, phib, st)) return -1;
        for (int i = 0; i < na; i++) {
          la_axpy(c, 32, d.modes[l0 + i], 1.0, 0.0, w1[i], PAR_ALL, st);
          status[0] += ls[i];
        }
        dfl_mark(c, 4);
      }
      // dfl_renormalize_modes (dfl_subspace.c:243-259): the global modes
      // orthonormalised in order, here by Cholesky QR over the lattice
      if (gram_supported(c)) {
        const int rc = dfl_cholqr(c, (const float4 *const *)dmodes, (float4 *const *)dmodes, true, st);
        if (rc < 0) return -1;
        if (rc) return fail("dfl_modes: the modes became linearly dependent");
      } else {
        for (int l = 0; l < d.Ns; l++) {
          for (int j = 0; j < l; j++) {
            double r[4];
            la_dot(c, 32, d.modes[j], d.modes[l], PAR_ALL, r);
            la_axpy(c, 32, d.modes[l], -(float)(r[0] + r[1]), -(float)(r[2] + r[3]), d.modes[j], PAR_ALL, st);
          }
          double r[2];
          la_norm2(c, 32, d.modes[l], PAR_ALL, r);
          float nrm = (float)sqrt((double)(float)(r[0] + r[1]));
          if (nrm != 0.0f) la_scale(c, 32, d.modes[l], 1.0f / nrm, PAR_ALL, st);
        }
      }
      dfl_mark(c, 5);
      if (dfl_subspace_dev(c, d.modes, st)) return -1;
      dfl_mark(c, 1);
    }
    const int nst = d.Ns * (n - 3);
    if (nst > 0) status[0] = (status[0] + nst / 2) / nst;
    // the modes in the final basis (little modes of the little solver)
    if (ltl_lmodes_from_fields(c, d.modes, st)) return -1;
  } else {
    if (dfl_subspace_dev(c, d.modes, st)) return -1;
  }
  // restore the mass and the eo flag
  c.eoflg = eo_save;
  if (c.m0 != m0_save) {
    if (sw_shift_mass(c, m0_save - c.m0, st)) return -1;
    c.m0 = m0_save;
  }
  d.aw_valid = d.awhat_valid = false;
  // the modes are regenerated from random fields by every call
  for (void *p : d.modes) cudaFree(p);
  d.modes.clear();
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : fail("dfl_modes: CUDA error");
}

}  // namespace qcd
