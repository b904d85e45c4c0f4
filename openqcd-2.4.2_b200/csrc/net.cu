// Learned preconditioner: a gauge-equivariant parallel-transport
// convolutional network (no reference counterpart).
//
// A field with C channels is C colour triplets per site; an FP32 spinor
// field in the library's layout holds four channels (its four spin
// components), so a C-channel activation is C/4 spinor fields.  One layer
// maps Cin to Cout channels by
//
//   y_o(x) = sum_{d=0..8} sum_i W_d[o][i] (T_d psi_i)(x),
//   T_0 psi(x) = psi(x),  T_{+mu} psi(x) = U(x,mu) psi(x+mu),
//   T_{-mu} psi(x) = U(x-mu,mu)^dag psi(x-mu),
//
// with complex weights acting on the channel index only: colour is moved
// by the links alone, so the layer commutes with gauge transformations.
// The network has three such layers, 4 -> 8 -> 8 -> 4 channels (12, 24,
// 24, 12 spin-colour components), and no nonlinearity: the map it learns,
// an approximation of Dw^-1, is linear (as in the published
// gauge-equivariant preconditioner models).  Direction index d: 0 self,
// 1 + 2 mu the forward hop (+mu), 2 + 2 mu the backward hop (-mu).
//
// Training (Adam on the real and imaginary parts of the 2304 weights) runs
// on the device with these kernels: the forward layer, its adjoint (the
// same kernel with weights W'_{dbar}[i][o] = conj(W_d[o][i]), dbar the
// opposite direction, since T_{+mu}^dag = T_{-mu}), and the weight
// gradient G_d[o][i] = sum_x g_o(x) . conj((T_d psi_i)(x)) as a reduction
// over site tiles.  Loss: the mean over a batch of |M r - e|^2 / |e|^2 for
// pairs (r, e) with Dw e = r.  Inference uses the weights rounded to FP16
// (arithmetic in FP32).
#include "lib.h"
#include <cuda_fp16.h>
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace qcd {

static const int NCH[4] = {4, 8, 8, 4};
static const int NLAY = 3;

static int wsize(int l) { return 9 * NCH[l + 1] * NCH[l]; }   // complex weights of layer l

template <int N> struct FPtr {
  float4 *p[N];
};

// ------------------------------------------------------------ layer kernel
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_ptconv(Geom g, const float2 *__restrict__ u, FPtr<CIN / 4> in,
                                                const float2 *__restrict__ w, FPtr<COUT / 4> out) {
  __shared__ float2 ws[9 * COUT * CIN];
  for (int q = threadIdx.x; q < 9 * COUT * CIN; q += blockDim.x) ws[q] = w[q];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.vol) return;
  const int chunk = i / g.vbh, s = i - chunk * g.vbh;
  const int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
  Site x;
  site_decode(g, p, blk, s, x);
  float ar[COUT][3], ai[COUT][3];
#pragma unroll
  for (int o = 0; o < COUT; o++)
#pragma unroll
    for (int c = 0; c < 3; c++) ar[o][c] = ai[o][c] = 0.0f;
#pragma unroll 1
  for (int d = 0; d < 9; d++) {
    int c2 = chunk, s2 = s;
    su3<float> uu;
    const int mu = (d - 1) >> 1;
    if (d > 0) {
      const int dir = (d & 1) ? 1 : -1;
      site_nbr(g, x, mu, dir, c2, s2);
      uu = dir > 0 ? Store<float>::load_link(u, chunk, mu, s, g.vbh) : Store<float>::load_link(u, c2, mu, s2, g.vbh);
    }
#pragma unroll
    for (int f = 0; f < CIN / 4; f++) {
      const spinor<float> v = Store<float>::load_spinor(in.p[f], c2, s2, g.vbh);
#pragma unroll
      for (int a = 0; a < 4; a++) {
        vec3<float> t = v.c[a];
        if (d > 0) t = (d & 1) ? umul(uu, v.c[a]) : udagmul(uu, v.c[a]);
        const int ci = 4 * f + a;
#pragma unroll
        for (int o = 0; o < COUT; o++) {
          const float2 wv = ws[(d * COUT + o) * CIN + ci];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            ar[o][c] += wv.x * t.c[c].re - wv.y * t.c[c].im;
            ai[o][c] += wv.x * t.c[c].im + wv.y * t.c[c].re;
          }
        }
      }
    }
  }
#pragma unroll
  for (int f = 0; f < COUT / 4; f++) {
    spinor<float> r;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int c = 0; c < 3; c++) r.c[a].c[c] = mk<float>(ar[4 * f + a][c], ai[4 * f + a][c]);
    Store<float>::store_spinor(out.p[f], chunk, s, g.vbh, r);
  }
}

// ------------------------------------------------------- weight gradient
// part[cta][d][o][i] = sum over the CTA's sites of g_o . conj(T_d psi_i):
// a tile of TSW sites is staged in shared memory (g and, direction by
// direction, the transported input), thread (pair, quarter) sums a quarter
// of the tile's sites for one (o, i) pair and all nine directions.
constexpr int TSW = 32, WG_GRID = 296;

template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_ptconv_wgrad(Geom g, const float2 *__restrict__ u, FPtr<CIN / 4> in,
                                                      FPtr<COUT / 4> gout, float2 *part) {
  __shared__ float2 G[TSW][COUT][3];
  __shared__ float2 Tt[TSW][CIN][3];
  const int q = threadIdx.x, pair = q >> 2, quarter = q & 3;
  const bool active = pair < COUT * CIN;
  const int o = active ? pair / CIN : 0, ii = active ? pair % CIN : 0;
  float accr[9], acci[9];
#pragma unroll
  for (int d = 0; d < 9; d++) accr[d] = acci[d] = 0.0f;
  for (int t0 = blockIdx.x * TSW; t0 < g.vol; t0 += gridDim.x * TSW) {
    // stage g for the tile
    for (int e = threadIdx.x; e < TSW * (COUT / 4); e += blockDim.x) {
      const int sl = e % TSW, f = e / TSW, site = t0 + sl;
      spinor<float> v;
      szero(v);
      if (site < g.vol) {
        const int chunk = site / g.vbh, s = site - chunk * g.vbh;
        v = Store<float>::load_spinor(gout.p[f], chunk, s, g.vbh);
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) G[sl][4 * f + a][c] = make_float2(v.c[a].c[c].re, v.c[a].c[c].im);
    }
#pragma unroll 1
    for (int d = 0; d < 9; d++) {
      __syncthreads();
      for (int e = threadIdx.x; e < TSW * (CIN / 4); e += blockDim.x) {
        const int sl = e % TSW, f = e / TSW, site = t0 + sl;
        spinor<float> v;
        szero(v);
        if (site < g.vol) {
          const int chunk = site / g.vbh, s = site - chunk * g.vbh;
          const int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
          if (d == 0) {
            v = Store<float>::load_spinor(in.p[f], chunk, s, g.vbh);
          } else {
            Site x;
            site_decode(g, p, blk, s, x);
            const int mu = (d - 1) >> 1, dir = (d & 1) ? 1 : -1;
            int c2, s2;
            site_nbr(g, x, mu, dir, c2, s2);
            const su3<float> uu =
                dir > 0 ? Store<float>::load_link(u, chunk, mu, s, g.vbh) : Store<float>::load_link(u, c2, mu, s2, g.vbh);
            const spinor<float> n = Store<float>::load_spinor(in.p[f], c2, s2, g.vbh);
#pragma unroll
            for (int a = 0; a < 4; a++) v.c[a] = dir > 0 ? umul(uu, n.c[a]) : udagmul(uu, n.c[a]);
          }
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int c = 0; c < 3; c++) Tt[sl][4 * f + a][c] = make_float2(v.c[a].c[c].re, v.c[a].c[c].im);
      }
      __syncthreads();
      if (active) {
        float sr = 0.0f, si = 0.0f;
        for (int sl = quarter; sl < TSW; sl += 4)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const float2 a = G[sl][o][c], b = Tt[sl][ii][c];
            sr += a.x * b.x + a.y * b.y;   // a conj(b)
            si += a.y * b.x - a.x * b.y;
          }
        accr[d] += sr;
        acci[d] += si;
      }
    }
    __syncthreads();
  }
  // sum the four quarters (adjacent lanes)
#pragma unroll
  for (int d = 0; d < 9; d++) {
    accr[d] += __shfl_xor_sync(0xffffffffu, accr[d], 1);
    acci[d] += __shfl_xor_sync(0xffffffffu, acci[d], 1);
    accr[d] += __shfl_xor_sync(0xffffffffu, accr[d], 2);
    acci[d] += __shfl_xor_sync(0xffffffffu, acci[d], 2);
  }
  if (active && quarter == 0)
#pragma unroll
    for (int d = 0; d < 9; d++)
      part[((size_t)blockIdx.x * 9 + d) * COUT * CIN + o * CIN + ii] = make_float2(accr[d], acci[d]);
}

// grad[j] += sum over CTAs of part[cta][j] (fixed order, double)
__global__ void k_wgrad_sum(const float2 *__restrict__ part, int nw, int ncta, double2 *grad) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nw) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < ncta; b++) {
    const float2 v = part[(size_t)b * nw + j];
    re += v.x;
    im += v.y;
  }
  grad[j].x += re;
  grad[j].y += im;
}

// ----------------------------------------------------------- host side
static int net_alloc(Ctx &c) {
  NetState &n = c.net;
  if (n.dev_w[0]) return 0;
  for (int l = 0; l < NLAY; l++) {
    if (cudaMalloc(&n.dev_w[l], wsize(l) * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&n.dev_wadj[l], wsize(l) * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&n.dev_w16[l], wsize(l) * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&n.dev_grad[l], wsize(l) * sizeof(double2)) != cudaSuccess)
      return fail("out of device memory (network)");
  }
  if (cudaMalloc(&n.part, (size_t)WG_GRID * 9 * 64 * sizeof(float2)) != cudaSuccess)
    return fail("out of device memory (network)");
  return 0;
}

// host weights -> device copies (FP32, adjoint, FP16-rounded)
static int net_upload(Ctx &c) {
  NetState &n = c.net;
  for (int l = 0; l < NLAY; l++) {
    const int ci = NCH[l], co = NCH[l + 1];
    std::vector<float2> w(wsize(l)), wa(wsize(l)), w16(wsize(l));
    for (int d = 0; d < 9; d++) {
      const int db = d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1);
      for (int o = 0; o < co; o++)
        for (int i = 0; i < ci; i++) {
          const int q = (d * co + o) * ci + i;
          const float re = n.w[l][2 * q], im = n.w[l][2 * q + 1];
          w[q] = make_float2(re, im);
          w16[q] = make_float2(__half2float(__float2half_rn(re)), __half2float(__float2half_rn(im)));
          // adjoint layer: co <- ci, direction db, entry [i][o] = conj(W_d[o][i])
          wa[(db * ci + i) * co + o] = make_float2(re, -im);
        }
    }
    cudaMemcpy(n.dev_w[l], w.data(), w.size() * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(n.dev_wadj[l], wa.data(), wa.size() * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(n.dev_w16[l], w16.data(), w16.size() * sizeof(float2), cudaMemcpyHostToDevice);
  }
  n.ready = true;
  return cudaGetLastError() == cudaSuccess ? 0 : fail("network: upload failed");
}

int net_set_weights(Ctx &c, const float *w) {
  if (net_alloc(c)) return -1;
  NetState &n = c.net;
  const float *p = w;
  for (int l = 0; l < NLAY; l++) {
    n.w[l].assign(p, p + 2 * wsize(l));
    p += 2 * wsize(l);
    n.m[l].assign(2 * wsize(l), 0.0f);
    n.v[l].assign(2 * wsize(l), 0.0f);
  }
  n.t = 0;
  return net_upload(c);
}

int net_get_weights(Ctx &c, float *w) {
  NetState &n = c.net;
  if (!n.ready) return fail("network: no weights");
  float *p = w;
  for (int l = 0; l < NLAY; l++) {
    std::copy(n.w[l].begin(), n.w[l].end(), p);
    p += 2 * wsize(l);
  }
  return 0;
}

int net_nweights() {
  int s = 0;
  for (int l = 0; l < NLAY; l++) s += 2 * wsize(l);
  return s;
}

// initial weights: the network starts close to (scale) x identity, with
// small random couplings to every direction and channel
int net_init(Ctx &c, uint64_t seed, float scale) {
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  std::vector<float> all;
  for (int l = 0; l < NLAY; l++) {
    const int ci = NCH[l], co = NCH[l + 1];
    for (int d = 0; d < 9; d++)
      for (int o = 0; o < co; o++)
        for (int i = 0; i < ci; i++) {
          float re = 0.02f * nd(rng) / std::sqrt((float)ci), im = 0.02f * nd(rng) / std::sqrt((float)ci);
          if (d == 0 && o == i) re += (l == 2 ? scale : 1.0f);
          all.push_back(re);
          all.push_back(im);
        }
  }
  return net_set_weights(c, all.data());
}

template <int CIN, int COUT>
static void layer(Ctx &c, const float2 *w, void *const *in, void *const *out, cudaStream_t st) {
  FPtr<CIN / 4> a;
  FPtr<COUT / 4> b;
  for (int f = 0; f < CIN / 4; f++) a.p[f] = (float4 *)in[f];
  for (int f = 0; f < COUT / 4; f++) b.p[f] = (float4 *)out[f];
  k_ptconv<CIN, COUT><<<(c.g.vol + 127) / 128, 128, 0, st>>>(c.g, c.u32, a, w, b);
}

template <int CIN, int COUT>
static void wgrad(Ctx &c, void *const *in, void *const *gout, double2 *grad, cudaStream_t st) {
  FPtr<CIN / 4> a;
  FPtr<COUT / 4> b;
  for (int f = 0; f < CIN / 4; f++) a.p[f] = (float4 *)in[f];
  for (int f = 0; f < COUT / 4; f++) b.p[f] = (float4 *)gout[f];
  k_ptconv_wgrad<CIN, COUT><<<WG_GRID, 256, 0, st>>>(c.g, c.u32, a, b, c.net.part);
  const int nw = 9 * CIN * COUT;
  k_wgrad_sum<<<(nw + 127) / 128, 128, 0, st>>>(c.net.part, nw, WG_GRID, grad);
}

static int net_fields(Ctx &c) {
  NetState &n = c.net;
  while (n.f.size() < 10) {
    void *p = nullptr;
    if (cudaMalloc(&p, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory (network)");
    n.f.push_back(p);
  }
  return 0;
}

// out = M in (FP32 device fields); half = use the FP16-rounded weights
int net_apply(Ctx &c, const void *in, void *out, bool half, cudaStream_t st) {
  NetState &n = c.net;
  if (!n.ready) return fail("network: no weights");
  if (!c.have_ud) return fail("network: no gauge field on the device");
  if (net_fields(c)) return -1;
  void *x0[1] = {const_cast<void *>(in)}, *a1[2] = {n.f[0], n.f[1]}, *a2[2] = {n.f[2], n.f[3]}, *y[1] = {out};
  float2 *const *W = half ? n.dev_w16 : n.dev_w;
  layer<4, 8>(c, W[0], x0, a1, st);
  layer<8, 8>(c, W[1], a1, a2, st);
  layer<8, 4>(c, W[2], a2, y, st);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("network: launch failed");
}

// loss |M r - e|^2 / |e|^2 * wt of one pair, gradient added into dev_grad
static int net_pair_grad(Ctx &c, const void *r, const void *e, double wt, double *loss, cudaStream_t st) {
  NetState &n = c.net;
  void *x0[1] = {const_cast<void *>(r)}, *a1[2] = {n.f[0], n.f[1]}, *a2[2] = {n.f[2], n.f[3]}, *y[1] = {n.f[4]};
  void *g3[1] = {n.f[4]}, *g2[2] = {n.f[5], n.f[6]}, *g1[2] = {n.f[7], n.f[8]};
  layer<4, 8>(c, n.dev_w[0], x0, a1, st);
  layer<8, 8>(c, n.dev_w[1], a1, a2, st);
  layer<8, 4>(c, n.dev_w[2], a2, y, st);
  double en[2], rn[2];
  la_norm2(c, 32, e, PAR_ALL, en);
  la_axpy(c, 32, y[0], -1.0, 0.0, e, PAR_ALL, st);        // y = M r - e
  la_norm2(c, 32, y[0], PAR_ALL, rn);
  const double e2 = en[0] + en[1], r2 = rn[0] + rn[1];
  if (!(e2 > 0.0)) return fail("network: a target field is zero");
  *loss = wt * r2 / e2;
  // G = 2 wt (M r - e) / |e|^2 is the gradient of the loss w.r.t. conj(y), doubled
  la_scale(c, 32, g3[0], 2.0 * wt / e2, PAR_ALL, st);
  wgrad<8, 4>(c, a2, g3, n.dev_grad[2], st);
  layer<4, 8>(c, n.dev_wadj[2], g3, g2, st);
  wgrad<8, 8>(c, a1, g2, n.dev_grad[1], st);
  layer<8, 8>(c, n.dev_wadj[1], g2, g1, st);
  wgrad<4, 8>(c, x0, g1, n.dev_grad[0], st);
  return cudaGetLastError() == cudaSuccess ? 0 : fail("network: launch failed");
}

static void grad_zero(Ctx &c, cudaStream_t st) {
  for (int l = 0; l < NLAY; l++) cudaMemsetAsync(c.net.dev_grad[l], 0, wsize(l) * sizeof(double2), st);
}

static void grad_read(Ctx &c, std::vector<double> *g) {
  for (int l = 0; l < NLAY; l++) {
    g[l].resize(2 * wsize(l));
    cudaMemcpy(g[l].data(), c.net.dev_grad[l], wsize(l) * sizeof(double2), cudaMemcpyDeviceToHost);
  }
}

// loss and gradient (d/dRe w, d/dIm w, packed like the weights) of one pair
int net_grad(Ctx &c, const void *r, const void *e, double *loss, float *grad) {
  NetState &n = c.net;
  if (!n.ready) return fail("network: no weights");
  if (!c.have_ud) return fail("network: no gauge field on the device");
  if (net_fields(c)) return -1;
  cudaStream_t st = c.stream;
  grad_zero(c, st);
  if (net_pair_grad(c, r, e, 1.0, loss, st)) return -1;
  cudaStreamSynchronize(st);
  std::vector<double> g[NLAY];
  grad_read(c, g);
  float *p = grad;
  for (int l = 0; l < NLAY; l++)
    for (size_t k = 0; k < g[l].size(); k++) *p++ = (float)g[l][k];
  return 0;
}

// mean loss and mean gradient over npairs pairs (one minibatch; a rank of a
// data-parallel training sums these over ranks before the Adam step)
int net_batch_grad(Ctx &c, int npairs, const void *const *r, const void *const *e, double *loss, float *grad) {
  NetState &n = c.net;
  if (!n.ready) return fail("network: no weights");
  if (!c.have_ud) return fail("network: no gauge field on the device");
  if (npairs < 1) return fail("network: no pairs");
  if (net_fields(c)) return -1;
  cudaStream_t st = c.stream;
  grad_zero(c, st);
  double tot = 0.0;
  for (int k = 0; k < npairs; k++) {
    double l = 0.0;
    if (net_pair_grad(c, r[k], e[k], 1.0 / npairs, &l, st)) return -1;
    tot += l;
  }
  cudaStreamSynchronize(st);
  std::vector<double> g[NLAY];
  grad_read(c, g);
  float *p = grad;
  for (int l = 0; l < NLAY; l++)
    for (size_t k = 0; k < g[l].size(); k++) *p++ = (float)g[l][k];
  *loss = tot;
  return 0;
}

// Adam (Kingma & Ba, 2015) on the real parameters
static void adam_step(NetState &n, const std::vector<double> *g, float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  n.t += 1;
  const float c1 = 1.0f - std::pow(b1, (float)n.t), c2 = 1.0f - std::pow(b2, (float)n.t);
  for (int l = 0; l < NLAY; l++)
    for (size_t k = 0; k < n.w[l].size(); k++) {
      const float gk = (float)g[l][k];
      n.m[l][k] = b1 * n.m[l][k] + (1.0f - b1) * gk;
      n.v[l][k] = b2 * n.v[l][k] + (1.0f - b2) * gk * gk;
      n.w[l][k] -= lr * (n.m[l][k] / c1) / (std::sqrt(n.v[l][k] / c2) + eps);
    }
}

// one Adam step with a given gradient (packed like the weights), then the
// device copies of the weights
int net_adam(Ctx &c, const float *grad, float lr) {
  NetState &n = c.net;
  if (!n.ready) return fail("network: no weights");
  std::vector<double> g[NLAY];
  const float *p = grad;
  for (int l = 0; l < NLAY; l++) {
    g[l].resize(n.w[l].size());
    for (size_t k = 0; k < g[l].size(); k++) g[l][k] = *p++;
  }
  adam_step(n, g, lr);
  return net_upload(c);
}

// steps of Adam on minibatches of `batch` pairs drawn from the npairs
// (r, e); loss_hist[s] = mean loss of step s
int net_train(Ctx &c, int npairs, const void *const *r, const void *const *e, int steps, int batch, float lr,
              uint64_t seed, float *loss_hist) {
  NetState &n = c.net;
  if (!n.ready) return fail("network: no weights (b200_net_init)");
  if (!c.have_ud) return fail("network: no gauge field on the device");
  if (npairs < 1 || batch < 1 || steps < 0) return fail("network: parameters out of range");
  if (net_fields(c)) return -1;
  cudaStream_t st = c.stream;
  std::mt19937_64 rng(seed);
  std::vector<double> g[NLAY];
  for (int s = 0; s < steps; s++) {
    grad_zero(c, st);
    double tot = 0.0;
    for (int b = 0; b < batch; b++) {
      const int k = (int)(rng() % (uint64_t)npairs);
      double l = 0.0;
      if (net_pair_grad(c, r[k], e[k], 1.0 / batch, &l, st)) return -1;
      tot += l;
    }
    cudaStreamSynchronize(st);
    grad_read(c, g);
    adam_step(n, g, lr);
    if (net_upload(c)) return -1;
    if (loss_hist) loss_hist[s] = (float)tot;
  }
  return 0;
}

// activation fields are sized for the geometry; the weights are kept
void net_fields_release(Ctx &c) {
  for (void *p : c.net.f) cudaFree(p);
  c.net.f.clear();
}

void net_release(Ctx &c) {
  NetState &n = c.net;
  for (int l = 0; l < NLAY; l++) {
    cudaFree(n.dev_w[l]);
    cudaFree(n.dev_wadj[l]);
    cudaFree(n.dev_w16[l]);
    cudaFree(n.dev_grad[l]);
  }
  cudaFree(n.part);
  for (void *p : n.f) cudaFree(p);
  n = NetState();
}

}  // namespace qcd
