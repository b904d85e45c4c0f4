// Several right-hand sides solved together (no reference counterpart; each
// system follows the reference's algorithm).
//
// gcr_batch runs the flexible GCR of modules/linsolv/fgcr.c:215 for nr
// systems in lock step: every system keeps its own Krylov space, scalars,
// restarts and stopping test, and leaves the batch as soon as it has
// converged (or failed), so the remaining systems' steps cost only their
// own work.  What the systems share is done once for all of them: with
// deflation (dfl_sap_gcr.c:212-241) the restriction, the little solve and
// the prolongation of every step run as multi-right-hand-side kernels that
// read the Ns basis fields and the little-operator matrices once per group
// of four systems.  Each system may have its own twisted mass (not with
// deflation, whose little operator depends on it).
//
// ltl_gcr_b is the little solver of ltl_gcr.c:155 for nr little systems in
// lock step, with per-system convergence.
#include "lib.h"
#include <array>
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace qcd {

// ------------------------------------------------- batched little GCR kernels
// Little vectors of system r: vector j of the system at base + (r*nvec + j)*nv.
// The CTAs of grid row y work on system act[y].
constexpr int BK = 32, BGRID = 148;

__device__ __forceinline__ const double2 *lvec(const double2 *base, int nvec, size_t nv, int r, int j) {
  return base + ((size_t)r * nvec + j) * nv;
}

__global__ void __launch_bounds__(256) k_bmdot(const double2 *__restrict__ base, int nvec, size_t nv,
                                               const int *__restrict__ act, int jq0, int k, int jy, int n,
                                               double2 *part) {
  __shared__ double2 red[8][BK];
  const int r = act[blockIdx.y];
  const double2 *y = lvec(base, nvec, nv, r, jy);
  double ar[BK], ai[BK];
#pragma unroll
  for (int j = 0; j < BK; j++) ar[j] = ai[j] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 yy = y[i];
#pragma unroll
    for (int j = 0; j < BK; j++)
      if (j < k) {
        const double2 q = lvec(base, nvec, nv, r, jq0 + j)[i];
        ar[j] += q.x * yy.x + q.y * yy.y;
        ai[j] += q.x * yy.y - q.y * yy.x;
      }
  }
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < BK; j++)
    if (j < k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ar[j] += __shfl_down_sync(0xffffffffu, ar[j], o);
        ai[j] += __shfl_down_sync(0xffffffffu, ai[j], o);
      }
      if (lane == 0) red[wp][j] = make_double2(ar[j], ai[j]);
    }
  __syncthreads();
  if ((int)threadIdx.x < k) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < 8; w++) {
      re += red[w][threadIdx.x].x;
      im += red[w][threadIdx.x].y;
    }
    part[((size_t)blockIdx.y * BGRID + blockIdx.x) * BK + threadIdx.x] = make_double2(re, im);
  }
}

// dots[r*64 + off + j] = sum over the CTAs of row y = slot (fixed order)
__global__ void k_bmdot_fin(const double2 *__restrict__ part, int k, const int *__restrict__ act, double2 *dots,
                            int off) {
  const int y = blockIdx.x, r = act[y], j = threadIdx.x;
  if (j >= k) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < BGRID; b++) {
    const double2 a = part[((size_t)y * BGRID + b) * BK + j];
    re += a.x;
    im += a.y;
  }
  dots[r * 64 + off + j] = make_double2(re, im);
}

// q_k -= sum_j dots_j q_j ; p_k -= sum_j dots_j p_j
__global__ void k_bgs_sub(double2 *base, int nvec, size_t nv, const int *__restrict__ act, int k,
                          const double2 *__restrict__ dots, int jq0, int jp0, int n) {
  __shared__ double2 c[BK];
  const int r = act[blockIdx.y];
  if ((int)threadIdx.x < k) c[threadIdx.x] = dots[r * 64 + threadIdx.x];
  __syncthreads();
  double2 *qk = (double2 *)lvec(base, nvec, nv, r, jq0 + k), *pk = (double2 *)lvec(base, nvec, nv, r, jp0 + k);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 q = qk[i], p = pk[i];
    for (int j = 0; j < k; j++) {
      const double2 a = lvec(base, nvec, nv, r, jq0 + j)[i], b = lvec(base, nvec, nv, r, jp0 + j)[i], z = c[j];
      q.x -= z.x * a.x - z.y * a.y; q.y -= z.x * a.y + z.y * a.x;
      p.x -= z.x * b.x - z.y * b.y; p.y -= z.x * b.y + z.y * b.x;
    }
    qk[i] = q;
    pk[i] = p;
  }
}

// q, p /= |q| with |q|^2 = dots[off] (unchanged when zero)
__global__ void k_bnorm(double2 *base, int nvec, size_t nv, const int *__restrict__ act,
                        const double2 *__restrict__ dots, int off, int jq, int jp, int n) {
  const int r = act[blockIdx.y];
  const double s2 = dots[r * 64 + off].x;
  if (!(s2 > 0.0)) return;
  const double f = 1.0 / sqrt(s2);
  double2 *q = (double2 *)lvec(base, nvec, nv, r, jq), *p = (double2 *)lvec(base, nvec, nv, r, jp);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 a = q[i], b = p[i];
    q[i] = make_double2(a.x * f, a.y * f);
    p[i] = make_double2(b.x * f, b.y * f);
  }
}

// x += z p ; rv -= z q with z = dots[off]
__global__ void k_bxr(double2 *base, int nvec, size_t nv, const int *__restrict__ act,
                      const double2 *__restrict__ dots, int off, int jx, int jr, int jp, int jq, int n) {
  const int r = act[blockIdx.y];
  const double2 z = dots[r * 64 + off];
  double2 *x = (double2 *)lvec(base, nvec, nv, r, jx), *rv = (double2 *)lvec(base, nvec, nv, r, jr);
  const double2 *p = lvec(base, nvec, nv, r, jp), *q = lvec(base, nvec, nv, r, jq);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 pp = p[i], qq = q[i];
    double2 xx = x[i], rr = rv[i];
    xx.x += z.x * pp.x - z.y * pp.y; xx.y += z.x * pp.y + z.y * pp.x;
    rr.x -= z.x * qq.x - z.y * qq.y; rr.y -= z.x * qq.y + z.y * qq.x;
    x[i] = xx;
    rv[i] = rr;
  }
}

// dst = src (sgn = 0) or dst = src - dst (sgn = 1), first n entries
__global__ void k_bcopy(double2 *base, int nvec, size_t nv, const int *__restrict__ act, int js, int jd, int n,
                        int sgn) {
  const int r = act[blockIdx.y];
  const double2 *a = lvec(base, nvec, nv, r, js);
  double2 *b = (double2 *)lvec(base, nvec, nv, r, jd);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 v = a[i];
    if (sgn) {
      const double2 w = b[i];
      b[i] = make_double2(v.x - w.x, v.y - w.y);
    } else {
      b[i] = v;
    }
  }
}

// ------------------------------------------------------------ little solver
struct LtlBatch {
  double2 *base = nullptr;
  int nvec = 0, nsys = 0;
  size_t nv = 0;
  double2 *part = nullptr, *dots = nullptr, *h_dots = nullptr;
  int *act = nullptr, *h_act = nullptr;
};
static LtlBatch g_lb;

static int ltl_batch_alloc(Ctx &c, int nr) {
  DflState &d = c.dfl;
  const int nvec = 2 * d.nkv + 6;
  if (g_lb.base && g_lb.nsys >= nr && g_lb.nvec == nvec && g_lb.nv == (size_t)d.nv) return 0;
  cudaFree(g_lb.base);
  cudaFree(g_lb.part);
  cudaFree(g_lb.dots);
  cudaFree(g_lb.act);
  if (g_lb.h_dots) cudaFreeHost(g_lb.h_dots);
  if (g_lb.h_act) cudaFreeHost(g_lb.h_act);
  g_lb = LtlBatch();
  g_lb.nvec = nvec;
  g_lb.nsys = nr;
  g_lb.nv = (size_t)d.nv;
  if (cudaMalloc(&g_lb.base, (size_t)nr * nvec * d.nv * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&g_lb.part, (size_t)nr * BGRID * BK * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&g_lb.dots, (size_t)nr * 64 * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&g_lb.act, nr * sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&g_lb.h_dots, (size_t)nr * 64 * sizeof(double2)) != cudaSuccess ||
      cudaMallocHost(&g_lb.h_act, nr * sizeof(int)) != cudaSuccess)
    return fail("out of device memory (batched little solver)");
  return 0;
}

void ltl_batch_release() {
  cudaFree(g_lb.base);
  cudaFree(g_lb.part);
  cudaFree(g_lb.dots);
  cudaFree(g_lb.act);
  if (g_lb.h_dots) cudaFreeHost(g_lb.h_dots);
  if (g_lb.h_act) cudaFreeHost(g_lb.h_act);
  g_lb = LtlBatch();
}

// ltl_gcr for nr little systems: eta[r] -> psi[r] (device little vectors of
// nv entries; psi[r] may equal eta[r]).  status[r] = GCR steps of system r.
int ltl_gcr_b(Ctx &c, double mu, int nr, const double2 *const *eta, double2 *const *psi, int *ifail, int *status,
              cudaStream_t st) {
  DflState &d = c.dfl;
  for (int r = 0; r < nr; r++) ifail[r] = status[r] = 0;
  if (dfl_set_Awhat(c, mu, st)) {
    for (int r = 0; r < nr; r++) {
      ifail[r] = -2;
      cudaMemsetAsync(psi[r], 0, (size_t)d.nv * sizeof(double2), st);
    }
    return 0;
  }
  if (d.nkv > BK) return fail("ltl_gcr: nkv must not exceed 32");
  if (ltl_batch_alloc(c, nr)) return -1;
  LtlBatch &B = g_lb;
  const int nkv = d.nkv, nvec = B.nvec, nbh = d.nb / 2;
  const size_t nv = B.nv, nvh = nv / 2;
  const int n = (int)nvh;
  enum { JX = 0, JR = 1, JT = 2, JEH = 3, JW = 4, JY = 5 };
  const int JP = 6, JQ = 6 + nkv;
  auto vecs = [&](int j) {
    std::vector<double2 *> v(nr);
    for (int r = 0; r < nr; r++) v[r] = B.base + ((size_t)r * nvec + j) * nv;
    return v;
  };
  const unsigned gv = (unsigned)std::min<size_t>((nvh + 255) / 256, 148);
  std::vector<int> act;
  auto set_act = [&](const std::vector<int> &a) {
    for (size_t i = 0; i < a.size(); i++) B.h_act[i] = a[i];
    cudaMemcpyAsync(B.act, B.h_act, a.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  };
  auto mdot = [&](int na, int jq0, int k, int jy, int off) {
    k_bmdot<<<dim3(BGRID, na), 256, 0, st>>>(B.base, nvec, nv, B.act, jq0, k, jy, n, B.part);
    k_bmdot_fin<<<na, 32, 0, st>>>(B.part, k, B.act, B.dots, off);
  };
  auto read_dots = [&]() {
    cudaMemcpyAsync(B.h_dots, B.dots, (size_t)nr * 64 * sizeof(double2), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
  };
  // sub-lists of pointers for the active systems
  auto pick = [&](const std::vector<double2 *> &v, const std::vector<int> &a) {
    std::vector<double2 *> o(a.size());
    for (size_t i = 0; i < a.size(); i++) o[i] = v[a[i]];
    return o;
  };
  const std::vector<double2 *> X = vecs(JX), R = vecs(JR), Tt = vecs(JT), EH = vecs(JEH), W = vecs(JW),
                               Y = vecs(JY);
  std::vector<const double2 *> ETA(eta, eta + nr);
  std::vector<double2 *> PSI(psi, psi + nr);
  // eh_e = Aee^-1 (eta_e - Aeo Aoo^-1 eta_o)
  for (int r = 0; r < nr; r++) cudaMemcpyAsync(W[r], eta[r], nv * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  little_b(c, nr, 3, nbh, nbh, d.Ainv, nullptr, ETA.data(), nullptr, W.data(), st);
  little_b(c, nr, 2, 0, nbh, nullptr, d.Ahop, ETA.data(), (const double2 *const *)W.data(), Tt.data(), st);
  little_b(c, nr, 3, 0, nbh, d.Ainv, nullptr, Tt.data(), nullptr, EH.data(), st);
  std::vector<int> all(nr);
  for (int r = 0; r < nr; r++) {
    all[r] = r;
    cudaMemsetAsync(X[r], 0, nvh * sizeof(double2), st);
    cudaMemcpyAsync(R[r], EH[r], nvh * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  }
  set_act(all);
  mdot(nr, JR, 1, JR, 34);
  read_dots();
  std::vector<double> rn(nr), tol(nr);
  for (int r = 0; r < nr; r++) {
    rn[r] = sqrt(B.h_dots[r * 64 + 34].x);
    tol[r] = d.res * rn[r];
    if (rn[r] > tol[r]) act.push_back(r);
  }
  int it = 0;
  while (!act.empty() && it < d.nmx) {
    for (int k = 0; k < nkv && !act.empty() && it < d.nmx; k++) {
      const int na = (int)act.size();
      set_act(act);
      // the iteration's launches as one CUDA graph per shape (the active
      // systems, k, the little operator in use); the active list itself
      // is copied to the device before the replay
      std::vector<uint64_t> key = {0x17a9ull, (uint64_t)na, (uint64_t)k, (uint64_t)(uintptr_t)B.base, nv,
                                   (uint64_t)nvec, (uint64_t)(uintptr_t)d.Mhop, (uint64_t)(uintptr_t)d.Mhop32,
                                   (uint64_t)(uintptr_t)B.act, (uint64_t)(uintptr_t)B.dots,
                                   (uint64_t)(uintptr_t)B.part, (uint64_t)(uintptr_t)d.nbr, (uint64_t)d.Ns};
      for (int r : act) key.push_back((uint64_t)r);
      const int rc = graph_run(c, key.data(), key.size() * sizeof(uint64_t), st, [&]() {
        k_bcopy<<<dim3(gv, na), 256, 0, st>>>(B.base, nvec, nv, B.act, JR, JP + k, n, 0);
        {
          const std::vector<double2 *> Pk = pick(vecs(JP + k), act), Qk = pick(vecs(JQ + k), act),
                                       Ya = pick(Y, act);
          dfl_Awhat_b(c, na, (const double2 *const *)Pk.data(), Qk.data(), Ya.data(), st);
        }
        if (k > 0)
          for (int pass = 0; pass < 2; pass++) {
            mdot(na, JQ, k, JQ + k, 0);
            k_bgs_sub<<<dim3(gv, na), 256, 0, st>>>(B.base, nvec, nv, B.act, k, B.dots, JQ, JP, n);
          }
        mdot(na, JQ + k, 1, JQ + k, 32);
        k_bnorm<<<dim3(gv, na), 256, 0, st>>>(B.base, nvec, nv, B.act, B.dots, 32, JQ + k, JP + k, n);
        mdot(na, JQ + k, 1, JR, 33);
        k_bxr<<<dim3(gv, na), 256, 0, st>>>(B.base, nvec, nv, B.act, B.dots, 33, JX, JR, JP + k, JQ + k, n);
        mdot(na, JR, 1, JR, 34);
        return cudaGetLastError() == cudaSuccess ? 0 : fail("ltl_gcr: launch failed");
      });
      if (rc) return -1;
      read_dots();
      it++;
      std::vector<int> keep;
      for (int r : act) {
        status[r] += 1;
        const double nq2 = B.h_dots[r * 64 + 32].x;
        rn[r] = sqrt(B.h_dots[r * 64 + 34].x);
        if (nq2 > 0.0 && rn[r] > tol[r]) keep.push_back(r);
      }
      act.swap(keep);
    }
    if (act.empty()) break;
    // restart the unconverged systems from their true residual
    const int na = (int)act.size();
    set_act(act);
    {
      const std::vector<double2 *> Xa = pick(X, act), Wa = pick(W, act), Ya = pick(Y, act);
      dfl_Awhat_b(c, na, (const double2 *const *)Xa.data(), Wa.data(), Ya.data(), st);
    }
    k_bcopy<<<dim3(gv, na), 256, 0, st>>>(B.base, nvec, nv, B.act, JEH, JW, n, 1);   // w = eh - w
    k_bcopy<<<dim3(gv, na), 256, 0, st>>>(B.base, nvec, nv, B.act, JW, JR, n, 0);    // r = w
    mdot(na, JR, 1, JR, 34);
    read_dots();
    std::vector<int> keep;
    for (int r : act) {
      rn[r] = sqrt(B.h_dots[r * 64 + 34].x);
      if (rn[r] > tol[r]) keep.push_back(r);
    }
    act.swap(keep);
  }
  for (int r = 0; r < nr; r++)
    if (rn[r] > tol[r]) ifail[r] = -1;
  // psi_e = x_e ; psi_o = Aoo^-1 (eta_o - Aoe x_e)
  for (int r = 0; r < nr; r++) cudaMemcpyAsync(psi[r], X[r], nvh * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  little_b(c, nr, 2, nbh, nbh, nullptr, d.Ahop, ETA.data(), (const double2 *const *)X.data(), Tt.data(), st);
  little_b(c, nr, 3, nbh, nbh, d.Ainv, nullptr, (const double2 *const *)Tt.data(), nullptr, PSI.data(), st);
  return 0;
}

// ------------------------------------------ fused orthogonalisation (FP32)
// One gcr_step of fgcr.c:157 for a system in three passes instead of about
// 5k+9: (1) all k products (chi_l, chi_k) in one pass over chi_k; (2)
// chi_k -= sum_l a_lk chi_l together with |chi_k|^2 and (chi_k, rho); (3)
// chi_k /= |chi_k|, rho -= c chi_k together with |rho|^2.  Products are
// accumulated in FP32 over runs of 16 float4, in double beyond, and summed
// over a fixed grid.  This is
// classical Gram-Schmidt where the reference applies the products one by
// one (modified Gram-Schmidt); in exact arithmetic the two agree.
constexpr int OG = 1184, OK_ = 32;
struct F2Ptrs {
  const float4 *p[OK_];
};

// products summed in FP32 over runs of 16 grid-stride steps, the runs in
// double (FP64 adds per element halved the speed of these kernels)
template <int KM>
__global__ void __launch_bounds__(256) k_fmdot(F2Ptrs q, int k, const float4 *__restrict__ y, size_t n,
                                               double2 *part) {
  __shared__ double2 red[8][KM];
  double ar[KM], ai[KM];
#pragma unroll
  for (int j = 0; j < KM; j++) ar[j] = ai[j] = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  while (i < n) {
    float fr[KM], fi[KM];
#pragma unroll
    for (int j = 0; j < KM; j++) fr[j] = fi[j] = 0.0f;
    for (int t = 0; t < 16 && i < n; t++, i += stride) {
      const float4 yy = __ldg(y + i);
#pragma unroll
      for (int j = 0; j < KM; j++)
        if (j < k) {
          const float4 a = __ldg(q.p[j] + i);
          fr[j] += a.x * yy.x + a.y * yy.y + a.z * yy.z + a.w * yy.w;
          fi[j] += a.x * yy.y - a.y * yy.x + a.z * yy.w - a.w * yy.z;
        }
    }
#pragma unroll
    for (int j = 0; j < KM; j++) {
      ar[j] += fr[j];
      ai[j] += fi[j];
    }
  }
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < KM; j++)
    if (j < k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ar[j] += __shfl_down_sync(0xffffffffu, ar[j], o);
        ai[j] += __shfl_down_sync(0xffffffffu, ai[j], o);
      }
      if (lane == 0) red[wp][j] = make_double2(ar[j], ai[j]);
    }
  __syncthreads();
  if ((int)threadIdx.x < k) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < 8; w++) {
      re += red[w][threadIdx.x].x;
      im += red[w][threadIdx.x].y;
    }
    part[blockIdx.x * OK_ + threadIdx.x] = make_double2(re, im);
  }
}

// out[j] = sum over the OG partials of product j: CTA j, fixed tree
__global__ void __launch_bounds__(256) k_fsum(const double2 *__restrict__ part, double2 *out) {
  __shared__ double2 red[256];
  const int j = blockIdx.x;
  double re = 0.0, im = 0.0;
  for (int b = threadIdx.x; b < OG; b += blockDim.x) {
    re += part[b * OK_ + j].x;
    im += part[b * OK_ + j].y;
  }
  red[threadIdx.x] = make_double2(re, im);
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      red[threadIdx.x].x += red[threadIdx.x + h].x;
      red[threadIdx.x].y += red[threadIdx.x + h].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0];
}

// block sums of two products into part[b*OK_ + 0, 1]
__device__ __forceinline__ void block_sum2(double a0, double a1, double a2, double2 *part) {
  __shared__ double red[3][8];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    a1 += __shfl_down_sync(0xffffffffu, a1, o);
    a2 += __shfl_down_sync(0xffffffffu, a2, o);
  }
  if (lane == 0) {
    red[0][wp] = a0;
    red[1][wp] = a1;
    red[2][wp] = a2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int w = 0; w < 8; w++) {
      s0 += red[0][w];
      s1 += red[1][w];
      s2 += red[2][w];
    }
    part[blockIdx.x * OK_] = make_double2(s0, 0.0);
    part[blockIdx.x * OK_ + 1] = make_double2(s1, s2);
  }
}

// The same three passes with the coefficients kept on the device: the
// products of pass (1) and the two sums of pass (2) are written to the
// system's record dsum (OK_ + 3 entries: a_lk, |chi_k|^2, (chi_k, rho),
// |rho|^2), pass (2) reads its coefficients there and pass (3) derives its
// scale and coefficient there exactly as the host does (float(sqrt(double
// (float |chi_k|^2))), 1.0f / b), so the host reads one record per system
// per step instead of waiting three times per system.
constexpr int DS = OK_ + 3;

template <int KM>
__global__ void __launch_bounds__(256) k_fgs_d(F2Ptrs q, int k, const double2 *__restrict__ coef, float4 *chik,
                                               const float4 *__restrict__ rho, size_t n, double2 *part) {
  float2 cz[KM];
#pragma unroll
  for (int j = 0; j < KM; j++)
    cz[j] = j < k ? make_float2((float)coef[j].x, (float)coef[j].y) : make_float2(0.0f, 0.0f);
  double nn = 0.0, dr = 0.0, di = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  while (i < n) {
    float fn = 0.0f, fr = 0.0f, fi = 0.0f;
    for (int t = 0; t < 16 && i < n; t++, i += stride) {
      float4 x = chik[i];
#pragma unroll
      for (int j = 0; j < KM; j++)
        if (j < k) {
          const float4 a = __ldg(q.p[j] + i);
          const float2 z = cz[j];
          x.x -= z.x * a.x - z.y * a.y;
          x.y -= z.x * a.y + z.y * a.x;
          x.z -= z.x * a.z - z.y * a.w;
          x.w -= z.x * a.w + z.y * a.z;
        }
      chik[i] = x;
      const float4 r = __ldg(rho + i);
      fn += x.x * x.x + x.y * x.y + x.z * x.z + x.w * x.w;
      fr += x.x * r.x + x.y * r.y + x.z * r.z + x.w * r.w;
      fi += x.x * r.y - x.y * r.x + x.z * r.w - x.w * r.z;
    }
    nn += fn;
    dr += fr;
    di += fi;
  }
  block_sum2(nn, dr, di, part);
}

__global__ void __launch_bounds__(256) k_fupd_d(float4 *chik, float4 *rho, const double2 *__restrict__ sums, size_t n,
                                                double2 *part) {
  const float bn = (float)sqrt((double)(float)sums[0].x);
  const float s = bn != 0.0f ? 1.0f / bn : 0.0f;
  const float2 c = make_float2((float)sums[1].x * s, (float)sums[1].y * s);
  double nn = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  while (i < n) {
    float fn = 0.0f;
    for (int t = 0; t < 16 && i < n; t++, i += stride) {
      float4 x = chik[i], r = rho[i];
      x.x *= s;
      x.y *= s;
      x.z *= s;
      x.w *= s;
      r.x -= c.x * x.x - c.y * x.y;
      r.y -= c.x * x.y + c.y * x.x;
      r.z -= c.x * x.z - c.y * x.w;
      r.w -= c.x * x.w + c.y * x.z;
      chik[i] = x;
      rho[i] = r;
      fn += r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w;
    }
    nn += fn;
  }
  block_sum2(nn, 0.0, 0.0, part);
}

struct OrthoBufs {
  double2 *part = nullptr;
  double2 *dsum = nullptr, *h_dsum = nullptr;   // DS entries per system
  int nsys = 0;
};
static OrthoBufs g_ob;

static int ortho_alloc() {
  if (g_ob.part) return 0;
  if (cudaMalloc(&g_ob.part, (size_t)OG * OK_ * sizeof(double2)) != cudaSuccess)
    return fail("out of memory (orthogonalisation buffers)");
  return 0;
}

static int dsum_alloc(int nr) {
  if (g_ob.nsys >= nr) return 0;
  cudaFree(g_ob.dsum);
  cudaFreeHost(g_ob.h_dsum);
  g_ob.dsum = g_ob.h_dsum = nullptr;
  g_ob.nsys = 0;
  if (cudaMalloc(&g_ob.dsum, (size_t)nr * DS * sizeof(double2)) != cudaSuccess ||
      cudaMallocHost(&g_ob.h_dsum, (size_t)nr * DS * sizeof(double2)) != cudaSuccess)
    return fail("out of memory (orthogonalisation buffers)");
  g_ob.nsys = nr;
  return 0;
}

// the passes of gcr_step_fused for one system, its record at dsum
static void gcr_step_dev(const Ctx &c, int k, const std::vector<void *> &chi, void *rho, double2 *dsum,
                         cudaStream_t st) {
  const size_t n = (size_t)c.g.vol * 6;
  F2Ptrs q;
  for (int j = 0; j < OK_; j++) q.p[j] = j < k ? (const float4 *)chi[j] : nullptr;
  if (k > 0) {
    if (k <= 8) k_fmdot<8><<<OG, 256, 0, st>>>(q, k, (const float4 *)chi[k], n, g_ob.part);
    else if (k <= 16) k_fmdot<16><<<OG, 256, 0, st>>>(q, k, (const float4 *)chi[k], n, g_ob.part);
    else k_fmdot<32><<<OG, 256, 0, st>>>(q, k, (const float4 *)chi[k], n, g_ob.part);
    k_fsum<<<k, 256, 0, st>>>(g_ob.part, dsum);
  }
  if (k <= 8) k_fgs_d<8><<<OG, 256, 0, st>>>(q, k, dsum, (float4 *)chi[k], (const float4 *)rho, n, g_ob.part);
  else if (k <= 16) k_fgs_d<16><<<OG, 256, 0, st>>>(q, k, dsum, (float4 *)chi[k], (const float4 *)rho, n, g_ob.part);
  else k_fgs_d<32><<<OG, 256, 0, st>>>(q, k, dsum, (float4 *)chi[k], (const float4 *)rho, n, g_ob.part);
  k_fsum<<<2, 256, 0, st>>>(g_ob.part, dsum + OK_);
  k_fupd_d<<<OG, 256, 0, st>>>((float4 *)chi[k], (float4 *)rho, dsum + OK_, n, g_ob.part);
  k_fsum<<<1, 256, 0, st>>>(g_ob.part, dsum + OK_ + 2);
}

// a_lk, b_k, c_k and rn of a system from its record, as gcr_step_fused sets them
static double gcr_step_coefs(int nkv, int k, const double2 *h, std::vector<cplxf> &a, std::vector<float> &b,
                             std::vector<cplxf> &cc) {
  for (int l = 0; l < k; l++) a[(size_t)nkv * l + k] = {(float)h[l].x, (float)h[l].y};
  const float bn = (float)sqrt((double)(float)h[OK_].x);
  b[k] = bn;
  const float s = bn != 0.0f ? 1.0f / bn : 0.0f;
  cc[k] = {(float)h[OK_ + 1].x * s, (float)h[OK_ + 1].y * s};
  return sqrt((double)(float)h[OK_ + 2].x);
}


// ------------------------------------------------------------- outer solver
struct SysState {
  double mu = 0.0, rho0 = 0.0, rn = 0.0, tol = 0.0, rn_old = 0.0;
  int k = 0, status = 0, ifail = 0, lstat = 0;
  bool active = false;
  std::vector<cplxf> a, cc;
  std::vector<float> b;
  void *rsd = nullptr, *rho = nullptr, *ws0 = nullptr;
  std::vector<void *> phi, chi;
};

struct BatchWs {
  std::vector<void *> f32, f64;
};
static BatchWs g_bw;

void gcr_batch_release() {
  for (void *p : g_bw.f32) cudaFree(p);
  for (void *p : g_bw.f64) cudaFree(p);
  g_bw = BatchWs();
  ltl_batch_release();
}

static int bw_reserve(Ctx &c, std::vector<void *> &v, size_t n, int prec) {
  while (v.size() < n) {
    void *p = nullptr;
    if (cudaMalloc(&p, spinor_bytes(c, prec)) != cudaSuccess) return fail("out of device memory (batch workspace)");
    v.push_back(p);
  }
  return 0;
}

// The little operators of the masses of a deflated batch: the first lives
// in the deflation state's own arrays, the others in arrays of the same
// sizes; use(j) points the state at set j.  The state's own arrays hold
// set 0 again when the batch ends (the destructor), marked stale.
struct LittleSets {
  Ctx *c = nullptr;
  void *own[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<std::array<void *, 5>> set;
  std::vector<double> mu;
  std::vector<int> fail;
  // The first mass in the library's own arrays (recomputed only if they
  // hold another mass); every further mass gets its own diagonal blocks,
  // inverses and preconditioned hops, and shares the hop matrices Ahop,
  // which do not depend on the mass.
  int build(Ctx &cc, const std::vector<double> &umu, cudaStream_t st) {
    c = &cc;
    DflState &d = cc.dfl;
    own[0] = d.Ablk; own[1] = d.Ainv; own[2] = d.Ahop; own[3] = d.Mhop; own[4] = d.Mhop32;
    const size_t m = (size_t)d.nb * d.Ns * d.Ns * sizeof(double2);
    const size_t sz[5] = {m, m, 8 * m, 8 * m, 4 * m};
    mu = umu;
    set.assign(umu.size(), {nullptr, nullptr, nullptr, nullptr, nullptr});
    fail.assign(umu.size(), 0);
    for (size_t j = 0; j < umu.size(); j++) {
      if (j > 0 && d.xsets.size() < j) {
        std::array<void *, 4> x = {nullptr, nullptr, nullptr, nullptr};
        const int ks[4] = {0, 1, 3, 4};
        for (int q = 0; q < 4; q++)
          if (cudaMalloc(&x[q], sz[ks[q]]) != cudaSuccess) {
            for (void *p : x) cudaFree(p);
            return qcd::fail("gcr_batch: out of device memory (little operators)");
          }
        d.xsets.push_back(x);
      }
      for (int k = 0; k < 5; k++) {
        if (j == 0 || k == 2) set[j][k] = own[k];
        else set[j][k] = d.xsets[j - 1][k < 2 ? k : k - 1];
      }
      point(j);
      // set 0: the operator of umu[0] if the arrays do not hold it yet
      // (with the hop matrices); sets j > 0: their diagonal part
      const int f = j == 0 ? dfl_set_Awhat(cc, umu[0], st) : dfl_set_Awhat(cc, umu[j], st, true);
      if (f < 0) return -1;
      fail[j] = f;
    }
    if (umu.size() > 1) point(0);
    return 0;
  }
  void point(size_t j) {
    DflState &d = c->dfl;
    d.Ablk = (double2 *)set[j][0]; d.Ainv = (double2 *)set[j][1]; d.Ahop = (double2 *)set[j][2];
    d.Mhop = (double2 *)set[j][3]; d.Mhop32 = (float2 *)set[j][4];
  }
  void use(Ctx &cc, size_t j) {
    if (set.size() <= 1) return;
    DflState &d = cc.dfl;
    point(j);
    d.aw_valid = d.awhat_valid = true;
    d.aw_mu = mu[j];
    d.aw_eo = cc.eoflg;
    d.awhat_fail = fail[j];
    d.awhat_ver++;
  }
  ~LittleSets() {
    if (!c || set.size() <= 1) return;
    DflState &d = c->dfl;
    cudaStreamSynchronize(c->stream);
    d.Ablk = (double2 *)own[0]; d.Ainv = (double2 *)own[1]; d.Ahop = (double2 *)own[2];
    d.Mhop = (double2 *)own[3]; d.Mhop32 = (float2 *)own[4];
    // the own arrays hold the operator of the first mass
    d.aw_valid = d.awhat_valid = true;
    d.aw_mu = mu[0];
    d.aw_eo = c->eoflg;
    d.awhat_fail = fail[0];
    d.awhat_ver++;
  }
};

// nr systems Dw(mu[r]) psi[r] = eta[r] (FP64 device fields), flexible GCR
// with SAP (dfl = 0) or deflated SAP (dfl = 1) preconditioning as in
// sap_gcr / dfl_sap_gcr.  rho[r] = residual norm, ifail[r], status[r] as
// there (status[r] = GCR steps; with deflation status[nr + r] = average
// little-solver steps).
int gcr_batch(Ctx &c, int nr, int dfl, int nkv, int nmx, int istop, double res, const double *mu,
              const void *const *eta, void *const *psi, double *rho, int *ifail, int *status) {
  cudaStream_t st = c.stream;
  DflState &d = c.dfl;
  if (nr < 1) return fail("gcr_batch: no systems");
  if (nkv < 1 || nmx < 1 || res <= DBL_EPSILON || istop < 0 || istop > 1) return fail("gcr_batch: parameters are out of range");
  if (!c.sap_set) return fail("gcr_batch: SAP parameters are not set");
  if (!c.have_ud || !c.have_sw) return fail("gcr_batch: gauge or SW field missing on the device");
  // the distinct twisted masses of the batch and each system's group; the
  // little operator depends on the mass, so each group has its own
  // (restriction, prolongation and SAP are shared by all systems)
  std::vector<double> umu;
  std::vector<int> grp(nr);
  for (int r = 0; r < nr; r++) {
    int j = 0;
    while (j < (int)umu.size() && umu[j] != mu[r]) j++;
    if (j == (int)umu.size()) umu.push_back(mu[r]);
    grp[r] = j;
  }
  LittleSets lsets;
  if (dfl) {
    if (!d.ready || !d.have_basis) return fail("gcr_batch: the deflation subspace is not set");
    if (dfl_batch_alloc(c)) return -1;
  }
  if (sap_prepare(c, st) || ortho_alloc() || dsum_alloc(nr)) return -1;
  const int per32 = 2 * nkv + 1 + (dfl ? 1 : 0);
  if (bw_reserve(c, g_bw.f32, (size_t)nr * per32 + 1, 32) || bw_reserve(c, g_bw.f64, (size_t)nr + 1, 64)) return -1;
  if (!c.tmp32 && cudaMalloc(&c.tmp32, spinor_bytes(c, 32)) != cudaSuccess) return fail("out of device memory");
  if (!c.tmp64 && cudaMalloc(&c.tmp64, spinor_bytes(c, 64)) != cudaSuccess) return fail("out of device memory");
  void *phib = g_bw.f32[(size_t)nr * per32], *wrk = g_bw.f64[nr];
  const KrylovOps o = dev_krylov_ops(c);
  const double PRECISION_LIMIT = (double)(100.0f * FLT_EPSILON);
  std::vector<SysState> S(nr);
  std::vector<double2 *> vd(nr);
  if (dfl) {
    if (ensure_lvd_n(c, nr)) return -1;
    for (int r = 0; r < nr; r++) vd[r] = d.lvd[r];
  }
  for (int r = 0; r < nr; r++) {
    SysState &y = S[r];
    y.mu = mu[r];
    y.a.resize((size_t)nkv * nkv);
    y.cc.resize(nkv);
    y.b.resize(nkv);
    y.rho = g_bw.f32[(size_t)r * per32];
    y.phi.assign(g_bw.f32.begin() + (size_t)r * per32 + 1, g_bw.f32.begin() + (size_t)r * per32 + 1 + nkv);
    y.chi.assign(g_bw.f32.begin() + (size_t)r * per32 + 1 + nkv, g_bw.f32.begin() + (size_t)r * per32 + 1 + 2 * nkv);
    y.ws0 = dfl ? g_bw.f32[(size_t)r * per32 + 2 * nkv + 1] : nullptr;
    y.rsd = g_bw.f64[r];
    ifail[r] = 0;
    status[r] = 0;
    if (dfl) status[nr + r] = 0;
    // source scale as in sap_gcr.c:200-215 (uniform norm) / dfl_sap_gcr.c (istop norm)
    double u[2];
    if (dfl && !istop) {
      la_norm2(c, 64, eta[r], PAR_ALL, u);
      y.rho0 = sqrt(u[0]);
    } else {
      la_unorm(c, 64, eta[r], PAR_ALL, u);
      y.rho0 = u[0];
    }
    if (y.rho0 == 0.0) {
      la_zero(c, 64, psi[r], PAR_ALL, st);
      rho[r] = 0.0;
      continue;
    }
    la_copy(c, 64, eta[r], 64, y.rsd, PAR_ALL, st);
    la_scale(c, 64, y.rsd, 1.0 / y.rho0, PAR_ALL, st);
    o.zero64(psi[r]);
    o.copy64to32(y.rsd, y.rho);
    y.rn = o.res32(y.rho, istop);
    y.tol = res * y.rn;
    y.rn_old = y.rn;
    y.k = 0;
    y.active = y.rn > y.tol;
  }
  if (c.isolv == 1 && (c.sw_inv_fail & 2)) {
    for (int r = 0; r < nr; r++) {
      ifail[r] = -3;
      S[r].active = false;
    }
  }
  if (dfl) {
    // one little operator per mass (set_Awhat, dfl_modes.c / Aw_ops.c:223)
    if (lsets.build(c, umu, st)) return -1;
    for (int r = 0; r < nr; r++)
      if (lsets.fail[grp[r]]) {
        ifail[r] = -2;
        S[r].active = false;
      }
  }
  for (;;) {
    std::vector<int> A;
    for (int r = 0; r < nr; r++)
      if (S[r].active) A.push_back(r);
    if (A.empty()) break;
    const int na = (int)A.size();
    // --- Mop for all active systems: phi_k = M rho, chi_k = D phi_k
    // (phase timers, when on: 3 deflation, 4 SAP, 2 rest of Mop,
    // 1 orthogonalisation, 0 restarts)
    dfl_mark(c, -1);
    if (dfl) {
      std::vector<const void *> rh(na);
      std::vector<double2 *> v(na);
      std::vector<void *> w0(na);
      std::vector<int> lf(na), ls(na);
      for (int i = 0; i < na; i++) {
        rh[i] = S[A[i]].rho;
        v[i] = vd[i];
        w0[i] = S[A[i]].ws0;
      }
      dfl_restrict_b(c, na, rh.data(), v.data(), st);
      // the little systems, one batch per mass
      for (int j = 0; j < (int)umu.size(); j++) {
        std::vector<double2 *> vj;
        std::vector<int> ij;
        for (int i = 0; i < na; i++)
          if (grp[A[i]] == j) {
            vj.push_back(v[i]);
            ij.push_back(i);
          }
        if (vj.empty()) continue;
        lsets.use(c, j);
        std::vector<int> lfj(vj.size()), lsj(vj.size());
        if (ltl_gcr_b(c, umu[j], (int)vj.size(), (const double2 *const *)vj.data(), vj.data(), lfj.data(),
                      lsj.data(), st))
          return -1;
        for (size_t q = 0; q < ij.size(); q++) {
          lf[ij[q]] = lfj[q];
          ls[ij[q]] = lsj[q];
        }
      }
      dfl_prolong_b(c, na, (const double2 *const *)v.data(), w0.data(), st);
      dfl_mark(c, 3);
      // SAP_MS systems per SAP launch
      for (int i0 = 0; i0 < na; i0 += SAP_MS) {
        const int m = na - i0 < SAP_MS ? na - i0 : SAP_MS;
        const void *rh[SAP_MS], *base[SAP_MS], *add[SAP_MS];
        void *ph[SAP_MS], *ch[SAP_MS], *in[SAP_MS], *rv[SAP_MS];
        float mus[SAP_MS];
        for (int q = 0; q < m; q++) {
          SysState &y = S[A[i0 + q]];
          ph[q] = y.phi[y.k];
          ch[q] = y.chi[y.k];
          // rho - D ws0, written where the SAP sequence reads its input
          in[q] = sap_input_field_multi(c, q, m);
          if (!in[q]) in[q] = ch[q];
          rv[q] = y.rho;
          rh[q] = in[q];
          base[q] = y.rho;
          add[q] = y.ws0;
          mus[q] = (float)y.mu;
          y.lstat += ls[i0 + q];
        }
        if (dirac_sys32(c, m, mus, &w0[i0], in, rv, st)) return fail("gcr_batch: Dirac launch failed");
        dfl_mark(c, 3);
        // SAP on them, then ch = rho - (final residual), ph += ws0
        if (sap_mop_multi(c, m, mus, c.isolv, c.nmr, c.ncy, rh, ph, ch, phib, st, base, add)) return -1;
        dfl_mark(c, 4);
      }
    } else {
      for (int i0 = 0; i0 < na; i0 += SAP_MS) {
        const int m = na - i0 < SAP_MS ? na - i0 : SAP_MS;
        const void *rh[SAP_MS];
        void *ph[SAP_MS], *ch[SAP_MS];
        float mus[SAP_MS];
        for (int q = 0; q < m; q++) {
          SysState &y = S[A[i0 + q]];
          rh[q] = y.rho;
          ph[q] = y.phi[y.k];
          ch[q] = y.chi[y.k];
          mus[q] = (float)y.mu;
        }
        dfl_mark(c, 2);
        if (sap_mop_multi(c, m, mus, c.isolv, c.nmr, c.ncy, rh, ph, ch, phib, st, nullptr, nullptr)) return -1;
        dfl_mark(c, 4);
      }
    }
    // --- the rest of gcr_step, and restarts, per system (fgcr.c:157-299):
    // with the fused passes, every system's passes first, then one read of
    // all their records
    const bool fused = istop == 0 && nkv <= OK_;
    if (fused) {
      // captured as one CUDA graph per step shape (the systems' k and
      // fields), replayed by later steps and solves of the same shape
      std::vector<uint64_t> key = {0x0e7a0ull, (uint64_t)na, (uint64_t)(size_t)c.g.vol};
      for (int i = 0; i < na; i++) {
        const SysState &y = S[A[i]];
        key.push_back((uint64_t)y.k);
        key.push_back((uint64_t)(uintptr_t)y.rho);
        for (int l = 0; l <= y.k; l++) key.push_back((uint64_t)(uintptr_t)y.chi[l]);
      }
      const int rc = graph_run(c, key.data(), key.size() * sizeof(uint64_t), st, [&]() {
        for (int i = 0; i < na; i++)
          gcr_step_dev(c, S[A[i]].k, S[A[i]].chi, S[A[i]].rho, g_ob.dsum + (size_t)i * DS, st);
        return cudaGetLastError() == cudaSuccess ? 0 : fail("gcr_batch: launch failed");
      });
      if (rc) return -1;
      cudaMemcpyAsync(g_ob.h_dsum, g_ob.dsum, (size_t)na * DS * sizeof(double2), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) return fail("gcr_batch: CUDA error");
    }
    for (int ia = 0; ia < na; ia++) {
      const int r = A[ia];
      SysState &y = S[r];
      const int k = y.k;
      if (fused) {
        y.rn = gcr_step_coefs(nkv, k, g_ob.h_dsum + (size_t)ia * DS, y.a, y.b, y.cc);
      } else {
        for (int l = 0; l < k; l++) {
          cplxf z = o.dot32(y.chi[l], y.chi[k]);
          y.a[(size_t)nkv * l + k] = z;
          o.axpy32(y.chi[k], -z.re, -z.im, y.chi[l]);
        }
        y.b[k] = o.normalize32(y.chi[k]);
        y.cc[k] = o.dot32(y.chi[k], y.rho);
        o.axpy32(y.rho, -y.cc[k].re, -y.cc[k].im, y.chi[k]);
        y.rn = o.res32(y.rho, istop);
      }
      y.status += 1;
      dfl_mark(c, 1);
      if (y.rn <= y.tol || y.rn < PRECISION_LIMIT * y.rn_old || k == nkv - 1 || y.status >= nmx) {
        // update_psi (fgcr.c:181)
        for (int l = k; l >= 0; l--) {
          cplxf z = y.cc[l];
          for (int i = l + 1; i <= k; i++) {
            cplxf al = y.a[(size_t)l * nkv + i];
            z.re -= al.re * y.cc[i].re - al.im * y.cc[i].im;
            z.im -= al.re * y.cc[i].im + al.im * y.cc[i].re;
          }
          float rb = 1.0f / y.b[l];
          y.cc[l].re = z.re * rb;
          y.cc[l].im = z.im * rb;
        }
        {
          std::vector<cplxf> cl;
          std::vector<void *> xl;
          for (int l = k; l >= 0; l--) {
            cl.push_back(y.cc[l]);
            xl.push_back(y.phi[l]);
          }
          o.lincomb32(y.rho, k + 1, cl.data(), xl.data());
        }
        o.add32to64(y.rho, psi[r]);
        dirac_op<double>(c, 0, y.mu, psi[r], wrk, c.tmp64, st);
        o.diff64to32(y.rsd, wrk, y.rho);
        y.rn = o.res32(y.rho, istop);
        y.k = 0;
        y.rn_old = y.rn;
        dfl_mark(c, 0);
        if (y.rn <= y.tol) {
          y.active = false;
        } else if (y.status >= nmx) {
          y.active = false;
          ifail[r] = -1;
        }
      } else {
        y.k = k + 1;
      }
    }
  }
  for (int r = 0; r < nr; r++) {
    SysState &y = S[r];
    if (y.rho0 == 0.0) continue;
    if (ifail[r] <= -2) {
      la_zero(c, 64, psi[r], PAR_ALL, st);
      rho[r] = y.rho0;
      continue;
    }
    la_scale(c, 64, psi[r], y.rho0, PAR_ALL, st);
    rho[r] = y.rn * y.rho0;
    status[r] = ifail[r] == -1 ? nmx : y.status;
    if (dfl && y.status > 0) status[nr + r] = (y.lstat + y.status / 2) / y.status;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("gcr_batch: CUDA error");
  return dfl ? dfl_batch_check(c) : 0;
}

}  // namespace qcd
