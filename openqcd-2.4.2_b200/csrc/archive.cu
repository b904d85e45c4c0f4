// Gauge-field and spinor-field files in openQCD's "universal" format
// (modules/archive/archive.c:804-977 export_cnfg/import_cnfg,
// modules/archive/sarchive.c:424-620 export_sfld/import_sfld, layout in
// main/README.io): the device<->disk bridge for real configurations and
// propagators.
//
// Configuration file: int32 N0..N3, double average plaquette
// (sum of Re tr U(p) over the 6 V plaquettes, divided by 6 V), then for every
// odd point x in lexicographic order (x3 fastest) the 8 links
// U(x,0), U(x-0,0), U(x,1), U(x-1,1), ..., U(x-3,3) as 3x3 complex doubles
// (row major), without the antiperiodic boundary phase.  Spinor file: int32
// N0..N3, eo, double |sd|^2 over the sites written, then the spinors of all
// sites (eo = 0) or of the even sites (eo = 1) in lexicographic order.
// Little-endian only (the byte swap of the reference for big-endian hosts is
// not needed on the hosts this library runs on).
#include "lib.h"
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace qcd {

// device site (chunk, s) of the global coordinates x
static void dev_site(const Ctx &c, const int x[4], int &chunk, int &s) {
  int n[4], y[4];
  for (int mu = 0; mu < 4; mu++) {
    n[mu] = x[mu] / c.g.bs[mu];
    y[mu] = x[mu] % c.g.bs[mu];
  }
  const int blk = ((n[0] * c.g.nb[1] + n[1]) * c.g.nb[2] + n[2]) * c.g.nb[3] + n[3];
  const int l = ((y[0] * c.g.bs[1] + y[1]) * c.g.bs[2] + y[2]) * c.g.bs[3] + y[3];
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  chunk = p * c.g.nbl + blk;
  s = l >> 1;
}

// ------------------------------------------------------------- plaquette
// Re tr U(p) summed over the 6 planes of every site, per-CTA partial sums
__global__ void k_plaq(Geom g, const double2 *__restrict__ u, double *part) {
  __shared__ double red[8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (i < g.vol) {
    const int chunk = i / g.vbh, s = i - chunk * g.vbh;
    const int p = chunk >= g.nbl, blk = chunk - p * g.nbl;
    Site x;
    site_decode(g, p, blk, s, x);
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        int cm, sm, cn, sn;
        site_nbr(g, x, mu, 1, cm, sm);
        site_nbr(g, x, nu, 1, cn, sn);
        const su3<double> a = Store<double>::load_link(u, chunk, mu, s, g.vbh);
        const su3<double> b = Store<double>::load_link(u, cm, nu, sm, g.vbh);
        const su3<double> cc = Store<double>::load_link(u, cn, mu, sn, g.vbh);
        const su3<double> d = Store<double>::load_link(u, chunk, nu, s, g.vbh);
        // tr[a b cc^dag d^dag] = sum_{ijkl} a_ij b_jk conj(cc_lk) conj(d_il)
        double tr = 0.0;
        for (int ii = 0; ii < 3; ii++)
          for (int l = 0; l < 3; l++) {
            // (a b)_{ik} . conj(cc_{lk}) summed over k, times conj(d_{il})
            double er = 0.0, ei = 0.0;
            for (int k = 0; k < 3; k++) {
              double abr = 0.0, abi = 0.0;
              for (int j = 0; j < 3; j++) {
                const cpx<double> x1 = a.e[3 * ii + j], y1 = b.e[3 * j + k];
                abr += x1.re * y1.re - x1.im * y1.im;
                abi += x1.re * y1.im + x1.im * y1.re;
              }
              const cpx<double> z = cc.e[3 * l + k];
              er += abr * z.re + abi * z.im;
              ei += abi * z.re - abr * z.im;
            }
            const cpx<double> w = d.e[3 * ii + l];
            tr += er * w.re + ei * w.im;
          }
        acc += tr;
      }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    part[blockIdx.x] = t;
  }
}

// Kahan sum of a host array in a fixed order
static double ksum(const std::vector<double> &v) {
  double s = 0.0, c = 0.0;
  for (double x : v) {
    const double y = x - c, t = s + y;
    c = (t - s) - y;
    s = t;
  }
  return s;
}

int plaq_sum(Ctx &c, double *sum) {
  if (dd_unsupported(c, "plaq_sum")) return -1;
  if (!c.have_ud) return fail("plaq_sum: no gauge field on the device");
  const int t = 256, nb = (c.g.vol + t - 1) / t;
  double *part = nullptr;
  if (cudaMalloc(&part, nb * sizeof(double)) != cudaSuccess) return fail("out of device memory");
  k_plaq<<<nb, t, 0, c.stream>>>(c.g, c.ud, part);
  std::vector<double> h(nb);
  cudaMemcpyAsync(h.data(), part, nb * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  cudaStreamSynchronize(c.stream);
  cudaFree(part);
  if (cudaGetLastError() != cudaSuccess) return fail("plaq_sum: CUDA error");
  *sum = ksum(h);
  return 0;
}

// ---------------------------------------------------------- configurations
// the antiperiodic phase of bc type 3 sits on U(x,0) with x0 = N0-1; with
// phase angles theta the spatial links carry exp(i theta[k-1]/N[k]) as well
// (set_ud_phase, modules/uflds/uflds.c:249-355), put on after reading a
// configuration and taken off before writing one
static bool phase_link(const Ctx &c, const int x[4], int mu) { return c.bc == 3 && mu == 0 && x[0] == c.g.L[0] - 1; }

int export_cnfg(Ctx &c, const char *out) {
  if (dd_unsupported(c, "export_cnfg")) return -1;
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (!c.have_ud) return fail("export_cnfg: no gauge field on the device");
  const int *L = c.g.L;
  const size_t nd = (size_t)c.g.vol * 36;
  std::vector<double2> hu(nd);
  if (cudaMemcpy(hu.data(), c.ud, nd * sizeof(double2), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail("export_cnfg: CUDA error");
  double ps = 0.0;
  if (plaq_sum(c, &ps)) return -1;
  double plaq = ps / (6.0 * (double)c.g.vol);
  FILE *f = fopen(out, "wb");
  if (!f) return fail("export_cnfg: unable to open output file");
  int32_t ls[4] = {L[0], L[1], L[2], L[3]};
  bool ok = fwrite(ls, sizeof(int32_t), 4, f) == 4 && fwrite(&plaq, sizeof(double), 1, f) == 1;
  std::vector<double> line((size_t)4 * L[3] * 18);
  double pr[3], pi[3];
  const bool phased = spatial_phases(c, pr, pi);
  for (int k = 0; k < 3; k++) pi[k] = -pi[k];   // the phase is taken off (set_phase(-1))
  int x[4];
  for (x[0] = 0; x[0] < L[0] && ok; x[0]++)
    for (x[1] = 0; x[1] < L[1] && ok; x[1]++)
      for (x[2] = 0; x[2] < L[2] && ok; x[2]++) {
        double *q = line.data();
        for (x[3] = 0; x[3] < L[3]; x[3]++) {
          if (!((x[0] + x[1] + x[2] + x[3]) & 1)) continue;
          for (int mu = 0; mu < 4; mu++)
            for (int dir = 0; dir < 2; dir++) {
              int y[4] = {x[0], x[1], x[2], x[3]};
              if (dir) y[mu] = (y[mu] + L[mu] - 1) % L[mu];
              int chunk, s;
              dev_site(c, y, chunk, s);
              const double sg = phase_link(c, y, mu) ? -1.0 : 1.0;
              for (int k = 0; k < 9; k++) {
                const double2 v = hu[(((size_t)chunk * 4 + mu) * 9 + k) * c.g.vbh + s];
                if (phased && mu > 0) {
                  *q++ = v.x * pr[mu - 1] - v.y * pi[mu - 1];
                  *q++ = v.x * pi[mu - 1] + v.y * pr[mu - 1];
                } else {
                  *q++ = sg * v.x;
                  *q++ = sg * v.y;
                }
              }
            }
        }
        ok = fwrite(line.data(), sizeof(double), line.size(), f) == line.size();
      }
  ok = (fclose(f) == 0) && ok;
  return ok ? 0 : fail("export_cnfg: incorrect write count");
}

int import_cnfg(Ctx &c, const char *in, int mask) {
  if (dd_unsupported(c, "import_cnfg")) return -1;
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  const int *L = c.g.L;
  FILE *f = fopen(in, "rb");
  if (!f) return fail("import_cnfg: unable to open input file");
  int32_t ls[4];
  double plaq0 = 0.0;
  if (fread(ls, sizeof(int32_t), 4, f) != 4 || fread(&plaq0, sizeof(double), 1, f) != 1) {
    fclose(f);
    return fail("import_cnfg: incorrect read count");
  }
  (void)mask;
  if (ls[0] != L[0] || ls[1] != L[1] || ls[2] != L[2] || ls[3] != L[3]) {
    fclose(f);
    return fail("import_cnfg: the lattice sizes of the file differ from the geometry (extension is not supported)");
  }
  const size_t nd = (size_t)c.g.vol * 36;
  std::vector<double2> hu(nd);
  std::vector<double> line((size_t)4 * L[3] * 18);
  double pr[3], pi[3];
  const bool phased = spatial_phases(c, pr, pi);
  int x[4];
  bool ok = true;
  for (x[0] = 0; x[0] < L[0] && ok; x[0]++)
    for (x[1] = 0; x[1] < L[1] && ok; x[1]++)
      for (x[2] = 0; x[2] < L[2] && ok; x[2]++) {
        ok = fread(line.data(), sizeof(double), line.size(), f) == line.size();
        const double *q = line.data();
        for (x[3] = 0; x[3] < L[3] && ok; x[3]++) {
          if (!((x[0] + x[1] + x[2] + x[3]) & 1)) continue;
          for (int mu = 0; mu < 4; mu++)
            for (int dir = 0; dir < 2; dir++) {
              int y[4] = {x[0], x[1], x[2], x[3]};
              if (dir) y[mu] = (y[mu] + L[mu] - 1) % L[mu];
              int chunk, s;
              dev_site(c, y, chunk, s);
              const double sg = phase_link(c, y, mu) ? -1.0 : 1.0;
              for (int k = 0; k < 9; k++) {
                double2 &d = hu[(((size_t)chunk * 4 + mu) * 9 + k) * c.g.vbh + s];
                if (phased && mu > 0)
                  d = make_double2(q[0] * pr[mu - 1] - q[1] * pi[mu - 1], q[0] * pi[mu - 1] + q[1] * pr[mu - 1]);
                else
                  d = make_double2(sg * q[0], sg * q[1]);
                q += 2;
              }
            }
        }
      }
  fclose(f);
  if (!ok) return fail("import_cnfg: incorrect read count");
  if (!c.ud && cudaMalloc(&c.ud, nd * sizeof(double2)) != cudaSuccess) return fail("out of device memory (links)");
  if (cudaMemcpy(c.ud, hu.data(), nd * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail("import_cnfg: CUDA error");
  c.have_ud = true;
  c.have_sw = false;   // the SW term belongs to the old field: recompute it
  if (links_refresh_f32(c, c.stream)) return -1;
  double plaq1 = 0.0;
  if (plaq_sum(c, &plaq1)) return -1;
  const double nplaq = 6.0 * (double)c.g.vol;
  plaq0 *= nplaq;
  // the check of archive.c:967-972
  double eps = std::sqrt(64.0 * nplaq) * DBL_EPSILON;
  eps += 64.0 * (std::fabs(plaq0) + std::fabs(plaq1)) * DBL_EPSILON;
  if (std::fabs(plaq1 - plaq0) > eps) return fail("import_cnfg: incorrect average plaquette");
  return 0;
}

// ---------------------------------------------------------- spinor fields
// reference-layout index of the site x (through the caller's ipt)
static size_t ref_index(const Ctx &c, const int x[4]) {
  int chunk, s;
  dev_site(c, x, chunk, s);
  return (size_t)c.h_dev2q[(size_t)chunk * c.g.vbh + s];
}

// qflt-style (TwoSum) accumulation of |sd|^2 over the first n sites
static double norm_sq(const double *sd, size_t n) {
  double h = 0.0, lo = 0.0;
  for (size_t i = 0; i < n * 24; i++) {
    const double x = sd[i] * sd[i];
    const double s = h + x, bb = s - h;
    lo += (h - (s - bb)) + (x - bb);
    h = s;
  }
  return h + lo;
}

int export_sfld(Ctx &c, const char *out, int eo, const void *sd) {
  if (dd_unsupported(c, "export_sfld")) return -1;
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (!c.have_ipt) return fail("export_sfld: no reference site order (pass ipt[] to the geometry call)");
  if (eo < 0 || eo > 1) return fail("export_sfld: parameter eo is out of range");
  const int *L = c.g.L;
  const size_t V = (size_t)c.g.vol;
  std::vector<double> h(V * 24);
  if (cudaMemcpy(h.data(), sd, V * 24 * sizeof(double), cudaMemcpyDefault) != cudaSuccess)
    return fail("export_sfld: cannot read the field");
  double norm = norm_sq(h.data(), eo ? V / 2 : V);
  FILE *f = fopen(out, "wb");
  if (!f) return fail("export_sfld: unable to open output file");
  int32_t ls[5] = {L[0], L[1], L[2], L[3], eo};
  bool ok = fwrite(ls, sizeof(int32_t), 5, f) == 5 && fwrite(&norm, sizeof(double), 1, f) == 1;
  std::vector<double> line((size_t)L[3] * 24);
  int x[4];
  for (x[0] = 0; x[0] < L[0] && ok; x[0]++)
    for (x[1] = 0; x[1] < L[1] && ok; x[1]++)
      for (x[2] = 0; x[2] < L[2] && ok; x[2]++) {
        size_t n = 0;
        for (x[3] = 0; x[3] < L[3]; x[3]++) {
          if (eo && ((x[0] + x[1] + x[2] + x[3]) & 1)) continue;
          std::memcpy(&line[24 * n], &h[24 * ref_index(c, x)], 24 * sizeof(double));
          n++;
        }
        ok = fwrite(line.data(), sizeof(double), 24 * n, f) == 24 * n;
      }
  ok = (fclose(f) == 0) && ok;
  return ok ? 0 : fail("export_sfld: incorrect write count");
}

int import_sfld(Ctx &c, const char *in, int eo, void *sd) {
  if (dd_unsupported(c, "import_sfld")) return -1;
  if (!c.ready) return fail("geometry not set (call b200_geometry first)");
  if (!c.have_ipt) return fail("import_sfld: no reference site order (pass ipt[] to the geometry call)");
  if (eo < 0 || eo > 1) return fail("import_sfld: parameter eo is out of range");
  const int *L = c.g.L;
  const size_t V = (size_t)c.g.vol;
  FILE *f = fopen(in, "rb");
  if (!f) return fail("import_sfld: unable to open input file");
  int32_t ls[5];
  double norm0 = 0.0;
  if (fread(ls, sizeof(int32_t), 5, f) != 5 || fread(&norm0, sizeof(double), 1, f) != 1) {
    fclose(f);
    return fail("import_sfld: incorrect read count");
  }
  if (ls[0] != L[0] || ls[1] != L[1] || ls[2] != L[2] || ls[3] != L[3] || ls[4] != eo) {
    fclose(f);
    return fail("import_sfld: lattice sizes or eo flag do not match");
  }
  std::vector<double> h(V * 24);
  if (cudaMemcpy(h.data(), sd, V * 24 * sizeof(double), cudaMemcpyDefault) != cudaSuccess) {
    fclose(f);
    return fail("import_sfld: cannot read the field");
  }
  std::vector<double> line((size_t)L[3] * 24);
  const size_t n3 = eo ? (size_t)L[3] / 2 : (size_t)L[3];
  int x[4];
  bool ok = true;
  for (x[0] = 0; x[0] < L[0] && ok; x[0]++)
    for (x[1] = 0; x[1] < L[1] && ok; x[1]++)
      for (x[2] = 0; x[2] < L[2] && ok; x[2]++) {
        ok = fread(line.data(), sizeof(double), 24 * n3, f) == 24 * n3;
        size_t n = 0;
        for (x[3] = 0; x[3] < L[3] && ok; x[3]++) {
          if (eo && ((x[0] + x[1] + x[2] + x[3]) & 1)) continue;
          std::memcpy(&h[24 * ref_index(c, x)], &line[24 * n], 24 * sizeof(double));
          n++;
        }
      }
  fclose(f);
  if (!ok) return fail("import_sfld: incorrect read count");
  const double norm1 = norm_sq(h.data(), eo ? V / 2 : V);
  // the check of sarchive.c:612-615
  if (std::fabs(norm1 - norm0) > 64.0 * (norm0 + norm1) * DBL_EPSILON) return fail("import_sfld: incorrect square norm");
  if (cudaMemcpy(sd, h.data(), V * 24 * sizeof(double), cudaMemcpyDefault) != cudaSuccess)
    return fail("import_sfld: cannot write the field");
  return 0;
}

}  // namespace qcd
