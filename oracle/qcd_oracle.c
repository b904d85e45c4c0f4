/*
 * CPU restatement of the reference's Dirac-operator / SAP+GCR path.
 * TEST INFRASTRUCTURE ONLY: the checker for the device library, never part of
 * the product.  Built by oracle/build_oracle.py into oracle/liboracle.so.
 *
 * Plain C, written for readability: one site at a time on a lexicographic
 * layout (site index x3 + L3*(x2 + L2*(x1 + L1*x0)), all parities mixed):
 *   spinor  : 24 reals per site (c1..c4, 3 complex each), double or float
 *   links   : U(x,mu) forward links, 18 doubles at [4*x + mu]
 *   pauli   : upper/lower 6x6 Hermitian, 36 reals at [2*x + half]
 * Each function names the reference function (file:line) it restates.  The
 * restatement is pinned against the reference library itself
 * (oracle/_ref, tests/test_oracle.py) on identical inputs.
 */
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>

typedef struct
{
   int L[4], vol;
} geom_t;

static int lex(const geom_t *g, const int x[4])
{
   return x[3] + g->L[3] * (x[2] + g->L[2] * (x[1] + g->L[1] * x[0]));
}

static void coords(const geom_t *g, int ix, int x[4])
{
   int mu;
   for (mu = 3; mu >= 0; mu--)
   {
      x[mu] = ix % g->L[mu];
      ix /= g->L[mu];
   }
}

static int nbr(const geom_t *g, int ix, int mu, int dir)
{
   int x[4];
   coords(g, ix, x);
   x[mu] = (x[mu] + dir + g->L[mu]) % g->L[mu];
   return lex(g, x);
}

static int parity(const geom_t *g, int ix)
{
   int x[4];
   coords(g, ix, x);
   return (x[0] + x[1] + x[2] + x[3]) & 1;
}

/* ----------------------------------------------------- generic precision */
/* The operator code is written once as a macro template over the real type
 * R; FP64 and FP32 instances follow the reference's Dw_dble.c and Dw.c. */

#define DEFINE_OPS(R, SFX)                                                           \
                                                                                     \
/* (A + i mu) w for packed Hermitian A (pauli_dble.c:1336 mul_pauli_dble) */         \
static void mul_pauli_##SFX(R mu, const R *u, const R *w, R *r)                      \
{                                                                                    \
   int i, j, k;                                                                      \
   R o[12];                                                                          \
   for (i = 0; i < 6; i++)                                                           \
   {                                                                                 \
      o[2 * i] = u[i] * w[2 * i] - mu * w[2 * i + 1];                                \
      o[2 * i + 1] = u[i] * w[2 * i + 1] + mu * w[2 * i];                            \
   }                                                                                 \
   k = 6;                                                                            \
   for (i = 0; i < 6; i++)                                                           \
      for (j = i + 1; j < 6; j++, k += 2)                                            \
      {                                                                              \
         R ar = u[k], ai = u[k + 1];                                                 \
         o[2 * i] += ar * w[2 * j] - ai * w[2 * j + 1];                              \
         o[2 * i + 1] += ar * w[2 * j + 1] + ai * w[2 * j];                          \
         o[2 * j] += ar * w[2 * i] + ai * w[2 * i + 1];                              \
         o[2 * j + 1] += ar * w[2 * i + 1] - ai * w[2 * i];                          \
      }                                                                              \
   memcpy(r, o, sizeof(o));                                                          \
}                                                                                    \
                                                                                     \
/* r = U v or U^dag v, v and r 3 complex */                                          \
static void su3mul_##SFX(const double *ud, int dag, const R *v, R *r)                \
{                                                                                    \
   int i, j;                                                                         \
   for (i = 0; i < 3; i++)                                                           \
   {                                                                                 \
      R re = 0, im = 0;                                                              \
      for (j = 0; j < 3; j++)                                                        \
      {                                                                              \
         R a = (R)ud[dag ? 2 * (3 * j + i) : 2 * (3 * i + j)];                       \
         R b = (R)ud[dag ? 2 * (3 * j + i) + 1 : 2 * (3 * i + j) + 1];               \
         if (dag) b = -b;                                                            \
         re += a * v[2 * j] - b * v[2 * j + 1];                                      \
         im += a * v[2 * j + 1] + b * v[2 * j];                                      \
      }                                                                              \
      r[2 * i] = re;                                                                 \
      r[2 * i + 1] = im;                                                             \
   }                                                                                 \
}                                                                                    \
                                                                                     \
/* h = a + f*b for 3-vectors, f in {+1,-1,+i,-i} coded 0..3 */                       \
static void comb_##SFX(const R *a, const R *b, int f, R *h)                          \
{                                                                                    \
   int i;                                                                            \
   for (i = 0; i < 3; i++)                                                           \
   {                                                                                 \
      R br = b[2 * i], bi = b[2 * i + 1];                                            \
      if (f == 0) { h[2*i] = a[2*i] + br; h[2*i+1] = a[2*i+1] + bi; }                \
      else if (f == 1) { h[2*i] = a[2*i] - br; h[2*i+1] = a[2*i+1] - bi; }           \
      else if (f == 2) { h[2*i] = a[2*i] - bi; h[2*i+1] = a[2*i+1] + br; }           \
      else { h[2*i] = a[2*i] + bi; h[2*i+1] = a[2*i+1] - br; }                       \
   }                                                                                 \
}                                                                                    \
                                                                                     \
/* r += f*c (f coded as in comb) */                                                  \
static void acc_##SFX(R *r, const R *c, int f)                                       \
{                                                                                    \
   int i;                                                                            \
   for (i = 0; i < 3; i++)                                                           \
   {                                                                                 \
      R cr = c[2 * i], ci = c[2 * i + 1];                                            \
      if (f == 0) { r[2*i] += cr; r[2*i+1] += ci; }                                  \
      else if (f == 1) { r[2*i] -= cr; r[2*i+1] -= ci; }                             \
      else if (f == 2) { r[2*i] -= ci; r[2*i+1] += cr; }                             \
      else { r[2*i] += ci; r[2*i+1] -= cr; }                                         \
   }                                                                                 \
}                                                                                    \
                                                                                     \
/* Hop term of direction mu at a site, forward (dir=+1, link U(x,mu), spinor    */   \
/* s(x+mu)) or backward (dir=-1, U(x-mu,mu)^dag, s(x-mu)); the projector rows  */   \
/* are those of doe() (Dw_dble.c:1114-1242): for each of the two Weyl rows,     */   \
/* h = s[a] + f s[b], c = U h, out[a] += c, out[b] += g c.                       */   \
static void hop_##SFX(int mu, int dir, const double *ud, const R *s, R *out)         \
{                                                                                    \
   /* {a, b, f, g} for row 1 and row 2, forward; backward flips f and g signs */     \
   static const int tab[4][2][4] = {                                                 \
      {{0, 2, 0, 0}, {1, 3, 0, 0}},                                                  \
      {{0, 3, 2, 3}, {1, 2, 2, 3}},                                                  \
      {{0, 3, 0, 0}, {1, 2, 1, 1}},                                                  \
      {{0, 2, 2, 3}, {1, 3, 3, 2}}};                                                 \
   int row;                                                                          \
   R h[6], c[6];                                                                     \
   for (row = 0; row < 2; row++)                                                     \
   {                                                                                 \
      int a = tab[mu][row][0], b = tab[mu][row][1];                                  \
      int f = tab[mu][row][2], gg = tab[mu][row][3];                                 \
      if (dir < 0)                                                                   \
      {                                                                              \
         f ^= 1;                                                                     \
         gg ^= 1;                                                                    \
      }                                                                              \
      comb_##SFX(s + 6 * a, s + 6 * b, f, h);                                        \
      su3mul_##SFX(ud, dir < 0, h, c);                                               \
      acc_##SFX(out + 6 * a, c, 0);                                                  \
      acc_##SFX(out + 6 * b, c, gg);                                                 \
   }                                                                                 \
}                                                                                    \
                                                                                     \
/* -1/2 sum_mu hop terms of s around site ix; in-block restriction if blk */         \
static void hopsum_##SFX(const geom_t *g, const double *U, const R *s, int ix,        \
                         const int *bs, R *out)                                      \
{                                                                                    \
   int mu, k, x[4];                                                                  \
   memset(out, 0, 24 * sizeof(R));                                                   \
   coords(g, ix, x);                                                                 \
   for (mu = 0; mu < 4; mu++)                                                        \
   {                                                                                 \
      if (!bs || (x[mu] % bs[mu]) + 1 < bs[mu])                                      \
      {                                                                              \
         int iy = nbr(g, ix, mu, +1);                                                \
         hop_##SFX(mu, +1, U + 18 * (4 * ix + mu), s + 24 * iy, out);                \
      }                                                                              \
      if (!bs || (x[mu] % bs[mu]) > 0)                                               \
      {                                                                              \
         int iy = nbr(g, ix, mu, -1);                                                \
         hop_##SFX(mu, -1, U + 18 * (4 * iy + mu), s + 24 * iy, out);                \
      }                                                                              \
   }                                                                                 \
   for (k = 0; k < 24; k++)                                                          \
      out[k] *= (R)(-0.5);                                                           \
}                                                                                    \
                                                                                     \
/* (A(x) + i mu gamma5) s(x): +mu on the upper, -mu on the lower Weyl half */        \
/* (pauli_dble.c:1840 apply_sw_dble) */                                              \
static void swsite_##SFX(const R *sw, int ix, R mu, const R *s, R *r)                \
{                                                                                    \
   R t[24];                                                                          \
   mul_pauli_##SFX(mu, sw + 72 * ix, s, t);                                          \
   mul_pauli_##SFX(-mu, sw + 72 * ix + 36, s + 12, t + 12);                          \
   memcpy(r, t, sizeof(t));                                                          \
}

DEFINE_OPS(double, d)
DEFINE_OPS(float, f)

/* --------------------------------------------------------- Dirac operators */
/* op: 0 Dw, 1 Dwee, 2 Dwoo, 3 Dwoe, 4 Dweo, 5 Dwhat (Dw_dble.c:1377-1889).
 * sw: SW field, swi: its inverse (used on odd sites by Dwhat), tm_eo: the
 * twisted-mass eo flag.  r is read and updated by Dweo, and keeps its other
 * parity untouched for the even/odd pieces. */
void or_dirac_dble(const int *L, int op, double mu, int tm_eo, const double *U, const double *sw,
                   const double *swi, const double *s, double *r)
{
   geom_t g;
   int ix, k;
   double muo = tm_eo ? 0.0 : mu, h[24], a[24];
   double *t = NULL;

   g.L[0] = L[0]; g.L[1] = L[1]; g.L[2] = L[2]; g.L[3] = L[3];
   g.vol = L[0] * L[1] * L[2] * L[3];
   if (op == 5)
   {
      /* t_o = A_o^-1 D_oe s_e */
      t = calloc((size_t)24 * g.vol, sizeof(double));
      for (ix = 0; ix < g.vol; ix++)
         if (parity(&g, ix) == 1)
         {
            hopsum_d(&g, U, s, ix, NULL, h);
            swsite_d(swi, ix, 0.0, h, t + 24 * ix);
         }
   }
   double *out = calloc((size_t)24 * g.vol, sizeof(double));
   memcpy(out, r, 24 * sizeof(double) * g.vol);
   for (ix = 0; ix < g.vol; ix++)
   {
      int p = parity(&g, ix);
      double *o = out + 24 * ix;
      switch (op)
      {
      case 0:
         swsite_d(sw, ix, p ? muo : mu, s + 24 * ix, a);
         hopsum_d(&g, U, s, ix, NULL, h);
         for (k = 0; k < 24; k++) o[k] = a[k] + h[k];
         break;
      case 1:
         if (p == 0) swsite_d(sw, ix, mu, s + 24 * ix, o);
         break;
      case 2:
         if (p == 1) swsite_d(sw, ix, muo, s + 24 * ix, o);
         break;
      case 3:
         if (p == 1) hopsum_d(&g, U, s, ix, NULL, o);
         break;
      case 4:
         if (p == 0)
         {
            hopsum_d(&g, U, s, ix, NULL, h);
            for (k = 0; k < 24; k++) o[k] -= h[k];
         }
         break;
      case 5:
         if (p == 0)
         {
            swsite_d(sw, ix, mu, s + 24 * ix, a);
            hopsum_d(&g, U, t, ix, NULL, h);
            for (k = 0; k < 24; k++) o[k] = a[k] - h[k];
         }
         break;
      }
   }
   memcpy(r, out, 24 * sizeof(double) * g.vol);
   free(out);
   free(t);
}

/* single-precision twin (Dw.c:973-1473) */
void or_dirac(const int *L, int op, float mu, int tm_eo, const double *U, const float *sw, const float *swi,
              const float *s, float *r)
{
   geom_t g;
   int ix, k;
   float muo = tm_eo ? 0.0f : mu, h[24], a[24];
   float *t = NULL;

   g.L[0] = L[0]; g.L[1] = L[1]; g.L[2] = L[2]; g.L[3] = L[3];
   g.vol = L[0] * L[1] * L[2] * L[3];
   if (op == 5)
   {
      t = calloc((size_t)24 * g.vol, sizeof(float));
      for (ix = 0; ix < g.vol; ix++)
         if (parity(&g, ix) == 1)
         {
            hopsum_f(&g, U, s, ix, NULL, h);
            swsite_f(swi, ix, 0.0f, h, t + 24 * ix);
         }
   }
   float *out = calloc((size_t)24 * g.vol, sizeof(float));
   memcpy(out, r, 24 * sizeof(float) * g.vol);
   for (ix = 0; ix < g.vol; ix++)
   {
      int p = parity(&g, ix);
      float *o = out + 24 * ix;
      switch (op)
      {
      case 0:
         swsite_f(sw, ix, p ? muo : mu, s + 24 * ix, a);
         hopsum_f(&g, U, s, ix, NULL, h);
         for (k = 0; k < 24; k++) o[k] = a[k] + h[k];
         break;
      case 1:
         if (p == 0) swsite_f(sw, ix, mu, s + 24 * ix, o);
         break;
      case 2:
         if (p == 1) swsite_f(sw, ix, muo, s + 24 * ix, o);
         break;
      case 3:
         if (p == 1) hopsum_f(&g, U, s, ix, NULL, o);
         break;
      case 4:
         if (p == 0)
         {
            hopsum_f(&g, U, s, ix, NULL, h);
            for (k = 0; k < 24; k++) o[k] -= h[k];
         }
         break;
      case 5:
         if (p == 0)
         {
            swsite_f(sw, ix, mu, s + 24 * ix, a);
            hopsum_f(&g, U, t, ix, NULL, h);
            for (k = 0; k < 24; k++) o[k] = a[k] - h[k];
         }
         break;
      }
   }
   memcpy(r, out, 24 * sizeof(float) * g.vol);
   free(out);
   free(t);
}

/* ------------------------------------------------------------- SW term */
/* Inverse of (A + i mu) by Gauss-Jordan elimination; returns the Hermitian
 * part in packed form and the safety flag of inv_pauli_dble
 * (pauli_dble.c:1718-1759: unsafe iff |M|_F^2 |M^-1|_F^2 > 1e4). */
int or_inv_pauli(double mu, const double *u, double *out)
{
   double ar[36], ai[36], br[36], bi[36], fn = 0.0, sm = 0.0;
   int i, j, k, c, r, ifail = 0;

   memset(ar, 0, sizeof(ar)); memset(ai, 0, sizeof(ai));
   memset(br, 0, sizeof(br)); memset(bi, 0, sizeof(bi));
   k = 6;
   for (i = 0; i < 6; i++)
   {
      ar[7 * i] = u[i]; ai[7 * i] = mu; br[7 * i] = 1.0;
      fn += u[i] * u[i] + mu * mu;
      for (j = i + 1; j < 6; j++, k += 2)
      {
         ar[6 * i + j] = u[k]; ai[6 * i + j] = u[k + 1];
         ar[6 * j + i] = u[k]; ai[6 * j + i] = -u[k + 1];
         fn += 2.0 * (u[k] * u[k] + u[k + 1] * u[k + 1]);
      }
   }
   for (c = 0; c < 6; c++)
   {
      int piv = c;
      double best = ar[7 * c] * ar[7 * c] + ai[7 * c] * ai[7 * c], pr, pi, d, qr, qi;
      for (r = c + 1; r < 6; r++)
      {
         double v = ar[6 * r + c] * ar[6 * r + c] + ai[6 * r + c] * ai[6 * r + c];
         if (v > best) { best = v; piv = r; }
      }
      if (best == 0.0) ifail = 1;
      if (piv != c)
         for (j = 0; j < 6; j++)
         {
            double t;
            t = ar[6*c+j]; ar[6*c+j] = ar[6*piv+j]; ar[6*piv+j] = t;
            t = ai[6*c+j]; ai[6*c+j] = ai[6*piv+j]; ai[6*piv+j] = t;
            t = br[6*c+j]; br[6*c+j] = br[6*piv+j]; br[6*piv+j] = t;
            t = bi[6*c+j]; bi[6*c+j] = bi[6*piv+j]; bi[6*piv+j] = t;
         }
      pr = ar[7 * c]; pi = ai[7 * c];
      d = pr * pr + pi * pi;
      if (d == 0.0) d = 1.0;
      qr = pr / d; qi = -pi / d;
      for (j = 0; j < 6; j++)
      {
         double xr = ar[6*c+j], xi = ai[6*c+j];
         ar[6*c+j] = xr * qr - xi * qi; ai[6*c+j] = xr * qi + xi * qr;
         xr = br[6*c+j]; xi = bi[6*c+j];
         br[6*c+j] = xr * qr - xi * qi; bi[6*c+j] = xr * qi + xi * qr;
      }
      for (r = 0; r < 6; r++)
      {
         double fr, fi;
         if (r == c) continue;
         fr = ar[6 * r + c]; fi = ai[6 * r + c];
         for (j = 0; j < 6; j++)
         {
            ar[6*r+j] -= fr * ar[6*c+j] - fi * ai[6*c+j];
            ai[6*r+j] -= fr * ai[6*c+j] + fi * ar[6*c+j];
            br[6*r+j] -= fr * br[6*c+j] - fi * bi[6*c+j];
            bi[6*r+j] -= fr * bi[6*c+j] + fi * br[6*c+j];
         }
      }
   }
   for (i = 0; i < 36; i++) sm += br[i] * br[i] + bi[i] * bi[i];
   if (1.0e-4 * fn * sm > 1.0) ifail = 1;
   k = 6;
   for (i = 0; i < 6; i++)
   {
      out[i] = br[7 * i];
      for (j = i + 1; j < 6; j++, k += 2)
      {
         out[k] = 0.5 * (br[6 * i + j] + br[6 * j + i]);
         out[k + 1] = 0.5 * (bi[6 * i + j] - bi[6 * j + i]);
      }
   }
   return ifail;
}

/* 3x3 complex helpers for the field tensor (18 doubles, row major) */
static void m3mul(const double *a, const double *b, double *c)
{
   int i, j, k;
   double t[18];
   for (i = 0; i < 3; i++)
      for (j = 0; j < 3; j++)
      {
         double re = 0, im = 0;
         for (k = 0; k < 3; k++)
         {
            re += a[2*(3*i+k)] * b[2*(3*k+j)] - a[2*(3*i+k)+1] * b[2*(3*k+j)+1];
            im += a[2*(3*i+k)] * b[2*(3*k+j)+1] + a[2*(3*i+k)+1] * b[2*(3*k+j)];
         }
         t[2*(3*i+j)] = re;
         t[2*(3*i+j)+1] = im;
      }
   memcpy(c, t, sizeof(t));
}

static void m3dag(const double *a, double *c)
{
   int i, j;
   double t[18];
   for (i = 0; i < 3; i++)
      for (j = 0; j < 3; j++)
      {
         t[2*(3*i+j)] = a[2*(3*j+i)];
         t[2*(3*i+j)+1] = -a[2*(3*j+i)+1];
      }
   memcpy(c, t, sizeof(t));
}

/* X += (M - M^dag)/8 in the 9-real U(3) algebra convention
 * (su3fcts/su3prod.c:56-63, prod2u3alg :2193, ftensor.c add_X2ft) */
static void add_ah(const double *m, double *X)
{
   X[0] += 0.125 * 2.0 * m[1];
   X[1] += 0.125 * 2.0 * m[9];
   X[2] += 0.125 * 2.0 * m[17];
   X[3] += 0.125 * (m[2] - m[6]);
   X[4] += 0.125 * (m[3] + m[7]);
   X[5] += 0.125 * (m[4] - m[12]);
   X[6] += 0.125 * (m[5] + m[13]);
   X[7] += 0.125 * (m[10] - m[14]);
   X[8] += 0.125 * (m[11] + m[15]);
}

/* F_{mu nu}(x): the four plaquettes with a corner at x, each read in the
 * orientation of tcharge/ftensor.c:141-192 (periodic lattice). */
static void ftensor_site(const geom_t *g, const double *U, int ix, int mu, int nu, double *X)
{
   double w1[18], w2[18], m[18], t[18];
   int c, a, b;
   memset(X, 0, 9 * sizeof(double));
   /* corner x */
   c = ix; a = nbr(g, c, mu, 1); b = nbr(g, c, nu, 1);
   m3mul(U + 18 * (4 * c + mu), U + 18 * (4 * a + nu), w1);
   m3dag(U + 18 * (4 * b + mu), t); m3dag(U + 18 * (4 * c + nu), m); m3mul(t, m, w2);
   m3mul(w1, w2, m); add_ah(m, X);
   /* corner x - mu - nu: w2 w1 */
   c = nbr(g, nbr(g, ix, mu, -1), nu, -1); a = nbr(g, c, mu, 1); b = nbr(g, c, nu, 1);
   m3mul(U + 18 * (4 * c + mu), U + 18 * (4 * a + nu), w1);
   m3dag(U + 18 * (4 * b + mu), t); m3dag(U + 18 * (4 * c + nu), m); m3mul(t, m, w2);
   m3mul(w2, w1, m); add_ah(m, X);
   /* corner x - nu: w1' w2', w1' = U(c,nu)^dag U(c,mu), w2' = U(c+mu,nu) U(c+nu,mu)^dag */
   c = nbr(g, ix, nu, -1); a = nbr(g, c, mu, 1); b = nbr(g, c, nu, 1);
   m3dag(U + 18 * (4 * c + nu), t); m3mul(t, U + 18 * (4 * c + mu), w1);
   m3dag(U + 18 * (4 * b + mu), t); m3mul(U + 18 * (4 * a + nu), t, w2);
   m3mul(w1, w2, m); add_ah(m, X);
   /* corner x - mu: w2' w1' */
   c = nbr(g, ix, mu, -1); a = nbr(g, c, mu, 1); b = nbr(g, c, nu, 1);
   m3dag(U + 18 * (4 * c + nu), t); m3mul(t, U + 18 * (4 * c + mu), w1);
   m3dag(U + 18 * (4 * b + mu), t); m3mul(U + 18 * (4 * a + nu), t, w2);
   m3mul(w2, w1, m); add_ah(m, X);
}

/* U(3) algebra -> packed Pauli entries, restated from u3_alg2pauli1/2/3
 * (sw_term/sw_term.c:145-219): {target, source, sign, add} */
static const int pm1[15][4] = {{10,0,-1,0},{12,4,-1,0},{13,3,1,0},{14,6,-1,0},{15,5,1,0},{18,4,-1,0},
   {19,3,-1,0},{20,1,-1,0},{22,8,-1,0},{23,7,1,0},{24,6,-1,0},{25,5,-1,0},{26,8,-1,0},{27,7,-1,0},
   {28,2,-1,0}};
static const int pm2[15][4] = {{11,0,1,0},{12,3,1,1},{13,4,1,1},{14,5,1,1},{15,6,1,1},{18,3,-1,1},
   {19,4,1,1},{21,1,1,0},{22,7,1,1},{23,8,1,1},{24,5,-1,1},{25,6,1,1},{26,7,-1,1},{27,8,1,1},
   {29,2,1,0}};
static const int pm3[18][4] = {{0,0,-1,0},{1,1,-1,0},{2,2,-1,0},{3,0,1,0},{4,1,1,0},{5,2,1,0},
   {6,4,-1,0},{7,3,1,0},{8,6,-1,0},{9,5,1,0},{16,8,-1,0},{17,7,1,0},{30,4,1,0},{31,3,-1,0},
   {32,6,1,0},{33,5,-1,0},{34,8,1,0},{35,7,-1,0}};

static void apply_pm(const int (*m)[4], int n, const double *X, double *u)
{
   int i;
   for (i = 0; i < n; i++)
   {
      double v = m[i][2] * X[m[i][1]];
      if (m[i][3]) u[m[i][0]] += v;
      else u[m[i][0]] = v;
   }
}

/* sw_term(NO_PTS) for periodic boundary conditions (sw_term.c:225-243,
 * :247-345): upper = c2 (F23-F01, F31-F02, F12-F03), lower with +, then
 * + (4+m0) on the diagonal; c2 = -csw/2.  sw[72*x + 36*half]. */
void or_sw_term(const int *L, double csw, double m0, const double *U, double *sw)
{
   geom_t g;
   int ix, n, k, half;
   static const int pl[6][2] = {{0, 1}, {0, 2}, {0, 3}, {2, 3}, {3, 1}, {1, 2}};
   double F[6][9], X[9], c2 = -0.5 * csw;

   g.L[0] = L[0]; g.L[1] = L[1]; g.L[2] = L[2]; g.L[3] = L[3];
   g.vol = L[0] * L[1] * L[2] * L[3];
   for (ix = 0; ix < g.vol; ix++)
   {
      for (n = 0; n < 6; n++)
         ftensor_site(&g, U, ix, pl[n][0], pl[n][1], F[n]);
      for (half = 0; half < 2; half++)
      {
         double sg = half ? 1.0 : -1.0, *u = sw + 72 * ix + 36 * half;
         for (k = 0; k < 9; k++) X[k] = c2 * (F[3][k] + sg * F[0][k]);
         apply_pm(pm1, 15, X, u);
         for (k = 0; k < 9; k++) X[k] = c2 * (F[4][k] + sg * F[1][k]);
         apply_pm(pm2, 15, X, u);
         for (k = 0; k < 9; k++) X[k] = c2 * (F[5][k] + sg * F[2][k]);
         apply_pm(pm3, 18, X, u);
         for (k = 0; k < 6; k++) u[k] += 4.0 + m0;
      }
   }
}

/* --------------------------------------------------------------- SAP */
/* Products of FP32 fields accumulated in double (linalg/salg.c:1050-1078). */
static double nsq_f(int n, const float *x)
{
   int i;
   double s = 0.0;
   for (i = 0; i < n; i++) s += (double)x[i] * x[i];
   return s;
}

static void dot_f(int n, const float *x, const float *y, double *re, double *im)
{
   int i;
   double a = 0.0, b = 0.0;
   for (i = 0; i < n; i += 2)
   {
      a += (double)x[i] * y[i] + (double)x[i + 1] * y[i + 1];
      b += (double)x[i] * y[i + 1] - (double)x[i + 1] * y[i];
   }
   *re = a;
   *im = b;
}

/* One SAP cycle (sap/sap.c:720), FP32.  Blocks of colour 0 (sum of block
 * coordinates even), then colour 1; per block nmr MR steps on the block
 * operator with zero exterior -- on Dhat (isolv=1, blk_solv.c:1153) or on Dw
 * (isolv=0, blk_solv.c:1117) -- then psi += phi, rho <- block residual
 * (update_flds0/1/2, sap.c:592-716), and rho -= D phi on the exterior faces
 * (Dw_bnd + sap_com). */
void or_sap(const int *L, const int *bs, float mu, int isolv, int nmr, int tm_eo, const double *U,
            const float *sw, const float *swi, float *psi, float *rho)
{
   geom_t g;
   int nb[4], nbl, vb, ic, b, i, k, mu_;
   g.L[0] = L[0]; g.L[1] = L[1]; g.L[2] = L[2]; g.L[3] = L[3];
   g.vol = L[0] * L[1] * L[2] * L[3];
   for (mu_ = 0; mu_ < 4; mu_++) nb[mu_] = L[mu_] / bs[mu_];
   nbl = nb[0] * nb[1] * nb[2] * nb[3];
   vb = bs[0] * bs[1] * bs[2] * bs[3];
   int *sites = malloc(sizeof(int) * vb);
   float *s0 = calloc((size_t)24 * g.vol, sizeof(float)), *s1 = calloc((size_t)24 * g.vol, sizeof(float));
   float *s2 = calloc((size_t)24 * g.vol, sizeof(float)), *w = calloc((size_t)24 * g.vol, sizeof(float));
   float *phi = calloc((size_t)24 * g.vol, sizeof(float));
   float h[24], a[24];
   float muo = tm_eo ? 0.0f : mu;

   for (ic = 0; ic < 2; ic++)
   {
      for (b = 0; b < nbl; b++)
      {
         int n[4], r = b, x[4], ns = 0;
         for (mu_ = 3; mu_ >= 0; mu_--) { n[mu_] = r % nb[mu_]; r /= nb[mu_]; }
         if (((n[0] + n[1] + n[2] + n[3]) & 1) != ic) continue;
         for (i = 0; i < vb; i++)
         {
            int q = i;
            for (mu_ = 3; mu_ >= 0; mu_--) { x[mu_] = n[mu_] * bs[mu_] + q % bs[mu_]; q /= bs[mu_]; }
            sites[ns++] = lex(&g, x);
         }
         if (isolv)
         {
            /* v_o = A_o^-1 rho_o ; s1_e = rho_e - D_eo v_o ; s0_e = 0 */
            for (i = 0; i < vb; i++)
               if (parity(&g, sites[i]) == 1)
                  swsite_f(swi, sites[i], 0.0f, rho + 24 * sites[i], w + 24 * sites[i]);
            for (i = 0; i < vb; i++)
               if (parity(&g, sites[i]) == 0)
               {
                  int ix = sites[i];
                  hopsum_f(&g, U, w, ix, bs, h);
                  for (k = 0; k < 24; k++) { s1[24*ix+k] = rho[24*ix+k] - h[k]; s0[24*ix+k] = 0.0f; }
               }
            for (int imr = 0; imr < nmr; imr++)
            {
               double rr = 0.0, zr = 0.0, zi = 0.0, tr, ti;
               for (i = 0; i < vb; i++)
                  if (parity(&g, sites[i]) == 1)
                  {
                     hopsum_f(&g, U, s1, sites[i], bs, h);
                     swsite_f(swi, sites[i], 0.0f, h, w + 24 * sites[i]);
                  }
               for (i = 0; i < vb; i++)
                  if (parity(&g, sites[i]) == 0)
                  {
                     int ix = sites[i];
                     swsite_f(sw, ix, mu, s1 + 24 * ix, a);
                     hopsum_f(&g, U, w, ix, bs, h);
                     for (k = 0; k < 24; k++) s2[24 * ix + k] = a[k] - h[k];
                     rr += nsq_f(24, s2 + 24 * ix);
                     dot_f(24, s2 + 24 * ix, s1 + 24 * ix, &tr, &ti);
                     zr += tr; zi += ti;
                  }
               float rf = (float)rr;
               if (rf < 2.0f * FLT_MIN) break;
               float ri = 1.0f / rf, fzr = (float)zr * ri, fzi = (float)zi * ri;
               for (i = 0; i < vb; i++)
                  if (parity(&g, sites[i]) == 0)
                  {
                     float *p0 = s0 + 24 * sites[i], *p1 = s1 + 24 * sites[i], *p2 = s2 + 24 * sites[i];
                     for (k = 0; k < 24; k += 2)
                     {
                        p0[k] += fzr * p1[k] - fzi * p1[k + 1];
                        p0[k + 1] += fzr * p1[k + 1] + fzi * p1[k];
                        p1[k] -= fzr * p2[k] - fzi * p2[k + 1];
                        p1[k + 1] -= fzr * p2[k + 1] + fzi * p2[k];
                     }
                  }
            }
            for (i = 0; i < vb; i++)
            {
               int ix = sites[i];
               float *ph = phi + 24 * ix;
               if (parity(&g, ix) == 1)
               {
                  float t[24], v[24];
                  hopsum_f(&g, U, s0, ix, bs, h);
                  swsite_f(swi, ix, 0.0f, h, t);
                  swsite_f(swi, ix, 0.0f, rho + 24 * ix, v);
                  for (k = 0; k < 24; k++) ph[k] = v[k] - t[k];
               }
            }
            for (i = 0; i < vb; i++)
            {
               int ix = sites[i];
               float *ph = phi + 24 * ix;
               if (parity(&g, ix) == 0)
               {
                  memcpy(ph, s0 + 24 * ix, 24 * sizeof(float));
                  memcpy(rho + 24 * ix, s1 + 24 * ix, 24 * sizeof(float));
               }
               else
               {
                  for (k = 0; k < 24; k += 2)
                  {
                     float m = (k < 12) ? -mu : mu;   /* rho_o = -i mu gamma5 phi_o */
                     if (tm_eo) m = 0.0f;
                     rho[24 * ix + k] = -m * ph[k + 1];
                     rho[24 * ix + k + 1] = m * ph[k];
                  }
               }
               for (k = 0; k < 24; k++) psi[24 * ix + k] += ph[k];
            }
         }
         else
         {
            for (i = 0; i < vb; i++)
            {
               int ix = sites[i];
               memcpy(s1 + 24 * ix, rho + 24 * ix, 24 * sizeof(float));
               memset(s0 + 24 * ix, 0, 24 * sizeof(float));
            }
            for (int imr = 0; imr < nmr; imr++)
            {
               double rr = 0.0, zr = 0.0, zi = 0.0, tr, ti;
               for (i = 0; i < vb; i++)
               {
                  int ix = sites[i];
                  swsite_f(sw, ix, parity(&g, ix) ? muo : mu, s1 + 24 * ix, a);
                  hopsum_f(&g, U, s1, ix, bs, h);
                  for (k = 0; k < 24; k++) s2[24 * ix + k] = a[k] + h[k];
                  rr += nsq_f(24, s2 + 24 * ix);
                  dot_f(24, s2 + 24 * ix, s1 + 24 * ix, &tr, &ti);
                  zr += tr; zi += ti;
               }
               float rf = (float)rr;
               if (rf < 2.0f * FLT_MIN) break;
               float ri = 1.0f / rf, fzr = (float)zr * ri, fzi = (float)zi * ri;
               for (i = 0; i < vb; i++)
               {
                  float *p0 = s0 + 24 * sites[i], *p1 = s1 + 24 * sites[i], *p2 = s2 + 24 * sites[i];
                  for (k = 0; k < 24; k += 2)
                  {
                     p0[k] += fzr * p1[k] - fzi * p1[k + 1];
                     p0[k + 1] += fzr * p1[k + 1] + fzi * p1[k];
                     p1[k] -= fzr * p2[k] - fzi * p2[k + 1];
                     p1[k + 1] -= fzr * p2[k + 1] + fzi * p2[k];
                  }
               }
            }
            for (i = 0; i < vb; i++)
            {
               int ix = sites[i];
               memcpy(phi + 24 * ix, s0 + 24 * ix, 24 * sizeof(float));
               memcpy(rho + 24 * ix, s1 + 24 * ix, 24 * sizeof(float));
               for (k = 0; k < 24; k++) psi[24 * ix + k] += s0[24 * ix + k];
            }
         }
      }
      /* exterior update: rho(y) -= D_{y,x} phi(x) for x in a colour-ic block,
       * y outside that block */
      for (i = 0; i < g.vol; i++)
      {
         int y[4], by = 0;
         coords(&g, i, y);
         for (mu_ = 0; mu_ < 4; mu_++) by += y[mu_] / bs[mu_];
         if ((by & 1) == ic) continue;
         memset(h, 0, sizeof(h));
         for (mu_ = 0; mu_ < 4; mu_++)
         {
            if (y[mu_] % bs[mu_] == bs[mu_] - 1)
            {
               int iz = nbr(&g, i, mu_, +1);
               hop_f(mu_, +1, U + 18 * (4 * i + mu_), phi + 24 * iz, h);
            }
            if (y[mu_] % bs[mu_] == 0)
            {
               int iz = nbr(&g, i, mu_, -1);
               hop_f(mu_, -1, U + 18 * (4 * iz + mu_), phi + 24 * iz, h);
            }
         }
         for (k = 0; k < 24; k++) rho[24 * i + k] += 0.5f * h[k];
      }
   }
   free(sites); free(s0); free(s1); free(s2); free(w); free(phi);
}

/* -------------------------------------------------------- GCR solver */
typedef struct { float re, im; } cf_t;

static double nsq_d(int n, const double *x)
{
   int i;
   double s = 0.0;
   for (i = 0; i < n; i++) s += x[i] * x[i];
   return s;
}

static double unorm_f(int vol, const float *x)
{
   int i;
   double m = 0.0;
   for (i = 0; i < vol; i++)
   {
      double t = nsq_f(24, x + 24 * i);
      if (t > m) m = t;
   }
   return (double)(float)sqrt(m);
}

static double unorm_d(int vol, const double *x)
{
   int i;
   double m = 0.0;
   for (i = 0; i < vol; i++)
   {
      double t = nsq_d(24, x + 24 * i);
      if (t > m) m = t;
   }
   return sqrt(m);
}

/* SAP+GCR (sap/sap_gcr.c:140) with flexible GCR (linsolv/fgcr.c:215):
 * FP32 Krylov space, double accumulation of products, FP64 true residual at
 * every restart, restart when rn < 100 FLT_EPSILON rn_old. */
double or_sap_gcr(const int *L, const int *bs, int isolv, int nmr, int ncy, int tm_eo, double csw_unused,
                  const double *U, const double *swd, const float *sw, const float *swi, int nkv, int nmx,
                  int istop, double res, double mu, const double *eta, double *psi, int *ifail, int *status)
{
   int vol = L[0] * L[1] * L[2] * L[3], n24 = 24 * vol;
   int k, l, i, j;
   double rho0, rn, rn_old, tol;
   const double PRECISION_LIMIT = (double)(100.0f * FLT_EPSILON);
   (void)csw_unused;

   ifail[0] = 0;
   status[0] = 0;
   rho0 = unorm_d(vol, eta);
   if (rho0 == 0.0)
   {
      memset(psi, 0, sizeof(double) * n24);
      return 0.0;
   }
   double *rsd = malloc(sizeof(double) * n24), *wrk = malloc(sizeof(double) * n24);
   float **phi = malloc(sizeof(float *) * nkv), **chi = malloc(sizeof(float *) * nkv);
   float *rho = malloc(sizeof(float) * n24);
   cf_t *a = malloc(sizeof(cf_t) * nkv * nkv), *c = malloc(sizeof(cf_t) * nkv);
   float *b = malloc(sizeof(float) * nkv);
   for (k = 0; k < nkv; k++)
   {
      phi[k] = malloc(sizeof(float) * n24);
      chi[k] = malloc(sizeof(float) * n24);
   }
   for (i = 0; i < n24; i++) rsd[i] = eta[i] / rho0;
   memset(psi, 0, sizeof(double) * n24);
   for (i = 0; i < n24; i++) rho[i] = (float)rsd[i];
   rn = istop ? unorm_f(vol, rho) : sqrt((double)(float)nsq_f(n24, rho));
   tol = res * rn;
   while (rn > tol)
   {
      rn_old = rn;
      for (k = 0;; k++)
      {
         /* Mop: phi = 0, chi = rho, ncy SAP cycles, chi = rho - chi */
         memset(phi[k], 0, sizeof(float) * n24);
         memcpy(chi[k], rho, sizeof(float) * n24);
         for (j = 0; j < ncy; j++)
            or_sap(L, bs, (float)mu, isolv, nmr, tm_eo, U, sw, swi, phi[k], chi[k]);
         for (i = 0; i < n24; i++) chi[k][i] = rho[i] - chi[k][i];
         for (l = 0; l < k; l++)
         {
            double re, im;
            dot_f(n24, chi[l], chi[k], &re, &im);
            a[nkv * l + k].re = (float)re;
            a[nkv * l + k].im = (float)im;
            for (i = 0; i < n24; i += 2)
            {
               float xr = chi[l][i], xi = chi[l][i + 1];
               chi[k][i] += -a[nkv*l+k].re * xr + a[nkv*l+k].im * xi;
               chi[k][i + 1] += -a[nkv*l+k].re * xi - a[nkv*l+k].im * xr;
            }
         }
         b[k] = (float)sqrt((double)(float)nsq_f(n24, chi[k]));
         for (i = 0; i < n24; i++) chi[k][i] *= 1.0f / b[k];
         {
            double re, im;
            dot_f(n24, chi[k], rho, &re, &im);
            c[k].re = (float)re;
            c[k].im = (float)im;
         }
         for (i = 0; i < n24; i += 2)
         {
            float xr = chi[k][i], xi = chi[k][i + 1];
            rho[i] += -c[k].re * xr + c[k].im * xi;
            rho[i + 1] += -c[k].re * xi - c[k].im * xr;
         }
         rn = istop ? unorm_f(vol, rho) : sqrt((double)(float)nsq_f(n24, rho));
         status[0] += 1;
         if ((rn <= tol) || (rn < PRECISION_LIMIT * rn_old) || (k == nkv - 1) || (status[0] >= nmx))
            break;
      }
      /* update_psi (fgcr.c:181) */
      for (l = k; l >= 0; l--)
      {
         cf_t z = c[l];
         for (i = l + 1; i <= k; i++)
         {
            z.re -= a[l * nkv + i].re * c[i].re - a[l * nkv + i].im * c[i].im;
            z.im -= a[l * nkv + i].re * c[i].im + a[l * nkv + i].im * c[i].re;
         }
         float r = 1.0f / b[l];
         c[l].re = z.re * r;
         c[l].im = z.im * r;
      }
      memset(rho, 0, sizeof(float) * n24);
      for (l = k; l >= 0; l--)
         for (i = 0; i < n24; i += 2)
         {
            float xr = phi[l][i], xi = phi[l][i + 1];
            rho[i] += c[l].re * xr - c[l].im * xi;
            rho[i + 1] += c[l].re * xi + c[l].im * xr;
         }
      for (i = 0; i < n24; i++) psi[i] += (double)rho[i];
      {
         double *swi_d = NULL;
         (void)swi_d;
         or_dirac_dble(L, 0, mu, tm_eo, U, swd, NULL, psi, wrk);
      }
      for (i = 0; i < n24; i++) rho[i] = (float)(rsd[i] - wrk[i]);
      rn = istop ? unorm_f(vol, rho) : sqrt((double)(float)nsq_f(n24, rho));
      if ((status[0] >= nmx) && (rn > tol))
      {
         status[0] = -1;
         break;
      }
   }
   for (i = 0; i < n24; i++) psi[i] *= rho0;
   rn *= rho0;
   if (status[0] < 0)
   {
      ifail[0] = -1;
      status[0] = nmx;
   }
   for (k = 0; k < nkv; k++) { free(phi[k]); free(chi[k]); }
   free(phi); free(chi); free(rho); free(a); free(c); free(b); free(rsd); free(wrk);
   return rn;
}
