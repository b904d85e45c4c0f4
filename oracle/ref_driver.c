/*
 * Test-infrastructure driver around the REFERENCE library (the reference's
 * own modules compiled in place by oracle/build_ref.py).  It is the oracle:
 * only tests/, the smoke check and bench.py's CPU-baseline leg load it.
 *
 * It exposes flat C entry points (prefix ref_) that Python reaches through
 * ctypes.  Spinor, gauge and SW arrays cross this boundary as plain doubles or
 * floats in the reference's own storage order:
 *   spinor_dble[VOLUME]   ipt order, even sites first (main/README.global)
 *   su3_dble[4*VOLUME]    8 links per odd site (main/README.global:229-262)
 *   pauli_dble[2*VOLUME]  upper/lower 6x6 at sw[2ix], sw[2ix+1]
 *                         (modules/sw_term/sw_term.c:42-44)
 *
 * Field generation follows the workload recipe: every link is exp(eps*X)
 * with X drawn by random_alg() (modules/linalg/liealg.c:289) and the SU(3)
 * exponential expXsu3() (modules/su3fcts/chexp.c:878); then set_bc() and
 * set_ud_phase() (modules/uflds/uflds.c:338) apply the boundary conditions.
 */
#define MAIN_PROGRAM

#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <omp.h>
#include "mpi.h"
#include "su3.h"
#include "flags.h"
#include "random.h"
#include "su3fcts.h"
#include "utils.h"
#include "lattice.h"
#include "uflds.h"
#include "sflds.h"
#include "linalg.h"
#include "sw_term.h"
#include "block.h"
#include "dirac.h"
#include "sap.h"
#include "linsolv.h"
#include "global.h"

static int initialised = 0;
static int nws = 0, nwsd = 0;

/* The OpenMP runtime is shared by every copy of the reference loaded into a
 * process, while each copy assumes exactly NTHREAD threads
 * (modules/utils/utils.c:195), so every entry point pins the team size. */
#define ENTER() omp_set_num_threads(NTHREAD)

int ref_volume(void) { ENTER(); return VOLUME; }
int ref_nthread(void) { ENTER(); return NTHREAD; }

void ref_dims(int *L)
{
   ENTER();
   L[0] = L0; L[1] = L1; L[2] = L2; L[3] = L3;
}

static void need_ws(int n, int nd)
{
   if (n > nws) { alloc_ws(n); nws = n; }
   if (nd > nwsd) { alloc_wsd(nd); nwsd = nd; }
}

static double bc_theta[3] = {0.0, 0.0, 0.0};

/* The spatial phase angles theta of set_bc_parms (flags/lat_parms.c), taken
 * by the first ref_init call of the process; set_ud_phase() then multiplies
 * U(x,k) by exp(i theta[k-1]/N[k]) (modules/uflds/uflds.c:249-300). */
void ref_set_theta(double t0, double t1, double t2)
{
   bc_theta[0] = t0; bc_theta[1] = t1; bc_theta[2] = t2;
}

/* Geometry, parameter data base and random-number generator.  Must be called
 * once per process before any other ref_ function. */
void ref_init_isw(int bc, int seed, double csw, double m0, int eoflg, int isw)
{
   ENTER();
   int provided;
   double phi[2] = {0.0, 0.0}, phip[2] = {0.0, 0.0}, theta[3];
   theta[0] = bc_theta[0]; theta[1] = bc_theta[1]; theta[2] = bc_theta[2];

   if (!initialised)
   {
      MPI_Init_thread(NULL, NULL, MPI_THREAD_FUNNELED, &provided);
      omp_set_num_threads(NTHREAD);
      omp_set_dynamic(0);
      set_lat_parms(6.0, 1.0, 0, NULL, isw, csw);
      set_bc_parms(bc, 1.0, 1.0, 1.0, 1.0, phi, phip, theta);
      start_ranlux(0, seed);
      geometry();
      chexp_init();
      initialised = 1;
   }
   set_sw_parms(m0);
   set_tm_parms(eoflg);
   need_ws(40, 8);
}

void ref_init(int bc, int seed, double csw, double m0, int eoflg)
{
   ref_init_isw(bc, seed, csw, m0, eoflg, 0);
}

void ref_set_sw_parms(double m0) { ENTER(); set_sw_parms(m0); set_flags(ERASED_SWD); }
void ref_set_tm_parms(int eoflg) { ENTER(); set_tm_parms(eoflg); }

void ref_set_sap_parms(int b0, int b1, int b2, int b3, int isolv, int nmr, int ncy)
{
   ENTER();
   int bs[4];
   bs[0] = b0; bs[1] = b1; bs[2] = b2; bs[3] = b3;
   set_sap_parms(bs, isolv, nmr, ncy);
}

/* Links U = exp(eps*X)*1 on all 4*VOLUME link slots, then boundary
 * conditions and phase.  Reseeds the generator first. */
void ref_gen_links(double eps, int seed)
{
   ENTER();
   int i;
   su3_dble *ud;
   su3_alg_dble X __attribute__((aligned(64)));

   start_ranlux(0, seed);
   ud = udfld();
   for (i = 0; i < 4 * VOLUME; i++)
   {
      memset(ud + i, 0, sizeof(su3_dble));
      ud[i].c11.re = 1.0;
      ud[i].c22.re = 1.0;
      ud[i].c33.re = 1.0;
      random_alg(1, 0, &X);
      expXsu3(eps, &X, ud + i);
   }
   set_flags(UPDATED_UD);
   set_flags(UNSET_UD_PHASE);
   set_bc();
   set_ud_phase();
}

void ref_random_ud(int seed)
{
   ENTER();
   start_ranlux(0, seed);
   random_ud();
   set_ud_phase();
}

void ref_get_ipt(int *out)
{
   ENTER();
   memcpy(out, ipt, VOLUME * sizeof(int));
}

void ref_get_ud(double *out) { ENTER(); memcpy(out, udfld(), 4 * VOLUME * sizeof(su3_dble)); }

void ref_set_ud(const double *in)
{
   ENTER();
   memcpy(udfld(), in, 4 * VOLUME * sizeof(su3_dble));
   set_flags(UPDATED_UD);
}

/* sw_term(set) with set = 0 (NO_PTS), 1 (EVEN_PTS), 2 (ODD_PTS),
 * 3 (ALL_PTS): compute the SW field and invert it on the given points
 * (modules/sw_term/sw_term.c:399).  Returns the reference's ifail. */
int ref_sw_term(int set)
{
   ENTER();
   ptset_t s = NO_PTS;
   if (set == 1) s = EVEN_PTS;
   else if (set == 2) s = ODD_PTS;
   else if (set == 3) s = ALL_PTS;
   return sw_term(s);
}

void ref_get_swd(double *out) { ENTER(); memcpy(out, swdfld(), 2 * VOLUME * sizeof(pauli_dble)); }

void ref_random_sd(int seed, double sigma, double *out)
{
   ENTER();
   spinor_dble **wsd;
   start_ranlux(0, seed);
   wsd = reserve_wsd(1);
   random_sd(VOLUME_TRD, 2, wsd[0], sigma);
   memcpy(out, wsd[0], VOLUME * sizeof(spinor_dble));
   release_wsd();
}

/* Double-precision operators: op = 0 Dw, 1 Dwee, 2 Dwoo, 3 Dwoe, 4 Dweo,
 * 5 Dwhat (modules/dirac/Dw_dble.c:1377-1889).  r is both read (Dweo
 * subtracts from it) and written. */
void ref_dirac_dble(int op, double mu, const double *s, double *r)
{
   ENTER();
   spinor_dble **wsd;
   wsd = reserve_wsd(2);
   memcpy(wsd[0], s, VOLUME * sizeof(spinor_dble));
   memcpy(wsd[1], r, VOLUME * sizeof(spinor_dble));
   switch (op)
   {
   case 0: Dw_dble(mu, wsd[0], wsd[1]); break;
   case 1: Dwee_dble(mu, wsd[0], wsd[1]); break;
   case 2: Dwoo_dble(mu, wsd[0], wsd[1]); break;
   case 3: Dwoe_dble(wsd[0], wsd[1]); break;
   case 4: Dweo_dble(wsd[0], wsd[1]); break;
   case 5: Dwhat_dble(mu, wsd[0], wsd[1]); break;
   default: break;
   }
   memcpy(r, wsd[1], VOLUME * sizeof(spinor_dble));
   release_wsd();
}

/* Single-precision twins (modules/dirac/Dw.c:973-1473).  The single-
 * precision gauge and SW fields are refreshed from the double-precision
 * ones first (assign_ud2u, assign_swd2sw). */
void ref_dirac(int op, float mu, const float *s, float *r)
{
   ENTER();
   spinor **ws;
   assign_ud2u();
   assign_swd2sw();
   ws = reserve_ws(2);
   memcpy(ws[0], s, VOLUME * sizeof(spinor));
   memcpy(ws[1], r, VOLUME * sizeof(spinor));
   switch (op)
   {
   case 0: Dw(mu, ws[0], ws[1]); break;
   case 1: Dwee(mu, ws[0], ws[1]); break;
   case 2: Dwoo(mu, ws[0], ws[1]); break;
   case 3: Dwoe(ws[0], ws[1]); break;
   case 4: Dweo(ws[0], ws[1]); break;
   case 5: Dwhat(mu, ws[0], ws[1]); break;
   default: break;
   }
   memcpy(r, ws[1], VOLUME * sizeof(spinor));
   release_ws();
}

/* One or more SAP cycles sap(mu,isolv,nmr,psi,rho) on single-precision
 * fields (modules/sap/sap.c:720), after the block-grid set-up sap_gcr()
 * performs (modules/sap/sap_gcr.c:150-200). */
int ref_sap(float mu, int isolv, int nmr, int ncy, float *psi, float *rho)
{
   ENTER();
   int nb, isw, n, ifail = 0;
   spinor **ws;

   blk_list(SAP_BLOCKS, &nb, &isw);
   if (nb == 0)
      alloc_bgr(SAP_BLOCKS);
   assign_ud2ubgr(SAP_BLOCKS);
   if (query_flags(SWD_UP2DATE) != 1 || query_flags(SWD_E_INVERTED) == 1 ||
       query_flags(SWD_O_INVERTED) == 1)
      sw_term(NO_PTS);
   ifail = assign_swd2swbgr(SAP_BLOCKS, isolv ? ODD_PTS : NO_PTS);

   ws = reserve_ws(2);
   memcpy(ws[0], psi, VOLUME * sizeof(spinor));
   memcpy(ws[1], rho, VOLUME * sizeof(spinor));
   for (n = 0; n < ncy; n++)
      sap(mu, isolv, nmr, ws[0], ws[1]);
   memcpy(psi, ws[0], VOLUME * sizeof(spinor));
   memcpy(rho, ws[1], VOLUME * sizeof(spinor));
   release_ws();
   return ifail;
}

/* The reference SAP+GCR solver (modules/sap/sap_gcr.c:140).  The SW term is
 * brought into the non-inverted state first, as the main programs do. */
double ref_sap_gcr(int nkv, int nmx, int istop, double res, double mu,
                   const double *eta, double *psi, int *ifail, int *status)
{
   ENTER();
   double rho;
   spinor_dble **wsd;

   need_ws(2 * nkv + 1 + 4, 8);
   wsd = reserve_wsd(2);
   memcpy(wsd[0], eta, VOLUME * sizeof(spinor_dble));
   rho = sap_gcr(nkv, nmx, istop, res, mu, wsd[0], wsd[1], ifail, status);
   memcpy(psi, wsd[1], VOLUME * sizeof(spinor_dble));
   release_wsd();
   return rho;
}

/* Wall-clock seconds for n applications of Dw_dble (op 0) or Dw (op 1) on a
 * Gaussian field, timed with the reference's MPI_Wtime. */
double ref_time_dirac(int op, double mu, int n)
{
   ENTER();
   int i;
   double t0, t1;
   spinor_dble **wsd;
   spinor **ws;

   if (op == 0)
   {
      wsd = reserve_wsd(2);
      random_sd(VOLUME_TRD, 2, wsd[0], 1.0);
      Dw_dble(mu, wsd[0], wsd[1]);
      t0 = MPI_Wtime();
      for (i = 0; i < n; i++)
         Dw_dble(mu, wsd[0], wsd[1]);
      t1 = MPI_Wtime();
      release_wsd();
   }
   else
   {
      assign_ud2u();
      assign_swd2sw();
      ws = reserve_ws(2);
      random_s(VOLUME_TRD, 2, ws[0], 1.0f);
      Dw((float)mu, ws[0], ws[1]);
      t0 = MPI_Wtime();
      for (i = 0; i < n; i++)
         Dw((float)mu, ws[0], ws[1]);
      t1 = MPI_Wtime();
      release_ws();
   }
   return t1 - t0;
}

/* The same timing of Dw_dble on the caller's source s (reference storage
 * order); the last application's result is copied to r. */
double ref_time_dirac_src(double mu, const double *s, double *r, int n)
{
   ENTER();
   int i;
   double t0, t1;
   spinor_dble **wsd;

   wsd = reserve_wsd(2);
   memcpy(wsd[0], s, VOLUME * sizeof(spinor_dble));
   Dw_dble(mu, wsd[0], wsd[1]);
   t0 = MPI_Wtime();
   for (i = 0; i < n; i++)
      Dw_dble(mu, wsd[0], wsd[1]);
   t1 = MPI_Wtime();
   memcpy(r, wsd[1], VOLUME * sizeof(spinor_dble));
   release_wsd();
   return t1 - t0;
}

/* Site-local SW term of the reference on caller arrays
 * (modules/sw_term/pauli_dble.c:1840, :1860; pauli.c:1107).  The reference's
 * AVX code needs 32-byte aligned matrices and spinors, so the caller's arrays
 * are copied into aligned buffers first. */
static void *aligned_copy(const void *p, size_t n)
{
   void *q = aligned_alloc(64, (n + 63) / 64 * 64);
   if (q != NULL && p != NULL)
      memcpy(q, p, n);
   return q;
}

void ref_apply_sw_dble(int vol, double mu, const double *m, const double *s, double *r)
{
   ENTER();
   size_t nm = (size_t)vol * 2 * sizeof(pauli_dble), ns = (size_t)vol * sizeof(spinor_dble);
   void *am = aligned_copy(m, nm), *as = aligned_copy(s, ns), *ar = aligned_copy(NULL, ns);
   apply_sw_dble(vol, mu, (pauli_dble *)am, (spinor_dble *)as, (spinor_dble *)ar);
   memcpy(r, ar, ns);
   free(am); free(as); free(ar);
}

void ref_apply_sw(int vol, float mu, const float *m, const float *s, float *r)
{
   ENTER();
   size_t nm = (size_t)vol * 2 * sizeof(pauli), ns = (size_t)vol * sizeof(spinor);
   void *am = aligned_copy(m, nm), *as = aligned_copy(s, ns), *ar = aligned_copy(NULL, ns);
   apply_sw(vol, mu, (pauli *)am, (spinor *)as, (spinor *)ar);
   memcpy(r, ar, ns);
   free(am); free(as); free(ar);
}

int ref_apply_swinv_dble(int vol, double mu, const double *m, const double *s, double *r)
{
   ENTER();
   int ifail;
   pauli_wsp_t *pwsp;
   size_t nm = (size_t)vol * 2 * sizeof(pauli_dble), ns = (size_t)vol * sizeof(spinor_dble);
   void *am = aligned_copy(m, nm), *as = aligned_copy(s, ns), *ar = aligned_copy(NULL, ns);
   pwsp = alloc_pauli_wsp();
   ifail = apply_swinv_dble(vol, mu, (pauli_dble *)am, (spinor_dble *)as, pwsp, (spinor_dble *)ar);
   free_pauli_wsp(pwsp);
   memcpy(r, ar, ns);
   free(am); free(as); free(ar);
   return ifail;
}

int ref_inv_pauli_dble(double mu, const double *m, double *im)
{
   ENTER();
   int ifail;
   pauli_wsp_t *pwsp;
   void *am = aligned_copy(m, sizeof(pauli_dble)), *ai = aligned_copy(NULL, sizeof(pauli_dble));
   pwsp = alloc_pauli_wsp();
   ifail = inv_pauli_dble(mu, (pauli_dble *)am, pwsp, (pauli_dble *)ai);
   free_pauli_wsp(pwsp);
   memcpy(im, ai, sizeof(pauli_dble));
   free(am); free(ai);
   return ifail;
}

/* Reference BLAS-1 on caller arrays of VOLUME sites (modules/linalg/
 * salg_dble.c:2611, :2729; salg.c:1223, :1289), called as the reference's
 * solvers do (vol = VOLUME_TRD, icom = 3). */
void ref_spinor_prod_dble(const double *s, const double *r, double *out)
{
   ENTER();
   complex_qflt z;
   spinor_dble **wsd = reserve_wsd(2);
   memcpy(wsd[0], s, VOLUME * sizeof(spinor_dble));
   memcpy(wsd[1], r, VOLUME * sizeof(spinor_dble));
   z = spinor_prod_dble(VOLUME_TRD, 3, wsd[0], wsd[1]);
   out[0] = z.re.q[0]; out[1] = z.re.q[1]; out[2] = z.im.q[0]; out[3] = z.im.q[1];
   release_wsd();
}

void ref_norm_square_dble(const double *s, double *out)
{
   ENTER();
   qflt q;
   spinor_dble **wsd = reserve_wsd(1);
   memcpy(wsd[0], s, VOLUME * sizeof(spinor_dble));
   q = norm_square_dble(VOLUME_TRD, 3, wsd[0]);
   out[0] = q.q[0]; out[1] = q.q[1];
   release_wsd();
}

void ref_spinor_prod(const float *s, const float *r, float *out)
{
   ENTER();
   complex z;
   spinor **ws = reserve_ws(2);
   memcpy(ws[0], s, VOLUME * sizeof(spinor));
   memcpy(ws[1], r, VOLUME * sizeof(spinor));
   z = spinor_prod(VOLUME_TRD, 3, ws[0], ws[1]);
   out[0] = z.re; out[1] = z.im;
   release_ws();
}

float ref_norm_square(const float *s)
{
   ENTER();
   float n;
   spinor **ws = reserve_ws(1);
   memcpy(ws[0], s, VOLUME * sizeof(spinor));
   n = norm_square(VOLUME_TRD, 3, ws[0]);
   release_ws();
   return n;
}

/* ------------------------------------------------------------ deflation */
/* Deflation parameters and workspaces (modules/flags/dfl_parms.c:209-380). */
#include "dfl.h"
#include "little.h"
#include "vflds.h"

static int dfl_nv = 0;

int ref_dfl_init(int b0, int b1, int b2, int b3, int Ns, int nkv, int nmx, double res, int nmx_gcr,
                 double res_gcr, double kappa, double mu, int ninv, int nmr, int ncy)
{
   ENTER();
   int bs[4], nb, isw;
   bs[0] = b0; bs[1] = b1; bs[2] = b2; bs[3] = b3;
   set_dfl_parms(bs, Ns);
   set_dfl_pro_parms(nkv, nmx, res, nmx_gcr, res_gcr);
   set_dfl_gen_parms(kappa, mu, ninv, nmr, ncy);
   if (dfl_nv != 0)
      return dfl_nv;
   alloc_wv(2 * nmx_gcr + 5);
   alloc_wvd(2 * nkv + 8);
   need_ws(Ns + 2 * 40 + 4, 8);
   blk_list(SAP_BLOCKS, &nb, &isw);
   if (nb == 0) alloc_bgr(SAP_BLOCKS);
   blk_list(DFL_BLOCKS, &nb, &isw);
   if (nb == 0) alloc_bgr(DFL_BLOCKS);
   blk_list(DFL_BLOCKS, &nb, &isw);
   dfl_nv = Ns * nb;
   return dfl_nv;
}

/* dfl_modes() (modules/dfl/dfl_modes.c:423): random fields, SAP smoothing,
 * deflated inverse iteration, dfl_subspace().  Returns ifail. */
int ref_dfl_modes(int seed, int *status)
{
   ENTER();
   int ifail = 0;
   start_ranlux(0, seed);
   dfl_modes(&ifail, status);
   return ifail;
}

/* The Ns start fields dfl_modes() draws after start_ranlux(0, seed)
 * (random_fields, modules/dfl/dfl_modes.c:248-264): every real component
 * uniform in [-0.5, 0.5), drawn with ranlxs by each OpenMP thread for its
 * VOLUME_TRD sites in turn, field after field.  Written one field after
 * another in ipt order. */
void ref_dfl_random_fields(int seed, int Ns, float *out)
{
   ENTER();
   int l;
   start_ranlux(0, seed);
   for (l = 0; l < Ns; l++)
   {
      float *f = out + (size_t)l * VOLUME * 24;
#pragma omp parallel
      {
         int k = omp_get_thread_num(), i, j;
         float *p = f + (size_t)k * VOLUME_TRD * 24;
         for (i = 0; i < VOLUME_TRD; i++, p += 24)
         {
            ranlxs(p, 24);
            for (j = 0; j < 24; j++)
               p[j] -= 0.5f;
         }
      }
   }
}

/* dfl_subspace() (modules/dfl/dfl_subspace.c:171) on Ns FP32 fields given
 * one after another in ipt order. */
void ref_dfl_subspace(int Ns, const float *modes)
{
   ENTER();
   int l;
   spinor **ws = reserve_ws(Ns);
   for (l = 0; l < Ns; l++)
      memcpy(ws[l], modes + (size_t)l * VOLUME * 24, VOLUME * sizeof(spinor));
   dfl_subspace(ws);
   release_ws();
}

/* Basis vector l of every DFL block, as one global field (ipt order). */
void ref_dfl_get_basis(int l, float *out)
{
   ENTER();
   int nb, isw, n;
   spinor **ws = reserve_ws(1);
   blk_list(DFL_BLOCKS, &nb, &isw);
   for (n = 0; n < nb; n++)
      assign_sblk2s(DFL_BLOCKS, n, ALL_PTS, l + 1, ws[0]);
   memcpy(out, ws[0], VOLUME * sizeof(spinor));
   release_ws();
}

static complex_dble *vd_copy(const double *v)
{
   complex_dble *p = aligned_alloc(64, ((size_t)dfl_nv * sizeof(complex_dble) + 63) / 64 * 64);
   if (v) memcpy(p, v, (size_t)dfl_nv * sizeof(complex_dble));
   else memset(p, 0, (size_t)dfl_nv * sizeof(complex_dble));
   return p;
}

void ref_dfl_s2vd(const float *s, double *vd)
{
   ENTER();
   spinor **ws = reserve_ws(1);
   complex_dble *v = vd_copy(NULL);
   memcpy(ws[0], s, VOLUME * sizeof(spinor));
   dfl_s2vd(ws[0], v);
   memcpy(vd, v, (size_t)dfl_nv * sizeof(complex_dble));
   free(v);
   release_ws();
}

void ref_dfl_vd2s(const double *vd, float *s)
{
   ENTER();
   spinor **ws = reserve_ws(1);
   complex_dble *v = vd_copy(vd);
   dfl_vd2s(v, ws[0]);
   memcpy(s, ws[0], VOLUME * sizeof(spinor));
   free(v);
   release_ws();
}

/* Little Dirac operator (modules/little/Aw_ops.c:186, :223; Aw_dble.c:122,
 * :361): which = 0 Aw_dble after set_Aw(mu), 1 Awhat_dble after
 * set_Awhat(mu) (even blocks only; w keeps its odd part). */
int ref_little(int which, double mu, const double *v, double *w)
{
   ENTER();
   int ifail = 0;
   complex_dble *a = vd_copy(v), *b = vd_copy(w);
   if (which == 0)
   {
      set_Aw(mu);
      Aw_dble(a, b);
   }
   else
   {
      ifail = set_Awhat(mu);
      if (which == 1) Awhat_dble(a, b);
      else if (which == 2) Aweeinv_dble(a, b);
      else if (which == 3) Awooinv_dble(a, b);
      else if (which == 4) Awoe_dble(a, b);
      else if (which == 5) Aweo_dble(a, b);
   }
   memcpy(w, b, (size_t)dfl_nv * sizeof(complex_dble));
   free(a);
   free(b);
   return ifail;
}

/* FP32 little operators (Aw.c:122, :361) on complex-float vectors, after
 * set_Aw(mu) / set_Awhat(mu): which = 0 Aw, 1 Awhat. */
int ref_little32(int which, double mu, const float *v, float *w)
{
   ENTER();
   int ifail = 0;
   size_t nb = (size_t)dfl_nv * sizeof(complex);
   complex *a = malloc(nb), *b = malloc(nb);
   memcpy(a, v, nb);
   memcpy(b, w, nb);
   if (which == 0)
   {
      set_Aw(mu);
      Aw(a, b);
   }
   else
   {
      ifail = set_Awhat(mu);
      if (which == 1) Awhat(a, b);
      else if (which == 2) Aweeinv(a, b);
      else if (which == 3) Awooinv(a, b);
      else if (which == 4) Awoe(a, b);
      else Aweo(a, b);
   }
   memcpy(w, b, nb);
   free(a);
   free(b);
   return ifail;
}

/* Little mode l of the last subspace: vflds()[Ns + l] (dfl_subspace.c:198). */
void ref_dfl_get_lmode(int l, float *out)
{
   ENTER();
   complex **vs = vflds();
   dfl_parms_t dp = dfl_parms();
   memcpy(out, vs[dp.Ns + l], (size_t)dfl_nv * sizeof(complex));
}

/* set_Awhat(mu) (which rebuilds the little modes, Aw_ops.c) and the inverse
 * little-little matrix (ltl_modes.c:301) into m (Ns*Ns complex). */
int ref_ltl_modes(double mu, double *m)
{
   ENTER();
   int ifail = set_Awhat(mu);
   dfl_parms_t dp = dfl_parms();
   memcpy(m, ltl_matrix(), (size_t)dp.Ns * dp.Ns * sizeof(complex_dble));
   return ifail;
}

/* ltl_modes.c projections on copies: which = 0 dfl_Lvd(v), 1 dfl_LRvd(v, w),
 * 2 dfl_RLvd(v, w); the little modes must be up to date (ref_ltl_modes). */
void ref_dfl_proj(int which, double *v, double *w)
{
   ENTER();
   complex_dble *a = vd_copy(v), *b = vd_copy(w);
   if (which == 0) dfl_Lvd(a);
   else if (which == 1) dfl_LRvd(a, b);
   else dfl_RLvd(a, b);
   memcpy(v, a, (size_t)dfl_nv * sizeof(complex_dble));
   memcpy(w, b, (size_t)dfl_nv * sizeof(complex_dble));
   free(a);
   free(b);
}

void ref_dfl_Lv(float *v)
{
   ENTER();
   size_t nb = (size_t)dfl_nv * sizeof(complex);
   complex *a = malloc(nb);
   memcpy(a, v, nb);
   dfl_Lv(a);
   memcpy(v, a, nb);
   free(a);
}

double ref_ltl_gcr(double mu, const double *eta, double *psi, int *ifail, int *status)
{
   ENTER();
   double rho;
   complex_dble *a = vd_copy(eta), *b = vd_copy(NULL);
   rho = ltl_gcr(mu, a, b, ifail, status);
   memcpy(psi, b, (size_t)dfl_nv * sizeof(complex_dble));
   free(a);
   free(b);
   return rho;
}

/* dfl_sap_gcr (modules/dfl/dfl_sap_gcr.c:353); status[3]. */
double ref_dfl_sap_gcr(int nkv, int nmx, int istop, double res, double mu, const double *eta, double *psi,
                       int *ifail, int *status)
{
   ENTER();
   double rho;
   spinor_dble **wsd;
   need_ws(2 * nkv + 4, 8);
   wsd = reserve_wsd(2);
   memcpy(wsd[0], eta, VOLUME * sizeof(spinor_dble));
   rho = dfl_sap_gcr(nkv, nmx, istop, res, mu, wsd[0], wsd[1], ifail, status);
   memcpy(psi, wsd[1], VOLUME * sizeof(spinor_dble));
   release_wsd();
   return rho;
}

/* Time one dfl_sap_gcr solve (wall clock, MPI_Wtime). */
double ref_time_dfl_sap_gcr(int nkv, int nmx, double res, double mu, const double *eta, int *status)
{
   ENTER();
   int ifail[1];
   double t0, t1;
   spinor_dble **wsd;
   need_ws(2 * nkv + 4, 8);
   wsd = reserve_wsd(2);
   memcpy(wsd[0], eta, VOLUME * sizeof(spinor_dble));
   t0 = MPI_Wtime();
   dfl_sap_gcr(nkv, nmx, 0, res, mu, wsd[0], wsd[1], ifail, status);
   t1 = MPI_Wtime();
   release_wsd();
   return t1 - t0;
}

double ref_time_sap_gcr(int nkv, int nmx, double res, double mu, const double *eta, int *status)
{
   ENTER();
   int ifail[1];
   double t0, t1;
   spinor_dble **wsd;
   need_ws(2 * nkv + 4, 8);
   wsd = reserve_wsd(2);
   memcpy(wsd[0], eta, VOLUME * sizeof(spinor_dble));
   t0 = MPI_Wtime();
   sap_gcr(nkv, nmx, 0, res, mu, wsd[0], wsd[1], ifail, status);
   t1 = MPI_Wtime();
   release_wsd();
   return t1 - t0;
}


/* ------------------------------------------------------------- archives */
/* export_cnfg / import_cnfg (modules/archive/archive.c:804, :878) and
 * export_sfld / import_sfld (modules/archive/sarchive.c:424, :522).  The
 * driver's gauge field carries the antiperiodic phase; the archive holds
 * the field without it, as the reference requires. */
#include "archive.h"

void ref_export_cnfg(const char *path)
{
   ENTER();
   unset_ud_phase();
   export_cnfg((char *)path);
   set_ud_phase();
}

void ref_import_cnfg(const char *path)
{
   ENTER();
   import_cnfg((char *)path, 0);
   set_ud_phase();
}

void ref_export_sfld(const char *path, int eo, const double *sd)
{
   ENTER();
   spinor_dble **wsd = reserve_wsd(1);
   memcpy(wsd[0], sd, VOLUME * sizeof(spinor_dble));
   export_sfld((char *)path, eo, wsd[0]);
   release_wsd();
}

void ref_import_sfld(const char *path, int eo, double *sd)
{
   ENTER();
   spinor_dble **wsd = reserve_wsd(1);
   memset(wsd[0], 0, VOLUME * sizeof(spinor_dble));
   import_sfld((char *)path, eo, wsd[0]);
   memcpy(sd, wsd[0], VOLUME * sizeof(spinor_dble));
   release_wsd();
}

double ref_plaq_sum(void)
{
   ENTER();
   return plaq_sum_dble(1);
}


/* ------------------------------------------------------------------ tmcg */
#include "forces.h"

double ref_tmcg(int eo, int nmx, int istop, double res, double mu, const double *eta, double *psi, int *ifail,
                int *status)
{
   ENTER();
   double rho;
   spinor_dble **wsd;
   need_ws(40, 8);
   wsd = reserve_wsd(2);
   memcpy(wsd[0], eta, VOLUME * sizeof(spinor_dble));
   memcpy(wsd[1], psi, VOLUME * sizeof(spinor_dble));
   if (eo)
      rho = tmcgeo(nmx, istop, res, mu, wsd[0], wsd[1], ifail, status);
   else
      rho = tmcg(nmx, istop, res, mu, wsd[0], wsd[1], ifail, status);
   memcpy(psi, wsd[1], VOLUME * sizeof(spinor_dble));
   release_wsd();
   return rho;
}


/* ----------------------------------------------------------------- tmcgm */
/* tmcgm (modules/forces/tmcgm.c:100) on copies of eta and of the nmu
 * solution fields psi[k] (psi: nmu consecutive fields) */
void ref_tmcgm(int nmx, int istop, const double *res, int nmu, const double *mu, const double *eta, double *psi,
               int *ifail, int *status)
{
   ENTER();
   int k;
   spinor_dble **wsd, *ps[64];
   need_ws(40, 2 * nmu + 8);
   wsd = reserve_wsd(1 + nmu);
   memcpy(wsd[0], eta, VOLUME * sizeof(spinor_dble));
   for (k = 0; k < nmu; k++)
   {
      ps[k] = wsd[1 + k];
      memcpy(ps[k], psi + (size_t)k * VOLUME * 24, VOLUME * sizeof(spinor_dble));
   }
   ifail[0] = 0;
   tmcgm(nmx, istop, (double *)res, nmu, (double *)mu, wsd[0], ps, ifail, status);
   for (k = 0; k < nmu; k++)
      memcpy(psi + (size_t)k * VOLUME * 24, ps[k], VOLUME * sizeof(spinor_dble));
   release_wsd();
}
