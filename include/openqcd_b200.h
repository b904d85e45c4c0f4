/*
 * openqcd_b200.h -- C interface of the B200 (sm_100a) implementation of
 * openQCD-2.4.2's Wilson-Dirac operator and SAP+GCR solver path.
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements with the reference's names, prototypes and
 *     argument meaning (include/dirac.h, include/sw_term.h, include/sap.h,
 *     include/linsolv.h of the reference).  Spinor arguments are arrays in the
 *     reference's storage order (ipt order, even sites first, VOLUME
 *     elements); they may live in host memory (pageable or pinned) or in
 *     device memory.  The calls are synchronous.  The gauge and SW fields
 *     these operators use are the library's device copies, loaded with
 *     b200_upload_ud()/b200_upload_swd() or generated on the device; they play
 *     the role of the reference's udfld()/swdfld() module globals.
 *
 *  2. b200_* management calls (geometry, parameters, field upload) and
 *     b200_dev_* calls on fields that stay on the device in the library's own
 *     block-major layout (used by solvers, tests and benchmarks).
 *
 * Error behaviour: the reference aborts the program on fatal errors
 * (modules/utils/error.c:119-200 error(), error_root()).  By default this
 * library does the same (message on stderr, exit(1)); after
 * b200_set_fatal(0) a failing call records the message, readable with
 * b200_last_error(), and returns (status -1 where the prototype returns int).
 * Recoverable solver failures use the reference's ifail/status codes.
 */
#ifndef OPENQCD_B200_H
#define OPENQCD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Types with the memory layout of the reference's include/su3.h:32-112,
 * defined here only when su3.h has not been included first. */
#ifndef SU3_H
typedef struct { float re, im; } complex;
typedef struct { double re, im; } complex_dble;
typedef struct { complex c1, c2, c3; } su3_vector;
typedef struct { complex_dble c1, c2, c3; } su3_vector_dble;
typedef struct { su3_vector c1, c2, c3, c4; } spinor;
typedef struct { su3_vector_dble c1, c2, c3, c4; } spinor_dble;
typedef struct { complex c11, c12, c13, c21, c22, c23, c31, c32, c33; } su3;
typedef struct { complex_dble c11, c12, c13, c21, c22, c23, c31, c32, c33; } su3_dble;
typedef struct { float u[36]; } pauli;
typedef struct { double u[36]; } pauli_dble;
typedef struct { double q[2]; } qflt;
typedef struct { qflt re, im; } complex_qflt;
#endif
#ifndef SW_TERM_H
typedef struct b200_pauli_wsp pauli_wsp_t;   /* unused here; kept for the prototype */
#endif

/* ------------------------------------------------------------------ state */

/* Select the CUDA device the library uses (default 0); call before
 * b200_geometry().  One process per GPU. */
int b200_set_device(int dev);

/* Lattice geometry.  L[4] lattice sizes (x0 = time), bs[4] the SAP block
 * size, which is also the tile of the device layout.  ipt (may be NULL) is
 * the reference's ipt[VOLUME] table (main/README.global:128-131); without it
 * only the b200_dev_* calls are available.  Replaces geometry()
 * (modules/lattice/geometry.c:273) for this library. */
int b200_geometry(const int L[4], const int bs[4], const int *ipt);

/* Domain decomposition along x0, as the reference's process grid with
 * NPROC0 > 1 (include/global.h:18-36): nproc0 ranks, this one at position
 * cpr0, each holding an L0 x L1 x L2 x L3 slab (L as given to b200_geometry,
 * the local lattice; the global time extent is nproc0 * L0).  Takes effect
 * at the next b200_geometry call; nproc0 = 1 switches it off.  L0 / bs0
 * must be even.  The transport is the caller's:
 *
 *  - xchg moves, per operator application, the x0-faces: send_dn (this
 *    rank's first time plane) to rank cpr0 - 1, where it arrives in
 *    recv_up, and send_up (the last plane) to rank cpr0 + 1, arriving in
 *    recv_dn (periodic in the rank index).  All four are device buffers of
 *    the library, `bytes` long.  The send buffers are written by work
 *    already enqueued on `stream` (a cudaStream_t); work the library
 *    enqueues on it after the call returns reads the receive buffers, so
 *    the callback either enqueues the transfers on that stream (NCCL) or
 *    synchronises it, copies, and returns when the data are in place.
 *  - gather is an all-gather of n doubles from every rank into out[nproc0 *
 *    n] (rank-major, host memory), used for the global sums, which every
 *    rank then adds in rank order in double-double (the reference's
 *    global_qsum, modules/utils/qsum.c:389).
 *
 * Available with it: the Dirac operators (device and drop-in entry
 * points), gauge and SW uploads/downloads, the SW term from the links,
 * apply_sw, the SAP cycle, sap_gcr, fgcr on device fields, the CG solvers
 * and the BLAS-1 reductions on device fields.  Not available (an error):
 * deflation, batched solves, the learned preconditioner, field files and
 * the plaquette, the allocation-free entry point.  Returns 0 or -1. */
typedef int (*b200_dd_exchange_fn)(void *send_dn, void *send_up, void *recv_up, void *recv_dn, size_t bytes,
                                   void *stream, void *user);
typedef int (*b200_dd_allgather_fn)(const double *in, double *out, int n, void *user);
int b200_dd_setup(int nproc0, int cpr0, b200_dd_exchange_fn xchg, b200_dd_allgather_fn gather, void *user);
/* The exchange buffers (send_dn, send_up, recv_up, recv_dn) and their size,
 * and the number of exchanges so far; returns nproc0. */
int b200_dd_info(void **bufs, size_t *bytes, long long *nexchange);
/* The global sum the reductions use: n (hi, lo) double-double pairs of this
 * rank (in[2k], in[2k+1]) summed over the ranks in rank order with TwoSum,
 * the same on every rank, into out (host code only, no device work). */
int b200_dd_global_sum(const double *in, double *out, int n);

/* Parameter data base: the values the reference reads from
 * set_lat_parms (modules/flags/lat_parms.c:216, csw), set_bc_parms (:516,
 * only type 3 = periodic gauge / antiperiodic quark fields is supported),
 * set_sw_parms (:920, m0), set_tm_parms (:963, eoflg) and set_sap_parms
 * (modules/flags/sap_parms.c:112). */
int b200_set_lat_parms(double csw);
/* the SW type isw of set_lat_parms (lat_parms.c:216): 0 traditional, 1
 * exponential form c exp{[csw/(4+m0)] (i/4) sigma F} (sw_term.c:46-49) */
int b200_set_sw_type(int isw);
int b200_set_bc_parms(int type);
/* The spatial phase angles theta[0..2] of set_bc_parms (lat_parms.c:516):
 * gauge fields made on the device (b200_random_ud) or read by import_cnfg
 * get the phase of set_ud_phase (modules/uflds/uflds.c:249-355), U(x,k)
 * times exp(i theta[k-1]/N[k]) besides the sign of the time links at
 * x0 = N0-1, and export_cnfg takes it off again; a field loaded with
 * b200_upload_ud is used as given (the caller has set its phase).  Default
 * 0; set it before the field is made or read. */
int b200_set_bc_theta(const double theta[3]);
int b200_set_sw_parms(double m0);
int b200_set_tm_parms(int eoflg);
int b200_set_sap_parms(const int bs[4], int isolv, int nmr, int ncy);

/* Gauge field in the reference's layout (udfld(), 4*VOLUME su3_dble, 8 links
 * per odd site, boundary phase already applied: modules/uflds/uflds.c:150,
 * :338).  Upload refreshes the FP32 copy (assign_ud2u, uflds.c:479). */
int b200_upload_ud(const su3_dble *ud);
int b200_download_ud(su3_dble *ud);

/* SW field in the reference's layout (swdfld(), 2*VOLUME pauli_dble, NOT
 * inverted, i.e. after sw_term(NO_PTS)).  Upload also forms the inverses
 * and FP32 copies (sw_term(ODD_PTS)/assign_swd2sw equivalents).  Returns 0,
 * or a bit mask of unsafe inversions (1 even, 2 odd sites; the reference's
 * Frobenius-condition criterion, pauli_dble.c:55-59). */
int b200_upload_swd(const pauli_dble *swd);
/* which = 0: the SW field, 1: its inverse on all sites (mu = 0). */
int b200_download_swd(pauli_dble *swd, int which);

/* sw_term(NO_PTS) (modules/sw_term/sw_term.c:399) on the device, from the
 * device gauge field; same return value as b200_upload_swd(). */
int b200_sw_term(void);

/* Test gauge field on the device: U = exp(eps X) per link, X drawn like the
 * reference's random_alg() (modules/linalg/liealg.c:289), antiperiodic
 * time boundary sign applied as set_ud_phase() does. */
int b200_random_ud(double eps, unsigned long long seed);

/* Page-locked host memory for reference-layout arrays (fast host<->device
 * transfers in the drop-in calls). */
void *b200_host_alloc(size_t bytes);
void b200_host_free(void *p);
/* Device-memory buffer of the given size, and a copy between any two
 * host/device addresses (cudaMemcpyDefault semantics), ordered on the
 * library's stream and complete when the call returns. */
void *b200_dev_alloc(size_t bytes);
int b200_memcpy(void *dst, const void *src, size_t bytes);

const char *b200_last_error(void);
/* Forget the recorded message (calls of void prototypes are checked by
 * clearing it before and reading it after). */
void b200_clear_error(void);
void b200_set_fatal(int on);
/* Wait for the library's stream; fails when a kernel gave up one of its
 * bounded waits for bulk copies (the flag is cleared by the call). */
int b200_sync(void);
int b200_volume(void);
/* No counterpart in the reference.  Self-check of that failure path: one CTA
 * waits, with at most `limit` polls (1 .. 2^22), on an mbarrier that nothing
 * completes, records the error and returns with nothing in flight.  Returns
 * -1 with the bounded-wait message when the path works; the context stays
 * usable. */
int b200_selfcheck_bounded_wait(int limit);

/* --------------------------------------- drop-in operators (dirac.h:24-52) */
/* Dw_dble.c:1377 */ void Dw_dble(double mu, spinor_dble *s, spinor_dble *r);
/* Dw_dble.c:1507 */ void Dwee_dble(double mu, spinor_dble *s, spinor_dble *r);
/* Dw_dble.c:1565 */ void Dwoo_dble(double mu, spinor_dble *s, spinor_dble *r);
/* Dw_dble.c:1627 */ void Dwoe_dble(spinor_dble *s, spinor_dble *r);
/* Dw_dble.c:1705 */ void Dweo_dble(spinor_dble *s, spinor_dble *r);
/* Dw_dble.c:1792 */ void Dwhat_dble(double mu, spinor_dble *s, spinor_dble *r);
/* Dw.c:973  */ void Dw(float mu, spinor *s, spinor *r);
/* Dw.c:1101 */ void Dwee(float mu, spinor *s, spinor *r);
/* Dw.c:1155 */ void Dwoo(float mu, spinor *s, spinor *r);
/* Dw.c:1213 */ void Dwoe(spinor *s, spinor *r);
/* Dw.c:1291 */ void Dweo(spinor *s, spinor *r);
/* Dw.c:1378 */ void Dwhat(float mu, spinor *s, spinor *r);

/* ------------------------------------ drop-in SW term (sw_term.h:37-56) */
/* pauli_dble.c:1840 */ void apply_sw_dble(int vol, double mu, pauli_dble *m, spinor_dble *s, spinor_dble *r);
/* pauli.c:1107      */ void apply_sw(int vol, float mu, pauli *m, spinor *s, spinor *r);
/* pauli_dble.c:1860 */ int apply_swinv_dble(int vol, double mu, pauli_dble *m, spinor_dble *s,
                                              pauli_wsp_t *pwsp, spinor_dble *r);

/* ------------------------------------------ drop-in solvers (sap.h:23-34) */
/* sap.c:720: one SAP cycle on single-precision fields psi, rho */
void sap(float mu, int isolv, int nmr, spinor *psi, spinor *rho);
/* sap_gcr.c:140: SAP-preconditioned flexible GCR; same ifail/status codes */
double sap_gcr(int nkv, int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi,
               int *ifail, int *status);

/* ------------------------------- drop-in BLAS-1 (linalg.h, salg*.c) */
/* vol sites; with icom & 0x2 the fields span vol sites per thread of the
 * caller's NTHREAD threads (b200_set_nthread, default 1); icom & 0x1 (MPI
 * sum) is a no-op here.  Arrays in host or device memory. */
int b200_set_nthread(int n);
/* salg_dble.c:2611 */ complex_qflt spinor_prod_dble(int vol, int icom, spinor_dble *s, spinor_dble *r);
/* salg_dble.c      */ qflt spinor_prod_re_dble(int vol, int icom, spinor_dble *s, spinor_dble *r);
/* salg_dble.c:2729 */ qflt norm_square_dble(int vol, int icom, spinor_dble *s);
/* salg_dble.c      */ void mulc_spinor_add_dble(int vol, int icom, spinor_dble *s, spinor_dble *r, complex_dble z);
/* salg_dble.c      */ void mulr_spinor_add_dble(int vol, int icom, spinor_dble *s, spinor_dble *r, double c);
/* salg_dble.c      */ void scale_dble(int vol, int icom, double c, spinor_dble *s);
/* salg_dble.c      */ double normalize_dble(int vol, int icom, spinor_dble *s);
/* salg.c:1223 */ complex spinor_prod(int vol, int icom, spinor *s, spinor *r);
/* salg.c      */ float spinor_prod_re(int vol, int icom, spinor *s, spinor *r);
/* salg.c:1289 */ float norm_square(int vol, int icom, spinor *s);
/* salg.c:1319 */ void mulc_spinor_add(int vol, int icom, spinor *s, spinor *r, complex z);
/* salg.c      */ void mulr_spinor_add(int vol, int icom, spinor *s, spinor *r, float c);
/* salg.c      */ void scale(int vol, int icom, float c, spinor *s);
/* salg.c:1415 */ float normalize(int vol, int icom, spinor *s);

/* fgcr.c:215: flexible GCR with the caller's operator Dop and
 * preconditioner Mop (called back with the caller's own arrays, which Dop
 * and Mop must be able to act on).  vol and the workspaces ws[2*nkv+1],
 * wsd[1] as in the reference (vol per thread, see b200_set_nthread). */
double fgcr(int vol, void (*Dop)(spinor_dble *s, spinor_dble *r), void (*Mop)(int k, spinor *rho, spinor *phi, spinor *chi),
            spinor **ws, spinor_dble **wsd, int nkv, int nmx, int istop, double res, spinor_dble *eta,
            spinor_dble *psi, int *status);

/* Storage precision of the links and SW matrices read by the even-odd SAP
 * block solver (no reference counterpart): 32 (default) as the reference;
 * 16 reads FP16 copies of them, with FP32 work vectors and arithmetic. */
int b200_set_sap_prec(int bits);
/* Dw (FP32, twisted mass mu) on n device fields (no reference
 * counterpart): r[j] = Dw s[j], or r[j] = sub[j] - Dw s[j] when sub is not
 * NULL, the subtraction fused into the operator's store. */
int b200_dev_dirac_multi(int n, float mu, void *const *s, void *const *r, void *const *sub);
/* Start (on != 0) or stop profiler collection around a region of interest
 * (for ncu --profile-from-start off). */
int b200_profiler(int on);
/* on != 0 (default): when every link satisfies the SU(3) relation
 * row3 = conj(row1 x row2), with the sign flipped on the time links at
 * x0 = N0-1 (the antiperiodic phase), the FP32 Dirac operators and the
 * even-odd SAP solver (block solves and block-boundary hops) read FP32
 * links as their first two rows and rebuild the third (no reference
 * counterpart; 2/3 of the link bytes, results equal to FP32 rounding).
 * Links with spatial phases (theta != 0) fail the check and are read in
 * full. */
int b200_set_sap_link12(int on);
/* 1 when the FP32 operators read 12-real links for the current gauge field
 * (on, and every link passed the check), 0 when they read 18 reals. */
int b200_links12_active(void);
/* mode != 0 (default): the FP64 operators with an SW term (all but
 * Dwoe_dble and Dweo_dble) stage each tile's SW matrices in shared memory
 * with bulk asynchronous copies; 0 reads them directly.  Same arithmetic,
 * identical results.  Returns the previous mode (no reference
 * counterpart). */
int b200_set_dw_staged(int mode);
/* Traversal order of the blocks in the full-lattice operator kernels (no
 * reference counterpart; results do not depend on it, only how long a
 * block's face data wait in L2 between uses): 0 Morton order of the block
 * coordinates (default), 1 lexicographic with x0 slowest, 2 lexicographic
 * with x0 fastest, 3 columns along x0 in Morton order of the spatial block
 * coordinates, 4 slabs of two block rows along x0, Morton order inside.
 * Returns the previous kind.  b200_tune_block_order times Dw_dble on the
 * resident fields under each kind (ms[kind], if ms is not null: 5 floats),
 * keeps the fastest and returns it. */
int b200_set_block_order(int kind);
/* Fix the launch variant of the even-odd SAP block kernel for the current
 * block size (the index of the autotuner's candidate list, 0..3), so that
 * separate runs use the same arithmetic; -1 lets the autotuner choose again
 * (no reference counterpart). */
int b200_set_sap_variant(int variant);
/* Block-shape autotuner (no reference counterpart).  For each candidate
 * SAP block shape cand[4 i .. 4 i + 3] (i < ncand) that fits the lattice,
 * the resident gauge and SW fields are laid out again with it, and nsteps
 * steps of the SAP-preconditioned GCR (current isolv, nmr, ncy) on a
 * Gaussian source are timed: score[i] = ln(|eta| / |residual|) / seconds
 * (-1 for shapes that do not fit).  Ns > 0: the shape is also the DFL
 * block; every candidate gets an Ns-mode subspace (dfl_modes with the
 * current generation parameters, not timed) and the deflated solver's
 * steps are timed.  The best shape stays in force (the geometry and the SAP
 * parameters now use it; deflation must be set up again); returns its
 * index.  Needs the ipt[] of the geometry call. */
int b200_tune_block_shape(const int *cand, int ncand, int nsteps, double mu, int Ns, float *score);
int b200_tune_block_order(float *ms);
/* on != 0 (default): the SAP preconditioner's launch sequence (ncy cycles of
 * block solves and boundary updates with the copies around them) is
 * captured as a CUDA graph on its first use with a given set of fields and
 * parameters and replayed afterwards; 0 launches the kernels one by one
 * (and frees the cached graphs).  Returns the previous setting.
 * b200_graphs_cached: the number of executable graphs held (no reference
 * counterpart). */
int b200_set_cuda_graphs(int on);
/* on != 0 (default): Dw_dble and Dw on page-locked host arrays run as a
 * pipeline (copy in, operator, copy out of different parts of the lattice
 * overlap) when the lattice has at least three block rows along x0 and can
 * be cut into at least three x0-slabs ("pieces", as thin as possible, at
 * least 131072 sites or a sixteenth of the lattice) that are contiguous
 * ranges of each parity half of the caller's storage order: planes for a
 * lexicographic order with x0 slowest, multiples of L0_TRD planes for
 * openQCD's ipt[].  The pieces are copied in and converted one by one; the operator
 * runs on a block row once the pieces holding it and its two neighbouring
 * planes are in; a piece is copied out once its rows are done.  Otherwise,
 * or with 0, the fields are copied whole.  Returns the previous setting.
 * b200_pipeline_slabs: the number of block rows of the pipeline,
 * b200_pipeline_pieces: the number of pieces (0: no pipeline);
 * b200_pipeline_used: 1 if the last Dw_dble or Dw call on host arrays ran
 * the pipeline, 0 if it copied the fields whole.  No reference
 * counterpart. */
int b200_set_pipeline(int on);
int b200_pipeline_slabs(void);
int b200_pipeline_pieces(void);
int b200_pipeline_used(void);
/* The numbers of pieces and block rows the pipeline would have for lattice
 * L, blocks bs and storage order ipt (host code only; needs no device and
 * no geometry call).  No reference counterpart. */
int b200_pipeline_plan(const int L[4], const int bs[4], const int *ipt, int *npieces, int *nslabs);
int b200_graphs_cached(void);
/* Launch variant of the SAP block kernel picked by the autotuner for the
 * current block size (prec 32, 16, or 12 for the 12-real links): index,
 * threads per block, time of one cycle's block sweeps in ms. */
int b200_sap_tuning(int prec, int *variant, int *threads, float *ms);

/* ------------------------------------------------------------- forces.h */
/* CG on the normal equations Dw(mu)^dag Dw(mu) psi = eta (cgne.c:452 with
 * the drivers of forces/tmcg.c): tmcg on all sites, tmcgeo with the even-odd
 * preconditioned Dwhat on the even sites (ifail -3: unsafe odd SW
 * inversion).  Reference-layout FP64 fields (host or device). */
/* tmcg.c:118 */ double tmcg(int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi,
                             int *ifail, int *status);
/* tmcg.c:206 */ double tmcgeo(int nmx, int istop, double res, double mu, spinor_dble *eta, spinor_dble *psi,
                               int *ifail, int *status);
/* the same on device fields in the library's layout (eo selects tmcgeo) */
double b200_dev_tmcg(int eo, int nmx, int istop, double res, double mu, const void *eta, void *psi, int *ifail,
                     int *status);
/* Multi-shift CG (linsolv/mscg.c:387 with the driver forces/tmcgm.c:100):
 * (Dwhat^dag Dwhat + mu[k]^2) psi[k] = eta on the even sites for nmu shifts
 * at once, each to its own relative residual res[k]; status = total CG
 * iterations including the final residual checks (ifail -1: not converged,
 * status nmx; -3: unsafe odd SW inversion).  Reference-layout FP64 fields
 * (host or device); the odd sites of psi[k] are kept. */
/* tmcgm.c:100 */ void tmcgm(int nmx, int istop, double *res, int nmu, double *mu, spinor_dble *eta,
                             spinor_dble **psi, int *ifail, int *status);
/* the same on device fields in the library's layout; returns 0, or -1 on an
 * error (message from b200_last_error) */
int b200_dev_tmcgm(int nmx, int istop, const double *res, int nmu, const double *mu, const void *eta,
                   void *const *psi, int *ifail, int *status);

/* ------------------------------------------------------ archive.h, uflds.h */
/* Files in openQCD's universal format (main/README.io), little-endian.  The
 * gauge field is read from / written to the device copy (the antiperiodic
 * phase is removed on export and applied on import); import requires the
 * file's lattice sizes to equal the geometry (no extension; mask unused)
 * and marks the SW term stale (call b200_sw_term()).  Spinor arrays are in
 * the reference layout (host or device). */
/* archive.c:804 */ void export_cnfg(char *out);
/* archive.c:878 */ void import_cnfg(char *in, int mask);
/* sarchive.c:424 */ void export_sfld(char *out, int eo, spinor_dble *sd);
/* sarchive.c:522 */ void import_sfld(char *in, int eo, spinor_dble *sd);
/* plaq_sum.c:161 plaq_sum_dble(1) of the device gauge field */
double b200_plaq_sum(void);

/* ------------------------------------------- deflation (dfl.h, little.h) */
/* Parameters of set_dfl_parms (modules/flags/dfl_parms.c:209; the DFL block
 * size must equal the geometry block size), set_dfl_pro_parms (:286) and
 * set_dfl_gen_parms (:360). */
int b200_set_dfl_parms(const int bs[4], int Ns);
int b200_set_dfl_pro_parms(int nkv, int nmx, double res, int nmx_gcr, double res_gcr);
int b200_set_dfl_gen_parms(double kappa, double mu, int ninv, int nmr, int ncy);
/* Ns * (number of DFL blocks): the length of a little vector. */
int b200_dfl_nv(void);
/* Phase timers of the deflation code (no reference counterpart): with on=1
 * the stream is synchronised at phase boundaries and seconds are summed into
 * six slots (SAP smoothing of the modes, block Gram-Schmidt, little operator
 * set-up, little solves, SAP in the preconditioner and inverse iteration,
 * the rest); out (6 doubles, may be NULL) receives the sums so far. */
int b200_dfl_profile(int on, double *out);
/* Device time (CUDA events) of n calls of one deflation kernel (no
 * reference counterpart): what = 0 restriction of an FP32 field, 1
 * prolongation, 2 Awhat_dble, 3 Aw_dble, 4 ltl_gcr on a random little
 * vector (its: GCR steps of the last solve), 5-7 the batched restriction,
 * prolongation and little solver on four right-hand sides. */
int b200_dfl_time(int what, int n, float *ms, int *its);
/* dfl_s2vd (dfl_subspace.c:83) and dfl_vd2s (:126) of nr fields at once
 * (1 <= nr <= 16; the batching has no reference counterpart): fields in the
 * reference layout, little vectors in the reference's block order, host or
 * device memory.  Four fields per pass run on the tensor cores (TF32
 * head/tail split products, FP32 accumulation, block sums in FP64), the rest
 * on the CUDA cores; the results are rounded to FP32 as the reference's. */
int b200_dfl_s2vd_multi(int nr, spinor *const *s, complex_dble *const *vd);
/* Awhat_dble (Aw_dble.c:361) of nr little vectors at once (1 <= nr <= 16;
 * the batching has no reference counterpart), after set_Awhat: the path of
 * the batched little solver, four vectors per pass with the preconditioned
 * hop matrices rounded to FP32 on the tensor cores (TF32 head/tail split
 * products, FP32 sums per matrix, FP64 across matrices), the rest in FP64.
 * Only the even blocks of w are written, as by Awhat_dble. */
int b200_Awhat_dble_multi(int nr, complex_dble *const *v, complex_dble *const *w);
int b200_dfl_vd2s_multi(int nr, complex_dble *const *vd, spinor *const *s);
/* Basis vector l of every block as one global FP32 field, reference layout. */
int b200_dfl_set_basis(int l, const spinor *field);
int b200_dfl_get_basis(int l, spinor *field);
/* dfl_modes.c:423 */ void dfl_modes(int *ifail, int *status);
int b200_dev_dfl_modes(unsigned long long seed, int *ifail, int *status);
/* No reference counterpart.  The start fields of the next dfl_modes call
 * (Ns FP32 fields in the reference's storage order, one after another),
 * in place of the library's own random fields: with the fields the
 * reference draws (random_fields, dfl_modes.c:248) the two generate the
 * same subspace up to rounding.  Used once. */
int b200_dfl_set_start_fields(const spinor *fields);
/* dfl_subspace.c:171 */ void dfl_subspace(spinor **mds);
/* dfl_subspace.c:83  */ void dfl_s2vd(spinor *s, complex_dble *vd);
/* dfl_subspace.c:126 */ void dfl_vd2s(complex_dble *vd, spinor *s);
/* Aw_ops.c:186 */ void set_Aw(double mu);
/* Aw_ops.c:223 */ int set_Awhat(double mu);
/* Aw_dble.c:122 */ void Aw_dble(complex_dble *v, complex_dble *w);
/* Aw_dble.c:361 */ void Awhat_dble(complex_dble *v, complex_dble *w);
/* The even-odd pieces of the little operator (even blocks first in a
 * little vector; the untouched half of w is unchanged) and the FP32 little
 * operators (FP32 arithmetic on the FP32-rounded matrices). */
/* Aw_dble.c:202 */ void Aweeinv_dble(complex_dble *v, complex_dble *w);
/* Aw_dble.c:234 */ void Awooinv_dble(complex_dble *v, complex_dble *w);
/* Aw_dble.c:266 */ void Awoe_dble(complex_dble *v, complex_dble *w);
/* Aw_dble.c:306 */ void Aweo_dble(complex_dble *v, complex_dble *w);
/* Aw.c:122 */ void Aw(complex *v, complex *w);
/* Aw.c:361 */ void Awhat(complex *v, complex *w);
/* Aw.c:202-359, the FP32 even-odd pieces (after set_Awhat): w_e = Aee^-1 v_e,
 * w_o = Aoo^-1 v_o, w_o = Aoe v_e, w_e = w_e - Aeo v_o */
/* Aw.c:202 */ void Aweeinv(complex *v, complex *w);
/* Aw.c:234 */ void Awooinv(complex *v, complex *w);
/* Aw.c:266 */ void Awoe(complex *v, complex *w);
/* Aw.c:306 */ void Aweo(complex *v, complex *w);
/* Global-mode ("little-little") deflation of the even-odd little system:
 * the little modes are the modes of the last dfl_subspace()/dfl_modes()
 * call in the block basis; set_ltl_modes returns 1 if the little-little
 * operator is not safely invertible.  ltl_matrix points to its inverse
 * (host memory, Ns x Ns row-major) until the next set_ltl_modes. */
/* ltl_modes.c:286 */ int set_ltl_modes(void);
/* ltl_modes.c:301 */ complex_dble *ltl_matrix(void);
/* ltl_modes.c:307 */ void dfl_Lvd(complex_dble *vd);
/* ltl_modes.c:339 */ void dfl_LRvd(complex_dble *vd, complex_dble *wd);
/* ltl_modes.c:382 */ void dfl_RLvd(complex_dble *vd, complex_dble *wd);
/* ltl_modes.c:417 */ void dfl_Lv(complex *v);
/* ltl_gcr solves the little equation with the solver chosen by
 * b200_set_ltl_solver: 0 (default) the device GCR on the even-odd little
 * system (status[1] = 0), 1 the reference's algorithm, flexible FP64 GCR
 * (fgcr4vd.c) preconditioned by FP32 GCR (gcr4v.c) with global-mode
 * deflation (status[1] = the FP32 GCR's Krylov vectors).  The deflated
 * solvers (dfl_sap_gcr, dfl_sap_gcr2) use the same choice.  Returns the
 * previous choice (no reference counterpart). */
/* ltl_gcr.c:155 */ double ltl_gcr(double mu, complex_dble *eta, complex_dble *psi, int *ifail, int *status);
int b200_set_ltl_solver(int kind);
/* RHS-tile autotuner of the multi-right-hand-side restriction and
 * prolongation: one, two or four fields per pass on the CUDA cores, or four
 * fields on the tensor cores, chosen by timing on the first call with four
 * or more fields per geometry and deflation set-up.  tile[0] restriction,
 * tile[1] prolongation (fields per pass, 0: not tuned yet), tc[k] = 1 when
 * the four-field pass of k runs on the tensor cores; ms[0..3] and ms[4..7]
 * the times of four fields with the kinds (1, 2, 4 on the CUDA cores, 4 on
 * the tensor cores).  No reference counterpart. */
int b200_rhs_tiles(int tile[2], int tc[2], float ms[8]);
/* Fixes the RHS tiles of the current geometry and deflation set-up
 * (tile[k] in {1, 2, 4}, tc[k] for four fields on the tensor cores; tile[k]
 * = 0 hands k back to the autotuner).  No reference counterpart. */
int b200_set_rhs_tiles(const int tile[2], const int tc[2]);
/* Little mode l (nv complex floats) for a subspace uploaded as a basis with
 * b200_dfl_set_basis; dfl_subspace() and dfl_modes() set them themselves
 * (no reference counterpart). */
int b200_dfl_set_lmode(int l, const complex *v);
/* dfl_sap_gcr.c:353 */ double dfl_sap_gcr(int nkv, int nmx, int istop, double res, double mu, spinor_dble *eta,
                                           spinor_dble *psi, int *ifail, int *status);
/* dfl_sap_gcr.c:383 */ double dfl_sap_gcr2(int nkv, int nmx, int istop, double res, double mu, spinor_dble *eta,
                                            spinor_dble *psi, int *ifail, int *status);
/* Several right-hand sides solved together (no reference counterpart):
 * nrhs systems Dw(mu[r]) psi[r] = eta[r] on device fields in the library's
 * layout, each by the algorithm of sap_gcr (dfl = 0) or dfl_sap_gcr
 * (dfl = 1, same mu for all systems) with its own Krylov space and stopping
 * test; a system leaves the batch when it has converged.  With deflation
 * the restriction, little solve and prolongation of all systems run as
 * multi-right-hand-side kernels.  rho[r], ifail[r] and status[r] as in the
 * single-system solvers (status[nrhs + r]: average little-solver steps). */
int b200_dev_gcr_batch(int nrhs, int dfl, int nkv, int nmx, int istop, double res, const double *mu,
                       void *const *eta, void *const *psi, double *rho, int *ifail, int *status);
/* Free the solvers' cached work fields. */
int b200_release_workspace(void);
double b200_dev_dfl_sap_gcr(int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                            int *ifail, int *status);

/* --------------------------------------------- learned preconditioner */
/* A gauge-equivariant parallel-transport convolutional network (no
 * reference counterpart): three linear layers of 4 -> 8 -> 8 -> 4 colour-
 * triplet channels with complex weights per direction (self and the 8
 * hops), colour moved by the links only.  Weights are packed per layer as
 * [9][Cout][Cin] complex floats (re, im); b200_net_nweights() floats in
 * all.  Fields are FP32 device fields in the library's layout. */
int b200_net_nweights(void);
/* weights close to scale * identity plus small random couplings */
int b200_net_init(unsigned long long seed, float scale);
int b200_net_set_weights(const float *w);
int b200_net_get_weights(float *w);
/* out = M in; half != 0 uses the FP16-rounded weights (FP32 arithmetic) */
int b200_net_apply(const void *in, void *out, int half);
/* loss |M r - e|^2/|e|^2 of one pair and its gradient with respect to the
 * real and imaginary parts of the weights (packed like the weights) */
int b200_net_grad(const void *r, const void *e, double *loss, float *grad);
/* mean loss and mean gradient over npairs pairs (one minibatch), and one
 * Adam step with a given gradient: the two halves of a training step, for
 * data-parallel training where the ranks sum their gradients in between
 * (openqcd_b200.net_train_data_parallel) */
int b200_net_batch_grad(int npairs, void *const *r, void *const *e, double *loss, float *grad);
int b200_net_adam_step(const float *grad, float lr);
/* steps of Adam on minibatches of `batch` of the npairs (r, e) pairs,
 * on the device; loss_hist[step] = minibatch loss (may be NULL) */
int b200_net_train(int npairs, void *const *r, void *const *e, int steps, int batch, float lr,
                   unsigned long long seed, float *loss_hist);
/* training pairs from the plain solver: r Gaussian, e = Dw(mu)^-1 r */
int b200_net_make_pairs(int npairs, void *const *r, void *const *e, double mu, double res,
                        unsigned long long seed);
/* (residual, SAP-error) pairs: r Gaussian, e = Dw(mu)^-1 r - M_sap r, the
 * error that ncy SAP cycles from zero (current SAP parameters) leave */
int b200_net_make_sap_pairs(int npairs, void *const *r, void *const *e, double mu, double res,
                            unsigned long long seed);
/* preconditioner of sap_gcr: 0 SAP (default), 1 the network (SAP once a
 * step reduces the residual by less than 10 %), 2 the network followed by
 * SAP on its residual, 3 none, 4 SAP plus the network's correction
 * M_sap r + N r (a network trained on SAP-error pairs; SAP alone once a
 * step reduces the residual by less than 10 %) */
int b200_set_precond(int kind);

/* ------------------------------------ device-resident fields (own layout) */
/* prec = 64 (spinor_dble) or 32 (spinor).  Operator codes for
 * b200_dev_dirac: 0 Dw, 1 Dwee, 2 Dwoo, 3 Dwoe, 4 Dweo, 5 Dwhat. */
void *b200_dev_alloc_spinor(int prec);
void b200_dev_free(void *p);
/* Point source: zero except component (spin, colour) = 1 at site x (x[0]
 * time); the sources of the batched-solve workload. */
int b200_dev_point_source(int prec, void *f, const int x[4], int spin, int colour);
int b200_dev_random_spinor(int prec, void *f, double sigma, unsigned long long seed);
int b200_dev_from_ref(int prec, const void *q, void *f);
int b200_dev_to_ref(int prec, const void *f, void *q);
int b200_dev_dirac(int prec, int op, double mu, const void *s, void *r);
int b200_dev_sap(float mu, int isolv, int nmr, int ncy, void *psi, void *rho);
double b200_dev_sap_gcr(int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                        int *ifail, int *status);
double b200_dev_norm2(int prec, const void *f);

/* No counterpart in the reference.  Dwhat_dble (even-odd preconditioned FP64
 * operator, as b200_dev_dirac(64, 5, ...)) on device-resident fields in the
 * library's layout, without allocating anything: for callers that cannot let
 * a library call cudaMalloc -- applications whose own memory pool already
 * holds the device (a further cudaMalloc would fail or fragment it) and
 * services whose device footprint must stay fixed after start-up.  The
 * odd-site intermediate lives in a static device array of 12 MiB (held by
 * every GPU that loads the library until exit), so lattices larger than
 * 131072 sites are rejected with an error.  The first call on a device looks
 * up the array's device address; make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * streams or host threads) race.  Returns when the result is complete. */
int b200_dev_Dwhat_dble_noalloc(double mu, const void *s, void *r);
/* Device time of n back-to-back operator applications, measured with CUDA
 * events on the library's stream; returns total milliseconds in *ms. */
int b200_dev_time_dirac(int prec, int op, double mu, const void *s, void *r, int n, float *ms);
/* Device time of n repetitions of ncy SAP cycles on FP32 device fields. */
int b200_dev_time_sap(float mu, int isolv, int nmr, int ncy, void *psi, void *rho, int n, float *ms);
/* Same, for Dw_dble through the drop-in entry point with host arrays in the
 * reference layout (host->device copy, layout conversion, operator,
 * conversion back, device->host copy), timed with events around each call. */
int b200_time_Dw_dble_host(double mu, spinor_dble *s, spinor_dble *r, int n, float *ms);

#ifdef __cplusplus
}
#endif
#endif
