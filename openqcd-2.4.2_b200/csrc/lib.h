// Internal host-side declarations: the library context (geometry, resident
// fields, parameters) and the launchers each .cu file provides.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <functional>
#include <string>
#include <array>
#include <vector>
#include "qcd.cuh"

// Transport callbacks of the domain decomposition (declared for callers in
// include/openqcd_b200.h with the same signatures).
typedef int (*b200_dd_exchange_fn)(void *send_dn, void *send_up, void *recv_up, void *recv_dn, size_t bytes,
                                   void *stream, void *user);
typedef int (*b200_dd_allgather_fn)(const double *in, double *out, int n, void *user);

namespace qcd {

struct LtlRef;

// Domain decomposition along x0 (dd.cu): ranks, the caller's transport and
// the four face buffers (send to the rank below, send to the rank above,
// received from above, received from below).
struct DDState {
  int np = 1, rank = 0;
  b200_dd_exchange_fn xchg = nullptr;
  b200_dd_allgather_fn gather = nullptr;
  void *user = nullptr;
  void *buf[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t bytes = 0;
  long long nxchg = 0;
};

// The host pipeline of Dw / Dw_dble works on two plans of x0-slabs.  A
// Slab is one block row, the unit of the operator launches: device blocks
// [b0, b1) (lexicographic block order, x0 slowest), planes [t0, t1).  A
// Piece is the unit of the transfers and layout conversions: planes
// [t0, t1) whose sites are the storage indices [q0[p], q1[p]) of each
// parity half of the caller's storage order.
struct Slab {
  int b0, b1;
  int t0, t1;
};
struct Piece {
  int t0, t1;
  int q0[2], q1[2];
};

// Deflation state (the reference's DFL block grid, little operator and
// parameter sets dfl_parms, dfl_pro_parms, dfl_gen_parms).
struct DflState {
  bool ready = false, have_basis = false, gen_set = false;
  int Ns = 0, nb = 0, nv = 0;
  int nkv = 16, nmx = 256, nmx_gcr = 24;
  double res = 1e-2, res_gcr = 1e-2;
  double gen_kappa = 0.125, gen_mu = 0.0;
  int gen_ninv = 4, gen_nmr = 4, gen_ncy = 4;
  int *vd2lex = nullptr, *nbr = nullptr;
  int *faces = nullptr, *nfc = nullptr, fmax = 0;   // block-face site lists
  double2 *rpart = nullptr;                          // restriction partial sums [nb][2][Ns]
  double2 *bpart = nullptr;                          // the same for batched restriction
  int *kerr = nullptr;                               // error flag of bounded waits in kernels
  std::vector<void *> basis, modes;
  // start fields of the next dfl_modes (b200_dfl_set_start_fields), used
  // instead of the library's own random fields, once
  std::vector<void *> start;
  bool use_start = false;
  void **d_basis = nullptr;
  double2 *Ablk = nullptr, *Ainv = nullptr, *Ahop = nullptr, *Mhop = nullptr;
  float2 *Mhop32 = nullptr;     // FP32 copy of Mhop (the batched little hops on the tensor cores)
  // Ablk, Ainv, Mhop, Mhop32 of the further masses of a batched solve
  // (kept between calls, so that their addresses, part of the keys of the
  // captured little-solver iterations, repeat)
  std::vector<std::array<void *, 4>> xsets;
  bool aw_valid = false, awhat_valid = false;
  int awhat_fail = 0, aw_eo = 0;
  double aw_mu = 0.0;
  std::vector<double2 *> lv, lvd;
  double2 **lvtab = nullptr;    // device table of the little solver's Krylov vectors
  double2 *ldots = nullptr, *lpart = nullptr, *h_ldots = nullptr;
  // Cholesky QR of the modes: Gram matrices (per block, then the lattice
  // sum), inverse Cholesky factors, failure flag
  double2 *gram = nullptr, *tri = nullptr;
  int *gfail = nullptr;
  // little solver: 0 the device GCR, 1 the reference's algorithm (ltl_ref.cu)
  int ltl_kind = 0;
  int awhat_ver = 0;   // incremented whenever the preconditioned operator is rebuilt
  struct LtlRef *ltlref = nullptr;
  int lvtab_nkv = 0;
  // phase timers (seconds): 0 SAP smoothing of the modes, 1 block
  // Gram-Schmidt, 2 little operator set-up, 3 little solves, 4 SAP in the
  // deflated preconditioner and inverse iteration, 5 everything else
  bool profile = false;
  double prof[6] = {0, 0, 0, 0, 0, 0};
  double prof_t0 = 0.0;
};

// The learned preconditioner (net.cu): host master weights with Adam
// moments, device copies (FP32, adjoint layers, FP16-rounded), gradient
// accumulators and activation fields.
struct NetState {
  bool ready = false;
  std::vector<float> w[3], m[3], v[3];
  int t = 0;
  float2 *dev_w[3] = {nullptr, nullptr, nullptr}, *dev_wadj[3] = {nullptr, nullptr, nullptr};
  float2 *dev_w16[3] = {nullptr, nullptr, nullptr};
  double2 *dev_grad[3] = {nullptr, nullptr, nullptr};
  float2 *part = nullptr;
  std::vector<void *> f;
};

constexpr int SAP_MS = 8;   // systems per SAP launch of the batched solvers

// Everything the reference keeps in module-global state for this path:
// geometry (lattice/geometry.c), the gauge field (uflds/uflds.c udfld/ufld),
// the SW field (sw_term/swflds.c swdfld/swfld) and the parameter data base
// (flags/lat_parms.c, flags/sap_parms.c).
struct Ctx {
  bool ready = false;
  int dev = 0;
  Geom g{};                     // device pointers inside point to the tables below
  int *d_bcoord = nullptr, *d_lcoord = nullptr;
  int *sched = nullptr;         // block traversal order for full-lattice kernels
  int block_order = 0;          // its kind (set_block_order in layout.cu)
  // reference (openQCD) storage order, when the caller supplied its ipt[]
  bool have_ipt = false;
  int *d_dev2q = nullptr;       // [vol] device site (chunk*vbh+s) -> reference index ix
  int *d_q2dev = nullptr;       // [vol] its inverse
  int *d_link2q = nullptr;      // [4*vol] (device site, mu) -> slot in the reference ud[4V]
  std::vector<int> h_dev2q;
  std::vector<int> h_ipt;       // the caller's ipt[] (for a change of block shape)
  // slab and piece plans for pipelined host transfers (both empty if the
  // storage order has no contiguous pieces), the identity block list, the
  // copy streams
  std::vector<Slab> slab;
  std::vector<Piece> piece;
  int *d_ident = nullptr;
  cudaStream_t st_in = nullptr, st_out = nullptr, st_cv = nullptr;
  std::vector<cudaEvent_t> slab_ev;
  int pipeline = 1;             // pipelined host transfers of Dw / Dw_dble when possible
  int pipeline_used = 0;        // whether the last host Dw / Dw_dble call ran the pipeline

  // parameters
  double csw = 0.0, m0 = 0.0;
  int bc = 3, eoflg = 0;
  double theta[3] = {0.0, 0.0, 0.0};   // spatial phase angles of set_bc_parms
  int isw = 0;                  // SW term: 0 traditional, 1 exponential
  int isolv = 1, nmr = 4, ncy = 5;
  bool sap_set = false;

  // resident fields
  double2 *ud = nullptr;        // FP64 forward links
  float2 *u32 = nullptr;        // FP32 copy (assign_ud2u)
  double2 *swd = nullptr;       // FP64 SW term, not inverted
  double2 *swd_inv = nullptr;   // FP64 inverse (mu = 0) on all sites
  float4 *sw32 = nullptr;       // FP32 copies (assign_swd2sw)
  float4 *sw32_inv = nullptr;
  // FP16 copies for the SAP block solver in half-precision storage
  // (links as __half2 planes, Pauli matrices as 4-half uint2 planes)
  int sap_prec = 32;
  void *u16 = nullptr, *sw16 = nullptr, *sw16_inv = nullptr;
  bool h16_valid = false;
  // SAP block-kernel launch variant chosen by the autotuner, per storage
  // precision (0: FP32, 1: FP16), for the block size it was tuned on
  int sap_variant[3] = {0, 0, 0}, sap_tuned_vbh[3] = {0, 0, 0};
  float sap_tuned_ms[3] = {0.0f, 0.0f, 0.0f};
  // 12-real FP32 links for the SAP block solver (first two rows; the third
  // is rebuilt), used when every link passes the SU(3) check
  int sap_link12 = 1;
  void *u12 = nullptr;
  bool u12_valid = false, u12_ok = false;
  bool have_ud = false, have_sw = false, sw_inv_ok = false;
  int sw_inv_fail = 0;

  // scratch
  void *tmp64 = nullptr;        // one FP64 spinor field
  void *tmp32 = nullptr;        // one FP32 spinor field
  void *stage = nullptr;        // staging buffer for reference-layout transfers
  size_t stage_bytes = 0;
  double *red = nullptr;        // reduction partials
  double *red_out = nullptr;    // reduction results (device)
  double *h_red = nullptr;      // pinned host mirror of red_out
  int red_blocks = 0;
  cudaStream_t stream = nullptr;
  // error flag of bounded waits in the operator kernels: page-locked host
  // memory mapped into the device (h_kerr host view, d_kerr device view)
  int *h_kerr = nullptr, *d_kerr = nullptr;
  // FP64 operators with an SW term: SW matrices staged in shared memory by
  // bulk copies (1) or read directly (0)
  int dw_staged = 1;
  // repeated launch sequences (the SAP preconditioner) run as CUDA graphs,
  // on three library-owned FP32 fields (solution, residual, block scratch)
  int use_graphs = 1;
  void *sap_fld[3] = {nullptr, nullptr, nullptr};
  // the same for up to SAP_MS systems at once (sap_mfld_n consecutive
  // fields each)
  void *sap_mfld[3] = {nullptr, nullptr, nullptr};
  int sap_mfld_n = 0;
  int nthread = 1;              // the caller's NTHREAD, for icom & 0x2 in the BLAS drop-ins
  void *fstage[3] = {nullptr, nullptr, nullptr};   // staging of host operands
  size_t fstage_bytes[3] = {0, 0, 0};
  std::vector<void *> ws32, ws64;   // solver workspaces (reserve_ws / reserve_wsd)
  DflState dfl;
  NetState net;
  DDState dd;
  DDGeom ddg{0, 0, nullptr, nullptr};   // this rank's slab (x0off, N0) for the kernels
  // preconditioner of sap_gcr: 0 SAP, 1 network (SAP when the residual
  // stalls), 2 network then SAP on the remainder, 3 none
  int precond = 0;
};

inline bool dd_on(const Ctx &c) { return c.dd.np > 1; }

Ctx &ctx();
void set_error(const std::string &msg);
int fail(const std::string &msg);   // records msg, returns -1 (or aborts in fatal mode)

size_t spinor_bytes(const Ctx &c, int prec);   // prec 64 or 32

// dd.cu: domain decomposition along x0
int dd_buffers(Ctx &c);
int dd_exchange(Ctx &c, size_t bytes, cudaStream_t st);
// pack the half-spinor faces of field t (links u: FP64, FP32 or 12-real
// FP32 with l12), exchange them, and return in g the geometry with the
// received faces attached
int dd_faces(Ctx &c, int prec, const void *t, const void *u, int l12, cudaStream_t st, DDGeom &dg);
int dd_links_after_upload(Ctx &c, const void *qud, cudaStream_t st);
int dd_links_after_download(Ctx &c, void *qud, cudaStream_t st);
// n (hi, lo) pairs summed (or maxed) over the ranks, in rank order
int dd_global(Ctx &c, double *res, int n, bool is_max);
int dd_all(Ctx &c, int flag);                       // 1 when flag is non-zero on every rank
int dd_rank0(Ctx &c, int value);                    // rank 0's value on every rank
int dd_unsupported(const Ctx &c, const char *what);  // fails under domain decomposition

// dirac.cu
template <typename R>
int dirac_op(const Ctx &c, int op, R mu, const void *s, void *r, void *tmp, cudaStream_t st);

// Dw on all sites of the blocks blocks[0..nblk) (device block indices)
template <typename R>
int dirac_dw_blocks(const Ctx &c, R mu, const void *s, void *r, const int *blocks, int nblk, cudaStream_t st);

int dwhat_dble_halfscratch(const Ctx &c, double mu, const void *s, void *r, void *odd_scratch, cudaStream_t st);

// layout.cu
int geometry_init(Ctx &c, const int L[4], const int bs[4], const int *ipt);
constexpr int kBlockOrders = 5;
int set_block_order(Ctx &c, int kind);   // block traversal order of the full-lattice kernels
int spinor_from_ref(const Ctx &c, int prec, const void *q, void *dev, cudaStream_t st);   // q: reference AoS on device
// the same for the device sites [d0, d0 + n) only
int spinor_from_ref_range(const Ctx &c, int prec, const void *q, void *dev, int d0, int n, cudaStream_t st);
int spinor_to_ref_range(const Ctx &c, int prec, const void *dev, void *q, int d0, int n, cudaStream_t st);
int spinor_from_ref_piece(const Ctx &c, int prec, const void *q, void *dev, const Piece &pc, cudaStream_t st);
void pipeline_plan(const int L[4], const int bs[4], const int *ipt, std::vector<Piece> &piece,
                   std::vector<Slab> &slab);
int spinor_to_ref(const Ctx &c, int prec, const void *dev, void *q, cudaStream_t st);
int links_from_ref(Ctx &c, const void *qud, cudaStream_t st);                           // qud on device
int links_to_ref(const Ctx &c, void *qud, cudaStream_t st);
int pauli_from_ref(Ctx &c, const void *qsw, cudaStream_t st);                           // qsw on device
int pauli_to_ref(const Ctx &c, int which, void *qsw, cudaStream_t st);

// sw.cu
int sw_refresh_derived(Ctx &c, cudaStream_t st, bool inv_given = false);   // inverses + FP32 copies from swd
int sw_compute(Ctx &c, cudaStream_t st);             // SW term from the links (sw_term)
int links_refresh_f32(Ctx &c, cudaStream_t st);      // u32 from ud
int apply_sw_ref_layout(int prec, int vol, double mu, const void *m, const void *s, void *r, cudaStream_t st);
int apply_swinv_ref_layout(int vol, double mu, const void *m, const void *s, void *r, int *d_fail,
                           cudaStream_t st);

// fields.cu
// exp(i theta[k]/N[k+1]) of the spatial links (set_phase, uflds.c:249-276);
// true when an angle is non-zero
bool spatial_phases(const Ctx &c, double pr[3], double pi[3]);
int gen_links(Ctx &c, double eps, uint64_t seed, cudaStream_t st);
int gen_spinor(const Ctx &c, int prec, void *dev, double sigma, uint64_t seed, cudaStream_t st);

// graph.cu: run launch() captured as a CUDA graph, replayed while key
// (the bytes of everything the launches depend on) repeats
int graph_run(Ctx &c, const void *key, size_t keylen, cudaStream_t st, const std::function<int()> &launch);
void graphs_release();
size_t graphs_cached();

// linalg.cu : BLAS-1 on device-layout spinor fields.  "n" = number of sites
// counted from the start of the field (vol for full fields, volh for even).
// Reductions accumulate in double per thread and in double-double across
// blocks, deterministically.
enum { PAR_ALL = 2, PAR_EVEN = 0, PAR_ODD = 1 };
int la_norm2(Ctx &c, int prec, const void *x, int par, double *res_dd);                 // |x|^2 -> (hi,lo)
int la_dot(Ctx &c, int prec, const void *x, const void *y, int par, double *res);       // (x,y) -> re,im (dd each)
int la_unorm(Ctx &c, int prec, const void *x, int par, double *res);                    // max site norm
int la_xr_norm2(Ctx &c, void *x, void *r, const void *p, const void *ap, double a, int par,
                double *res_dd);                                 // FP64: x += a p, r -= a ap, |r|^2
int la_mulg5_norm2(Ctx &c, void *x, int par, double *res_dd);    // FP64: x = g5 x, |x|^2
void la_zero(const Ctx &c, int prec, void *x, int par, cudaStream_t st);
void la_copy(const Ctx &c, int prec_in, const void *x, int prec_out, void *y, int par, cudaStream_t st);
void la_scale(const Ctx &c, int prec, void *x, double a, int par, cudaStream_t st);
void la_axpy(const Ctx &c, int prec, void *y, double are, double aim, const void *x, int par, cudaStream_t st);  // y += a x
void la_diff(const Ctx &c, int prec, const void *x, void *y, int par, cudaStream_t st);  // y = x - y
void la_add_s2sd(const Ctx &c, const void *s32, void *sd, int par, cudaStream_t st);    // sd += s
void la_diff_sd2s(const Ctx &c, const void *ad, const void *bd, void *r32, int par, cudaStream_t st);  // r = a - b

// blas.cu: layout-agnostic BLAS-1 on device-accessible arrays of nsite
// sites in the reference's order (24 reals per site)
int flat_scratch(Ctx &c, double **scratch, double **out);
int flat_dot(Ctx &c, int prec, const void *x, const void *y, size_t nsite, double *res_dd, double *scratch,
             double *out_dev);
int flat_norm2(Ctx &c, int prec, const void *x, size_t nsite, double *res_dd, double *scratch, double *out_dev);
int flat_umax(Ctx &c, int prec, const void *x, size_t nsite, double *res, double *scratch, double *out_dev);
void flat_axpy(Ctx &c, int prec, void *y, const void *x, size_t nsite, double ar, double ai);
void flat_scale(Ctx &c, int prec, void *y, size_t nsite, double a);
void flat_zero(Ctx &c, int prec, void *y, size_t nsite);
void flat_copy(Ctx &c, int pin, const void *x, int pout, void *y, size_t nsite);
void flat_add_s2sd(Ctx &c, const void *s, void *sd, size_t nsite);
void flat_diff_sd2s(Ctx &c, const void *a, const void *b, void *r, size_t nsite);
void flat_diff(Ctx &c, int prec, const void *x, void *y, size_t nsite);
// y = sum over l = 0..n-1 of (cre[l] + i cim[l]) x[l], FP32 fields, one pass
// per 16 terms
void la_lincomb32(const Ctx &c, void *y, int n, const float *cre, const float *cim, void *const *x,
                  cudaStream_t st);

// solver.cu: the GCR recursion over an abstract set of FP32/FP64 field
// operations, so the same code serves device-layout fields (sap_gcr) and
// caller arrays (the generic fgcr drop-in).
struct cplxf { float re, im; };
struct KrylovOps {
  std::function<double(const void *, int)> res32;                 // get_res (fgcr.c:128)
  std::function<cplxf(const void *, const void *)> dot32;         // spinor_prod
  std::function<float(void *)> normalize32;                        // normalize
  std::function<void(void *, float, float, const void *)> axpy32;  // mulc_spinor_add
  std::function<void(void *)> zero32, zero64;
  std::function<void(const void *, void *)> copy64to32;            // assign_sd2s
  std::function<void(const void *, void *)> add32to64;             // add_s2sd
  std::function<void(const void *, const void *, void *)> diff64to32;  // diff_sd2s
  // y = sum of c[l] x[l], l = 0..n-1 in this order (optional: without it
  // the recursion zeroes y and applies one axpy32 per term)
  std::function<void(void *, int, const cplxf *, void *const *)> lincomb32;
};
double fgcr_core(const KrylovOps &o, int nkv, int nmx, int istop, double res, const void *eta, void *psi,
                 int *status, const std::function<void(const void *, void *)> &Dop,
                 const std::function<void(int, const void *, void *, void *)> &Mop,
                 const std::vector<void *> &phi, const std::vector<void *> &chi, void *rho, void *wrk);

KrylovOps dev_krylov_ops(Ctx &c);
int flat_cdot(Ctx &c, const double2 *x, const double2 *y, size_t n, double *res_dd, double *scratch, double *out_dev);
void flat_caxpy(Ctx &c, double2 *y, const double2 *x, size_t n, double ar, double ai);
void flat_cscale(Ctx &c, double2 *y, size_t n, double a);
int sw_shift_mass(Ctx &c, double dm, cudaStream_t st);
int gen_uniform_spinor32(const Ctx &c, void *dev, uint64_t seed, cudaStream_t st);

// dfl.cu
int dfl_set_parms(Ctx &c, const int bs[4], int Ns);
void dfl_release(Ctx &c);
// ltl_ref.cu: the reference's little solver (fgcr4vd + gcr4v + global-mode
// deflation) and the FP32 little operators
void ltl_ref_release(Ctx &c);
void ltl_invalidate(Ctx &c);
void ltl_forget_lmodes(Ctx &c);
int ltl_lmodes_from_fields(Ctx &c, const std::vector<void *> &modes, cudaStream_t st);
int ltl_lmode_set(Ctx &c, int l, const void *v32);
int ltl_set_modes(Ctx &c);
double ltl_gcr_ref(Ctx &c, double mu, const double2 *eta, double2 *psi, int *ifail, int *status, cudaStream_t st);
void dfl_Lvd_dev(Ctx &c, double2 *vd);
void dfl_LRvd_dev(Ctx &c, double2 *vd, double2 *wd);
void dfl_RLvd_dev(Ctx &c, double2 *vd, double2 *wd);
void dfl_Lv_dev(Ctx &c, float2 *v);
int little32_apply(Ctx &c, int which, const float2 *v, float2 *w);
const double *ltl_matrix_host(Ctx &c);
// dfl_gram.cu
bool gram_supported(const Ctx &c);
int dfl_cholqr(Ctx &c, const float4 *const *dv, float4 *const *dw, bool global, cudaStream_t st);
// solver_cg.cu
double tmcg_dev(Ctx &c, int eo, int nmx, int istop, double res, double mu, const void *eta, void *psi, int *ifail,
                int *status);
int tmcgm_dev(Ctx &c, int nmx, int istop, const double *res, int nmu, const double *mu, const void *eta,
              void *const *psi, int *ifail, int *status);
// archive.cu
int plaq_sum(Ctx &c, double *sum);
int export_cnfg(Ctx &c, const char *out);
int import_cnfg(Ctx &c, const char *in, int mask);
int export_sfld(Ctx &c, const char *out, int eo, const void *sd);
int import_sfld(Ctx &c, const char *in, int eo, void *sd);
// net.cu
int net_set_weights(Ctx &c, const float *w);
int net_get_weights(Ctx &c, float *w);
int net_nweights();
int net_init(Ctx &c, uint64_t seed, float scale);
int net_apply(Ctx &c, const void *in, void *out, bool half, cudaStream_t st);
int net_grad(Ctx &c, const void *r, const void *e, double *loss, float *grad);
int net_batch_grad(Ctx &c, int npairs, const void *const *r, const void *const *e, double *loss, float *grad);
int net_adam(Ctx &c, const float *grad, float lr);
int net_train(Ctx &c, int npairs, const void *const *r, const void *const *e, int steps, int batch, float lr,
              uint64_t seed, float *loss_hist);
void net_release(Ctx &c);
void net_fields_release(Ctx &c);
// dfl_batch.cu: the deflation steps for nr right-hand sides at once
int dfl_batch_alloc(Ctx &c);
int dirac_multi32(const Ctx &c, int n, float mu, void *const *sv, void *const *rv, void *const *subv,
                  cudaStream_t st);
// r_j = sub_j - Dw(mu_j) s_j for n <= SAP_MS systems in one launch (FP32)
int dirac_sys32(const Ctx &c, int n, const float *mu, void *const *sv, void *const *rv, void *const *subv,
                cudaStream_t st);
void dfl_mark(Ctx &c, int k);
int ensure_lvd_n(Ctx &c, int n);
int dfl_batch_check(Ctx &c);
int set_rhs_tiles(Ctx &c, const int *tile, const int *tc);   // fixed RHS tiles (0: autotune)
int rhs_tiles(const Ctx &c, int *tile, int *tc, float *ms);   // RHS tiles (restrict, prolong) and the kinds' times
// solver_batch.cu
int ltl_gcr_b(Ctx &c, double mu, int nr, const double2 *const *eta, double2 *const *psi, int *ifail, int *status,
              cudaStream_t st);
int gcr_batch(Ctx &c, int nr, int dfl, int nkv, int nmx, int istop, double res, const double *mu,
              const void *const *eta, void *const *psi, double *rho, int *ifail, int *status);
void gcr_batch_release();
void ltl_batch_release();
void dfl_restrict_b(Ctx &c, int nr, const void *const *x, double2 *const *vd, cudaStream_t st);
void dfl_prolong_b(Ctx &c, int nr, const double2 *const *vd, void *const *s, cudaStream_t st);
void little_b(Ctx &c, int nr, int mode, int b0, int nblk, const double2 *A, const double2 *H,
              const double2 *const *v, const double2 *const *u, double2 *const *w, cudaStream_t st);
void dfl_Awhat_b(Ctx &c, int nr, const double2 *const *v, double2 *const *w, double2 *const *t, cudaStream_t st);
void dfl_Aw_b(Ctx &c, int nr, const double2 *const *v, double2 *const *w, cudaStream_t st);
void dfl_restrict(Ctx &c, int prec, const void *s, double2 *vd, cudaStream_t st);
void dfl_prolong(Ctx &c, const double2 *vd, void *s, cudaStream_t st);
int dfl_subspace_dev(Ctx &c, const std::vector<void *> &modes, cudaStream_t st, bool lmodes = false);
void dfl_Aweeinv(Ctx &c, const double2 *v, double2 *w, cudaStream_t st);
void dfl_Awooinv(Ctx &c, const double2 *v, double2 *w, cudaStream_t st);
void dfl_Awoe(Ctx &c, const double2 *v, double2 *w, cudaStream_t st);
void dfl_Aweo(Ctx &c, const double2 *v, double2 *w, cudaStream_t st);
// diag_only: recompute the diagonal blocks only (keeping d.Ahop, which
// does not depend on the twisted mass)
int dfl_set_Aw(Ctx &c, double mu, cudaStream_t st, bool diag_only = false);
int dfl_set_Awhat(Ctx &c, double mu, cudaStream_t st, bool diag_only = false);
void dfl_Aw(Ctx &c, const double2 *v, double2 *w, cudaStream_t st);
void dfl_Awhat(Ctx &c, const double2 *v, double2 *w, double2 *t, cudaStream_t st);
double dfl_ltl_gcr(Ctx &c, double mu, const double2 *eta, double2 *psi, int *ifail, int *status, cudaStream_t st);
double dfl_sap_gcr_dev(Ctx &c, int nkv, int nmx, int istop, double res, double mu, const void *eta, void *psi,
                       int *ifail, int *status);
int dfl_modes_dev(Ctx &c, uint64_t seed, int *ifail, int *status);

// sap.cu
int sap_prepare(Ctx &c, cudaStream_t st);
int sap_variant_threads(const Ctx &c, int slot);
int sap_set_variant(Ctx &c, int v);
int sap_storage_mode(Ctx &c);
int sap_cycle(Ctx &c, float mu, int isolv, int nmr, void *psi, void *rho, void *phi_blk, cudaStream_t st);
int sap_cycles(Ctx &c, float mu, int isolv, int nmr, int ncy, void *psi, void *rho, void *phi_blk,
               cudaStream_t st);
// the 12-real FP32 link copy (first two rows) when the 12-real reads are on
// and every link passed the SU(3) check with its boundary sign, else null
const void *links12(Ctx &c, cudaStream_t st);
// field the captured SAP sequence reads its input from (null when CUDA
// graphs are off); an rh written there is not copied again by sap_mop
void *sap_input_field(Ctx &c);
// psi = ncy cycles on rho = rh, then rho = rh - rho (the sap_gcr preconditioner)
int sap_mop(Ctx &c, float mu, int isolv, int nmr, int ncy, const void *rh, void *psi, void *rho, void *phi_blk,
            cudaStream_t st, const void *base = nullptr, const void *add = nullptr);
// ncy SAP cycles for n systems of one twisted mass on their own fields
int sap_cycles_multi(Ctx &c, int n, float mu, int isolv, int nmr, int ncy, void *const *psi, void *const *rho,
                     void *const *phi_blk, cudaStream_t st);
// the input field of system r (< n <= SAP_MS) of an sap_mop_multi call on
// n systems (null when CUDA graphs are off, with domain decomposition, or
// when the fields do not fit)
void *sap_input_field_multi(Ctx &c, int r, int n);
// sap_mop for ns systems (twisted masses mu[r]) with every SAP launch
// covering up to SAP_MS of them; base and add may be null (as in sap_mop),
// or arrays whose entries may be null
int sap_mop_multi(Ctx &c, int ns, const float *mu, int isolv, int nmr, int ncy, const void *const *rh,
                  void *const *psi, void *const *rho, void *phi_blk, cudaStream_t st, const void *const *base,
                  const void *const *add);

}  // namespace qcd
