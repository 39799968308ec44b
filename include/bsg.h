/*
 * bsg.h -- C ABI of the B200 M-scheme Hamiltonian engine (libbsgpu.so).
 *
 * The engine replaces BIGSTICK's on-the-fly factorized matvec and the Lanczos
 * loop around it.  The Fortran host keeps building the basis, sectors, jumps,
 * opbundles and uncoupled matrix elements; it passes plain pointers to those
 * module arrays through this ABI (an ISO_C_BINDING interface block).  The
 * arrays are uploaded to the device unchanged; every derived index the GPU
 * kernels need lives in separate device buffers.
 *
 * Index conventions are the reference's (Fortran, 1-based):
 *   basis state = pstart(ip) + nstart(in)  (pstart 0-based offset, nstart
 *   1-based), jump isd/fsd already hold pstart/nstart values, op labels and
 *   hmat indices are 1-based, cpnpair/dpnpair are 2-D Fortran arrays with
 *   bounds (-nhsps(-2):nhsps(2), -nhsps(-1):nhsps(1)), first index fastest.
 *
 * Every entry point returns an int status (BSG_OK == 0).  Nothing aborts,
 * traps or exits; the last error message is latched in the context.
 */
#ifndef BSG_H
#define BSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace the reference's `stop N`, e.g.
 *      src/bapplyhlibOMP.f90:943, :1446 and :1971) ---- */
#define BSG_OK               0
#define BSG_ERR_BAD_TABLE    1   /* table failed validation before upload      */
#define BSG_ERR_OOB_INDEX    2   /* an index points outside its array          */
#define BSG_ERR_CUDA         3   /* CUDA runtime error                         */
#define BSG_ERR_NOMEM        4   /* device or host allocation failed           */
#define BSG_ERR_TIMEOUT      5   /* a bounded device wait gave up              */
#define BSG_ERR_NAN          6   /* non-finite value found in a vector         */
#define BSG_ERR_ARG          7   /* bad argument                               */
#define BSG_ERR_UNSUPPORTED  8   /* valid input outside what this build covers */
#define BSG_ERR_NOT_CONVERGED 9  /* Lanczos hit its iteration cap              */

/* ---- opbundle optype / hchar (src/bmodules_parallel.f90:275-311) ---- */
#define BSG_OP_SPE 1
#define BSG_OP_PP  2
#define BSG_OP_NN  3
#define BSG_OP_PN  4
#define BSG_H_FWD  'f'
#define BSG_H_BWD  'b'
#define BSG_H_HERM 'h'

/* ---- vector precision (lanc_prec, src/bmodules_main.f90:171) ---- */
#define BSG_PREC_FP32 4
#define BSG_PREC_FP64 8

/* ---- bsg_applyh flags ---- */
#define BSG_ACCUMULATE   1   /* vout += H vin (the reference's semantics after
                                initialize_final zeroes vec2); else vout = H vin */
#define BSG_DEVICE_PTRS  2   /* vin/vout are device pointers; else host memory  */

/*
 * Plain pointers to the reference's module arrays after setup
 * (src/bigstick_main.f90:650-676: jumps sorted by sort_bundled_jumps,
 * hmat* filled by uncoupleXXtbme / count_uncouplepn).
 */
typedef struct bsg_tables {
    /* basis: src/bbasislib.f90:16-19, combinebasis :540-677 */
    int64_t dimbasis;
    int64_t nsd_p, nsd_n;              /* nXsd(1), nXsd(2)                   */
    const int64_t *pstart;             /* [nsd_p]                            */
    const int64_t *nstart;             /* [nsd_n]                            */

    /* one-body jumps: src/bmodules_main.f90:643-666 */
    int64_t np1b;
    const int64_t *p1b_isd, *p1b_fsd;
    const int16_t *p1b_cop, *p1b_dop;
    const int8_t  *p1b_phase;
    int64_t nn1b;
    const int64_t *n1b_isd, *n1b_fsd;
    const int16_t *n1b_cop, *n1b_dop;
    const int8_t  *n1b_phase;

    /* two-body jumps: src/bmodules_main.f90:668-680 */
    int64_t np2b;
    const int64_t *p2b_isd, *p2b_fsd;
    const int32_t *p2b_op;
    const int8_t  *p2b_phase;
    int64_t nn2b;
    const int64_t *n2b_isd, *n2b_fsd;
    const int32_t *n2b_op;
    const int8_t  *n2b_phase;

    /* uncoupled matrix elements, float32: src/bmodules_main.f90:873-875 */
    int64_t nmatpp, nmatnn, nmatpn;
    const float *hmatpp, *hmatnn, *hmatpn;   /* 1-based labels index these */

    /* cpnpair/dpnpair: src/btbmepn.f90:126-131 */
    int32_t nhsps_pl, nhsps_pr;        /* nhsps(-1), nhsps(1)                */
    int32_t nhsps_nl, nhsps_nr;        /* nhsps(-2), nhsps(2)                */
    const int64_t *cpnpair, *dpnpair;  /* [(nl+nr+1)*(pl+pr+1)], column-major */

    /* SPE case (only when call_spe, src/bsppot.f90:20-34): src/bdiagh.f90:5-13 */
    int32_t call_spe;
    const float *pspe_h;               /* [nsd_p] or NULL                    */
    const float *nspe_h;               /* [nsd_n] or NULL                    */

    /* opbundles as struct-of-arrays: src/bmodules_parallel.f90:275-311 */
    int64_t nbundles;
    const int32_t *optype;             /* BSG_OP_*                           */
    const int32_t *hchar;              /* 'f', 'b', 'h'                      */
    const int64_t *pxstart, *pxend, *nxstart, *nxend, *cstride;
} bsg_tables;

typedef struct bsg_config {
    int32_t device;        /* CUDA device ordinal                              */
    int32_t max_nb;        /* largest block size bsg_applyh will be given      */
    int32_t validate;      /* 1: run the host-side table validator at create   */
    int32_t pn_table_max;  /* largest (b,d) label-pair table of one neutron
                              operator (the PN-form shared-memory table); a
                              larger operator is split into sub-operators of
                              at most this many pairs.  0: 512 (384 for
                              bsg_create3) */
} bsg_config;

typedef struct bsg_ctx bsg_ctx;

/* Lanczos parameters (src/blanczosmain.f90:1413-2153, src/bmodules_flags.f90) */
typedef struct bsg_lanczos_params {
    int32_t nkeep;         /* states wanted                                    */
    int32_t niter;         /* iterations per restart cycle (max if no restart) */
    int32_t nthick_add;    /* extra Ritz vectors kept on thick restart (0: off)*/
    int32_t max_restarts;  /* max_num_thick_restart                            */
    int32_t nb;            /* block size: 1 = lanczos_p, >1 = lanczos_block     */
    int32_t matvec_prec;   /* BSG_PREC_FP32 or BSG_PREC_FP64 for applyH         */
    int32_t fixed_iter;    /* 1: run exactly niter iterations (no conv. test)  */
    int32_t ncheck;        /* states in the convergence test (nkeep+ncheck_ex) */
    double  converge_tol;  /* converge_tol0_def = 1e-3 (blanczoslib.f90:2642)  */
    int32_t want_vectors;  /* 1: return nkeep eigenvectors (fp64, dim x nkeep) */
    int32_t pivot;         /* 0: uniform 1/sqrt(dim) (blanczoslib.f90:825-831);
                              bsg_batch_lanczos also takes 1: a seeded random
                              normalized pivot per system (seed, system)   */
    uint64_t seed;         /* random restart / block pivot seed                */
    int32_t lanc_prec;     /* Lanczos vector storage (src/bmodules_main.f90:171):
                              BSG_PREC_FP32 or BSG_PREC_FP64 (0 = FP64); dots,
                              updates and alpha/beta accumulate in FP64 */
    int32_t reserved;
} bsg_lanczos_params;

typedef struct bsg_report {
    int32_t iterations;        /* iterations in the last cycle              */
    int32_t total_iterations;  /* including thick-restart cycles            */
    int32_t restarts;          /* thick restarts done                       */
    int32_t random_restarts;   /* beta collapses handled                    */
    int32_t matvecs;           /* applyH calls (block calls count once)     */
    int32_t converged;
    double  t_matvec_ms;       /* device time in applyH                     */
    double  t_reorth_ms;       /* device time in reorthogonalization        */
    double  t_eig_ms;          /* device time in projected eigen-solves     */
    double  t_total_ms;
} bsg_report;

/* ---- three-body opbundles (src/bapplyhlib1.f90:1390-2804) ---- */
#define BSG_OP_PPP 7   /* p3b jumps px, conjugate neutron SDs nx (as PP)       */
#define BSG_OP_NNN 8   /* proton SDs px (cstride), n3b jumps nx (as NN)        */
#define BSG_OP_PPN 9   /* p2b jumps px (pair labels), n1b jumps nx             */
#define BSG_OP_PNN 10  /* p1b jumps px, n2b jumps nx (pair labels)             */

/*
 * The arrays a three-body run adds (src/bmodules_3body.f90:26-103).  In such
 * a run the two-body jumps carry the labels of their created (cop) and
 * destroyed (dop) pair instead of a matrix-element label
 * (src/bjumplib_weld.f90:771-775): bsg_tables' p2b_op / n2b_op are unused
 * and the pair labels come from here.  Pair labels are 1-based indices of
 * the species' pair list (XX2(it)%pair).
 *   PPP: out(p3b_fsd + nstart(csd)) += hmatppp(p3b_op) * p3b_phase * in(p3b_isd + nstart(csd))
 *   NNN: out(n3b_fsd + pstart(csd)) += hmatnnn(n3b_op) * n3b_phase * in(...)
 *   PPN: xme = hmatppn(cppntriplet(bb,a) + dppntriplet(dd,c)) * phasep * phasen,
 *        bb/dd = p2b cop/dop, a/c = n1b cop/dop (src/bapplyhlib1.f90:2295-2562)
 *   PNN: xme = hmatpnn(cpnntriplet(bb,a) + dpnntriplet(dd,c)) * phasep * phasen,
 *        a/c = p1b cop/dop, bb/dd = n2b cop/dop (src/bapplyhlib1.f90:2033-2285)
 * 'f' bundles add out(statef) += xme*in(statei), 'b' bundles the transpose.
 * cppntriplet / dppntriplet are column-major [npairs_p x (nhsps_nl+nhsps_nr+1)]
 * as the reference's cppntriplet(npairs, -nhsps(-2):nhsps(2)): entry (bb, a)
 * at (bb-1) + (a + nhsps_nl)*npairs_p.  cpnntriplet / dpnntriplet likewise
 * [npairs_n x (nhsps_pl+nhsps_pr+1)], (bb, a) at (bb-1) + (a + nhsps_pl)*npairs_n.
 */
typedef struct bsg_tables3 {
    const int32_t *p2b_cop, *p2b_dop;   /* [np2b] created / destroyed proton pair */
    const int32_t *n2b_cop, *n2b_dop;   /* [nn2b]                                 */
    int64_t np3b;
    const int64_t *p3b_isd, *p3b_fsd;   /* pstart values                          */
    const int32_t *p3b_op;              /* 1-based hmatppp label                  */
    const int8_t  *p3b_phase;
    int64_t nn3b;
    const int64_t *n3b_isd, *n3b_fsd;   /* nstart values                          */
    const int32_t *n3b_op;              /* 1-based hmatnnn label                  */
    const int8_t  *n3b_phase;
    int64_t nmatppp, nmatnnn, nmatppn, nmatpnn;
    const float *hmatppp, *hmatnnn, *hmatppn, *hmatpnn;
    int32_t npairs_p, npairs_n;
    const int32_t *cppntriplet, *dppntriplet;
    const int32_t *cpnntriplet, *dpnntriplet;
} bsg_tables3;

/* ---- lifecycle ---- */
int  bsg_create(const bsg_tables *t, const bsg_config *cfg, bsg_ctx **out);
/* a three-body Hamiltonian: the bundles of t are applied as
 * applyHbundled_g does with threebody set (src/bapplyhlib1.f90:56-310): SPE,
 * PPP, PPN, PNN and NNN; PP, NN and PN bundles are skipped.  bsg_grad is
 * not available on such a context (BSG_ERR_UNSUPPORTED). */
int  bsg_create3(const bsg_tables *t, const bsg_tables3 *t3, const bsg_config *cfg, bsg_ctx **out);
/* bsg_validate_tables for a three-body run (t3 may be NULL: two-body) */
int  bsg_validate_tables3(const bsg_tables *t, const bsg_tables3 *t3, char *msg, size_t len);
int  bsg_destroy(bsg_ctx *ctx);
/* the validator bsg_create runs, on the host only (no GPU needed): every
 * index of every table checked against its array (the reference's own checks
 * are check_opbundle_bounds, src/bparallel_opbundles.f90:1232-1286, and the
 * range asserts of src/bapplyhlibOMP.f90:1968-1972); msg gets the reason */
int  bsg_validate_tables(const bsg_tables *t, char *msg, size_t len);
const char *bsg_strerror(int status);
/* copies the latched message of the last failing call on ctx */
int  bsg_last_error(const bsg_ctx *ctx, char *buf, size_t len);

/* ---- applyH: replaces applyHbundled_omp('n') (src/bapplyhlibOMP.f90:882)
 *      for nb == 1 and applyHbundled_block_omp (src/bapplyhlibOMP_block.f90:43)
 *      for nb > 1.  Vectors of nb interleaved vectors: element (state s,
 *      vector v) at (s-1)*nb + v (src/bmodules_block.f90:19-22).
 *      prec: BSG_PREC_FP32 (float vectors, fp32 accumulation) or
 *      BSG_PREC_FP64 (double vectors, fp32 matrix elements promoted). ---- */
int  bsg_applyh(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int flags);
/* same on a caller-provided cudaStream_t (device pointers only) */
int  bsg_applyh_stream(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec,
                       int flags, void *cuda_stream);

/* ---- applyH on host vectors with no device allocation.  No counterpart in
 *      the reference.  For callers that cannot allocate device memory when
 *      they need a matvec: hosts whose device memory is a fixed pool owned by
 *      another component, and drivers that must not grow the device
 *      footprint after set-up.  vin/vout are staged through one static
 *      __device__ array instead of buffers allocated on first use.  Each
 *      vector (dim*nb*element size) must fit in BSG_NOALLOC_MAX_VECTOR_BYTES,
 *      else BSG_ERR_ARG.  The call is synchronous: it waits for the
 *      context's stream before it returns.  The first call on a device looks
 *      up the array's address.  Row tiles: the context's
 *      own when an earlier applyH built them, else at most 65536 tiles in the
 *      static array (more: BSG_ERR_ARG).  All calls in the process share the
 *      array: calls that overlap on the GPU race.  Same semantics as
 *      bsg_applyh otherwise (host pointers only, BSG_ACCUMULATE honoured). ---- */
#define BSG_NOALLOC_MAX_VECTOR_BYTES (8u << 20)
int  bsg_applyh_noalloc(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int flags);

/* ---- Lanczos: replaces lanczos_p (src/blanczosmain.f90:1413) and
 *      lanczos_block (:1804) with thick restart; everything stays on the
 *      device.  evals[nkeep]; evecs (host, fp64, dim x nkeep column-major) or
 *      NULL.  pivot_vec: optional host fp64 start vector (dim*nb) or NULL. ---- */
int  bsg_lanczos(bsg_ctx *ctx, const bsg_lanczos_params *p, const double *pivot_vec,
                 double *evals, double *evecs, bsg_report *rep);

/* ---- adjoint: Hellmann-Feynman gradient dE_k/dhmat for the uncoupled
 *      matrix elements (the transposed-jump contraction of
 *      src/bdenslib4.f90:129-729).  evecs: host fp64 dim x nstates column-major
 *      (normalized).  Outputs (host, fp64): dpp[nstates*nmatpp],
 *      dnn[nstates*nmatnn], dpn[nstates*nmatpn], dspe_p[nstates*nsd_p] and
 *      dspe_n[nstates*nsd_n] (the last two only when call_spe; may be NULL). ---- */
int  bsg_grad(bsg_ctx *ctx, const double *evecs, int nstates,
              double *dpp, double *dnn, double *dpn, double *dspe_p, double *dspe_n);
/*      All states in one launch; every label's sum is accumulated exactly (to
 *      2^-64) in 128-bit fixed point with integer atomics, so the result is
 *      bitwise repeatable and independent of how the work is split. */

/* ---- one-body densities: replaces master_density1b_bundled
 *      (src/bdenslib1.f90:1506-1607), i.e. applyP1Bdenbundled_g and
 *      applyN1Bdenbundled_g (src/bdenslib3.f90:14-311), for every pair of
 *      nstates states in one call.  The tables are the one-body jumps that
 *      master1bodyjumps builds for densities (Delta Jz = 0 sector jumps,
 *      a+_c a_c included) in the jumpNbody arrays' types, bundled as the
 *      reference's P1B / N1B opbundles:
 *        P1B: jumps pxstart..pxend of p1b_*; conjugate neutron SDs
 *             nxstart..nxend step cstride; statei = p1b_isd + nstart(...)
 *             exactly as src/bdenslib3.f90:58-100 indexes it;
 *        N1B: jumps nxstart..nxend of n1b_*; conjugate proton SDs
 *             pxstart..pxend step cstride, pstride = pstart(pxstart+cstride)
 *             - pstart(pxstart); statei = n1b_isd + pstart(pxstart) +
 *             pstride*(k-1) (src/bdenslib3.f90:206-265).
 *      hchar 'f'/'h' adds psi_f(statef) psi_i(statei) phase to (cop, dop);
 *      'b' adds psi_f(statei) psi_i(statef) phase to (dop, cop).
 *      vecs: host fp64, dim x nstates column-major, nstates <= 32.
 *      Outputs (host fp64, zeroed first):
 *        p1bopme[((f*nstates + i)*nqp + c)*nqp + d] = <f| a+_c a_d |i>
 *      with nqp = nhsps_pl + nhsps_pr and c, d the combined s.p. index of a
 *      signed label (-l -> l-1 for l = 1..nhsps_pl, +r -> nhsps_pl + r - 1);
 *      n1bopme likewise with nqn = nhsps_nl + nhsps_nr.  The sum over each
 *      label runs in a fixed order: results are bitwise repeatable. ---- */
#define BSG_OP_P1B 5
#define BSG_OP_N1B 6
typedef struct bsg_density_tables {
    int64_t np1b;
    const int64_t *p1b_isd, *p1b_fsd;
    const int16_t *p1b_cop, *p1b_dop;
    const int8_t  *p1b_phase;
    int64_t nn1b;
    const int64_t *n1b_isd, *n1b_fsd;
    const int16_t *n1b_cop, *n1b_dop;
    const int8_t  *n1b_phase;
    int64_t nbundles;
    const int32_t *optype;             /* BSG_OP_P1B or BSG_OP_N1B           */
    const int32_t *hchar;              /* 'f', 'b', 'h'                      */
    const int64_t *pxstart, *pxend, *nxstart, *nxend, *cstride;
} bsg_density_tables;
int  bsg_density1b(bsg_ctx *ctx, const bsg_density_tables *dt, const double *vecs, int nstates,
                   double *p1bopme, double *n1bopme);

/* ---- one-body operator: replaces master_apply1bop (src/bdenslib1.f90:2612)
 *      with applyP1Bopbundled_g / applyN1Bopbundled_g (src/bdenslib3.f90:319-584)
 *      over the same density tables: vout = O vin with
 *      O = sum_cd ppot[c*nqp + d] a+_c a_d (protons) + npot[...] (neutrons),
 *      the reference's pPOT_h / nPOT_h on combined s.p. indices (the layout
 *      of p1bopme).  ppot or npot may be NULL (no such part).  vin, vout:
 *      host fp64, dim x nvec column-major.  Rows are owned by one writer per
 *      species and summed in a fixed order: bitwise repeatable. ---- */
int  bsg_apply1b(bsg_ctx *ctx, const bsg_density_tables *dt, const double *ppot, const double *npot,
                 const double *vin, double *vout, int nvec);

/* ---- batched systems: many independent Hamiltonians of uneven dimension
 *      (the reference runs one per process).  bsg_batch_applyh applies all of
 *      them in one persistent launch whose CTAs pull (system, row tile) work
 *      items heaviest first; vin[s]/vout[s] are device pointers of dim_s
 *      elements, launched on cuda_stream (NULL: the legacy default stream).  bsg_batch_lanczos runs lock-step scalar Lanczos on all
 *      systems for exactly p->niter iterations (uniform pivots, full
 *      classical Gram-Schmidt reorthogonalization) with each iteration
 *      captured once as a CUDA graph and replayed; evals[s*nkeep + k];
 *      evecs NULL or n host pointers of dim_s*nkeep doubles.  The tile width
 *      and CTA residency of the batched kernel come from bsg_batch_autotune
 *      (timed on the device) or bsg_batch_set_tuning. ---- */
typedef struct bsg_batch bsg_batch;
int  bsg_batch_create(int n, const bsg_tables *const *tables, const bsg_config *cfg, bsg_batch **out);
int  bsg_batch_destroy(bsg_batch *b);
int  bsg_batch_last_error(const bsg_batch *b, char *buf, size_t len);
int  bsg_batch_dims(const bsg_batch *b, int64_t *dims);
int  bsg_batch_system(const bsg_batch *b, int s, bsg_ctx **ctx);
int  bsg_batch_applyh(bsg_batch *b, const void *const *vin, void *const *vout, int prec, void *cuda_stream);
int  bsg_batch_autotune(bsg_batch *b, int *items, int *ctas_per_sm, double *best_ms);
int  bsg_batch_set_tuning(bsg_batch *b, int items, int ctas_per_sm);
int  bsg_batch_lanczos(bsg_batch *b, const bsg_lanczos_params *p, double *evals, double *const *evecs,
                       bsg_report *rep);
/* adjoint gradients of every system of the batch in one launch over all
 * (system, state, row tile) items (the per-system bsg_grad of each member,
 * bitwise equal to it): evecs[s] host fp64 dim_s x nstates column-major;
 * dpp[s], dnn[s], dpn[s] host fp64 [nstates x nmat*_s] (state-major), and
 * dspe_p[s] / dspe_n[s] for members with SPE bundles (arrays may be NULL).
 * kernel_ms (may be NULL): device time of the launch. */
int  bsg_batch_grad(bsg_batch *b, const double *const *evecs, int nstates, double *const *dpp,
                    double *const *dnn, double *const *dpn, double *const *dspe_p, double *const *dspe_n,
                    double *kernel_ms);

/* ---- on-device jump generation: the set-up stage that builds the jump
 *      tables (weld / master1bodyjumps / master2bodyjumps,
 *      src/bjumplib_weld.f90:296-809, src/bjumplib_master.f90:436-1196) and
 *      sorts the PN bundles' ranges (sort1bjumps, src/bsortjumpslib.f90
 *      :190-290), run as GPU kernels.  A species is described by its Slater
 *      determinants; the generated arrays are the jumpNbody arrays of bsg.h
 *      (p1b_*, n1b_*, p2b_*, n2b_*), in the host builder's order:
 *        one-body, per sector jump (is -> fs): source SD ascending, then the
 *          annihilated state k, then the created state i (a+_i a_k), the
 *          jumps whose final SD lies in fs;
 *        two-body, per sector: source SD, annihilated pair k<l, created pair
 *          i<j of the same (M, parity) section, isd >= fsd kept;
 *      isd/fsd hold pstart/nstart values, cop/dop the signed labels
 *      (q < nl: -(q+1), else q-nl+1), op the hmatpp/hmatnn label. ---- */
typedef struct bsg_species {
    int32_t nsps;                 /* s.p. states (at most 22)                  */
    int32_t nl;                   /* the first nl states have m < 0            */
    const int32_t *m2, *par;      /* 2m and parity (+1/-1) per s.p. state      */
    int64_t nsd;
    const uint64_t *sd_bits;      /* occupation bitmask per SD (bit q: state q)*/
    const int64_t *xstart;        /* pstart (protons) / nstart (neutrons) per SD */
    int32_t nsectors;
    const int64_t *sector_start, *sector_end;   /* 1-based SD range per sector */
} bsg_species;
typedef struct bsg_jumpgen bsg_jumpgen;
int  bsg_jumpgen_create(int device, const bsg_species *sp, bsg_jumpgen **out);
int  bsg_jumpgen_destroy(bsg_jumpgen *g);
int  bsg_jumpgen_last_error(const bsg_jumpgen *g, char *buf, size_t len);
/* one-body jumps of the sector jumps is[j] -> fs[j] (0-based sectors):
 * starts[0..nsj] receives the first jump of each (starts[nsj] = total); the
 * outputs (host arrays of starts[nsj] entries) may be NULL to count only */
int  bsg_jumpgen_one(bsg_jumpgen *g, int nsj, const int32_t *is, const int32_t *fs, int64_t *starts,
                     int64_t *isd, int64_t *fsd, int16_t *cop, int16_t *dop, int8_t *phase, double *kernel_ms);
/* two-body jumps inside the sectors sec[j] */
int  bsg_jumpgen_two(bsg_jumpgen *g, int nsec, const int32_t *sec, int64_t *starts,
                     int64_t *isd, int64_t *fsd, int32_t *op, int8_t *phase, double *kernel_ms);
/* sort1bjumps on the nr disjoint ranges [start, start+len) of host arrays of
 * n jumps: key fsd (by_fsd = 1, the proton side of PN bundles) or isd */
int  bsg_jumpgen_sort1(bsg_jumpgen *g, int nr, const int64_t *start, const int64_t *len, int by_fsd, int64_t n,
                       int64_t *isd, int64_t *fsd, int16_t *cop, int16_t *dop, int8_t *phase, double *kernel_ms);

/* ---- introspection used by tests and the benchmark ---- */
typedef struct bsg_stats {
    int64_t n_ops_pp, n_ops_nn, n_ops_pn, n_ops_spe;  /* inner-loop updates / matvec */
    int64_t jump_bytes;        /* bytes of jump + label tables uploaded        */
    int64_t derived_bytes;     /* bytes of derived device indices              */
    int64_t n_rows;            /* proton SDs (output rows)                     */
    int64_t n_contrib;         /* row contributions                            */
    int32_t kernel_launches_per_matvec;
    int32_t reserved;
    /* last bsg_density1b: device time of its kernels (ms), rows summed
     * (conjugate SDs over all jumps), launches */
    double  density_ms;
    int64_t density_rows;
    int32_t density_launches;
    int32_t reserved2;
    double  apply1b_ms;        /* last bsg_apply1b: device time of its kernels */
    double  grad_ms;           /* last bsg_grad: device time of its kernels    */
    /* three-body contexts: inner-loop updates per matvec of each kind */
    int64_t n_ops_ppp, n_ops_nnn, n_ops_ppn, n_ops_pnn;
} bsg_stats;
int  bsg_get_stats(const bsg_ctx *ctx, bsg_stats *st);

#ifdef __cplusplus
}
#endif
#endif /* BSG_H */
