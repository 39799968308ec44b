/*
 * bsg_host.h -- C ABI of the host-side table builder (libbsghost.so).
 *
 * In a BIGSTICK build the Fortran host produces the tables that bsg_create()
 * consumes (basis, sectors, jumps, opbundles, uncoupled matrix elements).  No
 * Fortran compiler is available to this project, so this CPU library restates
 * that setup for full (untruncated) M-scheme spaces and fills the same arrays,
 * in the same element types and with the same index conventions.  It is not
 * part of the GPU path: it only produces the inputs of bsg.h.
 *
 * Reference stages restated here:
 *   s.p. states      src/bspstates.f90:53-332 (extract_sps, sort_spsqn,
 *                    make_hspsqn)
 *   sectors, basis   src/bbasislib.f90:227-677 (count_create_sectors,
 *                    count_fill_sectors_w_blocks, combinebasis)
 *   jumps            src/bjumplib_weld.f90:296-809 (isd = blockstart-1 +
 *                    (iladd-1)*niradd + iradd; hermitian half isd >= fsd on
 *                    diagonal two-body blocks)
 *   opbundles        src/bparallel_opbundles.f90:36-708
 *   density jumps    src/bdenslib1.f90:190-213 (set1bsectorjumps,
 *                    master1bodyjumps) with P1B/N1B bundles as read by
 *                    src/bdenslib3.f90:14-311
 *   jump sort        src/bsortjumpslib.f90:21-290 (shell sort, fixed strides)
 *   matrix elements  src/btbme.f90:1209-1551, src/btbmepn.f90:177-587,
 *                    src/binput_tbme.f90:898-2027, src/bsppot.f90:20-238
 */
#ifndef BSG_HOST_H
#define BSG_HOST_H

#include <stdint.h>
#include "bsg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* one orbit line of an isospin .sps file: n l j w (src/binput.f90) */
typedef struct bsg_orbit {
    int32_t nr, l, j2, w;      /* j2 = 2j */
} bsg_orbit;

/* coupled J-T two-body matrix element line "a b c d J T V" of an isospin
 * .int file (src/binput_tbme.f90:898-1240), orbit labels 1-based */
typedef struct bsg_tbme {
    int32_t a, b, c, d, J, T;
    double v;
} bsg_tbme;

typedef struct bsg_model_spec {
    int32_t norb;
    const bsg_orbit *orbits;   /* same orbits for protons and neutrons      */
    int32_t np, nn;            /* valence protons, neutrons                 */
    int32_t jz2;               /* 2 x Jz of the system                      */
    int32_t parity;            /* +1 / -1 (ignored when all orbits share it) */
    int32_t ntbme;
    const bsg_tbme *tbme;
    const double *spe;         /* [norb] single-particle energies           */
    double spe_scale;          /* xspe                                      */
    double tbme_scale;         /* (A0/A)^x                                   */
} bsg_model_spec;

/* owning container: every pointer in .t points into memory owned here */
typedef struct bsg_host_tables {
    bsg_tables t;
    int32_t nsectors_p, nsectors_n;
    int64_t *psector_start, *psector_end;  /* 1-based SD ranges per sector */
    int32_t *psector_jz2, *psector_par;
    int64_t *nsector_start, *nsector_end;
    int32_t *nsector_jz2, *nsector_par;
    int32_t *psector_conj;                 /* conjugate neutron sector (1-based) */
    int32_t nhsps_p, nhsps_n;              /* total s.p. states per species */
    /* s.p. states in builder order: combined label q (0-based); signed label
     * is -(q+1) for q < nl (left, m<0) else q-nl+1 (right, m>=0) */
    int32_t *sp_orb_p, *sp_m2_p, *sp_orb_n, *sp_m2_n;
    uint64_t *sd_bits_p, *sd_bits_n;       /* occupation bitmasks per SD   */
    /* pair bookkeeping for the adjoint chain rule (coupled <- uncoupled) */
    int64_t npairs_pp, npairs_nn, npairs_pn;
    void *priv;                            /* builder internals            */
    /* one-body density jumps and P1B/N1B bundles for bsg_density1b
     * (master1bodyjumps for densities, src/bdenslib1.f90:190-213) */
    bsg_density_tables dt;
    /* three-body arrays (bsg_host_build3), NULL for a two-body build */
    const bsg_tables3 *t3;
} bsg_host_tables;

int  bsg_host_build(const bsg_model_spec *spec, bsg_host_tables **out);

/* A three-body Hamiltonian for bsg_create3: SPE bundles (pspe_h / nspe_h)
 * plus PPP, PPN, PNN and NNN bundles, no two-body bundles, as a BIGSTICK run
 * with three-body forces is laid out (src/bapplyhlib1.f90:56-310).  The
 * uncoupled three-body matrix elements are
 *   W(T, T') = w2 * <T| V2 |T'> / (A - 2) + w3 * R(T, T'),
 * where <T|V2|T'> is the two-body interaction of spec between three-particle
 * states (the reference converts two-body into three-body matrix elements
 * the same way, src/b3from2bme.f90; on A-particle states the w2 term alone is
 * exactly V2), and R a seeded symmetric part, uniform in [-1, 1), that keeps
 * M and parity: for the triplet keys kT, kT' (sorted combined s.p. labels q
 * of the builder's order -- PPP (p,p,p) kind 1, NNN (n,n,n) kind 2, PPN
 * (p,p,n) kind 3, PNN (p,n,n) kind 4) with lo <= hi in lexicographic order,
 *   x = seed; for v in (kind, lo..., hi...): x = mix(x ^ v);
 *   R = (x >> 11) * 2^-52 - 1,
 * mix the SplitMix64 finalizer of (x + 0x9E3779B97F4A7C15).  Two-body jumps
 * carry pair labels (t3->p2b_cop/dop), hmat of a diagonal label (T == T',
 * or equal pairs bb == dd for PPN / PNN) is halved since 'f' and 'b'
 * bundles both apply it, and three-body jumps inside a sector keep
 * isd >= fsd (src/bjumplib_weld.f90:1072-1076).  Needs A >= 3. */
typedef struct bsg_model3_spec {
    double w2;
    double w3;
    uint64_t seed;
} bsg_model3_spec;
int  bsg_host_build3(const bsg_model_spec *spec, const bsg_model3_spec *s3, bsg_host_tables **out);
void bsg_host_free(bsg_host_tables *h);
const char *bsg_host_last_error(void);

/* d hmat / d V_JT(ab,cd) chain-rule coefficients: for uncoupled label index
 * k (0-based) of species kind (0 = pp, 1 = nn, 2 = pn) the coefficient of
 * each file TBME line i: dhmat[k]/dV_i.  Dense [nmat x ntbme] double.
 * Also dhmat/dspe_a for each orbit ([nmat x norb]) through SPE subsumption. */
int  bsg_host_me_jacobian(const bsg_host_tables *h, int kind, double *d_tbme, double *d_spe);

#ifdef __cplusplus
}
#endif
#endif /* BSG_HOST_H */
