/*
 * ORACLE -- test infrastructure only.  Nothing in the product links, imports
 * or calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, as the checker.
 *
 * Plain-C restatement of BIGSTICK's factorized matvec on the host:
 *
 *   oracle_applyh()      applyHbundled_omp with one thread
 *                        (src/bapplyhlibOMP.f90:882-1657: SPE :988-1011,
 *                        NN :1012-1066, PP :1068-1241, PN :1242-1442) and its
 *                        block form applyHbundled_block_omp
 *                        (src/bapplyhlibOMP_block.f90:43-886) for nb > 1.
 *   oracle_applyh_rows() / oracle_applyh_owner()
 *                        applyHbundled_omp's owner-computes OpenMP
 *                        partition: every thread computes the output rows
 *                        getLoadDist gives it (src/bapplyhlibOMP.f90:34-868,
 *                        :954-1442).  The timed CPU baseline, and the checker
 *                        of systems too large for one thread (a few rows).
 *   oracle_applyh_omp()  the OpenMP serial-path split routines
 *                        applyhPPbundled_g / applyhNNbundled_g /
 *                        applyhPNbundled_g (src/bapplyhlib1.f90:325-818):
 *                        PP threads over neutron SD chunks, NN over proton SD
 *                        chunks, PN forward over proton-jump chunks cut at
 *                        p1b_fsd changes, PN backward over neutron-jump chunks
 *                        cut at n1b_isd changes (jumps are sorted that way,
 *                        src/bsortjumpslib.f90:57-95).
 *
 * Arithmetic follows the reference: xme is real(4) (hmat * phase), the update
 * is vout = vout + xme*vin in the vector precision (float for lanc_prec=4,
 * double for lanc_prec=8), accumulating into vout.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/bsg.h"

#define CPN(t, b, a) ((t)->cpnpair[(int64_t)((b) + (t)->nhsps_nl) + \
                      (int64_t)((a) + (t)->nhsps_pl) * (int64_t)((t)->nhsps_nl + (t)->nhsps_nr + 1)])
#define DPN(t, d, c) ((t)->dpnpair[(int64_t)((d) + (t)->nhsps_nl) + \
                      (int64_t)((c) + (t)->nhsps_pl) * (int64_t)((t)->nhsps_nl + (t)->nhsps_nr + 1)])

/* one bundle, serial, vector element type T, block size nb */
#define DEFINE_BUNDLE(T, NAME)                                                           \
static void NAME(const bsg_tables *t, int64_t ib, const T *vin, T *vout, int nb) {        \
    const int op = t->optype[ib];                                                        \
    const int hc = t->hchar[ib];                                                         \
    const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib];                              \
    const int64_t nx0 = t->nxstart[ib], nx1 = t->nxend[ib];                              \
    const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;                          \
    if (op == BSG_OP_SPE) {                                                              \
        for (int64_t ip = px0; ip <= px1; ++ip) {                                        \
            const float pspe = t->pspe_h[ip - 1];                                        \
            int64_t statef = t->pstart[ip - 1] + t->nstart[nx0 - 1];                     \
            for (int64_t in = nx0; in <= nx1; ++in) {                                    \
                const float nspe = t->nspe_h[in - 1];                                    \
                const float e = pspe + nspe;                                             \
                for (int v = 0; v < nb; ++v)                                             \
                    vout[(statef - 1) * nb + v] += vin[(statef - 1) * nb + v] * (T)e;    \
                ++statef;                                                                \
            }                                                                            \
        }                                                                                \
    } else if (op == BSG_OP_NN) {                                                        \
        const int64_t *s1 = hc == 'b' ? t->n2b_fsd : t->n2b_isd;                         \
        const int64_t *s2 = hc == 'b' ? t->n2b_isd : t->n2b_fsd;                         \
        for (int64_t csd = px0; csd <= px1; csd += cs) {                                 \
            const int64_t psd = t->pstart[csd - 1];                                      \
            for (int64_t x = nx0; x <= nx1; ++x) {                                       \
                float xme = t->hmatnn[t->n2b_op[x - 1] - 1];                             \
                xme = xme * (float)t->n2b_phase[x - 1];                                  \
                const int64_t si = s1[x - 1] + psd, sf = s2[x - 1] + psd;                \
                for (int v = 0; v < nb; ++v)                                             \
                    vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];          \
            }                                                                            \
        }                                                                                \
    } else if (op == BSG_OP_PP) {                                                        \
        const int64_t *s1 = hc == 'b' ? t->p2b_fsd : t->p2b_isd;                         \
        const int64_t *s2 = hc == 'b' ? t->p2b_isd : t->p2b_fsd;                         \
        for (int64_t x = px0; x <= px1; ++x) {                                           \
            float xme = t->hmatpp[t->p2b_op[x - 1] - 1];                                 \
            xme = xme * (float)t->p2b_phase[x - 1];                                      \
            const int64_t psdi = s1[x - 1], psdf = s2[x - 1];                            \
            for (int64_t csd = nx0; csd <= nx1; csd += cs) {                             \
                const int64_t nsd = t->nstart[csd - 1];                                  \
                const int64_t sf = psdf + nsd, si = psdi + nsd;                          \
                for (int v = 0; v < nb; ++v)                                             \
                    vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];          \
            }                                                                            \
        }                                                                                \
    } else if (op == BSG_OP_PN) {                                                        \
        for (int64_t pj = px0; pj <= px1; ++pj) {                                        \
            const int64_t psdi = t->p1b_isd[pj - 1], psdf = t->p1b_fsd[pj - 1];          \
            const int phasep = t->p1b_phase[pj - 1];                                     \
            const int a = t->p1b_cop[pj - 1], c = t->p1b_dop[pj - 1];                    \
            for (int64_t nj = nx0; nj <= nx1; ++nj) {                                    \
                const int b = t->n1b_cop[nj - 1], d = t->n1b_dop[nj - 1];                \
                const int phasen = t->n1b_phase[nj - 1];                                 \
                float xme = t->hmatpn[CPN(t, b, a) + DPN(t, d, c) - 1];                  \
                xme = xme * (float)phasep * (float)phasen;                               \
                const int64_t sf = t->n1b_fsd[nj - 1] + psdf;                            \
                const int64_t si = t->n1b_isd[nj - 1] + psdi;                            \
                if (hc != 'b') {                                                         \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];      \
                } else {                                                                 \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(si - 1) * nb + v] += (T)xme * vin[(sf - 1) * nb + v];      \
                }                                                                        \
            }                                                                            \
        }                                                                                \
    }                                                                                    \
}

DEFINE_BUNDLE(float, bundle_f32)
DEFINE_BUNDLE(double, bundle_f64)

/* vout += H vin over all opbundles, in table order (one thread) */
int oracle_applyh(const bsg_tables *t, const void *vin, void *vout, int nb, int prec) {
    if (!t || !vin || !vout || nb < 1) return BSG_ERR_ARG;
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        if (prec == BSG_PREC_FP32)
            bundle_f32(t, ib, (const float *)vin, (float *)vout, nb);
        else
            bundle_f64(t, ib, (const double *)vin, (double *)vout, nb);
    }
    return BSG_OK;
}

/* ------------------------------------------------------ three-body ---- */
/* The serial bundle loops of a three-body run (applyHbundled_g with
 * threebody set, src/bapplyhlib1.f90:160-235; block forms
 * src/bapplyhblocklib.f90:741-1541):
 *   PPP  applyhPPPbundled_g   (src/bapplyhlib1.f90:1390-1572)
 *   NNN  applyhNNNbundled_g   (:1579-1756)
 *   PNN  applyhPNNbundled_g   (:2033-2285)
 *   PPN  applyhPPNbundled_g   (:2295-2562)
 * xme real(4) = hmat * phase(s), vout(statef) += xme * vin(statei) for 'f',
 * the transpose for 'b'. */
#define TRIP(tab, np_, lab, sp, nl) ((tab)[(int64_t)((lab) - 1) + (int64_t)((sp) + (nl)) * (int64_t)(np_)])
#define DEFINE_BUNDLE3(T, NAME)                                                          \
static void NAME(const bsg_tables *t, const bsg_tables3 *u, int64_t ib, const T *vin,      \
                 T *vout, int nb) {                                                      \
    const int op = t->optype[ib];                                                        \
    const int hc = t->hchar[ib];                                                         \
    const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib];                              \
    const int64_t nx0 = t->nxstart[ib], nx1 = t->nxend[ib];                              \
    const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;                          \
    if (op == BSG_OP_PPP) {                                                              \
        const int64_t *s1 = hc == 'b' ? u->p3b_fsd : u->p3b_isd;                         \
        const int64_t *s2 = hc == 'b' ? u->p3b_isd : u->p3b_fsd;                         \
        for (int64_t csd = nx0; csd <= nx1; csd += cs) {                                 \
            const int64_t nsd = t->nstart[csd - 1];                                      \
            for (int64_t x = px0; x <= px1; ++x) {                                       \
                float xme = u->hmatppp[u->p3b_op[x - 1] - 1];                            \
                xme = xme * (float)u->p3b_phase[x - 1];                                  \
                const int64_t si = s1[x - 1] + nsd, sf = s2[x - 1] + nsd;                \
                for (int v = 0; v < nb; ++v)                                             \
                    vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];          \
            }                                                                            \
        }                                                                                \
    } else if (op == BSG_OP_NNN) {                                                       \
        const int64_t *s1 = hc == 'b' ? u->n3b_fsd : u->n3b_isd;                         \
        const int64_t *s2 = hc == 'b' ? u->n3b_isd : u->n3b_fsd;                         \
        for (int64_t csd = px0; csd <= px1; csd += cs) {                                 \
            const int64_t psd = t->pstart[csd - 1];                                      \
            for (int64_t x = nx0; x <= nx1; ++x) {                                       \
                float xme = u->hmatnnn[u->n3b_op[x - 1] - 1];                            \
                xme = xme * (float)u->n3b_phase[x - 1];                                  \
                const int64_t si = s1[x - 1] + psd, sf = s2[x - 1] + psd;                \
                for (int v = 0; v < nb; ++v)                                             \
                    vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];          \
            }                                                                            \
        }                                                                                \
    } else if (op == BSG_OP_PPN || op == BSG_OP_PNN) {                                   \
        const int ppn = (op == BSG_OP_PPN);                                              \
        for (int64_t pj = px0; pj <= px1; ++pj) {                                        \
            const int64_t psdi = ppn ? t->p2b_isd[pj - 1] : t->p1b_isd[pj - 1];          \
            const int64_t psdf = ppn ? t->p2b_fsd[pj - 1] : t->p1b_fsd[pj - 1];          \
            const int phasep = ppn ? t->p2b_phase[pj - 1] : t->p1b_phase[pj - 1];        \
            const int pc = ppn ? u->p2b_cop[pj - 1] : t->p1b_cop[pj - 1];                \
            const int pd = ppn ? u->p2b_dop[pj - 1] : t->p1b_dop[pj - 1];                \
            for (int64_t nj = nx0; nj <= nx1; ++nj) {                                    \
                const int phasen = ppn ? t->n1b_phase[nj - 1] : t->n2b_phase[nj - 1];    \
                const int nc = ppn ? t->n1b_cop[nj - 1] : u->n2b_cop[nj - 1];            \
                const int nd = ppn ? t->n1b_dop[nj - 1] : u->n2b_dop[nj - 1];            \
                int64_t lab;                                                             \
                if (ppn)                                                                 \
                    lab = (int64_t)TRIP(u->cppntriplet, u->npairs_p, pc, nc, t->nhsps_nl) + \
                          TRIP(u->dppntriplet, u->npairs_p, pd, nd, t->nhsps_nl);        \
                else                                                                     \
                    lab = (int64_t)TRIP(u->cpnntriplet, u->npairs_n, nc, pc, t->nhsps_pl) + \
                          TRIP(u->dpnntriplet, u->npairs_n, nd, pd, t->nhsps_pl);        \
                float xme = ppn ? u->hmatppn[lab - 1] : u->hmatpnn[lab - 1];             \
                xme = xme * (float)phasep * (float)phasen;                               \
                const int64_t nsdi = ppn ? t->n1b_isd[nj - 1] : t->n2b_isd[nj - 1];      \
                const int64_t nsdf = ppn ? t->n1b_fsd[nj - 1] : t->n2b_fsd[nj - 1];      \
                const int64_t si = nsdi + psdi, sf = nsdf + psdf;                        \
                if (hc != 'b') {                                                         \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];      \
                } else {                                                                 \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(si - 1) * nb + v] += (T)xme * vin[(sf - 1) * nb + v];      \
                }                                                                        \
            }                                                                            \
        }                                                                                \
    }                                                                                    \
}

DEFINE_BUNDLE3(float, bundle3_f32)
DEFINE_BUNDLE3(double, bundle3_f64)

/* vout += H vin for a three-body run: SPE and the three-body bundles, PP /
 * NN / PN bundles skipped (src/bapplyhlib1.f90:107-235) */
int oracle_applyh3(const bsg_tables *t, const bsg_tables3 *u, const void *vin, void *vout, int nb, int prec) {
    if (!t || !u || !vin || !vout || nb < 1) return BSG_ERR_ARG;
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        const int op = t->optype[ib];
        if (op == BSG_OP_PP || op == BSG_OP_NN || op == BSG_OP_PN) continue;
        if (op == BSG_OP_SPE) {
            if (prec == BSG_PREC_FP32)
                bundle_f32(t, ib, (const float *)vin, (float *)vout, nb);
            else
                bundle_f64(t, ib, (const double *)vin, (double *)vout, nb);
        } else if (prec == BSG_PREC_FP32) {
            bundle3_f32(t, u, ib, (const float *)vin, (float *)vout, nb);
        } else {
            bundle3_f64(t, u, ib, (const double *)vin, (double *)vout, nb);
        }
    }
    return BSG_OK;
}

/* the same for the listed bundles only (0-based indices): a bounded sample
 * of one matvec for the timed CPU baseline */
int oracle_applyh3_bundles(const bsg_tables *t, const bsg_tables3 *u, const void *vin, void *vout, int nb, int prec,
                           const int64_t *list, int64_t nlist) {
    if (!t || !u || !vin || !vout || nb < 1 || (nlist > 0 && !list)) return BSG_ERR_ARG;
    for (int64_t k = 0; k < nlist; ++k) {
        const int64_t ib = list[k];
        if (ib < 0 || ib >= t->nbundles) return BSG_ERR_ARG;
        const int op = t->optype[ib];
        if (op == BSG_OP_PP || op == BSG_OP_NN || op == BSG_OP_PN) continue;
        if (op == BSG_OP_SPE) {
            if (prec == BSG_PREC_FP32)
                bundle_f32(t, ib, (const float *)vin, (float *)vout, nb);
            else
                bundle_f64(t, ib, (const double *)vin, (double *)vout, nb);
        } else if (prec == BSG_PREC_FP32) {
            bundle3_f32(t, u, ib, (const float *)vin, (float *)vout, nb);
        } else {
            bundle3_f64(t, u, ib, (const double *)vin, (double *)vout, nb);
        }
    }
    return BSG_OK;
}

/* inner-loop updates of each three-body kind: ops[0..3] = PPP, NNN, PPN, PNN */
void oracle_count_ops3(const bsg_tables *t, int64_t *ops) {
    for (int k = 0; k < 4; ++k) ops[k] = 0;
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        const int op = t->optype[ib];
        const int64_t np_ = t->pxend[ib] - t->pxstart[ib] + 1, nn_ = t->nxend[ib] - t->nxstart[ib] + 1;
        const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;
        if (np_ <= 0 || nn_ <= 0) continue;
        if (op == BSG_OP_PPP) ops[0] += np_ * ((nn_ + cs - 1) / cs);
        else if (op == BSG_OP_NNN) ops[1] += ((np_ + cs - 1) / cs) * nn_;
        else if (op == BSG_OP_PPN) ops[2] += np_ * nn_;
        else if (op == BSG_OP_PNN) ops[3] += np_ * nn_;
    }
}

/* ----------------------------------------------------------- OpenMP ---- */
/* chunk boundaries of [lo, hi] (1-based, inclusive) into at most nthr pieces,
 * each cut moved forward until key[] changes (src/bsortjumpslib.f90:491-713
 * makes the same kind of cut for startp_thread / startn_thread) */
static int cut_ranges(int64_t lo, int64_t hi, const int64_t *key, int nthr, int64_t *starts) {
    const int64_t n = hi - lo + 1;
    int k = 0;
    starts[k++] = lo;
    for (int th = 1; th < nthr; ++th) {
        int64_t c = lo + (n * th) / nthr;
        if (c <= starts[k - 1]) continue;
        while (c <= hi && key[c - 1] == key[c - 2]) ++c;
        if (c > hi) break;
        if (c > starts[k - 1]) starts[k++] = c;
    }
    starts[k] = hi + 1;
    return k;
}

#define DEFINE_OMP(T, NAME)                                                              \
static void NAME(const bsg_tables *t, const T *vin, T *vout, int nb, int nthr,           \
                 int64_t *cuts) {                                                        \
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {                                       \
        const int op = t->optype[ib];                                                    \
        const int hc = t->hchar[ib];                                                     \
        const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib];                          \
        const int64_t nx0 = t->nxstart[ib], nx1 = t->nxend[ib];                          \
        const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;                      \
        if (op == BSG_OP_PP) {                                                           \
            const int64_t *s1 = hc == 'b' ? t->p2b_fsd : t->p2b_isd;                     \
            const int64_t *s2 = hc == 'b' ? t->p2b_isd : t->p2b_fsd;                     \
            const int64_t nc = (nx1 + cs - nx0) / cs;                                    \
            _Pragma("omp parallel num_threads(nthr)")                                    \
            {                                                                            \
                int me = 0, nt = 1;                                                      \
                OMP_IDS(me, nt);                                                         \
                const int64_t chunk = (nc + nt - 1) / nt;                                \
                const int64_t i0 = (int64_t)me * chunk, i1 = i0 + chunk < nc ? i0 + chunk : nc; \
                for (int64_t x = px0; x <= px1; ++x) {                                   \
                    float xme = t->hmatpp[t->p2b_op[x - 1] - 1];                         \
                    xme = xme * (float)t->p2b_phase[x - 1];                              \
                    const int64_t psdi = s1[x - 1], psdf = s2[x - 1];                    \
                    for (int64_t ic = i0; ic < i1; ++ic) {                               \
                        const int64_t nsd = t->nstart[nx0 + ic * cs - 1];                \
                        const int64_t sf = psdf + nsd, si = psdi + nsd;                  \
                        for (int v = 0; v < nb; ++v)                                     \
                            vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];  \
                    }                                                                    \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_NN) {                                                    \
            const int64_t *s1 = hc == 'b' ? t->n2b_fsd : t->n2b_isd;                     \
            const int64_t *s2 = hc == 'b' ? t->n2b_isd : t->n2b_fsd;                     \
            const int64_t nc = (px1 + cs - px0) / cs;                                    \
            _Pragma("omp parallel for schedule(static) num_threads(nthr)")               \
            for (int64_t ic = 0; ic < nc; ++ic) {                                        \
                const int64_t psd = t->pstart[px0 + ic * cs - 1];                        \
                for (int64_t x = nx0; x <= nx1; ++x) {                                   \
                    float xme = t->hmatnn[t->n2b_op[x - 1] - 1];                         \
                    xme = xme * (float)t->n2b_phase[x - 1];                              \
                    const int64_t si = s1[x - 1] + psd, sf = s2[x - 1] + psd;            \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];      \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_PN && hc != 'b') {                                       \
            const int k = cut_ranges(px0, px1, t->p1b_fsd, nthr, cuts);                  \
            _Pragma("omp parallel for schedule(dynamic,1) num_threads(nthr)")            \
            for (int th = 0; th < k; ++th) {                                             \
                for (int64_t pj = cuts[th]; pj < cuts[th + 1]; ++pj) {                   \
                    const int64_t psdi = t->p1b_isd[pj - 1], psdf = t->p1b_fsd[pj - 1];  \
                    const int phasep = t->p1b_phase[pj - 1];                             \
                    const int a = t->p1b_cop[pj - 1], c = t->p1b_dop[pj - 1];            \
                    for (int64_t nj = nx0; nj <= nx1; ++nj) {                            \
                        const int b = t->n1b_cop[nj - 1], d = t->n1b_dop[nj - 1];        \
                        float xme = t->hmatpn[CPN(t, b, a) + DPN(t, d, c) - 1];          \
                        xme = xme * (float)phasep * (float)t->n1b_phase[nj - 1];         \
                        const int64_t sf = t->n1b_fsd[nj - 1] + psdf;                    \
                        const int64_t si = t->n1b_isd[nj - 1] + psdi;                    \
                        for (int v = 0; v < nb; ++v)                                     \
                            vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];  \
                    }                                                                    \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_PN) {                                                    \
            const int k = cut_ranges(nx0, nx1, t->n1b_isd, nthr, cuts);                  \
            _Pragma("omp parallel for schedule(dynamic,1) num_threads(nthr)")            \
            for (int th = 0; th < k; ++th) {                                             \
                for (int64_t nj = cuts[th]; nj < cuts[th + 1]; ++nj) {                   \
                    const int64_t nsdi = t->n1b_isd[nj - 1], nsdf = t->n1b_fsd[nj - 1];  \
                    const int b = t->n1b_cop[nj - 1], d = t->n1b_dop[nj - 1];            \
                    const int phasen = t->n1b_phase[nj - 1];                             \
                    for (int64_t pj = px0; pj <= px1; ++pj) {                            \
                        const int a = t->p1b_cop[pj - 1], c = t->p1b_dop[pj - 1];        \
                        float xme = t->hmatpn[CPN(t, b, a) + DPN(t, d, c) - 1];          \
                        xme = xme * (float)t->p1b_phase[pj - 1] * (float)phasen;         \
                        const int64_t si = nsdi + t->p1b_isd[pj - 1];                    \
                        const int64_t sf = nsdf + t->p1b_fsd[pj - 1];                    \
                        for (int v = 0; v < nb; ++v)                                     \
                            vout[(si - 1) * nb + v] += (T)xme * vin[(sf - 1) * nb + v];  \
                    }                                                                    \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_SPE) {                                                   \
            const int64_t np_ = px1 - px0 + 1;                                           \
            _Pragma("omp parallel for schedule(static) num_threads(nthr)")               \
            for (int64_t k2 = 0; k2 < np_; ++k2) {                                       \
                const int64_t ip = px0 + k2;                                             \
                const float pspe = t->pspe_h[ip - 1];                                    \
                int64_t statef = t->pstart[ip - 1] + t->nstart[nx0 - 1];                 \
                for (int64_t in = nx0; in <= nx1; ++in) {                                \
                    const float e = pspe + t->nspe_h[in - 1];                            \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(statef - 1) * nb + v] += vin[(statef - 1) * nb + v] * (T)e; \
                    ++statef;                                                            \
                }                                                                        \
            }                                                                            \
        }                                                                                \
    }                                                                                    \
}

#ifdef _OPENMP
#define OMP_IDS(me, nt) do { me = omp_get_thread_num(); nt = omp_get_num_threads(); } while (0)
#else
#define OMP_IDS(me, nt) do { me = 0; nt = 1; } while (0)
#endif

DEFINE_OMP(float, omp_f32)
DEFINE_OMP(double, omp_f64)

/* vout += H vin with nthreads OpenMP threads (the CPU baseline) */
int oracle_applyh_omp(const bsg_tables *t, const void *vin, void *vout, int nb, int prec, int nthreads) {
    if (!t || !vin || !vout || nb < 1) return BSG_ERR_ARG;
    if (nthreads < 1) nthreads = 1;
    int64_t *cuts = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nthreads + 2));
    if (!cuts) return BSG_ERR_NOMEM;
    if (prec == BSG_PREC_FP32)
        omp_f32(t, (const float *)vin, (float *)vout, nb, nthreads, cuts);
    else
        omp_f64(t, (const double *)vin, (double *)vout, nb, nthreads, cuts);
    free(cuts);
    return BSG_OK;
}

/* ------------------------------------------ owner-computes partition ---- */
/* applyHbundled_omp gives each OpenMP thread the output rows whose pstart
 * value lies in [mybasisstart-1, mybasisstop) (getLoadDist buckets the work
 * of every jump by the pstart value of its output row and cuts the buckets
 * into equal-work runs, src/bapplyhlibOMP.f90:34-868); per bundle the thread
 * visits the jumps whose output row is its own (threadStart/threadStop, and
 * the rescans of the 'b' bundles that keep psdi in range, :1340-1356).
 * oracle_applyh_rows() is one owner's share: the outputs of the rows whose
 * pstart value r satisfies lo <= r < hi, in bundle order, every other output
 * untouched.  Output row of a jump: PP psdf (psdi for 'b'), NN and SPE
 * pstart(ip), PN p1b_fsd ('b': p1b_isd).  Rows are contiguous runs of basis
 * states (a proton SD and its neutron partners), so disjoint [lo, hi) ranges
 * write disjoint outputs. */
#define DEFINE_ROWS(T, NAME)                                                             \
static void NAME(const bsg_tables *t, const T *vin, T *vout, int nb, int64_t lo, int64_t hi) { \
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {                                       \
        const int op = t->optype[ib];                                                    \
        const int hc = t->hchar[ib];                                                     \
        const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib];                          \
        const int64_t nx0 = t->nxstart[ib], nx1 = t->nxend[ib];                          \
        const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;                      \
        if (op == BSG_OP_SPE) {                                                          \
            for (int64_t ip = px0; ip <= px1; ++ip) {                                    \
                const int64_t row = t->pstart[ip - 1];                                   \
                if (row < lo || row >= hi) continue;                                     \
                const float pspe = t->pspe_h[ip - 1];                                    \
                int64_t statef = row + t->nstart[nx0 - 1];                               \
                for (int64_t in = nx0; in <= nx1; ++in) {                                \
                    const float e = pspe + t->nspe_h[in - 1];                            \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(statef - 1) * nb + v] += vin[(statef - 1) * nb + v] * (T)e; \
                    ++statef;                                                            \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_NN) {                                                    \
            const int64_t *s1 = hc == 'b' ? t->n2b_fsd : t->n2b_isd;                     \
            const int64_t *s2 = hc == 'b' ? t->n2b_isd : t->n2b_fsd;                     \
            for (int64_t csd = px0; csd <= px1; csd += cs) {                             \
                const int64_t psd = t->pstart[csd - 1];                                  \
                if (psd < lo || psd >= hi) continue;                                     \
                for (int64_t x = nx0; x <= nx1; ++x) {                                   \
                    float xme = t->hmatnn[t->n2b_op[x - 1] - 1];                         \
                    xme = xme * (float)t->n2b_phase[x - 1];                              \
                    const int64_t si = s1[x - 1] + psd, sf = s2[x - 1] + psd;            \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];      \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_PP) {                                                    \
            const int64_t *s1 = hc == 'b' ? t->p2b_fsd : t->p2b_isd;                     \
            const int64_t *s2 = hc == 'b' ? t->p2b_isd : t->p2b_fsd;                     \
            for (int64_t x = px0; x <= px1; ++x) {                                       \
                const int64_t psdi = s1[x - 1], psdf = s2[x - 1];                        \
                if (psdf < lo || psdf >= hi) continue;                                   \
                float xme = t->hmatpp[t->p2b_op[x - 1] - 1];                             \
                xme = xme * (float)t->p2b_phase[x - 1];                                  \
                for (int64_t csd = nx0; csd <= nx1; csd += cs) {                         \
                    const int64_t nsd = t->nstart[csd - 1];                              \
                    const int64_t sf = psdf + nsd, si = psdi + nsd;                      \
                    for (int v = 0; v < nb; ++v)                                         \
                        vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];      \
                }                                                                        \
            }                                                                            \
        } else if (op == BSG_OP_PN) {                                                    \
            const int bwd = hc == 'b';                                                   \
            for (int64_t pj = px0; pj <= px1; ++pj) {                                    \
                const int64_t psdi = t->p1b_isd[pj - 1], psdf = t->p1b_fsd[pj - 1];      \
                const int64_t own = bwd ? psdi : psdf;                                   \
                if (own < lo || own >= hi) continue;                                     \
                const int phasep = t->p1b_phase[pj - 1];                                 \
                const int a = t->p1b_cop[pj - 1], c = t->p1b_dop[pj - 1];                \
                for (int64_t nj = nx0; nj <= nx1; ++nj) {                                \
                    const int b = t->n1b_cop[nj - 1], d = t->n1b_dop[nj - 1];            \
                    float xme = t->hmatpn[CPN(t, b, a) + DPN(t, d, c) - 1];              \
                    xme = xme * (float)phasep * (float)t->n1b_phase[nj - 1];             \
                    const int64_t sf = t->n1b_fsd[nj - 1] + psdf;                        \
                    const int64_t si = t->n1b_isd[nj - 1] + psdi;                        \
                    if (!bwd) {                                                          \
                        for (int v = 0; v < nb; ++v)                                     \
                            vout[(sf - 1) * nb + v] += (T)xme * vin[(si - 1) * nb + v];  \
                    } else {                                                             \
                        for (int v = 0; v < nb; ++v)                                     \
                            vout[(si - 1) * nb + v] += (T)xme * vin[(sf - 1) * nb + v];  \
                    }                                                                    \
                }                                                                        \
            }                                                                            \
        }                                                                                \
    }                                                                                    \
}

DEFINE_ROWS(float, rows_f32)
DEFINE_ROWS(double, rows_f64)

static int cmp_i64(const void *x, const void *y) {
    const int64_t a = *(const int64_t *)x, b = *(const int64_t *)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* index of the row whose start value is r in the ascending list rs[n] */
static int64_t row_index(const int64_t *rs, int64_t n, int64_t r) {
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) / 2;
        if (rs[mid] <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* The work getLoadDist buckets, per output row: row_start[] receives the
 * distinct pstart values in ascending order (the rows), ops[] the inner-loop
 * updates landing in each row (the bucket counts of src/bapplyhlibOMP.f90
 * :213-327 at row granularity).  Both arrays need nsd_p entries; returns the
 * number of rows. */
int64_t oracle_row_ops(const bsg_tables *t, int64_t *row_start, int64_t *ops) {
    int64_t n = t->nsd_p;
    memcpy(row_start, t->pstart, sizeof(int64_t) * (size_t)n);
    qsort(row_start, (size_t)n, sizeof(int64_t), cmp_i64);
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i)
        if (m == 0 || row_start[i] != row_start[m - 1]) row_start[m++] = row_start[i];
    memset(ops, 0, sizeof(int64_t) * (size_t)m);
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        const int op = t->optype[ib], hc = t->hchar[ib];
        const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib];
        const int64_t nx0 = t->nxstart[ib], nx1 = t->nxend[ib];
        const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;
        if (op == BSG_OP_SPE) {
            for (int64_t ip = px0; ip <= px1; ++ip) ops[row_index(row_start, m, t->pstart[ip - 1])] += nx1 - nx0 + 1;
        } else if (op == BSG_OP_NN) {
            for (int64_t csd = px0; csd <= px1; csd += cs) ops[row_index(row_start, m, t->pstart[csd - 1])] += nx1 - nx0 + 1;
        } else if (op == BSG_OP_PP) {
            const int64_t *s2 = hc == 'b' ? t->p2b_isd : t->p2b_fsd;
            const int64_t nc = (nx1 + cs - nx0) / cs;
            for (int64_t x = px0; x <= px1; ++x) ops[row_index(row_start, m, s2[x - 1])] += nc;
        } else if (op == BSG_OP_PN) {
            const int64_t *own = hc == 'b' ? t->p1b_isd : t->p1b_fsd;
            for (int64_t pj = px0; pj <= px1; ++pj) ops[row_index(row_start, m, own[pj - 1])] += nx1 - nx0 + 1;
        }
    }
    return m;
}

/* vout += H vin restricted to the rows with pstart value in [lo, hi) */
int oracle_applyh_rows(const bsg_tables *t, const void *vin, void *vout, int nb, int prec, int64_t lo, int64_t hi) {
    if (!t || !vin || !vout || nb < 1) return BSG_ERR_ARG;
    if (prec == BSG_PREC_FP32)
        rows_f32(t, (const float *)vin, (float *)vout, nb, lo, hi);
    else
        rows_f64(t, (const double *)vin, (double *)vout, nb, lo, hi);
    return BSG_OK;
}

/* The owner-computes matvec: range i is [bounds[2i], bounds[2i+1]) of row
 * start values, one range per OpenMP work item (dynamic schedule).  With
 * equal-work ranges that cover every row this is applyHbundled_omp's
 * partition; ranges that cover part of the rows compute those rows only. */
int oracle_applyh_owner(const bsg_tables *t, const void *vin, void *vout, int nb, int prec,
                        int nranges, const int64_t *bounds, int nthreads) {
    if (!t || !vin || !vout || nb < 1 || nranges < 0 || !bounds) return BSG_ERR_ARG;
    if (nthreads < 1) nthreads = 1;
    int st = BSG_OK;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int i = 0; i < nranges; ++i) {
        const int r = oracle_applyh_rows(t, vin, vout, nb, prec, bounds[2 * i], bounds[2 * i + 1]);
        if (r) st = r;
    }
    return st;
}

/* number of inner-loop updates one applyH executes (the N_ops of the
 * algorithmic-bytes model) split by optype */
void oracle_count_ops(const bsg_tables *t, int64_t *ops /* [4]: spe, pp, nn, pn */) {
    ops[0] = ops[1] = ops[2] = ops[3] = 0;
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;
        const int64_t np_ = t->pxend[ib] - t->pxstart[ib] + 1;
        const int64_t nn_ = t->nxend[ib] - t->nxstart[ib] + 1;
        switch (t->optype[ib]) {
        case BSG_OP_SPE: ops[0] += np_ * nn_; break;
        case BSG_OP_PP: ops[1] += np_ * ((nn_ + cs - 1) / cs); break;
        case BSG_OP_NN: ops[2] += ((np_ + cs - 1) / cs) * nn_; break;
        case BSG_OP_PN: ops[3] += np_ * nn_; break;
        }
    }
}

/* Two-body densities with both vectors equal to psi (FP64), the traversal of
 * applyh{PP,NN,PN}bundled_den (src/bdenslib4.f90:129-729): for every bundle
 * and every jump pair, dmat(label) += psi(f) * psi(i) * phase.  With the
 * Hamiltonian's own bundles this is dE/dhmat(label) (Hellmann-Feynman). SPE
 * bundles give d/dpspe_h and d/dnspe_h.  Outputs are accumulated (caller
 * zeroes them). */
int oracle_density(const bsg_tables *t, const double *psi, double *dpp, double *dnn, double *dpn,
                   double *dspe_p, double *dspe_n) {
    if (!t || !psi) return BSG_ERR_ARG;
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        const int op = t->optype[ib], hc = t->hchar[ib];
        const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib];
        const int64_t nx0 = t->nxstart[ib], nx1 = t->nxend[ib];
        const int64_t cs = t->cstride[ib] > 0 ? t->cstride[ib] : 1;
        if (op == BSG_OP_PP) {
            const int64_t *s1 = hc == 'b' ? t->p2b_fsd : t->p2b_isd;
            const int64_t *s2 = hc == 'b' ? t->p2b_isd : t->p2b_fsd;
            for (int64_t x = px0; x <= px1; ++x) {
                double s = 0.0;
                for (int64_t csd = nx0; csd <= nx1; csd += cs) {
                    const int64_t nsd = t->nstart[csd - 1];
                    s += psi[s2[x - 1] + nsd - 1] * psi[s1[x - 1] + nsd - 1];
                }
                dpp[t->p2b_op[x - 1] - 1] += s * t->p2b_phase[x - 1];
            }
        } else if (op == BSG_OP_NN) {
            const int64_t *s1 = hc == 'b' ? t->n2b_fsd : t->n2b_isd;
            const int64_t *s2 = hc == 'b' ? t->n2b_isd : t->n2b_fsd;
            for (int64_t csd = px0; csd <= px1; csd += cs) {
                const int64_t psd = t->pstart[csd - 1];
                for (int64_t x = nx0; x <= nx1; ++x)
                    dnn[t->n2b_op[x - 1] - 1] += psi[s2[x - 1] + psd - 1] * psi[s1[x - 1] + psd - 1] * t->n2b_phase[x - 1];
            }
        } else if (op == BSG_OP_PN) {
            for (int64_t pj = px0; pj <= px1; ++pj) {
                const int a = t->p1b_cop[pj - 1], c = t->p1b_dop[pj - 1];
                for (int64_t nj = nx0; nj <= nx1; ++nj) {
                    const int b = t->n1b_cop[nj - 1], d = t->n1b_dop[nj - 1];
                    const int64_t lab = CPN(t, b, a) + DPN(t, d, c);
                    const int64_t sf = t->n1b_fsd[nj - 1] + t->p1b_fsd[pj - 1];
                    const int64_t si = t->n1b_isd[nj - 1] + t->p1b_isd[pj - 1];
                    dpn[lab - 1] += psi[sf - 1] * psi[si - 1] * t->p1b_phase[pj - 1] * t->n1b_phase[nj - 1];
                }
            }
        } else if (op == BSG_OP_SPE && dspe_p && dspe_n) {
            for (int64_t ip = px0; ip <= px1; ++ip) {
                int64_t statef = t->pstart[ip - 1] + t->nstart[nx0 - 1];
                for (int64_t in = nx0; in <= nx1; ++in) {
                    const double p2 = psi[statef - 1] * psi[statef - 1];
                    dspe_p[ip - 1] += p2;
                    dspe_n[in - 1] += p2;
                    ++statef;
                }
            }
        }
    }
    return BSG_OK;
}
