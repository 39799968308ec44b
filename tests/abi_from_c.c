/*
 * abi_from_c.c -- a C caller of the two libraries through the headers
 * bsg.h and bsg_host.h alone, no Python: builds the tables of a model
 * (libbsghost.so), then on the GPU (libbsgpu.so) applies H once to host
 * vectors and runs Lanczos, the two calls a BIGSTICK host makes in place of
 * applyHbundled_omp (src/bapplyhlibOMP.f90:882) and lanczos_p
 * (src/blanczosmain.f90:1413).
 *
 *   abi_from_c SPEC VOUT
 *
 * SPEC is a text file:
 *   norb np nn jz2 parity spe_scale tbme_scale
 *   nr l j2 w spe                 (norb lines, the orbits of an .sps file)
 *   ntbme
 *   a b c d J T V                 (ntbme lines, as in an isospin .int file)
 * The program writes H vin (dim doubles, vin[i] = sin(0.1 i + 1)) to VOUT
 * and prints "dim D" and "eval K E" lines (five lowest states).  Any failing
 * call prints its status and message and exits 1.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "bsg.h"
#include "bsg_host.h"

#define NKEEP 5

static int fail_host(const char *what, int st)
{
    fprintf(stderr, "%s: %s: %s\n", what, bsg_strerror(st), bsg_host_last_error());
    return 1;
}

static int fail_ctx(const char *what, int st, const bsg_ctx *ctx)
{
    char msg[512] = "";
    if (ctx) bsg_last_error(ctx, msg, sizeof msg);
    fprintf(stderr, "%s: %s: %s\n", what, bsg_strerror(st), msg);
    return 1;
}

static int read_spec(FILE *f, bsg_model_spec *ms, bsg_orbit **orbs, double **spe, bsg_tbme **tb)
{
    if (fscanf(f, "%d %d %d %d %d %lf %lf", &ms->norb, &ms->np, &ms->nn, &ms->jz2,
               &ms->parity, &ms->spe_scale, &ms->tbme_scale) != 7 || ms->norb <= 0)
        return -1;
    *orbs = calloc((size_t)ms->norb, sizeof **orbs);
    *spe = calloc((size_t)ms->norb, sizeof **spe);
    if (!*orbs || !*spe) return -1;
    for (int i = 0; i < ms->norb; i++) {
        bsg_orbit *o = &(*orbs)[i];
        if (fscanf(f, "%d %d %d %d %lf", &o->nr, &o->l, &o->j2, &o->w, &(*spe)[i]) != 5)
            return -1;
    }
    if (fscanf(f, "%d", &ms->ntbme) != 1 || ms->ntbme < 0) return -1;
    *tb = calloc((size_t)(ms->ntbme > 0 ? ms->ntbme : 1), sizeof **tb);
    if (!*tb) return -1;
    for (int i = 0; i < ms->ntbme; i++) {
        bsg_tbme *t = &(*tb)[i];
        if (fscanf(f, "%d %d %d %d %d %d %lf", &t->a, &t->b, &t->c, &t->d, &t->J, &t->T,
                   &t->v) != 7)
            return -1;
    }
    ms->orbits = *orbs;
    ms->spe = *spe;
    ms->tbme = *tb;
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s SPEC VOUT\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "r");
    if (!f) {
        perror(argv[1]);
        return 1;
    }
    bsg_model_spec ms = {0};
    bsg_orbit *orbs = NULL;
    double *spe = NULL;
    bsg_tbme *tb = NULL;
    int bad = read_spec(f, &ms, &orbs, &spe, &tb);
    fclose(f);
    if (bad) {
        fprintf(stderr, "%s: malformed spec\n", argv[1]);
        return 1;
    }

    bsg_host_tables *h = NULL;
    int st = bsg_host_build(&ms, &h);
    if (st != BSG_OK) return fail_host("bsg_host_build", st);

    bsg_config cfg = {0};
    cfg.device = 0;
    cfg.max_nb = 1;
    cfg.validate = 1;
    bsg_ctx *ctx = NULL;
    st = bsg_create(&h->t, &cfg, &ctx);
    if (st != BSG_OK) return fail_ctx("bsg_create", st, ctx);

    int64_t dim = h->t.dimbasis;
    double *vin = malloc((size_t)dim * sizeof *vin);
    double *vout = malloc((size_t)dim * sizeof *vout);
    if (!vin || !vout) return 1;
    for (int64_t i = 0; i < dim; i++) vin[i] = sin(0.1 * (double)i + 1.0);
    st = bsg_applyh(ctx, vin, vout, 1, BSG_PREC_FP64, 0);
    if (st != BSG_OK) return fail_ctx("bsg_applyh", st, ctx);

    FILE *o = fopen(argv[2], "wb");
    if (!o || fwrite(vout, sizeof *vout, (size_t)dim, o) != (size_t)dim) {
        perror(argv[2]);
        return 1;
    }
    fclose(o);

    bsg_lanczos_params p = {0};
    p.nkeep = NKEEP;
    p.niter = 300;
    p.nb = 1;
    p.matvec_prec = BSG_PREC_FP64;
    p.ncheck = NKEEP + 5;
    p.converge_tol = 1e-3;
    p.pivot = 0;
    p.seed = 12345;
    p.lanc_prec = BSG_PREC_FP64;
    double evals[NKEEP];
    bsg_report rep;
    st = bsg_lanczos(ctx, &p, NULL, evals, NULL, &rep);
    if (st != BSG_OK) return fail_ctx("bsg_lanczos", st, ctx);

    printf("dim %lld\n", (long long)dim);
    for (int k = 0; k < NKEEP; k++) printf("eval %d %.17g\n", k, evals[k]);
    printf("iterations %d converged %d\n", rep.total_iterations, rep.converged);

    st = bsg_destroy(ctx);
    if (st != BSG_OK) return fail_ctx("bsg_destroy", st, NULL);
    bsg_host_free(h);
    free(vin);
    free(vout);
    free(orbs);
    free(spe);
    free(tb);
    return 0;
}
