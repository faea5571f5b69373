/*
 * ice_oracle.c -- TEST INFRASTRUCTURE: the CPU FP64 oracle of ICE's Eulerian
 * dispersed-phase time step (Explicit_Step, src/lib/numerics/time/explicit/
 * Mod_Explicit.f90:11-245) and of the set-up maps it reads (Pair_Connections,
 * io/IO_BC.f90:360-510; build_local_bc_index / collect_boundary_cells /
 * collect_owner_records, parallel/Mod_GhostExchange.f90:103-360).
 *
 * It is the checker of the CUDA product, never part of it: only tests/, the
 * smoke check and the CPU-baseline leg of bench.py load libice_oracle.so.
 *
 * The arrays keep the Fortran layouts of Allocate_Block (variable fastest,
 * gc = 2 ghost layers), every loop keeps the reference's order where the order
 * changes bits (boundary records in face order, then the interior faces of each
 * direction odd-then-even, Mod_Fluxes.f90:470-506), and the per-face and
 * per-cell arithmetic is ice_oracle_physics.h. The face fluxes of a direction
 * are computed once into a face buffer and gathered per cell, which gives the
 * bits of the reference's tile sweep for any thread count (OpenMP), as the
 * reference itself does (docs/user/parallel.md:44-46).
 *
 * Entry points mirror include/ice_gpu.h with the prefix orc_ instead of
 * ice_gpu_, so that a test drives the oracle and the CUDA library alike.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdarg.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "ice_oracle_physics.h"

#define MAXF ICE_GPU_MAX_FAMILIES
#define NCM  ICE_GPU_NCOND_MAX

typedef struct {
    double *prim, *prim_old, *residual, *source, *dt, *tau, *beta;
    double *imports;      /* the coupler's rates (nc per interior cell), or NULL */
    double *source_step;  /* two-way coupling: the step's weighted source (nc per interior cell) */
    unsigned char *inj;
} ofam;

typedef struct {
    int ni, nj, nk;
    double *face[3], *vol, *dl, *M;
    double *gprim, *gR, *ggam, *gk, *gmu;
    ofam fam[MAXF];
} oblk;

typedef struct {
    int b, i, j, k, f, type, p, bs, is, js, ks, fs, partner, owner, cf;
    double massflux, velocity, alpha, beta, temperature, radius, gfixed;
    int normal_dir;
    long d0; int n1, n2;  /* chimera: donors d0 .. d0+n1-1 of ghost layer 1, then n2 of layer 2 */
} orec;

typedef struct orc_ctx {
    ice_gpu_params P;
    int nb;
    oblk* blk;
    int nrec;
    orec* bc;
    int nchim, have_chim; /* chimera records and whether their donors are set */
    int have_imp[MAXF];   /* the family has the coupler's imports (set_imports) */
    int exchange;         /* two-way coupling: the step's source is kept (set_exchange) */
    int* cdon;            /* chimera donors: block, i, j, k (1-based) */
    double* cw;           /* their weights */
    int* grp_first;       /* nfam+1, 0-based into grp */
    int* grp;             /* records by family, table order */
    int bn[MAXF]; int* bfirst[MAXF]; int* brec[MAXF];   /* boundary cells (0-based record ids) */
    int nconn[MAXF]; double* connF[MAXF]; int nown[MAXF]; int* own[MAXF];
    double time, dtglobal;
    int iter, iter_from_call;
    long long nfloored;
    int status;
    double residuo[5], residuofam[5*MAXF];
    int have_norm;
    double res_reference; /* the first non-zero density residual of a steady run (0: none yet) */
    int res_end;          /* the last step ended the run on res-threshold */
    double* fbuf;         /* face flux scratch */
    size_t fbuf_n;
    /* the block split (set_partition, set_halo, set_exchange_hook): the blocks this rank steps (NULL:
     * every block), the exchange lists per kind and family, the hook and its buffers */
    int* owned;
    int nhs[3][MAXF], nhr[3][MAXF];
    int *hs[3][MAXF], *hr[3][MAXF];
    ice_gpu_exchange_fn hook;
    void* hook_user;
    double* hbuf;
    size_t hbuf_n;
    char err[512];
} orc_ctx;

/* The block split: a block this rank steps (every block without a partition). */
static inline int OWN(const orc_ctx* c, int b) { return !c->owned || c->owned[b]; }

static const int guide[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};

static int seterr(orc_ctx* c, int code, const char* fmt, ...) {
    if (c) { va_list ap; va_start(ap, fmt); vsnprintf(c->err, sizeof c->err, fmt, ap); va_end(ap); }
    return code;
}

/* index helpers: 1-based Fortran indices */
static inline long CI(const oblk* B, int i, int j, int k) {     /* (1-gc:n+gc)^3 */
    return ((long)(k + 1) * (B->nj + 4) + (j + 1)) * (B->ni + 4) + (i + 1);
}
static inline long II(const oblk* B, int i, int j, int k) {     /* (1:n)^3 */
    return ((long)(k - 1) * B->nj + (j - 1)) * B->ni + (i - 1);
}
static inline long RI(const oblk* B, int i, int j, int k) {     /* (0:n+1)^3 */
    return ((long)k * (B->nj + 2) + j) * (B->ni + 2) + i;
}
static inline long FI(const oblk* B, int d, int i, int j, int k) {
    if (d == 0) return ((long)(k - 1) * B->nj + (j - 1)) * (B->ni + 1) + i;
    if (d == 1) return ((long)(k - 1) * (B->nj + 1) + j) * B->ni + (i - 1);
    return ((long)k * B->nj + (j - 1)) * B->ni + (i - 1);
}
static inline long ncells_g(const oblk* B) { return (long)(B->ni + 4) * (B->nj + 4) * (B->nk + 4); }
static inline long ncells(const oblk* B) { return (long)B->ni * B->nj * B->nk; }
static inline long nring(const oblk* B) { return (long)(B->ni + 2) * (B->nj + 2) * (B->nk + 2); }
static inline long nfaces(const oblk* B, int d) {
    if (d == 0) return (long)(B->ni + 1) * B->nj * B->nk;
    if (d == 1) return (long)B->ni * (B->nj + 1) * B->nk;
    return (long)B->ni * B->nj * (B->nk + 1);
}
static inline int nc_of(const orc_ctx* c, int p) { return o_nbase(c->P.fam[p].closure); }
static inline const double* NRM(const oblk* B, int d, int i, int j, int k) { return B->face[d] + 4*FI(B, d, i, j, k); }

/* ------------------------------------------------------------- lifecycle */
int orc_create(const ice_gpu_params* P, int nb, const int* dims, orc_ctx** out) {
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    if (!c) return ICE_GPU_ENOMEM;
    c->P = *P; c->nb = nb;
    c->blk = (oblk*)calloc(nb, sizeof(oblk));
    for (int b = 0; b < nb; ++b) {
        oblk* B = &c->blk[b];
        B->ni = dims[3*b]; B->nj = dims[3*b+1]; B->nk = dims[3*b+2];
        for (int d = 0; d < 3; ++d) B->face[d] = (double*)calloc(4*nfaces(B, d), sizeof(double));
        B->vol = (double*)calloc(ncells(B), sizeof(double));
        B->dl = (double*)calloc(3*nring(B), sizeof(double));
        B->M = (double*)calloc(9*nring(B), sizeof(double));
        for (int p = 0; p < P->nfam; ++p) {
            int nc = nc_of(c, p);
            ofam* F = &B->fam[p];
            F->prim = (double*)malloc(sizeof(double)*nc*ncells_g(B));
            F->prim_old = (double*)malloc(sizeof(double)*nc*ncells_g(B));
            for (long q = 0; q < nc*ncells_g(B); ++q) { F->prim[q] = NAN; F->prim_old[q] = NAN; }
            F->residual = (double*)calloc(nc*ncells(B), sizeof(double));
            F->source = (double*)calloc(nc*ncells(B), sizeof(double));
            F->dt = (double*)calloc(ncells(B), sizeof(double));
            F->beta = (double*)malloc(sizeof(double)*ncells(B));
            for (long q = 0; q < ncells(B); ++q) F->beta[q] = 1.0;
            F->tau = (double*)malloc(sizeof(double)*ncells_g(B));
            for (long q = 0; q < ncells_g(B); ++q) F->tau[q] = INFINITY;
            F->inj = (unsigned char*)calloc(ncells_g(B), 1);
        }
    }
    *out = c;
    return 0;
}

int orc_destroy(orc_ctx* c) {
    if (!c) return 0;
    for (int b = 0; b < c->nb; ++b) {
        oblk* B = &c->blk[b];
        for (int d = 0; d < 3; ++d) free(B->face[d]);
        free(B->vol); free(B->dl); free(B->M);
        free(B->gprim); free(B->gR); free(B->ggam); free(B->gk); free(B->gmu);
        for (int p = 0; p < c->P.nfam; ++p) {
            ofam* F = &B->fam[p];
            free(F->prim); free(F->prim_old); free(F->residual); free(F->source);
            free(F->dt); free(F->beta); free(F->tau); free(F->inj); free(F->imports); free(F->source_step);
        }
    }
    free(c->blk); free(c->bc); free(c->grp_first); free(c->grp); free(c->cdon); free(c->cw);
    for (int p = 0; p < MAXF; ++p) { free(c->bfirst[p]); free(c->brec[p]); free(c->connF[p]); free(c->own[p]); }
    free(c->fbuf); free(c->hbuf); free(c->owned);
    for (int k = 0; k < 3; ++k) for (int p = 0; p < MAXF; ++p) { free(c->hs[k][p]); free(c->hr[k][p]); }
    free(c);
    return 0;
}

int orc_set_block(orc_ctx* c, int b1, const double* f1, const double* f2, const double* f3,
                  const double* vol, const double* dl, const double* M) {
    if (b1 < 1 || b1 > c->nb) return seterr(c, ICE_GPU_EINVAL, "block %d out of range", b1);
    oblk* B = &c->blk[b1 - 1];
    const double* fs[3] = {f1, f2, f3};
    for (int d = 0; d < 3; ++d) memcpy(B->face[d], fs[d], sizeof(double)*4*nfaces(B, d));
    memcpy(B->vol, vol, sizeof(double)*ncells(B));
    memcpy(B->dl, dl, sizeof(double)*3*nring(B));
    memcpy(B->M, M, sizeof(double)*9*nring(B));
    return 0;
}

int orc_set_gas(orc_ctx* c, int b1, const double* prim5, const double* R, const double* gam,
                const double* k, const double* mu) {
    if (b1 < 1 || b1 > c->nb) return seterr(c, ICE_GPU_EINVAL, "block %d out of range", b1);
    oblk* B = &c->blk[b1 - 1];
    long n = ncells(B);
    free(B->gprim); free(B->gR); free(B->ggam); free(B->gk); free(B->gmu);
    B->gprim = (double*)malloc(sizeof(double)*5*n); memcpy(B->gprim, prim5, sizeof(double)*5*n);
    B->gR = (double*)malloc(sizeof(double)*n); memcpy(B->gR, R, sizeof(double)*n);
    B->ggam = (double*)malloc(sizeof(double)*n); memcpy(B->ggam, gam, sizeof(double)*n);
    B->gk = (double*)malloc(sizeof(double)*n); memcpy(B->gk, k, sizeof(double)*n);
    B->gmu = (double*)malloc(sizeof(double)*n); memcpy(B->gmu, mu, sizeof(double)*n);
    return 0;
}

int orc_upload_state(orc_ctx* c, int b1, int p1, const double* prim, const unsigned char* inj) {
    if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam) return seterr(c, ICE_GPU_EINVAL, "bad block/family");
    oblk* B = &c->blk[b1 - 1];
    ofam* F = &B->fam[p1 - 1];
    int nc = nc_of(c, p1 - 1);
    memcpy(F->prim, prim, sizeof(double)*nc*ncells_g(B));
    if (inj) memcpy(F->inj, inj, ncells_g(B));
    return 0;
}

int orc_download_state(const orc_ctx* c, int b1, int p1, double* prim) {
    const oblk* B = &c->blk[b1 - 1];
    memcpy(prim, B->fam[p1 - 1].prim, sizeof(double)*nc_of(c, p1 - 1)*ncells_g(B));
    return 0;
}

/* tau and dt of the interior cells, for the tests */
int orc_download_aux(const orc_ctx* c, int b1, int p1, double* dt, double* tau, double* beta) {
    const oblk* B = &c->blk[b1 - 1];
    const ofam* F = &B->fam[p1 - 1];
    for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
        long q = II(B, i, j, k);
        if (dt) dt[q] = F->dt[q];
        if (tau) tau[q] = F->tau[CI(B, i, j, k)];
        if (beta) beta[q] = F->beta[q];
    }
    return 0;
}

int orc_set_time(orc_ctx* c, double time, int iter, int iter_from_call) {
    c->time = time; c->iter = iter; c->iter_from_call = iter_from_call;
    return 0;
}

int orc_set_res_reference(orc_ctx* c, double ref) {
    c->res_reference = ref;
    return 0;
}

int orc_get_res_reference(orc_ctx* c, double* ref) {
    if (!ref) return seterr(c, ICE_GPU_EINVAL, "get_res_reference: null pointer");
    *ref = c->res_reference;
    return 0;
}

int orc_update_params(orc_ctx* c, const ice_gpu_params* P) {
    if (P->nfam != c->P.nfam || P->ndir != c->P.ndir) return seterr(c, ICE_GPU_EINVAL, "nfam/ndir may not change");
    for (int p = 0; p < P->nfam; ++p)
        if (P->fam[p].closure != c->P.fam[p].closure) return seterr(c, ICE_GPU_EINVAL, "closures may not change");
    c->P = *P;
    return 0;
}

int orc_last_error(const orc_ctx* c, char* buf, int n) {
    if (c && n > 0) { strncpy(buf, c->err, n - 1); buf[n - 1] = 0; }
    return 0;
}

/* ------------------------------------------------------- connection pairing */
/* Pair_Connections (io/IO_BC.f90:360-510). rec: ICE_GPU_REC_INTS ints per record; fields
 * 12..14 (partner, owner, cf) are written. */
static void tangential(int f, int i, int j, int k, int* t) {
    if (f <= 2) { t[0] = j; t[1] = k; } else if (f <= 4) { t[0] = i; t[1] = k; } else { t[0] = i; t[1] = j; }
}
static int key_less(const int* a, const int* b) {
    for (int m = 0; m < 5; ++m) if (a[m] != b[m]) return a[m] < b[m];
    return 0;
}
int orc_pair_connections(int nb, const int* dims, int ngroups, int nrec, int* rec, char* err, int errlen) {
#define R(n, fld) rec[(long)(n)*ICE_GPU_REC_INTS + (fld)]
    enum { Fb, Fi, Fj, Fk, Ff, Ftype, Fp, Fbs, Fis, Fjs, Fks, Ffs, Fpartner, Fowner, Fcf };
    int** map = (int**)calloc((size_t)nb*6, sizeof(int*));
    int rc = 0;
    for (int n = 0; n < nrec; ++n) { if (R(n, Ftype) == 101 || R(n, Ftype) == 201) { R(n, Fpartner) = 0; R(n, Fowner) = 0; R(n, Fcf) = 0; } }
    for (int p = 1; p <= ngroups && !rc; ++p) {
        for (int n = p - 1; n < nrec; n += ngroups) {
            int ty = R(n, Ftype);
            if (ty != 101 && ty != 201) continue;
            int b = R(n, Fb), f = R(n, Ff), t[2], nt[2];
            int* d = (int*)&dims[3*(b - 1)];
            if (!map[(b - 1)*6 + f - 1]) {
                tangential(f, d[0], d[1], d[2], nt);
                map[(b - 1)*6 + f - 1] = (int*)calloc((size_t)nt[0]*nt[1] + 2, sizeof(int));
                map[(b - 1)*6 + f - 1][0] = nt[0]; map[(b - 1)*6 + f - 1][1] = nt[1];
            }
            tangential(f, R(n, Fi), R(n, Fj), R(n, Fk), t);
            int* m = map[(b - 1)*6 + f - 1];
            m[2 + (t[1] - 1)*m[0] + (t[0] - 1)] = n + 1;
        }
        for (int n = p - 1; n < nrec && !rc; n += ngroups) {
            int ty = R(n, Ftype);
            if (ty != 101 && ty != 201) continue;
            int b = R(n, Fbs), f = R(n, Ffs), q = 0, t[2];
            if (b >= 1 && b <= nb && f >= 1 && f <= 6 && map[(b - 1)*6 + f - 1]) {
                int* m = map[(b - 1)*6 + f - 1];
                tangential(f, R(n, Fis), R(n, Fjs), R(n, Fks), t);
                if (t[0] >= 1 && t[1] >= 1 && t[0] <= m[0] && t[1] <= m[1]) q = m[2 + (t[1] - 1)*m[0] + (t[0] - 1)];
            }
            if (q) {
                int qq = q - 1;
                if (R(qq, Fi) != R(n, Fis) || R(qq, Fj) != R(n, Fjs) || R(qq, Fk) != R(n, Fks)) q = 0;
            }
            if (!q) { snprintf(err, errlen, "record %d points at no connection record of its family", n + 1); rc = 1; break; }
            if (q == n + 1) { snprintf(err, errlen, "record %d points at its own cell and face", n + 1); rc = 1; break; }
            int qq = q - 1;
            if (R(qq, Ftype) != ty || R(qq, Fbs) != R(n, Fb) || R(qq, Ffs) != R(n, Ff) || R(qq, Fis) != R(n, Fi) ||
                R(qq, Fjs) != R(n, Fj) || R(qq, Fks) != R(n, Fk)) {
                snprintf(err, errlen, "record %d and record %d do not point at each other", n + 1, q); rc = 1; break;
            }
            int across = dims[3*(b - 1) + (f + 1)/2 - 1];
            if (across < 2) { snprintf(err, errlen, "record %d: block across has %d cell across its face", n + 1, across); rc = 1; break; }
            R(n, Fpartner) = q;
            int fn = R(n, Ff), fq = R(qq, Ff);
            if (fn % 2 == 0 && fq % 2 == 1) R(n, Fowner) = 1;
            else if (fn % 2 == 1 && fq % 2 == 0) R(n, Fowner) = 0;
            else {
                int k1[5] = {R(n, Fb), R(n, Ff), R(n, Fk), R(n, Fj), R(n, Fi)};
                int k2[5] = {R(qq, Fb), R(qq, Ff), R(qq, Fk), R(qq, Fj), R(qq, Fi)};
                R(n, Fowner) = key_less(k1, k2);
            }
        }
        if (!rc) {
            int nf = 0;
            for (int n = p - 1; n < nrec; n += ngroups) {
                int ty = R(n, Ftype);
                if ((ty != 101 && ty != 201) || !R(n, Fowner)) continue;
                ++nf;
                R(n, Fcf) = nf;
                R(R(n, Fpartner) - 1, Fcf) = nf;
            }
        }
        for (int q = 0; q < nb*6; ++q) { free(map[q]); map[q] = NULL; }
    }
    free(map);
    return rc ? ICE_GPU_EINVAL : 0;
#undef R
}

/* ------------------------------------------------------------- records */
/* build_local_bc_index + collect_boundary_cells + collect_owner_records
 * (Mod_GhostExchange.f90:103-360), one rank owning every block. */
int orc_set_records(orc_ctx* c, int nrec, const int* ri, const double* rr) {
    int nf = c->P.nfam;
    free(c->bc); c->bc = (orec*)calloc(nrec > 0 ? nrec : 1, sizeof(orec));
    c->nrec = nrec;
    for (int n = 0; n < nrec; ++n) {
        const int* q = ri + (long)n*ICE_GPU_REC_INTS;
        orec* r = &c->bc[n];
        r->b = q[0]; r->i = q[1]; r->j = q[2]; r->k = q[3]; r->f = q[4]; r->type = q[5]; r->p = q[6];
        r->bs = q[7]; r->is = q[8]; r->js = q[9]; r->ks = q[10]; r->fs = q[11];
        r->partner = q[12]; r->owner = q[13]; r->cf = q[14];
        const double* x = rr + (long)n*ICE_GPU_REC_REALS;
        r->massflux = x[0]; r->velocity = x[1]; r->alpha = x[2]; r->beta = x[3];
        r->temperature = x[4]; r->radius = x[5]; r->gfixed = x[6]; r->normal_dir = x[7] != 0.0;
        if (r->b < 1 || r->b > c->nb || r->p < 1 || r->p > nf || r->f < 1 || r->f > 6)
            return seterr(c, ICE_GPU_EINVAL, "record %d: bad block, family or face", n + 1);
        /* read_bc, IO_BC.f90:264-271: an injecting 401 or 403 inlet reads the gas speed, and a run
         * without a gas phase refuses it while the table is read (a zero-flux inlet mirrors) */
        if ((r->type == 401 || r->type == 403) && r->massflux != 0.0 && !c->P.coupled)
            return seterr(c, ICE_GPU_EINVAL, "record %d: inlet %d takes its speed from the gas, and the run has no gas",
                          n + 1, r->type);
    }
    c->nchim = 0;
    for (int n = 0; n < nrec; ++n) { c->nchim += c->bc[n].type == 102; c->bc[n].d0 = 0; c->bc[n].n1 = c->bc[n].n2 = 0; }
    c->have_chim = c->nchim == 0;
    /* records grouped by family, table order */
    free(c->grp_first); free(c->grp);
    c->grp_first = (int*)calloc(nf + 1, sizeof(int));
    c->grp = (int*)calloc(nrec > 0 ? nrec : 1, sizeof(int));
    int pos[MAXF] = {0};
    for (int n = 0; n < nrec; ++n) pos[c->bc[n].p - 1]++;
    c->grp_first[0] = 0;
    for (int p = 0; p < nf; ++p) c->grp_first[p + 1] = c->grp_first[p] + pos[p];
    for (int p = 0; p < nf; ++p) pos[p] = c->grp_first[p];
    for (int n = 0; n < nrec; ++n) c->grp[pos[c->bc[n].p - 1]++] = n;
    /* boundary cells per family: block by block in cell order (k, j, i), records by face (stable) */
    for (int p = 0; p < nf; ++p) {
        free(c->bfirst[p]); free(c->brec[p]);
        int ncell = 0, nr = 0;
        int* tmpfirst = NULL; int* tmprec = (int*)malloc(sizeof(int)*(nrec > 0 ? nrec : 1));
        int cap = 16; tmpfirst = (int*)malloc(sizeof(int)*cap);
        for (int b = 0; b < c->nb; ++b) {
            oblk* B = &c->blk[b];
            long nce = ncells(B);
            int* head = (int*)calloc(nce, sizeof(int));
            int* tail = (int*)calloc(nce, sizeof(int));
            int* next = (int*)calloc(nrec > 0 ? nrec : 1, sizeof(int));
            for (int n = 0; n < nrec; ++n) {
                orec* r = &c->bc[n];
                if (r->b != b + 1 || r->p != p + 1 || r->type == 0) continue;
                long q = II(B, r->i, r->j, r->k);
                next[n] = -1;
                if (!head[q]) head[q] = n + 1; else next[tail[q] - 1] = n;
                tail[q] = n + 1;
            }
            for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
                long q = II(B, i, j, k);
                if (!head[q]) continue;
                if (ncell + 2 > cap) { cap *= 2; tmpfirst = (int*)realloc(tmpfirst, sizeof(int)*cap); }
                tmpfirst[ncell++] = nr;
                int s0 = nr;
                for (int n = head[q] - 1; n >= 0; n = next[n]) tmprec[nr++] = n;
                for (int m = s0 + 1; m < nr; ++m) {          /* insertion sort by face, stable */
                    int n = tmprec[m], l = m - 1;
                    while (l >= s0 && c->bc[tmprec[l]].f > c->bc[n].f) { tmprec[l + 1] = tmprec[l]; --l; }
                    tmprec[l + 1] = n;
                }
            }
            free(head); free(tail); free(next);
        }
        tmpfirst[ncell] = nr;
        c->bn[p] = ncell; c->bfirst[p] = tmpfirst; c->brec[p] = tmprec;
        /* owners, table order within the family group */
        free(c->own[p]); free(c->connF[p]);
        int k = 0, ncf = 0;
        for (int ii = c->grp_first[p]; ii < c->grp_first[p + 1]; ++ii) {
            orec* r = &c->bc[c->grp[ii]];
            if ((r->type == 101 || r->type == 201)) { if (r->owner) ++k; if (r->cf > ncf) ncf = r->cf; }
        }
        c->nown[p] = k; c->nconn[p] = ncf;
        c->own[p] = (int*)malloc(sizeof(int)*(k > 0 ? k : 1));
        c->connF[p] = (double*)calloc((size_t)(ncf > 0 ? ncf : 1)*NCM, sizeof(double));
        k = 0;
        for (int ii = c->grp_first[p]; ii < c->grp_first[p + 1]; ++ii) {
            orec* r = &c->bc[c->grp[ii]];
            if ((r->type == 101 || r->type == 201) && r->owner) c->own[p][k++] = c->grp[ii];
        }
    }
    return 0;
}

int orc_index_maps(const orc_ctx* c, int p1, int* nbcell, int* first, int* nrecs, int* recs, int* nown, int* own) {
    int p = p1 - 1;
    *nbcell = c->bn[p];
    *nrecs = c->bfirst[p][c->bn[p]];
    *nown = c->nown[p];
    if (first) for (int q = 0; q <= c->bn[p]; ++q) first[q] = c->bfirst[p][q] + 1;
    if (recs) for (int q = 0; q < *nrecs; ++q) recs[q] = c->brec[p][q] + 1;
    if (own) for (int q = 0; q < c->nown[p]; ++q) own[q] = c->own[p][q] + 1;
    return 0;
}

/* The donors of the chimera records (ICE_bc_type%ni, donorID, volume_fraction;
 * Advanced_Types_m.f90:29-31, read by IO_BC.f90:209-236), in table order. */
int orc_set_chimera(orc_ctx* c, int nrec, const int* nchi, const int* donor, const double* weight) {
    if (!c) return ICE_GPU_EINVAL;
    if (nrec != c->nrec || (nrec > 0 && !nchi))
        return seterr(c, ICE_GPU_EINVAL, "set_chimera: %d records given, the table has %d", nrec, c->nrec);
    long tot = 0;
    for (int n = 0; n < nrec; ++n) {
        int n1 = nchi[2*n], n2 = nchi[2*n + 1];
        if (n1 < 0 || n2 < 0) return seterr(c, ICE_GPU_EINVAL, "record %d: negative donor count", n + 1);
        if (c->bc[n].type != 102 && (n1 || n2))
            return seterr(c, ICE_GPU_EINVAL, "record %d: donors given to a record of code %d", n + 1, c->bc[n].type);
        if (c->bc[n].type == 102 && (n1 < 1 || n2 < 1))
            return seterr(c, ICE_GPU_EINVAL, "record %d: a chimera record needs donors for both ghost layers", n + 1);
        tot += n1 + n2;
    }
    if (tot > 0 && (!donor || !weight)) return seterr(c, ICE_GPU_EINVAL, "set_chimera: null donor arrays");
    for (long s = 0; s < tot; ++s) {
        const int* d = donor + 4*s;
        if (d[0] < 1 || d[0] > c->nb) return seterr(c, ICE_GPU_EINVAL, "donor %ld: block %d", s + 1, d[0]);
        const oblk* B = &c->blk[d[0] - 1];
        if (d[1] < 1 || d[1] > B->ni || d[2] < 1 || d[2] > B->nj || d[3] < 1 || d[3] > B->nk)
            return seterr(c, ICE_GPU_EINVAL, "donor %ld: cell %d %d %d is not an interior cell of block %d",
                          s + 1, d[1], d[2], d[3], d[0]);
        if (!isfinite(weight[s])) return seterr(c, ICE_GPU_EINVAL, "donor %ld: weight is not finite", s + 1);
    }
    free(c->cdon); free(c->cw);
    c->cdon = (int*)malloc(sizeof(int)*4*(tot > 0 ? tot : 1));
    c->cw = (double*)malloc(sizeof(double)*(tot > 0 ? tot : 1));
    if (tot > 0) { memcpy(c->cdon, donor, sizeof(int)*4*tot); memcpy(c->cw, weight, sizeof(double)*tot); }
    long off = 0;
    for (int n = 0; n < nrec; ++n) {
        c->bc[n].d0 = off; c->bc[n].n1 = nchi[2*n]; c->bc[n].n2 = nchi[2*n + 1];
        off += nchi[2*n] + nchi[2*n + 1];
    }
    c->have_chim = 1;
    return 0;
}

/* ---------------------------------------------------------------- ghosts */
/* ghost_chimera (Lib_Ghost.f90:439-466): ghost cell g of layer `layer` is the weighted sum of its
 * donors' conservative states, in donor order, back to primitive (cons_2_prim with its floors). */
static void ghost_chimera(orc_ctx* c, const orec* r, int layer, double* g) {
    int pm = r->p - 1, nc = nc_of(c, pm), cl = c->P.fam[pm].closure;
    const ice_gpu_family* m = &c->P.fam[pm];
    long a = r->d0 + (layer == 1 ? 0 : r->n1), z = a + (layer == 1 ? r->n1 : r->n2);
    double cs[NCM], cd[NCM];
    for (int v = 0; v < nc; ++v) cs[v] = 0.0;
    for (long s = a; s < z; ++s) {
        const int* d = c->cdon + 4*s;
        oblk* D = &c->blk[d[0] - 1];
        const double* pd = D->fam[pm].prim + nc*CI(D, d[1], d[2], d[3]);
        o_prim2cons(cl, pd, cd, m);
        for (int v = 0; v < nc; ++v) cs[v] = cs[v] + c->cw[s]*cd[v];
    }
    o_cons2prim(cl, cs, g, m);
}

/* The face normal of a record's own face: dir(d)%f(ic,...) with ic = im - mod(fm,2) (Lib_Ghost.f90:114-123). */
static const double* rec_face(const oblk* B, const orec* r) {
    int f = r->f;
    if (f <= 2) return NRM(B, 0, r->i - (f % 2), r->j, r->k);
    if (f <= 4) return NRM(B, 1, r->i, r->j - (f % 2), r->k);
    return NRM(B, 2, r->i, r->j, r->k - (f % 2));
}

enum { GHOST_COPY = 0, GHOST_MIRROR = 1, GHOST_INJECT = 2 };
/* ghost_rule, Lib_Ghost.f90:395-413 */
static int ghost_rule(const orec* r, double veln) {
    int rule = GHOST_COPY;
    if (r->type == 200) rule = GHOST_MIRROR;
    else if (r->type == 300 || r->type == 301) {
        if (veln*(double)(1 - 2*(r->f % 2)) <= 0.0 || r->f == 3) rule = GHOST_MIRROR;
    } else if (r->type >= 401 && r->type <= 403) {
        if (!(veln*(double)(1 - 2*(r->f % 2)) > 0.0)) {
            rule = GHOST_INJECT;
            if (r->massflux == 0.0) rule = GHOST_MIRROR;
        }
    }
    return rule;
}

static void injected_velocity(double speed, const orec* r, const double* inward, double* v) {
    if (r->normal_dir) { v[0] = speed*inward[0]; v[1] = speed*inward[1]; v[2] = speed*inward[2]; }
    else {
        v[0] = speed*cos(r->beta)*cos(r->alpha);
        v[1] = speed*cos(r->beta)*sin(r->alpha);
        v[2] = speed*sin(r->beta);
    }
}

/* ghost_record (Lib_Ghost.f90:76-267) */
static void ghost_record(orc_ctx* c, const orec* r) {
    int pm = r->p - 1, nc = nc_of(c, pm), cl = c->P.fam[pm].closure, nb = o_nbase(cl);
    oblk* B = &c->blk[r->b - 1];
    double* P = B->fam[pm].prim;
    int im = r->i, jm = r->j, km = r->k, fm = r->f;
    int ig = im - guide[fm-1][0], jg = jm - guide[fm-1][1], kg = km - guide[fm-1][2];
    double* g = P + nc*CI(B, ig, jg, kg);
    const double* m = P + nc*CI(B, im, jm, km);
    switch (r->type) {
    case 101: case 201: {
        oblk* S = &c->blk[r->bs - 1];
        const double* s = S->fam[pm].prim + nc*CI(S, r->is, r->js, r->ks);
        for (int v = 0; v < nc; ++v) g[v] = s[v];
        break;
    }
    case 200: case 300: case 301: {
        const double* N = rec_face(B, r);
        double n[3] = {N[0], N[1], N[2]};
        for (int v = 0; v < nc; ++v) g[v] = m[v];
        double vel[3] = {m[1], m[2], m[3]};
        double veln = vel[0]*n[0] + vel[1]*n[1] + vel[2]*n[2];
        if (ghost_rule(r, veln) == GHOST_MIRROR) {
            for (int a = 0; a < 3; ++a) vel[a] = vel[a] - 2.0*veln*n[a];
            if (nb == 12) o_mirror_tensor(m + 4, n, g + 4);
        }
        g[1] = vel[0]; g[2] = vel[1]; g[3] = vel[2];
        break;
    }
    case 0: case 400:
        for (int v = 0; v < nc; ++v) g[v] = m[v];
        break;
    case 102:
        ghost_chimera(c, r, 1, g);
        break;
    case 401: case 402: case 403: {
        const double* N = rec_face(B, r);
        double n[3] = {N[0], N[1], N[2]};
        double vel[3] = {m[1], m[2], m[3]};
        double veln = vel[0]*n[0] + vel[1]*n[1] + vel[2]*n[2];
        int rule = ghost_rule(r, veln);
        B->fam[pm].inj[CI(B, ig, jg, kg)] = (rule == GHOST_INJECT);
        if (rule == GHOST_COPY) { for (int v = 0; v < nc; ++v) g[v] = m[v]; return; }
        if (rule == GHOST_MIRROR) {
            for (int v = 0; v < nc; ++v) g[v] = m[v];
            for (int a = 0; a < 3; ++a) vel[a] = vel[a] - 2.0*veln*n[a];
            g[1] = vel[0]; g[2] = vel[1]; g[3] = vel[2];
            if (nb == 12) o_mirror_tensor(m + 4, n, g + 4);
            return;
        }
        for (int v = 0; v < nc; ++v) g[v] = 0.0;
        double sgn = (double)(2*(fm % 2) - 1);
        double inward[3] = {sgn*n[0], sgn*n[1], sgn*n[2]};
        const double* gas = B->gprim ? B->gprim + 5*II(B, im, jm, km) : NULL;
        double v3[3];
        if (r->type == 401) {
            double vn = gas[1]*inward[0] + gas[2]*inward[1] + gas[3]*inward[2];
            injected_velocity(r->velocity*vn, r, inward, v3);
            g[1] = v3[0]; g[2] = v3[1]; g[3] = v3[2];
            g[0] = r->massflux*gas[0]/r->velocity;
            vn = fabs(g[1]*n[0] + g[2]*n[1] + g[3]*n[2]);
            if (r->gfixed > 0.0 && vn > 0.0) g[0] = g[0] + r->massflux*r->gfixed/vn;
            g[nb - 2] = r->temperature*gas[4];
        } else if (r->type == 402) {
            injected_velocity(r->velocity, r, inward, v3);
            g[1] = v3[0]; g[2] = v3[1]; g[3] = v3[2];
            double vn = g[1]*n[0] + g[2]*n[1] + g[3]*n[2];
            g[0] = r->massflux/fabs(vn);
            g[nb - 2] = r->temperature;
        } else {
            double vn = o_norm2(gas[1], gas[2], gas[3]);
            injected_velocity(r->velocity*vn, r, inward, v3);
            g[1] = v3[0]; g[2] = v3[1]; g[3] = v3[2];
            vn = g[1]*n[0] + g[2]*n[1] + g[3]*n[2];
            g[0] = r->massflux/fabs(vn);
            g[nb - 2] = r->temperature;
        }
        g[nb - 1] = g[0]/c->P.fam[pm].rho_al/(4.0/3.0*O_PI*pow(r->radius, 3.0));
        if (cl == ICE_CLOSURE_IG) g[4] = 1e-6;
        else if (cl == ICE_CLOSURE_AG) { g[4] = 1e-6; g[7] = 1e-6; g[9] = 1e-6; }
        break;
    }
    default: break;
    }
}

/* second_ghost_record (Lib_Ghost.f90:312-387) */
static void second_ghost_record(orc_ctx* c, const orec* r) {
    if (r->type == 0) return;
    int pm = r->p - 1, nc = nc_of(c, pm), nb = o_nbase(c->P.fam[pm].closure);
    oblk* B = &c->blk[r->b - 1];
    double* P = B->fam[pm].prim;
    int im = r->i, jm = r->j, km = r->k, fm = r->f;
    const int* gd = guide[fm - 1];
    int ig = im - gd[0], jg = jm - gd[1], kg = km - gd[2];
    int ig2 = im - 2*gd[0], jg2 = jm - 2*gd[1], kg2 = km - 2*gd[2];
    int ip = im + gd[0], jp = jm + gd[1], kp = km + gd[2];
    double* g2 = P + nc*CI(B, ig2, jg2, kg2);
    const double* g1 = P + nc*CI(B, ig, jg, kg);
    const double* m = P + nc*CI(B, im, jm, km);
    const double* mp = P + nc*CI(B, ip, jp, kp);
    switch (r->type) {
    case 101: case 201: {
        oblk* S = &c->blk[r->bs - 1];
        const int* gs = guide[r->fs - 1];
        const double* s = S->fam[pm].prim + nc*CI(S, r->is + gs[0], r->js + gs[1], r->ks + gs[2]);
        for (int v = 0; v < nc; ++v) g2[v] = s[v];
        break;
    }
    case 200: case 300: case 301: case 401: case 402: case 403: {
        const double* N = rec_face(B, r);
        double n[3] = {N[0], N[1], N[2]};
        double veln = m[1]*n[0] + m[2]*n[1] + m[3]*n[2];
        int rule = ghost_rule(r, veln);
        if (rule == GHOST_INJECT) { for (int v = 0; v < nc; ++v) g2[v] = g1[v]; }
        else {
            for (int v = 0; v < nc; ++v) g2[v] = mp[v];
            if (rule == GHOST_MIRROR) {
                double vel[3] = {mp[1], mp[2], mp[3]};
                double d = vel[0]*n[0] + vel[1]*n[1] + vel[2]*n[2];
                for (int a = 0; a < 3; ++a) g2[1 + a] = vel[a] - 2.0*d*n[a];
                if (nb == 12) o_mirror_tensor(mp + 4, n, g2 + 4);
            }
        }
        break;
    }
    case 102:
        ghost_chimera(c, r, 2, g2);
        break;
    default:
        for (int v = 0; v < nc; ++v) g2[v] = 3.0*g1[v] - 3.0*m[v] + mp[v];
        break;
    }
}

static void compute_ghost(orc_ctx* c, int p) {
    int lo = c->grp_first[p], hi = c->grp_first[p + 1];
    #pragma omp parallel for schedule(dynamic, 64)
    for (int ii = lo; ii < hi; ++ii) {
        const orec* r = &c->bc[c->grp[ii]];
        if (OWN(c, r->b - 1)) ghost_record(c, r);
    }
    #pragma omp parallel for schedule(dynamic, 64)
    for (int ii = lo; ii < hi; ++ii) {
        const orec* r = &c->bc[c->grp[ii]];
        if (OWN(c, r->b - 1)) second_ghost_record(c, r);
    }
}

/* ------------------------------------------------------ the block split */
/* One exchange of a split step (Mod_GhostExchange.f90:737-800 for the cells): pack the kind's send
 * entries of family p, let the hook move the buffers, unpack the receive entries. CELLS: the cells'
 * state into the local copy of the remote block; BETA: the Jameson weights of cells; FLUX: connection
 * face fluxes (nc each) by face number. */
static int halo_exchange(orc_ctx* c, int kind, int p) {
    if (!c->owned) return 0;
    int nc = nc_of(c, p), w = kind == ICE_GPU_HALO_BETA ? 1 : nc;
    long ns = (long)c->nhs[kind][p] * w, nr = (long)c->nhr[kind][p] * w;
    if (c->hbuf_n < (size_t)(ns + nr + 1)) {
        free(c->hbuf); c->hbuf_n = (size_t)(ns + nr + 1); c->hbuf = (double*)malloc(sizeof(double)*c->hbuf_n);
    }
    double* sb = c->hbuf; double* rb = c->hbuf + ns;
    for (int n = 0; n < c->nhs[kind][p]; ++n) {
        const int* e = c->hs[kind][p] + 4*n;
        if (kind == ICE_GPU_HALO_FLUX) { memcpy(sb + (long)n*w, c->connF[p] + (long)(e[0] - 1)*NCM, sizeof(double)*nc); continue; }
        oblk* B = &c->blk[e[0] - 1];
        if (kind == ICE_GPU_HALO_CELLS) memcpy(sb + (long)n*w, B->fam[p].prim + (long)nc*CI(B, e[1], e[2], e[3]), sizeof(double)*nc);
        else sb[n] = B->fam[p].beta[II(B, e[1], e[2], e[3])];
    }
    if (!c->hook) return seterr(c, ICE_GPU_ENOTREADY, "a split run needs its exchange hook (set_exchange_hook)");
    if (c->hook(c->hook_user, kind, p + 1, ns, sb, nr, rb) != 0)
        return seterr(c, ICE_GPU_EEXCH, "the exchange hook failed (kind %d, family %d)", kind, p + 1);
    for (int n = 0; n < c->nhr[kind][p]; ++n) {
        const int* e = c->hr[kind][p] + 4*n;
        if (kind == ICE_GPU_HALO_FLUX) { memcpy(c->connF[p] + (long)(e[0] - 1)*NCM, rb + (long)n*w, sizeof(double)*nc); continue; }
        oblk* B = &c->blk[e[0] - 1];
        if (kind == ICE_GPU_HALO_CELLS) memcpy(B->fam[p].prim + (long)nc*CI(B, e[1], e[2], e[3]), rb + (long)n*w, sizeof(double)*nc);
        else B->fam[p].beta[II(B, e[1], e[2], e[3])] = rb[n];
    }
    return 0;
}

/* The reductions of a split step: the minimum (DT) or the sum (NORM) over the ranks of n doubles. */
static int halo_reduce(orc_ctx* c, int kind, double* x, long n) {
    if (!c->owned) return 0;
    if (!c->hook) return seterr(c, ICE_GPU_ENOTREADY, "a split run needs its exchange hook (set_exchange_hook)");
    double* in = (double*)malloc(sizeof(double)*n);
    memcpy(in, x, sizeof(double)*n);
    int rc = c->hook(c->hook_user, kind, 0, n, in, n, x);
    free(in);
    return rc ? seterr(c, ICE_GPU_EEXCH, "the exchange hook failed (kind %d)", kind) : 0;
}

int orc_set_partition(orc_ctx* c, const int* owned) {
    if (!owned) { free(c->owned); c->owned = NULL; return 0; }
    if (c->P.irs) return seterr(c, ICE_GPU_EINVAL, "set_partition: IRS is not supported in a split run");
    if (c->nchim > 0) return seterr(c, ICE_GPU_EINVAL, "set_partition: chimera records are not supported in a split run");
    for (int p = 0; p < c->P.nfam; ++p)
        if (c->have_imp[p]) return seterr(c, ICE_GPU_EINVAL, "set_partition: imports are not supported in a split run");
    free(c->owned);
    c->owned = (int*)malloc(sizeof(int)*c->nb);
    for (int b = 0; b < c->nb; ++b) c->owned[b] = owned[b] != 0;
    return 0;
}

int orc_set_halo(orc_ctx* c, int kind, int p1, int nsend, const int* send, int nrecv, const int* recv) {
    if (kind < 0 || kind > 2 || p1 < 1 || p1 > c->P.nfam || nsend < 0 || nrecv < 0 ||
        (nsend > 0 && !send) || (nrecv > 0 && !recv))
        return seterr(c, ICE_GPU_EINVAL, "set_halo: bad arguments");
    int p = p1 - 1;
    for (int side = 0; side < 2; ++side) {
        int n = side ? nrecv : nsend;
        const int* e = side ? recv : send;
        for (int q = 0; q < n; ++q) {
            const int* x = e + 4*q;
            if (kind == ICE_GPU_HALO_FLUX) {
                if (x[0] < 1 || x[0] > c->nconn[p]) return seterr(c, ICE_GPU_EINVAL, "set_halo: connection face %d", x[0]);
                continue;
            }
            if (x[0] < 1 || x[0] > c->nb) return seterr(c, ICE_GPU_EINVAL, "set_halo: block %d", x[0]);
            const oblk* B = &c->blk[x[0] - 1];
            if (x[1] < 1 || x[1] > B->ni || x[2] < 1 || x[2] > B->nj || x[3] < 1 || x[3] > B->nk)
                return seterr(c, ICE_GPU_EINVAL, "set_halo: cell %d %d %d outside block %d", x[1], x[2], x[3], x[0]);
        }
    }
    free(c->hs[kind][p]); free(c->hr[kind][p]);
    c->hs[kind][p] = (int*)malloc(sizeof(int)*4*(nsend + 1));
    c->hr[kind][p] = (int*)malloc(sizeof(int)*4*(nrecv + 1));
    if (nsend) memcpy(c->hs[kind][p], send, sizeof(int)*4*nsend);
    if (nrecv) memcpy(c->hr[kind][p], recv, sizeof(int)*4*nrecv);
    c->nhs[kind][p] = nsend; c->nhr[kind][p] = nrecv;
    return 0;
}

int orc_set_exchange_hook(orc_ctx* c, ice_gpu_exchange_fn fn, void* user) {
    c->hook = fn; c->hook_user = user;
    return 0;
}

/* ---------------------------------------------------------------- beta */
static void compute_beta(orc_ctx* c, int p) {
    int nc = nc_of(c, p);
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            if (c->P.shock_detector) {
                const double* P = F->prim;
                F->beta[II(B, i, j, k)] = o_sd_rho(P[nc*CI(B, i, j, k)],
                    P[nc*CI(B, i - 1, j, k)], P[nc*CI(B, i + 1, j, k)],
                    P[nc*CI(B, i, j - 1, k)], P[nc*CI(B, i, j + 1, k)],
                    P[nc*CI(B, i, j, k - 1)], P[nc*CI(B, i, j, k + 1)]);
            } else F->beta[II(B, i, j, k)] = 1.0;
        }
    }
}

/* ---------------------------------------------------- boundary fluxes */
/* record_flux (Mod_BC_Fluxes.f90:180-272). Returns 1 on an unphysical first-order face. */
static int record_flux(orc_ctx* c, const orec* r, double* flux, const double* beta_face) {
    int pm = r->p - 1, nc = nc_of(c, pm);
    const ice_gpu_family* mat = &c->P.fam[pm];
    oblk* B = &c->blk[r->b - 1];
    ofam* F = &B->fam[pm];
    int i = r->i, j = r->j, k = r->k, f = r->f;
    const int* gd = guide[f - 1];
    int ig = i - gd[0], jg = j - gd[1], kg = k - gd[2];
    int ig2 = i - 2*gd[0], jg2 = j - 2*gd[1], kg2 = k - 2*gd[2];
    int ip = i + gd[0], jp = j + gd[1], kp = k + gd[2];
    int dir = (f + 1)/2 - 1;
    double bv = beta_face ? *beta_face : F->beta[II(B, i, j, k)];
    double pl[NCM], pr[NCM], fl[NCM];
    double dl0, dl1, dl2, dll, dlr;
    double dl_g1 = B->dl[3*RI(B, ig, jg, kg) + dir];
    double dl_m = B->dl[3*RI(B, i, j, k) + dir];
    double dl_4 = B->dl[3*RI(B, ip, jp, kp) + dir];
    const double* P = F->prim;
    int bad;
    if (f % 2 == 1) {
        /* dir(dir)%f(ig,jg,kg): the face below the cell along dir */
        const double* nrm = dir == 0 ? NRM(B, 0, ig, j, k) : dir == 1 ? NRM(B, 1, i, jg, k) : NRM(B, 2, i, j, kg);
        double n[3] = {nrm[0], nrm[1], nrm[2]}, area = nrm[3];
        dl0 = dl_g1; dl1 = 0.5*(dl_g1 + dl_m); dl2 = 0.5*(dl_m + dl_4);
        dll = 0.5*dl_g1; dlr = 0.5*dl_m;
        if (F->inj[CI(B, ig, jg, kg)]) { dl1 = 0.5*dl_m; dll = 0.0; }
        if (F->inj[CI(B, ip, jp, kp)]) dl2 = 0.5*dl_m;
        bad = o_reconstruct(mat->closure, c->P.limiter, P + nc*CI(B, ig2, jg2, kg2), P + nc*CI(B, ig, jg, kg),
                            P + nc*CI(B, i, j, k), P + nc*CI(B, ip, jp, kp), dl0, dl1, dl2, dll, dlr, pl, pr, bv);
        o_riemann(mat->riemann, mat->closure, pl, pr, n, fl, mat);
        for (int v = 0; v < nc; ++v) flux[v] = fl[v] * area;
    } else {
        const double* nrm = NRM(B, dir, i, j, k);
        double n[3] = {nrm[0], nrm[1], nrm[2]}, area = nrm[3];
        dl0 = 0.5*(dl_4 + dl_m); dl1 = 0.5*(dl_m + dl_g1); dl2 = dl_g1;
        dll = 0.5*dl_m; dlr = 0.5*dl_g1;
        if (F->inj[CI(B, ig, jg, kg)]) { dl1 = 0.5*dl_m; dlr = 0.0; }
        if (F->inj[CI(B, ip, jp, kp)]) dl0 = 0.5*dl_m;
        bad = o_reconstruct(mat->closure, c->P.limiter, P + nc*CI(B, ip, jp, kp), P + nc*CI(B, i, j, k),
                            P + nc*CI(B, ig, jg, kg), P + nc*CI(B, ig2, jg2, kg2), dl0, dl1, dl2, dll, dlr, pl, pr, bv);
        o_riemann(mat->riemann, mat->closure, pl, pr, n, fl, mat);
        for (int v = 0; v < nc; ++v) flux[v] = -(fl[v] * area);
    }
    return bad;
}

static int compute_bound(orc_ctx* c, int p) {
    int nc = nc_of(c, p), bad = 0;
    /* owner fluxes of the connection faces (owner_flux, Mod_BC_Fluxes.f90:151-170) */
    #pragma omp parallel for schedule(dynamic, 16) reduction(|:bad)
    for (int jj = 0; jj < c->nown[p]; ++jj) {
        const orec* r = &c->bc[c->own[p][jj]];
        if (!OWN(c, r->b - 1)) continue;
        const orec* q = &c->bc[r->partner - 1];
        double bq = c->blk[q->b - 1].fam[p].beta[II(&c->blk[q->b - 1], q->i, q->j, q->k)];
        double bo = c->blk[r->b - 1].fam[p].beta[II(&c->blk[r->b - 1], r->i, r->j, r->k)];
        double bf = o_min2(bo, bq);
        double fl[NCM];
        bad |= record_flux(c, r, fl, &bf);
        for (int v = 0; v < nc; ++v) c->connF[p][(long)(r->cf - 1)*NCM + v] = fl[v];
    }
    /* a split run: the fluxes of connection faces whose partner another rank steps go to it */
    if (bad) return bad;
    if (halo_exchange(c, ICE_GPU_HALO_FLUX, p)) return -1;
    /* boundary cells, records in face order (bound_cell, Mod_BC_Fluxes.f90:105-144) */
    #pragma omp parallel for schedule(dynamic, 16) reduction(|:bad)
    for (int cc = 0; cc < c->bn[p]; ++cc) {
        if (!OWN(c, c->bc[c->brec[p][c->bfirst[p][cc]]].b - 1)) continue;
        for (int rr = c->bfirst[p][cc]; rr < c->bfirst[p][cc + 1]; ++rr) {
            const orec* r = &c->bc[c->brec[p][rr]];
            oblk* B = &c->blk[r->b - 1];
            double fl[NCM];
            if (r->type == 200 && c->P.fam[p].closure == ICE_CLOSURE_MK) continue;
            if (r->type == 101 || r->type == 201) {
                const double* cf = c->connF[p] + (long)(r->cf - 1)*NCM;
                for (int v = 0; v < nc; ++v) fl[v] = r->owner ? cf[v] : -cf[v];
            } else bad |= record_flux(c, r, fl, NULL);
            double* res = B->fam[p].residual + (long)nc*II(B, r->i, r->j, r->k);
            for (int v = 0; v < nc; ++v) res[v] = res[v] + fl[v];
        }
    }
    return bad;
}

/* ------------------------------------------------------ interior fluxes */
/* face_flux + compute_flux_ (Mod_Fluxes.f90:599-685): the face between (i,j,k) and its upper
 * neighbour along d (0-based). */
static int face_flux(orc_ctx* c, oblk* B, int p, int d, int i, int j, int k, double* flux) {
    int nc = nc_of(c, p);
    const ice_gpu_family* mat = &c->P.fam[p];
    ofam* F = &B->fam[p];
    int o[3] = {d == 0, d == 1, d == 2};
    int dim[3] = {B->ni, B->nj, B->nk};
    int idx[3] = {i, j, k};
    double bf = o_min2(F->beta[II(B, i, j, k)], F->beta[II(B, i + o[0], j + o[1], k + o[2])]);
    double len[4];
    for (int s = -1; s <= 2; ++s) len[s + 1] = B->dl[3*RI(B, i + s*o[0], j + s*o[1], k + s*o[2]) + d];
    if (idx[d] == 1 && F->inj[CI(B, i - o[0], j - o[1], k - o[2])]) len[0] = 0.0;
    if (idx[d] == dim[d] - 1 && F->inj[CI(B, i + 2*o[0], j + 2*o[1], k + 2*o[2])]) len[3] = 0.0;
    double dl0 = 0.5*(len[0] + len[1]), dl1 = 0.5*(len[1] + len[2]), dl2 = 0.5*(len[2] + len[3]);
    double dll = 0.5*len[1], dlr = 0.5*len[2];
    const double* P = F->prim;
    double pl[NCM], pr[NCM], fl[NCM];
    int bad = o_reconstruct(mat->closure, c->P.limiter,
                            P + nc*CI(B, i - o[0], j - o[1], k - o[2]), P + nc*CI(B, i, j, k),
                            P + nc*CI(B, i + o[0], j + o[1], k + o[2]), P + nc*CI(B, i + 2*o[0], j + 2*o[1], k + 2*o[2]),
                            dl0, dl1, dl2, dll, dlr, pl, pr, bf);
    const double* nrm = NRM(B, d, i, j, k);
    double n[3] = {nrm[0], nrm[1], nrm[2]};
    o_riemann(mat->riemann, mat->closure, pl, pr, n, fl, mat);
    for (int v = 0; v < nc; ++v) flux[v] = fl[v] * nrm[3];
    return bad;
}

static int compute_flux(orc_ctx* c, int p) {
    int nc = nc_of(c, p), bad = 0;
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        int dim[3] = {B->ni, B->nj, B->nk};
        for (int d = 0; d < 3; ++d) {
            if (dim[d] < 2) continue;
            /* faces between cells c and c+1 along d, c = 1..n_d-1: stored at the lower cell */
            long nf = ncells(B);
            if (c->fbuf_n < (size_t)nf*nc) { free(c->fbuf); c->fbuf_n = (size_t)nf*nc; c->fbuf = (double*)malloc(sizeof(double)*c->fbuf_n); }
            double* fb = c->fbuf;
            int e0 = d == 0 ? B->ni - 1 : B->ni, e1 = d == 1 ? B->nj - 1 : B->nj, e2 = d == 2 ? B->nk - 1 : B->nk;
            #pragma omp parallel for collapse(2) schedule(static) reduction(|:bad)
            for (int k = 1; k <= e2; ++k) for (int j = 1; j <= e1; ++j) for (int i = 1; i <= e0; ++i)
                bad |= face_flux(c, B, p, d, i, j, k, fb + (long)nc*II(B, i, j, k));
            int o[3] = {d == 0, d == 1, d == 2};
            #pragma omp parallel for collapse(2) schedule(static)
            for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
                int idx[3] = {i, j, k};
                int ci = idx[d], n = dim[d];
                double* r = F->residual + (long)nc*II(B, i, j, k);
                const double* up = fb + (long)nc*II(B, i, j, k);
                const double* lo = ci > 1 ? fb + (long)nc*II(B, i - o[0], j - o[1], k - o[2]) : NULL;
                if (ci % 2 == 1) {
                    if (ci < n) for (int v = 0; v < nc; ++v) r[v] = r[v] - up[v];
                    if (ci > 1) for (int v = 0; v < nc; ++v) r[v] = r[v] + lo[v];
                } else {
                    for (int v = 0; v < nc; ++v) r[v] = r[v] + lo[v];
                    if (ci < n) for (int v = 0; v < nc; ++v) r[v] = r[v] - up[v];
                }
            }
        }
    }
    return bad;
}

/* ------------------------------------------------------------ sources */
static void compute_source(orc_ctx* c, int p) {
    int nc = nc_of(c, p);
    const ice_gpu_family* mat = &c->P.fam[p];
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            long q = II(B, i, j, k);
            double s[NCM];
            F->tau[CI(B, i, j, k)] = o_cell_source(mat->closure, F->prim + nc*CI(B, i, j, k), B->gprim + 5*q,
                                                   B->gR[q], B->ggam[q], B->gk[q], B->gmu[q], mat,
                                                   c->P.drag, c->P.heat, c->P.blow, s);
            for (int f = 0; f < mat->nfrozen; ++f) s[mat->frozen[f] - 1] = 0.0;
            for (int v = 0; v < nc; ++v) F->source[(long)nc*q + v] = s[v];
        }
    }
}

/* ------------------------------------------------- residual, IRS, update */
static void compute_residual(orc_ctx* c, int p) {
    int nc = nc_of(c, p);
    const ice_gpu_family* mat = &c->P.fam[p];
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        #pragma omp parallel for schedule(static)
        for (long q = 0; q < ncells(B); ++q) {
            double* r = F->residual + nc*q;
            const double* s = F->source + nc*q;
            for (int v = 0; v < nc; ++v) r[v] = (r[v]/B->vol[q] + s[v]) * F->dt[q];
            for (int f = 0; f < mat->nfrozen; ++f) r[mat->frozen[f] - 1] = 0.0;
        }
    }
}

/* residual_smoothing_ (Lib_IRS.f90:34-86) */
static void residual_smoothing(orc_ctx* c, int p) {
    int nc = nc_of(c, p);
    double beta = c->P.irs_beta;
    for (int d = 0; d < c->P.ndir; ++d) {
        for (int b = 0; b < c->nb; ++b) {
            oblk* B = &c->blk[b];
            double* res = B->fam[p].residual;
            int Nx = B->ni, Ny = B->nj, Nz = B->nk;
            long ns = (long)(Nx + 2)*(Ny + 2)*(Nz + 2);
#define SI(i, j, k) ((((long)(k))*(Ny + 2) + (j))*(Nx + 2) + (i))
            double* star = (double*)calloc(ns*nc, sizeof(double));
            double* rnew = (double*)calloc(ncells(B)*nc, sizeof(double));
            for (int k = 1; k <= Nz; ++k) for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i)
                for (int v = 0; v < nc; ++v) star[nc*SI(i, j, k) + v] = res[nc*II(B, i, j, k) + v];
            for (int k = 1; k <= Nz; ++k) for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i) {
                for (int v = 0; v < nc; ++v) {
                    if (d == 0 && i == 1) star[nc*SI(0, j, k) + v] = star[nc*SI(1, j, k) + v];
                    if (d == 0 && i == Nx) star[nc*SI(Nx + 1, j, k) + v] = star[nc*SI(Nx, j, k) + v];
                    if (d == 1 && j == 1) star[nc*SI(i, 0, k) + v] = star[nc*SI(i, 1, k) + v];
                    if (d == 1 && j == Ny) star[nc*SI(i, Ny + 1, k) + v] = star[nc*SI(i, Ny, k) + v];
                    if (d == 2 && k == 1) star[nc*SI(i, j, 0) + v] = star[nc*SI(i, j, 1) + v];
                    if (d == 2 && k == Nz) star[nc*SI(i, j, Nz + 1) + v] = star[nc*SI(i, j, Nz) + v];
                }
            }
            int o[3] = {d == 0, d == 1, d == 2};
            for (int sweep = 0; sweep < 2; ++sweep) {
                #pragma omp parallel for collapse(2) schedule(static)
                for (int k = 1; k <= Nz; ++k) for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i)
                    for (int v = 0; v < nc; ++v)
                        rnew[nc*II(B, i, j, k) + v] = (res[nc*II(B, i, j, k) + v] + beta*(star[nc*SI(i - o[0], j - o[1], k - o[2]) + v]
                                                      + star[nc*SI(i + o[0], j + o[1], k + o[2]) + v])) / (1.0 + 2.0*beta);
                for (int k = 1; k <= Nz; ++k) for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i)
                    for (int v = 0; v < nc; ++v) star[nc*SI(i, j, k) + v] = rnew[nc*II(B, i, j, k) + v];
            }
            memcpy(res, rnew, sizeof(double)*nc*ncells(B));
            free(star); free(rnew);
#undef SI
        }
    }
}

static const double RKC[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0/3.0}};

/* state_update / state_update_ (Lib_Newstate.f90:109-219) */
static int state_update(orc_ctx* c, int p, int srk) {
    int nc = nc_of(c, p), cl = c->P.fam[p].closure, bad = 0;
    const ice_gpu_family* mat = &c->P.fam[p];
    double rk = RKC[c->P.nrk - 1][srk - 1];
    long long nfl = 0;
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        #pragma omp parallel for collapse(2) schedule(static) reduction(|:bad) reduction(+:nfl)
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            double co[NCM], cn[NCM];
            double* pr = F->prim + nc*CI(B, i, j, k);
            const double* po = F->prim_old + nc*CI(B, i, j, k);
            const double* r = F->residual + (long)nc*II(B, i, j, k);
            o_prim2cons(cl, po, co, mat);
            o_prim2cons(cl, pr, cn, mat);
            for (int v = 0; v < nc; ++v) { double rr = (cn[v] - co[v] + r[v]) * rk; cn[v] = co[v] + rr; }
            if (cn[0] < 0.0) ++nfl;
            o_cons2prim(cl, cn, pr, mat);
            if (!o_check_prim(cl, pr)) bad = 1;
        }
    }
    c->nfloored += nfl;
    return bad;
}

/* ------------------------------------------------------------------ dt */
/* compute_dt / compute_dt_ (Mod_dt.f90:11-112, 256-275) */
static void compute_dt(orc_ctx* c, int p) {
    int nc = nc_of(c, p), cl = c->P.fam[p].closure, ndir = c->P.ndir;
    int tau_limit = c->P.coupled && c->P.tau_factor > 0.0;
    double dtmin = DBL_MAX;
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        #pragma omp parallel for collapse(2) schedule(static) reduction(min:dtmin)
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            long q = II(B, i, j, k);
            const double* pr = F->prim + nc*CI(B, i, j, k);
            const double* T = B->M + 9*RI(B, i, j, k);     /* column-major c(3,3): T(d,c) = T[3*c + d] */
            double dt = (double)1e+5f, rate = 0.0;
            for (int d = 0; d < ndir; ++d) {
                double gn = o_norm2(T[d], T[3 + d], T[6 + d]);
                double vs[3] = {T[d]/gn, T[3 + d]/gn, T[6 + d]/gn};
                rate = rate + (fabs(pr[1]*vs[0] + pr[2]*vs[1] + pr[3]*vs[2]) + o_wavespeed(cl, pr, vs)) * gn;
            }
            if (rate > 0.0) dt = o_min2(dt, 1.0/rate);
            dt = dt * c->P.cfl;
            if (c->iter <= c->P.cfl_ramp_iter) dt = dt * (double)c->iter / (double)c->P.cfl_ramp_iter;
            dt = o_min2(dt, c->P.dt_max);
            if (tau_limit) {
                double tau = F->tau[CI(B, i, j, k)];
                if (pr[0] > O_RHO_EMPTY && !o_not_finite(tau) && tau > 0.0) dt = o_min2(dt, c->P.tau_factor*tau);
            }
            F->dt[q] = dt;
            dtmin = o_min2(dtmin, dt);
        }
    }
    c->dtglobal = o_min2(c->dtglobal, dtmin);
}

/* The coupler's imports into family p1 of block b1 (ICE_cond_phase_type%imports, accumulated by
 * Mod_Exchange.f90:270-390), (nc, ni, nj, nk); NULL zeroes the block's. The first call allocates the
 * family's arrays (zero in every block). */
int orc_set_imports(orc_ctx* c, int b1, int p1, const double* imports) {
    if (c->owned) return seterr(c, ICE_GPU_EINVAL, "set_imports: imports are not supported in a split run");
    if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam) return seterr(c, ICE_GPU_EINVAL, "set_imports: bad block/family");
    int p = p1 - 1, nc = nc_of(c, p);
    oblk* Bq = &c->blk[b1 - 1];
    if (imports)
        for (long q = 0; q < ncells(Bq)*nc; ++q)
            if (!isfinite(imports[q])) return seterr(c, ICE_GPU_EINVAL, "set_imports: a rate is not finite");
    if (!c->have_imp[p]) {
        for (int b = 0; b < c->nb; ++b) c->blk[b].fam[p].imports = (double*)calloc((size_t)nc*ncells(&c->blk[b]), sizeof(double));
        c->have_imp[p] = 1;
    }
    double* d = Bq->fam[p].imports;
    for (long q = 0; q < ncells(Bq)*nc; ++q) d[q] = imports ? imports[q] : 0.0;
    return 0;
}

/* bound_empty_dt (Mod_dt.f90:134-214) with the coupler's imports as the source (no births of the
 * family's own, no burning family): an empty cell that a source fills steps no further than what
 * fills it. */
static void bound_empty_dt(orc_ctx* c, int p) {
    if (!c->have_imp[p]) return;
    int nc = nc_of(c, p), cl = c->P.fam[p].closure, ndir = c->P.ndir;
    double cfl = c->P.cfl;
    int filled = 0;
    double floor_dt = DBL_MAX, src_dt = DBL_MAX, umax[3] = {0.0, 0.0, 0.0};
    double ps[NCM];
    for (int b = 0; b < c->nb; ++b) {
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            long q = II(B, i, j, k);
            const double* pr = F->prim + nc*CI(B, i, j, k);
            const double* s = F->imports + nc*q;
            if (s[0] > 0.0) filled = 1;
            if (pr[0] > O_RHO_EMPTY) {
                floor_dt = o_min2(floor_dt, F->dt[q]);
                for (int a = 0; a < 3; ++a) umax[a] = o_max2(umax[a], fabs(pr[1 + a]));
                continue;
            }
            if (!(s[0] > 0.0)) continue;
            for (int v = 0; v < nc; ++v) ps[v] = pr[v];
            for (int a = 0; a < 3; ++a) ps[1 + a] = s[1 + a]/s[0];
            for (int a = 0; a < 3; ++a) umax[a] = o_max2(umax[a], fabs(ps[1 + a]));
            double dts = (double)1e+5f, rate = 0.0;
            const double* T = B->M + 9*RI(B, i, j, k);
            for (int d = 0; d < ndir; ++d) {
                double gn = o_norm2(T[d], T[3 + d], T[6 + d]);
                double vs[3] = {T[d]/gn, T[3 + d]/gn, T[6 + d]/gn};
                rate = rate + (fabs(ps[1]*vs[0] + ps[2]*vs[1] + ps[3]*vs[2]) + o_wavespeed(cl, ps, vs)) * gn;
            }
            if (rate > 0.0) dts = o_min2(dts, 1.0/rate);
            src_dt = o_min2(src_dt, dts*cfl);
        }
    }
    if (!filled) return;
    if (c->P.time_accurate) { c->dtglobal = o_min2(c->dtglobal, src_dt); return; }
    floor_dt = o_min2(floor_dt, src_dt);
    for (int b = 0; b < c->nb; ++b) {
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            const double* pr = F->prim + nc*CI(B, i, j, k);
            if (pr[0] > O_RHO_EMPTY) continue;
            const double* T = B->M + 9*RI(B, i, j, k);
            double rate = 0.0;
            for (int d = 0; d < ndir; ++d) {
                double sum = umax[0]*fabs(T[d]);
                sum = sum + umax[1]*fabs(T[3 + d]);
                sum = sum + umax[2]*fabs(T[6 + d]);
                rate = rate + sum;
            }
            double dts = floor_dt;
            if (rate > 0.0) dts = o_min2(dts, cfl/rate);
            long q = II(B, i, j, k);
            F->dt[q] = o_min2(F->dt[q], dts);
        }
    }
}

/* bound_removal_dt (Mod_dt.f90:220-242): a cell the coupler takes mass out of steps no further
 * than empties it. */
static void bound_removal_dt(orc_ctx* c, int p) {
    if (!c->have_imp[p]) return;
    int nc = nc_of(c, p);
    for (int b = 0; b < c->nb; ++b) {
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
            long q = II(B, i, j, k);
            double out = -F->imports[nc*q];
            if (!(out > 0.0)) continue;
            double dts = F->prim[nc*CI(B, i, j, k)]/out;
            if (c->P.time_accurate) c->dtglobal = o_min2(c->dtglobal, dts);
            else F->dt[q] = o_min2(F->dt[q], dts);
        }
    }
}

/* add_births (Lib_Residual.f90:164-210) with the coupler's imports: residual + imports * dt, then the
 * frozen slots to zero. */
static void add_births(orc_ctx* c, int p) {
    if (!c->have_imp[p]) return;
    int nc = nc_of(c, p);
    const ice_gpu_family* mat = &c->P.fam[p];
    for (int b = 0; b < c->nb; ++b) {
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        for (long q = 0; q < ncells(B); ++q) {
            double* r = F->residual + nc*q;
            for (int v = 0; v < nc; ++v) r[v] = r[v] + F->imports[nc*q + v]*F->dt[q];
            for (int f = 0; f < mat->nfrozen; ++f) r[mat->frozen[f] - 1] = 0.0;
        }
    }
}

/* Two-way coupling on or off (twcoupled): the step's weighted source of every family is kept. */
int orc_set_exchange(orc_ctx* c, int on) {
    if (on && !c->P.coupled) return seterr(c, ICE_GPU_EINVAL, "set_exchange: the run is not coupled to a gas");
    if (on && !c->exchange)
        for (int b = 0; b < c->nb; ++b) for (int p = 0; p < c->P.nfam; ++p) {
            oblk* B = &c->blk[b];
            free(B->fam[p].source_step);
            B->fam[p].source_step = (double*)calloc((size_t)nc_of(c, p)*ncells(B), sizeof(double));
        }
    c->exchange = on != 0;
    return 0;
}

/* add_stage_source (Mod_Explicit.f90:257-280) with RK_accumulate (Lib_RK.f90:28-44): stage 1 starts the
 * running sum, stage k > 1 makes it (sum + source) * c_k. After the last stage it is the step's source
 * (hand_step_source, Mod_Explicit.f90:284-300). With one stage it is that stage's source. */
static void add_stage_source(orc_ctx* c, int p, int srk) {
    static const double RKC[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0/3.0}};
    int nc = nc_of(c, p);
    double ck = RKC[c->P.nrk - 1][srk - 1];
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        ofam* F = &B->fam[p];
        for (long q = 0; q < (long)nc*ncells(B); ++q)
            F->source_step[q] = srk == 1 ? F->source[q] : (F->source_step[q] + F->source[q]) * ck;
    }
}

/* exchange_rate (Mod_Exchange.f90:60-78) of family p1 in block b1 over the last step: (5, ni, nj, nk) of
 * mass, momentum and energy the gas receives, the negated step source (no burning family). */
int orc_exchange_rate(orc_ctx* c, int b1, int p1, double* x) {
    if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam || !x) return seterr(c, ICE_GPU_EINVAL, "exchange_rate: bad arguments");
    if (!c->exchange) return seterr(c, ICE_GPU_ENOTREADY, "exchange_rate: exchange is off (set_exchange)");
    int p = p1 - 1, nc = nc_of(c, p), ie = o_nbase(c->P.fam[p].closure) - 2;
    oblk* B = &c->blk[b1 - 1];
    for (long q = 0; q < ncells(B); ++q) {
        const double* a = B->fam[p].source_step + (long)nc*q;
        x[5*q] = -a[0]; x[5*q + 1] = -a[1]; x[5*q + 2] = -a[2]; x[5*q + 3] = -a[3]; x[5*q + 4] = -a[ie];
    }
    return 0;
}

/* --------------------------------------------------------------- norm */
static int residual_norm(orc_ctx* c) {
    int nf = c->P.nfam;
    double* part = (double*)calloc((size_t)5*c->nb*nf, sizeof(double));
    for (int b = 0; b < c->nb; ++b) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        for (int p = 0; p < nf; ++p) {
            int nc = nc_of(c, p), iT = o_nbase(c->P.fam[p].closure) - 2;
            double* acc = part + 5*((long)b*nf + p);
            const double* n = B->fam[p].prim; const double* o = B->fam[p].prim_old;
            for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i) {
                long q = nc*CI(B, i, j, k);
                double r[5] = {fabs(n[q] - o[q]), fabs(n[q + 1] - o[q + 1]), fabs(n[q + 2] - o[q + 2]),
                               fabs(n[q + 3] - o[q + 3]), fabs(n[q + iT] - o[q + iT])};
                for (int m = 0; m < 5; ++m) acc[m] = acc[m] + r[m]*r[m];
            }
        }
    }
    /* a split run: every block's partial sums come from the one rank that steps it (the others add
     * zeros), so the sums below keep the block order of an unsplit run */
    if (halo_reduce(c, ICE_GPU_HALO_NORM, part, 5L*c->nb*nf)) { free(part); return ICE_GPU_EEXCH; }
    double tot[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < c->nb; ++b) for (int p = 0; p < nf; ++p) for (int m = 0; m < 5; ++m) tot[m] = tot[m] + part[5*((long)b*nf + p) + m];
    for (int m = 0; m < 5; ++m) c->residuo[m] = sqrt(tot[m]);
    for (int p = 0; p < nf; ++p) {
        double fam[5] = {0, 0, 0, 0, 0};
        for (int b = 0; b < c->nb; ++b) for (int m = 0; m < 5; ++m) fam[m] = fam[m] + part[5*((long)b*nf + p) + m];
        for (int m = 0; m < 5; ++m) c->residuofam[5*p + m] = sqrt(fam[m]);
    }
    free(part);
    c->have_norm = 1;
    return 0;
}

int orc_residual_norm(orc_ctx* c, double* total, double* fam) {
    if (residual_norm(c)) return ICE_GPU_EEXCH;
    memcpy(total, c->residuo, sizeof(double)*5);
    if (fam) memcpy(fam, c->residuofam, sizeof(double)*5*c->P.nfam);
    return 0;
}

/* ------------------------------------------------------------ the step */
static int due(int iter, int every) { return every > 0 && iter % every == 0; }

/* Explicit_Step (Mod_Explicit.f90:11-245) on the one-way-coupled, non-burning path. */
static int explicit_step(orc_ctx* c, ice_gpu_step_out* out) {
    int nf = c->P.nfam;
    c->iter += 1; c->iter_from_call += 1;
    c->dtglobal = (double)1e+5f;
    for (int p = 0; p < nf; ++p) { compute_dt(c, p); bound_empty_dt(c, p); bound_removal_dt(c, p); }
    if (halo_reduce(c, ICE_GPU_HALO_DT, &c->dtglobal, 1)) return ICE_GPU_EEXCH;
    if (c->P.time_accurate) {
        c->time = c->time + c->dtglobal;
        for (int b = 0; b < c->nb; ++b) for (int p = 0; p < nf; ++p) {
            if (!OWN(c, b)) continue;
            oblk* B = &c->blk[b];
            for (long q = 0; q < ncells(B); ++q) B->fam[p].dt[q] = c->dtglobal;
        }
    }
    for (int b = 0; b < c->nb; ++b) for (int p = 0; p < nf; ++p) {
        if (!OWN(c, b)) continue;
        oblk* B = &c->blk[b];
        int nc = nc_of(c, p);
        for (int k = 1; k <= B->nk; ++k) for (int j = 1; j <= B->nj; ++j) for (int i = 1; i <= B->ni; ++i)
            memcpy(B->fam[p].prim_old + nc*CI(B, i, j, k), B->fam[p].prim + nc*CI(B, i, j, k), sizeof(double)*nc);
    }
    for (int p = 0; p < nf; ++p) {
        for (int srk = 1; srk <= c->P.nrk; ++srk) {
            for (int b = 0; b < c->nb; ++b) if (OWN(c, b)) memset(c->blk[b].fam[p].residual, 0, sizeof(double)*nc_of(c, p)*ncells(&c->blk[b]));
            if (c->P.coupled) compute_source(c, p);
            if (c->P.coupled && c->exchange) add_stage_source(c, p, srk);
            if (halo_exchange(c, ICE_GPU_HALO_CELLS, p)) return ICE_GPU_EEXCH;
            compute_ghost(c, p);
            compute_beta(c, p);
            if (halo_exchange(c, ICE_GPU_HALO_BETA, p)) return ICE_GPU_EEXCH;
            int rb = compute_bound(c, p);
            if (rb < 0) return ICE_GPU_EEXCH;
            if (rb) { c->status |= ICE_GPU_ST_BAD_RECON; return ICE_GPU_ESTATE; }
            if (compute_flux(c, p)) { c->status |= ICE_GPU_ST_BAD_RECON; return ICE_GPU_ESTATE; }
            compute_residual(c, p);
            add_births(c, p);
            if (c->P.irs) residual_smoothing(c, p);
            if (state_update(c, p, srk)) { c->status |= ICE_GPU_ST_NAN_STATE; return ICE_GPU_ESTATE; }
        }
    }
    /* res-threshold ends a steady run once its density residual has fallen by res_threshold from the
     * first non-zero one (Mod_Explicit.f90:193-240): a residual of zero (a cloud at rest at its first
     * one-stage step) is no reference, and until one has come the residual ends nothing */
    int res_stop = !c->P.time_accurate && c->P.res_threshold > 0.0;
    int need_norm = res_stop || due(c->iter, c->P.res_diter) || due(c->iter, c->P.shell_diter) ||
                    c->iter_from_call >= c->P.itermax || c->time >= c->P.time_threshold;
    c->have_norm = 0;
    if (need_norm && residual_norm(c)) return ICE_GPU_EEXCH;
    if (res_stop && c->res_reference == 0.0) c->res_reference = c->residuo[0];
    c->res_end = res_stop && c->res_reference > 0.0 && c->residuo[0] <= c->P.res_threshold * c->res_reference;
    int endsim = c->iter_from_call >= c->P.itermax || c->res_end || c->time >= c->P.time_threshold;
    int iosim = (c->P.sol_diter > 0 && c->iter % c->P.sol_diter == 0);
    if (out) {
        out->todo = endsim ? 3 : iosim ? 2 : 1;
        out->have_norm = c->have_norm;
        memcpy(out->residual, c->residuo, sizeof(double)*5);
    }
    return 0;
}

int orc_step(orc_ctx* c, int nsteps, ice_gpu_step_out* out) {
    int rc = 0;
    if (c->nchim > 0 && !c->have_chim)
        return seterr(c, ICE_GPU_ENOTREADY, "%d chimera records have no donors (set_chimera)", c->nchim);
    /* the sources of a coupled run and the ghosts of its 401 and 403 inlets read the gas of their
     * block: a block without one is refused before any step (an uncoupled run's injecting 401 or 403
     * inlets were refused by set_records) */
    for (int b = 0; b < c->nb; ++b)
        if (c->P.coupled && !c->blk[b].gprim)
            return seterr(c, ICE_GPU_ENOTREADY, "a coupled run needs the gas of every block (block %d has none)", b + 1);
    c->res_end = 0;
    for (int s = 0; s < nsteps && !rc && !c->res_end; ++s) rc = explicit_step(c, out);
    if (out) {
        out->dtglobal = c->dtglobal; out->time = c->time; out->iter = c->iter;
        out->status = c->status; out->nfloored = c->nfloored; out->device_ms = 0.0;
        out->nrealized = 0;
    }
    return rc;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

/* ------------------------------------------------- unit-level entry points */
/* For the known-answer tests of the reference's unit suite. */
int orc_reconstruct(int closure, int limiter, const double* prev, const double* local, const double* next,
                    const double* next2, double dl0, double dl1, double dl2, double dll, double dlr,
                    double* priml, double* primr, double beta) {
    return o_reconstruct(closure, limiter, prev, local, next, next2, dl0, dl1, dl2, dll, dlr, priml, primr, beta);
}
double orc_limiter(int limiter, double x, double y, double cx, double cy) { return o_limiter(limiter, x, y, cx, cy); }
void orc_riemann(int solver, int closure, const double* p1, const double* p4, const double* n, double* f,
                 const ice_gpu_family* m) { o_riemann(solver, closure, p1, p4, n, f, m); }
double orc_cell_source(int closure, const double* p, const double* gas, double gR, double ggam, double gk, double gmu,
                       const ice_gpu_family* m, int drag, int heat, int blow, double* s) {
    return o_cell_source(closure, p, gas, gR, ggam, gk, gmu, m, drag, heat, blow, s);
}
double orc_drag(double Re, double Ma, double G, double Tr, int sel) { return o_drag(Re, Ma, G, Tr, sel); }
double orc_heat(double Re, double Pr, double Ma, int sel) { return o_heat(Re, Pr, Ma, sel); }
void orc_evaporation(double rhog, double Tg, double gamma, double Rg, double mug, double kg, double Tp, double dp,
                     double Re, int evap, int intf, const double* ep, double* mdot, double* Qd, int* ovr) {
    o_evaporation(rhog, Tg, gamma, Rg, mug, kg, Tp, dp, Re, evap, intf, ep, mdot, Qd, ovr);
}
double orc_blowing(double gamma, double Rg, double mug, double kg, double rhop, double dp, double mp, double mdot) {
    return o_blowing(gamma, Rg, mug, kg, rhop, dp, mp, mdot);
}
void orc_prim2cons(int cl, const double* p, double* c, const ice_gpu_family* m) { o_prim2cons(cl, p, c, m); }
/* the elementary functions of include/ice_math.h, for their accuracy test */
double orc_math(int fn, double x, double y) {
    switch (fn) {
    case 0: return ice_exp(x);
    case 1: return ice_log(x);
    case 2: return ice_pow(x, y);
    case 3: return ice_tanh(x);
    case 4: return ice_expm1(x);
    case 5: return ice_log10(x);
    }
    return 0.0;
}
void orc_cons2prim(int cl, const double* c, double* p, const ice_gpu_family* m) { o_cons2prim(cl, c, p, m); }
