/*
 * fdtd_oracle.c - CPU f64 restatement of the reference FDTD time step.
 *
 * TEST INFRASTRUCTURE ONLY (see fdtd_oracle.h): the checker for the GPU
 * engine. Each function names the reference lines (skyhoffert/CourantEM
 * solver/src/...) whose arithmetic it restates. The per-point operation order
 * is kept (bulk curl, then the CPML corrections axis by axis, then the post
 * phase in its fixed order) so that, fed the reference plan, it reproduces
 * the reference cem_step to the bit.
 */
#include "fdtd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define MU0 1.25663706212e-6
#define EPS0 8.8541878128e-12
#define MAXP 600

typedef struct {
    int n;
    int *comp;
    size_t *idx;
    double *w, *cs;
    double R;
    double *acc, *acc2; /* port: V and I; probes: acc */
} olist;

struct orc_sim {
    int n[3];
    size_t si, sj, N;
    double dt;
    const double *ca[3], *cb[3], *ide[3], *idh[3], *be[3], *ce[3], *bh[3], *ch[3], *d[3], *dd[3];
    int npml[6], has_pml;
    double *E[3], *H[3];
    double *psiE[3][2], *psiH[3][2];
    long step;
    int nf;
    double *freq, *phE, *phH, *rotE, *src_acc;
    int nport, nvp, nip;
    olist port[MAXP], vp[MAXP], ip[MAXP];
    double vold[MAXP];
    olist msrc;
    int has_msrc, excited;
    long nwave;
    double *wl, *wm;
    int nd, npole;
    int *dcomp;
    size_t *didx;
    double *dcb, *dbeta, *dk, *dJ, *dEold;
    int ns, nterm;
    int *scomp, *hcomp;
    size_t *sidx, *hidx;
    double *hw, *sc, *se, *sy;
};

static char g_err[128];
const char *orc_last_error(void) { return g_err; }

static size_t IDX(const orc_sim *o, int i, int j, int k) { return (size_t)i * o->si + (size_t)j * o->sj + (size_t)k; }

static int imax(int a, int b) { return a > b ? a : b; }

/* CPML slab ranges and compact layout (reference sim.c:641-678) */
static void ranges(const orc_sim *o, int a, int is_e, int r[2][2]) {
    int n = o->n[a], lo = o->npml[2 * a], hi = o->npml[2 * a + 1];
    if (is_e) {
        r[0][0] = 1; r[0][1] = lo;
        r[1][0] = n - hi; r[1][1] = n - 1;
        if (lo == 0) { r[0][0] = 1; r[0][1] = 0; }
        if (hi == 0) { r[1][0] = 1; r[1][1] = 0; }
    } else {
        r[0][0] = 0; r[0][1] = lo - 1;
        r[1][0] = n - hi; r[1][1] = n - 1;
    }
}
static size_t per_plane(const orc_sim *o, int a) {
    const int *n = o->n;
    return a == 0 ? (size_t)(n[1] + 1) * (n[2] + 1) : a == 1 ? (size_t)(n[0] + 1) * (n[2] + 1) : (size_t)(n[0] + 1) * (n[1] + 1);
}
static size_t nplanes(const orc_sim *o, int a, int is_e) {
    int r[2][2];
    ranges(o, a, is_e, r);
    size_t c = 0;
    for (int sd = 0; sd < 2; sd++) if (r[sd][1] >= r[sd][0]) c += (size_t)(r[sd][1] - r[sd][0] + 1);
    return c;
}
static size_t plane_of(const orc_sim *o, int a, int is_e, int idx) {
    int r[2][2];
    ranges(o, a, is_e, r);
    size_t lo = r[0][1] >= r[0][0] ? (size_t)(r[0][1] - r[0][0] + 1) : 0;
    return idx <= r[0][1] && idx >= r[0][0] ? (size_t)(idx - r[0][0]) : lo + (size_t)(idx - r[1][0]);
}
static size_t in_plane(const orc_sim *o, int a, int i, int j, int k) {
    return a == 0 ? (size_t)j * (o->n[2] + 1) + k : a == 1 ? (size_t)i * (o->n[2] + 1) + k : (size_t)i * (o->n[1] + 1) + j;
}

orc_sim *orc_create(int nx, int ny, int nz, double dt, const double *const *ca, const double *const *cb,
                    const double *const *ide, const double *const *idh, const double *const *be,
                    const double *const *ce, const double *const *bh, const double *const *ch,
                    const double *const *d, const double *const *dd, const int *npml) {
    orc_sim *o = calloc(1, sizeof *o);
    o->n[0] = nx; o->n[1] = ny; o->n[2] = nz;
    o->sj = (size_t)nz + 1;
    o->si = o->sj * ((size_t)ny + 1);
    o->N = o->si * ((size_t)nx + 1);
    o->dt = dt;
    for (int a = 0; a < 3; a++) {
        o->ca[a] = ca[a]; o->cb[a] = cb[a]; o->ide[a] = ide[a]; o->idh[a] = idh[a];
        o->be[a] = be[a]; o->ce[a] = ce[a]; o->bh[a] = bh[a]; o->ch[a] = ch[a]; o->d[a] = d[a]; o->dd[a] = dd[a];
        o->E[a] = calloc(o->N, sizeof(double));
        o->H[a] = calloc(o->N, sizeof(double));
    }
    for (int f = 0; f < 6; f++) { o->npml[f] = npml[f]; if (npml[f]) o->has_pml = 1; }
    if (o->has_pml)
        for (int c = 0; c < 3; c++)
            for (int w = 0; w < 2; w++) {
                int a = (c + w + 1) % 3;
                o->psiE[c][w] = calloc(nplanes(o, a, 1) * per_plane(o, a) + 1, sizeof(double));
                o->psiH[c][w] = calloc(nplanes(o, a, 0) * per_plane(o, a) + 1, sizeof(double));
            }
    o->excited = -1;
    return o;
}

static void free_list(olist *l) { free(l->comp); free(l->idx); free(l->w); free(l->cs); free(l->acc); free(l->acc2); }

void orc_destroy(orc_sim *o) {
    if (!o) return;
    for (int a = 0; a < 3; a++) {
        free(o->E[a]); free(o->H[a]);
        for (int w = 0; w < 2; w++) { free(o->psiE[a][w]); free(o->psiH[a][w]); }
    }
    for (int p = 0; p < o->nport; p++) free_list(&o->port[p]);
    for (int p = 0; p < o->nvp; p++) free_list(&o->vp[p]);
    for (int p = 0; p < o->nip; p++) free_list(&o->ip[p]);
    free_list(&o->msrc);
    free(o->freq); free(o->phE); free(o->phH); free(o->rotE); free(o->src_acc); free(o->wl); free(o->wm);
    free(o->dcomp); free(o->didx); free(o->dcb); free(o->dbeta); free(o->dk); free(o->dJ); free(o->dEold);
    free(o->scomp); free(o->hcomp); free(o->sidx); free(o->hidx); free(o->hw); free(o->sc); free(o->se); free(o->sy);
    free(o);
}

int orc_set_frequencies(orc_sim *o, int nf, const double *f) {
    o->nf = nf;
    o->freq = malloc(nf * sizeof(double));
    memcpy(o->freq, f, nf * sizeof(double));
    o->phE = calloc(2 * nf, sizeof(double));
    o->phH = calloc(2 * nf, sizeof(double));
    o->rotE = calloc(2 * nf, sizeof(double));
    o->src_acc = calloc(2 * nf, sizeof(double));
    /* rotation per step (reference sim.c:558-562) */
    for (int q = 0; q < nf; q++) {
        double w = 2 * M_PI * f[q];
        o->rotE[2 * q] = cos(w * o->dt);
        o->rotE[2 * q + 1] = -sin(w * o->dt);
    }
    return 0;
}

static void fill_list(orc_sim *o, olist *l, int n, const double *idx, const double *w, const double *cs) {
    l->n = n;
    l->comp = calloc(n ? n : 1, sizeof(int));
    l->idx = calloc(n ? n : 1, sizeof(size_t));
    l->w = calloc(n ? n : 1, sizeof(double));
    l->cs = calloc(n ? n : 1, sizeof(double));
    for (int e = 0; e < n; e++) {
        size_t g = (size_t)idx[e];
        l->comp[e] = (int)(g / o->N);
        l->idx[e] = g % o->N;
        l->w[e] = w[e];
        if (cs) l->cs[e] = cs[e];
    }
    l->acc = calloc(2 * o->nf, sizeof(double));
    l->acc2 = calloc(2 * o->nf, sizeof(double));
}

int orc_add_port(orc_sim *o, int n, const double *idx, const double *vw, const double *cs, double R) {
    if (o->nport >= MAXP || !o->nf) { strcpy(g_err, "port: set frequencies first / too many"); return -1; }
    olist *l = &o->port[o->nport];
    fill_list(o, l, n, idx, vw, cs);
    l->R = R;
    return o->nport++;
}

int orc_add_vprobe(orc_sim *o, int n, const double *idx, const double *w) {
    if (o->nvp >= MAXP || !o->nf) { strcpy(g_err, "vprobe"); return -1; }
    fill_list(o, &o->vp[o->nvp], n, idx, w, NULL);
    return o->nvp++;
}

int orc_add_iprobe(orc_sim *o, int n, const double *idx, const double *w) {
    if (o->nip >= MAXP || !o->nf) { strcpy(g_err, "iprobe"); return -1; }
    fill_list(o, &o->ip[o->nip], n, idx, w, NULL);   /* H indices arrive as (comp-3)*N + q */
    return o->nip++;
}

int orc_set_mode_source(orc_sim *o, int n, const double *idx, const double *w) {
    fill_list(o, &o->msrc, n, idx, w, NULL);
    return 0;
}

int orc_set_waveforms(orc_sim *o, long nsteps, const double *lumped, const double *mode, int excited, int has_mode) {
    o->nwave = nsteps;
    o->wl = malloc(nsteps * sizeof(double));
    o->wm = malloc(nsteps * sizeof(double));
    memcpy(o->wl, lumped, nsteps * sizeof(double));
    memcpy(o->wm, mode, nsteps * sizeof(double));
    o->excited = excited;
    o->has_msrc = has_mode;
    return 0;
}

int orc_set_disp(orc_sim *o, int nd, int npole, const double *idx, const double *cb, const double *beta,
                 const double *k) {
    o->nd = nd; o->npole = npole;
    o->dcomp = malloc(nd * sizeof(int));
    o->didx = malloc(nd * sizeof(size_t));
    o->dcb = malloc(nd * sizeof(double));
    o->dbeta = malloc((size_t)nd * npole * sizeof(double));
    o->dk = malloc(npole * sizeof(double));
    o->dJ = calloc((size_t)nd * npole, sizeof(double));
    o->dEold = calloc(nd, sizeof(double));
    for (int e = 0; e < nd; e++) {
        size_t g = (size_t)idx[e];
        o->dcomp[e] = (int)(g / o->N);
        o->didx[e] = g % o->N;
        o->dcb[e] = cb[e];
    }
    memcpy(o->dbeta, beta, (size_t)nd * npole * sizeof(double));
    memcpy(o->dk, k, npole * sizeof(double));
    return 0;
}

int orc_set_sibc(orc_sim *o, int ns, int nterm, const double *idx, const double *hidx, const double *hw,
                 const double *c, const double *e) {
    o->ns = ns; o->nterm = nterm;
    o->scomp = malloc(ns * sizeof(int));
    o->sidx = malloc(ns * sizeof(size_t));
    o->hcomp = malloc(4 * (size_t)ns * sizeof(int));
    o->hidx = malloc(4 * (size_t)ns * sizeof(size_t));
    o->hw = malloc(4 * (size_t)ns * sizeof(double));
    o->sc = malloc(nterm * sizeof(double));
    o->se = malloc(nterm * sizeof(double));
    o->sy = calloc((size_t)ns * nterm, sizeof(double));
    for (int q = 0; q < ns; q++) {
        size_t g = (size_t)idx[q];
        o->scomp[q] = (int)(g / o->N);
        o->sidx[q] = g % o->N;
        for (int f = 0; f < 4; f++) {
            size_t h = (size_t)hidx[4 * q + f];
            o->hcomp[4 * q + f] = (int)(h / o->N);
            o->hidx[4 * q + f] = h % o->N;
            o->hw[4 * q + f] = hw[4 * q + f];
        }
    }
    memcpy(o->sc, c, nterm * sizeof(double));
    memcpy(o->se, e, nterm * sizeof(double));
    return 0;
}

/* H update with the CPML corrections applied axis by axis afterwards
 * (reference sim.c:579-606 bulk, :680-754 psi recursions) */
static void update_h(orc_sim *o) {
    const int *n = o->n;
    const double dth = o->dt / MU0;
    const size_t st[3] = {o->si, o->sj, 1};
    for (int c = 0; c < 3; c++) {
        int a1 = (c + 1) % 3, a2 = (c + 2) % 3;
        int lim[3] = {n[0], n[1], n[2]};   /* H_c: index c runs to n[c] inclusive, others < n */
        lim[c] = n[c] + 1;
        double *Hc = o->H[c];
        const double *E1 = o->E[a2], *E2 = o->E[a1];
        for (int i = 0; i < lim[0]; i++)
            for (int j = 0; j < lim[1]; j++)
                for (int k = 0; k < lim[2]; k++) {
                    int ijk[3] = {i, j, k};
                    size_t q = IDX(o, i, j, k);
                    Hc[q] -= dth * ((E1[q + st[a1]] - E1[q]) * o->idh[a1][ijk[a1]] - (E2[q + st[a2]] - E2[q]) * o->idh[a2][ijk[a2]]);
                }
    }
    if (!o->has_pml) return;
    for (int a = 0; a < 3; a++) {
        int r[2][2];
        ranges(o, a, 0, r);
        /* the two H components with a derivative along a: c = a+2 (term 1) and c = a+1 (term 2) */
        const int cs2[2] = {(a + 2) % 3, (a + 1) % 3};
        for (int t = 0; t < 2; t++) {
            int c = cs2[t], w = t == 0 ? 0 : 1;
            int ec = t == 0 ? (c + 2) % 3 : (c + 1) % 3; /* differentiated E component */
            double sgn = t == 0 ? -1.0 : 1.0;
            double *psi = o->psiH[c][w];
            int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
            hi[c] = n[c] + 1;
            for (int sd = 0; sd < 2; sd++)
                for (int m = r[sd][0]; m <= r[sd][1]; m++) {
                    double b = o->bh[a][m], cc = o->ch[a][m], id = 1.0 / o->d[a][m];
                    size_t base = plane_of(o, a, 0, m) * per_plane(o, a);
                    int l2[3] = {lo[0], lo[1], lo[2]}, h2[3] = {hi[0], hi[1], hi[2]};
                    l2[a] = m; h2[a] = m + 1;
                    for (int i = l2[0]; i < h2[0]; i++)
                        for (int j = l2[1]; j < h2[1]; j++)
                            for (int k = l2[2]; k < h2[2]; k++) {
                                size_t q = IDX(o, i, j, k), p = base + in_plane(o, a, i, j, k);
                                psi[p] = b * psi[p] + cc * (o->E[ec][q + st[a]] - o->E[ec][q]) * id;
                                if (sgn < 0) o->H[c][q] -= dth * psi[p];
                                else o->H[c][q] += dth * psi[p];
                            }
                }
        }
    }
}

/* E update with the CPML corrections (reference sim.c:608-637 bulk, :756-832 psi) */
static void update_e(orc_sim *o) {
    const int *n = o->n;
    const size_t st[3] = {o->si, o->sj, 1};
    for (int c = 0; c < 3; c++) {
        int a1 = (c + 1) % 3, a2 = (c + 2) % 3;
        double *Ec = o->E[c];
        const double *H1 = o->H[a2], *H2 = o->H[a1];
        int lo[3] = {1, 1, 1}, hi[3] = {n[0], n[1], n[2]};  /* transverse 1..n-1, own 0..n-1 */
        lo[c] = 0;
        for (int i = lo[0]; i < hi[0]; i++)
            for (int j = lo[1]; j < hi[1]; j++)
                for (int k = lo[2]; k < hi[2]; k++) {
                    int ijk[3] = {i, j, k};
                    size_t q = IDX(o, i, j, k);
                    Ec[q] = o->ca[c][q] * Ec[q] + o->cb[c][q] * ((H1[q] - H1[q - st[a1]]) * o->ide[a1][ijk[a1]] - (H2[q] - H2[q - st[a2]]) * o->ide[a2][ijk[a2]]);
                }
    }
    if (!o->has_pml) return;
    for (int a = 0; a < 3; a++) {
        int r[2][2];
        ranges(o, a, 1, r);
        const int cs2[2] = {(a + 2) % 3, (a + 1) % 3};
        for (int t = 0; t < 2; t++) {
            int c = cs2[t], w = t == 0 ? 0 : 1;
            int hc = t == 0 ? (c + 2) % 3 : (c + 1) % 3;
            double *psi = o->psiE[c][w];
            int lo[3] = {1, 1, 1}, hi[3] = {n[0], n[1], n[2]};
            lo[c] = 0;
            for (int sd = 0; sd < 2; sd++)
                for (int m = r[sd][0]; m <= r[sd][1]; m++) {
                    double b = o->be[a][m], cc = o->ce[a][m], id = 1.0 / o->dd[a][m];
                    size_t base = plane_of(o, a, 1, m) * per_plane(o, a);
                    int l2[3] = {lo[0], lo[1], lo[2]}, h2[3] = {hi[0], hi[1], hi[2]};
                    if (m < lo[a] || m >= hi[a]) continue;
                    l2[a] = m; h2[a] = m + 1;
                    for (int i = l2[0]; i < h2[0]; i++)
                        for (int j = l2[1]; j < h2[1]; j++)
                            for (int k = l2[2]; k < h2[2]; k++) {
                                size_t q = IDX(o, i, j, k), p = base + in_plane(o, a, i, j, k);
                                psi[p] = b * psi[p] + cc * (o->H[hc][q] - o->H[hc][q - st[a]]) * id;
                                if (t == 0) o->E[c][q] += o->cb[c][q] * psi[p];
                                else o->E[c][q] -= o->cb[c][q] * psi[p];
                            }
                }
        }
    }
}

static void dft_add(double *acc, const double *ph, int nf, double v) {
    for (int f = 0; f < nf; f++) { acc[2 * f] += v * ph[2 * f]; acc[2 * f + 1] += v * ph[2 * f + 1]; }
}

static double line_sum(const orc_sim *o, const olist *l, int h) {
    double v = 0;
    for (int e = 0; e < l->n; e++) v += (h ? o->H[l->comp[e]] : o->E[l->comp[e]])[l->idx[e]] * l->w[e];
    return v;
}

/* one step: pre, H, mid, E, post (reference sim.c:867-933,951-960) */
static void one_step(orc_sim *o) {
    const int nf = o->nf;
    long sn = o->step;
    if ((sn & 1023) == 0)
        for (int f = 0; f < nf; f++) {
            double w = 2 * M_PI * o->freq[f], tE = (sn + 1) * o->dt, tH = (sn + 0.5) * o->dt;
            o->phE[2 * f] = cos(w * tE); o->phE[2 * f + 1] = -sin(w * tE);
            o->phH[2 * f] = cos(w * tH); o->phH[2 * f + 1] = -sin(w * tH);
        }
    update_h(o);
    for (int p = 0; p < o->nip; p++) dft_add(o->ip[p].acc, o->phH, nf, line_sum(o, &o->ip[p], 1) * o->dt);
    for (int p = 0; p < o->nport; p++) o->vold[p] = line_sum(o, &o->port[p], 0);
    for (int e = 0; e < o->nd; e++) o->dEold[e] = o->E[o->dcomp[e]][o->didx[e]];
    update_e(o);
    /* post (reference sim.c:894-933) */
    for (int e = 0; e < o->nd; e++) {   /* dispersive.c:93-100 */
        double acc = 0;
        for (int p = 0; p < o->npole; p++) acc += 0.5 * (1 + o->dk[p]) * o->dJ[(size_t)p * o->nd + e];
        o->E[o->dcomp[e]][o->didx[e]] -= o->dcb[e] * acc;
    }
    for (int q = 0; q < o->ns; q++) {   /* sibc.c:256-269 */
        double J = 0;
        for (int f = 0; f < 4; f++)
            if (o->hw[4 * q + f] != 0) J += o->hw[4 * q + f] * o->H[o->hcomp[4 * q + f]][o->hidx[4 * q + f]];
        double Ev = 0, *y = &o->sy[(size_t)q * o->nterm];
        for (int k = 0; k < o->nterm; k++) {
            y[k] = o->se[k] * y[k] + (1 - o->se[k]) * J;
            Ev += o->sc[k] * (J - y[k]);
        }
        o->E[o->scomp[q]][o->sidx[q]] = Ev;
    }
    double Vs = o->excited >= 0 && sn < o->nwave ? o->wl[sn] : 0.0;
    if (o->excited >= 0) {
        olist *pt = &o->port[o->excited];
        for (int e = 0; e < pt->n; e++) o->E[pt->comp[e]][pt->idx[e]] += pt->cs[e] * Vs;
        dft_add(o->src_acc, o->phH, nf, Vs * o->dt);
    }
    if (o->has_msrc) {
        double v = sn < o->nwave ? o->wm[sn] : 0.0;
        for (int e = 0; e < o->msrc.n; e++) o->E[o->msrc.comp[e]][o->msrc.idx[e]] += o->msrc.w[e] * v;
        dft_add(o->src_acc, o->phH, nf, v * o->dt);
    }
    if (o->nd) {   /* dispersive.c:102-112 */
        double idt = 1.0 / o->dt;
        for (int e = 0; e < o->nd; e++) {
            double dE = (o->E[o->dcomp[e]][o->didx[e]] - o->dEold[e]) * idt;
            for (int p = 0; p < o->npole; p++) {
                size_t q = (size_t)p * o->nd + e;
                o->dJ[q] = o->dk[p] * o->dJ[q] + o->dbeta[q] * dE;
            }
        }
    }
    for (int p = 0; p < o->nport; p++) {
        olist *pt = &o->port[p];
        double V = 0.5 * (line_sum(o, pt, 0) + o->vold[p]);
        double vs = p == o->excited ? Vs : 0.0;
        double I = (vs - V) / pt->R;
        dft_add(pt->acc, o->phH, nf, V * o->dt);
        dft_add(pt->acc2, o->phH, nf, I * o->dt);
    }
    for (int p = 0; p < o->nvp; p++) dft_add(o->vp[p].acc, o->phE, nf, line_sum(o, &o->vp[p], 0) * o->dt);
    for (int f = 0; f < nf; f++) {
        double a = o->phE[2 * f], b = o->phE[2 * f + 1], c = o->rotE[2 * f], d = o->rotE[2 * f + 1];
        o->phE[2 * f] = a * c - b * d; o->phE[2 * f + 1] = a * d + b * c;
        a = o->phH[2 * f]; b = o->phH[2 * f + 1];
        o->phH[2 * f] = a * c - b * d; o->phH[2 * f + 1] = a * d + b * c;
    }
    o->step++;
}

void orc_step(orc_sim *o, long n) { for (long t = 0; t < n; t++) one_step(o); }
long orc_step_count(const orc_sim *o) { return o->step; }

/* W = 1/2 sum (dt/cb) E^2 dV + 1/2 sum mu0 H^2 dV (reference sim.c:970-994) */
double orc_energy(const orc_sim *o) {
    const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
    double we = 0, wm = 0;
    for (int c = 0; c < 3; c++) {
        int ua = (c + 1) % 3, va = (c + 2) % 3;
        for (int i = 0; i <= nx; i++)
            for (int j = 0; j <= ny; j++)
                for (int k = 0; k <= nz; k++) {
                    int ijk[3] = {i, j, k};
                    size_t q = IDX(o, i, j, k);
                    if (ijk[c] < o->n[c] && o->cb[c][q] != 0) {
                        double vol = o->d[c][ijk[c]] * o->dd[ua][ijk[ua]] * o->dd[va][ijk[va]];
                        double eps = o->dt / o->cb[c][q];
                        we += 0.5 * eps * o->E[c][q] * o->E[c][q] * vol;
                    }
                    if (ijk[ua] < o->n[ua] && ijk[va] < o->n[va]) {
                        double vol = o->dd[c][ijk[c]] * o->d[ua][ijk[ua]] * o->d[va][ijk[va]];
                        wm += 0.5 * MU0 * o->H[c][q] * o->H[c][q] * vol;
                    }
                }
    }
    (void)imax;
    return we + wm;
}

double *orc_field(orc_sim *o, int comp) { return comp < 3 ? o->E[comp] : o->H[comp - 3]; }
const double *orc_port_v(const orc_sim *o, int p) { return o->port[p].acc; }
const double *orc_port_i(const orc_sim *o, int p) { return o->port[p].acc2; }
const double *orc_vprobe(const orc_sim *o, int p) { return o->vp[p].acc; }
const double *orc_iprobe(const orc_sim *o, int p) { return o->ip[p].acc; }
const double *orc_source_spectrum(const orc_sim *o) { return o->src_acc; }
