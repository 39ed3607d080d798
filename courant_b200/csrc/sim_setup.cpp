// Host-side simulation setup: creation, geometry, ports, probes and the FP64
// update plan built by cem_finalize.
//
// The plan must be the reference plan to the last bit, because the f64 core
// (skyhoffert/CourantEM solver/src/sim.c) is the oracle every result is judged
// against. Each formula therefore evaluates the same expression in the same
// order as the reference line cited beside it; the data structures, the loops
// and the device hand-off around them are this library's own.
#include "sim.hpp"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <thread>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace cb2 {

namespace {
thread_local char g_error[256] = "";
}

void set_error(const char *msg) {
    std::snprintf(g_error, sizeof g_error, "%s", msg);
}

// Area-weighted average of eps_r and sigma over the (up to) four cells sharing
// the edge along c at (i,j,k); any PEC cell makes the edge PEC.
// (reference sim.c:346-367)
void edge_material(const cem_sim *s, int c, int i, int j, int k, double *eps, double *sig, int *pec) {
    const int ua = (c + 1) % 3, va = (c + 2) % 3;
    double wsum = 0, es = 0, ss = 0;
    *pec = 0;
    for (int du = -1; du <= 0; du++)
        for (int dv = -1; dv <= 0; dv++) {
            int cc[3] = {i, j, k};
            cc[ua] += du;
            cc[va] += dv;
            if (cc[ua] < 0 || cc[ua] >= s->n[ua] || cc[va] < 0 || cc[va] >= s->n[va]) continue;
            if (cc[c] >= s->n[c]) continue;
            const size_t q = idx3(s, cc[0], cc[1], cc[2]);
            const double w = s->d[ua][cc[ua]] * s->d[va][cc[va]];
            if (s->cell_pec[q]) *pec = 1;
            es += w * s->eps_r[q];
            ss += w * s->sigma[q];
            wsum += w;
        }
    *eps = wsum > 0 ? es / wsum : 1.0;
    *sig = wsum > 0 ? ss / wsum : 0.0;
}

// Area-weighted Debye weights around an edge; returns 1 if any is non-zero.
// (reference dispersive.c:65-87)
int edge_debye(const cem_sim *s, int c, int i, int j, int k, double *deps) {
    if (!s->npole) return 0;
    const int ua = (c + 1) % 3, va = (c + 2) % 3;
    double wsum = 0;
    for (int p = 0; p < s->npole; p++) deps[p] = 0;
    for (int du = -1; du <= 0; du++)
        for (int dv = -1; dv <= 0; dv++) {
            int cc[3] = {i, j, k};
            cc[ua] += du;
            cc[va] += dv;
            if (cc[ua] < 0 || cc[ua] >= s->n[ua] || cc[va] < 0 || cc[va] >= s->n[va]) continue;
            const size_t q = idx3(s, cc[0], cc[1], cc[2]);
            const double w = s->d[ua][cc[ua]] * s->d[va][cc[va]];
            for (int p = 0; p < s->npole; p++) deps[p] += w * s->cell_deps[p][q];
            wsum += w;
        }
    int any = 0;
    for (int p = 0; p < s->npole; p++) {
        deps[p] = wsum > 0 ? deps[p] / wsum : 0;
        if (deps[p] != 0) any = 1;
    }
    return any;
}

// CPML slab ranges for derivative axis a: E auxiliaries live on nodes
// 1..lo and n-hi..n-1, H auxiliaries on cells 0..lo-1 and n-hi..n-1.
// (reference sim.c:641-653)
void pml_ranges(const cem_sim *s, int a, int is_e, int r[2][2]) {
    const int n = s->n[a], lo = s->npml[2 * a], hi = s->npml[2 * a + 1];
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

// Points per CPML plane normal to axis a (full node extent of the other two
// axes) and planes per axis: the compact auxiliary layout of the reference
// (sim.c:655-678), kept because checkpoints and cem_state_array expose it.
size_t pml_per(const cem_sim *s, int a) {
    const int *n = s->n;
    if (a == 0) return (size_t)(n[1] + 1) * (n[2] + 1);
    if (a == 1) return (size_t)(n[0] + 1) * (n[2] + 1);
    return (size_t)(n[0] + 1) * (n[1] + 1);
}

static size_t pml_planes(const cem_sim *s, int a, int is_e) {
    int r[2][2];
    pml_ranges(s, a, is_e, r);
    size_t planes = 0;
    for (int sd = 0; sd < 2; sd++)
        if (r[sd][1] >= r[sd][0]) planes += (size_t)(r[sd][1] - r[sd][0] + 1);
    return planes;
}

size_t psi_len(const cem_sim *s, int is_e, int comp, int w) {
    const int a = (comp + w + 1) % 3;
    return s->has_pml ? pml_planes(s, a, is_e) * pml_per(s, a) : 0;
}

double lumped_source_value(const cem_sim *s, double t) {
    if (s->src_port < 0) return 0.0;
    const double x = (t - s->src_t0) / s->src_tau;
    return s->src_amp * std::exp(-x * x);
}

}  // namespace cb2

using namespace cb2;

extern "C" {

const char *cem_last_error(void) { return g_error; }

const char *cem_version(void) {
#ifdef CEM_VERSION
    return CEM_VERSION;
#else
    return "dev";
#endif
}

size_t cem_index(const cem_sim *s, int i, int j, int k) { return idx3(s, i, j, k); }

void cem_dims(const cem_sim *s, int *nx, int *ny, int *nz) {
    *nx = s->n[0];
    *ny = s->n[1];
    *nz = s->n[2];
}

double cem_dt(const cem_sim *s) { return s->dt; }
long cem_step_count(const cem_sim *s) { return s->step; }
int cem_nfreq(const cem_sim *s) { return s->nf; }

cem_sim *cem_create(int nx, int ny, int nz, const double *x, const double *y, const double *z) {
    if (nx < 2 || ny < 2 || nz < 2) {
        set_error("grid needs at least 2 cells per axis");
        return nullptr;
    }
    cem_sim *s = nullptr;
    try {
        s = new cem_sim;
        s->n[0] = nx; s->n[1] = ny; s->n[2] = nz;
        const double *src[3] = {x, y, z};
        for (int a = 0; a < 3; a++) {
            const int n = s->n[a];
            s->node[a].assign(src[a], src[a] + n + 1);
            s->d[a].assign(n, 0.0);
            s->dd[a].assign(n + 1, 0.0);
            for (int i = 0; i < n; i++) {
                s->d[a][i] = src[a][i + 1] - src[a][i];
                if (!(s->d[a][i] > 0)) {
                    set_error("node coordinates must be strictly increasing");
                    delete s;
                    return nullptr;
                }
            }
            // dual spacing at nodes (reference sim.c:56-59)
            for (int i = 0; i <= n; i++) {
                const double lo = i > 0 ? s->d[a][i - 1] : 0.0, hi = i < n ? s->d[a][i] : 0.0;
                s->dd[a][i] = 0.5 * (lo + hi);
            }
        }
        s->sj = (size_t)nz + 1;
        s->si = s->sj * ((size_t)ny + 1);
        s->N = s->si * ((size_t)nx + 1);
        big_assign(s->eps_r, s->N, 1.0);
        big_assign(s->sigma, s->N, 0.0);
        big_assign(s->cell_pec, s->N, (uint8_t)0);
        for (int c = 0; c < 3; c++) big_assign(s->edge_pec[c], s->N, (uint8_t)0);
    } catch (const std::bad_alloc &) {
        delete s;
        set_error("out of memory");
        return nullptr;
    }
    return s;
}

void cem_destroy(cem_sim *s) {
    if (!s) return;
    modeports_release(s);
    delete s;
}

int cem_set_boundary(cem_sim *s, int face, int type, int ncells) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (face < 0 || face > 5) { set_error("bad face"); return -1; }
    const int a = face / 2;
    if (type == CEM_BC_CPML && (ncells < 1 || ncells * 2 >= s->n[a])) { set_error("bad CPML thickness"); return -1; }
    s->bc[face] = type;
    s->npml[face] = type == CEM_BC_CPML ? ncells : 0;
    return 0;
}

}  // extern "C"

namespace {

// Node nearest to pos along axis a (first one on ties). (reference sim.c:121-129)
int nearest_node(const cem_sim *s, int a, double pos) {
    int best = 0;
    double bd = std::fabs(s->node[a][0] - pos);
    for (int i = 1; i <= s->n[a]; i++) {
        const double dist = std::fabs(s->node[a][i] - pos);
        if (dist < bd) { bd = dist; best = i; }
    }
    return best;
}

// Cells whose centre lies in [lo, hi] along axis a. (reference sim.c:131-142)
bool cell_range(const cem_sim *s, int a, double lo, double hi, int *i0, int *i1) {
    *i0 = s->n[a];
    *i1 = -1;
    for (int i = 0; i < s->n[a]; i++) {
        const double c = 0.5 * (s->node[a][i] + s->node[a][i + 1]);
        if (c >= lo && c <= hi) {
            *i0 = std::min(*i0, i);
            *i1 = std::max(*i1, i);
        }
    }
    return *i1 >= *i0;
}

bool box_cells(const cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1, int r[3][2]) {
    const double lo[3] = {x0, y0, z0}, hi[3] = {x1, y1, z1};
    for (int a = 0; a < 3; a++)
        if (!cell_range(s, a, lo[a], hi[a], &r[a][0], &r[a][1])) return false;
    return true;
}

bool edge_column_ok(const cem_sim *s, int axis, int n1, int n2, int m0, int m1) {
    if (axis < 0 || axis > 2) return false;
    const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
    if (n1 < 0 || n1 > s->n[ua] || n2 < 0 || n2 > s->n[va]) return false;
    if (m0 < 0 || m1 > s->n[axis] || m1 <= m0) return false;
    return true;
}

size_t column_index(const cem_sim *s, int axis, int n1, int n2, int m) {
    int ijk[3];
    ijk[axis] = m;
    ijk[(axis + 1) % 3] = n1;
    ijk[(axis + 2) % 3] = n2;
    return idx3(s, ijk[0], ijk[1], ijk[2]);
}

}  // namespace

extern "C" {

int cem_material_box(cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1, double eps_r,
                     double sigma) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    int r[3][2];
    if (!box_cells(s, x0, x1, y0, y1, z0, z1, r)) return 0;
    for (int i = r[0][0]; i <= r[0][1]; i++)
        for (int j = r[1][0]; j <= r[1][1]; j++)
            for (int k = r[2][0]; k <= r[2][1]; k++) {
                const size_t q = idx3(s, i, j, k);
                s->eps_r[q] = eps_r;
                s->sigma[q] = sigma;
            }
    return 0;
}

int cem_pec_box(cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    int r[3][2];
    if (!box_cells(s, x0, x1, y0, y1, z0, z1, r)) return 0;
    for (int i = r[0][0]; i <= r[0][1]; i++)
        for (int j = r[1][0]; j <= r[1][1]; j++)
            for (int k = r[2][0]; k <= r[2][1]; k++) s->cell_pec[idx3(s, i, j, k)] = 1;
    return 0;
}

// Zero-thickness sheet on the node plane nearest pos: every tangential edge
// lying inside the rectangle becomes PEC. (reference sim.c:173-199)
int cem_pec_sheet(cem_sim *s, int axis, double pos, double a0, double a1, double b0, double b1) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (axis < 0 || axis > 2) { set_error("bad axis"); return -1; }
    const int m = nearest_node(s, axis, pos);
    const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
    const std::vector<double> &U = s->node[ua], &V = s->node[va];
    const double tol = 1e-9 * (U[s->n[ua]] - U[0] + V[s->n[va]] - V[0]);
    int ijk[3];
    ijk[axis] = m;
    for (int u = 0; u < s->n[ua]; u++) {
        if (U[u] < a0 - tol || U[u + 1] > a1 + tol) continue;
        for (int v = 0; v <= s->n[va]; v++) {
            if (V[v] < b0 - tol || V[v] > b1 + tol) continue;
            ijk[ua] = u; ijk[va] = v;
            s->edge_pec[ua][idx3(s, ijk[0], ijk[1], ijk[2])] = 1;
        }
    }
    for (int u = 0; u <= s->n[ua]; u++) {
        if (U[u] < a0 - tol || U[u] > a1 + tol) continue;
        for (int v = 0; v < s->n[va]; v++) {
            if (V[v] < b0 - tol || V[v + 1] > b1 + tol) continue;
            ijk[ua] = u; ijk[va] = v;
            s->edge_pec[va][idx3(s, ijk[0], ijk[1], ijk[2])] = 1;
        }
    }
    return 0;
}

int cem_pec_edges_plane(cem_sim *s, int axis, int m, const unsigned char *mask_u, const unsigned char *mask_v) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (axis < 0 || axis > 2 || m < 0 || m > s->n[axis]) { set_error("bad plane"); return -1; }
    const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
    const int nu = s->n[ua], nv = s->n[va];
    int ijk[3];
    ijk[axis] = m;
    if (mask_u)
        for (int u = 0; u < nu; u++)
            for (int v = 0; v <= nv; v++)
                if (mask_u[(size_t)u * (nv + 1) + v]) {
                    ijk[ua] = u; ijk[va] = v;
                    s->edge_pec[ua][idx3(s, ijk[0], ijk[1], ijk[2])] = 1;
                }
    if (mask_v)
        for (int u = 0; u <= nu; u++)
            for (int v = 0; v < nv; v++)
                if (mask_v[(size_t)u * nv + v]) {
                    ijk[ua] = u; ijk[va] = v;
                    s->edge_pec[va][idx3(s, ijk[0], ijk[1], ijk[2])] = 1;
                }
    return 0;
}

int cem_pec_cells(cem_sim *s, int i0, int j0, int k0, int ni, int nj, int nk, const unsigned char *mask) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (i0 < 0 || j0 < 0 || k0 < 0 || i0 + ni > s->n[0] || j0 + nj > s->n[1] || k0 + nk > s->n[2]) {
        set_error("bad cell box");
        return -1;
    }
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int k = 0; k < nk; k++)
                if (mask[((size_t)i * nj + j) * nk + k]) s->cell_pec[idx3(s, i0 + i, j0 + j, k0 + k)] = 1;
    return 0;
}

int cem_set_debye_poles(cem_sim *s, int npole, const double *f_p) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (s->npole) { set_error("Debye poles already set"); return -1; }
    if (npole < 1 || npole > kMaxPoles) { set_error("bad pole count"); return -1; }
    for (int p = 0; p < npole; p++)
        if (!(f_p[p] > 0)) { set_error("pole frequencies must be positive"); return -1; }
    try {
        for (int p = 0; p < npole; p++) {
            s->pole_f[p] = f_p[p];
            big_assign(s->cell_deps[p], s->N, 0.0);
        }
    } catch (const std::bad_alloc &) {
        set_error("out of memory");
        return -1;
    }
    s->npole = npole;
    return 0;
}

int cem_material_box_debye(cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1,
                           double eps_inf, double sigma, const double *deps) {
    if (!s->npole) { set_error("set Debye poles first"); return -1; }
    if (cem_material_box(s, x0, x1, y0, y1, z0, z1, eps_inf, sigma)) return -1;
    int r[3][2];
    if (!box_cells(s, x0, x1, y0, y1, z0, z1, r)) return 0;
    for (int i = r[0][0]; i <= r[0][1]; i++)
        for (int j = r[1][0]; j <= r[1][1]; j++)
            for (int k = r[2][0]; k <= r[2][1]; k++) {
                const size_t q = idx3(s, i, j, k);
                for (int p = 0; p < s->npole; p++) s->cell_deps[p][q] = deps[p];
            }
    return 0;
}

int cem_add_lumped_port(cem_sim *s, int axis, int n1, int n2, int m0, int m1, int dir, double R) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if ((int)s->port.size() >= kMaxPorts) { set_error("too many ports"); return -1; }
    if (!edge_column_ok(s, axis, n1, n2, m0, m1) || !(R > 0) || (dir != 1 && dir != -1)) {
        set_error("bad port definition");
        return -1;
    }
    LumpedPort p;
    p.axis = axis; p.dir = dir; p.R = R;
    for (int m = m0; m < m1; m++) {
        p.edge.push_back(column_index(s, axis, n1, n2, m));
        p.dl.push_back(s->d[axis][m]);
    }
    p.cs.assign(p.edge.size(), 0.0);
    s->port.push_back(std::move(p));
    return (int)s->port.size() - 1;
}

int cem_set_gaussian(cem_sim *s, int port, double amp, double t0, double tau) {
    if (port < 0 || port >= (int)s->port.size()) { set_error("bad port"); return -1; }
    s->src_port = port; s->src_amp = amp; s->src_t0 = t0; s->src_tau = tau;
    return 0;
}

int cem_set_frequencies(cem_sim *s, int nf, const double *f) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (nf < 1) { set_error("need at least one frequency"); return -1; }
    s->nf = nf;
    s->freq.assign(f, f + nf);
    return 0;
}

int cem_add_vprobe(cem_sim *s, int axis, int n1, int n2, int m0, int m1, int dir) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if ((int)s->vp.size() >= kMaxProbes) { set_error("too many probes"); return -1; }
    if (!edge_column_ok(s, axis, n1, n2, m0, m1)) { set_error("bad probe"); return -1; }
    VoltageProbe p;
    p.axis = axis; p.dir = dir;
    for (int m = m0; m < m1; m++) {
        p.edge.push_back(column_index(s, axis, n1, n2, m));
        p.dl.push_back(s->d[axis][m] * dir);
    }
    s->vp.push_back(std::move(p));
    return (int)s->vp.size() - 1;
}

// Circulation of H around a dual rectangle, current in +axis: bottom and top
// runs along ua, then right and left runs along va, with dual-length weights.
// (reference sim.c:309-340)
int cem_add_iprobe(cem_sim *s, int axis, int m, int u0, int u1, int v0, int v1) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if ((int)s->ip.size() >= kMaxProbes) { set_error("too many probes"); return -1; }
    if (axis < 0 || axis > 2) { set_error("bad current probe"); return -1; }
    const int ua = (axis + 1) % 3, va = (axis + 2) % 3;
    if (m < 0 || m >= s->n[axis] || u0 < 0 || u1 >= s->n[ua] || u1 <= u0 || v0 < 0 || v1 >= s->n[va] || v1 <= v0) {
        set_error("bad current probe");
        return -1;
    }
    CurrentProbe p;
    int ijk[3];
    ijk[axis] = m;
    auto add = [&](int comp, double w) {
        p.comp.push_back(comp);
        p.idx.push_back(idx3(s, ijk[0], ijk[1], ijk[2]));
        p.w.push_back(w);
    };
    for (int u = u0 + 1; u <= u1; u++) {
        ijk[ua] = u; ijk[va] = v0;
        add(3 + ua, s->dd[ua][u]);
        ijk[va] = v1;
        add(3 + ua, -s->dd[ua][u]);
    }
    for (int v = v0 + 1; v <= v1; v++) {
        ijk[va] = v; ijk[ua] = u1;
        add(3 + va, s->dd[va][v]);
        ijk[ua] = u0;
        add(3 + va, -s->dd[va][v]);
    }
    s->ip.push_back(std::move(p));
    return (int)s->ip.size() - 1;
}

}  // extern "C"

namespace {

// CPML grading on one axis: polynomial (m = 3) sigma and kappa, linear alpha,
// recursive-convolution b/c at nodes (E) and cells (H), and the kappa-scaled
// inverse spacings used by the bulk update. (reference sim.c:369-425)
// host threads for the whole-grid loops of finalize
int plane_threads() {
    const unsigned h = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(h ? h : 1u, 32u));
}

// f(t) for t in [0, n) on up to plane_threads() threads
template <class F>
void parallel_tasks(int n, F f) {
    const int nt = std::min(n, plane_threads());
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int w = 0; w < nt; w++)
        th.emplace_back([&] {
            for (int t = next++; t < n; t = next++) f(t);
        });
    for (auto &x : th) x.join();
}

// f(i0, i1) over slabs of the node planes [0, n)
template <class F>
void parallel_planes(int n, F f) {
    const int ns = std::max(1, std::min(n, 4 * plane_threads()));
    parallel_tasks(ns, [&](int sl) {
        f((int)((long long)n * sl / ns), (int)((long long)n * (sl + 1) / ns));
    });
}

void setup_pml_axis(cem_sim *s, int a) {
    const int n = s->n[a];
    s->ide[a].assign(n + 1, 0.0);
    s->idh[a].assign(n, 0.0);
    s->be[a].assign(n + 1, 0.0);
    s->ce[a].assign(n + 1, 0.0);
    s->bh[a].assign(n, 0.0);
    s->ch[a].assign(n, 0.0);
    s->pml_sn[a].assign(n + 1, 0.0);
    s->pml_an[a].assign(n + 1, 0.0);
    s->pml_kn[a].assign(n + 1, 1.0);
    s->pml_sc[a].assign(n, 0.0);
    s->pml_ac[a].assign(n, 0.0);
    s->pml_kc[a].assign(n, 1.0);
    for (int i = 0; i <= n; i++) s->ide[a][i] = s->dd[a][i] > 0 ? 1.0 / s->dd[a][i] : 0.0;
    for (int i = 0; i < n; i++) s->idh[a][i] = 1.0 / s->d[a][i];

    const double m = 3.0, kmax = 5.0, amax = 0.05;
    const std::vector<double> &x = s->node[a];
    for (int side = 0; side < 2; side++) {
        const int np = s->npml[2 * a + side];
        if (!np) continue;
        const double xi = side == 0 ? x[np] : x[n - np];
        const double L = side == 0 ? x[np] - x[0] : x[n] - x[n - np];
        const double dmean = L / np;
        const double smax = 0.8 * (m + 1) / (376.730313668 * dmean);
        auto profile = [&](double pos, double *sg, double *kp, double *al) {
            double depth = side == 0 ? (xi - pos) / L : (pos - xi) / L;
            if (depth <= 0) return false;
            if (depth > 1) depth = 1;
            *sg = smax * std::pow(depth, m);
            *kp = 1 + (kmax - 1) * std::pow(depth, m);
            *al = amax * (1 - depth);
            return true;
        };
        double sg, kp, al;
        for (int i = 0; i <= n; i++) {
            if (!profile(x[i], &sg, &kp, &al)) continue;
            const double b = std::exp(-(sg / kp + al) * s->dt / CEM_EPS0);
            s->be[a][i] = b;
            s->ce[a][i] = sg > 0 ? sg / (sg * kp + kp * kp * al) * (b - 1) : 0;
            s->ide[a][i] = 1.0 / (kp * s->dd[a][i]);
            s->pml_sn[a][i] = sg; s->pml_kn[a][i] = kp; s->pml_an[a][i] = al;
        }
        for (int i = 0; i < n; i++) {
            if (!profile(0.5 * (x[i] + x[i + 1]), &sg, &kp, &al)) continue;
            const double b = std::exp(-(sg / kp + al) * s->dt / CEM_EPS0);
            s->bh[a][i] = b;
            s->ch[a][i] = sg > 0 ? sg / (sg * kp + kp * kp * al) * (b - 1) : 0;
            s->idh[a][i] = 1.0 / (kp * s->d[a][i]);
            s->pml_sc[a][i] = sg; s->pml_kc[a][i] = kp; s->pml_ac[a][i] = al;
        }
    }
}

}  // namespace

extern "C" {

int cem_finalize(cem_sim *s, double cfl) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    // CEM_B200_TRACE=1: seconds per set-up stage on stderr
    static const bool trace = [] { const char *e = std::getenv("CEM_B200_TRACE"); return e && e[0] == '1'; }();
    auto t_last = std::chrono::steady_clock::now();
    auto tick = [&](const char *what) {
        if (!trace) return;
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "courant-b200: finalize %s %.3f s\n", what, std::chrono::duration<double>(now - t_last).count());
        t_last = now;
    };
    try {
        if (!s->nf) {
            const double f = 1e9;
            cem_set_frequencies(s, 1, &f);
        }
        // CFL time step from the smallest cell on each axis (reference sim.c:430-436)
        double dmin[3];
        for (int a = 0; a < 3; a++) dmin[a] = *std::min_element(s->d[a].begin(), s->d[a].end());
        if (!(cfl > 0 && cfl <= 1)) cfl = 0.99;
        s->dt = cfl / (CEM_C0 * std::sqrt(1 / (dmin[0] * dmin[0]) + 1 / (dmin[1] * dmin[1]) + 1 / (dmin[2] * dmin[2])));

        for (int a = 0; a < 3; a++) setup_pml_axis(s, a);
        s->has_pml = 0;
        for (int f = 0; f < 6; f++)
            if (s->npml[f]) s->has_pml = 1;
        tick("cpml profiles");

        const int nx = s->n[0], ny = s->n[1], nz = s->n[2];
        // per-edge coefficients, lossy dielectric by the semi-implicit average
        // (reference sim.c:450-465); every edge on its own, node planes in parallel
        for (int c = 0; c < 3; c++) {
            big_assign(s->ca[c], s->N, 0.0);
            big_assign(s->cb[c], s->N, 0.0);
        }
        parallel_planes(nx + 1, [&](int i0, int i1) {
            for (int c = 0; c < 3; c++)
                for (int i = i0; i < i1; i++)
                    for (int j = 0; j <= ny; j++)
                        for (int k = 0; k <= nz; k++) {
                            const int ijk[3] = {i, j, k};
                            if (ijk[c] >= s->n[c]) continue;
                            const size_t q = idx3(s, i, j, k);
                            double er, sg;
                            int pec;
                            edge_material(s, c, i, j, k, &er, &sg, &pec);
                            if (pec || s->edge_pec[c][q]) continue;   // ca = cb = 0
                            const double eps = er * CEM_EPS0, h = sg * s->dt / (2 * eps);
                            s->ca[c][q] = (1 - h) / (1 + h);
                            s->cb[c][q] = (s->dt / eps) / (1 + h);
                        }
        });

        tick("edge coefficients");
        // lumped ports: resistive voltage source spread over the column's edges
        // (reference sim.c:468-492)
        for (LumpedPort &pt : s->port) {
            double L = 0;
            for (double dl : pt.dl) L += dl;
            const int ua = (pt.axis + 1) % 3, va = (pt.axis + 2) % 3;
            for (size_t e = 0; e < pt.edge.size(); e++) {
                const size_t q = pt.edge[e];
                const int i = (int)(q / s->si), j = (int)((q % s->si) / s->sj), k = (int)(q % s->sj);
                const int ijk[3] = {i, j, k};
                const double A = s->dd[ua][ijk[ua]] * s->dd[va][ijk[va]];
                double er, sg;
                int pec;
                edge_material(s, pt.axis, i, j, k, &er, &sg, &pec);
                if (pec || s->edge_pec[pt.axis][q]) { set_error("port edge is PEC"); return -1; }
                const double eps = er * CEM_EPS0;
                const double Re = pt.R * pt.dl[e] / L;
                const double beta = s->dt * pt.dl[e] / (2 * Re * A * eps) + sg * s->dt / (2 * eps);
                s->ca[pt.axis][q] = (1 - beta) / (1 + beta);
                s->cb[pt.axis][q] = (s->dt / eps) / (1 + beta);
                pt.cs[e] = s->dt / (Re * A * eps * (1 + beta)) * (pt.dl[e] / L) * pt.dir;
            }
            pt.V.assign(2 * s->nf, 0.0);
            pt.I.assign(2 * s->nf, 0.0);
        }

        std::vector<uint8_t> is_port;
        if (!s->port.empty() && (s->npole || s->sibc_on)) {
            big_assign(is_port, s->N * 3, (uint8_t)0);
            for (const LumpedPort &pt : s->port)
                for (size_t q : pt.edge) is_port[pt.axis * s->N + q] = 1;
        }

        // Debye edges: eps -> eps_inf eps0 + sum beta_p / 2 in ca/cb, ADE tables.
        // Lumped-port edges keep their own coefficients. (reference sim.c:501-549)
        if (s->npole) {
            // each (component, slab of node planes) counts its Debye edges, then
            // writes them at its offset in the final lists: the lists join in
            // component, then plane order, the reference's edge order
            const int nslab = std::max(1, std::min(nx + 1, 4 * plane_threads()));
            const int ntask = 3 * nslab;
            auto walk = [&](int t, auto &&edge) {
                const int c = t / nslab, sl = t % nslab;
                const int i0 = (int)((long long)(nx + 1) * sl / nslab), i1 = (int)((long long)(nx + 1) * (sl + 1) / nslab);
                double dep[kMaxPoles];
                for (int i = i0; i < i1; i++)
                    for (int j = 0; j <= ny; j++)
                        for (int k = 0; k <= nz; k++) {
                            const int ijk[3] = {i, j, k};
                            if (ijk[c] >= s->n[c]) continue;
                            const size_t q = idx3(s, i, j, k);
                            if (s->cb[c][q] == 0 || (!is_port.empty() && is_port[c * s->N + q])) continue;
                            if (!edge_debye(s, c, i, j, k, dep)) continue;
                            edge(c, i, j, k, q, dep);
                        }
            };
            std::vector<size_t> first(ntask + 1, 0);
            parallel_tasks(ntask, [&](int t) {
                size_t n = 0;
                walk(t, [&](int, int, int, int, size_t, const double *) { n++; });
                first[t + 1] = n;
            });
            for (int t = 0; t < ntask; t++) first[t + 1] += first[t];
            const size_t total = first[ntask];
            s->ndisp = (int)total;
            big_assign(s->d_comp, total, 0);
            big_assign(s->d_idx, total, (size_t)0);
            big_assign(s->d_cb, total, 0.0);
            big_assign(s->d_beta, (size_t)s->npole * total, 0.0);
            parallel_tasks(ntask, [&](int t) {
                size_t at = first[t];
                walk(t, [&](int c, int i, int j, int k, size_t q, const double *dep) {
                    double er, sg;
                    int pec;
                    edge_material(s, c, i, j, k, &er, &sg, &pec);
                    double einst = er * CEM_EPS0;
                    for (int p = 0; p < s->npole; p++) {
                        const double tau = 1.0 / (2 * M_PI * s->pole_f[p]);
                        const double bt = CEM_EPS0 * dep[p] * s->dt / (tau * (1 + s->dt / (2 * tau)));
                        s->d_beta[(size_t)p * total + at] = bt;
                        einst += 0.5 * bt;
                    }
                    const double h = sg * s->dt / (2 * einst);
                    s->ca[c][q] = (1 - h) / (1 + h);
                    s->cb[c][q] = (s->dt / einst) / (1 + h);
                    s->d_comp[at] = c;
                    s->d_idx[at] = q;
                    s->d_cb[at] = s->cb[c][q];
                    at++;
                });
            });
            for (int p = 0; p < s->npole; p++) {
                const double tau = 1.0 / (2 * M_PI * s->pole_f[p]);
                s->d_k[p] = (1 - s->dt / (2 * tau)) / (1 + s->dt / (2 * tau));
            }
        }
        tick("lumped ports, Debye edges");
        if (sibc_finalize(s, is_port)) return -1;
        tick("surface impedance");

        for (VoltageProbe &p : s->vp) p.acc.assign(2 * s->nf, 0.0);
        for (CurrentProbe &p : s->ip) p.acc.assign(2 * s->nf, 0.0);
        s->src_acc.assign(2 * s->nf, 0.0);
        s->step = 0;
        s->finalized = 1;
        if (modeports_finalize(s)) {
            s->finalized = 0;
            return -1;
        }
        tick("mode ports");
    } catch (const std::bad_alloc &) {
        set_error("out of memory");
        return -1;
    }
    return 0;
}

// ---- results ------------------------------------------------------------

const double *cem_port_v(const cem_sim *s, int p) {
    if (p < 0 || p >= (int)s->port.size() || s->port[p].V.empty()) return nullptr;
    engine_pull(s, kGroupDft);
    engine_expose(s, kGroupDft);
    return s->port[p].V.data();
}

const double *cem_port_i(const cem_sim *s, int p) {
    if (p < 0 || p >= (int)s->port.size() || s->port[p].I.empty()) return nullptr;
    engine_pull(s, kGroupDft);
    engine_expose(s, kGroupDft);
    return s->port[p].I.data();
}

const double *cem_source_spectrum(const cem_sim *s) {
    if (s->src_acc.empty()) return nullptr;
    engine_pull(s, kGroupDft);
    engine_expose(s, kGroupDft);
    return s->src_acc.data();
}

const double *cem_vprobe(const cem_sim *s, int p) {
    if (p < 0 || p >= (int)s->vp.size() || s->vp[p].acc.empty()) return nullptr;
    engine_pull(s, kGroupDft);
    engine_expose(s, kGroupDft);
    return s->vp[p].acc.data();
}

const double *cem_iprobe(const cem_sim *s, int p) {
    if (p < 0 || p >= (int)s->ip.size() || s->ip[p].acc.empty()) return nullptr;
    engine_pull(s, kGroupDft);
    engine_expose(s, kGroupDft);
    return s->ip[p].acc.data();
}

double cem_port_impedance(const cem_sim *s, int p) { return p >= 0 && p < (int)s->port.size() ? s->port[p].R : 0; }
int cem_excited_port(const cem_sim *s) { return s->src_port; }

double *cem_field(cem_sim *s, int comp) {
    if (comp < 0 || comp > 5) return nullptr;
    const unsigned g = 1u << comp;
    host_state_alloc(s, g);
    engine_pull(s, g);
    engine_expose(s, g);
    return comp < 3 ? s->E[comp].data() : s->H[comp - 3].data();
}

}  // extern "C"
