// 2D full-wave eigenmode solver on a Yee cross-section (FP64, host).
//
// The physics is the reference's mode formulation (skyhoffert/CourantEM
// solver/src/mode2d.c:1-20), which the 3D mode ports must reproduce: fields
// ~ exp(-j beta x) along +x on the transverse Yee cell
//   E_u = Ey(j+1/2, k)   E_v = Ez(j, k+1/2)   E_w = Ex(j, k)
//   H_u = Hy(j, k+1/2)   H_v = Hz(j+1/2, k)   H_w = Hx(j+1/2, k+1/2)
// with beta e = P h, beta h = Q e, so beta^2 is an eigenvalue of A = P Q acting
// on the transverse E unknowns. Derivatives carry the stretched-coordinate PML
// factor 1/(s d), s = kappa + sigma/(alpha + j w eps0), and media are complex
// (eps - j sigma/w, Debye poles). The window's outer boundary is PEC.
//
// The solver is this library's own:
//  * A is assembled in closed form. Writing Q and P out, the longitudinal
//    field is E_w = w iw div_t(eps E_t) (the curl terms of H_u, H_v cancel in
//    the divergence), so each row of A is
//        w^2 mu0 eps E  -  curl_t curl_t E  +  grad_t(iw div_t(eps E_t))
//    with at most 15 couplings (E_u: k +- 1, j +- 1 and the four E_v around
//    it), computed directly instead of by applying the operator to probe
//    vectors.
//  * Unknowns on metal (and on the PEC window boundary) are not part of the
//    system at all; the rest are numbered j-major, then k, E_u before E_v, so
//    the band half-width is about 2 nz + 2.
//  * The band is factorised by LU with partial pivoting in row-major storage
//    (each row holds its band plus the pivoting fill), with the complex
//    arithmetic written out so the update loops vectorise.
//  * The eigenpair nearest sigma = (k0 n_guess)^2 comes from shifted inverse
//    iteration: converged when the eigenvalue estimate sigma + 1/<x, y> changes
//    by less than tol relatively and the phase-aligned iterate by less than
//    1e-10, the reference's stopping rule. When that has not happened within
//    maxit iterations (a second mode nearly as close to the shift), the shift
//    moves onto the current estimate and the band is factorised again, up to
//    three times; the reference's solver gives up there.
#include "sim.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

using cb2::cplx;

struct cem_mode2d {
    int ny = 0, nz = 0;
    std::vector<double> y, z;
    std::vector<double> hy, hz;    // cell sizes
    std::vector<double> gy, gz;    // dual sizes at the nodes (half cells at the ends)
    // media at the three E locations (u, v, w): relative permittivity,
    // conductivity, metal flag, Debye pole strengths (npole blocks)
    struct Media {
        std::vector<double> eps, sig, deps;
        std::vector<uint8_t> metal;
    } med[3];
    int npole = 0;
    double pole_f[cb2::kMaxPoles] = {};
    // stretching profiles: [0] y cells, [1] y nodes, [2] z cells, [3] z nodes
    std::vector<double> pml_s[4], pml_k[4], pml_a[4];
    double freq = 0;
    cplx beta = 0;
    std::vector<cplx> eu, ev, hu, hv;   // last mode (API layout: E_u/H_v at j*(nz+1)+k, E_v/H_u at j*nz+k)

    int at_u(int j, int k) const { return j * (nz + 1) + k; }   // E_u, H_v: j < ny, k <= nz
    int at_v(int j, int k) const { return j * nz + k; }         // E_v, H_u: j <= ny, k < nz
    int at_n(int j, int k) const { return j * (nz + 1) + k; }   // nodes
    int count(int which) const { return which == 0 ? ny * (nz + 1) : (which == 1 ? (ny + 1) * nz : (ny + 1) * (nz + 1)); }
};

namespace {

constexpr int U = 0, V = 1, W = 2;

// Coefficients of one angular frequency: 1/(s d) per grid line, absolute
// complex permittivity of E_u and E_v, and 1/eps at the E_w nodes (0 on metal).
struct Coeffs {
    std::vector<cplx> ryc, ryn, rzc, rzn;
    std::vector<cplx> eps_u, eps_v, inv_w;
};

Coeffs coefficients(const cem_mode2d &m, double w) {
    Coeffs c;
    const cplx jwe0(0.0, w * CEM_EPS0);
    auto inv_stretched = [&](int prof, int i, double d) {
        return 1.0 / ((m.pml_k[prof][i] + m.pml_s[prof][i] / (m.pml_a[prof][i] + jwe0)) * d);
    };
    for (int j = 0; j < m.ny; j++) c.ryc.push_back(inv_stretched(0, j, m.hy[j]));
    for (int j = 0; j <= m.ny; j++) c.ryn.push_back(inv_stretched(1, j, m.gy[j]));
    for (int k = 0; k < m.nz; k++) c.rzc.push_back(inv_stretched(2, k, m.hz[k]));
    for (int k = 0; k <= m.nz; k++) c.rzn.push_back(inv_stretched(3, k, m.gz[k]));
    cplx relax[cb2::kMaxPoles];
    for (int p = 0; p < m.npole; p++) relax[p] = 1.0 / cplx(1.0, w / (2 * M_PI * m.pole_f[p]));
    auto permittivity = [&](int which, int q) {
        const cem_mode2d::Media &md = m.med[which];
        cplx e = md.eps[q];
        const int n = m.count(which);
        for (int p = 0; p < m.npole; p++) e += md.deps[(size_t)p * n + q] * relax[p];
        return e * CEM_EPS0 - cplx(0.0, md.sig[q] / w);
    };
    for (int q = 0; q < m.count(U); q++) c.eps_u.push_back(permittivity(U, q));
    for (int q = 0; q < m.count(V); q++) c.eps_v.push_back(permittivity(V, q));
    for (int q = 0; q < m.count(W); q++) c.inv_w.push_back(m.med[W].metal[q] ? cplx(0.0) : 1.0 / permittivity(W, q));
    return c;
}

// Unknown numbering of the field points off metal: j-major, k, E_u before E_v.
struct Numbering {
    std::vector<int> of_u, of_v;    // system index of each E_u / E_v point, -1 on metal
    std::vector<int> where;         // per system index: 2 * point + (0 for E_u, 1 for E_v)
    int n = 0;
};

Numbering number_unknowns(const cem_mode2d &m) {
    Numbering o;
    o.of_u.assign(m.count(U), -1);
    o.of_v.assign(m.count(V), -1);
    for (int j = 0; j <= m.ny; j++)
        for (int k = 0; k <= m.nz; k++) {
            if (j < m.ny && !m.med[U].metal[m.at_u(j, k)]) {
                o.of_u[m.at_u(j, k)] = o.n++;
                o.where.push_back(2 * m.at_u(j, k));
            }
            if (k < m.nz && !m.med[V].metal[m.at_v(j, k)]) {
                o.of_v[m.at_v(j, k)] = o.n++;
                o.where.push_back(2 * m.at_v(j, k) + 1);
            }
        }
    return o;
}

// One assembled row: up to 16 (column, value) couplings.
struct Row {
    int n = 0;
    int col[16];
    cplx val[16];
    void add(int c, cplx v) {
        if (c < 0) return;
        for (int q = 0; q < n; q++)
            if (col[q] == c) { val[q] += v; return; }
        col[n] = c;
        val[n++] = v;
    }
};

// Row of A for E_u(j, k) or E_v(j, k) (which = U or V), every term of
//   w^2 mu0 eps E - curl curl E + grad(iw div(eps E)).
Row assemble_row(const cem_mode2d &m, const Coeffs &c, const Numbering &o, double w, int which, int j, int k) {
    const int ny = m.ny, nz = m.nz;
    const double wwm = w * w * CEM_MU0;
    Row r;
    auto u = [&](int jj, int kk) { return (jj >= 0 && jj < ny && kk >= 0 && kk <= nz) ? o.of_u[m.at_u(jj, kk)] : -1; };
    auto v = [&](int jj, int kk) { return (jj >= 0 && jj <= ny && kk >= 0 && kk < nz) ? o.of_v[m.at_v(jj, kk)] : -1; };
    auto eu = [&](int jj, int kk) { return c.eps_u[m.at_u(jj, kk)]; };
    auto ev = [&](int jj, int kk) { return c.eps_v[m.at_v(jj, kk)]; };
    // h_w(jc, kc) = ryc (E_v(jc+1) - E_v(jc)) - rzc (E_u(kc+1) - E_u(kc)), scaled by s
    auto hw = [&](int jc, int kc, cplx s) {
        const cplx a = s * c.ryc[jc], b = s * c.rzc[kc];
        r.add(v(jc + 1, kc), a);
        r.add(v(jc, kc), -a);
        r.add(u(jc, kc + 1), -b);
        r.add(u(jc, kc), b);
    };
    // iw div(eps E) at node (jn, kn), scaled by s
    auto div = [&](int jn, int kn, cplx s) {
        const cplx t = s * c.inv_w[m.at_n(jn, kn)];
        if (t == 0.0) return;
        const cplx ty = t * c.ryn[jn], tz = t * c.rzn[kn];
        if (jn < ny) r.add(u(jn, kn), ty * eu(jn, kn));
        if (jn > 0) r.add(u(jn - 1, kn), -ty * eu(jn - 1, kn));
        if (kn < nz) r.add(v(jn, kn), tz * ev(jn, kn));
        if (kn > 0) r.add(v(jn, kn - 1), -tz * ev(jn, kn - 1));
    };
    if (which == U) {
        r.add(u(j, k), wwm * eu(j, k));
        // - d/dz of h_w across the node line k (cells k-1, k)
        if (k < nz) hw(j, k, -c.rzn[k]);
        if (k > 0) hw(j, k - 1, c.rzn[k]);
        // d/dy of the divergence between nodes j and j+1
        div(j + 1, k, c.ryc[j]);
        div(j, k, -c.ryc[j]);
    } else {
        r.add(v(j, k), wwm * ev(j, k));
        // + d/dy of h_w across the node line j (cells j-1, j)
        if (j < ny) hw(j, k, c.ryn[j]);
        if (j > 0) hw(j - 1, k, -c.ryn[j]);
        div(j, k + 1, c.rzc[k]);
        div(j, k, -c.rzc[k]);
    }
    return r;
}

// Complex band matrix in row-major storage: row r keeps columns
// [r - kl, r + kl + ku] (the upper kl diagonals receive the pivoting fill),
// real and imaginary parts in two arrays of the same layout, so that the row
// updates run as plain vector loops.
struct Band {
    int n = 0, kl = 0, ku = 0, width = 0;
    std::vector<double> re, im;
    std::vector<double> lc;   // the multipliers again, column by column (kl complex per column), for the solves
    std::vector<int> piv;
    size_t at(int r, int c) const { return (size_t)r * width + (size_t)(c - r + kl); }
};

// dst -= l * src over len complex entries (split parts); the loop of the
// elimination and of nothing else, cloned for AVX2 machines (no contraction:
// every clone gives the same bits)
__attribute__((target_clones("arch=x86-64-v3", "default")))
void row_update(double *__restrict__ dr, double *__restrict__ di, const double *__restrict__ sr,
                const double *__restrict__ si, double lr, double li, int len) {
    for (int q = 0; q < len; q++) {
        dr[q] -= lr * sr[q] - li * si[q];
        di[q] -= lr * si[q] + li * sr[q];
    }
}

// LU with partial pivoting, column by column; multipliers stay in the rows
// they were computed for (interchanges apply from their step on).
bool band_factor(Band &B) {
    const int n = B.n, kl = B.kl, reach = B.kl + B.ku;
    double *re = B.re.data(), *im = B.im.data();
    B.piv.assign(n, 0);
    B.lc.assign((size_t)n * kl * 2, 0.0);
    for (int j = 0; j < n; j++) {
        const int last = std::min(n - 1, j + kl), cmax = std::min(n - 1, j + reach);
        int p = j;
        double best = -1;
        for (int i = j; i <= last; i++) {
            const size_t x = B.at(i, j);
            const double mag = std::hypot(re[x], im[x]);
            if (mag > best) { best = mag; p = i; }
        }
        B.piv[j] = p;
        if (!(best > 0)) return false;
        if (p != j) {
            const size_t rj = B.at(j, j), rp = B.at(p, j);
            for (int q = 0; q <= cmax - j; q++) {
                std::swap(re[rj + q], re[rp + q]);
                std::swap(im[rj + q], im[rp + q]);
            }
        }
        const size_t pr = B.at(j, j);
        const double den = re[pr] * re[pr] + im[pr] * im[pr];
        const double ir = re[pr] / den, ii = -im[pr] / den;   // 1 / pivot
        const int len = cmax - j;
        for (int i = j + 1; i <= last; i++) {
            const size_t ri = B.at(i, j);
            const double lr = re[ri] * ir - im[ri] * ii, li = re[ri] * ii + im[ri] * ir;
            re[ri] = lr;
            im[ri] = li;
            B.lc[((size_t)j * kl + (i - j - 1)) * 2] = lr;
            B.lc[((size_t)j * kl + (i - j - 1)) * 2 + 1] = li;
            if (lr == 0 && li == 0) continue;
            row_update(re + ri + 1, im + ri + 1, re + pr + 1, im + pr + 1, lr, li, len);
        }
    }
    return true;
}

// x <- (L U)^-1 P x (complex products written out: (a + ib)(c + id) =
// (ac - bd) + i(ad + bc), as std::complex forms them, without its NaN checks)
void band_solve(const Band &B, std::vector<cplx> &xv) {
    const int n = B.n, kl = B.kl, reach = B.kl + B.ku;
    const double *re = B.re.data(), *im = B.im.data();
    double *x = reinterpret_cast<double *>(xv.data());
    for (int j = 0; j < n; j++) {
        const int p = B.piv[j];
        if (p != j) {
            std::swap(x[2 * j], x[2 * p]);
            std::swap(x[2 * j + 1], x[2 * p + 1]);
        }
        const double xr = x[2 * j], xi = x[2 * j + 1];
        if (xr == 0 && xi == 0) continue;
        const double *l = B.lc.data() + (size_t)j * kl * 2;
        const int m = std::min(n - 1, j + kl) - j;
        double *y = x + 2 * (j + 1);
        for (int q = 0; q < m; q++) {
            y[2 * q] -= l[2 * q] * xr - l[2 * q + 1] * xi;
            y[2 * q + 1] -= l[2 * q] * xi + l[2 * q + 1] * xr;
        }
    }
    for (int j = n - 1; j >= 0; j--) {
        const int cmax = std::min(n - 1, j + reach);
        const size_t row = B.at(j, j);
        double sr = x[2 * j], si = x[2 * j + 1];
        for (int q = 1; q <= cmax - j; q++) {
            const double ar = re[row + q], ai = im[row + q];
            const double xr = x[2 * (j + q)], xi = x[2 * (j + q) + 1];
            sr -= ar * xr - ai * xi;
            si -= ar * xi + ai * xr;
        }
        const double dr = re[row], di = im[row];
        const double den = dr * dr + di * di;
        x[2 * j] = (sr * dr + si * di) / den;
        x[2 * j + 1] = (si * dr - sr * di) / den;
    }
}

double norm2(const std::vector<cplx> &x) {
    double s = 0;
    for (const cplx &v : x) s += std::norm(v);
    return std::sqrt(s);
}

cplx inner(const std::vector<cplx> &a, const std::vector<cplx> &b) {   // sum conj(a) b, written out
    double sr = 0, si = 0;
    for (size_t q = 0; q < a.size(); q++) {
        const double ar = a[q].real(), ai = a[q].imag(), br = b[q].real(), bi = b[q].imag();
        sr += ar * br - -ai * bi;
        si += ar * bi + -ai * br;
    }
    return cplx(sr, si);
}

// h = Q e / beta for the API's H_u, H_v arrays
void magnetic_field(cem_mode2d &m, const Coeffs &c, double w) {
    const int ny = m.ny, nz = m.nz;
    std::vector<cplx> hw((size_t)ny * nz);
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++)
            hw[(size_t)j * nz + k] = (m.ev[m.at_v(j + 1, k)] - m.ev[m.at_v(j, k)]) * c.ryc[j] -
                                     (m.eu[m.at_u(j, k + 1)] - m.eu[m.at_u(j, k)]) * c.rzc[k];
    const double g = 1.0 / (w * CEM_MU0);
    for (int j = 0; j <= ny; j++)
        for (int k = 0; k < nz; k++) {
            const cplx d = (j < ny ? hw[(size_t)j * nz + k] : 0.0) - (j > 0 ? hw[(size_t)(j - 1) * nz + k] : 0.0);
            m.hu[m.at_v(j, k)] = (-w * c.eps_v[m.at_v(j, k)] * m.ev[m.at_v(j, k)] - g * d * c.ryn[j]) / m.beta;
        }
    for (int j = 0; j < ny; j++)
        for (int k = 0; k <= nz; k++) {
            const cplx d = (k < nz ? hw[(size_t)j * nz + k] : 0.0) - (k > 0 ? hw[(size_t)j * nz + k - 1] : 0.0);
            m.hv[m.at_u(j, k)] = (w * c.eps_u[m.at_u(j, k)] * m.eu[m.at_u(j, k)] - g * d * c.rzn[k]) / m.beta;
        }
}

}  // namespace

namespace cb2 {
double mode_freq_hint(const cem_mode2d *m) { return m->freq; }

void mode2d_copy_mode(cem_mode2d *dst, const cem_mode2d *src) {
    dst->freq = src->freq;
    dst->beta = src->beta;
    dst->eu = src->eu;
    dst->ev = src->ev;
    dst->hu = src->hu;
    dst->hv = src->hv;
}
}

extern "C" {

cem_mode2d *cem_mode2d_create(int ny, int nz, const double *y, const double *z) {
    cem_mode2d *m = new cem_mode2d;
    m->ny = ny;
    m->nz = nz;
    m->y.assign(y, y + ny + 1);
    m->z.assign(z, z + nz + 1);
    // dual sizes: half of each neighbouring cell
    m->gy.assign(ny + 1, 0.0);
    m->gz.assign(nz + 1, 0.0);
    for (int j = 0; j < ny; j++) {
        m->hy.push_back(y[j + 1] - y[j]);
        m->gy[j] += m->hy[j] / 2;
        m->gy[j + 1] += m->hy[j] / 2;
    }
    for (int k = 0; k < nz; k++) {
        m->hz.push_back(z[k + 1] - z[k]);
        m->gz[k] += m->hz[k] / 2;
        m->gz[k + 1] += m->hz[k] / 2;
    }
    for (int which = 0; which < 3; which++) {
        cem_mode2d::Media &md = m->med[which];
        md.eps.assign(m->count(which), 1.0);
        md.sig.assign(m->count(which), 0.0);
        md.metal.assign(m->count(which), 0);
    }
    const int len[4] = {ny, ny + 1, nz, nz + 1};
    for (int a = 0; a < 4; a++) {
        m->pml_s[a].assign(len[a], 0.0);
        m->pml_k[a].assign(len[a], 1.0);
        m->pml_a[a].assign(len[a], 0.0);
    }
    // the window's outer boundary is a perfect conductor
    for (int j = 0; j < ny; j++) m->med[U].metal[m->at_u(j, 0)] = m->med[U].metal[m->at_u(j, nz)] = 1;
    for (int k = 0; k < nz; k++) m->med[V].metal[m->at_v(0, k)] = m->med[V].metal[m->at_v(ny, k)] = 1;
    for (int j = 0; j <= ny; j++) m->med[W].metal[m->at_n(j, 0)] = m->med[W].metal[m->at_n(j, nz)] = 1;
    for (int k = 0; k <= nz; k++) m->med[W].metal[m->at_n(0, k)] = m->med[W].metal[m->at_n(ny, k)] = 1;
    m->eu.assign(m->count(U), cplx(0));
    m->ev.assign(m->count(V), cplx(0));
    m->hu.assign(m->count(V), cplx(0));
    m->hv.assign(m->count(U), cplx(0));
    return m;
}

void cem_mode2d_destroy(cem_mode2d *m) { delete m; }

void cem_mode2d_set_debye(cem_mode2d *m, int npole, const double *f_p, const double *deps_u, const double *deps_v,
                          const double *deps_w) {
    npole = std::min(npole, cb2::kMaxPoles);
    m->npole = npole;
    std::copy(f_p, f_p + npole, m->pole_f);
    const double *src[3] = {deps_u, deps_v, deps_w};
    for (int which = 0; which < 3; which++)
        m->med[which].deps.assign(src[which], src[which] + (size_t)npole * m->count(which));
}

void cem_mode2d_set_media(cem_mode2d *m, const double *epsr_u, const double *epsr_v, const double *epsr_w,
                          const unsigned char *pec_u, const unsigned char *pec_v, const unsigned char *pec_w) {
    const double *eps[3] = {epsr_u, epsr_v, epsr_w};
    const unsigned char *pec[3] = {pec_u, pec_v, pec_w};
    for (int which = 0; which < 3; which++) {
        cem_mode2d::Media &md = m->med[which];
        for (int q = 0; q < m->count(which); q++) {
            md.eps[q] = eps[which][q];
            md.metal[q] |= pec[which][q];   // the boundary stays metal
        }
    }
}

void cem_mode2d_set_loss(cem_mode2d *m, const double *sig_u, const double *sig_v, const double *sig_w) {
    const double *sig[3] = {sig_u, sig_v, sig_w};
    for (int which = 0; which < 3; which++) m->med[which].sig.assign(sig[which], sig[which] + m->count(which));
}

void cem_mode2d_set_pml(cem_mode2d *m, int which, const double *sigma, const double *kappa, const double *alpha) {
    if (which < 0 || which > 3) return;
    const int len = (which < 2 ? m->ny : m->nz) + (which & 1);
    m->pml_s[which].assign(sigma, sigma + len);
    m->pml_k[which].assign(kappa, kappa + len);
    m->pml_a[which].assign(alpha, alpha + len);
}

// 0: converged; 1: not within maxit iterations and three refined shifts (the last iterate is kept); -1: singular
int cem_mode2d_solve(cem_mode2d *m, double f, double neff_guess, const double *start, int maxit, double tol) {
    const int ny = m->ny, nz = m->nz;
    const double w = 2 * M_PI * f, k0 = w / CEM_C0;
    const cplx sigma = k0 * k0 * neff_guess * neff_guess;
    const Coeffs c = coefficients(*m, w);
    const Numbering o = number_unknowns(*m);
    const int n = o.n;
    if (n == 0) return -1;
    // rows of A and the band they need
    std::vector<Row> rows(n);
    int half = 0;
    for (int g = 0; g < n; g++) {
        const int pt = o.where[g] >> 1, which = o.where[g] & 1;
        const int j = which == U ? pt / (nz + 1) : pt / nz, k = which == U ? pt % (nz + 1) : pt % nz;
        rows[g] = assemble_row(*m, c, o, w, which, j, k);
        rows[g].add(g, 0.0);   // the diagonal always has an entry for the shift
        for (int q = 0; q < rows[g].n; q++) half = std::max(half, std::abs(rows[g].col[q] - g));
    }
    Band B;
    B.n = n;
    B.kl = B.ku = half;
    B.width = 2 * half + half + 1;
    // LU of A - shift I
    auto factor = [&](cplx shift) {
        B.re.assign((size_t)n * B.width, 0.0);
        B.im.assign((size_t)n * B.width, 0.0);
        for (int g = 0; g < n; g++)
            for (int q = 0; q < rows[g].n; q++) {
                const cplx v = rows[g].val[q] - (rows[g].col[q] == g ? shift : cplx(0.0));
                const size_t e = B.at(g, rows[g].col[q]);
                B.re[e] += v.real();
                B.im[e] += v.imag();
            }
        return band_factor(B);
    };
    static const bool trace = [] { const char *e = std::getenv("CEM_B200_TRACE"); return e && e[0] == '1'; }();
    const auto t0 = std::chrono::steady_clock::now();
    int iters = 0, factors = 1;
    if (!factor(sigma)) return -1;
    const double t_factor = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    // start vector: the given field (API layout: E_u then E_v, complex) or a fixed pseudo-random one
    std::vector<cplx> x(n), y(n);
    if (start) {
        const cplx *st = reinterpret_cast<const cplx *>(start);
        for (int g = 0; g < n; g++) {
            const int pt = o.where[g] >> 1;
            x[g] = (o.where[g] & 1) ? st[m->count(U) + pt] : st[pt];
        }
    } else {
        uint64_t s = 0x9e3779b97f4a7c15ull;
        for (int g = 0; g < n; g++) {
            s ^= s << 13; s ^= s >> 7; s ^= s << 17;   // xorshift64
            x[g] = (double)(s >> 11) * 0x1.0p-53 - 0.5;
        }
    }
    double nx = norm2(x);
    if (!(nx > 0)) return -1;
    for (cplx &v : x) v /= nx;
    cplx lam = sigma;
    // inverse iteration with shift `shift`, from x; true when converged
    auto iterate = [&](cplx shift, int its) {
        cplx lam_prev = 0;
        for (int it = 0; it < its; it++) {
            iters++;
            y = x;
            band_solve(B, y);
            const cplx mu = inner(x, y);
            lam = shift + 1.0 / mu;
            const double ny2 = norm2(y);
            for (cplx &v : y) v /= ny2;
            // change of the iterate with its global phase aligned to the previous one
            const cplx ph = inner(y, x);
            const cplx rot = std::abs(ph) > 0 ? ph / std::abs(ph) : cplx(1.0);
            double d = 0;
            for (int g = 0; g < n; g++) {
                const double yr = y[g].real(), yi = y[g].imag();
                const double dr = (yr * rot.real() - yi * rot.imag()) - x[g].real();
                const double di = (yr * rot.imag() + yi * rot.real()) - x[g].imag();
                d += dr * dr + di * di;
            }
            x.swap(y);
            if (it >= 2 && std::abs(lam - lam_prev) < tol * std::abs(lam) && std::sqrt(d) < 1e-10) return true;
            lam_prev = lam;
        }
        return false;
    };
    int rc = iterate(sigma, maxit) ? 0 : 1;
    // Where a second mode lies nearly as close to the shift, inverse iteration
    // crawls and stops at maxit (the reference's solver returns there). This
    // solver then moves the shift onto the estimate of the mode it has been
    // converging to and iterates again (up to three times): with the shift at
    // the eigenvalue the other modes fall away at once.
    for (int refine = 0; rc == 1 && refine < 3; refine++) {
        const cplx shift = lam;
        factors++;
        if (!factor(shift)) break;
        if (iterate(shift, 60)) rc = 0;
    }
    // largest component real and positive; scatter into the API arrays
    int imax = 0;
    for (int g = 1; g < n; g++)
        if (std::abs(x[g]) > std::abs(x[imax])) imax = g;
    const cplx fix = std::conj(x[imax]) / std::abs(x[imax]);
    std::fill(m->eu.begin(), m->eu.end(), cplx(0));
    std::fill(m->ev.begin(), m->ev.end(), cplx(0));
    for (int g = 0; g < n; g++) {
        const int pt = o.where[g] >> 1;
        ((o.where[g] & 1) ? m->ev : m->eu)[pt] = x[g] * fix;
    }
    if (trace)
        std::fprintf(stderr, "courant-b200: mode solve f %.4g GHz n %d half %d: first factor %.3f s, %d factors, "
                     "%d iterations, %.3f s in all, rc %d\n", f * 1e-9, n, half, t_factor, factors, iters,
                     std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(), rc);
    cplx bt = std::sqrt(lam);
    if (bt.real() < 0) bt = -bt;
    m->beta = bt;
    m->freq = f;
    magnetic_field(*m, c, w);
    return rc;
}

double cem_mode2d_beta(const cem_mode2d *m) { return m->beta.real(); }
double cem_mode2d_alpha(const cem_mode2d *m) { return -m->beta.imag(); }
const double *cem_mode2d_eu(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->eu.data()); }
const double *cem_mode2d_ev(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->ev.data()); }
const double *cem_mode2d_hu(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->hu.data()); }
const double *cem_mode2d_hv(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->hv.data()); }

// Real part of the complex power flow 1/2 integral (E_t x H_t*) . x dA.
double cem_mode2d_power(const cem_mode2d *m) {
    double p = 0;
    for (int j = 0; j < m->ny; j++)
        for (int k = 0; k <= m->nz; k++) {
            const int q = m->at_u(j, k);
            p += (m->eu[q] * std::conj(m->hv[q])).real() * m->hy[j] * m->gz[k];
        }
    for (int j = 0; j <= m->ny; j++)
        for (int k = 0; k < m->nz; k++) {
            const int q = m->at_v(j, k);
            p -= (m->ev[q] * std::conj(m->hu[q])).real() * m->gy[j] * m->hz[k];
        }
    return 0.5 * p;
}

// V = -integral of Ez from k0 to k1 on node column j0; I = circulation of H
// (+x current) around the dual rectangle (ja+1/2 .. jb+1/2) x (ka+1/2 .. kb+1/2).
void cem_mode2d_vi(const cem_mode2d *m, int j0, int k0, int k1, int ja, int jb, int ka, int kb, double *V,
                   double *Iout) {
    cplx v = 0, i = 0;
    for (int k = k0; k < k1; k++) v -= m->ev[m->at_v(j0, k)] * m->hz[k];
    for (int j = ja + 1; j <= jb; j++) i += (m->hu[m->at_v(j, ka)] - m->hu[m->at_v(j, kb)]) * m->gy[j];
    for (int k = ka + 1; k <= kb; k++) i += (m->hv[m->at_u(jb, k)] - m->hv[m->at_u(ja, k)]) * m->gz[k];
    V[0] = v.real();
    V[1] = v.imag();
    Iout[0] = i.real();
    Iout[1] = i.imag();
}

// Conductor attenuation of the last mode by perturbation (the reference's
// definition, solver/src/mode2d.c:444-498): every metal segment of the
// section that faces a field cell outside the PML loses Rs/2 |J|^2 per unit
// length, with the transverse surface current |H_w| = |curl_w E| / (w mu0) on
// the segment and the longitudinal one from the transverse H at its two end
// points (half a segment each); alpha_c = P_loss / (2 P).
double cem_mode2d_conductor_alpha(const cem_mode2d *m, double Rs) {
    const int ny = m->ny, nz = m->nz;
    const cem_mode2d::Media &mu = m->med[U], &mv = m->med[V];
    auto solid = [&](int j, int k) {   // cell (j, k) enclosed by metal on all four sides
        return j >= 0 && j < ny && k >= 0 && k < nz && mu.metal[m->at_u(j, k)] && mu.metal[m->at_u(j, k + 1)] &&
               mv.metal[m->at_v(j, k)] && mv.metal[m->at_v(j + 1, k)];
    };
    const double wm = 2 * M_PI * m->freq * CEM_MU0;
    auto hw_mag = [&](int j, int k) {
        const cplx cw = (m->ev[m->at_v(j + 1, k)] - m->ev[m->at_v(j, k)]) / m->hy[j] -
                        (m->eu[m->at_u(j, k + 1)] - m->eu[m->at_u(j, k)]) / m->hz[k];
        return std::abs(cw) / wm;
    };
    double loss = 0;
    for (int j = 0; j < ny; j++)   // y-directed segments (E_u points on metal)
        for (int k = 0; k <= nz; k++) {
            if (!mu.metal[m->at_u(j, k)] || m->pml_s[0][j] > 0 || m->pml_s[3][k] > 0) continue;
            for (int kc : {k, k - 1}) {
                if (kc < 0 || kc >= nz || solid(j, kc)) continue;
                const double h = hw_mag(j, kc);
                loss += 0.5 * Rs * h * h * m->hy[j];
                for (int jn : {j, j + 1}) {
                    if (mv.metal[m->at_v(jn, kc)]) continue;
                    const double t = std::abs(m->hu[m->at_v(jn, kc)]);
                    loss += 0.25 * Rs * t * t * m->hy[j];
                }
            }
        }
    for (int j = 0; j <= ny; j++)   // z-directed segments (E_v points on metal)
        for (int k = 0; k < nz; k++) {
            if (!mv.metal[m->at_v(j, k)] || m->pml_s[1][j] > 0 || m->pml_s[2][k] > 0) continue;
            for (int jc : {j, j - 1}) {
                if (jc < 0 || jc >= ny || solid(jc, k)) continue;
                const double h = hw_mag(jc, k);
                loss += 0.5 * Rs * h * h * m->hz[k];
                for (int kn : {k, k + 1}) {
                    if (mu.metal[m->at_u(jc, kn)]) continue;
                    const double t = std::abs(m->hv[m->at_u(jc, kn)]);
                    loss += 0.25 * Rs * t * t * m->hz[k];
                }
            }
        }
    const double P = cem_mode2d_power(m);
    return P > 0 ? loss / (2 * P) : 0;
}

}  // extern "C"
