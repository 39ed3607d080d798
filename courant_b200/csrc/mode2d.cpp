// 2D full-wave eigenmode solver on a Yee cross-section (FP64, host).
//
// Propagation along +x with fields ~ exp(-j beta x); transverse unknowns
//   E_u = Ey(j+1/2,k)  E_v = Ez(j,k+1/2)  E_w = Ex(j,k)
//   H_u = Hy(j,k+1/2)  H_v = Hz(j+1/2,k)  H_w = Hx(j+1/2,k+1/2)
// with beta e = P h, beta h = Q e, i.e. beta^2 e = (P Q) e. Complex arithmetic
// carries the stretched-coordinate PML (s = kappa + sigma/(alpha + j w eps0)),
// conductivity and Debye dispersion. P Q is applied matrix-free, assembled in
// band storage by probing with coloured unit vectors, factorised by a banded
// LU with partial pivoting, and the eigenpair nearest (k0 n_guess)^2 is found
// by shifted inverse iteration.
//
// The formulation, unknown ordering, probing pattern, shift and start vector
// are those of the reference solver (skyhoffert/CourantEM solver/src/mode2d.c),
// because the 3D mode-port results must match the oracle; std::complex<double>
// under GCC performs the same IEEE complex operations as C99 double complex.
#include "sim.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

using cb2::cplx;

struct cem_mode2d {
    int ny = 0, nz = 0;
    std::vector<double> y, z, dy, dz, ddy, ddz;
    std::vector<double> er_u, er_v, er_w, sg_u, sg_v, sg_w;
    std::vector<uint8_t> pec_u, pec_v, pec_w;
    int npole = 0;
    double pole_f[cb2::kMaxPoles] = {};
    std::vector<double> dp_u, dp_v, dp_w;   // npole blocks
    std::vector<double> ps[4], pk[4], pa[4];   // PML sigma/kappa/alpha: y cells, y nodes, z cells, z nodes
    double freq = 0;
    cplx beta = 0;
    std::vector<cplx> eu, ev, hu, hv;

    // flat indices: E_u and H_v (j<ny, k<=nz), E_v and H_u (j<=ny, k<nz), nodes, cells
    int iu(int j, int k) const { return j * (nz + 1) + k; }
    int iv(int j, int k) const { return j * nz + k; }
    int in(int j, int k) const { return j * (nz + 1) + k; }
    int ic(int j, int k) const { return j * nz + k; }
    int nu() const { return ny * (nz + 1); }
    int nv() const { return (ny + 1) * nz; }
    int nn() const { return (ny + 1) * (nz + 1); }
};

namespace {

// Coefficients for one angular frequency.
struct Coef {
    std::vector<cplx> iyc, iyn, izc, izn;   // 1/(s d) at y cells, y nodes, z cells, z nodes
    std::vector<cplx> eu, ev, iw;           // complex permittivity of E_u, E_v; 1/eps at E_w (0 on PEC)
};

Coef make_coef(const cem_mode2d &m, double w) {
    const int ny = m.ny, nz = m.nz;
    Coef c;
    const cplx jw = cplx(0.0, 1.0) * w * CEM_EPS0;
    auto stretch = [&](int a, int i) { return m.pk[a][i] + m.ps[a][i] / (m.pa[a][i] + jw); };
    c.iyc.resize(ny); c.iyn.resize(ny + 1); c.izc.resize(nz); c.izn.resize(nz + 1);
    for (int j = 0; j < ny; j++) c.iyc[j] = 1.0 / (stretch(0, j) * m.dy[j]);
    for (int j = 0; j <= ny; j++) c.iyn[j] = 1.0 / (stretch(1, j) * m.ddy[j]);
    for (int k = 0; k < nz; k++) c.izc[k] = 1.0 / (stretch(2, k) * m.dz[k]);
    for (int k = 0; k <= nz; k++) c.izn[k] = 1.0 / (stretch(3, k) * m.ddz[k]);
    cplx dfac[cb2::kMaxPoles];
    for (int p = 0; p < m.npole; p++) dfac[p] = 1.0 / (1.0 + cplx(0.0, 1.0) * w / (2 * M_PI * m.pole_f[p]));
    const cplx jay(0.0, 1.0);
    auto permittivity = [&](double er, const std::vector<double> &dp, size_t stride, size_t q, double sg) {
        cplx e = er;
        for (int p = 0; p < m.npole; p++) e += dp[(size_t)p * stride + q] * dfac[p];
        return e * CEM_EPS0 - jay * sg / w;
    };
    const int nu = m.nu(), nv = m.nv(), nn = m.nn();
    c.eu.resize(nu); c.ev.resize(nv); c.iw.resize(nn);
    for (int q = 0; q < nu; q++) c.eu[q] = permittivity(m.er_u[q], m.dp_u, nu, q, m.sg_u[q]);
    for (int q = 0; q < nv; q++) c.ev[q] = permittivity(m.er_v[q], m.dp_v, nv, q, m.sg_v[q]);
    for (int q = 0; q < nn; q++)
        c.iw[q] = m.pec_w[q] ? cplx(0) : 1.0 / permittivity(m.er_w[q], m.dp_w, nn, q, m.sg_w[q]);
    return c;
}

// h = Q e (curl of E and Faraday's law); hw: work array over cells
void apply_q(const cem_mode2d &m, const Coef &c, double w, const cplx *eu, const cplx *ev, cplx *hu, cplx *hv,
             cplx *hw) {
    const int ny = m.ny, nz = m.nz;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++)
            hw[m.ic(j, k)] = (ev[m.iv(j + 1, k)] - ev[m.iv(j, k)]) * c.iyc[j] - (eu[m.iu(j, k + 1)] - eu[m.iu(j, k)]) * c.izc[k];
    const double cc = 1.0 / (w * CEM_MU0);
    for (int j = 0; j <= ny; j++)
        for (int k = 0; k < nz; k++) {
            const cplx r = (j < ny ? hw[m.ic(j, k)] : 0.0) - (j > 0 ? hw[m.ic(j - 1, k)] : 0.0);
            hu[m.iv(j, k)] = -w * c.ev[m.iv(j, k)] * ev[m.iv(j, k)] - cc * r * c.iyn[j];
        }
    for (int j = 0; j < ny; j++)
        for (int k = 0; k <= nz; k++) {
            const cplx r = (k < nz ? hw[m.ic(j, k)] : 0.0) - (k > 0 ? hw[m.ic(j, k - 1)] : 0.0);
            hv[m.iu(j, k)] = w * c.eu[m.iu(j, k)] * eu[m.iu(j, k)] - cc * r * c.izn[k];
        }
}

// e = P h (Ampere's law with the longitudinal E eliminated); ew: work array over nodes
void apply_p(const cem_mode2d &m, const Coef &c, double w, const cplx *hu, const cplx *hv, cplx *eu, cplx *ev,
             cplx *ew) {
    const int ny = m.ny, nz = m.nz;
    for (int j = 0; j <= ny; j++)
        for (int k = 0; k <= nz; k++) {
            const cplx du = ((j < ny ? hv[m.iu(j, k)] : 0.0) - (j > 0 ? hv[m.iu(j - 1, k)] : 0.0)) * c.iyn[j];
            const cplx dv = ((k < nz ? hu[m.iv(j, k)] : 0.0) - (k > 0 ? hu[m.iv(j, k - 1)] : 0.0)) * c.izn[k];
            ew[m.in(j, k)] = (du - dv) * c.iw[m.in(j, k)];
        }
    const double cc = 1.0 / w;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k <= nz; k++)
            eu[m.iu(j, k)] = w * CEM_MU0 * hv[m.iu(j, k)] + cc * (ew[m.in(j + 1, k)] - ew[m.in(j, k)]) * c.iyc[j];
    for (int j = 0; j <= ny; j++)
        for (int k = 0; k < nz; k++)
            ev[m.iv(j, k)] = -w * CEM_MU0 * hu[m.iv(j, k)] + cc * (ew[m.in(j, k + 1)] - ew[m.in(j, k)]) * c.izc[k];
}

// Unknown ordering: j outer, k inner, E_u and E_v interleaved, which keeps the
// half-bandwidth near 2 (nz + 2).
struct Unknowns {
    std::vector<int> kind, idx;   // kind 0: E_u, 1: E_v
    int n = 0;
};

Unknowns make_unknowns(const cem_mode2d &m) {
    Unknowns o;
    for (int j = 0; j <= m.ny; j++)
        for (int k = 0; k <= m.nz; k++) {
            if (j < m.ny) { o.kind.push_back(0); o.idx.push_back(m.iu(j, k)); }
            if (k < m.nz) { o.kind.push_back(1); o.idx.push_back(m.iv(j, k)); }
        }
    o.n = (int)o.kind.size();
    return o;
}

bool unknown_is_pec(const cem_mode2d &m, const Unknowns &o, int g) {
    return o.kind[g] == 0 ? m.pec_u[o.idx[g]] != 0 : m.pec_v[o.idx[g]] != 0;
}

// Complex band matrix in LAPACK gbtrf layout: element (i, j) at
// ab[j*ldab + kl + ku + i - j], kl rows of fill kept above the band for pivoting.
struct Band {
    int n, kl, ku, ldab;
    std::vector<cplx> ab;
    std::vector<int> ipiv;
    Band(int n_, int bw) : n(n_), kl(bw), ku(bw), ldab(3 * bw + 1), ab((size_t)(3 * bw + 1) * n_), ipiv(n_) {}
    cplx &at(int i, int j) { return ab[(size_t)j * ldab + (kl + ku + i - j)]; }

    int factor() {
        const int kv = ku + kl;
        for (int j = 0; j < n; j++) {
            const int last = std::min(j + kl, n - 1);
            int p = j;
            double best = std::abs(at(j, j));
            for (int i = j + 1; i <= last; i++) {
                const double v = std::abs(at(i, j));
                if (v > best) { best = v; p = i; }
            }
            ipiv[j] = p;
            if (best == 0) return -1;
            const int jmax = std::min(j + kv, n - 1);
            if (p != j)
                for (int c = j; c <= jmax; c++) std::swap(at(j, c), at(p, c));
            const cplx piv = at(j, j);
            for (int i = j + 1; i <= last; i++) {
                at(i, j) /= piv;
                const cplx l = at(i, j);
                if (l == 0.0) continue;
                for (int c = j + 1; c <= jmax; c++) at(i, c) -= l * at(j, c);
            }
        }
        return 0;
    }

    void solve(cplx *x) {
        const int kv = ku + kl;
        for (int j = 0; j < n; j++) {
            const int p = ipiv[j];
            if (p != j) std::swap(x[j], x[p]);
            const int last = std::min(j + kl, n - 1);
            for (int i = j + 1; i <= last; i++) x[i] -= at(i, j) * x[j];
        }
        for (int j = n - 1; j >= 0; j--) {
            x[j] /= at(j, j);
            const int first = std::max(j - kv, 0);
            for (int i = first; i < j; i++) x[i] -= at(i, j) * x[j];
        }
    }
};

struct Work {
    std::vector<cplx> eu, ev, hu, hv, wk;
    explicit Work(const cem_mode2d &m) : eu(m.nu()), ev(m.nv()), hu(m.nv()), hv(m.nu()), wk(m.nn()) {}
};

void apply_a(const cem_mode2d &m, const Coef &c, const Unknowns &o, double w, const cplx *x, cplx *y, Work &W) {
    std::fill(W.eu.begin(), W.eu.end(), cplx(0));
    std::fill(W.ev.begin(), W.ev.end(), cplx(0));
    for (int g = 0; g < o.n; g++) {
        if (unknown_is_pec(m, o, g)) continue;
        (o.kind[g] == 0 ? W.eu : W.ev)[o.idx[g]] = x[g];
    }
    apply_q(m, c, w, W.eu.data(), W.ev.data(), W.hu.data(), W.hv.data(), W.wk.data());
    apply_p(m, c, w, W.hu.data(), W.hv.data(), W.eu.data(), W.ev.data(), W.wk.data());
    for (int g = 0; g < o.n; g++)
        y[g] = unknown_is_pec(m, o, g) ? cplx(0) : (o.kind[g] == 0 ? W.eu : W.ev)[o.idx[g]];
}

}  // namespace

namespace cb2 {
double mode_freq_hint(const cem_mode2d *m) { return m->freq; }
}

extern "C" {

cem_mode2d *cem_mode2d_create(int ny, int nz, const double *y, const double *z) {
    cem_mode2d *m = new cem_mode2d;
    m->ny = ny; m->nz = nz;
    m->y.assign(y, y + ny + 1);
    m->z.assign(z, z + nz + 1);
    m->dy.resize(ny); m->dz.resize(nz);
    m->ddy.assign(ny + 1, 0.0); m->ddz.assign(nz + 1, 0.0);
    // dual spacings accumulated half-cell by half-cell (reference mode2d.c:64-65)
    for (int j = 0; j < ny; j++) { m->dy[j] = y[j + 1] - y[j]; m->ddy[j] += m->dy[j] / 2; m->ddy[j + 1] += m->dy[j] / 2; }
    for (int k = 0; k < nz; k++) { m->dz[k] = z[k + 1] - z[k]; m->ddz[k] += m->dz[k] / 2; m->ddz[k + 1] += m->dz[k] / 2; }
    const int nu = m->nu(), nv = m->nv(), nn = m->nn();
    m->er_u.assign(nu, 1.0); m->er_v.assign(nv, 1.0); m->er_w.assign(nn, 1.0);
    m->sg_u.assign(nu, 0.0); m->sg_v.assign(nv, 0.0); m->sg_w.assign(nn, 0.0);
    m->pec_u.assign(nu, 0); m->pec_v.assign(nv, 0); m->pec_w.assign(nn, 0);
    const int len[4] = {ny, ny + 1, nz, nz + 1};
    for (int a = 0; a < 4; a++) {
        m->ps[a].assign(len[a], 0.0);
        m->pk[a].assign(len[a], 1.0);
        m->pa[a].assign(len[a], 0.0);
    }
    // the window's outer boundary is PEC
    for (int j = 0; j < ny; j++) m->pec_u[m->iu(j, 0)] = m->pec_u[m->iu(j, nz)] = 1;
    for (int k = 0; k < nz; k++) m->pec_v[m->iv(0, k)] = m->pec_v[m->iv(ny, k)] = 1;
    for (int j = 0; j <= ny; j++) m->pec_w[m->in(j, 0)] = m->pec_w[m->in(j, nz)] = 1;
    for (int k = 0; k <= nz; k++) m->pec_w[m->in(0, k)] = m->pec_w[m->in(ny, k)] = 1;
    m->eu.assign(nu, cplx(0)); m->ev.assign(nv, cplx(0));
    m->hu.assign(nv, cplx(0)); m->hv.assign(nu, cplx(0));
    return m;
}

void cem_mode2d_destroy(cem_mode2d *m) { delete m; }

void cem_mode2d_set_debye(cem_mode2d *m, int npole, const double *f_p, const double *deps_u, const double *deps_v,
                          const double *deps_w) {
    if (npole > cb2::kMaxPoles) npole = cb2::kMaxPoles;
    m->npole = npole;
    std::memcpy(m->pole_f, f_p, npole * sizeof(double));
    m->dp_u.assign(deps_u, deps_u + (size_t)npole * m->nu());
    m->dp_v.assign(deps_v, deps_v + (size_t)npole * m->nv());
    m->dp_w.assign(deps_w, deps_w + (size_t)npole * m->nn());
}

void cem_mode2d_set_media(cem_mode2d *m, const double *epsr_u, const double *epsr_v, const double *epsr_w,
                          const unsigned char *pec_u, const unsigned char *pec_v, const unsigned char *pec_w) {
    for (int q = 0; q < m->nu(); q++) { m->er_u[q] = epsr_u[q]; m->pec_u[q] |= pec_u[q]; }
    for (int q = 0; q < m->nv(); q++) { m->er_v[q] = epsr_v[q]; m->pec_v[q] |= pec_v[q]; }
    for (int q = 0; q < m->nn(); q++) { m->er_w[q] = epsr_w[q]; m->pec_w[q] |= pec_w[q]; }
}

void cem_mode2d_set_loss(cem_mode2d *m, const double *sig_u, const double *sig_v, const double *sig_w) {
    m->sg_u.assign(sig_u, sig_u + m->nu());
    m->sg_v.assign(sig_v, sig_v + m->nv());
    m->sg_w.assign(sig_w, sig_w + m->nn());
}

void cem_mode2d_set_pml(cem_mode2d *m, int which, const double *sigma, const double *kappa, const double *alpha) {
    if (which < 0 || which > 3) return;
    const int len[4] = {m->ny, m->ny + 1, m->nz, m->nz + 1};
    m->ps[which].assign(sigma, sigma + len[which]);
    m->pk[which].assign(kappa, kappa + len[which]);
    m->pa[which].assign(alpha, alpha + len[which]);
}

int cem_mode2d_solve(cem_mode2d *m, double f, double neff_guess, const double *start, int maxit, double tol) {
    const int ny = m->ny, nz = m->nz;
    const double w = 2 * M_PI * f, k0 = w / CEM_C0;
    const cplx shift = k0 * k0 * neff_guess * neff_guess;
    const Coef c = make_coef(*m, w);
    const Unknowns o = make_unknowns(*m);
    const int n = o.n, bw = 2 * (nz + 2) + 2;
    Band B(n, bw);
    std::vector<cplx> x(n), y(n);
    Work W(*m);

    // assemble the band by probing: unknowns Wc apart never share a band column
    const int Wc = 2 * bw + 1;
    for (int col = 0; col < Wc; col++) {
        std::fill(x.begin(), x.end(), cplx(0));
        for (int g = col; g < n; g += Wc) x[g] = 1.0;
        apply_a(*m, c, o, w, x.data(), y.data(), W);
        for (int g = col; g < n; g += Wc) {
            const int lo = std::max(g - bw, 0), hi = std::min(g + bw, n - 1);
            for (int r = lo; r <= hi; r++) B.at(r, g) = y[r];
        }
    }
    // PEC unknowns are pushed far from the shift so they never attract the iteration
    const double big = -1e6 * (std::abs(shift) + 1.0);
    for (int g = 0; g < n; g++) {
        if (unknown_is_pec(*m, o, g)) B.at(g, g) = big;
        B.at(g, g) -= shift;
    }
    if (B.factor()) return -1;

    if (start) {
        const cplx *st = reinterpret_cast<const cplx *>(start);
        for (int g = 0; g < n; g++) x[g] = o.kind[g] == 0 ? st[o.idx[g]] : st[ny * (nz + 1) + o.idx[g]];
    } else {
        unsigned lcg = 12345u;
        for (int g = 0; g < n; g++) {
            lcg = lcg * 1103515245u + 12345u;
            x[g] = ((lcg >> 8) & 0xffff) / 65536.0 - 0.5;
        }
    }
    cplx lam = shift, lam_old = 0;
    std::vector<cplx> xo(n, cplx(0));
    int rc = 1;
    for (int it = 0; it < maxit; it++) {
        double nx2 = 0;
        for (int g = 0; g < n; g++) nx2 += std::real(x[g] * std::conj(x[g]));
        const double inv = 1 / std::sqrt(nx2);
        for (int g = 0; g < n; g++) x[g] *= inv;
        // converge the phase-aligned vector as well as lambda: the source
        // profile comes from the vector
        cplx ph = 0;
        for (int g = 0; g < n; g++) ph += std::conj(xo[g]) * x[g];
        double dv = 0;
        if (std::abs(ph) > 0) {
            ph = std::conj(ph) / std::abs(ph);
            for (int g = 0; g < n; g++) {
                const cplx d = x[g] * ph - xo[g];
                dv += std::real(d * std::conj(d));
            }
        } else {
            dv = 1;
        }
        xo = x;
        y = x;
        B.solve(y.data());
        cplx mu = 0;
        for (int g = 0; g < n; g++) mu += std::conj(x[g]) * y[g];
        lam = shift + 1.0 / mu;
        x = y;
        if (it > 2 && std::abs(lam - lam_old) < tol * std::abs(lam) && std::sqrt(dv) < 1e-10) { rc = 0; break; }
        lam_old = lam;
    }
    // normalise and make the largest component real
    double nx2 = 0, amax = 0;
    cplx ph = 1;
    for (int g = 0; g < n; g++) {
        nx2 += std::real(x[g] * std::conj(x[g]));
        if (std::abs(x[g]) > amax) { amax = std::abs(x[g]); ph = std::conj(x[g]) / amax; }
    }
    const double inv = 1 / std::sqrt(nx2);
    std::fill(m->eu.begin(), m->eu.end(), cplx(0));
    std::fill(m->ev.begin(), m->ev.end(), cplx(0));
    for (int g = 0; g < n; g++) {
        if (unknown_is_pec(*m, o, g)) continue;
        (o.kind[g] == 0 ? m->eu : m->ev)[o.idx[g]] = x[g] * inv * ph;
    }
    cplx bt = std::sqrt(lam);
    if (std::real(bt) < 0) bt = -bt;
    m->beta = bt;
    m->freq = f;
    apply_q(*m, c, w, m->eu.data(), m->ev.data(), m->hu.data(), m->hv.data(), W.wk.data());
    for (cplx &v : m->hu) v /= bt;
    for (cplx &v : m->hv) v /= bt;
    return rc;
}

double cem_mode2d_beta(const cem_mode2d *m) { return std::real(m->beta); }
double cem_mode2d_alpha(const cem_mode2d *m) { return -std::imag(m->beta); }
const double *cem_mode2d_eu(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->eu.data()); }
const double *cem_mode2d_ev(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->ev.data()); }
const double *cem_mode2d_hu(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->hu.data()); }
const double *cem_mode2d_hv(const cem_mode2d *m) { return reinterpret_cast<const double *>(m->hv.data()); }

// Real part of the complex power 1/2 sum (Eu Hv* - Ev Hu*) dA.
double cem_mode2d_power(const cem_mode2d *m) {
    const int ny = m->ny, nz = m->nz;
    cplx P = 0;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k <= nz; k++) P += m->eu[m->iu(j, k)] * std::conj(m->hv[m->iu(j, k)]) * m->dy[j] * m->ddz[k];
    for (int j = 0; j <= ny; j++)
        for (int k = 0; k < nz; k++) P -= m->ev[m->iv(j, k)] * std::conj(m->hu[m->iv(j, k)]) * m->ddy[j] * m->dz[k];
    return 0.5 * std::real(P);
}

// V = -sum Ez dz on node column j0, k0..k1; I = circulation of H around the
// dual rectangle (ja+1/2..jb+1/2) x (ka+1/2..kb+1/2), current in +x.
void cem_mode2d_vi(const cem_mode2d *m, int j0, int k0, int k1, int ja, int jb, int ka, int kb, double *V,
                   double *Iout) {
    cplx v = 0, c = 0;
    for (int k = k0; k < k1; k++) v -= m->ev[m->iv(j0, k)] * m->dz[k];
    for (int j = ja + 1; j <= jb; j++) c += (m->hu[m->iv(j, ka)] - m->hu[m->iv(j, kb)]) * m->ddy[j];
    for (int k = ka + 1; k <= kb; k++) c += (m->hv[m->iu(jb, k)] - m->hv[m->iu(ja, k)]) * m->ddz[k];
    V[0] = std::real(v); V[1] = std::imag(v);
    Iout[0] = std::real(c); Iout[1] = std::imag(c);
}

// Conductor attenuation by perturbation: P_loss = Rs/2 sum |n x H|^2 dl over
// metal surfaces facing a field cell, alpha_c = P_loss / (2 P).
// (reference mode2d.c:444-498)
double cem_mode2d_conductor_alpha(const cem_mode2d *m, double Rs) {
    const int ny = m->ny, nz = m->nz;
    auto solid = [&](int j, int k) {
        return j >= 0 && j < ny && k >= 0 && k < nz && m->pec_u[m->iu(j, k)] && m->pec_u[m->iu(j, k + 1)] &&
               m->pec_v[m->iv(j, k)] && m->pec_v[m->iv(j + 1, k)];
    };
    const double w = 2 * M_PI * m->freq;
    auto curl_w = [&](int j, int k) {
        return (m->ev[m->iv(j + 1, k)] - m->ev[m->iv(j, k)]) / m->dy[j] - (m->eu[m->iu(j, k + 1)] - m->eu[m->iu(j, k)]) / m->dz[k];
    };
    double loss = 0;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k <= nz; k++) {
            if (!m->pec_u[m->iu(j, k)]) continue;
            if (m->ps[0][j] > 0 || m->ps[3][k] > 0) continue;   // metal inside the PML is not the device
            for (int side = 0; side < 2; side++) {
                const int kc = side == 0 ? k : k - 1;
                if (kc < 0 || kc >= nz || solid(j, kc)) continue;
                const double hw = std::abs(curl_w(j, kc)) / (w * CEM_MU0);
                loss += 0.5 * Rs * hw * hw * m->dy[j];
                for (int e = 0; e < 2; e++) {
                    const int jn = j + e;
                    if (m->pec_v[m->iv(jn, kc)]) continue;
                    const double hu = std::abs(m->hu[m->iv(jn, kc)]);
                    loss += 0.5 * Rs * hu * hu * 0.5 * m->dy[j];
                }
            }
        }
    for (int j = 0; j <= ny; j++)
        for (int k = 0; k < nz; k++) {
            if (!m->pec_v[m->iv(j, k)]) continue;
            if (m->ps[1][j] > 0 || m->ps[2][k] > 0) continue;
            for (int side = 0; side < 2; side++) {
                const int jc = side == 0 ? j : j - 1;
                if (jc < 0 || jc >= ny || solid(jc, k)) continue;
                const double hw = std::abs(curl_w(jc, k)) / (w * CEM_MU0);
                loss += 0.5 * Rs * hw * hw * m->dz[k];
                for (int e = 0; e < 2; e++) {
                    const int kn = k + e;
                    if (m->pec_u[m->iu(jc, kn)]) continue;
                    const double hv = std::abs(m->hv[m->iu(jc, kn)]);
                    loss += 0.5 * Rs * hv * hv * 0.5 * m->dz[k];
                }
            }
        }
    const double P = cem_mode2d_power(m);
    return P > 0 ? loss / (2 * P) : 0;
}

}  // extern "C"
