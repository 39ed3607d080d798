// Material model fits done once on the host in FP64: the Lawson-Hanson
// non-negative least squares solver, the Djordjevic-Sarkar -> Debye fit, the
// surface-impedance (SIBC) Foster fit and the discovery of lossy metal edges.
//
// These feed coefficients into the plan, so each step follows the reference
// arithmetic (skyhoffert/CourantEM solver/src/sibc.c, dispersive.c) in the
// same order, which keeps the fitted values bit-identical to the oracle's.
#include "sim.hpp"

#include <cmath>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace cb2 {

// Lawson-Hanson NNLS for a small dense problem, A column-major (m x n).
// Passive-set least squares by normal equations and Gaussian elimination with
// partial pivoting. (reference sibc.c:45-111)
void nnls(int m, int n, const double *A, const double *b, double *x) {
    std::vector<int> passive(n, 0), active_idx(n);
    std::vector<double> w(n), z(n), r(m), M((size_t)n * n), g(n);
    auto col = [&](int j) { return A + (size_t)j * m; };
    for (int j = 0; j < n; j++) x[j] = 0;
    for (int outer = 0; outer < 3 * n; outer++) {
        for (int i = 0; i < m; i++) {
            r[i] = b[i];
            for (int j = 0; j < n; j++) r[i] -= col(j)[i] * x[j];
        }
        int jmax = -1;
        double wmax = 1e-14;
        for (int j = 0; j < n; j++) {
            w[j] = 0;
            for (int i = 0; i < m; i++) w[j] += col(j)[i] * r[i];
            if (!passive[j] && w[j] > wmax) { wmax = w[j]; jmax = j; }
        }
        if (jmax < 0) break;
        passive[jmax] = 1;
        for (int inner = 0; inner < 3 * n; inner++) {
            int np = 0;
            for (int j = 0; j < n; j++)
                if (passive[j]) active_idx[np++] = j;
            for (int a = 0; a < np; a++) {
                const double *ca = col(active_idx[a]);
                g[a] = 0;
                for (int i = 0; i < m; i++) g[a] += ca[i] * b[i];
                for (int c = 0; c < np; c++) {
                    const double *cc = col(active_idx[c]);
                    double acc = 0;
                    for (int i = 0; i < m; i++) acc += ca[i] * cc[i];
                    M[a * np + c] = acc;
                }
            }
            for (int a = 0; a < np; a++) {
                int piv = a;
                for (int q = a + 1; q < np; q++)
                    if (std::fabs(M[q * np + a]) > std::fabs(M[piv * np + a])) piv = q;
                if (piv != a) {
                    for (int c = 0; c < np; c++) std::swap(M[a * np + c], M[piv * np + c]);
                    std::swap(g[a], g[piv]);
                }
                for (int q = a + 1; q < np; q++) {
                    const double l = M[q * np + a] / M[a * np + a];
                    for (int c = a; c < np; c++) M[q * np + c] -= l * M[a * np + c];
                    g[q] -= l * g[a];
                }
            }
            for (int a = np - 1; a >= 0; a--) {
                double acc = g[a];
                for (int c = a + 1; c < np; c++) acc -= M[a * np + c] * z[active_idx[c]];
                z[active_idx[a]] = acc / M[a * np + a];
            }
            bool feasible = true;
            for (int a = 0; a < np; a++)
                if (z[active_idx[a]] <= 0) feasible = false;
            if (feasible) {
                for (int a = 0; a < np; a++) x[active_idx[a]] = z[active_idx[a]];
                break;
            }
            double alpha = 1;
            for (int a = 0; a < np; a++) {
                const int j = active_idx[a];
                if (z[j] <= 0) {
                    const double t = x[j] / (x[j] - z[j]);
                    if (t < alpha) alpha = t;
                }
            }
            for (int a = 0; a < np; a++) {
                const int j = active_idx[a];
                x[j] += alpha * (z[j] - x[j]);
                if (x[j] <= 1e-300) { x[j] = 0; passive[j] = 0; }
            }
        }
    }
}

namespace {

// Target surface impedance Zs = (1+j) Rs K(w) of a good conductor with an
// optional roughness factor (Groisse or single-size Huray). (reference sibc.c:26-42)
void zs_target(double f, double sigma, int rough, double p1, double p2, double *re, double *im) {
    const double w = 2 * M_PI * f;
    const double rs = std::sqrt(w * CEM_MU0 / (2 * sigma));
    double K = 1;
    const double delta = std::sqrt(2 / (w * CEM_MU0 * sigma));
    if (rough == 1) {
        K = 1 + std::exp(-std::pow(delta / (2 * p1), 1.6));
    } else if (rough == 2) {
        const double a = p1;
        K = 1 + p2 * 4 * M_PI * a * a / (1 + delta / a + delta * delta / (2 * a * a));
    }
    *re = rs * K;
    *im = rs * K;
}

// Djordjevic-Sarkar log term over the 1 kHz .. 1 THz relaxation band
void ds_logterm(double f, double *re, double *im) {
    const double m1 = 3, m2 = 12;
    const double w1 = 2 * M_PI * std::pow(10, m1), w2 = 2 * M_PI * std::pow(10, m2);
    const double w = 2 * M_PI * f;
    const double nr = w2 * w2 + w * w, dr = w1 * w1 + w * w;
    const double ar = std::atan2(w, w2) - std::atan2(w, w1);
    *re = 0.5 * std::log(nr / dr) / std::log(10.0) / (m2 - m1);
    *im = ar / std::log(10.0) / (m2 - m1);
}

// Is the E edge along c at ijk metal? Out-of-range edges and tangential edges
// on a PEC outer face count as metal. (reference sibc.c:173-184)
bool edge_is_metal(const cem_sim *s, int c, const int *ijk) {
    for (int a = 0; a < 3; a++) {
        const int lim = a == c ? s->n[a] - 1 : s->n[a];
        if (ijk[a] < 0 || ijk[a] > lim) return true;
    }
    for (int a = 0; a < 3; a++) {
        if (a == c) continue;
        if (ijk[a] == 0 && s->bc[2 * a] == CEM_BC_PEC) return true;
        if (ijk[a] == s->n[a] && s->bc[2 * a + 1] == CEM_BC_PEC) return true;
    }
    return s->cb[c][idx3(s, ijk[0], ijk[1], ijk[2])] == 0;
}

}  // namespace

// Every metal edge facing at least one non-metal neighbour edge (outside the
// CPML slabs, not a lumped-port edge) becomes a surface-impedance edge with
// J = sum over faces of the signed tangential H, averaged. (reference sibc.c:186-253)
int sibc_finalize(cem_sim *s, const std::vector<uint8_t> &is_port) {
    if (!s->sibc_on) return 0;
    const int nx = s->n[0], ny = s->n[1], nz = s->n[2];
    s->sb_comp.clear(); s->sb_idx.clear(); s->sb_nf.clear();
    s->sb_hc.clear(); s->sb_hi.clear(); s->sb_sg.clear();
    for (int c = 0; c < 3; c++) {
        const int ua = (c + 1) % 3, va = (c + 2) % 3;
        for (int i = 0; i <= nx; i++)
            for (int j = 0; j <= ny; j++)
                for (int k = 0; k <= nz; k++) {
                    const int ijk[3] = {i, j, k};
                    if (ijk[c] >= s->n[c]) continue;
                    const size_t q = idx3(s, i, j, k);
                    if (!edge_is_metal(s, c, ijk)) continue;
                    if (!is_port.empty() && is_port[c * s->N + q]) continue;
                    bool in_pml = false;
                    for (int a = 0; a < 3; a++) {
                        const int lo = s->npml[2 * a], hi = s->npml[2 * a + 1];
                        if (a == c) {
                            if (ijk[a] < lo || ijk[a] >= s->n[a] - hi) in_pml = true;
                        } else if (ijk[a] < lo || ijk[a] > s->n[a] - hi) {
                            in_pml = true;
                        }
                    }
                    if (in_pml) continue;
                    int nface = 0, hc[4];
                    size_t hi[4];
                    double sg[4];
                    int nb[3];
                    auto shifted = [&](int axis, int delta) {
                        nb[0] = ijk[0]; nb[1] = ijk[1]; nb[2] = ijk[2];
                        nb[axis] += delta;
                        return nb;
                    };
                    if (!edge_is_metal(s, c, shifted(va, +1))) { hc[nface] = ua; hi[nface] = q; sg[nface] = -1; nface++; }
                    if (!edge_is_metal(s, c, shifted(va, -1))) {
                        hc[nface] = ua; hi[nface] = idx3(s, nb[0], nb[1], nb[2]); sg[nface] = 1; nface++;
                    }
                    if (!edge_is_metal(s, c, shifted(ua, +1))) { hc[nface] = va; hi[nface] = q; sg[nface] = 1; nface++; }
                    if (!edge_is_metal(s, c, shifted(ua, -1))) {
                        hc[nface] = va; hi[nface] = idx3(s, nb[0], nb[1], nb[2]); sg[nface] = -1; nface++;
                    }
                    if (!nface) continue;
                    s->sb_comp.push_back(c);
                    s->sb_idx.push_back(q);
                    s->sb_nf.push_back(nface);
                    for (int f = 0; f < 4; f++) {
                        const bool has = f < nface;
                        s->sb_hc.push_back(has ? hc[f] : 0);
                        s->sb_hi.push_back(has ? hi[f] : 0);
                        s->sb_sg.push_back(has ? sg[f] / nface : 0.0);
                    }
                }
    }
    s->nsb = (int)s->sb_idx.size();
    for (int k = 0; k < s->sibc_npole; k++) s->sibc_e[k] = std::exp(-s->sibc_a[k] * s->dt);
    return 0;
}

}  // namespace cb2

using namespace cb2;

extern "C" {

void cem_conductor_zs(const cem_sim *s, double f, double *re, double *im) {
    const double w = 2 * M_PI * f;
    *re = *im = 0;
    for (int k = 0; k < s->sibc_npole; k++) {
        const double a = s->sibc_a[k], d = w * w + a * a;
        *re += s->sibc_c[k] * w * w / d;
        *im += s->sibc_c[k] * w * a / d;
    }
}

double cem_conductor_fit_error(const cem_sim *s) { return s->sibc_fit_err; }

// Passive Foster fit Z(s) ~ sum_k c_k s/(s + a_k), a_k log-spaced one decade
// beyond the band on each side, c_k >= 0 by NNLS on relative error.
// (reference sibc.c:115-156)
int cem_set_conductor_loss(cem_sim *s, double sigma, int rough, double p1, double p2, double fmin, double fmax) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if (!(sigma > 0) || !(fmax > fmin) || !(fmin > 0)) { set_error("bad conductor-loss parameters"); return -1; }
    s->sibc_on = 1;
    s->sibc_sigma = sigma;
    s->sibc_rough = rough; s->sibc_p1 = p1; s->sibc_p2 = p2;
    const int K = kSibcTerms, M = 200;
    std::vector<double> A((size_t)2 * M * K), b(2 * M);
    for (int k = 0; k < K; k++) s->sibc_a[k] = 2 * M_PI * fmin / 10 * std::pow(100 * fmax / fmin, (double)k / (K - 1));
    for (int i = 0; i < M; i++) {
        const double f = fmin * std::pow(fmax / fmin, (double)i / (M - 1)), w = 2 * M_PI * f;
        double re, im;
        zs_target(f, sigma, rough, p1, p2, &re, &im);
        const double scale = 1 / std::hypot(re, im);
        b[i] = re * scale;
        b[M + i] = im * scale;
        for (int k = 0; k < K; k++) {
            const double a = s->sibc_a[k], d = w * w + a * a;
            A[(size_t)k * 2 * M + i] = w * w / d * scale;
            A[(size_t)k * 2 * M + M + i] = w * a / d * scale;
        }
    }
    nnls(2 * M, K, A.data(), b.data(), s->sibc_c);
    s->sibc_npole = K;
    double worst = 0;
    for (int i = 0; i < M; i++) {
        const double f = fmin * std::pow(fmax / fmin, (double)i / (M - 1)), w = 2 * M_PI * f;
        double re, im, fr = 0, fi = 0;
        zs_target(f, sigma, rough, p1, p2, &re, &im);
        for (int k = 0; k < K; k++) {
            const double a = s->sibc_a[k], d = w * w + a * a;
            fr += s->sibc_c[k] * w * w / d;
            fi += s->sibc_c[k] * w * a / d;
        }
        const double e = std::hypot(fr - re, fi - im) / std::hypot(re, im);
        if (e > worst) worst = e;
    }
    s->sibc_fit_err = worst;
    return 0;
}

// Djordjevic-Sarkar (Dk, Df at fref) fitted by npole Debye poles log-spaced
// over [fmin/10, 10 fmax] with non-negative weights; returns the worst relative
// loss-tangent error over [fmin, fmax]. (reference dispersive.c:123-171)
double cem_fit_djordjevic_sarkar(double dk, double df, double fref, double fmin, double fmax, int npole,
                                 double *eps_inf, double *f_p, double *deps) {
    double Lr, Li;
    ds_logterm(fref, &Lr, &Li);
    const double d_eps = -dk * df / Li;
    const double e_inf_ds = dk - d_eps * Lr;
    const int M = 200, K = npole + 1;
    std::vector<double> A((size_t)2 * M * K), b(2 * M), x(K);
    for (int p = 0; p < npole; p++)
        f_p[p] = fmin / 10 * std::pow(100 * fmax / fmin, npole > 1 ? (double)p / (npole - 1) : 0.5);
    const double wr = 1 / dk, wi = 1 / std::fmax(dk * df, 1e-6);
    for (int i = 0; i < M; i++) {
        const double f = fmin * std::pow(fmax / fmin, (double)i / (M - 1));
        double re, im;
        ds_logterm(f, &re, &im);
        const double er = e_inf_ds + d_eps * re, ei = d_eps * im;
        b[i] = er * wr;
        b[M + i] = ei * wi;
        for (int p = 0; p < npole; p++) {
            const double r = f / f_p[p], d = 1 + r * r;
            A[(size_t)p * 2 * M + i] = (1 / d) * wr;
            A[(size_t)p * 2 * M + M + i] = (-r / d) * wi;
        }
        A[(size_t)npole * 2 * M + i] = wr;
        A[(size_t)npole * 2 * M + M + i] = 0;
    }
    nnls(2 * M, K, A.data(), b.data(), x.data());
    *eps_inf = x[npole];
    for (int p = 0; p < npole; p++) deps[p] = x[p];
    double worst = 0;
    for (int i = 0; i < M; i++) {
        const double f = fmin * std::pow(fmax / fmin, (double)i / (M - 1));
        double re, im;
        ds_logterm(f, &re, &im);
        const double er = e_inf_ds + d_eps * re, ei = d_eps * im;
        double fr = x[npole], fi = 0;
        for (int p = 0; p < npole; p++) {
            const double r = f / f_p[p], d = 1 + r * r;
            fr += x[p] / d;
            fi += -x[p] * r / d;
        }
        const double t0 = -ei / er, t1 = -fi / fr, e = std::fabs(t1 - t0) / t0;
        if (e > worst) worst = e;
    }
    return worst;
}

}  // extern "C"
