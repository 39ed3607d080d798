// Mode ports on x-directed lines: the eigenmode source profile, the wave
// separation at the monitor plane, two-port renormalisation, and the
// cross-section extraction that feeds the 2D solver. All FP64 on the host.
//
// The discrete-consistency rules (frequency pre-warping, kappa -> beta by the
// arcsine mapping, V interpolated to the current's half plane) and the retry
// ladder of the mode search are those of the reference
// (skyhoffert/CourantEM solver/src/modeport.c), so the wave amplitudes match
// the oracle when fed the same probe spectra.
#include "sim.hpp"

#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

using namespace cb2;

namespace {

// frequency at which the continuous-time 2D problem matches the leapfrog
// scheme (reference modeport.c:64-67)
double warp(const cem_sim *s, double f) { return 2.0 / s->dt * std::sin(M_PI * f * s->dt) / (2 * M_PI); }

}  // namespace

namespace cb2 {

double mode_source_value(const cem_sim *s, double t) {
    if (s->msrc < 0) return 0;
    const double x = (t - s->msrc_t0) / s->msrc_tau;
    return -2 * x * std::exp(-x * x);   // tau d/dt of exp(-x^2): zero DC
}

void modeports_release(cem_sim *s) {
    for (ModePort &p : s->mport) {
        cem_mode2d_destroy(p.xs);
        p.xs = nullptr;
    }
}

// Solve each port's mode at f0 on the monitor-plane cross-section and turn
// its transverse E into source weights on the i_src plane, oriented so the
// source voltage is positive. (reference modeport.c:70-122) The ports are
// independent and are solved on one thread each.
namespace {
int finalize_port(cem_sim *s, ModePort &p) {
    {
        const cem_mode_port_def &d = p.def;
        p.xs = cem_cross_section_x(s, d.i_mon, d.j0, d.j1, d.k0, d.k1);
        if (!p.xs) return -1;
        static const double tries[] = {1.0, 1.08, 0.93, 1.16, 0.87};
        bool ok = false;
        for (int t = 0; t < 5 && !ok; t++) {
            if (!cem_mode2d_solve(p.xs, warp(s, d.f0), p.def.neff0 * tries[t], nullptr, 300, 1e-13)) {
                ok = true;
                p.def.neff0 *= tries[t];
                p.xs_fresh_fw = warp(s, d.f0);
            }
        }
        if (!ok) {
            set_error("mode port: eigenmode did not converge");
            return -1;
        }
        const int ny = d.j1 - d.j0, nz = d.k1 - d.k0;
        const double *eu = cem_mode2d_eu(p.xs), *ev = cem_mode2d_ev(p.xs);
        double vmax = 0;
        for (int i = 0; i < ny * (nz + 1); i++) vmax = std::fabs(eu[2 * i]) > vmax ? std::fabs(eu[2 * i]) : vmax;
        for (int i = 0; i < (ny + 1) * nz; i++) vmax = std::fabs(ev[2 * i]) > vmax ? std::fabs(ev[2 * i]) : vmax;
        p.src_comp.clear(); p.src_idx.clear(); p.src_w.clear();
        for (int j = 0; j < ny; j++)
            for (int k = 0; k <= nz; k++) {
                const double w = eu[2 * (j * (nz + 1) + k)] / vmax;
                if (w == 0) continue;
                const size_t q = idx3(s, d.i_src, d.j0 + j, d.k0 + k);
                if (s->cb[1][q] == 0) continue;
                p.src_comp.push_back(1); p.src_idx.push_back(q); p.src_w.push_back(w);
            }
        for (int j = 0; j <= ny; j++)
            for (int k = 0; k < nz; k++) {
                const double w = ev[2 * (j * nz + k)] / vmax;
                if (w == 0) continue;
                const size_t q = idx3(s, d.i_src, d.j0 + j, d.k0 + k);
                if (s->cb[2][q] == 0) continue;
                p.src_comp.push_back(2); p.src_idx.push_back(q); p.src_w.push_back(w);
            }
        double V[2], Iv[2];
        cem_mode2d_vi(p.xs, d.vj - d.j0, d.vk0 - d.k0, d.vk1 - d.k0, d.ja - d.j0, d.jb - d.j0, d.ka - d.k0,
                      d.kb - d.k0, V, Iv);
        if (-V[0] * d.vsign < 0)
            for (double &w : p.src_w) w = -w;
    }
    return 0;
}
}  // namespace

int modeports_finalize(cem_sim *s) {
    // errors are kept per thread: each port's message comes back with its return code
    std::vector<int> rc(s->mport.size(), 0);
    std::vector<std::string> msg(s->mport.size());
    std::vector<std::thread> th;
    for (size_t q = 0; q < s->mport.size(); q++)
        th.emplace_back([s, q, &rc, &msg] {
            rc[q] = finalize_port(s, s->mport[q]);
            if (rc[q]) msg[q] = cem_last_error();
        });
    for (auto &t : th) t.join();
    for (size_t q = 0; q < rc.size(); q++)
        if (rc[q]) {
            set_error(msg[q].c_str());
            return -1;
        }
    return 0;
}

}  // namespace cb2

namespace {

// Mode at every output frequency, walking outward from the frequency nearest
// f0 and seeding each solve with the previous mode so the same mode is
// tracked; kappa -> beta by the arcsine mapping of the leapfrog grid, Z0 from
// the mode's own V and I. (reference modeport.c:146-201)
//
// The walk starts with a fresh solve at the frequency nearest f0 and a solve
// seeded with it there, as both of the reference's passes do; their results
// are the same, so they run once, on the port's own cross-section, and the
// upward walk continues on a second cross-section given a copy of that mode,
// on its own thread, while the downward walk continues on the port's own one,
// which ends on the lowest frequency's mode as in a walk up then down.

// the seeded solve at frequency q from xs's last mode, and the port's figures there
int port_step(const cem_sim *s, ModePort &p, cem_mode2d *xs, int q, std::vector<double> &start) {
    const cem_mode_port_def &d = p.def;
    const int ny = d.j1 - d.j0, nz = d.k1 - d.k0;
    const double dx = s->d[0][d.i_mon];
    const double fw = warp(s, s->freq[q]);
    const double ng = cem_mode2d_beta(xs) / (2 * M_PI * mode_freq_hint(xs) / CEM_C0);
    std::memcpy(start.data(), cem_mode2d_eu(xs), 2 * ny * (nz + 1) * sizeof(double));
    std::memcpy(start.data() + 2 * ny * (nz + 1), cem_mode2d_ev(xs), 2 * (ny + 1) * nz * sizeof(double));
    if (cem_mode2d_solve(xs, fw, ng, start.data(), 300, 1e-13)) return -1;
    const cplx kc = cem_mode2d_beta(xs) - cplx(0.0, 1.0) * cem_mode2d_alpha(xs);
    const cplx b3 = 2 / dx * std::asin(kc * dx / 2.0);
    p.kappa[2 * q] = std::real(kc); p.kappa[2 * q + 1] = std::imag(kc);
    p.beta[q] = std::real(b3);
    p.alpha[q] = -std::imag(b3);
    if (s->sibc_on) {
        double zr, zi;
        cem_conductor_zs(s, s->freq[q], &zr, &zi);
        p.alpha_c[q] = cem_mode2d_conductor_alpha(xs, zr);
        p.alpha[q] += p.alpha_c[q];
    }
    double V[2], Iv[2];
    cem_mode2d_vi(xs, d.vj - d.j0, d.vk0 - d.k0, d.vk1 - d.k0, d.ja - d.j0, d.jb - d.j0, d.ka - d.k0, d.kb - d.k0,
                  V, Iv);
    // cem_mode2d_vi returns -sum Ez dz; the port voltage is vsign * sum Ez dz
    const cplx Z = (double)(-d.vsign) * cplx(V[0], V[1]) / cplx(Iv[0], Iv[1]);
    p.z0[2 * q] = std::real(Z); p.z0[2 * q + 1] = std::imag(Z);
    return 0;
}

std::vector<double> start_buffer(const ModePort &p) {
    const int ny = p.def.j1 - p.def.j0, nz = p.def.k1 - p.def.k0;
    return std::vector<double>(2 * (size_t)(ny * (nz + 1) + (ny + 1) * nz));
}

// frequencies q0, q0 + stepq, ... to the end of the list, each seeded with the previous mode
int port_walk(const cem_sim *s, ModePort &p, cem_mode2d *xs, int q0, int stepq) {
    std::vector<double> start = start_buffer(p);
    for (int q = q0; q >= 0 && q < s->nf; q += stepq)
        if (port_step(s, p, xs, q, start)) return -1;
    return 0;
}

int solve_port_modes(cem_sim *s, ModePort &p) {
    const int nf = s->nf;
    const cem_mode_port_def &d = p.def;
    p.z0.assign(2 * nf, 0.0);
    p.beta.assign(nf, 0.0);
    p.alpha.assign(nf, 0.0);
    p.kappa.assign(2 * nf, 0.0);
    p.alpha_c.assign(nf, 0.0);
    int q0 = 0;
    for (int q = 0; q < nf; q++)
        if (std::fabs(s->freq[q] - d.f0) < std::fabs(s->freq[q0] - d.f0)) q0 = q;
    auto fail = [] {
        set_error("mode port: eigenmode did not converge at an output frequency");
        return -1;
    };
    std::vector<double> start = start_buffer(p);
    // the unseeded solve at the starting frequency: finalize's, when f0 is that frequency (an
    // unseeded solve depends on nothing but the section, the frequency and the shift)
    const double fw0 = warp(s, s->freq[q0]);
    if (p.xs_fresh_fw != fw0) cem_mode2d_solve(p.xs, fw0, d.neff0, nullptr, 300, 1e-13);
    p.xs_fresh_fw = -1;
    if (port_step(s, p, p.xs, q0, start)) return fail();
    cem_mode2d *up = cem_cross_section_x(s, d.i_mon, d.j0, d.j1, d.k0, d.k1);
    if (!up) return -1;
    mode2d_copy_mode(up, p.xs);
    int rc_up = 0;
    std::thread t([&] { rc_up = port_walk(s, p, up, q0 + 1, 1); });
    const int rc_down = port_walk(s, p, p.xs, q0 - 1, -1);
    t.join();
    cem_mode2d_destroy(up);
    if (rc_up || rc_down) return fail();
    p.solved = true;
    return 0;
}

// the output-frequency modes of every mode port not solved yet, one thread per port
int solve_all_ports(cem_sim *s) {
    std::vector<std::thread> th;
    std::vector<int> rc(s->mport.size(), 0);
    std::vector<std::string> msg(s->mport.size());
    for (size_t q = 0; q < s->mport.size(); q++)
        if (!s->mport[q].solved)
            th.emplace_back([s, q, &rc, &msg] {
                rc[q] = solve_port_modes(s, s->mport[q]);
                if (rc[q]) msg[q] = cem_last_error();
            });
    for (auto &t : th) t.join();
    for (size_t q = 0; q < rc.size(); q++)
        if (rc[q]) {
            set_error(msg[q].c_str());
            return -1;
        }
    return 0;
}

}  // namespace

extern "C" {

int cem_add_mode_port(cem_sim *s, const cem_mode_port_def *d) {
    if (s->finalized) { set_error("already finalized"); return -1; }
    if ((int)s->mport.size() >= kMaxModePorts) { set_error("too many mode ports"); return -1; }
    if (d->i_mon < 1 || d->i_mon + 1 > s->n[0] || d->i_src < 1 || d->i_src >= s->n[0] || d->j0 < 0 ||
        d->j1 > s->n[1] || d->k0 < 0 || d->k1 > s->n[2] || (d->dir != 1 && d->dir != -1)) {
        set_error("bad mode port definition");
        return -1;
    }
    if ((d->dir == 1 && d->i_src >= d->i_mon) || (d->dir == -1 && d->i_src <= d->i_mon + 1)) {
        set_error("mode port source must lie behind the monitor (away from the device)");
        return -1;
    }
    ModePort p;
    p.def = *d;
    if (!(p.def.neff0 > 0)) p.def.neff0 = 1.0;
    p.vp0 = cem_add_vprobe(s, CEM_Z, d->i_mon, d->vj, d->vk0, d->vk1, d->vsign);
    p.vp1 = cem_add_vprobe(s, CEM_Z, d->i_mon + 1, d->vj, d->vk0, d->vk1, d->vsign);
    p.ip = cem_add_iprobe(s, CEM_X, d->i_mon, d->ja, d->jb, d->ka, d->kb);
    if (p.vp0 < 0 || p.vp1 < 0 || p.ip < 0) return -1;
    s->mport.push_back(std::move(p));
    return (int)s->mport.size() - 1;
}

int cem_add_mode_port_args(cem_sim *s, int dir, int i_src, int i_mon, int j0, int j1, int k0, int k1, int vj,
                           int vk0, int vk1, int vsign, int ja, int jb, int ka, int kb, double x_ref, double f0,
                           double neff0) {
    const cem_mode_port_def d = {dir, i_src, i_mon, j0, j1, k0, k1, vj, vk0, vk1, vsign, ja, jb, ka, kb, x_ref, f0, neff0};
    return cem_add_mode_port(s, &d);
}

int cem_set_mode_excitation(cem_sim *s, int port, double t0, double tau) {
    if (port < 0 || port >= (int)s->mport.size()) { set_error("bad mode port"); return -1; }
    s->msrc = port; s->msrc_t0 = t0; s->msrc_tau = tau;
    return 0;
}

// Incident and outgoing waves at the reference plane, normalised to the
// port's Z0(f). (reference modeport.c:203-227)
int cem_mode_port_waves(cem_sim *s, int port, double *a, double *b, double *z0, double *beta) {
    if (port < 0 || port >= (int)s->mport.size() || !s->finalized) { set_error("bad mode port"); return -1; }
    ModePort &p = s->mport[port];
    if (!p.solved && solve_all_ports(s)) return -1;
    const double *V0 = cem_vprobe(s, p.vp0), *V1 = cem_vprobe(s, p.vp1), *Ix = cem_iprobe(s, p.ip);
    const cem_mode_port_def &d = p.def;
    const double dx = s->d[0][d.i_mon];
    const double xmon = 0.5 * (s->node[0][d.i_mon] + s->node[0][d.i_mon + 1]);
    const double dist = d.dir * (d.x_ref - xmon);   // monitor -> reference, into the device
    const cplx J(0.0, 1.0);
    for (int q = 0; q < s->nf; q++) {
        const cplx Z = p.z0[2 * q] + J * p.z0[2 * q + 1];
        const cplx g = p.alpha[q] + J * p.beta[q];
        const cplx c = std::cosh(g * dx / 2.0);
        const cplx V = ((V0[2 * q] + V1[2 * q]) + J * (V0[2 * q + 1] + V1[2 * q + 1])) / (2.0 * c);
        const cplx Iin = (double)d.dir * (Ix[2 * q] + J * Ix[2 * q + 1]);
        const cplx sq = 2.0 * std::sqrt(Z);
        cplx A = (V + Z * Iin) / sq, Bw = (V - Z * Iin) / sq;
        A *= std::exp(-g * dist);
        Bw *= std::exp(g * dist);
        a[2 * q] = std::real(A); a[2 * q + 1] = std::imag(A);
        b[2 * q] = std::real(Bw); b[2 * q + 1] = std::imag(Bw);
        if (z0) z0[q] = std::real(Z);
        if (beta) beta[q] = p.beta[q];
    }
    return 0;
}

int cem_mode_port_alpha(const cem_sim *s, int port, double *alpha) {
    if (port < 0 || port >= (int)s->mport.size() || !s->mport[port].solved) { set_error("mode port not solved"); return -1; }
    std::memcpy(alpha, s->mport[port].alpha.data(), s->nf * sizeof(double));
    return 0;
}

int cem_mode_port_alpha_c(const cem_sim *s, int port, double *alpha_c) {
    if (port < 0 || port >= (int)s->mport.size() || !s->mport[port].solved) { set_error("mode port not solved"); return -1; }
    std::memcpy(alpha_c, s->mport[port].alpha_c.data(), s->nf * sizeof(double));
    return 0;
}

// S' = (Z - zref)(Z + zref)^-1 with Z = sqrt(Zd) (I + S)(I - S)^-1 sqrt(Zd).
// (reference modeport.c:242-264)
void cem_s2_renormalize(double *Sv, double z1, double z2, double zref) {
    const cplx J(0.0, 1.0);
    const cplx S[2][2] = {{Sv[0] + J * Sv[1], Sv[2] + J * Sv[3]}, {Sv[4] + J * Sv[5], Sv[6] + J * Sv[7]}};
    const cplx A[2][2] = {{1.0 - S[0][0], -S[0][1]}, {-S[1][0], 1.0 - S[1][1]}};
    const cplx det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    const cplx Ai[2][2] = {{A[1][1] / det, -A[0][1] / det}, {-A[1][0] / det, A[0][0] / det}};
    const cplx B[2][2] = {{1.0 + S[0][0], S[0][1]}, {S[1][0], 1.0 + S[1][1]}};
    cplx Zn[2][2], Z[2][2], R[2][2];
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) Zn[r][c] = B[r][0] * Ai[0][c] + B[r][1] * Ai[1][c];
    const double sq[2] = {std::sqrt(z1), std::sqrt(z2)};
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) Z[r][c] = sq[r] * Zn[r][c] * sq[c];
    const cplx P[2][2] = {{Z[0][0] + zref, Z[0][1]}, {Z[1][0], Z[1][1] + zref}};
    const cplx Mm[2][2] = {{Z[0][0] - zref, Z[0][1]}, {Z[1][0], Z[1][1] - zref}};
    const cplx dp = P[0][0] * P[1][1] - P[0][1] * P[1][0];
    const cplx Pi[2][2] = {{P[1][1] / dp, -P[0][1] / dp}, {-P[1][0] / dp, P[0][0] / dp}};
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) R[r][c] = Mm[r][0] * Pi[0][c] + Mm[r][1] * Pi[1][c];
    Sv[0] = std::real(R[0][0]); Sv[1] = std::imag(R[0][0]); Sv[2] = std::real(R[0][1]); Sv[3] = std::imag(R[0][1]);
    Sv[4] = std::real(R[1][0]); Sv[5] = std::imag(R[1][0]); Sv[6] = std::real(R[1][1]); Sv[7] = std::imag(R[1][1]);
}

// Cross-section of the finalized 3D sim on x node plane i: cell-averaged
// materials and Debye weights, PEC from the update coefficients, and the 3D
// CPML profiles inside the window. (reference sim.c:1026-1079)
cem_mode2d *cem_cross_section_x(const cem_sim *s, int i, int j0, int j1, int k0, int k1) {
    if (!s->finalized || i < 0 || i >= s->n[0] || j0 < 0 || j1 > s->n[1] || k0 < 0 || k1 > s->n[2] || j1 - j0 < 2 ||
        k1 - k0 < 2) {
        set_error("bad cross-section window");
        return nullptr;
    }
    const int ny = j1 - j0, nz = k1 - k0, np = s->npole;
    cem_mode2d *m = cem_mode2d_create(ny, nz, s->node[1].data() + j0, s->node[2].data() + k0);
    const int nu = ny * (nz + 1), nv = (ny + 1) * nz, nn = (ny + 1) * (nz + 1);
    std::vector<double> eu(nu), ev(nv), ew(nn), su(nu, 0.0), sv(nv, 0.0), sw(nn, 0.0);
    std::vector<unsigned char> pu(nu, 0), pv(nv, 0), pw(nn, 0);
    std::vector<double> du((size_t)np * nu, 0.0), dv((size_t)np * nv, 0.0), dw((size_t)np * nn, 0.0);
    double dep[kMaxPoles];
    int pec;
    // one unknown family per component: (component, count in y, count in z, outputs)
    auto fill = [&](int comp, int jcount, int kcount, std::vector<double> &er, std::vector<double> &sg,
                    std::vector<unsigned char> &pe, std::vector<double> &dp, int ntot) {
        for (int j = 0; j < jcount; j++)
            for (int k = 0; k < kcount; k++) {
                const size_t q = idx3(s, i, j0 + j, k0 + k);
                const int o = j * kcount + k;
                if (s->cb[comp][q] == 0) { pe[o] = 1; er[o] = 1; continue; }
                edge_material(s, comp, i, j0 + j, k0 + k, &er[o], &sg[o], &pec);
                if (np && edge_debye(s, comp, i, j0 + j, k0 + k, dep))
                    for (int p = 0; p < np; p++) dp[(size_t)p * ntot + o] = dep[p];
            }
    };
    fill(1, ny, nz + 1, eu, su, pu, du, nu);       // E_u = Ey
    fill(2, ny + 1, nz, ev, sv, pv, dv, nv);       // E_v = Ez
    fill(0, ny + 1, nz + 1, ew, sw, pw, dw, nn);   // E_w = Ex
    if (np) cem_mode2d_set_debye(m, np, s->pole_f, du.data(), dv.data(), dw.data());
    cem_mode2d_set_media(m, eu.data(), ev.data(), ew.data(), pu.data(), pv.data(), pw.data());
    cem_mode2d_set_loss(m, su.data(), sv.data(), sw.data());
    cem_mode2d_set_pml(m, 0, s->pml_sc[1].data() + j0, s->pml_kc[1].data() + j0, s->pml_ac[1].data() + j0);
    cem_mode2d_set_pml(m, 1, s->pml_sn[1].data() + j0, s->pml_kn[1].data() + j0, s->pml_an[1].data() + j0);
    cem_mode2d_set_pml(m, 2, s->pml_sc[2].data() + k0, s->pml_kc[2].data() + k0, s->pml_ac[2].data() + k0);
    cem_mode2d_set_pml(m, 3, s->pml_sn[2].data() + k0, s->pml_kn[2].data() + k0, s->pml_an[2].data() + k0);
    return m;
}

}  // extern "C"
