// Plan export for external steppers, sample push-back, checkpoints, state
// arrays, and the time-stepping entry points of the C ABI.
//
// Plan and checkpoint formats are the reference's (skyhoffert/CourantEM
// solver/src/export.c): indices as doubles in the global comp*N + q space,
// checkpoints as an 8-double header plus blocks in a fixed order. Keeping the
// formats lets a run move between this library and the reference core.
#include "sim.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

using namespace cb2;

namespace {

constexpr double kCheckpointMagic = 20261017.0;

void phasors_at(const cem_sim *s, long step, std::vector<double> &phE, std::vector<double> &phH) {
    phE.assign(2 * s->nf, 0.0);
    phH.assign(2 * s->nf, 0.0);
    const double tE = (step + 1) * s->dt, tH = (step + 0.5) * s->dt;
    for (int f = 0; f < s->nf; f++) {
        const double w = 2 * M_PI * s->freq[f];
        phE[2 * f] = std::cos(w * tE); phE[2 * f + 1] = -std::sin(w * tE);
        phH[2 * f] = std::cos(w * tH); phH[2 * f + 1] = -std::sin(w * tH);
    }
}

// Walk the checkpoint blocks in the reference order (export.c:187-213);
// visit(ptr, n) gets each block's host array (or nullptr when absent).
template <class F>
size_t checkpoint_blocks(cem_sim *s, F visit) {
    size_t o = 0;
    auto block = [&](double *p, size_t n) { visit(p, n, o); o += n; };
    for (int c = 0; c < 3; c++) block(s->E[c].empty() ? nullptr : s->E[c].data(), s->N);
    for (int c = 0; c < 3; c++) block(s->H[c].empty() ? nullptr : s->H[c].data(), s->N);
    if (s->has_pml)
        for (int c = 0; c < 3; c++)
            for (int w = 0; w < 2; w++) {
                block(s->psiE[c][w].empty() ? nullptr : s->psiE[c][w].data(), psi_len(s, 1, c, w));
                block(s->psiH[c][w].empty() ? nullptr : s->psiH[c][w].data(), psi_len(s, 0, c, w));
            }
    if (s->ndisp) {
        block(s->d_J.empty() ? nullptr : s->d_J.data(), (size_t)s->npole * s->ndisp);
        block(s->d_Eold.empty() ? nullptr : s->d_Eold.data(), s->ndisp);
    }
    if (s->nsb) block(s->sb_y.empty() ? nullptr : s->sb_y.data(), (size_t)s->nsb * s->sibc_npole);
    for (LumpedPort &p : s->port) {
        block(p.V.data(), 2 * s->nf);
        block(p.I.data(), 2 * s->nf);
    }
    for (VoltageProbe &p : s->vp) block(p.acc.data(), 2 * s->nf);
    for (CurrentProbe &p : s->ip) block(p.acc.data(), 2 * s->nf);
    block(s->src_acc.data(), 2 * s->nf);
    block(s->phE.empty() ? nullptr : s->phE.data(), 2 * s->nf);
    block(s->phH.empty() ? nullptr : s->phH.data(), 2 * s->nf);
    return o;
}

size_t checkpoint_body(const cem_sim *s) {
    return checkpoint_blocks(const_cast<cem_sim *>(s), [](double *, size_t, size_t) {});
}

void report(const char *what) {
    std::fprintf(stderr, "courant-b200: %s: %s\n", what, cem_last_error());
}

}  // namespace

extern "C" {

// which: 0 ca, 1 cb, 2 ide, 3 idh, 4 be, 5 ce, 6 bh, 7 ch, 8 d, 9 dd (reference export.c:13-31)
const double *cem_plan_array(const cem_sim *s, int which, int comp) {
    if (!s->finalized || comp < 0 || comp > 2) return nullptr;
    switch (which) {
    case 0: return s->ca[comp].data();
    case 1: return s->cb[comp].data();
    case 2: return s->ide[comp].data();
    case 3: return s->idh[comp].data();
    case 4: return s->be[comp].data();
    case 5: return s->ce[comp].data();
    case 6: return s->bh[comp].data();
    case 7: return s->ch[comp].data();
    case 8: return s->d[comp].data();
    case 9: return s->dd[comp].data();
    default: return nullptr;
    }
}

int cem_plan_npml(const cem_sim *s, int face) { return face >= 0 && face < 6 ? s->npml[face] : 0; }
int cem_plan_has_pml(const cem_sim *s) { return s->has_pml; }
int cem_plan_nport(const cem_sim *s) { return (int)s->port.size(); }
int cem_plan_nvprobe(const cem_sim *s) { return (int)s->vp.size(); }
int cem_plan_niprobe(const cem_sim *s) { return (int)s->ip.size(); }
int cem_plan_ndisp(const cem_sim *s) { return s->ndisp; }
int cem_plan_nsibc(const cem_sim *s) { return s->nsb; }
int cem_plan_npole(const cem_sim *s) { return s->npole; }
int cem_plan_excited_lumped(const cem_sim *s) { return s->src_port; }

int cem_plan_port(const cem_sim *s, int p, double *idx, double *vw, double *cs) {
    if (p < 0 || p >= (int)s->port.size()) return -1;
    const LumpedPort &pt = s->port[p];
    for (size_t e = 0; e < pt.edge.size(); e++) {
        if (idx) idx[e] = (double)(pt.axis * s->N + pt.edge[e]);
        if (vw) vw[e] = pt.dl[e] * pt.dir;
        if (cs) cs[e] = pt.cs[e];
    }
    return (int)pt.edge.size();
}

int cem_plan_vprobe(const cem_sim *s, int p, double *idx, double *w) {
    if (p < 0 || p >= (int)s->vp.size()) return -1;
    const VoltageProbe &v = s->vp[p];
    for (size_t e = 0; e < v.edge.size(); e++) {
        if (idx) idx[e] = (double)(v.axis * s->N + v.edge[e]);
        if (w) w[e] = v.dl[e];
    }
    return (int)v.edge.size();
}

int cem_plan_iprobe(const cem_sim *s, int p, double *idx, double *w) {
    if (p < 0 || p >= (int)s->ip.size()) return -1;
    const CurrentProbe &c = s->ip[p];
    for (size_t e = 0; e < c.idx.size(); e++) {
        if (idx) idx[e] = (double)((c.comp[e] - 3) * s->N + c.idx[e]);
        if (w) w[e] = c.w[e];
    }
    return (int)c.idx.size();
}

int cem_plan_mode_source(const cem_sim *s, double *idx, double *w) {
    if (s->msrc < 0) return 0;
    const ModePort &p = s->mport[s->msrc];
    for (size_t i = 0; i < p.src_idx.size(); i++) {
        if (idx) idx[i] = (double)(p.src_comp[i] * s->N + p.src_idx[i]);
        if (w) w[i] = p.src_w[i];
    }
    return (int)p.src_idx.size();
}

// source waveforms at H times t = (n + 1/2) dt for n0 .. n0+n-1 (reference export.c:89-99)
void cem_plan_waveforms(const cem_sim *s, long n0, int n, double *lumped, double *mode) {
    for (int q = 0; q < n; q++) {
        const double t = (n0 + q + 0.5) * s->dt;
        if (lumped) lumped[q] = lumped_source_value(s, t);
        if (mode) mode[q] = mode_source_value(s, t);
    }
}

int cem_plan_disp(const cem_sim *s, double *idx, double *cb, double *beta, double *k) {
    for (int e = 0; e < s->ndisp; e++) {
        if (idx) idx[e] = (double)(s->d_comp[e] * s->N + s->d_idx[e]);
        if (cb) cb[e] = s->d_cb[e];
    }
    if (beta && !s->d_beta.empty()) std::memcpy(beta, s->d_beta.data(), s->d_beta.size() * sizeof(double));
    if (k) std::memcpy(k, s->d_k, s->npole * sizeof(double));
    return s->ndisp;
}

int cem_plan_sibc(const cem_sim *s, double *idx, double *hidx, double *hw, double *c, double *e, int *nterm) {
    for (int q = 0; q < s->nsb; q++) {
        if (idx) idx[q] = (double)(s->sb_comp[q] * s->N + s->sb_idx[q]);
        for (int f = 0; f < 4; f++) {
            const bool has = f < s->sb_nf[q];
            if (hidx) hidx[4 * q + f] = has ? (double)(s->sb_hc[4 * q + f] * s->N + s->sb_hi[4 * q + f]) : 0;
            if (hw) hw[4 * q + f] = has ? s->sb_sg[4 * q + f] : 0;
        }
    }
    if (c) std::memcpy(c, s->sibc_c, s->sibc_npole * sizeof(double));
    if (e) std::memcpy(e, s->sibc_e, s->sibc_npole * sizeof(double));
    if (nterm) *nterm = s->sibc_npole;
    return s->nsb;
}

// Samples recorded by an external engine, folded into the DFTs exactly as the
// reference does it (export.c:121-149), on the host in FP64.
void cem_push_samples(cem_sim *s, int n, const double *ip, const double *vold, const double *vnew, const double *vp) {
    if (engine_pull(s, kGroupDft)) return;
    const int nf = s->nf;
    std::vector<double> phE, phH;
    auto acc = [nf](double *a, const std::vector<double> &ph, double v) {
        for (int f = 0; f < nf; f++) { a[2 * f] += v * ph[2 * f]; a[2 * f + 1] += v * ph[2 * f + 1]; }
    };
    const int nip = (int)s->ip.size(), nport = (int)s->port.size(), nvp = (int)s->vp.size();
    for (int q = 0; q < n; q++) {
        const long st = s->step;
        const double tH = (st + 0.5) * s->dt;
        phasors_at(s, st, phE, phH);
        for (int p = 0; p < nip; p++) acc(s->ip[p].acc.data(), phH, ip[(size_t)q * nip + p] * s->dt);
        double Vs = 0;
        if (s->src_port >= 0) {
            Vs = lumped_source_value(s, tH);
            acc(s->src_acc.data(), phH, Vs * s->dt);
        }
        if (s->msrc >= 0) acc(s->src_acc.data(), phH, mode_source_value(s, tH) * s->dt);
        for (int p = 0; p < nport; p++) {
            LumpedPort &pt = s->port[p];
            const double V = 0.5 * (vnew[(size_t)q * nport + p] + vold[(size_t)q * nport + p]);
            const double vs = p == s->src_port ? Vs : 0.0;
            const double I = (vs - V) / pt.R;
            acc(pt.V.data(), phH, V * s->dt);
            acc(pt.I.data(), phH, I * s->dt);
        }
        for (int p = 0; p < nvp; p++) acc(s->vp[p].acc.data(), phE, vp[(size_t)q * nvp + p] * s->dt);
        s->step++;
    }
    engine_host_modified(s, kGroupDft);
}

size_t cem_checkpoint_size(const cem_sim *s) {
    if (!s->finalized) return 0;
    return 8 + checkpoint_body(s);
}

int cem_checkpoint_save(const cem_sim *cs, double *buf) {
    cem_sim *s = const_cast<cem_sim *>(cs);
    if (!s->finalized) { set_error("not finalized"); return -1; }
    if (engine_pull(s, kGroupAll)) return -1;
    phasors_at(s, s->step, s->phE, s->phH);
    // the ADE stores E before the last E update; the device folds that value
    // into the same pass, so the current E at the dispersive edges stands in
    if (s->ndisp) {
        s->d_Eold.resize(s->ndisp);
        for (int e = 0; e < s->ndisp; e++) s->d_Eold[e] = s->E[s->d_comp[e]][s->d_idx[e]];
    }
    const size_t body = checkpoint_body(s);
    const double hdr[8] = {kCheckpointMagic, 1, (double)s->N, (double)s->nf, (double)s->step, (double)body,
                           (double)(s->port.size() + 100 * s->vp.size() + 10000 * s->ip.size()),
                           (double)(s->ndisp + s->nsb)};
    std::memcpy(buf, hdr, sizeof hdr);
    checkpoint_blocks(s, [buf](double *p, size_t n, size_t o) {
        if (p) std::memcpy(buf + 8 + o, p, n * sizeof(double));
        else std::memset(buf + 8 + o, 0, n * sizeof(double));
    });
    return 0;
}

int cem_checkpoint_load(cem_sim *s, const double *buf) {
    if (!s->finalized) { set_error("not finalized"); return -1; }
    const size_t body = checkpoint_body(s);
    if (buf[0] != kCheckpointMagic || buf[1] != 1 || buf[2] != (double)s->N || buf[3] != (double)s->nf ||
        buf[5] != (double)body || buf[6] != (double)(s->port.size() + 100 * s->vp.size() + 10000 * s->ip.size()) ||
        buf[7] != (double)(s->ndisp + s->nsb)) {
        set_error("checkpoint does not match this simulation");
        return -1;
    }
    host_state_alloc(s, kGroupAll);
    s->phE.assign(2 * s->nf, 0.0);
    s->phH.assign(2 * s->nf, 0.0);
    checkpoint_blocks(s, [buf](double *p, size_t n, size_t o) {
        if (p) std::memcpy(p, buf + 8 + o, n * sizeof(double));
    });
    s->step = (long)buf[4];
    engine_host_modified(s, kGroupAll);
    return 0;
}

// which: 0 psiE[comp][w], 1 psiH[comp][w], 2 Debye J, 3 Debye E_old, 4 SIBC states
// (reference export.c:244-268). The pointer stays in step with the device.
double *cem_state_array(cem_sim *s, int which, int comp, int w) {
    if (!s->finalized) return nullptr;
    unsigned g;
    switch (which) {
    case 0: case 1:
        if (!s->has_pml || comp < 0 || comp > 2 || w < 0 || w > 1) return nullptr;
        g = kGroupPsi; break;
    case 2: case 3:
        if (!s->ndisp) return nullptr;
        g = kGroupDebye; break;
    case 4:
        if (!s->nsb) return nullptr;
        g = kGroupSibc; break;
    default: return nullptr;
    }
    if (engine_pull(s, g)) return nullptr;
    engine_expose(s, g);
    switch (which) {
    case 0: return s->psiE[comp][w].data();
    case 1: return s->psiH[comp][w].data();
    case 2: return s->d_J.data();
    case 3: return s->d_Eold.data();
    default: return s->sb_y.data();
    }
}

size_t cem_state_len(const cem_sim *s, int which, int comp, int w) {
    switch (which) {
    case 0: return s->finalized ? psi_len(s, 1, comp, w) : 0;
    case 1: return s->finalized ? psi_len(s, 0, comp, w) : 0;
    case 2: return s->ndisp ? (size_t)s->npole * s->ndisp : 0;
    case 3: return s->ndisp ? (size_t)s->ndisp : 0;
    case 4: return s->nsb ? (size_t)s->nsb * s->sibc_npole : 0;
    default: return 0;
    }
}

void cem_set_step(cem_sim *s, long step) {
    // the DFT ring is indexed by step: fold pending rows before renumbering
    if (engine_has_device(s)) engine_pull(s, kGroupDft);
    s->step = step;
}

void cem_step(cem_sim *s, long n) {
    if (!s->finalized) return;
    if (engine_step(s, n)) report("cem_step");
}

double cem_energy(const cem_sim *s) {
    if (!s->finalized) return 0;
    double W = 0;
    if (engine_energy(s, &W)) {   // device failure: NaN, so no run-control test passes on it
        report("cem_energy");
        return std::numeric_limits<double>::quiet_NaN();
    }
    return W;
}

// Energy-decay run control (reference sim.c:996-1012).
long cem_run(cem_sim *s, long max_steps, double decay, int check_every) {
    if (!s->finalized) return 0;
    if (check_every < 1) check_every = 200;
    const long start = s->step;
    double t_src_end = s->src_port >= 0 ? s->src_t0 + 6 * s->src_tau : 0;
    if (s->msrc >= 0 && s->msrc_t0 + 6 * s->msrc_tau > t_src_end) t_src_end = s->msrc_t0 + 6 * s->msrc_tau;
    double peak = 0;
    while (s->step - start < max_steps) {
        long chunk = check_every;
        if (s->step - start + chunk > max_steps) chunk = max_steps - (s->step - start);
        if (engine_step(s, chunk)) { report("cem_run"); break; }
        double W = 0;
        if (engine_energy(s, &W)) { report("cem_run"); break; }
        if (W > peak) peak = W;
        if (s->step * s->dt > t_src_end && peak > 0 && W < decay * peak) break;
    }
    return s->step - start;
}

// Phased stepping (reference sim.c:863-933): the same kernels as cem_step,
// launched phase by phase; H and E accept any slab split.
void cem_mt_pre(cem_sim *s) {
    if (s->finalized && engine_phase(s, 0, 0, 0)) report("cem_mt_pre");
}
void cem_mt_H(cem_sim *s, int i0, int i1) {
    if (s->finalized && engine_phase(s, 1, i0, i1)) report("cem_mt_H");
}
void cem_mt_mid(cem_sim *s) {
    if (s->finalized && engine_phase(s, 2, 0, 0)) report("cem_mt_mid");
}
void cem_mt_E(cem_sim *s, int i0, int i1) {
    if (s->finalized && engine_phase(s, 3, i0, i1)) report("cem_mt_E");
}
void cem_mt_post(cem_sim *s) {
    if (s->finalized && engine_phase(s, 4, 0, 0)) report("cem_mt_post");
}

}  // extern "C"
