// Internal host-side state of libcourant_b200.
//
// The host keeps the FP64 "plan" of a simulation (node coordinates, cell
// materials, per-edge update coefficients, CPML profiles, port/probe/source
// tables) in the same index space as the reference core (k fastest, stride
// sj = nz+1, si = (ny+1)(nz+1); reference sim_internal.h:151-153). Everything
// that evolves in time lives on the device (engine.cu) once the first step
// has run; host copies of that state exist only when a caller asks for them.
#pragma once

#include "../../include/courant.h"

#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <sys/mman.h>

namespace cb2 {

// A large host array set to n copies of val: capacity reserved first (fresh
// pages, untouched), advised for transparent huge pages, then filled, so that
// its first touch faults in 2 MB pages instead of 4 kB ones (set-up of a
// large grid otherwise spends most of its time in page faults).
template <class T>
void big_assign(std::vector<T> &v, size_t n, const T &val) {
    std::vector<T>().swap(v);
    v.reserve(n);
    constexpr uintptr_t kHuge = (uintptr_t)2 << 20;
    if (n * sizeof(T) >= 2 * kHuge) {
        const uintptr_t b = reinterpret_cast<uintptr_t>(v.data());
        const uintptr_t a = (b + kHuge - 1) & ~(kHuge - 1), e = (b + n * sizeof(T)) & ~(kHuge - 1);
        if (e > a) madvise(reinterpret_cast<void *>(a), e - a, MADV_HUGEPAGE);
    }
    v.assign(n, val);
}

// Limits of the reference core (sim_internal.h:14-15,42-43); kept so the same
// programs hit the same errors.
constexpr int kMaxPorts = 16;
constexpr int kMaxProbes = 256;
constexpr int kMaxModePorts = 8;
constexpr int kMaxPoles = 16;
constexpr int kSibcTerms = 12;   // Foster terms of the surface-impedance fit (sibc.c:122)

using cplx = std::complex<double>;

void set_error(const char *msg);

struct LumpedPort {
    int axis = 0, dir = 1;
    double R = 50.0;
    std::vector<size_t> edge;   // field index of each edge of the column
    std::vector<double> dl;     // edge lengths
    std::vector<double> cs;     // source coefficient per edge (per volt of Vs)
    std::vector<double> V, I;   // host copies of the DFT accumulators, 2*nf
};

struct VoltageProbe {
    int axis = 0, dir = 1;
    std::vector<size_t> edge;
    std::vector<double> dl;     // signed edge lengths (dl * dir)
    std::vector<double> acc;
};

struct CurrentProbe {
    std::vector<int> comp;      // 3..5
    std::vector<size_t> idx;
    std::vector<double> w;      // signed dual lengths
    std::vector<double> acc;
};

struct ModePort {
    cem_mode_port_def def{};
    int vp0 = -1, vp1 = -1, ip = -1;      // probe indices created for the port
    std::vector<int> src_comp;            // 1 (Ey) or 2 (Ez)
    std::vector<size_t> src_idx;
    std::vector<double> src_w;            // source profile on the i_src plane
    cem_mode2d *xs = nullptr;             // cross-section at the monitor plane
    double xs_fresh_fw = -1;              // xs holds the unseeded solve at this warped frequency and neff0 (-1: not)
    std::vector<double> z0, kappa;        // complex, 2*nf
    std::vector<double> beta, alpha, alpha_c;
    bool solved = false;
};

struct Device;  // device-resident time-stepping state (engine.cu)
void device_release(Device *d);

}  // namespace cb2

struct cem_sim {
    int n[3] = {0, 0, 0};
    std::vector<double> node[3], d[3], dd[3];
    size_t si = 0, sj = 0, N = 0;

    // cell materials (cells use the point index; only i<nx, j<ny, k<nz are used)
    std::vector<double> eps_r, sigma;
    std::vector<uint8_t> cell_pec;
    std::vector<uint8_t> edge_pec[3];

    int bc[6] = {0, 0, 0, 0, 0, 0}, npml[6] = {0, 0, 0, 0, 0, 0};
    int has_pml = 0;

    // FP64 plan (cem_plan_array)
    std::vector<double> ca[3], cb[3];
    std::vector<double> ide[3], idh[3], be[3], ce[3], bh[3], ch[3];
    std::vector<double> pml_sn[3], pml_kn[3], pml_an[3], pml_sc[3], pml_kc[3], pml_ac[3];

    double dt = 0;
    long step = 0;
    int finalized = 0;

    // lumped ports and the Gaussian source
    std::vector<cb2::LumpedPort> port;
    int src_port = -1;
    double src_amp = 0, src_t0 = 0, src_tau = 1;
    std::vector<double> src_acc;

    // frequencies and probes
    int nf = 0;
    std::vector<double> freq;
    std::vector<cb2::VoltageProbe> vp;
    std::vector<cb2::CurrentProbe> ip;

    // mode ports
    std::vector<cb2::ModePort> mport;
    int msrc = -1;
    double msrc_t0 = 0, msrc_tau = 1;

    // Debye dispersion: global poles, per-cell weights, per-edge tables
    int npole = 0;
    double pole_f[cb2::kMaxPoles] = {};
    std::vector<double> cell_deps[cb2::kMaxPoles];
    int ndisp = 0;
    std::vector<int> d_comp;
    std::vector<size_t> d_idx;
    std::vector<double> d_cb, d_beta;   // d_beta pole-major: p*ndisp + e
    double d_k[cb2::kMaxPoles] = {};
    std::vector<double> d_J, d_Eold;    // host copies of the ADE state (reference layout)

    // surface impedance
    int sibc_on = 0, sibc_rough = 0, sibc_npole = 0;
    double sibc_sigma = 0, sibc_p1 = 0, sibc_p2 = 0, sibc_fit_err = 0;
    double sibc_a[cb2::kSibcTerms] = {}, sibc_c[cb2::kSibcTerms] = {}, sibc_e[cb2::kSibcTerms] = {};
    int nsb = 0;
    std::vector<int> sb_comp, sb_nf, sb_hc;   // sb_hc: 4 per edge
    std::vector<size_t> sb_idx, sb_hi;        // sb_hi: 4 per edge
    std::vector<double> sb_sg;                // 4 per edge, already divided by the face count
    std::vector<double> sb_y;                 // host copy of the recursive-convolution states

    // host copies of time-dependent state, materialised on demand
    std::vector<double> E[3], H[3];
    std::vector<double> psiE[3][2], psiH[3][2];
    std::vector<double> phE, phH;             // phasor snapshot for checkpoints

    // Coherence of the host copies with the device state, one bit per state
    // group (cb2::StateGroup). host_valid: the host copy holds the current
    // values; dev_valid: the device copy does; exposed: a caller holds a
    // pointer into the host copy and may read or write it between calls.
    // With neither bit set the state is all zeros (freshly finalized).
    unsigned host_valid = 0, dev_valid = 0, exposed = 0;
    int kernel_choice = -1;   // -1: environment default, 0: separate H/E kernels, 1: fused
    int tune_choice = -1;     // -1: environment default (CEM_B200_TUNE), 0: default launch shape, 1: tuned

    std::unique_ptr<cb2::Device, void (*)(cb2::Device *)> dev{nullptr, cb2::device_release};
};

namespace cb2 {

inline size_t idx3(const cem_sim *s, int i, int j, int k) {
    return (size_t)i * s->si + (size_t)j * s->sj + (size_t)k;
}

// setup helpers shared across translation units
void edge_material(const cem_sim *s, int c, int i, int j, int k, double *eps, double *sig, int *pec);
int edge_debye(const cem_sim *s, int c, int i, int j, int k, double *deps);
size_t psi_len(const cem_sim *s, int is_e, int comp, int w);
void pml_ranges(const cem_sim *s, int a, int is_e, int r[2][2]);
size_t pml_per(const cem_sim *s, int a);
int sibc_finalize(cem_sim *s, const std::vector<uint8_t> &is_port);
int modeports_finalize(cem_sim *s);
void modeports_release(cem_sim *s);
double mode_source_value(const cem_sim *s, double t);
double lumped_source_value(const cem_sim *s, double t);
double mode_freq_hint(const cem_mode2d *m);
// the last mode of src (frequency, beta, fields) into dst, a cross-section of the same geometry
void mode2d_copy_mode(cem_mode2d *dst, const cem_mode2d *src);
void nnls(int m, int n, const double *A, const double *b, double *x);

// Host views of time-dependent state. Groups let the engine move only what a
// caller has asked for between host and device.
enum StateGroup : unsigned {
    kGroupE0 = 1u << 0, kGroupE1 = 1u << 1, kGroupE2 = 1u << 2,
    kGroupH0 = 1u << 3, kGroupH1 = 1u << 4, kGroupH2 = 1u << 5,
    kGroupPsi = 1u << 6, kGroupDebye = 1u << 7, kGroupSibc = 1u << 8, kGroupDft = 1u << 9,
    kGroupFields = 0x3f, kGroupAll = 0x3ff,
};

// engine entry points (engine.cu); all return 0 or -1 with the error set
int engine_step(cem_sim *s, long n);
int engine_phase(cem_sim *s, int phase, int i0, int i1);   // cem_mt_* on the device
int engine_energy(const cem_sim *s, double *out);
int engine_pull(const cem_sim *s, unsigned groups);   // device -> host copies (host becomes valid)
void engine_expose(const cem_sim *s, unsigned groups);  // caller holds pointers into these host copies
void engine_host_modified(cem_sim *s, unsigned groups); // host copies were changed by the library
bool engine_has_device(const cem_sim *s);
void host_state_alloc(cem_sim *s, unsigned groups);

}  // namespace cb2
