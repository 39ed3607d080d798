// The export table of the Node shim: one entry per function of the
// reference TypeScript wrapper's Exports interface
// (skyhoffert/CourantEM web/src/solver/courant.ts:19-85), each translating JS
// numbers to the courant.h call and the result back (see shim.hpp).
#include <cmath>
#include <limits>
#include <stdexcept>

#include "shim.hpp"

namespace cnapi {

namespace {

using Fn = double (*)(Shim &, const double *);
constexpr double kUndefined = std::numeric_limits<double>::quiet_NaN();

struct Export {
    const char *name;
    int arity;
    bool void_result;
    Fn fn;
};

int I(const double *a, int k) { return (int)a[k]; }
double *P(Shim &s, const double *a, int k) { return static_cast<double *>(s.ptr(a[k])); }

// a call on the simulation in a[0], with its live arrays synchronised around it
template <class F>
double on_sim(Shim &s, const double *a, F f) {
    cem_sim *sim = s.sim(a[0]);
    s.sync_in(a[0]);
    const double r = f(sim);
    s.sync_out(a[0]);
    return r;
}

size_t points(Shim &s, cem_sim *sim) {
    int nx, ny, nz;
    s.lib().cem_dims(sim, &nx, &ny, &nz);
    return (size_t)(nx + 1) * (ny + 1) * (nz + 1);
}

// length of a cem_plan_array result (which 0-1: per point; 2-9 per grid line,
// nodes (n+1) for ide, be, ce, dd and cells (n) for idh, bh, ch, d)
size_t plan_len(Shim &s, cem_sim *sim, int which, int comp) {
    int n[3];
    s.lib().cem_dims(sim, &n[0], &n[1], &n[2]);
    if (which <= 1) return (size_t)(n[0] + 1) * (n[1] + 1) * (n[2] + 1);
    if (comp < 0 || comp > 2) return 0;
    const bool nodes = which == 2 || which == 4 || which == 5 || which == 9;
    return (size_t)n[comp] + (nodes ? 1 : 0);
}

double spectrum(Shim &s, const double *a, int kind, const double *(*get)(const cnapi::Lib &, cem_sim *, int)) {
    return on_sim(s, a, [&](cem_sim *sim) {
        const int idx = kind == 4 ? 0 : I(a, 1);
        return s.mirror(a[0], kind, idx, 0, get(s.lib(), sim, idx), 2 * (size_t)s.lib().cem_nfreq(sim), false);
    });
}

#define SIM(body) [](Shim &s, const double *a) -> double { return on_sim(s, a, [&](cem_sim *sim) -> double { body; }); }
#define SIMV(body) [](Shim &s, const double *a) -> double { return on_sim(s, a, [&](cem_sim *sim) -> double { body; return 0; }); }

const Export kExports[] = {
    {"cem_last_error", 0, false, [](Shim &s, const double *) -> double { return s.string_mirror(s.lib().cem_last_error()); }},
    {"cem_create", 6, false, [](Shim &s, const double *a) -> double {
         return s.new_handle(s.lib().cem_create(I(a, 0), I(a, 1), I(a, 2), P(s, a, 3), P(s, a, 4), P(s, a, 5)));
     }},
    {"cem_destroy", 1, true, [](Shim &s, const double *a) -> double {
         s.lib().cem_destroy(s.sim(a[0]));
         s.drop_handle(a[0]);
         return 0;
     }},
    {"cem_set_boundary", 4, false, SIM(return s.lib().cem_set_boundary(sim, I(a, 1), I(a, 2), I(a, 3)))},
    {"cem_material_box", 9, false, SIM(return s.lib().cem_material_box(sim, a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]))},
    {"cem_pec_box", 7, false, SIM(return s.lib().cem_pec_box(sim, a[1], a[2], a[3], a[4], a[5], a[6]))},
    {"cem_pec_sheet", 7, false, SIM(return s.lib().cem_pec_sheet(sim, I(a, 1), a[2], a[3], a[4], a[5], a[6]))},
    {"cem_add_lumped_port", 8, false,
     SIM(return s.lib().cem_add_lumped_port(sim, I(a, 1), I(a, 2), I(a, 3), I(a, 4), I(a, 5), I(a, 6), a[7]))},
    {"cem_set_gaussian", 5, false, SIM(return s.lib().cem_set_gaussian(sim, I(a, 1), a[2], a[3], a[4]))},
    {"cem_set_frequencies", 3, false, SIM(return s.lib().cem_set_frequencies(sim, I(a, 1), P(s, a, 2)))},
    {"cem_add_vprobe", 7, false, SIM(return s.lib().cem_add_vprobe(sim, I(a, 1), I(a, 2), I(a, 3), I(a, 4), I(a, 5), I(a, 6)))},
    {"cem_add_iprobe", 7, false, SIM(return s.lib().cem_add_iprobe(sim, I(a, 1), I(a, 2), I(a, 3), I(a, 4), I(a, 5), I(a, 6)))},
    {"cem_finalize", 2, false, SIM(return s.lib().cem_finalize(sim, a[1]))},
    {"cem_dt", 1, false, SIM(return s.lib().cem_dt(sim))},
    {"cem_step_count", 1, false, SIM(return (double)s.lib().cem_step_count(sim))},
    {"cem_step", 2, true, SIMV(s.lib().cem_step(sim, (long)a[1]))},
    {"cem_energy", 1, false, SIM(return s.lib().cem_energy(sim))},
    {"cem_nfreq", 1, false, SIM(return s.lib().cem_nfreq(sim))},
    {"cem_port_v", 2, false, [](Shim &s, const double *a) -> double {
         return spectrum(s, a, 0, [](const Lib &l, cem_sim *x, int p) { return l.cem_port_v(x, p); });
     }},
    {"cem_port_i", 2, false, [](Shim &s, const double *a) -> double {
         return spectrum(s, a, 1, [](const Lib &l, cem_sim *x, int p) { return l.cem_port_i(x, p); });
     }},
    {"cem_source_spectrum", 1, false, [](Shim &s, const double *a) -> double {
         return spectrum(s, a, 4, [](const Lib &l, cem_sim *x, int) { return l.cem_source_spectrum(x); });
     }},
    {"cem_vprobe", 2, false, [](Shim &s, const double *a) -> double {
         return spectrum(s, a, 2, [](const Lib &l, cem_sim *x, int p) { return l.cem_vprobe(x, p); });
     }},
    {"cem_iprobe", 2, false, [](Shim &s, const double *a) -> double {
         return spectrum(s, a, 3, [](const Lib &l, cem_sim *x, int p) { return l.cem_iprobe(x, p); });
     }},
    {"cem_add_mode_port_args", 19, false,
     SIM(return s.lib().cem_add_mode_port_args(sim, I(a, 1), I(a, 2), I(a, 3), I(a, 4), I(a, 5), I(a, 6), I(a, 7), I(a, 8),
                                              I(a, 9), I(a, 10), I(a, 11), I(a, 12), I(a, 13), I(a, 14), I(a, 15), a[16],
                                              a[17], a[18]))},
    {"cem_set_mode_excitation", 4, false, SIM(return s.lib().cem_set_mode_excitation(sim, I(a, 1), a[2], a[3]))},
    {"cem_mode_port_waves", 6, false,
     SIM(return s.lib().cem_mode_port_waves(sim, I(a, 1), P(s, a, 2), P(s, a, 3), P(s, a, 4), P(s, a, 5)))},
    {"cem_set_debye_poles", 3, false, SIM(return s.lib().cem_set_debye_poles(sim, I(a, 1), P(s, a, 2)))},
    {"cem_material_box_debye", 10, false,
     SIM(return s.lib().cem_material_box_debye(sim, a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], P(s, a, 9)))},
    {"cem_set_conductor_loss", 7, false,
     SIM(return s.lib().cem_set_conductor_loss(sim, a[1], I(a, 2), a[3], a[4], a[5], a[6]))},
    {"cem_conductor_fit_error", 1, false, SIM(return s.lib().cem_conductor_fit_error(sim))},
    {"cem_fit_djordjevic_sarkar", 9, false, [](Shim &s, const double *a) -> double {
         return s.lib().cem_fit_djordjevic_sarkar(a[0], a[1], a[2], a[3], a[4], I(a, 5), P(s, a, 6), P(s, a, 7), P(s, a, 8));
     }},
    {"cem_s2_renormalize", 4, true, [](Shim &s, const double *a) -> double {
         s.lib().cem_s2_renormalize(P(s, a, 0), a[1], a[2], a[3]);
         return 0;
     }},
    {"cem_plan_array", 3, false, SIM({
         const size_t n = plan_len(s, sim, I(a, 1), I(a, 2));
         return s.mirror(a[0], 10 + I(a, 1), I(a, 2), 0, s.lib().cem_plan_array(sim, I(a, 1), I(a, 2)), n, false);
     })},
    {"cem_plan_npml", 2, false, SIM(return s.lib().cem_plan_npml(sim, I(a, 1)))},
    {"cem_plan_has_pml", 1, false, SIM(return s.lib().cem_plan_has_pml(sim))},
    {"cem_plan_nport", 1, false, SIM(return s.lib().cem_plan_nport(sim))},
    {"cem_plan_nvprobe", 1, false, SIM(return s.lib().cem_plan_nvprobe(sim))},
    {"cem_plan_niprobe", 1, false, SIM(return s.lib().cem_plan_niprobe(sim))},
    {"cem_plan_ndisp", 1, false, SIM(return s.lib().cem_plan_ndisp(sim))},
    {"cem_state_len", 4, false, SIM(return (double)s.lib().cem_state_len(sim, I(a, 1), I(a, 2), I(a, 3)))},
    {"cem_plan_nsibc", 1, false, SIM(return s.lib().cem_plan_nsibc(sim))},
    {"cem_plan_port", 5, false,
     SIM(return s.lib().cem_plan_port(sim, I(a, 1), P(s, a, 2), P(s, a, 3), P(s, a, 4)))},
    {"cem_plan_vprobe", 4, false, SIM(return s.lib().cem_plan_vprobe(sim, I(a, 1), P(s, a, 2), P(s, a, 3)))},
    {"cem_plan_iprobe", 4, false, SIM(return s.lib().cem_plan_iprobe(sim, I(a, 1), P(s, a, 2), P(s, a, 3)))},
    {"cem_plan_mode_source", 3, false, SIM(return s.lib().cem_plan_mode_source(sim, P(s, a, 1), P(s, a, 2)))},
    {"cem_plan_waveforms", 5, true,
     SIMV(s.lib().cem_plan_waveforms(sim, (long)a[1], I(a, 2), P(s, a, 3), P(s, a, 4)))},
    {"cem_plan_excited_lumped", 1, false, SIM(return s.lib().cem_plan_excited_lumped(sim))},
    {"cem_push_samples", 6, true,
     SIMV(s.lib().cem_push_samples(sim, I(a, 1), P(s, a, 2), P(s, a, 3), P(s, a, 4), P(s, a, 5)))},
    {"cem_field", 2, false, SIM({
         return s.mirror(a[0], 30, I(a, 1), 0, s.lib().cem_field(sim, I(a, 1)), points(s, sim), true);
     })},
    {"cem_plan_npole", 1, false, SIM(return s.lib().cem_plan_npole(sim))},
    {"cem_plan_disp", 5, false,
     SIM(return s.lib().cem_plan_disp(sim, P(s, a, 1), P(s, a, 2), P(s, a, 3), P(s, a, 4)))},
    {"cem_plan_sibc", 7, false, SIM(return s.lib().cem_plan_sibc(sim, P(s, a, 1), P(s, a, 2), P(s, a, 3), P(s, a, 4),
                                                                 P(s, a, 5), static_cast<int *>(s.ptr(a[6]))))},
    {"cem_checkpoint_size", 1, false, SIM(return (double)s.lib().cem_checkpoint_size(sim))},
    {"cem_checkpoint_save", 2, false, SIM(return s.lib().cem_checkpoint_save(sim, P(s, a, 1)))},
    {"cem_checkpoint_load", 2, false, SIM(return s.lib().cem_checkpoint_load(sim, P(s, a, 1)))},
    {"cem_state_array", 4, false, SIM({
         const size_t n = s.lib().cem_state_len(sim, I(a, 1), I(a, 2), I(a, 3));
         return s.mirror(a[0], 40 + I(a, 1), I(a, 2), I(a, 3), s.lib().cem_state_array(sim, I(a, 1), I(a, 2), I(a, 3)), n, true);
     })},
};
#undef SIM
#undef SIMV

constexpr int kCount = (int)(sizeof kExports / sizeof kExports[0]);

}  // namespace

const std::vector<std::string> &Shim::names() {
    static const std::vector<std::string> v = [] {
        std::vector<std::string> out;
        for (const Export &e : kExports) out.push_back(e.name);
        return out;
    }();
    return v;
}

int Shim::find(const std::string &name) {
    for (int q = 0; q < kCount; q++)
        if (name == kExports[q].name) return q;
    return -1;
}

int Shim::arity(int index) { return index >= 0 && index < kCount ? kExports[index].arity : -1; }

double Shim::call(int index, const double *args, bool *undefined_result) {
    if (index < 0 || index >= kCount) throw std::invalid_argument("no such export");
    const Export &e = kExports[index];
    const double r = e.fn(*this, args);
    if (undefined_result) *undefined_result = e.void_result;
    return e.void_result ? kUndefined : r;
}

}  // namespace cnapi
