/*
 * fdtd_oracle.h - CPU f64 restatement of the reference FDTD time step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU engine is compared
 * against; nothing in the product links it. It consumes an update plan
 * exported through the courant.h plan API (cem_plan_*, cem_plan_waveforms)
 * and advances fields in double precision with the operations and order of
 * skyhoffert/CourantEM solver/src/sim.c:569-933, dispersive.c:89-112 and
 * sibc.c:256-269 (each function in fdtd_oracle.c cites its lines).
 *
 * Parity pin: driven by the reference library's own plan, this restatement
 * reproduces the reference cem_step bit for bit (tests/test_oracle_pin.py),
 * and the reference's parity scene reproduces tests/golden/parity_scene.txt.
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H

#include <stddef.h>

typedef struct orc_sim orc_sim;

/* Plan arrays are borrowed (the caller keeps them alive): ca, cb (N each,
 * per component), ide/be/ce (n+1 per axis), idh/bh/ch/d (n per axis), dd (n+1). */
orc_sim *orc_create(int nx, int ny, int nz, double dt, const double *const *ca, const double *const *cb,
                    const double *const *ide, const double *const *idh, const double *const *be,
                    const double *const *ce, const double *const *bh, const double *const *ch,
                    const double *const *d, const double *const *dd, const int *npml);
void orc_destroy(orc_sim *o);

/* frequencies (Hz) of the DFT probes */
int orc_set_frequencies(orc_sim *o, int nf, const double *f);
/* lumped port: global E indices (comp*N + q), dl*dir weights, source coefficients, R */
int orc_add_port(orc_sim *o, int n, const double *idx, const double *vw, const double *cs, double R);
int orc_add_vprobe(orc_sim *o, int n, const double *idx, const double *w);
int orc_add_iprobe(orc_sim *o, int n, const double *idx, const double *w);
/* excited mode-port source entries */
int orc_set_mode_source(orc_sim *o, int n, const double *idx, const double *w);
/* source waveforms at H times for steps 0..nsteps-1 (cem_plan_waveforms); excited = excited lumped port or -1 */
int orc_set_waveforms(orc_sim *o, long nsteps, const double *lumped, const double *mode, int excited, int has_mode);
int orc_set_disp(orc_sim *o, int nd, int npole, const double *idx, const double *cb, const double *beta,
                 const double *k);
int orc_set_sibc(orc_sim *o, int ns, int nterm, const double *idx, const double *hidx, const double *hw,
                 const double *c, const double *e);

void orc_step(orc_sim *o, long n);
long orc_step_count(const orc_sim *o);
double orc_energy(const orc_sim *o);

/* comp 0..5 = Ex..Hz, N doubles, writable (initial conditions) */
double *orc_field(orc_sim *o, int comp);
/* interleaved re/im, 2*nf */
const double *orc_port_v(const orc_sim *o, int p);
const double *orc_port_i(const orc_sim *o, int p);
const double *orc_vprobe(const orc_sim *o, int p);
const double *orc_iprobe(const orc_sim *o, int p);
const double *orc_source_spectrum(const orc_sim *o);
const char *orc_last_error(void);

#endif
