/*
 * courant.h - flat C ABI of the Courant EM FDTD core, served by libcourant_b200.
 *
 * Every declaration below has the same name, argument list and meaning as the
 * reference header of skyhoffert/CourantEM (solver/include/courant.h); the line
 * cited beside each group is the reference declaration it stands in for, so a
 * program written against the reference links against libcourant_b200 with
 * only its link line changed.
 *
 * What differs is underneath: the geometry, materials and update coefficients
 * are built in FP64 on the host exactly as the reference builds them, and the
 * time loop (H/E updates with CPML, Debye currents, surface impedance, sources
 * and the DFT probes) runs on an NVIDIA B200 in hand-written CUDA. Fields and
 * auxiliary states are FP32 on the device; the DFT accumulators are FP64.
 *
 * Grid: cell (i,j,k) spans [x_i,x_i+1] x [y_j,y_j+1] x [z_k,z_k+1];
 *   Ex(i+1/2,j,k) Ey(i,j+1/2,k) Ez(i,j,k+1/2) Hx(i,j+1/2,k+1/2) Hy(i+1/2,j,k+1/2)
 *   Hz(i+1/2,j+1/2,k); every component is addressed by its integer parts in an
 *   (nx+1)(ny+1)(nz+1) array with k fastest (reference courant.h:8-12).
 *
 * Host pointers returned by cem_field, cem_port_v, cem_vprobe, ... stay valid
 * until cem_destroy. Once such a pointer has been handed out, every call that
 * advances the simulation refreshes the memory behind it before returning, and
 * values written into a field pointer are taken up by the next step.
 *
 * Errors: functions returning int give -1 and set cem_last_error(); device
 * failures inside void functions (cem_step) also set cem_last_error(), print
 * one line on stderr, and leave the step count unchanged.
 */
#ifndef COURANT_H
#define COURANT_H

#include <stddef.h>

#if defined(__GNUC__)
#define CEM_API __attribute__((visibility("default")))
#else
#define CEM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* physical constants (reference courant.h:33-35) */
#define CEM_C0 299792458.0
#define CEM_MU0 1.25663706212e-6
#define CEM_EPS0 8.8541878128e-12

/* axes, faces (2*axis + side), boundary kinds (reference courant.h:37-40) */
enum { CEM_X = 0, CEM_Y = 1, CEM_Z = 2 };
enum { CEM_XLO = 0, CEM_XHI, CEM_YLO, CEM_YHI, CEM_ZLO, CEM_ZHI };
enum { CEM_BC_PEC = 0, CEM_BC_CPML = 1 };

typedef struct cem_sim cem_sim;

/* ---- lifecycle (reference courant.h:47-49) ------------------------------ */
/* Node coordinates x[nx+1], y[ny+1], z[nz+1], strictly increasing. */
CEM_API cem_sim *cem_create(int nx, int ny, int nz, const double *x, const double *y, const double *z);
CEM_API void cem_destroy(cem_sim *s);
CEM_API const char *cem_last_error(void);

/* CPML of ncells cells on a face, or PEC (default). (reference courant.h:53) */
CEM_API int cem_set_boundary(cem_sim *s, int face, int type, int ncells);

/* ---- materials and geometry (reference courant.h:58-95) ----------------- */
CEM_API int cem_material_box(cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1,
                             double eps_r, double sigma);
CEM_API int cem_set_debye_poles(cem_sim *s, int npole, const double *f_p);
CEM_API int cem_material_box_debye(cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1,
                                   double eps_inf, double sigma, const double *deps);
CEM_API int cem_set_conductor_loss(cem_sim *s, double sigma, int rough, double p1, double p2, double fmin,
                                   double fmax);
CEM_API double cem_conductor_fit_error(const cem_sim *s);
CEM_API void cem_conductor_zs(const cem_sim *s, double f, double *re, double *im);
CEM_API double cem_fit_djordjevic_sarkar(double dk, double df, double fref, double fmin, double fmax, int npole,
                                         double *eps_inf, double *f_p, double *deps);
CEM_API int cem_pec_box(cem_sim *s, double x0, double x1, double y0, double y1, double z0, double z1);
CEM_API int cem_pec_sheet(cem_sim *s, int axis, double pos, double a0, double a1, double b0, double b1);
CEM_API int cem_pec_edges_plane(cem_sim *s, int axis, int m, const unsigned char *mask_u,
                                const unsigned char *mask_v);
CEM_API int cem_pec_cells(cem_sim *s, int i0, int j0, int k0, int ni, int nj, int nk, const unsigned char *mask);

/* ---- ports and excitation (reference courant.h:106-110) ----------------- */
CEM_API int cem_add_lumped_port(cem_sim *s, int axis, int n1, int n2, int m0, int m1, int dir, double R);
CEM_API int cem_set_gaussian(cem_sim *s, int port, double amp, double t0, double tau);

/* ---- frequency-domain probes (reference courant.h:114-122) -------------- */
CEM_API int cem_set_frequencies(cem_sim *s, int nf, const double *f);
CEM_API int cem_add_vprobe(cem_sim *s, int axis, int n1, int n2, int m0, int m1, int dir);
CEM_API int cem_add_iprobe(cem_sim *s, int axis, int m, int a0, int a1, int b0, int b1);

/* ---- running (reference courant.h:127-137) ------------------------------ */
CEM_API int cem_finalize(cem_sim *s, double courant_number);
CEM_API double cem_dt(const cem_sim *s);
CEM_API long cem_step_count(const cem_sim *s);
/* Advance n steps on the device (replaces reference sim.c:951-960). */
CEM_API void cem_step(cem_sim *s, long n);
/* Energy-decay run control (replaces reference sim.c:996-1012). */
CEM_API long cem_run(cem_sim *s, long max_steps, double decay, int check_every);
/* Field energy, an FP64 reduction on the device (replaces reference sim.c:970-994). */
CEM_API double cem_energy(const cem_sim *s);

/* ---- results: interleaved re/im, 2*nf (reference courant.h:141-148) ----- */
CEM_API int cem_nfreq(const cem_sim *s);
CEM_API const double *cem_port_v(const cem_sim *s, int port);
CEM_API const double *cem_port_i(const cem_sim *s, int port);
CEM_API const double *cem_source_spectrum(const cem_sim *s);
CEM_API const double *cem_vprobe(const cem_sim *s, int probe);
CEM_API const double *cem_iprobe(const cem_sim *s, int probe);
CEM_API double cem_port_impedance(const cem_sim *s, int port);
CEM_API int cem_excited_port(const cem_sim *s);

/* ---- raw fields: comp 0..2 = Ex,Ey,Ez, 3..5 = Hx,Hy,Hz (reference courant.h:151-153) */
CEM_API double *cem_field(cem_sim *s, int comp);
CEM_API size_t cem_index(const cem_sim *s, int i, int j, int k);
CEM_API void cem_dims(const cem_sim *s, int *nx, int *ny, int *nz);

/* ---- 2D eigenmode solver (reference courant.h:158-195) ------------------ */
typedef struct cem_mode2d cem_mode2d;
CEM_API cem_mode2d *cem_mode2d_create(int ny, int nz, const double *y, const double *z);
CEM_API void cem_mode2d_destroy(cem_mode2d *m);
CEM_API void cem_mode2d_set_media(cem_mode2d *m, const double *epsr_u, const double *epsr_v, const double *epsr_w,
                                  const unsigned char *pec_u, const unsigned char *pec_v, const unsigned char *pec_w);
CEM_API int cem_mode2d_solve(cem_mode2d *m, double f, double neff_guess, const double *start, int maxit, double tol);
CEM_API void cem_mode2d_set_debye(cem_mode2d *m, int npole, const double *f_p, const double *deps_u,
                                  const double *deps_v, const double *deps_w);
CEM_API void cem_mode2d_set_loss(cem_mode2d *m, const double *sig_u, const double *sig_v, const double *sig_w);
CEM_API void cem_mode2d_set_pml(cem_mode2d *m, int which, const double *sigma, const double *kappa,
                                const double *alpha);
CEM_API double cem_mode2d_beta(const cem_mode2d *m);
CEM_API double cem_mode2d_alpha(const cem_mode2d *m);
CEM_API const double *cem_mode2d_eu(const cem_mode2d *m);
CEM_API const double *cem_mode2d_ev(const cem_mode2d *m);
CEM_API const double *cem_mode2d_hu(const cem_mode2d *m);
CEM_API const double *cem_mode2d_hv(const cem_mode2d *m);
CEM_API double cem_mode2d_power(const cem_mode2d *m);
CEM_API double cem_mode2d_conductor_alpha(const cem_mode2d *m, double Rs);
CEM_API void cem_mode2d_vi(const cem_mode2d *m, int j0, int k0, int k1, int ja, int jb, int ka, int kb, double *V,
                           double *I);

/* ---- mode ports on x-directed lines (reference courant.h:198-229) -------- */
typedef struct {
    int dir;                 /* +1 if the device under test lies on the +x side */
    int i_src;               /* x node plane of the modal source */
    int i_mon;               /* x node plane of the monitor (V at i_mon, i_mon+1; I at cell i_mon) */
    int j0, j1, k0, k1;      /* cross-section window in y/z nodes, PEC on its edge */
    int vj, vk0, vk1, vsign; /* voltage path along z at y node vj: V = vsign * sum Ez dz */
    int ja, jb, ka, kb;      /* current loop over dual nodes (ja+1/2..jb+1/2) x (ka+1/2..kb+1/2) */
    double x_ref;            /* reference plane (m) */
    double f0;               /* frequency of the source mode profile (Hz) */
    double neff0;            /* effective index guess for the mode search */
} cem_mode_port_def;

CEM_API int cem_add_mode_port(cem_sim *s, const cem_mode_port_def *d);
CEM_API int cem_add_mode_port_args(cem_sim *s, int dir, int i_src, int i_mon, int j0, int j1, int k0, int k1, int vj,
                                   int vk0, int vk1, int vsign, int ja, int jb, int ka, int kb, double x_ref,
                                   double f0, double neff0);
CEM_API int cem_set_mode_excitation(cem_sim *s, int port, double t0, double tau);
CEM_API int cem_mode_port_waves(cem_sim *s, int port, double *a, double *b, double *z0, double *beta);
CEM_API int cem_mode_port_alpha(const cem_sim *s, int port, double *alpha);
CEM_API int cem_mode_port_alpha_c(const cem_sim *s, int port, double *alpha_c);
CEM_API void cem_s2_renormalize(double *S, double z1, double z2, double zref);

/* ---- update plan for external steppers (reference courant.h:232-251) ---- */
CEM_API const double *cem_plan_array(const cem_sim *s, int which, int comp);
CEM_API int cem_plan_npml(const cem_sim *s, int face);
CEM_API int cem_plan_has_pml(const cem_sim *s);
CEM_API int cem_plan_nport(const cem_sim *s);
CEM_API int cem_plan_nvprobe(const cem_sim *s);
CEM_API int cem_plan_niprobe(const cem_sim *s);
CEM_API int cem_plan_ndisp(const cem_sim *s);
CEM_API int cem_plan_nsibc(const cem_sim *s);
CEM_API int cem_plan_port(const cem_sim *s, int p, double *idx, double *vw, double *cs);
CEM_API int cem_plan_vprobe(const cem_sim *s, int p, double *idx, double *w);
CEM_API int cem_plan_iprobe(const cem_sim *s, int p, double *idx, double *w);
CEM_API int cem_plan_mode_source(const cem_sim *s, double *idx, double *w);
CEM_API void cem_plan_waveforms(const cem_sim *s, long n0, int n, double *lumped, double *mode);
CEM_API int cem_plan_excited_lumped(const cem_sim *s);
CEM_API int cem_plan_npole(const cem_sim *s);
CEM_API int cem_plan_disp(const cem_sim *s, double *idx, double *cb, double *beta, double *k);
CEM_API int cem_plan_sibc(const cem_sim *s, double *idx, double *hidx, double *hw, double *c, double *e, int *nterm);
CEM_API void cem_push_samples(cem_sim *s, int n, const double *ip, const double *vold, const double *vnew,
                              const double *vp);

/* ---- checkpoints (reference courant.h:255-261) --------------------------- */
CEM_API size_t cem_checkpoint_size(const cem_sim *s);
CEM_API int cem_checkpoint_save(const cem_sim *s, double *buf);
CEM_API int cem_checkpoint_load(cem_sim *s, const double *buf);
CEM_API double *cem_state_array(cem_sim *s, int which, int comp, int w);
CEM_API size_t cem_state_len(const cem_sim *s, int which, int comp, int w);

/* ---- phased stepping and misc (reference courant.h:265-277) -------------- */
/* The phases run on the device in stream order; cem_mt_H/cem_mt_E accept any
 * slab split and the result does not depend on it. */
CEM_API void cem_mt_pre(cem_sim *s);
CEM_API const char *cem_version(void);
CEM_API void cem_mt_H(cem_sim *s, int i0, int i1);
CEM_API void cem_mt_mid(cem_sim *s);
CEM_API void cem_mt_E(cem_sim *s, int i0, int i1);
CEM_API void cem_mt_post(cem_sim *s);
CEM_API void cem_set_step(cem_sim *s, long step);
CEM_API cem_mode2d *cem_cross_section_x(const cem_sim *s, int i, int j0, int j1, int k0, int k1);

#ifdef __cplusplus
}
#endif
#endif
