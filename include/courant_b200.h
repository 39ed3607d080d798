/*
 * courant_b200.h - extensions of libcourant_b200 beyond courant.h.
 *
 * These entry points have no counterpart in the reference core: they expose
 * device-side timing and sizes of a simulation for benchmarking and
 * profiling. Everything else a caller needs is in courant.h.
 */
#ifndef COURANT_B200_H
#define COURANT_B200_H

#include "courant.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Advance n steps like cem_step and report the device time they took on the
 * engine's stream (CUDA events around the launches), in milliseconds.
 * Returns 0, or -1 with cem_last_error() set. */
CEM_API int cemx_step_timed(cem_sim *s, long n, double *gpu_ms);

/* Advance n steps with a CUDA event pair around every kernel launch and
 * accumulate per-kernel device time (ms) and launch counts, in the order
 * H update, E update, surface impedance, probes, DFT fold. Arrays hold 5
 * entries. The events serialise nothing but add recording overhead, so use
 * cemx_step_timed for throughput. Returns 0 or -1. */
CEM_API int cemx_profile_steps(cem_sim *s, long n, double *kernel_ms, long *launches);

/* Sizes of a finalized simulation, n entries of:
 *   0 cells nx*ny*nz, 1 points N, 2 CPML E auxiliaries, 3 CPML H auxiliaries,
 *   4 Debye edges, 5 Debye poles, 6 surface-impedance edges, 7 their terms,
 *   8..10 coefficient-table entries of Ex/Ey/Ez (0 before the first step),
 *   11 device bytes held (0 before the first step), 12 kernel launches per step.
 * Returns 0 or -1. */
CEM_API int cemx_sizes(const cem_sim *s, long long *out, int n);

/* CUDA device on which simulations created (first stepped) afterwards by
 * this thread will live; default: the current device. Returns 0 or -1. */
CEM_API int cemx_select_device(int device);

/* Copy the time-dependent state of s to the host and release its device
 * memory; the next device operation uploads plan and state again. Returns 0
 * or -1. */
CEM_API int cemx_release_device(cem_sim *s);

/* Time-step kernel of s: 1 = the single-pass fused H+E kernel (TMA-staged),
 * 0 = separate H and E kernels (the ones the cem_mt_* phases use). Both give
 * bit-identical fields. The default is 0, or CEM_B200_FUSED=1 from the
 * environment. Returns the previous setting, or -1. */
CEM_API int cemx_use_fused(cem_sim *s, int on);

/* Wait for all device work of s. Returns 0 or -1. */
CEM_API int cemx_synchronize(cem_sim *s);

#ifdef __cplusplus
}
#endif
#endif
