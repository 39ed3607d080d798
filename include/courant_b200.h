/*
 * courant_b200.h - extensions of libcourant_b200 beyond courant.h.
 *
 * These entry points have no counterpart in the reference core: device-side
 * timing and sizes for benchmarking and profiling, device selection and
 * device-state control, the kernel choice, an energy evaluation that
 * allocates nothing, and batches of simulations advanced together. Everything
 * else a caller needs is in courant.h.
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
 *   11 device bytes held (0 before the first step), 12 kernel launches per step,
 *   13-17 point-components the update classes cover per step (H fast, H
 *   general, E fast, E general, E Debye; 0 before the first step),
 *   18 points of the Debye boxes (all three components).
 * Returns 0 or -1. */
CEM_API int cemx_sizes(const cem_sim *s, long long *out, int n);

/* CUDA device on which simulations created (first stepped) afterwards by
 * this thread will live; default: the current device. Returns 0 or -1. */
CEM_API int cemx_select_device(int device);

/* Create the device state of s now (plan tables, fields, uploads) on CUDA
 * device `device` (-1: the thread's selected or current device), instead of at
 * its first step; lets a caller move this host work off a thread that keeps
 * the GPU busy. Returns 0 or -1. */
CEM_API int cemx_prepare_device(cem_sim *s, int device);

/* Copy the time-dependent state of s to the host and release its device
 * memory; the next device operation uploads plan and state again. Returns 0
 * or -1. */
CEM_API int cemx_release_device(cem_sim *s);

/* Time-step kernel of s: 1 = the single-pass fused H+E kernel (TMA-staged),
 * 0 = separate H and E kernels (the ones the cem_mt_* phases use). Both give
 * bit-identical fields. The default is 0, or CEM_B200_FUSED=1 from the
 * environment. Returns the previous setting, or -1. */
CEM_API int cemx_use_fused(cem_sim *s, int on);

/* Launch-shape tuner (no counterpart in the reference core). With tuning on,
 * the first cem_step call of at least 2048 steps on a simulation's device
 * state chooses its launch shape - the thin-segment threshold of the update
 * kernels' thread spaces (8, 16 or 32 points), the z CPML slabs inside the
 * lean kernels' rows or as general blocks, general CPML blocks on a second
 * stream or after the others, 16, 32 or 64 steps per replayed CUDA graph - by
 * timing about 672 of those steps under each choice in turn (every choice
 * computes the same bits, so they are ordinary steps), and records the result
 * per grid shape (cells, poles, surface impedance, CPML faces) in a cache file,
 * $CEM_B200_TUNE_CACHE or ~/.cache/courant-b200/launch-shapes.txt, which later
 * simulations of the same shape read instead of measuring. Off by default, or
 * CEM_B200_TUNE=1 from the environment. Returns the previous setting, or -1. */
CEM_API int cemx_tune(cem_sim *s, int on);

/* The launch shape in use: out[0] tuned (0/1), out[1] taken from the cache,
 * out[2] thin-segment threshold, out[3] second stream (0/1), out[4] steps per
 * graph, out[5] tuned ms per step (0 if not tuned), out[6] z tails (the z
 * CPML slabs inside the lean kernels' rows, 0/1). Returns 0 or -1. */
CEM_API int cemx_tune_state(const cem_sim *s, double *out, int n);

/* Stored electromagnetic energy of s, like cem_energy (no counterpart in the
 * reference core: it replaces nothing there), computed without allocating
 * device memory. For callers that must not allocate while stepping: a
 * serving process that has handed all free HBM to simulation instances (any
 * cudaMalloc may fail there), or one that cannot accept the device-wide
 * synchronisation a cudaFree implies. cem_energy may allocate: it creates
 * the device state of a simulation that has none yet. This call uses the
 * same kernels, so it returns the same value bit for bit, but keeps its
 * block partials in one static device array per process and device (512 KiB,
 * 65536 partials, about 16.7 million grid points); nothing in it has to
 * start at zero. Every call looks up that array's address on the
 * simulation's device (cudaGetSymbolAddress; the first lookup on a device
 * loads the module there, so make a first call before any stream capture on
 * that device) and leaves the caller's current device as it found it. Calls
 * for simulations on the same device share the array and race if they
 * overlap on the GPU (serialise them across threads).
 * Fails (-1, cem_last_error() set) when s has no device state yet (step it
 * first), when field pointers handed out by cem_field are live, or when the
 * grid needs more than 65536 partials (use cem_energy). Returns 0 or -1. */
CEM_API int cemx_energy_noalloc(cem_sim *s, double *energy);

/* Batches (no counterpart in the reference core). A batch advances several
 * finalized simulations on one device together: every batched launch walks a
 * work-list of blocks across all members (H, E, surface impedance, probes),
 * and runs of 16 steps replay one CUDA graph captured per composition. Each member
 * computes the same bits as when stepped alone with cem_step. Members keep
 * their own device state, so results are read with the usual courant.h calls
 * between runs. A simulation belongs to at most one batch and must not be
 * stepped by other calls while it is a member. */
typedef struct cemx_batch cemx_batch;

/* A batch on CUDA device `device` (-1: the current device); NULL on error. */
CEM_API cemx_batch *cemx_batch_create(int device);

/* Stop and free the batch (not its members). */
CEM_API void cemx_batch_destroy(cemx_batch *b);

/* Add a finalized simulation with a budget of `steps` further steps; creates
 * its device state on the batch's device. Returns its member index or -1. */
CEM_API int cemx_batch_add(cemx_batch *b, cem_sim *s, long steps);

/* Remove a member (its state stays on the device). Returns 0 or -1. */
CEM_API int cemx_batch_remove(cemx_batch *b, cem_sim *s);

/* Steps a member still has to run, or -1 when s is not a member. */
CEM_API long cemx_batch_left(const cemx_batch *b, const cem_sim *s);

/* Advance every member by up to max_steps (each stops at its budget).
 * Returns the number of members still short of their budget, or -1. */
CEM_API int cemx_batch_run(cemx_batch *b, long max_steps);

/* on = 1: the next run picks the work-list order (member-major or plane by
 * plane across members) by timing real steps, once per batch composition per
 * process. Returns the previous setting. */
CEM_API int cemx_batch_tune(cemx_batch *b, int on);

/* Statistics of the last run, n entries of: device ms, steps, launches
 * (graph launches count once), graph length, work-list order, members.
 * Returns 0 or -1. */
CEM_API int cemx_batch_stats(const cemx_batch *b, double *out, int n);

/* Wait for all device work of s. Returns 0 or -1. */
CEM_API int cemx_synchronize(cem_sim *s);

#ifdef __cplusplus
}
#endif
#endif
