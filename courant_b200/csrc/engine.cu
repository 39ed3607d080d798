// Device time stepping for libcourant_b200 (NVIDIA B200, sm_100a).
//
// Replaces the reference time loop (skyhoffert/CourantEM solver/src/sim.c:569-960,
// dispersive.c:89-112, sibc.c:256-269, modeport.c:124-135) with four kernels
// per step, all in stream order:
//
//   k_update_h   H bulk curl fused with the CPML psi_H recursions
//   k_update_e   E bulk curl fused with the CPML psi_E recursions, PEC/sheet
//                masking, the lumped and mode sources and the Debye ADE
//                currents (correction and update in one pass per edge)
//   k_sibc       surface-impedance edges (recursive convolution), if any
//   k_post       probe/port line integrals by warp reductions into a sample
//                ring; k_dft folds the ring into FP64 DFT accumulators
//
// Layout in HBM: fields and auxiliary states are FP32, structure of arrays,
// in the reference index space q = i*si + j*sj + k (k fastest), so a warp
// reads 32 consecutive words of a (j,k) plane. Each E edge carries a 16-bit
// material index into a per-component coefficient table (ca-1, cb, source
// coefficient, Debye beta/dt per pole). Coefficients that are close to 1 are
// stored as their difference from 1 (ca-1, b-1, 1-k, 1-e) so FP32 keeps the
// decay rates accurate over tens of thousands of steps.
#include "sim.hpp"
#include "spaces.hpp"
#include "../../include/courant_b200.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <map>
#include <atomic>
#include <sys/stat.h>
#include <array>
#include <chrono>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace cb2 {

constexpr int kRing = 1024;          // sample rows kept on the device between DFT flushes
#ifndef CB2_BLOCK
#define CB2_BLOCK 128
#endif
constexpr int kBlock = CB2_BLOCK;   // threads per block of the update and SIBC kernels
constexpr int kEnergyBlock = 256;   // threads per block of the energy kernel (one partial per block)
constexpr int kMaxSlots = 2 * kMaxProbes + kMaxPorts;
constexpr int kPostThreads = 1024;   // k_post: one block
constexpr int kMaxGridY = 65535;     // launches over node planes are split into chunks of this many
constexpr int kPostStage = 4096;     // probe edge products staged in shared memory
constexpr unsigned kFlagDisp = 1, kFlagSrc = 2, kFlagMode = 4;   // table entry flags: Debye, lumped source, mode source

// ---------------------------------------------------------------- arguments

// Device index space: rows padded to 32 bytes, q = i*si + j*sj + k with
// sj = round_up(nz+1, 8) and si = (ny+1)*sj; padding elements (k > nz) stay
// zero and belong to no field component. Host copies use the reference index
// space (sj = nz+1) and are converted row by row at transfer.
struct Geom {
    int n[3];
    long long si;
    int sj, plane;
    unsigned long long sj_magic;   // j = (m * sj_magic) >> 40 for m < plane
};

struct PmlAxis {
    const int *plane_h, *plane_e;        // CPML plane of a cell / node, -1 outside
    const float *bm1_h, *cid_h;          // b-1 and c/d at cells (H auxiliaries)
    const float *bm1_e, *cid_e;          // b-1 and c/dd at nodes (E auxiliaries)
    int planes;                          // planes in the CPML slabs of this axis (cells and nodes alike)
    const int *zoff_h, *zoff_e;          // z axis: position of k in its column window, -1 outside
    int zw_h, zw_e;                      // z axis: window points per (i, j) column
};

// Device layout of the CPML auxiliaries, in the padded index space so that
// four consecutive k move as one aligned float4:
//   x slabs  plane * si + j * sj + k
//   y slabs  (i * planes + plane) * sj + k
//   z slabs  (i * (ny+1) + j) * zw + zoff[k], where each (i, j) column keeps
//            a window of whole 4-point groups covering its z slabs.
// Host copies use the reference's compact layout (sim.c:655-678) and are
// converted at transfer.

// Thread spaces of the update kernels. A space is a list of rectangles of a
// node plane: k range [ks, ke) in whole 4-point groups, rows [js, js + rows).
// One thread per 4-point group; the rectangles' threads follow one another
// (rectangle q holds threads [t0[q], t0[q + 1])), row by row within a
// rectangle, so the threads of a row are consecutive (k neighbours move by
// shuffle) and a warp mostly shares its k pattern. The k axis is cut at the z
// CPML slabs and (E) the Debye boxes, the rows at the inner edges of the y
// slabs and (E) the boxes' rows. Each update has three spaces: the fast
// rectangles (no point of any component has a CPML auxiliary on a
// derivative axis or a Debye current) and the general ones of the interior
// node planes [p0, p1), and all rectangles for the other planes.
constexpr int kMaxRects = 12;
struct Space {
    int n;
    int ks[kMaxRects], ke[kMaxRects], js[kMaxRects];
    int t0[kMaxRects + 1];                  // t0[n]: threads of the space
    unsigned long long magic[kMaxRects];    // row in its rectangle of thread t - t0: ((t - t0) * magic) >> 40
};
// E only: kDebye, the interior rectangles that meet a Debye box but no CPML
// slab (the lean Debye kernel's space; general otherwise).
constexpr int kFast = 0, kGeneral = 1, kAll = 2, kDebye = 3, kSpaces = 4;

struct StepArgs {
    Geom g;
    float *E[3], *H[3];
    const float *hc[3];      // dt/mu0 * idh per axis (cells)
    const float *ec[3];      // ide per axis (nodes)
    float dth;
    int has_pml;
    PmlAxis pml[3];
    float *psiH[3][2], *psiE[3][2];
    const unsigned short *mat[3];
    const float *tab[3];          // field-major: ca-1, cb, cs, beta_p/dt (p = 0..P-1)
    const float4 *tab4[3];        // packed per entry: ca-1, cb, cs, flags (bit pattern)
    const float4 *beta4[3];       // per entry: beta_p/dt of the P poles, nb4 float4 (zero beyond P)
    int nb4;
    int ntab[3];
    int npole;
    float omk[kMaxPoles], hk[kMaxPoles];
    float *J[3];
    int jbox[3][6];          // i0, j0, k0, ni, nj, nk of each component's Debye box
    double dt;
    double src_amp, src_t0, src_tau;   // lumped Gaussian (amp 0 when none)
    int msrc_on, i_src;
    double m_t0, m_tau;
    const float *wsrc[2];    // mode-source weights of Ey and Ez on plane i_src
    const long long *dstep;
    const float *srcv;       // lumped Vs and modal Vm at this step's H time, FP32 (source_values)
    // [H, E]: k ranges [zt[u][0], zt[u][1]) and [zt[u][2], zt[u][3]) (four-point groups) where the
    // lean kernels' rows reach into a z CPML slab and take its auxiliaries (empty: they never do)
    int zt[2][4];
    // thread spaces last: batched kernels stage the arguments before them
    Space sp[2][4];          // [H, E][kFast, kGeneral, kAll, kDebye]
    int p0[2], p1[2];        // interior node planes of H and E
};

struct SibcArgs {
    int ns, K;
    const unsigned char *ecomp;
    const unsigned *eidx;
    const uchar4 *hcomp;     // H component of each face (0..2)
    const uint4 *hidx;       // H index of each face
    const float4 *hw;        // face weights (0 beyond the face count)
    float *y;                // K * ns, term-major
    float c[kSibcTerms], ome[kSibcTerms];
    float *E[3];
    const float *H[3];
};

// buffers of one fused step: read the old, write the new
struct FusedArgs {
    const float *Eo[3], *Ho[3];
    float *En[3], *Hn[3];
    float *psiHo[3][2];   // read only
    float *psiHn[3][2];
    int *error;           // set when a bounded wait gives up
};

// TMA descriptors of the old E and H buffers of one parity (3D tiled: k, j, i)
struct TmaMaps {
    CUtensorMap e[3], h[3];
};

struct PostArgs {
    int nin;                 // input slots: nip current probes, nport ports, nvp voltage probes
    int nip, nport, nvp, nslot;
    const int *off;          // nin + 1 entry offsets
    const unsigned char *ecomp;   // 0..5
    const unsigned *eidx;
    const double *ew;
    const double *R;
    double *vold;
    int src_port;
    double src_amp, src_t0, src_tau, dt;
    int msrc_on;
    double m_t0, m_tau;
    double *ring;            // kRing * nslot
    const float *F[6];
    long long *dstep;
    float *srcv;             // source values of the step the E update runs next
    int advance;             // 1: count this step
};

// --------------------------------------------------------------- helpers

// Source waveforms, with every rounding explicit so that each kernel that
// inlines them gives the same bits.
__device__ __forceinline__ double gauss(double t, double amp, double t0, double tau) {
    const double x = __ddiv_rn(__dsub_rn(t, t0), tau);
    return __dmul_rn(amp, exp(-__dmul_rn(x, x)));
}

__device__ __forceinline__ double dgauss(double t, double t0, double tau) {
    const double x = __ddiv_rn(__dsub_rn(t, t0), tau);
    return __dmul_rn(__dmul_rn(-2.0, x), exp(-__dmul_rn(x, x)));
}

// ------------------------------------------------- per-point arithmetic
//
// The H and E updates of one point are written once, with explicit
// round-to-nearest intrinsics (no contraction left to the compiler), and
// shared by the fused step and the separate phase kernels: both give the
// same bits, as cem_step and the cem_mt_* phases do in the reference
// (sim.c:863-866).

// CPML recursion psi' = psi + (b-1) psi + (c/d) diff
__device__ __forceinline__ float psi_next(float psi, float bm1, float cid, float diff) {
    return __fmaf_rn(bm1, psi, __fmaf_rn(cid, diff, psi));
}

// Values of a (j,k) column that stay fixed while a thread marches along x:
// update coefficients and CPML plane indices (-1 outside the slabs).
struct Column {
    float hcy, hcz, ecy, ecz;
    int phj, phk, pej, pek;
};

__device__ __forceinline__ Column column_at(const StepArgs &a, int j, int k) {
    const int ny = a.g.n[1], nz = a.g.n[2];
    Column c;
    c.hcy = j < ny ? a.hc[1][j] : 0.f;
    c.hcz = k < nz ? a.hc[2][k] : 0.f;
    c.ecy = a.ec[1][j];
    c.ecz = a.ec[2][k];
    c.phj = c.phk = c.pej = c.pek = -1;
    if (a.has_pml) {
        if (j < ny) c.phj = a.pml[1].plane_h[j];
        if (k < nz) c.phk = a.pml[2].plane_h[k];
        c.pej = a.pml[1].plane_e[j];
        c.pek = a.pml[2].plane_e[k];
    }
    return c;
}

// Values of node plane i, the same for every thread of the plane.
struct Plane {
    float hcx, ecx;
    int phi, pei;
};

__device__ __forceinline__ Plane plane_at(const StepArgs &a, int i) {
    const int nx = a.g.n[0];
    Plane p;
    p.hcx = i < nx ? a.hc[0][i] : 0.f;
    p.ecx = a.ec[0][i];
    p.phi = a.has_pml && i < nx ? a.pml[0].plane_h[i] : -1;
    p.pei = a.has_pml ? a.pml[0].plane_e[i] : -1;
    return p;
}

// device index of the CPML auxiliary at (i, j, k) for derivative axis A,
// E (nodes) or H (cells); plane: the point's slab plane on axis A (x, y)
template <int A, bool E>
__device__ __forceinline__ int psi_at(const StepArgs &a, int plane, int i, int j, int k) {
    if (A == 0) return plane * (int)a.g.si + j * a.g.sj + k;
    if (A == 1) return (i * a.pml[1].planes + plane) * a.g.sj + k;
    return (i * (a.g.n[1] + 1) + j) * (E ? a.pml[2].zw_e : a.pml[2].zw_h) +
           (E ? a.pml[2].zoff_e : a.pml[2].zoff_h)[k];
}

// H component C at (i, j, k) (reference sim.c:579-606, CPML :680-754):
//   H_C -= dt/mu0 [ (d1 c1 + psi_{C,0}) - (d2 c2 + psi_{C,1}) ]
// with d1 = dE_{C+2} along axis C+1, d2 = dE_{C+1} along axis C+2, c1, c2 the
// kappa-scaled inverse cell sizes times dt/mu0. in1, in2: the point lies in
// the CPML slab of that derivative axis; s1, s2 then hold the old auxiliary
// on entry and the new one on exit.
template <int C>
__device__ __forceinline__ float h_value(const StepArgs &a, int i, int j, int k, float h, float d1, float d2,
                                         float c1, float c2, bool in1, bool in2, float &s1, float &s2) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int idx[3] = {i, j, k};
    float t1 = __fmul_rn(d1, c1), t2 = __fmul_rn(d2, c2);
    if (in1) {
        s1 = psi_next(s1, a.pml[A1].bm1_h[idx[A1]], a.pml[A1].cid_h[idx[A1]], d1);
        t1 = __fmaf_rn(a.dth, s1, t1);
    }
    if (in2) {
        s2 = psi_next(s2, a.pml[A2].bm1_h[idx[A2]], a.pml[A2].cid_h[idx[A2]], d2);
        t2 = __fmaf_rn(a.dth, s2, t2);
    }
    return __fsub_rn(h, __fsub_rn(t1, t2));
}

// h_value with the auxiliaries read from `pin` and, when STORE, written to
// `pout`; p1, p2 are the CPML planes of the two derivative axes (-1 outside).
template <int C, bool STORE>
__device__ __forceinline__ float h_comp(const StepArgs &a, float *const (&pin)[3][2], float *const (&pout)[3][2],
                                        int i, int j, int k, float h, float d1, float d2, float c1, float c2, int p1,
                                        int p2) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    int x1 = 0, x2 = 0;
    float s1 = 0.f, s2 = 0.f;
    if (p1 >= 0) { x1 = psi_at<A1, false>(a, p1, i, j, k); s1 = pin[C][0][x1]; }
    if (p2 >= 0) { x2 = psi_at<A2, false>(a, p2, i, j, k); s2 = pin[C][1][x2]; }
    const float r = h_value<C>(a, i, j, k, h, d1, d2, c1, c2, p1 >= 0, p2 >= 0, s1, s2);
    if (STORE) {
        if (p1 >= 0) pout[C][0][x1] = s1;
        if (p2 >= 0) pout[C][1][x2] = s2;
    }
    return r;
}

// All three H components at (i, j, k) for the fused step. e*: E at the point;
// *_jp, *_kp: at j+1, k+1; ey1, ez1: at i+1. h* in: old, out: new.
template <bool STORE>
__device__ __forceinline__ void h_point(const StepArgs &a, const Column &col, const Plane &pl,
                                        float *const (&pin)[3][2], float *const (&pout)[3][2], int i, int j, int k,
                                        float ex, float ey, float ez, float ez_jp, float ex_jp, float ey_kp,
                                        float ex_kp, float ey1, float ez1, float &hx, float &hy, float &hz) {
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    if (j < ny && k < nz)
        hx = h_comp<0, STORE>(a, pin, pout, i, j, k, hx, __fsub_rn(ez_jp, ez), __fsub_rn(ey_kp, ey), col.hcy, col.hcz,
                              col.phj, col.phk);
    if (k < nz && i < nx)
        hy = h_comp<1, STORE>(a, pin, pout, i, j, k, hy, __fsub_rn(ex_kp, ex), __fsub_rn(ez1, ez), col.hcz, pl.hcx,
                              col.phk, pl.phi);
    if (j < ny && i < nx)
        hz = h_comp<2, STORE>(a, pin, pout, i, j, k, hz, __fsub_rn(ey1, ey), __fsub_rn(ex_jp, ex), pl.hcx, col.hcy,
                              pl.phi, col.phj);
}

// Per-edge epilogue: material table, Debye correction, sources.
//   E = E + (ca-1) E + cb [curl - sum_p hk_p J_p] + cs Vs(t) + w Vm(t)
// t: the edge's packed table entry (ca-1, cb, cs, flags); jsum: sum_p hk_p J_p
// of the edge's Debye currents (debye_sum), used when t flags the edge
// dispersive; sv: this step's source values (source_values).
// (reference sim.c:608-637, :894-910; dispersive.c:93-104; modeport.c:130-135)
template <int C>
__device__ __forceinline__ float e_finish(const StepArgs &a, const float4 t, float e_old, float curl, int j, int k,
                                          const float2 sv, float jsum) {
    const unsigned flag = __float_as_uint(t.w);
    const float base = __fmaf_rn(t.x, e_old, e_old);
    if (!flag) return __fmaf_rn(t.y, curl, base);
    if (flag & kFlagDisp) curl = __fsub_rn(curl, jsum);
    float e = __fmaf_rn(t.y, curl, base);
    if (flag & kFlagSrc) e = __fmaf_rn(t.z, sv.x, e);
    if (C > 0 && (flag & kFlagMode)) {
        const float w = a.wsrc[C - 1][j * (a.g.n[2] + 1) + k];
        if (w != 0.f) e = __fmaf_rn(w, sv.y, e);
    }
    return e;
}

// sum_p hk_p J_p accumulated in pole order, one term at a time
__device__ __forceinline__ float debye_term(const StepArgs &a, int p, float jp, float acc) {
    return __fmaf_rn(a.hk[p], jp, acc);
}

// beta_p/dt of pole p for table entry mi of component C (packed table)
template <int C>
__device__ __forceinline__ float beta_at(const StepArgs &a, int mi, int p) {
    return __ldg(reinterpret_cast<const float *>(a.beta4[C] + mi * a.nb4) + p);
}

// Debye current update of pole p of a dispersive edge (reference
// dispersive.c:105-112): J_p += -(1-k_p) J_p + beta_p/dt (E_new - E_old),
// bidt = beta_p/dt of the edge's table entry
__device__ __forceinline__ float debye_next(const StepArgs &a, int p, float bidt, float de, float jp) {
    return __fmaf_rn(bidt, de, __fmaf_rn(-a.omk[p], jp, jp));
}

// E component C at (i, j, k) (reference sim.c:608-637, CPML :756-832):
//   E_C = ca E + cb [ (d1 c1 + psi_{C,0}) - (d2 c2 + psi_{C,1}) ] + epilogue
// with d1 = dH_{C+2} along axis C+1, d2 = dH_{C+1} along axis C+2; in1, in2,
// s1, s2 as for h_value.
template <int C>
__device__ __forceinline__ float e_value(const StepArgs &a, const float4 t, int i, int j, int k, const float2 sv,
                                         float e, float d1, float d2, float c1, float c2, bool in1, bool in2,
                                         float &s1, float &s2, float jsum) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int idx[3] = {i, j, k};
    float t1 = __fmul_rn(d1, c1), t2 = __fmul_rn(d2, c2);
    if (in1) {
        s1 = psi_next(s1, a.pml[A1].bm1_e[idx[A1]], a.pml[A1].cid_e[idx[A1]], d1);
        t1 = __fadd_rn(t1, s1);
    }
    if (in2) {
        s2 = psi_next(s2, a.pml[A2].bm1_e[idx[A2]], a.pml[A2].cid_e[idx[A2]], d2);
        t2 = __fadd_rn(t2, s2);
    }
    return e_finish<C>(a, t, e, __fsub_rn(t1, t2), j, k, sv, jsum);
}

// offset of (i, j, k) in component C's dense Debye box, -1 outside
template <int C>
__device__ __forceinline__ int jbox_at(const StepArgs &a, int i, int j, int k) {
    const int *bx = a.jbox[C];
    const int di = i - bx[0], dj = j - bx[1], dk = k - bx[2];
    if ((unsigned)di >= (unsigned)bx[3] || (unsigned)dj >= (unsigned)bx[4] || (unsigned)dk >= (unsigned)bx[5]) return -1;
    return (di * bx[4] + dj) * bx[5] + dk;
}

template <int C>
__device__ __forceinline__ int jbox_volume(const StepArgs &a) {
    return a.jbox[C][3] * a.jbox[C][4] * a.jbox[C][5];
}

// Element of pole p's current at offset o of a Debye box of `vol` points
// with P poles. CB2_JLAYOUT 0: one box-sized plane per pole; 1: the P poles
// of each four-point group side by side (one thread's currents are P
// consecutive float4).
#ifndef CB2_JLAYOUT
#define CB2_JLAYOUT 0
#endif
__host__ __device__ __forceinline__ size_t jaddr(int P, size_t vol, int p, size_t o) {
#if CB2_JLAYOUT
    (void)vol;
    return ((o >> 2) * (size_t)P + (size_t)p) * 4 + (o & 3);
#else
    (void)P;
    return (size_t)p * vol + o;
#endif
}

// E value with auxiliaries and Debye currents read and written in place
// (fused step; p1, p2: CPML planes as for h_comp; mi: table index)
template <int C, int P>
__device__ __forceinline__ float e_comp(const StepArgs &a, int i, int j, int k, const float2 sv, float e, float d1,
                                        float d2, float c1, float c2, int p1, int p2, int mi) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    int x1 = 0, x2 = 0;
    float s1 = 0.f, s2 = 0.f;
    if (p1 >= 0) { x1 = psi_at<A1, true>(a, p1, i, j, k); s1 = a.psiE[C][0][x1]; }
    if (p2 >= 0) { x2 = psi_at<A2, true>(a, p2, i, j, k); s2 = a.psiE[C][1][x2]; }
    const float4 t = __ldg(a.tab4[C] + mi);
    const bool disp = P > 0 && (__float_as_uint(t.w) & kFlagDisp);
    float jsum = 0.f;
    int jo = 0;
    const int jvol = P > 0 ? jbox_volume<C>(a) : 0;
    if (disp) {
        jo = jbox_at<C>(a, i, j, k);
#pragma unroll
        for (int p = 0; p < P; p++) jsum = debye_term(a, p, a.J[C][jaddr(P, jvol, p, jo)], jsum);
    }
    const float r = e_value<C>(a, t, i, j, k, sv, e, d1, d2, c1, c2, p1 >= 0, p2 >= 0, s1, s2, jsum);
    if (p1 >= 0) a.psiE[C][0][x1] = s1;
    if (p2 >= 0) a.psiE[C][1][x2] = s2;
    if (disp) {
        const float de = __fsub_rn(r, e);
#pragma unroll
        for (int p = 0; p < P; p++) {
            float *jp = a.J[C] + jaddr(P, jvol, p, jo);
            *jp = debye_next(a, p, beta_at<C>(a, mi, p), de, *jp);
        }
    }
    return r;
}

// All three E components at (i, j, k) for the fused step. h*: H at the point;
// *_jm, *_km: at j-1, k-1; hy_p, hz_p: at i-1. e* in: old, out: new.
template <int P>
__device__ __forceinline__ void e_point(const StepArgs &a, const Column &col, const Plane &pl, int i, int j, int k,
                                        const float2 sv, float hx, float hy, float hz, float hz_jm, float hx_jm,
                                        float hy_km, float hx_km, float hy_p, float hz_p, int m0, int m1, int m2,
                                        float &ex, float &ey, float &ez) {
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    if (i >= nx) return;
    const bool jin = j >= 1 && j < ny, kin = k >= 1 && k < nz;
    if (jin && kin)
        ex = e_comp<0, P>(a, i, j, k, sv, ex, __fsub_rn(hz, hz_jm), __fsub_rn(hy, hy_km), col.ecy, col.ecz, col.pej,
                          col.pek, m0);
    if (i < 1) return;
    if (j < ny && kin)
        ey = e_comp<1, P>(a, i, j, k, sv, ey, __fsub_rn(hx, hx_km), __fsub_rn(hz, hz_p), col.ecz, pl.ecx, col.pek,
                          pl.pei, m1);
    if (jin && k < nz)
        ez = e_comp<2, P>(a, i, j, k, sv, ez, __fsub_rn(hy, hy_p), __fsub_rn(hx, hx_jm), pl.ecx, col.ecy, pl.pei,
                          col.pej, m2);
}

// ------------------------------------------------ separate phase kernels
//
// One thread per field component and per four consecutive k points of one
// padded row (one aligned float4) of one node plane. Fields move as 16-byte
// loads and stores, material indices as 8-byte loads; the k+1 / k-1
// neighbour of the four points comes from the adjacent lane by a warp
// shuffle (the lane at the warp's edge loads it). The CPML auxiliaries and
// Debye currents of all four points are loaded before any arithmetic, so
// their latencies overlap. Points a component does not own (boundary
// tangential E, row padding) are written back unchanged.

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, const float4 &v) { *reinterpret_cast<float4 *>(p) = v; }

// values at q+1 .. q+4 from v = values at q .. q+3: the next lane's first
// element, unless this lane ends a run of consecutive points (`edge`: last
// lane of the warp or of its segment row), which loads p[4] when `need`.
// Every lane of the warp must call it.
__device__ __forceinline__ float4 next_k(const float4 &v, const float *p, bool need, bool edge) {
    float w = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (edge && need) w = __ldg(p + 4);
    return make_float4(v.y, v.z, v.w, w);
}

// values at q-1 .. q+2 (a lane that starts a run loads p[-1] when `need`)
__device__ __forceinline__ float4 prev_k(const float4 &v, const float *p, bool need, bool edge) {
    float w = __shfl_up_sync(0xffffffffu, v.w, 1);
    if (edge && need) w = __ldg(p - 1);
    return make_float4(w, v.x, v.y, v.z);
}

// Position of this thread (block b of a space): row j and first point k4 of
// its four, the k range [ks, ke) of its rectangle, whether it has work
// (`act`; a thread past the end takes the last thread's position) and whether
// the next lane holds the next four points of the same row (`cont`).
struct RowPos {
    int j, k4, ks, ke;
    bool act, cont;
};

__device__ __forceinline__ RowPos space_pos(const Space &sp, int b) {
    const int t = b * kBlock + threadIdx.x, nt = sp.t0[sp.n];
    RowPos r;
    r.act = t < nt;
    const int tc = r.act ? t : nt - 1;
    int q = 0;
    while (q + 1 < sp.n && tc >= sp.t0[q + 1]) q++;
    const int tl = tc - sp.t0[q];
    r.ks = sp.ks[q];
    r.ke = sp.ke[q];
    const int nk4 = (r.ke - r.ks) >> 2;
    const int row = (int)(((unsigned long long)tl * sp.magic[q]) >> 40);
    r.j = sp.js[q] + row;
    r.k4 = r.ks + 4 * (tl - row * nk4);
    r.cont = (threadIdx.x & 31) != 31 && r.k4 + 4 < r.ke && t + 1 < nt;
    return r;
}

template <int A>
__device__ __forceinline__ int stride_of(const StepArgs &a) {
    return A == 0 ? (int)a.g.si : (A == 1 ? a.g.sj : 1);
}

__device__ __forceinline__ float lane4(const float4 &v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

__device__ __forceinline__ void set4(float4 &v, int e, float x) {
    if (e == 0) v.x = x;
    else if (e == 1) v.y = x;
    else if (e == 2) v.z = x;
    else v.w = x;
}

__device__ __forceinline__ int lane4i(const int4 &v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// Where four points k4 .. k4+3 of row (i, j) stand for component C: the
// CPML planes of the derivative axes (x, y: the row's; z: per point), and
// whether any of them needs the general path (CPML; for E also the Debye box,
// jo4 >= 0 the points' offset in it).
struct Where {
    int pi, pj;
    int4 pk;
    int jo4;
    bool gen;
};

template <int C>
__device__ __forceinline__ Where h_where(const StepArgs &a, int i, int j, int k4) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    Where w{-1, -1, make_int4(-1, -1, -1, -1), -1, false};
    if (a.has_pml) {
        if ((A1 == 0 || A2 == 0) && i < a.g.n[0]) w.pi = a.pml[0].plane_h[i];
        if ((A1 == 1 || A2 == 1) && j < a.g.n[1]) w.pj = a.pml[1].plane_h[j];
        if (A1 == 2 || A2 == 2) w.pk = __ldg(reinterpret_cast<const int4 *>(a.pml[2].plane_h + k4));
    }
    w.gen = w.pi >= 0 || w.pj >= 0 || max(max(w.pk.x, w.pk.y), max(w.pk.z, w.pk.w)) >= 0;
    return w;
}

// H component C at points k4 .. k4+3 of row (i, j) from the E values there
// (e2 = E_{C+2}, e1 = E_{C+1}) and one step along the derivative axes (e2n
// along C+1, e1n along C+2), h the old H, w from h_where; the new H goes to
// hq.
template <int C>
__device__ __forceinline__ void h_points(const StepArgs &a, int i, int j, int k4, float *hq, const Where &w,
                                         const float4 &e2, const float4 &e2n, const float4 &e1, const float4 &e1n,
                                         float4 h) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    constexpr bool kz = A1 == 2 || A2 == 2;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    // coefficients and CPML planes of the derivative axes
    const float ci = a.hc[0][min(i, nx - 1)], cj = a.hc[1][min(j, ny - 1)];
    const float4 ck = ldg4(a.hc[2] + k4);
    const int pi = w.pi, pj = w.pj;
    const int4 pk = w.pk;
    const int pa[3] = {pi, pj, max(max(pk.x, pk.y), max(pk.z, pk.w))};
    if (!w.gen) {
        // no CPML on either derivative axis at any of the four points
        float s = 0.f;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int k = k4 + e;
            if (!(kz ? k < nz : k <= nz)) continue;
            const float c[3] = {ci, cj, lane4(ck, e)};
            set4(h, e, h_value<C>(a, i, j, k, lane4(h, e), __fsub_rn(lane4(e2n, e), lane4(e2, e)),
                                  __fsub_rn(lane4(e1n, e), lane4(e1, e)), c[A1], c[A2], false, false, s, s));
        }
        st4(hq, h);
        return;
    }
    // CPML on a derivative axis: the auxiliaries of the four points move as
    // float4 (padded layout); only points inside a slab change theirs
    const bool any1 = pa[A1] >= 0, any2 = pa[A2] >= 0;
    const int x1 = any1 ? psi_at<A1, false>(a, pa[A1], i, j, k4) : 0;
    const int x2 = any2 ? psi_at<A2, false>(a, pa[A2], i, j, k4) : 0;
    float4 s1 = any1 ? ld4(a.psiH[C][0] + x1) : z4;
    float4 s2 = any2 ? ld4(a.psiH[C][1] + x2) : z4;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = k4 + e;
        if (!(kz ? k < nz : k <= nz)) continue;
        const bool in1 = A1 == 2 ? lane4i(pk, e) >= 0 : any1;
        const bool in2 = A2 == 2 ? lane4i(pk, e) >= 0 : any2;
        float q1 = lane4(s1, e), q2 = lane4(s2, e);
        const float c[3] = {ci, cj, lane4(ck, e)};
        set4(h, e, h_value<C>(a, i, j, k, lane4(h, e), __fsub_rn(lane4(e2n, e), lane4(e2, e)),
                              __fsub_rn(lane4(e1n, e), lane4(e1, e)), c[A1], c[A2], in1, in2, q1, q2));
        set4(s1, e, q1);
        set4(s2, e, q2);
    }
    st4(hq, h);
    if (any1) st4(a.psiH[C][0] + x1, s1);
    if (any2) st4(a.psiH[C][1] + x2, s2);
}

// H component C on points k4 .. k4+3 of row (i, j) (segment [ks, ke)).
// FAST: the block lies where no point has a CPML auxiliary (short path only,
// fewer registers); the arithmetic is the same.
template <int C, bool FAST>
__device__ __forceinline__ void h_vec(const StepArgs &a, int i, const RowPos &r) {
    const int j = r.j, k4 = r.k4;
    const int m = j * a.g.sj + k4;
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    // derivative axes x and y need i < nx, j < ny (the row's own axis goes to n)
    const bool valid = r.act && (!(A1 == 0 || A2 == 0) || i < nx) && (!(A1 == 1 || A2 == 1) || j < ny);
    const Where w = valid && !FAST ? h_where<C>(a, i, j, k4) : Where{-1, -1, make_int4(-1, -1, -1, -1), -1, false};
    const bool row = valid;
    const int q = i * (int)a.g.si + m;
    const float *__restrict__ E2 = a.E[A2];
    const float *__restrict__ E1 = a.E[A1];
    float *__restrict__ H = a.H[C];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 e2 = z4, e1 = z4, h = z4, e2n = z4, e1n = z4;
    if (row) {
        e2 = ldg4(E2 + q);
        e1 = ldg4(E1 + q);
        h = ld4(H + q);
        if (A1 != 2) e2n = ldg4(E2 + q + stride_of<A1>(a));
        if (A2 != 2) e1n = ldg4(E1 + q + stride_of<A2>(a));
    }
    // the next lane holds the next four points only if it is in the same run and loaded them
    const bool nb = __shfl_down_sync(0xffffffffu, row, 1);
    const bool edge = (threadIdx.x & 31) == 31 || k4 + 4 >= r.ke || !nb;
    if (A1 == 2) e2n = next_k(e2, E2 + q, row && k4 + 4 <= nz, edge);
    if (A2 == 2) e1n = next_k(e1, E1 + q, row && k4 + 4 <= nz, edge);
    if (!row) return;
    h_points<C>(a, i, j, k4, H + q, w, e2, e2n, e1, e1n, h);
}

// e_where: as h_where for E; CPML planes of nodes, and the Debye box
template <int C, int P>
__device__ __forceinline__ Where e_where(const StepArgs &a, int i, int j, int k4) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    Where w{-1, -1, make_int4(-1, -1, -1, -1), -1, false};
    if (a.has_pml) {
        if (A1 == 0 || A2 == 0) w.pi = a.pml[0].plane_e[i];
        if (A1 == 1 || A2 == 1) w.pj = a.pml[1].plane_e[j];
        if (A1 == 2 || A2 == 2) w.pk = __ldg(reinterpret_cast<const int4 *>(a.pml[2].plane_e + k4));
    }
    // the four points' offset in the Debye box, whose k extent is aligned to
    // four points: all four are inside or all outside
    const int *bx = a.jbox[C];
    if (P > 0 && k4 >= bx[2] && k4 < bx[2] + bx[5]) w.jo4 = jbox_at<C>(a, i, j, k4);
    w.gen = w.pi >= 0 || w.pj >= 0 || max(max(w.pk.x, w.pk.y), max(w.pk.z, w.pk.w)) >= 0 || w.jo4 >= 0;
    return w;
}

// E component C at points k4 .. k4+3 of row (i, j) from the H values there
// (h2 = H_{C+2}, h1 = H_{C+1}) and one step back along the derivative axes
// (h2m along C+1, h1m along C+2), the old E ev and the material indices mv,
// w from e_where; the new E goes to eq. Points with no CPML on a derivative
// axis and outside the Debye box take a short path (sources included); the
// others update CPML auxiliaries and Debye currents, the currents of all
// four points read in one pass (sum_p hk_p J_p) and re-read from L1 for
// their update.
template <int C, int P>
__device__ __forceinline__ void e_points(const StepArgs &a, int i, int j, int k4, float *eq, const Where &w,
                                         const float4 &h2, const float4 &h2m, const float4 &h1, const float4 &h1m,
                                         float4 ev, const uint2 mv, const float2 sv) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int nz = a.g.n[2];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float ci = a.ec[0][i], cj = a.ec[1][j];
    const float4 ck = ldg4(a.ec[2] + k4);
    const int pi = w.pi, pj = w.pj;
    const int4 pk = w.pk;
    const int pa[3] = {pi, pj, max(max(pk.x, pk.y), max(pk.z, pk.w))};
    const int jo4 = w.jo4;
    const bool box = jo4 >= 0;
    const int mi[4] = {(int)(mv.x & 0xffffu), (int)(mv.x >> 16), (int)(mv.y & 0xffffu), (int)(mv.y >> 16)};
    float4 t[4];
    unsigned flags = 0;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        t[e] = __ldg(a.tab4[C] + mi[e]);   // index 0 (PEC, padding) for points E does not own
        flags |= __float_as_uint(t[e].w);
    }
    // sources (lumped and modal) need no general path: their flags are
    // handled by e_finish; dispersive edges lie inside the Debye box
    if (!w.gen) {
        float s = 0.f;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int k = k4 + e;
            if (!(C == 2 ? k < nz : (k >= 1 && k < nz))) continue;
            const float c[3] = {ci, cj, lane4(ck, e)};
            set4(ev, e, e_value<C>(a, t[e], i, j, k, sv, lane4(ev, e), __fsub_rn(lane4(h2, e), lane4(h2m, e)),
                                   __fsub_rn(lane4(h1, e), lane4(h1m, e)), c[A1], c[A2], false, false, s, s, 0.f));
        }
        st4(eq, ev);
        return;
    }
    const bool any1 = pa[A1] >= 0, any2 = pa[A2] >= 0;
    const int x1 = any1 ? psi_at<A1, true>(a, pa[A1], i, j, k4) : 0;
    const int x2 = any2 ? psi_at<A2, true>(a, pa[A2], i, j, k4) : 0;
    float4 s1 = any1 ? ld4(a.psiE[C][0] + x1) : z4;
    float4 s2 = any2 ? ld4(a.psiE[C][1] + x2) : z4;
    float jsum[4] = {0.f, 0.f, 0.f, 0.f};
    const int jvol = P > 0 ? jbox_volume<C>(a) : 0;
    // sum_p hk_p J_p of the four points (currents of points that are not
    // dispersive are never written and stay zero; their sum is unused)
    if (P > 0 && box) {
#pragma unroll
        for (int p = 0; p < (P > 0 ? P : 1); p++) {
            const float4 jp = ld4(a.J[C] + jaddr(P, jvol, p, jo4));
#pragma unroll
            for (int e = 0; e < 4; e++) jsum[e] = debye_term(a, p, lane4(jp, e), jsum[e]);
        }
    }
    float4 eo = ev;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = k4 + e;
        if (!(C == 2 ? k < nz : (k >= 1 && k < nz))) continue;
        const bool in1 = A1 == 2 ? lane4i(pk, e) >= 0 : any1;
        const bool in2 = A2 == 2 ? lane4i(pk, e) >= 0 : any2;
        float q1 = lane4(s1, e), q2 = lane4(s2, e);
        const float c[3] = {ci, cj, lane4(ck, e)};
        set4(ev, e, e_value<C>(a, t[e], i, j, k, sv, lane4(ev, e), __fsub_rn(lane4(h2, e), lane4(h2m, e)),
                               __fsub_rn(lane4(h1, e), lane4(h1m, e)), c[A1], c[A2], in1, in2, q1, q2, jsum[e]));
        set4(s1, e, q1);
        set4(s2, e, q2);
    }
    st4(eq, ev);
    if (any1) st4(a.psiE[C][0] + x1, s1);
    if (any2) st4(a.psiE[C][1] + x2, s2);
    if (P > 0 && box && (flags & kFlagDisp)) {
        bool disp[4];
        float de[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int k = k4 + e;
            disp[e] = (C == 2 ? k < nz : (k >= 1 && k < nz)) && (__float_as_uint(t[e].w) & kFlagDisp);
            de[e] = __fsub_rn(lane4(ev, e), lane4(eo, e));
        }
#pragma unroll
        for (int p = 0; p < (P > 0 ? P : 1); p++) {
            float *jp = a.J[C] + jaddr(P, jvol, p, jo4);
            float4 jv = ld4(jp);
#pragma unroll
            for (int e = 0; e < 4; e++)
                if (disp[e]) set4(jv, e, debye_next(a, p, beta_at<C>(a, mi[e], p), de[e], lane4(jv, e)));
            st4(jp, jv);
        }
    }
}

// E component C on points k4 .. k4+3 of row (i, j) (segment [ks, ke));
// FAST as for h_vec: no CPML auxiliary and no Debye current in the block.
template <int C, int P, bool FAST>
__device__ __forceinline__ void e_vec(const StepArgs &a, int i, const RowPos &r, const float2 sv) {
    const int j = r.j, k4 = r.k4;
    const int m = j * a.g.sj + k4;
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int nx = a.g.n[0], ny = a.g.n[1];
    // own axis: index < n; transverse axes: 1 <= index < n
    const bool valid = r.act && i < nx && (C == 0 || i >= 1) && (C == 1 ? j < ny : (j >= 1 && j < ny));
    const Where w = valid && !FAST ? e_where<C, P>(a, i, j, k4) : Where{-1, -1, make_int4(-1, -1, -1, -1), -1, false};
    const bool row = valid;
    const int q = i * (int)a.g.si + m;
    const float *__restrict__ H2 = a.H[A2];
    const float *__restrict__ H1 = a.H[A1];
    float *__restrict__ E = a.E[C];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 h2 = z4, h1 = z4, ev = z4, h2m = z4, h1m = z4;
    uint2 mv = make_uint2(0, 0);
    if (row) {
        h2 = ldg4(H2 + q);
        h1 = ldg4(H1 + q);
        ev = ld4(E + q);
        mv = __ldg(reinterpret_cast<const uint2 *>(a.mat[C] + q));
        if (A1 != 2) h2m = ldg4(H2 + q - stride_of<A1>(a));
        if (A2 != 2) h1m = ldg4(H1 + q - stride_of<A2>(a));
    }
    // the previous lane holds the previous four points only if it is in the same run and loaded them
    const bool pb = __shfl_up_sync(0xffffffffu, row, 1);
    const bool edge = (threadIdx.x & 31) == 0 || k4 == r.ks || !pb;
    if (A1 == 2) h2m = prev_k(h2, H2 + q, row && k4 > 0, edge);
    if (A2 == 2) h1m = prev_k(h1, H1 + q, row && k4 > 0, edge);
    if (!row) return;
    e_points<C, P>(a, i, j, k4, E + q, w, h2, h2m, h1, h1m, ev, mv, sv);
}

// whether the group at k4 of a lean kernel's row lies in a z tail (StepArgs::zt)
__device__ __forceinline__ bool in_ztail(const int (&zt)[4], int k4) {
    return (k4 >= zt[0] && k4 < zt[1]) || (k4 >= zt[2] && k4 < zt[3]);
}

// Where of a z-tail group: lean rows lie on interior planes outside the y
// slabs, so only the z planes of the four points are looked up (the x and y
// ones are -1 by construction, which the compiler sees)
__device__ __forceinline__ Where ztail_where(const int *plane_z, int k4) {
    const int4 pk = __ldg(reinterpret_cast<const int4 *>(plane_z + k4));
    return Where{-1, -1, pk, -1, max(max(pk.x, pk.y), max(pk.z, pk.w)) >= 0};
}

// H component C at points k4 .. k4+3 of row (i, j) of a fast piece: the
// short path of h_points (no auxiliaries), every rounding the same; groups of
// a z tail take h_points itself. All lanes of the warp call it (the k+1
// neighbours move by shuffle).
template <int C>
__device__ __forceinline__ void h_lean(const StepArgs &a, int i, const RowPos &p) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    constexpr bool kz = A1 == 2 || A2 == 2;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int j = p.j, k4 = p.k4;
    const bool row = p.act && (!(A1 == 0 || A2 == 0) || i < nx) && (!(A1 == 1 || A2 == 1) || j < ny);
    const int q = i * (int)a.g.si + j * a.g.sj + k4;
    const float *__restrict__ E2 = a.E[A2];
    const float *__restrict__ E1 = a.E[A1];
    float *__restrict__ H = a.H[C];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 e2 = z4, e1 = z4, h = z4, e2n = z4, e1n = z4;
    if (row) {
        e2 = ldg4(E2 + q);
        e1 = ldg4(E1 + q);
        h = ld4(H + q);
        if (A1 != 2) e2n = ldg4(E2 + q + stride_of<A1>(a));
        if (A2 != 2) e1n = ldg4(E1 + q + stride_of<A2>(a));
    }
    if (A1 == 2) e2n = next_k(e2, E2 + q, row && k4 + 4 <= nz, !p.cont);
    if (A2 == 2) e1n = next_k(e1, E1 + q, row && k4 + 4 <= nz, !p.cont);
    if (!row) return;
    if (kz && in_ztail(a.zt[0], k4)) {
        h_points<C>(a, i, j, k4, H + q, ztail_where(a.pml[2].plane_h, k4), e2, e2n, e1, e1n, h);
        return;
    }
    const float ci = __ldg(a.hc[0] + i), cj = __ldg(a.hc[1] + j);
    const float4 ck = ldg4(a.hc[2] + k4);
    float s = 0.f;
    float4 r = h;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = k4 + e;
        const float c[3] = {ci, cj, lane4(ck, e)};
        const float v = h_value<C>(a, i, j, k, lane4(h, e), __fsub_rn(lane4(e2n, e), lane4(e2, e)),
                                   __fsub_rn(lane4(e1n, e), lane4(e1, e)), c[A1], c[A2], false, false, s, s);
        if (kz ? k < nz : k <= nz) set4(r, e, v);
    }
    st4(H + q, r);
}

// E component C at points k4 .. k4+3 of row (i, j) of a fast piece: the
// short path of e_points (material table, sources; no auxiliaries, no Debye
// currents), every rounding the same; groups of a z tail take e_points itself
template <int C>
__device__ __forceinline__ void e_lean(const StepArgs &a, int i, const RowPos &p, const float2 sv) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    constexpr bool kz = A1 == 2 || A2 == 2;
    const int ny = a.g.n[1], nz = a.g.n[2];
    const int j = p.j, k4 = p.k4;
    const bool row = p.act && (C == 0 || i >= 1) && (C == 1 ? j < ny : (j >= 1 && j < ny));
    const int q = i * (int)a.g.si + j * a.g.sj + k4;
    const float *__restrict__ H2 = a.H[A2];
    const float *__restrict__ H1 = a.H[A1];
    float *__restrict__ E = a.E[C];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 h2 = z4, h1 = z4, ev = z4, h2m = z4, h1m = z4;
    uint2 mv = make_uint2(0, 0);
    if (row) {
        h2 = ldg4(H2 + q);
        h1 = ldg4(H1 + q);
        ev = ld4(E + q);
        mv = __ldg(reinterpret_cast<const uint2 *>(a.mat[C] + q));
        if (A1 != 2) h2m = ldg4(H2 + q - stride_of<A1>(a));
        if (A2 != 2) h1m = ldg4(H1 + q - stride_of<A2>(a));
    }
    // the previous lane holds the previous four points unless this lane starts a warp or a row
    const bool first = (threadIdx.x & 31) == 0 || k4 == p.ks;
    if (A1 == 2) h2m = prev_k(h2, H2 + q, row && k4 > 0, first);
    if (A2 == 2) h1m = prev_k(h1, H1 + q, row && k4 > 0, first);
    if (!row) return;
    if (kz && in_ztail(a.zt[1], k4)) {
        e_points<C, 0>(a, i, j, k4, E + q, ztail_where(a.pml[2].plane_e, k4), h2, h2m, h1, h1m, ev, mv, sv);
        return;
    }
    const float ci = __ldg(a.ec[0] + i), cj = __ldg(a.ec[1] + j);
    const float4 ck = ldg4(a.ec[2] + k4);
    const int mi[4] = {(int)(mv.x & 0xffffu), (int)(mv.x >> 16), (int)(mv.y & 0xffffu), (int)(mv.y >> 16)};
    float s = 0.f;
    float4 r = ev;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = k4 + e;
        const float4 t = __ldg(a.tab4[C] + mi[e]);
        const float c[3] = {ci, cj, lane4(ck, e)};
        const float v = e_value<C>(a, t, i, j, k, sv, lane4(ev, e), __fsub_rn(lane4(h2, e), lane4(h2m, e)),
                                   __fsub_rn(lane4(h1, e), lane4(h1m, e)), c[A1], c[A2], false, false, s, s, 0.f);
        if (C == 2 ? k < nz : (k >= 1 && k < nz)) set4(r, e, v);
    }
    st4(E + q, r);
}

// E component C at points k4 .. k4+3 of row (i, j) of a Debye piece: no
// CPML auxiliary on a derivative axis but the z slab of a z tail (whose
// groups take e_points), the points in or beside the component's Debye box.
// The P pole currents of the four points are read once as float4 and kept in
// registers for both sum_p hk_p J_p and their own update, then written once;
// beta_p/dt comes packed per table entry. Every rounding is that of e_points.
template <int C, int P>
__device__ __forceinline__ void e_debye(const StepArgs &a, int i, const RowPos &p, const float2 sv) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    constexpr int NB = (P + 3) / 4;
    const int ny = a.g.n[1], nz = a.g.n[2];
    const int j = p.j, k4 = p.k4;
    const bool row = p.act && (C == 0 || i >= 1) && (C == 1 ? j < ny : (j >= 1 && j < ny));
    const int q = i * (int)a.g.si + j * a.g.sj + k4;
    const float *__restrict__ H2 = a.H[A2];
    const float *__restrict__ H1 = a.H[A1];
    float *__restrict__ E = a.E[C];
    float *__restrict__ Jc = a.J[C];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 h2 = z4, h1 = z4, ev = z4, h2m = z4, h1m = z4;
    uint2 mv = make_uint2(0, 0);
    // the four points' offset in the Debye box (k extent aligned to four: all in or all out)
    const int *bx = a.jbox[C];
    const int jo4 = row && k4 >= bx[2] && k4 < bx[2] + bx[5] ? jbox_at<C>(a, i, j, k4) : -1;
    const int jvol = jbox_volume<C>(a);
    float4 J[P > 0 ? P : 1];
    if (row) {
        h2 = ldg4(H2 + q);
        h1 = ldg4(H1 + q);
        ev = ld4(E + q);
        mv = __ldg(reinterpret_cast<const uint2 *>(a.mat[C] + q));
        if (A1 != 2) h2m = ldg4(H2 + q - stride_of<A1>(a));
        if (A2 != 2) h1m = ldg4(H1 + q - stride_of<A2>(a));
    }
#pragma unroll
    for (int pp = 0; pp < P; pp++) J[pp] = jo4 >= 0 ? ld4(Jc + jaddr(P, jvol, pp, jo4)) : z4;
    const bool first = (threadIdx.x & 31) == 0 || k4 == p.ks;
    if (A1 == 2) h2m = prev_k(h2, H2 + q, row && k4 > 0, first);
    if (A2 == 2) h1m = prev_k(h1, H1 + q, row && k4 > 0, first);
    if (!row) return;
    // a z tail above the box (tails exist only where no box reaches a z slab)
    if ((A1 == 2 || A2 == 2) && in_ztail(a.zt[1], k4)) {
        e_points<C, 0>(a, i, j, k4, E + q, ztail_where(a.pml[2].plane_e, k4), h2, h2m, h1, h1m, ev, mv, sv);
        return;
    }
    const float ci = __ldg(a.ec[0] + i), cj = __ldg(a.ec[1] + j);
    const float4 ck = ldg4(a.ec[2] + k4);
    const int mi[4] = {(int)(mv.x & 0xffffu), (int)(mv.x >> 16), (int)(mv.y & 0xffffu), (int)(mv.y >> 16)};
    float s = 0.f;
    float4 r = ev;
    float de[4];
    bool disp[4];
    bool any = false;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = k4 + e;
        const float4 t = __ldg(a.tab4[C] + mi[e]);
        float jsum = 0.f;
#pragma unroll
        for (int pp = 0; pp < P; pp++) jsum = debye_term(a, pp, lane4(J[pp], e), jsum);
        const float c[3] = {ci, cj, lane4(ck, e)};
        const float v = e_value<C>(a, t, i, j, k, sv, lane4(ev, e), __fsub_rn(lane4(h2, e), lane4(h2m, e)),
                                   __fsub_rn(lane4(h1, e), lane4(h1m, e)), c[A1], c[A2], false, false, s, s, jsum);
        const bool own = C == 2 ? k < nz : (k >= 1 && k < nz);
        if (own) set4(r, e, v);
        disp[e] = own && jo4 >= 0 && (__float_as_uint(t.w) & kFlagDisp);
        de[e] = __fsub_rn(v, lane4(ev, e));
        any = any || disp[e];
    }
    st4(E + q, r);
    if (!any) return;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        if (!disp[e]) continue;
        float b[4 * (NB > 0 ? NB : 1)];
#pragma unroll
        for (int h = 0; h < NB; h++) {
            const float4 v = __ldg(a.beta4[C] + mi[e] * NB + h);
            b[4 * h] = v.x; b[4 * h + 1] = v.y; b[4 * h + 2] = v.z; b[4 * h + 3] = v.w;
        }
#pragma unroll
        for (int pp = 0; pp < P; pp++) set4(J[pp], e, debye_next(a, pp, b[pp], de[e], lane4(J[pp], e)));
    }
#pragma unroll
    for (int pp = 0; pp < P; pp++) st4(Jc + jaddr(P, jvol, pp, jo4), J[pp]);
}

// H over node planes [i0, i0 + gridDim.y) (cem_mt_H and the unfused step)
// Resident blocks (of kBlock threads) per SM the update kernels are
// compiled for: register caps of 51 and 64 per thread for the general H and
// E kernels at the default 10 and 8 (the rarer CPML and Debye paths spill a
// little), 40 and 64 for the lean ones at 12 and 8 (the z-tail path of the
// lean kernels fits without spilling; at 16 and 10 it spills, and on the
// large board the step is 5% slower)
#ifndef CB2_H_MINBLOCKS
#define CB2_H_MINBLOCKS 10
#endif
#ifndef CB2_E_MINBLOCKS
#define CB2_E_MINBLOCKS 8
#endif

#ifndef CB2_HF_MINBLOCKS
#define CB2_HF_MINBLOCKS 12
#endif
#ifndef CB2_EF_MINBLOCKS
#define CB2_EF_MINBLOCKS 8
#endif

// H on the fast rectangles of node planes [i0, i0 + gridDim.y); block x:
// block x / 3 of the space, component x % 3
__global__ void __launch_bounds__(kBlock, CB2_HF_MINBLOCKS) k_update_h_fast(const StepArgs a, int i0) {
    const int comp = blockIdx.x % 3;
    const RowPos p = space_pos(a.sp[0][kFast], blockIdx.x / 3);
    const int i = i0 + blockIdx.y;
    if (comp == 0) h_lean<0>(a, i, p);
    else if (comp == 1) h_lean<1>(a, i, p);
    else h_lean<2>(a, i, p);
}

// E on the fast rectangles of node planes [i0, i0 + gridDim.y)
__global__ void __launch_bounds__(kBlock, CB2_EF_MINBLOCKS) k_update_e_fast(const StepArgs a, int i0) {
    const int comp = blockIdx.x % 3;
    const RowPos p = space_pos(a.sp[1][kFast], blockIdx.x / 3);
    const int i = i0 + blockIdx.y;
    const float2 sv = *reinterpret_cast<const float2 *>(a.srcv);
    if (comp == 0) e_lean<0>(a, i, p, sv);
    else if (comp == 1) e_lean<1>(a, i, p, sv);
    else e_lean<2>(a, i, p, sv);
}

#ifndef CB2_ED_MINBLOCKS
#define CB2_ED_MINBLOCKS 6
#endif

// E on the Debye rectangles of node planes [i0, i0 + gridDim.y) (P poles)
template <int P>
__global__ void __launch_bounds__(kBlock, CB2_ED_MINBLOCKS) k_update_e_debye(const StepArgs a, int i0) {
    const int comp = blockIdx.x % 3;
    const RowPos p = space_pos(a.sp[1][kDebye], blockIdx.x / 3);
    const int i = i0 + blockIdx.y;
    const float2 sv = *reinterpret_cast<const float2 *>(a.srcv);
    if (comp == 0) e_debye<0, P>(a, i, p, sv);
    else if (comp == 1) e_debye<1, P>(a, i, p, sv);
    else e_debye<2, P>(a, i, p, sv);
}

// Position in the general space of update U: the general rectangles on an
// interior node plane i, all rectangles on the others
template <int U>
__device__ __forceinline__ RowPos general_pos(const StepArgs &a, int i, int b) {
    return i >= a.p0[U] && i < a.p1[U] ? space_pos(a.sp[U][kGeneral], b) : space_pos(a.sp[U][kAll], b);
}

// Work entry of the general blocks: x node plane, y block of the plane's
// general space (component y % 3, block y / 3).
__global__ void __launch_bounds__(kBlock, CB2_H_MINBLOCKS) k_update_h(const StepArgs a, const int2 *work) {
    const int2 w = work[blockIdx.x];
    const int comp = w.y % 3;
    const RowPos r = general_pos<0>(a, w.x, w.y / 3);
    if (comp == 0) h_vec<0, false>(a, w.x, r);
    else if (comp == 1) h_vec<1, false>(a, w.x, r);
    else h_vec<2, false>(a, w.x, r);
}

// E over the general blocks (P Debye poles)
template <int P>
__global__ void __launch_bounds__(kBlock, CB2_E_MINBLOCKS) k_update_e(const StepArgs a, const int2 *work) {
    const int2 w = work[blockIdx.x];
    const int comp = w.y % 3;
    const RowPos r = general_pos<1>(a, w.x, w.y / 3);
    const float2 sv = *reinterpret_cast<const float2 *>(a.srcv);
    if (comp == 0) e_vec<0, P, false>(a, w.x, r, sv);
    else if (comp == 1) e_vec<1, P, false>(a, w.x, r, sv);
    else e_vec<2, P, false>(a, w.x, r, sv);
}

constexpr unsigned kWaitLimit = 1u << 24;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait; on timeout the error flag is set and the copies in flight
// get a second bounded wait, so the block never leaves with TMA writes pending
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int *err) {
    for (unsigned it = 0; it < kWaitLimit; it++)
        if (mbar_try(bar, parity)) return true;
    atomicExch(err, 1);
    for (unsigned it = 0; it < kWaitLimit; it++)
        if (mbar_try(bar, parity)) break;
    return false;
}

// ------------------------------------------------------- fused H + E step

// One time step in a single pass over the fields. A block owns a (j,k) tile
// of kFK x kFJ points and marches over kFX node planes along x. Per plane,
// one thread arms an mbarrier and issues TMA bulk tensor copies of E_old (the
// tile plus a one-point halo: box 40 x 10) and H_old (the tile plus the low
// halo: box 40 x 9) into shared-memory rings of three and two planes, two
// planes ahead of the arithmetic. At plane i the block computes H_new(i) on
// the tile and, redundantly, on its low halo, then E_new(i) on the tile from
// those values and H_new(i-1) kept in registers. Fields and H auxiliaries
// are read from the old buffers and written to the new ones, so the
// redundant halo work never sees a neighbour's updated values. Per step the
// fields are read once and written once: 48 bytes per cell instead of 72 for
// separate H and E passes. The x coordinate of every box starts 4 elements
// before the tile (16-byte aligned); out-of-grid elements read as zero.
constexpr int kFK = 32, kFJ = 8, kFX = 16, kFT = kFK * kFJ;
constexpr int kBX = kFK + 8;                                   // box width: k0-4 .. k0+35
constexpr int kRJ = kFJ + 2, kHJ = kFJ + 1;                    // E rows j0-1..j0+8, H rows j0-1..j0+7
constexpr int kHK = kFK + 1;                                   // H region width: k0-1 .. k0+31
constexpr int kHalo = kHK + kFJ;                               // halo H points per plane
constexpr int kEBox = kRJ * kBX * 4, kHBox = kHJ * kBX * 4;    // bytes per component box
constexpr int kEStride = (kEBox + 127) / 128 * 128, kHStride = (kHBox + 127) / 128 * 128;
constexpr int kOffE = 0;                                       // 3 slots x 3 components
constexpr int kOffH = kOffE + 9 * kEStride;                    // 2 slots x 3 components
constexpr int kOffHn = kOffH + 6 * kHStride;                   // H_new of the current plane [3][kHJ][kHK]
constexpr int kOffBar = (kOffHn + 3 * kHJ * kHK * 4 + 15) / 16 * 16;
constexpr int kFusedSmem = kOffBar + 5 * 8;
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y, int z, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <int P>
__global__ void __launch_bounds__(kFT, 3) k_step_fused(const StepArgs a, const FusedArgs f,
                                                       const __grid_constant__ TmaMaps maps) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(smem + kOffBar);   // E slots 0-2, H slots 3-4
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kFK + tx;
    const int k0 = blockIdx.x * kFK, j0 = blockIdx.y * kFJ;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int sj = a.g.sj, si = (int)a.g.si;
    const int ib = blockIdx.z * kFX, ie = min(ib + kFX, nx + 1);
    const int j = j0 + ty, k = k0 + tx;
    const bool inside = j <= ny && k <= nz;

    auto Eb = [&](int slot, int c) { return reinterpret_cast<float *>(smem + kOffE + (slot * 3 + c) * kEStride); };
    auto Hb = [&](int slot, int c) { return reinterpret_cast<float *>(smem + kOffH + (slot * 3 + c) * kHStride); };
    float *Hn = reinterpret_cast<float *>(smem + kOffHn);   // [3][kHJ][kHK]
    // Every copy issued is waited for: E planes up to e_last (E(ie) feeds H(ie-1)),
    // H planes up to ie-1. Every thread tracks the same pending and parity bits;
    // thread 0 alone issues.
    const int e_last = min(ie, nx), h_last = ie - 1;
    unsigned eph = 0, hph = 0, epend = 0, hpend = 0;   // per slot: phase parity, copy in flight
    bool ok = true;
    auto issue_e = [&](int p) {
        if (p > e_last) return;
        const int sl = p % 3;
        epend |= 1u << sl;
        if (tid != 0) return;
        unsigned long long *b = bar + sl;
        mbar_expect(b, 3 * kEBox);
        for (int c = 0; c < 3; c++) tma_load(Eb(sl, c), &maps.e[c], k0 - 4, j0 - 1, p, b);
    };
    auto issue_h = [&](int p) {
        if (p > h_last) return;
        const int sl = p % 2;
        hpend |= 1u << sl;
        if (tid != 0) return;
        unsigned long long *b = bar + 3 + sl;
        mbar_expect(b, 3 * kHBox);
        for (int c = 0; c < 3; c++) tma_load(Hb(sl, c), &maps.h[c], k0 - 4, j0 - 1, p, b);
    };
    auto wait_e = [&](int p) {
        const int sl = p % 3;
        ok &= mbar_wait(bar + sl, (eph >> sl) & 1u, f.error);
        eph ^= 1u << sl;
        epend &= ~(1u << sl);
    };
    auto wait_h = [&](int p) {
        const int sl = p % 2;
        ok &= mbar_wait(bar + 3 + sl, (hph >> sl) & 1u, f.error);
        hph ^= 1u << sl;
        hpend &= ~(1u << sl);
    };
    // after a timed-out wait: give every copy still in flight a bounded wait, then leave
    auto drain = [&]() {
        for (int sl = 0; sl < 3; sl++)
            if (epend & (1u << sl)) mbar_wait(bar + sl, (eph >> sl) & 1u, f.error);
        for (int sl = 0; sl < 2; sl++)
            if (hpend & (1u << sl)) mbar_wait(bar + 3 + sl, (hph >> sl) & 1u, f.error);
    };
    // H_new at (p, jj, kk); the E region column of kk is x = kk - k0 + 4, its row rj = jj - j0 + 1
    auto h_at = [&](const Column &col, const Plane &pl, int p, int jj, int kk, bool own, float &hx, float &hy,
                    float &hz) {
        const int rj = jj - j0 + 1, x = kk - k0 + 4;
        const float *e0 = Eb(p % 3, 0), *e1 = Eb(p % 3, 1), *e2 = Eb(p % 3, 2);
        const float *n1 = Eb((p + 1) % 3, 1), *n2 = Eb((p + 1) % 3, 2);
        const int o = rj * kBX + x;
        hx = Hb(p % 2, 0)[o]; hy = Hb(p % 2, 1)[o]; hz = Hb(p % 2, 2)[o];
        if (own)
            h_point<true>(a, col, pl, f.psiHo, f.psiHn, p, jj, kk, e0[o], e1[o], e2[o], e2[o + kBX], e0[o + kBX],
                          e1[o + 1], e0[o + 1], n1[o], n2[o], hx, hy, hz);
        else
            h_point<false>(a, col, pl, f.psiHo, f.psiHn, p, jj, kk, e0[o], e1[o], e2[o], e2[o + kBX], e0[o + kBX],
                           e1[o + 1], e0[o + 1], n1[o], n2[o], hx, hy, hz);
    };
    int hj = -1, hk = -1;
    if (tid < kHK) { hj = j0 - 1; hk = k0 - 1 + tid; }
    else if (tid < kHalo) { hj = j0 + (tid - kHK); hk = k0 - 1; }
    const bool halo = tid < kHalo && hj >= 0 && hk >= 0 && hj <= ny && hk <= nz;
    const Column col = column_at(a, min(j, ny), min(k, nz));
    const Column hcol = column_at(a, halo ? hj : 0, halo ? hk : 0);

    if (tid == 0) {
        for (int q = 0; q < 5; q++) mbar_init(bar + q);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (ib >= 1) { issue_e(ib - 1); issue_h(ib - 1); }
    issue_e(ib);
    issue_h(ib);
    issue_e(ib + 1);
    const float2 sv = *reinterpret_cast<const float2 *>(a.srcv);
    float hy_prev = 0.f, hz_prev = 0.f;
    if (ib >= 1) { wait_e(ib - 1); wait_h(ib - 1); }
    wait_e(ib);
    if (__syncthreads_or(!ok)) { drain(); return; }
    if (ib >= 1) {
        if (inside) {   // H_new(ib-1) at the own point, for the x-derivatives of E at ib
            float hx, hy, hz;
            h_at(col, plane_at(a, ib - 1), ib - 1, j, k, false, hx, hy, hz);
            hy_prev = hy;
            hz_prev = hz;
        }
        __syncthreads();   // the first copies of the loop reuse the slots of plane ib-1
    }
    for (int i = ib; i < ie; i++) {
        if (tid == 0) asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // generic reads before async writes
        issue_e(i + 2);
        issue_h(i + 1);
        const int q = i * si + j * sj + k;
        int m0 = 0, m1 = 0, m2 = 0;
        if (inside && i < nx) { m0 = a.mat[0][q]; m1 = a.mat[1][q]; m2 = a.mat[2][q]; }
        if (i < nx) wait_e(i + 1);
        wait_h(i);
        if (__syncthreads_or(!ok)) { drain(); return; }
        const Plane pl = plane_at(a, i);
        float hx = 0.f, hy = 0.f, hz = 0.f;
        if (inside) {
            h_at(col, pl, i, j, k, true, hx, hy, hz);
            const int o = (ty + 1) * kHK + tx + 1;
            Hn[o] = hx; Hn[kHJ * kHK + o] = hy; Hn[2 * kHJ * kHK + o] = hz;
            f.Hn[0][q] = hx; f.Hn[1][q] = hy; f.Hn[2][q] = hz;
        }
        if (halo) {
            float gx, gy, gz;
            h_at(hcol, pl, i, hj, hk, false, gx, gy, gz);
            const int o = (hj - j0 + 1) * kHK + (hk - k0 + 1);
            Hn[o] = gx; Hn[kHJ * kHK + o] = gy; Hn[2 * kHJ * kHK + o] = gz;
        }
        __syncthreads();
        if (inside) {
            const int x = tx + 4, o = (ty + 1) * kBX + x;
            float ex = Eb(i % 3, 0)[o], ey = Eb(i % 3, 1)[o], ez = Eb(i % 3, 2)[o];
            const int h = (ty + 1) * kHK + tx + 1;
            e_point<P>(a, col, pl, i, j, k, sv, hx, hy, hz, Hn[2 * kHJ * kHK + h - kHK], Hn[h - kHK],
                    Hn[kHJ * kHK + h - 1], Hn[h - 1], hy_prev, hz_prev, m0, m1, m2, ex, ey, ez);
            f.En[0][q] = ex; f.En[1][q] = ey; f.En[2][q] = ez;
        }
        hy_prev = hy;
        hz_prev = hz;
        __syncthreads();
    }
}

// launchers of the pole-count instantiations
using EKernel = void (*)(StepArgs, const int2 *);
using HKernel = void (*)(StepArgs, int);
using FKernel = void (*)(StepArgs, FusedArgs, TmaMaps);
#define CB2_POLES(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)
#define CB2_EK(p) k_update_e<p>,
#define CB2_FK(p) k_step_fused<p>,
#define CB2_DK(p) k_update_e_debye<p>,
const EKernel kEKernels[] = {CB2_POLES(CB2_EK)};
const FKernel kFKernels[] = {CB2_POLES(CB2_FK)};
const HKernel kEDKernels[] = {CB2_POLES(CB2_DK)};
#undef CB2_EK
#undef CB2_FK
#undef CB2_DK
#undef CB2_POLES

// ------------------------------------------------------------------- SIBC

// E = sum_k c_k (J - y_k) with y_k += (1 - e_k)(J - y_k), J from the faces' H.
// (reference sibc.c:256-269)
__device__ __forceinline__ void sibc_edge(const SibcArgs &a, int e) {
    // every load first: face tables (16-byte vectors), the convolution
    // states, then the H values of the faces
    const float4 w4 = __ldg(a.hw + e);
    const uint4 i4 = __ldg(a.hidx + e);
    const uchar4 c4 = __ldg(a.hcomp + e);
    const unsigned char ec = __ldg(a.ecomp + e);
    const unsigned ei = __ldg(a.eidx + e);
    float y[kSibcTerms];
#pragma unroll
    for (int k = 0; k < kSibcTerms; k++)
        if (k < a.K) y[k] = a.y[(long long)k * a.ns + e];
    const float w[4] = {w4.x, w4.y, w4.z, w4.w};
    const unsigned hi[4] = {i4.x, i4.y, i4.z, i4.w};
    const int hc[4] = {c4.x, c4.y, c4.z, c4.w};
    float h[4];
#pragma unroll
    for (int f = 0; f < 4; f++) h[f] = w[f] != 0.f ? __ldg(a.H[hc[f]] + hi[f]) : 0.f;
    // explicit roundings: the same bits in every kernel that inlines this
    float J = 0.f;
#pragma unroll
    for (int f = 0; f < 4; f++)
        if (w[f] != 0.f) J = __fmaf_rn(w[f], h[f], J);
    float E = 0.f;
#pragma unroll
    for (int k = 0; k < kSibcTerms; k++) {
        if (k < a.K) {
            y[k] = __fmaf_rn(a.ome[k], __fsub_rn(J, y[k]), y[k]);
            E = __fmaf_rn(a.c[k], __fsub_rn(J, y[k]), E);
        }
    }
#pragma unroll
    for (int k = 0; k < kSibcTerms; k++)
        if (k < a.K) a.y[(long long)k * a.ns + e] = y[k];
    a.E[ec][ei] = E;
}

__global__ void __launch_bounds__(kBlock) k_sibc(const SibcArgs a) {
    const int e = blockIdx.x * kBlock + threadIdx.x;
    if (e < a.ns) sibc_edge(a, e);
}

// ------------------------------------------------- probes, ports, DFT ring

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// FP32 source values the E update of step n adds: the lumped Gaussian Vs and
// the differentiated modal Gaussian Vm at the H time (n + 1/2) dt (reference
// sim.c:834-838,900-909, modeport.c:124-135). Computed once per step.
__device__ __forceinline__ void source_values(const PostArgs &a, long long n, float *out) {
    const double tH = __dmul_rn(__dadd_rn((double)n, 0.5), a.dt);
    out[0] = a.src_port >= 0 ? (float)gauss(tH, a.src_amp, a.src_t0, a.src_tau) : 0.f;
    out[1] = a.msrc_on ? (float)dgauss(tH, a.m_t0, a.m_tau) : 0.f;
}

// Line integrals of every input slot (warp per slot), then port V/I and the
// source value, written as one row of the sample ring. With advance = 0 it
// only refreshes the port voltages before the E update (vold).
__device__ __forceinline__ void post_block(const PostArgs &a) {
    __shared__ double res[kMaxSlots];
    __shared__ double val[kPostStage];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int first = a.advance ? 0 : a.nip, last = a.advance ? a.nin : a.nip + a.nport;
    // all edge products at once (their loads overlap), then per-slot sums in
    // a fixed order: lane-strided partial sums and a warp reduction
    const int e0 = a.off[first], e1 = a.off[last];
    const bool staged = e1 - e0 <= kPostStage;
    if (staged) {
        for (int e = e0 + threadIdx.x; e < e1; e += kPostThreads)
            val[e - e0] = __dmul_rn((double)a.F[a.ecomp[e]][a.eidx[e]], a.ew[e]);
        __syncthreads();
    }
    for (int s = first + warp; s < last; s += kPostThreads / 32) {
        double v = 0;
        for (int e = a.off[s] + lane; e < a.off[s + 1]; e += 32)
            v = __dadd_rn(v, staged ? val[e - e0] : __dmul_rn((double)a.F[a.ecomp[e]][a.eidx[e]], a.ew[e]));
        v = warp_sum(v);
        if (lane == 0) res[s] = v;
    }
    __syncthreads();
    const long long step = *a.dstep;
    if (!a.advance) {
        if (threadIdx.x < a.nport) a.vold[threadIdx.x] = res[a.nip + threadIdx.x];
        return;
    }
    double *row = a.ring + (long long)(step % kRing) * a.nslot;
    const double tH = __dmul_rn(__dadd_rn((double)step, 0.5), a.dt);
    const double vs = a.src_port >= 0 ? gauss(tH, a.src_amp, a.src_t0, a.src_tau) : 0.0;
    for (int s = threadIdx.x; s < a.nip; s += kPostThreads) row[s] = res[s];
    for (int p = threadIdx.x; p < a.nport; p += kPostThreads) {
        const double vnew = res[a.nip + p];
        const double V = __dmul_rn(0.5, __dadd_rn(vnew, a.vold[p]));
        a.vold[p] = vnew;
        const double I = __ddiv_rn(__dsub_rn(p == a.src_port ? vs : 0.0, V), a.R[p]);
        row[a.nip + 2 * p] = V;
        row[a.nip + 2 * p + 1] = I;
    }
    if (threadIdx.x == 0) {
        double src = a.src_port >= 0 ? vs : 0.0;
        if (a.msrc_on) src = __dadd_rn(src, dgauss(tH, a.m_t0, a.m_tau));
        row[a.nip + 2 * a.nport] = src;
    }
    for (int s = threadIdx.x; s < a.nvp; s += kPostThreads) row[a.nip + 2 * a.nport + 1 + s] = res[a.nip + a.nport + s];
    __syncthreads();
    if (threadIdx.x == 0) {
        *a.dstep = step + 1;
        source_values(a, step + 1, a.srcv);
    }
}

__global__ void __launch_bounds__(kPostThreads) k_post(const PostArgs a) { post_block(a); }

// source values for the step count held on the device (after it was set from the host)
__global__ void k_source_values(const PostArgs a) { source_values(a, *a.dstep, a.srcv); }

// acc[slot][f] += (sample * dt) e^{-j w t} for each pending row in step order,
// t the slot's sampling time: (n + 1/2) dt for H-time slots, (n + 1) dt for
// the voltage probes (reference sim.c:840-861,872-933). Adding row by row
// into the accumulator, as the reference does, makes the result independent
// of where the ring was flushed (checkpoint resume stays bit-exact).
__global__ void k_dft(const double *ring, int nslot, int first_e_slot, long long step0, int count, double dt,
                      const double *omega, int nf, double *acc) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (f >= nf) return;
    const double w = omega[f];
    const double toff = s >= first_e_slot ? 1.0 : 0.5;
    double *a = acc + (long long)s * 2 * nf + 2 * f;
    double re = a[0], im = a[1];
    for (int r = 0; r < count; r++) {
        const long long n = step0 + r;
        const double v = ring[(n % kRing) * nslot + s] * dt;
        double sn, cs;
        sincos(w * (((double)n + toff) * dt), &sn, &cs);
        re += v * cs;
        im += v * -sn;
    }
    a[0] = re;
    a[1] = im;
}

// ------------------------------------------------------- batched kernels
//
// Several simulations on one device advance together: each launch walks a
// work-list of blocks across all of them. A block stages its simulation's
// arguments in shared memory and then runs exactly the per-simulation code
// (h_vec, e_vec, sibc_edge, post_block), so every simulation computes the
// same bits alone and in a batch.

// this simulation's arguments (their first `bytes`), copied to shared memory
// by the whole block
template <class T>
__device__ __forceinline__ const T &stage_args(const T *src, unsigned *buf, int bytes = sizeof(T)) {
    static_assert(sizeof(T) % 4 == 0, "arguments copied as 4-byte words");
    const unsigned *s = reinterpret_cast<const unsigned *>(src);
    for (int q = threadIdx.x; q < bytes / 4; q += blockDim.x) buf[q] = s[q];
    __syncthreads();
    return *reinterpret_cast<const T *>(buf);
}

// the update kernels stage the arguments before the thread spaces; a thread
// reads its position from the spaces in global memory
constexpr int kStaged = (int)offsetof(StepArgs, sp);
static_assert(kStaged % 4 == 0, "staged arguments end on a 4-byte boundary");

// work entry: x simulation, y block of the plane (component = y % 3), z node plane
// A batched update block walks kPerBlock consecutive work entries (x
// member, y block of the plane incl. component, z node plane) and stages a
// member's arguments only when the member changes: the arguments before the
// thread spaces, the interior planes and the spaces it walks (the fast one,
// or the general one and the one of all rectangles), each at its own offset,
// so the buffer reads as the member's StepArgs.
constexpr int kPerBlock = 4;

template <int U, bool FAST>
__device__ __forceinline__ void stage_member(const StepArgs *args, int x, unsigned *buf) {
    __syncthreads();   // every thread is done with the previous member
    const unsigned *s = reinterpret_cast<const unsigned *>(args + x);
    for (int q = threadIdx.x; q < kStaged / 4; q += blockDim.x) buf[q] = s[q];
    constexpr int sw = (int)(sizeof(Space) / 4);
    const int c0 = FAST ? kFast : kGeneral;
    for (int c = c0; c < (FAST ? kFast + 1 : kSpaces); c++) {
        const int off = (int)((offsetof(StepArgs, sp) + (U * kSpaces + c) * sizeof(Space)) / 4);
        for (int q = threadIdx.x; q < sw; q += blockDim.x) buf[off + q] = s[off + q];
    }
    constexpr int po = (int)(offsetof(StepArgs, p0) / 4);
    if (threadIdx.x < 4) buf[po + threadIdx.x] = s[po + threadIdx.x];   // p0[2], p1[2]
    __syncthreads();
}

// FAST: the members' fast rectangles (the lean kernels' code), else their general blocks
template <bool FAST>
__global__ void __launch_bounds__(kBlock, FAST ? CB2_HF_MINBLOCKS : CB2_H_MINBLOCKS)
    k_batch_h(const StepArgs *args, const int4 *work, int n) {
    static_assert(offsetof(StepArgs, p0) % 4 == 0 && offsetof(StepArgs, p1) == offsetof(StepArgs, p0) + 8, "p0, p1");
    __shared__ unsigned buf[sizeof(StepArgs) / 4];
    const StepArgs &a = *reinterpret_cast<const StepArgs *>(buf);
    int staged = -1;
    const int e1 = min(n, (int)(blockIdx.x + 1) * kPerBlock);
    for (int e = blockIdx.x * kPerBlock; e < e1; e++) {
        const int4 w = work[e];
        if (w.x != staged) {
            stage_member<0, FAST>(args, w.x, buf);
            staged = w.x;
        }
        const RowPos r = FAST ? space_pos(a.sp[0][kFast], w.y / 3) : general_pos<0>(a, w.z, w.y / 3);
        const int comp = w.y % 3;
        if (FAST) {
            if (comp == 0) h_lean<0>(a, w.z, r);
            else if (comp == 1) h_lean<1>(a, w.z, r);
            else h_lean<2>(a, w.z, r);
        } else {
            if (comp == 0) h_vec<0, false>(a, w.z, r);
            else if (comp == 1) h_vec<1, false>(a, w.z, r);
            else h_vec<2, false>(a, w.z, r);
        }
    }
}

template <int P, bool FAST>
__global__ void __launch_bounds__(kBlock, FAST ? CB2_EF_MINBLOCKS : CB2_E_MINBLOCKS)
    k_batch_e(const StepArgs *args, const int4 *work, int n) {
    __shared__ unsigned buf[sizeof(StepArgs) / 4];
    const StepArgs &a = *reinterpret_cast<const StepArgs *>(buf);
    int staged = -1;
    const int e1 = min(n, (int)(blockIdx.x + 1) * kPerBlock);
    for (int e = blockIdx.x * kPerBlock; e < e1; e++) {
        const int4 w = work[e];
        if (w.x != staged) {
            stage_member<1, FAST>(args, w.x, buf);
            staged = w.x;
        }
        // general entries: w.w = 1 for blocks of the Debye space (general code, the same bits)
        const RowPos r = FAST ? space_pos(a.sp[1][kFast], w.y / 3)
                              : (w.w ? space_pos(a.sp[1][kDebye], w.y / 3) : general_pos<1>(a, w.z, w.y / 3));
        const float2 sv = *reinterpret_cast<const float2 *>(a.srcv);
        const int comp = w.y % 3;
        if (FAST) {
            if (comp == 0) e_lean<0>(a, w.z, r, sv);
            else if (comp == 1) e_lean<1>(a, w.z, r, sv);
            else e_lean<2>(a, w.z, r, sv);
        } else {
            if (comp == 0) e_vec<0, P, false>(a, w.z, r, sv);
            else if (comp == 1) e_vec<1, P, false>(a, w.z, r, sv);
            else e_vec<2, P, false>(a, w.z, r, sv);
        }
    }
}

using BEKernel = void (*)(const StepArgs *, const int4 *, int);
#define CB2_BE(p) k_batch_e<p, false>,
const BEKernel kBEKernels[] = {CB2_BE(0) CB2_BE(1) CB2_BE(2) CB2_BE(3) CB2_BE(4) CB2_BE(5) CB2_BE(6) CB2_BE(7) CB2_BE(8)
                                   CB2_BE(9) CB2_BE(10) CB2_BE(11) CB2_BE(12) CB2_BE(13) CB2_BE(14) CB2_BE(15)
                                       CB2_BE(16)};
#undef CB2_BE

// work entry: x simulation, y first edge of the block
__global__ void __launch_bounds__(kBlock) k_batch_sibc(const SibcArgs *args, const int2 *work) {
    __shared__ unsigned buf[sizeof(SibcArgs) / 4];
    const int2 w = work[blockIdx.x];
    const SibcArgs &a = stage_args(args + w.x, buf);
    const int e = w.y + threadIdx.x;
    if (e < a.ns) sibc_edge(a, e);
}

// one block per simulation
__global__ void __launch_bounds__(kPostThreads) k_batch_post(const PostArgs *args) { post_block(args[blockIdx.x]); }

// ----------------------------------------------------------------- energy

struct EnergyArgs {
    Geom g;
    const float *F[6];
    const unsigned short *mat[3];
    const double *cb64[3];
    const double *d[3], *dd[3];
    double dt;
    double *partial;
};

// W = 1/2 sum eps E^2 dV + 1/2 sum mu0 H^2 dV with eps = dt/cb (reference sim.c:970-994)
__global__ void __launch_bounds__(kEnergyBlock) k_energy(const EnergyArgs a, int i0) {
    __shared__ double red[kEnergyBlock / 32];
    const int i = i0 + blockIdx.y;
    const int m = blockIdx.x * kEnergyBlock + threadIdx.x;
    double acc = 0;
    const int j = (int)(((unsigned long long)m * a.g.sj_magic) >> 40);
    const int k = m - j * a.g.sj;
    if (m < a.g.plane && k <= a.g.n[2]) {
        const long long q = (long long)i * a.g.si + m;
        const int idx[3] = {i, j, k};
        for (int c = 0; c < 3; c++) {
            const int ua = (c + 1) % 3, va = (c + 2) % 3;
            if (idx[c] < a.g.n[c]) {
                const double cb = a.cb64[c][a.mat[c][q]];
                if (cb != 0) {
                    const double vol = a.d[c][idx[c]] * a.dd[ua][idx[ua]] * a.dd[va][idx[va]];
                    const double e = a.F[c][q];
                    acc += 0.5 * (a.dt / cb) * e * e * vol;
                }
            }
            if (idx[ua] < a.g.n[ua] && idx[va] < a.g.n[va]) {
                const double vol = a.dd[c][idx[c]] * a.d[ua][idx[ua]] * a.d[va][idx[va]];
                const double h = a.F[3 + c][q];
                acc += 0.5 * CEM_MU0 * h * h * vol;
            }
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < kEnergyBlock / 32; w++) s += red[w];
        a.partial[(long long)i * gridDim.x + blockIdx.x] = s;
    }
}

// fixed-order sum of the block partials (deterministic)
__global__ void k_sum(const double *partial, long long n, double *out) {
    __shared__ double red[1024];
    double s = 0;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) s += partial[q];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// ------------------------------------------------------------ device state

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

struct Device {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool failed = false;
    std::string error_msg;

    Geom g{};
    size_t Np = 0;   // points in the padded device index space
    // fields and H auxiliaries are double-buffered: the fused step reads
    // buffer `cur` and writes buffer cur^1 (the other kernels work in place on cur)
    DevBuf<float> E[2][3], H[2][3];
    int cur = 0;
    bool use_fused = false;  // CEM_B200_FUSED=1 selects the single-pass H+E kernel
    DevBuf<float> hc[3], ec[3];
    DevBuf<int> plane_h[3], plane_e[3];
    DevBuf<float> bm1_h[3], cid_h[3], bm1_e[3], cid_e[3];
    DevBuf<float> psiH[2][3][2], psiE[3][2];
    size_t psi_len_h[3][2] = {}, psi_len_e[3][2] = {};   // reference (host) lengths
    size_t psi_dev_h[3][2] = {}, psi_dev_e[3][2] = {};   // device lengths
    int zplanes = 0;   // planes of the z CPML slabs (same count for cells and nodes)
    int pml_planes[3] = {0, 0, 0};
    DevBuf<int> zoff_h, zoff_e;
    int zw_h = 0, zw_e = 0;
    std::vector<int> zoff_host[2];   // H, E
    DevBuf<unsigned short> mat[3];
    DevBuf<float> tab[3];
    DevBuf<float4> tab4[3];
    DevBuf<float4> beta4[3];   // beta_p/dt per table entry, (P + 3) / 4 float4 each
    DevBuf<double> cb64[3];
    int ntab[3] = {0, 0, 0};
    DevBuf<float> J[3];
    int jbox[3][6] = {};
    // Update kernels [H, E]: thread spaces [kFast, kGeneral, kAll], the
    // interior node planes [p0, p1), and the work-list of the general blocks
    // (entries: node plane, block of the plane's general space incl.
    // component) in plane order; wl_start[u][i] is the first entry of plane i.
    Space sp[2][kSpaces]{};
    int p0[2] = {0, 0}, p1[2] = {0, 0};
    int zt[2][4] = {};       // z CPML groups the lean kernels' rows reach (StepArgs::zt)
    DevBuf<int2> wl[2];
    std::vector<int> wl_start[2];
    DevBuf<float> wsrc[2];
    // SIBC
    DevBuf<unsigned char> sb_ecomp;
    DevBuf<unsigned> sb_eidx;
    DevBuf<uchar4> sb_hcomp;
    DevBuf<uint4> sb_hidx;
    DevBuf<float4> sb_hw;
    DevBuf<float> sb_y;
    // probes
    int nip = 0, nport = 0, nvp = 0, nin = 0, nslot = 0;
    std::vector<unsigned long long> probe_e;   // (component, index) of the probes' E edges, sorted
    bool post_beside_sibc = false;             // no probe edge is a surface-impedance edge
    DevBuf<int> off;
    DevBuf<unsigned char> ecomp;
    DevBuf<unsigned> eidx;
    DevBuf<double> ew, R, vold, ring, acc, omega;
    DevBuf<long long> dstep;
    DevBuf<float> srcv;
    // energy
    DevBuf<double> d64[3], dd64[3], partial, scalar;
    // pending DFT rows [ring_first, ring_first + ring_count)
    long long ring_first = 0;
    int ring_count = 0;
    bool vold_valid = false;

    TmaMaps maps[2]{};
    DevBuf<int> error;
    StepArgs sa[2]{};
    SibcArgs sb[2]{};
    PostArgs pa[2]{};
    EnergyArgs ea[2]{};
    FusedArgs fa[2]{};

    // second stream and fork/join events: the general blocks of an update run
    // beside its fast pieces
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // runs of kGraphSteps whole steps replay one captured graph (CEM_B200_GRAPHS=0: never)
    bool use_graphs = true;
    // launch shape, chosen by the tuner per grid shape (defaults otherwise):
    // k segments thinner than `thin` points join a neighbour; general blocks on
    // the second stream beside the others (`side_on`) or after them on the main
    // one; `graph_steps` steps per replayed graph
    int thin = 16;
    bool side_on = true;
    int graph_steps = 32;
    // the z CPML slabs run inside the lean kernels' rows (z tails) or as general blocks;
    // by default tails from 2 M cells (CEM_B200_ZTAIL=0/1/2 forces): on smaller grids the lean
    // and general kernels each fit in a wave or two and run side by side, and keeping the
    // slab apart balances the two streams (121 x 62 x 40 line: 16.3 against 18.2 us per step;
    // 1498 x 1014 x 64 board: 3.21 against 3.01 ms)
    bool ztail = true;
    // z tails as rectangles of their own in the lean space (the default; CEM_B200_ZTAIL=1:
    // inside the rows' other pieces): a row's slab groups follow its other groups in the
    // same launch, but no warp mixes the two paths (lossy 2-port line: 154.5 against 165.3 us
    // per step; the large boards equal)
    bool ztail_split = true;
    // with z tails, E rows are not cut at the Debye boxes: a row that meets a box is one
    // piece of the Debye space, air and tail included (CEM_B200_ROWS=0/1)
    bool whole_rows = false;
    bool tune = false, tuned = false, tuned_from_cache = false;
    double tuned_ms = 0;
    cudaEvent_t tev[2] = {nullptr, nullptr};   // tuner timing
    cudaGraphExec_t graph = nullptr;

    ~Device() {
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t e : tev)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
};

void device_release(Device *d) { delete d; }

namespace {

// optional per-kernel timing: when set, an event pair brackets every launch
struct KernelTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    cudaStream_t stream = nullptr;
    void begin(int k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, stream);
        ev.push_back(e);
        kind.push_back(k);
    }
    void end() {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, stream);
        ev.push_back(e);
        kind.push_back(-1);
    }
};
KernelTimer *g_timer = nullptr;
thread_local int g_selected_device = -1;

inline void t_begin(int k) { if (g_timer) g_timer->begin(k); }
inline void t_end() { if (g_timer) g_timer->end(); }

bool fail(cem_sim *s, const char *what, cudaError_t e) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "CUDA %s: %s", what, cudaGetErrorString(e));
    set_error(msg);
    std::fprintf(stderr, "courant-b200: %s\n", msg);
    if (s->dev) {
        s->dev->failed = true;
        s->dev->error_msg = msg;
    }
    return false;
}

#define CB2_CHECK(s, call)                                  \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return fail((s), #call, e_); \
    } while (0)

// All copies and fills are ordered on the engine stream (a non-blocking
// stream does not synchronise with the legacy default stream).
bool h2d(cem_sim *s, void *dst, const void *src, size_t bytes) {
    if (!bytes) return true;
    CB2_CHECK(s, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->dev->stream));
    CB2_CHECK(s, cudaStreamSynchronize(s->dev->stream));   // src may be a temporary
    return true;
}

bool d2h(cem_sim *s, void *dst, const void *src, size_t bytes) {
    if (!bytes) return true;
    CB2_CHECK(s, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->dev->stream));
    CB2_CHECK(s, cudaStreamSynchronize(s->dev->stream));
    return true;
}

bool zero_dev(cem_sim *s, void *p, size_t bytes) {
    if (!bytes || !p) return true;
    CB2_CHECK(s, cudaMemsetAsync(p, 0, bytes, s->dev->stream));
    return true;
}

template <class T>
bool dev_alloc(cem_sim *s, DevBuf<T> &b, size_t n) {
    b.n = n;
    if (!n) return true;
    CB2_CHECK(s, cudaMalloc(&b.p, n * sizeof(T)));
    return true;
}

template <class T>
bool dev_upload(cem_sim *s, DevBuf<T> &b, const std::vector<T> &v) {
    if (!dev_alloc(s, b, v.size())) return false;
    return h2d(s, b.p, v.data(), v.size() * sizeof(T));
}

// length of a per-axis array of n cells / n+1 nodes, padded past round_up(n+1, 4)
size_t axis_padded(int n) { return (size_t)(n + 1 + 3) / 4 * 4 + 4; }

// reference index q -> padded device index
unsigned dev_index(const cem_sim *s, const Device &D, size_t q) {
    const size_t i = q / s->si, r = q % s->si, j = r / s->sj, k = r % s->sj;
    return (unsigned)(i * D.g.si + j * D.g.sj + k);   // < 2^31 (checked at device creation)
}

std::vector<float> to_f32(const std::vector<double> &v) {
    std::vector<float> o(v.size());
    for (size_t i = 0; i < v.size(); i++) o[i] = (float)v[i];
    return o;
}

// Material tables: deduplicate the FP32 coefficient tuples of every E edge of
// one component. Entry 0 is PEC (ca-1 = -1, cb = 0).
struct TableBuilder {
    int nf;   // fields per entry
    std::vector<float> rows;        // entry-major while building
    std::vector<unsigned char> flags;
    std::vector<double> cb64;
    std::unordered_map<std::string, int> index;
    explicit TableBuilder(int nfields) : nf(nfields) {
        std::vector<float> pec(nf, 0.f);
        pec[0] = -1.f;
        add(pec.data(), 0, 0.0);
    }
    int add(const float *row, unsigned char flag, double cb) {
        std::string key(reinterpret_cast<const char *>(row), nf * sizeof(float));
        key.push_back((char)flag);
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        const int id = (int)flags.size();
        index.emplace(std::move(key), id);
        rows.insert(rows.end(), row, row + nf);
        flags.push_back(flag);
        cb64.push_back(cb);
        return id;
    }
    std::vector<float> field_major() const {
        const size_t n = flags.size();
        std::vector<float> o(n * nf);
        for (size_t e = 0; e < n; e++)
            for (int f = 0; f < nf; f++) o[f * n + e] = rows[e * nf + f];
        return o;
    }
};

// Material tables of the three E components. Entries are
// numbered in order of first appearance along (i, j, k); a point whose
// coefficient row equals the previous point's takes its entry without a
// lookup. The lumped-source and Debye edges of a component are walked as
// sorted lists beside the grid loop (reference indices grow with it).
bool build_tables(cem_sim *s, Device &D) {
    const int P = s->npole;
    const int nfields = 3 + P;
    // per-edge extras: lumped source coefficient (excited port only), Debye beta/dt
    std::vector<std::vector<std::pair<size_t, double>>> src(3);
    if (s->src_port >= 0) {
        const LumpedPort &pt = s->port[s->src_port];
        for (size_t e = 0; e < pt.edge.size(); e++) src[pt.axis].push_back({pt.edge[e], pt.cs[e]});
    }
    std::vector<std::vector<std::pair<size_t, int>>> disp(3);
    {
        size_t count[3] = {0, 0, 0};
        for (int e = 0; e < s->ndisp; e++) count[s->d_comp[e]]++;
        for (int c = 0; c < 3; c++) disp[c].reserve(count[c]);
    }
    for (int e = 0; e < s->ndisp; e++) disp[s->d_comp[e]].push_back({s->d_idx[e], e});
    auto by_index = [](const auto &x, const auto &y) { return x.first < y.first; };
    for (int c = 0; c < 3; c++) {   // stable: of equal indices the last one counts, as a map assignment would
        std::stable_sort(src[c].begin(), src[c].end(), by_index);
        if (!std::is_sorted(disp[c].begin(), disp[c].end(), by_index))   // finalize lists them in index order
            std::stable_sort(disp[c].begin(), disp[c].end(), by_index);
    }
    // mode-source weights of Ey, Ez on the source plane (reference index j*(nz+1)+k)
    int msrc_i = -1;
    std::vector<float> wsrc[2];
    if (s->msrc >= 0) {
        const ModePort &mp = s->mport[s->msrc];
        msrc_i = mp.def.i_src;
        for (int c = 0; c < 2; c++) wsrc[c].assign((size_t)(s->n[1] + 1) * (s->n[2] + 1), 0.f);
        for (size_t e = 0; e < mp.src_idx.size(); e++)
            wsrc[mp.src_comp[e] - 1][mp.src_idx[e] % s->si] += (float)mp.src_w[e];
    }
    const int *n = s->n;
    // Each component's node planes are cut into slabs that build tables of
    // their own in parallel; the slabs' tables then merge in slab order, so
    // entries keep their numbering by first appearance along (i, j, k), and the
    // slabs' indices are renumbered.
    struct Slab {
        std::unique_ptr<TableBuilder> tb;
        int box_lo[3], box_hi[3];
        bool overflow = false;
        int i0 = 0, i1 = 0;
    };
    struct Built {
        TableBuilder tb;
        std::vector<unsigned short> mat;
        int box_lo[3], box_hi[3];
        bool overflow = false;
        explicit Built(int nf) : tb(nf) {}
    };
    std::vector<std::unique_ptr<Built>> out;
    for (int c = 0; c < 3; c++) {
        out.emplace_back(new Built(nfields));
        big_assign(out[c]->mat, (size_t)D.Np, (unsigned short)0);
    }
    const int nthreads = (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    const int nslab = std::max(1, std::min(n[0] + 1, nthreads));
    std::vector<Slab> slabs(3 * (size_t)nslab);
    auto run_parallel = [&](int ntask, auto f) {
        std::atomic<int> next{0};
        std::vector<std::thread> th;
        for (int w = 0; w < std::min(ntask, nthreads); w++)
            th.emplace_back([&] {
                for (int t = next++; t < ntask; t = next++) f(t);
            });
        for (auto &x : th) x.join();
    };
    auto build = [&](int t) {
        const int c = t / nslab, sl = t % nslab;
        Slab &b = slabs[t];
        b.tb.reset(new TableBuilder(nfields));
        TableBuilder &tb = *b.tb;
        std::vector<unsigned short> &mat = out[c]->mat;
        b.i0 = (int)((long long)(n[0] + 1) * sl / nslab);
        b.i1 = (int)((long long)(n[0] + 1) * (sl + 1) / nslab);
        std::vector<float> row(nfields), prev(nfields);
        unsigned char prev_flag = 0;
        int prev_id = -1;
        for (int a = 0; a < 3; a++) { b.box_lo[a] = n[a]; b.box_hi[a] = -1; }
        const auto &sc = src[c];
        const auto &dc = disp[c];
        const size_t q0 = idx3(s, b.i0, 0, 0);
        auto first_at = [q0](const auto &v) {
            return (size_t)(std::lower_bound(v.begin(), v.end(), q0, [](const auto &x, size_t q) { return x.first < q; }) -
                            v.begin());
        };
        size_t ss = first_at(sc), ds = first_at(dc);
        for (int i = b.i0; i < b.i1; i++)
            for (int j = 0; j <= n[1]; j++)
                for (int k = 0; k <= n[2]; k++) {
                    const int ijk[3] = {i, j, k};
                    if (ijk[c] >= n[c]) continue;
                    const size_t q = idx3(s, i, j, k);
                    const double ca = s->ca[c][q], cb = s->cb[c][q];
                    if (cb == 0 && ca == 0) continue;   // PEC: entry 0
                    std::fill(row.begin(), row.end(), 0.f);
                    row[0] = (float)(ca - 1.0);
                    row[1] = (float)cb;
                    unsigned char flag = 0;
                    while (ss < sc.size() && sc[ss].first < q) ss++;
                    if (ss < sc.size() && sc[ss].first == q) {
                        while (ss + 1 < sc.size() && sc[ss + 1].first == q) ss++;
                        row[2] = (float)sc[ss].second;
                        flag |= kFlagSrc;
                    }
                    if (c > 0 && i == msrc_i && wsrc[c - 1][(size_t)j * (n[2] + 1) + k] != 0.f) flag |= kFlagMode;
                    while (ds < dc.size() && dc[ds].first < q) ds++;
                    if (ds < dc.size() && dc[ds].first == q) {
                        while (ds + 1 < dc.size() && dc[ds + 1].first == q) ds++;
                        flag |= kFlagDisp;
                        for (int p = 0; p < P; p++)
                            row[3 + p] = (float)(s->d_beta[(size_t)p * s->ndisp + dc[ds].second] / s->dt);
                        for (int a = 0; a < 3; a++) {
                            b.box_lo[a] = std::min(b.box_lo[a], ijk[a]);
                            b.box_hi[a] = std::max(b.box_hi[a], ijk[a]);
                        }
                    }
                    int id = prev_id;
                    if (id < 0 || flag != prev_flag || std::memcmp(row.data(), prev.data(), nfields * sizeof(float))) {
                        id = tb.add(row.data(), flag, cb);
                        prev = row;
                        prev_flag = flag;
                        prev_id = id;
                    }
                    if (id > 65535) {
                        b.overflow = true;
                        return;
                    }
                    mat[(size_t)i * D.g.si + (size_t)j * D.g.sj + k] = (unsigned short)id;
                }
    };
    run_parallel(3 * nslab, build);
    // merge: the slabs' entries join each component's table in slab order
    std::vector<std::vector<int>> remap(slabs.size());
    for (int c = 0; c < 3; c++) {
        Built &b = *out[c];
        for (int a = 0; a < 3; a++) { b.box_lo[a] = n[a]; b.box_hi[a] = -1; }
        for (int sl = 0; sl < nslab && !b.overflow; sl++) {
            Slab &x = slabs[(size_t)c * nslab + sl];
            if (x.overflow) { b.overflow = true; break; }
            const TableBuilder &t = *x.tb;
            std::vector<int> &rm = remap[(size_t)c * nslab + sl];
            rm.resize(t.flags.size());
            for (size_t l = 0; l < t.flags.size(); l++) {
                rm[l] = b.tb.add(&t.rows[l * nfields], t.flags[l], t.cb64[l]);
                if (rm[l] > 65535) { b.overflow = true; break; }
            }
            for (int a = 0; a < 3; a++) {
                b.box_lo[a] = std::min(b.box_lo[a], x.box_lo[a]);
                b.box_hi[a] = std::max(b.box_hi[a], x.box_hi[a]);
            }
        }
    }
    run_parallel(3 * nslab, [&](int t) {
        const int c = t / nslab;
        if (out[c]->overflow) return;
        const Slab &x = slabs[t];
        const std::vector<int> &rm = remap[t];
        unsigned short *m = out[c]->mat.data();
        for (size_t q = (size_t)x.i0 * D.g.si; q < (size_t)x.i1 * D.g.si; q++) m[q] = (unsigned short)rm[m[q]];
    });
    for (int c = 0; c < 3; c++) {
        Built &b = *out[c];
        if (b.overflow) {
            set_error("more than 65535 distinct update coefficients on one component");
            return false;
        }
        TableBuilder &tb = b.tb;
        const int *box_lo = b.box_lo, *box_hi = b.box_hi;
        D.ntab[c] = (int)tb.flags.size();
        if (!dev_upload(s, D.mat[c], b.mat)) return false;
        if (!dev_upload(s, D.tab[c], tb.field_major())) return false;
        {
            const size_t ne = tb.flags.size();
            std::vector<float4> packed(ne);
            for (size_t e = 0; e < ne; e++) {
                unsigned fl = tb.flags[e];
                float fbits;
                std::memcpy(&fbits, &fl, 4);
                packed[e] = make_float4(tb.rows[e * nfields], tb.rows[e * nfields + 1], tb.rows[e * nfields + 2], fbits);
            }
            if (!dev_upload(s, D.tab4[c], packed)) return false;
            const int nb4 = (P + 3) / 4;
            if (nb4) {
                std::vector<float4> beta(ne * nb4, make_float4(0.f, 0.f, 0.f, 0.f));
                for (size_t e = 0; e < ne; e++)
                    for (int p = 0; p < P; p++)
                        reinterpret_cast<float *>(&beta[e * nb4])[p] = tb.rows[e * nfields + 3 + p];
                if (!dev_upload(s, D.beta4[c], beta)) return false;
            }
        }
        if (!dev_upload(s, D.cb64[c], tb.cb64)) return false;
        if (box_hi[0] >= 0) {
            for (int a = 0; a < 3; a++) {
                D.jbox[c][a] = box_lo[a];
                D.jbox[c][3 + a] = box_hi[a] - box_lo[a] + 1;
                if (a == 2) {   // k extent aligned to 4 points: the currents of four points move as a float4
                    D.jbox[c][2] = box_lo[2] / 4 * 4;
                    D.jbox[c][5] = (box_hi[2] + 1 - D.jbox[c][2] + 3) / 4 * 4;
                }
            }
            const size_t vol = (size_t)D.jbox[c][3] * D.jbox[c][4] * D.jbox[c][5];
            if (!dev_alloc(s, D.J[c], vol * P)) return false;
        }
    }
    return true;
}

bool build_pml(cem_sim *s, Device &D) {
    for (int a = 0; a < 3; a++) {
        const int n = s->n[a];
        const size_t np = axis_padded(n);   // padded so four consecutive k load as one int4
        std::vector<int> ph(np, -1), pe(np, -1);
        std::vector<float> bh(np, 0.f), chh(np, 0.f), be(np, 0.f), cee(np, 0.f);
        int r[2][2];
        pml_ranges(s, a, 0, r);
        const int lo_h = r[0][1] >= r[0][0] ? r[0][1] - r[0][0] + 1 : 0;
        for (int sd = 0; sd < 2; sd++)
            for (int i = r[sd][0]; i <= r[sd][1]; i++) ph[i] = sd == 0 ? i - r[0][0] : lo_h + (i - r[1][0]);
        pml_ranges(s, a, 1, r);
        const int lo_e = r[0][1] >= r[0][0] ? r[0][1] - r[0][0] + 1 : 0;
        for (int sd = 0; sd < 2; sd++)
            for (int i = r[sd][0]; i <= r[sd][1]; i++) pe[i] = sd == 0 ? i - r[0][0] : lo_e + (i - r[1][0]);
        for (int i = 0; i < n; i++) {
            bh[i] = (float)(s->bh[a][i] - 1.0);
            chh[i] = (float)(s->ch[a][i] * (1.0 / s->d[a][i]));
        }
        for (int i = 0; i <= n; i++) {
            be[i] = (float)(s->be[a][i] - 1.0);
            cee[i] = (float)(s->ce[a][i] * (s->dd[a][i] > 0 ? 1.0 / s->dd[a][i] : 0.0));
        }
        if (!s->has_pml) {
            std::fill(ph.begin(), ph.end(), -1);
            std::fill(pe.begin(), pe.end(), -1);
        }
        if (!dev_upload(s, D.plane_h[a], ph) || !dev_upload(s, D.plane_e[a], pe) || !dev_upload(s, D.bm1_h[a], bh) ||
            !dev_upload(s, D.cid_h[a], chh) || !dev_upload(s, D.bm1_e[a], be) || !dev_upload(s, D.cid_e[a], cee))
            return false;
    }
    for (int a = 0; a < 3; a++) {
        int r[2][2], planes = 0;
        pml_ranges(s, a, 0, r);
        for (int sd = 0; sd < 2; sd++) planes += r[sd][1] >= r[sd][0] ? r[sd][1] - r[sd][0] + 1 : 0;
        D.pml_planes[a] = s->has_pml ? planes : 0;
    }
    D.zplanes = D.pml_planes[2];
    // z windows: whole 4-point groups covering the slabs of each (i, j) column
    const int nzp = (int)axis_padded(s->n[2]);
    for (int is_e = 0; is_e < 2; is_e++) {
        std::vector<int> &zo = D.zoff_host[is_e];
        zo.assign(nzp, -1);
        int width = 0;
        if (s->has_pml) {
            int r[2][2];
            pml_ranges(s, 2, is_e, r);
            std::vector<std::pair<int, int>> win;
            for (int sd = 0; sd < 2; sd++)
                if (r[sd][1] >= r[sd][0]) win.push_back({r[sd][0] / 4 * 4, (r[sd][1] + 1 + 3) / 4 * 4});
            if (win.size() == 2 && win[1].first < win[0].second) {   // overlapping windows merge
                win[0].second = std::max(win[0].second, win[1].second);
                win.pop_back();
            }
            for (const auto &wd : win) {
                for (int k = wd.first; k < wd.second; k++) zo[k] = width + (k - wd.first);
                width += wd.second - wd.first;
            }
        }
        (is_e ? D.zw_e : D.zw_h) = width;
        if (!dev_upload(s, is_e ? D.zoff_e : D.zoff_h, zo)) return false;
    }
    const size_t nx1 = s->n[0] + 1, ny1 = s->n[1] + 1;
    for (int c = 0; c < 3; c++)
        for (int w = 0; w < 2; w++) {
            D.psi_len_h[c][w] = psi_len(s, 0, c, w);
            D.psi_len_e[c][w] = psi_len(s, 1, c, w);
            const int ax = (c + w + 1) % 3;
            size_t nh = 0, ne = 0;
            if (D.psi_len_h[c][w]) {
                if (ax == 0) nh = ne = (size_t)D.pml_planes[0] * D.g.si;
                else if (ax == 1) nh = ne = nx1 * D.pml_planes[1] * D.g.sj;
                else { nh = nx1 * ny1 * D.zw_h; ne = nx1 * ny1 * D.zw_e; }
            }
            D.psi_dev_h[c][w] = nh;
            D.psi_dev_e[c][w] = ne;
            if (!dev_alloc(s, D.psiH[0][c][w], nh + 4) || !dev_alloc(s, D.psiH[1][c][w], nh + 4) ||
                !dev_alloc(s, D.psiE[c][w], ne + 4))
                return false;
            // padding slots of the layout are read and written back unchanged: they must stay finite
            if (!zero_dev(s, D.psiH[1][c][w].p, D.psiH[1][c][w].n * 4)) return false;
        }
    return true;
}

bool build_probes(cem_sim *s, Device &D) {
    D.nip = (int)s->ip.size();
    D.nport = (int)s->port.size();
    D.nvp = (int)s->vp.size();
    D.nin = D.nip + D.nport + D.nvp;
    D.nslot = D.nip + 2 * D.nport + 1 + D.nvp;
    std::vector<int> off{0};
    std::vector<unsigned char> comp;
    std::vector<unsigned> idx;
    std::vector<double> w;
    for (const CurrentProbe &p : s->ip) {
        for (size_t e = 0; e < p.idx.size(); e++) {
            comp.push_back((unsigned char)p.comp[e]); idx.push_back(dev_index(s, D, p.idx[e])); w.push_back(p.w[e]);
        }
        off.push_back((int)idx.size());
    }
    for (const LumpedPort &p : s->port) {
        for (size_t e = 0; e < p.edge.size(); e++) {
            comp.push_back((unsigned char)p.axis); idx.push_back(dev_index(s, D, p.edge[e])); w.push_back(p.dl[e] * p.dir);
        }
        off.push_back((int)idx.size());
    }
    for (const VoltageProbe &p : s->vp) {
        for (size_t e = 0; e < p.edge.size(); e++) {
            comp.push_back((unsigned char)p.axis); idx.push_back(dev_index(s, D, p.edge[e])); w.push_back(p.dl[e]);
        }
        off.push_back((int)idx.size());
    }
    D.probe_e.clear();
    for (size_t e = 0; e < idx.size(); e++)
        if (comp[e] < 3) D.probe_e.push_back((unsigned long long)comp[e] << 32 | idx[e]);
    std::sort(D.probe_e.begin(), D.probe_e.end());
    std::vector<double> R;
    for (const LumpedPort &p : s->port) R.push_back(p.R);
    std::vector<double> omega(s->nf);
    for (int f = 0; f < s->nf; f++) omega[f] = 2 * M_PI * s->freq[f];
    if (!dev_upload(s, D.off, off) || !dev_upload(s, D.ecomp, comp) || !dev_upload(s, D.eidx, idx) ||
        !dev_upload(s, D.ew, w) || !dev_upload(s, D.R, R) || !dev_upload(s, D.omega, omega))
        return false;
    if (!dev_alloc(s, D.vold, std::max(D.nport, 1)) || !dev_alloc(s, D.ring, (size_t)kRing * D.nslot) ||
        !dev_alloc(s, D.acc, (size_t)D.nslot * 2 * s->nf) || !dev_alloc(s, D.dstep, 1) ||
        !dev_alloc(s, D.srcv, 2))
        return false;
    return true;
}

bool build_sibc(cem_sim *s, Device &D) {
    if (!s->nsb) return true;
    const size_t ns = (size_t)s->nsb;
    std::vector<unsigned char> ecomp(ns);
    std::vector<unsigned> eidx(ns);
    std::vector<uchar4> hcomp(ns);
    std::vector<uint4> hidx(ns);
    std::vector<float4> hw(ns);
    for (size_t e = 0; e < ns; e++) {
        ecomp[e] = (unsigned char)s->sb_comp[e];
        eidx[e] = dev_index(s, D, s->sb_idx[e]);
        unsigned char c[4] = {0, 0, 0, 0};
        unsigned q[4] = {0, 0, 0, 0};
        float w[4] = {0.f, 0.f, 0.f, 0.f};
        for (int f = 0; f < 4 && f < s->sb_nf[e]; f++) {
            c[f] = (unsigned char)s->sb_hc[4 * e + f];
            q[f] = dev_index(s, D, s->sb_hi[4 * e + f]);
            w[f] = (float)s->sb_sg[4 * e + f];
        }
        hcomp[e] = make_uchar4(c[0], c[1], c[2], c[3]);
        hidx[e] = make_uint4(q[0], q[1], q[2], q[3]);
        hw[e] = make_float4(w[0], w[1], w[2], w[3]);
    }
    // the probe pass may run beside the surface impedance when it reads none of its edges
    D.post_beside_sibc = true;
    for (size_t e = 0; e < ns && D.post_beside_sibc; e++)
        D.post_beside_sibc = !std::binary_search(D.probe_e.begin(), D.probe_e.end(),
                                                  (unsigned long long)ecomp[e] << 32 | eidx[e]);
    return dev_upload(s, D.sb_ecomp, ecomp) && dev_upload(s, D.sb_hcomp, hcomp) && dev_upload(s, D.sb_eidx, eidx) &&
           dev_upload(s, D.sb_hidx, hidx) && dev_upload(s, D.sb_hw, hw) &&
           dev_alloc(s, D.sb_y, ns * s->sibc_npole);
}

// blocks of a space
int space_blocks(const Space &sp) { return (sp.t0[sp.n] + kBlock - 1) / kBlock; }

// The thread spaces of update u (0 H, 1 E) and its general work-list.
// k is cut at the z CPML slabs (cells for H, nodes for E) and, for E, at the
// Debye boxes: a slab's start rounded down and its end up to a multiple of
// 4, so that the slab's k range holds every 4-point group that reaches into
// it. The rows are cut at the inner edges of the y slabs and, for E, at the
// boxes' rows. Interior planes: the longest run of node planes outside the
// x slabs. A rectangle is general when its rows reach a y slab, or (E) it
// meets a Debye box whose planes meet the interior ones, or its k range
// reaches a z slab while the z slabs are not tails (below); consecutive row
// ranges of one class and k range merge. Z tails (Device::ztail, when no such
// box reaches a z slab's k range): the z slabs make no rectangle general; the
// lean (and Debye) kernels take the slab's auxiliaries for the groups inside
// it (the general kernel's point code, the same bits). The slab's groups are
// rectangles of their own in the lean space (Device::ztail_split, cut after
// the thin merges) or pieces of the rows above the boxes.
bool build_spaces(cem_sim *s, Device &D, int u) {
    const Geom &g = D.g;
    const int nx = s->n[0], rows = s->n[1] + 1;
    const int planes = u ? nx : nx + 1;
    auto slab = [&](int a, int idx) {
        if (!s->has_pml) return false;
        int r[2][2];
        pml_ranges(s, a, u, r);
        if (idx >= s->n[a] && !u) return false;   // cells end at n-1
        for (int sd = 0; sd < 2; sd++)
            if (idx >= r[sd][0] && idx <= r[sd][1]) return true;
        return false;
    };
    int p0 = 0, p1 = 0;
    for (int i = 0; i < planes;) {
        if (slab(0, i)) { i++; continue; }
        int e = i;
        while (e < planes && !slab(0, e)) e++;
        if (e - i > p1 - p0) { p0 = i; p1 = e; }
        i = e;
    }
    // boxes whose planes meet the interior ones
    std::vector<const int *> boxes;
    for (int c = 0; u && c < 3; c++) {
        const int *bx = D.jbox[c];
        if (bx[3] * bx[4] * bx[5] > 0 && bx[0] < p1 && bx[0] + bx[3] > p0) boxes.push_back(bx);
    }
    // k groups up to the last node (nz); the row padding beyond is never touched
    const int kmax = (s->n[2] + 1 + 3) / 4 * 4;
    std::vector<int> kb{0, kmax}, jb{0, rows};
    auto kcut = [&](int c) { if (c > 0 && c < kmax) kb.push_back(c); };
    auto jcut = [&](int c) { if (c > 0 && c < rows) jb.push_back(c); };
    for (int q = 0; q < 4; q++) D.zt[u][q] = 0;
    if (s->has_pml) {
        int r[2][2];
        pml_ranges(s, 2, u, r);
        int zg[2][2] = {{0, 0}, {0, 0}};   // the slabs' group-aligned k ranges
        bool tails = D.ztail;
        for (int sd = 0; sd < 2; sd++)
            if (r[sd][1] >= r[sd][0]) {
                zg[sd][0] = r[sd][0] / 4 * 4;
                zg[sd][1] = (r[sd][1] + 1 + 3) / 4 * 4;
                for (const int *bx : boxes)
                    if (bx[2] < zg[sd][1] && bx[2] + bx[5] > zg[sd][0]) tails = false;
            }
        for (int sd = 0; sd < 2; sd++) {
            if (zg[sd][1] <= zg[sd][0]) continue;
            if (tails) { D.zt[u][2 * sd] = zg[sd][0]; D.zt[u][2 * sd + 1] = zg[sd][1]; }
            else { kcut(zg[sd][0]); kcut(zg[sd][1]); }
        }
        pml_ranges(s, 1, u, r);
        if (r[0][1] >= r[0][0]) jcut(r[0][1] + 1);
        if (r[1][1] >= r[1][0]) jcut(r[1][0]);
    }
    const bool tails = D.zt[u][1] > D.zt[u][0] || D.zt[u][3] > D.zt[u][2];
    for (const int *bx : boxes) {
        if (!(tails && D.whole_rows)) {
            kcut(bx[2] / 4 * 4);
            kcut((bx[2] + bx[5] + 3) / 4 * 4);
        }
        jcut(bx[1]);
        jcut(bx[1] + bx[4]);
    }
    for (auto *v : {&kb, &jb}) {
        std::sort(v->begin(), v->end());
        v->erase(std::unique(v->begin(), v->end()), v->end());
    }
    // thin k segments join a neighbour (spaces.hpp); with z tails a slab
    // makes no segment general (the lean and Debye kernels take its groups)
    merge_thin_segments(kb, [&](int ks, int ke) {
        bool zs = false, deb = false;
        for (int k = ks; k < ke && !zs; k++) zs = slab(2, k);
        for (const int *bx : boxes) deb = deb || (ke > bx[2] && ks < bx[2] + bx[5]);
        if (zs && !tails) return 2;
        return deb ? 1 : 0;
    }, D.thin);
    if (tails && D.ztail_split) {   // the slabs' groups as segments of their own, after the thin merges
        for (int q = 0; q < 4; q += 2)
            if (D.zt[u][q + 1] > D.zt[u][q]) { kcut(D.zt[u][q]); kcut(D.zt[u][q + 1]); }
        std::sort(kb.begin(), kb.end());
        kb.erase(std::unique(kb.begin(), kb.end()), kb.end());
    }
    struct Rect { int ks, ke, js, je; };
    std::vector<Rect> cls[kSpaces];
    for (size_t q = 0; q + 1 < kb.size(); q++) {
        const int ks = kb[q], ke = kb[q + 1];
        bool zs = false;
        for (int k = ks; k < ke; k++) zs = zs || slab(2, k);
        cls[kAll].push_back({ks, ke, 0, rows});
        for (size_t r = 0; r + 1 < jb.size(); r++) {
            const int js = jb[r], je = jb[r + 1];
            bool pml = zs && !tails, deb = false;
            for (int j = js; j < je && !pml; j++) pml = slab(1, j);
            for (const int *bx : boxes)
                deb = deb || (ke > bx[2] && ks < bx[2] + bx[5] && je > bx[1] && js < bx[1] + bx[4]);
            std::vector<Rect> &v = cls[pml ? kGeneral : (deb ? kDebye : kFast)];
            if (!v.empty() && v.back().ks == ks && v.back().je == js) v.back().je = je;
            else v.push_back({ks, ke, js, je});
        }
    }
    if (p1 <= p0 || (int)cls[kFast].size() > kMaxRects || (int)cls[kGeneral].size() > kMaxRects ||
        (int)cls[kDebye].size() > kMaxRects) {
        cls[kFast].clear();   // no interior planes, or too many rectangles: every block general
        cls[kDebye].clear();
        cls[kGeneral] = cls[kAll];
    }
    if ((int)cls[kAll].size() > kMaxRects) {
        set_error("too many k segments");
        return false;
    }
    for (int c = 0; c < kSpaces; c++) {
        Space &sp = D.sp[u][c];
        sp = Space{};
        long long t = 0;
        for (const Rect &r : cls[c]) {
            const long long nk4 = (r.ke - r.ks) / 4, nr = r.je - r.js;
            if (nr * nk4 * nk4 >= (1ll << 40)) {
                set_error("grid too large for the update layout");
                return false;
            }
            sp.ks[sp.n] = r.ks;
            sp.ke[sp.n] = r.ke;
            sp.js[sp.n] = r.js;
            sp.t0[sp.n] = (int)t;
            sp.magic[sp.n] = ((1ull << 40) + (unsigned long long)nk4 - 1) / (unsigned long long)nk4;
            sp.n++;
            t += nr * nk4;
        }
        if (t >= (1ll << 31) - kBlock) {
            set_error("grid too large for the update layout");
            return false;
        }
        sp.t0[sp.n] = (int)t;
    }
    D.p0[u] = p0;
    D.p1[u] = p1;
    // general work-list: the general space on interior planes, every rectangle elsewhere
    std::vector<int2> wl;
    std::vector<int> &st = D.wl_start[u];
    st.assign(planes + 1, 0);
    const int ng = space_blocks(D.sp[u][kGeneral]), na = space_blocks(D.sp[u][kAll]);
    for (int i = 0; i < planes; i++) {
        st[i] = (int)wl.size();
        const int nb = i >= p0 && i < p1 ? ng : na;
        for (int b = 0; b < 3 * nb; b++) wl.push_back(make_int2(i, b));
    }
    st[planes] = (int)wl.size();
    return wl.empty() || dev_upload(s, D.wl[u], wl);
}

bool build_sources(cem_sim *s, Device &D) {
    const size_t plane = (size_t)(s->n[1] + 1) * (s->n[2] + 1);
    if (s->msrc >= 0) {
        const ModePort &p = s->mport[s->msrc];
        std::vector<float> w[2] = {std::vector<float>(plane, 0.f), std::vector<float>(plane, 0.f)};
        for (size_t e = 0; e < p.src_idx.size(); e++) {
            const size_t q = p.src_idx[e];
            const size_t jk = q % s->si;   // j*sj + k on the i_src plane
            w[p.src_comp[e] - 1][jk] += (float)p.src_w[e];
        }
        if (!dev_upload(s, D.wsrc[0], w[0]) || !dev_upload(s, D.wsrc[1], w[1])) return false;
    }
    return true;
}

void fill_args_for(cem_sim *s, Device &D, int cur) {
    StepArgs &a = D.sa[cur];
    a = StepArgs{};
    a.g = D.g;
    for (int u = 0; u < 2; u++) {
        for (int c = 0; c < kSpaces; c++) a.sp[u][c] = D.sp[u][c];
        a.p0[u] = D.p0[u];
        a.p1[u] = D.p1[u];
        for (int q = 0; q < 4; q++) a.zt[u][q] = D.zt[u][q];
    }
    for (int c = 0; c < 3; c++) {
        a.E[c] = D.E[cur][c].p;
        a.H[c] = D.H[cur][c].p;
        a.hc[c] = D.hc[c].p;
        a.ec[c] = D.ec[c].p;
        a.pml[c] = PmlAxis{D.plane_h[c].p, D.plane_e[c].p, D.bm1_h[c].p, D.cid_h[c].p, D.bm1_e[c].p, D.cid_e[c].p,
                           D.pml_planes[c], D.zoff_h.p, D.zoff_e.p, D.zw_h, D.zw_e};
        for (int w = 0; w < 2; w++) {
            a.psiH[c][w] = D.psiH[cur][c][w].p;
            a.psiE[c][w] = D.psiE[c][w].p;
        }
        a.mat[c] = D.mat[c].p;
        a.tab[c] = D.tab[c].p;
        a.tab4[c] = D.tab4[c].p;
        a.beta4[c] = D.beta4[c].p;
        a.ntab[c] = D.ntab[c];
        a.J[c] = D.J[c].p;
        for (int q = 0; q < 6; q++) a.jbox[c][q] = D.jbox[c][q];
    }
    a.dth = (float)(s->dt / CEM_MU0);
    a.has_pml = s->has_pml;
    a.npole = s->npole;
    a.nb4 = (s->npole + 3) / 4;
    for (int p = 0; p < s->npole; p++) {
        const double tau = 1.0 / (2 * M_PI * s->pole_f[p]);
        const double r = s->dt / (2 * tau);
        a.omk[p] = (float)(2 * r / (1 + r));   // 1 - k_p
        a.hk[p] = (float)(0.5 * (1 + s->d_k[p]));
    }
    a.dt = s->dt;
    a.src_amp = s->src_port >= 0 ? s->src_amp : 0.0;
    a.src_t0 = s->src_t0;
    a.src_tau = s->src_tau;
    a.msrc_on = s->msrc >= 0;
    if (a.msrc_on) {
        a.i_src = s->mport[s->msrc].def.i_src;
        a.m_t0 = s->msrc_t0;
        a.m_tau = s->msrc_tau;
        a.wsrc[0] = D.wsrc[0].p;
        a.wsrc[1] = D.wsrc[1].p;
    }
    a.dstep = D.dstep.p;
    a.srcv = D.srcv.p;

    FusedArgs &f = D.fa[cur];
    f.error = D.error.p;
    for (int c = 0; c < 3; c++) {
        f.Eo[c] = D.E[cur][c].p; f.Ho[c] = D.H[cur][c].p;
        f.En[c] = D.E[cur ^ 1][c].p; f.Hn[c] = D.H[cur ^ 1][c].p;
        for (int w = 0; w < 2; w++) {
            f.psiHo[c][w] = D.psiH[cur][c][w].p;
            f.psiHn[c][w] = D.psiH[cur ^ 1][c][w].p;
        }
    }

    SibcArgs &b = D.sb[cur];
    b = SibcArgs{};
    b.ns = s->nsb;
    b.K = s->sibc_npole;
    b.ecomp = D.sb_ecomp.p; b.eidx = D.sb_eidx.p; b.hcomp = D.sb_hcomp.p; b.hidx = D.sb_hidx.p; b.hw = D.sb_hw.p;
    b.y = D.sb_y.p;
    for (int k = 0; k < s->sibc_npole; k++) {
        b.c[k] = (float)s->sibc_c[k];
        b.ome[k] = (float)(-std::expm1(-s->sibc_a[k] * s->dt));   // 1 - e_k without cancellation
    }
    for (int c = 0; c < 3; c++) { b.E[c] = D.E[cur][c].p; b.H[c] = D.H[cur][c].p; }

    PostArgs &p = D.pa[cur];
    p = PostArgs{};
    p.nin = D.nin; p.nip = D.nip; p.nport = D.nport; p.nvp = D.nvp; p.nslot = D.nslot;
    p.off = D.off.p; p.ecomp = D.ecomp.p; p.eidx = D.eidx.p; p.ew = D.ew.p; p.R = D.R.p; p.vold = D.vold.p;
    p.src_port = s->src_port;
    p.src_amp = s->src_amp; p.src_t0 = s->src_t0; p.src_tau = s->src_tau; p.dt = s->dt;
    p.msrc_on = s->msrc >= 0; p.m_t0 = s->msrc_t0; p.m_tau = s->msrc_tau;
    p.ring = D.ring.p;
    for (int c = 0; c < 3; c++) { p.F[c] = D.E[cur][c].p; p.F[3 + c] = D.H[cur][c].p; }
    p.dstep = D.dstep.p;
    p.srcv = D.srcv.p;

    EnergyArgs &e = D.ea[cur];
    e.g = D.g;
    for (int c = 0; c < 3; c++) {
        e.F[c] = D.E[cur][c].p; e.F[3 + c] = D.H[cur][c].p;
        e.mat[c] = D.mat[c].p; e.cb64[c] = D.cb64[c].p;
        e.d[c] = D.d64[c].p; e.dd[c] = D.dd64[c].p;
    }
    e.dt = s->dt;
    e.partial = D.partial.p;
}

void fill_args(cem_sim *s, Device &D) {
    fill_args_for(s, D, 0);
    fill_args_for(s, D, 1);
}

bool create_device_impl(cem_sim *s);

// a device that failed to build is dropped, so the next call starts over
bool create_device(cem_sim *s) {
    if (s->dev) return !s->dev->failed;
    if (create_device_impl(s)) return true;
    s->dev.reset();
    return false;
}

// 3D tiled TMA descriptor of one field buffer (padded layout), box kBX x rows x 1
bool make_tmap(cem_sim *s, CUtensorMap *map, const float *base, unsigned rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            set_error("cuTensorMapEncodeTiled unavailable");
            return false;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const Device &D = *s->dev;
    const cuuint64_t dims[3] = {(cuuint64_t)s->n[2] + 1, (cuuint64_t)s->n[1] + 1, (cuuint64_t)s->n[0] + 1};
    const cuuint64_t strides[2] = {(cuuint64_t)D.g.sj * 4, (cuuint64_t)D.g.si * 4};
    const cuuint32_t box[3] = {(cuuint32_t)kBX, rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed");
        return false;
    }
    return true;
}

bool create_device_impl(cem_sim *s) {
    if (!s->finalized) { set_error("not finalized"); return false; }
    int ndev = 0;
    cudaError_t err = cudaGetDeviceCount(&ndev);
    if (err != cudaSuccess || ndev == 0) {
        set_error("no CUDA device: libcourant_b200 steps only on the GPU");
        std::fprintf(stderr, "courant-b200: no CUDA device: libcourant_b200 steps only on the GPU\n");
        return false;
    }
    s->dev.reset(new Device);
    Device &D = *s->dev;
    if (g_selected_device >= 0) CB2_CHECK(s, cudaSetDevice(g_selected_device));
    CB2_CHECK(s, cudaGetDevice(&D.device));
    if (const char *e = std::getenv("CEM_B200_FUSED")) D.use_fused = e[0] == '1';
    if (const char *e = std::getenv("CEM_B200_GRAPHS")) D.use_graphs = e[0] != '0';
    D.ztail = (long long)s->n[0] * s->n[1] * s->n[2] >= 2000000;
    if (const char *e = std::getenv("CEM_B200_ZTAIL")) {
        D.ztail = e[0] != '0';
        D.ztail_split = e[0] != '1';
    }
    if (const char *e = std::getenv("CEM_B200_ROWS")) D.whole_rows = e[0] == '1';
    if (s->kernel_choice >= 0) D.use_fused = s->kernel_choice == 1;
    if (const char *e = std::getenv("CEM_B200_TUNE")) D.tune = e[0] == '1';
    if (s->tune_choice >= 0) D.tune = s->tune_choice == 1;
    CB2_CHECK(s, cudaStreamCreateWithFlags(&D.stream, cudaStreamNonBlocking));
    CB2_CHECK(s, cudaStreamCreateWithFlags(&D.side, cudaStreamNonBlocking));
    CB2_CHECK(s, cudaEventCreateWithFlags(&D.fork, cudaEventDisableTiming));
    CB2_CHECK(s, cudaEventCreateWithFlags(&D.join, cudaEventDisableTiming));
    Geom &g = D.g;
    for (int a = 0; a < 3; a++) g.n[a] = s->n[a];
    g.sj = (s->n[2] + 1 + 7) / 8 * 8;
    g.si = (long long)(s->n[1] + 1) * g.sj;
    g.plane = (int)g.si;
    g.sj_magic = ((1ull << 40) + g.sj - 1) / g.sj;
    D.Np = (size_t)g.si * (s->n[0] + 1);
    if ((double)g.plane * (double)g.sj >= 1099511627776.0 || D.Np >= (1ull << 31)) {
        set_error("grid too large: more than 2^31 points");
        return false;
    }
    for (int c = 0; c < 3; c++) {
        for (int b = 0; b < 2; b++)
            if (!dev_alloc(s, D.E[b][c], D.Np) || !dev_alloc(s, D.H[b][c], D.Np) ||
                !zero_dev(s, D.E[b][c].p, D.Np * 4) || !zero_dev(s, D.H[b][c].p, D.Np * 4))
                return false;
        // per-axis coefficients, zero-padded so four consecutive k load as one float4
        std::vector<double> hc(axis_padded(s->n[c]), 0.0), ec(axis_padded(s->n[c]), 0.0);
        for (int i = 0; i < s->n[c]; i++) hc[i] = s->dt / CEM_MU0 * s->idh[c][i];
        for (int i = 0; i <= s->n[c]; i++) ec[i] = s->ide[c][i];
        if (!dev_upload(s, D.hc[c], to_f32(hc)) || !dev_upload(s, D.ec[c], to_f32(ec))) return false;
        if (!dev_upload(s, D.d64[c], s->d[c]) || !dev_upload(s, D.dd64[c], s->dd[c])) return false;
    }
    // CEM_B200_TRACE=1: the host time of each set-up phase on stderr
    static const bool trace = [] { const char *e = std::getenv("CEM_B200_TRACE"); return e && e[0] == '1'; }();
    auto t0 = std::chrono::steady_clock::now();
    auto phase = [&](const char *name, bool ok) {
        if (trace) {
            const auto t1 = std::chrono::steady_clock::now();
            std::fprintf(stderr, "courant-b200: device set-up %-8s %8.3f s\n", name,
                         std::chrono::duration<double>(t1 - t0).count());
            t0 = t1;
        }
        return ok;
    };
    if (!phase("fields", true) || !phase("pml", build_pml(s, D)) || !phase("tables", build_tables(s, D)) ||
        !phase("probes", build_probes(s, D)) || !phase("sibc", build_sibc(s, D)) ||
        !phase("sources", build_sources(s, D)) || !phase("spaces", build_spaces(s, D, 0) && build_spaces(s, D, 1)))
        return false;
    for (int b = 0; b < 2; b++)
        for (int c = 0; c < 3; c++)
            if (!make_tmap(s, &D.maps[b].e[c], D.E[b][c].p, kRJ) || !make_tmap(s, &D.maps[b].h[c], D.H[b][c].p, kHJ))
                return false;
    if (!dev_alloc(s, D.error, 1) || !zero_dev(s, D.error.p, 4)) return false;
    CB2_CHECK(s, cudaFuncSetAttribute(kFKernels[s->npole], cudaFuncAttributeMaxDynamicSharedMemorySize, kFusedSmem));
    const long long nblk = (long long)((g.plane + kEnergyBlock - 1) / kEnergyBlock) * (s->n[0] + 1);
    if (!dev_alloc(s, D.partial, (size_t)nblk) || !dev_alloc(s, D.scalar, 1)) return false;
    fill_args(s, D);
    return true;
}

// ----------------------------------------------------- host <-> device moves

// a field in the reference layout -> the padded device layout, and back
bool upload_field(cem_sim *s, float *dst, const std::vector<double> &src) {
    const Device &D = *s->dev;
    std::vector<float> tmp(D.Np, 0.f);
    const int nx = s->n[0], ny = s->n[1], nz = s->n[2];
    for (int i = 0; i <= nx; i++)
        for (int j = 0; j <= ny; j++) {
            const double *r = &src[(size_t)i * s->si + (size_t)j * s->sj];
            float *o = &tmp[(size_t)i * D.g.si + (size_t)j * D.g.sj];
            for (int k = 0; k <= nz; k++) o[k] = (float)r[k];
        }
    return h2d(s, dst, tmp.data(), tmp.size() * 4);
}

bool download_field(cem_sim *s, std::vector<double> &dst, const float *src) {
    const Device &D = *s->dev;
    std::vector<float> tmp(D.Np);
    if (!d2h(s, tmp.data(), src, tmp.size() * 4)) return false;
    dst.resize(s->N);
    const int nx = s->n[0], ny = s->n[1], nz = s->n[2];
    for (int i = 0; i <= nx; i++)
        for (int j = 0; j <= ny; j++) {
            const float *r = &tmp[(size_t)i * D.g.si + (size_t)j * D.g.sj];
            double *o = &dst[(size_t)i * s->si + (size_t)j * s->sj];
            for (int k = 0; k <= nz; k++) o[k] = r[k];
        }
    return true;
}

// pack the host DFT accumulators in slot order: I probes, port V/I, source, V probes
std::vector<double *> dft_slots(cem_sim *s) {
    std::vector<double *> v;
    for (CurrentProbe &p : s->ip) v.push_back(p.acc.data());
    for (LumpedPort &p : s->port) { v.push_back(p.V.data()); v.push_back(p.I.data()); }
    v.push_back(s->src_acc.data());
    for (VoltageProbe &p : s->vp) v.push_back(p.acc.data());
    return v;
}

bool flush_dft(cem_sim *s) {
    Device &D = *s->dev;
    if (!D.ring_count) return true;
    dim3 grid((s->nf + 127) / 128, D.nslot);
    t_begin(4);
    k_dft<<<grid, 128, 0, D.stream>>>(D.ring.p, D.nslot, D.nip + 2 * D.nport + 1, D.ring_first, D.ring_count, s->dt,
                                      D.omega.p, s->nf, D.acc.p);
    t_end();
    CB2_CHECK(s, cudaGetLastError());
    D.ring_first += D.ring_count;
    D.ring_count = 0;
    return true;
}

// Reference compact index -> device index of every auxiliary of array
// (c, w) (derivative axis (c + w + 1) % 3), E (nodes) or H (cells).
template <class F>
void psi_map(const cem_sim *s, const Device &D, bool is_e, int c, int w, F visit) {
    const int ax = (c + w + 1) % 3, nx = s->n[0], ny = s->n[1], nz = s->n[2];
    const size_t per = pml_per(s, ax);
    const int planes = D.pml_planes[ax];
    for (int pl = 0; pl < planes; pl++) {
        if (ax == 0) {
            for (int j = 0; j <= ny; j++)
                for (int k = 0; k <= nz; k++)
                    visit(pl * per + (size_t)j * (nz + 1) + k, (size_t)pl * D.g.si + (size_t)j * D.g.sj + k);
        } else if (ax == 1) {
            for (int i = 0; i <= nx; i++)
                for (int k = 0; k <= nz; k++)
                    visit(pl * per + (size_t)i * (nz + 1) + k, ((size_t)i * planes + pl) * D.g.sj + k);
        } else {
            int r[2][2];
            pml_ranges(s, 2, is_e, r);
            const int nlo = r[0][1] >= r[0][0] ? r[0][1] - r[0][0] + 1 : 0;
            const int kz = pl < nlo ? r[0][0] + pl : r[1][0] + (pl - nlo);
            const size_t zw = is_e ? D.zw_e : D.zw_h, zo = D.zoff_host[is_e][kz];
            for (int i = 0; i <= nx; i++)
                for (int j = 0; j <= ny; j++)
                    visit(pl * per + (size_t)i * (ny + 1) + j, ((size_t)i * (ny + 1) + j) * zw + zo);
        }
    }
}

bool psi_upload(cem_sim *s, bool is_e, int c, int w, const std::vector<double> &v, float *dst) {
    const Device &D = *s->dev;
    const size_t n = is_e ? D.psi_dev_e[c][w] : D.psi_dev_h[c][w];
    if (!n) return true;
    std::vector<float> o(n + 4, 0.f);
    if (!v.empty()) psi_map(s, D, is_e, c, w, [&](size_t r, size_t d) { o[d] = (float)v[r]; });
    return h2d(s, dst, o.data(), o.size() * sizeof(float));
}

bool psi_download(cem_sim *s, bool is_e, int c, int w, std::vector<double> &v, const float *src) {
    const Device &D = *s->dev;
    const size_t n = is_e ? D.psi_dev_e[c][w] : D.psi_dev_h[c][w];
    v.assign(is_e ? D.psi_len_e[c][w] : D.psi_len_h[c][w], 0.0);
    if (!n) return true;
    std::vector<float> o(n);
    if (!d2h(s, o.data(), src, n * sizeof(float))) return false;
    psi_map(s, D, is_e, c, w, [&](size_t r, size_t d) { v[r] = o[d]; });
    return true;
}

bool upload_group(cem_sim *s, unsigned g, bool from_host) {
    Device &D = *s->dev;
    for (int c = 0; c < 3; c++) {
        if (g & (kGroupE0 << c)) {
            if (from_host) { if (!upload_field(s, D.E[D.cur][c].p, s->E[c])) return false; }
            else if (!zero_dev(s, D.E[D.cur][c].p, D.Np * sizeof(float))) return false;
            D.vold_valid = false;
        }
        if (g & (kGroupH0 << c)) {
            if (from_host) { if (!upload_field(s, D.H[D.cur][c].p, s->H[c])) return false; }
            else if (!zero_dev(s, D.H[D.cur][c].p, D.Np * sizeof(float))) return false;
        }
    }
    if (g & kGroupPsi)
        for (int c = 0; c < 3; c++)
            for (int w = 0; w < 2; w++) {
                if (from_host) {
                    if (!psi_upload(s, true, c, w, s->psiE[c][w], D.psiE[c][w].p) ||
                        !psi_upload(s, false, c, w, s->psiH[c][w], D.psiH[D.cur][c][w].p))
                        return false;
                } else if (!zero_dev(s, D.psiE[c][w].p, D.psiE[c][w].n * 4) ||
                           !zero_dev(s, D.psiH[D.cur][c][w].p, D.psiH[D.cur][c][w].n * 4)) {
                    return false;
                }
            }
    if (g & kGroupDebye)
        for (int c = 0; c < 3; c++) {
            if (!D.J[c].p) continue;
            if (!from_host) { if (!zero_dev(s, D.J[c].p, D.J[c].n * 4)) return false; continue; }
            const int *bx = D.jbox[c];
            const size_t vol = (size_t)bx[3] * bx[4] * bx[5];
            std::vector<float> box(D.J[c].n, 0.f);
            for (int e = 0; e < s->ndisp; e++) {
                if (s->d_comp[e] != c) continue;
                const size_t q = s->d_idx[e];
                const int i = (int)(q / s->si), j = (int)((q % s->si) / s->sj), k = (int)(q % s->sj);
                const size_t o = ((size_t)(i - bx[0]) * bx[4] + (j - bx[1])) * bx[5] + (k - bx[2]);
                for (int p = 0; p < s->npole; p++) box[jaddr(s->npole, vol, p, o)] = (float)s->d_J[(size_t)p * s->ndisp + e];
            }
            if (!h2d(s, D.J[c].p, box.data(), box.size() * 4)) return false;
        }
    if ((g & kGroupSibc) && s->nsb) {
        if (!from_host) {
            if (!zero_dev(s, D.sb_y.p, D.sb_y.n * 4)) return false;
        } else {
            const int K = s->sibc_npole, ns = s->nsb;
            std::vector<float> y((size_t)K * ns);
            for (int e = 0; e < ns; e++)
                for (int k = 0; k < K; k++) y[(size_t)k * ns + e] = (float)s->sb_y[(size_t)e * K + k];
            if (!h2d(s, D.sb_y.p, y.data(), y.size() * 4)) return false;
        }
    }
    if (g & kGroupDft) {
        const size_t len = 2 * (size_t)s->nf;
        std::vector<double> acc((size_t)D.nslot * len, 0.0);
        if (from_host) {
            std::vector<double *> slots = dft_slots(s);
            for (size_t q = 0; q < slots.size(); q++) std::memcpy(&acc[q * len], slots[q], len * sizeof(double));
        }
        if (!h2d(s, D.acc.p, acc.data(), acc.size() * sizeof(double))) return false;
        D.ring_first = s->step;
        D.ring_count = 0;
    }
    return true;
}

bool download_group(cem_sim *s, unsigned g) {
    Device &D = *s->dev;
    if ((g & kGroupDft) && !flush_dft(s)) return false;
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    for (int c = 0; c < 3; c++) {
        if ((g & (kGroupE0 << c)) && !download_field(s, s->E[c], D.E[D.cur][c].p)) return false;
        if ((g & (kGroupH0 << c)) && !download_field(s, s->H[c], D.H[D.cur][c].p)) return false;
    }
    if (g & kGroupPsi)
        for (int c = 0; c < 3; c++)
            for (int w = 0; w < 2; w++)
                if (!psi_download(s, true, c, w, s->psiE[c][w], D.psiE[c][w].p) ||
                    !psi_download(s, false, c, w, s->psiH[c][w], D.psiH[D.cur][c][w].p))
                    return false;
    if (g & kGroupDebye) {
        s->d_J.assign((size_t)s->npole * s->ndisp, 0.0);
        if (s->d_Eold.size() != (size_t)s->ndisp) s->d_Eold.assign(s->ndisp, 0.0);
        for (int c = 0; c < 3; c++) {
            if (!D.J[c].p) continue;
            std::vector<float> box(D.J[c].n);
            if (!d2h(s, box.data(), D.J[c].p, box.size() * 4)) return false;
            const int *bx = D.jbox[c];
            const size_t vol = (size_t)bx[3] * bx[4] * bx[5];
            for (int e = 0; e < s->ndisp; e++) {
                if (s->d_comp[e] != c) continue;
                const size_t q = s->d_idx[e];
                const int i = (int)(q / s->si), j = (int)((q % s->si) / s->sj), k = (int)(q % s->sj);
                const size_t o = ((size_t)(i - bx[0]) * bx[4] + (j - bx[1])) * bx[5] + (k - bx[2]);
                for (int p = 0; p < s->npole; p++) s->d_J[(size_t)p * s->ndisp + e] = box[jaddr(s->npole, vol, p, o)];
            }
        }
    }
    if ((g & kGroupSibc) && s->nsb) {
        const int K = s->sibc_npole, ns = s->nsb;
        std::vector<float> y((size_t)K * ns);
        if (!d2h(s, y.data(), D.sb_y.p, y.size() * 4)) return false;
        s->sb_y.resize((size_t)K * ns);
        for (int e = 0; e < ns; e++)
            for (int k = 0; k < K; k++) s->sb_y[(size_t)e * K + k] = y[(size_t)k * ns + e];
    }
    if (g & kGroupDft) {
        const size_t len = 2 * (size_t)s->nf;
        std::vector<double> acc((size_t)D.nslot * len);
        if (!d2h(s, acc.data(), D.acc.p, acc.size() * sizeof(double))) return false;
        std::vector<double *> slots = dft_slots(s);
        for (size_t q = 0; q < slots.size(); q++) std::memcpy(slots[q], &acc[q * len], len * sizeof(double));
    }
    return true;
}

// Make the device state current before a device operation.
bool begin_device_op(cem_sim *s) {
    if (!create_device(s)) return false;
    Device &D = *s->dev;
    if (D.failed) { set_error(D.error_msg.c_str()); return false; }
    CB2_CHECK(s, cudaSetDevice(D.device));
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    const unsigned need = (~s->dev_valid | s->exposed) & kGroupAll;
    for (unsigned g = 1; g & kGroupAll; g <<= 1) {
        if (!(need & g)) continue;
        if (!upload_group(s, g, (s->host_valid & g) != 0)) return false;
    }
    s->dev_valid = kGroupAll;
    if (D.ring_count == 0) D.ring_first = s->step;
    long long st = s->step;
    CB2_CHECK(s, cudaMemcpyAsync(D.dstep.p, &st, sizeof st, cudaMemcpyHostToDevice, D.stream));
    k_source_values<<<1, 1, 0, D.stream>>>(D.pa[D.cur]);
    CB2_CHECK(s, cudaGetLastError());
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    if (!D.vold_valid && D.nport) {
        PostArgs pa = D.pa[D.cur];
        pa.advance = 0;
        k_post<<<1, kPostThreads, 0, D.stream>>>(pa);
        CB2_CHECK(s, cudaGetLastError());
        D.vold_valid = true;
    }
    s->host_valid = 0;
    return true;
}

// After a device operation: refresh what callers hold pointers to.
bool end_device_op(cem_sim *s) {
    Device &D = *s->dev;
    if (D.use_fused) {
        int err = 0;
        if (!d2h(s, &err, D.error.p, sizeof err)) return false;
        if (err) {
            D.failed = true;
            D.error_msg = "device: a TMA wait in the fused step timed out";
            set_error(D.error_msg.c_str());
            std::fprintf(stderr, "courant-b200: %s\n", D.error_msg.c_str());
            return false;
        }
    }
    if (s->exposed) {
        if (!download_group(s, s->exposed)) return false;
        s->host_valid |= s->exposed;
    }
    return true;
}

// Surface impedance, then the probe pass (probes, ports, sample ring, step
// count). SIBC writes E only on its own edges and the probes only read, so
// when no probe edge is a SIBC edge the two run side by side (SIBC on the
// second stream, joined before the next step); one after the other while
// kernels are timed one by one.
void launch_sibc_post(cem_sim *s, Device &D) {
    PostArgs pa = D.pa[D.cur];
    pa.advance = 1;
    const bool beside = s->nsb && D.post_beside_sibc && !g_timer;
    const unsigned nb = (unsigned)((s->nsb + kBlock - 1) / kBlock);
    if (beside) {
        cudaEventRecord(D.fork, D.stream);
        cudaStreamWaitEvent(D.side, D.fork, 0);
        k_sibc<<<nb, kBlock, 0, D.side>>>(D.sb[D.cur]);
        cudaEventRecord(D.join, D.side);
    } else if (s->nsb) {
        t_begin(2);
        k_sibc<<<nb, kBlock, 0, D.stream>>>(D.sb[D.cur]);
        t_end();
    }
    t_begin(3);
    k_post<<<1, kPostThreads, 0, D.stream>>>(pa);
    t_end();
    if (beside) cudaStreamWaitEvent(D.stream, D.join, 0);
}

// one whole step: the fused H+E pass, then SIBC, probes and the step count
bool launch_fused_step(cem_sim *s) {
    Device &D = *s->dev;
    if (D.ring_count == kRing && !flush_dft(s)) return false;
    const dim3 grid((s->n[2] + 1 + kFK - 1) / kFK, (s->n[1] + 1 + kFJ - 1) / kFJ, (s->n[0] + 1 + kFX - 1) / kFX);
    t_begin(1);
    kFKernels[s->npole]<<<grid, dim3(kFK, kFJ), kFusedSmem, D.stream>>>(D.sa[D.cur], D.fa[D.cur], D.maps[D.cur]);
    t_end();
    D.cur ^= 1;
    launch_sibc_post(s, D);
    D.ring_count++;
    s->step++;
    CB2_CHECK(s, cudaGetLastError());
    return true;
}

bool launch_step(cem_sim *s, int phase_mask, int i0, int i1) {
    Device &D = *s->dev;
    if (phase_mask == (1 | 4 | 8) && i0 <= 0 && i1 > s->n[0] && D.use_fused) return launch_fused_step(s);
    const int nx = s->n[0];
    const dim3 blk(kBlock);
    // general work-list entries of update u for node planes [a, b)
    auto span = [&](int u, int a, int b, const int2 *&p) {
        const std::vector<int> &st = D.wl_start[u];
        p = D.wl[u].p + st[a];
        return (unsigned)(st[b] - st[a]);
    };
    // fast (or Debye) rectangles of update u on node planes [a, b)
    auto fast = [&](int u, int a, int b, auto kernel, int cls = kFast) {
        const int nb = space_blocks(D.sp[u][cls]);
        const int c0 = std::max(a, D.p0[u]), c1 = std::min(b, D.p1[u]);
        if (nb == 0) return;
        for (int c = c0; c < c1; c += kMaxGridY)
            kernel<<<dim3(3 * nb, std::min(kMaxGridY, c1 - c)), blk, 0, D.stream>>>(D.sa[D.cur], c);
    };
    // the general blocks go to the side stream (after the work so far on the
    // main one), the fast pieces to the main stream, which then waits for both
    auto fork = [&]() {
        cudaEventRecord(D.fork, D.stream);
        cudaStreamWaitEvent(D.side, D.fork, 0);
    };
    auto join = [&]() { cudaStreamWaitEvent(D.stream, D.join, 0); };
    if (phase_mask & 1) {   // H over node planes [i0, i1) within [0, nx]
        const int a = std::max(0, i0), b = std::min(nx + 1, i1);
        if (b > a) {
            t_begin(0);
            const int2 *w;
            const unsigned n = span(0, a, b, w);
            if (n && D.side_on) {
                fork();
                k_update_h<<<n, blk, 0, D.side>>>(D.sa[D.cur], w);
                cudaEventRecord(D.join, D.side);
            }
            fast(0, a, b, k_update_h_fast);
            if (n && !D.side_on) k_update_h<<<n, blk, 0, D.stream>>>(D.sa[D.cur], w);
            if (n && D.side_on) join();
            t_end();
        }
    }
    if (phase_mask & 2) {   // port voltages before the E update
        PostArgs pa = D.pa[D.cur];
        pa.advance = 0;
        if (D.nport) k_post<<<1, kPostThreads, 0, D.stream>>>(pa);
    }
    if (phase_mask & 4) {   // E over node planes [i0, i1) within [0, nx)
        const int a = std::max(0, i0), b = std::min(nx, i1);
        if (b > a) {
            t_begin(1);
            const int2 *w;
            const unsigned n = span(1, a, b, w);
            if (n && D.side_on) {
                fork();
                kEKernels[s->npole]<<<n, blk, 0, D.side>>>(D.sa[D.cur], w);
                cudaEventRecord(D.join, D.side);
            }
            fast(1, a, b, k_update_e_fast);
            fast(1, a, b, kEDKernels[s->npole], kDebye);
            if (n && !D.side_on) kEKernels[s->npole]<<<n, blk, 0, D.stream>>>(D.sa[D.cur], w);
            if (n && D.side_on) join();
            t_end();
        }
    }
    if (phase_mask & 8) {   // surface impedance, probes, step count
        if (D.ring_count == kRing && !flush_dft(s)) return false;
        launch_sibc_post(s, D);
        D.ring_count++;
        s->step++;
    }
    CB2_CHECK(s, cudaGetLastError());
    return true;
}

}  // namespace

// ------------------------------------------------------------ engine API

void host_state_alloc(cem_sim *s, unsigned groups) {
    for (int c = 0; c < 3; c++) {
        if ((groups & (kGroupE0 << c)) && s->E[c].size() != s->N) s->E[c].assign(s->N, 0.0);
        if ((groups & (kGroupH0 << c)) && s->H[c].size() != s->N) s->H[c].assign(s->N, 0.0);
    }
    if ((groups & kGroupPsi) && s->finalized)
        for (int c = 0; c < 3; c++)
            for (int w = 0; w < 2; w++) {
                if (s->psiE[c][w].size() != psi_len(s, 1, c, w)) s->psiE[c][w].assign(psi_len(s, 1, c, w), 0.0);
                if (s->psiH[c][w].size() != psi_len(s, 0, c, w)) s->psiH[c][w].assign(psi_len(s, 0, c, w), 0.0);
            }
    if ((groups & kGroupDebye) && s->finalized) {
        if (s->d_J.size() != (size_t)s->npole * s->ndisp) s->d_J.assign((size_t)s->npole * s->ndisp, 0.0);
        if (s->d_Eold.size() != (size_t)s->ndisp) s->d_Eold.assign(s->ndisp, 0.0);
    }
    if ((groups & kGroupSibc) && s->finalized && s->sb_y.size() != (size_t)s->nsb * s->sibc_npole)
        s->sb_y.assign((size_t)s->nsb * s->sibc_npole, 0.0);
}

bool engine_has_device(const cem_sim *s) { return s->dev != nullptr; }

int engine_pull(const cem_sim *cs, unsigned groups) {
    cem_sim *s = const_cast<cem_sim *>(cs);
    const unsigned missing = groups & ~s->host_valid & kGroupAll;
    if (!missing) return 0;
    host_state_alloc(s, missing);
    const unsigned from_dev = s->dev && !s->dev->failed ? missing & s->dev_valid : 0u;
    if (from_dev && !download_group(s, from_dev)) return -1;
    // groups valid nowhere are all zero: the freshly allocated host copies
    if (missing & ~from_dev) {
        for (int c = 0; c < 3; c++) {
            if (missing & ~from_dev & (kGroupE0 << c)) std::fill(s->E[c].begin(), s->E[c].end(), 0.0);
            if (missing & ~from_dev & (kGroupH0 << c)) std::fill(s->H[c].begin(), s->H[c].end(), 0.0);
        }
    }
    s->host_valid |= missing;
    return 0;
}

void engine_expose(const cem_sim *cs, unsigned groups) { const_cast<cem_sim *>(cs)->exposed |= groups; }

void engine_host_modified(cem_sim *s, unsigned groups) {
    s->host_valid |= groups;
    s->dev_valid &= ~groups;
}

namespace {

constexpr int kGraphSteps = 32;   // divides kRing: graph runs fill the sample ring exactly

// n whole steps. With graphs on (separate H and E kernels, not while kernels
// are timed one by one), a run of kGraphSteps steps that needs no DFT flush
// replays one graph captured from the same launches; the others go one by one.
// The graph holds the kernels' arguments, which stay fixed for the life of
// the device state.
bool run_steps(cem_sim *s, long n) {
    Device &D = *s->dev;
    const bool graphs = D.use_graphs && !D.use_fused && !g_timer;
    for (long it = 0; it < n;) {
        const int gs = D.graph_steps;
        if (graphs && n - it >= gs && D.ring_count + gs <= kRing) {
            if (!D.graph) {
                const int rc = D.ring_count;
                const long st = s->step;
                CB2_CHECK(s, cudaStreamBeginCapture(D.stream, cudaStreamCaptureModeThreadLocal));
                bool ok = true;
                for (int q = 0; q < gs && ok; q++) ok = launch_step(s, 1 | 4 | 8, 0, s->n[0] + 1);
                cudaGraph_t g = nullptr;
                const cudaError_t ec = cudaStreamEndCapture(D.stream, &g);
                D.ring_count = rc;
                s->step = st;
                if (!ok) {
                    if (g) cudaGraphDestroy(g);
                    return false;
                }
                CB2_CHECK(s, ec);
                const cudaError_t ei = cudaGraphInstantiate(&D.graph, g, 0);
                cudaGraphDestroy(g);
                if (ei != cudaSuccess) D.graph = nullptr;
                CB2_CHECK(s, ei);
            }
            CB2_CHECK(s, cudaGraphLaunch(D.graph, D.stream));
            D.ring_count += gs;
            s->step += gs;
            it += gs;
        } else {
            if (!launch_step(s, 1 | 4 | 8, 0, s->n[0] + 1)) return false;
            it++;
        }
    }
    CB2_CHECK(s, cudaGetLastError());
    return true;
}

// ------------------------------------------------------------------- tuner
//
// The launch shape of a simulation (thin-segment threshold of the thread
// spaces, general blocks on the second stream or after the others, steps per
// replayed graph) is chosen per grid shape: measured on the simulation's own
// first steps (every choice computes the same bits, so these are ordinary
// steps) and kept in a cache file, one line per grid shape, that later
// processes read instead of measuring again.

std::mutex g_shape_mu;
bool g_shape_loaded = false;
std::map<std::string, std::array<double, 5>> g_shapes;   // key -> thin, side, graph steps, ms per step, z tails

std::string shape_cache_path() {
    if (const char *p = std::getenv("CEM_B200_TUNE_CACHE")) return p;
    std::string base;
    if (const char *x = std::getenv("XDG_CACHE_HOME")) base = x;
    else if (const char *h = std::getenv("HOME")) base = std::string(h) + "/.cache";
    else base = "/tmp";
    return base + "/courant-b200/launch-shapes.txt";
}

std::string shape_key(const cem_sim *s) {
    char k[160];
    std::snprintf(k, sizeof k, "%dx%dx%d/p%d/sibc%d/pml%d.%d.%d.%d.%d.%d", s->n[0], s->n[1], s->n[2], s->npole,
                  s->nsb > 0, s->npml[0], s->npml[1], s->npml[2], s->npml[3], s->npml[4], s->npml[5]);
    return k;
}

void load_shapes() {   // g_shape_mu held
    if (g_shape_loaded) return;
    g_shape_loaded = true;
    FILE *f = std::fopen(shape_cache_path().c_str(), "r");
    if (!f) return;
    // lines: key thin side graph ms [ztail] (lines without the z-tail choice keep the default: -1)
    char line[400], key[200];
    while (std::fgets(line, sizeof line, f)) {
        double v[5] = {0, 0, 0, 0, -1};
        if (std::sscanf(line, "%199s %lf %lf %lf %lf %lf", key, &v[0], &v[1], &v[2], &v[3], &v[4]) >= 5)
            g_shapes[key] = {v[0], v[1], v[2], v[3], v[4]};
    }
    std::fclose(f);
}

void store_shape(const std::string &key, const std::array<double, 5> &v) {   // g_shape_mu held
    g_shapes[key] = v;
    const std::string path = shape_cache_path();
    for (size_t q = 1; q < path.size(); q++)   // mkdir -p of the directory
        if (path[q] == '/') mkdir(path.substr(0, q).c_str(), 0755);
    if (FILE *f = std::fopen(path.c_str(), "a")) {
        std::fprintf(f, "%s %g %g %g %.6g %g\n", key.c_str(), v[0], v[1], v[2], v[3], v[4]);
        std::fclose(f);
    }
}

bool apply_shape(cem_sim *s, Device &D, int thin, bool side, int graph, bool ztail) {
    const bool respace = thin != D.thin || ztail != D.ztail;
    if (respace) {
        D.thin = thin;
        D.ztail = ztail;
        if (!build_spaces(s, D, 0) || !build_spaces(s, D, 1)) return false;
        fill_args(s, D);
    }
    if (respace || graph != D.graph_steps) {
        if (D.graph) cudaGraphExecDestroy(D.graph);
        D.graph = nullptr;
        D.graph_steps = graph;
    }
    D.side_on = side;
    return true;
}

// device milliseconds per step of `n` steps (after `warm` untimed ones)
bool shape_ms(cem_sim *s, long warm, long n, double *ms, long *used) {
    Device &D = *s->dev;
    if (!D.tev[0]) {
        CB2_CHECK(s, cudaEventCreate(&D.tev[0]));
        CB2_CHECK(s, cudaEventCreate(&D.tev[1]));
    }
    if (!run_steps(s, warm)) return false;
    CB2_CHECK(s, cudaEventRecord(D.tev[0], D.stream));
    if (!run_steps(s, n)) return false;
    CB2_CHECK(s, cudaEventRecord(D.tev[1], D.stream));
    CB2_CHECK(s, cudaEventSynchronize(D.tev[1]));
    float f = 0;
    CB2_CHECK(s, cudaEventElapsedTime(&f, D.tev[0], D.tev[1]));
    *ms = f / n;
    *used += warm + n;
    return true;
}

// choose the launch shape of s (cache, else coordinate descent over the
// choices, 672 steps); `used` returns the steps it ran
bool tune_shape(cem_sim *s, long *used) {
    Device &D = *s->dev;
    const std::string key = shape_key(s);
    std::lock_guard<std::mutex> lock(g_shape_mu);
    load_shapes();
    auto it = g_shapes.find(key);
    D.tuned = true;
    if (it != g_shapes.end()) {
        D.tuned_from_cache = true;
        D.tuned_ms = it->second[3];
        const bool zt = it->second[4] < 0 ? D.ztail : it->second[4] != 0;
        return apply_shape(s, D, (int)it->second[0], it->second[1] != 0, (int)it->second[2], zt);
    }
    int thin = D.thin, graph = D.graph_steps;
    bool side = D.side_on, zt = D.ztail;
    double best;
    if (!shape_ms(s, 32, 64, &best, used)) return false;
    auto trial = [&](int t, bool sd, int g, bool z) {
        double ms;
        if (!apply_shape(s, D, t, sd, g, z) || !shape_ms(s, 32, 64, &ms, used)) return false;
        if (ms < 0.995 * best) { best = ms; thin = t; side = sd; graph = g; zt = z; }
        return apply_shape(s, D, thin, side, graph, zt);
    };
    if (!trial(thin, side, graph, !zt)) return false;
    for (int t : {8, 32}) if (!trial(t, side, graph, zt)) return false;
    if (!trial(thin, !side, graph, zt)) return false;
    for (int g : {16, 64}) if (!trial(thin, side, g, zt)) return false;
    D.tuned_ms = best;
    store_shape(key, {(double)thin, side ? 1.0 : 0.0, (double)graph, best, zt ? 1.0 : 0.0});
    return true;
}

}  // namespace

int engine_step(cem_sim *s, long n) {
    if (n <= 0) return 0;
    if (!begin_device_op(s)) return -1;
    Device &D = *s->dev;
    if (D.tune && !D.tuned && !D.use_fused && n >= 2048 && !g_timer) {
        long used = 0;
        if (!tune_shape(s, &used)) return -1;
        n -= used;
    }
    if (!run_steps(s, n)) return -1;
    if (!end_device_op(s)) return -1;
    return 0;
}

int engine_phase(cem_sim *s, int phase, int i0, int i1) {
    if (!begin_device_op(s)) return -1;
    static const int masks[5] = {0, 1, 2, 4, 8};
    if (phase < 0 || phase > 4) return 0;
    if (phase == 2) s->dev->vold_valid = true;
    if (!launch_step(s, masks[phase], i0, i1)) return -1;
    if (!end_device_op(s)) return -1;
    return 0;
}

namespace {
bool energy_on_device(cem_sim *s, double *out) {
    if (!begin_device_op(s)) return false;
    Device &D = *s->dev;
    const int gx = (D.g.plane + kEnergyBlock - 1) / kEnergyBlock;
    for (int c0 = 0; c0 <= s->n[0]; c0 += kMaxGridY)
        k_energy<<<dim3(gx, std::min(kMaxGridY, s->n[0] + 1 - c0)), kEnergyBlock, 0, D.stream>>>(D.ea[D.cur], c0);
    k_sum<<<1, 1024, 0, D.stream>>>(D.partial.p, (long long)gx * (s->n[0] + 1), D.scalar.p);
    CB2_CHECK(s, cudaGetLastError());
    CB2_CHECK(s, cudaMemcpyAsync(out, D.scalar.p, sizeof(double), cudaMemcpyDeviceToHost, D.stream));
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    return end_device_op(s);
}
}  // namespace

int engine_energy(const cem_sim *cs, double *out) {
    return energy_on_device(const_cast<cem_sim *>(cs), out) ? 0 : -1;
}

// ------------------------------------------- energy without device allocation
//
// cemx_energy_noalloc runs k_energy and k_sum exactly as energy_on_device
// does, but its block partials and its result live in this file-scope array
// instead of the simulation's own buffers. Every slot is written before it is
// read, so nothing has to start at zero. One array per device and process:
// calls for different simulations on one device must not overlap in time.
constexpr long long kNoAllocPartials = 65536;   // 512 KiB of block partials
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocPartials + 1];   // + the result

// Address of g_noalloc_scratch on the current device. In host code the
// array's name is only a host-side stand-in, so the device address is looked
// up on every call (cheap once the module is loaded, allocates nothing, and
// stays right after a cudaDeviceReset tears the module down and reloads it).
double *noalloc_scratch() {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "cemx_energy_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        set_error(msg);
        return nullptr;
    }
    return static_cast<double *>(p);
}

bool energy_noalloc_on(cem_sim *s, Device &D, double *out) {
    const int gx = (D.g.plane + kEnergyBlock - 1) / kEnergyBlock;
    const long long nblk = (long long)gx * (s->n[0] + 1);
    double *scratch = noalloc_scratch();
    if (!scratch) return false;
    EnergyArgs ea = D.ea[D.cur];
    ea.partial = scratch;
    for (int c0 = 0; c0 <= s->n[0]; c0 += kMaxGridY)
        k_energy<<<dim3(gx, std::min(kMaxGridY, s->n[0] + 1 - c0)), kEnergyBlock, 0, D.stream>>>(ea, c0);
    k_sum<<<1, 1024, 0, D.stream>>>(scratch, nblk, scratch + kNoAllocPartials);
    CB2_CHECK(s, cudaGetLastError());
    CB2_CHECK(s, cudaMemcpyAsync(out, scratch + kNoAllocPartials, sizeof(double), cudaMemcpyDeviceToHost, D.stream));
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    return true;
}

bool energy_noalloc(cem_sim *s, double *out) {
    if (!s->dev) {
        set_error("cemx_energy_noalloc: no device state (step the simulation first; this call never creates it)");
        return false;
    }
    Device &D = *s->dev;
    if (D.failed) { set_error(D.error_msg.c_str()); return false; }
    if ((s->dev_valid & kGroupFields) != kGroupFields || (s->exposed & kGroupFields)) {
        set_error("cemx_energy_noalloc: fields are held or modified on the host; use cem_energy");
        return false;
    }
    const int gx = (D.g.plane + kEnergyBlock - 1) / kEnergyBlock;
    const long long nblk = (long long)gx * (s->n[0] + 1);
    if (nblk > kNoAllocPartials) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "cemx_energy_noalloc: grid needs %lld block partials, above the static scratch of %lld; "
                      "use cem_energy", nblk, kNoAllocPartials);
        set_error(msg);
        return false;
    }
    // run on the simulation's device and give the caller back its current device
    int prev = -1;
    CB2_CHECK(s, cudaGetDevice(&prev));
    CB2_CHECK(s, cudaSetDevice(D.device));
    const bool ok = energy_noalloc_on(s, D, out);
    const cudaError_t e = cudaSetDevice(prev);
    if (ok && e != cudaSuccess) return fail(s, "cudaSetDevice(previous device)", e);
    return ok;
}

}  // namespace cb2

using namespace cb2;

namespace {
bool timed_steps(cem_sim *s, long n, double *ms) {
    if (!begin_device_op(s)) return false;
    Device &D = *s->dev;
    cudaEvent_t e0, e1;
    CB2_CHECK(s, cudaEventCreate(&e0));
    CB2_CHECK(s, cudaEventCreate(&e1));
    CB2_CHECK(s, cudaEventRecord(e0, D.stream));
    if (!run_steps(s, n)) return false;
    CB2_CHECK(s, cudaEventRecord(e1, D.stream));
    CB2_CHECK(s, cudaEventSynchronize(e1));
    float t = 0;
    CB2_CHECK(s, cudaEventElapsedTime(&t, e0, e1));
    *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return end_device_op(s);
}

bool profiled_steps(cem_sim *s, long n, double *kernel_ms, long *launches) {
    if (!begin_device_op(s)) return false;
    Device &D = *s->dev;
    KernelTimer timer;
    timer.stream = D.stream;
    g_timer = &timer;
    bool ok = true;
    for (long it = 0; it < n && ok; it++) ok = launch_step(s, 1 | 4 | 8, 0, s->n[0] + 1);
    if (ok) ok = flush_dft(s);
    g_timer = nullptr;
    if (!ok) return false;
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    for (int k = 0; k < 5; k++) { kernel_ms[k] = 0; launches[k] = 0; }
    for (size_t q = 0; q + 1 < timer.ev.size(); q += 2) {
        float t = 0;
        CB2_CHECK(s, cudaEventElapsedTime(&t, timer.ev[q], timer.ev[q + 1]));
        kernel_ms[timer.kind[q]] += t;
        launches[timer.kind[q]]++;
    }
    for (cudaEvent_t e : timer.ev) cudaEventDestroy(e);
    return end_device_op(s);
}
}  // namespace

// ------------------------------------------------------------------ batches

// Simulations advanced together on one device (cemx_batch_*). Each member
// keeps its own device state; the batch holds device copies of the members'
// kernel arguments and the work-lists of the batched kernels, rebuilt when
// the set of members still short of their step budget changes, and a CUDA
// graph of `chunk` batched steps, captured once per work-list.
struct cemx_batch {
    struct Member {
        cem_sim *s;
        long left;   // steps still to run
    };
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Member> members;
    std::vector<int> active;                 // members in the work-lists
    DevBuf<StepArgs> args;
    DevBuf<SibcArgs> sargs;
    DevBuf<PostArgs> pargs;
    DevBuf<int4> work_h[2];                  // H blocks: fast, general
    DevBuf<int4> work_ef;                    // E fast blocks of all members
    std::map<int, DevBuf<int4>> work_e;      // E general blocks, by pole count
    DevBuf<int2> work_s;
    size_t nh[2] = {0, 0}, nef = 0, ns = 0;
    std::map<int, size_t> ne;
    bool dirty = true;
    int order = 0;                           // work-list order: 0 member-major, 1 plane-interleaved
    int chunk = 256;                         // steps between the host's checks of budgets and rings
    bool tune = false, tuned = false;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;   // timing of the tuning chunks
    cudaStream_t side = nullptr;             // general blocks beside the fast ones; SIBC beside the probes
    bool sibc_beside = false;                // no member's probes read a SIBC edge
    cudaEvent_t fork = nullptr, join = nullptr;
    double last_ms = 0;
    long last_steps = 0, last_launches = 0;
};

namespace {

bool batch_fail(const char *what, cudaError_t e) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "batch: CUDA %s: %s", what, cudaGetErrorString(e));
    set_error(msg);
    return false;
}
#define CB2_BCHECK(call)                                   \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return batch_fail(#call, e_); \
    } while (0)

template <class T>
bool batch_upload(DevBuf<T> &b, const std::vector<T> &v) {
    if (b.p) { cudaFree(b.p); b.p = nullptr; b.n = 0; }
    if (v.empty()) return true;
    CB2_BCHECK(cudaMalloc(&b.p, v.size() * sizeof(T)));
    b.n = v.size();
    CB2_BCHECK(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return true;
}

void batch_drop_graph(cemx_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
}

// work-lists of the members still short of their budget
bool batch_rebuild(cemx_batch *b) {
    batch_drop_graph(b);
    b->active.clear();
    for (int m = 0; m < (int)b->members.size(); m++)
        if (b->members[m].left > 0) b->active.push_back(m);
    std::vector<StepArgs> sa;
    std::vector<SibcArgs> sb;
    std::vector<PostArgs> pa;
    std::vector<int4> wh[2], wef;
    std::map<int, std::vector<int4>> we;
    std::vector<int2> ws;
    int maxp = 0;
    for (int x = 0; x < (int)b->active.size(); x++) {
        cem_sim *s = b->members[b->active[x]].s;
        Device &D = *s->dev;
        sa.push_back(D.sa[D.cur]);
        sb.push_back(D.sb[D.cur]);
        pa.push_back(D.pa[D.cur]);
        pa.back().advance = 1;
        maxp = std::max(maxp, s->n[0] + 1);
        for (int e0 = 0; e0 < s->nsb; e0 += kBlock) ws.push_back(make_int2(x, e0));
    }
    // H over planes 0..nx, E over 0..nx-1; member-major, or plane by plane
    // across members; fast and general blocks as the member's own lists
    auto add_plane = [&](int x, int i) {
        cem_sim *s = b->members[b->active[x]].s;
        const Device &D = *s->dev;
        // interior planes: the fast and the general space; elsewhere every rectangle
        auto blocks = [&](int u, int c) { return 3 * space_blocks(D.sp[u][c]); };
        const bool ih = i >= D.p0[0] && i < D.p1[0], ie = i >= D.p0[1] && i < D.p1[1];
        if (i <= s->n[0]) {
            for (int bx = 0; ih && bx < blocks(0, kFast); bx++) wh[0].push_back(make_int4(x, bx, i, 0));
            for (int bx = 0; bx < blocks(0, ih ? kGeneral : kAll); bx++) wh[1].push_back(make_int4(x, bx, i, 0));
        }
        if (i < s->n[0]) {
            for (int bx = 0; ie && bx < blocks(1, kFast); bx++) wef.push_back(make_int4(x, bx, i, 0));
            for (int bx = 0; bx < blocks(1, ie ? kGeneral : kAll); bx++)
                we[s->npole].push_back(make_int4(x, bx, i, 0));
            for (int bx = 0; ie && bx < blocks(1, kDebye); bx++) we[s->npole].push_back(make_int4(x, bx, i, 1));
        }
    };
    if (b->order == 0) {
        for (int x = 0; x < (int)b->active.size(); x++)
            for (int i = 0; i <= b->members[b->active[x]].s->n[0]; i++) add_plane(x, i);
    } else {
        for (int i = 0; i < maxp; i++)
            for (int x = 0; x < (int)b->active.size(); x++) add_plane(x, i);
    }
    if (!batch_upload(b->args, sa) || !batch_upload(b->sargs, sb) || !batch_upload(b->pargs, pa) ||
        !batch_upload(b->work_h[0], wh[0]) || !batch_upload(b->work_h[1], wh[1]) || !batch_upload(b->work_ef, wef) ||
        !batch_upload(b->work_s, ws))
        return false;
    b->work_e.clear();
    b->ne.clear();
    for (auto &kv : we) {
        if (!batch_upload(b->work_e[kv.first], kv.second)) return false;
        b->ne[kv.first] = kv.second.size();
    }
    b->sibc_beside = true;
    for (int m : b->active) b->sibc_beside = b->sibc_beside && b->members[m].s->dev->post_beside_sibc;
    b->nh[0] = wh[0].size();
    b->nh[1] = wh[1].size();
    b->nef = wef.size();
    b->ns = ws.size();
    b->dirty = false;
    return true;
}

// blocks of a batched update launch over n work entries
unsigned blocks_for(size_t n) { return (unsigned)((n + kPerBlock - 1) / kPerBlock); }

// one batched time step: H (fast, general blocks), E (fast blocks; general
// blocks one launch per pole count), SIBC, probes
int batch_step(cemx_batch *b) {
    int launches = 0;
    // general blocks on the side stream beside the fast ones, joined before the next phase
    auto fork = [&]() {
        cudaEventRecord(b->fork, b->stream);
        cudaStreamWaitEvent(b->side, b->fork, 0);
    };
    auto join = [&]() {
        cudaEventRecord(b->join, b->side);
        cudaStreamWaitEvent(b->stream, b->join, 0);
    };
    if (b->nh[1]) {
        fork();
        k_batch_h<false><<<blocks_for(b->nh[1]), kBlock, 0, b->side>>>(b->args.p, b->work_h[1].p, (int)b->nh[1]);
        launches++;
    }
    if (b->nh[0]) {
        k_batch_h<true><<<blocks_for(b->nh[0]), kBlock, 0, b->stream>>>(b->args.p, b->work_h[0].p, (int)b->nh[0]);
        launches++;
    }
    if (b->nh[1]) join();
    bool side = false;
    for (auto &kv : b->ne)
        if (kv.second) {
            if (!side) fork();
            side = true;
            kBEKernels[kv.first]<<<blocks_for(kv.second), kBlock, 0, b->side>>>(b->args.p, b->work_e[kv.first].p,
                                                                               (int)kv.second);
            launches++;
        }
    if (b->nef) {
        k_batch_e<0, true><<<blocks_for(b->nef), kBlock, 0, b->stream>>>(b->args.p, b->work_ef.p, (int)b->nef);
        launches++;
    }
    if (side) join();
    const bool beside = b->ns && b->sibc_beside;
    if (beside) fork();
    if (b->ns) {
        k_batch_sibc<<<(unsigned)b->ns, kBlock, 0, beside ? b->side : b->stream>>>(b->sargs.p, b->work_s.p);
        launches++;
    }
    k_batch_post<<<(unsigned)b->active.size(), kPostThreads, 0, b->stream>>>(b->pargs.p);
    if (beside) join();
    return launches + 1;
}

// n batched steps, through the cached graph when n is the chunk length
// n batched steps: whole runs of kBatchGraph steps replay the graph captured
// for the current composition (captured once per composition, so a change of
// members costs one short capture), the rest go step by step
constexpr int kBatchGraph = 16;

bool batch_launch(cemx_batch *b, int n) {
    if (n >= kBatchGraph) {
        if (!b->graph || b->graph_steps != kBatchGraph) {
            batch_drop_graph(b);
            cudaGraph_t g = nullptr;
            CB2_BCHECK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            for (int q = 0; q < kBatchGraph; q++) batch_step(b);
            CB2_BCHECK(cudaStreamEndCapture(b->stream, &g));
            const cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) { b->graph = nullptr; return batch_fail("cudaGraphInstantiate", e); }
            b->graph_steps = kBatchGraph;
        }
        for (int q = 0; q + kBatchGraph <= n; q += kBatchGraph) {
            CB2_BCHECK(cudaGraphLaunch(b->graph, b->stream));
            b->last_launches += 1;
        }
    }
    for (int q = n / kBatchGraph * kBatchGraph; q < n; q++) b->last_launches += batch_step(b);
    CB2_BCHECK(cudaGetLastError());
    return true;
}

// Per-composition choice of chunk length and work-list order, found by timing
// real batched steps once and kept for the process.
std::mutex g_tune_mu;
std::map<std::string, std::pair<int, int>> g_tuned;

// cache-file key of a batch composition: FNV-1a hash of its signature and the member count
std::string batch_key(const std::string &sig) {
    unsigned long long h = 1469598103934665603ull;
    int members = 0;
    for (char c : sig) {
        h = (h ^ (unsigned char)c) * 1099511628211ull;
        members += c == ';';
    }
    char k[64];
    std::snprintf(k, sizeof k, "batch/%016llx/%d", h, members);
    return k;
}

std::string batch_signature(const cemx_batch *b) {
    std::vector<std::string> v;
    for (int m : b->active) {
        const cem_sim *s = b->members[m].s;
        char k[96];
        std::snprintf(k, sizeof k, "%dx%dx%d/p%d/s%d", s->n[0], s->n[1], s->n[2], s->npole, s->nsb);
        v.push_back(k);
    }
    std::sort(v.begin(), v.end());
    std::string sig;
    for (auto &x : v) sig += x + ";";
    return sig;
}

}  // namespace

extern "C" {

int cemx_step_timed(cem_sim *s, long n, double *gpu_ms) {
    if (!s->finalized) { set_error("not finalized"); return -1; }
    return timed_steps(s, n, gpu_ms) ? 0 : -1;
}

int cemx_profile_steps(cem_sim *s, long n, double *kernel_ms, long *launches) {
    if (!s->finalized) { set_error("not finalized"); return -1; }
    return profiled_steps(s, n, kernel_ms, launches) ? 0 : -1;
}

int cemx_sizes(const cem_sim *s, long long *out, int n) {
    if (!s->finalized) { set_error("not finalized"); return -1; }
    long long v[19] = {0};
    v[0] = (long long)s->n[0] * s->n[1] * s->n[2];
    v[1] = (long long)s->N;
    for (int c = 0; c < 3; c++)
        for (int w = 0; w < 2; w++) {
            v[2] += (long long)psi_len(s, 1, c, w);
            v[3] += (long long)psi_len(s, 0, c, w);
        }
    v[4] = s->ndisp;
    v[5] = s->npole;
    v[6] = s->nsb;
    v[7] = s->sibc_npole;
    if (s->dev) {
        for (int c = 0; c < 3; c++) v[8 + c] = s->dev->ntab[c];
        long long bytes = 0;
        const Device &D = *s->dev;
        for (int c = 0; c < 3; c++) {
            bytes += (long long)(2 * D.E[0][c].n + 2 * D.H[0][c].n + D.hc[c].n + D.ec[c].n) * 4 +
                     (long long)D.mat[c].n * 2 + (long long)D.tab[c].n * 4 + (long long)D.J[c].n * 4;
            for (int w = 0; w < 2; w++) bytes += (long long)(D.psiE[c][w].n + 2 * D.psiH[0][c][w].n) * 4;
        }
        bytes += (long long)D.sb_y.n * 4 + (long long)(D.sb_hw.n + D.sb_hidx.n) * 16 + (long long)D.sb_eidx.n * 4 +
                 (long long)(D.ring.n + D.acc.n) * 8;
        v[11] = bytes;
    }
    // kernels per step: H and E, each over its fast and general blocks (or one
    // fused kernel), SIBC when present, the probe pass
    int upd = 4;
    if (s->dev && s->dev->use_fused) upd = 1;
    else if (s->dev)
        for (int u = 0; u < 2; u++) {
            const Device &D = *s->dev;
            upd -= space_blocks(D.sp[u][kFast]) == 0 || D.p1[u] <= D.p0[u];
            upd -= D.wl_start[u].empty() || D.wl_start[u].back() == 0;
            upd += u == 1 && space_blocks(D.sp[u][kDebye]) > 0 && D.p1[u] > D.p0[u];
        }
    v[12] = upd + 1 + (s->nsb ? 1 : 0);
    // point-components each update class covers per step (4 points per thread,
    // 3 components): H fast, H general, E fast, E general, E Debye; and the
    // Debye boxes' points (pole currents move for all of them)
    if (s->dev) {
        const Device &D = *s->dev;
        for (int u = 0; u < 2; u++) {
            const long long inner = std::max(0, D.p1[u] - D.p0[u]), planes = u ? s->n[0] : s->n[0] + 1;
            auto pts = [&](int c) { return 12LL * D.sp[u][c].t0[D.sp[u][c].n]; };
            const bool split = space_blocks(D.sp[u][kFast]) + space_blocks(D.sp[u][kDebye]) > 0 && inner > 0;
            const long long fast = split ? pts(kFast) * inner : 0, deb = split ? pts(kDebye) * inner : 0;
            const long long gen = split ? pts(kGeneral) * inner + pts(kAll) * (planes - inner) : pts(kAll) * planes;
            v[13 + 2 * u] = fast;
            v[14 + 2 * u] = gen;
            if (u == 1) v[17] = deb;
        }
        for (int c = 0; c < 3; c++) v[18] += (long long)D.jbox[c][3] * D.jbox[c][4] * D.jbox[c][5];
    }
    for (int q = 0; q < n && q < 19; q++) out[q] = v[q];
    return 0;
}

int cemx_select_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        set_error("no such CUDA device");
        return -1;
    }
    g_selected_device = device;
    return 0;
}

int cemx_prepare_device(cem_sim *s, int device) {
    if (!s || !s->finalized) { set_error("not finalized"); return -1; }
    const int prev = g_selected_device;
    if (device >= 0) g_selected_device = device;
    const bool ok = begin_device_op(s) && end_device_op(s);
    g_selected_device = prev;
    return ok ? 0 : -1;
}

int cemx_release_device(cem_sim *s) {
    if (!s->dev) return 0;
    if (engine_pull(s, kGroupAll)) return -1;
    s->dev.reset();
    s->dev_valid = 0;
    return 0;
}

int cemx_use_fused(cem_sim *s, int on) {
    const int prev = s->dev ? (s->dev->use_fused ? 1 : 0) : (s->kernel_choice >= 0 ? s->kernel_choice : 0);
    s->kernel_choice = on ? 1 : 0;
    if (s->dev) s->dev->use_fused = on != 0;
    return prev;
}

int cemx_tune(cem_sim *s, int on) {
    if (!s) { set_error("null simulation"); return -1; }
    const int prev = s->dev ? (s->dev->tune ? 1 : 0) : (s->tune_choice >= 0 ? s->tune_choice : 0);
    s->tune_choice = on ? 1 : 0;
    if (s->dev) s->dev->tune = on != 0;
    return prev;
}

int cemx_tune_state(const cem_sim *s, double *out, int n) {
    if (!s || !out) { set_error("null argument"); return -1; }
    double v[7] = {0, 0, 16, 1, 32, 0, 1};
    if (s->dev) {
        const Device &D = *s->dev;
        v[0] = D.tuned;
        v[1] = D.tuned_from_cache;
        v[2] = D.thin;
        v[3] = D.side_on;
        v[4] = D.graph_steps;
        v[5] = D.tuned_ms;
        v[6] = D.ztail;
    }
    for (int q = 0; q < n && q < 7; q++) out[q] = v[q];
    return 0;
}

int cemx_energy_noalloc(cem_sim *s, double *out) {
    if (!s || !out) { set_error("cemx_energy_noalloc: null argument"); return -1; }
    if (!s->finalized) { set_error("not finalized"); return -1; }
    return energy_noalloc(s, out) ? 0 : -1;
}


cemx_batch *cemx_batch_create(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        set_error("no CUDA device: libcourant_b200 steps only on the GPU");
        return nullptr;
    }
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) { set_error("no current CUDA device"); return nullptr; }
    if (device >= n) { set_error("no such CUDA device"); return nullptr; }
    cemx_batch *b = new cemx_batch;
    b->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaEventCreate(&b->tev0) != cudaSuccess || cudaEventCreate(&b->tev1) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess) {
        set_error("batch: cannot create its stream");
        cemx_batch_destroy(b);
        return nullptr;
    }
    return b;
}

void cemx_batch_destroy(cemx_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    b->work_e.clear();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->tev0) cudaEventDestroy(b->tev0);
    if (b->tev1) cudaEventDestroy(b->tev1);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int cemx_batch_add(cemx_batch *b, cem_sim *s, long steps) {
    if (!b || !s) { set_error("batch: null argument"); return -1; }
    if (!s->finalized) { set_error("not finalized"); return -1; }
    if (steps < 0) { set_error("batch: negative step count"); return -1; }
    for (auto &m : b->members)
        if (m.s == s) { set_error("batch: simulation already a member"); return -1; }
    const int prev = g_selected_device;
    g_selected_device = b->device;
    const bool ok = create_device(s);
    g_selected_device = prev;
    if (!ok) return -1;
    if (s->dev->device != b->device) { set_error("batch: simulation lives on another device"); return -1; }
    b->members.push_back({s, steps});
    b->dirty = true;
    return (int)b->members.size() - 1;
}

int cemx_batch_remove(cemx_batch *b, cem_sim *s) {
    if (!b) { set_error("batch: null argument"); return -1; }
    for (size_t m = 0; m < b->members.size(); m++)
        if (b->members[m].s == s) {
            cudaSetDevice(b->device);
            cudaStreamSynchronize(b->stream);
            b->members.erase(b->members.begin() + m);
            b->dirty = true;
            return 0;
        }
    set_error("batch: not a member");
    return -1;
}

long cemx_batch_left(const cemx_batch *b, const cem_sim *s) {
    if (!b) return -1;
    for (const auto &m : b->members)
        if (m.s == s) return m.left;
    return -1;
}

int cemx_batch_tune(cemx_batch *b, int on) {
    if (!b) return -1;
    const int prev = b->tune ? 1 : 0;
    b->tune = on != 0;
    b->tuned = false;
    return prev;
}

int cemx_batch_run(cemx_batch *b, long max_steps) {
    if (!b) { set_error("batch: null argument"); return -1; }
    if (cudaSetDevice(b->device) != cudaSuccess) { set_error("batch: cannot select its device"); return -1; }
    std::vector<cem_sim *> touched;
    for (auto &m : b->members)
        if (m.left > 0) {
            if (!begin_device_op(m.s)) return -1;
            touched.push_back(m.s);
        }
    b->last_ms = 0;
    b->last_steps = 0;
    b->last_launches = 0;
    if (cudaEventRecord(b->ev0, b->stream) != cudaSuccess) { set_error("batch: event"); return -1; }
    long done = 0;
    while (done < max_steps) {
        if (b->dirty && !batch_rebuild(b)) return -1;
        if (b->active.empty()) break;
        if (b->tune && !b->tuned) {
            // chunk length and work-list order: cached per composition, else timed on real steps
            const std::string sig = batch_signature(b);
            std::pair<int, int> best{b->chunk, b->order};
            bool cached = false;
            {   // this process's choices, then the launch-shape cache file
                std::lock_guard<std::mutex> lock(g_tune_mu);
                auto it = g_tuned.find(sig);
                if (it != g_tuned.end()) { best = it->second; cached = true; }
            }
            if (!cached) {
                std::lock_guard<std::mutex> lock(g_shape_mu);
                load_shapes();
                auto it = g_shapes.find(batch_key(sig));
                if (it != g_shapes.end()) { best = {(int)it->second[0], (int)it->second[1]}; cached = true; }
            }
            if (!cached) {
                long minleft = max_steps - done;
                for (int m : b->active) minleft = std::min(minleft, b->members[m].left);
                float best_ms = 1e30f;
                for (int order = 0; order < 2; order++)
                    for (int ch : {64}) {
                        if (2 * ch > minleft) continue;   // one warm-up and one timed chunk
                        if (b->order != order) { b->order = order; if (!batch_rebuild(b)) return -1; }
                        b->chunk = ch;
                        float ms = 0;
                        for (int rep = 0; rep < 2; rep++) {
                            for (int m : b->active) {
                                Device &D = *b->members[m].s->dev;
                                if (D.ring_count + ch > kRing) {
                                    const cudaError_t e = cudaStreamSynchronize(b->stream);
                                    if (e != cudaSuccess) { batch_fail("cudaStreamSynchronize", e); return -1; }
                                    if (!flush_dft(b->members[m].s) || cudaStreamSynchronize(D.stream) != cudaSuccess)
                                        return -1;
                                }
                            }
                            cudaError_t e = cudaEventRecord(b->tev0, b->stream);
                            if (e != cudaSuccess) { batch_fail("cudaEventRecord", e); return -1; }
                            if (!batch_launch(b, ch)) return -1;
                            if ((e = cudaEventRecord(b->tev1, b->stream)) != cudaSuccess ||
                                (e = cudaEventSynchronize(b->tev1)) != cudaSuccess ||
                                (e = cudaEventElapsedTime(&ms, b->tev0, b->tev1)) != cudaSuccess)
                            { batch_fail("tuning timer", e); return -1; }
                            for (int m : b->active) {
                                b->members[m].s->step += ch;
                                b->members[m].s->dev->ring_count += ch;
                                b->members[m].left -= ch;
                            }
                            done += ch;
                            minleft -= ch;
                            b->last_steps += ch;
                        }
                        if (ms / ch < best_ms) { best_ms = ms / ch; best = {ch, order}; }
                    }
                {
                    std::lock_guard<std::mutex> lock(g_tune_mu);
                    g_tuned[sig] = best;
                }
                std::lock_guard<std::mutex> lock(g_shape_mu);
                store_shape(batch_key(sig), {(double)best.first, (double)best.second, 0.0, best_ms});
            }
            b->tuned = true;
            if (b->order != best.second) { b->order = best.second; b->dirty = true; }
            for (int m : b->active)
                if (b->members[m].left <= 0) b->dirty = true;
            continue;
        }
        long n = std::min<long>(b->chunk, max_steps - done);
        for (int m : b->active) n = std::min(n, b->members[m].left);
        for (int m : b->active) {
            Device &D = *b->members[m].s->dev;
            if (D.ring_count + n > kRing) {   // room in the sample ring for n rows
                cudaStreamSynchronize(b->stream);
                if (!flush_dft(b->members[m].s) || cudaStreamSynchronize(D.stream) != cudaSuccess) return -1;
            }
        }
        if (!batch_launch(b, (int)n)) return -1;
        for (int m : b->active) {
            cemx_batch::Member &mb = b->members[m];
            mb.s->step += n;
            mb.s->dev->ring_count += n;
            mb.left -= n;
            if (mb.left == 0) b->dirty = true;
        }
        done += n;
        b->last_steps += n;
    }
    float ms = 0;
    if (cudaEventRecord(b->ev1, b->stream) != cudaSuccess || cudaEventSynchronize(b->ev1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, b->ev0, b->ev1) != cudaSuccess) {
        set_error("batch: a batched launch failed");
        return -1;
    }
    b->last_ms = ms;
    for (cem_sim *s : touched)
        if (!end_device_op(s)) return -1;
    int left = 0;
    for (auto &m : b->members) left += m.left > 0;
    return left;
}

int cemx_batch_stats(const cemx_batch *b, double *out, int n) {
    if (!b) return -1;
    const double v[6] = {b->last_ms, (double)b->last_steps, (double)b->last_launches, (double)kBatchGraph,
                         (double)b->order, (double)b->members.size()};
    for (int q = 0; q < n && q < 6; q++) out[q] = v[q];
    return 0;
}

int cemx_synchronize(cem_sim *s) {
    if (!s->dev) return 0;
    cudaError_t e = cudaStreamSynchronize(s->dev->stream);
    if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

}  // extern "C"
