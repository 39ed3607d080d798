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
#include "../../include/courant_b200.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace cb2 {

constexpr int kRing = 1024;          // sample rows kept on the device between DFT flushes
constexpr int kBlock = 256;
constexpr int kMaxSlots = 2 * kMaxProbes + kMaxPorts;
constexpr unsigned kFlagDisp = 1, kFlagSrc = 2;

// ---------------------------------------------------------------- arguments

// Device index space: rows padded to 16 bytes, q = i*si + j*sj + k with
// sj = round_up(nz+1, 4) and si = (ny+1)*sj; padding elements (k > nz) stay
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
    int per;                             // points per plane
    int planes;                          // planes in the CPML slabs of this axis (z-axis layout stride)
};

// Device layout of the CPML auxiliaries: x and y slabs as in the reference
// (plane-major, then the in-plane index); z slabs with the plane index
// fastest, ((i*(ny+1) + j) * planes + plane), so the z-slab cells of one k
// row sit next to each other. Host copies use the reference layout.

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
    const unsigned char *tflag[3];
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
};

struct SibcArgs {
    int ns, K;
    const int *ecomp;
    const long long *eidx;
    const int *hcomp;        // 4 per edge
    const long long *hidx;   // 4 per edge
    const float *hw;         // 4 per edge (0 beyond the face count)
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
    const long long *eidx;
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
    int advance;             // 1: count this step
};

// --------------------------------------------------------------- helpers

__device__ __forceinline__ double gauss(double t, double amp, double t0, double tau) {
    const double x = (t - t0) / tau;
    return amp * exp(-x * x);
}

__device__ __forceinline__ double dgauss(double t, double t0, double tau) {
    const double x = (t - t0) / tau;
    return -2 * x * exp(-x * x);
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

// compact index of a CPML auxiliary for derivative axis A (device layout, see PmlAxis)
template <int A>
__device__ __forceinline__ int psi_at(const StepArgs &a, int plane, int i, int j, int k) {
    if (A == 0) return plane * a.pml[0].per + j * (a.g.n[2] + 1) + k;
    if (A == 1) return plane * a.pml[1].per + i * (a.g.n[2] + 1) + k;
    return (i * (a.g.n[1] + 1) + j) * a.pml[2].planes + plane;
}

// H component C at (i, j, k) (reference sim.c:579-606, CPML :680-754):
//   H_C -= dt/mu0 [ (d1 c1 + psi_{C,0}) - (d2 c2 + psi_{C,1}) ]
// with d1 = dE_{C+2} along axis C+1, d2 = dE_{C+1} along axis C+2, c1, c2 the
// kappa-scaled inverse cell sizes times dt/mu0, p1, p2 the CPML planes of the
// two derivative axes (-1 outside). psi read from `pin`, written to `pout`
// when STORE.
template <int C, bool STORE>
__device__ __forceinline__ float h_comp(const StepArgs &a, float *const (&pin)[3][2], float *const (&pout)[3][2],
                                        int i, int j, int k, float h, float d1, float d2, float c1, float c2, int p1,
                                        int p2) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int idx[3] = {i, j, k};
    float t1 = __fmul_rn(d1, c1), t2 = __fmul_rn(d2, c2);
    if (p1 >= 0) {
        const int x = psi_at<A1>(a, p1, i, j, k);
        const float psi = psi_next(pin[C][0][x], a.pml[A1].bm1_h[idx[A1]], a.pml[A1].cid_h[idx[A1]], d1);
        if (STORE) pout[C][0][x] = psi;
        t1 = __fmaf_rn(a.dth, psi, t1);
    }
    if (p2 >= 0) {
        const int x = psi_at<A2>(a, p2, i, j, k);
        const float psi = psi_next(pin[C][1][x], a.pml[A2].bm1_h[idx[A2]], a.pml[A2].cid_h[idx[A2]], d2);
        if (STORE) pout[C][1][x] = psi;
        t2 = __fmaf_rn(a.dth, psi, t2);
    }
    return __fsub_rn(h, __fsub_rn(t1, t2));
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

// Per-edge epilogue: material table, Debye correction and update, sources.
//   E = E + (ca-1) E + cb [curl - sum_p hk_p J_p] + cs Vs(t) + w Vm(t)
//   J_p += -(1-k_p) J_p + beta_p/dt (E_new - E_old)
// P (the number of Debye poles) is a template parameter so the pole loops
// unroll and the currents stay in registers.
// (reference sim.c:608-637, :894-910; dispersive.c:93-112; modeport.c:130-135)
template <int C, int P>
__device__ __forceinline__ float e_finish(const StepArgs &a, int mi, float e_old, float curl, int i, int j, int k,
                                          long long step) {
    const float4 t = __ldg(a.tab4[C] + mi);   // ca-1, cb, cs, flags
    const unsigned flag = __float_as_uint(t.w);
    const float base = __fmaf_rn(t.x, e_old, e_old);
    if (!flag) return __fmaf_rn(t.y, curl, base);
    int jo = 0, jvol = 0;
    float jv[P > 0 ? P : 1];
    if (P > 0 && (flag & kFlagDisp)) {
        const int *bx = a.jbox[C];
        jvol = bx[3] * bx[4] * bx[5];
        jo = ((i - bx[0]) * bx[4] + (j - bx[1])) * bx[5] + (k - bx[2]);
        float acc = 0.f;
#pragma unroll
        for (int p = 0; p < P; p++) {
            jv[p] = a.J[C][p * jvol + jo];
            acc = __fmaf_rn(a.hk[p], jv[p], acc);
        }
        curl = __fsub_rn(curl, acc);
    }
    float e = __fmaf_rn(t.y, curl, base);
    if (flag & kFlagSrc) {
        const double tH = ((double)step + 0.5) * a.dt;
        e = __fmaf_rn(t.z, (float)gauss(tH, a.src_amp, a.src_t0, a.src_tau), e);
    }
    if (C > 0 && a.msrc_on && i == a.i_src) {
        const float w = a.wsrc[C - 1][j * (a.g.n[2] + 1) + k];
        if (w != 0.f) {
            const double tH = ((double)step + 0.5) * a.dt;
            e = __fmaf_rn(w, (float)dgauss(tH, a.m_t0, a.m_tau), e);
        }
    }
    if (P > 0 && (flag & kFlagDisp)) {
        const float de = __fsub_rn(e, e_old);
        const int nt = a.ntab[C];
#pragma unroll
        for (int p = 0; p < P; p++) {
            const float bidt = __ldg(a.tab[C] + (3 + p) * nt + mi);
            a.J[C][p * jvol + jo] = __fmaf_rn(bidt, de, __fmaf_rn(-a.omk[p], jv[p], jv[p]));
        }
    }
    return e;
}

// E component C at (i, j, k) (reference sim.c:608-637, CPML :756-832):
//   E_C = ca E + cb [ (d1 c1 + psi_{C,0}) - (d2 c2 + psi_{C,1}) ] + epilogue
// with d1 = dH_{C+2} along axis C+1, d2 = dH_{C+1} along axis C+2.
template <int C, int P>
__device__ __forceinline__ float e_comp(const StepArgs &a, int i, int j, int k, long long step, float e, float d1,
                                        float d2, float c1, float c2, int p1, int p2, int mi) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int idx[3] = {i, j, k};
    float t1 = __fmul_rn(d1, c1), t2 = __fmul_rn(d2, c2);
    if (p1 >= 0) {
        float *arr = a.psiE[C][0];
        const int x = psi_at<A1>(a, p1, i, j, k);
        const float psi = psi_next(arr[x], a.pml[A1].bm1_e[idx[A1]], a.pml[A1].cid_e[idx[A1]], d1);
        arr[x] = psi;
        t1 = __fadd_rn(t1, psi);
    }
    if (p2 >= 0) {
        float *arr = a.psiE[C][1];
        const int x = psi_at<A2>(a, p2, i, j, k);
        const float psi = psi_next(arr[x], a.pml[A2].bm1_e[idx[A2]], a.pml[A2].cid_e[idx[A2]], d2);
        arr[x] = psi;
        t2 = __fadd_rn(t2, psi);
    }
    return e_finish<C, P>(a, mi, e, __fsub_rn(t1, t2), i, j, k, step);
}

// All three E components at (i, j, k) for the fused step. h*: H at the point;
// *_jm, *_km: at j-1, k-1; hy_p, hz_p: at i-1. e* in: old, out: new.
template <int P>
__device__ __forceinline__ void e_point(const StepArgs &a, const Column &col, const Plane &pl, int i, int j, int k,
                                        long long step, float hx, float hy, float hz, float hz_jm, float hx_jm,
                                        float hy_km, float hx_km, float hy_p, float hz_p, int m0, int m1, int m2,
                                        float &ex, float &ey, float &ez) {
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    if (i >= nx) return;
    const bool jin = j >= 1 && j < ny, kin = k >= 1 && k < nz;
    if (jin && kin)
        ex = e_comp<0, P>(a, i, j, k, step, ex, __fsub_rn(hz, hz_jm), __fsub_rn(hy, hy_km), col.ecy, col.ecz, col.pej,
                       col.pek, m0);
    if (i < 1) return;
    if (j < ny && kin)
        ey = e_comp<1, P>(a, i, j, k, step, ey, __fsub_rn(hx, hx_km), __fsub_rn(hz, hz_p), col.ecz, pl.ecx, col.pek,
                       pl.pei, m1);
    if (jin && k < nz)
        ez = e_comp<2, P>(a, i, j, k, step, ez, __fsub_rn(hy, hy_p), __fsub_rn(hx, hx_jm), pl.ecx, col.ecy, pl.pei,
                       col.pej, m2);
}

// ------------------------------------------------ separate phase kernels
//
// One thread per field component of a (j,k) column, marching over kU node
// planes along x with the loads of all kU planes issued before any
// arithmetic. The three components of a chunk of the plane sit in adjacent
// blocks, so the neighbour values they share come from L2.

constexpr int kU = 4;

template <int A>
__device__ __forceinline__ int stride_of(const StepArgs &a) {
    return A == 0 ? (int)a.g.si : (A == 1 ? a.g.sj : 1);
}

template <int C>
__device__ __forceinline__ void h_march(const StepArgs &a, int ib, int ie, int j, int k, int m) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int jk[3] = {0, j, k};
    if ((A1 != 0 && jk[A1] >= a.g.n[A1]) || (A2 != 0 && jk[A2] >= a.g.n[A2]) || k > nz) return;
    const int last = (A1 == 0 || A2 == 0) ? min(ie, nx) : ie;   // an x-derivative needs plane i+1
    const int si = (int)a.g.si, s1 = stride_of<A1>(a), s2 = stride_of<A2>(a);
    const float *__restrict__ E2 = a.E[A2];
    const float *__restrict__ E1 = a.E[A1];
    float *__restrict__ H = a.H[C];
    float e2[kU], e2n[kU], e1[kU], e1n[kU], h[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
        const int q = (ib + u) * si + m;
        if (ib + u < last) {
            e2[u] = E2[q]; e2n[u] = E2[q + s1]; e1[u] = E1[q]; e1n[u] = E1[q + s2]; h[u] = H[q];
        }
    }
    const float cj = a.hc[1][min(j, ny - 1)], ck = a.hc[2][min(k, nz - 1)];
    const int pj = a.has_pml && j < ny ? a.pml[1].plane_h[j] : -1, pk = a.has_pml && k < nz ? a.pml[2].plane_h[k] : -1;
#pragma unroll
    for (int u = 0; u < kU; u++) {
        const int i = ib + u;
        if (i >= last) break;
        const float ci = a.hc[0][min(i, nx - 1)];
        const int pi = a.has_pml && i < nx ? a.pml[0].plane_h[i] : -1;
        const float c[3] = {ci, cj, ck};
        const int pp[3] = {pi, pj, pk};
        H[i * si + m] = h_comp<C, true>(a, a.psiH, a.psiH, i, j, k, h[u], __fsub_rn(e2n[u], e2[u]),
                                        __fsub_rn(e1n[u], e1[u]), c[A1], c[A2], pp[A1], pp[A2]);
    }
}

template <int C, int P>
__device__ __forceinline__ void e_march(const StepArgs &a, int ib, int ie, int j, int k, int m, long long step) {
    constexpr int A1 = (C + 1) % 3, A2 = (C + 2) % 3;
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int jk[3] = {0, j, k};
    // own axis: index < n; transverse axes: 1 <= index < n
    if (C != 0 && jk[C] >= a.g.n[C]) return;
    if (A1 != 0 && (jk[A1] < 1 || jk[A1] >= a.g.n[A1])) return;
    if (A2 != 0 && (jk[A2] < 1 || jk[A2] >= a.g.n[A2])) return;
    const int first = C == 0 ? ib : max(ib, 1), last = min(ie, nx);
    const int si = (int)a.g.si, s1 = stride_of<A1>(a), s2 = stride_of<A2>(a);
    const float *__restrict__ H2 = a.H[A2];
    const float *__restrict__ H1 = a.H[A1];
    float *__restrict__ E = a.E[C];
    const unsigned short *__restrict__ M = a.mat[C];
    float h2[kU], h2m[kU], h1[kU], h1m[kU], e[kU];
    int mi[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
        const int i = ib + u, q = i * si + m;
        if (i >= first && i < last) {
            h2[u] = H2[q]; h2m[u] = H2[q - s1]; h1[u] = H1[q]; h1m[u] = H1[q - s2]; e[u] = E[q]; mi[u] = M[q];
        }
    }
    const float cj = a.ec[1][j], ck = a.ec[2][k];
    const int pj = a.has_pml ? a.pml[1].plane_e[j] : -1, pk = a.has_pml ? a.pml[2].plane_e[k] : -1;
#pragma unroll
    for (int u = 0; u < kU; u++) {
        const int i = ib + u;
        if (i < first || i >= last) continue;
        const float c[3] = {a.ec[0][i], cj, ck};
        const int pp[3] = {a.has_pml ? a.pml[0].plane_e[i] : -1, pj, pk};
        E[i * si + m] = e_comp<C, P>(a, i, j, k, step, e[u], __fsub_rn(h2[u], h2m[u]), __fsub_rn(h1[u], h1m[u]),
                                     c[A1], c[A2], pp[A1], pp[A2], mi[u]);
    }
}

// H over node planes [i0, i1) (cem_mt_H and the unfused step)
__global__ void __launch_bounds__(kBlock, 6) k_update_h(const StepArgs a, int i0, int i1) {
    const int comp = blockIdx.x % 3;
    const int m = (blockIdx.x / 3) * kBlock + threadIdx.x;
    if (m >= a.g.plane) return;
    const int ib = i0 + blockIdx.y * kU, ie = min(ib + kU, i1);
    const int j = (int)(((unsigned long long)m * a.g.sj_magic) >> 40);
    const int k = m - j * a.g.sj;
    if (comp == 0) h_march<0>(a, ib, ie, j, k, m);
    else if (comp == 1) h_march<1>(a, ib, ie, j, k, m);
    else h_march<2>(a, ib, ie, j, k, m);
}

// E over node planes [i0, i1) (cem_mt_E and the unfused step)
template <int P>
__global__ void __launch_bounds__(kBlock, 3) k_update_e(const StepArgs a, int i0, int i1) {
    const int comp = blockIdx.x % 3;
    const int m = (blockIdx.x / 3) * kBlock + threadIdx.x;
    if (m >= a.g.plane) return;
    const int ib = i0 + blockIdx.y * kU, ie = min(ib + kU, i1);
    const int j = (int)(((unsigned long long)m * a.g.sj_magic) >> 40);
    const int k = m - j * a.g.sj;
    const long long step = *a.dstep;
    if (comp == 0) e_march<0, P>(a, ib, ie, j, k, m, step);
    else if (comp == 1) e_march<1, P>(a, ib, ie, j, k, m, step);
    else e_march<2, P>(a, ib, ie, j, k, m, step);
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
    const long long step = *a.dstep;
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
            e_point<P>(a, col, pl, i, j, k, step, hx, hy, hz, Hn[2 * kHJ * kHK + h - kHK], Hn[h - kHK],
                    Hn[kHJ * kHK + h - 1], Hn[h - 1], hy_prev, hz_prev, m0, m1, m2, ex, ey, ez);
            f.En[0][q] = ex; f.En[1][q] = ey; f.En[2][q] = ez;
        }
        hy_prev = hy;
        hz_prev = hz;
        __syncthreads();
    }
}

// launchers of the pole-count instantiations
using EKernel = void (*)(StepArgs, int, int);
using FKernel = void (*)(StepArgs, FusedArgs, TmaMaps);
#define CB2_POLES(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)
#define CB2_EK(p) k_update_e<p>,
#define CB2_FK(p) k_step_fused<p>,
const EKernel kEKernels[] = {CB2_POLES(CB2_EK)};
const FKernel kFKernels[] = {CB2_POLES(CB2_FK)};
#undef CB2_EK
#undef CB2_FK
#undef CB2_POLES

// ------------------------------------------------------------------- SIBC

// E = sum_k c_k (J - y_k) with y_k += (1 - e_k)(J - y_k), J from the faces' H.
// (reference sibc.c:256-269)
__global__ void __launch_bounds__(kBlock) k_sibc(const SibcArgs a) {
    const int e = blockIdx.x * kBlock + threadIdx.x;
    if (e >= a.ns) return;
    float J = 0.f;
    for (int f = 0; f < 4; f++) {
        const float w = a.hw[4 * e + f];
        if (w != 0.f) J += w * a.H[a.hcomp[4 * e + f]][a.hidx[4 * e + f]];
    }
    float E = 0.f;
    for (int k = 0; k < a.K; k++) {
        float y = a.y[(long long)k * a.ns + e];
        y += a.ome[k] * (J - y);
        a.y[(long long)k * a.ns + e] = y;
        E += a.c[k] * (J - y);
    }
    a.E[a.ecomp[e]][a.eidx[e]] = E;
}

// ------------------------------------------------- probes, ports, DFT ring

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Line integrals of every input slot (warp per slot), then port V/I and the
// source value, written as one row of the sample ring. With advance = 0 it
// only refreshes the port voltages before the E update (vold).
__global__ void __launch_bounds__(kBlock) k_post(const PostArgs a) {
    __shared__ double res[kMaxSlots];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int first = a.advance ? 0 : a.nip, last = a.advance ? a.nin : a.nip + a.nport;
    for (int s = first + warp; s < last; s += kBlock / 32) {
        double v = 0;
        for (int e = a.off[s] + lane; e < a.off[s + 1]; e += 32)
            v += (double)a.F[a.ecomp[e]][a.eidx[e]] * a.ew[e];
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
    const double tH = ((double)step + 0.5) * a.dt;
    const double vs = a.src_port >= 0 ? gauss(tH, a.src_amp, a.src_t0, a.src_tau) : 0.0;
    for (int s = threadIdx.x; s < a.nip; s += kBlock) row[s] = res[s];
    for (int p = threadIdx.x; p < a.nport; p += kBlock) {
        const double vnew = res[a.nip + p];
        const double V = 0.5 * (vnew + a.vold[p]);
        a.vold[p] = vnew;
        const double I = ((p == a.src_port ? vs : 0.0) - V) / a.R[p];
        row[a.nip + 2 * p] = V;
        row[a.nip + 2 * p + 1] = I;
    }
    if (threadIdx.x == 0) {
        double src = a.src_port >= 0 ? vs : 0.0;
        if (a.msrc_on) src += dgauss(tH, a.m_t0, a.m_tau);
        row[a.nip + 2 * a.nport] = src;
    }
    for (int s = threadIdx.x; s < a.nvp; s += kBlock) row[a.nip + 2 * a.nport + 1 + s] = res[a.nip + a.nport + s];
    __syncthreads();
    if (threadIdx.x == 0) *a.dstep = step + 1;
}

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
__global__ void __launch_bounds__(kBlock) k_energy(const EnergyArgs a) {
    __shared__ double red[kBlock / 32];
    const int i = blockIdx.y;
    const int m = blockIdx.x * kBlock + threadIdx.x;
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
        for (int w = 0; w < kBlock / 32; w++) s += red[w];
        a.partial[(long long)blockIdx.y * gridDim.x + blockIdx.x] = s;
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
    size_t psi_len_h[3][2] = {}, psi_len_e[3][2] = {};
    int zplanes = 0;   // planes of the z CPML slabs (same count for cells and nodes)
    DevBuf<unsigned short> mat[3];
    DevBuf<float> tab[3];
    DevBuf<float4> tab4[3];
    DevBuf<unsigned char> tflag[3];
    DevBuf<double> cb64[3];
    int ntab[3] = {0, 0, 0};
    DevBuf<float> J[3];
    int jbox[3][6] = {};
    DevBuf<float> wsrc[2];
    // SIBC
    DevBuf<int> sb_ecomp, sb_hcomp;
    DevBuf<long long> sb_eidx, sb_hidx;
    DevBuf<float> sb_hw, sb_y;
    // probes
    int nip = 0, nport = 0, nvp = 0, nin = 0, nslot = 0;
    DevBuf<int> off;
    DevBuf<unsigned char> ecomp;
    DevBuf<long long> eidx;
    DevBuf<double> ew, R, vold, ring, acc, omega;
    DevBuf<long long> dstep;
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

    ~Device() {
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

// reference index q -> padded device index
long long dev_index(const cem_sim *s, const Device &D, size_t q) {
    const size_t i = q / s->si, r = q % s->si, j = r / s->sj, k = r % s->sj;
    return (long long)(i * D.g.si + j * D.g.sj + k);
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

bool build_tables(cem_sim *s, Device &D) {
    const int P = s->npole;
    const int nfields = 3 + P;
    // per-edge extras: lumped source coefficient (excited port only), Debye beta/dt
    std::vector<std::unordered_map<size_t, double>> src(3);
    if (s->src_port >= 0) {
        const LumpedPort &pt = s->port[s->src_port];
        for (size_t e = 0; e < pt.edge.size(); e++) src[pt.axis][pt.edge[e]] = pt.cs[e];
    }
    std::vector<std::unordered_map<size_t, int>> disp(3);
    for (int e = 0; e < s->ndisp; e++) disp[s->d_comp[e]][s->d_idx[e]] = e;
    const int *n = s->n;
    for (int c = 0; c < 3; c++) {
        TableBuilder tb(nfields);
        std::vector<unsigned short> mat(D.Np, 0);
        std::vector<float> row(nfields);
        int box_lo[3] = {n[0], n[1], n[2]}, box_hi[3] = {-1, -1, -1};
        std::string last_key;
        for (int i = 0; i <= n[0]; i++)
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
                    auto it = src[c].find(q);
                    if (it != src[c].end()) { row[2] = (float)it->second; flag |= kFlagSrc; }
                    auto dt_ = disp[c].find(q);
                    if (dt_ != disp[c].end()) {
                        flag |= kFlagDisp;
                        for (int p = 0; p < P; p++)
                            row[3 + p] = (float)(s->d_beta[(size_t)p * s->ndisp + dt_->second] / s->dt);
                        for (int a = 0; a < 3; a++) {
                            box_lo[a] = std::min(box_lo[a], ijk[a]);
                            box_hi[a] = std::max(box_hi[a], ijk[a]);
                        }
                    }
                    const int id = tb.add(row.data(), flag, cb);
                    if (id > 65535) {
                        set_error("more than 65535 distinct update coefficients on one component");
                        return false;
                    }
                    mat[(size_t)i * D.g.si + (size_t)j * D.g.sj + k] = (unsigned short)id;
                }
        D.ntab[c] = (int)tb.flags.size();
        if (!dev_upload(s, D.mat[c], mat)) return false;
        if (!dev_upload(s, D.tab[c], tb.field_major())) return false;
        if (!dev_upload(s, D.tflag[c], tb.flags)) return false;
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
        }
        if (!dev_upload(s, D.cb64[c], tb.cb64)) return false;
        if (box_hi[0] >= 0) {
            for (int a = 0; a < 3; a++) {
                D.jbox[c][a] = box_lo[a];
                D.jbox[c][3 + a] = box_hi[a] - box_lo[a] + 1;
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
        std::vector<int> ph(n, -1), pe(n + 1, -1);
        std::vector<float> bh(n, 0.f), chh(n, 0.f), be(n + 1, 0.f), cee(n + 1, 0.f);
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
    {
        int r[2][2], planes = 0;
        pml_ranges(s, 2, 0, r);
        for (int sd = 0; sd < 2; sd++) planes += r[sd][1] >= r[sd][0] ? r[sd][1] - r[sd][0] + 1 : 0;
        D.zplanes = planes;
    }
    for (int c = 0; c < 3; c++)
        for (int w = 0; w < 2; w++) {
            D.psi_len_h[c][w] = psi_len(s, 0, c, w);
            D.psi_len_e[c][w] = psi_len(s, 1, c, w);
            if (!dev_alloc(s, D.psiH[0][c][w], D.psi_len_h[c][w] + 1) ||
                !dev_alloc(s, D.psiH[1][c][w], D.psi_len_h[c][w] + 1) || !dev_alloc(s, D.psiE[c][w], D.psi_len_e[c][w] + 1))
                return false;
            // unused slots of the compact layout are read by nobody but must stay finite
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
    std::vector<long long> idx;
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
    std::vector<double> R;
    for (const LumpedPort &p : s->port) R.push_back(p.R);
    std::vector<double> omega(s->nf);
    for (int f = 0; f < s->nf; f++) omega[f] = 2 * M_PI * s->freq[f];
    if (!dev_upload(s, D.off, off) || !dev_upload(s, D.ecomp, comp) || !dev_upload(s, D.eidx, idx) ||
        !dev_upload(s, D.ew, w) || !dev_upload(s, D.R, R) || !dev_upload(s, D.omega, omega))
        return false;
    if (!dev_alloc(s, D.vold, std::max(D.nport, 1)) || !dev_alloc(s, D.ring, (size_t)kRing * D.nslot) ||
        !dev_alloc(s, D.acc, (size_t)D.nslot * 2 * s->nf) || !dev_alloc(s, D.dstep, 1))
        return false;
    return true;
}

bool build_sibc(cem_sim *s, Device &D) {
    if (!s->nsb) return true;
    std::vector<int> ecomp(s->sb_comp), hcomp(s->sb_hc);
    std::vector<long long> eidx(s->nsb), hidx(4 * (size_t)s->nsb);
    std::vector<float> hw(4 * (size_t)s->nsb);
    for (int e = 0; e < s->nsb; e++) {
        eidx[e] = dev_index(s, D, s->sb_idx[e]);
        for (int f = 0; f < 4; f++) {
            hidx[4 * e + f] = f < s->sb_nf[e] ? dev_index(s, D, s->sb_hi[4 * e + f]) : 0;
            hw[4 * e + f] = f < s->sb_nf[e] ? (float)s->sb_sg[4 * e + f] : 0.f;
        }
    }
    return dev_upload(s, D.sb_ecomp, ecomp) && dev_upload(s, D.sb_hcomp, hcomp) && dev_upload(s, D.sb_eidx, eidx) &&
           dev_upload(s, D.sb_hidx, hidx) && dev_upload(s, D.sb_hw, hw) &&
           dev_alloc(s, D.sb_y, (size_t)s->nsb * s->sibc_npole);
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
    for (int c = 0; c < 3; c++) {
        a.E[c] = D.E[cur][c].p;
        a.H[c] = D.H[cur][c].p;
        a.hc[c] = D.hc[c].p;
        a.ec[c] = D.ec[c].p;
        a.pml[c] = PmlAxis{D.plane_h[c].p, D.plane_e[c].p, D.bm1_h[c].p, D.cid_h[c].p, D.bm1_e[c].p, D.cid_e[c].p,
                           (int)pml_per(s, c), D.zplanes};
        for (int w = 0; w < 2; w++) {
            a.psiH[c][w] = D.psiH[cur][c][w].p;
            a.psiE[c][w] = D.psiE[c][w].p;
        }
        a.mat[c] = D.mat[c].p;
        a.tab[c] = D.tab[c].p;
        a.tflag[c] = D.tflag[c].p;
        a.tab4[c] = D.tab4[c].p;
        a.ntab[c] = D.ntab[c];
        a.J[c] = D.J[c].p;
        for (int q = 0; q < 6; q++) a.jbox[c][q] = D.jbox[c][q];
    }
    a.dth = (float)(s->dt / CEM_MU0);
    a.has_pml = s->has_pml;
    a.npole = s->npole;
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
    if (s->kernel_choice >= 0) D.use_fused = s->kernel_choice == 1;
    CB2_CHECK(s, cudaStreamCreateWithFlags(&D.stream, cudaStreamNonBlocking));
    Geom &g = D.g;
    for (int a = 0; a < 3; a++) g.n[a] = s->n[a];
    g.sj = (s->n[2] + 1 + 3) / 4 * 4;
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
        std::vector<double> hc(s->n[c]);
        for (int i = 0; i < s->n[c]; i++) hc[i] = s->dt / CEM_MU0 * s->idh[c][i];
        if (!dev_upload(s, D.hc[c], to_f32(hc)) || !dev_upload(s, D.ec[c], to_f32(s->ide[c]))) return false;
        if (!dev_upload(s, D.d64[c], s->d[c]) || !dev_upload(s, D.dd64[c], s->dd[c])) return false;
    }
    if (!build_pml(s, D) || !build_tables(s, D) || !build_probes(s, D) || !build_sibc(s, D) || !build_sources(s, D))
        return false;
    for (int b = 0; b < 2; b++)
        for (int c = 0; c < 3; c++)
            if (!make_tmap(s, &D.maps[b].e[c], D.E[b][c].p, kRJ) || !make_tmap(s, &D.maps[b].h[c], D.H[b][c].p, kHJ))
                return false;
    if (!dev_alloc(s, D.error, 1) || !zero_dev(s, D.error.p, 4)) return false;
    CB2_CHECK(s, cudaFuncSetAttribute(kFKernels[s->npole], cudaFuncAttributeMaxDynamicSharedMemorySize, kFusedSmem));
    const long long nblk = (long long)((g.plane + kBlock - 1) / kBlock) * (s->n[0] + 1);
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

bool upload_f32(cem_sim *s, float *dst, const std::vector<double> &src, size_t n) {
    if (!n) return true;
    std::vector<float> tmp(n);
    for (size_t i = 0; i < n; i++) tmp[i] = (float)src[i];
    return h2d(s, dst, tmp.data(), n * sizeof(float));
}

bool download_f32(cem_sim *s, std::vector<double> &dst, const float *src, size_t n) {
    dst.resize(n);
    if (!n) return true;
    std::vector<float> tmp(n);
    if (!d2h(s, tmp.data(), src, n * sizeof(float))) return false;
    for (size_t i = 0; i < n; i++) dst[i] = tmp[i];
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

// reference compact layout <-> device layout (z-axis slabs transposed)
bool psi_is_z(int c, int w) { return (c + w + 1) % 3 == 2; }

std::vector<double> psi_to_device(const cem_sim *s, const Device &D, int c, int w, const std::vector<double> &v) {
    if (!psi_is_z(c, w) || v.empty()) return v;
    const size_t per = pml_per(s, 2), P = (size_t)D.zplanes;
    std::vector<double> o(v.size());
    for (size_t pl = 0; pl < P; pl++)
        for (size_t x = 0; x < per; x++) o[x * P + pl] = v[pl * per + x];
    return o;
}

void psi_to_host(const cem_sim *s, const Device &D, int c, int w, std::vector<double> &v) {
    if (!psi_is_z(c, w) || v.empty()) return;
    const size_t per = pml_per(s, 2), P = (size_t)D.zplanes;
    std::vector<double> o(v.size());
    for (size_t pl = 0; pl < P; pl++)
        for (size_t x = 0; x < per; x++) o[pl * per + x] = v[x * P + pl];
    v.swap(o);
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
                    if (!upload_f32(s, D.psiE[c][w].p, psi_to_device(s, D, c, w, s->psiE[c][w]), D.psi_len_e[c][w]) ||
                        !upload_f32(s, D.psiH[D.cur][c][w].p, psi_to_device(s, D, c, w, s->psiH[c][w]), D.psi_len_h[c][w]))
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
                for (int p = 0; p < s->npole; p++) box[p * vol + o] = (float)s->d_J[(size_t)p * s->ndisp + e];
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
                if (!download_f32(s, s->psiE[c][w], D.psiE[c][w].p, D.psi_len_e[c][w]) ||
                    !download_f32(s, s->psiH[c][w], D.psiH[D.cur][c][w].p, D.psi_len_h[c][w]))
                    return false;
                else {
                    psi_to_host(s, D, c, w, s->psiE[c][w]);
                    psi_to_host(s, D, c, w, s->psiH[c][w]);
                }
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
                for (int p = 0; p < s->npole; p++) s->d_J[(size_t)p * s->ndisp + e] = box[p * vol + o];
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
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    if (!D.vold_valid && D.nport) {
        PostArgs pa = D.pa[D.cur];
        pa.advance = 0;
        k_post<<<1, kBlock, 0, D.stream>>>(pa);
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

// one whole step: the fused H+E pass, then SIBC, probes and the step count
bool launch_fused_step(cem_sim *s) {
    Device &D = *s->dev;
    if (D.ring_count == kRing && !flush_dft(s)) return false;
    const dim3 grid((s->n[2] + 1 + kFK - 1) / kFK, (s->n[1] + 1 + kFJ - 1) / kFJ, (s->n[0] + 1 + kFX - 1) / kFX);
    t_begin(1);
    kFKernels[s->npole]<<<grid, dim3(kFK, kFJ), kFusedSmem, D.stream>>>(D.sa[D.cur], D.fa[D.cur], D.maps[D.cur]);
    t_end();
    D.cur ^= 1;
    if (s->nsb) { t_begin(2); k_sibc<<<(s->nsb + kBlock - 1) / kBlock, kBlock, 0, D.stream>>>(D.sb[D.cur]); t_end(); }
    PostArgs pa = D.pa[D.cur];
    pa.advance = 1;
    t_begin(3);
    k_post<<<1, kBlock, 0, D.stream>>>(pa);
    t_end();
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
    const int gx = (D.g.plane + kBlock - 1) / kBlock;
    if (phase_mask & 1) {   // H over node planes [i0, i1) within [0, nx]
        const int a = std::max(0, i0), b = std::min(nx + 1, i1);
        if (b > a) {
            t_begin(0);
            k_update_h<<<dim3(3 * gx, (b - a + kU - 1) / kU), blk, 0, D.stream>>>(D.sa[D.cur], a, b);
            t_end();
        }
    }
    if (phase_mask & 2) {   // port voltages before the E update
        PostArgs pa = D.pa[D.cur];
        pa.advance = 0;
        if (D.nport) k_post<<<1, kBlock, 0, D.stream>>>(pa);
    }
    if (phase_mask & 4) {   // E over node planes [i0, i1) within [0, nx)
        const int a = std::max(0, i0), b = std::min(nx, i1);
        if (b > a) {
            t_begin(1);
            kEKernels[s->npole]<<<dim3(3 * gx, (b - a + kU - 1) / kU), blk, 0, D.stream>>>(D.sa[D.cur], a, b);
            t_end();
        }
    }
    if (phase_mask & 8) {   // surface impedance, probes, step count
        if (D.ring_count == kRing && !flush_dft(s)) return false;
        if (s->nsb) { t_begin(2); k_sibc<<<(s->nsb + kBlock - 1) / kBlock, blk, 0, D.stream>>>(D.sb[D.cur]); t_end(); }
        PostArgs pa = D.pa[D.cur];
        pa.advance = 1;
        t_begin(3);
        k_post<<<1, kBlock, 0, D.stream>>>(pa);
        t_end();
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

int engine_step(cem_sim *s, long n) {
    if (n <= 0) return 0;
    if (!begin_device_op(s)) return -1;
    for (long it = 0; it < n; it++)
        if (!launch_step(s, 1 | 4 | 8, 0, s->n[0] + 1)) return -1;
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
    const int gx = (D.g.plane + kBlock - 1) / kBlock;
    k_energy<<<dim3(gx, s->n[0] + 1), kBlock, 0, D.stream>>>(D.ea[D.cur]);
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

constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_addr[kMaxScratchDevices] = {};

// Address of g_noalloc_scratch on `device`, which must be current. Looked up
// once per device; later calls only read the cached pointer.
double *noalloc_scratch(int device) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (device < 0 || device >= kMaxScratchDevices) {
        set_error("cemx_energy_noalloc: device ordinal beyond the 64 this library tracks");
        return nullptr;
    }
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            char msg[256];
            std::snprintf(msg, sizeof msg, "cemx_energy_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            set_error(msg);
            return nullptr;
        }
        g_scratch_addr[device] = static_cast<double *>(p);
    }
    return g_scratch_addr[device];
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
    const int gx = (D.g.plane + kBlock - 1) / kBlock;
    const long long nblk = (long long)gx * (s->n[0] + 1);
    if (nblk > kNoAllocPartials) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "cemx_energy_noalloc: grid needs %lld block partials, above the static scratch of %lld; "
                      "use cem_energy", nblk, kNoAllocPartials);
        set_error(msg);
        return false;
    }
    CB2_CHECK(s, cudaSetDevice(D.device));
    double *scratch = noalloc_scratch(D.device);
    if (!scratch) return false;
    EnergyArgs ea = D.ea[D.cur];
    ea.partial = scratch;
    k_energy<<<dim3(gx, s->n[0] + 1), kBlock, 0, D.stream>>>(ea);
    k_sum<<<1, 1024, 0, D.stream>>>(scratch, nblk, scratch + kNoAllocPartials);
    CB2_CHECK(s, cudaGetLastError());
    CB2_CHECK(s, cudaMemcpyAsync(out, scratch + kNoAllocPartials, sizeof(double), cudaMemcpyDeviceToHost, D.stream));
    CB2_CHECK(s, cudaStreamSynchronize(D.stream));
    return true;
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
    for (long it = 0; it < n; it++)
        if (!launch_step(s, 1 | 4 | 8, 0, s->n[0] + 1)) return false;
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
    long long v[13] = {0};
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
        bytes += (long long)(D.sb_y.n + D.sb_hw.n) * 4 + (long long)(D.sb_eidx.n + D.sb_hidx.n) * 8 +
                 (long long)(D.ring.n + D.acc.n) * 8;
        v[11] = bytes;
    }
    v[12] = 3 + (s->nsb ? 1 : 0);
    for (int q = 0; q < n && q < 13; q++) out[q] = v[q];
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

int cemx_energy_noalloc(cem_sim *s, double *out) {
    if (!s || !out) { set_error("cemx_energy_noalloc: null argument"); return -1; }
    if (!s->finalized) { set_error("not finalized"); return -1; }
    return energy_noalloc(s, out) ? 0 : -1;
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
