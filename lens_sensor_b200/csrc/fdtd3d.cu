// 3D Yee CPML step for sm_100a.
//
// Math (planar_3d/boundaries3d.py:311-362, CPML_3D.step_H / step_E):
//   H += Ch*(d1 - d2); strip corrections H += (+Ch)*(psi1 + (1/k-1)*d1),
//                                        H += (-Ch)*(psi2 + (1/k-1)*d2)
//   E <- D*E (lossy);  E += ce*(d1 - d2) on the interior; strip corrections with
//   coef +ce / -ce;  PEC on the absorbing faces; then the Huygens source
//   (fdtd3d_core.py:1116-1127: the source follows the step and its PEC).
// psi lives only in the PML strips (lens_fdtd.h); elsewhere it is exactly 0.
//
// Two execution paths share the per-cell arithmetic:
//  * fused3d  (field buffer 1 present): ONE pass per step.  A CTA owns a tile
//    of 8 rows (y) x 32 lanes (z) and streams an x-chunk.  Per x-plane, TMA
//    (cp.async.bulk.tensor) stages E(i+1) with a 1-cell y/z halo, H(i) with
//    the low halo and the coefficient tile into a 4/3/3-deep shared-memory
//    ring guarded by mbarriers; the CTA computes H(i) on the tile plus its low
//    halo (the halo redundantly, psi read-only there), then E(i) on the tile.
//    Reads buffer `cur`, writes the other: each field element crosses HBM once
//    per step (72 B per cell update for the lossy case, 60 lossless).
//  * h3d + e3d (in place, no buffer 1): two streaming passes.
#include <cuda.h>
#include <algorithm>

#include <cmath>

#include "lens_common.cuh"

namespace {

constexpr int BK = 32;  // tile lanes along z (contiguous)
constexpr int BJ = 8;   // tile rows along y
constexpr int NT = BK * BJ;

// Kernel-side view of a grid with the read (r*) and write (w*) buffers resolved.
struct K3 {
    int nx, ny, nz, P;
    const float *ex, *ey, *ez, *hx, *hy, *hz;
    float *wex, *wey, *wez, *whx, *why, *whz;
    const float *pr[LENS_NPSI];
    float *pw[LENS_NPSI];
    const float *ce_x, *ce_y, *ce_z, *da_x, *da_y, *da_z;
    float ch;
    LensAxis ax, ay, az;
    int pec[6];
    LensSource src;
    int src_comp;
    int *flag;
    const unsigned char *ctype, *cexpl;  // coefficient column form (LensGrid3D)
    const float *ctab;
    int ntype;
    int wd_plane;  // watchdog self-test: offset of the plane whose E copy CTA 0 withholds (-1: normal step)
};

struct Hv {
    float x, y, z;
};

// psi = b*psi_old + c*d (written only by the owning thread); returns psi + (1/k-1)*d.
__device__ __forceinline__ float psi_upd(const float *pr, float *pw, size_t idx, bool own,
                                         const LensProfile &pf, int m, float d) {
    const float p = pf.b[m] * pr[idx] + pf.c[m] * d;
    if (own) pw[idx] = p;
    return p + (pf.ik[m] - 1.0f) * d;
}

// H(i,j,k) from old H and the E values around it.
//   e*   : E(i,j,k)      e*k : E(i,j,k+1)    e*j : E(i,j+1,k)    e*n : E(i+1,j,k)
__device__ __forceinline__ Hv h_cell(const K3 &g, int i, int j, int k, Hv h, float ex, float ey,
                                     float ez, float exk, float eyk, float exj, float ezj, float ezn,
                                     float eyn, bool own) {
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const float ch = g.ch;
    const int sz = strip_of(k, g.az.h.lo, g.az.h.hi, g.az.h.n);
    const int sy = strip_of(j, g.ay.h.lo, g.ay.h.hi, g.ay.h.n);
    const int sx = strip_of(i, g.ax.h.lo, g.ax.h.hi, g.ax.h.n);
    const size_t c = ((size_t)i * ny + j) * P + k;  // psi is full-domain, same index as the fields
    Hv o = h;
    if (j < ny - 1 && k < nz - 1) {
        const float d1 = eyk - ey, d2 = ezj - ez;
        float v = h.x + ch * (d1 - d2);
        if (sz >= 0)
            v = v + ch * psi_upd(g.pr[LENS_PSI_HX_Z], g.pw[LENS_PSI_HX_Z], c,
                                 own, g.az.h, k, d1);
        if (sy >= 0)
            v = v + (-ch) * psi_upd(g.pr[LENS_PSI_HX_Y], g.pw[LENS_PSI_HX_Y], c,
                                    own, g.ay.h, j, d2);
        o.x = v;
    }
    if (i < nx - 1 && k < nz - 1) {
        const float d1 = ezn - ez, d2 = exk - ex;
        float v = h.y + ch * (d1 - d2);
        if (sx >= 0)
            v = v + ch * psi_upd(g.pr[LENS_PSI_HY_X], g.pw[LENS_PSI_HY_X], c,
                                 own, g.ax.h, i, d1);
        if (sz >= 0)
            v = v + (-ch) * psi_upd(g.pr[LENS_PSI_HY_Z], g.pw[LENS_PSI_HY_Z], c,
                                    own, g.az.h, k, d2);
        o.y = v;
    }
    if (i < nx - 1 && j < ny - 1) {
        const float d1 = exj - ex, d2 = eyn - ey;
        float v = h.z + ch * (d1 - d2);
        if (sy >= 0)
            v = v + ch * psi_upd(g.pr[LENS_PSI_HZ_Y], g.pw[LENS_PSI_HZ_Y], c,
                                 own, g.ay.h, j, d1);
        if (sx >= 0)
            v = v + (-ch) * psi_upd(g.pr[LENS_PSI_HZ_X], g.pw[LENS_PSI_HZ_X], c,
                                    own, g.ax.h, i, d2);
        o.z = v;
    }
    return o;
}

__device__ __forceinline__ float src3(const K3 &g, const LensStepTable &tab, int n, int i, int j,
                                      int k) {
    const LensSource &s = g.src;
    const int q = n - tab.t0;
    const size_t m = (size_t)j * s.pitch_k + k;
    if (i == s.ix) return (tab.env[q] * sinf(tab.wt[q] + s.ph1[m])) * s.amp[m];
    return -((tab.env[q] * sinf(tab.wt[q] + s.ph2[m])) * s.amp[m]);
}

__device__ __forceinline__ bool is_src(const K3 &g, int comp, int i, int j, int k) {
    return g.src_comp == comp && g.src.ix >= 0 && (i == g.src.ix || i == g.src.ix + 1) && j < g.src.nj &&
           k < g.src.nk;
}

struct Coef {
    float cx, cy, cz, dx, dy, dz;
};

// E(i,j,k) from old E, the new H around it and the coefficients.
//   h = H(i,j,k); hxk/hyk = H(i,j,k-1); hxj/hzj = H(i,j-1,k); hym/hzm = H(i-1,j,k)
__device__ __forceinline__ Hv e_cell(const K3 &g, const LensStepTable &tab, int n, int i, int j, int k,
                                     Hv e, Hv h, float hxk, float hyk, float hxj, float hzj, float hym,
                                     float hzm, const Coef &c, bool lossy) {
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const size_t c0 = ((size_t)i * ny + j) * P + k;  // psi index (full-domain)
    const int sz = strip_of(k, g.az.e.lo, g.az.e.hi, g.az.e.n);
    const int sy = strip_of(j, g.ay.e.lo, g.ay.e.hi, g.ay.e.n);
    const int sx = strip_of(i, g.ax.e.lo, g.ax.e.hi, g.ax.e.n);
    const bool iin = i >= 1 && i <= nx - 2, jin = j >= 1 && j <= ny - 2, kin = k >= 1 && k <= nz - 2;
    Hv o = e;
    if (i < nx - 1) {  // Ex (nx-1, ny, nz)
        float v = lossy ? e.x * c.dx : e.x;
        if (jin && kin) {
            const float d1 = h.z - hzj, d2 = h.y - hyk;
            v = v + c.cx * (d1 - d2);
            if (sy >= 0)
                v = v + c.cx * psi_upd(g.pr[LENS_PSI_EX_Y], g.pw[LENS_PSI_EX_Y], c0,
                                       true, g.ay.e, j, d1);
            if (sz >= 0)
                v = v + (-c.cx) * psi_upd(g.pr[LENS_PSI_EX_Z], g.pw[LENS_PSI_EX_Z], c0,
                                          true, g.az.e, k, d2);
        }
        if ((g.pec[2] && j == 0) || (g.pec[3] && j == ny - 1) || (g.pec[4] && k == 0) ||
            (g.pec[5] && k == nz - 1))
            v = 0.f;
        if (is_src(g, 0, i, j, k)) v += src3(g, tab, n, i, j, k);
        o.x = v;
    }
    if (j < ny - 1) {  // Ey (nx, ny-1, nz)
        float v = lossy ? e.y * c.dy : e.y;
        if (iin && kin) {
            const float d1 = h.x - hxk, d2 = h.z - hzm;
            v = v + c.cy * (d1 - d2);
            if (sz >= 0)
                v = v + c.cy * psi_upd(g.pr[LENS_PSI_EY_Z], g.pw[LENS_PSI_EY_Z], c0,
                                       true, g.az.e, k, d1);
            if (sx >= 0)
                v = v + (-c.cy) * psi_upd(g.pr[LENS_PSI_EY_X], g.pw[LENS_PSI_EY_X], c0,
                                          true, g.ax.e, i, d2);
        }
        if ((g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1) || (g.pec[4] && k == 0) ||
            (g.pec[5] && k == nz - 1))
            v = 0.f;
        if (is_src(g, 1, i, j, k)) v += src3(g, tab, n, i, j, k);
        o.y = v;
    }
    if (k < nz - 1) {  // Ez (nx, ny, nz-1)
        float v = lossy ? e.z * c.dz : e.z;
        if (iin && jin) {
            const float d1 = h.y - hym, d2 = h.x - hxj;
            v = v + c.cz * (d1 - d2);
            if (sx >= 0)
                v = v + c.cz * psi_upd(g.pr[LENS_PSI_EZ_X], g.pw[LENS_PSI_EZ_X], c0,
                                       true, g.ax.e, i, d1);
            if (sy >= 0)
                v = v + (-c.cz) * psi_upd(g.pr[LENS_PSI_EZ_Y], g.pw[LENS_PSI_EZ_Y], c0,
                                          true, g.ay.e, j, d2);
        }
        if ((g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1) || (g.pec[2] && j == 0) ||
            (g.pec[3] && j == ny - 1))
            v = 0.f;
        if (is_src(g, 2, i, j, k)) v += src3(g, tab, n, i, j, k);
        o.z = v;
    }
    return o;
}

__device__ __forceinline__ void plane3(const LensEpi3D &ep, const LensStepTable &tab, int n, int p,
                                       int pair, size_t vol, size_t jk, float e, float h) {
    const int q = n - tab.t0;
    double *a = ep.plane_acc + ((size_t)(p * 2 + pair) * 4) * vol + jk;
    a[0] += (double)e * (double)tab.pe[2 * q];
    a[vol] += (double)e * (double)tab.pe[2 * q + 1];
    a[2 * vol] += (double)h * (double)tab.ph[2 * q];
    a[3 * vol] += (double)h * (double)tab.ph[2 * q + 1];
}

// End of a detector-box range on an axis of extent `ext` with numpy slice
// semantics: a negative end counts from that component's own end
// (fdtd3d_core.py:1139-1142 uses slice(n_sp, -n_sp) on Ex, Ey and Ez alike).
__host__ __device__ __forceinline__ int box_end(int e, int ext) { return e < 0 ? ext + e : (e < ext ? e : ext); }

// Is (i, j, k) of component c (0 Ex, 1 Ey, 2 Ez) inside box bx?
__device__ __forceinline__ bool in_box(const int *bx, int c, int i, int j, int k, int nx, int ny, int nz) {
    return i >= bx[0] && i < box_end(bx[1], nx - (c == 0)) && j >= bx[2] && j < box_end(bx[3], ny - (c == 1)) &&
           k >= bx[4] && k < box_end(bx[5], nz - (c == 2));
}

// Epilogue of one cell after its E update.  All 32 lanes of a warp must call it.
//   detector boxes: sum of Ex^2+Ey^2+Ez^2 in FP64 (fdtd3d_core.py:477-481)
//   DFT windows:    complex float32 sums of each selected component (the
//                   reference's complex64 accumulator, fdtd3d_core.py:1150-1158)
//   flux planes:    FP64 DFT of E and of the x-averaged H (flux.py:28-41)
__device__ __forceinline__ void epi_cell(const K3 &g, const LensStepTable &tab, const LensEpi3D &ep,
                                         int n, int i, int j, int k, bool in, Hv e, float hym,
                                         float hzm, Hv h, bool vol_dft = true, bool boxes = true) {
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const bool vx = in && i < nx - 1, vy = in && j < ny - 1, vz = in && k < nz - 1;
    if (boxes && ep.nbox > 0) {
        const int bk0 = blockIdx.x * BK, bj0 = blockIdx.y * BJ;
        for (int b = 0; b < ep.nbox; ++b) {
            const int *bx = ep.box[b];
            if (i < bx[0] || i >= box_end(bx[1], nx) || box_end(bx[3], ny) <= bj0 || bx[2] >= bj0 + BJ ||
                box_end(bx[5], nz) <= bk0 || bx[4] >= bk0 + BK)
                continue;  // block-uniform
            double v = 0.0;
            if (vx && in_box(bx, 0, i, j, k, nx, ny, nz)) v += (double)(e.x * e.x);
            if (vy && in_box(bx, 1, i, j, k, nx, ny, nz)) v += (double)(e.y * e.y);
            if (vz && in_box(bx, 2, i, j, k, nx, ny, nz)) v += (double)(e.z * e.z);
            warp_atomic_add(ep.box_acc + b, v);
        }
    }
    const bool win = n >= ep.dft_n0 && n < ep.dft_n1;
    const bool prevw = ep.conv_prev && n >= ep.prev_n0 && n < ep.prev_n1;
    if (!in || !(win || prevw)) return;
    const size_t o = ((size_t)i * ny + j) * P + k;
    const float f = g.src_comp == 1 ? e.y : (g.src_comp == 2 ? e.z : e.x);
    const bool vf = g.src_comp == 1 ? vy : (g.src_comp == 2 ? vz : vx);
    const int q = n - tab.t0;
    const float pr = tab.pe[2 * q], pim = tab.pe[2 * q + 1];
    if (prevw && vf && k == ep.conv_k)
        kahan_add(reinterpret_cast<float4 *>(ep.conv_prev) + (size_t)i * g.src.nj + j, f * pr, f * pim);
    if (!win) return;
    if (vol_dft) {
        const float v[3] = {e.x, e.y, e.z};
        const bool ok[3] = {vx, vy, vz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (ep.dft[c] && ok[c]) {
                float2 *a = reinterpret_cast<float2 *>(ep.dft[c]) + o;
                float2 s = *a;
                s.x += v[c] * pr;
                s.y += v[c] * pim;
                *a = s;
            }
        }
    }
    if (ep.conv_last && vf && k == ep.conv_k)
        kahan_add(reinterpret_cast<float4 *>(ep.conv_last) + (size_t)i * g.src.nj + j, f * pr, f * pim);
    for (int p = 0; p < ep.nplane; ++p) {
        if (i != ep.plane[p]) continue;
        const size_t S = (size_t)ny * P, jk = (size_t)j * P + k;
        if (vy) plane3(ep, tab, n, p, 0, S, jk, e.y, 0.5f * (hzm + h.z));
        if (vz) plane3(ep, tab, n, p, 1, S, jk, e.z, 0.5f * (hym + h.y));
    }
}

// ============================================================ in-place passes
// A block owns a BJ x BK (y, z) tile and streams an x-chunk; x-neighbours are
// carried in registers, z-neighbours come by warp shuffle, y-neighbours via L1.
__global__ void __launch_bounds__(NT) h3d(const K3 g, int chunk) {
    const int lane = threadIdx.x;
    const int k = blockIdx.x * BK + lane, j = blockIdx.y * BJ + threadIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const int x0 = blockIdx.z * chunk, x1 = min(nx, x0 + chunk);
    const bool act = k < nz && j < ny;
    const size_t S = (size_t)ny * P;
    size_t o = ((size_t)x0 * ny + j) * P + k;
    float ex = 0.f, ey = 0.f, ez = 0.f;
    if (act) {
        ex = g.ex[o];
        ey = g.ey[o];
        ez = g.ez[o];
    }
    for (int i = x0; i < x1; ++i, o += S) {
        float exn = 0.f, eyn = 0.f, ezn = 0.f, ezj = 0.f, exj = 0.f;
        if (act) {
            if (i + 1 < nx) {
                exn = g.ex[o + S];
                eyn = g.ey[o + S];
                ezn = g.ez[o + S];
            }
            if (j + 1 < ny) {
                ezj = g.ez[o + P];
                exj = g.ex[o + P];
            }
        }
        float eyk = __shfl_down_sync(0xffffffffu, ey, 1);
        float exk = __shfl_down_sync(0xffffffffu, ex, 1);
        if (lane == BK - 1 && act && k + 1 < nz) {
            eyk = g.ey[o + 1];
            exk = g.ex[o + 1];
        }
        if (act) {
            const Hv h0{g.hx[o], g.hy[o], g.hz[o]};
            const Hv h = h_cell(g, i, j, k, h0, ex, ey, ez, exk, eyk, exj, ezj, ezn, eyn, true);
            g.whx[o] = h.x;
            g.why[o] = h.y;
            g.whz[o] = h.z;
        }
        ex = exn;
        ey = eyn;
        ez = ezn;
    }
}

__global__ void __launch_bounds__(NT)
    e3d(const K3 g, const LensStepTable tab, const LensEpi3D ep, int n, int chunk) {
    const int lane = threadIdx.x;
    const int k = blockIdx.x * BK + lane, j = blockIdx.y * BJ + threadIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const int x0 = blockIdx.z * chunk, x1 = min(nx, x0 + chunk);
    const bool in = k < nz && j < ny;
    const bool lossy = g.da_x != nullptr;
    const size_t S = (size_t)ny * P;
    size_t o = ((size_t)x0 * ny + j) * P + k;
    float hym = 0.f, hzm = 0.f;
    if (in && x0 >= 1) {
        hym = g.hy[o - S];
        hzm = g.hz[o - S];
    }
    for (int i = x0; i < x1; ++i, o += S) {
        Hv h{0.f, 0.f, 0.f};
        float hzj = 0.f, hxj = 0.f;
        if (in) {
            h = Hv{g.hx[o], g.hy[o], g.hz[o]};
            if (j >= 1) {
                hzj = g.hz[o - P];
                hxj = g.hx[o - P];
            }
        }
        float hyk = __shfl_up_sync(0xffffffffu, h.y, 1);
        float hxk = __shfl_up_sync(0xffffffffu, h.x, 1);
        if (lane == 0 && in && k >= 1) {
            hyk = g.hy[o - 1];
            hxk = g.hx[o - 1];
        }
        Hv e{0.f, 0.f, 0.f};
        if (in) {
            Coef c{g.ce_x[o], g.ce_y[o], g.ce_z[o], 1.f, 1.f, 1.f};
            if (lossy) {
                c.dx = g.da_x[o];
                c.dy = g.da_y[o];
                c.dz = g.da_z[o];
            }
            e = e_cell(g, tab, n, i, j, k, Hv{g.ex[o], g.ey[o], g.ez[o]}, h, hxk, hyk, hxj, hzj, hym,
                       hzm, c, lossy);
            g.wex[o] = e.x;
            g.wey[o] = e.y;
            g.wez[o] = e.z;
        }
        epi_cell(g, tab, ep, n, i, j, k, in, e, hym, hzm, h);
        hym = h.y;
        hzm = h.z;
    }
}

// ============================================================ fused TMA pass
// A CTA owns a tile of TJ = 14 rows (y) x TK = 32 lanes (z) and streams an
// x-chunk.  Warps 0..6 own rows 2w and 2w+1 (H and E); warp 7 computes H on
// the halo row j0-1 (all lanes) and the halo column k0-1 (lanes 0..13), and its
// lane 0 drives the E ring.  Per x-plane, TMA stages E with a one-cell halo
// (rows j0-1..j0+14, z k0-4..k0+35) into a 4-deep mbarrier ring and the old H
// and coefficient tiles of the owner cells into a 3-deep ring; the halo cells'
// old H and (in CPML tiles) psi are read with coalesced loads issued one phase
// ahead.  One CTA barrier per plane publishes the new H tile (shared memory)
// for the E update.  Reads buffer `cur`, writes the
// other: 72 B per cell update (lossy), 60 B lossless, plus psi in the strips.
constexpr int TJ = 14, TK = 32;             // 7 owner warps + 1 halo warp = 8 warps
constexpr int NOW = TJ / 2;                  // owner warps (2 rows each)
constexpr int NW3 = NOW + 1;                 // + halo warp
constexpr int EK = TK + 8, EJ = TJ + 2;      // E box
constexpr int E_BYTES = EK * EJ * 4;
constexpr int E_SLOT = ((E_BYTES + 127) / 128) * 128;
constexpr int NSE = 3;                       // E ring depth (x-planes)
constexpr int SHK = TK + 1, SHJ = TJ + 1;    // new H tile: z k0-1..k0+31, y j0-1..j0+TJ-1
constexpr int SH_N = SHK * SHJ;
constexpr int EF = E_SLOT / 4;
constexpr int HT = TK * TJ;                  // floats of one owner tile (z k0..k0+31, y j0..j0+TJ-1)
constexpr int NHC = 3;                       // H + coefficient ring depth (x-planes)
constexpr int HC_SLOT = 9 * HT * 4;          // Hx, Hy, Hz, ce_x, ce_y, ce_z, D_x, D_y, D_z
constexpr int OFF_HC = NSE * 3 * E_SLOT;
constexpr int OFF_SH = OFF_HC + NHC * HC_SLOT;
constexpr int OFF_PT = OFF_SH + ((2 * 3 * SH_N * 4 + 127) / 128) * 128;
constexpr int NT3 = NW3 * 32;                // threads of a CTA
constexpr int OFF_HS = OFF_PT + (((6 * (TK + 1 + TJ + 1)) * 4 + 127) / 128) * 128;
constexpr int HS_STAGE = 12 * NT3;           // H-psi of a thread's two cells, 6 components each
constexpr int OFF_BAR = OFF_HS + 2 * HS_STAGE * 4;
constexpr int OFF_CT = OFF_BAR + (NSE + NHC) * 8;  // coefficient column types: the tile's rows
constexpr int SMEM3 = OFF_CT + LENS_MAX_CTYPE * 6 * TJ * 4;
static_assert(OFF_HC % 128 == 0 && HC_SLOT % 128 == 0 && (HT * 4) % 128 == 0, "TMA alignment");
static_assert(OFF_SH % 128 == 0 && OFF_BAR % 8 == 0, "alignment");

struct EMaps {
    CUtensorMap e[3];  // Ex, Ey, Ez of the read buffer, box EK x EJ x 1
    CUtensorMap h[3];  // Hx, Hy, Hz of the read buffer, box TK x TJ x 1
    CUtensorMap c[6];  // ce_x, ce_y, ce_z, D_x, D_y, D_z, box TK x TJ x 1
};

__device__ __forceinline__ uint32_t s_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// Bounded wait for phase `parity` of an mbarrier; false if it gave up.  Each
// try_wait may suspend the thread for up to 1 us (suspend-time hint), so the
// bound (2^20 tries) is about a second.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int tries = 1 << 20) {
    uint32_t ok = 0;
    for (int t = 0; t < tries && !ok; ++t) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(1000u)
            : "memory");
    }
    return ok != 0;
}

__device__ __forceinline__ void tma3(uint32_t dst, const CUtensorMap *m, int c0, int c1, int c2,
                                     uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// does [a, b] meet a psi strip of profile p?
__host__ __device__ __forceinline__ bool meets(int a, int b, const LensProfile &p) {
    return (p.lo > 0 && a < p.lo) || (p.hi > 0 && b >= p.n - p.hi);
}

__host__ __device__ __forceinline__ bool in_strip(const LensProfile &p, int m) {
    return m >= 0 && m < p.n && (m < p.lo || m >= p.n - p.hi);
}

// psi = b*psi_old + c*d (stored when wr); returns psi + km*d, km = 1/kappa - 1.
template <typename IX>
__device__ __forceinline__ float psi_u(float b, float c, float km, float old, float d, float *pw, IX idx,
                                       bool wr) {
    const float v = b * old + c * d;
    if (wr) pw[idx] = v;
    return v + km * d;
}

// CPML profile tables of a CPML tile in shared memory: rows (b, c, 1/kappa-1) of
// the half-node (H) then the integer-node (E) profile, for z = k0-1 .. k0+TK-1
// (ZN entries) and y = j0-1 .. j0+TJ-1 (YN entries); zero outside the profile.
constexpr int ZN = TK + 1, YN = TJ + 1;

__device__ __forceinline__ void fill_row(float *t, int stride, const LensProfile &p, int m) {
    const bool in = m >= 0 && m < p.n;
    t[0] = in ? __ldg(p.b + m) : 0.f;
    t[stride] = in ? __ldg(p.c + m) : 0.f;
    t[2 * stride] = in ? __ldg(p.ik + m) - 1.0f : 0.f;
}

// Values of one x-plane (uniform): H profile at i (half node), E profile at i.
struct PX {
    float hb, hc, hk, eb, ec, ek;
};

__device__ __forceinline__ PX px_at(const K3 &g, int i) {
    PX v{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (in_strip(g.ax.h, i)) {
        v.hb = __ldg(g.ax.h.b + i); v.hc = __ldg(g.ax.h.c + i); v.hk = __ldg(g.ax.h.ik + i) - 1.0f;
    }
    if (in_strip(g.ax.e, i)) {
        v.eb = __ldg(g.ax.e.b + i); v.ec = __ldg(g.ax.e.c + i); v.ek = __ldg(g.ax.e.ik + i) - 1.0f;
    }
    return v;
}

constexpr int MAXCH = 96;
constexpr int MAXPERM = 4096;  // CPML tiles that can be reordered (more: the plain order)
// Work of one step: every (z-tile, y-tile, x-chunk).  The CPML tiles (outside
// the lean core [lo, hi): CPML-free, interior) come first, the longer CTAs
// starting early; within each group the order is chunk, y-tile, z-tile (z
// fastest), so that CTAs sharing E halo lines run together.
struct Work {
    int ntz, nty, nc;
    int lo[3], hi[3];  // lean core: z-tiles, y-tiles, chunks
    int plo[3], phi[3];  // z-tiles, y-tiles, chunks without z / y / x CPML psi
    int x[MAXCH + 1];  // chunk c covers planes [x[c], x[c+1])
    int nperm;                    // CTAs [0, nperm) take tile perm[id] (0: the order above)
    unsigned short perm[MAXPERM];  // CPML tiles ordered by the pass they run, most axes first
};

// Tile of CTA `id` (see Work); returns true for a lean tile.
__host__ __device__ __forceinline__ bool work_tile(const Work &wk, int id, int &tz, int &ty, int &c) {
    const int ntz = wk.ntz, nty = wk.nty;
    const int nlz = wk.hi[0] - wk.lo[0], nly = wk.hi[1] - wk.lo[1], nlc = wk.hi[2] - wk.lo[2];
    const int full = nty * ntz;                  // CPML tiles of a CPML chunk
    const int part = full - nly * nlz;           // CPML tiles of a lean chunk
    const int nstrip = (wk.nc - nlc) * full + nlc * part;
    if (id >= nstrip) {  // lean core, z fastest
        int q = id - nstrip;
        tz = wk.lo[0] + q % nlz;
        q /= nlz;
        ty = wk.lo[1] + q % nly;
        c = wk.lo[2] + q / nly;
        return true;
    }
    const int before = wk.lo[2] * full;          // CPML tiles of the chunks before the lean ones
    int rem;
    if (id < before) {
        c = id / full;
        rem = id % full;
    } else if (id < before + nlc * part) {
        c = wk.lo[2] + (id - before) / part;
        rem = (id - before) % part;
        // rows before the lean rows are whole, the lean rows lack their lean z-tiles
        const int r0 = wk.lo[1] * ntz, rp = nly * (ntz - nlz);
        if (rem >= r0 && rem < r0 + rp) {
            const int q = rem - r0, w = ntz - nlz;
            ty = wk.lo[1] + q / w;
            const int t = q % w;
            tz = t < wk.lo[0] ? t : t + nlz;
            return false;
        }
        if (rem >= r0 + rp) rem -= rp - nly * ntz;  // map to whole-row numbering
    } else {
        const int q = id - before - nlc * part;
        c = wk.hi[2] + q / full;
        rem = q % full;
    }
    ty = rem / ntz;
    tz = rem % ntz;
    return false;
}

// CPML axes whose psi a tile carries (template mask M of the tile pass).
enum : unsigned { AXZ = 1u, AXY = 2u, AXX = 4u, AXALL = 7u };

// Per-cell flags of an owner row.
enum : unsigned {
    F_IN = 1u, F_HX = 2u, F_HY = 4u, F_HZ = 8u,     // in the domain; H components that update
    F_EXU = 16u, F_EYU = 32u, F_EZU = 64u,          // E components whose curl term applies (j,k part)
    F_EYV = 128u, F_EZV = 256u,                     // Ey, Ez exist (j < ny-1, k < nz-1)
    F_PJ = 512u, F_PK = 1024u,                      // on a PEC face in y / z
    F_ZH = 2048u, F_YH = 4096u, F_ZE = 8192u, F_YE = 16384u   // in a z / y psi strip (H / E)
};

__device__ __forceinline__ unsigned cell_flags(const K3 &g, const LensEpi3D &ep, int j, int k) {
    const int ny = g.ny, nz = g.nz;
    unsigned f = 0;
    if (j < 0 || k < 0 || j >= ny || k >= nz) return 0;
    f |= F_IN;
    if (j < ny - 1 && k < nz - 1) f |= F_HX;
    if (k < nz - 1) f |= F_HY | F_EZV;
    if (j < ny - 1) f |= F_HZ | F_EYV;
    const bool jin = j >= 1 && j <= ny - 2, kin = k >= 1 && k <= nz - 2;
    if (jin && kin) f |= F_EXU;
    if (kin && j < ny - 1) f |= F_EYU;
    if (jin && k < nz - 1) f |= F_EZU;
    if ((g.pec[2] && j == 0) || (g.pec[3] && j == ny - 1)) f |= F_PJ;
    if ((g.pec[4] && k == 0) || (g.pec[5] && k == nz - 1)) f |= F_PK;
    if (in_strip(g.az.h, k)) f |= F_ZH;
    if (in_strip(g.ay.h, j)) f |= F_YH;
    if (in_strip(g.az.e, k)) f |= F_ZE;
    if (in_strip(g.ay.e, j)) f |= F_YE;
    return f;
}

// Read-only global load issued where it is written: the volatile asm keeps the
// compiler from sinking a prefetch toward its first use (the scoreboard then
// waits at the use, after the work placed in between).
__device__ __forceinline__ float ldg_early(const float *p) {
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ unsigned ldg_u8_early(const unsigned char *p) {
    unsigned v;
    asm volatile("ld.global.nc.u8 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// 4-byte asynchronous global -> shared copy (zero fill when !pred: nothing is read).
__device__ __forceinline__ void cp_async4(uint32_t dst, const float *src, bool pred) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(pred ? 4 : 0)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Stage the H-psi of one cell (hx_z, hx_y, hy_x, hy_z, hz_y, hz_x) into dst + q*NT3*4;
// only the components of the axes in M (the others are never read).
template <unsigned M, typename IX>
__device__ __forceinline__ void stage_hpsi(uint32_t dst, const K3 &g, IX o, unsigned f, bool xh) {
    const bool in = f & F_IN, z = in && (f & F_ZH), y = in && (f & F_YH), x = in && xh;
    const bool on[6] = {z, y, x, z, y, x};
    constexpr unsigned ax[6] = {AXZ, AXY, AXX, AXZ, AXY, AXX};
#pragma unroll
    for (int q = 0; q < 6; ++q)
        if (M & ax[q]) cp_async4(dst + q * NT3 * 4, on[q] ? g.pr[q] + o : g.pr[q], on[q]);
}

// A CPML tile that carries the psi of one axis only.
template <unsigned M>
constexpr bool single_axis() {
    return M == AXZ || M == AXY || M == AXX;
}

// Stage the E-psi of one cell of a single-axis tile beside its H-psi: E component e
// (ex_y, ex_z, ey_z, ey_x, ez_x, ez_y) into slot e, a slot the H-psi of that one
// axis leaves free (z: H 0, 3 / E 1, 2; y: H 1, 4 / E 0, 5; x: H 2, 5 / E 3, 4).
template <unsigned M, typename IX>
__device__ __forceinline__ void stage_epsi(uint32_t dst, const K3 &g, IX o, unsigned f, bool xe) {
    const bool in = f & F_IN, z = in && (f & F_ZE), y = in && (f & F_YE), x = in && xe;
    const bool on[6] = {y, z, z, x, x, y};
    constexpr unsigned ax[6] = {AXY, AXZ, AXZ, AXX, AXX, AXY};
#pragma unroll
    for (int e = 0; e < 6; ++e)
        if (M & ax[e]) cp_async4(dst + e * NT3 * 4, on[e] ? g.pr[6 + e] + o : g.pr[6 + e], on[e]);
}

// psi values of one cell (E-psi: ex_y, ex_z, ey_z, ey_x, ez_x, ez_y)
struct P6 {
    float v[6];
};

// E-psi values of one cell: ex_y, ex_z, ey_z, ey_x, ez_x, ez_y (LENS_PSI_* 6..11),
// of the axes in M
template <unsigned M, typename IX>
__device__ __forceinline__ void load_epsi(P6 &p, const K3 &g, IX o, unsigned f, bool xe) {
#pragma unroll
    for (int q = 0; q < 6; ++q) p.v[q] = 0.f;
    if ((M & AXY) && (f & F_YE)) {
        p.v[0] = ldg_early(g.pr[LENS_PSI_EX_Y] + o);
        p.v[5] = ldg_early(g.pr[LENS_PSI_EZ_Y] + o);
    }
    if ((M & AXZ) && (f & F_ZE)) {
        p.v[1] = ldg_early(g.pr[LENS_PSI_EX_Z] + o);
        p.v[2] = ldg_early(g.pr[LENS_PSI_EY_Z] + o);
    }
    if ((M & AXX) && xe) {
        p.v[3] = ldg_early(g.pr[LENS_PSI_EY_X] + o);
        p.v[4] = ldg_early(g.pr[LENS_PSI_EZ_X] + o);
    }
}

struct F3 {
    float x, y, z;
};

// New H of one cell from old H and E around it (boundaries3d.py:311-331):
//   e = E(i,j,k); exk, eyk = E(i,j,k+1); exj, ezj = E(i,j+1,k); eyn, ezn = E(i+1,j,k).
// iok: i < nx-1 (Hy, Hz exist).  ST: CPML tile (psi corrections in the strips).
// zt / yt: the cell's entries of the z / y profile tables; x: this plane's x values.
template <bool ST, unsigned M, typename IX>
__device__ __forceinline__ F3 h_new(const K3 &g, F3 h, float ex, float ey, float ez, float exk, float eyk,
                                    float exj, float ezj, float eyn, float ezn, unsigned f, bool iok,
                                    const float *zt, const float *yt, const PX &x, const float *hs, IX o,
                                    bool wr, bool xh) {
    // hs: this cell's staged H-psi, component q at hs[q * NT3]
    const float ch = g.ch;
    const float d1x = eyk - ey, d2x = ezj - ez;
    const float d1y = ezn - ez, d2y = exk - ex;
    const float d1z = exj - ex, d2z = eyn - ey;
    // !ST: a CPML-free interior tile (every component of every cell updates)
    if (!ST || (f & F_HX)) {
        float v = h.x + ch * (d1x - d2x);
        if (ST) {
            if ((M & AXZ) && (f & F_ZH)) v = v + ch * psi_u(zt[0], zt[ZN], zt[2 * ZN], hs[0 * NT3], d1x, g.pw[LENS_PSI_HX_Z], o, wr);
            if ((M & AXY) && (f & F_YH)) v = v + (-ch) * psi_u(yt[0], yt[YN], yt[2 * YN], hs[1 * NT3], d2x, g.pw[LENS_PSI_HX_Y], o, wr);
        }
        h.x = v;
    }
    if (!ST || (iok && (f & F_HY))) {
        float v = h.y + ch * (d1y - d2y);
        if (ST) {
            if ((M & AXX) && xh) v = v + ch * psi_u(x.hb, x.hc, x.hk, hs[2 * NT3], d1y, g.pw[LENS_PSI_HY_X], o, wr);
            if ((M & AXZ) && (f & F_ZH)) v = v + (-ch) * psi_u(zt[0], zt[ZN], zt[2 * ZN], hs[3 * NT3], d2y, g.pw[LENS_PSI_HY_Z], o, wr);
        }
        h.y = v;
    }
    if (!ST || (iok && (f & F_HZ))) {
        float v = h.z + ch * (d1z - d2z);
        if (ST) {
            if ((M & AXY) && (f & F_YH)) v = v + ch * psi_u(yt[0], yt[YN], yt[2 * YN], hs[4 * NT3], d1z, g.pw[LENS_PSI_HZ_Y], o, wr);
            if ((M & AXX) && xh) v = v + (-ch) * psi_u(x.hb, x.hc, x.hk, hs[5 * NT3], d2z, g.pw[LENS_PSI_HZ_X], o, wr);
        }
        h.z = v;
    }
    return h;
}

// Coefficients of one cell: ce_x, ce_y, ce_z and (lossy) D_x, D_y, D_z.
struct C6 {
    float cx, cy, cz, dx, dy, dz;
};

template <typename IX>
__device__ __forceinline__ void load_coef(C6 &c, const K3 &g, IX o, bool lossy) {
    c.cx = __ldg(g.ce_x + o);
    c.cy = __ldg(g.ce_y + o);
    c.cz = __ldg(g.ce_z + o);
    if (lossy) {
        c.dx = __ldg(g.da_x + o);
        c.dy = __ldg(g.da_y + o);
        c.dz = __ldg(g.da_z + o);
    } else {
        c.dx = c.dy = c.dz = 1.f;
    }
}

// Plane-uniform data of the E update.
struct PlE {
    bool iok, iin, pec_i, xe, src;
    float sgn;  // +1 on plane src.ix, -1 on src.ix+1
    float env, wt;
};

// New E of one cell (boundaries3d.py:333-362, fdtd3d_core.py:1116-1127):
//   D*E, curl of the new H (h = H(i,j,k), hxk/hyk = H(i,j,k-1), hxj/hzj = H(i,j-1,k),
//   hym/hzm = H(i-1,j,k)), psi in the strips, PEC on the absorbing faces, source.
template <bool ST, unsigned M, typename IX>
__device__ __forceinline__ F3 e_new(const K3 &g, F3 e, F3 h, float hxk, float hyk, float hxj, float hzj,
                                    float hym, float hzm, const C6 &c, unsigned f, const PlE &pl, int j,
                                    int k, const float *zt, const float *yt, const PX &x, const P6 &ps,
                                    IX o) {
    const float d1x = h.z - hzj, d2x = h.y - hyk;  // Ex
    const float d1y = h.x - hxk, d2y = h.z - hzm;  // Ey
    const float d1z = h.y - hym, d2z = h.x - hxj;  // Ez
    float vx = e.x * c.dx, vy = e.y * c.dy, vz = e.z * c.dz;
    // !ST: a CPML-free interior tile (all curl terms apply, no PEC, all components exist)
    const bool ux = !ST || (pl.iok && (f & F_EXU)), uy = !ST || (pl.iin && (f & F_EYU)),
               uz = !ST || (pl.iin && (f & F_EZU));
    if (ux) vx = vx + c.cx * (d1x - d2x);
    if (uy) vy = vy + c.cy * (d1y - d2y);
    if (uz) vz = vz + c.cz * (d1z - d2z);
    if (ST) {
        if (ux) {
            if ((M & AXY) && (f & F_YE)) vx = vx + c.cx * psi_u(yt[3 * YN], yt[4 * YN], yt[5 * YN], ps.v[0], d1x, g.pw[LENS_PSI_EX_Y], o, true);
            if ((M & AXZ) && (f & F_ZE)) vx = vx + (-c.cx) * psi_u(zt[3 * ZN], zt[4 * ZN], zt[5 * ZN], ps.v[1], d2x, g.pw[LENS_PSI_EX_Z], o, true);
        }
        if (uy) {
            if ((M & AXZ) && (f & F_ZE)) vy = vy + c.cy * psi_u(zt[3 * ZN], zt[4 * ZN], zt[5 * ZN], ps.v[2], d1y, g.pw[LENS_PSI_EY_Z], o, true);
            if ((M & AXX) && pl.xe) vy = vy + (-c.cy) * psi_u(x.eb, x.ec, x.ek, ps.v[3], d2y, g.pw[LENS_PSI_EY_X], o, true);
        }
        if (uz) {
            if ((M & AXX) && pl.xe) vz = vz + c.cz * psi_u(x.eb, x.ec, x.ek, ps.v[4], d1z, g.pw[LENS_PSI_EZ_X], o, true);
            if ((M & AXY) && (f & F_YE)) vz = vz + (-c.cz) * psi_u(yt[3 * YN], yt[4 * YN], yt[5 * YN], ps.v[5], d2z, g.pw[LENS_PSI_EZ_Y], o, true);
        }
    }
    if (ST) {
        if (!pl.iok || (f & (F_PJ | F_PK))) vx = 0.f;
        if (!(f & F_EYV) || pl.pec_i || (f & F_PK)) vy = 0.f;
        if (!(f & F_EZV) || pl.pec_i || (f & F_PJ)) vz = 0.f;
    }
    if (pl.src && j < g.src.nj && k < g.src.nk) {
        const size_t m = (size_t)j * g.src.pitch_k + k;
        const float *ph = pl.sgn > 0.f ? g.src.ph1 : g.src.ph2;
        const float s = pl.sgn * ((pl.env * sinf(pl.wt + __ldg(ph + m))) * __ldg(g.src.amp + m));
        if (g.src_comp == 0) vx += s;
        else if (g.src_comp == 1) vy += s;
        else vz += s;
    }
    return F3{vx, vy, vz};
}

// IX: index type of the field volumes (32-bit when nx*ny*pitch < 2^31).  ST: a
// tile that touches a CPML strip or a domain face (per-cell flags); M: the axes
// whose CPML psi the tile carries (a subset of ST tiles' work; 0 for faces only).
template <bool ST, unsigned M, typename IX>
__device__ __forceinline__ void tile3d(const EMaps &tm, const K3 &g, const LensStepTable &tab,
                                       const LensEpi3D &ep, int n, int epi, int k0, int j0, int x0,
                                       int x1, unsigned char *smem) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int nx = g.nx, ny = g.ny, P = g.P;
    const IX S = (IX)ny * P;
    const int xs = x0 > 0 ? x0 - 1 : 0;  // plane x0-1: its H feeds E(x0)
    const uint32_t sbase = s_addr(smem), bar0 = sbase + OFF_BAR, barh = bar0 + 8u * NSE;
    const float *sE = reinterpret_cast<const float *>(smem);
    const float *sHC = reinterpret_cast<const float *>(smem + OFF_HC);
    float *sH = reinterpret_cast<float *>(smem + OFF_SH);
    float *sZT = reinterpret_cast<float *>(smem + OFF_PT), *sYT = sZT + 6 * ZN;
    const bool lossy = g.da_x != nullptr;
    const int ncoef = lossy ? 6 : 3;
    const bool owner = w < NOW;
    const bool prod = (w == NOW && lane == 0);
    const int q0 = n - tab.t0;

    // ---- producer (lane 0 of the halo warp): E ring and H/coefficient ring.
    // E(p) sits in slot (p-xs) % NSE, HC(p) in slot (p-xs) % NHC; the u-th fill of a
    // slot completes mbarrier phase u.  Every thread waits itself for the planes it
    // reads (E(i+1) and HC(i) at the top of iteration i), so a late copy stalls only
    // the warps that need it; the CTA barrier of each plane orders the slot reuse.
    // After a wait gives up a thread awaits nothing more and the producer issues
    // nothing more (the flag reports it); the producer drains the copies in flight
    // (bounded) before the CTA exits.
    bool ok = true;
    int ie = xs - 1, we = xs - 1, ih = xs - 1, wh = xs - 1;
    // watchdog self-test (lens_fdtd3d_watchdog_test): CTA 0 withholds one plane's
    // E copy and every wait of the launch is bounded at a few hundred tries
    const bool wd = g.wd_plane >= 0;
    const int tries = wd ? 256 : (1 << 20);
    auto issue_e = [&](int p) {
        const int s = (p - xs) % NSE;
        const uint32_t bar = bar0 + 8u * s;
        if (wd && blockIdx.x == 0 && p == xs + g.wd_plane) {
            ie = p;  // never armed: the waits on this plane run out
            return;
        }
        mbar_expect(bar, 3 * E_BYTES);
#pragma unroll
        for (int q = 0; q < 3; ++q) tma3(sbase + (s * 3 + q) * E_SLOT, &tm.e[q], k0 - 4, j0 - 1, p, bar);
        ie = p;
    };
    // the coefficient boxes of plane p only where its 32-column group holds a
    // column without a type (the others come from the type table in shared memory)
    auto issue_hc = [&](int p) {
        const int s = (p - xs) % NHC;
        const uint32_t bar = barh + 8u * s, dst = sbase + OFF_HC + s * HC_SLOT;
        const int nc = (!g.ctype || g.cexpl[(size_t)p * (P / TK) + k0 / TK]) ? ncoef : 0;
        mbar_expect(bar, (3 + nc) * HT * 4);
#pragma unroll
        for (int q = 0; q < 3; ++q) tma3(dst + q * HT * 4, &tm.h[q], k0, j0, p, bar);
        for (int q = 0; q < nc; ++q) tma3(dst + (3 + q) * HT * 4, &tm.c[q], k0, j0, p, bar);
        ih = p;
    };
    if (prod) {
        for (int q = 0; q < NSE + NHC; ++q) mbar_init(bar0 + 8u * q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int p = xs; p <= min(x1, xs + NSE - 1); ++p) issue_e(p);
        for (int p = xs; p <= min(x1 - 1, xs + NHC - 1); ++p) issue_hc(p);
    }
    // consumer side: slot and phase parity of E(i), E(i+1) and HC(i) (ring counters)
    int se = 0, sn = 1 % NSE, sh = 0;
    unsigned pe = 0u, pn = NSE == 1 ? 1u : 0u, ph = 0u;

    // ---- per-thread cells.  Owners: rows a = j0+2w, b = a+1 at k = k0+lane.
    // Halo warp: A = (j0-1, k0+lane), B = (j0+lane, k0-1) for lane < TJ.
    const int k = owner ? k0 + lane : 0;
    const int ja = owner ? j0 + 2 * w : 0, jb = ja + 1;
    const int kA = k0 + lane, jA = j0 - 1, kB = k0 - 1, jB = j0 + lane;
    unsigned fa, fb;
    int ea, sa;            // E-box / new-H tile index of the first cell
    IX oa, ob;             // in-plane offsets
    if (owner) {
        fa = cell_flags(g, ep, ja, k);
        fb = cell_flags(g, ep, jb, k);
        ea = (2 * w + 1) * EK + lane + 4;
        sa = (2 * w + 1) * SHK + lane + 1;
        oa = (IX)ja * P + k;
        ob = oa + P;
    } else {
        fa = cell_flags(g, ep, jA, kA);
        fb = lane < TJ ? cell_flags(g, ep, jB, kB) : 0u;
        ea = lane + 4;
        sa = lane + 1;
        oa = (fa & F_IN) ? (IX)jA * P + kA : 0;
        ob = (fb & F_IN) ? (IX)jB * P + kB : 0;
    }
    const int hl = lane < TJ ? lane : TJ - 1;  // lanes >= TJ of the halo warp compute a discarded copy
    const int eb = owner ? ea + EK : (hl + 1) * EK + 3;
    const int sb = owner ? sa + SHK : (hl + 1) * SHK;
    const int ta = 2 * w * TK + lane;          // owner tile index of row a (row b: ta + TK)
    // profile-table entries of the two cells
    const float *zta = sZT + lane + 1, *ztb = owner ? zta : sZT;
    const float *yta = sYT + (owner ? 2 * w + 1 : 0), *ytb = owner ? yta + 1 : sYT + hl + 1;
    if (ST && (M & (AXZ | AXY))) {
        const int t = w * TK + lane;
        if ((M & AXZ) && t < ZN) {
            fill_row(sZT + t, ZN, g.az.h, k0 - 1 + t);
            fill_row(sZT + 3 * ZN + t, ZN, g.az.e, k0 - 1 + t);
        } else if ((M & AXY) && t >= ZN && t < ZN + YN) {
            fill_row(sYT + (t - ZN), YN, g.ay.h, j0 - 1 + (t - ZN));
            fill_row(sYT + 3 * YN + (t - ZN), YN, g.ay.e, j0 - 1 + (t - ZN));
        }
    }

    // halo warp: old H by loads one plane ahead; CPML tiles: psi one phase ahead
    //   after the H phase of plane i: halo old H of plane i+1, E-psi of plane i;
    //   after the E phase of plane i: H-psi of plane i+1.
    F3 hoa{0.f, 0.f, 0.f}, hob{0.f, 0.f, 0.f};
    P6 epa, epb;
    const int tid = w * 32 + lane;
    const uint32_t hs_s = sbase + OFF_HS + tid * 4;  // this thread's H-psi staging slot
    const float *hs_p = reinterpret_cast<const float *>(smem + OFF_HS) + tid;
    auto load_hold = [&](int p) {
        const IX base = (IX)p * S;
        if (fa & F_IN) hoa = F3{ldg_early(g.hx + base + oa), ldg_early(g.hy + base + oa), ldg_early(g.hz + base + oa)};
        if (fb & F_IN) hob = F3{ldg_early(g.hx + base + ob), ldg_early(g.hy + base + ob), ldg_early(g.hz + base + ob)};
    };
    // H-psi of plane p into staging buffer (p - xs) & 1 (cp.async, one plane ahead)
    auto stage_hp = [&](int p) {
        const IX base = (IX)p * S;
        const bool xh = (M & AXX) && in_strip(g.ax.h, p);
        const uint32_t d = hs_s + (((unsigned)(p - xs) & 1u) * HS_STAGE) * 4;
        stage_hpsi<M>(d, g, base + oa, fa, xh);
        stage_hpsi<M>(d + 6 * NT3 * 4, g, base + ob, fb, xh);
        if (single_axis<M>() && owner && p >= x0) {  // E-psi of plane p, read in its E phase
            const bool xe = (M & AXX) && in_strip(g.ax.e, p);
            stage_epsi<M>(d, g, base + oa, fa, xe);
            stage_epsi<M>(d + 6 * NT3 * 4, g, base + ob, fb, xe);
        }
        cp_async_commit();
    };
    auto load_ep = [&](int p) {
        const IX base = (IX)p * S;
        const bool xe = (M & AXX) && in_strip(g.ax.e, p);
        if (fa & F_IN) load_epsi<M>(epa, g, base + oa, fa, xe);
        if (fb & F_IN) load_epsi<M>(epb, g, base + ob, fb, xe);
    };
    if (!owner) load_hold(xs);
    if (ST && M) stage_hp(xs);
    if (ST && M && !single_axis<M>() && owner) load_ep(x0);
    // coefficient column types: the tile's rows of the type table into shared
    // memory; each owner lane's column type one plane ahead
    float *sCT = reinterpret_cast<float *>(smem + OFF_CT);
    const bool ccol = g.ctype != nullptr;
    if (ccol)
        for (int t = tid; t < g.ntype * 6 * TJ; t += NT3) {
            const int r = t % TJ, q = t / TJ;
            sCT[t] = j0 + r < ny ? __ldg(g.ctab + (size_t)q * ny + j0 + r) : 0.f;
        }
    unsigned tcn = (owner && ccol) ? ldg_u8_early(g.ctype + (IX)xs * P + k) : 255u;

    const float env = tab.env[q0], wt = tab.wt[q0];

    // E(i) of the owner cells at (j, k): Ey, Ez carried from the previous plane's "next" reads
    float cya = 0.f, cza = 0.f, cyb = 0.f, czb = 0.f;
    float hyma = 0.f, hzma = 0.f, hymb = 0.f, hzmb = 0.f;  // new H(i-1)
    __syncthreads();  // the mbarriers are initialised
    if (ok) ok = mbar_wait(bar0, 0u, tries);  // E(xs)
    if (prod && ok) we = xs;
    if (owner) {  // plane xs sits in slot 0
        cya = sE[EF + ea];
        cza = sE[2 * EF + ea];
        cyb = sE[EF + eb];
        czb = sE[2 * EF + eb];
    }

    for (int i = xs; i < x1; ++i) {
        const bool eon = i >= x0;
        const unsigned u = i - xs;
        const unsigned tc = tcn;  // column type of (i, k)
        if (owner && ccol && i + 1 < x1) tcn = ldg_u8_early(g.ctype + (IX)(i + 1) * P + k);
        if (ok) ok = mbar_wait(bar0 + 8u * sn, pn, tries);   // E(i+1)
        if (ok) ok = mbar_wait(barh + 8u * sh, ph, tries);   // HC(i)
        if (prod && ok) { we = i + 1; wh = i; }
        const float *eC = sE + se * 3 * EF, *eN = sE + sn * 3 * EF;
        const float *hc = sHC + sh * (HC_SLOT / 4);
        float *shw = sH + (u & 1) * 3 * SH_N;
        const bool iok = i < nx - 1;
        const bool xh = ST && (M & AXX) && in_strip(g.ax.h, i);
        const PX px = (ST && (M & AXX)) ? px_at(g, i) : PX{};
        const IX base = (IX)i * S;
        F3 ha{0.f, 0.f, 0.f}, hb{0.f, 0.f, 0.f};
        float exa = 0.f, exb = 0.f, nya = 0.f, nza = 0.f, nyb = 0.f, nzb = 0.f;
        const float *hs = hs_p + (u & 1u) * HS_STAGE;  // staged H-psi of plane i (own slots)
        if (ST && M) cp_async_wait_all();
        // ---------------- H(i)
        if (owner) {
            exa = eC[ea];
            const float exa1 = eC[ea + 1], eya1 = eC[EF + ea + 1];
            exb = eC[eb];
            const float exb1 = eC[eb + 1], eyb1 = eC[EF + eb + 1];
            const float exc = eC[eb + EK], ezc = eC[2 * EF + eb + EK];
            nya = eN[EF + ea];
            nza = eN[2 * EF + ea];
            nyb = eN[EF + eb];
            nzb = eN[2 * EF + eb];
            const F3 h0a{hc[ta], hc[HT + ta], hc[2 * HT + ta]};
            const F3 h0b{hc[ta + TK], hc[HT + ta + TK], hc[2 * HT + ta + TK]};
            const bool wr = eon;
            ha = h_new<ST, M, IX>(g, h0a, exa, cya, cza, exa1, eya1, exb, czb, nya, nza, fa, iok, zta, yta, px,
                               hs, base + oa, wr, xh);
            hb = h_new<ST, M, IX>(g, h0b, exb, cyb, czb, exb1, eyb1, exc, ezc, nyb, nzb, fb, iok, ztb, ytb, px,
                               hs + 6 * NT3, base + ob, wr, xh);
        } else if (eon) {
            // halo cells: A on row 0 of the boxes, B on column 0 (read-only psi)
            const float *c = eC + ea;
            ha = h_new<ST, M, IX>(g, hoa, c[0], c[EF], c[2 * EF], c[1], c[EF + 1], c[EK], c[2 * EF + EK],
                               eN[EF + ea], eN[2 * EF + ea], fa, iok, zta, yta, px, hs, base + oa, false, xh);
            const float *d = eC + eb;
            hb = h_new<ST, M, IX>(g, hob, d[0], d[EF], d[2 * EF], d[1], d[EF + 1], d[EK], d[2 * EF + EK],
                               eN[EF + eb], eN[2 * EF + eb], fb, iok, ztb, ytb, px, hs + 6 * NT3, base + ob, false, xh);
        }
        if (owner || eon) {
            shw[sa] = ha.x;
            shw[SH_N + sa] = ha.y;
            shw[2 * SH_N + sa] = ha.z;
            if (owner || lane < TJ) {
                shw[sb] = hb.x;
                shw[SH_N + sb] = hb.y;
                shw[2 * SH_N + sb] = hb.z;
            }
        }
        if (!owner && i + 1 < x1) load_hold(i + 1);
        if (ST && M && i + 1 < x1) stage_hp(i + 1);
        __syncthreads();
        if (prod && ok) {
            if (i + NSE <= x1) issue_e(i + NSE);                        // E(i)'s slot is free
            if (i - 1 >= xs && i - 1 + NHC <= x1 - 1) issue_hc(i - 1 + NHC);  // HC(i-1)'s slot is free
        }

        // ---------------- E(i)
        if (owner && eon) {
            PlE pl;
            pl.iok = iok;
            pl.iin = i >= 1 && i <= nx - 2;
            pl.pec_i = (g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1);
            pl.xe = ST && (M & AXX) && in_strip(g.ax.e, i);
            pl.src = g.src.ix >= 0 && (i == g.src.ix || i == g.src.ix + 1);
            pl.sgn = i == g.src.ix ? 1.f : -1.f;
            pl.env = env;
            pl.wt = wt;
            const float hxja = shw[sa - SHK], hzja = shw[2 * SH_N + sa - SHK];
            const float hxka = shw[sa - 1], hyka = shw[SH_N + sa - 1];
            const float hxkb = shw[sb - 1], hykb = shw[SH_N + sb - 1];
            // coefficients: the staged boxes (a column without a type) or the type table
            const bool tb = tc != 255u;
            const float *cs = tb ? sCT + tc * (6 * TJ) + 2 * w : hc + 3 * HT + ta;
            const int st = tb ? TJ : HT, nb = tb ? 1 : TK;  // coefficient stride, row b offset
            const C6 ca{cs[0], cs[st], cs[2 * st], lossy ? cs[3 * st] : 1.f, lossy ? cs[4 * st] : 1.f,
                        lossy ? cs[5 * st] : 1.f};
            cs += nb;
            const C6 cb{cs[0], cs[st], cs[2 * st], lossy ? cs[3 * st] : 1.f, lossy ? cs[4 * st] : 1.f,
                        lossy ? cs[5 * st] : 1.f};
            if (ST && single_axis<M>()) {  // E-psi staged beside the H-psi of this plane
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    epa.v[e] = hs[e * NT3];
                    epb.v[e] = hs[(6 + e) * NT3];
                }
            }
            const F3 Ea = e_new<ST, M, IX>(g, F3{exa, cya, cza}, ha, hxka, hyka, hxja, hzja, hyma, hzma, ca, fa,
                                        pl, ja, k, zta, yta, px, epa, base + oa);
            const F3 Eb = e_new<ST, M, IX>(g, F3{exb, cyb, czb}, hb, hxkb, hykb, ha.x, ha.z, hymb, hzmb, cb, fb,
                                        pl, jb, k, ztb, ytb, px, epb, base + ob);
            if (!ST || (fa & F_IN)) {
                const IX o = base + oa;
                g.whx[o] = ha.x; g.why[o] = ha.y; g.whz[o] = ha.z;
                g.wex[o] = Ea.x; g.wey[o] = Ea.y; g.wez[o] = Ea.z;
            }
            if (!ST || (fb & F_IN)) {
                const IX o = base + ob;
                g.whx[o] = hb.x; g.why[o] = hb.y; g.whz[o] = hb.z;
                g.wex[o] = Eb.x; g.wey[o] = Eb.y; g.wez[o] = Eb.z;
            }
        }
        if (ST && M && !single_axis<M>() && owner && i + 1 < x1) load_ep(i + 1);
        // carry; advance the ring counters
        cya = nya; cza = nza; cyb = nyb; czb = nzb;
        hyma = ha.y; hzma = ha.z; hymb = hb.y; hzmb = hb.z;
        se = sn; pe = pn;
        if (++sn == NSE) { sn = 0; pn ^= 1u; }
        if (++sh == NHC) { sh = 0; ph ^= 1u; }
    }
    if (!ok && g.flag) atomicOr(g.flag, 1);
    if (prod && !ok) {
        for (int p = we + 1; p <= ie; ++p) mbar_wait(bar0 + 8u * ((p - xs) % NSE), ((p - xs) / NSE) & 1, tries);
        for (int p = wh + 1; p <= ih; ++p) mbar_wait(barh + 8u * ((p - xs) % NHC), ((p - xs) / NHC) & 1, tries);
        if (g.flag) atomicOr(g.flag, 1);
    }
}

template <typename IX>
__global__ void __launch_bounds__(NW3 * 32, 2)
    yee3d(const __grid_constant__ EMaps tm, const K3 g, const LensStepTable tab, const LensEpi3D ep, int n,
          int epi, const __grid_constant__ Work wk) {
    int tz, ty, c;
    const bool lean = work_tile(wk, blockIdx.x < wk.nperm ? (int)wk.perm[blockIdx.x] : (int)blockIdx.x, tz, ty, c);
    extern __shared__ __align__(128) unsigned char smem[];
    const int k0 = tz * TK, j0 = ty * TJ, x0 = wk.x[c], x1 = wk.x[c + 1];
    if (lean) {
        tile3d<false, 0u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem);
        return;
    }
    if (sizeof(IX) > 4) {  // very large grids: one generic CPML pass
        tile3d<true, AXALL, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem);
        return;
    }
    const unsigned m = ((tz < wk.plo[0] || tz >= wk.phi[0]) ? AXZ : 0u) |
                       ((ty < wk.plo[1] || ty >= wk.phi[1]) ? AXY : 0u) |
                       ((c < wk.plo[2] || c >= wk.phi[2]) ? AXX : 0u);
    switch (m) {  // tile pass specialised on the CPML axes it carries
        case 0u: tile3d<true, 0u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        case 1u: tile3d<true, 1u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        case 2u: tile3d<true, 2u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        case 3u: tile3d<true, 3u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        case 4u: tile3d<true, 4u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        case 5u: tile3d<true, 5u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        case 6u: tile3d<true, 6u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
        default: tile3d<true, 7u, IX>(tm, g, tab, ep, n, epi, k0, j0, x0, x1, smem); break;
    }
}

// Window epilogue after a fused step (DFT / convergence windows): volume DFTs,
// convergence planes and flux planes of the NEW fields (g reads the buffer the
// step wrote).  A separate streaming pass keeps the step kernel's registers for
// its pipeline: it reads E once (12 B per cell) and updates the complex
// accumulators (16 B per component and cell) on window steps only.
constexpr int WK = 4;  // window epilogue: cells per thread along z

__global__ void __launch_bounds__(NT) win3d(const K3 g, const LensStepTable tab, const LensEpi3D ep, int n) {
    const int k0 = (blockIdx.x * BK + threadIdx.x) * WK, j = blockIdx.y * BJ + threadIdx.y, i = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    if (k0 >= P || j >= ny) return;  // no warp-collective operations below
    const size_t S = (size_t)ny * P, o = i * S + (size_t)j * P + k0;
    const bool win = n >= ep.dft_n0 && n < ep.dft_n1;
    const int q = n - tab.t0;
    const float pr = tab.pe[2 * q], pim = tab.pe[2 * q + 1];
    // E of WK cells; the step leaves zero wherever a component does not exist
    // (its last plane / row / column, the z padding), so those sums stay zero
    const float4 E[3] = {*reinterpret_cast<const float4 *>(g.ex + o), *reinterpret_cast<const float4 *>(g.ey + o),
                         *reinterpret_cast<const float4 *>(g.ez + o)};
    if (win) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (!ep.dft[c]) continue;
            float4 *a = reinterpret_cast<float4 *>(ep.dft[c] + 2 * o);
            float4 s0 = a[0], s1 = a[1];
            s0.x += E[c].x * pr; s0.y += E[c].x * pim; s0.z += E[c].y * pr; s0.w += E[c].y * pim;
            s1.x += E[c].z * pr; s1.y += E[c].z * pim; s1.z += E[c].w * pr; s1.w += E[c].w * pim;
            a[0] = s0;
            a[1] = s1;
        }
    }
    const bool conv = (win && ep.conv_last) || (ep.conv_prev && n >= ep.prev_n0 && n < ep.prev_n1);
    bool fl = false;
    for (int p = 0; p < ep.nplane; ++p) fl |= (i == ep.plane[p]);
    const bool cz = conv && ep.conv_k >= k0 && ep.conv_k < k0 + WK;
    if (!cz && !(win && fl)) return;
    const float ev[3][WK] = {{E[0].x, E[0].y, E[0].z, E[0].w}, {E[1].x, E[1].y, E[1].z, E[1].w},
                             {E[2].x, E[2].y, E[2].z, E[2].w}};
#pragma unroll
    for (int m = 0; m < WK; ++m) {
        const int k = k0 + m;
        if (k >= nz || !((cz && k == ep.conv_k) || (win && fl))) continue;
        const size_t om = o + m;
        Hv h{0.f, 0.f, 0.f};
        float hym = 0.f, hzm = 0.f;
        if (fl) {
            h = Hv{g.hx[om], g.hy[om], g.hz[om]};
            hym = g.hy[om - S];
            hzm = g.hz[om - S];
        }
        epi_cell(g, tab, ep, n, i, j, k, true, Hv{ev[0][m], ev[1][m], ev[2][m]}, hym, hzm, h, false, false);
    }
}

// ============================================================ detector boxes
// Detector box sums of the new E after a fused step (fdtd3d_core.py:477-481):
// sum over the box of Ex^2 + Ey^2 + Ez^2, each component over its own slice
// (box_end), squares in float32 summed in FP64.  One launch for every box:
// blockIdx.z runs over the boxes' planes in groups of BOXX (xb[b] is the first
// group of box b); all loads of a thread are issued before its sums; one FP64
// atomic per CTA.
constexpr int BOXX = 2;

struct BoxGrid {
    int xb[LENS_MAX_BOX + 1];
};

__global__ void __launch_bounds__(NT) box3d(const K3 g, const LensEpi3D ep, const BoxGrid bg) {
    int b = 0;
    while (b + 1 < ep.nbox && (int)blockIdx.z >= bg.xb[b + 1]) ++b;
    const int *bx = ep.box[b];
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const int k = bx[4] + blockIdx.x * BK + threadIdx.x, j = bx[2] + blockIdx.y * BJ + threadIdx.y;
    const int i0 = bx[0] + ((int)blockIdx.z - bg.xb[b]) * BOXX, i1 = min(i0 + BOXX, box_end(bx[1], nx));
    const bool col = j >= 0 && j < ny && k >= 0 && k < nz && k < box_end(bx[5], nz) && j < box_end(bx[3], ny);
    float e[BOXX][3];
#pragma unroll
    for (int q = 0; q < BOXX; ++q) {
        const int i = i0 + q;
        const size_t o = ((size_t)i * ny + j) * P + k;
        const bool pl = col && i >= 0 && i < i1;
        e[q][0] = (pl && i < nx - 1 && in_box(bx, 0, i, j, k, nx, ny, nz)) ? g.ex[o] : 0.f;
        e[q][1] = (pl && j < ny - 1 && in_box(bx, 1, i, j, k, nx, ny, nz)) ? g.ey[o] : 0.f;
        e[q][2] = (pl && k < nz - 1 && in_box(bx, 2, i, j, k, nx, ny, nz)) ? g.ez[o] : 0.f;
    }
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < BOXX; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) v += (double)(e[q][c] * e[q][c]);
    __shared__ double red[NT / 32];
    v = warp_sum(v);
    if (threadIdx.x == 0) red[threadIdx.y] = v;
    __syncthreads();
    if (threadIdx.y == 0) {
        v = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0 && v != 0.0) atomicAdd(ep.box_acc + b, v);
        // a NaN or infinity in a detector box marks the solve invalid (flag bit 2)
        if (threadIdx.x == 0 && g.flag && !isfinite(v)) atomicOr(g.flag, 2);
    }
}

// ============================================================ stitch drive
// Soft injection of the previous window's CW field into the first O x-planes of
// the new E (fdtd3d_core.py:1614-1617): for Ex, Ey and Ez
//   F = w_i * (env * Re(D e^{+i w t})) + (1 - w_i) * F
// with D the handed-over complex amplitude and w_i the cosine taper.  Rounded
// operation by operation (no contraction) like the complex64 / float32 NumPy
// expression; e^{+iwt} is the conjugate of the table's DFT phase.
__global__ void __launch_bounds__(NT) drive3d(const K3 g, const LensStepTable tab, const LensDrive3D d, int n) {
    const int k = blockIdx.x * BK + threadIdx.x, j = blockIdx.y * BJ + threadIdx.y, i = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (k >= nz || j >= ny || i >= d.nplanes) return;
    const size_t o = ((size_t)i * ny + j) * g.P + k;
    const int q = n - tab.t0;
    const float c = tab.pe[2 * q], s = -tab.pe[2 * q + 1], env = tab.env[q];
    const float w = d.taper[i], w1 = d.taper[d.nplanes + i];
    float *F[3] = {g.wex, g.wey, g.wez};
    const bool ok[3] = {i < nx - 1, j < ny - 1, k < nz - 1};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        if (!ok[m]) continue;
        const float2 D = reinterpret_cast<const float2 *>(d.hand[m])[o];
        const float re = __fsub_rn(__fmul_rn(D.x, c), __fmul_rn(D.y, s));
        const float v = __fmul_rn(w, __fmul_rn(env, re));
        F[m][o] = __fadd_rn(v, __fmul_rn(w1, F[m][o]));
    }
}

// ============================================================ Iavg
// Square of component F mapped onto the target grid (fdtd3d_core.py:438-461):
// x: equal extent or one shorter (mean of the clipped neighbours i-1, i);
// y, z: one longer (mean of j, j+1) or one shorter (edges copied, else mean of j-1, j).
struct Ext {
    int nx, ny, nz;
};

__device__ __forceinline__ float sqx(const float *F, const Ext &f, int tnx, int P, int ny, int i, int j,
                                     int k) {
    if (f.nx == tnx) {
        const float a = F[((size_t)i * ny + j) * P + k];
        return a * a;
    }
    const int i0 = min(max(i - 1, 0), f.nx - 1), i1 = min(max(i, 0), f.nx - 1);
    const float a = F[((size_t)i0 * ny + j) * P + k], b = F[((size_t)i1 * ny + j) * P + k];
    return 0.5f * (a * a + b * b);
}

__device__ __forceinline__ float sqxy(const float *F, const Ext &f, const Ext &t, int P, int ny, int i,
                                      int j, int k) {
    if (f.ny == t.ny) return sqx(F, f, t.nx, P, ny, i, j, k);
    if (f.ny == t.ny + 1)
        return 0.5f * (sqx(F, f, t.nx, P, ny, i, j, k) + sqx(F, f, t.nx, P, ny, i, j + 1, k));
    if (j == 0) return sqx(F, f, t.nx, P, ny, i, 0, k);
    if (j == t.ny - 1) return sqx(F, f, t.nx, P, ny, i, f.ny - 1, k);
    return 0.5f * (sqx(F, f, t.nx, P, ny, i, j - 1, k) + sqx(F, f, t.nx, P, ny, i, j, k));
}

__device__ __forceinline__ float sq_on_grid(const float *F, const Ext &f, const Ext &t, int P, int ny,
                                            int i, int j, int k) {
    if (f.nz == t.nz) return sqxy(F, f, t, P, ny, i, j, k);
    if (f.nz == t.nz + 1) return 0.5f * (sqxy(F, f, t, P, ny, i, j, k) + sqxy(F, f, t, P, ny, i, j, k + 1));
    if (k == 0) return sqxy(F, f, t, P, ny, i, j, 0);
    if (k == t.nz - 1) return sqxy(F, f, t, P, ny, i, j, f.nz - 1);
    return 0.5f * (sqxy(F, f, t, P, ny, i, j, k - 1) + sqxy(F, f, t, P, ny, i, j, k));
}

// nxt <= nx: only planes [0, nxt) of the components take part, as for the slices
// Ex[:nxt-1], Ey[:nxt], Ez[:nxt] (fdtd3d_core.py:1650).
__global__ void __launch_bounds__(NT) accum_e2(const K3 g, int target, int nxt, float *iavg) {
    const int k = blockIdx.x * BK + threadIdx.x, j = blockIdx.y * BJ + threadIdx.y, i = blockIdx.z;
    const int ny = g.ny, nz = g.nz, P = g.P;
    const Ext ex{nxt - 1, ny, nz}, ey{nxt, ny - 1, nz}, ez{nxt, ny, nz - 1};
    const Ext t = target == 1 ? ey : ez;
    if (i >= t.nx || j >= t.ny || k >= t.nz) return;
    const float a = sq_on_grid(g.ex, ex, t, P, ny, i, j, k);
    const float b = sq_on_grid(g.ey, ey, t, P, ny, i, j, k);
    const float d = sq_on_grid(g.ez, ez, t, P, ny, i, j, k);
    iavg[((size_t)i * ny + j) * P + k] += (a + b) + d;
}

// ============================================================ host side
bool ax_ok(const LensAxis &a, int n) { return lens_profile_ok(a.e, n) && lens_profile_ok(a.h, n - 1); }

int psi_width(const LensGrid3D *g, int q) {
    switch (q) {
        case LENS_PSI_HX_Z: case LENS_PSI_HY_Z: return g->az.h.lo + g->az.h.hi;
        case LENS_PSI_EX_Z: case LENS_PSI_EY_Z: return g->az.e.lo + g->az.e.hi;
        case LENS_PSI_HX_Y: case LENS_PSI_HZ_Y: return g->ay.h.lo + g->ay.h.hi;
        case LENS_PSI_EX_Y: case LENS_PSI_EZ_Y: return g->ay.e.lo + g->ay.e.hi;
        case LENS_PSI_HY_X: case LENS_PSI_HZ_X: return g->ax.h.lo + g->ax.h.hi;
        default: return g->ax.e.lo + g->ax.e.hi;
    }
}

bool buffer_ok(const LensGrid3D *g, int b) {
    for (int c = 0; c < 6; ++c)
        if (!g->f[b][c]) return false;
    for (int q = 0; q < LENS_NPSI; ++q)
        if (psi_width(g, q) > 0 && !g->psi[b][q]) return false;
    return true;
}

bool has_buffer1(const LensGrid3D *g) {
    for (int c = 0; c < 6; ++c)
        if (g->f[1][c]) return true;
    return false;
}

bool grid3d_ok(const LensGrid3D *g) {
    if (!g || g->nx < 3 || g->ny < 3 || g->nz < 3 || g->pitch < g->nz || (g->pitch % 32)) return false;
    if (g->cur != 0 && g->cur != 1) return false;
    if (!buffer_ok(g, g->cur)) return false;
    if (has_buffer1(g) && !buffer_ok(g, 1 - g->cur)) return false;
    if (!g->ce_x || !g->ce_y || !g->ce_z) return false;
    const bool d0 = !g->da_x, d1 = !g->da_y, d2 = !g->da_z;
    if (d0 != d1 || d1 != d2) return false;
    if (!ax_ok(g->ax, g->nx) || !ax_ok(g->ay, g->ny) || !ax_ok(g->az, g->nz)) return false;
    if (g->ctype && (!g->ctab || !g->cexpl || g->ntype < 1 || g->ntype > LENS_MAX_CTYPE)) return false;
    if (g->src.ix >= 0) {
        if (!g->src.amp || !g->src.ph1 || !g->src.ph2 || g->src.ix + 1 >= g->nx) return false;
        if (g->src_comp < 0 || g->src_comp > 2 || g->src.pitch_k < g->src.nk) return false;
        if (g->src.nj < 0 || g->src.nk < 0) return false;
    }
    return true;
}

bool epi3d_ok(const LensEpi3D *ep, const LensStepTable *t, const LensGrid3D *g) {
    if (!ep) return true;
    if (ep->nbox < 0 || ep->nbox > LENS_MAX_BOX || (ep->nbox > 0 && !ep->box_acc)) return false;
    if (ep->nplane < 0 || ep->nplane > LENS_MAX_PLANE || (ep->nplane > 0 && !ep->plane_acc)) return false;
    for (int p = 0; p < ep->nplane; ++p)
        if (ep->plane[p] < 1 || ep->plane[p] > g->nx - 2) return false;
    const bool dft = ep->dft[0] || ep->dft[1] || ep->dft[2] || ep->nplane > 0 || ep->conv_prev ||
                     ep->conv_last;
    return !dft || (t->pe && t->ph);
}

int epi3d_active(const LensEpi3D *e, int n) {
    if (e->nbox > 0) return 1;
    if (n >= e->dft_n0 && n < e->dft_n1 &&
        (e->dft[0] || e->dft[1] || e->dft[2] || e->nplane > 0 || e->conv_last))
        return 1;
    return (e->conv_prev && n >= e->prev_n0 && n < e->prev_n1) ? 1 : 0;
}

// Kernel view: read buffer rb, write buffer wb (equal for the in-place passes).
K3 view(const LensGrid3D *g, int rb, int wb) {
    K3 k{};
    k.nx = g->nx; k.ny = g->ny; k.nz = g->nz; k.P = g->pitch;
    k.ex = g->f[rb][0]; k.ey = g->f[rb][1]; k.ez = g->f[rb][2];
    k.hx = g->f[rb][3]; k.hy = g->f[rb][4]; k.hz = g->f[rb][5];
    k.wex = g->f[wb][0]; k.wey = g->f[wb][1]; k.wez = g->f[wb][2];
    k.whx = g->f[wb][3]; k.why = g->f[wb][4]; k.whz = g->f[wb][5];
    for (int q = 0; q < LENS_NPSI; ++q) {
        k.pr[q] = g->psi[rb][q];
        k.pw[q] = g->psi[wb][q];
    }
    k.ce_x = g->ce_x; k.ce_y = g->ce_y; k.ce_z = g->ce_z;
    k.da_x = g->da_x; k.da_y = g->da_y; k.da_z = g->da_z;
    k.ch = g->ch; k.ax = g->ax; k.ay = g->ay; k.az = g->az;
    for (int q = 0; q < 6; ++q) k.pec[q] = g->pec[q];
    k.src = g->src; k.src_comp = g->src_comp; k.flag = g->flag;
    k.ctype = g->ctype; k.cexpl = g->cexpl; k.ctab = g->ctab; k.ntype = g->ntype;
    k.wd_plane = -1;
    return k;
}

// x-chunks of the fused pass: the planes that carry x CPML psi get chunks of
// their own, the rest is cut into pieces of about `target` planes.  Returns the
// chunk count; x[c] is the first plane of chunk c, strip[c] != 0 for CPML chunks.
int make_chunks(const LensGrid3D *g, int target, int *x, int *strip) {
    const int nx = g->nx;
    int n = 0;
    int lo = g->ax.h.lo > g->ax.e.lo ? g->ax.h.lo : g->ax.e.lo;
    int hi = nx - 1 - g->ax.h.hi;
    if (nx - g->ax.e.hi < hi) hi = nx - g->ax.e.hi;
    lo = lo > 0 ? lo + 1 : 0;  // the next chunk's warm-up plane lo must be strip-free too
    if (hi < lo) hi = lo;
    auto add = [&](int a, int b, int s) {
        if (b <= a || n >= MAXCH) return;
        x[n] = a;
        strip[n] = s;
        x[++n] = b;
    };
    if (lo > 0) add(0, lo, 1);
    const int mid = hi - lo;
    if (mid > 0) {
        int pieces = (mid + target / 2) / target;
        if (pieces < 1) pieces = 1;
        if (pieces > MAXCH - 4) pieces = MAXCH - 4;
        for (int q = 0; q < pieces; ++q)
            add(lo + (int)((long)mid * q / pieces), lo + (int)((long)mid * (q + 1) / pieces), 0);
    }
    if (hi < nx) add(hi, nx, 1);
    return n;
}

// Lean (CPML-free) range [l0, l1) of a sequence of tiles; empty when the lean
// tiles are not one contiguous run.
template <class F>
void lean_range(int count, F is_strip, int &l0, int &l1) {
    l0 = 0;
    while (l0 < count && is_strip(l0)) ++l0;
    l1 = l0;
    while (l1 < count && !is_strip(l1)) ++l1;
    for (int q = l1; q < count; ++q)
        if (!is_strip(q)) l0 = l1 = 0;
}

// Work of the fused pass: all tiles, and the CPML-free interior core.  The chunk length is chosen so that the CTAs
// fill whole waves of `slots` resident CTAs: estimated time = waves x (planes
// per chunk + 1 warm-up plane).
Work make_work(const LensGrid3D *g, int slots) {
    Work wk{};
    int cstrip[MAXCH];
    const int ntz = g->pitch / TK, nty = (g->ny + TJ - 1) / TJ;
    int target = 32;
    double best = 1e300;
    for (int t = 12; t <= 96; t += 2) {
        const int nc = make_chunks(g, t, wk.x, cstrip);
        const double waves = std::ceil((double)ntz * nty * nc / (slots > 0 ? slots : 1));
        const double cost = waves * ((double)g->nx / nc + 1.0);
        if (cost < best - 1e-9) {
            best = cost;
            target = t;
        }
    }
    const int nc = make_chunks(g, target, wk.x, cstrip);
    int z0, z1, y0, y1, c0, c1;
    // a lean tile has no psi strip cell (owners and halo) and lies inside the
    // domain's interior: every component of every cell exists and updates
    lean_range(ntz, [&](int t) {
        const int k0 = t * TK;
        return meets(k0 - 1, k0 + TK - 1, g->az.h) || meets(k0, k0 + TK - 1, g->az.e) || k0 < 1 ||
               k0 + TK - 1 > g->nz - 2;
    }, z0, z1);
    lean_range(nty, [&](int t) {
        const int j0 = t * TJ;
        return meets(j0 - 1, j0 + TJ - 1, g->ay.h) || meets(j0, j0 + TJ - 1, g->ay.e) || j0 < 1 ||
               j0 + TJ - 1 > g->ny - 2;
    }, y0, y1);
    lean_range(nc, [&](int c) { return cstrip[c] != 0 || wk.x[c] < 1 || wk.x[c + 1] > g->nx - 1; }, c0, c1);
    // tiles / chunks without psi of an axis (a contiguous run, else none: every
    // tile then carries that axis, which is always correct)
    lean_range(ntz, [&](int t) {
        const int k0 = t * TK;
        return meets(k0 - 1, k0 + TK - 1, g->az.h) || meets(k0, k0 + TK - 1, g->az.e);
    }, wk.plo[0], wk.phi[0]);
    lean_range(nty, [&](int t) {
        const int j0 = t * TJ;
        return meets(j0 - 1, j0 + TJ - 1, g->ay.h) || meets(j0, j0 + TJ - 1, g->ay.e);
    }, wk.plo[1], wk.phi[1]);
    lean_range(nc, [&](int c) {
        const int a = wk.x[c], b = wk.x[c + 1];
        return meets(a > 0 ? a - 1 : 0, b - 1, g->ax.h) || meets(a, b - 1, g->ax.e);
    }, wk.plo[2], wk.phi[2]);
    if (z1 == z0 || y1 == y0 || c1 == c0) z0 = z1 = y0 = y1 = c0 = c1 = 0;
    wk.ntz = ntz; wk.nty = nty; wk.nc = nc;
    wk.lo[0] = z0; wk.hi[0] = z1;
    wk.lo[1] = y0; wk.hi[1] = y1;
    wk.lo[2] = c0; wk.hi[2] = c1;
    // CPML tiles grouped by the specialised pass they run (tiles of more axes first), so
    // that CTAs resident together mostly share their code
    const int nlean = (z1 - z0) * (y1 - y0) * (c1 - c0);
    const int nstrip = ntz * nty * nc - nlean;
    wk.nperm = 0;
    if (nstrip > 0 && nstrip <= MAXPERM) {
        unsigned char mk[MAXPERM];
        for (int id = 0; id < nstrip; ++id) {
            int tz, ty, c;
            work_tile(wk, id, tz, ty, c);
            const unsigned m = ((tz < wk.plo[0] || tz >= wk.phi[0]) ? AXZ : 0u) |
                               ((ty < wk.plo[1] || ty >= wk.phi[1]) ? AXY : 0u) |
                               ((c < wk.plo[2] || c >= wk.phi[2]) ? AXX : 0u);
            const int axes = (m & 1u) + ((m >> 1) & 1u) + ((m >> 2) & 1u);
            mk[id] = (unsigned char)((3 - axes) * 8 + (7 - m));  // sort key: more axes first, then the mask
        }
        int n = 0;
        for (int key = 0; key < 32; ++key)
            for (int id = 0; id < nstrip; ++id)
                if (mk[id] == key) wk.perm[n++] = (unsigned short)id;
        wk.nperm = n;
    }
    return wk;
}

// x-chunk length: about `target` planes, enough CTAs that the last wave's tail is short.
int chunk_len(int nx, int target) {
    int nch = (nx + target / 2) / target;
    if (nch < 1) nch = 1;
    return (nx + nch - 1) / nch;
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// Tensor map of a padded (nx, ny, pitch) float array with a (bk, bj, 1) box;
// out-of-range elements of a box read as zero.
bool encode(CUtensorMap *m, const float *base, const LensGrid3D *g, int bk, int bj) {
    EncodeTiled fn = encoder();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g->pitch, (cuuint64_t)g->ny, (cuuint64_t)g->nx};
    const cuuint64_t strides[2] = {(cuuint64_t)g->pitch * 4, (cuuint64_t)g->pitch * g->ny * 4};
    const cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)bj, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The two-pass path sums the detector boxes inside its E pass, before a drive
// could act, so a driven step takes no boxes.
bool drive3d_ok(const LensDrive3D *d, const LensStepTable *t, const LensGrid3D *g, const LensEpi3D *ep) {
    if (!d) return true;
    if (ep && ep->nbox > 0) return false;
    if (d->nplanes < 1 || d->nplanes > g->nx - 1 || !d->taper || !t->pe || !t->env) return false;
    for (int m = 0; m < 3; ++m)
        if (!d->hand[m] || (reinterpret_cast<uintptr_t>(d->hand[m]) & 7)) return false;
    return true;
}

// Steps [n0, n0+nsteps): the Yee update (source included), then the optional
// stitch drive on the new E, then the epilogue that reads the new E.
int step3d(LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep, const LensDrive3D *dr, int n0,
           int nsteps, void *stream, int wd_plane = -1) {
    if (!grid3d_ok(g) || nsteps < 0 || !lens_table_ok(tab, n0, nsteps) || !epi3d_ok(ep, tab, g) ||
        !drive3d_ok(dr, tab, g, ep))
        return LENS_ERR_ARG;
    LensEpi3D e{};  // zero: no boxes, empty windows, no planes
    if (ep) e = *ep;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 blk(BK, BJ);
    const dim3 grd_d(g->pitch / BK, (g->ny + BJ - 1) / BJ, dr ? dr->nplanes : 1);
    if (!has_buffer1(g)) {
        const K3 k = view(g, g->cur, g->cur);
        const int chunk = chunk_len(g->nx, 96);
        const dim3 grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, (g->nx + chunk - 1) / chunk);
        for (int n = n0; n < n0 + nsteps; ++n) {
            h3d<<<grd, blk, 0, s>>>(k, chunk);
            if (dr) {
                // the in-place E pass folds the epilogue in; with a drive the
                // epilogue must see the driven E, so it runs as a pass of its own
                e3d<<<grd, blk, 0, s>>>(k, *tab, LensEpi3D{}, n, chunk);
                drive3d<<<grd_d, blk, 0, s>>>(k, *tab, *dr, n);
                if (epi3d_active(&e, n))
                    win3d<<<dim3((g->pitch + BK * WK - 1) / (BK * WK), (g->ny + BJ - 1) / BJ, g->nx), blk, 0, s>>>(
                        k, *tab, e, n);
            } else {
                e3d<<<grd, blk, 0, s>>>(k, *tab, e, n, chunk);
            }
        }
        return lens_cuda_status();
    }
    // every TMA base address must be 16-byte aligned
    const float *bases[6] = {g->ce_x, g->ce_y, g->ce_z, g->da_x, g->da_y, g->da_z};
    for (int q = 0; q < 6; ++q)
        if (reinterpret_cast<uintptr_t>(bases[q]) & 15) return LENS_ERR_ARG;
    for (int b = 0; b < 2; ++b) {
        for (int c = 0; c < 6; ++c)
            if (reinterpret_cast<uintptr_t>(g->f[b][c]) & 15) return LENS_ERR_ARG;
        for (int q = 0; q < LENS_NPSI; ++q)
            if (!g->psi[b][q] || (reinterpret_cast<uintptr_t>(g->psi[b][q]) & 15)) return LENS_ERR_ARG;
    }
    const bool ix32 = (double)g->nx * g->ny * g->pitch < 2147483647.0;
    if (cudaFuncSetAttribute(yee3d<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM3) != cudaSuccess ||
        cudaFuncSetAttribute(yee3d<size_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM3) != cudaSuccess)
        return LENS_ERR_CUDA;
    EMaps tm[2];
    for (int rb = 0; rb < 2; ++rb) {
        for (int c = 0; c < 3; ++c)
            if (!encode(&tm[rb].e[c], g->f[rb][c], g, EK, EJ) || !encode(&tm[rb].h[c], g->f[rb][3 + c], g, TK, TJ))
                return LENS_ERR_CUDA;
        for (int c = 0; c < 6; ++c)
            if (!encode(&tm[rb].c[c], c < 3 ? bases[c] : (g->da_x ? bases[c] : bases[c - 3]), g, TK, TJ))
                return LENS_ERR_CUDA;
    }
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return LENS_ERR_CUDA;
    const Work wk = make_work(g, 2 * nsm);
    const int nblk = wk.ntz * wk.nty * wk.nc;
    // box-sum grid: the largest y-z extent of the boxes, their plane groups stacked in z
    BoxGrid bgr{};
    int bgx = 0, bgy = 0, bgz = 0;
    for (int b = 0; b < e.nbox; ++b) {
        const int *bx = e.box[b];
        const int zl = box_end(bx[5], g->nz) - bx[4], yl = box_end(bx[3], g->ny) - bx[2],
                  xl = box_end(bx[1], g->nx) - bx[0];
        bgr.xb[b] = bgz;
        if (zl > 0 && yl > 0 && xl > 0) {
            bgx = std::max(bgx, (zl + BK - 1) / BK);
            bgy = std::max(bgy, (yl + BJ - 1) / BJ);
            bgz += (xl + BOXX - 1) / BOXX;
        }
    }
    bgr.xb[e.nbox] = bgz;
    const dim3 grd_w((g->pitch + BK * WK - 1) / (BK * WK), (g->ny + BJ - 1) / BJ, g->nx);
    for (int n = n0; n < n0 + nsteps; ++n) {
        const int rb = g->cur;
        K3 k = view(g, rb, 1 - rb);
        k.wd_plane = wd_plane;
        const int ea = epi3d_active(&e, n);
        if (ix32)
            yee3d<uint32_t><<<nblk, dim3(TK, NW3), SMEM3, s>>>(tm[rb], k, *tab, e, n, ea, wk);
        else
            yee3d<size_t><<<nblk, dim3(TK, NW3), SMEM3, s>>>(tm[rb], k, *tab, e, n, ea, wk);
        if (dr) drive3d<<<grd_d, blk, 0, s>>>(view(g, 1 - rb, 1 - rb), *tab, *dr, n);
        if (e.nbox > 0 && bgz > 0)  // detector boxes of the new E, every box in one launch
            box3d<<<dim3(bgx, bgy, bgz), blk, 0, s>>>(view(g, 1 - rb, 1 - rb), e, bgr);
        if (ea && ((n >= e.dft_n0 && n < e.dft_n1) || (e.conv_prev && n >= e.prev_n0 && n < e.prev_n1)))
            win3d<<<grd_w, blk, 0, s>>>(view(g, 1 - rb, 1 - rb), *tab, e, n);
        g->cur = 1 - rb;
    }
    return lens_cuda_status();
}

}  // namespace

extern "C" int lens_fdtd3d_step(LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep, int n0,
                                int nsteps, void *stream) {
    return step3d(g, tab, ep, nullptr, n0, nsteps, stream);
}

extern "C" int lens_fdtd3d_step_driven(LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep,
                                       const LensDrive3D *drive, int n0, int nsteps, void *stream) {
    if (!drive) return LENS_ERR_ARG;
    return step3d(g, tab, ep, drive, n0, nsteps, stream);
}

extern "C" int lens_fdtd3d_watchdog_test(LensGrid3D *g, const LensStepTable *tab, int n0, int offset, void *stream) {
    if (!g || !g->flag || !has_buffer1(g) || offset < 0 || offset > 1) return LENS_ERR_ARG;
    return step3d(g, tab, nullptr, nullptr, n0, 1, stream, offset);
}

extern "C" int lens_fdtd3d_accum_e2(const LensGrid3D *g, int target, int nx_target, float *iavg, void *stream) {
    if (!grid3d_ok(g) || !iavg || (target != 1 && target != 2) || nx_target < 2 || nx_target > g->nx)
        return LENS_ERR_ARG;
    const dim3 blk(BK, BJ), grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, nx_target);
    accum_e2<<<grd, blk, 0, static_cast<cudaStream_t>(stream)>>>(view(g, g->cur, g->cur), target, nx_target,
                                                                  iavg);
    return lens_cuda_status();
}

extern "C" int lens_version(void) { return 100; }

extern "C" int lens_abi_sizes(int *sizes, int n) {
    const int v[15] = {(int)sizeof(LensProfile), (int)sizeof(LensAxis), (int)sizeof(LensStepTable),
                       (int)sizeof(LensSource),  (int)sizeof(LensTE2D), (int)sizeof(LensTM2D),
                       (int)sizeof(LensEpi2D),   (int)sizeof(LensGrid3D), (int)sizeof(LensEpi3D),
                       (int)sizeof(LensInst2D),  (int)sizeof(LensDrive3D), (int)sizeof(LensDrive2D),
                       (int)sizeof(LensTB2D), (int)sizeof(LensTB3D), (int)sizeof(LensRsOut2D)};
    for (int q = 0; q < n && q < 15; ++q) sizes[q] = v[q];
    return 15;
}

extern "C" const char *lens_status_string(int status) {
    switch (status) {
        case LENS_OK: return "ok";
        case LENS_ERR_ARG: return "invalid argument";
        case LENS_ERR_CUDA: return "CUDA launch or runtime error";
        case LENS_ERR_SIZE: return "size exceeds the supported maximum";
        default: return "unknown status";
    }
}
