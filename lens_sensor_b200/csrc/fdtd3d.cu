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
    return g.src_comp == comp && (i == g.src.ix || i == g.src.ix + 1) && j < g.src.nj &&
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

// Epilogue of one cell after its E update.  All 32 lanes of a warp must call it.
//   detector boxes: sum of Ex^2+Ey^2+Ez^2 in FP64 (fdtd3d_core.py:477-481)
//   DFT windows:    compensated float32 (Kahan) complex sums of each selected component
//   flux planes:    FP64 DFT of E and of the x-averaged H (flux.py:28-41)
__device__ __forceinline__ void epi_cell(const K3 &g, const LensStepTable &tab, const LensEpi3D &ep,
                                         int n, int i, int j, int k, bool in, Hv e, float hym,
                                         float hzm, Hv h, bool vol_dft = true) {
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const bool vx = in && i < nx - 1, vy = in && j < ny - 1, vz = in && k < nz - 1;
    if (ep.nbox > 0) {
        const int bk0 = blockIdx.x * BK, bj0 = blockIdx.y * BJ;
        for (int b = 0; b < ep.nbox; ++b) {
            const int *bx = ep.box[b];
            if (i < bx[0] || i >= bx[1] || bx[3] <= bj0 || bx[2] >= bj0 + BJ || bx[5] <= bk0 ||
                bx[4] >= bk0 + BK)
                continue;  // block-uniform
            const bool inb = j >= bx[2] && j < bx[3] && k >= bx[4] && k < bx[5];
            double v = 0.0;
            if (inb) {
                if (vx) v += (double)(e.x * e.x);
                if (vy) v += (double)(e.y * e.y);
                if (vz) v += (double)(e.z * e.z);
            }
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
        if (ep.dft[0] && vx) kahan_add(reinterpret_cast<float4 *>(ep.dft[0]) + o, e.x * pr, e.x * pim);
        if (ep.dft[1] && vy) kahan_add(reinterpret_cast<float4 *>(ep.dft[1]) + o, e.y * pr, e.y * pim);
        if (ep.dft[2] && vz) kahan_add(reinterpret_cast<float4 *>(ep.dft[2]) + o, e.z * pr, e.z * pim);
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
// CTA = 10 warps: warps 0..7 own the tile rows j0..j0+7 (H and E), warp 8
// computes H on the halo row j0-1, warp 9 (lanes 0..7) H on the halo column
// k0-1, and lane 31 of warp 9 issues the TMA copies.  Every (j, k) dependent
// quantity (validity, strip slot, CPML profile values, source profile) is
// computed once per thread; i dependent ones once per plane.
constexpr int FW = BJ + 2;
constexpr int EK = BK + 8, EJ = BJ + 2;    // E box:   z k0-4..k0+35, y j0-1..j0+8
constexpr int HK = BK + 4, HJ = BJ + 1;    // H box:   z k0-4..k0+31, y j0-1..j0+7
constexpr int SHK = BK + 1, SHJ = BJ + 1;  // new H:   z k0-1..k0+31, y j0-1..j0+7
constexpr int NSE = 4, NSH = 3, NSC = 3;   // ring depths (x-planes)
constexpr int E_BYTES = EK * EJ * 4, E_SLOT = 1664;
constexpr int H_BYTES = HK * HJ * 4, H_SLOT = 1408;
constexpr int C_BYTES = BK * BJ * 4;
constexpr int SH_N = SHK * SHJ;
constexpr int OFF_H = NSE * 3 * E_SLOT;
constexpr int OFF_C = OFF_H + NSH * 3 * H_SLOT;
constexpr int OFF_SH = OFF_C + NSC * 6 * C_BYTES;
constexpr int OFF_BAR = OFF_SH + ((2 * 3 * SH_N * 4 + 127) / 128) * 128;
constexpr int SMEM_LEAN = OFF_BAR + (NSE + NSH + NSC) * 8;
// strip CTAs also stage psi: 6 H-psi tiles per H stage, 6 E-psi tiles per C stage
constexpr int OFF_HP = ((SMEM_LEAN + 127) / 128) * 128;
constexpr int OFF_EP = OFF_HP + NSH * 6 * H_SLOT;
constexpr int SMEM_STRIP = OFF_EP + NSC * 6 * C_BYTES;
static_assert(E_SLOT % 128 == 0 && E_SLOT >= E_BYTES, "E slot");
static_assert(H_SLOT % 128 == 0 && H_SLOT >= H_BYTES, "H slot");
static_assert(OFF_H % 128 == 0 && OFF_C % 128 == 0 && OFF_SH % 128 == 0, "alignment");

struct TMaps {
    CUtensorMap e[3];  // E of the read buffer, box EK x EJ x 1
    CUtensorMap h[3];  // H of the read buffer, box HK x HJ x 1
    CUtensorMap c[6];  // ce_x, ce_y, ce_z, D_x, D_y, D_z, box BK x BJ x 1
    CUtensorMap p[12]; // psi of the read buffer (LENS_PSI_* order): H-psi box HK x HJ, E-psi BK x BJ
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
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok = 0;
    for (int t = 0; t < (1 << 20) && !ok; ++t) {
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

// CPML values of one coordinate: inside a psi strip?  and b, c, 1/kappa - 1.
struct PV {
    int s;
    float b, c, km;
};

__device__ __forceinline__ PV pv_at(const LensProfile &p, int m) {
    PV r{-1, 1.f, 0.f, 0.f};
    if (m >= 0 && m < p.n) {
        r.s = strip_of(m, p.lo, p.hi, p.n);
        if (r.s >= 0) {
            r.b = p.b[m];
            r.c = p.c[m];
            r.km = p.ik[m] - 1.0f;
        }
    }
    return r;
}

// psi update: stores the new psi (owner only) and returns psi + (1/kappa - 1)*d.
__device__ __forceinline__ float psi_u(float old, const PV &v, float d, float *pw, size_t idx, bool wr) {
    const float p = v.b * old + v.c * d;
    if (wr) pw[idx] = p;
    return p + v.km * d;
}

// does [a, b] meet a psi strip of profile p?
__device__ __forceinline__ bool meets(int a, int b, const LensProfile &p) {
    return (p.lo > 0 && a < p.lo) || (p.hi > 0 && b >= p.n - p.hi);
}

constexpr int MAXCH = 96;
// x-decomposition: chunk c covers planes [x[c], x[c+1]); strip[c] != 0 when a
// plane of the chunk (or the plane before it) lies in an x CPML strip.
struct Chunks {
    int n;
    int x[MAXCH + 1];
    int strip[MAXCH];
};

// Ring slot (stage) and phase parity of the u-th use, tracked incrementally.
struct Ring {
    int s, ph;
    int n;
    __device__ __forceinline__ void next() {
        if (++s == n) {
            s = 0;
            ph ^= 1;
        }
    }
};

// One launch per block category: ST = false runs only the blocks whose tile
// and x-chunk meet no CPML strip (no psi at all), ST = true the others, whose
// psi tiles are staged by TMA next to the field tiles.  Only the producer lane
// waits on the mbarriers; the other warps sleep in the CTA barrier.
template <bool ST, bool DF>
__global__ void __launch_bounds__(FW * 32, ST ? 2 : 3)
    fused3d(const __grid_constant__ TMaps tm, const K3 g, const LensStepTable tab,
            const LensEpi3D ep, int n, int epi, const __grid_constant__ Chunks chs) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int k0 = blockIdx.x * BK, j0 = blockIdx.y * BJ;
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const int x0 = chs.x[blockIdx.z], x1 = chs.x[blockIdx.z + 1];
    // block category (uniform); psi tiles this CTA needs
    const bool nz_h = meets(k0 - 1, k0 + BK - 1, g.az.h), ny_h = meets(j0 - 1, j0 + BJ - 1, g.ay.h);
    const bool nz_e = meets(k0, k0 + BK - 1, g.az.e), ny_e = meets(j0, j0 + BJ - 1, g.ay.e);
    if ((nz_h || ny_h || nz_e || ny_e || chs.strip[blockIdx.z] != 0) != ST) return;
    extern __shared__ __align__(128) unsigned char smem[];
    const float *sE = reinterpret_cast<const float *>(smem);
    const float *sHo = reinterpret_cast<const float *>(smem + OFF_H);
    const float *sC = reinterpret_cast<const float *>(smem + OFF_C);
    float *sH = reinterpret_cast<float *>(smem + OFF_SH);
    const float *sHP = reinterpret_cast<const float *>(smem + OFF_HP);
    const float *sEP = reinterpret_cast<const float *>(smem + OFF_EP);
    const uint32_t sbase = s_addr(smem);
    const uint32_t bar0 = sbase + OFF_BAR;
    const int xs = x0 > 0 ? x0 - 1 : 0;  // plane x0-1: its H feeds E(x0)
    const bool lossy = g.da_x != nullptr;
    const int ncoef = lossy ? 6 : 3;
    const bool prod = (w == FW - 1 && lane == 31);
    const float ch = g.ch;

    // ---- thread role: the cell (j, k) whose H this thread computes
    const bool own = w < BJ;
    int j, k, ej, ek, sa;
    if (own) {
        j = j0 + w; k = k0 + lane; ej = w + 1; ek = lane + 4; sa = (w + 1) * SHK + lane + 1;
    } else if (w == BJ) {
        j = j0 - 1; k = k0 + lane; ej = 0; ek = lane + 4; sa = lane + 1;
    } else {
        j = j0 + lane; k = k0 - 1; ej = lane + 1; ek = 3; sa = (lane + 1) * SHK;
    }
    const bool hrole = own || w == BJ || lane < BJ;
    const bool hact = hrole && j >= 0 && j < ny && k >= 0 && k < nz;
    const int ea = ej * EK + ek, ha = ej * HK + ek;
    const bool hx_ok = hact && j < ny - 1 && k < nz - 1, hy_k = hact && k < nz - 1, hz_j = hact && j < ny - 1;
    const bool ein = own && j < ny && k < nz;
    const bool jin = j >= 1 && j <= ny - 2, kin = k >= 1 && k <= nz - 2;
    const bool pec_j = (g.pec[2] && j == 0) || (g.pec[3] && j == ny - 1);
    const bool pec_k = (g.pec[4] && k == 0) || (g.pec[5] && k == nz - 1);
    float s_amp = 0.f, s_ph1 = 0.f, s_ph2 = 0.f;
    if (ein && g.src.ix >= 0 && j < g.src.nj && k < g.src.nk) {
        const size_t m = (size_t)j * g.src.pitch_k + k;
        s_amp = g.src.amp[m];
        s_ph1 = g.src.ph1[m];
        s_ph2 = g.src.ph2[m];
    }
    PV zh{-1, 1.f, 0.f, 0.f}, yh = zh, ze = zh, ye = zh;
    if (ST) {
        zh = pv_at(g.az.h, k); yh = pv_at(g.ay.h, j);
        ze = pv_at(g.az.e, k); ye = pv_at(g.ay.e, j);
    }
    const size_t S = (size_t)ny * P;
    size_t o = ((size_t)xs * ny + j) * P + k;  // field / psi index of (xs, j, k)

    auto issue_e = [&](int p, int s) {
        const uint32_t bar = bar0 + 8u * s;
        mbar_expect(bar, 3 * E_BYTES);
        for (int c = 0; c < 3; ++c) tma3(sbase + (s * 3 + c) * E_SLOT, &tm.e[c], k0 - 4, j0 - 1, p, bar);
    };
    auto issue_h = [&](int p, int s) {
        const uint32_t bar = bar0 + 8u * (NSE + s);
        int np = 0;
        bool pn[6] = {false, false, false, false, false, false};
        if (ST) {
            const bool xh = meets(p, p, g.ax.h);
            pn[0] = nz_h; pn[1] = ny_h; pn[2] = xh; pn[3] = nz_h; pn[4] = ny_h; pn[5] = xh;
            for (int q = 0; q < 6; ++q) np += pn[q];
        }
        mbar_expect(bar, (3 + np) * H_BYTES);
        for (int c = 0; c < 3; ++c) tma3(sbase + OFF_H + (s * 3 + c) * H_SLOT, &tm.h[c], k0 - 4, j0 - 1, p, bar);
        if (ST)
            for (int q = 0; q < 6; ++q)
                if (pn[q]) tma3(sbase + OFF_HP + (s * 6 + q) * H_SLOT, &tm.p[q], k0 - 4, j0 - 1, p, bar);
    };
    auto issue_c = [&](int p, int s) {
        const uint32_t bar = bar0 + 8u * (NSE + NSH + s);
        int np = 0;
        bool pn[6] = {false, false, false, false, false, false};
        if (ST) {
            const bool xe = meets(p, p, g.ax.e);
            pn[0] = ny_e; pn[1] = nz_e; pn[2] = nz_e; pn[3] = xe; pn[4] = xe; pn[5] = ny_e;
            for (int q = 0; q < 6; ++q) np += pn[q];
        }
        mbar_expect(bar, (ncoef + np) * C_BYTES);
        for (int c = 0; c < ncoef; ++c) tma3(sbase + OFF_C + (s * 6 + c) * C_BYTES, &tm.c[c], k0, j0, p, bar);
        if (ST)
            for (int q = 0; q < 6; ++q)
                if (pn[q]) tma3(sbase + OFF_EP + (s * 6 + q) * C_BYTES, &tm.p[6 + q], k0, j0, p, bar);
    };
    // rings: E holds planes xs.., H planes xs.., C planes x0..; the producer lane
    // issues and waits, everybody else only uses __syncthreads
    Ring we{0, 0, NSE}, wh{0, 0, NSH}, wc{0, 0, NSC};  // waiter cursors
    Ring fe{0, 0, NSE}, fh{0, 0, NSH}, fc{0, 0, NSC};  // fill cursors
    bool ok = true;
    if (prod) {
        for (int q = 0; q < NSE + NSH + NSC; ++q) mbar_init(bar0 + 8u * q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int p = xs; p <= min(x1, xs + NSE - 1); ++p, fe.next()) issue_e(p, fe.s);
        for (int p = xs; p <= min(x1 - 1, xs + NSH - 1); ++p, fh.next()) issue_h(p, fh.s);
        for (int p = x0; p <= min(x1 - 1, x0 + NSC - 1); ++p, fc.next()) issue_c(p, fc.s);
        ok &= mbar_wait(bar0 + 8u * we.s, we.ph);  // E(xs)
        we.next();
        ok &= mbar_wait(bar0 + 8u * we.s, we.ph);  // E(xs+1)
        ok &= mbar_wait(bar0 + 8u * (NSE + wh.s), wh.ph);  // H(xs)
        wh.next();
    }
    __syncthreads();
    const int EF = E_SLOT / 4, HF = H_SLOT / 4, CF = C_BYTES / 4;
    const int q0 = n - tab.t0;
    const float env = tab.env[q0], wt = tab.wt[q0];
    const bool win = DF && epi && n >= ep.dft_n0 && n < ep.dft_n1;
    float hym = 0.f, hzm = 0.f;  // own H(i-1), new
    int se = 0, sh = 0, sc = 0;  // stage of E(i), H(i), C(i)
    for (int i = xs; i < x1; ++i, o += S) {
        const bool eon = i >= x0;
        const int se1 = se + 1 == NSE ? 0 : se + 1;
        const float *eC = sE + se * 3 * EF;
        const float *eN = sE + se1 * 3 * EF;
        const float *hO = sHo + sh * 3 * HF;
        float *shw = sH + ((i - xs) & 1) * 3 * SH_N;
        const bool iok = i < nx - 1;

        // DFT accumulators of this plane: loaded now, used after the H phase
        float4 acc[DF ? 3 : 1];
        const bool dft_now = DF && win && ein && eon;
        if (DF && dft_now) {
#pragma unroll
            for (int c = 0; c < (DF ? 3 : 1); ++c)
                if (ep.dft[c]) acc[c] = reinterpret_cast<const float4 *>(ep.dft[c])[o];
        }
        // ---- H(i) at (j, k)
        const float ex = eC[ea], ey = eC[EF + ea], ez = eC[2 * EF + ea];
        float hx = 0.f, hy = 0.f, hz = 0.f;
        if (hact) {
            hx = hO[ha];
            hy = hO[HF + ha];
            hz = hO[2 * HF + ha];
            const float dxz = eC[EF + ea + 1] - ey, dxy = eC[2 * EF + ea + EK] - ez;  // Hx terms
            const float dyx = eN[2 * EF + ea] - ez, dyz = eC[ea + 1] - ex;          // Hy terms
            const float dzy = eC[ea + EK] - ex, dzx = eN[EF + ea] - ey;             // Hz terms
            if (hx_ok) hx = hx + ch * (dxz - dxy);
            if (iok && hy_k) hy = hy + ch * (dyx - dyz);
            if (iok && hz_j) hz = hz + ch * (dzy - dzx);
            if (ST) {
                const bool wr = own && eon;  // psi of this plane is written by its owner only
                const PV xh = pv_at(g.ax.h, i);
                const float *hp = sHP + sh * 6 * HF + ha;
                if (hx_ok) {
                    if (zh.s >= 0) hx = hx + ch * psi_u(hp[0], zh, dxz, g.pw[LENS_PSI_HX_Z], o, wr);
                    if (yh.s >= 0) hx = hx + (-ch) * psi_u(hp[HF], yh, dxy, g.pw[LENS_PSI_HX_Y], o, wr);
                }
                if (iok && hy_k) {
                    if (xh.s >= 0) hy = hy + ch * psi_u(hp[2 * HF], xh, dyx, g.pw[LENS_PSI_HY_X], o, wr);
                    if (zh.s >= 0) hy = hy + (-ch) * psi_u(hp[3 * HF], zh, dyz, g.pw[LENS_PSI_HY_Z], o, wr);
                }
                if (iok && hz_j) {
                    if (yh.s >= 0) hz = hz + ch * psi_u(hp[4 * HF], yh, dzy, g.pw[LENS_PSI_HZ_Y], o, wr);
                    if (xh.s >= 0) hz = hz + (-ch) * psi_u(hp[5 * HF], xh, dzx, g.pw[LENS_PSI_HZ_X], o, wr);
                }
            }
        }
        if (hrole) {
            shw[sa] = hx;
            shw[SH_N + sa] = hy;
            shw[2 * SH_N + sa] = hz;
        }
        if (prod) {  // data of this plane's E phase and of the next plane's H phase
            if (eon) {
                ok &= mbar_wait(bar0 + 8u * (NSE + NSH + wc.s), wc.ph);
                wc.next();
            }
            if (i + 2 <= x1) {
                we.next();
                ok &= mbar_wait(bar0 + 8u * we.s, we.ph);
            }
            if (i + 1 <= x1 - 1) {
                ok &= mbar_wait(bar0 + 8u * (NSE + wh.s), wh.ph);
                wh.next();
            }
        }
        __syncthreads();
        // E(i) and H(i) stages are free now, and the coefficients of plane i-1
        if (prod) {
            if (i + NSE <= x1) {
                issue_e(i + NSE, fe.s);
                fe.next();
            }
            if (i + NSH <= x1 - 1) {
                issue_h(i + NSH, fh.s);
                fh.next();
            }
            if (i - 1 >= x0 && i - 1 + NSC <= x1 - 1) {
                issue_c(i - 1 + NSC, fc.s);
                fc.next();
            }
        }
        if (own && eon) {
            Hv e{0.f, 0.f, 0.f};
            if (ein) {
                g.whx[o] = hx;
                g.why[o] = hy;
                g.whz[o] = hz;
                const int ca = w * BK + lane;
                const float *cs = sC + sc * 6 * CF + ca;
                const bool iin = i >= 1 && i <= nx - 2;
                const bool pec_i = (g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1);
                float src = 0.f;
                if (i == g.src.ix) src = (env * sinf(wt + s_ph1)) * s_amp;
                else if (g.src.ix >= 0 && i == g.src.ix + 1) src = -((env * sinf(wt + s_ph2)) * s_amp);
                const float hzj = shw[2 * SH_N + sa - SHK], hyk = shw[SH_N + sa - 1];
                const float hxk = shw[sa - 1], hxj = shw[sa - SHK];
                const float d1x = hz - hzj, d2x = hy - hyk;  // Ex
                const float d1y = hx - hxk, d2y = hz - hzm;  // Ey
                const float d1z = hy - hym, d2z = hx - hxj;  // Ez
                float vx = ex, vy = ey, vz = ez;
                if (iok) {
                    if (lossy) vx = vx * cs[3 * CF];
                    if (jin && kin) vx = vx + cs[0] * (d1x - d2x);
                }
                if (j < ny - 1) {
                    if (lossy) vy = vy * cs[4 * CF];
                    if (iin && kin) vy = vy + cs[CF] * (d1y - d2y);
                }
                if (k < nz - 1) {
                    if (lossy) vz = vz * cs[5 * CF];
                    if (iin && jin) vz = vz + cs[2 * CF] * (d1z - d2z);
                }
                if (ST) {
                    const PV xe = pv_at(g.ax.e, i);
                    const float *pp = sEP + sc * 6 * CF + ca;
                    if (iok && jin && kin) {
                        const float cx = cs[0];
                        if (ye.s >= 0) vx = vx + cx * psi_u(pp[0], ye, d1x, g.pw[LENS_PSI_EX_Y], o, true);
                        if (ze.s >= 0) vx = vx + (-cx) * psi_u(pp[CF], ze, d2x, g.pw[LENS_PSI_EX_Z], o, true);
                    }
                    if (j < ny - 1 && iin && kin) {
                        const float cy = cs[CF];
                        if (ze.s >= 0) vy = vy + cy * psi_u(pp[2 * CF], ze, d1y, g.pw[LENS_PSI_EY_Z], o, true);
                        if (xe.s >= 0) vy = vy + (-cy) * psi_u(pp[3 * CF], xe, d2y, g.pw[LENS_PSI_EY_X], o, true);
                    }
                    if (k < nz - 1 && iin && jin) {
                        const float cz = cs[2 * CF];
                        if (xe.s >= 0) vz = vz + cz * psi_u(pp[4 * CF], xe, d1z, g.pw[LENS_PSI_EZ_X], o, true);
                        if (ye.s >= 0) vz = vz + (-cz) * psi_u(pp[5 * CF], ye, d2z, g.pw[LENS_PSI_EZ_Y], o, true);
                    }
                }
                if (iok) {
                    if (pec_j || pec_k) vx = 0.f;
                    if (g.src_comp == 0) vx += src;
                    e.x = vx;
                }
                if (j < ny - 1) {
                    if (pec_i || pec_k) vy = 0.f;
                    if (g.src_comp == 1) vy += src;
                    e.y = vy;
                }
                if (k < nz - 1) {
                    if (pec_i || pec_j) vz = 0.f;
                    if (g.src_comp == 2) vz += src;
                    e.z = vz;
                }
                g.wex[o] = e.x;
                g.wey[o] = e.y;
                g.wez[o] = e.z;
            }
            if (DF && dft_now) {
                const float pr = tab.pe[2 * q0], pim = tab.pe[2 * q0 + 1];
                const bool vx = iok, vy = j < ny - 1, vz = k < nz - 1;
                if (ep.dft[0] && vx) {
                    kahan_reg(acc[0], e.x * pr, e.x * pim);
                    reinterpret_cast<float4 *>(ep.dft[0])[o] = acc[0];
                }
                if (ep.dft[1] && vy) {
                    kahan_reg(acc[DF ? 1 : 0], e.y * pr, e.y * pim);
                    reinterpret_cast<float4 *>(ep.dft[1])[o] = acc[DF ? 1 : 0];
                }
                if (ep.dft[2] && vz) {
                    kahan_reg(acc[DF ? 2 : 0], e.z * pr, e.z * pim);
                    reinterpret_cast<float4 *>(ep.dft[2])[o] = acc[DF ? 2 : 0];
                }
            }
            if (epi) epi_cell(g, tab, ep, n, i, j, k, ein, e, hym, hzm, Hv{hx, hy, hz}, !DF);
        }
        if (eon) sc = sc + 1 == NSC ? 0 : sc + 1;
        se = se1;
        sh = sh + 1 == NSH ? 0 : sh + 1;
        hym = hy;
        hzm = hz;
    }
    if (prod && !ok && g.flag) atomicExch(g.flag, 1);
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

__global__ void __launch_bounds__(NT) accum_e2(const K3 g, int target, float *iavg) {
    const int k = blockIdx.x * BK + threadIdx.x, j = blockIdx.y * BJ + threadIdx.y, i = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.P;
    const Ext ex{nx - 1, ny, nz}, ey{nx, ny - 1, nz}, ez{nx, ny, nz - 1};
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
    return k;
}

// x-chunks of the fused pass: the planes that carry x CPML psi get chunks of
// their own, the rest is cut into pieces of about `target` planes.
Chunks make_chunks(const LensGrid3D *g, int target) {
    Chunks c{};
    const int nx = g->nx;
    int lo = g->ax.h.lo > g->ax.e.lo ? g->ax.h.lo : g->ax.e.lo;
    int hi = nx - 1 - g->ax.h.hi;
    if (nx - g->ax.e.hi < hi) hi = nx - g->ax.e.hi;
    lo = lo > 0 ? lo + 1 : 0;  // the next chunk's warm-up plane lo must be strip-free too
    if (hi < lo) hi = lo;
    auto add = [&](int a, int b, int strip) {
        if (b <= a || c.n >= MAXCH) return;
        c.x[c.n] = a;
        c.strip[c.n] = strip;
        c.x[++c.n] = b;
    };
    if (lo > 0) add(0, lo, 1);
    const int mid = hi - lo;
    if (mid > 0) {
        int pieces = (mid + target / 2) / target;
        if (pieces < 1) pieces = 1;
        if (pieces > MAXCH - 4) pieces = MAXCH - 4;
        for (int q = 0; q < pieces; ++q) add(lo + (int)((long)mid * q / pieces), lo + (int)((long)mid * (q + 1) / pieces), 0);
    }
    if (hi < nx) add(hi, nx, 1);
    return c;
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

}  // namespace

extern "C" int lens_fdtd3d_step(LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep, int n0,
                                int nsteps, void *stream) {
    if (!grid3d_ok(g) || nsteps < 0 || !lens_table_ok(tab, n0, nsteps) || !epi3d_ok(ep, tab, g))
        return LENS_ERR_ARG;
    LensEpi3D e{};  // zero: no boxes, empty windows, no planes
    if (ep) e = *ep;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 blk(BK, BJ);
    if (!has_buffer1(g)) {
        const K3 k = view(g, g->cur, g->cur);
        const int chunk = chunk_len(g->nx, 96);
        const dim3 grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, (g->nx + chunk - 1) / chunk);
        for (int n = n0; n < n0 + nsteps; ++n) {
            h3d<<<grd, blk, 0, s>>>(k, chunk);
            e3d<<<grd, blk, 0, s>>>(k, *tab, e, n, chunk);
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
    if (cudaFuncSetAttribute(fused3d<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LEAN) !=
            cudaSuccess ||
        cudaFuncSetAttribute(fused3d<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LEAN) !=
            cudaSuccess ||
        cudaFuncSetAttribute(fused3d<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_STRIP) !=
            cudaSuccess ||
        cudaFuncSetAttribute(fused3d<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_STRIP) !=
            cudaSuccess)
        return LENS_ERR_CUDA;
    TMaps tm[2];
    for (int rb = 0; rb < 2; ++rb) {
        bool ok = true;
        for (int c = 0; c < 3; ++c) {
            ok = ok && encode(&tm[rb].e[c], g->f[rb][c], g, EK, EJ);
            ok = ok && encode(&tm[rb].h[c], g->f[rb][3 + c], g, HK, HJ);
            ok = ok && encode(&tm[rb].c[c], bases[c], g, BK, BJ);
            ok = ok && encode(&tm[rb].c[3 + c], g->da_x ? bases[3 + c] : bases[c], g, BK, BJ);
        }
        for (int q = 0; q < LENS_NPSI; ++q)  // H-psi tiles like H, E-psi tiles like the coefficients
            ok = ok && encode(&tm[rb].p[q], g->psi[rb][q], g, q < 6 ? HK : BK, q < 6 ? HJ : BJ);
        if (!ok) return LENS_ERR_CUDA;
    }
    const Chunks chs = make_chunks(g, 40);
    const dim3 grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, chs.n);
    for (int n = n0; n < n0 + nsteps; ++n) {
        const int rb = g->cur;
        const K3 k = view(g, rb, 1 - rb);
        const int ea = epi3d_active(&e, n);
        const bool df = ea && n >= e.dft_n0 && n < e.dft_n1 && (e.dft[0] || e.dft[1] || e.dft[2]);
        if (df) {
            fused3d<true, true><<<grd, dim3(BK, FW), SMEM_STRIP, s>>>(tm[rb], k, *tab, e, n, ea, chs);
            fused3d<false, true><<<grd, dim3(BK, FW), SMEM_LEAN, s>>>(tm[rb], k, *tab, e, n, ea, chs);
        } else {
            fused3d<true, false><<<grd, dim3(BK, FW), SMEM_STRIP, s>>>(tm[rb], k, *tab, e, n, ea, chs);
            fused3d<false, false><<<grd, dim3(BK, FW), SMEM_LEAN, s>>>(tm[rb], k, *tab, e, n, ea, chs);
        }
        g->cur = 1 - rb;
    }
    return lens_cuda_status();
}

extern "C" int lens_fdtd3d_accum_e2(const LensGrid3D *g, int target, float *iavg, void *stream) {
    if (!grid3d_ok(g) || !iavg || (target != 1 && target != 2)) return LENS_ERR_ARG;
    const dim3 blk(BK, BJ), grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, g->nx);
    accum_e2<<<grd, blk, 0, static_cast<cudaStream_t>(stream)>>>(view(g, g->cur, g->cur), target, iavg);
    return lens_cuda_status();
}

extern "C" int lens_version(void) { return 100; }

extern "C" int lens_abi_sizes(int *sizes, int n) {
    const int v[9] = {(int)sizeof(LensProfile), (int)sizeof(LensAxis), (int)sizeof(LensStepTable),
                      (int)sizeof(LensSource),  (int)sizeof(LensTE2D), (int)sizeof(LensTM2D),
                      (int)sizeof(LensEpi2D),   (int)sizeof(LensGrid3D), (int)sizeof(LensEpi3D)};
    for (int q = 0; q < n && q < 9; ++q) sizes[q] = v[q];
    return 9;
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
