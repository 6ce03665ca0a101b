// 3D Yee CPML step for sm_100a: H half step, then E half step with loss
// damping, CPML psi strips, PEC, Huygens source and epilogues fused.
//
// Follows planar_3d/boundaries3d.py:311-362 (CPML_3D.step_H / step_E):
//   H += Ch*(d1 - d2);  strip corrections  H += (+Ch)*(psi1 + (1/k-1)*d1),
//                                          H += (-Ch)*(psi2 + (1/k-1)*d2)
//   E <- D*E (lossy);   E += ce*(d1 - d2) on the interior, strip corrections
//   with coef = +ce / -ce; PEC on the absorbing faces; then the source
//   (fdtd3d_core.py:1127, after the step and its PEC).
// psi is stored only in the PML strips (header lens_fdtd.h); outside them
// the correction is exactly zero and skipped.
//
// Thread mapping: one thread per cell (i, j, k); a block is 32 contiguous z
// cells x 8 rows in y, gridDim.z runs over x.
#include "lens_common.cuh"

namespace {

constexpr int BK = 32;
constexpr int BJ = 8;

struct Idx {
    int i, j, k;
    size_t o;
};

__device__ __forceinline__ Idx cell(const LensGrid3D &g) {
    Idx c;
    c.k = blockIdx.x * BK + threadIdx.x;
    c.j = blockIdx.y * BJ + threadIdx.y;
    c.i = blockIdx.z;
    c.o = ((size_t)c.i * g.ny + c.j) * g.pitch + c.k;
    return c;
}

// psi update on a strip cell:  psi = b*psi + c*d ; returns psi + (1/k - 1)*d.
__device__ __forceinline__ float psi_step(float *q, const LensProfile &pr, int m, float d) {
    const float p = pr.b[m] * (*q) + pr.c[m] * d;
    *q = p;
    return p + (pr.ik[m] - 1.0f) * d;
}

__global__ void __launch_bounds__(BK *BJ) h3d(const LensGrid3D g) {
    const Idx c = cell(g);
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.pitch;
    if (c.k >= nz || c.j >= ny) return;
    const size_t S = (size_t)ny * P;
    const size_t o = c.o;
    const float ch = g.ch;
    const int i = c.i, j = c.j, k = c.k;
    if (j < ny - 1 && k < nz - 1) {  // Hx
        const float d1 = g.ey[o + 1] - g.ey[o];  // dEy/dz
        const float d2 = g.ez[o + P] - g.ez[o];  // dEz/dy
        float h = g.hx[o] + ch * (d1 - d2);
        int s = strip_of(k, g.az.h.lo, g.az.h.hi, g.az.h.n);
        if (s >= 0)
            h = h + ch * psi_step(g.psi_hx_z + ((size_t)i * ny + j) * (g.az.h.lo + g.az.h.hi) + s,
                                  g.az.h, k, d1);
        s = strip_of(j, g.ay.h.lo, g.ay.h.hi, g.ay.h.n);
        if (s >= 0)
            h = h + (-ch) * psi_step(g.psi_hx_y + ((size_t)i * (g.ay.h.lo + g.ay.h.hi) + s) * P + k,
                                     g.ay.h, j, d2);
        g.hx[o] = h;
    }
    if (i < nx - 1 && k < nz - 1) {  // Hy
        const float d1 = g.ez[o + S] - g.ez[o];  // dEz/dx
        const float d2 = g.ex[o + 1] - g.ex[o];  // dEx/dz
        float h = g.hy[o] + ch * (d1 - d2);
        int s = strip_of(i, g.ax.h.lo, g.ax.h.hi, g.ax.h.n);
        if (s >= 0)
            h = h + ch * psi_step(g.psi_hy_x + ((size_t)s * ny + j) * P + k, g.ax.h, i, d1);
        s = strip_of(k, g.az.h.lo, g.az.h.hi, g.az.h.n);
        if (s >= 0)
            h = h + (-ch) * psi_step(g.psi_hy_z + ((size_t)i * ny + j) * (g.az.h.lo + g.az.h.hi) + s,
                                     g.az.h, k, d2);
        g.hy[o] = h;
    }
    if (i < nx - 1 && j < ny - 1) {  // Hz
        const float d1 = g.ex[o + P] - g.ex[o];  // dEx/dy
        const float d2 = g.ey[o + S] - g.ey[o];  // dEy/dx
        float h = g.hz[o] + ch * (d1 - d2);
        int s = strip_of(j, g.ay.h.lo, g.ay.h.hi, g.ay.h.n);
        if (s >= 0)
            h = h + ch * psi_step(g.psi_hz_y + ((size_t)i * (g.ay.h.lo + g.ay.h.hi) + s) * P + k,
                                  g.ay.h, j, d1);
        s = strip_of(i, g.ax.h.lo, g.ax.h.hi, g.ax.h.n);
        if (s >= 0)
            h = h + (-ch) * psi_step(g.psi_hz_x + ((size_t)s * ny + j) * P + k, g.ax.h, i, d2);
        g.hz[o] = h;
    }
}

__device__ __forceinline__ float src3(const LensGrid3D &g, const LensStepTable &tab, int n, int i,
                                      int j, int k) {
    const LensSource &s = g.src;
    const int q = n - tab.t0;
    const size_t m = (size_t)j * s.pitch_k + k;
    if (i == s.ix) return (tab.env[q] * sinf(tab.wt[q] + s.ph1[m])) * s.amp[m];
    return -((tab.env[q] * sinf(tab.wt[q] + s.ph2[m])) * s.amp[m]);
}

__device__ __forceinline__ bool is_src(const LensGrid3D &g, int comp, int i, int j, int k) {
    return g.src_comp == comp && (i == g.src.ix || i == g.src.ix + 1) && j < g.src.nj &&
           k < g.src.nk;
}

__device__ __forceinline__ void plane3(const LensEpi3D &ep, const LensStepTable &tab, int n,
                                       int p, int pair, size_t vol, size_t jk, float e, float h) {
    const int q = n - tab.t0;
    double *a = ep.plane_acc + ((size_t)(p * 2 + pair) * 4) * vol + jk;
    a[0] += (double)e * (double)tab.pe[2 * q];
    a[vol] += (double)e * (double)tab.pe[2 * q + 1];
    a[2 * vol] += (double)h * (double)tab.ph[2 * q];
    a[3 * vol] += (double)h * (double)tab.ph[2 * q + 1];
}

__global__ void __launch_bounds__(BK *BJ)
    e3d(const LensGrid3D g, const LensStepTable tab, const LensEpi3D ep, int n) {
    const Idx c = cell(g);
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.pitch;
    const int i = c.i, j = c.j, k = c.k;
    const bool in = (k < nz && j < ny);
    const size_t S = (size_t)ny * P;
    const size_t o = c.o;
    const bool vx = in && i < nx - 1, vy = in && j < ny - 1, vz = in && k < nz - 1;
    float ex = 0.f, ey = 0.f, ez = 0.f;
    if (vx) {
        ex = g.ex[o];
        if (g.da_x) ex = ex * g.da_x[o];
        if (j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
            const float d1 = g.hz[o] - g.hz[o - P];  // dHz/dy
            const float d2 = g.hy[o] - g.hy[o - 1];  // dHy/dz
            const float cc = g.ce_x[o];
            ex = ex + cc * (d1 - d2);
            int s = strip_of(j, g.ay.e.lo, g.ay.e.hi, g.ay.e.n);
            if (s >= 0)
                ex = ex + cc * psi_step(g.psi_ex_y + ((size_t)i * (g.ay.e.lo + g.ay.e.hi) + s) * P + k,
                                        g.ay.e, j, d1);
            s = strip_of(k, g.az.e.lo, g.az.e.hi, g.az.e.n);
            if (s >= 0)
                ex = ex + (-cc) * psi_step(g.psi_ex_z + ((size_t)i * ny + j) * (g.az.e.lo + g.az.e.hi) + s,
                                           g.az.e, k, d2);
        }
        if ((g.pec[2] && j == 0) || (g.pec[3] && j == ny - 1) || (g.pec[4] && k == 0) ||
            (g.pec[5] && k == nz - 1))
            ex = 0.f;
        if (is_src(g, 0, i, j, k)) ex += src3(g, tab, n, i, j, k);
        g.ex[o] = ex;
    }
    if (vy) {
        ey = g.ey[o];
        if (g.da_y) ey = ey * g.da_y[o];
        if (i >= 1 && i <= nx - 2 && k >= 1 && k <= nz - 2) {
            const float d1 = g.hx[o] - g.hx[o - 1];  // dHx/dz
            const float d2 = g.hz[o] - g.hz[o - S];  // dHz/dx
            const float cc = g.ce_y[o];
            ey = ey + cc * (d1 - d2);
            int s = strip_of(k, g.az.e.lo, g.az.e.hi, g.az.e.n);
            if (s >= 0)
                ey = ey + cc * psi_step(g.psi_ey_z + ((size_t)i * ny + j) * (g.az.e.lo + g.az.e.hi) + s,
                                        g.az.e, k, d1);
            s = strip_of(i, g.ax.e.lo, g.ax.e.hi, g.ax.e.n);
            if (s >= 0)
                ey = ey + (-cc) * psi_step(g.psi_ey_x + ((size_t)s * ny + j) * P + k, g.ax.e, i, d2);
        }
        if ((g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1) || (g.pec[4] && k == 0) ||
            (g.pec[5] && k == nz - 1))
            ey = 0.f;
        if (is_src(g, 1, i, j, k)) ey += src3(g, tab, n, i, j, k);
        g.ey[o] = ey;
    }
    if (vz) {
        ez = g.ez[o];
        if (g.da_z) ez = ez * g.da_z[o];
        if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
            const float d1 = g.hy[o] - g.hy[o - S];  // dHy/dx
            const float d2 = g.hx[o] - g.hx[o - P];  // dHx/dy
            const float cc = g.ce_z[o];
            ez = ez + cc * (d1 - d2);
            int s = strip_of(i, g.ax.e.lo, g.ax.e.hi, g.ax.e.n);
            if (s >= 0)
                ez = ez + cc * psi_step(g.psi_ez_x + ((size_t)s * ny + j) * P + k, g.ax.e, i, d1);
            s = strip_of(j, g.ay.e.lo, g.ay.e.hi, g.ay.e.n);
            if (s >= 0)
                ez = ez + (-cc) * psi_step(g.psi_ez_y + ((size_t)i * (g.ay.e.lo + g.ay.e.hi) + s) * P + k,
                                           g.ay.e, j, d2);
        }
        if ((g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1) || (g.pec[2] && j == 0) ||
            (g.pec[3] && j == ny - 1))
            ez = 0.f;
        if (is_src(g, 2, i, j, k)) ez += src3(g, tab, n, i, j, k);
        g.ez[o] = ez;
    }

    // ---------------------------------------------------------- epilogue
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
                if (vx) v += (double)(ex * ex);
                if (vy) v += (double)(ey * ey);
                if (vz) v += (double)(ez * ez);
            }
            warp_atomic_add(ep.box_acc + b, v);
        }
    }
    if (!in) return;
    const bool win = n >= ep.dft_n0 && n < ep.dft_n1;
    const bool prevw = ep.conv_prev && n >= ep.prev_n0 && n < ep.prev_n1;
    if (!win && !prevw) return;
    const float f = g.src_comp == 1 ? ey : (g.src_comp == 2 ? ez : ex);
    const bool vf = g.src_comp == 1 ? vy : (g.src_comp == 2 ? vz : vx);
    if (prevw && vf && k == ep.conv_k) {
        const float *pq = tab.pe + 2 * (n - tab.t0);
        kahan_add(reinterpret_cast<float4 *>(ep.conv_prev) + (size_t)i * g.src.nj + j, f * pq[0],
                  f * pq[1]);
    }
    if (!win) return;
    const float *pe = tab.pe + 2 * (n - tab.t0);
    if (ep.dft[0] && vx) kahan_add(reinterpret_cast<float4 *>(ep.dft[0]) + o, ex * pe[0], ex * pe[1]);
    if (ep.dft[1] && vy) kahan_add(reinterpret_cast<float4 *>(ep.dft[1]) + o, ey * pe[0], ey * pe[1]);
    if (ep.dft[2] && vz) kahan_add(reinterpret_cast<float4 *>(ep.dft[2]) + o, ez * pe[0], ez * pe[1]);
    if (ep.conv_last && vf && k == ep.conv_k)
        kahan_add(reinterpret_cast<float4 *>(ep.conv_last) + (size_t)i * g.src.nj + j, f * pe[0],
                  f * pe[1]);
    if (ep.nplane > 0 && i >= 1) {
        for (int p = 0; p < ep.nplane; ++p) {
            if (i != ep.plane[p]) continue;
            const size_t jk = (size_t)j * P + k;
            if (vy) plane3(ep, tab, n, p, 0, S, jk, ey, 0.5f * (g.hz[o - S] + g.hz[o]));
            if (vz) plane3(ep, tab, n, p, 1, S, jk, ez, 0.5f * (g.hy[o - S] + g.hy[o]));
        }
    }
}

// ---------------------------------------------------------------- Iavg
// Square of component F mapped onto the target grid (fdtd3d_core.py:438-461):
// x: equal extent or one shorter (average of clipped neighbours i-1, i);
// y, z: one longer (mean of j, j+1) or one shorter (edges copied, else mean of j-1, j).
struct Ext {
    int nx, ny, nz;
};

__device__ __forceinline__ float sqx(const float *F, const Ext &f, int tnx, int P, int ny, int i,
                                     int j, int k) {
    if (f.nx == tnx) {
        const float a = F[((size_t)i * ny + j) * P + k];
        return a * a;
    }
    const int i0 = min(max(i - 1, 0), f.nx - 1), i1 = min(max(i, 0), f.nx - 1);
    const float a = F[((size_t)i0 * ny + j) * P + k], b = F[((size_t)i1 * ny + j) * P + k];
    return 0.5f * (a * a + b * b);
}

__device__ __forceinline__ float sqxy(const float *F, const Ext &f, const Ext &t, int P, int ny,
                                      int i, int j, int k) {
    if (f.ny == t.ny) return sqx(F, f, t.nx, P, ny, i, j, k);
    if (f.ny == t.ny + 1) return 0.5f * (sqx(F, f, t.nx, P, ny, i, j, k) + sqx(F, f, t.nx, P, ny, i, j + 1, k));
    if (j == 0) return sqx(F, f, t.nx, P, ny, i, 0, k);
    if (j == t.ny - 1) return sqx(F, f, t.nx, P, ny, i, f.ny - 1, k);
    return 0.5f * (sqx(F, f, t.nx, P, ny, i, j - 1, k) + sqx(F, f, t.nx, P, ny, i, j, k));
}

__device__ __forceinline__ float sq_on_grid(const float *F, const Ext &f, const Ext &t, int P,
                                            int ny, int i, int j, int k) {
    if (f.nz == t.nz) return sqxy(F, f, t, P, ny, i, j, k);
    if (f.nz == t.nz + 1)
        return 0.5f * (sqxy(F, f, t, P, ny, i, j, k) + sqxy(F, f, t, P, ny, i, j, k + 1));
    if (k == 0) return sqxy(F, f, t, P, ny, i, j, 0);
    if (k == t.nz - 1) return sqxy(F, f, t, P, ny, i, j, f.nz - 1);
    return 0.5f * (sqxy(F, f, t, P, ny, i, j, k - 1) + sqxy(F, f, t, P, ny, i, j, k));
}

__global__ void __launch_bounds__(BK *BJ) accum_e2(const LensGrid3D g, int target, float *iavg) {
    const Idx c = cell(g);
    const int nx = g.nx, ny = g.ny, nz = g.nz, P = g.pitch;
    const Ext ex{nx - 1, ny, nz}, ey{nx, ny - 1, nz}, ez{nx, ny, nz - 1};
    const Ext t = target == 1 ? ey : ez;
    if (c.i >= t.nx || c.j >= t.ny || c.k >= t.nz) return;
    const float a = sq_on_grid(g.ex, ex, t, P, ny, c.i, c.j, c.k);
    const float b = sq_on_grid(g.ey, ey, t, P, ny, c.i, c.j, c.k);
    const float d = sq_on_grid(g.ez, ez, t, P, ny, c.i, c.j, c.k);
    iavg[c.o] += (a + b) + d;
}

bool ax_ok(const LensAxis &a, int n) { return lens_profile_ok(a.e, n) && lens_profile_ok(a.h, n - 1); }

bool grid3d_ok(const LensGrid3D *g) {
    if (!g || g->nx < 3 || g->ny < 3 || g->nz < 3 || g->pitch < g->nz || (g->pitch % 32)) return false;
    if (!g->ex || !g->ey || !g->ez || !g->hx || !g->hy || !g->hz || !g->ce_x || !g->ce_y || !g->ce_z)
        return false;
    const bool d0 = !g->da_x, d1 = !g->da_y, d2 = !g->da_z;
    if (d0 != d1 || d1 != d2) return false;
    if (!ax_ok(g->ax, g->nx) || !ax_ok(g->ay, g->ny) || !ax_ok(g->az, g->nz)) return false;
    const bool need[12] = {g->az.h.lo + g->az.h.hi > 0, g->ay.h.lo + g->ay.h.hi > 0,
                           g->ax.h.lo + g->ax.h.hi > 0, g->az.h.lo + g->az.h.hi > 0,
                           g->ay.h.lo + g->ay.h.hi > 0, g->ax.h.lo + g->ax.h.hi > 0,
                           g->ay.e.lo + g->ay.e.hi > 0, g->az.e.lo + g->az.e.hi > 0,
                           g->az.e.lo + g->az.e.hi > 0, g->ax.e.lo + g->ax.e.hi > 0,
                           g->ax.e.lo + g->ax.e.hi > 0, g->ay.e.lo + g->ay.e.hi > 0};
    const float *ps[12] = {g->psi_hx_z, g->psi_hx_y, g->psi_hy_x, g->psi_hy_z, g->psi_hz_y, g->psi_hz_x,
                           g->psi_ex_y, g->psi_ex_z, g->psi_ey_z, g->psi_ey_x, g->psi_ez_x, g->psi_ez_y};
    for (int q = 0; q < 12; ++q)
        if (need[q] && !ps[q]) return false;
    if (g->src.ix >= 0) {
        if (!g->src.amp || !g->src.ph1 || !g->src.ph2 || g->src.ix + 1 >= g->nx) return false;
        if (g->src_comp < 0 || g->src_comp > 2 || g->src.pitch_k < g->src.nk) return false;
    }
    return true;
}

bool epi3d_ok(const LensEpi3D *ep, const LensStepTable *t, const LensGrid3D *g) {
    if (!ep) return true;
    if (ep->nbox < 0 || ep->nbox > LENS_MAX_BOX || (ep->nbox > 0 && !ep->box_acc)) return false;
    if (ep->nplane < 0 || ep->nplane > LENS_MAX_PLANE || (ep->nplane > 0 && !ep->plane_acc))
        return false;
    for (int p = 0; p < ep->nplane; ++p)
        if (ep->plane[p] < 1 || ep->plane[p] > g->nx - 2) return false;
    const bool dft = ep->dft[0] || ep->dft[1] || ep->dft[2] || ep->nplane > 0 || ep->conv_prev ||
                     ep->conv_last;
    return !dft || (t->pe && t->ph);
}

}  // namespace

extern "C" int lens_fdtd3d_step(const LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep,
                                int n0, int nsteps, void *stream) {
    if (!grid3d_ok(g) || nsteps < 0 || !lens_table_ok(tab, n0, nsteps) || !epi3d_ok(ep, tab, g))
        return LENS_ERR_ARG;
    LensEpi3D e{};  // zero: no boxes, empty windows, no planes
    if (ep) e = *ep;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 blk(BK, BJ), grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, g->nx);
    for (int n = n0; n < n0 + nsteps; ++n) {
        h3d<<<grd, blk, 0, s>>>(*g);
        e3d<<<grd, blk, 0, s>>>(*g, *tab, e, n);
    }
    return lens_cuda_status();
}

extern "C" int lens_fdtd3d_accum_e2(const LensGrid3D *g, int target, float *iavg, void *stream) {
    if (!grid3d_ok(g) || !iavg || (target != 1 && target != 2)) return LENS_ERR_ARG;
    const dim3 blk(BK, BJ), grd(g->pitch / BK, (g->ny + BJ - 1) / BJ, g->nx);
    accum_e2<<<grd, blk, 0, static_cast<cudaStream_t>(stream)>>>(*g, target, iavg);
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
