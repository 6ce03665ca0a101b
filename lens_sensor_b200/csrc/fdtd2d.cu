// 2D TE / TM CPML Yee step for sm_100a, with source, PEC and epilogues fused.
//
// One step = H half step (one launch) + E half step (one launch; TE also runs
// the epilogue there, TM needs node averages of the new E and runs it in a
// third, light launch).  Each thread owns one node (i, j); a block covers 8
// rows x 32 contiguous columns so every global access is a coalesced 128-byte
// row segment.
//
// Arithmetic follows planar_beads/boundaries.py:164-274 term by term:
//   TE  psi_Hxy = b*psi + c*dEz/dy;  Hx -= Ch*(dEz/dy/kappa + psi)      (:186-194)
//       psi_Hyx likewise along x;    Hy += Ch*(dEz/dx/kappa + psi)
//       Ez = CeE*Ez + CeH*(dHy/dx/kx + psi_x - dHx/dy/ky - psi_y)       (:196-205)
//   TM  Hz -= Ch*((dEy/dx/kx + psi) - (dEx/dy/ky + psi))                (:240-247)
//       E <- D*E (loss, fdtd2d_core.py:796-797), Ex += Ca_ex*(...),
//       Ey += -Ca_ey*(...)                                               (:249-258)
// then the Huygens source (vcsel.py:151-156) and the PEC termination
// (boundaries.py:207-215, 260-268) in the reference order (inject, then PEC).
#include "lens_common.cuh"

namespace {

constexpr int BX = 32;  // columns (contiguous j) per block
constexpr int BY = 8;   // rows (i) per block

__device__ __forceinline__ float src_term(const LensSource &s, const LensStepTable &tab, int n,
                                          int i, int j) {
    // vcsel.py:151-156: F[ix] += env*sin(wt + ph1)*amp ; F[ix+1] -= env*sin(wt + ph2)*amp
    const int k = n - tab.t0;
    if (i == s.ix) return (tab.env[k] * sinf(tab.wt[k] + s.ph1[j])) * s.amp[j];
    return -((tab.env[k] * sinf(tab.wt[k] + s.ph2[j])) * s.amp[j]);
}

// Epilogue on one node: detector boxes (FP64), compensated DFTs, intensity average.
// Every lane of the warp must call it (the box sums use warp shuffles).
__device__ __forceinline__ void epilogue_node(const LensEpi2D &ep, const LensStepTable &tab,
                                              int n, int i, int j, bool valid, size_t o,
                                              float field, float inten, float exn) {
    if (ep.nbox > 0) {
        const int bi0 = blockIdx.y * BY, bj0 = blockIdx.x * BX;
        for (int b = 0; b < ep.nbox; ++b) {
            const int *bx = ep.box[b];
            // block-uniform test: does this block touch box b at all?
            if (bx[1] <= bi0 || bx[0] >= bi0 + BY || bx[3] <= bj0 || bx[2] >= bj0 + BX) continue;
            const bool in = valid && i >= bx[0] && i < bx[1] && j >= bx[2] && j < bx[3];
            warp_atomic_add(ep.box_acc + b, in ? (double)inten : 0.0);
        }
    }
    if (!valid) return;
    const int k = n - tab.t0;
    if (n >= ep.dft_n0 && n < ep.dft_n1) {
        const float pr = tab.pe[2 * k], pi = tab.pe[2 * k + 1];
        if (ep.dft) kahan_add(reinterpret_cast<float4 *>(ep.dft) + o, field * pr, field * pi);
        if (ep.dft_ex) kahan_add(reinterpret_cast<float4 *>(ep.dft_ex) + o, exn * pr, exn * pi);
    }
    if (ep.dft_prev && n >= ep.prev_n0 && n < ep.prev_n1) {
        const float pr = tab.pe[2 * k], pi = tab.pe[2 * k + 1];
        kahan_add(reinterpret_cast<float4 *>(ep.dft_prev) + o, field * pr, field * pi);
    }
    if (ep.iavg && n >= ep.iavg_n0) ep.iavg[o] += inten;
}

// Plane DFT for the Poynting flux (flux.py:28-41): E on the plane, H averaged.
__device__ __forceinline__ void plane_node(const LensEpi2D &ep, const LensStepTable &tab, int n,
                                           int p, int pitch, int j, float e, float h) {
    const int k = n - tab.t0;
    double *a = ep.plane_acc + (size_t)p * 4 * pitch + j;
    const double er = tab.pe[2 * k], ei = tab.pe[2 * k + 1];
    const double hr = tab.ph[2 * k], hi = tab.ph[2 * k + 1];
    a[0] += (double)e * er;
    a[pitch] += (double)e * ei;
    a[2 * pitch] += (double)h * hr;
    a[3 * pitch] += (double)h * hi;
}

// Time-domain Poynting term of one plane cell (fdtd2d_core.py:489-497): the
// FP32 product of E and H averaged onto the E plane, summed in FP64.
__device__ __forceinline__ void sx_node(const LensEpi2D &ep, int p, int pitch, int j, float e, float h0, float h1) {
    const float h = __fmul_rn(0.5f, __fadd_rn(h0, h1));
    ep.sx_acc[(size_t)p * pitch + j] += (double)__fmul_rn(e, h);
}

__device__ __forceinline__ bool in_window(const LensEpi2D &ep, int n) {
    return n >= ep.dft_n0 && n < ep.dft_n1;
}

// Stitch drive of one cell of the driven component (rows i < d.nplanes):
// w * (env * Re(D e^{iwt})) in FP64 plus (1 - w) * E in FP32, rounded to FP32.
__device__ __forceinline__ float drive2(const LensDrive2D &d, const LensStepTable &tab, int n, int i,
                                        size_t o, float e) {
    const double *t = d.tab + 3 * (size_t)(n - tab.t0);
    const float2 D = reinterpret_cast<const float2 *>(d.hand)[o];
    const double re = __dsub_rn(__dmul_rn((double)D.x, t[1]), __dmul_rn((double)D.y, t[2]));
    const double din = __dmul_rn(t[0], re);
    const float w = d.taper[i];
    return (float)__dadd_rn(__dmul_rn((double)w, din), (double)__fmul_rn(__fsub_rn(1.0f, w), e));
}

// ------------------------------------------------------------------ TE
__global__ void __launch_bounds__(BX *BY) te2d_h(const LensTE2D g) {
    const int j = blockIdx.x * BX + threadIdx.x;
    const int i = blockIdx.y * BY + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int P = g.pitch;
    const size_t o = (size_t)i * P + j;
    const float ez = g.ez[o];
    if (j < g.ny - 1) {
        const float d = g.ez[o + 1] - ez;
        float p = 0.f;
        const int s = strip_of(j, g.ay.h.lo, g.ay.h.hi, g.ay.h.n);
        if (s >= 0) {
            float *q = g.psi_hxy + (size_t)i * (g.ay.h.lo + g.ay.h.hi) + s;
            p = g.ay.h.b[j] * (*q) + g.ay.h.c[j] * d;
            *q = p;
        }
        g.hx[o] = g.hx[o] - g.ch * (d * g.ay.h.ik[j] + p);
    }
    if (i < g.nx - 1) {
        const float d = g.ez[o + P] - ez;
        float p = 0.f;
        const int s = strip_of(i, g.ax.h.lo, g.ax.h.hi, g.ax.h.n);
        if (s >= 0) {
            float *q = g.psi_hyx + (size_t)s * P + j;
            p = g.ax.h.b[i] * (*q) + g.ax.h.c[i] * d;
            *q = p;
        }
        g.hy[o] = g.hy[o] + g.ch * (d * g.ax.h.ik[i] + p);
    }
}

__global__ void __launch_bounds__(BX *BY)
    te2d_e(const LensTE2D g, const LensStepTable tab, const LensEpi2D ep, int n, const LensDrive2D d) {
    const int j = blockIdx.x * BX + threadIdx.x;
    const int i = blockIdx.y * BY + threadIdx.y;
    const bool valid = i < g.nx && j < g.ny;
    const int P = g.pitch;
    const size_t o = (size_t)i * P + j;
    float ez = 0.f;
    if (valid) {
        ez = g.ez[o];
        if (i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1) {
            const float dhy = g.hy[o] - g.hy[o - P];
            const float dhx = g.hx[o] - g.hx[o - 1];
            float qx = 0.f, qy = 0.f;
            int s = strip_of(i, g.ax.e.lo, g.ax.e.hi, g.ax.e.n);
            if (s >= 0) {
                float *q = g.psi_ezx + (size_t)s * P + j;
                qx = g.ax.e.b[i] * (*q) + g.ax.e.c[i] * dhy;
                *q = qx;
            }
            s = strip_of(j, g.ay.e.lo, g.ay.e.hi, g.ay.e.n);
            if (s >= 0) {
                float *q = g.psi_ezy + (size_t)i * (g.ay.e.lo + g.ay.e.hi) + s;
                qy = g.ay.e.b[j] * (*q) + g.ay.e.c[j] * dhx;
                *q = qy;
            }
            ez = g.ce_e[o] * ez +
                 g.ce_h[o] * (dhy * g.ax.e.ik[i] + qx - dhx * g.ay.e.ik[j] - qy);
        }
        if (g.src.ix >= 0 && (i == g.src.ix || i == g.src.ix + 1) && j < g.src.nj)
            ez += src_term(g.src, tab, n, i, j);
        if (i < d.nplanes) ez = drive2(d, tab, n, i, o, ez);
        if ((g.pec[0] && i == 0) || (g.pec[1] && i == g.nx - 1) || (g.pec[2] && j == 0) ||
            (g.pec[3] && j == g.ny - 1))
            ez = 0.f;
        g.ez[o] = ez;
        if (ep.nplane > 0 && in_window(ep, n)) {
            for (int p = 0; p < ep.nplane; ++p)
                if (i == ep.plane[p])
                    plane_node(ep, tab, n, p, P, j, ez, 0.5f * (g.hy[o - P] + g.hy[o]));
        }
        for (int p = 0; p < ep.nsx; ++p)
            if (i == ep.sx_plane[p]) sx_node(ep, p, P, j, ez, g.hy[o - P], g.hy[o]);
    }
    epilogue_node(ep, tab, n, i, j, valid, o, ez, ez * ez, 0.f);
}

// ------------------------------------------------------------------ TM
__global__ void __launch_bounds__(BX *BY) tm2d_h(const LensTM2D g) {
    const int j = blockIdx.x * BX + threadIdx.x;
    const int i = blockIdx.y * BY + threadIdx.y;
    if (i >= g.nx - 1 || j >= g.ny - 1) return;
    const int P = g.pitch;
    const size_t o = (size_t)i * P + j;
    const float dyx = g.ey[o + P] - g.ey[o];
    const float dxy = g.ex[o + 1] - g.ex[o];
    float px = 0.f, py = 0.f;
    int s = strip_of(i, g.ax.h.lo, g.ax.h.hi, g.ax.h.n);
    if (s >= 0) {
        float *q = g.psi_hzx + (size_t)s * P + j;
        px = g.ax.h.b[i] * (*q) + g.ax.h.c[i] * dyx;
        *q = px;
    }
    s = strip_of(j, g.ay.h.lo, g.ay.h.hi, g.ay.h.n);
    if (s >= 0) {
        float *q = g.psi_hzy + (size_t)i * (g.ay.h.lo + g.ay.h.hi) + s;
        py = g.ay.h.b[j] * (*q) + g.ay.h.c[j] * dxy;
        *q = py;
    }
    g.hz[o] = g.hz[o] - g.ch * ((dyx * g.ax.h.ik[i] + px) - (dxy * g.ay.h.ik[j] + py));
}

__global__ void __launch_bounds__(BX *BY)
    tm2d_e(const LensTM2D g, const LensStepTable tab, int n, const LensDrive2D d) {
    const int j = blockIdx.x * BX + threadIdx.x;
    const int i = blockIdx.y * BY + threadIdx.y;
    const int P = g.pitch;
    const size_t o = (size_t)i * P + j;
    if (i < g.nx - 1 && j < g.ny) {  // Ex at (i+1/2, j)
        float e = g.ex[o];
        if (g.da_x) e = e * g.da_x[o];
        if (j > 0 && j < g.ny - 1) {
            const float d = g.hz[o] - g.hz[o - 1];
            float p = 0.f;
            const int s = strip_of(j, g.ay.e.lo, g.ay.e.hi, g.ay.e.n);
            if (s >= 0) {
                float *q = g.psi_exy + (size_t)i * (g.ay.e.lo + g.ay.e.hi) + s;
                p = g.ay.e.b[j] * (*q) + g.ay.e.c[j] * d;
                *q = p;
            }
            e = e + g.ca_x[o] * (d * g.ay.e.ik[j] + p);
        }
        if ((g.pec[2] && j == 0) || (g.pec[3] && j == g.ny - 1)) e = 0.f;
        g.ex[o] = e;
    }
    if (i < g.nx && j < g.ny - 1) {  // Ey at (i, j+1/2)
        float e = g.ey[o];
        if (g.da_y) e = e * g.da_y[o];
        if (i > 0 && i < g.nx - 1) {
            const float d = g.hz[o] - g.hz[o - P];
            float p = 0.f;
            const int s = strip_of(i, g.ax.e.lo, g.ax.e.hi, g.ax.e.n);
            if (s >= 0) {
                float *q = g.psi_eyx + (size_t)s * P + j;
                p = g.ax.e.b[i] * (*q) + g.ax.e.c[i] * d;
                *q = p;
            }
            e = e + (-g.ca_y[o]) * (d * g.ax.e.ik[i] + p);
        }
        if (g.src.ix >= 0 && (i == g.src.ix || i == g.src.ix + 1) && j < g.src.nj)
            e += src_term(g.src, tab, n, i, j);
        if (i < d.nplanes) e = drive2(d, tab, n, i, o, e);
        if ((g.pec[0] && i == 0) || (g.pec[1] && i == g.nx - 1)) e = 0.f;
        g.ey[o] = e;
    }
}

// Node averages of the new TM fields (fdtd2d_core.py:458-486) and the epilogue.
__global__ void __launch_bounds__(BX *BY)
    tm2d_epi(const LensTM2D g, const LensStepTable tab, const LensEpi2D ep, int n) {
    const int j = blockIdx.x * BX + threadIdx.x;
    const int i = blockIdx.y * BY + threadIdx.y;
    const bool valid = i < g.nx && j < g.ny;
    const int P = g.pitch;
    const size_t o = (size_t)i * P + j;
    float field = 0.f, inten = 0.f, exn = 0.f;
    if (valid) {
        const int ny = g.ny, nx = g.nx;
        const float *ey = g.ey + (size_t)i * P;
        field = (j == 0) ? ey[0] : (j == ny - 1) ? ey[ny - 2] : 0.5f * (ey[j - 1] + ey[j]);
        float s2;
        if (i == 0) {
            const float a = g.ex[j];
            s2 = a * a;
            exn = a;
        } else if (i == nx - 1) {
            const float a = g.ex[(size_t)(nx - 2) * P + j];
            s2 = a * a;
            exn = a;
        } else {
            const float a = g.ex[o - P], b = g.ex[o];
            s2 = 0.5f * (a * a + b * b);
            exn = 0.5f * (a + b);
        }
        inten = field * field + s2;
        if (in_window(ep, n)) {  // stitch: Ey on its own grid, Ex^2 on the nodes
            if (ep.dft_raw && j < ny - 1) {
                const int k = n - tab.t0;
                const float v = g.ey[o];
                kahan_add(reinterpret_cast<float4 *>(ep.dft_raw) + o, v * tab.pe[2 * k], v * tab.pe[2 * k + 1]);
            }
            if (ep.ex2) ep.ex2[o] += s2;
        }
        if (ep.nplane > 0 && in_window(ep, n) && j < ny - 1) {
            for (int p = 0; p < ep.nplane; ++p)
                if (i == ep.plane[p])
                    plane_node(ep, tab, n, p, P, j, g.ey[o], 0.5f * (g.hz[o - P] + g.hz[o]));
        }
        if (j < ny - 1)
            for (int p = 0; p < ep.nsx; ++p)
                if (i == ep.sx_plane[p]) sx_node(ep, p, P, j, g.ey[o], g.hz[o - P], g.hz[o]);
    }
    epilogue_node(ep, tab, n, i, j, valid, o, field, inten, exn);
}

bool epi2d_active(const LensEpi2D *ep, int n) {
    if (!ep) return false;
    if (ep->nbox > 0 || ep->nsx > 0) return true;
    if ((ep->dft || ep->dft_ex || ep->dft_raw || ep->ex2 || ep->nplane > 0) && n >= ep->dft_n0 && n < ep->dft_n1)
        return true;
    if (ep->dft_prev && n >= ep->prev_n0 && n < ep->prev_n1) return true;
    return ep->iavg && n >= ep->iavg_n0;
}

bool epi2d_ok(const LensEpi2D *ep, const LensStepTable *t, int nx) {
    if (!ep) return true;
    if (ep->nbox < 0 || ep->nbox > LENS_MAX_BOX || (ep->nbox > 0 && !ep->box_acc)) return false;
    if (ep->nplane < 0 || ep->nplane > LENS_MAX_PLANE || (ep->nplane > 0 && !ep->plane_acc))
        return false;
    for (int p = 0; p < ep->nplane; ++p)  // H is averaged over rows il-1 and il
        if (ep->plane[p] < 1 || ep->plane[p] > nx - 2) return false;
    if (ep->nsx < 0 || ep->nsx > LENS_MAX_PLANE || (ep->nsx > 0 && !ep->sx_acc)) return false;
    for (int p = 0; p < ep->nsx; ++p)
        if (ep->sx_plane[p] < 1 || ep->sx_plane[p] > nx - 2) return false;
    const bool dft = ep->dft || ep->dft_ex || ep->dft_prev || ep->dft_raw || ep->nplane > 0;
    return !dft || (t->pe && t->ph);
}

template <class G>
bool grid2d_ok(const G *g) {
    return g && g->nx >= 3 && g->ny >= 3 && g->pitch >= g->ny && (g->pitch % 32) == 0 &&
           lens_profile_ok(g->ax.e, g->nx) && lens_profile_ok(g->ax.h, g->nx - 1) &&
           lens_profile_ok(g->ay.e, g->ny) && lens_profile_ok(g->ay.h, g->ny - 1) &&
           (g->src.ix < 0 || (g->src.amp && g->src.ph1 && g->src.ph2 && g->src.ix + 1 < g->nx));
}

// psi arrays of the strips each kernel updates (te2d_h/te2d_e, tm2d_h/tm2d_e)
bool psi2d_ok(const LensTE2D *g) {
    return lens_psi_ok(g->ay.h, g->psi_hxy) && lens_psi_ok(g->ax.h, g->psi_hyx) &&
           lens_psi_ok(g->ax.e, g->psi_ezx) && lens_psi_ok(g->ay.e, g->psi_ezy);
}

bool psi2d_ok(const LensTM2D *g) {
    return lens_psi_ok(g->ax.h, g->psi_hzx) && lens_psi_ok(g->ay.h, g->psi_hzy) &&
           lens_psi_ok(g->ay.e, g->psi_exy) && lens_psi_ok(g->ax.e, g->psi_eyx);
}

LensEpi2D empty_epi() {
    LensEpi2D e{};
    e.dft_n0 = e.dft_n1 = 0;
    e.prev_n0 = e.prev_n1 = 0;
    e.iavg_n0 = 1 << 30;
    return e;
}

// A drive table must cover the steps run, its amplitudes the driven rows.
bool drive2d_ok(const LensDrive2D *d, const LensStepTable *tab, int nx) {
    return !d || d->nplanes == 0 || (d->nplanes > 0 && d->nplanes <= nx && d->taper && d->hand && d->tab &&
                                     (reinterpret_cast<uintptr_t>(d->hand) & 7) == 0 && tab);
}

int te2d_run(const LensTE2D *g, const LensStepTable *tab, const LensEpi2D *ep, const LensDrive2D *dr, int n0,
             int nsteps, void *stream) {
    if (!grid2d_ok(g) || !psi2d_ok(g) || !g->ez || !g->hx || !g->hy || !g->ce_e || !g->ce_h || nsteps < 0 ||
        !lens_table_ok(tab, n0, nsteps) || !epi2d_ok(ep, tab, g->nx) || !drive2d_ok(dr, tab, g->nx))
        return LENS_ERR_ARG;
    const LensEpi2D e = ep ? *ep : empty_epi();
    const LensDrive2D d = dr ? *dr : LensDrive2D{};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 blk(BX, BY), grd((g->ny + BX - 1) / BX, (g->nx + BY - 1) / BY);
    for (int n = n0; n < n0 + nsteps; ++n) {
        te2d_h<<<grd, blk, 0, s>>>(*g);
        te2d_e<<<grd, blk, 0, s>>>(*g, *tab, e, n, d);
    }
    return lens_cuda_status();
}

int tm2d_run(const LensTM2D *g, const LensStepTable *tab, const LensEpi2D *ep, const LensDrive2D *dr, int n0,
             int nsteps, void *stream) {
    if (!grid2d_ok(g) || !psi2d_ok(g) || !g->ex || !g->ey || !g->hz || !g->ca_x || !g->ca_y ||
        (!g->da_x) != (!g->da_y) || nsteps < 0 || !lens_table_ok(tab, n0, nsteps) ||
        !epi2d_ok(ep, tab, g->nx) || !drive2d_ok(dr, tab, g->nx))
        return LENS_ERR_ARG;
    const LensEpi2D e = ep ? *ep : empty_epi();
    const LensDrive2D d = dr ? *dr : LensDrive2D{};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 blk(BX, BY), grd((g->ny + BX - 1) / BX, (g->nx + BY - 1) / BY);
    for (int n = n0; n < n0 + nsteps; ++n) {
        tm2d_h<<<grd, blk, 0, s>>>(*g);
        tm2d_e<<<grd, blk, 0, s>>>(*g, *tab, n, d);
        if (epi2d_active(&e, n)) tm2d_epi<<<grd, blk, 0, s>>>(*g, *tab, e, n);
    }
    return lens_cuda_status();
}

}  // namespace

extern "C" int lens_te2d_step(const LensTE2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                              int n0, int nsteps, void *stream) {
    return te2d_run(g, tab, ep, nullptr, n0, nsteps, stream);
}

extern "C" int lens_tm2d_step(const LensTM2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                              int n0, int nsteps, void *stream) {
    return tm2d_run(g, tab, ep, nullptr, n0, nsteps, stream);
}

extern "C" int lens_te2d_step_driven(const LensTE2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                                     const LensDrive2D *drive, int n0, int nsteps, void *stream) {
    if (!drive) return LENS_ERR_ARG;
    return te2d_run(g, tab, ep, drive, n0, nsteps, stream);
}

extern "C" int lens_tm2d_step_driven(const LensTM2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                                     const LensDrive2D *drive, int n0, int nsteps, void *stream) {
    if (!drive) return LENS_ERR_ARG;
    return tm2d_run(g, tab, ep, drive, n0, nsteps, stream);
}
