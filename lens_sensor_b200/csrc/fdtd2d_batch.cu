// Batched 2D TE/TM steps for sm_100a: many independent solves of uneven sizes
// advanced together (tear-film / bead sweeps).
//
// One launch per half step covers every tile of every instance (128 columns x
// 2 * blockDim.y rows; a thread updates 4 columns of 2 rows); block b reads its
// instance from the plan's owner table (lens_batch2d_plan).  The per-cell arithmetic is term for
// term the single-grid kernels' (fdtd2d.cu, after planar_beads/boundaries.py:
// 164-274, source vcsel.py:151-156, loss fdtd2d_core.py:796-797), with the
// fields read and written in the batch's storage type (FP32, FP16 or BF16) and
// all arithmetic in FP32.
//
// Launches per step: H, E (TE: + node DFT), and on DFT-window steps a TM node
// epilogue (Ey averaged onto the nodes, fdtd2d_core.py:458-465).  A span of
// steps is graph-capturable: the host issues only kernel launches.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>

#include "lens_common.cuh"
#include "lens_store.cuh"

namespace {

constexpr int BXB = 32;  // lanes along y (contiguous)

// A block covers a tile of TW = 128 columns (y, contiguous) x blockDim.y * RB
// rows (x) of one instance: each thread updates VEC = 4 consecutive columns of
// RB consecutive rows, with one 16-byte (FP32) or 8-byte (FP16/BF16) access per
// field and row, all issued before the arithmetic; the single column beyond
// the thread's four (j+4 for H, j-1 for E) is a scalar load that hits the line
// the neighbouring lane brought in.  The H and E passes are held to 64
// registers (4 blocks of 256 threads per SM): they wait on memory, and the
// extra resident warps hide more of that latency than registers would save.
// owner[b] is the instance of block b and blk[q] its first block; the
// descriptor fields are read through the read-only cache (every thread of the
// block reads the same words).
constexpr int RB = 2;
constexpr int VEC = 4;
constexpr int TW = BXB * VEC;

struct Tile {
    const LensInst2D *g;
    int i, j;  // first row and first column of this thread
};

__device__ __forceinline__ Tile tile_of(const LensInst2D *inst, const int *blk, const int *owner, int b) {
    const int q = __ldg(owner + b);
    const LensInst2D *g = inst + q;
    const int t = b - __ldg(blk + q);
    const int ntj = (__ldg(&g->ny) + TW - 1) / TW;
    return Tile{g, (t / ntj) * (int)blockDim.y * RB + (int)threadIdx.y * RB,
                (t % ntj) * TW + (int)threadIdx.x * VEC};
}

// Read-only view of one instance descriptor (loads through the non-coherent cache).
struct V {
    const LensInst2D *p;
    __device__ __forceinline__ int pol() const { return __ldg(&p->pol); }
    __device__ __forceinline__ int nx() const { return __ldg(&p->nx); }
    __device__ __forceinline__ int ny() const { return __ldg(&p->ny); }
    __device__ __forceinline__ int pitch() const { return __ldg(&p->pitch); }
    __device__ __forceinline__ void *f(int q) const {
        return reinterpret_cast<void *>(__ldg(reinterpret_cast<const unsigned long long *>(&p->f[q])));
    }
    __device__ __forceinline__ const float *c(int q) const {
        return reinterpret_cast<const float *>(__ldg(reinterpret_cast<const unsigned long long *>(&p->c[q])));
    }
    __device__ __forceinline__ float *psi(int q) const {
        return reinterpret_cast<float *>(__ldg(reinterpret_cast<const unsigned long long *>(&p->psi[q])));
    }
    __device__ __forceinline__ float ch() const { return __ldg(&p->ch); }
    // coefficient q of row i from column j0 on: the row-type table where row i
    // has a type, else the instance's own array
    __device__ __forceinline__ const float *crow(int q, int ncoef, int i, int j0, size_t o) const {
        const unsigned char *rt = reinterpret_cast<const unsigned char *>(
            __ldg(reinterpret_cast<const unsigned long long *>(&p->rtype)));
        const unsigned t = rt ? __ldg(rt + i) : 255u;
        if (t == 255u) return c(q) + o;
        const float *tab = reinterpret_cast<const float *>(__ldg(reinterpret_cast<const unsigned long long *>(&p->ctab)));
        return tab + ((size_t)t * ncoef + q) * (size_t)pitch() + j0;
    }
    __device__ __forceinline__ const LensProfile &prof(bool x, bool e) const {
        return x ? (e ? p->ax.e : p->ax.h) : (e ? p->ay.e : p->ay.h);
    }
};

__device__ __forceinline__ float src_b(const LensSource &s, const LensStepTable &tab, int n, int i, int j) {
    const int k = n - tab.t0;
    if (i == s.ix) return (tab.env[k] * sinf(tab.wt[k] + s.ph1[j])) * s.amp[j];
    return -((tab.env[k] * sinf(tab.wt[k] + s.ph2[j])) * s.amp[j]);
}

__device__ __forceinline__ void dft_node(const LensInst2D *g, const LensStepTable &tab, int n, size_t o, float v) {
    float *d = reinterpret_cast<float *>(__ldg(reinterpret_cast<const unsigned long long *>(&g->dft)));
    if (d && n >= __ldg(&g->dft_n0) && n < __ldg(&g->dft_n1)) {
        const int k = n - tab.t0;
        float2 *a = reinterpret_cast<float2 *>(d) + o;
        float2 s = *a;
        s.x += v * tab.pe[2 * k];
        s.y += v * tab.pe[2 * k + 1];
        *a = s;
    }
}

// A zero the compiler cannot see through: the lean passes add it where the
// general passes add a psi term, so both evaluate the same expression shapes.
__device__ __forceinline__ float opaque_zero() {
    float z;
    asm volatile("mov.b32 %0, 0;" : "=f"(z));
    return z;
}

// Rows [i0, i0 + RB) / columns [j0, j0 + VEC) of a thread clear of a profile's
// psi strips ([lo, n - hi) is strip-free), of the faces and of the source rows:
// a warp whose threads are all clear takes the lean passes below (no per-cell
// tests); a warp with one thread at a face or in a strip takes the general pass.
__device__ __forceinline__ bool clear_of(const LensProfile &p, int a, int b, int lo_min, int hi_max) {
    return a >= max(p.lo, lo_min) && b <= min(p.n - p.hi, hi_max);
}

// psi update at profile entry m: psi = b*psi + c*d, stored; returns the new psi.
__device__ __forceinline__ float psi_step(const LensProfile &pf, int m, float *q, float d) {
    const float p = __ldg(pf.b + m) * (*q) + __ldg(pf.c + m) * d;
    *q = p;
    return p;
}

// H of tile b (boundaries.py:186-194 / 240-247).
template <typename T>
__device__ __forceinline__ void h_tile(const LensInst2D *inst, const int *blk, const int *owner, int b) {
    const Tile tl = tile_of(inst, blk, owner, b);
    const V g{tl.g};
    const int i0 = tl.i, j0 = tl.j, nx = g.nx(), ny = g.ny(), P = g.pitch();
    if (i0 >= nx || j0 >= ny) return;   // j0 < ny <= P: the four columns lie inside the row pitch
    const float ch = g.ch();
    using S = St<T>;
    const LensProfile &xh = g.prof(true, false), &yh = g.prof(false, false);
    const int wy = yh.lo + yh.hi;
    if (g.pol() == 0) {  // TE: Hx, Hy from Ez (boundaries.py:186-194)
        const void *ezp = g.f(0);
        void *hxp = g.f(1), *hyp = g.f(2);
        float ez[RB + 1][VEC], ezn[RB], hx[RB][VEC], hy[RB][VEC];
#pragma unroll
        for (int r = 0; r <= RB; ++r) {
            const bool in = i0 + r < nx;
            f4_to(in ? S::ld4(ezp, (size_t)(i0 + r) * P + j0) : make_float4(0.f, 0.f, 0.f, 0.f), ez[r]);
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const size_t o = (size_t)(i0 + r) * P + j0;
            const bool in = i0 + r < nx;
            ezn[r] = (in && j0 + VEC < ny) ? S::ld(ezp, o + VEC) : 0.f;
            f4_to(in ? S::ld4(hxp, o) : make_float4(0.f, 0.f, 0.f, 0.f), hx[r]);
            f4_to(in ? S::ld4(hyp, o) : make_float4(0.f, 0.f, 0.f, 0.f), hy[r]);
        }
        if (__all_sync(__activemask(), clear_of(xh, i0, i0 + RB, 0, nx - 1) && clear_of(yh, j0, j0 + VEC, 0, ny - 1))) {
            const float z = opaque_zero();  // lean: every Hx and Hy updates, no psi
#pragma unroll
            for (int r = 0; r < RB; ++r) {
                const int i = i0 + r;
                const size_t o = (size_t)i * P + j0;
                const float ki = __ldg(xh.ik + i);
                float nhx[VEC], nhy[VEC];
#pragma unroll
                for (int c = 0; c < VEC; ++c) {
                    const float d = (c + 1 < VEC ? ez[r][c + 1] : ezn[r]) - ez[r][c];
                    nhx[c] = hx[r][c] - ch * (d * __ldg(yh.ik + j0 + c) + z);
                    const float d2 = ez[r + 1][c] - ez[r][c];
                    nhy[c] = hy[r][c] + ch * (d2 * ki + z);
                }
                S::st4(hxp, o, to_f4(nhx));
                S::st4(hyp, o, to_f4(nhy));
            }
            return;
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const int i = i0 + r;
            if (i >= nx) break;
            const size_t o = (size_t)i * P + j0;
            float nhx[VEC], nhy[VEC];
            const int s = i < nx - 1 ? strip_of(i, xh.lo, xh.hi, xh.n) : -1;
            const float ki = i < nx - 1 ? __ldg(xh.ik + i) : 0.f;
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
                const int j = j0 + c;
                nhx[c] = hx[r][c];
                nhy[c] = hy[r][c];
                if (j < ny - 1) {
                    const float d = (c + 1 < VEC ? ez[r][c + 1] : ezn[r]) - ez[r][c];
                    float p = 0.f;
                    const int sj = strip_of(j, yh.lo, yh.hi, yh.n);
                    if (sj >= 0) p = psi_step(yh, j, g.psi(0) + (size_t)i * wy + sj, d);
                    nhx[c] = hx[r][c] - ch * (d * __ldg(yh.ik + j) + p);
                }
                if (i < nx - 1 && j < ny) {
                    const float d = ez[r + 1][c] - ez[r][c];
                    float p = 0.f;
                    if (s >= 0) p = psi_step(xh, i, g.psi(1) + (size_t)s * P + j, d);
                    nhy[c] = hy[r][c] + ch * (d * ki + p);
                }
            }
            S::st4(hxp, o, to_f4(nhx));
            S::st4(hyp, o, to_f4(nhy));
        }
        return;
    }
    // TM: Hz from Ex, Ey (boundaries.py:240-247)
    if (i0 >= nx - 1) return;
    const void *exp_ = g.f(0), *eyp = g.f(1);
    void *hzp = g.f(2);
    float ey[RB + 1][VEC], ex[RB][VEC], exn[RB], hz[RB][VEC];
#pragma unroll
    for (int r = 0; r <= RB; ++r) {
        const bool in = i0 + r < nx;
        f4_to(in ? S::ld4(eyp, (size_t)(i0 + r) * P + j0) : make_float4(0.f, 0.f, 0.f, 0.f), ey[r]);
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const size_t o = (size_t)(i0 + r) * P + j0;
        const bool in = i0 + r < nx - 1;
        f4_to(in ? S::ld4(exp_, o) : make_float4(0.f, 0.f, 0.f, 0.f), ex[r]);
        exn[r] = (in && j0 + VEC < ny) ? S::ld(exp_, o + VEC) : 0.f;
        f4_to(in ? S::ld4(hzp, o) : make_float4(0.f, 0.f, 0.f, 0.f), hz[r]);
    }
    if (__all_sync(__activemask(), clear_of(xh, i0, i0 + RB, 0, nx - 1) && clear_of(yh, j0, j0 + VEC, 0, ny - 1))) {
        const float z = opaque_zero();  // lean: every Hz updates, no psi
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const int i = i0 + r;
            const size_t o = (size_t)i * P + j0;
            const float ki = __ldg(xh.ik + i);
            float nhz[VEC];
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
                const float dyx = ey[r + 1][c] - ey[r][c], dxy = (c + 1 < VEC ? ex[r][c + 1] : exn[r]) - ex[r][c];
                nhz[c] = hz[r][c] - ch * ((dyx * ki + z) - (dxy * __ldg(yh.ik + j0 + c) + z));
            }
            S::st4(hzp, o, to_f4(nhz));
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const int i = i0 + r;
        if (i >= nx - 1) break;
        const size_t o = (size_t)i * P + j0;
        const int s = strip_of(i, xh.lo, xh.hi, xh.n);
        const float ki = __ldg(xh.ik + i);
        float nhz[VEC];
#pragma unroll
        for (int c = 0; c < VEC; ++c) {
            const int j = j0 + c;
            nhz[c] = hz[r][c];
            if (j < ny - 1) {
                const float dyx = ey[r + 1][c] - ey[r][c], dxy = (c + 1 < VEC ? ex[r][c + 1] : exn[r]) - ex[r][c];
                float px = 0.f, py = 0.f;
                const int sj = strip_of(j, yh.lo, yh.hi, yh.n);
                if (s >= 0) px = psi_step(xh, i, g.psi(0) + (size_t)s * P + j, dyx);
                if (sj >= 0) py = psi_step(yh, j, g.psi(1) + (size_t)i * wy + sj, dxy);
                nhz[c] = hz[r][c] - ch * ((dyx * ki + px) - (dxy * __ldg(yh.ik + j) + py));
            }
        }
        S::st4(hzp, o, to_f4(nhz));
    }
}

// E of tile b at batch step n (boundaries.py:196-215 / 249-268), source, PEC, node DFT.
template <typename T>
__device__ __forceinline__ void e_tile(const LensInst2D *inst, const int *blk, const int *owner, const LensStepTable &tab,
                                       int n, int b) {
    const Tile tl = tile_of(inst, blk, owner, b);
    const V g{tl.g};
    const int i0 = tl.i, j0 = tl.j, nx = g.nx(), ny = g.ny(), P = g.pitch();
    if (i0 >= nx || j0 >= ny) return;
    using S = St<T>;
    const LensProfile &xe = g.prof(true, true), &ye = g.prof(false, true);
    const int wy = ye.lo + ye.hi;
    const LensSource &src = tl.g->src;
    const int *pec = tl.g->pec;
    const int six = __ldg(&src.ix), snj = __ldg(&src.nj);
    n -= __ldg(&tl.g->n_start);  // the instance's own step
    const int pec0 = __ldg(pec), pec1 = __ldg(pec + 1), pec2 = __ldg(pec + 2), pec3 = __ldg(pec + 3);
    if (g.pol() == 0) {  // TE: Ez (boundaries.py:196-215), source, PEC, node DFT
        void *ezp = g.f(0);
        const void *hxp = g.f(1), *hyp = g.f(2);
        float hy[RB + 1][VEC], hx[RB][VEC], hxp1[RB], ez[RB][VEC];
#pragma unroll
        for (int r = 0; r <= RB; ++r) {  // hy[r] = Hy(i0 + r - 1)
            const int i = i0 + r - 1;
            f4_to((i >= 0 && i < nx) ? S::ld4(hyp, (size_t)i * P + j0) : make_float4(0.f, 0.f, 0.f, 0.f), hy[r]);
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const int i = i0 + r;
            const size_t o = (size_t)i * P + j0;
            const bool in = i < nx;
            f4_to(in ? S::ld4(hxp, o) : make_float4(0.f, 0.f, 0.f, 0.f), hx[r]);
            hxp1[r] = (in && j0 >= 1) ? S::ld(hxp, o - 1) : 0.f;       // Hx(i, j0-1)
            f4_to(in ? S::ld4(ezp, o) : make_float4(0.f, 0.f, 0.f, 0.f), ez[r]);
        }
        if (__all_sync(__activemask(), clear_of(xe, i0, i0 + RB, 1, nx - 1) && clear_of(ye, j0, j0 + VEC, 1, ny - 1) &&
                                           (six < 0 || six + 1 < i0 || six >= i0 + RB))) {
            const float z = opaque_zero();  // lean: interior cells, no psi, source or PEC
            float *dft = reinterpret_cast<float *>(__ldg(reinterpret_cast<const unsigned long long *>(&tl.g->dft)));
            const bool win = dft && n >= __ldg(&tl.g->dft_n0) && n < __ldg(&tl.g->dft_n1);
#pragma unroll
            for (int r = 0; r < RB; ++r) {
                const int i = i0 + r;
                const size_t o = (size_t)i * P + j0;
                const float ki = __ldg(xe.ik + i);
                float c0[VEC], c1[VEC], v4[VEC];
                f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(0, 2, i, j0, o))), c0);
                f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(1, 2, i, j0, o))), c1);
#pragma unroll
                for (int c = 0; c < VEC; ++c) {
                    const float dhy = hy[r + 1][c] - hy[r][c], dhx = hx[r][c] - (c > 0 ? hx[r][c - 1] : hxp1[r]);
                    v4[c] = c0[c] * ez[r][c] + c1[c] * (dhy * ki + z - dhx * __ldg(ye.ik + j0 + c) - z);
                }
                S::st4(ezp, o, to_f4(v4));
                if (win) {  // dft_node on the four cells
                    const int k = n - tab.t0;
                    const float pr = tab.pe[2 * k], pim = tab.pe[2 * k + 1];
                    float4 *a = reinterpret_cast<float4 *>(dft + 2 * o);
                    float4 s0 = a[0], s1 = a[1];
                    s0.x += v4[0] * pr; s0.y += v4[0] * pim; s0.z += v4[1] * pr; s0.w += v4[1] * pim;
                    s1.x += v4[2] * pr; s1.y += v4[2] * pim; s1.z += v4[3] * pr; s1.w += v4[3] * pim;
                    a[0] = s0;
                    a[1] = s1;
                }
            }
            return;
        }
        if (__all_sync(__activemask(), clear_of(xe, i0, i0 + RB, 1, nx - 1) &&
                                           (six < 0 || six + 1 < i0 || six >= i0 + RB))) {
            // rows clear of x strips, x faces and the source: the y tests only
            const float z = opaque_zero();
#pragma unroll
            for (int r = 0; r < RB; ++r) {
                const int i = i0 + r;
                const size_t o = (size_t)i * P + j0;
                const float ki = __ldg(xe.ik + i);
                float c0[VEC], c1[VEC], v4[VEC];
                f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(0, 2, i, j0, o))), c0);
                f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(1, 2, i, j0, o))), c1);
#pragma unroll
                for (int c = 0; c < VEC; ++c) {
                    const int j = j0 + c;
                    float v = ez[r][c];
                    if (j > 0 && j < ny - 1) {
                        const float dhy = hy[r + 1][c] - hy[r][c], dhx = hx[r][c] - (c > 0 ? hx[r][c - 1] : hxp1[r]);
                        float qy = z;
                        const int sj = strip_of(j, ye.lo, ye.hi, ye.n);
                        if (sj >= 0) qy = psi_step(ye, j, g.psi(3) + (size_t)i * wy + sj, dhx);
                        v = c0[c] * v + c1[c] * (dhy * ki + z - dhx * __ldg(ye.ik + j) - qy);
                    }
                    if ((pec2 && j == 0) || (pec3 && j == ny - 1)) v = 0.f;
                    if (j >= ny) v = 0.f;
                    v4[c] = v;
                    if (j < ny) dft_node(tl.g, tab, n, o + c, v);
                }
                S::st4(ezp, o, to_f4(v4));
            }
            return;
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const int i = i0 + r;
            if (i >= nx) break;
            const size_t o = (size_t)i * P + j0;
            const int s = (i > 0 && i < nx - 1) ? strip_of(i, xe.lo, xe.hi, xe.n) : -1;
            const float ki = __ldg(xe.ik + i);
            float c0[VEC], c1[VEC], v4[VEC];
            f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(0, 2, i, j0, o))), c0);
            f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(1, 2, i, j0, o))), c1);
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
                const int j = j0 + c;
                float v = ez[r][c];
                if (j > 0 && j < ny - 1 && i > 0 && i < nx - 1) {
                    const float dhy = hy[r + 1][c] - hy[r][c], dhx = hx[r][c] - (c > 0 ? hx[r][c - 1] : hxp1[r]);
                    float qx = 0.f, qy = 0.f;
                    const int sj = strip_of(j, ye.lo, ye.hi, ye.n);
                    if (s >= 0) qx = psi_step(xe, i, g.psi(2) + (size_t)s * P + j, dhy);
                    if (sj >= 0) qy = psi_step(ye, j, g.psi(3) + (size_t)i * wy + sj, dhx);
                    v = c0[c] * v + c1[c] * (dhy * ki + qx - dhx * __ldg(ye.ik + j) - qy);
                }
                if ((i == six || i == six + 1) && j < snj) v += src_b(src, tab, n, i, j);
                if ((pec0 && i == 0) || (pec1 && i == nx - 1) || (pec2 && j == 0) || (pec3 && j == ny - 1)) v = 0.f;
                if (j >= ny) v = 0.f;
                v4[c] = v;
                if (j < ny) dft_node(tl.g, tab, n, o + c, v);
            }
            S::st4(ezp, o, to_f4(v4));
        }
        return;
    }
    // TM: loss damping, Ex / Ey (boundaries.py:249-268), source, PEC
    void *exp_ = g.f(0), *eyp = g.f(1);
    const void *hzp = g.f(2);
    const float *dax = g.c(2), *day = g.c(3);
    float hz[RB + 1][VEC], hzp1[RB], ex[RB][VEC], ey[RB][VEC];
#pragma unroll
    for (int r = 0; r <= RB; ++r) {  // hz[r] = Hz(i0 + r - 1)
        const int i = i0 + r - 1;
        f4_to((i >= 0 && i < nx - 1) ? S::ld4(hzp, (size_t)i * P + j0) : make_float4(0.f, 0.f, 0.f, 0.f), hz[r]);
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const int i = i0 + r;
        const size_t o = (size_t)i * P + j0;
        f4_to(i < nx - 1 ? S::ld4(exp_, o) : make_float4(0.f, 0.f, 0.f, 0.f), ex[r]);
        hzp1[r] = (i < nx - 1 && j0 >= 1) ? S::ld(hzp, o - 1) : 0.f;   // Hz(i, j0-1)
        f4_to(i < nx ? S::ld4(eyp, o) : make_float4(0.f, 0.f, 0.f, 0.f), ey[r]);
    }
    if (__all_sync(__activemask(), clear_of(xe, i0, i0 + RB, 1, nx - 1) && clear_of(ye, j0, j0 + VEC, 1, ny - 1) &&
                                       (six < 0 || six + 1 < i0 || six >= i0 + RB))) {
        const float z = opaque_zero();  // lean: interior cells, no psi, source or PEC
        const int nq = dax ? 4 : 2;
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const int i = i0 + r;
            const size_t o = (size_t)i * P + j0;
            float ax_[VEC], ay_[VEC], dx_[VEC], dy_[VEC];
            f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(0, nq, i, j0, o))), ax_);
            f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(1, nq, i, j0, o))), ay_);
            f4_to(dax ? __ldg(reinterpret_cast<const float4 *>(g.crow(2, nq, i, j0, o))) : make_float4(1.f, 1.f, 1.f, 1.f),
                  dx_);
            f4_to(day ? __ldg(reinterpret_cast<const float4 *>(g.crow(3, nq, i, j0, o))) : make_float4(1.f, 1.f, 1.f, 1.f),
                  dy_);
            const float ki = __ldg(xe.ik + i);
            float nex[VEC], ney[VEC];
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
                float e = ex[r][c];
                if (dax) e = e * dx_[c];
                const float d = hz[r + 1][c] - (c > 0 ? hz[r + 1][c - 1] : hzp1[r]);
                nex[c] = e + ax_[c] * (d * __ldg(ye.ik + j0 + c) + z);
                float e2 = ey[r][c];
                if (day) e2 = e2 * dy_[c];
                const float d2 = hz[r + 1][c] - hz[r][c];
                ney[c] = e2 + (-ay_[c]) * (d2 * ki + z);
            }
            S::st4(exp_, o, to_f4(nex));
            S::st4(eyp, o, to_f4(ney));
        }
        return;
    }
    if (__all_sync(__activemask(), clear_of(xe, i0, i0 + RB, 1, nx - 1) &&
                                       (six < 0 || six + 1 < i0 || six >= i0 + RB))) {
        // rows clear of x strips, x faces and the source: the y tests only
        const float z = opaque_zero();
        const int nq = dax ? 4 : 2;
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const int i = i0 + r;
            const size_t o = (size_t)i * P + j0;
            float ax_[VEC], ay_[VEC], dx_[VEC], dy_[VEC];
            f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(0, nq, i, j0, o))), ax_);
            f4_to(__ldg(reinterpret_cast<const float4 *>(g.crow(1, nq, i, j0, o))), ay_);
            f4_to(dax ? __ldg(reinterpret_cast<const float4 *>(g.crow(2, nq, i, j0, o))) : make_float4(1.f, 1.f, 1.f, 1.f),
                  dx_);
            f4_to(day ? __ldg(reinterpret_cast<const float4 *>(g.crow(3, nq, i, j0, o))) : make_float4(1.f, 1.f, 1.f, 1.f),
                  dy_);
            const float ki = __ldg(xe.ik + i);
            float nex[VEC], ney[VEC];
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
                const int j = j0 + c;
                nex[c] = ex[r][c];
                ney[c] = ey[r][c];
                if (j < ny) {  // Ex at (i+1/2, j)
                    float e = ex[r][c];
                    if (dax) e = e * dx_[c];
                    if (j > 0 && j < ny - 1) {
                        const float d = hz[r + 1][c] - (c > 0 ? hz[r + 1][c - 1] : hzp1[r]);
                        float p = z;
                        const int sj = strip_of(j, ye.lo, ye.hi, ye.n);
                        if (sj >= 0) p = psi_step(ye, j, g.psi(2) + (size_t)i * wy + sj, d);
                        e = e + ax_[c] * (d * __ldg(ye.ik + j) + p);
                    }
                    if ((pec2 && j == 0) || (pec3 && j == ny - 1)) e = 0.f;
                    nex[c] = e;
                }
                if (j < ny - 1) {  // Ey at (i, j+1/2)
                    float e = ey[r][c];
                    if (day) e = e * dy_[c];
                    const float d = hz[r + 1][c] - hz[r][c];
                    ney[c] = e + (-ay_[c]) * (d * ki + z);
                }
            }
            S::st4(exp_, o, to_f4(nex));
            S::st4(eyp, o, to_f4(ney));
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const int i = i0 + r;
        if (i >= nx) break;
        const size_t o = (size_t)i * P + j0;
        const int nq = dax ? 4 : 2;
        const float4 ax4 = __ldg(reinterpret_cast<const float4 *>(g.crow(0, nq, i, j0, o)));
        const float4 ay4 = __ldg(reinterpret_cast<const float4 *>(g.crow(1, nq, i, j0, o)));
        const float4 dx4 = dax ? __ldg(reinterpret_cast<const float4 *>(g.crow(2, nq, i, j0, o)))
                               : make_float4(1.f, 1.f, 1.f, 1.f);
        const float4 dy4 = day ? __ldg(reinterpret_cast<const float4 *>(g.crow(3, nq, i, j0, o)))
                               : make_float4(1.f, 1.f, 1.f, 1.f);
        float ax_[VEC], ay_[VEC], dx_[VEC], dy_[VEC];
        f4_to(ax4, ax_); f4_to(ay4, ay_); f4_to(dx4, dx_); f4_to(dy4, dy_);
        const int s = (i > 0 && i < nx - 1) ? strip_of(i, xe.lo, xe.hi, xe.n) : -1;
        const float ki = __ldg(xe.ik + i);
        float nex[VEC], ney[VEC];
#pragma unroll
        for (int c = 0; c < VEC; ++c) {
            const int j = j0 + c;
            const bool jin = j > 0 && j < ny - 1;
            nex[c] = ex[r][c];
            ney[c] = ey[r][c];
            if (i < nx - 1 && j < ny) {  // Ex at (i+1/2, j)
                float e = ex[r][c];
                if (dax) e = e * dx_[c];
                if (jin) {
                    const float d = hz[r + 1][c] - (c > 0 ? hz[r + 1][c - 1] : hzp1[r]);
                    float p = 0.f;
                    const int sj = strip_of(j, ye.lo, ye.hi, ye.n);
                    if (sj >= 0) p = psi_step(ye, j, g.psi(2) + (size_t)i * wy + sj, d);
                    e = e + ax_[c] * (d * __ldg(ye.ik + j) + p);
                }
                if ((pec2 && j == 0) || (pec3 && j == ny - 1)) e = 0.f;
                nex[c] = e;
            }
            if (j < ny - 1) {  // Ey at (i, j+1/2)
                float e = ey[r][c];
                if (day) e = e * dy_[c];
                if (i > 0 && i < nx - 1) {
                    const float d = hz[r + 1][c] - hz[r][c];
                    float p = 0.f;
                    if (s >= 0) p = psi_step(xe, i, g.psi(3) + (size_t)s * P + j, d);
                    e = e + (-ay_[c]) * (d * ki + p);
                }
                if ((i == six || i == six + 1) && j < snj) e += src_b(src, tab, n, i, j);
                if ((pec0 && i == 0) || (pec1 && i == nx - 1)) e = 0.f;
                ney[c] = e;
            }
        }
        if (i < nx - 1) S::st4(exp_, o, to_f4(nex));
        S::st4(eyp, o, to_f4(ney));
    }
}

// TM node DFT of tile b: Ey averaged onto the nodes (fdtd2d_core.py:458-465).
template <typename T>
__device__ __forceinline__ void node_tile(const LensInst2D *inst, const int *blk, const int *owner,
                                          const LensStepTable &tab, int n, int b) {
    const Tile tl = tile_of(inst, blk, owner, b);
    const V g{tl.g};
    if (g.pol() != 1) return;
    const int i0 = tl.i, j0 = tl.j, nx = g.nx(), ny = g.ny(), P = g.pitch();
    if (i0 >= nx || j0 >= ny) return;
    n -= __ldg(&tl.g->n_start);
    using S = St<T>;
    const void *p1 = g.f(1);
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const int i = i0 + r;
        if (i >= nx) break;
        const size_t row = (size_t)i * P;
#pragma unroll
        for (int c = 0; c < VEC; ++c) {
            const int j = j0 + c;
            if (j >= ny) break;
            const float v = (j == 0) ? S::ld(p1, row) : (j == ny - 1) ? S::ld(p1, row + ny - 2)
                                                                    : 0.5f * (S::ld(p1, row + j - 1) + S::ld(p1, row + j));
            dft_node(tl.g, tab, n, row + j, v);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256, 4) b2d_h(const LensInst2D *inst, const int *blk, const int *owner) {
    h_tile<T>(inst, blk, owner, blockIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(256, 4)
    b2d_e(const LensInst2D *inst, const int *blk, const int *owner, const LensStepTable tab, int n) {
    e_tile<T>(inst, blk, owner, tab, n, blockIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(256)
    b2d_tm_node(const LensInst2D *inst, const int *blk, const int *owner, const LensStepTable tab, int n) {
    node_tile<T>(inst, blk, owner, tab, n, blockIdx.x);
}

// ------------------------------------------------------ persistent batched run
// One cooperative launch advances the whole batch by nsteps: the blocks (all
// resident at once) stride over the batch's tiles in each phase and meet at a
// grid barrier between the H and E phases of every step (and after the TM node
// DFT on its window steps), so a batch whose state fits in L2 keeps it there
// across steps and no launch gap separates them.  Tile b is always handled by
// block b mod gridDim.x, so a thread's DFT sums stay its own.
//
// Barrier: sync[0] counts the arrivals of the current generation sync[1]; the
// last block to arrive resets the count and opens the next generation.  Every
// wait is bounded (PB_TRIES polls of at least 64 ns, about a second); a wait that
// runs out, or sees another block's error, sets *err and the kernel returns.
constexpr long long PB_TRIES = 1LL << 24;

__device__ __forceinline__ bool grid_barrier(unsigned *sync, int *err) {
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        volatile unsigned *gen = sync + 1;
        volatile int *verr = err;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(sync, 1u) == gridDim.x - 1) {
            atomicExch(sync, 0u);
            __threadfence();
            atomicAdd(sync + 1, 1u);
        } else {
            long long t = 0;
            while (*gen == g) {
                if (*verr || ++t > PB_TRIES) {
                    atomicOr(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *reinterpret_cast<volatile int *>(err) == 0;
}

template <typename T>
__global__ void __launch_bounds__(256, 3)
    pb2d(const LensInst2D *inst, const int *blk, const int *owner, int nblk, const LensStepTable tab, int n0,
         int nsteps, int tm_lo, int tm_hi, unsigned *sync, int *err) {
    for (int n = n0; n < n0 + nsteps; ++n) {
        for (int b = blockIdx.x; b < nblk; b += gridDim.x) h_tile<T>(inst, blk, owner, b);
        if (!grid_barrier(sync, err)) return;
        for (int b = blockIdx.x; b < nblk; b += gridDim.x) e_tile<T>(inst, blk, owner, tab, n, b);
        if (!grid_barrier(sync, err)) return;
        // the node DFT reads Ey of the neighbouring tile's first column: after the E
        // barrier; the next E phase that rewrites Ey comes after the next H barrier
        if (n >= tm_lo && n < tm_hi)
            for (int b = blockIdx.x; b < nblk; b += gridDim.x) node_tile<T>(inst, blk, owner, tab, n, b);
    }
}

bool inst_ok(const LensInst2D &g) {
    if ((g.pol != 0 && g.pol != 1) || g.nx < 3 || g.ny < 3 || g.pitch < g.ny || (g.pitch % 32)) return false;
    if (!g.f[0] || !g.f[1] || !g.f[2] || !g.c[0] || !g.c[1]) return false;
    if (g.pol == 1 && (!g.c[2]) != (!g.c[3])) return false;
    if (g.rtype && !g.ctab) return false;
    if (!lens_profile_ok(g.ax.e, g.nx) || !lens_profile_ok(g.ax.h, g.nx - 1) || !lens_profile_ok(g.ay.e, g.ny) ||
        !lens_profile_ok(g.ay.h, g.ny - 1))
        return false;
    if (g.src.ix >= 0 && (!g.src.amp || !g.src.ph1 || !g.src.ph2 || g.src.ix + 1 >= g.nx || g.src.nj > g.ny))
        return false;
    // psi[q] of the strip it serves: TE hxy (y, H), hyx (x, H), ezx (x, E), ezy (y, E);
    // TM hzx (x, H), hzy (y, H), exy (y, E), eyx (x, E)
    const LensProfile *strip[2][4] = {{&g.ay.h, &g.ax.h, &g.ax.e, &g.ay.e}, {&g.ax.h, &g.ay.h, &g.ay.e, &g.ax.e}};
    for (int q = 0; q < 4; ++q)
        if (!lens_psi_ok(*strip[g.pol][q], g.psi[q])) return false;
    return true;
}

long inst_blocks(const LensInst2D &g, int by) {
    return (long)((g.ny + TW - 1) / TW) * ((g.nx + by * RB - 1) / (by * RB));
}

template <typename T>
void launch(const LensInst2D *dev, const int *blk, const int *owner, int ninst, int nblk, int by,
            const LensStepTable &tab, int n0, int nsteps, bool tm_dft, const LensInst2D *host, cudaStream_t s) {
    const dim3 b(BXB, by);
    for (int n = n0; n < n0 + nsteps; ++n) {
        b2d_h<T><<<nblk, b, 0, s>>>(dev, blk, owner);
        b2d_e<T><<<nblk, b, 0, s>>>(dev, blk, owner, tab, n);
        if (tm_dft) {
            bool any = false;
            for (int q = 0; q < ninst && !any; ++q)
                any = host[q].pol == 1 && host[q].dft && n - host[q].n_start >= host[q].dft_n0 &&
                      n - host[q].n_start < host[q].dft_n1;
            if (any) b2d_tm_node<T><<<nblk, b, 0, s>>>(dev, blk, owner, tab, n);
        }
    }
}

}  // namespace

extern "C" int lens_batch2d_plan(const LensInst2D *inst, int ninst, int by, int *blk, int *owner) {
    if (!inst || !blk || ninst < 1 || by < 1 || BXB * by > 256) return LENS_ERR_ARG;
    long tot = 0;
    for (int q = 0; q < ninst; ++q) {
        if (!inst_ok(inst[q])) return LENS_ERR_ARG;
        blk[q] = (int)tot;
        const long nb = inst_blocks(inst[q], by);
        if (tot + nb > 0x7fffffffL) return LENS_ERR_SIZE;
        if (owner)
            for (long b = 0; b < nb; ++b) owner[tot + b] = q;
        tot += nb;
    }
    blk[ninst] = (int)tot;
    return (int)tot;
}

extern "C" int lens_batch2d_step(const LensInst2D *inst_host, const LensInst2D *inst_dev, const int *blk_dev,
                                 const int *owner_dev, int ninst, int storage, int by, const LensStepTable *tab,
                                 int n0, int nsteps, void *stream) {
    if (!inst_host || !inst_dev || !blk_dev || !owner_dev || ninst < 1 || by < 1 || BXB * by > 256 || nsteps < 0)
        return LENS_ERR_ARG;
    long tot = 0;
    bool tm_dft = false, any_dft = false;
    for (int q = 0; q < ninst; ++q) {
        if (!inst_ok(inst_host[q]) || !lens_table_ok(tab, n0 - inst_host[q].n_start, nsteps)) return LENS_ERR_ARG;
        tot += inst_blocks(inst_host[q], by);
        tm_dft = tm_dft || (inst_host[q].pol == 1 && inst_host[q].dft);
        any_dft = any_dft || inst_host[q].dft;
    }
    if (tot > 0x7fffffffL) return LENS_ERR_SIZE;
    if (any_dft && !tab->pe) return LENS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nblk = (int)tot;
    switch (storage) {
        case LENS_F32:
            launch<float>(inst_dev, blk_dev, owner_dev, ninst, nblk, by, *tab, n0, nsteps, tm_dft, inst_host, s);
            break;
        case LENS_F16:
            launch<__half>(inst_dev, blk_dev, owner_dev, ninst, nblk, by, *tab, n0, nsteps, tm_dft, inst_host, s);
            break;
        case LENS_BF16:
            launch<__nv_bfloat16>(inst_dev, blk_dev, owner_dev, ninst, nblk, by, *tab, n0, nsteps, tm_dft,
                                  inst_host, s);
            break;
        default: return LENS_ERR_ARG;
    }
    return lens_cuda_status();
}

namespace {

// Batch steps on which a TM instance accumulates its node DFT: [lo, hi) (empty: lo = hi).
void tm_window(const LensInst2D *inst, int ninst, int &lo, int &hi) {
    lo = 1 << 30;
    hi = -(1 << 30);
    for (int q = 0; q < ninst; ++q) {
        const LensInst2D &g = inst[q];
        if (g.pol != 1 || !g.dft) continue;
        lo = std::min(lo, g.dft_n0 + g.n_start);
        hi = std::max(hi, g.dft_n1 + g.n_start);
    }
    if (hi < lo) lo = hi = 0;
}

template <typename T>
int run_persistent(const LensInst2D *dev, const int *blk, const int *owner, int nblk, int by, const LensStepTable &tab,
                   int n0, int nsteps, int tm_lo, int tm_hi, unsigned *sync, int *err, cudaStream_t s) {
    int dv = 0, nsm = 0, per = 0, coop = 0;
    if (cudaGetDevice(&dv) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dv) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dv) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pb2d<T>, BXB * by, 0) != cudaSuccess)
        return LENS_ERR_CUDA;
    if (!coop || per < 1) return LENS_ERR_CUDA;
    const int grid = std::min(nblk, per * nsm);
    if (cudaMemsetAsync(sync, 0, 2 * sizeof(unsigned), s) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess)
        return LENS_ERR_CUDA;
    LensStepTable t = tab;
    void *args[] = {(void *)&dev, (void *)&blk, (void *)&owner, (void *)&nblk, (void *)&t, (void *)&n0,
                    (void *)&nsteps, (void *)&tm_lo, (void *)&tm_hi, (void *)&sync, (void *)&err};
    if (cudaLaunchCooperativeKernel((const void *)pb2d<T>, dim3(grid), dim3(BXB, by), args, 0, s) != cudaSuccess)
        return LENS_ERR_CUDA;
    return LENS_OK;
}

}  // namespace

extern "C" int lens_batch2d_run(const LensInst2D *inst_host, const LensInst2D *inst_dev, const int *blk_dev,
                                const int *owner_dev, int ninst, int storage, int by, const LensStepTable *tab, int n0,
                                int nsteps, unsigned *sync, int *err, void *stream) {
    if (!inst_host || !inst_dev || !blk_dev || !owner_dev || !sync || !err || ninst < 1 || by < 1 ||
        BXB * by > 256 || nsteps < 0)
        return LENS_ERR_ARG;
    long tot = 0;
    bool any_dft = false;
    for (int q = 0; q < ninst; ++q) {
        if (!inst_ok(inst_host[q]) || !lens_table_ok(tab, n0 - inst_host[q].n_start, nsteps)) return LENS_ERR_ARG;
        tot += inst_blocks(inst_host[q], by);
        any_dft = any_dft || inst_host[q].dft;
    }
    if (tot > 0x7fffffffL) return LENS_ERR_SIZE;
    if (any_dft && !tab->pe) return LENS_ERR_ARG;
    if (nsteps == 0) return LENS_OK;
    int lo, hi;
    tm_window(inst_host, ninst, lo, hi);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int st;
    switch (storage) {
        case LENS_F32: st = run_persistent<float>(inst_dev, blk_dev, owner_dev, (int)tot, by, *tab, n0, nsteps, lo, hi, sync, err, s); break;
        case LENS_F16: st = run_persistent<__half>(inst_dev, blk_dev, owner_dev, (int)tot, by, *tab, n0, nsteps, lo, hi, sync, err, s); break;
        case LENS_BF16:
            st = run_persistent<__nv_bfloat16>(inst_dev, blk_dev, owner_dev, (int)tot, by, *tab, n0, nsteps, lo, hi, sync, err, s);
            break;
        default: return LENS_ERR_ARG;
    }
    if (st != LENS_OK) {
        cudaGetLastError();
        return st;
    }
    return lens_cuda_status();
}

// ------------------------------------------------------ allocation-free variant
// lens_batch2d_step needs device copies of the instance descriptors and of the
// block plan, which the caller allocates.  Callers that cannot allocate device
// memory at all (a host application whose allocator owns the GPU, code running
// under a fixed memory budget or inside a loop where cudaMalloc's implicit
// synchronisation is not allowed) use lens_batch2d_step_noalloc instead: the
// descriptors, the block offsets and the owner table live in one file-scope
// device array of fixed size, which every GPU that loads this library holds
// until the process exits.
namespace {

constexpr int NA_MAX_INST = 512;                 // instances per call
constexpr int NA_MAX_BLOCKS = 1 << 21;           // tiles per call (128 x 2*by nodes each)
constexpr size_t NA_DESC_BYTES = ((NA_MAX_INST * sizeof(LensInst2D) + 255) / 256) * 256;
constexpr size_t NA_BLK_BYTES = (((NA_MAX_INST + 1) * sizeof(int) + 255) / 256) * 256;
constexpr size_t NA_BYTES = NA_DESC_BYTES + NA_BLK_BYTES + (size_t)NA_MAX_BLOCKS * sizeof(int);

static __device__ __align__(256) unsigned char g_batch2d_scratch[NA_BYTES];

// Device address of the scratch array on the current device, looked up once per
// device (host code must not use the array's name as a device address).
constexpr int NA_MAX_DEV = 64;
std::atomic<unsigned char *> na_addr[NA_MAX_DEV];

int na_scratch(unsigned char **p) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return LENS_ERR_CUDA;
    if (dev < 0 || dev >= NA_MAX_DEV) return LENS_ERR_ARG;
    unsigned char *a = na_addr[dev].load();
    if (!a) {
        void *v = nullptr;
        if (cudaGetSymbolAddress(&v, g_batch2d_scratch) != cudaSuccess || !v) return LENS_ERR_CUDA;
        a = static_cast<unsigned char *>(v);
        na_addr[dev].store(a);
    }
    *p = a;
    return LENS_OK;
}

// owner[b] = instance of block b (binary search over the block offsets).
__global__ void na_owner(const int *blk, int ninst, int *owner, int nblk) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blk[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    owner[b] = lo;
}

}  // namespace

extern "C" int lens_batch2d_step_noalloc(const LensInst2D *inst, int ninst, int storage, int by,
                                         const LensStepTable *tab, int n0, int nsteps, void *stream) {
    if (!inst || ninst < 1 || by < 1 || BXB * by > 256 || nsteps < 0 ||
        (storage != LENS_F32 && storage != LENS_F16 && storage != LENS_BF16))
        return LENS_ERR_ARG;
    if (ninst > NA_MAX_INST) return LENS_ERR_SIZE;
    int blk[NA_MAX_INST + 1];
    long tot = 0;
    bool tm_dft = false, any_dft = false;
    for (int q = 0; q < ninst; ++q) {
        if (!inst_ok(inst[q]) || !lens_table_ok(tab, n0 - inst[q].n_start, nsteps)) return LENS_ERR_ARG;
        blk[q] = (int)tot;
        tot += inst_blocks(inst[q], by);
        if (tot > NA_MAX_BLOCKS) return LENS_ERR_SIZE;
        tm_dft = tm_dft || (inst[q].pol == 1 && inst[q].dft);
        any_dft = any_dft || inst[q].dft;
    }
    blk[ninst] = (int)tot;
    if (any_dft && !tab->pe) return LENS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the descriptors and block offsets are copied from host memory at call time;
    // a captured copy would re-read that memory at every replay, so a capturing
    // stream is refused before anything is enqueued
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return LENS_ERR_ARG;
    }
    if (cap != cudaStreamCaptureStatusNone) return LENS_ERR_ARG;
    unsigned char *base = nullptr;
    const int st = na_scratch(&base);
    if (st != LENS_OK) return st;
    LensInst2D *desc = reinterpret_cast<LensInst2D *>(base);
    int *blk_dev = reinterpret_cast<int *>(base + NA_DESC_BYTES);
    int *owner = reinterpret_cast<int *>(base + NA_DESC_BYTES + NA_BLK_BYTES);
    // every table is rewritten in full by each call (nothing carries over)
    if (cudaMemcpyAsync(desc, inst, ninst * sizeof(LensInst2D), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(blk_dev, blk, (ninst + 1) * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return LENS_ERR_CUDA;
    const int nblk = (int)tot;
    na_owner<<<(nblk + 255) / 256, 256, 0, s>>>(blk_dev, ninst, owner, nblk);
    switch (storage) {
        case LENS_F32: launch<float>(desc, blk_dev, owner, ninst, nblk, by, *tab, n0, nsteps, tm_dft, inst, s); break;
        case LENS_F16: launch<__half>(desc, blk_dev, owner, ninst, nblk, by, *tab, n0, nsteps, tm_dft, inst, s); break;
        default: launch<__nv_bfloat16>(desc, blk_dev, owner, ninst, nblk, by, *tab, n0, nsteps, tm_dft, inst, s);
    }
    return lens_cuda_status();
}
