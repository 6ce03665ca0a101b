// Temporally blocked 3D Yee CPML step for sm_100a: LENS_TB3_K = 2 time steps per
// launch with every per-step epilogue fused.
//
// Per cell the arithmetic is the fused single-step kernel's (fdtd3d.cu, after
// planar_3d/boundaries3d.py:311-362: H += Ch*(d1 - d2) with the strip
// corrections, E <- D*E, the curl and its strip corrections, PEC on the
// absorbing faces, then the Huygens source of fdtd3d_core.py:1116-1127).  What
// changes is how often a field crosses HBM: once per two steps.
//
// A CTA of 16 warps owns a tile of 12 rows (y) x 28 lanes (z) and streams an
// x-chunk; warp w holds row j0 - 2 + w, lane l holds z = k0 - 2 + l, so the two
// rows / lanes on each side are halo that neighbouring tiles own.  At plane
// iteration t the CTA loads plane t of the read buffer (level 0) and advances
// level 1 on plane t - 1 and level 2 on plane t - 2: level s reads level s-1 on
// planes i and i+1 and its own H on plane i-1, all in registers; z-neighbours
// come by warp shuffle and y-neighbours through shared-memory rows (the E rows
// of a level double-buffered by plane parity, so two barriers per plane
// suffice).  Level s is exact on planes [x0-2+s, x1+2-s), rows
// [j0-2+s, j0+14-s) and lanes [k0-2+s, k0+30-s) (clipped to the domain, whose
// faces are exact): level 2 is exact on the owned part, which is written to
// the other field buffer.
//
// CPML psi is per-cell state: level 1 of the twelve psi volumes goes to a
// scratch set on the cells where level 1 is exact (any other CTA that writes
// such a cell writes the same bits, and a CTA reads level 1 only where it wrote
// it itself); level 2 goes to the other psi buffer on the owned cells.
//
// Epilogues of both steps on the owned cells, from registers: detector box
// sums of Ex^2 + Ey^2 + Ez^2 (FP64, one atomic per warp and box per launch,
// fdtd3d_core.py:477-481), the volume DFTs (complex float32, :1150-1158), the
// convergence planes (compensated) and the flux planes (FP64, flux.py:28-41).
// There are no waits between CTAs and no pipeline barriers that could stall.
#include "lens_common.cuh"

namespace {

constexpr int K = LENS_TB3_K;   // time levels per launch
constexpr int NW = 16;          // warps of a CTA = rows of its tile
constexpr int RO = NW - 2 * K;  // owned rows
constexpr int ZO = 32 - 2 * K;  // owned lanes
constexpr unsigned FULL = 0xffffffffu;
static_assert(K == 2, "the kernel unrolls two levels");

struct T3 {
    int nx, ny, nz, P;
    const float *fi[6];          // read buffer: Ex Ey Ez Hx Hy Hz
    float *fo[6];                // write buffer
    const float *pin[LENS_NPSI]; // psi level 0
    float *plv[LENS_NPSI];       // psi level 1 (scratch)
    float *pout[LENS_NPSI];      // psi level 2
    const float *ce[3], *da[3];  // da[0] NULL: lossless
    float ch;
    LensAxis ax, ay, az;
    int pec[6];
    LensSource src;
    int src_comp;
    int *flag;
    const unsigned char *ctype;  // column form of the coefficients (LensGrid3D)
    const float *ctab;
    int ntz, nty, chunk;
};

struct V6 {
    float ex, ey, ez, hx, hy, hz;
};

__device__ __forceinline__ V6 zero6() { return V6{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}; }

__device__ __forceinline__ bool in_strip(const LensProfile &p, int m) {
    return m >= 0 && m < p.n && (m < p.lo || m >= p.n - p.hi);
}

__device__ __forceinline__ int box_end(int e, int ext) { return e < 0 ? ext + e : (e < ext ? e : ext); }

__device__ __forceinline__ bool in_box(const int *bx, int c, int i, int j, int k, int nx, int ny, int nz) {
    return i >= bx[0] && i < box_end(bx[1], nx - (c == 0)) && j >= bx[2] && j < box_end(bx[3], ny - (c == 1)) &&
           k >= bx[4] && k < box_end(bx[5], nz - (c == 2));
}

// Lane-constant facts of a cell (j, k) of the tile.
struct Cell {
    int j, k;
    bool in;                     // inside the domain
    bool hx, hyk, hzj;           // Hx exists; Hy, Hz exist apart from the x condition
    bool exu, eyu, ezu;          // curl terms apply (apart from the x condition)
    bool eyv, ezv;               // Ey, Ez exist
    bool pj, pk;                 // on a PEC face in y / z
    bool zh, yh, ze, ye;         // in a z / y psi strip (H / E profiles)
    bool own;                    // owned (j, k)
    bool ex1;                    // exact (j, k) at level 1
};

// psi = b*old + c*d with old from level s-1; level s stored where `wr`; returns psi + km*d.
template <int S>
__device__ __forceinline__ float psi3(const T3 &g, int q, const LensProfile &pf, int m, size_t o, float d, bool wr) {
    const float old = S == 1 ? __ldg(g.pin[q] + o) : g.plv[q][o];
    const float p = __ldg(pf.b + m) * old + __ldg(pf.c + m) * d;
    if (wr) {
        if (S == 1) g.plv[q][o] = p;
        else g.pout[q][o] = p;
    }
    return p + (__ldg(pf.ik + m) - 1.0f) * d;
}

// Coefficients of cell (i, j, k): ce_x, ce_y, ce_z, D_x, D_y, D_z.
__device__ __forceinline__ void coef6(const T3 &g, int i, const Cell &c, size_t o, float *cf) {
    const bool lossy = g.da[0] != nullptr;
    unsigned t = 255u;
    if (g.ctype) t = __ldg(g.ctype + (size_t)i * g.P + c.k);
    if (t != 255u) {
        const float *tb = g.ctab + (size_t)t * 6 * g.ny + c.j;
#pragma unroll
        for (int q = 0; q < 3; ++q) cf[q] = __ldg(tb + (size_t)q * g.ny);
#pragma unroll
        for (int q = 3; q < 6; ++q) cf[q] = lossy ? __ldg(tb + (size_t)q * g.ny) : 1.f;
    } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) cf[q] = __ldg(g.ce[q] + o);
#pragma unroll
        for (int q = 3; q < 6; ++q) cf[q] = lossy ? __ldg(g.da[q - 3] + o) : 1.f;
    }
}

// Shared rows: E exchange per level (Ez, Ex of row w for row w-1's H), H exchange
// (Hz, Hx of row w for row w+1's E).
struct Smem {
    float e[K][2][2][NW][32];    // level s-1 (0 loaded, 1 computed), plane parity, {Ez, Ex}
    float h[K][2][NW][32];       // level s: {Hz, Hx}
};

struct Epi {
    double box[LENS_MAX_BOX];
};

// One level: H then E on plane i (uniform), from P = level s-1 on plane i,
// C = level s-1 on plane i+1, Hp = level s on plane i-1.  Returns level s on plane i.
template <int S>
__device__ __forceinline__ V6 level(const T3 &g, const LensStepTable &tab, const LensEpi3D &ep, int n, int i,
                                    int x0, int x1, const Cell &c, const V6 &P, const V6 &C, const V6 &Hp,
                                    const float (*se)[NW][32], float (*sh)[NW][32], int w, int lane, Epi &acc) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool iin_dom = i >= 0 && i < nx;
    const bool iok = i < nx - 1;
    // neighbours of level s-1: k+1 by shuffle, j+1 from the shared row above
    const float eyk = __shfl_down_sync(FULL, P.ey, 1), exk = __shfl_down_sync(FULL, P.ex, 1);
    const int wu = w + 1 < NW ? w + 1 : w, wd = w > 0 ? w - 1 : 0;
    const float ezj = se[0][wu][lane], exj = se[1][wu][lane];
    const size_t o = ((size_t)(iin_dom ? i : 0) * ny + (c.in ? c.j : 0)) * g.P + (c.in ? c.k : 0);
    const bool live = iin_dom && c.in;
    // exactness of this cell at this level (psi stores)
    const bool xex = i >= max(0, x0 - K + S) && i < min(nx, x1 + K - S);
    const bool own = c.own && i >= x0 && i < x1;
    const bool wr = S == K ? own : (xex && c.ex1);
    V6 N = P;
    const float ch = g.ch;
    if (live) {
        const float d1x = eyk - P.ey, d2x = ezj - P.ez;
        const float d1y = C.ez - P.ez, d2y = exk - P.ex;
        const float d1z = exj - P.ex, d2z = C.ey - P.ey;
        if (c.hx) {
            float v = P.hx + ch * (d1x - d2x);
            if (c.zh) v = v + ch * psi3<S>(g, LENS_PSI_HX_Z, g.az.h, c.k, o, d1x, wr);
            if (c.yh) v = v + (-ch) * psi3<S>(g, LENS_PSI_HX_Y, g.ay.h, c.j, o, d2x, wr);
            N.hx = v;
        }
        const bool xh = iok && in_strip(g.ax.h, i);
        if (iok && c.hyk) {
            float v = P.hy + ch * (d1y - d2y);
            if (xh) v = v + ch * psi3<S>(g, LENS_PSI_HY_X, g.ax.h, i, o, d1y, wr);
            if (c.zh) v = v + (-ch) * psi3<S>(g, LENS_PSI_HY_Z, g.az.h, c.k, o, d2y, wr);
            N.hy = v;
        }
        if (iok && c.hzj) {
            float v = P.hz + ch * (d1z - d2z);
            if (c.yh) v = v + ch * psi3<S>(g, LENS_PSI_HZ_Y, g.ay.h, c.j, o, d1z, wr);
            if (xh) v = v + (-ch) * psi3<S>(g, LENS_PSI_HZ_X, g.ax.h, i, o, d2z, wr);
            N.hz = v;
        }
    }
    sh[0][w][lane] = N.hz;
    sh[1][w][lane] = N.hx;
    __syncthreads();
    // neighbours of the new H: k-1 by shuffle, j-1 from the shared row below
    const float hyk = __shfl_up_sync(FULL, N.hy, 1), hxk = __shfl_up_sync(FULL, N.hx, 1);
    const float hzj = sh[0][wd][lane], hxj = sh[1][wd][lane];
    if (live) {
        float cf[6];
        coef6(g, i, c, o, cf);
        const bool iin = i >= 1 && i <= nx - 2;
        const bool pec_i = (g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1);
        const bool xe = in_strip(g.ax.e, i);
        const float d1x = N.hz - hzj, d2x = N.hy - hyk;
        const float d1y = N.hx - hxk, d2y = N.hz - Hp.hz;
        const float d1z = N.hy - Hp.hy, d2z = N.hx - hxj;
        float vx = P.ex * cf[3], vy = P.ey * cf[4], vz = P.ez * cf[5];
        if (iok && c.exu) {
            vx = vx + cf[0] * (d1x - d2x);
            if (c.ye) vx = vx + cf[0] * psi3<S>(g, LENS_PSI_EX_Y, g.ay.e, c.j, o, d1x, wr);
            if (c.ze) vx = vx + (-cf[0]) * psi3<S>(g, LENS_PSI_EX_Z, g.az.e, c.k, o, d2x, wr);
        }
        if (iin && c.eyu) {
            vy = vy + cf[1] * (d1y - d2y);
            if (c.ze) vy = vy + cf[1] * psi3<S>(g, LENS_PSI_EY_Z, g.az.e, c.k, o, d1y, wr);
            if (xe) vy = vy + (-cf[1]) * psi3<S>(g, LENS_PSI_EY_X, g.ax.e, i, o, d2y, wr);
        }
        if (iin && c.ezu) {
            vz = vz + cf[2] * (d1z - d2z);
            if (xe) vz = vz + cf[2] * psi3<S>(g, LENS_PSI_EZ_X, g.ax.e, i, o, d1z, wr);
            if (c.ye) vz = vz + (-cf[2]) * psi3<S>(g, LENS_PSI_EZ_Y, g.ay.e, c.j, o, d2z, wr);
        }
        if (!iok || c.pj || c.pk) vx = 0.f;
        if (!c.eyv || pec_i || c.pk) vy = 0.f;
        if (!c.ezv || pec_i || c.pj) vz = 0.f;
        const LensSource &s = g.src;
        if (s.ix >= 0 && (i == s.ix || i == s.ix + 1) && c.j < s.nj && c.k < s.nk) {
            const int q = n - tab.t0;
            const size_t m = (size_t)c.j * s.pitch_k + c.k;
            const float sv = i == s.ix ? (__ldg(tab.env + q) * sinf(__ldg(tab.wt + q) + __ldg(s.ph1 + m))) * __ldg(s.amp + m)
                                       : -((__ldg(tab.env + q) * sinf(__ldg(tab.wt + q) + __ldg(s.ph2 + m))) * __ldg(s.amp + m));
            if (g.src_comp == 0) vx += sv;
            else if (g.src_comp == 1) vy += sv;
            else vz += sv;
        }
        N.ex = vx;
        N.ey = vy;
        N.ez = vz;
        // ---- epilogue of step n on the owned cells
        if (own) {
            const bool vxv = iok, vyv = c.eyv, vzv = c.ezv;
#pragma unroll
            for (int b = 0; b < LENS_MAX_BOX; ++b) {
                if (b >= ep.nbox) break;
                const int *bx = ep.box[b];
                double v = 0.0;
                if (vxv && in_box(bx, 0, i, c.j, c.k, nx, ny, nz)) v += (double)(vx * vx);
                if (vyv && in_box(bx, 1, i, c.j, c.k, nx, ny, nz)) v += (double)(vy * vy);
                if (vzv && in_box(bx, 2, i, c.j, c.k, nx, ny, nz)) v += (double)(vz * vz);
                acc.box[b] += v;
            }
            const bool win = n >= ep.dft_n0 && n < ep.dft_n1;
            const bool prevw = ep.conv_prev && n >= ep.prev_n0 && n < ep.prev_n1;
            if (win || prevw) {
                const int q = n - tab.t0;
                const float pr = __ldg(tab.pe + 2 * q), pim = __ldg(tab.pe + 2 * q + 1);
                const float f = g.src_comp == 1 ? vy : (g.src_comp == 2 ? vz : vx);
                const bool vf = g.src_comp == 1 ? vyv : (g.src_comp == 2 ? vzv : vxv);
                if (prevw && vf && c.k == ep.conv_k && c.j < g.src.nj)
                    kahan_add(reinterpret_cast<float4 *>(ep.conv_prev) + (size_t)i * g.src.nj + c.j, f * pr, f * pim);
                if (win) {
                    const float v3[3] = {vx, vy, vz};
                    const bool ok3[3] = {vxv, vyv, vzv};
#pragma unroll
                    for (int q3 = 0; q3 < 3; ++q3) {
                        if (ep.dft[q3] && ok3[q3]) {
                            float2 *a = reinterpret_cast<float2 *>(ep.dft[q3]) + o;
                            float2 sacc = *a;
                            sacc.x += v3[q3] * pr;
                            sacc.y += v3[q3] * pim;
                            *a = sacc;
                        }
                    }
                    if (ep.conv_last && vf && c.k == ep.conv_k && c.j < g.src.nj)
                        kahan_add(reinterpret_cast<float4 *>(ep.conv_last) + (size_t)i * g.src.nj + c.j, f * pr, f * pim);
                    for (int p = 0; p < ep.nplane; ++p) {
                        if (i != ep.plane[p]) continue;
                        const size_t vol = (size_t)ny * g.P, jk = (size_t)c.j * g.P + c.k;
                        const float qr = __ldg(tab.ph + 2 * q), qi = __ldg(tab.ph + 2 * q + 1);
                        if (vyv) {
                            double *a = ep.plane_acc + ((size_t)(p * 2 + 0) * 4) * vol + jk;
                            const float h = 0.5f * (Hp.hz + N.hz);
                            a[0] += (double)vy * (double)pr;
                            a[vol] += (double)vy * (double)pim;
                            a[2 * vol] += (double)h * (double)qr;
                            a[3 * vol] += (double)h * (double)qi;
                        }
                        if (vzv) {
                            double *a = ep.plane_acc + ((size_t)(p * 2 + 1) * 4) * vol + jk;
                            const float h = 0.5f * (Hp.hy + N.hy);
                            a[0] += (double)vz * (double)pr;
                            a[vol] += (double)vz * (double)pim;
                            a[2 * vol] += (double)h * (double)qr;
                            a[3 * vol] += (double)h * (double)qi;
                        }
                    }
                }
            }
        }
    }
    return N;
}

__device__ __forceinline__ V6 load6(const T3 &g, int t, const Cell &c) {
    if (t < 0 || t >= g.nx || !c.in) return zero6();
    const size_t o = ((size_t)t * g.ny + c.j) * g.P + c.k;
    return V6{__ldg(g.fi[0] + o), __ldg(g.fi[1] + o), __ldg(g.fi[2] + o),
              __ldg(g.fi[3] + o), __ldg(g.fi[4] + o), __ldg(g.fi[5] + o)};
}

__global__ void __launch_bounds__(NW * 32, 1)
    tb3d(const __grid_constant__ T3 g, const LensStepTable tab, const __grid_constant__ LensEpi3D ep, int n0) {
    __shared__ Smem sm;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tz = blockIdx.x % g.ntz, ty = (blockIdx.x / g.ntz) % g.nty, cx = blockIdx.x / (g.ntz * g.nty);
    const int j0 = ty * RO, k0 = tz * ZO;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int x0 = cx * g.chunk, x1 = min(nx, x0 + g.chunk);
    Cell c;
    c.j = j0 - K + w;
    c.k = k0 - K + lane;
    c.in = c.j >= 0 && c.j < ny && c.k >= 0 && c.k < nz;
    const bool jin = c.j >= 1 && c.j <= ny - 2, kin = c.k >= 1 && c.k <= nz - 2;
    c.hx = c.in && c.j < ny - 1 && c.k < nz - 1;
    c.hyk = c.in && c.k < nz - 1;
    c.hzj = c.in && c.j < ny - 1;
    c.exu = c.in && jin && kin;
    c.eyu = c.in && kin && c.j < ny - 1;
    c.ezu = c.in && jin && c.k < nz - 1;
    c.eyv = c.in && c.j < ny - 1;
    c.ezv = c.in && c.k < nz - 1;
    c.pj = (g.pec[2] && c.j == 0) || (g.pec[3] && c.j == ny - 1);
    c.pk = (g.pec[4] && c.k == 0) || (g.pec[5] && c.k == nz - 1);
    c.zh = c.in && in_strip(g.az.h, c.k);
    c.yh = c.in && in_strip(g.ay.h, c.j);
    c.ze = c.in && in_strip(g.az.e, c.k);
    c.ye = c.in && in_strip(g.ay.e, c.j);
    c.own = c.in && c.j >= j0 && c.j < j0 + RO && c.k >= k0 && c.k < k0 + ZO;
    c.ex1 = c.in && c.j >= max(0, j0 - K + 1) && c.j < min(ny, j0 + RO + K - 1) && c.k >= max(0, k0 - K + 1) &&
            c.k < min(nz, k0 + ZO + K - 1);
    Epi acc;
#pragma unroll
    for (int b = 0; b < LENS_MAX_BOX; ++b) acc.box[b] = 0.0;
    V6 L0 = zero6(), L1 = zero6(), H2 = zero6();  // level 0 on plane t-1, level 1 on t-2, level 2 H on t-3
    const int t0 = x0 - K, t1 = x1 + K;
    V6 nxt = load6(g, t0, c);
    for (int t = t0; t < t1; ++t) {
        const V6 cur = nxt;
        if (t + 1 < t1) nxt = load6(g, t + 1, c);
        const int par = t & 1;
        // level 0 of plane t: its E rows for level 1 at the next plane
        sm.e[0][par ^ 1][0][w][lane] = cur.ez;
        sm.e[0][par ^ 1][1][w][lane] = cur.ex;
        // level 1 on plane t - 1
        const V6 E1 = level<1>(g, tab, ep, n0, t - 1, x0, x1, c, L0, cur, L1, sm.e[0][par], sm.h[0], w, lane, acc);
        sm.e[1][par ^ 1][0][w][lane] = E1.ez;
        sm.e[1][par ^ 1][1][w][lane] = E1.ex;
        // level 2 on plane t - 2
        const V6 E2 = level<2>(g, tab, ep, n0 + 1, t - 2, x0, x1, c, L1, E1, H2, sm.e[1][par], sm.h[1], w, lane, acc);
        const int i2 = t - 2;
        if (c.own && i2 >= x0 && i2 < x1) {
            const size_t o = ((size_t)i2 * ny + c.j) * g.P + c.k;
            g.fo[0][o] = E2.ex; g.fo[1][o] = E2.ey; g.fo[2][o] = E2.ez;
            g.fo[3][o] = E2.hx; g.fo[4][o] = E2.hy; g.fo[5][o] = E2.hz;
        }
        L0 = cur;
        L1 = E1;
        H2 = E2;
    }
    // detector boxes: one FP64 atomic per warp and box; a non-finite sum marks the solve
#pragma unroll
    for (int b = 0; b < LENS_MAX_BOX; ++b) {
        if (b >= ep.nbox) break;
        const double v = warp_sum(acc.box[b]);
        if (lane == 0) {
            if (v != 0.0) atomicAdd(ep.box_acc + b, v);
            if (g.flag && !isfinite(v)) atomicOr(g.flag, 2);
        }
    }
}

}  // namespace

// Host side (in fdtd3d.cu's translation unit the grid checks live; this file
// repeats the few it needs).
namespace {

bool tb3_grid_ok(const LensGrid3D *g) {
    if (!g || g->nx < 3 || g->ny < 3 || g->nz < 3 || g->pitch < g->nz || (g->pitch % 32)) return false;
    if (g->cur != 0 && g->cur != 1) return false;
    for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 6; ++c)
            if (!g->f[b][c]) return false;
    if (!g->ce_x || !g->ce_y || !g->ce_z) return false;
    if ((!g->da_x) != (!g->da_y) || (!g->da_y) != (!g->da_z)) return false;
    const LensAxis *a[3] = {&g->ax, &g->ay, &g->az};
    const int n[3] = {g->nx, g->ny, g->nz};
    for (int q = 0; q < 3; ++q)
        if (!lens_profile_ok(a[q]->e, n[q]) || !lens_profile_ok(a[q]->h, n[q] - 1)) return false;
    if (g->ctype && (!g->ctab || g->ntype < 1 || g->ntype > LENS_MAX_CTYPE)) return false;
    if (g->src.ix >= 0) {
        if (!g->src.amp || !g->src.ph1 || !g->src.ph2 || g->src.ix + 1 >= g->nx) return false;
        if (g->src_comp < 0 || g->src_comp > 2 || g->src.pitch_k < g->src.nk || g->src.nj < 0 || g->src.nk < 0)
            return false;
    }
    return true;
}

}  // namespace

extern "C" int lens_fdtd3d_step_tb(LensGrid3D *g, const LensTB3D *tb, const LensStepTable *tab, const LensEpi3D *ep,
                                   int n0, int nsteps, void *stream) {
    if (!tb3_grid_ok(g) || !tb || tb->chunk < 1 || nsteps < 0 || nsteps % K || !lens_table_ok(tab, n0, nsteps))
        return LENS_ERR_ARG;
    for (int q = 0; q < LENS_NPSI; ++q)
        if (!g->psi[0][q] || !g->psi[1][q] || !tb->psi_lv[q]) return LENS_ERR_ARG;
    LensEpi3D e{};
    if (ep) e = *ep;
    if (e.nbox < 0 || e.nbox > LENS_MAX_BOX || (e.nbox > 0 && !e.box_acc)) return LENS_ERR_ARG;
    if (e.nplane < 0 || e.nplane > LENS_MAX_PLANE || (e.nplane > 0 && !e.plane_acc)) return LENS_ERR_ARG;
    for (int p = 0; p < e.nplane; ++p)
        if (e.plane[p] < 1 || e.plane[p] > g->nx - 2) return LENS_ERR_ARG;
    const bool dft = e.dft[0] || e.dft[1] || e.dft[2] || e.nplane > 0 || e.conv_prev || e.conv_last;
    if (dft && (!tab->pe || !tab->ph)) return LENS_ERR_ARG;
    if ((e.conv_prev || e.conv_last) && g->src.nj < 1) return LENS_ERR_ARG;
    T3 k{};
    k.nx = g->nx; k.ny = g->ny; k.nz = g->nz; k.P = g->pitch;
    k.ce[0] = g->ce_x; k.ce[1] = g->ce_y; k.ce[2] = g->ce_z;
    k.da[0] = g->da_x; k.da[1] = g->da_y; k.da[2] = g->da_z;
    k.ch = g->ch;
    k.ax = g->ax; k.ay = g->ay; k.az = g->az;
    for (int q = 0; q < 6; ++q) k.pec[q] = g->pec[q];
    k.src = g->src;
    k.src_comp = g->src_comp;
    k.flag = g->flag;
    k.ctype = g->ctype;
    k.ctab = g->ctab;
    k.ntz = (g->nz + ZO - 1) / ZO;
    k.nty = (g->ny + RO - 1) / RO;
    k.chunk = tb->chunk;
    const int nch = (g->nx + tb->chunk - 1) / tb->chunk;
    const long nblk = (long)k.ntz * k.nty * nch;
    if (nblk > 0x7fffffffL) return LENS_ERR_SIZE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int m = 0; m < nsteps / K; ++m) {
        const int rb = g->cur;
        for (int q = 0; q < 6; ++q) {
            k.fi[q] = g->f[rb][q];
            k.fo[q] = g->f[1 - rb][q];
        }
        for (int q = 0; q < LENS_NPSI; ++q) {
            k.pin[q] = g->psi[rb][q];
            k.plv[q] = tb->psi_lv[q];
            k.pout[q] = g->psi[1 - rb][q];
        }
        tb3d<<<(unsigned)nblk, NW * 32, 0, s>>>(k, *tab, e, n0 + m * K);
        g->cur = 1 - rb;
    }
    return lens_cuda_status();
}
