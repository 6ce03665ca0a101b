// Temporally blocked 2D TE/TM steps for sm_100a: LENS_TB_K = 4 time steps per
// launch, for one grid or a batch of uneven grids.
//
// Per cell the arithmetic is the single-step kernels' (fdtd2d_batch.cu, after
// planar_beads/boundaries.py:164-274, the source of vcsel.py:151-156 and the
// loss damping of fdtd2d_core.py:796-797); what changes is how often a field
// crosses HBM: once per K steps instead of once per step.
//
// Work unit = one warp = a tile of 128 columns (y, contiguous; 4 per lane) by a
// chunk of rows (x).  The warp streams its rows: at iteration t it loads row t
// of the fields (level 0) and advances level s = 1..K on row t - s, so level s
// reads level s-1 on rows t-s and t-s+1 and its own previous row t-s-1; every
// level is one row of registers (4 columns x 3 fields per lane).  Neighbouring
// columns come by warp shuffle.  The result after K steps is exact on the
// tile's owned part: rows [x0, x1) and the inner 128 - 2K columns; the K
// columns on each side and the K rows before and after the chunk are halo,
// recomputed by the neighbouring units (an exact domain face needs no halo).
// At level s a warp's values are exact on rows [x0-K+s, x1+K-s) and columns
// [c0-K+s, c0+128-K-s) (clipped to the domain).
//
// Fields are double-buffered across launches (a launch reads one buffer and
// writes the owned cells of the other), so a unit's halo reads never see a
// neighbour's new values.  CPML psi, which is per-cell state like the fields,
// keeps levels 1..K-1 in a scratch array: a warp writes psi level s only where
// its level-s values are exact, where any other warp that writes the same cell
// writes the same bits, and it reads level s-1 only where it wrote it itself;
// level K goes to the other psi buffer on the owned cells.
//
// Epilogue: the node-field DFT over the instance's window (TE Ez, TM Ey on the
// nodes, fdtd2d_core.py:458-465, 838-847), accumulated on the owned cells only,
// plain (re, im) or compensated (re, im, c_re, c_im).
#include "lens_common.cuh"
#include "lens_store.cuh"

namespace {

constexpr int K = LENS_TB_K;        // time steps per launch
constexpr int TV = 4;               // columns per lane
constexpr int TC = 32 * TV;         // columns of a warp tile
constexpr int TO = TC - 2 * K;      // owned columns of a warp tile
constexpr int TW = 4;               // warps per block
constexpr unsigned FULL = 0xffffffffu;
static_assert(K % TV == 0, "the halo must be whole lanes so every vector access stays 16-byte aligned");

struct F3 {
    float a[TV], b[TV], c[TV];  // TE Ez, Hx, Hy; TM Ex, Ey, Hz
};

__device__ __forceinline__ void zero3(F3 &f) {
#pragma unroll
    for (int c = 0; c < TV; ++c) f.a[c] = f.b[c] = f.c[c] = 0.f;
}

template <typename T>
__device__ __forceinline__ void load3(F3 &f, void *const *p, int t, int j0, int nx, int P) {
    if (t >= 0 && t < nx && j0 >= 0 && j0 < P) {
        using S = St<T>;
        const size_t o = (size_t)t * P + j0;
        f4_to(S::ld4(p[0], o), f.a);
        f4_to(S::ld4(p[1], o), f.b);
        f4_to(S::ld4(p[2], o), f.c);
    } else {
        zero3(f);
    }
}

__device__ __forceinline__ unsigned long long ldu64(const void *p) {
    return __ldg(reinterpret_cast<const unsigned long long *>(p));
}

// Everything a warp needs about its unit, read once.
struct Unit {
    const LensInst2D *g;
    int pol, nx, ny, P, nst;
    int x0, x1, c0, cA;      // owned rows [x0, x1), owned columns [c0, c0 + TO), first tile column
    int j0;                  // this lane's first column
    void *fi[3], *fo[3];     // fields read / written by this launch
    const float *pin[4];     // psi level 0
    float *pout[4];          // psi level K
    float *lv;               // psi levels 1..K-1
    size_t lvoff[4], lvtot;  // offset of psi q inside one level, floats per level
    int wid[4];              // strip widths of the four psi arrays
    bool kahan;
    float *dft;
    int dft_n0, dft_n1;
};

// Strip width and size of psi q: TE hxy (y, H), hyx (x, H), ezx (x, E), ezy (y, E);
// TM hzx (x, H), hzy (y, H), exy (y, E), eyx (x, E).  x arrays are (w, P), y arrays (nx, w).
__device__ __forceinline__ bool psi_is_x(int pol, int q) { return pol == 0 ? (q == 1 || q == 2) : (q == 0 || q == 3); }

__device__ __forceinline__ const LensProfile &psi_prof(const LensInst2D *g, int pol, int q) {
    // the profile whose strip psi q serves
    if (pol == 0) return q == 0 ? g->ay.h : q == 1 ? g->ax.h : q == 2 ? g->ax.e : g->ay.e;
    return q == 0 ? g->ax.h : q == 1 ? g->ay.h : q == 2 ? g->ay.e : g->ax.e;
}

// psi update of level s at (row r, column j): read level s-1, write level s where
// `wr` (exact cells; owned cells at level K).  m: profile entry, sidx: strip index.
template <int S>
__device__ __forceinline__ float psi_lv(const Unit &u, int q, const LensProfile &pf, int m, int sidx, int r, int j,
                                        float d, bool wr) {
    const bool xs = psi_is_x(u.pol, q);
    const size_t idx = xs ? (size_t)sidx * u.P + j : (size_t)r * u.wid[q] + sidx;
    float old;
    if (S == 1) old = __ldg(u.pin[q] + idx);
    else old = u.lv[(size_t)(S - 2) * u.lvtot + u.lvoff[q] + idx];
    const float p = __ldg(pf.b + m) * old + __ldg(pf.c + m) * d;
    if (wr) {
        if (S == K) u.pout[q][idx] = p;
        else u.lv[(size_t)(S - 1) * u.lvtot + u.lvoff[q] + idx] = p;
    }
    return p;
}

__device__ __forceinline__ const float *crow(const LensInst2D *g, int q, int ncoef, int i, int j0, int P) {
    const unsigned char *rt = reinterpret_cast<const unsigned char *>(ldu64(&g->rtype));
    const unsigned t = rt ? __ldg(rt + i) : 255u;
    if (t == 255u) return reinterpret_cast<const float *>(ldu64(&g->c[q])) + (size_t)i * P + j0;
    const float *tab = reinterpret_cast<const float *>(ldu64(&g->ctab));
    return tab + ((size_t)t * ncoef + q) * (size_t)P + j0;
}

__device__ __forceinline__ float src_term(const LensInst2D *g, const LensStepTable &tab, int step, int r, int j) {
    const int k = step - tab.t0;
    const float *amp = reinterpret_cast<const float *>(ldu64(&g->src.amp));
    if (r == __ldg(&g->src.ix)) {
        const float *ph1 = reinterpret_cast<const float *>(ldu64(&g->src.ph1));
        return (__ldg(tab.env + k) * sinf(__ldg(tab.wt + k) + __ldg(ph1 + j))) * __ldg(amp + j);
    }
    const float *ph2 = reinterpret_cast<const float *>(ldu64(&g->src.ph2));
    return -((__ldg(tab.env + k) * sinf(__ldg(tab.wt + k) + __ldg(ph2 + j))) * __ldg(amp + j));
}

// DFT of the node value v at (r, j) for the instance's own step `step`.
__device__ __forceinline__ void dft_add(const Unit &u, const LensStepTable &tab, int step, int r, int j, float v) {
    const int k = step - tab.t0;
    const float pr = __ldg(tab.pe + 2 * k), pim = __ldg(tab.pe + 2 * k + 1);
    const size_t o = (size_t)r * u.P + j;
    if (u.kahan) {
        kahan_add(reinterpret_cast<float4 *>(u.dft) + o, v * pr, v * pim);
    } else {
        float2 *a = reinterpret_cast<float2 *>(u.dft) + o;
        float2 s = *a;
        s.x += v * pr;
        s.y += v * pim;
        *a = s;
    }
}

// Exactness of level s on row r / column j (see the header).
template <int S>
__device__ __forceinline__ bool row_exact(const Unit &u, int r) {
    return r >= max(0, u.x0 - K + S) && r < min(u.nx, u.x1 + K - S);
}
template <int S>
__device__ __forceinline__ bool col_exact(const Unit &u, int j) {
    return j >= max(0, u.cA + S) && j < min(u.ny, u.cA + TC - S);
}
__device__ __forceinline__ bool owned(const Unit &u, int r, int j) {
    return r >= u.x0 && r < u.x1 && j >= u.c0 && j < u.c0 + TO && j < u.ny;
}

// ------------------------------------------------------------------------ TE
// Level S on row r: P = level S-1 on row r, C = level S-1 on row r+1, Q = level S
// on row r-1; N = level S on row r.
template <int S>
__device__ __forceinline__ void te_level(const Unit &u, const LensStepTable &tab, int step, int r, const F3 &P,
                                         const F3 &C, const F3 &Q, F3 &N, const float *kyh, const float *kye) {
    const LensInst2D *g = u.g;
    const int nx = u.nx, ny = u.ny, j0 = u.j0;
    const float enext = __shfl_down_sync(FULL, P.a[0], 1);  // Ez(r, j0 + 4)
    if (r < 0 || r >= nx) {  // uniform over the warp (one row per level)
        zero3(N);
        return;
    }
    const float ch = __ldg(&g->ch);
    const LensProfile &xh = g->ax.h, &xe = g->ax.e, &yh = g->ay.h, &ye = g->ay.e;
    const bool rex = row_exact<S>(u, r);
    // ---- H (boundaries.py:186-194)
    const int sxh = r < nx - 1 ? strip_of(r, xh.lo, xh.hi, xh.n) : -1;
    const float kxh = r < nx - 1 ? __ldg(xh.ik + r) : 0.f;
#pragma unroll
    for (int c = 0; c < TV; ++c) {
        const int j = j0 + c;
        float hx = P.b[c], hy = P.c[c];
        if (j >= 0 && j < ny - 1) {
            const float d = (c + 1 < TV ? P.a[c + 1] : enext) - P.a[c];
            float p = 0.f;
            const int sj = strip_of(j, yh.lo, yh.hi, yh.n);
            if (sj >= 0) p = psi_lv<S>(u, 0, yh, j, sj, r, j, d, S == K ? owned(u, r, j) : (rex && col_exact<S>(u, j)));
            hx = P.b[c] - ch * (d * kyh[c] + p);
        }
        if (r < nx - 1 && j >= 0 && j < ny) {
            const float d = C.a[c] - P.a[c];
            float p = 0.f;
            if (sxh >= 0) p = psi_lv<S>(u, 1, xh, r, sxh, r, j, d, S == K ? owned(u, r, j) : (rex && col_exact<S>(u, j)));
            hy = P.c[c] + ch * (d * kxh + p);
        }
        N.b[c] = hx;
        N.c[c] = hy;
    }
    // ---- E (boundaries.py:196-215), source, PEC
    const float hxm = __shfl_up_sync(FULL, N.b[TV - 1], 1);  // Hx(r, j0 - 1)
    const bool rin = r >= 1 && r <= nx - 2;
    const int sxe = rin ? strip_of(r, xe.lo, xe.hi, xe.n) : -1;
    const float kxe = __ldg(xe.ik + r);
    const int six = __ldg(&g->src.ix), snj = __ldg(&g->src.nj);
    const bool srow = six >= 0 && (r == six || r == six + 1);
    const int pec0 = __ldg(g->pec), pec1 = __ldg(g->pec + 1), pec2 = __ldg(g->pec + 2), pec3 = __ldg(g->pec + 3);
    float c0[TV], c1[TV];
    if (j0 >= 0 && j0 < u.P) {
        f4_to(__ldg(reinterpret_cast<const float4 *>(crow(g, 0, 2, r, j0, u.P))), c0);
        f4_to(__ldg(reinterpret_cast<const float4 *>(crow(g, 1, 2, r, j0, u.P))), c1);
    } else {
#pragma unroll
        for (int c = 0; c < TV; ++c) c0[c] = c1[c] = 0.f;
    }
#pragma unroll
    for (int c = 0; c < TV; ++c) {
        const int j = j0 + c;
        float v = P.a[c];
        if (rin && j >= 1 && j <= ny - 2) {
            const float dhy = N.c[c] - Q.c[c], dhx = N.b[c] - (c > 0 ? N.b[c - 1] : hxm);
            float qx = 0.f, qy = 0.f;
            const bool wr = S == K ? owned(u, r, j) : (rex && col_exact<S>(u, j));
            const int sj = strip_of(j, ye.lo, ye.hi, ye.n);
            if (sxe >= 0) qx = psi_lv<S>(u, 2, xe, r, sxe, r, j, dhy, wr);
            if (sj >= 0) qy = psi_lv<S>(u, 3, ye, j, sj, r, j, dhx, wr);
            v = c0[c] * v + c1[c] * (dhy * kxe + qx - dhx * kye[c] - qy);
        }
        if (srow && j >= 0 && j < snj) v += src_term(g, tab, step, r, j);
        if ((pec0 && r == 0) || (pec1 && r == nx - 1) || (pec2 && j == 0) || (pec3 && j == ny - 1)) v = 0.f;
        if (j < 0 || j >= ny) v = 0.f;
        N.a[c] = v;
    }
    if (u.dft && step >= u.dft_n0 && step < u.dft_n1 && r >= u.x0 && r < u.x1) {
#pragma unroll
        for (int c = 0; c < TV; ++c)
            if (owned(u, r, j0 + c)) dft_add(u, tab, step, r, j0 + c, N.a[c]);
    }
}

// ------------------------------------------------------------------------ TM
template <int S>
__device__ __forceinline__ void tm_level(const Unit &u, const LensStepTable &tab, int step, int r, const F3 &P,
                                         const F3 &C, const F3 &Q, F3 &N, const float *kyh, const float *kye) {
    const LensInst2D *g = u.g;
    const int nx = u.nx, ny = u.ny, j0 = u.j0;
    const float exn = __shfl_down_sync(FULL, P.a[0], 1);  // Ex(r, j0 + 4)
    if (r < 0 || r >= nx) {  // uniform over the warp (one row per level)
        zero3(N);
        return;
    }
    const float ch = __ldg(&g->ch);
    const LensProfile &xh = g->ax.h, &xe = g->ax.e, &yh = g->ay.h, &ye = g->ay.e;
    const bool rex = row_exact<S>(u, r);
    // ---- Hz (boundaries.py:240-247)
    const int sxh = r < nx - 1 ? strip_of(r, xh.lo, xh.hi, xh.n) : -1;
    const float kxh = r < nx - 1 ? __ldg(xh.ik + r) : 0.f;
#pragma unroll
    for (int c = 0; c < TV; ++c) {
        const int j = j0 + c;
        float hz = P.c[c];
        if (r < nx - 1 && j >= 0 && j < ny - 1) {
            const float dyx = C.b[c] - P.b[c], dxy = (c + 1 < TV ? P.a[c + 1] : exn) - P.a[c];
            float px = 0.f, py = 0.f;
            const bool wr = S == K ? owned(u, r, j) : (rex && col_exact<S>(u, j));
            const int sj = strip_of(j, yh.lo, yh.hi, yh.n);
            if (sxh >= 0) px = psi_lv<S>(u, 0, xh, r, sxh, r, j, dyx, wr);
            if (sj >= 0) py = psi_lv<S>(u, 1, yh, j, sj, r, j, dxy, wr);
            hz = P.c[c] - ch * ((dyx * kxh + px) - (dxy * kyh[c] + py));
        }
        N.c[c] = hz;
    }
    // ---- loss damping, Ex / Ey (boundaries.py:249-268), source, PEC
    const float hzm = __shfl_up_sync(FULL, N.c[TV - 1], 1);  // Hz(r, j0 - 1)
    const bool lossy = ldu64(&g->c[2]) != 0ull;
    const int nq = lossy ? 4 : 2;
    float ax_[TV], ay_[TV], dx_[TV], dy_[TV];
#pragma unroll
    for (int c = 0; c < TV; ++c) ax_[c] = ay_[c] = 0.f, dx_[c] = dy_[c] = 1.f;
    if (j0 >= 0 && j0 < u.P) {
        f4_to(__ldg(reinterpret_cast<const float4 *>(crow(g, 0, nq, r, j0, u.P))), ax_);
        f4_to(__ldg(reinterpret_cast<const float4 *>(crow(g, 1, nq, r, j0, u.P))), ay_);
        if (lossy) {
            f4_to(__ldg(reinterpret_cast<const float4 *>(crow(g, 2, nq, r, j0, u.P))), dx_);
            f4_to(__ldg(reinterpret_cast<const float4 *>(crow(g, 3, nq, r, j0, u.P))), dy_);
        }
    }
    const bool rin = r >= 1 && r <= nx - 2;
    const int sxe = rin ? strip_of(r, xe.lo, xe.hi, xe.n) : -1;
    const float kxe = __ldg(xe.ik + r);
    const int six = __ldg(&g->src.ix), snj = __ldg(&g->src.nj);
    const bool srow = six >= 0 && (r == six || r == six + 1);
    const int pec0 = __ldg(g->pec), pec1 = __ldg(g->pec + 1), pec2 = __ldg(g->pec + 2), pec3 = __ldg(g->pec + 3);
#pragma unroll
    for (int c = 0; c < TV; ++c) {
        const int j = j0 + c;
        const bool wr = S == K ? owned(u, r, j) : (rex && col_exact<S>(u, j));
        float ex = P.a[c], ey = P.b[c];
        if (r < nx - 1 && j >= 0 && j < ny) {  // Ex at (r+1/2, j)
            float e = ex;
            if (lossy) e = e * dx_[c];
            if (j >= 1 && j <= ny - 2) {
                const float d = N.c[c] - (c > 0 ? N.c[c - 1] : hzm);
                float p = 0.f;
                const int sj = strip_of(j, ye.lo, ye.hi, ye.n);
                if (sj >= 0) p = psi_lv<S>(u, 2, ye, j, sj, r, j, d, wr);
                e = e + ax_[c] * (d * kye[c] + p);
            }
            if ((pec2 && j == 0) || (pec3 && j == ny - 1)) e = 0.f;
            ex = e;
        }
        if (j >= 0 && j < ny - 1) {  // Ey at (r, j+1/2)
            float e = ey;
            if (lossy) e = e * dy_[c];
            if (rin) {
                const float d = N.c[c] - Q.c[c];
                float p = 0.f;
                if (sxe >= 0) p = psi_lv<S>(u, 3, xe, r, sxe, r, j, d, wr);
                e = e + (-ay_[c]) * (d * kxe + p);
            }
            if (srow && j < snj) e += src_term(g, tab, step, r, j);
            if ((pec0 && r == 0) || (pec1 && r == nx - 1)) e = 0.f;
            ey = e;
        }
        N.a[c] = ex;
        N.b[c] = ey;
    }
    // node DFT of Ey averaged onto the nodes (fdtd2d_core.py:458-465)
    const float eym = __shfl_up_sync(FULL, N.b[TV - 1], 1);  // Ey(r, j0 - 1)
    if (u.dft && step >= u.dft_n0 && step < u.dft_n1 && r >= u.x0 && r < u.x1) {
#pragma unroll
        for (int c = 0; c < TV; ++c) {
            const int j = j0 + c;
            if (!owned(u, r, j)) continue;
            float v;
            if (j == 0) v = N.b[0];
            else if (j == ny - 1) v = c > 0 ? N.b[c - 1] : eym;
            else v = 0.5f * ((c > 0 ? N.b[c - 1] : eym) + N.b[c]);
            dft_add(u, tab, step, r, j, v);
        }
    }
}

template <int S>
__device__ __forceinline__ void level(const Unit &u, const LensStepTable &tab, int n0, int r, const F3 &P, const F3 &C,
                                      const F3 &Q, F3 &N, const float *kyh, const float *kye) {
    const int step = n0 + S - 1 - u.nst;  // the instance's own step of level S
    if (u.pol == 0) te_level<S>(u, tab, step, r, P, C, Q, N, kyh, kye);
    else tm_level<S>(u, tab, step, r, P, C, Q, N, kyh, kye);
}

template <typename T>
__global__ void __launch_bounds__(TW * 32)
    tb2d(const LensTB2D *inst, const int *first, int ninst, int nunits, int chunk, const LensStepTable tab, int n0,
         int par) {
    const int unit = blockIdx.x * TW + (threadIdx.x >> 5);
    if (unit >= nunits) return;  // whole warps leave together
    const int lane = threadIdx.x & 31;
    // instance of this unit: the last q with first[q] <= unit
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(first + mid) <= unit) lo = mid;
        else hi = mid - 1;
    }
    const LensTB2D *d = inst + lo;
    const LensInst2D *g = &d->g;
    Unit u;
    u.g = g;
    u.pol = __ldg(&g->pol);
    u.nx = __ldg(&g->nx);
    u.ny = __ldg(&g->ny);
    u.P = __ldg(&g->pitch);
    u.nst = __ldg(&g->n_start);
    const int ntc = (u.ny + TO - 1) / TO;
    const int w = unit - __ldg(first + lo);
    u.c0 = (w % ntc) * TO;
    u.cA = u.c0 - K;
    u.x0 = (w / ntc) * chunk;
    u.x1 = min(u.nx, u.x0 + chunk);
    u.j0 = u.cA + lane * TV;
    for (int q = 0; q < 3; ++q) {
        void *b0 = reinterpret_cast<void *>(ldu64(&g->f[q])), *b1 = reinterpret_cast<void *>(ldu64(&d->f1[q]));
        u.fi[q] = par ? b1 : b0;
        u.fo[q] = par ? b0 : b1;
    }
    size_t off = 0;
    for (int q = 0; q < 4; ++q) {
        const LensProfile &pf = psi_prof(g, u.pol, q);
        u.wid[q] = __ldg(&pf.lo) + __ldg(&pf.hi);
        float *b0 = reinterpret_cast<float *>(ldu64(&g->psi[q])), *b1 = reinterpret_cast<float *>(ldu64(&d->psi1[q]));
        u.pin[q] = par ? b1 : b0;
        u.pout[q] = par ? b0 : b1;
        u.lvoff[q] = off;
        off += u.wid[q] == 0 ? 0 : (psi_is_x(u.pol, q) ? (size_t)u.wid[q] * u.P : (size_t)u.nx * u.wid[q]);
    }
    u.lvtot = off;
    u.lv = reinterpret_cast<float *>(ldu64(&d->psi_lv));
    u.kahan = __ldg(&d->dft_kahan) != 0;
    u.dft = reinterpret_cast<float *>(ldu64(&g->dft));
    u.dft_n0 = __ldg(&g->dft_n0);
    u.dft_n1 = __ldg(&g->dft_n1);
    // 1/kappa of this lane's columns (loop-invariant): H (half nodes), E (nodes)
    const LensProfile &yh = g->ay.h, &ye = g->ay.e;
    float kyh[TV], kye[TV];
#pragma unroll
    for (int c = 0; c < TV; ++c) {
        const int j = u.j0 + c;
        kyh[c] = (j >= 0 && j < u.ny - 1) ? __ldg(yh.ik + j) : 0.f;
        kye[c] = (j >= 0 && j < u.ny) ? __ldg(ye.ik + j) : 0.f;
    }
    const int P = u.P, nx = u.nx;
    using St_ = St<T>;
    // st[s]: level s on its previous row (level 0: the last loaded row)
    F3 st[K + 1];
#pragma unroll
    for (int s = 0; s <= K; ++s) zero3(st[s]);
    const int t0 = u.x0 - K, t1 = u.x1 + K;  // rows loaded: [t0, t1)
    F3 nxt;
    load3<T>(nxt, u.fi, t0, u.j0, nx, P);
    // the last owned row x1 - 1 leaves level K at t = t1 - 1
    for (int t = t0; t < t1; ++t) {
        F3 cur = nxt;
        if (t + 1 < t1) load3<T>(nxt, u.fi, t + 1, u.j0, nx, P);
        // level s on row t - s: P = level s-1 on row t-s (its previous row),
        // C = level s-1 on row t-s+1 (just computed), Q = level s on row t-s-1
        F3 pv = st[0];
        st[0] = cur;
        F3 cv = cur;
#define LENS_TB_LEVEL(S_)                                                  \
        {                                                                  \
            F3 nv;                                                         \
            level<S_>(u, tab, n0, t - S_, pv, cv, st[S_], nv, kyh, kye);   \
            pv = st[S_];                                                   \
            st[S_] = nv;                                                   \
            cv = nv;                                                       \
        }
        LENS_TB_LEVEL(1)
        LENS_TB_LEVEL(2)
        LENS_TB_LEVEL(3)
        LENS_TB_LEVEL(4)
#undef LENS_TB_LEVEL
        // level K is final on the owned part of row t - K
        const int r = t - K;
        if (r >= u.x0 && r < u.x1 && u.j0 >= u.c0 && u.j0 < u.c0 + TO && u.j0 < P) {
            const size_t o = (size_t)r * P + u.j0;
            St_::st4(u.fo[0], o, to_f4(st[K].a));
            St_::st4(u.fo[1], o, to_f4(st[K].b));
            St_::st4(u.fo[2], o, to_f4(st[K].c));
        }
    }
}
static_assert(K == 4, "tb2d unrolls four levels");

// Host-side checks of an instance (the single-step batched kernels' rules).
bool tb_inst_ok(const LensInst2D &g) {
    if ((g.pol != 0 && g.pol != 1) || g.nx < 3 || g.ny < 3 || g.pitch < g.ny || (g.pitch % 32)) return false;
    if (!g.f[0] || !g.f[1] || !g.f[2] || !g.c[0] || !g.c[1]) return false;
    if (g.pol == 1 && (!g.c[2]) != (!g.c[3])) return false;
    if (g.rtype && !g.ctab) return false;
    if (!lens_profile_ok(g.ax.e, g.nx) || !lens_profile_ok(g.ax.h, g.nx - 1) || !lens_profile_ok(g.ay.e, g.ny) ||
        !lens_profile_ok(g.ay.h, g.ny - 1))
        return false;
    if (g.src.ix >= 0 && (!g.src.amp || !g.src.ph1 || !g.src.ph2 || g.src.ix + 1 >= g.nx || g.src.nj > g.ny))
        return false;
    const LensProfile *strip[2][4] = {{&g.ay.h, &g.ax.h, &g.ax.e, &g.ay.e}, {&g.ax.h, &g.ay.h, &g.ay.e, &g.ax.e}};
    for (int q = 0; q < 4; ++q)
        if (!lens_psi_ok(*strip[g.pol][q], g.psi[q])) return false;
    return true;
}

bool tb_ok(const LensTB2D &d) {
    const LensInst2D &g = d.g;
    if (!tb_inst_ok(g) || !d.f1[0] || !d.f1[1] || !d.f1[2]) return false;
    for (int q = 0; q < 4; ++q)
        if (g.psi[q] && !d.psi1[q]) return false;
    const bool any = g.ax.e.lo + g.ax.e.hi + g.ax.h.lo + g.ax.h.hi + g.ay.e.lo + g.ay.e.hi + g.ay.h.lo + g.ay.h.hi > 0;
    if (any && !d.psi_lv) return false;
    return true;
}

long tb_units(const LensInst2D &g, int chunk) {
    return (long)((g.ny + TO - 1) / TO) * ((g.nx + chunk - 1) / chunk);
}

}  // namespace

extern "C" int lens_tb2d_plan(const LensTB2D *inst, int ninst, int chunk, int *first) {
    if (!inst || ninst < 1 || chunk < 1 || !first) return LENS_ERR_ARG;
    long tot = 0;
    for (int q = 0; q < ninst; ++q) {
        if (!tb_ok(inst[q])) return LENS_ERR_ARG;
        first[q] = (int)tot;
        tot += tb_units(inst[q].g, chunk);
        if (tot > 0x7fffffffL - TW) return LENS_ERR_SIZE;
    }
    first[ninst] = (int)tot;
    return (int)tot;
}

extern "C" int lens_tb2d_step(const LensTB2D *inst_host, const LensTB2D *inst_dev, const int *first_dev, int ninst,
                              int chunk, int storage, const LensStepTable *tab, int n0, int nsteps, void *stream) {
    if (!inst_host || !inst_dev || !first_dev || ninst < 1 || chunk < 1 || nsteps < 0 || nsteps % (2 * K))
        return LENS_ERR_ARG;
    long tot = 0;
    bool any_dft = false;
    for (int q = 0; q < ninst; ++q) {
        const LensInst2D &g = inst_host[q].g;
        if (!tb_ok(inst_host[q]) || n0 < g.n_start || !lens_table_ok(tab, n0 - g.n_start, nsteps)) return LENS_ERR_ARG;
        if (g.dft && (reinterpret_cast<uintptr_t>(g.dft) & 15)) return LENS_ERR_ARG;
        tot += tb_units(g, chunk);
        any_dft = any_dft || g.dft;
    }
    if (tot > 0x7fffffffL - TW) return LENS_ERR_SIZE;
    if (any_dft && !tab->pe) return LENS_ERR_ARG;
    const int nunits = (int)tot;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = (nunits + TW - 1) / TW;
    for (int m = 0; m < nsteps / K; ++m) {
        const int par = m & 1;
        const int n = n0 + m * K;
        switch (storage) {
            case LENS_F32: tb2d<float><<<nb, TW * 32, 0, s>>>(inst_dev, first_dev, ninst, nunits, chunk, *tab, n, par); break;
            case LENS_F16: tb2d<__half><<<nb, TW * 32, 0, s>>>(inst_dev, first_dev, ninst, nunits, chunk, *tab, n, par); break;
            case LENS_BF16:
                tb2d<__nv_bfloat16><<<nb, TW * 32, 0, s>>>(inst_dev, first_dev, ninst, nunits, chunk, *tab, n, par);
                break;
            default: return LENS_ERR_ARG;
        }
    }
    return lens_cuda_status();
}
