// Resident batched 2D solves for sm_100a: a group of 2D TE/TM instances whose
// whole state fits on the chip is advanced by many steps in ONE cooperative
// launch, the fields held in registers from the first step to the last.
//
// A CTA owns a band of `rows` consecutive x rows of one instance and every y
// column of it: thread (lane, warp) holds column j = 32*warp + lane of each of
// its rows in registers (three field arrays of RM floats).  Per step:
//   H phase: neighbour terms along y from the next lane (shuffle) or, for lane
//            31, from lane 0 of the next warp (shared memory); along x from the
//            thread's own next row, and for the band's last row from the next
//            band's first row (its E field of the previous step);
//   E phase: the same towards -y / -x, the band's first row taking the previous
//            band's last H row of this step.
// Bands exchange those single rows through L2 only: a thread publishes its
// column of the row as one 64-bit word {value, step tag} (one single-copy-atomic
// store, no fence and no flag), and the neighbour's thread of the same column
// polls that word until the tag of the step it needs appears.  Every poll is
// bounded; a wait that runs out sets *err, and all CTAs leave the step loop at
// their next CTA barrier (or when they see *err), write their state back and
// end.  Interior rows are updated before each wait, so the waits overlap them.
// Each slot of the halo rows is double-buffered by step parity; the exchange
// order (a band's E(n) needs the previous band's H(n), which needed this band's
// E(n-1)) keeps a slot from being rewritten before its reader is done with it.
//
// Bands clear of the x CPML strips, the source rows and the x faces run lean
// rows (the y strip and face terms by selects, no branch); the others run the
// general rows.  The per-cell arithmetic is term for
// term that of the batched kernels (fdtd2d_batch.cu, after
// planar_beads/boundaries.py:164-274, source vcsel.py:151-156, loss
// fdtd2d_core.py:796-797, TM nodes fdtd2d_core.py:458-465).  The band's
// coefficient rows and the CPML psi of its strip cells live in shared memory
// for the launch.  The node DFT is accumulated into the instance's dft array as
// (re, im) or, per instance, compensated (re, im, c_re, c_im).  Storage is FP32
// only: the state never leaves the chip between the first and the last step.
#include <algorithm>

#include "lens_common.cuh"

namespace {

constexpr int RS_MAXW = 18;                  // warps per CTA: ny <= 576
// The register file is split over the SM's four schedulers, a warp's registers
// on one of them: a CTA of up to 16 warps (ny <= 512) has 128 registers per
// thread, one of 17 or 18 warps (ny <= 576) 96 (the "wide" launches).
constexpr int RS_NT_NARROW = 512, RS_NT_WIDE = RS_MAXW * 32;
constexpr int RS_MAXWY = 64;                 // psi strip width of one y staggering (lo + hi)
constexpr long long RS_TRIES = 1LL << 22;    // polls per wait (each an L2 round trip, >= 0.3 us)
constexpr unsigned FULL = 0xffffffffu;

constexpr int RS_MAXCTA = 512;                // bands per launch
struct RPlan {
    int ninst, rows, nc;              // most rows of a band; coefficients per row held in shared memory
    int first[LENS_RS_MAX_INST + 1];  // first CTA of instance q; first[ninst] = grid
    LensRsOut2D out[LENS_RS_MAX_INST];
    short lo[RS_MAXCTA];              // first row of each band (a band ends where the instance's next begins)
    long long tries;                  // polls per wait
    int wd_cta;                       // watchdog self-test: this band withholds its E row of step 1 (-1: none)
};

// Row flags (RowC.flags): the row exists in the band, i < nx-1 (TE Hy / TM Hz
// and Ex rows), 0 < i < nx-1 (E curl rows), source rows ix (+) / ix+1 (-), PEC
// x face, psi of an x strip (H / E).
enum : unsigned { R_REAL = 1u, R_HOK = 2u, R_IN = 4u, R_SRCP = 8u, R_SRCM = 16u, R_XPEC = 32u, R_XH = 64u, R_XE = 128u };
constexpr unsigned R_LEAN = R_REAL | R_HOK | R_IN;
// Thread flags: j < ny-1, j < ny, 0 < j < ny-1, PEC y face, source column
// (j < src.nj).  The y-strip psi needs no flag: outside the strips a column's
// psi slot is a zero slot with b = c = 0.
enum : unsigned { T_HX = 1u, T_JLT = 2u, T_JIN = 4u, T_JPEC = 32u, T_SRCJ = 64u };
// Band flags
enum : unsigned { B_PREV = 1u, B_NEXT = 2u, B_LOSSY = 4u, B_KAHAN = 8u };

// Row constants of a band (shared memory): x profile values and strip indices.
struct __align__(16) RowC {
    float kxh, kxe, bxh, cxh, bxe, cxe;
    int sxh_sxe;         // x-strip index of the H psi (low 16 bits) and E psi (high 16 bits)
    unsigned flags;
};
static_assert(sizeof(RowC) % 16 == 0 && alignof(RowC) == 16, "row constants: whole 16-byte vectors");

// Band constants (shared memory, read into registers before the step loop).
struct Band {
    float *f[3];
    float *pxh, *pxe, *pyh, *pye;  // psi by role: x strips (w, pitch), y strips (nx, w)
    float *dft, *frames;
    const float *amp, *ph1, *ph2;
    int nx, ny, P, lo, R, wyh, wye, snj, dft_n0, dft_n1, n_start, every, nframes;
    unsigned flags;
    float ch;
};

__device__ __forceinline__ void put_tag(unsigned long long *p, float v, unsigned tag) {
    const unsigned long long w = ((unsigned long long)tag << 32) | __float_as_uint(v);
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}

// Value of the word at p once its tag is `tag`; false if the wait ran out or
// another CTA reported an error.
__device__ __forceinline__ bool get_tag(const unsigned long long *p, unsigned tag, const int *err, float &v,
                                        long long tries) {
    for (long long t = 0;; ++t) {
        unsigned long long w;
        asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
        if ((unsigned)(w >> 32) == tag) {
            v = __uint_as_float((unsigned)w);
            return true;
        }
        if (t >= tries) return false;
        if ((t & 255) == 255 && *reinterpret_cast<const volatile int *>(err)) return false;
    }
}

// A zero the compiler cannot see through: the lean rows add it where the
// general rows add a psi term, so both evaluate the same expression shapes.
__device__ __forceinline__ float opaque_zero() {
    float z;
    asm volatile("mov.b32 %0, 0;" : "=f"(z));
    return z;
}

__device__ __forceinline__ void dft_add(float *dft, bool kahan, size_t o, float v, float pr, float pim) {
    if (kahan) {
        kahan_add(reinterpret_cast<float4 *>(dft) + o, v * pr, v * pim);
    } else {
        float2 *a = reinterpret_cast<float2 *>(dft) + o;
        float2 s = *a;
        s.x += v * pr;
        s.y += v * pim;
        *a = s;
    }
}

// Band constants, row constants and the band's coefficient rows of CTA `cta`
// into shared memory.
template <int RM, int POL>
__device__ __forceinline__ void band_setup(const LensInst2D *gp, const RPlan &pl, int q, int cta, int NT, Band &B,
                                           RowC *rowc, float *ypc, float *cs) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int nx = gp->nx, ny = gp->ny, P = gp->pitch;
    const int lo = pl.lo[cta], hi = cta + 1 < pl.first[q + 1] ? pl.lo[cta + 1] : nx;
    const int six = gp->src.ix;
    const bool lossy = POL == 1 && gp->c[2] != nullptr;
    if (w == 0 && lane == 0) {
        for (int k = 0; k < 3; ++k) B.f[k] = static_cast<float *>(gp->f[k]);
        B.pxh = gp->psi[POL ? 0 : 1];
        B.pxe = gp->psi[POL ? 3 : 2];
        B.pyh = gp->psi[POL ? 1 : 0];
        B.pye = gp->psi[POL ? 2 : 3];
        B.dft = gp->dft;
        B.frames = pl.out[q].frames;
        B.every = pl.out[q].every;
        B.nframes = pl.out[q].nframes;
        B.amp = gp->src.amp;
        B.ph1 = gp->src.ph1;
        B.ph2 = gp->src.ph2;
        B.snj = gp->src.nj;
        B.nx = nx;
        B.ny = ny;
        B.P = P;
        B.lo = lo;
        B.R = hi - lo;
        B.wyh = gp->ay.h.lo + gp->ay.h.hi;
        B.wye = gp->ay.e.lo + gp->ay.e.hi;
        B.dft_n0 = gp->dft_n0;
        B.dft_n1 = gp->dft_n1;
        B.n_start = gp->n_start;
        B.flags = (cta > pl.first[q] ? B_PREV : 0u) | (hi < nx ? B_NEXT : 0u) | (lossy ? B_LOSSY : 0u) |
                  (pl.out[q].kahan ? B_KAHAN : 0u);
        B.ch = gp->ch;
    }
    if (w == 0 && lane < RM) {  // RM <= 32
        const int r = lane, i = lo + r;
        const LensProfile xh = gp->ax.h, xe = gp->ax.e;
        RowC rc;
        rc.kxh = rc.kxe = rc.bxh = rc.cxh = rc.bxe = rc.cxe = 0.f;
        int sh = -1, se = -1;
        unsigned f = 0;
        if (i < hi) {
            f = R_REAL;
            if (i < nx - 1) {
                f |= R_HOK;
                rc.kxh = __ldg(xh.ik + i);
                sh = strip_of(i, xh.lo, xh.hi, xh.n);
                if (sh >= 0) {
                    rc.bxh = __ldg(xh.b + i);
                    rc.cxh = __ldg(xh.c + i);
                    f |= R_XH;
                }
            }
            rc.kxe = __ldg(xe.ik + i);
            if (i > 0 && i < nx - 1) {
                f |= R_IN;
                se = strip_of(i, xe.lo, xe.hi, xe.n);
                if (se >= 0) {
                    rc.bxe = __ldg(xe.b + i);
                    rc.cxe = __ldg(xe.c + i);
                    f |= R_XE;
                }
            }
            if (six >= 0 && i == six) f |= R_SRCP;
            if (six >= 0 && i == six + 1) f |= R_SRCM;
            if ((gp->pec[0] && i == 0) || (gp->pec[1] && i == nx - 1)) f |= R_XPEC;
        }
        rc.sxh_sxe = (sh & 0xffff) | (se << 16);
        rc.flags = f;
        rowc[r] = rc;
    }
    // y profile values of the strip columns: ypc[0..3][sj] = b_h, c_h, b_e, c_e
    const int j = w * 32 + lane;
    const LensProfile yh = gp->ay.h, ye = gp->ay.e;
    const int sjh = (j < ny - 1) ? strip_of(j, yh.lo, yh.hi, yh.n) : -1;
    const int sje = (j > 0 && j < ny - 1) ? strip_of(j, ye.lo, ye.hi, ye.n) : -1;
    if (sjh >= 0) {
        ypc[sjh] = __ldg(yh.b + j);
        ypc[RS_MAXWY + sjh] = __ldg(yh.c + j);
    }
    if (sje >= 0) {
        ypc[2 * RS_MAXWY + sje] = __ldg(ye.b + j);
        ypc[3 * RS_MAXWY + sje] = __ldg(ye.c + j);
    }
    // the band's coefficient rows, typed or not: cs[(r * nc + k) * NT + j]
    const int nci = POL == 0 ? 2 : (lossy ? 4 : 2);
    for (int r = 0; r < RM; ++r) {
        const int i = lo + r;
        const unsigned t = (i < hi && gp->rtype) ? gp->rtype[i] : 255u;
        for (int k = 0; k < pl.nc; ++k) {
            float v = 0.f;
            if (i < hi && j < ny && k < nci)
                v = t == 255u ? __ldg(gp->c[k] + (size_t)i * P + j) : __ldg(gp->ctab + ((size_t)t * nci + k) * P + j);
            cs[(r * pl.nc + k) * NT + j] = v;
        }
    }
}

template <int RM, int POL>
__device__ __forceinline__ void rs_band(const LensInst2D *__restrict__ insts, const RPlan &pl, const LensStepTable &tab,
                                        int n0, int nsteps, unsigned long long *halo, int *err, unsigned char *smem) {
    const int lane = threadIdx.x, w = threadIdx.y, W = blockDim.y, NT = 32 * W;
    const int j = w * 32 + lane;
    const int cta = blockIdx.x;
    int q = 0;
    while (q + 1 < pl.ninst && cta >= pl.first[q + 1]) ++q;
    const LensInst2D *gp = insts + q;
    const int NC = pl.nc;

    // shared memory: coefficient rows [RM][NC][NT], x-strip psi (H, E) [RM][NT],
    // y-strip psi (H, E) [RM][RS_MAXWY], y profile values of the strip columns
    // [4][RS_MAXWY], warp-edge columns zb / xb / eb [RM][RS_MAXW], row constants
    // [RM], band constants
    float *cs = reinterpret_cast<float *>(smem);
    float *xps_h = cs + RM * NC * NT;
    float *xps_e = xps_h + RM * NT;
    float *yps_h = xps_e + RM * NT;
    float *yps_e = yps_h + RM * RS_MAXWY;
    float *ypc = yps_e + RM * RS_MAXWY;
    float *zb = ypc + 4 * RS_MAXWY;      // lane 0 of each warp: E field read at j+1 (TE Ez, TM Ex)
    float *xb = zb + RM * RS_MAXW;       // lane 31: H field read at j-1 (TE Hx, TM Hz)
    float *eb = xb + RM * RS_MAXW;       // lane 31: TM Ey (node average)
    float *junk = eb + RM * RS_MAXW;     // [NT]: the y-psi slot of a column outside the y strips (stays 0)
    // the row constants are read as 16-byte vectors: their array starts on a 16-byte boundary
    RowC *rowc = reinterpret_cast<RowC *>((reinterpret_cast<uintptr_t>(junk + NT) + 15) & ~uintptr_t(15));
    for (int t = threadIdx.y * 32 + threadIdx.x; t < 2 * RM * NT + 2 * RM * RS_MAXWY; t += NT) xps_h[t] = 0.f;
    junk[w * 32 + lane] = 0.f;
    Band &B = *reinterpret_cast<Band *>(rowc + RM);
    band_setup<RM, POL>(gp, pl, q, cta, NT, B, rowc, ypc, cs);
    __syncthreads();

    const int ny = B.ny, R = B.R;
    const unsigned bf = B.flags;
    const float ch = B.ch;
    const bool lossy = bf & B_LOSSY;
    const int sjh = (j < ny - 1) ? strip_of(j, gp->ay.h.lo, gp->ay.h.hi, ny - 1) : -1;
    const int sje = (j > 0 && j < ny - 1) ? strip_of(j, gp->ay.e.lo, gp->ay.e.hi, ny) : -1;
    const float kyh = j < ny - 1 ? __ldg(gp->ay.h.ik + j) : 0.f, kye = j < ny ? __ldg(gp->ay.e.ik + j) : 0.f;
    const float byh = sjh >= 0 ? ypc[sjh] : 0.f, cyh = sjh >= 0 ? ypc[RS_MAXWY + sjh] : 0.f;
    const float bye = sje >= 0 ? ypc[2 * RS_MAXWY + sje] : 0.f, cye = sje >= 0 ? ypc[3 * RS_MAXWY + sje] : 0.f;
    // y-psi slot of row r: yqh + r * ysh (H), yqe + r * yse (E); outside the strips a
    // zero slot of this thread's own, with b = c = 0, so the psi terms need no branch
    float *yqh = sjh >= 0 ? yps_h + sjh : junk + j, *yqe = sje >= 0 ? yps_e + sje : junk + j;
    const int ysh = sjh >= 0 ? RS_MAXWY : 0, yse = sje >= 0 ? RS_MAXWY : 0;
    unsigned tf = 0;
    if (j < ny - 1) tf |= T_HX;
    if (j < ny) tf |= T_JLT;
    if (j > 0 && j < ny - 1) tf |= T_JIN;
    if ((gp->pec[2] && j == 0) || (gp->pec[3] && j == ny - 1)) tf |= T_JPEC;
    if (j < B.snj) tf |= T_SRCJ;
    bool band_lean = true;
#pragma unroll
    for (int r = 0; r < RM; ++r) {
        const unsigned f = rowc[r].flags;
        if (f & R_REAL) band_lean = band_lean && f == R_LEAN;
    }
    // every warp of a band clear of x strips, source rows and x faces runs the lean rows
    const bool lean = band_lean;
    const float *csj = cs + j;

    // ---- state in: fields (registers), psi strips (shared memory)
    float fa[RM], fb[RM], fc[RM];
#pragma unroll
    for (int r = 0; r < RM; ++r) {
        const bool in = r < R && j < ny;
        const size_t o = (size_t)(B.lo + r) * B.P + j;
        fa[r] = in ? B.f[0][o] : 0.f;
        fb[r] = in ? B.f[1][o] : 0.f;
        fc[r] = in ? B.f[2][o] : 0.f;
        if (r < R) {
            const RowC &rc = rowc[r];
            const int sh = (int)(short)(rc.sxh_sxe & 0xffff), se = rc.sxh_sxe >> 16;
            if (sh >= 0 && j < ny) xps_h[r * NT + j] = B.pxh[(size_t)sh * B.P + j];
            if (se >= 0 && j < ny) xps_e[r * NT + j] = B.pxe[(size_t)se * B.P + j];
            if (sjh >= 0) yps_h[r * RS_MAXWY + sjh] = B.pyh[(size_t)(B.lo + r) * B.wyh + sjh];
            if (sje >= 0) yps_e[r * RS_MAXWY + sje] = B.pye[(size_t)(B.lo + r) * B.wye + sje];
        }
    }
    // E field of the next band's first row before the first step (TE Ez, TM Ey)
    float e_next0 = 0.f;
    if ((bf & B_NEXT) && j < ny) e_next0 = B.f[POL == 0 ? 0 : 1][(size_t)(B.lo + R) * B.P + j];
    // halo words: [cta][kind 0: first E row, 1: last H row][slot][NT]
    const size_t hq = (size_t)2 * NT;
    unsigned long long *h_my = halo + (size_t)cta * 2 * hq + j;
    const unsigned long long *h_next_e = halo + (size_t)(cta + 1) * 2 * hq + j;
    const unsigned long long *h_prev_h = halo + (size_t)max(cta - 1, 0) * 2 * hq + hq + j;
    if (lane == 0)
        for (int r = 0; r < RM; ++r) zb[r * RS_MAXW + w] = fa[r];
    __syncthreads();

    const float z = opaque_zero();
    // neighbour along +y (lane 31: lane 0 of the next warp) / -y (lane 0: lane 31 of the previous warp)
    auto nb_up = [&](float v, int r) {
        float u = __shfl_down_sync(FULL, v, 1);
        if (lane == 31) u = (w + 1 < W) ? zb[r * RS_MAXW + w + 1] : 0.f;
        return u;
    };
    auto nb_dn = [&](const float *edge, float v, int r) {
        float u = __shfl_up_sync(FULL, v, 1);
        if (lane == 0) u = w > 0 ? edge[r * RS_MAXW + w - 1] : 0.f;
        return u;
    };
    // thread tests, as booleans
    const bool t_hx = tf & T_HX, t_jlt = tf & T_JLT, t_jin = tf & T_JIN, t_zero = (tf & T_JPEC) || !(tf & T_JLT),
               t_jpec = tf & T_JPEC, t_src = tf & T_SRCJ;
    // The general rows evaluate every update and keep it where it applies
    // (selects): psi slots exist for every row and column (zero outside the
    // strips, with b = c = 0 there), so no psi term is a branch and the
    // compiler interleaves the rows.  A psi value is stored back only where the
    // batched kernels update it.
    // H of row r below the band's last (TE: also Hx of every row, the last included)
    auto h_gen = [&](int r) {
        const RowC rc = rowc[r];
        const unsigned rf = rc.flags;
        const bool below = r + 1 < R;
        if (POL == 0) {
            const float ez = fa[r];
            const float d = nb_up(ez, r) - ez;
            float *qy = yqh + r * ysh;
            const float py = byh * (*qy) + cyh * d;  // psi_hxy (the zero slot outside the strip)
            *qy = py;
            const float hx = fb[r] - ch * (d * kyh + py);  // Hx (boundaries.py:186-190)
            fb[r] = t_hx ? hx : fb[r];
            if (r + 1 < RM) {  // Hy (:191-194)
                const float d2 = fa[r + 1] - ez;
                float *qx = xps_h + r * NT + j;
                const float ox = *qx, px = rc.bxh * ox + rc.cxh * d2;
                const bool on = below && (rf & R_HOK) && t_jlt;
                *qx = on ? px : ox;
                const float hy = fc[r] + ch * (d2 * rc.kxh + px);
                fc[r] = on ? hy : fc[r];
            }
        } else if (r + 1 < RM) {  // Hz (boundaries.py:240-247)
            const float ex = fa[r];
            const float dyx = fb[r + 1] - fb[r], dxy = nb_up(ex, r) - ex;
            const bool on = below && (rf & R_HOK) && t_hx;
            float *qx = xps_h + r * NT + j, *qy = yqh + r * ysh;
            const float ox = *qx, oy = *qy;
            const float px = rc.bxh * ox + rc.cxh * dyx, py = byh * oy + cyh * dxy;
            *qx = on ? px : ox;
            *qy = on ? py : oy;
            const float hz = fc[r] - ch * ((dyx * rc.kxh + px) - (dxy * kyh + py));
            fc[r] = on ? hz : fc[r];
        }
    };
    // the band's last row (TE Hy, TM Hz) from en: the E field of row i+1 (TE Ez, TM Ey)
    auto h_last = [&](int r, float en) {
        const RowC rc = rowc[r];
        const unsigned rf = rc.flags;
        if (POL == 0) {
            const float d2 = en - fa[r];
            float *qx = xps_h + r * NT + j;
            const float ox = *qx, px = rc.bxh * ox + rc.cxh * d2;
            const bool on = (rf & R_HOK) && t_jlt;
            *qx = on ? px : ox;
            const float hy = fc[r] + ch * (d2 * rc.kxh + px);
            fc[r] = on ? hy : fc[r];
        } else {
            const float ex = fa[r];
            const float dyx = en - fb[r], dxy = nb_up(ex, r) - ex;
            const bool on = (rf & R_HOK) && t_hx;
            float *qx = xps_h + r * NT + j, *qy = yqh + r * ysh;
            const float ox = *qx, oy = *qy;
            const float px = rc.bxh * ox + rc.cxh * dyx, py = byh * oy + cyh * dxy;
            *qx = on ? px : ox;
            *qy = on ? py : oy;
            const float hz = fc[r] - ch * ((dyx * rc.kxh + px) - (dxy * kyh + py));
            fc[r] = on ? hz : fc[r];
        }
    };
    // Rows of a band clear of x strips, source rows and x faces (every real row
    // R_LEAN), any warp: the lean arithmetic plus the y-strip psi through the
    // thread's psi slots (zero outside the strips) and the column selects.
    auto h_lean = [&](int r) {  // every row: TE Hx; rows below the band's last: Hy / Hz
        const float kx = rowc[r].kxh;
        const bool below = r + 1 < R;
        float *qy = yqh + r * ysh;
        const float oy = *qy;
        if (POL == 0) {
            const float ez = fa[r];
            const float d = nb_up(ez, r) - ez;
            const float py = byh * oy + cyh * d;
            *qy = py;
            const float hx = fb[r] - ch * (d * kyh + py);
            fb[r] = t_hx ? hx : fb[r];
            if (r + 1 < RM) {
                const float hy = fc[r] + ch * ((fa[r + 1] - ez) * kx + z);
                fc[r] = (below && t_jlt) ? hy : fc[r];
            }
        } else if (r + 1 < RM) {
            const float ex = fa[r];
            const float dyx = fb[r + 1] - fb[r], dxy = nb_up(ex, r) - ex;
            const bool on = below && t_hx;
            const float py = byh * oy + cyh * dxy;
            *qy = on ? py : oy;
            const float hz = fc[r] - ch * ((dyx * kx + z) - (dxy * kyh + py));
            fc[r] = on ? hz : fc[r];
        }
    };
    auto h_lean_last = [&](int r, float en) {  // the band's last row from the next band's first E row
        const float kx = rowc[r].kxh;
        if (POL == 0) {
            const float hy = fc[r] + ch * ((en - fa[r]) * kx + z);
            fc[r] = t_jlt ? hy : fc[r];
        } else {
            float *qy = yqh + r * ysh;
            const float oy = *qy;
            const float ex = fa[r];
            const float dyx = en - fb[r], dxy = nb_up(ex, r) - ex;
            const float py = byh * oy + cyh * dxy;
            *qy = t_hx ? py : oy;
            const float hz = fc[r] - ch * ((dyx * kx + z) - (dxy * kyh + py));
            fc[r] = t_hx ? hz : fc[r];
        }
    };
    auto e_lean = [&](int r, float hm) {  // hm: the H field of row i-1 (TE Hy, TM Hz)
        const float kx = rowc[r].kxe;
        float *qy = yqe + r * yse;
        const float oy = *qy;
        if (POL == 0) {
            const float hx = fb[r];
            const float dhy = fc[r] - hm, dhx = hx - nb_dn(xb, hx, r);
            const float py = bye * oy + cye * dhx;
            *qy = py;
            const float c0 = csj[(r * NC) * NT], c1 = csj[(r * NC + 1) * NT];
            const float vn = c0 * fa[r] + c1 * (dhy * kx + z - dhx * kye - py);
            const float v = t_jin ? vn : fa[r];
            fa[r] = t_zero ? 0.f : v;
        } else {
            const float hz = fc[r];
            const float d = hz - nb_dn(xb, hz, r), d2 = hz - hm;
            const float py = bye * oy + cye * d;
            *qy = py;
            float e = fa[r] * (lossy ? csj[(r * NC + 2) * NT] : 1.f);
            const float en = e + csj[(r * NC) * NT] * (d * kye + py);
            e = t_jin ? en : e;
            e = t_jpec ? 0.f : e;
            fa[r] = t_jlt ? e : fa[r];
            const float e2 = fb[r] * (lossy ? csj[(r * NC + 3) * NT] : 1.f);
            const float e2n = e2 + (-csj[(r * NC + 1) * NT]) * (d2 * kx + z);
            fb[r] = t_hx ? e2n : fb[r];
        }
    };
    // source term of row flags rf at table row k (vcsel.py:151-156)
    auto src_term = [&](unsigned rf, int k) {
        const float s = (__ldg(tab.env + k) * sinf(__ldg(tab.wt + k) + __ldg(((rf & R_SRCP) ? B.ph1 : B.ph2) + j))) *
                        __ldg(B.amp + j);
        return (rf & R_SRCP) ? s : -s;
    };
    // E of row r (any band) at table row k; hm: the H field of row i-1 (TE Hy, TM Hz)
    auto e_row = [&](int r, float hm, int k) {
        const RowC rc = rowc[r];
        const unsigned rf = rc.flags;
        const bool rin = rf & R_IN;
        if (POL == 0) {
            const float hx = fb[r];
            const float dhy = fc[r] - hm, dhx = hx - nb_dn(xb, hx, r);
            float *qx = xps_e + r * NT + j, *qy = yqe + r * yse;
            const float ox = *qx, oy = *qy;
            const float px = rc.bxe * ox + rc.cxe * dhy, py = bye * oy + cye * dhx;
            *qx = t_jin ? px : ox;  // zero outside the x strips (b = c = 0)
            *qy = rin ? py : oy;
            const float c0 = csj[(r * NC) * NT], c1 = csj[(r * NC + 1) * NT];
            float v = fa[r];
            const float vn = c0 * v + c1 * (dhy * rc.kxe + px - dhx * kye - py);  // Ez (boundaries.py:196-215)
            v = (rin && t_jin) ? vn : v;
            if ((rf & (R_SRCP | R_SRCM)) && t_src) v += src_term(rf, k);
            fa[r] = ((rf & R_XPEC) || t_zero) ? 0.f : v;
        } else {
            const float hz = fc[r];
            const float d = hz - nb_dn(xb, hz, r), d2 = hz - hm;
            float *qx = xps_e + r * NT + j, *qy = yqe + r * yse;
            const float ox = *qx, oy = *qy;
            const float py = bye * oy + cye * d, px = rc.bxe * ox + rc.cxe * d2;
            *qy = (rf & R_HOK) ? py : oy;
            *qx = t_hx ? px : ox;
            // Ex at (i+1/2, j) (boundaries.py:249-258)
            float e = fa[r] * (lossy ? csj[(r * NC + 2) * NT] : 1.f);
            const float en = e + csj[(r * NC) * NT] * (d * kye + py);
            e = t_jin ? en : e;
            e = t_jpec ? 0.f : e;
            fa[r] = ((rf & R_HOK) && t_jlt) ? e : fa[r];
            // Ey at (i, j+1/2) (:259-268)
            float e2 = fb[r] * (lossy ? csj[(r * NC + 3) * NT] : 1.f);
            const float e2n = e2 + (-csj[(r * NC + 1) * NT]) * (d2 * rc.kxe + px);
            e2 = rin ? e2n : e2;
            if ((rf & (R_SRCP | R_SRCM)) && t_src) e2 += src_term(rf, k);
            e2 = (rf & R_XPEC) ? 0.f : e2;
            fb[r] = t_hx ? e2 : fb[r];
        }
    };

    bool bad = false;
    for (int u = 0; u < nsteps; ++u) {
        const int m = n0 + u - B.n_start;  // the instance's own step
        const int k = m - tab.t0;
        // ------------------------------------------------------------ H phase
        if (lean) {
#pragma unroll
            for (int r = 0; r < RM; ++r) h_lean(r);
        } else {
#pragma unroll
            for (int r = 0; r < RM; ++r)
                if (r < R) h_gen(r);  // short bands (x strips, source rows) skip the template's spare rows
        }
        // the band's last row: the next band's first E row of the previous step
        float en = 0.f;
        if (bf & B_NEXT) {
            if (u == 0) en = e_next0;
            else if (!bad && !get_tag(h_next_e + ((u - 1) & 1) * NT, (unsigned)u, err, en, pl.tries)) bad = true;
        }
#pragma unroll
        for (int r = 0; r < RM; ++r) {
            if (r == R - 1) {
                if (lean) h_lean_last(r, en);
                else h_last(r, en);
                if (bf & B_NEXT) put_tag(h_my + hq + (u & 1) * NT, fc[r], (unsigned)(u + 1));
            }
        }
        if (lane == 31)
#pragma unroll
            for (int r = 0; r < RM; ++r) xb[r * RS_MAXW + w] = POL == 0 ? fb[r] : fc[r];
        if (__syncthreads_or(bad)) break;

        // ------------------------------------------------------------ E phase
        if (lean) {  // rows 1.. (row 0 after the previous band's H row)
#pragma unroll
            for (int r = 1; r < RM; ++r) e_lean(r, fc[r - 1]);
        } else {
#pragma unroll
            for (int r = 1; r < RM; ++r)
                if (r < R) e_row(r, fc[r - 1], k);
        }
        float hp = 0.f;  // the previous band's last H row of this step
        if ((bf & B_PREV) && !bad && !get_tag(h_prev_h + (u & 1) * NT, (unsigned)(u + 1), err, hp, pl.tries)) bad = true;
        if (lean) e_lean(0, hp);
        else e_row(0, hp, k);
        if ((bf & B_PREV) && !(cta == pl.wd_cta && u == 1))
            put_tag(h_my + (u & 1) * NT, POL == 0 ? fa[0] : fb[0], (unsigned)(u + 1));
        const bool win = B.dft && m >= B.dft_n0 && m < B.dft_n1;
        if (POL == 0 && win && (tf & T_JLT)) {  // node DFT of Ez
            const float pr = __ldg(tab.pe + 2 * k), pim = __ldg(tab.pe + 2 * k + 1);
#pragma unroll
            for (int r = 0; r < RM; ++r)
                if (r < R) dft_add(B.dft, bf & B_KAHAN, (size_t)(B.lo + r) * B.P + j, fa[r], pr, pim);
        }
        if (B.frames && (m + 1) % B.every == 0 && (m + 1) / B.every <= B.nframes) {
            const int nyf = POL == 0 ? ny : ny - 1;
            float *fr = B.frames + (size_t)((m + 1) / B.every - 1) * B.nx * nyf;
#pragma unroll
            for (int r = 0; r < RM; ++r)
                if (r < R && j < nyf) fr[(size_t)(B.lo + r) * nyf + j] = POL == 0 ? fa[r] : fb[r];
        }
        if (lane == 0)
#pragma unroll
            for (int r = 0; r < RM; ++r) zb[r * RS_MAXW + w] = fa[r];
        if (POL == 1 && lane == 31)
#pragma unroll
            for (int r = 0; r < RM; ++r) eb[r * RS_MAXW + w] = fb[r];
        if (__syncthreads_or(bad)) break;
        if (POL == 1 && win) {  // TM node DFT: Ey averaged onto the nodes (fdtd2d_core.py:458-465)
            const float pr = __ldg(tab.pe + 2 * k), pim = __ldg(tab.pe + 2 * k + 1);
#pragma unroll
            for (int r = 0; r < RM; ++r) {
                if (r < R) {
                    const float ey = fb[r];
                    const float eyl = nb_dn(eb, ey, r);
                    if (tf & T_JLT) {
                        const float v = j == 0 ? ey : (j == ny - 1 ? eyl : 0.5f * (eyl + ey));
                        dft_add(B.dft, bf & B_KAHAN, (size_t)(B.lo + r) * B.P + j, v, pr, pim);
                    }
                }
            }
        }
    }
    if (bad) atomicOr(err, 1);

    // ---- state out
#pragma unroll
    for (int r = 0; r < RM; ++r) {
        if (r < R && j < ny) {
            const size_t o = (size_t)(B.lo + r) * B.P + j;
            B.f[0][o] = fa[r];
            B.f[1][o] = fb[r];
            B.f[2][o] = fc[r];
        }
        if (r < R) {
            const RowC &rc = rowc[r];
            const int sh = (int)(short)(rc.sxh_sxe & 0xffff), se = rc.sxh_sxe >> 16;
            if (sh >= 0 && j < ny) B.pxh[(size_t)sh * B.P + j] = xps_h[r * NT + j];
            if (se >= 0 && j < ny) B.pxe[(size_t)se * B.P + j] = xps_e[r * NT + j];
            if (sjh >= 0) B.pyh[(size_t)(B.lo + r) * B.wyh + sjh] = yps_h[r * RS_MAXWY + sjh];
            if (sje >= 0) B.pye[(size_t)(B.lo + r) * B.wye + sje] = yps_e[r * RS_MAXWY + sje];
        }
    }
}

template <int RM, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 1)
    rs2d(const LensInst2D *__restrict__ insts, const RPlan pl, const LensStepTable tab, int n0, int nsteps,
         unsigned long long *halo, int *err) {
    extern __shared__ __align__(16) unsigned char smem[];
    int q = 0;
    while (q + 1 < pl.ninst && (int)blockIdx.x >= pl.first[q + 1]) ++q;
    if (__ldg(&insts[q].pol) == 0) rs_band<RM, 0>(insts, pl, tab, n0, nsteps, halo, err, smem);
    else rs_band<RM, 1>(insts, pl, tab, n0, nsteps, halo, err, smem);
}

constexpr int RS_NRM = 6;
constexpr int RS_RM[RS_NRM] = {8, 11, 12, 14, 16, 20};   // row templates (the wide launches: 12, 16, 20)

size_t rs_smem(int rm, int W, int nc) {
    const int NT = 32 * W;
    return (size_t)(rm * nc * NT + 2 * rm * NT + 2 * rm * RS_MAXWY + 4 * RS_MAXWY + 3 * rm * RS_MAXW + NT) * sizeof(float) +
           16 + rm * sizeof(RowC) + sizeof(Band);  // 16: the row constants' alignment
}

const void *rs_kernel(int rm, bool wide) {
    if (wide) {
        switch (rm) {
            case 12: return (const void *)rs2d<12, RS_NT_WIDE>;
            case 16: return (const void *)rs2d<16, RS_NT_WIDE>;
            case 20: return (const void *)rs2d<20, RS_NT_WIDE>;
            default: return nullptr;
        }
    }
    switch (rm) {
        case 8: return (const void *)rs2d<8, RS_NT_NARROW>;
        case 11: return (const void *)rs2d<11, RS_NT_NARROW>;
        case 12: return (const void *)rs2d<12, RS_NT_NARROW>;
        case 14: return (const void *)rs2d<14, RS_NT_NARROW>;
        case 16: return (const void *)rs2d<16, RS_NT_NARROW>;
        default: return (const void *)rs2d<20, RS_NT_NARROW>;
    }
}

bool rs_inst_ok(const LensInst2D &g) {
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

// Relative cost of a row: lean bands run the lean rows, a band holding any x
// strip, source or face row runs the general rows, so such bands get fewer
// rows.  3.4 is the ratio that gave the fastest step on the B200 (config 0:
// 4.26 us per step at 1.6, 3.79 at 2.4, 3.29 at 3.4 and at 4.0); it also
// covers a band's fixed costs (two barriers, two halo exchanges per step).
constexpr int RS_COST_LEAN = 10, RS_COST_SPECIAL = 34;

bool row_special(const LensInst2D &g, int i) {
    if (i <= 0 || i >= g.nx - 1) return true;  // faces (and the row without Hy / Hz)
    if (g.src.ix >= 0 && (i == g.src.ix || i == g.src.ix + 1)) return true;
    const LensProfile &h = g.ax.h, &e = g.ax.e;
    return i < h.lo || i >= h.n - h.hi || i < e.lo || i >= e.n - e.hi;  // in an x strip (H or E psi)
}

// Bands of instance g with cost at most T and at most rmx rows each (greedy:
// every band as long as it may be); their first rows into lo (when not NULL).
int rs_bands(const LensInst2D &g, int T, int rmx, short *lo) {
    int n = 0;
    for (int i = 0; i < g.nx;) {
        int r = 0;
        bool sp = false;
        while (i + r < g.nx && r < rmx) {
            const bool sp2 = sp || row_special(g, i + r);
            if (r > 0 && (r + 1) * (sp2 ? RS_COST_SPECIAL : RS_COST_LEAN) > T) break;
            sp = sp2;
            ++r;
        }
        if (lo) lo[n] = (short)i;
        ++n;
        i += r;
    }
    return n;
}

// The least band cost T with which the instances' bands (at most rmx rows each)
// number at most avail; -1 when none does.
int rs_threshold(const LensInst2D *inst, int ninst, int avail, int rmx) {
    auto count = [&](int T) {
        long n = 0;
        for (int q = 0; q < ninst; ++q) n += rs_bands(inst[q], T, rmx, nullptr);
        return n;
    };
    int hi_t = rmx * RS_COST_SPECIAL;  // every band at most rmx rows
    if (avail < 1 || count(hi_t) > avail) return -1;
    int lo_t = RS_COST_LEAN - 1;        // infeasible: one lean row per band is the least
    while (hi_t - lo_t > 1) {
        const int mid = (lo_t + hi_t) / 2;
        if (count(mid) <= avail) hi_t = mid;
        else lo_t = mid;
    }
    return hi_t;
}

// Plan of a resident group on this device: the row template RM, the most rows of
// a band, warps per CTA, the CTA count, the coefficients per row and (when lo is
// not NULL) the first row of every band, instance after instance.  The bands
// minimise the largest band cost within the SMs' resident CTAs.  LENS_ERR_SIZE
// when the group does not fit.
int rs_plan(const LensInst2D *inst, int ninst, int &rm, int &rows, int &W, int &nctas, int &nc, short *lo) {
    if (!inst || ninst < 1 || ninst > LENS_RS_MAX_INST) return ninst > LENS_RS_MAX_INST ? LENS_ERR_SIZE : LENS_ERR_ARG;
    int ny_max = 0;
    nc = 2;
    for (int q = 0; q < ninst; ++q) {
        if (!rs_inst_ok(inst[q])) return LENS_ERR_ARG;
        const LensInst2D &g = inst[q];
        if (g.ay.e.lo + g.ay.e.hi > RS_MAXWY || g.ay.h.lo + g.ay.h.hi > RS_MAXWY || g.nx > 32767) return LENS_ERR_SIZE;
        ny_max = std::max(ny_max, g.ny);
        if (g.pol == 1 && g.c[2]) nc = 4;
    }
    W = (ny_max + 31) / 32;
    if (W > RS_MAXW) return LENS_ERR_SIZE;
    int dev = 0, nsm = 0, smax = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return LENS_ERR_CUDA;
    const bool wide = 32 * W > RS_NT_NARROW;
    int best_t = -1, best_rm = 0;
    for (int t = 0; t < RS_NRM; ++t) {
        const int cand = RS_RM[t];
        const void *k = rs_kernel(cand, wide);
        const size_t sm = rs_smem(cand, W, nc);
        if (!k || sm > (size_t)smax) continue;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
            return LENS_ERR_CUDA;
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 32 * W, sm) != cudaSuccess) return LENS_ERR_CUDA;
        const long avail = std::min((long)per * nsm, (long)RS_MAXCTA);
        const int tt = rs_threshold(inst, ninst, (int)avail, cand);
        if (tt > 0 && (best_t < 0 || tt < best_t)) {
            best_t = tt;
            best_rm = cand;
        }
    }
    if (best_t < 0) return LENS_ERR_SIZE;
    rm = best_rm;
    nctas = 0;
    rows = 0;
    for (int q = 0; q < ninst; ++q) {
        short tmp[RS_MAXCTA];
        const int n = rs_bands(inst[q], best_t, rm, tmp);
        for (int b = 0; b < n; ++b) {
            const int end = b + 1 < n ? tmp[b + 1] : inst[q].nx;
            rows = std::max(rows, end - tmp[b]);
            if (lo) lo[nctas + b] = tmp[b];
        }
        nctas += n;
    }
    return LENS_OK;
}

}  // namespace

extern "C" int lens_rs2d_plan(const LensInst2D *inst, int ninst, int *rows, int *ctas, int *threads) {
    int rm = 0, r = 0, W = 0, n = 0, nc = 0;
    const int st = rs_plan(inst, ninst, rm, r, W, n, nc, nullptr);
    if (st != LENS_OK) {
        cudaGetLastError();
        return st;
    }
    if (rows) *rows = r;
    if (ctas) *ctas = n;
    if (threads) *threads = 32 * W;
    return LENS_OK;
}

extern "C" int lens_rs2d_bands(const LensInst2D *inst, int ninst, int ctas, int max_rows, short *first_rows,
                               int capacity) {
    if (!inst || ninst < 1 || ctas < 1 || max_rows < 1 || !first_rows || capacity < 1) return LENS_ERR_ARG;
    for (int q = 0; q < ninst; ++q)
        if (!rs_inst_ok(inst[q]) || inst[q].nx > 32767) return LENS_ERR_ARG;
    const int T = rs_threshold(inst, ninst, std::min(ctas, capacity), max_rows);
    if (T < 0) return LENS_ERR_SIZE;
    int n = 0;
    for (int q = 0; q < ninst; ++q) n += rs_bands(inst[q], T, max_rows, first_rows + n);
    return n;
}

extern "C" size_t lens_rs2d_scratch_bytes(int ctas, int threads) {
    if (ctas < 1 || threads < 1) return 0;
    return (size_t)ctas * 4 * (size_t)threads * sizeof(unsigned long long);
}

namespace {

int rs_run(const LensInst2D *inst_host, const LensInst2D *inst_dev, const LensRsOut2D *out, int ninst,
           const LensStepTable *tab, int n0, int nsteps, void *scratch, size_t scratch_bytes, int *err, void *stream,
           long long tries, int wd) {
    if (!inst_host || !inst_dev || !scratch || !err || nsteps < 0) return LENS_ERR_ARG;
    int rm = 0, rows = 0, W = 0, nctas = 0, nc = 0;
    RPlan pl{};
    int st = rs_plan(inst_host, ninst, rm, rows, W, nctas, nc, pl.lo);
    if (st != LENS_OK) {
        cudaGetLastError();
        return st;
    }
    bool any_dft = false;
    for (int q = 0; q < ninst; ++q) {
        const LensInst2D &g = inst_host[q];
        if (n0 < g.n_start || !lens_table_ok(tab, n0 - g.n_start, nsteps)) return LENS_ERR_ARG;
        any_dft = any_dft || g.dft;
        if (out && out[q].frames && (out[q].every < 1 || out[q].nframes < 0)) return LENS_ERR_ARG;
    }
    if (any_dft && !tab->pe) return LENS_ERR_ARG;
    if (scratch_bytes < lens_rs2d_scratch_bytes(nctas, 32 * W)) return LENS_ERR_SIZE;
    if (nsteps == 0) return LENS_OK;
    int dev = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        !coop) {
        cudaGetLastError();
        return LENS_ERR_CUDA;
    }
    pl.ninst = ninst;
    pl.tries = tries;
    pl.wd_cta = -1;
    if (wd) {  // the second band of the first instance withholds a row: it must exist
        if (nctas < 2 || nsteps < 3 || inst_host[0].nx <= pl.lo[1]) return LENS_ERR_ARG;
        pl.wd_cta = 1;
    }
    pl.rows = rows;
    pl.nc = nc;
    int c = 0;
    for (int q = 0; q < ninst; ++q) {
        pl.first[q] = c;
        while (c < nctas && (c == pl.first[q] || pl.lo[c] != 0)) ++c;  // the next instance's bands start at row 0
        pl.out[q] = out ? out[q] : LensRsOut2D{nullptr, 0, 0, 0};
    }
    pl.first[ninst] = c;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(scratch, 0, lens_rs2d_scratch_bytes(nctas, 32 * W), s) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess)
        return LENS_ERR_CUDA;
    LensStepTable t = *tab;
    unsigned long long *halo = static_cast<unsigned long long *>(scratch);
    void *args[] = {(void *)&inst_dev, (void *)&pl, (void *)&t, (void *)&n0, (void *)&nsteps, (void *)&halo,
                    (void *)&err};
    if (cudaLaunchCooperativeKernel(rs_kernel(rm, 32 * W > RS_NT_NARROW), dim3(nctas), dim3(32, W), args,
                                    rs_smem(rm, W, nc), s) != cudaSuccess) {
        cudaGetLastError();
        return LENS_ERR_CUDA;
    }
    return lens_cuda_status();
}

}  // namespace

extern "C" int lens_rs2d_run(const LensInst2D *inst_host, const LensInst2D *inst_dev, const LensRsOut2D *out,
                             int ninst, const LensStepTable *tab, int n0, int nsteps, void *scratch,
                             size_t scratch_bytes, int *err, void *stream) {
    return rs_run(inst_host, inst_dev, out, ninst, tab, n0, nsteps, scratch, scratch_bytes, err, stream, RS_TRIES, 0);
}

// Watchdog self-test: the same launch with every wait cut to 1024 polls and the
// second band of the first instance withholding its first E row of step 1, so
// the first band's wait at step 2 runs out; *err must become nonzero, every
// CTA must leave its step loop and the stream stays usable.
extern "C" int lens_rs2d_watchdog_test(const LensInst2D *inst_host, const LensInst2D *inst_dev, int ninst,
                                       const LensStepTable *tab, int n0, int nsteps, void *scratch,
                                       size_t scratch_bytes, int *err, void *stream) {
    return rs_run(inst_host, inst_dev, nullptr, ninst, tab, n0, nsteps, scratch, scratch_bytes, err, stream, 1024, 1);
}
