/*
 * lens_fdtd.h - C ABI of the B200 (sm_100a) FDTD time-stepping engine.
 *
 * Drop-in for the hot loop of s1alknau/lens_sensor's native solver:
 *   2D TE  CPML step   planar_beads/boundaries.py:164-221 (CPML_TE.update_H/update_E/terminate)
 *                      planar_beads/fused2d.py:41-68, 105-115 (te_update_H / te_update_E)
 *   2D TM  CPML step   planar_beads/boundaries.py:224-274, fused2d.py:69-94, 118-126
 *                      + loss damping planar_beads/fdtd2d_core.py:796-797
 *   3D     CPML step   planar_3d/boundaries3d.py:262-362 (CPML_3D.step/step_H/step_E)
 *   source             common/vcsel.py:151-156 (HuygensSource.inject)
 *   epilogues          planar_beads/fdtd2d_core.py:834-850, planar_3d/fdtd3d_core.py:1139-1158,
 *                      common/flux.py:19-57 (PlaneFluxDFT.add)
 *
 * Conventions
 *  - Plain C: no CUDA or torch types.  Every pointer is a DEVICE pointer owned by
 *    the caller (the Python host allocates with PyTorch); the library allocates
 *    nothing and keeps no global state, so distinct solves are independent.
 *  - Every entry point returns an int status (LENS_OK = 0, negative on error) and
 *    never aborts.  `stream` is a cudaStream_t passed as void* (NULL = legacy
 *    default stream); all work is enqueued on it asynchronously.
 *  - Layout: every 2D array of a grid is stored as nx rows of `pitch` floats
 *    (pitch >= ny, multiple of 32); every 3D array as nx*ny rows of `pitch`
 *    floats along z (pitch >= nz, multiple of 32).  A staggered component
 *    occupies the leading part of its rows (e.g. 2D Hx = (nx, ny-1)); padding is
 *    never read for a valid update and stays zero.
 *  - CPML psi is updated only in the strips where the profile's c != 0 (leading
 *    `lo` and trailing `hi` entries of the profile); the 2D strip arrays and the
 *    3D psi volumes are documented with each grid.  Outside the strips psi is
 *    identically zero.  A profile with a strip (lo + hi > 0) needs the psi
 *    arrays that strip serves; a NULL one is refused with LENS_ERR_ARG before
 *    anything is launched.
 */
#ifndef LENS_FDTD_H
#define LENS_FDTD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LENS_OK 0
#define LENS_ERR_ARG (-1)
#define LENS_ERR_CUDA (-2)
#define LENS_ERR_SIZE (-3)

#define LENS_MAX_CTYPE 4
#define LENS_MAX_BOX 4
#define LENS_MAX_PLANE 4

/* One staggering of one CPML axis: b, c and 1/kappa, each of length n. */
typedef struct {
    const float *b, *c, *ik;
    int n;      /* profile length (N integer nodes, or N-1 half nodes) */
    int lo, hi; /* psi strip widths: entries [0,lo) and [n-hi,n) carry psi */
} LensProfile;

typedef struct {
    LensProfile e; /* integer nodes, length N     (boundaries.py:104-151 "e") */
    LensProfile h; /* half nodes,    length N - 1 (boundaries.py:104-151 "h") */
} LensAxis;

/* Per-step scalars computed once on the host (float64 math, float32 stored).
 * Step n reads entry n - t0 (0 <= n - t0 < n_table). */
typedef struct {
    const float *wt;  /* float32(omega * n * dt)        (vcsel.py:154-155)       */
    const float *env; /* source envelope at t = n*dt    (fdtd2d_core.py:784-787)  */
    const float *pe;  /* (re, im) of exp(-i w t_n)              : DFT of E       */
    const float *ph;  /* (re, im) of exp(-i w (t_n - dt/2))     : DFT of H (flux) */
    int t0, n_table;
} LensStepTable;

/* One-way Huygens soft-source pair on x-planes ix (+) and ix+1 (-). */
typedef struct {
    int ix;                        /* -1: no source                       */
    const float *amp, *ph1, *ph2;  /* 2D: length nj; 3D: (nj, pitch_k)    */
    int nj, nk, pitch_k;           /* source plane extent (2D: nk = 1)    */
} LensSource;

/* ---------------------------------------------------------------- 2D grids */
typedef struct {
    int nx, ny, pitch;           /* node counts; row pitch of every array      */
    float *ez, *hx, *hy;         /* Ez (nx,ny) Hx (nx,ny-1) Hy (nx-1,ny)       */
    const float *ce_e, *ce_h;    /* Ce_E, Ce_H (nx,ny)  fdtd2d_core.py:262-270 */
    float ch;                    /* dt/(mu0 dx)                                */
    LensAxis ax, ay;
    float *psi_hxy;              /* (nx, ay.h.lo+ay.h.hi)                      */
    float *psi_hyx;              /* (ax.h.lo+ax.h.hi, pitch)                   */
    float *psi_ezx;              /* (ax.e.lo+ax.e.hi, pitch)                   */
    float *psi_ezy;              /* (nx, ay.e.lo+ay.e.hi)                      */
    int pec[4];                  /* PEC on x-lo, x-hi, y-lo, y-hi              */
    LensSource src;              /* drives Ez                                  */
} LensTE2D;

typedef struct {
    int nx, ny, pitch;
    float *ex, *ey, *hz;         /* Ex (nx-1,ny) Ey (nx,ny-1) Hz (nx-1,ny-1)   */
    const float *ca_x, *ca_y;    /* Ca_ex (nx-1,ny) Ca_ey (nx,ny-1)            */
    const float *da_x, *da_y;    /* loss damping D or NULL (lossless)          */
    float ch;
    LensAxis ax, ay;
    float *psi_hzx;              /* (ax.h.lo+ax.h.hi, pitch)                   */
    float *psi_hzy;              /* (nx, ay.h.lo+ay.h.hi)                      */
    float *psi_exy;              /* (nx, ay.e.lo+ay.e.hi)                      */
    float *psi_eyx;              /* (ax.e.lo+ax.e.hi, pitch)                   */
    int pec[4];
    LensSource src;              /* drives Ey (source on the Ey grid)          */
} LensTM2D;

/* Epilogue of a 2D step (all optional; a NULL pointer or empty window = off).
 * "field" is Ez (TE) or Ey averaged onto the nodes (TM, fdtd2d_core.py:458-465);
 * I = |E|^2 on the nodes (TE Ez^2, TM field^2 + <Ex^2> fdtd2d_core.py:477-486). */
typedef struct {
    int nbox;
    int box[LENS_MAX_BOX][4];    /* [x0,x1) x [y0,y1) on the nodes            */
    double *box_acc;             /* nbox float64 sums of I, added every step  */
    int dft_n0, dft_n1;          /* steps [n0,n1): acc += field * pe[n]        */
    float *dft;                  /* (nx, pitch) x {re, im, c_re, c_im}: Kahan  */
    float *dft_ex;               /* TM: same for Ex on the nodes, or NULL      */
    int prev_n0, prev_n1;        /* second window (CW convergence test)        */
    float *dft_prev;             /* same layout as dft, or NULL                */
    int iavg_n0;                 /* steps >= iavg_n0: iavg += I                */
    float *iavg;                 /* (nx, pitch) or NULL                        */
    int nplane;
    int plane[LENS_MAX_PLANE];   /* x-planes il (1 <= il <= nx-2)              */
    double *plane_acc;           /* per plane: 4 rows of pitch doubles:
                                    E re, E im, H re, H im (H = mean of il-1, il);
                                    accumulated during the dft window          */
    float *dft_raw;              /* TM: Ey on its own grid (nx, pitch), Kahan
                                    layout as dft, during the dft window, or NULL */
    float *ex2;                  /* TM: Ex^2 on the nodes summed during the dft
                                    window (nx, pitch), or NULL                */
    int nsx;                     /* time-domain Poynting planes (every step)   */
    int sx_plane[LENS_MAX_PLANE];/* x-planes il (1 <= il <= nx-2)              */
    double *sx_acc;              /* per plane: pitch doubles, acc[j] += the
                                    FP32 product E(il,j) * (H(il-1,j) + H(il,j))/2
                                    (TE Ez*Hy, TM Ey*Hz; the TE flux is minus the
                                    sum, fdtd2d_core.py:489-497)              */
} LensEpi2D;

/* Advance `nsteps` steps starting at step n0 (t = n*dt, n = n0 ... n0+nsteps-1). */
int lens_te2d_step(const LensTE2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                   int n0, int nsteps, void *stream);
int lens_tm2d_step(const LensTM2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                   int n0, int nsteps, void *stream);

/* Stitch-window drive of a 2D grid (fdtd2d_core.py:1439-1440, 1462-1463): after
 * each E update, before the PEC termination, the first nplanes x-rows of the
 * driven component (TE: Ez, TM: Ey) become
 *     w_i * (env * Re(D e^{+i w t})) + (1 - w_i) * E
 * evaluated as the reference does: the complex64 amplitude D times the
 * complex128 phase in FP64, w_i * (...) in FP64, (1 - w_i) * E in FP32, the sum
 * rounded to FP32.                                                          */
typedef struct {
    int nplanes;                 /* O driven rows (0: no drive)                */
    const float *taper;          /* O weights w_i                              */
    const float *hand;           /* (O, pitch) x {re, im}: complex amplitudes   */
    const double *tab;           /* per step n - t0: env, cos(w t), sin(w t)    */
} LensDrive2D;

/* lens_te2d_step / lens_tm2d_step with a stitch drive (no counterpart entry in
 * the reference: its stitch loop assigns the overlap rows in NumPy).         */
int lens_te2d_step_driven(const LensTE2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                          const LensDrive2D *drive, int n0, int nsteps, void *stream);
int lens_tm2d_step_driven(const LensTM2D *g, const LensStepTable *tab, const LensEpi2D *ep,
                          const LensDrive2D *drive, int n0, int nsteps, void *stream);

/* ------------------------------------------------------- batched 2D solves
 * Many independent 2D solves of uneven sizes (TE and TM mixed) advanced together:
 * one launch per half step covers every tile of every instance, so a sweep of
 * small grids runs at the memory rate instead of the launch rate, and a span of
 * steps can be captured into one CUDA graph by the caller.  Field storage is
 * FP32, FP16 or BF16 for the whole batch (arithmetic is FP32 throughout);
 * coefficients, CPML psi and the DFT stay FP32.  The per-cell update is the one
 * of lens_te2d_step / lens_tm2d_step; the epilogue is the node-field DFT
 * (Ez for TE, Ey averaged onto the nodes for TM) over [dft_n0, dft_n1).    */
#define LENS_F32 0
#define LENS_F16 1
#define LENS_BF16 2

typedef struct {
    int pol;                     /* 0 TE (Ez, Hx, Hy), 1 TM (Ex, Ey, Hz)       */
    int nx, ny, pitch;
    void *f[3];                  /* TE ez, hx, hy / TM ex, ey, hz (storage type) */
    const float *c[4];           /* TE ce_e, ce_h / TM ca_x, ca_y, da_x, da_y   */
    float ch;
    LensAxis ax, ay;
    float *psi[4];               /* TE hxy, hyx, ezx, ezy / TM hzx, hzy, exy, eyx
                                    (shapes as in LensTE2D / LensTM2D)          */
    int pec[4];
    LensSource src;              /* drives Ez (TE) or Ey (TM)                   */
    int dft_n0, dft_n1;          /* in the instance's own steps                 */
    float *dft;                  /* (nx, pitch) x {re, im} or NULL              */
    int n_start;                 /* batch step at which this instance's step 0
                                    runs: its own step is n - n_start (source
                                    time, DFT window, table row), so instances
                                    can join a batch that is already running    */
    /* Optional row form of the coefficients (NULL rtype: every row from c[]).
       A layered instance repeats a few coefficient rows (over y) on almost
       every x row: rtype[i] < ntype names row i's type in ctab, laid out
       (type, coefficient q, pitch); 255 reads row i from c[].  Values are
       c[]'s own, bit for bit.                                                */
    const unsigned char *rtype;  /* (nx) or NULL                                */
    const float *ctab;           /* (ntype, ncoef, pitch), ncoef = TE 2 / TM 2
                                    or 4 (with damping)                       */
} LensInst2D;

/* Block plan of a batch for tiles of 128 columns x 2*by rows: writes blk[0..ninst]
 * (first block of each instance) and, when owner is not NULL, owner[b] (the
 * instance of block b, one entry per block); returns the block count, or < 0. */
int lens_batch2d_plan(const LensInst2D *inst, int ninst, int by, int *blk, int *owner);

/* Advance every instance by nsteps from batch step n0.  inst_host / inst_dev:
 * the same instance array in host and device memory; blk_dev / owner_dev: the
 * plan's tables in device memory; storage: LENS_F32 / LENS_F16 / LENS_BF16.
 * The table must hold every instance's own steps [n0 - n_start, n0 + nsteps -
 * n_start).                                                                  */
int lens_batch2d_step(const LensInst2D *inst_host, const LensInst2D *inst_dev, const int *blk_dev,
                      const int *owner_dev, int ninst, int storage, int by, const LensStepTable *tab,
                      int n0, int nsteps, void *stream);

/* The same steps as lens_batch2d_step in ONE persistent cooperative launch:
 * every resident block strides over the batch's tiles, phase by phase (H, E,
 * and the TM node DFT on its window steps), and the blocks meet at a grid
 * barrier between phases, so a batch whose state fits in L2 keeps it there
 * across steps and no launch gap separates the steps.  sync: 2 device words of
 * barrier state and err: a device int, both the caller's (zeroed by the call
 * on `stream` before the launch).  Every barrier wait is bounded (about a
 * second); if one runs out *err becomes nonzero, the launch ends and the
 * results are invalid.  The device must support cooperative launches.  No
 * counterpart entry in the reference (its loop advances one step per call,
 * fdtd2d_core.py:781-847).                                                   */
int lens_batch2d_run(const LensInst2D *inst_host, const LensInst2D *inst_dev, const int *blk_dev,
                     const int *owner_dev, int ninst, int storage, int by, const LensStepTable *tab, int n0,
                     int nsteps, unsigned *sync, int *err, void *stream);

/* Same step as lens_batch2d_step for callers that cannot allocate device
 * memory (an application that owns the GPU allocator, a fixed memory budget, a
 * loop where cudaMalloc's implicit synchronisation is not allowed).  No
 * counterpart in the reference.  The descriptors (inst, in host memory), the
 * block offsets and the owner table are placed in one fixed device array of
 * about 8.6 MB that every GPU loading this library holds until the process
 * exits; at most 512 instances and 2^21 tiles (128 x 2*by nodes each) per call,
 * larger calls return LENS_ERR_SIZE.  Nothing is allocated.  The first call on
 * a device looks up that array's device address and keeps it for the life of
 * the process (a cudaDeviceReset of that device invalidates it: do not reset a
 * device that has run this call).  inst is copied to the device with
 * cudaMemcpyAsync on `stream`: from pageable memory the copy is staged before
 * the call returns, from page-locked memory it runs later, so a page-locked inst
 * must stay unchanged until the stream has reached the call.  The call is not
 * capturable: on a stream that is capturing it returns LENS_ERR_ARG before
 * anything is enqueued.  Every call rewrites the whole array (nothing carries
 * over between calls), so calls that overlap on the GPU (other streams, other
 * threads) race on it; the fields, psi and DFT buffers are the caller's as
 * usual.                                                                     */
int lens_batch2d_step_noalloc(const LensInst2D *inst, int ninst, int storage, int by,
                              const LensStepTable *tab, int n0, int nsteps, void *stream);

/* ------------------------------------------- temporally blocked 2D solves
 * The batched 2D step with LENS_TB_K time steps per launch: each field value
 * crosses HBM once per K steps instead of once per step.  A warp streams a tile
 * of 128 columns (y) down a chunk of rows (x) and advances K time levels held
 * in registers, one row behind the other; the K columns on each side of the
 * tile and the K rows before and after the chunk are recomputed halo.  Fields
 * and psi are double-buffered: a launch reads buffer `b` and writes buffer
 * 1 - b, starting from buffer 0, so nsteps must be a multiple of 2*K and the
 * state ends in buffer 0 again.  The CPML psi of the K-1 intermediate levels
 * live in a scratch array.  Epilogue: the node-field DFT of LensInst2D (Ez for
 * TE, Ey on the nodes for TM) over its window, accumulated as (re, im) or, with
 * dft_kahan, compensated (re, im, c_re, c_im) as the single-grid epilogue
 * does.  Every instance must have started (n_start <= n0).                  */
#define LENS_TB_K 4

typedef struct {
    LensInst2D g;                /* the instance; g.f and g.psi are buffer 0    */
    void *f1[3];                 /* buffer 1 of the fields (same layout as g.f) */
    float *psi1[4];              /* buffer 1 of the psi arrays (shapes of g.psi) */
    float *psi_lv;               /* scratch of the intermediate psi levels:
                                    (LENS_TB_K - 1) x the sum of the four psi
                                    array sizes (x strips w x pitch, y strips
                                    nx x w; an empty strip takes no space), or
                                    NULL when the instance has no strip        */
    int dft_kahan;               /* g.dft layout: 1 (re, im, c_re, c_im), 0 (re, im) */
} LensTB2D;

/* Units (warps) of a temporally blocked batch with row chunks of `chunk` rows:
 * writes first[0..ninst] (first unit of each instance) and returns the unit
 * count, or < 0. */
int lens_tb2d_plan(const LensTB2D *inst, int ninst, int chunk, int *first);

/* Advance every instance by nsteps (a multiple of 2 * LENS_TB_K) from batch
 * step n0, LENS_TB_K steps per launch.  inst_host / inst_dev: the same
 * descriptors in host and device memory; first_dev: the plan's first[] in
 * device memory; storage: LENS_F32 / LENS_F16 / LENS_BF16 (all arithmetic
 * FP32).  Replaces the per-step loop of fdtd2d_core.py:781-847 (no counterpart
 * entry in the reference, which advances one step per call).                */
int lens_tb2d_step(const LensTB2D *inst_host, const LensTB2D *inst_dev, const int *first_dev, int ninst,
                   int chunk, int storage, const LensStepTable *tab, int n0, int nsteps, void *stream);

/* ------------------------------------------------- resident 2D solves
 * A group of FP32 instances whose state fits on the chip, advanced by nsteps
 * in ONE cooperative launch that keeps every field value in registers from the
 * first step to the last: a CTA owns a band of x rows of one instance (every y
 * column, ny <= 576), and neighbouring bands exchange one row per half step
 * through L2 as {value, step tag} words.  No counterpart entry in the
 * reference (its loop advances one step per call, fdtd2d_core.py:781-847);
 * the per-cell update is lens_batch2d_step's.  Outputs per instance: the node
 * DFT into g.dft over [dft_n0, dft_n1) as (re, im), or compensated (re, im,
 * c_re, c_im) with kahan = 1, and optional snapshot frames of the driven raw
 * component (TE Ez (nx, ny), TM Ey (nx, ny - 1)): frame f holds the field after
 * the instance's own step (f + 1) * every - 1.  Every instance must have started
 * (n_start <= n0).  Waits between bands are bounded (a few seconds at most); if
 * one runs out *err becomes nonzero, the launch ends and the results are
 * invalid.                                                                   */
#define LENS_RS_MAX_INST 32

typedef struct {
    float *frames;      /* NULL: none                                          */
    int every, nframes; /* frame cadence (own steps) and the frames' count     */
    int kahan;          /* g.dft layout: 1 (re, im, c_re, c_im), 0 (re, im)    */
} LensRsOut2D;

/* Band plan on the current device: rows per band, CTAs and threads per CTA;
 * LENS_ERR_SIZE when the group does not fit on the chip (more bands than
 * resident CTAs at 20 rows per band, ny > 576, a y strip wider than 64, or
 * more than LENS_RS_MAX_INST instances).                                     */
int lens_rs2d_plan(const LensInst2D *inst, int ninst, int *rows, int *ctas, int *threads);

/* The plan's band partition, host only (no device is touched): the instances'
 * rows cut into at most `ctas` bands of at most max_rows rows, a row of an x
 * CPML strip, a source row or a face row costing 3.4 rows elsewhere, the
 * largest band cost as small as it can be.  Writes the first row of every band,
 * instance after instance, into first_rows (capacity entries) and returns the
 * band count; LENS_ERR_SIZE when the rows do not fit.                        */
int lens_rs2d_bands(const LensInst2D *inst, int ninst, int ctas, int max_rows, short *first_rows, int capacity);

/* Bytes of the halo scratch of a plan (device memory, the caller's).        */
size_t lens_rs2d_scratch_bytes(int ctas, int threads);

/* Advance every instance by nsteps from batch step n0.  inst_host / inst_dev:
 * the same descriptors in host and device memory; out: NULL or ninst entries
 * (host memory); scratch: scratch_bytes of device memory; err: a device int.
 * The call zeroes scratch and *err on `stream` before the launch.  The launch
 * occupies every SM it plans for (one band per SM) and its bands wait on each
 * other: issue resident launches one after another (one stream, or streams
 * ordered by events), not side by side with other long-running work.         */
int lens_rs2d_run(const LensInst2D *inst_host, const LensInst2D *inst_dev, const LensRsOut2D *out, int ninst,
                  const LensStepTable *tab, int n0, int nsteps, void *scratch, size_t scratch_bytes, int *err,
                  void *stream);

/* Watchdog self-test of the waits between bands (no counterpart in the
 * reference): lens_rs2d_run's launch with every wait cut to 1024 polls and the
 * second band of the first instance withholding its first E row of step 1.
 * The first band's wait at step 2 runs out, *err becomes nonzero and every CTA
 * leaves its step loop (no fault, no hang).  Needs a first instance of two or
 * more bands and nsteps >= 3; the fields are left invalid.                   */
int lens_rs2d_watchdog_test(const LensInst2D *inst_host, const LensInst2D *inst_dev, int ninst,
                            const LensStepTable *tab, int n0, int nsteps, void *scratch, size_t scratch_bytes,
                            int *err, void *stream);

/* ---------------------------------------------------------------- 3D grid */
/* psi arrays of the 3D CPML (boundaries3d.py:286-302), in this order.  Each is a
 * full (nx, ny, pitch) volume like the fields, so a CTA stages psi with the same
 * TMA tiles as the fields; only cells inside the strip of the named profile are
 * ever read or written (elsewhere psi is identically zero).                    */
enum {
    LENS_PSI_HX_Z, LENS_PSI_HX_Y, LENS_PSI_HY_X, LENS_PSI_HY_Z, LENS_PSI_HZ_Y, LENS_PSI_HZ_X,
    LENS_PSI_EX_Y, LENS_PSI_EX_Z, LENS_PSI_EY_Z, LENS_PSI_EY_X, LENS_PSI_EZ_X, LENS_PSI_EZ_Y,
    LENS_NPSI
};

typedef struct {
    int nx, ny, nz, pitch;       /* node counts; z pitch of every array        */
    /* Field buffers b = 0, 1: f[b] = {Ex, Ey, Ez, Hx, Hy, Hz} with
       Ex (nx-1,ny,nz) Ey (nx,ny-1,nz) Ez (nx,ny,nz-1)
       Hx (nx,ny-1,nz-1) Hy (nx-1,ny,nz-1) Hz (nx-1,ny-1,nz).
       With buffer 1 present (all six pointers and all psi[1]) a step reads
       buffer `cur`, writes buffer 1-cur in one fused pass and flips `cur`;
       with buffer 1 NULL the step updates buffer `cur` in place (two passes). */
    float *f[2][6];
    float *psi[2][LENS_NPSI];
    int cur;
    const float *ce_x, *ce_y, *ce_z;  /* staggered update factors (fdtd3d_core.py:305-378) */
    const float *da_x, *da_y, *da_z;  /* staggered loss damping or NULL (fdtd3d_core.py:606-613) */
    float ch;
    LensAxis ax, ay, az;
    int pec[6];                  /* PEC on x-lo, x-hi, y-lo, y-hi, z-lo, z-hi  */
    LensSource src;              /* plane (nj, nk) of the driven component     */
    int src_comp;                /* 0 Ex, 1 Ey, 2 Ez                           */
    int *flag;                   /* optional device int: bit 1 set when a
                                    pipeline wait gave up, bit 2 when a detector
                                    box sum was not finite (results invalid)   */
    /* Optional column form of the six coefficient volumes (NULL ctype: the
       fused step reads every coefficient from the volumes).  A layered slab
       repeats a few coefficient columns (over y) at almost every (x, z): the
       fused step then reads those from ctab and the volumes only where
       ctype == 255.  Values are the volumes' own, bit for bit.              */
    const unsigned char *ctype;  /* (nx, pitch): column type 0..ntype-1 of the
                                    cells (i, *, k), or 255 (read the volumes) */
    const float *ctab;           /* (ntype, 6, ny): ce_x, ce_y, ce_z, D_x, D_y,
                                    D_z down each column type                  */
    const unsigned char *cexpl;  /* (nx, pitch/32): nonzero where the 32-column
                                    group of plane i holds a type-255 column   */
    int ntype;                   /* 1..4 (LENS_MAX_CTYPE)                      */
} LensGrid3D;

typedef struct {
    int nbox;
    int box[LENS_MAX_BOX][6];    /* [x0,x1) [y0,y1) [z0,z1), applied to Ex, Ey, Ez; an end
                                    < 0 counts from each component's own end (numpy
                                    slice(a, -b), fdtd3d_core.py:1139-1142)           */
    double *box_acc;             /* nbox sums of Ex^2+Ey^2+Ez^2 (fdtd3d_core.py:477-481) */
    int dft_n0, dft_n1;
    float *dft[3];               /* per component (or NULL): (nx,ny,pitch) x {re,im} */
    int conv_k;                  /* z index of the convergence plane (driven component) */
    int prev_n0, prev_n1;        /* previous window for the convergence test */
    float *conv_prev, *conv_last;/* (nx, nj) x {re,im,c_re,c_im} planes or NULL */
    int nplane;
    int plane[LENS_MAX_PLANE];
    double *plane_acc;           /* per plane: 2 pairs (Ey/Hz, Ez/Hy) x 4 x (ny*pitch) doubles */
} LensEpi3D;

/* Stitch-window drive (fdtd3d_core.py:1614-1617): after each E update the first
 * nplanes x-planes of Ex, Ey and Ez become
 *     w_i * (env * Re(D e^{+i w t})) + (1 - w_i) * E
 * with D the complex amplitude handed over from the previous window.          */
typedef struct {
    int nplanes;                 /* O: driven planes, 1 <= O <= nx-1            */
    const float *taper;          /* 2*O floats: w_0..w_{O-1}, then 1-w_0..1-w_{O-1} */
    const float *hand[3];        /* Ex, Ey, Ez amplitudes: (O, ny, pitch) x {re, im} */
} LensDrive3D;

/* Advance nsteps; updates g->cur when the fused (double-buffered) path runs. */
int lens_fdtd3d_step(LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep,
                     int n0, int nsteps, void *stream);

/* The same steps with the stitch drive applied to every new E before the
 * epilogue reads it (replaces the per-step overlap assignment of
 * fdtd3d_core.py:1611-1617 in run_3d_stitched).  The epilogue may hold DFT
 * windows, flux planes and convergence planes but no detector boxes.          */
int lens_fdtd3d_step_driven(LensGrid3D *g, const LensStepTable *tab, const LensEpi3D *ep,
                            const LensDrive3D *drive, int n0, int nsteps, void *stream);

/* Temporally blocked 3D step: LENS_TB3_K = 2 time steps per launch, each field
 * value crossing HBM once per two steps, with the step's epilogues fused
 * (detector boxes, volume DFTs, convergence and flux planes of LensEpi3D).  A
 * CTA streams a tile of 12 rows (y) x 28 lanes (z) down an x-chunk of `chunk`
 * planes, advancing two time levels one plane apart; the two cells around the
 * tile and the two planes around the chunk are recomputed halo.  Needs both
 * field and psi buffers (each launch reads buffer cur, writes 1 - cur and flips
 * cur) and psi_lv: a scratch set of the twelve psi volumes ((nx, ny, pitch)
 * each, touched only in the strips) holding the intermediate level.  nsteps
 * must be even; no stitch drive.  Replaces the per-step loop of
 * fdtd3d_core.py:1106-1158 (the reference advances one step per call).      */
#define LENS_TB3_K 2

typedef struct {
    float *psi_lv[LENS_NPSI];    /* intermediate-level psi volumes             */
    int chunk;                   /* x-planes per CTA (>= 1)                    */
} LensTB3D;

int lens_fdtd3d_step_tb(LensGrid3D *g, const LensTB3D *tb, const LensStepTable *tab, const LensEpi3D *ep,
                        int n0, int nsteps, void *stream);

/* Self-test of the fused step's failure detection (no counterpart in the
 * reference, whose NumPy loop has no device waits): one fused step in which the
 * first CTA of the launch withholds the E copy of one x-plane of its chunk (the
 * plane `offset` = 0 or 1 after the first plane it stages) and every pipeline
 * wait is bounded at 256 tries instead of about a second, so that CTA's waits
 * run out: it stops, drains its copies in flight, sets bit 1 of *g->flag and
 * returns, and the launch ends normally.  The step's results are invalid; the
 * grid and the context stay usable (reset the flag, restore the fields).
 * Needs the fused path (buffer 1) and g->flag.                              */
int lens_fdtd3d_watchdog_test(LensGrid3D *g, const LensStepTable *tab, int n0, int offset, void *stream);

/* Iavg += |E|^2 of all three components mapped onto the grid of component
 * `target` (1 Ey, 2 Ez) exactly as fdtd3d_core.py:438-474 (_sq_on_grid/_accum_E2),
 * over the x-planes [0, nx_target) of the slices Ex[:nx_target-1], Ey[:nx_target],
 * Ez[:nx_target] (nx_target = nx: the whole grid; a stitch window passes its
 * assembled width, fdtd3d_core.py:1650).                                     */
int lens_fdtd3d_accum_e2(const LensGrid3D *g, int target, int nx_target, float *iavg, void *stream);

/* Library identity and error text. */
int lens_version(void);
const char *lens_status_string(int status);

/* sizeof of the ABI structs, in this order: LensProfile, LensAxis, LensStepTable,
 * LensSource, LensTE2D, LensTM2D, LensEpi2D, LensGrid3D, LensEpi3D, LensInst2D,
 * LensDrive3D, LensDrive2D, LensTB2D, LensTB3D, LensRsOut2D.  Writes min(n, 15)
 * entries and returns 15 (bindings check their mirrors). */
int lens_abi_sizes(int *sizes, int n);

#ifdef __cplusplus
}
#endif
#endif /* LENS_FDTD_H */
