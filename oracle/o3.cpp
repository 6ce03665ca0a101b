// CPU restatement of the oracle's 3D CPML step (TEST INFRASTRUCTURE ONLY).
//
// Same algorithm and the same operation order, value by value, as
// oracle/fdtd_oracle.py Grid3D.step (itself the reference's CPML_3D.step,
// planar_3d/boundaries3d.py:311-362, with _PsiStrip.add_into :240-251), in
// float32 or float64 fields, multi-threaded over x-planes (std::thread).  It
// exists so the FP64 run of a full-size workload (480 x 192 x 256 cells, 4000
// steps) finishes in minutes instead of hours; tests/test_oracle_c.py checks it
// against the NumPy oracle bit for bit in both precisions.
//
// Arrays are the reference's shapes, C-contiguous:
//   Ex (nx-1,ny,nz) Ey (nx,ny-1,nz) Ez (nx,ny,nz-1)
//   Hx (nx,ny-1,nz-1) Hy (nx-1,ny,nz-1) Hz (nx-1,ny-1,nz)
// Coefficients are float32 volumes of the E shapes, widened to the field type
// before use (NumPy's float32 * float64 promotion).  psi arrays are whole
// volumes of the shape the oracle's strip lives in (the H shape for H psi,
// the interior block E[1:-1...] for E psi); only strip cells are touched.
// The source injection and every epilogue stay in NumPy on the same arrays.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off: no fused multiply-add,
// every operation rounded as NumPy rounds it).
#include <cstddef>
#include <cstdlib>
#include <thread>
#include <vector>

namespace {

// fn(i) for i in [0, n), the range split into contiguous pieces over the host
// threads (O3_THREADS, else all hardware threads).
template <typename F>
void par_for(int n, const F &fn) {
    int t = (int)std::thread::hardware_concurrency();
    if (const char *e = std::getenv("O3_THREADS")) t = std::atoi(e);
    if (t < 1) t = 1;
    if (t > n) t = n;
    std::vector<std::thread> th;
    for (int q = 0; q < t; ++q)
        th.emplace_back([&, q] {
            for (int i = (int)((long)n * q / t); i < (int)((long)n * (q + 1) / t); ++i) fn(i);
        });
    for (auto &x : th) x.join();
}

template <typename R>
struct Prof {
    const R *b, *c, *km;  // km = 1/kappa - 1, formed in the field type as the oracle does
    int n, lo, hi;        // length along the axis; strip cells [0, lo) and [n - hi, n)
    bool in(int m) const { return m < lo || m >= n - hi; }
};

template <typename R>
struct G3 {
    int nx, ny, nz;
    R *ex, *ey, *ez, *hx, *hy, *hz;
    const float *cex, *cey, *cez, *dax, *day, *daz;
    R ch;
    // psi order (LENS_PSI_*): hx_z hx_y hy_x hy_z hz_y hz_x ex_y ex_z ey_z ey_x ez_x ez_y
    R *psi[12];
    Prof<R> pf[12];
    int pec[6];  // x-lo x-hi y-lo y-hi z-lo z-hi
};

// psi = b*psi + c*d; returns psi + km*d (the strip's add term)
template <typename R>
inline R strip_term(R *p, const Prof<R> &f, int m, R d) {
    R v = *p * f.b[m];
    v = v + f.c[m] * d;
    *p = v;
    return v + f.km[m] * d;
}

template <typename R>
void step(const G3<R> &g) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const R ch = g.ch;
    // index helpers: arrays of extents (a, b, c)
    auto id = [](int i, int j, int k, int b, int c) { return ((size_t)i * b + j) * c + k; };
    // ---------------- H (old E)
    par_for(nx, [&](int i) {
        for (int j = 0; j < ny - 1; ++j)
            for (int k = 0; k < nz - 1; ++k) {  // Hx (nx, ny-1, nz-1)
                const R d1 = g.ey[id(i, j, k + 1, ny - 1, nz)] - g.ey[id(i, j, k, ny - 1, nz)];
                const R d2 = g.ez[id(i, j + 1, k, ny, nz - 1)] - g.ez[id(i, j, k, ny, nz - 1)];
                const size_t o = id(i, j, k, ny - 1, nz - 1);
                R h = g.hx[o] + ch * (d1 - d2);
                if (g.pf[0].in(k)) h = h + ch * strip_term(g.psi[0] + o, g.pf[0], k, d1);
                if (g.pf[1].in(j)) h = h + (-ch) * strip_term(g.psi[1] + o, g.pf[1], j, d2);
                g.hx[o] = h;
            }
        if (i < nx - 1) {
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz - 1; ++k) {  // Hy (nx-1, ny, nz-1)
                    const R d1 = g.ez[id(i + 1, j, k, ny, nz - 1)] - g.ez[id(i, j, k, ny, nz - 1)];
                    const R d2 = g.ex[id(i, j, k + 1, ny, nz)] - g.ex[id(i, j, k, ny, nz)];
                    const size_t o = id(i, j, k, ny, nz - 1);
                    R h = g.hy[o] + ch * (d1 - d2);
                    if (g.pf[2].in(i)) h = h + ch * strip_term(g.psi[2] + o, g.pf[2], i, d1);
                    if (g.pf[3].in(k)) h = h + (-ch) * strip_term(g.psi[3] + o, g.pf[3], k, d2);
                    g.hy[o] = h;
                }
            for (int j = 0; j < ny - 1; ++j)
                for (int k = 0; k < nz; ++k) {  // Hz (nx-1, ny-1, nz)
                    const R d1 = g.ex[id(i, j + 1, k, ny, nz)] - g.ex[id(i, j, k, ny, nz)];
                    const R d2 = g.ey[id(i + 1, j, k, ny - 1, nz)] - g.ey[id(i, j, k, ny - 1, nz)];
                    const size_t o = id(i, j, k, ny - 1, nz);
                    R h = g.hz[o] + ch * (d1 - d2);
                    if (g.pf[4].in(j)) h = h + ch * strip_term(g.psi[4] + o, g.pf[4], j, d1);
                    if (g.pf[5].in(i)) h = h + (-ch) * strip_term(g.psi[5] + o, g.pf[5], i, d2);
                    g.hz[o] = h;
                }
        }
    });
    // ---------------- E (new H): damping, curl on the interior block, strips, PEC
    const bool lossy = g.dax != nullptr;
    par_for(nx, [&](int i) {
        if (i < nx - 1) {  // Ex (nx-1, ny, nz); curl on [:, 1:-1, 1:-1]
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    const size_t o = id(i, j, k, ny, nz);
                    R v = g.ex[o];
                    if (lossy) v = v * (R)g.dax[o];
                    if (j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1) {
                        const R d1 = g.hz[id(i, j, k, ny - 1, nz)] - g.hz[id(i, j - 1, k, ny - 1, nz)];
                        const R d2 = g.hy[id(i, j, k, ny, nz - 1)] - g.hy[id(i, j, k - 1, ny, nz - 1)];
                        const R c = (R)g.cex[o];
                        v = v + c * (d1 - d2);
                        const size_t q = id(i, j - 1, k - 1, ny - 2, nz - 2);
                        if (g.pf[6].in(j - 1)) v = v + c * strip_term(g.psi[6] + q, g.pf[6], j - 1, d1);
                        if (g.pf[7].in(k - 1)) v = v + (-c) * strip_term(g.psi[7] + q, g.pf[7], k - 1, d2);
                    }
                    if ((g.pec[2] && j == 0) || (g.pec[3] && j == ny - 1) || (g.pec[4] && k == 0) ||
                        (g.pec[5] && k == nz - 1))
                        v = 0;
                    g.ex[o] = v;
                }
        }
        for (int j = 0; j < ny - 1; ++j)  // Ey (nx, ny-1, nz); curl on [1:-1, :, 1:-1]
            for (int k = 0; k < nz; ++k) {
                const size_t o = id(i, j, k, ny - 1, nz);
                R v = g.ey[o];
                if (lossy) v = v * (R)g.day[o];
                if (i >= 1 && i < nx - 1 && k >= 1 && k < nz - 1) {
                    const R d1 = g.hx[id(i, j, k, ny - 1, nz - 1)] - g.hx[id(i, j, k - 1, ny - 1, nz - 1)];
                    const R d2 = g.hz[id(i, j, k, ny - 1, nz)] - g.hz[id(i - 1, j, k, ny - 1, nz)];
                    const R c = (R)g.cey[o];
                    v = v + c * (d1 - d2);
                    const size_t q = id(i - 1, j, k - 1, ny - 1, nz - 2);
                    if (g.pf[8].in(k - 1)) v = v + c * strip_term(g.psi[8] + q, g.pf[8], k - 1, d1);
                    if (g.pf[9].in(i - 1)) v = v + (-c) * strip_term(g.psi[9] + q, g.pf[9], i - 1, d2);
                }
                if ((g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1) || (g.pec[4] && k == 0) ||
                    (g.pec[5] && k == nz - 1))
                    v = 0;
                g.ey[o] = v;
            }
        for (int j = 0; j < ny; ++j)  // Ez (nx, ny, nz-1); curl on [1:-1, 1:-1, :]
            for (int k = 0; k < nz - 1; ++k) {
                const size_t o = id(i, j, k, ny, nz - 1);
                R v = g.ez[o];
                if (lossy) v = v * (R)g.daz[o];
                if (i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1) {
                    const R d1 = g.hy[id(i, j, k, ny, nz - 1)] - g.hy[id(i - 1, j, k, ny, nz - 1)];
                    const R d2 = g.hx[id(i, j, k, ny - 1, nz - 1)] - g.hx[id(i, j - 1, k, ny - 1, nz - 1)];
                    const R c = (R)g.cez[o];
                    v = v + c * (d1 - d2);
                    const size_t q = id(i - 1, j - 1, k, ny - 2, nz - 1);
                    if (g.pf[10].in(i - 1)) v = v + c * strip_term(g.psi[10] + q, g.pf[10], i - 1, d1);
                    if (g.pf[11].in(j - 1)) v = v + (-c) * strip_term(g.psi[11] + q, g.pf[11], j - 1, d2);
                }
                if ((g.pec[0] && i == 0) || (g.pec[1] && i == nx - 1) || (g.pec[2] && j == 0) ||
                    (g.pec[3] && j == ny - 1))
                    v = 0;
                g.ez[o] = v;
            }
    });
}

// Flat argument list shared by both precisions: field pointers are R*.
template <typename R>
void run(int nx, int ny, int nz, void *const *f, const float *const *coef, double ch, void *const *psi,
         const void *const *pb, const void *const *pc, const void *const *pk, const int *plen, const int *plo,
         const int *phi, const int *pec) {
    G3<R> g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    R **fp[6] = {&g.ex, &g.ey, &g.ez, &g.hx, &g.hy, &g.hz};
    for (int q = 0; q < 6; ++q) *fp[q] = static_cast<R *>(f[q]);
    g.cex = coef[0]; g.cey = coef[1]; g.cez = coef[2];
    g.dax = coef[3]; g.day = coef[4]; g.daz = coef[5];
    g.ch = (R)ch;
    for (int q = 0; q < 12; ++q) {
        g.psi[q] = static_cast<R *>(psi[q]);
        g.pf[q] = Prof<R>{static_cast<const R *>(pb[q]), static_cast<const R *>(pc[q]),
                          static_cast<const R *>(pk[q]), plen[q], plo[q], phi[q]};
    }
    for (int q = 0; q < 6; ++q) g.pec[q] = pec[q];
    step(g);
}

}  // namespace

extern "C" {

// One step of the fields `f` (Ex, Ey, Ez, Hx, Hy, Hz) in float64 (dbl != 0) or
// float32.  coef: ce_x, ce_y, ce_z, D_x, D_y, D_z (D NULL: lossless).  ch: the
// H update factor in the field type (float64(float32(ch)) for float64 fields).
// Per psi q: pb/pc/pk the strip profile (b, c, 1/kappa - 1) along its axis in
// the field type, plen its length, plo/phi its strip widths.
void o3_step(int dbl, int nx, int ny, int nz, void *const *f, const float *const *coef, double ch,
             void *const *psi, const void *const *pb, const void *const *pc, const void *const *pk,
             const int *plen, const int *plo, const int *phi, const int *pec) {
    if (dbl)
        run<double>(nx, ny, nz, f, coef, ch, psi, pb, pc, pk, plen, plo, phi, pec);
    else
        run<float>(nx, ny, nz, f, coef, ch, psi, pb, pc, pk, plen, plo, phi, pec);
}

int o3_version(void) { return 1; }
}
