/*
 * lbm_oracle.c -- CPU oracle for the D3Q19 stream-collide hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is called only from tests/, from the smoke check and
 * from the timed CPU-baseline leg of bench.py.  Nothing in the product links it.
 *
 * It restates the reference's CPU twin (floodsim/lbm3d.py:179-330, the Numba
 * `step`/`feq1`/`bc` functions) in plain C.  The Numba functions store
 * populations in float32 arrays but infer float64 for most scalars, because
 * float32 (op) float64 and float32 (op) int64 both promote to float64.  The
 * `_f32` functions below reproduce that typing operation by operation: every
 * scalar Numba types as float64 is a `double` here, and a value is rounded to
 * float at exactly the points where Numba stores into a float32 array or
 * multiplies two float32 values.  Compile with -ffp-contract=off so that each
 * operation rounds as written.  Numba compiles `step` with fastmath=True, so
 * LLVM may contract or reassociate its float64 arithmetic; the two therefore
 * agree to within one float32 ulp per step rather than bit-for-bit.
 *
 * The `_f64` functions are the same algorithm with float64 storage and float64
 * arithmetic throughout: the FP64 oracle used for error statements.
 *
 * Layout (floodsim/lbm3d.py:9): f[i*N + c], c = x + nx*(y + ny*z), N = nx*ny*nz.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

/* D3Q19 velocity set, weights, opposite and lid-mirror tables
 * (floodsim/lbm3d.py:16-21). */
static const int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const int MIRZ[19] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};

/* W as float64 (floodsim/lbm3d.py:19) and as the float32 copy the Numba twin
 * captures (`w = W.astype(np.float32)`, floodsim/lbm3d.py:183-184). */
static double W64(int i) { return i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0); }
static float W32(int i) { return (float)W64(i); }

/* The wall function of the Numba step (floodsim/lbm3d.py:224-252): f[i] of the wall directions
 * (wl[i] set, holding the bounced populations) take the moving-wall correction sized from the
 * previous step's velocity (px, py, pz) and density rw of the cell, its friction cf and the
 * reference speed uref (<= 0: the local tangential speed).  (nwx, nwy, nwz) = -sum of the wall
 * directions' c_i. */
static void wall_fn_f32(float *f, const int *wl, double nwx, double nwy, double nwz, float cf,
                        float px, float py, float pz, float rw, float uref)
{
        const double nn = sqrt(nwx * nwx + nwy * nwy + nwz * nwz);
        const double afx = (wl[1] ? 1.0 : 0.0) + (wl[2] ? 1.0 : 0.0);
        const double afy = (wl[3] ? 1.0 : 0.0) + (wl[4] ? 1.0 : 0.0);
        const double afz = (wl[5] ? 1.0 : 0.0) + (wl[6] ? 1.0 : 0.0);
        const double area = sqrt(afx * afx + afy * afy + afz * afz);
        if (cf > 0.0f && nn > 0.0 && area > 0.0) {
            const double ex = nwx / nn, ey = nwy / nn, ez = nwz / nn;
            const double un = (double)px * ex + (double)py * ey + (double)pz * ez;
            double tx = (double)px - un * ex, ty = (double)py - un * ey, tz = (double)pz - un * ez;
            const double ut = sqrt(tx * tx + ty * ty + tz * tz);
            if (ut > 1e-7) {
                tx = tx / ut; ty = ty / ut; tz = tz / ut;
                double D = 0.0, K = 0.0;
                for (int i = 0; i < 19; ++i)
                    if (wl[i]) {
                        const double ct = CX[i] * tx + CY[i] * ty + CZ[i] * tz;
                        D += ct * (double)f[i];
                        K += (double)W32(i) * ct * ct;
                    }
                if (K > 0.0) {
                    const double U = uref > 0.0f ? (double)uref : ut;
                    const float rwcf = rw * cf;             /* float32 * float32 stays float32 */
                    const double us0 = (-2.0 * D - (double)rwcf * U * U * area) / (6.0 * (double)rw * K);
                    double us = us0 > -ut ? us0 : -ut;      /* min(max(us0, -ut), ut) */
                    us = us < ut ? us : ut;
                    for (int i = 0; i < 19; ++i)
                        if (wl[i])
                            f[i] = (float)((double)f[i] + 6.0 * (double)W32(i) * (double)rw
                                           * (CX[i] * tx + CY[i] * ty + CZ[i] * tz) * us);
                }
            }
        }
}

/* ------------------------------------------------------------------------ */
/* Numba-typed step: floodsim/lbm3d.py:186-294                               */
/* ------------------------------------------------------------------------ */
/* tau0_x: NULL, or the relaxation time at zero strain per x column (an outlet sponge,
 * which the reference does not have; NULL is the reference). */
static void step_f32(const float *fs, float *fd, const uint8_t *solid,
                     const float *Fx, const float *Fy, const float *Fz,
                     float *rho_o, float *ux_o, float *uy_o, float *uz_o,
                     const float *cfw, const float *uref,
                     int64_t nx, int64_t ny, int64_t nz, float tau0_all, float csmag2, const float *tau0_x)
{
    const int64_t N = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        const int64_t x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        if (solid[c]) {                                     /* lbm3d.py:193-198 */
            rho_o[c] = 1.0f; ux_o[c] = 0.0f; uy_o[c] = 0.0f; uz_o[c] = 0.0f;
            continue;
        }
        float f[19];
        int wl[19];
        double nwx = 0.0, nwy = 0.0, nwz = 0.0;
        for (int i = 0; i < 19; ++i) {                      /* lbm3d.py:204-223 */
            wl[i] = 0;
            int64_t xs = x - CX[i], ys = y - CY[i], zs = z - CZ[i];
            int ii = i;
            if (xs < 0 || xs >= nx) { f[i] = fs[(int64_t)i * N + c]; continue; }
            if (zs >= nz) { zs = z; ii = MIRZ[i]; }
            int wall = (ys < 0 || ys >= ny || zs < 0);
            int64_t s = 0;
            if (!wall) { s = xs + nx * (ys + ny * zs); wall = solid[s] != 0; }
            if (wall) { wl[i] = 1; nwx -= CX[i]; nwy -= CY[i]; nwz -= CZ[i]; }
            f[i] = wall ? fs[(int64_t)OPP[i] * N + c] : fs[(int64_t)ii * N + s];
        }
        wall_fn_f32(f, wl, nwx, nwy, nwz, cfw[c], ux_o[c], uy_o[c], uz_o[c], rho_o[c], uref[c]);
        double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;        /* lbm3d.py:253-264 */
        for (int i = 0; i < 19; ++i) {
            r += (double)f[i];
            mx += (double)f[i] * CX[i];
            my += (double)f[i] * CY[i];
            mz += (double)f[i] * CZ[i];
        }
        const float fx = Fx[c], fy = Fy[c], fz = Fz[c];
        const double ux = (mx + 0.5 * fx) / r, uy = (my + 0.5 * fy) / r, uz = (mz + 0.5 * fz) / r;
        const double usq = ux * ux + uy * uy + uz * uz;
        float feq[19];
        double pxx = 0.0, pyy = 0.0, pzz = 0.0, pxy = 0.0, pxz = 0.0, pyz = 0.0;
        for (int i = 0; i < 19; ++i) {                      /* lbm3d.py:265-276 */
            const double cu = 3.0 * (CX[i] * ux + CY[i] * uy + CZ[i] * uz);
            feq[i] = (float)((double)W32(i) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * usq));
            const float fn = f[i] - feq[i];                 /* float32 - float32 */
            pxx += (double)(CX[i] * CX[i]) * fn;
            pyy += (double)(CY[i] * CY[i]) * fn;
            pzz += (double)(CZ[i] * CZ[i]) * fn;
            pxy += (double)(CX[i] * CY[i]) * fn;
            pxz += (double)(CX[i] * CZ[i]) * fn;
            pyz += (double)(CY[i] * CZ[i]) * fn;
        }
        const double qn = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + 2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
        const float tau0 = tau0_x ? tau0_x[x] : tau0_all;
        const float t2 = tau0 * tau0;                       /* float32 * float32 */
        const double tau = 0.5 * ((double)tau0 + sqrt((double)t2 + 18.0 * 1.41421356 * (double)csmag2 * qn / r));
        const double om = 1.0 / tau;
        const double sf = 1.0 - 0.5 * om;
        for (int i = 0; i < 19; ++i) {                      /* lbm3d.py:281-290 */
            const double w = (double)W32(i);
            const double fneq = 4.5 * w * ((CX[i] * CX[i] - 1.0 / 3.0) * pxx + (CY[i] * CY[i] - 1.0 / 3.0) * pyy
                                           + (CZ[i] * CZ[i] - 1.0 / 3.0) * pzz
                                           + 2.0 * ((double)(CX[i] * CY[i]) * pxy + (double)(CX[i] * CZ[i]) * pxz
                                                    + (double)(CY[i] * CZ[i]) * pyz));
            const double cu = CX[i] * ux + CY[i] * uy + CZ[i] * uz;
            const double cF = (double)CX[i] * fx + (double)CY[i] * fy + (double)CZ[i] * fz;
            const double src = sf * w * (3.0 * ((CX[i] - ux) * fx + (CY[i] - uy) * fy + (CZ[i] - uz) * fz)
                                         + 9.0 * cu * cF);
            const double fneq1 = -1.5 * w * cF;
            fd[(int64_t)i * N + c] = (float)((double)feq[i] + (1.0 - om) * (fneq + fneq1) + src);
        }
        rho_o[c] = (float)r; ux_o[c] = (float)ux; uy_o[c] = (float)uy; uz_o[c] = (float)uz;
    }
}

/* feq1 (floodsim/lbm3d.py:296-299) specialised to the three argument typings
 * `bc` calls it with. */
void oracle_step_f32(const float *fs, float *fd, const uint8_t *solid,
                     const float *Fx, const float *Fy, const float *Fz,
                     float *rho_o, float *ux_o, float *uy_o, float *uz_o,
                     const float *cfw, const float *uref,
                     int64_t nx, int64_t ny, int64_t nz, float tau0, float csmag2)
{
    step_f32(fs, fd, solid, Fx, Fy, Fz, rho_o, ux_o, uy_o, uz_o, cfw, uref, nx, ny, nz, tau0, csmag2, NULL);
}

void oracle_step_f32_x(const float *fs, float *fd, const uint8_t *solid,
                       const float *Fx, const float *Fy, const float *Fz,
                       float *rho_o, float *ux_o, float *uy_o, float *uz_o,
                       const float *cfw, const float *uref,
                       int64_t nx, int64_t ny, int64_t nz, const float *tau0_x, float csmag2)
{
    step_f32(fs, fd, solid, Fx, Fy, Fz, rho_o, ux_o, uy_o, uz_o, cfw, uref, nx, ny, nz, 0.0f, csmag2, tau0_x);
}

static double feq1_dd(int i, double r, double ux, double uy, double uz)
{   /* r, u all float64 */
    const double cu = 3.0 * (CX[i] * ux + CY[i] * uy + CZ[i] * uz);
    return (double)W32(i) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * (ux * ux + uy * uy + uz * uz));
}
static double feq1_in(int i, double r, float uin)
{   /* inlet: ux = uin[j] is float32, uy = uz = 0.0 (float64); ux*ux stays float32 */
    const double cu = 3.0 * ((double)CX[i] * uin + CY[i] * 0.0 + CZ[i] * 0.0);
    const float u2 = uin * uin;
    return (double)W32(i) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * ((double)u2 + 0.0 * 0.0 + 0.0 * 0.0));
}
static double feq1_out(int i, float rho_out, double ux, double uy, double uz)
{   /* outlet: r = rho_out is float32, so w[i]*r stays float32 */
    const double cu = 3.0 * (CX[i] * ux + CY[i] * uy + CZ[i] * uz);
    const float wr = W32(i) * rho_out;
    return (double)wr * (1.0 + cu + 0.5 * cu * cu - 1.5 * (ux * ux + uy * uy + uz * uz));
}

/* Numba-typed inlet/outlet boundary: floodsim/lbm3d.py:301-328. */
void oracle_bc_f32(float *fd, const uint8_t *solid, const float *uin,
                   int64_t nx, int64_t ny, int64_t nz, float rho_out)
{
    const int64_t N = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny * nz; ++j) {
        const int64_t y = j % ny, z = j / ny, row = nx * (y + ny * z);
        for (int side = 0; side < 2; ++side) {
            const int64_t c0 = side == 0 ? row : row + nx - 1;
            const int64_t c1 = side == 0 ? row + 1 : row + nx - 2;
            if (solid[c0] || solid[c1]) continue;
            double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
            for (int i = 0; i < 19; ++i) {
                const float v = fd[(int64_t)i * N + c1];
                r += (double)v; mx += (double)v * CX[i]; my += (double)v * CY[i]; mz += (double)v * CZ[i];
            }
            const double ux = mx / r, uy = my / r, uz = mz / r;
            for (int i = 0; i < 19; ++i) {
                const double a = side == 0 ? feq1_in(i, r, uin[j]) : feq1_out(i, rho_out, ux, uy, uz);
                fd[(int64_t)i * N + c0] = (float)(a + ((double)fd[(int64_t)i * N + c1] - feq1_dd(i, r, ux, uy, uz)));
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* FP64 oracle: same algorithm, float64 storage and arithmetic.              */
/* ------------------------------------------------------------------------ */
static void step_f64(const double *fs, double *fd, const uint8_t *solid,
                     const double *Fx, const double *Fy, const double *Fz,
                     double *rho_o, double *ux_o, double *uy_o, double *uz_o,
                     const double *cfw, const double *uref,
                     int64_t nx, int64_t ny, int64_t nz, double tau0_all, double csmag2, const double *tau0_x)
{
    const int64_t N = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        const int64_t x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        if (solid[c]) { rho_o[c] = 1.0; ux_o[c] = 0.0; uy_o[c] = 0.0; uz_o[c] = 0.0; continue; }
        double f[19];
        int wl[19];
        double nwx = 0.0, nwy = 0.0, nwz = 0.0;
        for (int i = 0; i < 19; ++i) {
            wl[i] = 0;
            int64_t xs = x - CX[i], ys = y - CY[i], zs = z - CZ[i];
            int ii = i;
            if (xs < 0 || xs >= nx) { f[i] = fs[(int64_t)i * N + c]; continue; }
            if (zs >= nz) { zs = z; ii = MIRZ[i]; }
            int wall = (ys < 0 || ys >= ny || zs < 0);
            int64_t s = 0;
            if (!wall) { s = xs + nx * (ys + ny * zs); wall = solid[s] != 0; }
            if (wall) { wl[i] = 1; nwx -= CX[i]; nwy -= CY[i]; nwz -= CZ[i]; }
            f[i] = wall ? fs[(int64_t)OPP[i] * N + c] : fs[(int64_t)ii * N + s];
        }
        const double cf = cfw[c];
        const double nn = sqrt(nwx * nwx + nwy * nwy + nwz * nwz);
        const double afx = wl[1] + wl[2], afy = wl[3] + wl[4], afz = wl[5] + wl[6];
        const double area = sqrt(afx * afx + afy * afy + afz * afz);
        if (cf > 0.0 && nn > 0.0 && area > 0.0) {
            const double ex = nwx / nn, ey = nwy / nn, ez = nwz / nn;
            const double px = ux_o[c], py = uy_o[c], pz = uz_o[c];
            const double un = px * ex + py * ey + pz * ez;
            double tx = px - un * ex, ty = py - un * ey, tz = pz - un * ez;
            const double ut = sqrt(tx * tx + ty * ty + tz * tz);
            if (ut > 1e-7) {
                tx /= ut; ty /= ut; tz /= ut;
                const double rw = rho_o[c];
                double D = 0.0, K = 0.0;
                for (int i = 0; i < 19; ++i)
                    if (wl[i]) {
                        const double ct = CX[i] * tx + CY[i] * ty + CZ[i] * tz;
                        D += ct * f[i];
                        K += W64(i) * ct * ct;
                    }
                if (K > 0.0) {
                    const double U = uref[c] > 0.0 ? uref[c] : ut;
                    const double us0 = (-2.0 * D - rw * cf * U * U * area) / (6.0 * rw * K);
                    double us = us0 > -ut ? us0 : -ut;
                    us = us < ut ? us : ut;
                    for (int i = 0; i < 19; ++i)
                        if (wl[i]) f[i] += 6.0 * W64(i) * rw * (CX[i] * tx + CY[i] * ty + CZ[i] * tz) * us;
                }
            }
        }
        double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
        for (int i = 0; i < 19; ++i) { r += f[i]; mx += f[i] * CX[i]; my += f[i] * CY[i]; mz += f[i] * CZ[i]; }
        const double fx = Fx[c], fy = Fy[c], fz = Fz[c];
        const double ux = (mx + 0.5 * fx) / r, uy = (my + 0.5 * fy) / r, uz = (mz + 0.5 * fz) / r;
        const double usq = ux * ux + uy * uy + uz * uz;
        double feq[19];
        double pxx = 0.0, pyy = 0.0, pzz = 0.0, pxy = 0.0, pxz = 0.0, pyz = 0.0;
        for (int i = 0; i < 19; ++i) {
            const double cu = 3.0 * (CX[i] * ux + CY[i] * uy + CZ[i] * uz);
            feq[i] = W64(i) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * usq);
            const double fn = f[i] - feq[i];
            pxx += CX[i] * CX[i] * fn; pyy += CY[i] * CY[i] * fn; pzz += CZ[i] * CZ[i] * fn;
            pxy += CX[i] * CY[i] * fn; pxz += CX[i] * CZ[i] * fn; pyz += CY[i] * CZ[i] * fn;
        }
        const double qn = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + 2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
        const double tau0 = tau0_x ? tau0_x[x] : tau0_all;
        const double tau = 0.5 * (tau0 + sqrt(tau0 * tau0 + 18.0 * 1.41421356 * csmag2 * qn / r));
        const double om = 1.0 / tau, sf = 1.0 - 0.5 * om;
        for (int i = 0; i < 19; ++i) {
            const double w = W64(i);
            const double fneq = 4.5 * w * ((CX[i] * CX[i] - 1.0 / 3.0) * pxx + (CY[i] * CY[i] - 1.0 / 3.0) * pyy
                                           + (CZ[i] * CZ[i] - 1.0 / 3.0) * pzz
                                           + 2.0 * (CX[i] * CY[i] * pxy + CX[i] * CZ[i] * pxz + CY[i] * CZ[i] * pyz));
            const double cu = CX[i] * ux + CY[i] * uy + CZ[i] * uz;
            const double cF = CX[i] * fx + CY[i] * fy + CZ[i] * fz;
            const double src = sf * w * (3.0 * ((CX[i] - ux) * fx + (CY[i] - uy) * fy + (CZ[i] - uz) * fz) + 9.0 * cu * cF);
            const double fneq1 = -1.5 * w * cF;
            fd[(int64_t)i * N + c] = feq[i] + (1.0 - om) * (fneq + fneq1) + src;
        }
        rho_o[c] = r; ux_o[c] = ux; uy_o[c] = uy; uz_o[c] = uz;
    }
}

void oracle_step_f64(const double *fs, double *fd, const uint8_t *solid,
                     const double *Fx, const double *Fy, const double *Fz,
                     double *rho_o, double *ux_o, double *uy_o, double *uz_o,
                     const double *cfw, const double *uref,
                     int64_t nx, int64_t ny, int64_t nz, double tau0, double csmag2)
{
    step_f64(fs, fd, solid, Fx, Fy, Fz, rho_o, ux_o, uy_o, uz_o, cfw, uref, nx, ny, nz, tau0, csmag2, NULL);
}

void oracle_step_f64_x(const double *fs, double *fd, const uint8_t *solid,
                       const double *Fx, const double *Fy, const double *Fz,
                       double *rho_o, double *ux_o, double *uy_o, double *uz_o,
                       const double *cfw, const double *uref,
                       int64_t nx, int64_t ny, int64_t nz, const double *tau0_x, double csmag2)
{
    step_f64(fs, fd, solid, Fx, Fy, Fz, rho_o, ux_o, uy_o, uz_o, cfw, uref, nx, ny, nz, 0.0, csmag2, tau0_x);
}

static double feq64(int i, double r, double ux, double uy, double uz)
{
    const double cu = 3.0 * (CX[i] * ux + CY[i] * uy + CZ[i] * uz);
    return W64(i) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * (ux * ux + uy * uy + uz * uz));
}

/* FP64 inlet/outlet boundary (floodsim/lbm3d.py:301-328 in float64). */
void oracle_bc_f64(double *fd, const uint8_t *solid, const double *uin,
                   int64_t nx, int64_t ny, int64_t nz, double rho_out)
{
    const int64_t N = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny * nz; ++j) {
        const int64_t y = j % ny, z = j / ny, row = nx * (y + ny * z);
        for (int side = 0; side < 2; ++side) {
            const int64_t c0 = side == 0 ? row : row + nx - 1;
            const int64_t c1 = side == 0 ? row + 1 : row + nx - 2;
            if (solid[c0] || solid[c1]) continue;
            double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
            for (int i = 0; i < 19; ++i) {
                const double v = fd[(int64_t)i * N + c1];
                r += v; mx += v * CX[i]; my += v * CY[i]; mz += v * CZ[i];
            }
            const double ux = mx / r, uy = my / r, uz = mz / r;
            for (int i = 0; i < 19; ++i) {
                const double a = side == 0 ? feq64(i, r, uin[j], 0.0, 0.0) : feq64(i, rho_out, ux, uy, uz);
                fd[(int64_t)i * N + c0] = a + (fd[(int64_t)i * N + c1] - feq64(i, r, ux, uy, uz));
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Column-mean reference speed for the wall model: floodsim/reach3d.py:412-418
 * U(y,x) = sqrt((sum_z ux*fl)^2 + (sum_z uy*fl)^2) / ncol, written to uref at
 * bed/bank wall cells and 0 elsewhere.  float32 throughout, z summed in order
 * (NumPy's axis-0 reduction of a C-contiguous array adds the z slabs in turn). */
void oracle_update_uref_f32(const float *ux, const float *uy, const uint8_t *solid,
                            const uint8_t *bedwall, float *uref,
                            int64_t nx, int64_t ny, int64_t nz)
{
    const int64_t plane = nx * ny;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < plane; ++q) {
        float sx = 0.0f, sy = 0.0f;
        int64_t nf = 0;
        for (int64_t z = 0; z < nz; ++z) {
            const int64_t c = q + plane * z;
            const float fl = solid[c] ? 0.0f : 1.0f;
            sx = sx + ux[c] * fl;
            sy = sy + uy[c] * fl;
            nf += !solid[c];
        }
        const float ncol = (float)(nf > 1 ? nf : 1);
        const float U = sqrtf(sx * sx + sy * sy) / ncol;
        for (int64_t z = 0; z < nz; ++z) {
            const int64_t c = q + plane * z;
            uref[c] = bedwall[c] ? U : 0.0f;
        }
    }
}

void oracle_update_uref_f64(const double *ux, const double *uy, const uint8_t *solid,
                            const uint8_t *bedwall, double *uref,
                            int64_t nx, int64_t ny, int64_t nz)
{
    const int64_t plane = nx * ny;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < plane; ++q) {
        double sx = 0.0, sy = 0.0;
        int64_t nf = 0;
        for (int64_t z = 0; z < nz; ++z) {
            const int64_t c = q + plane * z;
            if (!solid[c]) { sx += ux[c]; sy += uy[c]; ++nf; }
        }
        const double U = sqrt(sx * sx + sy * sy) / (double)(nf > 1 ? nf : 1);
        for (int64_t z = 0; z < nz; ++z) {
            const int64_t c = q + plane * z;
            uref[c] = bedwall[c] ? U : 0.0;
        }
    }
}

/* Force on each body (hull) by momentum exchange, for the bounce-back of the step that follows
 * the state (fs = post-collision populations of the last step, rho/ux/uy/uz/uref its fields):
 * a fluid cell whose pull source x - c_i lies in body k (body[s] = k, 1..nbody) gets f_i back
 * as the bounced f_opp(i), after the wall function of floodsim/lbm3d.py:224-252, and the body
 * receives -c_i (f_opp(i) + f_i) for that link (floodsim has no force readout; this sums its
 * own bounce-back rule).  Under the rigid lid a -z mover's source is mirrored into the own
 * layer (lbm3d.py:54); when that source is a body cell the body takes the horizontal part of
 * the link and the lid the vertical one.  out[3*(k-1) + d] += the component d, in float64, in lattice units
 * (momentum per cell volume per step).  Serial, in cell order. */
void oracle_body_forces_f32(const float *fs, const uint8_t *solid, const uint8_t *body, int nbody,
                            const float *rho_o, const float *ux_o, const float *uy_o, const float *uz_o,
                            const float *cfw, const float *uref, int64_t nx, int64_t ny, int64_t nz,
                            double *out)
{
    const int64_t N = nx * ny * nz;
    for (int k = 0; k < 3 * nbody; ++k) out[k] = 0.0;
    for (int64_t c = 0; c < N; ++c) {
        if (solid[c]) continue;
        const int64_t x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        float f[19];
        int wl[19], bk[19];
        int any = 0;
        double nwx = 0.0, nwy = 0.0, nwz = 0.0;
        for (int i = 0; i < 19; ++i) {
            wl[i] = 0; bk[i] = 0;
            f[i] = 0.0f;
            int64_t xs = x - CX[i], ys = y - CY[i], zs = z - CZ[i];
            if (xs < 0 || xs >= nx) continue;
            int lid = 0;
            if (zs >= nz) { zs = z; lid = 1; }              /* the lid mirrors: source in the own layer */
            int wall = (ys < 0 || ys >= ny || zs < 0);
            int64_t s = 0;
            if (!wall) { s = xs + nx * (ys + ny * zs); wall = solid[s] != 0; }
            if (wall) {
                wl[i] = 1; nwx -= CX[i]; nwy -= CY[i]; nwz -= CZ[i];
                f[i] = fs[(int64_t)OPP[i] * N + c];
                if (!(ys < 0 || ys >= ny || zs < 0) && body[s] > 0 && body[s] <= nbody) {
                    bk[i] = body[s] * (lid ? -1 : 1);      /* negative: through the lid */
                    any = 1;
                }
            }
        }
        if (!any) continue;
        wall_fn_f32(f, wl, nwx, nwy, nwz, cfw[c], ux_o[c], uy_o[c], uz_o[c], rho_o[c], uref[c]);
        for (int i = 0; i < 19; ++i)
            if (bk[i]) {
                const double m = (double)fs[(int64_t)OPP[i] * N + c] + (double)f[i];
                double *o = out + 3 * ((bk[i] < 0 ? -bk[i] : bk[i]) - 1);
                o[0] -= CX[i] * m; o[1] -= CY[i] * m;
                if (bk[i] > 0) o[2] -= CZ[i] * m;         /* through the lid the lid takes the vertical part */
            }
    }
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
