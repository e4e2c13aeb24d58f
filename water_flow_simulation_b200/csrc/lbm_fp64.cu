// lbm_fp64.cu -- the float64 solver of the accuracy statements.
//
// The 16-bit and float32 paths state their water-level and bed-shear error against a run of
// the same algorithm in float64.  The CPU oracle does that up to config-1 sizes; at 36M cells
// and 20k steps it would take hours.  These kernels are that float64 run on the GPU: the
// reference's step (floodsim/lbm3d.py:31-138), inlet/outlet (lbm3d.py:140-175) and the
// column-mean wall speed of Run3D._update_uref (floodsim/reach3d.py:412-418), in the
// reference layout (f[i*N + c], c = x + nx*(y + ny*z)) with float64 populations, fields,
// forces and arithmetic throughout.  One thread per cell: these runs check accuracy, they
// are not the product's speed path.  The CPU oracle's float64 functions pin them
// (tests/test_gpu_fp64.py).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "d3q19.cuh"
#include "errors.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Equilibrium of direction i at density r and velocity (ux, uy, uz) (floodsim/lbm3d.py:140-143).
__device__ __forceinline__ double feq64(int i, double r, double ux, double uy, double uz)
{
    const double cu = 3.0 * (cx(i) * ux + cy(i) * uy + cz(i) * uz);
    return wgt64(i) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * (ux * ux + uy * uy + uz * uz));
}

__global__ void __launch_bounds__(128) k_step_f64(const double* __restrict__ fs, double* __restrict__ fd,
        const uint8_t* __restrict__ solid, const double* __restrict__ Fx, const double* __restrict__ Fy,
        const double* __restrict__ Fz, double* __restrict__ rho, double* __restrict__ vx, double* __restrict__ vy,
        double* __restrict__ vz, const double* __restrict__ cfw, const double* __restrict__ uref,
        int nx, int ny, int nz, double tau0, double csmag2, int sponge_cols, double sponge_tau)
{
    const long long N = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    if (solid[c]) { rho[c] = 1.0; vx[c] = 0.0; vy[c] = 0.0; vz[c] = 0.0; return; }
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long long)nx * ny));
    if (sponge_cols > 0 && x >= nx - sponge_cols) {         // optional outlet sponge
        const double s = (double)(x - (nx - sponge_cols) + 1) / sponge_cols;
        tau0 = tau0 + (sponge_tau - tau0) * (s * s);
    }

    // Pull with half-way bounce-back at y walls, the bed and solids, and the lid mirror
    // (lbm3d.py:42-59).  Pulls across x = 0 / nx-1 keep the cell's own value.
    double f[Q];
    uint32_t wall = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int xs = x - cx(i), ys = y - cy(i);
        int zs = z - cz(i), src_dir = i;
        if (xs < 0 || xs >= nx) { f[i] = fs[(long long)i * N + c]; continue; }
        if (zs >= nz) { zs = z; src_dir = mirz(i); }
        bool w = ys < 0 || ys >= ny || zs < 0;
        long long s = 0;
        if (!w) { s = xs + (long long)nx * (ys + (long long)ny * zs); w = solid[s] != 0; }
        if (w) wall |= 1u << i;
        f[i] = w ? fs[(long long)opp(i) * N + c] : fs[(long long)src_dir * N + s];
    }

    // Wall function (lbm3d.py:61-101): slip velocity along the wall, sized so that the
    // momentum the bounced populations carry matches the drag cf*rho*U^2 over the wall area.
    const double cf = cfw[c];
    double nwx = 0.0, nwy = 0.0, nwz = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i)
        if (wall & (1u << i)) { nwx -= cx(i); nwy -= cy(i); nwz -= cz(i); }
    const double nn = sqrt(nwx * nwx + nwy * nwy + nwz * nwz);
    const double ax = (double)(((wall >> 1) & 1) + ((wall >> 2) & 1));
    const double ay = (double)(((wall >> 3) & 1) + ((wall >> 4) & 1));
    const double az = (double)(((wall >> 5) & 1) + ((wall >> 6) & 1));
    const double area = sqrt(ax * ax + ay * ay + az * az);
    if (cf > 0.0 && nn > 0.0 && area > 0.0) {
        const double ex = nwx / nn, ey = nwy / nn, ez = nwz / nn;
        const double px = vx[c], py = vy[c], pz = vz[c];
        const double un = px * ex + py * ey + pz * ez;
        double tx = px - un * ex, ty = py - un * ey, tz = pz - un * ez;
        const double ut = sqrt(tx * tx + ty * ty + tz * tz);
        if (ut > 1e-7) {
            tx /= ut; ty /= ut; tz /= ut;
            const double rw = rho[c];
            double D = 0.0, K = 0.0;
#pragma unroll
            for (int i = 0; i < Q; ++i)
                if (wall & (1u << i)) {
                    const double ct = cx(i) * tx + cy(i) * ty + cz(i) * tz;
                    D += ct * f[i];
                    K += wgt64(i) * ct * ct;
                }
            if (K > 0.0) {
                const double U = uref[c] > 0.0 ? uref[c] : ut;
                const double us = fmin(fmax((-2.0 * D - rw * cf * U * U * area) / (6.0 * rw * K), -ut), ut);
#pragma unroll
                for (int i = 0; i < Q; ++i)
                    if (wall & (1u << i)) f[i] += 6.0 * wgt64(i) * rw * (cx(i) * tx + cy(i) * ty + cz(i) * tz) * us;
            }
        }
    }

    // Regularized BGK with Smagorinsky and Guo forcing (lbm3d.py:103-137).
    double r = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) { r += f[i]; jx += cx(i) * f[i]; jy += cy(i) * f[i]; jz += cz(i) * f[i]; }
    const double gx = Fx[c], gy = Fy[c], gz = Fz[c];
    const double ux = (jx + 0.5 * gx) / r, uy = (jy + 0.5 * gy) / r, uz = (jz + 0.5 * gz) / r;
    double pxx = 0.0, pyy = 0.0, pzz = 0.0, pxy = 0.0, pxz = 0.0, pyz = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const double d = f[i] - feq64(i, r, ux, uy, uz);
        pxx += cx(i) * cx(i) * d; pyy += cy(i) * cy(i) * d; pzz += cz(i) * cz(i) * d;
        pxy += cx(i) * cy(i) * d; pxz += cx(i) * cz(i) * d; pyz += cy(i) * cz(i) * d;
    }
    const double qn = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + 2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
    const double tau = 0.5 * (tau0 + sqrt(tau0 * tau0 + 18.0 * 1.41421356 * csmag2 * qn / r));
    const double om = 1.0 / tau, sf = 1.0 - 0.5 * om;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const double w = wgt64(i);
        const double reg = 4.5 * w * ((cx(i) * cx(i) - 1.0 / 3.0) * pxx + (cy(i) * cy(i) - 1.0 / 3.0) * pyy
                                      + (cz(i) * cz(i) - 1.0 / 3.0) * pzz
                                      + 2.0 * (cx(i) * cy(i) * pxy + cx(i) * cz(i) * pxz + cy(i) * cz(i) * pyz));
        const double cu = cx(i) * ux + cy(i) * uy + cz(i) * uz;
        const double cg = cx(i) * gx + cy(i) * gy + cz(i) * gz;
        const double guo = sf * w * (3.0 * ((cx(i) - ux) * gx + (cy(i) - uy) * gy + (cz(i) - uz) * gz) + 9.0 * cu * cg);
        fd[(long long)i * N + c] = feq64(i, r, ux, uy, uz) + (1.0 - om) * (reg - 1.5 * w * cg) + guo;
    }
    rho[c] = r; vx[c] = ux; vy[c] = uy; vz[c] = uz;
}

// Inlet velocity at x = 0, outlet density at x = nx-1: non-equilibrium extrapolation from
// x = 1 / nx-2 (lbm3d.py:145-175).
__global__ void k_bc_f64(double* __restrict__ fd, const uint8_t* __restrict__ solid, const double* __restrict__ uin,
                         int nx, int ny, int nz, double rho_out)
{
    const long long N = (long long)nx * ny * nz;
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (long long)ny * nz) return;
    const long long row = (long long)nx * j;          // j = y + ny*z
    for (int side = 0; side < 2; ++side) {
        const long long c0 = side == 0 ? row : row + nx - 1, c1 = side == 0 ? row + 1 : row + nx - 2;
        if (solid[c0] || solid[c1]) continue;
        double g[Q], r = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            g[i] = fd[(long long)i * N + c1];
            r += g[i]; jx += cx(i) * g[i]; jy += cy(i) * g[i]; jz += cz(i) * g[i];
        }
        const double ux = jx / r, uy = jy / r, uz = jz / r;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const double e = side == 0 ? feq64(i, r, uin[j], 0.0, 0.0) : feq64(i, rho_out, ux, uy, uz);
            fd[(long long)i * N + c0] = e + (g[i] - feq64(i, r, ux, uy, uz));
        }
    }
}

// Column-mean speed U(y,x) = |sum_z (ux, uy) over fluid cells| / max(n_fluid, 1), written to
// uref at bed/bank wall cells and 0 elsewhere (floodsim/reach3d.py:412-418).
__global__ void k_uref_f64(const double* __restrict__ vx, const double* __restrict__ vy,
                           const uint8_t* __restrict__ solid, const uint8_t* __restrict__ bedwall,
                           double* __restrict__ uref, int nx, int ny, int nz)
{
    const long long plane = (long long)nx * ny;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= plane) return;
    double sx = 0.0, sy = 0.0;
    int nf = 0;
    for (int z = 0; z < nz; ++z) {
        const long long c = q + plane * z;
        if (!solid[c]) { sx += vx[c]; sy += vy[c]; ++nf; }
    }
    const double U = sqrt(sx * sx + sy * sy) / (double)(nf > 1 ? nf : 1);
    for (int z = 0; z < nz; ++z) {
        const long long c = q + plane * z;
        uref[c] = bedwall[c] ? U : 0.0;
    }
}

int check_dims(const char* what, int nx, int ny, int nz)
{
    if (nx < 3 || ny < 1 || nz < 1) return fail(LBM_ERR_ARG, "%s: bad lattice %dx%dx%d", what, nx, ny, nz);
    return 0;
}

}  // namespace

extern "C" {

int lbm_step_f64(const double* fs, double* fd, const uint8_t* solid, const double* Fx, const double* Fy,
                 const double* Fz, double* rho, double* ux, double* uy, double* uz, const double* cfw,
                 const double* uref, int nx, int ny, int nz, double tau0, double csmag2, int sponge_cols,
                 double sponge_tau, void* stream)
{
    g_err[0] = 0;
    if (!fs || !fd || !solid || !Fx || !Fy || !Fz || !rho || !ux || !uy || !uz || !cfw || !uref)
        return fail(LBM_ERR_ARG, "lbm_step_f64: NULL array");
    if (int e = check_dims("lbm_step_f64", nx, ny, nz)) return e;
    if (sponge_cols < 0 || sponge_cols > nx - 2 || (sponge_cols > 0 && !(sponge_tau >= tau0 && sponge_tau < 2.0)))
        return fail(LBM_ERR_ARG, "lbm_step_f64: bad sponge (%d columns, tau %g)", sponge_cols, sponge_tau);
    if (fs == fd) return fail(LBM_ERR_ARG, "lbm_step_f64: fs and fd must differ");
    const long long N = (long long)nx * ny * nz;
    k_step_f64<<<(unsigned)((N + 127) / 128), 128, 0, as_stream(stream)>>>(fs, fd, solid, Fx, Fy, Fz, rho, ux, uy,
                                                                         uz, cfw, uref, nx, ny, nz, tau0, csmag2,
                                                                         sponge_cols, sponge_tau);
    return check_launch("lbm_step_f64");
}

int lbm_bc_f64(double* fd, const uint8_t* solid, const double* uin, int nx, int ny, int nz, double rho_out,
               void* stream)
{
    g_err[0] = 0;
    if (!fd || !solid || !uin) return fail(LBM_ERR_ARG, "lbm_bc_f64: NULL array");
    if (int e = check_dims("lbm_bc_f64", nx, ny, nz)) return e;
    const long long M = (long long)ny * nz;
    k_bc_f64<<<(unsigned)((M + 127) / 128), 128, 0, as_stream(stream)>>>(fd, solid, uin, nx, ny, nz, rho_out);
    return check_launch("lbm_bc_f64");
}

int lbm_update_uref_f64(const double* ux, const double* uy, const uint8_t* solid, const uint8_t* bedwall,
                        double* uref, int nx, int ny, int nz, void* stream)
{
    g_err[0] = 0;
    if (!ux || !uy || !solid || !bedwall || !uref) return fail(LBM_ERR_ARG, "lbm_update_uref_f64: NULL array");
    if (int e = check_dims("lbm_update_uref_f64", nx, ny, nz)) return e;
    const long long P = (long long)nx * ny;
    k_uref_f64<<<(unsigned)((P + 127) / 128), 128, 0, as_stream(stream)>>>(ux, uy, solid, bedwall, uref, nx, ny,
                                                                          nz);
    return check_launch("lbm_update_uref_f64");
}

}  // extern "C"
