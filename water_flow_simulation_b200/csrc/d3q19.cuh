// d3q19.cuh -- D3Q19 lattice constants and the per-cell physics shared by every kernel.
//
// The velocity set, weights, opposite and lid-mirror maps are the reference's
// (floodsim/lbm3d.py:16-21); they are constexpr functions so that, inside fully
// unrolled direction loops, every c_i, w_i and index folds to a literal.
#pragma once
#include <cstdint>

namespace wfs {

constexpr int Q = 19;

__host__ __device__ constexpr int cx(int i) {
    return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1
         : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int i) {
    return (i == 3 || i == 7 || i == 10 || i == 15 || i == 17) ? 1
         : (i == 4 || i == 8 || i == 9 || i == 16 || i == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int i) {
    return (i == 5 || i == 11 || i == 14 || i == 15 || i == 18) ? 1
         : (i == 6 || i == 12 || i == 13 || i == 16 || i == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
// reflection in the rigid lid: swaps the +z and -z member of each z-moving pair
__host__ __device__ constexpr int mirz(int i) {
    return i == 5 ? 6 : i == 6 ? 5 : i == 11 ? 13 : i == 13 ? 11 : i == 12 ? 14 : i == 14 ? 12
         : i == 15 ? 17 : i == 17 ? 15 : i == 16 ? 18 : i == 18 ? 16 : i;
}
__host__ __device__ constexpr float wgt(int i) {
    return i == 0 ? 1.0f / 3.0f : (i < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
}
__host__ __device__ constexpr double wgt64(int i) {
    return i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// Cell flag word (one uint32 per cell).
constexpr uint32_t FLAG_WALLS = 0x0007FFFEu;   // bit i (1..18): pull source of direction i is a wall
constexpr uint32_t FLAG_SOLID = 1u << 19;      // solid cell (never collided)
constexpr uint32_t FLAG_FORCE = 1u << 20;      // body force is non-zero here
constexpr uint32_t FLAG_WALLFN = 1u << 21;     // wall function applies (cf > 0 and a usable wall normal)
constexpr uint32_t FLAG_BEDWALL = 1u << 22;    // bed/bank wall cell: reference speed is the column mean
constexpr uint32_t FLAG_GHOST = 1u << 23;      // x padding beyond nx (treated as solid)

// Regularized-BGK + Smagorinsky + Guo collision (floodsim/lbm3d.py:103-137), in
// moment space.  With the half-force velocity u = (j + F/2)/rho and the
// non-equilibrium stress Pi = sum c c f - rho (u u + I/3), the reference's
//   feq_i + (1 - om) (fneq_i + fneq1_i) + src_i
// is exactly  w_i [ A0 + c_i.B + c_i.C.c_i ]  with
//   A0 = rho - 1.5 rho u^2 - 1.5 (1-om) tr Pi - 3 sf u.F
//   B  = 3 rho u + (3 sf - 1.5 (1-om)) F
//   C  = 4.5 [ rho u u + (1-om) Pi + sf (u F + F u) ]      (sf = 1 - om/2)
// which needs no per-direction equilibrium.  On return f holds the post-collision
// populations and r/ux/uy/uz the cell's density and velocity.
__host__ __device__ __forceinline__ void collide(float (&f)[Q], float fx, float fy, float fz, float tau0, float csmag2,
                                        float& r, float& ux, float& uy, float& uz)
{
    const float s1 = f[1] + f[2], d1 = f[1] - f[2];
    const float s3 = f[3] + f[4], d3 = f[3] - f[4];
    const float s5 = f[5] + f[6], d5 = f[5] - f[6];
    const float s7 = f[7] + f[8], d7 = f[7] - f[8];
    const float s9 = f[9] + f[10], d9 = f[9] - f[10];
    const float s11 = f[11] + f[12], d11 = f[11] - f[12];
    const float s13 = f[13] + f[14], d13 = f[13] - f[14];
    const float s15 = f[15] + f[16], d15 = f[15] - f[16];
    const float s17 = f[17] + f[18], d17 = f[17] - f[18];
    r = f[0] + (s1 + s3 + s5) + (s7 + s9 + s11) + (s13 + s15 + s17);
    const float jx = d1 + d7 + d9 + d11 + d13;
    const float jy = d3 + d7 - d9 + d15 + d17;
    const float jz = d5 + d11 - d13 + d15 - d17;
    const float sxx = s1 + s7 + s9 + s11 + s13;
    const float syy = s3 + s7 + s9 + s15 + s17;
    const float szz = s5 + s11 + s13 + s15 + s17;
    const float sxy = s7 - s9, sxz = s11 - s13, syz = s15 - s17;

    const float ir = 1.0f / r;
    ux = (jx + 0.5f * fx) * ir;
    uy = (jy + 0.5f * fy) * ir;
    uz = (jz + 0.5f * fz) * ir;
    const float r3 = r * (1.0f / 3.0f);
    const float pxx = sxx - r * ux * ux - r3, pyy = syy - r * uy * uy - r3, pzz = szz - r * uz * uz - r3;
    const float pxy = sxy - r * ux * uy, pxz = sxz - r * ux * uz, pyz = syz - r * uy * uz;

    const float qn = sqrtf(pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pxz * pxz + pyz * pyz));
    const float tau = 0.5f * (tau0 + sqrtf(tau0 * tau0 + 18.0f * 1.41421356f * csmag2 * qn * ir));
    const float om = 1.0f / tau;
    const float k1 = 1.0f - om, sf = 1.0f - 0.5f * om;

    const float usq = ux * ux + uy * uy + uz * uz;
    const float uF = ux * fx + uy * fy + uz * fz;
    const float A0 = r - 1.5f * (r * usq + k1 * (pxx + pyy + pzz)) - 3.0f * sf * uF;
    const float bf = 3.0f * sf - 1.5f * k1;
    const float Bx = 3.0f * r * ux + bf * fx, By = 3.0f * r * uy + bf * fy, Bz = 3.0f * r * uz + bf * fz;
    const float Cxx = 4.5f * (r * ux * ux + k1 * pxx + 2.0f * sf * ux * fx);
    const float Cyy = 4.5f * (r * uy * uy + k1 * pyy + 2.0f * sf * uy * fy);
    const float Czz = 4.5f * (r * uz * uz + k1 * pzz + 2.0f * sf * uz * fz);
    const float Cxy2 = 9.0f * (r * ux * uy + k1 * pxy + sf * (ux * fy + fx * uy));
    const float Cxz2 = 9.0f * (r * ux * uz + k1 * pxz + sf * (ux * fz + fx * uz));
    const float Cyz2 = 9.0f * (r * uy * uz + k1 * pyz + sf * (uy * fz + fy * uz));

    constexpr float w0 = wgt(0), w1 = wgt(1), w2 = wgt(7);
    f[0] = w0 * A0;
    float b;
    b = A0 + Cxx;                 f[1] = w1 * (b + Bx);  f[2] = w1 * (b - Bx);
    b = A0 + Cyy;                 f[3] = w1 * (b + By);  f[4] = w1 * (b - By);
    b = A0 + Czz;                 f[5] = w1 * (b + Bz);  f[6] = w1 * (b - Bz);
    b = A0 + Cxx + Cyy + Cxy2;    f[7] = w2 * (b + (Bx + By));  f[8] = w2 * (b - (Bx + By));
    b = A0 + Cxx + Cyy - Cxy2;    f[9] = w2 * (b + (Bx - By));  f[10] = w2 * (b - (Bx - By));
    b = A0 + Cxx + Czz + Cxz2;    f[11] = w2 * (b + (Bx + Bz)); f[12] = w2 * (b - (Bx + Bz));
    b = A0 + Cxx + Czz - Cxz2;    f[13] = w2 * (b + (Bx - Bz)); f[14] = w2 * (b - (Bx - Bz));
    b = A0 + Cyy + Czz + Cyz2;    f[15] = w2 * (b + (By + Bz)); f[16] = w2 * (b - (By + Bz));
    b = A0 + Cyy + Czz - Cyz2;    f[17] = w2 * (b + (By - Bz)); f[18] = w2 * (b - (By - Bz));
}

// Wall function (floodsim/lbm3d.py:61-101): moving-wall bounce-back whose tangential
// wall speed u_s makes the momentum a cell gives its wall faces per step equal
// the log-law/Manning shear rho*cf*U^2*area.  `wm` is the cell's wall mask
// (bits 1..18), f[i] at a wall direction already holds the bounced f*_opp,
// (px,py,pz,rw) are the cell's previous-step velocity and density, and
// `uref` the reference speed (<= 0 means: use the local tangential speed).
//
// Evaluated in float64, as the reference's CPU twin does (floodsim/lbm3d.py:230-252):
// the tangent t = u_t/|u_t| is ill-conditioned where |u_t| is small, and in float32
// its rounding alone moves wall cells by ~1e-6 of max|u| per step.  It runs only at
// wall-function cells, and B200 issues FP64 at half the FP32 rate.
__host__ __device__ __forceinline__ void wall_function(float (&f)[Q], uint32_t wm, float cf, float px, float py, float pz,
                                                       float rw, float uref)
{
    int nwx = 0, nwy = 0, nwz = 0;
#pragma unroll
    for (int i = 1; i < Q; ++i)
        if (wm & (1u << i)) { nwx -= cx(i); nwy -= cy(i); nwz -= cz(i); }
    const int n2 = nwx * nwx + nwy * nwy + nwz * nwz;
    const int afx = (int)(((wm >> 1) & 1u) + ((wm >> 2) & 1u));
    const int afy = (int)(((wm >> 3) & 1u) + ((wm >> 4) & 1u));
    const int afz = (int)(((wm >> 5) & 1u) + ((wm >> 6) & 1u));
    const int a2 = afx * afx + afy * afy + afz * afz;
    if (n2 <= 0 || a2 <= 0) return;
    const double nn = sqrt((double)n2), area = sqrt((double)a2);
    const double ex = nwx / nn, ey = nwy / nn, ez = nwz / nn;
    const double un = (double)px * ex + (double)py * ey + (double)pz * ez;
    double tx = px - un * ex, ty = py - un * ey, tz = pz - un * ez;
    const double ut = sqrt(tx * tx + ty * ty + tz * tz);
    if (!(ut > 1e-7)) return;
    tx /= ut; ty /= ut; tz /= ut;
    double D = 0.0, K = 0.0;
#pragma unroll
    for (int i = 1; i < Q; ++i)
        if (wm & (1u << i)) {
            const double ct = cx(i) * tx + cy(i) * ty + cz(i) * tz;
            D += ct * (double)f[i];
            K += (double)wgt(i) * ct * ct;
        }
    if (!(K > 0.0)) return;
    const double U = uref > 0.f ? (double)uref : ut;
    const double us0 = (-2.0 * D - (double)(rw * cf) * U * U * area) / (6.0 * (double)rw * K);
    const double us = fmin(fmax(us0, -ut), ut);
    const double g = 6.0 * (double)rw * us;
#pragma unroll
    for (int i = 1; i < Q; ++i)
        if (wm & (1u << i)) f[i] = (float)((double)f[i] + g * (double)wgt(i) * (cx(i) * tx + cy(i) * ty + cz(i) * tz));
}

// Second-order equilibrium of direction i (floodsim/lbm3d.py:140-143).
template <int I>
__host__ __device__ __forceinline__ float feq_dir(float r, float ux, float uy, float uz)
{
    const float cu = 3.f * ((float)cx(I) * ux + (float)cy(I) * uy + (float)cz(I) * uz);
    return wgt(I) * r * (1.f + cu + 0.5f * cu * cu - 1.5f * (ux * ux + uy * uy + uz * uz));
}

// Inlet velocity / outlet pressure by non-equilibrium extrapolation
// (floodsim/lbm3d.py:153-174): g = post-collision populations of the interior
// neighbour (x=1 or x=nx-2), out = the boundary cell's new populations.
// inlet: density from the neighbour, velocity (uin,0,0);
// outlet: density rho_out, velocity from the neighbour.
template <bool INLET>
__host__ __device__ __forceinline__ void nebb(const float (&g)[Q], float (&out)[Q], float uin, float rho_out)
{
    float r = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        r += g[i];
        mx += (float)cx(i) * g[i];
        my += (float)cy(i) * g[i];
        mz += (float)cz(i) * g[i];
    }
    const float ir = 1.0f / r;
    const float ux = mx * ir, uy = my * ir, uz = mz * ir;
#define WFS_NEBB(I)                                                                          \
    out[I] = (INLET ? feq_dir<I>(r, uin, 0.f, 0.f) : feq_dir<I>(rho_out, ux, uy, uz))        \
             + (g[I] - feq_dir<I>(r, ux, uy, uz));
    WFS_NEBB(0) WFS_NEBB(1) WFS_NEBB(2) WFS_NEBB(3) WFS_NEBB(4) WFS_NEBB(5) WFS_NEBB(6)
    WFS_NEBB(7) WFS_NEBB(8) WFS_NEBB(9) WFS_NEBB(10) WFS_NEBB(11) WFS_NEBB(12) WFS_NEBB(13)
    WFS_NEBB(14) WFS_NEBB(15) WFS_NEBB(16) WFS_NEBB(17) WFS_NEBB(18)
#undef WFS_NEBB
}

}  // namespace wfs
