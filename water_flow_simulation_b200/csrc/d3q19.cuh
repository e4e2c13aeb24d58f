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

// A float product rounded on its own (never fused into a later add).
__host__ __device__ __forceinline__ float mul_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}

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
    // tau0^2 and 18 sqrt(2) Cs^2 are rounded explicitly: they are lattice constants, and a compiler
    // that hoists them out of a loop (or not) must not change how they fuse into what follows
    const float tau0sq = mul_rn(tau0, tau0), smag = mul_rn(18.0f * 1.41421356f, csmag2);
    const float tau = 0.5f * (tau0 + sqrtf(tau0sq + smag * qn * ir));
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

// Direction masks over bits 1..18 (bit i = direction i), for popcount sums over a wall mask.
template <typename P>
__host__ __device__ constexpr uint32_t dir_mask(P pred)
{
    uint32_t m = 0;
    for (int i = 1; i < Q; ++i)
        if (pred(i)) m |= 1u << i;
    return m;
}
__host__ __device__ __forceinline__ int popc32(uint32_t v)
{
#ifdef __CUDA_ARCH__
    return __popc(v);
#else
    return __builtin_popcount(v);
#endif
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
// its rounding alone moves wall cells by ~1e-6 of max|u| per step.
//
// The reference's sums over the wall directions are regrouped so that only one pass over
// the populations remains: with c_i the wall directions' velocities,
//   n = -sum c_i                         (popcounts of the mask: c components are 0, +-1)
//   D = sum (c_i.t) f_i = t . J,          J = sum c_i f_i
//   K = sum w_i (c_i.t)^2 = t^T M t,      M = sum w_i c_i c_i^T  (popcounts again)
// and the update f_i += g w_i (c_i.t) is f_i += w_i c_i.(g t); the unit vectors are never
// formed (see below), which leaves two square roots and two divisions.  The float64 results
// differ from the per-direction sums only by float64 reassociation.
__host__ __device__ __forceinline__ void wall_function(float (&f)[Q], uint32_t wm, float cf, float px, float py, float pz,
                                                       float rw, float uref)
{
    constexpr uint32_t PX = dir_mask([](int i) { return cx(i) == 1; }), NX = dir_mask([](int i) { return cx(i) == -1; });
    constexpr uint32_t PY = dir_mask([](int i) { return cy(i) == 1; }), NY = dir_mask([](int i) { return cy(i) == -1; });
    constexpr uint32_t PZ = dir_mask([](int i) { return cz(i) == 1; }), NZ = dir_mask([](int i) { return cz(i) == -1; });
    constexpr uint32_t AXIS = 0x7Eu;                                          // directions 1..6 (weight 1/18)
    constexpr uint32_t XY_SAME = dir_mask([](int i) { return cx(i) * cy(i) == 1; });
    constexpr uint32_t XY_OPP = dir_mask([](int i) { return cx(i) * cy(i) == -1; });
    constexpr uint32_t XZ_SAME = dir_mask([](int i) { return cx(i) * cz(i) == 1; });
    constexpr uint32_t XZ_OPP = dir_mask([](int i) { return cx(i) * cz(i) == -1; });
    constexpr uint32_t YZ_SAME = dir_mask([](int i) { return cy(i) * cz(i) == 1; });
    constexpr uint32_t YZ_OPP = dir_mask([](int i) { return cy(i) * cz(i) == -1; });
    const uint32_t wx = wm & (PX | NX), wy = wm & (PY | NY), wz = wm & (PZ | NZ);
    const int nwx = popc32(wm & NX) - popc32(wm & PX);
    const int nwy = popc32(wm & NY) - popc32(wm & PY);
    const int nwz = popc32(wm & NZ) - popc32(wm & PZ);
    const int n2 = nwx * nwx + nwy * nwy + nwz * nwz;
    const int afx = (int)(((wm >> 1) & 1u) + ((wm >> 2) & 1u));
    const int afy = (int)(((wm >> 3) & 1u) + ((wm >> 4) & 1u));
    const int afz = (int)(((wm >> 5) & 1u) + ((wm >> 6) & 1u));
    const int a2 = afx * afx + afy * afy + afz * afz;
    if (n2 <= 0 || a2 <= 0) return;
    // Tangential velocity t = p - (p.n) n / |n|^2 (n the integer wall normal: no square root
    // needed for it), ut = |t|.  With the unit tangent t/ut the reference's slip speed is
    //   us0 = (-2 D - rw cf U^2 area) / (6 rw K),  D = (t.J)/ut,  K = (t^T M t)/ut^2,
    // clamped to [-ut, ut], and the update f_i += w_i c_i.(6 rw us t/ut); so with
    //   s = us0/ut = (-2 (t.J) - rw cf U^2 area ut) / (6 rw t^T M t)
    // the update is f_i += w_i c_i.(6 rw clamp(s, -1, 1) t): one square root for ut, one for
    // the face area, one division -- the same quantities as the reference's, regrouped.
    const double area = sqrt((double)a2);
    const double pn = (double)px * nwx + (double)py * nwy + (double)pz * nwz;
    const double q = pn / (double)n2;
    const double tx = px - q * nwx, ty = py - q * nwy, tz = pz - q * nwz;
    const double ut = sqrt(tx * tx + ty * ty + tz * tz);
    if (!(ut > 1e-7)) return;
    double jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
    for (int i = 1; i < Q; ++i)
        if (wm & (1u << i)) {
            const double fi = (double)f[i];
            if (cx(i) == 1) jx += fi; else if (cx(i) == -1) jx -= fi;
            if (cy(i) == 1) jy += fi; else if (cy(i) == -1) jy -= fi;
            if (cz(i) == 1) jz += fi; else if (cz(i) == -1) jz -= fi;
        }
    const double tJ = tx * jx + ty * jy + tz * jz;
    const double w1 = (double)wgt(1), w2 = (double)wgt(7);
    const double mxx = w1 * popc32(wx & AXIS) + w2 * popc32(wx & ~AXIS);
    const double myy = w1 * popc32(wy & AXIS) + w2 * popc32(wy & ~AXIS);
    const double mzz = w1 * popc32(wz & AXIS) + w2 * popc32(wz & ~AXIS);
    const double mxy = w2 * (popc32(wm & XY_SAME) - popc32(wm & XY_OPP));
    const double mxz = w2 * (popc32(wm & XZ_SAME) - popc32(wm & XZ_OPP));
    const double myz = w2 * (popc32(wm & YZ_SAME) - popc32(wm & YZ_OPP));
    const double tMt = tx * tx * mxx + ty * ty * myy + tz * tz * mzz + 2.0 * (tx * ty * mxy + tx * tz * mxz + ty * tz * myz);
    if (!(tMt > 0.0)) return;
    const double U = uref > 0.f ? (double)uref : ut;
    const double s0 = (-2.0 * tJ - (double)(rw * cf) * U * U * area * ut) / (6.0 * (double)rw * tMt);
    const double sc = fmin(fmax(s0, -1.0), 1.0);
    const double g = 6.0 * (double)rw * sc;
    const double gx = g * tx, gy = g * ty, gz = g * tz;
#pragma unroll
    for (int i = 1; i < Q; ++i)
        if (wm & (1u << i)) {
            double ct = 0.0;
            if (cx(i)) ct += cx(i) * gx;
            if (cy(i)) ct += cy(i) * gy;
            if (cz(i)) ct += cz(i) * gz;
            f[i] = (float)((double)f[i] + (double)wgt(i) * ct);
        }
}

// Inlet velocity / outlet pressure by non-equilibrium extrapolation
// (floodsim/lbm3d.py:153-174): g = post-collision populations of the interior
// neighbour (x=1 or x=nx-2), out = the boundary cell's new populations,
//   out_i = feq_i(rho_b, u_b) + g_i - feq_i(rho_g, u_g),
// inlet: rho_b = rho_g, u_b = (uin,0,0); outlet: rho_b = rho_out, u_b = u_g.
// The difference of the two second-order equilibria is itself a quadratic form,
//   feq_i(rho_b, u_b) - feq_i(rho_g, u_g) = w_i [A + c_i.B + c_i.C.c_i],
//   A = -1.5 (rho_b u_b^2 - rho_g u_g^2) + (rho_b - rho_g),
//   B = 3 (rho_b u_b - rho_g u_g),  C = 4.5 (rho_b u_b u_b - rho_g u_g u_g),
// so it is evaluated like the collision's output stage (one pass, no per-direction
// equilibria); the result differs from the reference's order of operations only by
// float32 rounding.
template <bool INLET>
__host__ __device__ __forceinline__ void nebb(const float (&g)[Q], float (&out)[Q], float uin, float rho_out)
{
    const float s1 = g[1] + g[2], d1 = g[1] - g[2];
    const float s3 = g[3] + g[4], d3 = g[3] - g[4];
    const float s5 = g[5] + g[6], d5 = g[5] - g[6];
    const float s7 = g[7] + g[8], d7 = g[7] - g[8];
    const float s9 = g[9] + g[10], d9 = g[9] - g[10];
    const float s11 = g[11] + g[12], d11 = g[11] - g[12];
    const float s13 = g[13] + g[14], d13 = g[13] - g[14];
    const float s15 = g[15] + g[16], d15 = g[15] - g[16];
    const float s17 = g[17] + g[18], d17 = g[17] - g[18];
    const float r = g[0] + (s1 + s3 + s5) + (s7 + s9 + s11) + (s13 + s15 + s17);
    const float mx = d1 + d7 + d9 + d11 + d13;
    const float my = d3 + d7 - d9 + d15 + d17;
    const float mz = d5 + d11 - d13 + d15 - d17;
    const float ir = 1.0f / r;
    const float ux = mx * ir, uy = my * ir, uz = mz * ir;
    // rho_b u_b and rho_b u_b u_b minus the same of g
    float rb, bx, by, bz;
    if (INLET) { rb = r; bx = uin; by = 0.f; bz = 0.f; }
    else       { rb = rho_out; bx = ux; by = uy; bz = uz; }
    const float A = (rb - r) - 1.5f * (rb * (bx * bx + by * by + bz * bz) - r * (ux * ux + uy * uy + uz * uz));
    const float Bx = 3.0f * (rb * bx - r * ux), By = 3.0f * (rb * by - r * uy), Bz = 3.0f * (rb * bz - r * uz);
    const float Cxx = 4.5f * (rb * bx * bx - r * ux * ux);
    const float Cyy = 4.5f * (rb * by * by - r * uy * uy);
    const float Czz = 4.5f * (rb * bz * bz - r * uz * uz);
    const float Cxy2 = 9.0f * (rb * bx * by - r * ux * uy);
    const float Cxz2 = 9.0f * (rb * bx * bz - r * ux * uz);
    const float Cyz2 = 9.0f * (rb * by * bz - r * uy * uz);
    constexpr float w0 = wgt(0), w1 = wgt(1), w2 = wgt(7);
    out[0] = g[0] + w0 * A;
    float b;
    b = A + Cxx;                 out[1] = g[1] + w1 * (b + Bx);  out[2] = g[2] + w1 * (b - Bx);
    b = A + Cyy;                 out[3] = g[3] + w1 * (b + By);  out[4] = g[4] + w1 * (b - By);
    b = A + Czz;                 out[5] = g[5] + w1 * (b + Bz);  out[6] = g[6] + w1 * (b - Bz);
    b = A + Cxx + Cyy + Cxy2;    out[7] = g[7] + w2 * (b + (Bx + By));  out[8] = g[8] + w2 * (b - (Bx + By));
    b = A + Cxx + Cyy - Cxy2;    out[9] = g[9] + w2 * (b + (Bx - By));  out[10] = g[10] + w2 * (b - (Bx - By));
    b = A + Cxx + Czz + Cxz2;    out[11] = g[11] + w2 * (b + (Bx + Bz)); out[12] = g[12] + w2 * (b - (Bx + Bz));
    b = A + Cxx + Czz - Cxz2;    out[13] = g[13] + w2 * (b + (Bx - Bz)); out[14] = g[14] + w2 * (b - (Bx - Bz));
    b = A + Cyy + Czz + Cyz2;    out[15] = g[15] + w2 * (b + (By + Bz)); out[16] = g[16] + w2 * (b - (By + Bz));
    b = A + Cyy + Czz - Cyz2;    out[17] = g[17] + w2 * (b + (By - Bz)); out[18] = g[18] + w2 * (b - (By - Bz));
}

}  // namespace wfs
