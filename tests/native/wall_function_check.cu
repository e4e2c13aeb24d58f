// Host-side check of the kernels' wall function (d3q19.cuh: wall_function, regrouped sums, no
// unit vectors) against the reference's per-direction form (floodsim/lbm3d.py:224-252, as the
// CPU oracle states it) on random wall masks, populations and velocities.  Prints the largest
// difference of an updated population relative to that population: cases the wall function
// changed, cases run, populations that differ, largest relative difference.
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <random>
#include "../../water_flow_simulation_b200/csrc/d3q19.cuh"
using namespace wfs;

static void reference_form(float (&f)[Q], uint32_t wm, float cf, float px, float py, float pz, float rw, float uref)
{
    double nwx = 0, nwy = 0, nwz = 0;
    int wl[Q];
    for (int i = 0; i < Q; ++i) {
        wl[i] = (i > 0 && (wm >> i) & 1u) ? 1 : 0;
        if (wl[i]) { nwx -= cx(i); nwy -= cy(i); nwz -= cz(i); }
    }
    const double nn = std::sqrt(nwx * nwx + nwy * nwy + nwz * nwz);
    const double afx = wl[1] + wl[2], afy = wl[3] + wl[4], afz = wl[5] + wl[6];
    const double area = std::sqrt(afx * afx + afy * afy + afz * afz);
    if (!(cf > 0.0f && nn > 0.0 && area > 0.0)) return;
    const double ex = nwx / nn, ey = nwy / nn, ez = nwz / nn;
    const double un = (double)px * ex + (double)py * ey + (double)pz * ez;
    double tx = px - un * ex, ty = py - un * ey, tz = pz - un * ez;
    const double ut = std::sqrt(tx * tx + ty * ty + tz * tz);
    if (!(ut > 1e-7)) return;
    tx /= ut; ty /= ut; tz /= ut;
    double D = 0, K = 0;
    for (int i = 0; i < Q; ++i)
        if (wl[i]) {
            const double ct = cx(i) * tx + cy(i) * ty + cz(i) * tz;
            D += ct * (double)f[i];
            K += (double)wgt(i) * ct * ct;
        }
    if (!(K > 0.0)) return;
    const double U = uref > 0.0f ? (double)uref : ut;
    const float rwcf = rw * cf;
    const double us0 = (-2.0 * D - (double)rwcf * U * U * area) / (6.0 * (double)rw * K);
    double us = us0 > -ut ? us0 : -ut;
    us = us < ut ? us : ut;
    for (int i = 0; i < Q; ++i)
        if (wl[i]) f[i] = (float)((double)f[i] + 6.0 * (double)wgt(i) * (double)rw * (cx(i) * tx + cy(i) * ty + cz(i) * tz) * us);
}

int main()
{
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U01(0.0, 1.0);
    double worst = 0.0;
    long changed = 0, cases = 0, updated = 0;
    for (int n = 0; n < 200000; ++n) {
        uint32_t wm = 0;
        for (int i = 1; i < Q; ++i)
            if (U01(rng) < 0.3) wm |= 1u << i;
        float f[Q], g[Q], f0[Q];
        for (int i = 0; i < Q; ++i) f0[i] = f[i] = g[i] = (float)(wgt(i) * (1.0 + 0.3 * (U01(rng) - 0.5)));
        const float px = (float)(0.1 * (U01(rng) - 0.5)), py = (float)(0.05 * (U01(rng) - 0.5)),
                    pz = (float)(0.02 * (U01(rng) - 0.5));
        const float cf = (float)(0.01 * U01(rng)), rw = (float)(1.0 + 0.01 * (U01(rng) - 0.5));
        const float uref = U01(rng) < 0.5 ? 0.0f : (float)(0.08 * U01(rng));
        reference_form(f, wm, cf, px, py, pz, rw, uref);
        wall_function(g, wm, cf, px, py, pz, rw, uref);
        ++cases;
        bool moved = false;
        for (int i = 0; i < Q; ++i) moved |= f[i] != f0[i];
        updated += moved;
        for (int i = 0; i < Q; ++i) {
            if (f[i] != g[i]) ++changed;
            const double d = std::fabs((double)f[i] - (double)g[i]) / std::fabs((double)f[i]);
            if (d > worst) worst = d;
        }
    }
    std::printf("%ld %ld %ld %.3e\n", updated, cases, changed, worst);
    return 0;
}
