// readouts.cuh -- FP64 device reductions of the along-stream profiles (floodsim/reach3d.py:545-568).
// Included inside the anonymous namespace of lbm_kernels.cu.
//
// Per x station, over the fluid cells of the cross-section (y, z), in float64:
//   PROF_Q        sum ux                      (discharge / (dx^2 * velocity scale))
//   PROF_UXX      sum ux^2                    (momentum flux)
//   PROF_DRHO     sum (rho - 1)               (pressure part of the momentum balance)
//   PROF_MASS     sum rho
//   PROF_NFLUID   fluid cells
//   PROF_TOP_N    fluid cells of the top layer (z = nz-1, under the rigid lid)
//   PROF_TOP_DRHO sum (rho - 1) over the top layer   (lid water level)
//   PROF_TOP_UX   sum ux over the top layer          (surface speed)
//   PROF_UMAX     max |u|
// and per (y, x) column the largest |u|^2 of a fluid cell whose lower neighbour is solid
// or the bed (the bed-shear cell of floodsim/reach3d.py:562-566).  The fields are either
// the time-average sums (avg, scaled by inv_navg: ux, uy, uz, rho, |u|, ux^2 at m*cells)
// or, without avg, the instantaneous rho/ux/uy/uz.  The sums are deterministic: pass 1
// writes per-chunk partials, pass 2 adds the chunks in order.
#pragma once

enum ProfField {
    PROF_Q = 0, PROF_UXX, PROF_DRHO, PROF_MASS, PROF_NFLUID, PROF_TOP_N, PROF_TOP_DRHO, PROF_TOP_UX, PROF_UMAX,
    PROF_NF
};

struct CellFields {
    double rho, ux, sp, uxx;
};

__device__ __forceinline__ CellFields cell_fields(const lbm_lattice& L, long long c, double inv_navg)
{
    CellFields r;
    if (L.avg) {
        const long long S = L.cells;
        r.ux = (double)L.avg[c] * inv_navg;
        r.rho = (double)L.avg[3 * S + c] * inv_navg;
        r.sp = (double)L.avg[4 * S + c] * inv_navg;
        r.uxx = (double)L.avg[5 * S + c] * inv_navg;
    } else {
        const double u = L.ux[c], v = L.uy[c], w = L.uz[c];
        r.ux = u;
        r.rho = L.rho[c];
        r.sp = sqrt(u * u + v * v + w * w);
        r.uxx = u * u;
    }
    return r;
}

// Pass 1: thread = x station, blockIdx.y = chunk of `rows_per_chunk` rows (row = z*ny + y).
__global__ void k_profile_partials(const lbm_lattice L, double inv_navg, int rows_per_chunk, double* __restrict__ part)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= L.nx) return;
    const int rows = L.ny * L.nz;
    const int r0 = blockIdx.y * rows_per_chunk, r1 = min(r0 + rows_per_chunk, rows);
    double acc[PROF_NF];
#pragma unroll
    for (int k = 0; k < PROF_NF; ++k) acc[k] = 0.0;
    for (int r = r0; r < r1; ++r) {
        const long long c = (long long)r * L.pitch + x;
        if (L.flags[c] & FLAG_SOLID) continue;
        const CellFields f = cell_fields(L, c, inv_navg);
        acc[PROF_Q] += f.ux;
        acc[PROF_UXX] += f.uxx;
        acc[PROF_DRHO] += f.rho - 1.0;
        acc[PROF_MASS] += f.rho;
        acc[PROF_NFLUID] += 1.0;
        acc[PROF_UMAX] = fmax(acc[PROF_UMAX], f.sp);
        if (r / L.ny == L.nz - 1) {
            acc[PROF_TOP_N] += 1.0;
            acc[PROF_TOP_DRHO] += f.rho - 1.0;
            acc[PROF_TOP_UX] += f.ux;
        }
    }
#pragma unroll
    for (int k = 0; k < PROF_NF; ++k) part[((long long)blockIdx.y * PROF_NF + k) * L.nx + x] = acc[k];
}

// Pass 2: prof[k*nx + x] = the chunks' partials added in chunk order (max for PROF_UMAX).
__global__ void k_profile_sum(const double* __restrict__ part, int nchunks, int nx, double* __restrict__ prof)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // k*nx + x
    if (i >= (long long)PROF_NF * nx) return;
    const int k = (int)(i / nx);
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ++ch) {
        const double v = part[(long long)ch * PROF_NF * nx + i];
        s = k == PROF_UMAX ? fmax(s, v) : s + v;
    }
    prof[i] = s;
}

// Bed-shear cells: thread = (y, x); max over z of |u|^2 at fluid cells above solid or the bed.
__global__ void k_bed_speed2(const lbm_lattice L, double inv_navg, double* __restrict__ sp2)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;    // x + nx*y
    if (q >= (long long)L.nx * L.ny) return;
    const int x = (int)(q % L.nx), y = (int)(q / L.nx);
    const long long plane = (long long)L.ny * L.pitch;
    double m = 0.0;
    bool below_solid = true;                                                 // z = 0 sits on the bed
    for (int z = 0; z < L.nz; ++z) {
        const long long c = z * plane + (long long)y * L.pitch + x;
        const bool solid = L.flags[c] & FLAG_SOLID;
        if (!solid && below_solid) {
            const double s = cell_fields(L, c, inv_navg).sp;
            m = fmax(m, s * s);
        }
        below_solid = solid;
    }
    sp2[q] = m;
}

// ---------------------------------------------------------------------------------------------
// FP64 force sums: the force on each body (hull) by momentum exchange, and the body force the
// lattice applies (propellers, jets).  No counterpart in the reference, which infers the boats'
// net force from the momentum-flux difference along the reach (floodsim/reach3d.py:604-609).
//
// From a state (f = the stored post-collision populations of the last step, rho/u its fields,
// colU or uref the wall-model speed) the next step pulls, at a fluid cell x whose source
// x - c_i is a solid cell of body k, the bounced f_opp(i)(x) as f_i(x), corrected by the wall
// function (floodsim/lbm3d.py:61-101); body k then receives -c_i (f_opp(i)(x) + f_i(x)) over
// that link -- its horizontal part only where the source was mirrored by the rigid lid
// (a -z mover under the lid, floodsim/lbm3d.py:54), the lid taking the vertical part.  acc[3*(k-1) + d]: the sum for body k (1..nbody); acc[3*nbody + d]: the applied
// body force, sum of F * force_scale over forced fluid cells.  Lattice units (momentum per
// cell volume per step).  A grid of kBodyBlocks blocks, each thread summing its cells in order,
// then each block in a fixed tree order, then the blocks in order: deterministic.
// ---------------------------------------------------------------------------------------------
constexpr int kMaxBodies = 16;
constexpr int kBodyBlocks = 1024;
constexpr int kBodyThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kBodyThreads) k_body_forces(const lbm_lattice L, const T* __restrict__ f,
                                                              float inv_scale, const uint8_t* __restrict__ body,
                                                              int nbody, bool ucol, double* __restrict__ part)
{
    __shared__ double red[kBodyThreads];
    const int nacc = 3 * nbody + 3;
    double acc[3 * kMaxBodies + 3];
#pragma unroll
    for (int k = 0; k < 3 * kMaxBodies + 3; ++k) acc[k] = 0.0;
    const long long plane = (long long)L.ny * L.pitch;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < L.cells;
         c += (long long)gridDim.x * blockDim.x) {
        const uint32_t fk = L.flags[c];
        if (fk & FLAG_SOLID) continue;
        if (fk & FLAG_FORCE) {
            acc[3 * nbody + 0] += (double)(L.Fx[c] * L.force_scale);
            acc[3 * nbody + 1] += (double)(L.Fy[c] * L.force_scale);
            acc[3 * nbody + 2] += (double)(L.Fz[c] * L.force_scale);
        }
        const uint32_t wm = fk & FLAG_WALLS;
        if (!wm) continue;
        const int x = (int)(c % L.pitch), y = (int)((c / L.pitch) % L.ny), z = (int)(c / plane);
        int bk[Q];
        bool any = false;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            bk[i] = 0;
            if (i == 0 || !(wm & (1u << i))) continue;
            int zs = z - cz(i);
            const int xs = x - cx(i), ys = y - cy(i);
            const bool lid = zs >= L.nz;                 // mirrored into the own layer (the lid's rule)
            if (lid) zs = z;
            if (zs < 0 || ys < 0 || ys >= L.ny || xs < 0 || xs >= L.nx) continue;   // bed, y walls, x edges
            const int b = body[zs * plane + (long long)ys * L.pitch + xs];
            if (b > 0 && b <= nbody) { bk[i] = lid ? -b : b; any = true; }
        }
        if (!any) continue;
        float fw[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i)
            fw[i] = (i > 0 && (wm & (1u << i))) ? ldpop(f + (long long)opp(i) * L.cells + c, i, inv_scale) : 0.f;
        float bounced[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) bounced[i] = fw[i];
        if (fk & FLAG_WALLFN) {
            const float U = ucol ? ((fk & FLAG_BEDWALL) ? L.colU[(long long)y * L.pitch + x] : 0.f) : L.uref[c];
            wall_function(fw, wm, L.cfw[c], L.ux[c], L.uy[c], L.uz[c], L.rho[c], U);
        }
#pragma unroll
        for (int i = 1; i < Q; ++i)
            if (bk[i]) {
                const double m = (double)bounced[i] + (double)fw[i];
                double* a = acc + 3 * ((bk[i] < 0 ? -bk[i] : bk[i]) - 1);
                a[0] -= cx(i) * m;
                a[1] -= cy(i) * m;
                if (bk[i] > 0) a[2] -= cz(i) * m;      // through the lid: the lid takes the vertical part
            }
    }
    for (int k = 0; k < nacc; ++k) {
        red[threadIdx.x] = acc[k];
        __syncthreads();
        for (int s = kBodyThreads / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * nacc + k] = red[0];
        __syncthreads();
    }
}

// out[k] = the blocks' partials of component k added in block order.
__global__ void k_body_forces_sum(const double* __restrict__ part, int nblocks, int nacc, double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nacc) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += part[(long long)b * nacc + k];
    out[k] = s;
}
