/*
 * lbm_b200.h -- C ABI of liblbm_b200.so, the B200 (sm_100a) D3Q19 solver kernels.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (cudaStream_t passed as void*, NULL = legacy default stream), returns an int
 * status (LBM_OK or a negative LBM_ERR_*) and never throws; the message of the
 * last failure on the calling thread is available from lbm_last_error().
 * Kernels are enqueued asynchronously on the given stream.
 *
 * Two families:
 *
 * 1. lbm_step / lbm_bc: the reference's two solver kernels with their exact
 *    argument lists and array layout (f[i*N + c], c = x + nx*(y + ny*z)).  They
 *    are what a ctypes/cupy binding of floodsim/lbm3d.py would call in place of
 *    its NVRTC-compiled CUDA_SRC.
 *
 * 2. The fused path (lbm_lattice + lbm_fused_step): one kernel per time step
 *    that streams, bounces back, applies the wall function, collides, applies
 *    the inlet/outlet condition and, on output steps, writes the macroscopic
 *    fields, the column-mean wall-model speed and the time averages.  Arrays
 *    use an x pitch `pitch` >= nx (a multiple of 4): cell (x,y,z) is at
 *    x + pitch*(y + ny*z) and population i of it at i*cells + that.  With
 *    pitch == nx this is the reference layout.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 113     /* major*100 + minor; lbm_abi_version() returns it */

#define LBM_OK 0
#define LBM_ERR_ARG (-1)          /* bad size, pointer, alignment or option */
#define LBM_ERR_CUDA (-2)         /* a CUDA runtime call or kernel launch failed */
#define LBM_ERR_UNSUPPORTED (-3)  /* valid request this build does not implement */

/* Cell flag bits (uint32 per cell), built by lbm_build_flags. */
#define LBM_FLAG_WALLS 0x0007FFFEu     /* bit i: the pull source of direction i is a wall */
#define LBM_FLAG_SOLID (1u << 19)
#define LBM_FLAG_FORCE (1u << 20)
#define LBM_FLAG_WALLFN (1u << 21)
#define LBM_FLAG_BEDWALL (1u << 22)
#define LBM_FLAG_GHOST (1u << 23)

/* lbm_fused_step mode bits */
#define LBM_STEP_OUTPUT 1u       /* write rho/u of every cell (else only where the wall function reads them) */
#define LBM_STEP_UREF_COLUMN 2u  /* wall model reads the column-mean speed colU; an OUTPUT step refreshes it */
#define LBM_STEP_ACCUMULATE 4u   /* an OUTPUT step adds ux,uy,uz,rho,|u|,ux^2 into avg[0..5] */
#define LBM_STEP_SKIP_PLAIN 8u   /* split pipeline: leave out the plain-segment kernel this call */
#define LBM_STEP_SKIP_SPECIAL 16u /* split pipeline: leave out the special/solid/column-mean kernels; a
                                    step split in two calls runs the plain part first */
#define LBM_STEP_OVERLAP 32u     /* split pipeline: run the edge and special kernels on a side stream of
                                    the library (one per CUDA context, created by the first such call:
                                    make it before any stream capture), forked from `stream` before
                                    the plain kernel and joined back after it, so that they share the
                                    SMs with it; tile.ctas_per_sm then bounds the plain kernel alone.
                                    Ignored with either SKIP bit. */

/* Message of the last failed call on this thread ("" if none). */
const char *lbm_last_error(void);

/* LBM_ABI_VERSION of the built library. */
int lbm_abi_version(void);

/* Replaces the `lbm_step` kernel of floodsim/lbm3d.py:31-138 (launched at
 * lbm3d.py:400-403): one pull stream-collide step of all N = nx*ny*nz cells,
 * fs -> fd, writing rho/ux/uy/uz (read back as the previous step at wall-function
 * cells).  solid: uint8[N]; Fx,Fy,Fz,cfw,uref,rho,ux,uy,uz: float[N];
 * fs,fd: float[19*N]. */
int lbm_step(const float *fs, float *fd, const uint8_t *solid,
             const float *Fx, const float *Fy, const float *Fz,
             float *rho, float *ux, float *uy, float *uz,
             const float *cfw, const float *uref,
             int nx, int ny, int nz, float tau0, float csmag2, void *stream);

/* Replaces the `lbm_bc` kernel of floodsim/lbm3d.py:145-175 (launched at
 * lbm3d.py:404): inlet velocity uin[y + ny*z] at x=0 and outlet density rho_out
 * at x=nx-1, in place on fd. */
int lbm_bc(float *fd, const uint8_t *solid, const float *uin,
           int nx, int ny, int nz, float rho_out, void *stream);

/* The reach builder's full arrays (build_reach / wall_cf, floodsim/reach3d.py:201-297,
 * 315-343), reference layout c = x + nx*(y + ny*z).  lbm_build_reach_masks: bed = outside[y]
 * or z < kb[y*nx + x]; solid = bed, or inside a hull segment of column x: segs[3k..3k+2] =
 * (y0, y1, z0) for k in [seg_off[x], seg_off[x+1]), solid for y0 <= y <= y1 and z >= z0.
 * lbm_build_reach_walls: fluid cells joined by a D3Q19 link to the bed (the bed below z = 0
 * and the y edges counting as bed; x beyond the ends read as the end columns) get
 * bedwall = 1 and cf = cf_col[y*nx + x]; other fluid cells joined to a hull (solid, not bed)
 * get cf = cf_hull; the first and last two x columns get neither.  hull_scratch: N bytes.
 * No counterpart in the reference (its builder is host NumPy). */
int lbm_build_reach_masks(int nx, int ny, int nz, const int32_t *kb, const uint8_t *outside,
                          const int32_t *seg_off, const int32_t *segs, uint8_t *solid, uint8_t *bed,
                          void *stream);
int lbm_build_reach_walls(int nx, int ny, int nz, const uint8_t *solid, const uint8_t *bed,
                          uint8_t *hull_scratch, const float *cf_col, float cf_hull, float *cf,
                          uint8_t *bedwall, void *stream);

/* Float64 solver of the accuracy statements (no counterpart in the reference, which
 * has no float64 GPU path).  lbm_step_f64 / lbm_bc_f64 are lbm_step / lbm_bc with
 * float64 populations, fields, forces and arithmetic (floodsim/lbm3d.py:31-175 in
 * float64); lbm_update_uref_f64 is Run3D._update_uref (floodsim/reach3d.py:412-418), and
 * sponge_cols / sponge_tau the outlet sponge of lbm_lattice (0: none):
 * uref = |sum over the fluid cells of a z column of (ux, uy)| / their count, at cells
 * where bedwall != 0, else 0.  Same layout as lbm_step; one thread per cell. */
int lbm_step_f64(const double *fs, double *fd, const uint8_t *solid,
                 const double *Fx, const double *Fy, const double *Fz,
                 double *rho, double *ux, double *uy, double *uz,
                 const double *cfw, const double *uref,
                 int nx, int ny, int nz, double tau0, double csmag2,
                 int sponge_cols, double sponge_tau, void *stream);
int lbm_bc_f64(double *fd, const uint8_t *solid, const double *uin,
               int nx, int ny, int nz, double rho_out, void *stream);
int lbm_update_uref_f64(const double *ux, const double *uy, const uint8_t *solid,
                        const uint8_t *bedwall, double *uref, int nx, int ny, int nz, void *stream);

/* Lattice description for the fused path.  All pointers are device memory;
 * per-cell arrays hold `cells` = pitch*ny*nz entries. */
typedef struct lbm_lattice {
    int32_t nx, ny, nz, pitch;
    int64_t cells;
    float tau0, csmag2;     /* relaxation time at zero strain; Smagorinsky constant squared */
    float rho_out;          /* outlet density (1.0 in floodsim) */
    float force_scale;      /* multiplies Fx,Fy,Fz (the force ramp of Run3D) */
    const uint32_t *flags;  /* cell flag words */
    const float *Fx, *Fy, *Fz;
    const float *cfw;       /* wall-function friction coefficient tau = rho cf U^2 */
    const float *uref;      /* per-cell reference speed (used without LBM_STEP_UREF_COLUMN) */
    const float *uin;       /* inlet profile, nz*ny, index y + ny*z */
    float *rho, *ux, *uy, *uz;
    float *colU;            /* column-mean speed, ny*pitch, index x + pitch*y */
    float *avg;             /* 6*cells accumulators, or NULL */
    int32_t *status;        /* device status word: bit 0 = non-finite or non-positive density seen,
                               bit 1 = a bounded wait for staged data ran out (data not trusted) */
    /* Work lists of pipeline LBM_PIPE_SPLIT (lbm_build_worklists): ids (z*ny + y)*nseg + seg
     * of the plain, solid, special and edge row segments of 32*list_cells_per_lane cells. */
    const uint32_t *rows_plain, *rows_solid, *rows_special;
    int32_t n_plain, n_solid, n_special, list_cells_per_lane;
    const uint32_t *rows_edge;
    int32_t n_edge;
    /* Optional outlet sponge (no counterpart in the reference; 0 = the reference's outlet):
     * over the last sponge_cols x columns the relaxation time at zero strain rises from tau0
     * to sponge_tau as tau0 + (sponge_tau - tau0) s^2, s = (x - (nx - sponge_cols) + 1) /
     * sponge_cols, damping the backflow the fixed-pressure outlet does not.  Split pipeline
     * only; segments that reach into the sponge are special segments. */
    int32_t sponge_cols;
    float sponge_tau;
    int32_t reserved;
} lbm_lattice;

/* Launch shape of lbm_fused_step.
 *   pipeline LBM_PIPE_REGISTER: a warp covers 32*cells_per_lane cells of a row with
 *     V-wide register loads and warp shuffles (cells_per_lane 2 or 4; warps 1..4 per
 *     CTA; stages unused);
 *   pipeline LBM_PIPE_TMA: `warps` (2, 4 or 8) consumer warps cover 32*warps cells of a
 *     row, one per thread, fed by one producer warp whose bulk asynchronous copies stage
 *     the 19 source rows (+ a 16-byte halo) and the flag row into a ring of `stages`
 *     (2..8) shared-memory slots and copy the output rows back (cells_per_lane 1).
 *   pipeline LBM_PIPE_ASYNC: every warp is independent and covers 64 cells of a row,
 *     two per lane (cells_per_lane 2); it stages the 19 source rows (+ one halo cell
 *     each side) and the flag row of the next stages-1 rows into a private ring of
 *     `stages` (2..4) shared-memory slots with cp.async while colliding the current row
 *     (warps 1..8 per CTA).
 *   pipeline LBM_PIPE_SPLIT: the register/shuffle pull over static work lists of row
 *     segments (lbm_build_worklists): plain interior segments run a lean kernel that reads
 *     no flag words, edge segments the same plus the x-edge copies and inlet/outlet
 *     extrapolation, special segments (walls, bed, lid, banks, hulls, forcing) a separately
 *     compiled general one, and solid segments move no populations (cells_per_lane 2 or 4
 *     as the lists were built; warps 1..4 per CTA).
 * ctas_per_sm: resident CTAs per SM of the persistent grid (0 = as many as fit). */
#define LBM_PIPE_REGISTER 0
#define LBM_PIPE_TMA 1
#define LBM_PIPE_ASYNC 2
#define LBM_PIPE_SPLIT 3
typedef struct lbm_tile {
    int32_t pipeline, cells_per_lane, warps, stages, ctas_per_sm;
} lbm_tile;

/* Fills flags (cells entries) from solid (uint8, pitched, x >= nx ignored) and
 * lat->Fx/Fy/Fz/cfw and the optional bedwall mask (uint8, pitched; NULL = none).
 * Wall bits follow floodsim/lbm3d.py:50-58. */
int lbm_build_flags(const lbm_lattice *lat, const uint8_t *solid, const uint8_t *bedwall,
                    uint32_t *flags, void *stream);

/* 1D-profile start, floodsim/lbm3d.py:362-364 + 377-384: f = feq(rho=1,
 * u=(uin(y,z),0,0)) for fluid cells, feq(1,0) for solid and padding cells,
 * evaluated in float64 like the reference's NumPy code.  f: float[19*cells]. */
int lbm_init_equilibrium(const lbm_lattice *lat, float *f, void *stream);

/* Classifies every row segment of 32*cells_per_lane cells (cells_per_lane 2, 4 or 8; from
 * lat->flags, which must be built) and writes each class's segment ids, in increasing order:
 *   plain   -- open row (1 <= y <= ny-2, 1 <= z <= nz-1, the row under the rigid lid
 *              included), x clear of 0 and nx-1, and no cell solid, walled, forced or
 *              under the wall function;
 *   edge    -- the same, but holding x = 0 or x = nx-1 (and possibly x padding);
 *   solid   -- every cell solid or padding;
 *   special -- all others (walls, bed, lid, banks, hulls, forcing).
 * Each of the four arrays and `scratch` (uint8) must hold nseg*ny*nz entries, nseg =
 * ceil(pitch / (32*cells_per_lane)); counts (device, int32[4]) receives the list lengths in
 * the order plain, solid, special, edge.  Rebuild whenever the flags change. */
int lbm_build_worklists(const lbm_lattice *lat, int cells_per_lane, uint8_t *scratch, uint32_t *plain,
                        uint32_t *solid, uint32_t *special, uint32_t *edge, int32_t *counts, void *stream);

/* lbm_build_worklists without the caller's scratch buffer; no counterpart in the reference
 * (floodsim has no work lists).  For callers that may not allocate device memory while they
 * run: hosts whose own allocator reserves the GPU up front and permits no other allocation,
 * and time loops that cannot take cudaMalloc/cudaFree's device-wide synchronisation.  It
 * calls no allocator: the scratch is a 4 MiB array of the library (held on every GPU that
 * loads it, until exit).  Limit: nseg*ny*nz <= 4194304 row segments; larger lattices return
 * LBM_ERR_ARG with a message naming the limit (checked before the other arguments).  The
 * array's address belongs to a CUDA context: the first call in each context (a device's
 * primary context, a context the host created itself, the new primary context after
 * cudaDeviceReset) looks it up there and caches it under the context's id, so make that call
 * before any stream capture in that context.  All calls in a context share the array: calls
 * whose kernels overlap on the GPU (other streams, other host threads) race.
 * Outputs and their sizes are those of lbm_build_worklists. */
int lbm_build_worklists_noalloc(const lbm_lattice *lat, int cells_per_lane, uint32_t *plain,
                                uint32_t *solid, uint32_t *special, uint32_t *edge, int32_t *counts,
                                void *stream);

/* One fused time step fs -> fd (see the file comment); mode = LBM_STEP_* bits. */
int lbm_fused_step(const lbm_lattice *lat, const float *fs, float *fd, uint32_t mode,
                   const lbm_tile *tile, void *stream);

/* 16-bit population storage (no counterpart in the reference, whose populations are float32).
 * Element i*cells + c holds fp16_rn((f_i - w_i) * scale): the population's deviation from its
 * lattice weight, times `scale`, a power of two in [2^-8, 2^24] chosen per lattice (LBM_ERR_ARG
 * otherwise).  Scaling is exact, so `scale` only places the fp16 exponent range: deviations up to
 * 65504/scale are representable and those above 2^-14/scale keep fp16's 11-bit significand.
 * Collision runs in float32 exactly as in lbm_fused_step; a step moves 76 bytes per cell. */

/* The start state of lbm_init_equilibrium, stored 16-bit.  h: uint16[19*cells]. */
int lbm_init_equilibrium_h(const lbm_lattice *lat, uint16_t *h, float scale, void *stream);

/* float populations f[19*cells] -> 16-bit storage (round to nearest) and back. */
int lbm_pack_populations(const lbm_lattice *lat, const float *f, uint16_t *h, float scale, void *stream);
int lbm_unpack_populations(const lbm_lattice *lat, const uint16_t *h, float *f, float scale, void *stream);

/* One fused time step hs -> hd on 16-bit storage; same physics, modes and fields as
 * lbm_fused_step.  Requires pitch % 8 == 0, work lists built with cells_per_lane 2, 4 or 8 (row
 * segments of 64, 128 or 256 cells) and tile {LBM_PIPE_SPLIT, that cells_per_lane, warps 1..4,
 * stages, ctas_per_sm} (NULL tile = 2 cells per lane, 4 warps, as many CTAs per SM as fit).
 * Plain segments move `stages` = 8 (or 0) cells per lane with 16-byte accesses, or 4 cells per
 * lane with 8-byte accesses (stages = 4, lists of 64 or 128 cells); edge and special segments
 * run the general path with 2 cells per lane (cells_per_lane 2) or 4 (one pass, or two for
 * 256-cell segments). */
int lbm_fused_step_h(const lbm_lattice *lat, const uint16_t *hs, uint16_t *hd, float scale, uint32_t mode,
                     const lbm_tile *tile, void *stream);

/* Batched 16-bit solves (no counterpart in the reference, which runs one case at a time):
 * `count` lattices (boat cases of any sizes, one run) advanced by one launch per kernel class
 * per step.  Every table is in device memory:
 *   lat          count lattice descriptors (each as for lbm_fused_step_h, with its own work
 *                lists built for cells_per_lane 2 and the same uref mode for all);
 *   pull_offsets count * lbm_batch_pull_offsets_bytes() bytes, filled by lbm_batch_init;
 *   scale        count 16-bit storage scales;
 *   pop0, pop1   count population buffers each (uint16[19*cells] of that lattice);
 *   rows_*       the cases' work lists concatenated, each entry (case << 24) | segment id
 *                (segment ids below 2^24);
 *   max_columns  the largest ny*pitch, max_rows the largest ny*nz of the lattices.
 * A step reads pop0 and writes pop1 when parity is 0, the reverse when it is 1; the rest of
 * the lattice descriptors (force_scale, fields, status) are read from device memory at run
 * time, so a chunk of steps can be captured in a CUDA graph once and replayed. */
typedef struct lbm_batch {
    int32_t count, max_columns, max_rows, reserved;
    const lbm_lattice *lat;
    void *pull_offsets;
    const float *scale;
    uint16_t *const *pop0;
    uint16_t *const *pop1;
    const uint32_t *rows_plain, *rows_solid, *rows_special, *rows_edge;
    int32_t n_plain, n_solid, n_special, n_edge;
} lbm_batch;

int lbm_batch_pull_offsets_bytes(void);
int lbm_batch_init(const lbm_batch *b, void *stream);

/* One step of every lattice of the batch; mode = LBM_STEP_* bits (for all lattices); tile
 * {LBM_PIPE_SPLIT, 2, warps 1..4, stages (plain-kernel cells per lane 8, or 4; 0 = 8),
 * ctas_per_sm}, NULL = {LBM_PIPE_SPLIT, 2, 4, 0, 0}. */
int lbm_batch_step_h(const lbm_batch *b, int parity, uint32_t mode, const lbm_tile *tile, void *stream);

/* `nsteps` steps of every lattice of the batch in ONE persistent, cooperative launch (no
 * counterpart in the reference): every CTA stays resident for the chunk, the steps are
 * separated by grid-wide barriers, and within a step the special, edge and plain segments of
 * all cases are interleaved over all warps.  Step s reads pop0 when (parity0 + s) is even.
 * mode: the inner steps' bits (LBM_STEP_UREF_COLUMN or 0); last_mode: the last step's, with
 * LBM_STEP_OUTPUT (and optionally LBM_STEP_ACCUMULATE) and the same UREF_COLUMN bit.  The same
 * populations and fields as nsteps calls of lbm_batch_step_h, bit for bit.  sync: 4 uint32 of
 * device memory the call clears and the barriers use (one chunk at a time per sync buffer).
 * Every barrier wait is bounded (2 s of the GPU's global timer); if one runs out the chunk stops
 * and bit 1 of every case's status word is set. */
int lbm_batch_chunk_h(const lbm_batch *b, int parity0, int nsteps, uint32_t mode, uint32_t last_mode,
                      uint32_t *sync, void *stream);

/* Along-stream profiles in float64 (floodsim/reach3d.py:545-568 reduces the same sums with
 * NumPy on the host).  From lat->avg (the time-average sums, scaled by inv_navg) when it is
 * not NULL, else from the instantaneous lat->rho/ux/uy/uz, over the fluid cells:
 *   prof[k*nx + x], k = 0 sum ux, 1 sum ux^2, 2 sum (rho-1), 3 sum rho, 4 fluid cells,
 *   5 top-layer (z = nz-1) fluid cells, 6 top-layer sum (rho-1), 7 top-layer sum ux,
 *   8 max |u|;
 *   bed_speed2[x + nx*y] = the largest |u|^2 of a fluid cell whose lower neighbour is solid
 *   or the bed (the bed-shear cells).
 * All in lattice units, each sum over one cross-section x.  Deterministic: the sums are
 * added in a fixed order.  scratch: lbm_profiles_scratch_doubles(lat) doubles. */
int64_t lbm_profiles_scratch_doubles(const lbm_lattice *lat);
int lbm_profiles(const lbm_lattice *lat, double inv_navg, double *prof, double *bed_speed2, double *scratch,
                 void *stream);

/* Float64 force sums (no counterpart in the reference, which infers the boats' net force from
 * the momentum-flux difference along the reach, floodsim/reach3d.py:604-609).  From the state
 * f (the populations the last step stored, float or, _h, 16-bit with its scale) and the fields
 * and wall-model speed the next step reads (colU with LBM_STEP_UREF_COLUMN in mode, else
 * lat->uref): the next step's bounce-back at every fluid cell whose pull source x - c_i is a
 * cell of body k (body[c] = k in 1..nbody, pitched like the flags; 0 = not a body) returns the
 * cell's own f_opp(i), corrected by the wall function of floodsim/lbm3d.py:61-101, as f_i, and
 * body k receives -c_i (f_opp(i) + f_i) over that link (momentum exchange; where the source was
 * mirrored by the rigid lid into the cell's own layer, only its horizontal part).
 *   out[3*(k-1) + d]  force on body k, component d (x, y, z);
 *   out[3*nbody + d]  the body force the step applies: sum of F * force_scale over forced
 *                     fluid cells (propellers and jets).
 * Lattice units (momentum per cell volume per step; times rho dx^4/dt^2 gives newtons).
 * nbody <= 16; body may be NULL when nbody == 0.  Deterministic (fixed summation order).
 * scratch: lbm_body_forces_scratch_doubles(nbody) doubles. */
int64_t lbm_body_forces_scratch_doubles(int nbody);
int lbm_body_forces(const lbm_lattice *lat, const float *f, const uint8_t *body, int nbody, uint32_t mode,
                    double *out, double *scratch, void *stream);
int lbm_body_forces_h(const lbm_lattice *lat, const uint16_t *h, float scale, const uint8_t *body, int nbody,
                      uint32_t mode, double *out, double *scratch, void *stream);

/* The web viewer's velocity export (floodsim/web3d.py:35-56, STRIDE 2): the time-averaged
 * velocity (the float32 sums lat->avg over navg outputs, times vel = dx/dt) averaged over
 * the fluid cells of each 2 x 2 horizontal block and quantised to int8 with one scale,
 * float32(max |component| / 126): q[b*3 + k] = clip(round-half-even(v / scale), +-126), or
 * -128 for a block without fluid; sp[b] = float32 |v| of the block (0 without fluid).
 * Blocks b = i + nx2*(j + ny2*z), nx2 = nx/2, ny2 = ny/2 (lbm_export_blocks returns their
 * count).  pooled: caller scratch of 4 floats per block (16-byte aligned); umax_bits: one
 * device word, returns the bits of max |component| (0 when every component is 0).  Bit for
 * bit the reference's arithmetic. */
int64_t lbm_export_blocks(const lbm_lattice *lat);
int lbm_export_velocity(const lbm_lattice *lat, int navg, float vel, float *pooled,
                        uint32_t *umax_bits, int8_t *q, float *sp, void *stream);

/* Tracer particles (Run3D.move_particles, floodsim/reach3d.py:508-536): P holds n
 * positions (x, y, z) in float64 metres, row-major (n x 3), with x from the inlet face, y
 * from the first lattice row and z from the domain bottom.  Each particle moves by the
 * velocity of the cell it is in (lat->ux/uy/uz, lattice units) times vel (m/s per lattice
 * unit) times dt (s), in the reference's float32 arithmetic; one that leaves the domain,
 * stops being finite or lands in a solid cell restarts in [0, 2 dx) x a random fluid cell of
 * the x = 1 column: inlet[] holds z*ny + y of those cells.  Restart positions come from
 * SplitMix64 of (seed, counter, particle), so pass a new counter per call.  respawned: one
 * device int incremented per restart (or NULL). */
int lbm_move_particles(const lbm_lattice *lat, double *P, int64_t n, float vel, float dt, double dx,
                       const int32_t *inlet, int32_t n_inlet, uint64_t seed, uint64_t counter,
                       int32_t *respawned, void *stream);

/* BF16 tensor-core GEMM of the learned warm start (no counterpart in the reference):
 * D[M x N] = A[M x K] * B[N x K]^T, A and B bf16 row-major with K contiguous (leading
 * dimensions lda, ldb; K, lda, ldb multiples of 8; A, B 16-byte aligned), products accumulated
 * in float32 on the tensor cores (tcgen05, accumulator in tensor memory).  epilogue:
 * 0 D float = acc; 1 D float += acc; 2 D bf16 = acc + bias[n]; 3 D bf16 = max(acc + bias[n], 0);
 * 4 D float = acc + bias[n] (bias may be NULL).  err (device int) is set to 1 if a tile's wait for its tensor-core
 * operations ran out (the result is then not valid).  Products with M >= 1024 and N >= 128 run a
 * persistent kernel that holds one SM's whole tensor memory (512 columns) and most of its shared
 * memory per CTA, one CTA per SM; smaller ones one 128-row tile per CTA.  Both read A and B
 * through tensor maps of this GPU's memory (no multicast): A and B must be on the current
 * device. */
int lbm_gemm_bf16(const uint16_t *A, int lda, const uint16_t *B, int ldb, int M, int N, int K, void *D, int ldd,
                  int epilogue, const float *bias, int *err, void *stream);

/* Support kernels of the learned warm start's network (no counterpart in the reference).
 * Activations are channels-last bf16 (x[v*C + c], voxel v = x + X*(y + Y*z) of a (Z, Y, X)
 * grid); a 3x3x3 tap t = (dz+1)*9 + (dy+1)*3 + (dx+1), zero outside the grid.
 *   im2col     col[v][t*C + c] = x[tap t of v][c]                (C a multiple of 8)
 *   col2im     dx[v][c] = sum of dcol[u][t*C + c] over the (u, t) that read v   (float)
 *   transpose  out[c][r] = in[r][c] (bf16, R rows -> Rp >= R columns, zero padded)
 *   act_grad   g = dy * (y > 0) (relu) or dy, as bf16; dbias[c] += column sums of g
 *   pool2      2x2x2 average (even grid sizes) and pool2_back its gradient (added to din when
 *              accumulate is set)
 *   up2_add    out = nearest 2x upsampling of coarse + skip, and up2_back the coarse gradient
 *   mse        masked mean-square error of pred[v][0..nout) (row stride Cp): loss += and dpred
 *   adam       Adam step on float32 weights (bias-corrected, step >= 1), refreshing a bf16 copy */
int lbm_nn_im2col(const uint16_t *x, int C, int X, int Y, int Z, uint16_t *col, void *stream);
int lbm_nn_col2im(const float *dcol, int C, int X, int Y, int Z, float *dx, void *stream);
int lbm_nn_transpose(const uint16_t *in, int64_t R, int C, int64_t Rp, uint16_t *out, void *stream);
int lbm_nn_act_grad(const float *dy, const uint16_t *y, int64_t V, int C, int relu, uint16_t *g, float *dbias,
                    void *stream);
int lbm_nn_pool2(const uint16_t *in, int C, int X, int Y, int Z, uint16_t *out, void *stream);
int lbm_nn_pool2_back(const float *dout, int C, int X, int Y, int Z, float *din, int accumulate, void *stream);
int lbm_nn_up2_add(const uint16_t *coarse, const uint16_t *skip, int C, int X, int Y, int Z, uint16_t *out,
                   void *stream);
int lbm_nn_up2_back(const float *dout, int C, int X, int Y, int Z, float *dcoarse, void *stream);
int lbm_nn_mse(const float *pred, int Cp, const float *target, int nout, const float *mask, int64_t V, float inv_n,
               float *dpred, float *loss, void *stream);
int lbm_nn_adam(float *w, const float *g, float *m, float *s, int64_t n, float lr, float b1, float b2, float eps,
                int step, uint16_t *wbf16, void *stream);

/* Start state from a coarse flow prediction (learned warm start; no counterpart in the
 * reference).  coarse: float (Z*Y*X, stride >= 4), channels (du, v, w, drho) per coarse voxel
 * of factor^3 cells; per fluid cell, trilinear between voxel centres: u = (uin(y,z) + du*su,
 * v*su, w*su), rho = 1 + drho*srho.  Writes f (float[19*cells]) = feq(rho, u) and the fields
 * rho/ux/uy/uz; solid and padding cells at rest. */
int lbm_lift_coarse(const lbm_lattice *lat, const float *coarse, int stride, int X, int Y, int Z, int factor,
                    float su, float srho, float *f, void *stream);

/* Number of streaming multiprocessors of the current device. */
int lbm_device_sm_count(void);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
