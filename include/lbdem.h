/*
 * lbdem.h -- C ABI of the B200 (sm_100a) resolved LBM-DEM step library
 * (liblbdem.so).  Plain pointers, sizes and POD descriptors; no torch types.
 *
 * Conventions
 *  - Every entry point is asynchronous on the caller's CUDA stream (`stream`
 *    is a cudaStream_t passed as void*; NULL = legacy default stream).
 *  - The library never allocates or frees device memory: every buffer is
 *    owned by the caller and passed in (the Python layer uses torch tensors).
 *  - Return value: LBDEM_OK or an LBDEM_ERR_* code (argument/launch errors,
 *    detected on the host).  Numerical/capacity faults found on the device are
 *    OR-ed into a caller-provided int32 status word (LBDEM_ST_* bits) that the
 *    caller reads at a synchronisation point of its choice.
 *  - Per-cell arrays (rho, vel, links, keys, ...) are x fastest: cell
 *    (x, y, z) -> (z*Ny + y)*Nx + x, vector fields as SoA planes of Ncells.
 *    (The reference's Taichi fields are indexed [i, j, k] = [x, y, z].)
 *  - Populations are blocked by 32 cells along x: with NB = ceil(Nx/32),
 *    population q of cell (x, y, z) is element
 *        ((z*Ny + y)*NB + x/32)*19*32 + q*32 + x%32
 *    (buffer of 19*32*NB*Ny*Nz elements; lanes x >= Nx of the last block are
 *    padding).  The lagged Smagorinsky state uses the same blocking with 5
 *    values per cell.
 *  - Populations are stored as scaled deviations from the lattice weights,
 *    h_q = (f_q - w_q) * S / w_q with S = 1 (FP32) or scale16 (FP16 / BF16);
 *    arithmetic is FP32 in every form.
 *  - Particle (DEM) state is FP64, array-of-structures (n, 3) like the
 *    reference's Grain fields.
 *
 * Reference interfaces replaced (dasfadwqd/LBDEM-Taichi):
 *  lbdem_lattice_init     <- PSCLattice3D.initialize      src/lbdem/psclattice3d.py:60-78
 *  lbdem_psc_map          <- PSCLattice3D.grains2lattice  src/lbdem/psclattice3d.py:84-182
 *  lbdem_psc_step_*       <- PSCLattice3D.collide + BasicLattice3D.stream
 *                            src/lbdem/psclattice3d.py:187-358,
 *                            src/lbm3d/lbm_solver3d.py:176-342,460-513,
 *                            src/lbm3d/lbm_foecelover.py:52-68
 *  lbdem_stream_moments_* <- BasicLattice3D.stream (+compute_rho_vel)
 *                            src/lbm3d/lbm_solver3d.py:197-303
 *  lbdem_psc_decode       <- PSCLattice3D fields id/volfrac/weight/velsolid
 *                            src/lbdem/psclattice3d.py:45-52
 *  lbdem_dem_bin,
 *  lbdem_dem_substeps     <- DEMSolver.run_simulation     src/dem3d/demsolver/demsolver.py:848-862
 *                            (BPCD bpcd.py:67-152, resolve :638-740,
 *                             resolve_wall :809-838, update :514-636,
 *                             hertz.py:45-153, linear.py:43-152)
 *  lbdem_build_links      <- CellType dispatch in BasicLattice3D.stream
 *                            src/lbm3d/lbm_solver3d.py:203-236
 *  lbdem_boundary_cells   <- second pass of BasicLattice3D.stream (wet-node cells)
 *                            src/lbm3d/lbm_solver3d.py:242-250
 *  lbdem_global_sums_f64  <- (no counterpart; FP64 conservation totals)
 *  lbdem_psc_map_smooth,
 *  lbdem_psc_step_adjoint_f32,
 *  lbdem_psc_force_adjoint <- (no counterpart; the reference has no gradients:
 *                            reverse mode of PSCLattice3D.collide + stream +
 *                            lattice2grains, psclattice3d.py:187-358,
 *                            lbm_solver3d.py:197-240, lbm_foecelover.py:52-68,
 *                            on a frozen bed with a smooth solid fraction)
 */
#ifndef LBDEM_H
#define LBDEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBDEM_ABI_VERSION 4

/* return codes */
#define LBDEM_OK 0
#define LBDEM_ERR_ARG 1
#define LBDEM_ERR_LAUNCH 2
#define LBDEM_ERR_UNSUPPORTED 3

/* device status bits (OR-ed into *status) */
#define LBDEM_ST_NAN 1u              /* non-finite population or moment */
#define LBDEM_ST_RHO 2u              /* density <= 0 in a fluid cell */
#define LBDEM_ST_VELMAX 4u           /* |u| >= sqrt(2/3) (lbm_solver3d.py:94,301) */
#define LBDEM_ST_CONTACT_OVERFLOW 8u /* more contacts than max_coordinate_number */
#define LBDEM_ST_GRID_OVERFLOW 16u   /* particle outside the broad-phase grid */
#define LBDEM_ST_GID_OVERFLOW 32u    /* more than 2^24-1 particles in the PSC map */
#define LBDEM_ST_CELL_OVERFLOW 64u   /* a broad-phase cell holds more than cell_cap particles */
#define LBDEM_ST_WAIT_TIMEOUT 128u   /* a bounded wait for an asynchronous copy gave up */
#define LBDEM_ST_PIPELINE_MARGIN 256u /* a particle moved farther in one step than the margin a
                                         pipelined step assumed (lbdem_psc_near_blocks) */

/* storage forms */
#define LBDEM_F32 0
#define LBDEM_F16 1
#define LBDEM_BF16 2

/* Smagorinsky modes */
#define LBDEM_SMAG_OFF 0
#define LBDEM_SMAG_REFERENCE 1 /* lagged: feq and omega of the previous collide (lbm_solver3d.py:460-513) */
#define LBDEM_SMAG_LOCAL 2     /* current feq, omega0 prefactor; no per-cell state */

/* CellType bits (src/lbm3d/lbmutils.py:69-97) */
#define LBDEM_CT_FLUID 1
#define LBDEM_CT_OBSTACLE 8
#define LBDEM_CT_FREE_SLIP 16
#define LBDEM_CT_VEL_LADD 32
#define LBDEM_CT_VEL_ZOUHE 64
#define LBDEM_CT_VEL_EXIT 128
#define LBDEM_CT_PRE_ZOUHE 256
#define LBDEM_CT_VEL_INLET_LADD 262144
#define LBDEM_CT_RIGHT 4096    /* face bits of open-boundary cells (x = Nx-1) */
#define LBDEM_CT_LEFT 8192     /* x = 0 */
#define LBDEM_CT_TOP 16384     /* y = Ny-1 */
#define LBDEM_CT_BOTTOM 32768  /* y = 0 */
#define LBDEM_CT_FRONT 65536   /* z = Nz-1 */
#define LBDEM_CT_BACK 131072   /* z = 0 */

/* link-mask bit of a FLUID cell (the value of every mask of an all-FLUID lattice) */
#define LBDEM_LINK_FLUID (1u << 20)

typedef struct lbdem_lattice {
    int32_t nx, ny, nz;
    int32_t storage;       /* LBDEM_F32 / LBDEM_F16 / LBDEM_BF16 */
    float omega0;          /* 1/tau */
    float smag_cs;         /* Smagorinsky constant */
    int32_t smag_mode;     /* LBDEM_SMAG_* */
    int32_t force_on;      /* 1: add w_q rho (c_q . F)/cs^2 to post-collision populations */
    float force[3];        /* body force, lattice units */
    float scale16;         /* storage scale of the 16-bit forms */
    void *f[2];            /* population buffers, 19*32*NB*Ny*Nz elements of the storage type (blocked) */
    float *rho;            /* Ncells, FP32 (moments; also the initial state) */
    float *vel;            /* 3*Ncells, FP32 SoA (ux | uy | uz) */
    void *aux;             /* lagged state (drho, u, omega) of the last collision, 5*32*NB*Ny*Nz of the
                              storage type, or FP16 with aux_half (blocked): required by LBDEM_SMAG_REFERENCE and by
                              lbdem_stress, NULL otherwise (then the step neither reads nor writes it) */
    const uint32_t *links; /* per-cell link mask from lbdem_build_links */
    int32_t *status;       /* device status word */
    const uint32_t *moving; /* per-cell bit q: neighbour x - c_q is a moving wall (VEL_LADD), from
                               lbdem_build_links; NULL when the lattice has no moving walls.  The
                               wall velocity is read from vel at the wall cell, the lagged density
                               of the cell from rho (the step keeps it current for these cells).
                               Also set for Ladd velocity inlets (VEL_INLET_LADD), whose links
                               use the inlet's velocity and density. */
    /* Open boundaries (Zou-He velocity / pressure, convective exits, Ladd
     * inlets, free-slip neighbours): the cells listed by lbdem_boundary_cells
     * are streamed and collided by a boundary pass that every step and
     * stream call runs after its main kernel.  bnd_na + bnd_nb = 0 (and the
     * pointers NULL) for a lattice without such cells. */
    const int32_t *ct;          /* CellType per cell (device), required when bnd_na + bnd_nb > 0 */
    const uint32_t *bnd_cells;  /* bnd_na first-pass cells, then bnd_nb second-pass cells (exits, inlets) */
    uint32_t bnd_na, bnd_nb;
    void *bnd_f0;               /* 19 * bnd_nb elements of the storage type ([q][t], t = second-pass index):
                                   the Ladd inlets' constant populations, captured by the first step after
                                   lattice_init or a stream call; required when bnd_nb > 0 */
    int32_t bnd_slip;           /* 1: the lattice has FREE_SLIP cells (their mirrors read inlets'
                                   post-collision populations, which are then stored) */
    float *stress;              /* optional 7 * Ncells FP32 planes (xx, yy, zz, xy, xz, yz, shear
                                   magnitude): when not NULL, lbdem_psc_step_* also writes the stress
                                   diagnostics of the post-stream state it gathers (its input) -- what
                                   lbdem_stress would give for that state, fused into the step
                                   (BasicLattice3D.compute_stress, src/lbm3d/lbm_solver3d.py:347-404).
                                   Needs aux; not supported with boundary-pass cells (bnd_na + bnd_nb
                                   > 0) nor by lbdem_psc_step_phase, which ignores it. */
    uint32_t links_all;         /* nonzero: every cell's link mask equals this value (a lattice without
                                   walls or special cells, all FLUID: the mask lbdem_build_links gives
                                   is then LBDEM_LINK_FLUID everywhere); the step kernels then read no
                                   per-cell masks.  0: read links[]. */
    int32_t aux_half;           /* 1: aux holds FP16 elements under FP32 storage -- the lagged state at
                                   half the bytes (20 B per cell less traffic for the step with
                                   LBDEM_SMAG_REFERENCE), rounded to FP16 between steps; no counterpart
                                   in the reference, whose lagged state is FP32.  0: aux has the storage
                                   type.  Must be 0 for the 16-bit storage forms. */
} lbdem_lattice;

typedef struct lbdem_grains {
    int32_t n;
    const double *pos;     /* (n,3) physical */
    const double *radius;  /* (n) */
    const double *vel;     /* (n,3) */
    const double *omega;   /* (n,3) */
    double *force_fluid;   /* (n,3) written by lbdem_psc_step_* (physical units) */
    double *moment_fluid;  /* (n,3) */
} lbdem_grains;

typedef struct lbdem_psc {
    double dx, dt, rho_unit;   /* UnitConverter(dx, dt, rho) */
    double xmin, ymin, zmin;   /* DEM domain minimum (config.domain) */
    int32_t skip_inlet;        /* 1: VEL_INLET_LADD cells are also skipped by the map */
    uint32_t *key;             /* Ncells owner keys (0 = no solid) */
    float *table;              /* 16*n floats per particle: floor(centre), frac(centre), v*dt/dx, omega*dt */
    double *prev;              /* 4*n: lattice centre and mapping radius of the previous map */
    int32_t have_prev;         /* 1: prev holds a map to clear */
    float *hydro_out;          /* optional per-cell hydrodynamic force (3*Ncells) or NULL */
    float *eps;                /* smooth solid fraction per cell (lbdem_psc_map_smooth), or NULL:
                                  the step then takes the exact 5^3 count from the key */
    /* Map reuse (no counterpart in the reference, which remaps every step): with
     * map_moved set (2 uint32 of caller device memory) and map_reuse = 1,
     * lbdem_psc_map first checks whether any particle's lattice centre or
     * mapping radius differs from the previous exact map's; if none does, the
     * owner keys are already exact and only the particle table and the force
     * accumulators are refreshed.  Set map_reuse = 0 whenever the cell types
     * (link masks) changed since the previous map.  map_parity is the
     * library's own toggle (start at 0). */
    uint32_t *map_moved;
    int32_t map_reuse;
    int32_t map_parity;
    /* Periodic images (no counterpart in the reference, whose mapping never
     * wraps, psclattice3d.py:102-108): wrap[a] = 1 maps a sphere that crosses
     * the periodic faces of axis a also through its image shifted by
     * period[a] lattice units (the DEM domain length / dx), and the step takes
     * the minimum image for lever arms and solid velocities.  The exact map
     * only; 0 everywhere reproduces the reference. */
    int32_t wrap[3];
    double period[3];
    /* Pipelined stepping (lbdem_psc_near_blocks / lbdem_psc_step_phase): the
     * DEM's periodic axes, and the largest distance (lattice units) a particle
     * may move between two maps; the map flags LBDEM_ST_PIPELINE_MARGIN when a
     * particle moved farther (minimum image on periodic axes).  0 = no check. */
    int32_t periodic[3];
    double disp_limit;
} lbdem_psc;

typedef struct lbdem_dem {
    int32_t n, maxc;
    int32_t model;                 /* 0 Hertz-Mindlin, 1 linear */
    double dt, g[3];
    double dom_min[3], dom_max[3]; /* config.domain */
    int32_t periodic[3];
    double bp_min[3];              /* broad-phase origin (init_particle_fields domain_min) */
    double cell_size;              /* 4 * max radius (bpcd.py:42) */
    int32_t gdim[3];               /* dense broad-phase grid, cells -1 .. gdim-2 per axis */
    /* materials: [0] particles, [1] walls */
    double E[2], nu[2], mu[2], e[2], kn[2], ks[2], dpn[2], dps[2];
    double wall_n[18], wall_d[6];
    int32_t wall_periodic[6];
    /* grains (n,...) */
    double *pos, *vel, *acc, *force, *quat, *omega, *omega_dot, *moment, *inertia, *mass, *radius;
    double *force_fluid, *moment_fluid;
    int32_t *freeze, *fixvel;
    /* contacts: n*maxc slots owned by the lower index, wall contacts n*6;
     * cfn = slots in use at the start of a sub-step, cf_add = slots appended
     * during it (zero between sub-steps) */
    int32_t *cf_j, *cf_active, *cfn, *cf_add;
    double *cf_shear, *cf_pos, *cf_force;
    int32_t *wcf_active;
    double *wcf_shear, *wcf_pos, *wcf_force;
    /* broad-phase scratch (caller-owned) */
    int32_t cell_cap;      /* particles a broad-phase cell can list */
    int32_t *cell_count;   /* 2 * prod(gdim), zero-initialised once (double-buffered counts) */
    int32_t *cell_list;    /* prod(gdim) * cell_cap particle ids */
    double *acc_force;     /* (n,3) contact force accumulator, zero between sub-steps */
    double *acc_moment;    /* (n,3) contact moment accumulator, zero between sub-steps */
    int32_t parity;        /* which half of cell_count holds the current binning */
    int32_t *status;
    uint32_t *sync;        /* 2 words of caller-owned device memory for the grid barrier of the
                              single-launch sub-step kernel (reset by the library on every call) */
    int32_t wrap_pairs;    /* 0: the reference's broad phase, which never proposes a pair across a
                              periodic face (bpcd.py:154-194, cells not wrapped); 1: also probe the
                              cells around a particle's periodic image when it lies within one
                              broad-phase cell of a periodic face (needs every periodic length
                              >= 4 cells; no counterpart in the reference) */
} lbdem_dem;

int lbdem_abi_version(void);
const char *lbdem_last_error(void);

int lbdem_build_links(const int32_t *ct, int32_t nx, int32_t ny, int32_t nz, int32_t skip_inlet,
                      uint32_t *links, uint32_t *moving, void *stream);

/* Deterministic list (lattice order) of the cells that the boundary pass
 * handles, from the link masks: first-pass cells (Zou-He, free-slip
 * neighbours), then second-pass cells (exits and Ladd inlets, which read their
 * interior neighbour's fresh moments).  counts (device, 2 uint32) receives
 * (n_a, n_b); at most `capacity` indices are written to `cells`, so a caller
 * reads counts and calls again with a larger array when n_a + n_b exceeds it.
 * scratch: 2 * Ny * Nz int32 of caller memory. */
int lbdem_boundary_cells(const uint32_t *links, int32_t nx, int32_t ny, int32_t nz, uint32_t *cells,
                         uint32_t capacity, uint32_t *counts, int32_t *scratch, void *stream);

int lbdem_lattice_init(const lbdem_lattice *L, int32_t buf, void *stream);

int lbdem_psc_map(const lbdem_lattice *L, lbdem_psc *P, const lbdem_grains *G, void *stream);

/* Clear, ahead of the next lbdem_psc_map, the owner keys that the previous
 * exact map claimed (the cells within each particle's previous mapping reach,
 * from P->prev), and set P->have_prev = 0 so that the next map claims on clear
 * keys without a clearing pass of its own (and does not reuse the previous
 * map).  It reads only P->prev and writes only the keys, so it may run on
 * another stream beside the DEM sub-steps once the last reader of the keys
 * (the step, lbdem_psc_decode) is done; the next map must be ordered after
 * it.  No counterpart in the reference, which rebuilds its fields every step.
 * Not with P->disp_limit > 0 (pipelined stepping checks displacements in the
 * map's own clearing pass): LBDEM_ERR_UNSUPPORTED. */
int lbdem_psc_map_clear(const lbdem_lattice *L, lbdem_psc *P, const lbdem_grains *G, void *stream);

/* One fused pass: [stream of the pending post-collision populations in
 * f[src] (gather=1) | read populations in place (gather=0)] -> moments ->
 * Smagorinsky omega -> equilibrium -> PSC / BGK collision -> body force ->
 * post-collision populations into f[dst]; hydrodynamic force and torque of
 * every particle accumulated into G->force_fluid / G->moment_fluid
 * (zeroed by lbdem_psc_map).  P/G may be NULL for a particle-free lattice.
 * With L->stress set, the stress diagnostics of the gathered state are
 * written too.  Three kernels implement the gathered step and give identical
 * populations: one gathers with per-thread loads; the others (rows of up to
 * 256 cells) have a producer warp copy whole upwind rows into shared memory
 * with the tensor memory accelerator, several rows ahead of the warps that
 * collide them, one cell per thread or -- 16-bit storage, even Nx, an even
 * number of x-blocks -- two x-adjacent cells per thread in f32x2 arithmetic
 * (its force sums group the cells differently: the same forces to FP32
 * rounding).  Defaults: two cells per thread where it applies, else one, for
 * 16-bit storage; per-thread gathers for FP32.  LBDEM_STEP_KERNEL=simt, =rows
 * or =rows2 in the environment selects one form for every storage. */
int lbdem_psc_step_f32(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src,
                       int32_t dst, int32_t gather, void *stream);
int lbdem_psc_step_f16(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src,
                       int32_t dst, int32_t gather, void *stream);
int lbdem_psc_step_bf16(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src,
                        int32_t dst, int32_t gather, void *stream);

/* Pipelined stepping (no counterpart in the reference: a scheduling of the
 * same step).  The fused step of a coupled lattice only needs the particle map
 * in the x-blocks (32 cells of a row) that some particle can reach; all other
 * blocks can be streamed and collided while the DEM sub-steps and the next
 * map still run on another stream.
 *
 * lbdem_psc_near_blocks: mask[(z*Ny + y)*NB + x/32] = 1 for every x-block
 * holding a cell within (mapping reach + margin) of a particle's current
 * centre, or of its periodic image along P->periodic axes (mask: Ny*Nz*NB
 * bytes of scratch); then the list `blocks` (Ny*Nz*NB uint32) holds the
 * counts[0] far blocks (ascending) from its start and the counts[1] near
 * blocks (ascending) packed at its end, each entry z << 20 | y << 8 | x/32.
 * counts: device uint32 array of 2 + 2 * ceil(Ny*Nz*NB / 1024) words (the
 * tail is scratch).  Lattices beyond Nx = 8192, Ny = 4096 or Nz = 4096 get
 * LBDEM_ERR_UNSUPPORTED.
 *
 * lbdem_psc_step_phase: one gathered step (gather = 1) restricted to
 *   phase 1: the far blocks, as pure fluid (no keys read, no force);
 *   phase 2: the near blocks, with the map and force reduction, then the
 *            boundary pass.
 * Phase 1 and phase 2 together equal lbdem_psc_step_* when no particle moved
 * farther than the margin between the lists and the map (checked by
 * lbdem_psc_map when P->disp_limit > 0).  Periodic images (P->wrap) are not
 * supported here (LBDEM_ERR_UNSUPPORTED).  entries: the caller's estimate of
 * the phase's list length (e.g. the length an earlier step's lists had, read
 * back asynchronously), or 0.  With 0 the launch covers every x-block and the
 * CTAs past the device-side length exit at once; with an estimate it covers
 * that many entries and a second, grid-striding launch of one CTA per SM
 * processes any beyond them, so every listed block is stepped either way. */
int lbdem_psc_near_blocks(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, double margin,
                          uint8_t *mask, uint32_t *blocks, uint32_t *counts, void *stream);
int lbdem_psc_step_phase(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src,
                         int32_t dst, int32_t phase, const uint32_t *blocks, const uint32_t *counts,
                         uint32_t entries, void *stream);

/* Stream the post-collision populations of f[src] into f[dst] and write
 * rho/vel of FLUID cells (the reference's stream(), no collision). */
int lbdem_stream_moments(const lbdem_lattice *L, int32_t src, int32_t dst, void *stream);

/* Stress diagnostics (BasicLattice3D.compute_stress, src/lbm3d/lbm_solver3d.py:347-404)
 * of the post-stream populations in f[buf] against the lagged state in aux:
 * out = 7 FP32 planes of Ncells (xx, yy, zz, xy, xz, yz, shear magnitude). */
int lbdem_stress(const lbdem_lattice *L, int32_t buf, float *out, void *stream);

/* Expand the owner keys into the reference's per-cell PSC fields. */
int lbdem_psc_decode(const lbdem_lattice *L, const lbdem_psc *P, int32_t *id, float *volfrac,
                     float *weight, float *velsolid, void *stream);

/* ---------------------------------------------------------------------------
 * Differentiable drag on a frozen particle bed (reverse mode).
 *
 * The reference's solid fraction is a count of 5^3 sub-points, piecewise
 * constant in the particle position; for gradients the map can instead use a
 * smooth fraction of the same effective radius r = R/dx - 1/2:
 *     t = clamp(r - d + 1/2, 0, 1),  eps = t^2 (3 - 2t)      (d: centre distance)
 * owner = the particle of largest eps (ties: lowest id), other cells free.
 * Model differentiated: FP32 storage, Smagorinsky off, constant omega, frozen
 * particles (u_s = 0), uniform body force F on every updated cell.  Loss:
 *     L = e . sum_particles force_fluid   after the step-N kernel
 * (e: 3 doubles, physical units of force_fluid).
 * ------------------------------------------------------------------------- */

/* Smooth map: fills P->key and P->eps (both Ncells), the particle table and
 * zeroes the force accumulators.  scratch: Ncells uint64 (caller-owned). */
int lbdem_psc_map_smooth(const lbdem_lattice *L, lbdem_psc *P, const lbdem_grains *G, uint64_t *scratch,
                         void *stream);

/* Reverse of one lbdem_psc_step_f32 (step n) on the lattice L (P->eps set).
 *  f_prev  populations the forward step n read (blocked, as L->f)
 *  lam_in  dL/d(post-collision populations of step n), blocked FP32 in units
 *          of f (ignored when seed = 1: step n is the last step)
 *  lam_out dL/d(f_prev), blocked FP32, written when gather = 1 (step n
 *          streamed f_prev; gather = 0 for the first step after initialize)
 *  bbar    Ncells FP32, dL/dB of every cell's PSC weight, accumulated (+=)
 *  gbar    3 doubles, dL/dF accumulated (+=), F in lattice units
 *  loss_dir 3 doubles, e of the loss */
int lbdem_psc_step_adjoint_f32(const lbdem_lattice *L, const lbdem_psc *P, const void *f_prev, const float *lam_in,
                               float *lam_out, float *bbar, double *gbar, const double *loss_dir, int32_t gather,
                               int32_t seed, void *stream);

/* Position gradient from dL/dB: pos_bar (n,3 doubles, physical units) +=
 * sum over each particle's owned cells of bbar dB/deps deps/dpos. */
int lbdem_psc_force_adjoint(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, const float *bbar,
                            double *pos_bar, void *stream);

int lbdem_dem_bin(lbdem_dem *D, void *stream);

/* Kernels launched by the calling thread's last lbdem_dem_substeps (1 for the
 * single-launch form, 2 per sub-step for the split form); for launch counts. */
int lbdem_dem_launches_last(void);
/* nsub DEM sub-steps on the stream, in one of these forms (same contact sets
 * and states; only the order of the atomic force sums differs):
 *   n <= 16:  one 128-thread block, block barriers between the phases;
 *   n <= 64:  one 512-thread block (cluster launch), block barriers;
 *   larger, with D->sync (2 words of device memory) and all contact lanes
 *            in one resident wave: one cooperative launch, bounded grid
 *            barriers (LBDEM_ST_WAIT_TIMEOUT if one gives up);
 *   otherwise two launches per sub-step (contacts, integration) in 64-thread
 *            blocks, which also share the GPU with a step on another stream. */
int lbdem_dem_substeps(lbdem_dem *D, int32_t nsub, void *stream);

/* FP64 totals over the updated (non-skipped) cells of population buffer
 * f[buf]: out[0] = sum of rho, out[1..3] = sum of momentum.  Valid in either
 * state of the buffer (post-stream or post-collision: streaming conserves
 * both).  `partials` is caller scratch of LBDEM_SUM_PARTIALS doubles. */
#define LBDEM_SUM_BLOCKS 1184
#define LBDEM_SUM_PARTIALS (4 * LBDEM_SUM_BLOCKS)
int lbdem_global_sums_f64(const lbdem_lattice *L, int32_t buf, double *out, double *partials,
                          void *stream);

/* Same totals as lbdem_global_sums_f64 without any caller scratch and without
 * allocating: for callers that own the lattice buffers but have no device
 * allocator of their own -- a host reaching the library only through this C
 * ABI with buffers lent by another component, or a process whose GPU memory is
 * fully reserved by a framework's caching allocator.  No counterpart in the
 * reference.  The block partials live in a library-owned device array of
 * 4 * 2048 doubles (64 KB, held by every GPU that loads the library until the
 * process exits), which covers lattices of up to 2^26 = 67,108,864 cells
 * (512 x 512 x 256); larger lattices return LBDEM_ERR_ARG before any device
 * work.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture; the
 * address is kept for the life of the process, so a device that the caller
 * resets (cudaDeviceReset) must not be given to this function again.  Every
 * call shares the array: calls that may overlap on the GPU (different streams
 * without ordering) race; each call overwrites every partial it reads, so no
 * clearing is needed between calls. */
int lbdem_global_sums_f64_noalloc(const lbdem_lattice *L, int32_t buf, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* LBDEM_H */
