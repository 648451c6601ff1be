// PSC particle -> lattice mapping (grains2lattice, psclattice3d.py:84-182).
//
// The reference loops over every cell and, inside, over every grain
// (O(cells x grains)).  Here each particle scatters over the cells its sphere
// can touch and claims them with atomicMax on a 32-bit owner key that encodes
// the reference's winner rule, so the result is identical for any order.
//
// Decisions are the reference's FP64 comparisons (operation order kept, and
// this file is compiled with -fmad=false so nothing is contracted); an FP32
// pre-classification with a proven margin decides the clear cases, so the 5^3
// sub-sample counts match the reference bit for bit at FP32 speed.
#include <math.h>
#include <string.h>

#include "common.cuh"

namespace lbdem {

struct MapArgs {
    int n, nx, ny, nz;
    int keys_only;           // the clearing pass zeroes the previous map's keys only (no table, no force reset)
    int table_in_scatter;    // no clearing pass runs: the scatter writes the table and resets the forces
    double dx, dt, xmin, ymin, zmin;
    const double *pos, *radius, *vel, *omega;
    const uint32_t *links;
    uint32_t *key;
    float4 *table;
    double *prev;
    int have_prev;
    uint32_t *moved;         // map reuse: set when a particle moved since the previous map (device word), or NULL
    uint32_t *moved_next;    // the next call's word, cleared here
    double *ff, *mf;
    int32_t *status;
    int wrap[3];             // periodic images along each axis (0: the reference's unwrapped mapping)
    double period[3];        // image shift per axis, lattice units
    int periodic[3];         // DEM periodic axes (pipelined stepping: near-block images, displacement check)
    double disp_limit;       // largest allowed centre displacement between two maps (0: no check)
};

constexpr double HALF_DIAG = 0.8660254037844386;  // 0.5 * sqrt(3.0), psclattice3d.py:111
// Largest distance of a 5^3 sub-point (offsets -0.4 .. 0.4 per axis,
// psclattice3d.py:121-128) from its cell centre, 0.4 sqrt(3), rounded up.
constexpr double SUB_REACH = 0.6928204;

__device__ __forceinline__ void particle_lattice(const MapArgs &a, int g, double &xc, double &yc, double &zc,
                                                 double &r) {
    // psclattice3d.py:102-105
    xc = (a.pos[3 * g + 0] - a.xmin + 0.5 * a.dx) / a.dx;
    yc = (a.pos[3 * g + 1] - a.ymin + 0.5 * a.dx) / a.dx;
    zc = (a.pos[3 * g + 2] - a.zmin + 0.5 * a.dx) / a.dx;
    r = (a.radius[g] - 0.5 * a.dx) / a.dx;
}

// Image shifts of a sphere centre c with reach `reach` along `axis`: 0, plus
// one periodic image when the sphere crosses a periodic face (wrap mode).
__device__ __forceinline__ int image_shifts(const MapArgs &a, int axis, double c, double reach, int n, double sh[2]) {
    sh[0] = 0.0;
    sh[1] = 0.0;
    if (!a.wrap[axis]) return 1;
    if (c - reach < 0.0) { sh[1] = a.period[axis]; return 2; }
    if (c + reach > (double)(n - 1)) { sh[1] = -a.period[axis]; return 2; }
    return 1;
}

// Particle g's row of the FP32 table the step reads, and its force
// accumulators reset (one thread).
__device__ __forceinline__ void particle_table(const MapArgs &a, int g) {
    for (int t = 0; t < 3; ++t) a.ff[3 * g + t] = a.mf[3 * g + t] = 0.0;
    double xc, yc, zc, r;
    particle_lattice(a, g, xc, yc, zc, r);
    const double fx = floor(xc), fy = floor(yc), fz = floor(zc);
    // cell-centre offsets are formed as (x - floor) - frac in FP32 (exact
    // integer part), keeping the lever arm accurate to ~1e-7 lattice units
    a.table[4 * g + 0] = make_float4((float)fx, (float)fy, (float)fz, 0.f);
    a.table[4 * g + 1] = make_float4((float)(xc - fx), (float)(yc - fy), (float)(zc - fz), 0.f);
    const double s = a.dt / a.dx;
    a.table[4 * g + 2] = make_float4((float)(a.vel[3 * g] * s), (float)(a.vel[3 * g + 1] * s),
                                     (float)(a.vel[3 * g + 2] * s), 0.f);
    a.table[4 * g + 3] = make_float4((float)(a.omega[3 * g] * a.dt), (float)(a.omega[3 * g + 1] * a.dt),
                                     (float)(a.omega[3 * g + 2] * a.dt), 0.f);
}

// Clear the cells claimed by the previous map (conservative shell), zero the
// force accumulators, and write the FP32 particle table used by the step.
// With map reuse (a.moved set) a particle clears its old shell only if its
// lattice centre or mapping radius changed, and flags the change; the scatter
// then re-claims every particle's cells if any particle moved and is skipped
// otherwise.  That is exact: an unmoved particle's old keys are still its own
// valid claims, and atomicMax against them gives the same winners.
// WRAP: the map has periodic images (a.wrap); without them the image loops
// compile to the single original sphere.
template <bool WRAP>
__global__ void __launch_bounds__(128) k_map_clear(const MapArgs a) {
    const int g = blockIdx.x;
    bool clear = a.have_prev != 0;
    if (a.disp_limit > 0.0 && a.have_prev && threadIdx.x == 0) {
        // pipelined stepping: the near-block mask assumed at most disp_limit
        double xc, yc, zc, r;
        particle_lattice(a, g, xc, yc, zc, r);
        double d[3] = {xc - a.prev[4 * g], yc - a.prev[4 * g + 1], zc - a.prev[4 * g + 2]};
        for (int t = 0; t < 3; ++t)
            if (a.periodic[t] && a.period[t] > 0.0) d[t] -= a.period[t] * rint(d[t] / a.period[t]);
        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > a.disp_limit * a.disp_limit)
            atomicOr(a.status, (int)LBDEM_ST_PIPELINE_MARGIN);
    }
    if (a.moved != nullptr) {
        if (g == 0 && threadIdx.x == 0) *a.moved_next = 0u;
        double xc, yc, zc, r;
        particle_lattice(a, g, xc, yc, zc, r);
        const double *p = a.prev + 4 * (size_t)g;
        const bool moved = !(xc == p[0] && yc == p[1] && zc == p[2] && r == p[3]);
        if (moved && threadIdx.x == 0) *a.moved = 1u;
        clear = clear && moved;
    }
    const double lim = a.prev[4 * g + 3] + HALF_DIAG + 1e-6;
    double shx[2], shy[2], shz[2];
    shx[0] = shy[0] = shz[0] = 0.0;
    int nix = clear ? 1 : 0, niy = 1, niz = 1;
    if constexpr (WRAP) {
        if (clear) {
            nix = image_shifts(a, 0, a.prev[4 * g], lim, a.nx, shx);
            niy = image_shifts(a, 1, a.prev[4 * g + 1], lim, a.ny, shy);
            niz = image_shifts(a, 2, a.prev[4 * g + 2], lim, a.nz, shz);
        }
    }
    for (int im = 0; im < nix * niy * niz; ++im) {
        const double pxc = a.prev[4 * g] + shx[im % nix], pyc = a.prev[4 * g + 1] + shy[(im / nix) % niy];
        const double pzc = a.prev[4 * g + 2] + shz[im / (nix * niy)];
        if (lim > 0.0) {
            const int x0 = max(0, (int)floor(pxc - lim)), x1 = min(a.nx - 1, (int)ceil(pxc + lim));
            const int y0 = max(0, (int)floor(pyc - lim)), y1 = min(a.ny - 1, (int)ceil(pyc + lim));
            const int z0 = max(0, (int)floor(pzc - lim)), z1 = min(a.nz - 1, (int)ceil(pzc + lim));
            const int ex = x1 - x0 + 1, ey = y1 - y0 + 1, ez = z1 - z0 + 1;
            if (ex > 0 && ey > 0 && ez > 0) {
                const unsigned exy = (unsigned)ex * (unsigned)ey, tot = exy * (unsigned)ez;
                const float lim2 = (float)(lim * lim) + 1e-3f;
                for (unsigned t = threadIdx.x; t < tot; t += blockDim.x) {
                    const unsigned kz = t / exy, rem = t - kz * exy, jy = rem / (unsigned)ex;
                    const int i = x0 + (int)(rem - jy * (unsigned)ex), j = y0 + (int)jy, k = z0 + (int)kz;
                    const float ddx = (float)(pxc - i), ddy = (float)(pyc - j), ddz = (float)(pzc - k);
                    if (ddx * ddx + ddy * ddy + ddz * ddz < lim2)
                        a.key[((size_t)k * a.ny + j) * a.nx + i] = 0u;
                }
            }
        }
    }
    if (threadIdx.x == 0 && !a.keys_only) particle_table(a, g);
}

// Exact FP64 sub-cell test, in the reference's operation order
// (psclattice3d.py:125-128): sqrt(dx^2 + dy^2 + dz^2) < r.
__device__ __forceinline__ bool subcell_inside_exact(double xc, double yc, double zc, int i, int j, int k, int ii,
                                                     int jj, int kk, double r) {
    const double ox = xc - (((double)i - 0.4) + 0.2 * ii);
    const double oy = yc - (((double)j - 0.4) + 0.2 * jj);
    const double oz = zc - (((double)k - 0.4) + 0.2 * kk);
    return sqrt((ox * ox + oy * oy) + oz * oz) < r;
}

// One block per particle -- or, with few particles, gridDim.y blocks sharing
// its bounding box in contiguous ranges of cells, so that a lone sphere does
// not map on one SM -- two phases per chunk of the box:
//  1. each thread classifies one cell -- outside / fully covered / partial
//     (psclattice3d.py:108-113).  FP32 with a safety margin decides the clear
//     cases; the exact FP64 comparisons run only for cells near a threshold.
//     Full covers are claimed at once, and so are partial cells whose 125
//     sub-points all lie inside the sphere; partial cells with sub-points on
//     both sides of the surface go to a shared list (those with none inside
//     are dropped).
//  2. one thread per partial cell counts its 5^3 sub-points
//     (psclattice3d.py:121-131) from the squared per-axis offsets; the few
//     cells with a sub-point near the surface are recounted one warp per
//     cell (25 lanes x 5, __reduce_add_sync).  A sub-point whose
//     FP32 squared distance lies within 1e-4 (1 + r^2) of r^2 is re-tested
//     with the reference's exact FP64 expression (|s32 - s64| < 2e-5 (1 + r^2)
//     for these offsets), so counts are bit-exact.
constexpr int MAP_CHUNK = 2048;         // box cells classified per round (shared-memory lists)
constexpr int MAP_THREADS = 256;
constexpr int MAP_MIN_BLOCKS = 5;       // per SM (46 registers, 40 KB of shared memory each)
constexpr int MAP_SPLIT_BELOW = 592;   // 148 SMs x 4 blocks

// Five 256-thread blocks per SM (46 registers, 40 KB of shared memory each);
// the image form keeps four (it would spill at five).
template <bool WRAP>
__global__ void __launch_bounds__(MAP_THREADS, WRAP ? 4 : MAP_MIN_BLOCKS) k_map_scatter(const MapArgs a) {
    __shared__ float4 s_off[MAP_CHUNK];   // (xc - i, yc - j, zc - k) in FP32; w = global cell index
    __shared__ int s_amb[MAP_CHUNK];      // partial cells needing the exact recount (index into s_off)
    __shared__ int s_n, s_na;
    const int g = blockIdx.x;
    if (a.moved != nullptr && *a.moved == 0u) return;   // reuse: nothing moved, keys unchanged (clear pass ran)
    double xc0, yc0, zc0, r;
    particle_lattice(a, g, xc0, yc0, zc0, r);
    if (threadIdx.x == 0 && blockIdx.y == 0) {
        a.prev[4 * g] = xc0; a.prev[4 * g + 1] = yc0; a.prev[4 * g + 2] = zc0; a.prev[4 * g + 3] = r;
    }
    const double t_out = r + HALF_DIAG, t_in = r - HALF_DIAG;
    // the sphere, and in wrap mode its periodic images (block-uniform loop;
    // none for a radius that reaches no cell centre)
    double shx[2], shy[2], shz[2];
    shx[0] = shy[0] = shz[0] = 0.0;
    int nix = 1, niy = 1, niz = 1;
    if constexpr (WRAP) {
        nix = image_shifts(a, 0, xc0, t_out, a.nx, shx);
        niy = image_shifts(a, 1, yc0, t_out, a.ny, shy);
        niz = image_shifts(a, 2, zc0, t_out, a.nz, shz);
    }
    const int nimg = t_out > 0.0 ? nix * niy * niz : 0;
    for (int im = 0; im < nimg; ++im) {
        const double xc = xc0 + shx[im % nix], yc = yc0 + shy[(im / nix) % niy], zc = zc0 + shz[im / (nix * niy)];
        const int x0 = max(0, (int)floor(xc - t_out)), x1 = min(a.nx - 1, (int)ceil(xc + t_out));
        const int y0 = max(0, (int)floor(yc - t_out)), y1 = min(a.ny - 1, (int)ceil(yc + t_out));
        const int z0 = max(0, (int)floor(zc - t_out)), z1 = min(a.nz - 1, (int)ceil(zc + t_out));
        const int ex = x1 - x0 + 1, ey = y1 - y0 + 1, ez = z1 - z0 + 1;
        if (ex <= 0 || ey <= 0 || ez <= 0) continue;
        const uint32_t gbits = 0xFFFFFFu - (uint32_t)g;
        const float out2 = (float)(t_out * t_out), marg_o = (float)(1e-4 * (1.0 + t_out * t_out));
        const float in2 = t_in > 0.0 ? (float)(t_in * t_in) : -1.f, marg_i = (float)(1e-4 * (1.0 + t_in * t_in));
        const double rr = r > 0.0 ? r * r : 0.0;
        const float band = (float)(1e-4 * (1.0 + rr));
        // sub-points lie within SUB_REACH of their cell centre: a partial cell
        // whose centre is within r - SUB_REACH counts all 125, one beyond
        // r + SUB_REACH none (FP32 with the same kind of margin)
        const double t_all = r - SUB_REACH, t_none = r + SUB_REACH;
        const float all2 = t_all > 0.0 ? (float)(t_all * t_all) : -1.f, marg_a = (float)(1e-4 * (1.0 + t_all * t_all));
        const float none2 = (float)(t_none * t_none), marg_n = (float)(1e-4 * (1.0 + t_none * t_none));
        const float lo = (float)rr - band, hi = (float)rr + band;
        const unsigned tot = (unsigned)ex * (unsigned)ey * (unsigned)ez;
        // this block's range of the box's cells
        const unsigned per = (tot + gridDim.y - 1) / gridDim.y;
        const unsigned beg = min(tot, blockIdx.y * per), end = min(tot, beg + per);
        // this thread's first cell, then advance by blockDim cells with carries
        // (every chunk but the last is a whole number of blockDim steps)
        const unsigned bd = blockDim.x;
        const int adx = (int)(bd % (unsigned)ex), ady = (int)((bd / (unsigned)ex) % (unsigned)ey);
        const int adz = (int)(bd / ((unsigned)ex * (unsigned)ey));
        const unsigned t0 = beg + threadIdx.x;
        int ix = (int)(t0 % (unsigned)ex), jy = (int)((t0 / (unsigned)ex) % (unsigned)ey);
        int kz = (int)(t0 / ((unsigned)ex * (unsigned)ey));
        for (unsigned base = beg; base < end; base += MAP_CHUNK) {
            if (threadIdx.x == 0) s_n = s_na = 0;
            __syncthreads();
            const unsigned lim = min(end, base + MAP_CHUNK);
            for (unsigned t = base + threadIdx.x; t < lim; t += bd) {
                const int i = x0 + ix, j = y0 + jy, k = z0 + kz;
                ix += adx; jy += ady; kz += adz;
                if (ix >= ex) { ix -= ex; ++jy; }
                if (jy >= ey) { jy -= ey; ++kz; }
                const float fx = (float)(xc - (double)i), fy = (float)(yc - (double)j), fz = (float)(zc - (double)k);
                const float d2 = (fx * fx + fy * fy) + fz * fz;
                if (d2 > out2 + marg_o) continue;                 // certainly dist >= t_out
                const unsigned c = ((unsigned)k * (unsigned)a.ny + (unsigned)j) * (unsigned)a.nx + (unsigned)i;
                if (a.links[c] & LINK_MAP_SKIP) continue;
                int full;
                if (d2 < in2 - marg_i) {
                    full = 1;                                     // certainly dist <= t_in
                } else if (d2 < out2 - marg_o && d2 > in2 + marg_i) {
                    full = 0;                                     // certainly partial
                } else {
                    const double ddx = xc - i, ddy = yc - j, ddz = zc - k;
                    const double dist = sqrt((ddx * ddx + ddy * ddy) + ddz * ddz);
                    if (dist >= t_out) continue;
                    full = dist <= t_in;
                }
                if (full) {
                    atomicMax(a.key + c, KEY_FULL | gbits);
                } else if (r > 0.0 && d2 < all2 - marg_a) {
                    atomicMax(a.key + c, (125u << 24) | gbits);   // every sub-point inside
                } else if (r > 0.0 && !(d2 > none2 + marg_n)) {
                    const int slot = atomicAdd(&s_n, 1);
                    s_off[slot] = make_float4(fx, fy, fz, __uint_as_float(c));
                }
            }
            __syncthreads();
            const int n = s_n;
            // 2a. one thread per partial cell: 25 columns x 5 sub-points from the
            // squared per-axis offsets (-fmad=false).  Per column (x, y) the five
            // z terms are compared with lo - s_xy and hi - s_xy (their rounding is
            // far inside the band), so a point counts when its squared distance is
            // certainly below r^2 and the cell is ambiguous when a point lies
            // between the two thresholds (the two counts differ); ambiguous cells
            // go to a second list for an exact warp recount.
            for (int e = threadIdx.x; e < n; e += bd) {
                const float4 o = s_off[e];
                float ox2[5], oy2[5], oz2[5];
    #pragma unroll
                for (int m = 0; m < 5; ++m) {
                    const float sh = 0.4f - 0.2f * (float)m;
                    const float ox = o.x + sh, oy = o.y + sh, oz = o.z + sh;
                    ox2[m] = ox * ox;
                    oy2[m] = oy * oy;
                    oz2[m] = oz * oz;
                }
                int cnt = 0, cnt_hi = 0;
    #pragma unroll
                for (int ia = 0; ia < 5; ++ia)
    #pragma unroll
                    for (int ja = 0; ja < 5; ++ja) {
                        const float sxy = ox2[ia] + oy2[ja];
                        const float tl = lo - sxy, th = hi - sxy;
    #pragma unroll
                        for (int kk = 0; kk < 5; ++kk) {
                            cnt += oz2[kk] < tl;
                            cnt_hi += oz2[kk] <= th;
                        }
                    }
                if (cnt_hi != cnt) {
                    s_amb[atomicAdd(&s_na, 1)] = e;
                } else if (cnt > 0) {   // eps = 0 never beats the empty cell (strict >)
                    atomicMax(a.key + __float_as_uint(o.w), ((uint32_t)cnt << 24) | gbits);
                }
            }
            __syncthreads();
            // 2b. cells with near-surface sub-points: one warp per cell, lane
            // (ii, jj) < 25 tests its column of five; points inside the band are
            // re-tested with the reference's exact FP64 expression
            const int na = s_na;
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
            const int ii = lane / 5, jj = lane % 5;
            const float oxl = 0.4f - 0.2f * (float)ii, oyl = 0.4f - 0.2f * (float)jj;
            for (int e2 = warp; e2 < na; e2 += nwarp) {
                const float4 o = s_off[s_amb[e2]];
                const unsigned c = __float_as_uint(o.w);
                int cnt = 0;
                if (lane < 25) {
                    const int i = (int)(c % (unsigned)a.nx), j = (int)((c / (unsigned)a.nx) % (unsigned)a.ny);
                    const int k = (int)(c / ((unsigned)a.nx * (unsigned)a.ny));
                    const float ox = o.x + oxl, oy = o.y + oyl;
                    const float sxy = ox * ox + oy * oy;
                    for (int kk = 0; kk < 5; ++kk) {
                        const float oz = o.z + (0.4f - 0.2f * (float)kk);
                        const float sd = sxy + oz * oz;
                        if (sd < lo) ++cnt;
                        else if (sd <= hi) cnt += subcell_inside_exact(xc, yc, zc, i, j, k, ii, jj, kk, r);
                    }
                }
                cnt = __reduce_add_sync(0xffffffffu, cnt);
                if (lane == 0 && cnt > 0) atomicMax(a.key + c, ((uint32_t)cnt << 24) | gbits);
            }
            __syncthreads();
        }
    }
    // without a clearing pass the table row and the force reset are written
    // here, last, where the registers of the claims are free again
    if (a.table_in_scatter && threadIdx.x == 0 && blockIdx.y == 0) particle_table(a, g);
}


// Near-block mask for pipelined stepping: every x-block (32 cells of a row)
// holding a cell within the particle's mapping reach plus `margin` of its
// lattice centre (per row: the chord of that ball), and
// of the centre's periodic image when the sphere's reach crosses a periodic
// face (a particle that crosses the face reappears there).  One block per
// particle; the stores are idempotent.
__global__ void __launch_bounds__(128) k_near_blocks(const MapArgs a, double margin, uint8_t *near) {
    const int g = blockIdx.x;
    double xc0, yc0, zc0, r;
    particle_lattice(a, g, xc0, yc0, zc0, r);
    const double reach = r + HALF_DIAG + margin;
    if (!(reach > 0.0)) return;
    const int nb = (a.nx + 31) / 32;
    const int n3[3] = {a.nx, a.ny, a.nz};
    const double c3[3] = {xc0, yc0, zc0};
    double sh[3][2];
    int ni[3];
    for (int t = 0; t < 3; ++t) {
        sh[t][0] = sh[t][1] = 0.0;
        ni[t] = 1;
        if (a.periodic[t] && a.period[t] > 0.0) {
            if (c3[t] - reach < 0.0) { sh[t][1] = a.period[t]; ni[t] = 2; }
            else if (c3[t] + reach > (double)(n3[t] - 1)) { sh[t][1] = -a.period[t]; ni[t] = 2; }
        }
    }
    for (int im = 0; im < ni[0] * ni[1] * ni[2]; ++im) {
        const double xc = xc0 + sh[0][im % ni[0]], yc = yc0 + sh[1][(im / ni[0]) % ni[1]];
        const double zc = zc0 + sh[2][im / (ni[0] * ni[1])];
        const int x0 = max(0, (int)floor(xc - reach)), x1 = min(a.nx - 1, (int)ceil(xc + reach));
        const int y0 = max(0, (int)floor(yc - reach)), y1 = min(a.ny - 1, (int)ceil(yc + reach));
        const int z0 = max(0, (int)floor(zc - reach)), z1 = min(a.nz - 1, (int)ceil(zc + reach));
        if (x1 < x0 || y1 < y0 || z1 < z0) continue;
        // one thread per (y, z) row of the box: the row's chord of the reach ball
        const int ey = y1 - y0 + 1;
        const unsigned tot = (unsigned)ey * (unsigned)(z1 - z0 + 1);
        for (unsigned t = threadIdx.x; t < tot; t += blockDim.x) {
            const int y = y0 + (int)(t % (unsigned)ey), z = z0 + (int)(t / (unsigned)ey);
            const double dy = (double)y - yc, dz = (double)z - zc;
            const double w2 = reach * reach - dy * dy - dz * dz;
            if (w2 < 0.0) continue;
            const double w = sqrt(w2);
            const int xa = max(0, (int)floor(xc - w)), xb = min(a.nx - 1, (int)ceil(xc + w));
            if (xb < xa) continue;
            uint8_t *rowp = near + ((size_t)z * a.ny + y) * nb;
            for (int b = xa >> 5; b <= (xb >> 5); ++b) rowp[b] = 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Smooth solid fraction (differentiable stand-in for the 5^3 count): the same
// effective radius r = R/dx - 1/2 (psclattice3d.py:105), a C1 ramp of one
// lattice spacing across the surface,
//     t = clamp(r - d + 1/2, 0, 1),  eps = t^2 (3 - 2t),
// owner = largest eps (ties: lowest id) through atomicMax on
// (float bits of eps) << 32 | (0xFFFFFFFF - id); no periodic images, and
// map-skipped cells stay free, as in the reference mapping.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_map_smooth(const MapArgs a, unsigned long long *scratch) {
    const int g = blockIdx.x;
    double xc, yc, zc, r;
    particle_lattice(a, g, xc, yc, zc, r);
    const double lim = r + 0.5;
    if (!(lim > 0.0)) return;
    const int x0 = max(0, (int)floor(xc - lim)), x1 = min(a.nx - 1, (int)ceil(xc + lim));
    const int y0 = max(0, (int)floor(yc - lim)), y1 = min(a.ny - 1, (int)ceil(yc + lim));
    const int z0 = max(0, (int)floor(zc - lim)), z1 = min(a.nz - 1, (int)ceil(zc + lim));
    const int ex = x1 - x0 + 1, ey = y1 - y0 + 1, ez = z1 - z0 + 1;
    if (ex <= 0 || ey <= 0 || ez <= 0) return;
    const unsigned exy = (unsigned)ex * (unsigned)ey, tot = exy * (unsigned)ez;
    for (unsigned t = threadIdx.x; t < tot; t += blockDim.x) {
        const unsigned kz = t / exy, rem = t - kz * exy, jy = rem / (unsigned)ex;
        const int i = x0 + (int)(rem - jy * (unsigned)ex), j = y0 + (int)jy, k = z0 + (int)kz;
        const size_t c = ((size_t)k * a.ny + j) * a.nx + i;
        if (a.links[c] & LINK_MAP_SKIP) continue;
        const double dxv = xc - i, dyv = yc - j, dzv = zc - k;
        const double d = sqrt(dxv * dxv + dyv * dyv + dzv * dzv);
        double tt = r - d + 0.5;
        if (tt <= 0.0) continue;
        if (tt > 1.0) tt = 1.0;
        const float e = (float)(tt * tt * (3.0 - 2.0 * tt));
        if (!(e > 0.f)) continue;
        const unsigned long long kk =
            ((unsigned long long)__float_as_uint(e) << 32) | (unsigned long long)(0xFFFFFFFFu - (unsigned)g);
        atomicMax(scratch + c, kk);
    }
}

__global__ void k_map_smooth_decode(size_t nc, const unsigned long long *scratch, uint32_t *key, float *eps) {
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const unsigned long long kk = scratch[c];
    if (!kk) {
        key[c] = 0u;
        eps[c] = 0.f;
        return;
    }
    const unsigned g = 0xFFFFFFFFu - (unsigned)(kk & 0xFFFFFFFFull);
    const float e = __uint_as_float((unsigned)(kk >> 32));
    key[c] = (e >= 1.f ? KEY_FULL : 0u) | (0xFFFFFFu - g);
    eps[c] = e;
}

}  // namespace lbdem

extern "C" int lbdem_psc_map_smooth(const lbdem_lattice *L, lbdem_psc *P, const lbdem_grains *G,
                                    uint64_t *scratch, void *stream) {
    using namespace lbdem;
    if (!L || !P || !G || !P->key || !P->eps || !P->table || !L->links || !scratch) {
        set_error("psc_map_smooth: bad arguments (key, eps, table, links and scratch are required)");
        return LBDEM_ERR_ARG;
    }
    if (P->wrap[0] || P->wrap[1] || P->wrap[2]) {
        set_error("psc_map_smooth: the smooth solid fraction has no periodic images");
        return LBDEM_ERR_UNSUPPORTED;
    }
    if (G->n > 0xFFFFFF) {
        set_error("psc_map_smooth: %d particles exceed the 2^24-1 owner-key range", G->n);
        return LBDEM_ERR_ARG;
    }
    if (!(P->dx > 0.0) || !(P->dt > 0.0)) {
        set_error("psc_map_smooth: dx and dt must be positive");
        return LBDEM_ERR_ARG;
    }
    const size_t nc = (size_t)L->nx * L->ny * L->nz;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(scratch, 0, nc * sizeof(uint64_t), st) != cudaSuccess) return check_launch("psc_map_smooth");
    if (G->n > 0) {
        MapArgs a;
    a.keys_only = 0;
    a.table_in_scatter = 0;
        a.n = G->n; a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
        a.dx = P->dx; a.dt = P->dt; a.xmin = P->xmin; a.ymin = P->ymin; a.zmin = P->zmin;
        a.pos = G->pos; a.radius = G->radius; a.vel = G->vel; a.omega = G->omega;
        a.links = L->links;
        a.key = P->key;
        a.table = (float4 *)P->table;
        a.prev = P->prev;
        a.have_prev = 0;
        a.ff = G->force_fluid; a.mf = G->moment_fluid;
        a.status = L->status;
        a.moved = a.moved_next = nullptr;
        a.disp_limit = 0.0;
        a.periodic[0] = a.periodic[1] = a.periodic[2] = 0;
        a.wrap[0] = a.wrap[1] = a.wrap[2] = 0;   // the smooth map has no periodic images
        a.period[0] = a.period[1] = a.period[2] = 0.0;
        k_map_clear<false><<<G->n, 128, 0, st>>>(a);
        k_map_smooth<<<G->n, 256, 0, st>>>(a, reinterpret_cast<unsigned long long *>(scratch));
    }
    k_map_smooth_decode<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(
        nc, reinterpret_cast<const unsigned long long *>(scratch), P->key, P->eps);
    P->have_prev = 0;   // every key is rewritten; a later exact map must not rely on a clear shell
    return check_launch("psc_map_smooth");
}

using namespace lbdem;

extern "C" int lbdem_psc_map(const lbdem_lattice *L, lbdem_psc *P, const lbdem_grains *G, void *stream) {
    if (!L || !P || !G || !P->key || !P->table || !P->prev || !L->links) {
        set_error("psc_map: bad arguments");
        return LBDEM_ERR_ARG;
    }
    if (G->n <= 0) return LBDEM_OK;
    if (G->n > 0xFFFFFF) {
        set_error("psc_map: %d particles exceed the 2^24-1 owner-key range", G->n);
        return LBDEM_ERR_ARG;
    }
    if (!(P->dx > 0.0) || !(P->dt > 0.0)) {
        set_error("psc_map: dx and dt must be positive");
        return LBDEM_ERR_ARG;
    }
    MapArgs a;
    a.keys_only = 0;
    a.table_in_scatter = 0;
    a.n = G->n; a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.dx = P->dx; a.dt = P->dt; a.xmin = P->xmin; a.ymin = P->ymin; a.zmin = P->zmin;
    a.pos = G->pos; a.radius = G->radius; a.vel = G->vel; a.omega = G->omega;
    a.links = L->links;
    a.key = P->key;
    a.table = (float4 *)P->table;
    a.prev = P->prev;
    a.have_prev = P->have_prev;
    a.ff = G->force_fluid; a.mf = G->moment_fluid;
    a.status = L->status;
    a.moved = a.moved_next = nullptr;
    for (int t = 0; t < 3; ++t) {
        a.wrap[t] = P->wrap[t] != 0;
        a.period[t] = P->period[t];
        a.periodic[t] = P->periodic[t] != 0;
        if (a.wrap[t] && !(P->period[t] >= 1.0)) {
            set_error("psc_map: periodic images need a positive period (axis %d)", t);
            return LBDEM_ERR_ARG;
        }
    }
    a.disp_limit = P->disp_limit;
    cudaStream_t st = (cudaStream_t)stream;
    if (P->map_moved && P->map_reuse && P->have_prev) {
        // the previous exact map's centres are in prev: skip the remap when none changed
        const int par = P->map_parity & 1;
        a.moved = P->map_moved + par;
        a.moved_next = P->map_moved + (1 - par);
        P->map_parity = 1 - par;
    }
    // fewer particles than about four blocks per SM: split each box over several blocks
    const dim3 sgrid((unsigned)G->n, (unsigned)(G->n >= MAP_SPLIT_BELOW ? 1 : min(16, (MAP_SPLIT_BELOW + G->n - 1) / G->n)));
    // with nothing to clear or check (keys cleared ahead by lbdem_psc_map_clear,
    // or the first map) the scatter writes the table itself: one launch
    const bool clear_pass = a.have_prev || a.moved != nullptr || a.disp_limit > 0.0;
    a.table_in_scatter = !clear_pass;
    if (a.wrap[0] || a.wrap[1] || a.wrap[2]) {
        if (clear_pass) k_map_clear<true><<<G->n, 128, 0, st>>>(a);
        k_map_scatter<true><<<sgrid, MAP_THREADS, 0, st>>>(a);
    } else {
        if (clear_pass) k_map_clear<false><<<G->n, 128, 0, st>>>(a);
        k_map_scatter<false><<<sgrid, MAP_THREADS, 0, st>>>(a);
    }
    P->have_prev = 1;
    return check_launch("psc_map");
}

extern "C" int lbdem_psc_map_clear(const lbdem_lattice *L, lbdem_psc *P, const lbdem_grains *G, void *stream) {
    if (!L || !P || !G || !P->key || !P->prev) {
        set_error("psc_map_clear: bad arguments");
        return LBDEM_ERR_ARG;
    }
    if (P->disp_limit > 0.0) {
        set_error("psc_map_clear: pipelined stepping (disp_limit > 0) checks displacements in the map's own clear");
        return LBDEM_ERR_UNSUPPORTED;
    }
    if (G->n <= 0 || !P->have_prev) return LBDEM_OK;
    MapArgs a;
    memset(&a, 0, sizeof(a));
    a.keys_only = 1;
    a.n = G->n; a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.key = P->key;
    a.prev = P->prev;
    a.have_prev = 1;
    a.status = L->status;
    for (int t = 0; t < 3; ++t) {
        a.wrap[t] = P->wrap[t] != 0;
        a.period[t] = P->period[t];
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (a.wrap[0] || a.wrap[1] || a.wrap[2]) k_map_clear<true><<<G->n, 128, 0, st>>>(a);
    else k_map_clear<false><<<G->n, 128, 0, st>>>(a);
    P->have_prev = 0;
    return check_launch("psc_map_clear");
}

// Ordered block lists (ascending ids, so each phase walks memory in order):
// far blocks from the front of `blocks`, near blocks packed at its end.
// Chunks of 1024 block ids: per-chunk counts, one scan over the chunks, then
// each chunk writes its ids at its offsets (warp ballots + a CTA prefix).
constexpr int LIST_CHUNK = 1024;

__global__ void __launch_bounds__(LIST_CHUNK) k_list_count(const uint8_t *mask, uint32_t nblocks, uint32_t *chunk_n) {
    const uint32_t id = blockIdx.x * LIST_CHUNK + threadIdx.x;
    const int nearb = id < nblocks && mask[id] != 0;
    const int n_near = __syncthreads_count(nearb);
    if (threadIdx.x == 0) {
        const uint32_t valid = min((uint32_t)LIST_CHUNK, nblocks - blockIdx.x * LIST_CHUNK);
        chunk_n[2 * blockIdx.x] = valid - (uint32_t)n_near;
        chunk_n[2 * blockIdx.x + 1] = (uint32_t)n_near;
    }
}

// exclusive scan of the (far, near) chunk counts in place; totals to counts[0..1]
__global__ void __launch_bounds__(1024) k_list_scan(uint32_t *chunk_n, uint32_t nchunks, uint32_t *counts) {
    __shared__ uint32_t sf[1024], sn[1024];
    const int t = threadIdx.x;
    uint32_t cf = 0, cn = 0;
    for (uint32_t base = 0; base < nchunks; base += 1024) {
        const uint32_t i = base + t;
        const uint32_t vf = i < nchunks ? chunk_n[2 * i] : 0u, vn = i < nchunks ? chunk_n[2 * i + 1] : 0u;
        sf[t] = vf;
        sn[t] = vn;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const uint32_t af = t >= o ? sf[t - o] : 0u, an = t >= o ? sn[t - o] : 0u;
            __syncthreads();
            sf[t] += af;
            sn[t] += an;
            __syncthreads();
        }
        if (i < nchunks) {
            chunk_n[2 * i] = cf + sf[t] - vf;
            chunk_n[2 * i + 1] = cn + sn[t] - vn;
        }
        const uint32_t tf = sf[1023], tn = sn[1023];
        __syncthreads();
        cf += tf;
        cn += tn;
    }
    if (t == 0) {
        counts[0] = cf;
        counts[1] = cn;
    }
}

// list entry: z (bits 20-31) | y (bits 8-19) | x-block (bits 0-7), so the step decodes it with shifts
__global__ void __launch_bounds__(LIST_CHUNK) k_list_fill(const uint8_t *mask, uint32_t nblocks, uint32_t nb, uint32_t ny,
                                                          const uint32_t *chunk_n, const uint32_t *counts,
                                                          uint32_t *blocks) {
    __shared__ uint32_t wf[LIST_CHUNK / 32], wn[LIST_CHUNK / 32];
    const uint32_t id = blockIdx.x * LIST_CHUNK + threadIdx.x;
    const bool in = id < nblocks;
    const bool nearb = in && mask[id] != 0, farb = in && !nearb;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, below = (1u << lane) - 1u;
    const unsigned mf = __ballot_sync(0xffffffffu, farb), mn = __ballot_sync(0xffffffffu, nearb);
    if (lane == 0) {
        wf[warp] = (uint32_t)__popc(mf);
        wn[warp] = (uint32_t)__popc(mn);
    }
    __syncthreads();
    uint32_t pf = 0, pn = 0;
    for (unsigned w = 0; w < warp; ++w) {
        pf += wf[w];
        pn += wn[w];
    }
    const uint32_t row = id / nb, code = ((row / ny) << 20) | ((row % ny) << 8) | (id - row * nb);
    if (farb) blocks[chunk_n[2 * blockIdx.x] + pf + __popc(mf & below)] = code;
    if (nearb) blocks[nblocks - counts[1] + chunk_n[2 * blockIdx.x + 1] + pn + __popc(mn & below)] = code;
}

extern "C" int lbdem_psc_near_blocks(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G,
                                     double margin, uint8_t *near, uint32_t *blocks, uint32_t *counts,
                                     void *stream) {
    using namespace lbdem;
    if (!L || !P || !G || !near || !blocks || !counts || L->nx <= 0 || L->ny <= 0 || L->nz <= 0 ||
        !(margin >= 0.0)) {
        set_error("psc_near_blocks: bad arguments");
        return LBDEM_ERR_ARG;
    }
    if (!(P->dx > 0.0)) {
        set_error("psc_near_blocks: dx must be positive");
        return LBDEM_ERR_ARG;
    }
    const size_t nb = ((size_t)L->nx + 31) / 32;
    const size_t nblocks = nb * (size_t)L->ny * L->nz;
    if (nblocks >= (1ull << 32)) {
        set_error("psc_near_blocks: too many x-blocks");
        return LBDEM_ERR_ARG;
    }
    if (nb > 256 || L->ny > 4096 || L->nz > 4096) {
        set_error("psc_near_blocks: block lists cover Nx <= 8192, Ny <= 4096, Nz <= 4096");
        return LBDEM_ERR_UNSUPPORTED;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(near, 0, nblocks, st) != cudaSuccess) return check_launch("near_blocks");
    MapArgs a;
    a.keys_only = 0;
    a.table_in_scatter = 0;
    memset(&a, 0, sizeof(a));
    a.n = G->n; a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.dx = P->dx; a.dt = P->dt; a.xmin = P->xmin; a.ymin = P->ymin; a.zmin = P->zmin;
    a.pos = G->pos; a.radius = G->radius;
    for (int t = 0; t < 3; ++t) {
        a.periodic[t] = P->periodic[t] != 0;
        a.period[t] = P->period[t];
    }
    if (G->n > 0) k_near_blocks<<<G->n, 128, 0, st>>>(a, margin, near);
    // ordered lists; the chunk counts live in the tail of counts (2 + 2 * chunks words)
    const uint32_t nchunks = (uint32_t)((nblocks + LIST_CHUNK - 1) / LIST_CHUNK);
    uint32_t *chunk_n = counts + 2;
    k_list_count<<<nchunks, LIST_CHUNK, 0, st>>>(near, (uint32_t)nblocks, chunk_n);
    k_list_scan<<<1, 1024, 0, st>>>(chunk_n, nchunks, counts);
    k_list_fill<<<nchunks, LIST_CHUNK, 0, st>>>(near, (uint32_t)nblocks, (uint32_t)nb, (uint32_t)L->ny, chunk_n, counts,
                                                blocks);
    return check_launch("near_blocks");
}
