// PSC particle -> lattice mapping (grains2lattice, psclattice3d.py:84-182).
//
// The reference loops over every cell and, inside, over every grain
// (O(cells x grains)).  Here each particle scatters over the cells its sphere
// can touch and claims them with atomicMax on a 32-bit owner key that encodes
// the reference's winner rule, so the result is identical for any order.
//
// The geometry is FP64 with the reference's operation order; this file is
// compiled with -fmad=false so no multiply-add is contracted and the 5^3
// sub-sample counts match the reference bit for bit.
#include <math.h>

#include "common.cuh"

namespace lbdem {

struct MapArgs {
    int n, nx, ny, nz;
    double dx, dt, xmin, ymin, zmin;
    const double *pos, *radius, *vel, *omega;
    const uint32_t *links;
    uint32_t *key;
    float4 *table;
    double *prev;
    int have_prev;
    double *ff, *mf;
    int32_t *status;
};

constexpr double HALF_DIAG = 0.8660254037844386;  // 0.5 * sqrt(3.0), psclattice3d.py:111

__device__ __forceinline__ void particle_lattice(const MapArgs &a, int g, double &xc, double &yc, double &zc,
                                                 double &r) {
    // psclattice3d.py:102-105
    xc = (a.pos[3 * g + 0] - a.xmin + 0.5 * a.dx) / a.dx;
    yc = (a.pos[3 * g + 1] - a.ymin + 0.5 * a.dx) / a.dx;
    zc = (a.pos[3 * g + 2] - a.zmin + 0.5 * a.dx) / a.dx;
    r = (a.radius[g] - 0.5 * a.dx) / a.dx;
}

// Clear the cells claimed by the previous map (conservative shell), zero the
// force accumulators, and write the FP32 particle table used by the step.
__global__ void __launch_bounds__(128) k_map_clear(const MapArgs a) {
    const int g = blockIdx.x;
    if (a.have_prev) {
        const double pxc = a.prev[4 * g], pyc = a.prev[4 * g + 1], pzc = a.prev[4 * g + 2];
        const double lim = a.prev[4 * g + 3] + HALF_DIAG + 1e-6;
        if (lim > 0.0) {
            const int x0 = max(0, (int)floor(pxc - lim)), x1 = min(a.nx - 1, (int)ceil(pxc + lim));
            const int y0 = max(0, (int)floor(pyc - lim)), y1 = min(a.ny - 1, (int)ceil(pyc + lim));
            const int z0 = max(0, (int)floor(pzc - lim)), z1 = min(a.nz - 1, (int)ceil(pzc + lim));
            const int ex = x1 - x0 + 1, ey = y1 - y0 + 1, ez = z1 - z0 + 1;
            if (ex > 0 && ey > 0 && ez > 0) {
                const long long tot = (long long)ex * ey * ez;
                const double lim2 = lim * lim;
                for (long long t = threadIdx.x; t < tot; t += blockDim.x) {
                    const int i = x0 + (int)(t % ex), j = y0 + (int)((t / ex) % ey), k = z0 + (int)(t / ((long long)ex * ey));
                    const double ddx = pxc - i, ddy = pyc - j, ddz = pzc - k;
                    if (ddx * ddx + ddy * ddy + ddz * ddz < lim2)
                        a.key[((size_t)k * a.ny + j) * a.nx + i] = 0u;
                }
            }
        }
    }
    if (threadIdx.x == 0) {
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
}

// 5^3 sub-cell count (psclattice3d.py:121-131): sqrt(s) < r decided exactly;
// s is formed in the reference's order ((dx^2 + dy^2) + dz^2), the square
// root is only evaluated when s lies within a few ulps of r^2.
__device__ __forceinline__ int subcell_count(double xc, double yc, double zc, int i, int j, int k, double r) {
    if (!(r > 0.0)) return 0;
    double sx2[5], sy2[5], sz2[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const double ox = xc - (((double)i - 0.4) + 0.2 * t);
        const double oy = yc - (((double)j - 0.4) + 0.2 * t);
        const double oz = zc - (((double)k - 0.4) + 0.2 * t);
        sx2[t] = ox * ox;
        sy2[t] = oy * oy;
        sz2[t] = oz * oz;
    }
    const double rr = r * r;
    const double lo = rr * (1.0 - 0x1p-45), hi = rr * (1.0 + 0x1p-45);
    int cnt = 0;
#pragma unroll
    for (int ii = 0; ii < 5; ++ii)
#pragma unroll
        for (int jj = 0; jj < 5; ++jj) {
            const double sxy = sx2[ii] + sy2[jj];
#pragma unroll
            for (int kk = 0; kk < 5; ++kk) {
                const double s = sxy + sz2[kk];
                if (s < lo) cnt++;
                else if (s <= hi && sqrt(s) < r) cnt++;
            }
        }
    return cnt;
}

__global__ void __launch_bounds__(256) k_map_scatter(const MapArgs a) {
    const int g = blockIdx.x;
    double xc, yc, zc, r;
    particle_lattice(a, g, xc, yc, zc, r);
    if (threadIdx.x == 0) {
        a.prev[4 * g] = xc; a.prev[4 * g + 1] = yc; a.prev[4 * g + 2] = zc; a.prev[4 * g + 3] = r;
    }
    const double t_out = r + HALF_DIAG, t_in = r - HALF_DIAG;
    if (!(t_out > 0.0)) return;
    const int x0 = max(0, (int)floor(xc - t_out)), x1 = min(a.nx - 1, (int)ceil(xc + t_out));
    const int y0 = max(0, (int)floor(yc - t_out)), y1 = min(a.ny - 1, (int)ceil(yc + t_out));
    const int z0 = max(0, (int)floor(zc - t_out)), z1 = min(a.nz - 1, (int)ceil(zc + t_out));
    const int ex = x1 - x0 + 1, ey = y1 - y0 + 1, ez = z1 - z0 + 1;
    if (ex <= 0 || ey <= 0 || ez <= 0) return;
    const uint32_t gbits = 0xFFFFFFu - (uint32_t)g;
    const long long tot = (long long)ex * ey * ez;
    for (long long t = threadIdx.x; t < tot; t += blockDim.x) {
        const int i = x0 + (int)(t % ex), j = y0 + (int)((t / ex) % ey), k = z0 + (int)(t / ((long long)ex * ey));
        const size_t c = ((size_t)k * a.ny + j) * a.nx + i;
        if (a.links[c] & LINK_MAP_SKIP) continue;
        const double ddx = xc - i, ddy = yc - j, ddz = zc - k;
        const double dist = sqrt((ddx * ddx + ddy * ddy) + ddz * ddz);
        if (dist >= t_out) continue;
        uint32_t kv;
        if (dist <= t_in) {
            kv = KEY_FULL | gbits;
        } else {
            const int cnt = subcell_count(xc, yc, zc, i, j, k, r);
            if (cnt == 0) continue;   // eps = 0 never beats the empty cell (strict >)
            kv = ((uint32_t)cnt << 24) | gbits;
        }
        atomicMax(a.key + c, kv);
    }
}

}  // namespace lbdem

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
    cudaStream_t st = (cudaStream_t)stream;
    k_map_clear<<<G->n, 128, 0, st>>>(a);
    k_map_scatter<<<G->n, 256, 0, st>>>(a);
    P->have_prev = 1;
    return check_launch("psc_map");
}
