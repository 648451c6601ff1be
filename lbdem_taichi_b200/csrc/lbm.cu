// Lattice kernels: the fused PSC collide-stream step and its helpers.
//
// Data layout (HBM): populations are structure-of-arrays, x fastest,
// population q of cell c at q*Ncells + c, in two buffers (pull scheme: the
// step reads post-collision populations of the previous step from f[src],
// streams them by gathering from the 18 upwind neighbours, collides, and
// writes post-collision populations of this step to f[dst]).  One thread per
// cell, 32 consecutive x per warp, so every direction is one coalesced
// 128 B (FP32) / 64 B (16-bit) access per warp (+1 element shift for c_x != 0).
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "common.cuh"

namespace lbdem {

static thread_local char g_err[512];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return LBDEM_ERR_LAUNCH;
    }
    return LBDEM_OK;
}

struct StepArgs {
    int nx, ny, nz;
    size_t nc;
    float omega0, inv_omega0, smag_c2;
    int force_on;
    float f3x, f3y, f3z;   // 3 * body force (1/cs^2 folded in)
    float dec;             // w_q * dec = decode factor of population q (16-bit forms)
    float enc;             // enc / w_q = encode factor
    const void *src;
    void *dst;
    void *aux;
    const uint32_t *links;
    const uint8_t *row_simple;
    const uint32_t *key;
    const float4 *table;
    double fscale, tscale;
    double *force_fluid, *moment_fluid;
    float *hydro_out;
    int32_t *status;
};

// ---------------------------------------------------------------------------
// population gather (pull streaming, lbm_solver3d.py:207-236 for FLUID and
// OBSTACLE neighbours; periodic wrap as compute_neigh_index :308-342)
// ---------------------------------------------------------------------------
template <typename T, bool GATHER>
__device__ __forceinline__ void load_populations(const T *__restrict__ src, size_t nc, int x, int y, int z,
                                                 int nx, int ny, int nz, uint32_t cell, uint32_t lk, float dec,
                                                 float d[Q]) {
    if (GATHER) {
        const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            T v;
            if (q != 0 && (lk & LINK_BB(q))) {
                v = Store<T>::ld(src + (size_t)qinv(q) * nc + cell);
            } else {
                const int xs = cx(q) == 1 ? xm : (cx(q) == -1 ? xp : x);
                const int ys = cy(q) == 1 ? ym : (cy(q) == -1 ? yp : y);
                const int zs = cz(q) == 1 ? zm : (cz(q) == -1 ? zp : z);
                v = Store<T>::ld(src + (size_t)q * nc + ((uint32_t)(zs * ny + ys) * (uint32_t)nx + xs));
            }
            d[q] = Store<T>::dec(v, wq(q) * dec);
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q] = Store<T>::dec(Store<T>::ld(src + (size_t)q * nc + cell), wq(q) * dec);
    }
}

__device__ __forceinline__ unsigned lane_id() {
    return (threadIdx.y * blockDim.x + threadIdx.x) & 31u;
}

// ---------------------------------------------------------------------------
// fused step
// ---------------------------------------------------------------------------
template <typename T, bool GATHER, int SMAG>
__global__ void __launch_bounds__(256) k_psc_step(const StepArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t nc = a.nc;
    const bool inb = (x < nx) && (y < ny);
    const uint32_t cell = inb ? (uint32_t)(z * ny + y) * (uint32_t)nx + (uint32_t)x : 0u;

    uint32_t lk = LINK_FLUID;
    if (inb && !a.row_simple[z * ny + y]) lk = a.links[cell];
    const bool act = inb && !(lk & LINK_SKIP);

    float d[Q];
    if (act) {
        load_populations<T, GATHER>((const T *)a.src, nc, x, y, z, nx, ny, nz, cell, lk, a.dec, d);
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q] = 0.f;
    }

    // D3Q19 directions come in opposite pairs (q, q+1) for odd q (c_{q+1} = -c_q):
    // symmetric sums sp = d_q + d_{q+1} and antisymmetric sums am = d_q - d_{q+1}
    // carry every moment needed below.
    float sp[9], am[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        sp[p] = d[2 * p + 1] + d[2 * p + 2];
        am[p] = d[2 * p + 1] - d[2 * p + 2];
    }
    // moments (compute_rho_vel, lbm_solver3d.py:276-303), deviation form
    float drho = d[0];
#pragma unroll
    for (int p = 0; p < 9; ++p) drho += sp[p];
    float jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int q = 2 * p + 1;
        if (cx(q)) jx += cx(q) * am[p];
        if (cy(q)) jy += cy(q) * am[p];
        if (cz(q)) jz += cz(q) * am[p];
    }
    const float rho = 1.f + drho;
    const float irho = 1.f / rho;
    const float ux = jx * irho, uy = jy * irho, uz = jz * irho;
    const float usq = ux * ux + uy * uy + uz * uz;
    if (act) {
        uint32_t bad = 0;
        if (!isfinite(rho) || !isfinite(usq)) bad |= LBDEM_ST_NAN;
        if (rho <= 0.f) bad |= LBDEM_ST_RHO;
        if (usq >= 2.f / 3.f) bad |= LBDEM_ST_VELMAX;
        if (bad) atomicOr(a.status, (int)bad);
    }

    // Smagorinsky relaxation frequency (computeOmega, lbm_solver3d.py:460-513)
    float om = a.omega0;
    if (SMAG != LBDEM_SMAG_OFF) {
        float sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            if (cx(q)) sxx += sp[p];
            if (cy(q)) syy += sp[p];
            if (cz(q)) szz += sp[p];
            if (cx(q) * cy(q)) sxy += cx(q) * cy(q) * sp[p];
            if (cx(q) * cz(q)) sxz += cx(q) * cz(q) * sp[p];
            if (cy(q) * cz(q)) syz += cy(q) * cz(q) * sp[p];
        }
        // second moment of the equilibrium: rho cs^2 delta + rho u u
        float er, eux, euy, euz, pref;
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            const T *ax = (const T *)a.aux;
            if (act) {
                er = aux_dec<T>(ax[cell]);
                eux = aux_dec<T>(ax[nc + cell]);
                euy = aux_dec<T>(ax[2 * nc + cell]);
                euz = aux_dec<T>(ax[3 * nc + cell]);
                pref = aux_dec<T>(ax[4 * nc + cell]);
            } else {
                er = eux = euy = euz = 0.f;
                pref = a.omega0;
            }
        } else {
            er = drho; eux = ux; euy = uy; euz = uz;
            pref = a.omega0;
        }
        const float erho = 1.f + er;
        const float pxx = sxx - (er * CS2 + erho * eux * eux);
        const float pyy = syy - (er * CS2 + erho * euy * euy);
        const float pzz = szz - (er * CS2 + erho * euz * euz);
        const float pxy = sxy - erho * eux * euy;
        const float pxz = sxz - erho * eux * euz;
        const float pyz = syz - erho * euy * euz;
        const float pi = sqrtf(2.f * (pxx * pxx + pyy * pyy + pzz * pzz + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz)));
        const float rate = pref * (0.5f / CS2) * irho * pi;
        const float nut = a.smag_c2 * rate;
        om = 1.f / (a.inv_omega0 + nut * (1.f / CS2));
        if (SMAG == LBDEM_SMAG_REFERENCE && act) {
            T *ax = (T *)a.aux;
            ax[cell] = aux_enc<T>(drho);
            ax[nc + cell] = aux_enc<T>(ux);
            ax[2 * nc + cell] = aux_enc<T>(uy);
            ax[3 * nc + cell] = aux_enc<T>(uz);
            ax[4 * nc + cell] = aux_enc<T>(om);
        }
    }

    // Collision, one opposite pair (q, q+1) at a time, in place in d[].
    // Equilibrium deviations feq - w (compute_feq, lbm_solver3d.py:255-271):
    // fe_q = A + B, fe_{q+1} = A - B with A = w (drho + rho (4.5 cu^2 - 1.5 u^2)),
    // B = 3 w rho cu.  Body force w rho (c . F)/cs^2 (lbm_foecelover.py:150-164)
    // is odd in c: +g on q, -g on q+1 (g = 0 when no force is set).
    const float base = -1.5f * usq;
    const float gx = rho * a.f3x, gy = rho * a.f3y, gz = rho * a.f3z;

    uint32_t key = 0;
    if (a.key != nullptr && act) key = a.key[cell];
    int gid = -1;
    float hx = 0.f, hy = 0.f, hz = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
    if (key) {
        // PSC weighted collision (psclattice3d.py:240-261; B from the current
        // omega as hybridlattice.py:236-245; solid velocity :160-182):
        // fpc = f + B Os + (1-B) Of, Os_q = f_{qbar} - feq_{qbar} + feqs_q - f_q,
        // Of = -omega (f - feq), hydroforce -= B Os_q c_q
        gid = (int)key_gid(key);
        const float eps = (key & KEY_FULL) ? 1.f : (float)key_count(key) * (1.f / 125.f);
        const float taum = 1.f / om - 0.5f;
        const float Bw = eps * taum / ((1.f - eps) + taum);
        const float Bf = (1.f - Bw) * om;
        const float4 t0 = a.table[4 * gid + 0], t1 = a.table[4 * gid + 1];
        const float4 t2 = a.table[4 * gid + 2], t3 = a.table[4 * gid + 3];
        const float rx = ((float)x - t0.x) - t1.x;
        const float ry = ((float)y - t0.y) - t1.y;
        const float rz = ((float)z - t0.z) - t1.z;
        const float sx = t2.x + (t3.y * rz - t3.z * ry);
        const float sy = t2.y + (t3.z * rx - t3.x * rz);
        const float sz = t2.z + (t3.x * ry - t3.y * rx);
        const float sbase = -1.5f * (sx * sx + sy * sy + sz * sz);
        {
            const float fe0 = wq(0) * (drho + rho * base);
            const float fs0 = wq(0) * (drho + rho * sbase);
            d[0] = d[0] + Bw * (fs0 - fe0) - Bf * (d[0] - fe0);
        }
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            const float cu = cx(q) * ux + cy(q) * uy + cz(q) * uz;
            const float A = wq(q) * (drho + rho * (4.5f * cu * cu + base));
            const float B = wq(q) * 3.f * rho * cu;
            const float cus = cx(q) * sx + cy(q) * sy + cz(q) * sz;
            const float As = wq(q) * (drho + rho * (4.5f * cus * cus + sbase));
            const float Bs = wq(q) * 3.f * rho * cus;
            const float dq = d[q], db = d[q + 1];
            const float osq = db - (A - B) + (As + Bs) - dq;
            const float osb = dq - (A + B) + (As - Bs) - db;
            const float g = wq(q) * (cx(q) * gx + cy(q) * gy + cz(q) * gz);
            d[q] = dq + Bw * osq - Bf * (dq - (A + B)) + g;
            d[q + 1] = db + Bw * osb - Bf * (db - (A - B)) - g;
            const float m = Bw * (osq - osb);   // B Os_q c_q + B Os_{q+1} c_{q+1}
            if (cx(q)) hx -= cx(q) * m;
            if (cy(q)) hy -= cy(q) * m;
            if (cz(q)) hz -= cz(q) * m;
        }
        tx = ry * hz - rz * hy;
        ty = rz * hx - rx * hz;
        tz = rx * hy - ry * hx;
        if (a.hydro_out) {
            a.hydro_out[cell] = hx;
            a.hydro_out[nc + cell] = hy;
            a.hydro_out[2 * nc + cell] = hz;
        }
    } else {
        d[0] = d[0] + om * (wq(0) * (drho + rho * base) - d[0]);
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            const float cu = cx(q) * ux + cy(q) * uy + cz(q) * uz;
            const float A = wq(q) * (drho + rho * (4.5f * cu * cu + base));
            const float B = wq(q) * 3.f * rho * cu;
            const float g = wq(q) * (cx(q) * gx + cy(q) * gy + cz(q) * gz);
            d[q] = d[q] + om * ((A + B) - d[q]) + g;
            d[q + 1] = d[q + 1] + om * ((A - B) - d[q + 1]) - g;
        }
    }

    if (act) {
        T *dst = (T *)a.dst;
#pragma unroll
        for (int q = 0; q < Q; ++q) dst[(size_t)q * nc + cell] = Store<T>::enc(d[q], a.enc / wq(q));
    }

    // hydrodynamic force/torque per particle (lattice2grains,
    // psclattice3d.py:316-358): warp-segmented sum over runs of equal owner
    // id, one FP64 atomic per run and component.
    if (a.key != nullptr && __any_sync(0xffffffffu, gid >= 0)) {
        const unsigned lane = lane_id();
        const int gnext = __shfl_down_sync(0xffffffffu, gid, 1);
        const int gprev = __shfl_up_sync(0xffffffffu, gid, 1);
        const unsigned tails = __ballot_sync(0xffffffffu, lane == 31 || gnext != gid);
        const unsigned mytail = (unsigned)(__ffs(tails >> lane) - 1) + lane;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float vx = __shfl_down_sync(0xffffffffu, hx, o);
            const float vy = __shfl_down_sync(0xffffffffu, hy, o);
            const float vz = __shfl_down_sync(0xffffffffu, hz, o);
            const float wx = __shfl_down_sync(0xffffffffu, tx, o);
            const float wy = __shfl_down_sync(0xffffffffu, ty, o);
            const float wz = __shfl_down_sync(0xffffffffu, tz, o);
            if (lane + o <= mytail) {
                hx += vx; hy += vy; hz += vz;
                tx += wx; ty += wy; tz += wz;
            }
        }
        const bool head = lane == 0 || gprev != gid;
        if (head && gid >= 0) {
            double *F = a.force_fluid + 3 * (size_t)gid;
            double *M = a.moment_fluid + 3 * (size_t)gid;
            atomicAdd(F + 0, (double)hx * a.fscale);
            atomicAdd(F + 1, (double)hy * a.fscale);
            atomicAdd(F + 2, (double)hz * a.fscale);
            atomicAdd(M + 0, (double)tx * a.tscale);
            atomicAdd(M + 1, (double)ty * a.tscale);
            atomicAdd(M + 2, (double)tz * a.tscale);
        }
    }
}

// stream only: move post-collision populations to their cells and compute
// rho/u of FLUID cells (BasicLattice3D.stream, lbm_solver3d.py:197-240)
template <typename T>
__global__ void __launch_bounds__(256) k_stream_moments(const StepArgs a, float *rho_out, float *vel_out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t nc = a.nc;
    if (x >= nx || y >= ny) return;
    const uint32_t cell = (uint32_t)(z * ny + y) * (uint32_t)nx + (uint32_t)x;
    uint32_t lk = LINK_FLUID;
    if (!a.row_simple[z * ny + y]) lk = a.links[cell];
    if (lk & LINK_SKIP) return;
    const T *src = (const T *)a.src;
    T *dst = (T *)a.dst;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        T v;
        if (q != 0 && (lk & LINK_BB(q))) {
            v = src[(size_t)qinv(q) * nc + cell];
        } else {
            const int xs = cx(q) == 1 ? xm : (cx(q) == -1 ? xp : x);
            const int ys = cy(q) == 1 ? ym : (cy(q) == -1 ? yp : y);
            const int zs = cz(q) == 1 ? zm : (cz(q) == -1 ? zp : z);
            v = src[(size_t)q * nc + ((uint32_t)(zs * ny + ys) * (uint32_t)nx + xs)];
        }
        dst[(size_t)q * nc + cell] = v;
        const float dq = Store<T>::dec(v, wq(q) * a.dec);
        drho += dq;
        jx += cx(q) * dq;
        jy += cy(q) * dq;
        jz += cz(q) * dq;
    }
    if (lk & LINK_FLUID) {
        const float rho = 1.f + drho;
        rho_out[cell] = rho;
        vel_out[cell] = jx / rho;
        vel_out[nc + cell] = jy / rho;
        vel_out[2 * nc + cell] = jz / rho;
    }
}

// f = feq(rho, u) (initialize, psclattice3d.py:60-75)
template <typename T>
__global__ void k_init(const StepArgs a, const float *rho_in, const float *vel_in, int smag_ref) {
    const size_t nc = a.nc;
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    T *dst = (T *)a.dst;
    const bool skip = (a.links[c] & LINK_SKIP) != 0;
    const float rho = skip ? 1.f : rho_in[c];
    const float ux = skip ? 0.f : vel_in[c], uy = skip ? 0.f : vel_in[nc + c], uz = skip ? 0.f : vel_in[2 * nc + c];
    const float drho = rho - 1.f;
    const float usq = ux * ux + uy * uy + uz * uz;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float cu = cx(q) * ux + cy(q) * uy + cz(q) * uz;
        const float fe = wq(q) * (drho + rho * (3.f * cu + 4.5f * cu * cu - 1.5f * usq));
        dst[(size_t)q * nc + c] = Store<T>::enc(fe, a.enc / wq(q));
    }
    if (smag_ref) {
        T *ax = (T *)a.aux;
        ax[c] = aux_enc<T>(drho);
        ax[nc + c] = aux_enc<T>(ux);
        ax[2 * nc + c] = aux_enc<T>(uy);
        ax[3 * nc + c] = aux_enc<T>(uz);
        ax[4 * nc + c] = aux_enc<T>(a.omega0);
    }
}

// link masks from CellType (lbm_solver3d.py:203-236)
__global__ void k_links(const int32_t *ct, int nx, int ny, int nz, int skip_inlet, uint32_t *links) {
    const size_t nc = (size_t)nx * ny * nz;
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((size_t)nx * ny));
    const int32_t own = ct[c];
    uint32_t L = 0;
    if (own & (LBDEM_CT_OBSTACLE | LBDEM_CT_VEL_LADD | LBDEM_CT_FREE_SLIP | LBDEM_CT_VEL_INLET_LADD)) L |= LINK_SKIP;
    int32_t mskip = LBDEM_CT_OBSTACLE | LBDEM_CT_VEL_LADD | LBDEM_CT_FREE_SLIP;
    if (skip_inlet) mskip |= LBDEM_CT_VEL_INLET_LADD;
    if (own & mskip) L |= LINK_MAP_SKIP;
    if (own & LBDEM_CT_FLUID) L |= LINK_FLUID;
    const int32_t prop = LBDEM_CT_FLUID | LBDEM_CT_VEL_ZOUHE | LBDEM_CT_VEL_EXIT | LBDEM_CT_PRE_ZOUHE;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        int xn = x - cx(q), yn = y - cy(q), zn = z - cz(q);
        xn = xn >= nx ? 0 : (xn < 0 ? nx - 1 : xn);
        yn = yn >= ny ? 0 : (yn < 0 ? ny - 1 : yn);
        zn = zn >= nz ? 0 : (zn < 0 ? nz - 1 : zn);
        const int32_t ctn = ct[((size_t)zn * ny + yn) * nx + xn];
        if (!(ctn & prop) && (ctn & LBDEM_CT_OBSTACLE)) L |= LINK_BB(q);
    }
    links[c] = L;
}

// row flag: every cell of the (y,z) row is an updated FLUID cell without
// bounce-back links, so the step needs no per-cell link read there
__global__ void k_rows(const uint32_t *links, int nx, int nrows, uint8_t *row_simple) {
    const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= nrows) return;
    const uint32_t bad_mask = LINK_SKIP | 0x7FFFEu;
    int ok = 1;
    for (int x = lane; x < nx; x += 32) {
        const uint32_t L = links[(size_t)row * nx + x];
        if ((L & bad_mask) || !(L & LINK_FLUID)) ok = 0;
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) row_simple[row] = (uint8_t)ok;
}

// per-cell PSC fields from the owner keys (psclattice3d.py:45-52, 144-182)
template <typename T>
__global__ void k_decode(const StepArgs a, int smag_ref, int32_t *id, float *volfrac, float *weight,
                         float *velsolid) {
    const size_t nc = a.nc;
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const uint32_t key = a.key ? a.key[c] : 0u;
    if (!key) {
        id[c] = -1;
        volfrac[c] = 0.f;
        weight[c] = 0.f;
        velsolid[c] = velsolid[nc + c] = velsolid[2 * nc + c] = 0.f;
        return;
    }
    const int x = (int)(c % a.nx), y = (int)((c / a.nx) % a.ny), z = (int)(c / ((size_t)a.nx * a.ny));
    const int gid = (int)key_gid(key);
    const float eps = (key & KEY_FULL) ? 1.f : (float)key_count(key) * (1.f / 125.f);
    const float om = smag_ref ? aux_dec<T>(((const T *)a.aux)[4 * nc + c]) : a.omega0;
    const float taum = 1.f / om - 0.5f;
    id[c] = gid;
    volfrac[c] = eps;
    weight[c] = eps * taum / ((1.f - eps) + taum);
    const float4 t0 = a.table[4 * gid + 0], t1 = a.table[4 * gid + 1];
    const float4 t2 = a.table[4 * gid + 2], t3 = a.table[4 * gid + 3];
    const float rx = ((float)x - t0.x) - t1.x, ry = ((float)y - t0.y) - t1.y, rz = ((float)z - t0.z) - t1.z;
    velsolid[c] = t2.x + (t3.y * rz - t3.z * ry);
    velsolid[nc + c] = t2.y + (t3.z * rx - t3.x * rz);
    velsolid[2 * nc + c] = t2.z + (t3.x * ry - t3.y * rx);
}

// FP64 totals (deterministic two-pass block reduction, no atomics)
template <typename T>
__global__ void __launch_bounds__(256) k_sums(const StepArgs a, double *partials) {
    const size_t nc = a.nc;
    double m = 0, px = 0, py = 0, pz = 0;
    const T *f = (const T *)a.src;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (a.links[c] & LINK_SKIP) continue;
        float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float dq = Store<T>::dec(f[(size_t)q * nc + c], wq(q) * a.dec);
            dr += dq; jx += cx(q) * dq; jy += cy(q) * dq; jz += cz(q) * dq;
        }
        m += 1.0 + (double)dr;
        px += jx; py += jy; pz += jz;
    }
    __shared__ double sh[4][256];
    sh[0][threadIdx.x] = m; sh[1][threadIdx.x] = px; sh[2][threadIdx.x] = py; sh[3][threadIdx.x] = pz;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) partials[4 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_sums_final(const double *partials, int nblocks, double *out) {
    if (threadIdx.x < 4) {
        double s = 0;
        for (int b = 0; b < nblocks; ++b) s += partials[4 * b + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int fill_args(const lbdem_lattice *L, StepArgs &a) {
    if (!L || L->nx <= 0 || L->ny <= 0 || L->nz <= 0) {
        set_error("invalid lattice descriptor");
        return LBDEM_ERR_ARG;
    }
    if ((size_t)L->nx * L->ny * L->nz >= (1ull << 32)) {
        set_error("lattice has %zu cells; at most 2^32-1 supported", (size_t)L->nx * L->ny * L->nz);
        return LBDEM_ERR_ARG;
    }
    memset(&a, 0, sizeof(a));
    a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.nc = (size_t)L->nx * L->ny * L->nz;
    a.omega0 = L->omega0;
    a.inv_omega0 = 1.f / L->omega0;
    a.smag_c2 = L->smag_cs * L->smag_cs;
    a.force_on = L->force_on;
    a.f3x = 3.f * L->force[0]; a.f3y = 3.f * L->force[1]; a.f3z = 3.f * L->force[2];
    if (L->storage == LBDEM_F32) {
        a.dec = 1.f; a.enc = 1.f;
    } else {
        if (!(L->scale16 > 0.f)) {
            set_error("scale16 must be positive for 16-bit storage");
            return LBDEM_ERR_ARG;
        }
        a.dec = 1.f / L->scale16;
        a.enc = L->scale16;
    }
    a.aux = L->aux;
    a.links = L->links;
    a.row_simple = L->row_simple;
    a.status = L->status;
    if (!a.links || !a.row_simple || !a.status) {
        set_error("links, row_simple and status are required");
        return LBDEM_ERR_ARG;
    }
    if (L->smag_mode == LBDEM_SMAG_REFERENCE && !L->aux) {
        set_error("LBDEM_SMAG_REFERENCE needs the aux buffer");
        return LBDEM_ERR_ARG;
    }
    return LBDEM_OK;
}

static void step_geometry(const lbdem_lattice *L, dim3 &grid, dim3 &block) {
    int bx = ((L->nx + 31) / 32) * 32;
    if (bx > 256) bx = 256;
    int by = 256 / bx;
    if (by > L->ny) by = L->ny;
    block = dim3(bx, by, 1);
    grid = dim3((L->nx + bx - 1) / bx, (L->ny + by - 1) / by, L->nz);
}

template <typename T>
static int launch_step(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int src, int dst,
                       int gather, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (src < 0 || src > 1 || dst < 0 || dst > 1 || src == dst) {
        set_error("src/dst must be 0/1 and distinct");
        return LBDEM_ERR_ARG;
    }
    a.src = L->f[src];
    a.dst = L->f[dst];
    if (P && G && G->n > 0) {
        if (!P->key || !P->table || !G->force_fluid || !G->moment_fluid) {
            set_error("PSC step needs key, table and force accumulators");
            return LBDEM_ERR_ARG;
        }
        a.key = P->key;
        a.table = (const float4 *)P->table;
        a.fscale = P->rho_unit * (P->dx * P->dx * P->dx * P->dx) / (P->dt * P->dt);
        a.tscale = a.fscale * P->dx;
        a.force_fluid = G->force_fluid;
        a.moment_fluid = G->moment_fluid;
        a.hydro_out = P->hydro_out;
    }
    dim3 grid, block;
    step_geometry(L, grid, block);
#define LBDEM_STEP_CASE(G_, S_) k_psc_step<T, G_, S_><<<grid, block, 0, st>>>(a)
    if (gather) {
        if (L->smag_mode == LBDEM_SMAG_OFF) LBDEM_STEP_CASE(true, LBDEM_SMAG_OFF);
        else if (L->smag_mode == LBDEM_SMAG_REFERENCE) LBDEM_STEP_CASE(true, LBDEM_SMAG_REFERENCE);
        else LBDEM_STEP_CASE(true, LBDEM_SMAG_LOCAL);
    } else {
        if (L->smag_mode == LBDEM_SMAG_OFF) LBDEM_STEP_CASE(false, LBDEM_SMAG_OFF);
        else if (L->smag_mode == LBDEM_SMAG_REFERENCE) LBDEM_STEP_CASE(false, LBDEM_SMAG_REFERENCE);
        else LBDEM_STEP_CASE(false, LBDEM_SMAG_LOCAL);
    }
#undef LBDEM_STEP_CASE
    return check_launch("psc_step");
}

template <typename T>
static int launch_stream_moments(const lbdem_lattice *L, int src, int dst, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (src < 0 || src > 1 || dst < 0 || dst > 1 || src == dst || !L->rho || !L->vel) {
        set_error("stream_moments: bad buffers");
        return LBDEM_ERR_ARG;
    }
    a.src = L->f[src];
    a.dst = L->f[dst];
    dim3 grid, block;
    step_geometry(L, grid, block);
    k_stream_moments<T><<<grid, block, 0, st>>>(a, L->rho, L->vel);
    return check_launch("stream_moments");
}

template <typename T>
static int launch_init(const lbdem_lattice *L, int buf, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (buf < 0 || buf > 1 || !L->rho || !L->vel) {
        set_error("lattice_init: bad buffers");
        return LBDEM_ERR_ARG;
    }
    a.dst = L->f[buf];
    const unsigned nb = (unsigned)((a.nc + 255) / 256);
    k_init<T><<<nb, 256, 0, st>>>(a, L->rho, L->vel, L->smag_mode == LBDEM_SMAG_REFERENCE);
    return check_launch("lattice_init");
}

template <typename T>
static int launch_decode(const lbdem_lattice *L, const lbdem_psc *P, int32_t *id, float *vf, float *w, float *vs,
                         cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (P) {
        a.key = P->key;
        a.table = (const float4 *)P->table;
    }
    const unsigned nb = (unsigned)((a.nc + 255) / 256);
    k_decode<T><<<nb, 256, 0, st>>>(a, L->smag_mode == LBDEM_SMAG_REFERENCE, id, vf, w, vs);
    return check_launch("psc_decode");
}

template <typename T>
static int launch_sums(const lbdem_lattice *L, int buf, double *out, double *partials, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (buf < 0 || buf > 1 || !out || !partials) {
        set_error("global_sums: bad arguments");
        return LBDEM_ERR_ARG;
    }
    a.src = L->f[buf];
    k_sums<T><<<LBDEM_SUM_BLOCKS, 256, 0, st>>>(a, partials);
    k_sums_final<<<1, 32, 0, st>>>(partials, LBDEM_SUM_BLOCKS, out);
    return check_launch("global_sums");
}

}  // namespace lbdem

using namespace lbdem;

extern "C" {

int lbdem_abi_version(void) { return LBDEM_ABI_VERSION; }

const char *lbdem_last_error(void) { return g_err; }

int lbdem_build_links(const int32_t *ct, int32_t nx, int32_t ny, int32_t nz, int32_t skip_inlet, uint32_t *links,
                      uint8_t *row_simple, void *stream) {
    if (!ct || !links || !row_simple || nx <= 0 || ny <= 0 || nz <= 0) {
        set_error("build_links: bad arguments");
        return LBDEM_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nc = (size_t)nx * ny * nz;
    k_links<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(ct, nx, ny, nz, skip_inlet, links);
    const int nrows = ny * nz;
    k_rows<<<(nrows + 7) / 8, 256, 0, st>>>(links, nx, nrows, row_simple);
    return check_launch("build_links");
}

int lbdem_lattice_init(const lbdem_lattice *L, int32_t buf, void *stream) {
    if (!L) return LBDEM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (L->storage) {
        case LBDEM_F32: return launch_init<float>(L, buf, st);
        case LBDEM_F16: return launch_init<__half>(L, buf, st);
        case LBDEM_BF16: return launch_init<__nv_bfloat16>(L, buf, st);
    }
    set_error("unknown storage form %d", L->storage);
    return LBDEM_ERR_ARG;
}

int lbdem_psc_step_f32(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src, int32_t dst,
                       int32_t gather, void *stream) {
    if (!L || L->storage != LBDEM_F32) { set_error("psc_step_f32: storage mismatch"); return LBDEM_ERR_ARG; }
    return launch_step<float>(L, P, G, src, dst, gather, (cudaStream_t)stream);
}

int lbdem_psc_step_f16(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src, int32_t dst,
                       int32_t gather, void *stream) {
    if (!L || L->storage != LBDEM_F16) { set_error("psc_step_f16: storage mismatch"); return LBDEM_ERR_ARG; }
    return launch_step<__half>(L, P, G, src, dst, gather, (cudaStream_t)stream);
}

int lbdem_psc_step_bf16(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src, int32_t dst,
                        int32_t gather, void *stream) {
    if (!L || L->storage != LBDEM_BF16) { set_error("psc_step_bf16: storage mismatch"); return LBDEM_ERR_ARG; }
    return launch_step<__nv_bfloat16>(L, P, G, src, dst, gather, (cudaStream_t)stream);
}

int lbdem_stream_moments(const lbdem_lattice *L, int32_t src, int32_t dst, void *stream) {
    if (!L) return LBDEM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (L->storage) {
        case LBDEM_F32: return launch_stream_moments<float>(L, src, dst, st);
        case LBDEM_F16: return launch_stream_moments<__half>(L, src, dst, st);
        case LBDEM_BF16: return launch_stream_moments<__nv_bfloat16>(L, src, dst, st);
    }
    set_error("unknown storage form %d", L->storage);
    return LBDEM_ERR_ARG;
}

int lbdem_psc_decode(const lbdem_lattice *L, const lbdem_psc *P, int32_t *id, float *volfrac, float *weight,
                     float *velsolid, void *stream) {
    if (!L || !id || !volfrac || !weight || !velsolid) { set_error("psc_decode: bad arguments"); return LBDEM_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    switch (L->storage) {
        case LBDEM_F32: return launch_decode<float>(L, P, id, volfrac, weight, velsolid, st);
        case LBDEM_F16: return launch_decode<__half>(L, P, id, volfrac, weight, velsolid, st);
        case LBDEM_BF16: return launch_decode<__nv_bfloat16>(L, P, id, volfrac, weight, velsolid, st);
    }
    set_error("unknown storage form %d", L->storage);
    return LBDEM_ERR_ARG;
}

int lbdem_global_sums_f64(const lbdem_lattice *L, int32_t buf, double *out, double *partials, void *stream) {
    if (!L) return LBDEM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (L->storage) {
        case LBDEM_F32: return launch_sums<float>(L, buf, out, partials, st);
        case LBDEM_F16: return launch_sums<__half>(L, buf, out, partials, st);
        case LBDEM_BF16: return launch_sums<__nv_bfloat16>(L, buf, out, partials, st);
    }
    set_error("unknown storage form %d", L->storage);
    return LBDEM_ERR_ARG;
}

}  // extern "C"
