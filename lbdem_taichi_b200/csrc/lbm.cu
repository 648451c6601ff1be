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
#include <cstdlib>
#include <cstring>
#include <mutex>

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
    int kernel_choice;         // LBDEM_STEP_KERNEL: 0 default, 1 one cell/thread, 2 two cells/thread, 3 staged rows
    uint32_t qoff[Q];          // q * Ncells: element offset of population q (kernel-parameter constants)
};

// Pull streaming (lbm_solver3d.py:207-236 for FLUID and OBSTACLE neighbours;
// periodic wrap as compute_neigh_index :308-342) is inlined in the kernels.

__device__ __forceinline__ unsigned lane_id() {
    return (threadIdx.y * blockDim.x + threadIdx.x) & 31u;
}

// ---------------------------------------------------------------------------
// fused step: per-cell collision (shared by the 1- and 2-cell kernels)
// ---------------------------------------------------------------------------
// d[]: deviations f - w of the streamed populations, overwritten with the
// post-collision deviations.  aux[5]: previous (drho, ux, uy, uz, omega) in,
// current out (reference Smagorinsky mode).  key: PSC owner key of the cell.
// Outputs gid (-1 if no solid) and the cell's hydrodynamic force h and torque
// arm product t (lattice units).
template <int SMAG>
__device__ __forceinline__ void collide_cell(const StepArgs &a, float d[Q], bool act, uint32_t cell, int x, int y,
                                             int z, float aux[5], uint32_t key, int &gid, float &hx, float &hy,
                                             float &hz, float &tx, float &ty, float &tz) {
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
            er = aux[0]; eux = aux[1]; euy = aux[2]; euz = aux[3]; pref = aux[4];
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
        aux[0] = drho; aux[1] = ux; aux[2] = uy; aux[3] = uz; aux[4] = om;
    }

    // Collision, one opposite pair (q, q+1) at a time, in place in d[].
    // Equilibrium deviations feq - w (compute_feq, lbm_solver3d.py:255-271):
    // fe_q = A + B, fe_{q+1} = A - B with A = w (drho + rho (4.5 cu^2 - 1.5 u^2)),
    // B = 3 w rho cu.  Body force w rho (c . F)/cs^2 (lbm_foecelover.py:150-164)
    // is odd in c: +g on q, -g on q+1 (g = 0 when no force is set).
    const float base = -1.5f * usq;
    const float gx = rho * a.f3x, gy = rho * a.f3y, gz = rho * a.f3z;

    gid = -1;
    hx = hy = hz = tx = ty = tz = 0.f;
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
            a.hydro_out[a.nc + cell] = hy;
            a.hydro_out[2 * a.nc + cell] = hz;
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

}

// Warp-segmented sum of (h, t) over runs of equal owner id, one FP64 atomic
// per run and component (lattice2grains, psclattice3d.py:316-358).
__device__ __forceinline__ void reduce_forces(const StepArgs &a, int gid, float hx, float hy, float hz, float tx,
                                              float ty, float tz) {
    if (!__any_sync(0xffffffffu, gid >= 0)) return;
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

// ---------------------------------------------------------------------------
// packed FP32x2 arithmetic (sm_100 FFMA2/FADD2/FMUL2): two cells per thread,
// cell A in .x and cell B in .y, every operation IEEE round-to-nearest per lane
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    // packed subtract (PTX sub.rn.f32x2, sm_100+)
    unsigned long long ra = *reinterpret_cast<unsigned long long *>(&a);
    unsigned long long rb = *reinterpret_cast<unsigned long long *>(&b), rd;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    return *reinterpret_cast<float2 *>(&rd);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dot3_2(int ax, int ay, int az, float2 x, float2 y, float2 z) {
    // c . v with c in {-1, 0, 1}^3 folded at compile time
    float2 r = f2(0.f);
    bool first = true;
    if (ax) { r = ax > 0 ? x : make_float2(-x.x, -x.y); first = false; }
    if (ay) { r = first ? (ay > 0 ? y : make_float2(-y.x, -y.y)) : (ay > 0 ? add2(r, y) : sub2(r, y)); first = false; }
    if (az) { r = first ? (az > 0 ? z : make_float2(-z.x, -z.y)) : (az > 0 ? add2(r, z) : sub2(r, z)); }
    return r;
}

// Same semantics as collide_cell, on two cells at once.  Lanes whose cell is
// not updated (act false) carry zeros and their results are discarded.  When
// either cell is owned by a particle the PSC form is evaluated for both, with
// weight B = 0 on a fluid cell, which reduces it exactly to BGK.
template <int SMAG>
__device__ __forceinline__ void collide_pair(const StepArgs &a, float2 d[Q], bool acta, bool actb, int x0, int y,
                                             int z, uint32_t cell0, float2 aux[5], uint32_t keya, uint32_t keyb,
                                             int &ga, int &gb, float ha[6], float hb[6]) {
    float2 sp[9], am[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        sp[p] = add2(d[2 * p + 1], d[2 * p + 2]);
        am[p] = sub2(d[2 * p + 1], d[2 * p + 2]);
    }
    float2 drho = d[0];
#pragma unroll
    for (int p = 0; p < 9; ++p) drho = add2(drho, sp[p]);
    float2 jx = f2(0.f), jy = f2(0.f), jz = f2(0.f);
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int q = 2 * p + 1;
        if (cx(q)) jx = cx(q) > 0 ? add2(jx, am[p]) : sub2(jx, am[p]);
        if (cy(q)) jy = cy(q) > 0 ? add2(jy, am[p]) : sub2(jy, am[p]);
        if (cz(q)) jz = cz(q) > 0 ? add2(jz, am[p]) : sub2(jz, am[p]);
    }
    const float2 rho = add2(f2(1.f), drho);
    const float2 irho = make_float2(1.f / rho.x, 1.f / rho.y);
    const float2 ux = mul2(jx, irho), uy = mul2(jy, irho), uz = mul2(jz, irho);
    const float2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
    {
        uint32_t bad = 0;
        if (acta) {
            if (!isfinite(rho.x) || !isfinite(usq.x)) bad |= LBDEM_ST_NAN;
            if (rho.x <= 0.f) bad |= LBDEM_ST_RHO;
            if (usq.x >= 2.f / 3.f) bad |= LBDEM_ST_VELMAX;
        }
        if (actb) {
            if (!isfinite(rho.y) || !isfinite(usq.y)) bad |= LBDEM_ST_NAN;
            if (rho.y <= 0.f) bad |= LBDEM_ST_RHO;
            if (usq.y >= 2.f / 3.f) bad |= LBDEM_ST_VELMAX;
        }
        if (bad) atomicOr(a.status, (int)bad);
    }
    float2 om = f2(a.omega0);
    if (SMAG != LBDEM_SMAG_OFF) {
        float2 sxx = f2(0.f), syy = f2(0.f), szz = f2(0.f), sxy = f2(0.f), sxz = f2(0.f), syz = f2(0.f);
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            if (cx(q)) sxx = add2(sxx, sp[p]);
            if (cy(q)) syy = add2(syy, sp[p]);
            if (cz(q)) szz = add2(szz, sp[p]);
            if (cx(q) * cy(q)) sxy = cx(q) * cy(q) > 0 ? add2(sxy, sp[p]) : sub2(sxy, sp[p]);
            if (cx(q) * cz(q)) sxz = cx(q) * cz(q) > 0 ? add2(sxz, sp[p]) : sub2(sxz, sp[p]);
            if (cy(q) * cz(q)) syz = cy(q) * cz(q) > 0 ? add2(syz, sp[p]) : sub2(syz, sp[p]);
        }
        float2 er, eux, euy, euz, pref;
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            er = aux[0]; eux = aux[1]; euy = aux[2]; euz = aux[3]; pref = aux[4];
        } else {
            er = drho; eux = ux; euy = uy; euz = uz;
            pref = f2(a.omega0);
        }
        const float2 erho = add2(f2(1.f), er);
        const float2 ecs = mul2(er, f2(CS2));
        const float2 pxx = sub2(sxx, fma2(mul2(erho, eux), eux, ecs));
        const float2 pyy = sub2(syy, fma2(mul2(erho, euy), euy, ecs));
        const float2 pzz = sub2(szz, fma2(mul2(erho, euz), euz, ecs));
        const float2 pxy = sub2(sxy, mul2(mul2(erho, eux), euy));
        const float2 pxz = sub2(sxz, mul2(mul2(erho, eux), euz));
        const float2 pyz = sub2(syz, mul2(mul2(erho, euy), euz));
        const float2 off = fma2(pxy, pxy, fma2(pxz, pxz, mul2(pyz, pyz)));
        const float2 dia = fma2(pxx, pxx, fma2(pyy, pyy, mul2(pzz, pzz)));
        const float2 pi2 = mul2(f2(2.f), fma2(f2(2.f), off, dia));
        const float2 pi = make_float2(sqrtf(pi2.x), sqrtf(pi2.y));
        const float2 rate = mul2(mul2(pref, f2(0.5f / CS2)), mul2(irho, pi));
        const float2 den = fma2(mul2(f2(a.smag_c2), rate), f2(1.f / CS2), f2(a.inv_omega0));
        om = make_float2(1.f / den.x, 1.f / den.y);
        aux[0] = drho; aux[1] = ux; aux[2] = uy; aux[3] = uz; aux[4] = om;
    }
    const float2 base = mul2(f2(-1.5f), usq);
    const float2 gx = mul2(rho, f2(a.f3x)), gy = mul2(rho, f2(a.f3y)), gz = mul2(rho, f2(a.f3z));
    ga = gb = -1;
#pragma unroll
    for (int k = 0; k < 6; ++k) ha[k] = hb[k] = 0.f;
    if (keya | keyb) {
        float2 Bw = f2(0.f), sx = f2(0.f), sy = f2(0.f), sz = f2(0.f);
        float rxa = 0.f, rya = 0.f, rza = 0.f, rxb = 0.f, ryb = 0.f, rzb = 0.f;
        if (keya) {
            ga = (int)key_gid(keya);
            const float eps = (keya & KEY_FULL) ? 1.f : (float)key_count(keya) * (1.f / 125.f);
            const float taum = 1.f / om.x - 0.5f;
            Bw.x = eps * taum / ((1.f - eps) + taum);
            const float4 t0 = a.table[4 * ga + 0], t1 = a.table[4 * ga + 1];
            const float4 t2 = a.table[4 * ga + 2], t3 = a.table[4 * ga + 3];
            rxa = ((float)x0 - t0.x) - t1.x; rya = ((float)y - t0.y) - t1.y; rza = ((float)z - t0.z) - t1.z;
            sx.x = t2.x + (t3.y * rza - t3.z * rya);
            sy.x = t2.y + (t3.z * rxa - t3.x * rza);
            sz.x = t2.z + (t3.x * rya - t3.y * rxa);
        }
        if (keyb) {
            gb = (int)key_gid(keyb);
            const float eps = (keyb & KEY_FULL) ? 1.f : (float)key_count(keyb) * (1.f / 125.f);
            const float taum = 1.f / om.y - 0.5f;
            Bw.y = eps * taum / ((1.f - eps) + taum);
            const float4 t0 = a.table[4 * gb + 0], t1 = a.table[4 * gb + 1];
            const float4 t2 = a.table[4 * gb + 2], t3 = a.table[4 * gb + 3];
            rxb = ((float)(x0 + 1) - t0.x) - t1.x; ryb = ((float)y - t0.y) - t1.y; rzb = ((float)z - t0.z) - t1.z;
            sx.y = t2.x + (t3.y * rzb - t3.z * ryb);
            sy.y = t2.y + (t3.z * rxb - t3.x * rzb);
            sz.y = t2.z + (t3.x * ryb - t3.y * rxb);
        }
        const float2 Bf = mul2(sub2(f2(1.f), Bw), om);
        const float2 sbase = mul2(f2(-1.5f), fma2(sx, sx, fma2(sy, sy, mul2(sz, sz))));
        float2 hx = f2(0.f), hy = f2(0.f), hz = f2(0.f);
        {
            const float2 fe0 = mul2(f2(wq(0)), fma2(rho, base, drho));
            const float2 fs0 = mul2(f2(wq(0)), fma2(rho, sbase, drho));
            d[0] = sub2(fma2(Bw, sub2(fs0, fe0), d[0]), mul2(Bf, sub2(d[0], fe0)));
        }
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            const float2 cu = dot3_2(cx(q), cy(q), cz(q), ux, uy, uz);
            const float2 A = mul2(f2(wq(q)), fma2(rho, fma2(mul2(f2(4.5f), cu), cu, base), drho));
            const float2 B = mul2(mul2(f2(3.f * wq(q)), rho), cu);
            const float2 cus = dot3_2(cx(q), cy(q), cz(q), sx, sy, sz);
            const float2 As = mul2(f2(wq(q)), fma2(rho, fma2(mul2(f2(4.5f), cus), cus, sbase), drho));
            const float2 Bs = mul2(mul2(f2(3.f * wq(q)), rho), cus);
            const float2 dq = d[q], db = d[q + 1];
            const float2 feq = add2(A, B), feb = sub2(A, B);
            const float2 osq = sub2(add2(sub2(db, feb), add2(As, Bs)), dq);
            const float2 osb = sub2(add2(sub2(dq, feq), sub2(As, Bs)), db);
            const float2 g = mul2(f2(wq(q)), dot3_2(cx(q), cy(q), cz(q), gx, gy, gz));
            d[q] = add2(sub2(fma2(Bw, osq, dq), mul2(Bf, sub2(dq, feq))), g);
            d[q + 1] = sub2(sub2(fma2(Bw, osb, db), mul2(Bf, sub2(db, feb))), g);
            const float2 m = mul2(Bw, sub2(osq, osb));
            if (cx(q)) hx = cx(q) > 0 ? sub2(hx, m) : add2(hx, m);
            if (cy(q)) hy = cy(q) > 0 ? sub2(hy, m) : add2(hy, m);
            if (cz(q)) hz = cz(q) > 0 ? sub2(hz, m) : add2(hz, m);
        }
        if (keya) {
            ha[0] = hx.x; ha[1] = hy.x; ha[2] = hz.x;
            ha[3] = rya * hz.x - rza * hy.x; ha[4] = rza * hx.x - rxa * hz.x; ha[5] = rxa * hy.x - rya * hx.x;
            if (a.hydro_out) {
                a.hydro_out[cell0] = hx.x; a.hydro_out[a.nc + cell0] = hy.x; a.hydro_out[2 * a.nc + cell0] = hz.x;
            }
        }
        if (keyb) {
            hb[0] = hx.y; hb[1] = hy.y; hb[2] = hz.y;
            hb[3] = ryb * hz.y - rzb * hy.y; hb[4] = rzb * hx.y - rxb * hz.y; hb[5] = rxb * hy.y - ryb * hx.y;
            if (a.hydro_out) {
                const uint32_t c1 = cell0 + 1;
                a.hydro_out[c1] = hx.y; a.hydro_out[a.nc + c1] = hy.y; a.hydro_out[2 * a.nc + c1] = hz.y;
            }
        }
    } else {
        d[0] = fma2(om, sub2(mul2(f2(wq(0)), fma2(rho, base, drho)), d[0]), d[0]);
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            const float2 cu = dot3_2(cx(q), cy(q), cz(q), ux, uy, uz);
            const float2 A = mul2(f2(wq(q)), fma2(rho, fma2(mul2(f2(4.5f), cu), cu, base), drho));
            const float2 B = mul2(mul2(f2(3.f * wq(q)), rho), cu);
            const float2 g = mul2(f2(wq(q)), dot3_2(cx(q), cy(q), cz(q), gx, gy, gz));
            d[q] = add2(fma2(om, sub2(add2(A, B), d[q]), d[q]), g);
            d[q + 1] = sub2(fma2(om, sub2(sub2(A, B), d[q + 1]), d[q + 1]), g);
        }
    }
}

// ---------------------------------------------------------------------------
// fused step, one cell per thread (any lattice size)
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
    // Issue the 19 gather loads first (their addresses never depend on the
    // link mask), then resolve the link mask and re-fetch bounce-back
    // directions on the few cells next to an obstacle.  Element indices are
    // 32-bit: the source cell of direction q is a wrapped row base (9 per
    // thread) plus a wrapped x offset, plus q*Ncells from the parameters.
    const int xc_ = inb ? x : 0, yc_ = inb ? y : 0;
    const uint32_t cellc = inb ? cell : 0u;
    const uint32_t unx = (uint32_t)nx, nxy = (uint32_t)nx * (uint32_t)ny;
    const T *__restrict__ src = (const T *)a.src;
    T raw[Q];
    if (GATHER) {
        const uint32_t r0 = (uint32_t)(z * ny + yc_) * unx;
        const uint32_t dym = yc_ == 0 ? (uint32_t)(ny - 1) * unx : (uint32_t)(-(int)nx);
        const uint32_t dyp = yc_ == ny - 1 ? (uint32_t)(-(int)((ny - 1) * nx)) : unx;
        const uint32_t dzm = z == 0 ? (uint32_t)(nz - 1) * nxy : (uint32_t)(-(int)nxy);
        const uint32_t dzp = z == nz - 1 ? (uint32_t)(-(int)((nz - 1) * nxy)) : nxy;
        const uint32_t xm = xc_ == 0 ? (uint32_t)(nx - 1) : (uint32_t)(xc_ - 1);
        const uint32_t xp = xc_ == nx - 1 ? 0u : (uint32_t)(xc_ + 1);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const uint32_t ry = cy(q) == 1 ? dym : (cy(q) == -1 ? dyp : 0u);
            const uint32_t rz = cz(q) == 1 ? dzm : (cz(q) == -1 ? dzp : 0u);
            const uint32_t xs = cx(q) == 1 ? xm : (cx(q) == -1 ? xp : (uint32_t)xc_);
            raw[q] = Store<T>::ld(src + (r0 + ry + rz + xs + a.qoff[q]));
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) raw[q] = Store<T>::ld(src + (cellc + a.qoff[q]));
    }
    float aux[5] = {0.f, 0.f, 0.f, 0.f, a.omega0};
    if (SMAG == LBDEM_SMAG_REFERENCE && inb) {
        const T *ax = (const T *)a.aux;
#pragma unroll
        for (int k = 0; k < 5; ++k) aux[k] = aux_dec<T>(ax[cell + a.qoff[k]]);
    }
    const uint32_t key = (a.key != nullptr && inb) ? a.key[cell] : 0u;
    uint32_t lk = LINK_FLUID;
    if (inb && !a.row_simple[z * ny + y]) lk = a.links[cell];
    const bool act = inb && !(lk & LINK_SKIP);
    if (GATHER && (lk & 0x7FFFEu)) {
#pragma unroll
        for (int q = 1; q < Q; ++q)
            if (lk & LINK_BB(q)) raw[q] = Store<T>::ld(src + (cellc + a.qoff[qinv(q)]));
    }
    float d[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) d[q] = act ? Store<T>::dec(raw[q], wq(q) * a.dec) : 0.f;
    int gid;
    float hx, hy, hz, tx, ty, tz;
    collide_cell<SMAG>(a, d, act, cell, x, y, z, aux, act ? key : 0u, gid, hx, hy, hz, tx, ty, tz);
    if (act) {
        T *dst = (T *)a.dst;
#pragma unroll
        for (int q = 0; q < Q; ++q) dst[cell + a.qoff[q]] = Store<T>::enc(d[q], a.enc / wq(q));
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            T *ax = (T *)a.aux;
#pragma unroll
            for (int k = 0; k < 5; ++k) ax[cell + a.qoff[k]] = aux_enc<T>(aux[k]);
        }
    }
    if (a.key != nullptr) reduce_forces(a, gid, hx, hy, hz, tx, ty, tz);
}

// ---------------------------------------------------------------------------
// fused step, two x-neighbouring cells per thread (Nx % 64 == 0): pair loads
// and stores (8 B FP32 / 4 B 16-bit); a warp covers 64 cells of one row, so
// the x-shifted directions come from the aligned pair loads of the
// neighbouring lane (one shuffle) plus one extra element at the warp edge.
// ---------------------------------------------------------------------------
template <typename T> struct Pair;
template <> struct Pair<float> {
    using V = float2;
    __device__ __forceinline__ static V ld(const float *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }
    __device__ __forceinline__ static void st(float *p, V v) { *reinterpret_cast<float2 *>(p) = v; }
    __device__ __forceinline__ static float lo(V v) { return v.x; }
    __device__ __forceinline__ static float hi(V v) { return v.y; }
    __device__ __forceinline__ static V make(float a, float b) { return make_float2(a, b); }
    __device__ __forceinline__ static float2 dec(V v, float) { return v; }
    __device__ __forceinline__ static V enc(float2 d, float) { return d; }
    __device__ __forceinline__ static float2 adec(V v) { return v; }
    __device__ __forceinline__ static V aenc(float2 d) { return d; }
    __device__ __forceinline__ static float shup(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
    __device__ __forceinline__ static float shdn(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
};
template <> struct Pair<__half> {
    using V = __half2;
    __device__ __forceinline__ static V ld(const __half *p) { return __ldg(reinterpret_cast<const __half2 *>(p)); }
    __device__ __forceinline__ static void st(__half *p, V v) { *reinterpret_cast<__half2 *>(p) = v; }
    __device__ __forceinline__ static __half lo(V v) { return __low2half(v); }
    __device__ __forceinline__ static __half hi(V v) { return __high2half(v); }
    __device__ __forceinline__ static V make(__half a, __half b) { return __halves2half2(a, b); }
    __device__ __forceinline__ static float2 dec(V v, float s) { return mul2(__half22float2(v), f2(s)); }
    __device__ __forceinline__ static V enc(float2 d, float s) { return __float22half2_rn(mul2(d, f2(s))); }
    __device__ __forceinline__ static float2 adec(V v) { return __half22float2(v); }
    __device__ __forceinline__ static V aenc(float2 d) { return __float22half2_rn(d); }
    __device__ __forceinline__ static __half shup(__half v) {
        return __ushort_as_half((unsigned short)__shfl_up_sync(0xffffffffu, (unsigned)__half_as_ushort(v), 1));
    }
    __device__ __forceinline__ static __half shdn(__half v) {
        return __ushort_as_half((unsigned short)__shfl_down_sync(0xffffffffu, (unsigned)__half_as_ushort(v), 1));
    }
};
template <> struct Pair<__nv_bfloat16> {
    using V = __nv_bfloat162;
    __device__ __forceinline__ static V ld(const __nv_bfloat16 *p) {
        return __ldg(reinterpret_cast<const __nv_bfloat162 *>(p));
    }
    __device__ __forceinline__ static void st(__nv_bfloat16 *p, V v) { *reinterpret_cast<__nv_bfloat162 *>(p) = v; }
    __device__ __forceinline__ static __nv_bfloat16 lo(V v) { return __low2bfloat16(v); }
    __device__ __forceinline__ static __nv_bfloat16 hi(V v) { return __high2bfloat16(v); }
    __device__ __forceinline__ static V make(__nv_bfloat16 a, __nv_bfloat16 b) { return __halves2bfloat162(a, b); }
    __device__ __forceinline__ static float2 dec(V v, float s) { return mul2(__bfloat1622float2(v), f2(s)); }
    __device__ __forceinline__ static V enc(float2 d, float s) { return __float22bfloat162_rn(mul2(d, f2(s))); }
    __device__ __forceinline__ static float2 adec(V v) { return __bfloat1622float2(v); }
    __device__ __forceinline__ static V aenc(float2 d) { return __float22bfloat162_rn(d); }
    __device__ __forceinline__ static __nv_bfloat16 shup(__nv_bfloat16 v) {
        return __ushort_as_bfloat16((unsigned short)__shfl_up_sync(0xffffffffu, (unsigned)__bfloat16_as_ushort(v), 1));
    }
    __device__ __forceinline__ static __nv_bfloat16 shdn(__nv_bfloat16 v) {
        return __ushort_as_bfloat16((unsigned short)__shfl_down_sync(0xffffffffu, (unsigned)__bfloat16_as_ushort(v), 1));
    }
};

template <typename T, bool GATHER, int SMAG>
__global__ void __launch_bounds__(128) k_psc_step2(const StepArgs a) {
    using P = Pair<T>;
    using V = typename P::V;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int tx2 = blockIdx.x * blockDim.x + threadIdx.x;   // pair index along x
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    const size_t nc = a.nc;
    const bool inb = y < ny;                                  // x always in range (Nx % 64 == 0)
    const int x0 = 2 * tx2;
    const int yc_ = inb ? y : 0;
    const uint32_t cell0 = (uint32_t)(z * ny + yc_) * (uint32_t)nx + (uint32_t)x0;
    const unsigned lane = lane_id();
    const T *__restrict__ src = (const T *)a.src;
    V rv[Q];   // streamed populations of cells (x0, x0+1)
    const uint32_t unx = (uint32_t)nx, nxy = (uint32_t)nx * (uint32_t)ny;
    if (GATHER) {
        const uint32_t r0 = (uint32_t)(z * ny + yc_) * unx;
        const uint32_t dym = yc_ == 0 ? (uint32_t)(ny - 1) * unx : (uint32_t)(-(int)nx);
        const uint32_t dyp = yc_ == ny - 1 ? (uint32_t)(-(int)((ny - 1) * nx)) : unx;
        const uint32_t dzm = z == 0 ? (uint32_t)(nz - 1) * nxy : (uint32_t)(-(int)nxy);
        const uint32_t dzp = z == nz - 1 ? (uint32_t)(-(int)((nz - 1) * nxy)) : nxy;
        // x of the element just left of this warp's 64 cells, and just right of them
        const int wx0 = x0 - 2 * (int)lane;
        const uint32_t xl = wx0 == 0 ? (uint32_t)(nx - 1) : (uint32_t)(wx0 - 1);
        const uint32_t xr = wx0 + 64 == nx ? 0u : (uint32_t)(wx0 + 64);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const uint32_t ry = cy(q) == 1 ? dym : (cy(q) == -1 ? dyp : 0u);
            const uint32_t rz = cz(q) == 1 ? dzm : (cz(q) == -1 ? dzp : 0u);
            const T *row = src + (r0 + ry + rz + a.qoff[q]);
            const V v = P::ld(row + x0);
            if (cx(q) == 0) {
                rv[q] = v;
            } else if (cx(q) == 1) {        // source x-1: (x0-1, x0)
                T left = P::shup(P::hi(v));
                if (lane == 0) left = Store<T>::ld(row + xl);
                rv[q] = P::make(left, P::lo(v));
            } else {                        // source x+1: (x0+1, x0+2)
                T right = P::shdn(P::lo(v));
                if (lane == 31) right = Store<T>::ld(row + xr);
                rv[q] = P::make(P::hi(v), right);
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) rv[q] = P::ld(src + (cell0 + a.qoff[q]));
    }
    float2 aux[5] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(a.omega0)};
    if (SMAG == LBDEM_SMAG_REFERENCE && inb) {
        const T *ax = (const T *)a.aux;
#pragma unroll
        for (int k = 0; k < 5; ++k) aux[k] = P::adec(P::ld(ax + (cell0 + a.qoff[k])));
    }
    uint2 key = make_uint2(0u, 0u);
    if (a.key != nullptr && inb) key = *reinterpret_cast<const uint2 *>(a.key + cell0);
    uint32_t la = LINK_FLUID, lb = LINK_FLUID;
    if (inb && !a.row_simple[z * ny + y]) {
        const uint2 l = *reinterpret_cast<const uint2 *>(a.links + cell0);
        la = l.x;
        lb = l.y;
    }
    const bool acta = inb && !(la & LINK_SKIP), actb = inb && !(lb & LINK_SKIP);
    if (GATHER && ((la | lb) & 0x7FFFEu)) {
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            const T lo = (la & LINK_BB(q)) ? Store<T>::ld(src + (cell0 + a.qoff[qinv(q)])) : P::lo(rv[q]);
            const T hi = (lb & LINK_BB(q)) ? Store<T>::ld(src + (cell0 + 1 + a.qoff[qinv(q)])) : P::hi(rv[q]);
            rv[q] = P::make(lo, hi);
        }
    }
    float2 d[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        d[q] = P::dec(rv[q], wq(q) * a.dec);
        if (!acta) d[q].x = 0.f;
        if (!actb) d[q].y = 0.f;
    }
    int ga, gb;
    float ha[6], hb[6];
    collide_pair<SMAG>(a, d, acta, actb, x0, y, z, cell0, aux, acta ? key.x : 0u, actb ? key.y : 0u, ga, gb, ha, hb);
    T *dst = (T *)a.dst;
    if (acta && actb) {
#pragma unroll
        for (int q = 0; q < Q; ++q) P::st(dst + (cell0 + a.qoff[q]), P::enc(d[q], a.enc / wq(q)));
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            T *ax = (T *)a.aux;
#pragma unroll
            for (int k = 0; k < 5; ++k) P::st(ax + (cell0 + a.qoff[k]), P::aenc(aux[k]));
        }
    } else if (acta || actb) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const V v = P::enc(d[q], a.enc / wq(q));
            if (acta) dst[cell0 + a.qoff[q]] = P::lo(v);
            if (actb) dst[cell0 + 1 + a.qoff[q]] = P::hi(v);
        }
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            T *ax = (T *)a.aux;
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const V v = P::aenc(aux[k]);
                if (acta) ax[cell0 + a.qoff[k]] = P::lo(v);
                if (actb) ax[cell0 + 1 + a.qoff[k]] = P::hi(v);
            }
        }
    }
    if (a.key != nullptr) {
        reduce_forces(a, ga, ha[0], ha[1], ha[2], ha[3], ha[4], ha[5]);
        reduce_forces(a, gb, hb[0], hb[1], hb[2], hb[3], hb[4], hb[5]);
    }
}

// ---------------------------------------------------------------------------
// fused step with rows staged in shared memory by asynchronous bulk copies
// (cp.async.bulk on the TMA engine, completion counted on an mbarrier).
// A block owns whole lattice rows (fixed y, z; all x) and walks them
// persistently with a two-stage ring: while the threads collide row k from
// one stage, the copies of row k+1 land in the other.  Per row and stage:
// for each direction q the source row (y - c_qy, z - c_qz), periodic in y and
// z through the row index, plus the Smagorinsky state and the owner keys of
// the row itself.  x +/- 1 neighbours (periodic in x) are read from shared
// memory.  Requires Nx * sizeof(T) % 16 == 0 and Nx % blockDim.x == 0.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~2^22 polls (each poll may suspend the thread
// for a short while), flags LBDEM_ST_WAIT_TIMEOUT and reports failure.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int32_t *status) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(status, (int)LBDEM_ST_WAIT_TIMEOUT);
    return false;
}

template <typename T, int SMAG>
struct RowStage {
    // element offsets of each staged row inside one stage
    static __host__ __device__ size_t pop(int q, int nx) { return (size_t)q * nx; }
    static __host__ __device__ size_t aux(int k, int nx) { return (size_t)(Q + k) * nx; }
    static __host__ __device__ int rows() { return Q + (SMAG == LBDEM_SMAG_REFERENCE ? 5 : 0); }
    static __host__ __device__ size_t bytes(int nx, bool keys) {
        return (size_t)rows() * nx * sizeof(T) + (keys ? (size_t)nx * sizeof(uint32_t) : 0);
    }
};

template <typename T, int SMAG>
__global__ void __launch_bounds__(256, 3) k_psc_step_rows(const StepArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bars[2];
    using RS = RowStage<T, SMAG>;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t nc = a.nc;
    const int nrows = ny * nz;
    const bool keys = a.key != nullptr;
    const size_t stage_bytes = RS::bytes(nx, keys);
    const uint32_t row_bytes = (uint32_t)(nx * sizeof(T));
    const T *__restrict__ src = (const T *)a.src;
    T *dst = (T *)a.dst;

    auto stage_ptr = [&](int s) { return reinterpret_cast<T *>(smem + (size_t)s * stage_bytes); };
    auto key_ptr = [&](int s) {
        return reinterpret_cast<uint32_t *>(smem + (size_t)s * stage_bytes + (size_t)RS::rows() * nx * sizeof(T));
    };
    // one elected thread fills a stage with the rows needed by lattice row r
    auto issue = [&](int r, int s) {
        const int z = r / ny, y = r - z * ny;
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
        T *st = stage_ptr(s);
        mbar_expect_tx(&bars[s], (uint32_t)stage_bytes);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int ys = cy(q) == 1 ? ym : (cy(q) == -1 ? yp : y);
            const int zs = cz(q) == 1 ? zm : (cz(q) == -1 ? zp : z);
            bulk_g2s(st + RS::pop(q, nx), src + (size_t)q * nc + (size_t)(zs * ny + ys) * nx, row_bytes, &bars[s]);
        }
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            const T *ax = (const T *)a.aux;
#pragma unroll
            for (int k = 0; k < 5; ++k)
                bulk_g2s(st + RS::aux(k, nx), ax + (size_t)k * nc + (size_t)r * nx, row_bytes, &bars[s]);
        }
        if (keys) bulk_g2s(key_ptr(s), a.key + (size_t)r * nx, (uint32_t)(nx * sizeof(uint32_t)), &bars[s]);
    };

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int r = blockIdx.x;
    if (threadIdx.x == 0 && r < nrows) issue(r, 0);
    bool ok = true;
    int kfail = -1, rnfail = nrows;
    for (int k = 0; r < nrows; ++k, r += gridDim.x) {
        const int s = k & 1;
        const int rn = r + gridDim.x;
        if (threadIdx.x == 0 && rn < nrows) {
            // the stage about to be refilled was last read before the
            // __syncthreads that closed the previous iteration
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(rn, s ^ 1);
        }
        ok = mbar_wait_bounded(&bars[s], (uint32_t)((k >> 1) & 1), a.status);
        if (!__syncthreads_and(ok)) {
            kfail = k;
            rnfail = rn;
            break;
        }
        const int z = r / ny, y = r - z * ny;
        const bool simple = a.row_simple[r] != 0;
        const T *st = stage_ptr(s);
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            const uint32_t cell = (uint32_t)r * (uint32_t)nx + (uint32_t)x;
            const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
            const uint32_t lk = simple ? LINK_FLUID : a.links[cell];
            const bool act = !(lk & LINK_SKIP);
            float d[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int xs = cx(q) == 1 ? xm : (cx(q) == -1 ? xp : x);
                T v = st[RS::pop(q, nx) + xs];
                if (q != 0 && (lk & LINK_BB(q))) v = Store<T>::ld(src + (size_t)qinv(q) * nc + cell);
                d[q] = act ? Store<T>::dec(v, wq(q) * a.dec) : 0.f;
            }
            float aux[5] = {0.f, 0.f, 0.f, 0.f, a.omega0};
            if (SMAG == LBDEM_SMAG_REFERENCE) {
#pragma unroll
                for (int kk = 0; kk < 5; ++kk) aux[kk] = aux_dec<T>(st[RS::aux(kk, nx) + x]);
            }
            const uint32_t key = (keys && act) ? key_ptr(s)[x] : 0u;
            int gid;
            float hx, hy, hz, tx, ty, tz;
            collide_cell<SMAG>(a, d, act, cell, x, y, z, aux, key, gid, hx, hy, hz, tx, ty, tz);
            if (act) {
#pragma unroll
                for (int q = 0; q < Q; ++q) dst[(size_t)q * nc + cell] = Store<T>::enc(d[q], a.enc / wq(q));
                if (SMAG == LBDEM_SMAG_REFERENCE) {
                    T *ax = (T *)a.aux;
#pragma unroll
                    for (int kk = 0; kk < 5; ++kk) ax[(size_t)kk * nc + cell] = aux_enc<T>(aux[kk]);
                }
            }
            if (keys) reduce_forces(a, gid, hx, hy, hz, tx, ty, tz);
        }
        __syncthreads();
    }
    // after a timeout, wait (bounded again) for this block's copies still in
    // flight before its shared memory is released
    if (kfail >= 0 && threadIdx.x == 0) {
        mbar_wait_bounded(&bars[kfail & 1], (uint32_t)((kfail >> 1) & 1), a.status);
        if (rnfail < nrows) mbar_wait_bounded(&bars[(kfail + 1) & 1], (uint32_t)(((kfail + 1) >> 1) & 1), a.status);
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
    if ((size_t)L->nx * L->ny * L->nz * Q >= (1ull << 32)) {
        set_error("lattice has %zu cells; element offsets are 32-bit, so at most %llu cells are supported",
                  (size_t)L->nx * L->ny * L->nz, (unsigned long long)((1ull << 32) / Q - 1));
        return LBDEM_ERR_ARG;
    }
    memset(&a, 0, sizeof(a));
    a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.nc = (size_t)L->nx * L->ny * L->nz;
    for (int q = 0; q < Q; ++q) a.qoff[q] = (uint32_t)(q * a.nc);
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
    {
        const char *k = getenv("LBDEM_STEP_KERNEL");
        a.kernel_choice = (k && strcmp(k, "one") == 0) ? 1
                          : (k && strcmp(k, "pair") == 0) ? 2
                          : (k && strcmp(k, "rows") == 0) ? 3 : 0;
    }
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
    // Rows staged in shared memory by bulk copies (opt-in: measured slower
    // than the register-gather kernels on 256^3, see the design notes).
    if (gather && a.kernel_choice == 3 && (L->nx % 32) == 0) {
        const bool keys = a.key != nullptr;
        size_t stage = 0;
        void (*kern)(StepArgs) = nullptr;
        if (L->smag_mode == LBDEM_SMAG_OFF) {
            kern = k_psc_step_rows<T, LBDEM_SMAG_OFF>;
            stage = RowStage<T, LBDEM_SMAG_OFF>::bytes(L->nx, keys);
        } else if (L->smag_mode == LBDEM_SMAG_REFERENCE) {
            kern = k_psc_step_rows<T, LBDEM_SMAG_REFERENCE>;
            stage = RowStage<T, LBDEM_SMAG_REFERENCE>::bytes(L->nx, keys);
        } else {
            kern = k_psc_step_rows<T, LBDEM_SMAG_LOCAL>;
            stage = RowStage<T, LBDEM_SMAG_LOCAL>::bytes(L->nx, keys);
        }
        const size_t smem = 2 * stage;
        if (smem <= 200 * 1024) {
            const int nt = L->nx < 256 ? L->nx : 256;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess) {
                int per_sm = 0, dev = 0, nsm = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem) == cudaSuccess && per_sm > 0) {
                    const int nrows = L->ny * L->nz;
                    int nb = per_sm * nsm;
                    if (nb > nrows) nb = nrows;
                    kern<<<nb, nt, smem, st>>>(a);
                    return check_launch("psc_step (rows)");
                }
            }
            cudaGetLastError();
        }
    }
    dim3 grid, block;
    // Two cells per thread with packed FP32x2 arithmetic pays off where the
    // step is issue-bound (16-bit storage); the FP32 form is memory-bound and
    // runs fastest one cell per thread.  Needs Nx % 64 == 0.
    const bool pairs = (L->nx % 64) == 0 &&
                       (a.kernel_choice == 2 || (a.kernel_choice == 0 && L->storage != LBDEM_F32));
    if (pairs) {
        int bx = L->nx / 2;
        if (bx > 128) bx = 128;
        int by = 128 / bx;
        if (by > L->ny) by = L->ny;
        block = dim3(bx, by, 1);
        grid = dim3(L->nx / 2 / bx, (L->ny + by - 1) / by, L->nz);
    } else {
        step_geometry(L, grid, block);
    }
#define LBDEM_STEP_CASE(G_, S_)                                            \
    do {                                                                   \
        if (pairs) k_psc_step2<T, G_, S_><<<grid, block, 0, st>>>(a);      \
        else k_psc_step<T, G_, S_><<<grid, block, 0, st>>>(a);             \
    } while (0)
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

// ---------------------------------------------------------------------------
// Allocation-free FP64 totals: the block partials live in a file-scope device
// array instead of caller scratch.  One block per NOALLOC_CELLS_PER_BLOCK
// cells, at most NOALLOC_MAX_BLOCKS blocks, so lattices of up to
// 4096 * 65536 = 2^28 cells are covered (32 KB of device memory, held by every
// GPU that loads the library until the process exits).
// ---------------------------------------------------------------------------
constexpr int NOALLOC_MAX_BLOCKS = 4096;
constexpr size_t NOALLOC_CELLS_PER_BLOCK = 65536;
static __device__ __align__(256) double g_noalloc_partials[4 * NOALLOC_MAX_BLOCKS];

// Device address of g_noalloc_partials for the current device, looked up once
// per device (the host-side symbol is only a stand-in and must never be passed
// to a kernel).
static double *noalloc_partials_address() {
    static std::mutex mu;
    static double *addr[256] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        set_error("global_sums_f64_noalloc: no current CUDA device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            set_error("global_sums_f64_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return nullptr;
        }
        addr[dev] = static_cast<double *>(p);
    }
    return addr[dev];
}

template <typename T>
static int launch_sums_noalloc(const lbdem_lattice *L, int buf, double *out, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (buf < 0 || buf > 1 || !out) {
        set_error("global_sums_f64_noalloc: bad arguments");
        return LBDEM_ERR_ARG;
    }
    const size_t nb = (a.nc + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK;
    if (nb > (size_t)NOALLOC_MAX_BLOCKS) {
        set_error("global_sums_f64_noalloc: lattice has %zu cells; the allocation-free sums cover at most %zu "
                  "cells (use lbdem_global_sums_f64 with caller scratch)",
                  a.nc, (size_t)NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK);
        return LBDEM_ERR_ARG;
    }
    double *partials = noalloc_partials_address();
    if (!partials) return LBDEM_ERR_LAUNCH;
    a.src = L->f[buf];
    // every block writes its own four partials, so nothing needs clearing
    k_sums<T><<<(unsigned)nb, 256, 0, st>>>(a, partials);
    k_sums_final<<<1, 32, 0, st>>>(partials, (int)nb, out);
    return check_launch("global_sums_f64_noalloc");
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

int lbdem_global_sums_f64_noalloc(const lbdem_lattice *L, int32_t buf, double *out, void *stream) {
    if (!L) return LBDEM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (L->storage) {
        case LBDEM_F32: return launch_sums_noalloc<float>(L, buf, out, st);
        case LBDEM_F16: return launch_sums_noalloc<__half>(L, buf, out, st);
        case LBDEM_BF16: return launch_sums_noalloc<__nv_bfloat16>(L, buf, out, st);
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
