// Lattice kernels: the fused PSC collide-stream step and its helpers.
//
// Data layout (HBM): populations are blocked by 32 cells along x ("AoSoA"):
// row r = z*Ny + y holds ceil(Nx/32) x-blocks, each block 19 populations x
// 32 lanes, so population q of cell (x, y, z) is element
//   (r * NB + x/32) * 19*32 + q*32 + x%32,   NB = ceil(Nx/32),
// in two buffers (pull scheme: the step reads post-collision populations of
// the previous step from f[src], streams them by gathering from the 18 upwind
// neighbours, collides, and writes post-collision populations of this step to
// f[dst]).  One thread per cell, a warp is one x-block, so every direction is
// one coalesced 128 B (FP32) / 64 B (16-bit) access per warp (+1 element
// shift for c_x != 0), and all 19 populations of a cell sit at compile-time
// offsets q*32 from one address.  The lagged Smagorinsky state (5 values per
// cell) uses the same blocking with 5 instead of 19.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

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
    float omega0, inv_omega0, smag_k;   // smag_k = 4.5 Cs^2 (strain-rate factor folded)
    float S;                            // storage scale: h = (f - w) S / w
    float W0, W1, W2;                   // lattice weights / S (moments from h)
    float g3x, g3y, g3z;                // 3 S F: body force in h units per unit density
    float dec;                          // 1/S  (f - w = h w dec; auxiliary kernels)
    float enc;                          // S
    const void *src;
    void *dst;
    void *aux;
    const uint32_t *links;
    const uint32_t *moving;    // velocity-link bits per cell (VEL_LADD / VEL_INLET_LADD neighbours), or NULL
    float *rho;                // lagged density of moving-wall-adjacent cells (read, then rewritten);
                               // inlet densities; moments of LINK_KEEP cells
    float *vel;                // wall / inlet velocities (SoA planes); moments of LINK_KEEP cells
    const int32_t *ct;         // CellType (boundary pass only)
    void *bnd_f0;              // populations of the second-pass cells, [q][t] (Ladd inlets' constant f)
    uint32_t bnd_nb;           // second-pass cells (row length of bnd_f0)
    int slip;                  // the lattice has free-slip cells (their mirrors read inlets' post-collision f)
    const uint32_t *key;
    const float *eps;          // smooth solid fraction per cell, or NULL (exact count in the key)
    const float4 *table;
    double fscale, tscale;
    double *force_fluid, *moment_fluid;
    float *hydro_out;
    int32_t *status;
    uint32_t nb;               // x-blocks per row, ceil(Nx / 32)
    uint32_t rs;               // population elements per row, nb * 19 * 32
    uint32_t ars;              // auxiliary elements per row, nb * 5 * 32
    int keep_lag;              // aux present: keep (drho, u, omega) of every collision (stress diagnostics)
    float per_x, per_y, per_z;  // periodic-image lengths (lattice units) of the map, 0: no images
    float iper_x, iper_y, iper_z;   // their reciprocals (0 without images)
    int wrap_any;                   // some axis has periodic images
    const uint32_t *blist;          // pipelined step: x-block ids (row * nb + x/32) of this phase
    const uint32_t *bcount;         // their number (device)
    int bfrom_end;                  // the list is read from the end of blist (near blocks)
    uint32_t nblocks;               // rows * nb
    float *stress_out;              // 7 planes of Ncells: stress of the gathered state (fused output), or NULL
    uint32_t links_all;             // nonzero: the link mask of every cell (no per-cell masks are read)
    uint32_t lbase;                 // listed launches: index of the first list entry of this launch
    int aux16;                      // FP32 storage with the lagged state in FP16 (aux is __half)
};

// Lagged-state element idx of aux (the blocked offsets do not depend on the
// element width): the storage type, or FP16 under FP32 storage with aux16.
// LAGM: the width as a template argument (LAG_STORE: the storage type,
// LAG_HALF: FP16; the fused step's own instantiations) or read from a.aux16
// (LAG_RUNTIME: every other kernel).
constexpr int LAG_STORE = 0, LAG_HALF = 1, LAG_RUNTIME = 2;
// Element `base + off` (off a compile-time constant at the call sites, so it
// folds into the address).
template <typename T, int LAGM = LAG_RUNTIME>
__device__ __forceinline__ float lag_ld(const StepArgs &a, uint32_t base, uint32_t off) {
    if constexpr (sizeof(T) == 4 && LAGM != LAG_STORE) {
        if (LAGM == LAG_HALF || a.aux16) return __half2float((static_cast<const __half *>(a.aux) + base)[off]);
    }
    return aux_dec<T>((static_cast<const T *>(a.aux) + base)[off]);
}
template <typename T, int LAGM = LAG_RUNTIME>
__device__ __forceinline__ void lag_st(const StepArgs &a, uint32_t base, uint32_t off, float v) {
    if constexpr (sizeof(T) == 4 && LAGM != LAG_STORE) {
        if (LAGM == LAG_HALF || a.aux16) {
            (static_cast<__half *>(a.aux) + base)[off] = __float2half_rn(v);
            return;
        }
    }
    (static_cast<T *>(a.aux) + base)[off] = aux_enc<T>(v);
}

// Pull streaming (lbm_solver3d.py:207-236 for FLUID and OBSTACLE neighbours;
// periodic wrap as compute_neigh_index :308-342) is inlined in the kernels.

__device__ __forceinline__ unsigned lane_id() {
    return (threadIdx.y * blockDim.x + threadIdx.x) & 31u;
}

// Hardware reciprocal and square root (PTX rcp.approx / sqrt.approx, at most
// one ulp from the rounded result): the step uses them for 1/rho, the
// Smagorinsky relaxation frequency and the PSC weight, where an ulp is far
// below the FP32 tolerance of the whole step.
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_fast(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ---------------------------------------------------------------------------
// Lane-generic arithmetic: the collision is written over a value type V with
// Lanes<V> (cells per value) so that a packed form can reuse it; the step
// instantiates it for V = float, one cell per thread.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }

// Packed FP32 pairs (B200 f32x2 FMA / add): two independent FP32 operations per
// issued instruction, each lane rounded exactly as its scalar form.  The
// collision runs its per-direction-pair arithmetic two pairs at a time.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

template <class V> struct Lanes;
template <> struct Lanes<float> {
    static constexpr int N = 1;
    __device__ __forceinline__ static float splat(float s) { return s; }
    __device__ __forceinline__ static float get(float v, int) { return v; }
    __device__ __forceinline__ static void set(float &v, int, float s) { v = s; }
    __device__ __forceinline__ static float rcp(float v) { return rcp_fast(v); }
    __device__ __forceinline__ static float sqrt(float v) { return sqrt_fast(v); }
};
// Two cells per thread: V = float2, every operation one f32x2 instruction
// rounded per lane exactly as its scalar form (a - b as fma(b, -1, a)).
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return sub2(a, b); }
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
template <> struct Lanes<float2> {
    static constexpr int N = 2;
    __device__ __forceinline__ static float2 splat(float s) { return make_float2(s, s); }
    __device__ __forceinline__ static float get(float2 v, int i) { return i ? v.y : v.x; }
    __device__ __forceinline__ static void set(float2 &v, int i, float s) {
        if (i) v.y = s;
        else v.x = s;
    }
    __device__ __forceinline__ static float2 rcp(float2 v) { return make_float2(rcp_fast(v.x), rcp_fast(v.y)); }
    __device__ __forceinline__ static float2 sqrt(float2 v) { return make_float2(sqrt_fast(v.x), sqrt_fast(v.y)); }
};
// c_q . (x, y, z) for odd q (whose first non-zero component is +1), with the
// zero components dropped at compile time (q is a constant after unrolling;
// 0 * v is not foldable under IEEE rules).
template <class V>
__device__ __forceinline__ V cdot(int q, V x, V y, V z) {
    V r = x;
    bool first = true;
    if (cx(q)) { r = x; first = false; }
    if (cy(q)) { r = first ? y : (cy(q) > 0 ? r + y : r - y); first = false; }
    if (cz(q)) { r = first ? z : (cz(q) > 0 ? r + z : r - z); }
    return r;
}

// Per-cell results of the collision needed by the force reduction.
struct CellForce {
    int gid;                       // owner particle, -1 if none
    float hx, hy, hz, tx, ty, tz;  // hydrodynamic force and torque (lattice units)
    float rho;                     // density of the collision
};

// Minimum image of a lever-arm component along an axis mapped with periodic
// images: r - P rint(r / P); with P = 1/P = 0 (no images) it returns r exactly.
__device__ __forceinline__ float min_image(float r, float P, float iP) { return fmaf(-P, rintf(r * iP), r); }

// PSC quantities of one cell owned by a particle (psclattice3d.py:144-182;
// B from the current omega as hybridlattice.py:236-245): weight B, 3 u_s,
// and the cell's force B (j - rho u_s) with its torque about the centre.
// WRAP: the map has periodic images, lever arms take the minimum image (the
// branch-free form is the identity where an axis has none).
template <bool WRAP>
__device__ __forceinline__ float psc_cell(const StepArgs &a, uint32_t key, float eps_smooth, float om, float rho,
                                          float jx, float jy, float jz, int x, int y, int z, float &s3x, float &s3y,
                                          float &s3z, CellForce &cf) {
    cf.gid = (int)key_gid(key);
    const float eps = a.eps ? eps_smooth : ((key & KEY_FULL) ? 1.f : (float)key_count(key) * (1.f / 125.f));
    const float taum = rcp_fast(om) - 0.5f;
    const float Bw = eps * taum * rcp_fast((1.f - eps) + taum);
    const float4 t0 = a.table[4 * cf.gid + 0], t1 = a.table[4 * cf.gid + 1];
    const float4 t2 = a.table[4 * cf.gid + 2], t3 = a.table[4 * cf.gid + 3];
    // integer part first (exact), then the fractional centre: image cells round as interior ones
    float ix = (float)x - t0.x, iy = (float)y - t0.y, iz = (float)z - t0.z;
    if constexpr (WRAP) {
        ix = min_image(ix, a.per_x, a.iper_x);
        iy = min_image(iy, a.per_y, a.iper_y);
        iz = min_image(iz, a.per_z, a.iper_z);
    }
    const float rx = ix - t1.x, ry = iy - t1.y, rz = iz - t1.z;
    const float sx = t2.x + (t3.y * rz - t3.z * ry);
    const float sy = t2.y + (t3.z * rx - t3.x * rz);
    const float sz = t2.z + (t3.x * ry - t3.y * rx);
    s3x = 3.f * sx; s3y = 3.f * sy; s3z = 3.f * sz;
    cf.hx = Bw * fmaf(-rho, sx, jx);
    cf.hy = Bw * fmaf(-rho, sy, jy);
    cf.hz = Bw * fmaf(-rho, sz, jz);
    cf.tx = ry * cf.hz - rz * cf.hy;
    cf.ty = rz * cf.hx - rx * cf.hz;
    cf.tz = rx * cf.hy - ry * cf.hx;
    return Bw;
}

// ---------------------------------------------------------------------------
// fused step: collision in scaled-deviation ("h") form
// ---------------------------------------------------------------------------
// Populations are carried as h_q = (f_q - w_q) S / w_q.  Because w_q = w_qbar,
// the BGK, PSC and body-force updates of the reference are w-free in h:
//   feq_h = S (drho + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2))      (compute_feq)
//   g_h   = 3 S rho (c.F)                          (ForcedLattice3D, added last)
// and the weights only enter the moments (W_k = w_k / S).  h[] holds the
// streamed populations; every post-collision population goes to out(q, h_q)
// as soon as it is known (registers are the occupancy limit).  aux[5]:
// previous (drho, ux, uy, uz, omega); the current ones go to aux_out(k, v)
// (reference Smagorinsky mode).  psc: the warp holds at least one owned cell (warp-
// uniform), so every cell takes the PSC form, fluid cells with B = 0.
// macro(rho, 3ux, 3uy, 3uz) receives the moments once they are known.
// OVR: collide with the density and velocity in ovr[4] = (rho, ux, uy, uz)
// instead of the moments of h -- the boundary pass, where a wet-node rule set
// them (the reference always collides with its rho / vel fields).
// PACK_PSC: the PSC pair updates also run two pairs per f32x2 instruction
// (same rounding per lane; needs the registers of the row-staged kernel).
template <class V, int SMAG, bool OVR = false, bool WRAP = false, bool PACK_PSC = false, class HA, class Out,
          class AuxOut, class Macro>
__device__ __forceinline__ void collide(const StepArgs &a, const HA &h, const bool act[], const int xs[], int y,
                                        int z, const V aux[5], bool psc, const uint32_t key[], const float eps[],
                                        CellForce cf[], Out &&out, AuxOut &&aux_out, Macro &&macro,
                                        const float *ovr = nullptr) {
    using L = Lanes<V>;
    // Opposite pairs (q, q+1), q odd: sp = h_q + h_{q+1}, am = h_q - h_{q+1}.
    // Pair p = (q-1)/2 has direction c_q: p0 (1,0,0), p1 (0,1,0), p2 (0,0,1),
    // p3 (1,1,0), p4 (1,-1,0), p5 (1,0,1), p6 (1,0,-1), p7 (0,1,1), p8 (0,1,-1).
    V sp[9], am[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        sp[p] = h[2 * p + 1] + h[2 * p + 2];
        am[p] = h[2 * p + 1] - h[2 * p + 2];
    }
    // moments (compute_rho_vel, lbm_solver3d.py:276-303)
    const V W1 = L::splat(a.W1), W2 = L::splat(a.W2);
    const V pxy = sp[3] + sp[4], pxz = sp[5] + sp[6], pyz = sp[7] + sp[8];
    V drho = vfma(L::splat(a.W0), h[0], vfma(W1, (sp[0] + sp[1]) + sp[2], W2 * ((pxy + pxz) + pyz)));
    V jx = vfma(W1, am[0], W2 * ((am[3] + am[4]) + (am[5] + am[6])));
    V jy = vfma(W1, am[1], W2 * ((am[3] - am[4]) + (am[7] + am[8])));
    V jz = vfma(W1, am[2], W2 * ((am[5] - am[6]) + (am[7] - am[8])));
    if constexpr (OVR) {
        // PSC force with the set (rho, u): -B sum_q Os_q c_q = B (2 j - rho (u + u_s)),
        // i.e. the closed form below with j replaced by 2 j - rho u
        const V r = L::splat(ovr[0]);
        jx = vfma(L::splat(2.f), jx, -r * L::splat(ovr[1]));
        jy = vfma(L::splat(2.f), jy, -r * L::splat(ovr[2]));
        jz = vfma(L::splat(2.f), jz, -r * L::splat(ovr[3]));
        drho = r - L::splat(1.f);
    }
    const V rho = L::splat(1.f) + drho;
    const V irho = L::rcp(rho);
    const V i3 = L::splat(3.f) * irho;
    V u3x, u3y, u3z;                                                               // 3u
    if constexpr (OVR) {
        u3x = L::splat(3.f * ovr[1]); u3y = L::splat(3.f * ovr[2]); u3z = L::splat(3.f * ovr[3]);
    } else {
        u3x = jx * i3; u3y = jy * i3; u3z = jz * i3;
    }
    macro(rho, u3x, u3y, u3z);
    const V nU = vfma(u3x, u3x, vfma(u3y, u3y, u3z * u3z)) * L::splat(-1.f / 3.f);   // -3 u^2
#pragma unroll
    for (int i = 0; i < L::N; ++i) {
        const float r = L::get(rho, i), U = -L::get(nU, i);
        if (act[i] && !(r > 0.f && r < 3.0e38f && U < 2.f)) {
            uint32_t bad = 0;
            if (!isfinite(r) || !isfinite(U)) bad |= LBDEM_ST_NAN;
            if (r <= 0.f) bad |= LBDEM_ST_RHO;
            if (U >= 2.f) bad |= LBDEM_ST_VELMAX;
            atomicOr(a.status, (int)(bad ? bad : LBDEM_ST_NAN));
        }
    }

    // Smagorinsky relaxation frequency (computeOmega, lbm_solver3d.py:460-513):
    // Pi = sum c c (f - feq_lagged); omega = 1 / (1/omega0 + 3 Cs^2 rate),
    // rate = omega_prev / (2 cs^2 rho) sqrt(2 Pi:Pi)
    V om = L::splat(a.omega0);
    if (SMAG != LBDEM_SMAG_OFF) {
        const V sxx = vfma(W1, sp[0], W2 * (pxy + pxz));
        const V syy = vfma(W1, sp[1], W2 * (pxy + pyz));
        const V szz = vfma(W1, sp[2], W2 * (pxz + pyz));
        const V sxy = W2 * (sp[3] - sp[4]);
        const V sxz = W2 * (sp[5] - sp[6]);
        const V syz = W2 * (sp[7] - sp[8]);
        // second moment of the equilibrium deviation: drho cs^2 delta + rho u u
        const V third = L::splat(1.f / 3.f);
        V er, eux, euy, euz, pref;
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            er = aux[0]; eux = aux[1]; euy = aux[2]; euz = aux[3]; pref = aux[4];
        } else {
            er = drho; eux = u3x * third; euy = u3y * third; euz = u3z * third;
            pref = L::splat(a.omega0);
        }
        const V erho = L::splat(1.f) + er;
        const V ecs = er * third;
        const V qx = erho * eux, qy = erho * euy;
        const V Pxx = sxx - vfma(qx, eux, ecs);
        const V Pyy = syy - vfma(qy, euy, ecs);
        const V Pzz = szz - vfma(erho * euz, euz, ecs);
        const V Pxy = sxy - qx * euy;
        const V Pxz = sxz - qx * euz;
        const V Pyz = syz - qy * euz;
        const V diag = vfma(Pxx, Pxx, vfma(Pyy, Pyy, Pzz * Pzz));
        const V offd = vfma(Pxy, Pxy, vfma(Pxz, Pxz, Pyz * Pyz));
        const V pi = L::sqrt(vfma(L::splat(4.f), offd, L::splat(2.f) * diag));
        om = L::rcp(vfma(L::splat(a.smag_k) * pref, irho * pi, L::splat(a.inv_omega0)));
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            aux_out(0, drho);
            aux_out(1, u3x * third);
            aux_out(2, u3y * third);
            aux_out(3, u3z * third);
            aux_out(4, om);
        }
    }

    if (SMAG != LBDEM_SMAG_REFERENCE && a.keep_lag) {
        // lagged state for the stress diagnostics: this collision's moments and omega
        const V third = L::splat(1.f / 3.f);
        aux_out(0, drho);
        aux_out(1, u3x * third);
        aux_out(2, u3y * third);
        aux_out(3, u3z * third);
        aux_out(4, om);
    }
    const V S = L::splat(a.S);
    const V SR = S * rho;
    const V rg3x = rho * L::splat(a.g3x), rg3y = rho * L::splat(a.g3y), rg3z = rho * L::splat(a.g3z);
#pragma unroll
    for (int i = 0; i < L::N; ++i) {
        cf[i].gid = -1;
        cf[i].hx = cf[i].hy = cf[i].hz = cf[i].tx = cf[i].ty = cf[i].tz = 0.f;
        cf[i].rho = L::get(rho, i);
    }
    if (!psc) {
        // BGK: h' = (1-om) h + om feq_h + g_h, one opposite pair at a time.
        // om feq_h = k0 + k2 (v^2 - U) +/- om S rho v, v = c.(3u); the odd part
        // and the body force combine into c.V, V = om S rho 3u + 3 S rho F.
        const V k0 = om * S * drho;
        const V k2 = L::splat(0.5f) * om * SR;
        const V omc = L::splat(1.f) - om;
        const V ks = om * SR;
        const V Vx = vfma(ks, u3x, rg3x), Vy = vfma(ks, u3y, rg3y), Vz = vfma(ks, u3z, rg3z);
        out(0, vfma(omc, h[0], vfma(k2, nU, k0)));
        if constexpr (L::N == 1) {
            // pairs (0,1) (2,3) (4,5) (6,7) packed, pair 8 scalar
            const float2 k2_ = f2(k2, k2), k0_ = f2(k0, k0), nU_ = f2(nU, nU), omc_ = f2(omc, omc);
#pragma unroll
            for (int p = 0; p < 8; p += 2) {
                const int q = 2 * p + 1, r = q + 2;
                const float2 v = f2(cdot(q, u3x, u3y, u3z), cdot(r, u3x, u3y, u3z));
                const float2 cv = f2(cdot(q, Vx, Vy, Vz), cdot(r, Vx, Vy, Vz));
                const float2 e = fma2(k2_, fma2(v, v, nU_), k0_);
                const float2 hp = fma2(omc_, f2(h[q], h[r]), add2(e, cv));
                const float2 hm = fma2(omc_, f2(h[q + 1], h[r + 1]), sub2(e, cv));
                out(q, hp.x); out(q + 1, hm.x); out(r, hp.y); out(r + 1, hm.y);
            }
            const V v = cdot(17, u3x, u3y, u3z);
            const V cv = cdot(17, Vx, Vy, Vz);
            const V e = vfma(k2, vfma(v, v, nU), k0);
            out(17, vfma(omc, h[17], e + cv));
            out(18, vfma(omc, h[18], e - cv));
        } else {
#pragma unroll
            for (int p = 0; p < 9; ++p) {
                const int q = 2 * p + 1;
                const V v = cdot(q, u3x, u3y, u3z);
                const V cv = cdot(q, Vx, Vy, Vz);
                const V e = vfma(k2, vfma(v, v, nU), k0);
                out(q, vfma(omc, h[q], e + cv));
                out(q + 1, vfma(omc, h[q + 1], e - cv));
            }
        }
        return;
    }
    // PSC weighted collision (psclattice3d.py:240-261):
    //   fpc = f + B Os + (1-B) Of,  Os_q = f_qbar - feq_qbar + feqs_q - f_q,
    //   Of = -om (f - feq),  hydroforce -= B sum_q Os_q c_q.
    // Per pair, with Bf = (1-B) om, c1 = 1 - B - Bf, feq = A +/- Bo,
    // feqs = As +/- Bso (solid velocity u_s, same rho):
    //   h_q'    = c1 h_q + B h_qbar + E + O,  h_qbar' = c1 h_qbar + B h_q + E - O,
    //   E = Bf A + B (As - A),  O = (B + Bf) Bo + B Bso + g_h.
    // sum_q Os_q c_q = rho (u_s - u) exactly for this equilibrium, so the
    // cell's force is B (j - rho u_s) (psc_cell).
    V Bw = L::splat(0.f), s3x = Bw, s3y = Bw, s3z = Bw;
#pragma unroll
    for (int i = 0; i < L::N; ++i) {
        if (key[i]) {
            float sx, sy, sz;
            L::set(Bw, i, psc_cell<WRAP>(a, key[i], eps[i], L::get(om, i), L::get(rho, i), L::get(jx, i), L::get(jy, i),
                                   L::get(jz, i), xs[i], y, z, sx, sy, sz, cf[i]));
            L::set(s3x, i, sx); L::set(s3y, i, sy); L::set(s3z, i, sz);
        }
    }
    const V Bf = (L::splat(1.f) - Bw) * om;
    const V nUs = vfma(s3x, s3x, vfma(s3y, s3y, s3z * s3z)) * L::splat(-1.f / 3.f);
    const V k2 = L::splat(0.5f) * SR;
    const V eA = k2 * (Bf - Bw), eS = k2 * Bw, e0 = Bf * (S * drho);
    const V c1 = (L::splat(1.f) - Bf) - Bw;
    const V ca = L::splat(0.5f) * (c1 + Bw);   // (c1 + B)/2
    const V cb = L::splat(0.5f) * (c1 - Bw);   // (c1 - B)/2
    const V kb = (Bw + Bf) * SR, ks = Bw * SR;
    const V Vx = vfma(kb, u3x, vfma(ks, s3x, rg3x));
    const V Vy = vfma(kb, u3y, vfma(ks, s3y, rg3y));
    const V Vz = vfma(kb, u3z, vfma(ks, s3z, rg3z));
    // q = 0: h0' = (c1 + B) h0 + Bf A0 + B (As0 - A0), A0 = S drho - k2 U
    out(0, vfma(c1 + Bw, h[0], vfma(eA, nU, vfma(eS, nUs, e0))));
    if constexpr (PACK_PSC && L::N == 1) {
        // pairs (0,1) (2,3) (4,5) (6,7) packed, pair 8 scalar
        const float2 eA_ = f2(eA, eA), nU_ = f2(nU, nU), eS_ = f2(eS, eS), nUs_ = f2(nUs, nUs), e0_ = f2(e0, e0);
        const float2 ca_ = f2(ca, ca), cb_ = f2(cb, cb);
#pragma unroll
        for (int p = 0; p < 8; p += 2) {
            const int q = 2 * p + 1, r = q + 2;
            const float2 v = f2(cdot(q, u3x, u3y, u3z), cdot(r, u3x, u3y, u3z));
            const float2 vs = f2(cdot(q, s3x, s3y, s3z), cdot(r, s3x, s3y, s3z));
            const float2 O = f2(cdot(q, Vx, Vy, Vz), cdot(r, Vx, Vy, Vz));
            const float2 E = fma2(eA_, fma2(v, v, nU_), fma2(eS_, fma2(vs, vs, nUs_), e0_));
            const float2 SE = fma2(ca_, f2(sp[p], sp[p + 1]), E);
            const float2 AO = fma2(cb_, f2(am[p], am[p + 1]), O);
            const float2 hp = add2(SE, AO), hm = sub2(SE, AO);
            out(q, hp.x); out(q + 1, hm.x); out(r, hp.y); out(r + 1, hm.y);
        }
        const V v = cdot(17, u3x, u3y, u3z);
        const V vs = cdot(17, s3x, s3y, s3z);
        const V O = cdot(17, Vx, Vy, Vz);
        const V E = vfma(eA, vfma(v, v, nU), vfma(eS, vfma(vs, vs, nUs), e0));
        const V SE = vfma(ca, sp[8], E);
        const V AO = vfma(cb, am[8], O);
        out(17, SE + AO);
        out(18, SE - AO);
    } else {
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int q = 2 * p + 1;
            const V v = cdot(q, u3x, u3y, u3z);
            const V vs = cdot(q, s3x, s3y, s3z);
            const V O = cdot(q, Vx, Vy, Vz);
            const V E = vfma(eA, vfma(v, v, nU), vfma(eS, vfma(vs, vs, nUs), e0));
            const V SE = vfma(ca, sp[p], E);
            const V AO = vfma(cb, am[p], O);
            out(q, SE + AO);
            out(q + 1, SE - AO);
        }
    }
}

// Warp-segmented sum of (h, t) over runs of equal owner id, one FP64 atomic
// per run and component (lattice2grains, psclattice3d.py:316-358).
__device__ __forceinline__ void reduce_forces(const StepArgs &a, CellForce c) {
    const unsigned lane = lane_id();
    const int gid = c.gid;
    const int gnext = __shfl_down_sync(0xffffffffu, gid, 1);
    const int gprev = __shfl_up_sync(0xffffffffu, gid, 1);
    const unsigned tails = __ballot_sync(0xffffffffu, lane == 31 || gnext != gid);
    const unsigned mytail = (unsigned)(__ffs(tails >> lane) - 1) + lane;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float vx = __shfl_down_sync(0xffffffffu, c.hx, o);
        const float vy = __shfl_down_sync(0xffffffffu, c.hy, o);
        const float vz = __shfl_down_sync(0xffffffffu, c.hz, o);
        const float wx = __shfl_down_sync(0xffffffffu, c.tx, o);
        const float wy = __shfl_down_sync(0xffffffffu, c.ty, o);
        const float wz = __shfl_down_sync(0xffffffffu, c.tz, o);
        if (lane + o <= mytail) {
            c.hx += vx; c.hy += vy; c.hz += vz;
            c.tx += wx; c.ty += wy; c.tz += wz;
        }
    }
    const bool head = lane == 0 || gprev != gid;
    if (head && gid >= 0) {
        double *F = a.force_fluid + 3 * (size_t)gid;
        double *M = a.moment_fluid + 3 * (size_t)gid;
        atomicAdd(F + 0, (double)c.hx * a.fscale);
        atomicAdd(F + 1, (double)c.hy * a.fscale);
        atomicAdd(F + 2, (double)c.hz * a.fscale);
        atomicAdd(M + 0, (double)c.tx * a.tscale);
        atomicAdd(M + 1, (double)c.ty * a.tscale);
        atomicAdd(M + 2, (double)c.tz * a.tscale);
    }
}

// ---------------------------------------------------------------------------
// fused step, one cell per thread
// ---------------------------------------------------------------------------
#ifndef ONE_THREADS
#define ONE_THREADS 256
#endif
#ifndef ONE_MIN_BLOCKS
#define ONE_MIN_BLOCKS 4
#endif

// Moving walls (VEL_LADD neighbours, lbm_solver3d.py:222-225): the bounced
// population gains 2 w_q rho (c_q . u_wall)/cs^2, rho being the cell's density
// of the previous collision (kept in rho[] for these cells) and u_wall the
// velocity stored at the wall cell; in h units that is 6 S rho (c_q . u_wall).
// Ladd inlets (VEL_INLET_LADD neighbours, :225-229) use the inlet's density.
__device__ __forceinline__ void moving_wall_terms(const StepArgs &a, uint32_t cell, int x, int y, int z, float h[Q]) {
    const uint32_t mv = a.moving[cell];
    const float k = 6.f * a.S;
    const float rc = a.rho[cell];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        if (!(mv & LINK_BB(q))) continue;
        int xn = x - cx(q), yn = y - cy(q), zn = z - cz(q);
        xn = xn < 0 ? nx - 1 : (xn >= nx ? 0 : xn);
        yn = yn < 0 ? ny - 1 : (yn >= ny ? 0 : yn);
        zn = zn < 0 ? nz - 1 : (zn >= nz ? 0 : zn);
        const size_t n = ((size_t)zn * ny + yn) * nx + xn;
        const float cu = cx(q) * a.vel[n] + cy(q) * a.vel[a.nc + n] + cz(q) * a.vel[2 * a.nc + n];
        const float r = (a.links[n] & LINK_INLET) ? a.rho[n] : rc;
        h[q] += k * r * cu;
    }
}

// Stress diagnostics of the state the step gathers (compute_stress,
// lbm_solver3d.py:347-404, evaluated on the post-stream populations h[] of
// this cell and the lagged (drho, u, omega) of its last collision in lag[]),
// written as an optional output of the fused step:
// sigma = -(1 - omega/2) (sum c c (f - w) - (drho cs^2 delta + rho u u)),
// 7 planes (xx, yy, zz, xy, xz, yz, shear magnitude), the same values as
// k_stress computes from the materialised state.
__device__ __forceinline__ void write_stress(const StepArgs &a, const float h[Q], const float lag[5], uint32_t cell) {
    float sp[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) sp[p] = h[2 * p + 1] + h[2 * p + 2];
    const float W1 = a.W1, W2 = a.W2;
    const float pxy = sp[3] + sp[4], pxz = sp[5] + sp[6], pyz = sp[7] + sp[8];
    const float sxx = fmaf(W1, sp[0], W2 * (pxy + pxz));
    const float syy = fmaf(W1, sp[1], W2 * (pxy + pyz));
    const float szz = fmaf(W1, sp[2], W2 * (pxz + pyz));
    const float sxy = W2 * (sp[3] - sp[4]), sxz = W2 * (sp[5] - sp[6]), syz = W2 * (sp[7] - sp[8]);
    const float dr = lag[0], ux = lag[1], uy = lag[2], uz = lag[3], om = lag[4];
    const float rho = 1.f + dr, ecs = dr * CS2;
    const float k = -(1.f - 0.5f * om);
    const float txy = k * (sxy - rho * ux * uy), txz = k * (sxz - rho * ux * uz), tyz = k * (syz - rho * uy * uz);
    float *o = a.stress_out + cell;
    const size_t nc = a.nc;
    o[0] = k * (sxx - (ecs + rho * ux * ux));
    o[nc] = k * (syy - (ecs + rho * uy * uy));
    o[2 * nc] = k * (szz - (ecs + rho * uz * uz));
    o[3 * nc] = txy;
    o[4 * nc] = txz;
    o[5 * nc] = tyz;
    o[6 * nc] = sqrtf(0.5f * (txy * txy + txz * txz + tyz * tyz));
}

// The part of the fused step after the loads: bounce-back refetch, moving
// walls, optional stress, collision, stores and the force reduction of one
// cell, given its streamed populations raw[] (storage type), the lagged state
// aux[], its owner key and link mask.  Shared by the kernel that gathers with
// its own loads and the one that stages rows in shared memory.
// psc_given: the collision form when the caller has decided it (0 BGK, 1
// PSC); -1: PSC when any cell of the warp is owned (a warp is one x-block).
template <typename T, bool GATHER, int SMAG, bool WRAP, bool STRESS, bool PACK_PSC = false, int LAGM = LAG_RUNTIME>
__device__ __forceinline__ void step_cell(const StepArgs &a, int x, int y, int z, bool inb, uint32_t cell,
                                          uint32_t own, uint32_t aown, T raw[Q], float aux[5], uint32_t key,
                                          uint32_t lk, int psc_given = -1) {
    const bool act = inb && !(lk & (LINK_SKIP | LINK_DEFER));
    if (!act) key = 0u;
    if (GATHER && (lk & 0x7FFFEu)) {
        const T *p = static_cast<const T *>(a.src) + own;
#pragma unroll
        for (int q = 1; q < Q; ++q)
            if (lk & LINK_BB(q)) raw[q] = Store<T>::ld(p + qinv(q) * 32);
    }
    float h[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) h[q] = Store<T>::widen(raw[q]);
    if (GATHER && (lk & LINK_MOVING)) moving_wall_terms(a, cell, x, y, z, h);
    if constexpr (STRESS) {
        if (act) write_stress(a, h, aux, cell);
    }
    const unsigned owners = __ballot_sync(0xffffffffu, key != 0u);
    const bool psc = a.key != nullptr && (psc_given >= 0 ? psc_given != 0 : owners != 0u);
    CellForce cf[1];
    const bool acts[1] = {act};
    const int xs[1] = {x};
    const uint32_t keys[1] = {key};
    const float epss[1] = {(a.eps != nullptr && key) ? a.eps[cell] : 0.f};
    // post-collision values overwrite h[] and aux[] and are stored together
    collide<float, SMAG, false, WRAP, PACK_PSC>(
        a, h, acts, xs, y, z, aux, psc, keys, epss, cf, [&](int q, float v) { h[q] = v; },
        [&](int k, float v) { aux[k] = v; },
        [&](float r, float u3x, float u3y, float u3z) {
            // post-stream moments of an exit's / inlet's interior neighbour, read by the boundary pass
            if (GATHER && act && (lk & LINK_KEEP) && a.vel != nullptr) {
                a.rho[cell] = r;
                a.vel[cell] = u3x * (1.f / 3.f);
                a.vel[a.nc + cell] = u3y * (1.f / 3.f);
                a.vel[2 * a.nc + cell] = u3z * (1.f / 3.f);
            }
        });
    if (act && (lk & LINK_MOVING)) a.rho[cell] = cf[0].rho;   // lagged density of the next stream
    if (act) {
        T *d = static_cast<T *>(a.dst) + own;
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q * 32] = Store<T>::narrow(h[q]);
        if (SMAG == LBDEM_SMAG_REFERENCE || a.keep_lag) {
#pragma unroll
            for (int k = 0; k < 5; ++k) lag_st<T, LAGM>(a, aown, k * 32, aux[k]);
        }
        if (a.hydro_out) {
            a.hydro_out[cell] = cf[0].hx;
            a.hydro_out[a.nc + cell] = cf[0].hy;
            a.hydro_out[2 * a.nc + cell] = cf[0].hz;
        }
    }
    if (a.key != nullptr && owners != 0u) reduce_forces(a, cf[0]);
}

// The fused step of the cell (x, y, z) of this thread: gathers, lagged state,
// key and link mask, then step_cell.
template <typename T, bool GATHER, int SMAG, bool WRAP, bool STRESS, int LAGM = LAG_RUNTIME>
__device__ __forceinline__ void step_at(const StepArgs &a, int x, int y, int z) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool inb = (x < nx) && (y < ny);
    const int xc_ = inb ? x : 0, yc_ = inb ? y : 0;
    const uint32_t row = (uint32_t)(z * ny + yc_);
    const uint32_t cell = row * (uint32_t)nx + (uint32_t)xc_;
    const uint32_t rs = a.rs;                         // elements per row of populations
    const uint32_t r0 = row * rs;
    const uint32_t own = r0 + xslot((uint32_t)xc_, QB);
    // Issue the 19 gather loads first (their addresses never depend on the
    // link mask), then resolve the link mask and re-fetch bounce-back
    // directions on the few cells next to an obstacle.  One pointer per
    // upwind (row, x) slot; the direction index is an immediate offset.
    const T *__restrict__ src = static_cast<const T *>(a.src);
    T raw[Q];
    if (GATHER) {
        const uint32_t dym = yc_ == 0 ? (uint32_t)(ny - 1) * rs : (uint32_t)(-(int)rs);
        const uint32_t dyp = yc_ == ny - 1 ? (uint32_t)(-(int)((ny - 1) * rs)) : rs;
        const uint32_t zs = (uint32_t)ny * rs;
        const uint32_t dzm = z == 0 ? (uint32_t)(nz - 1) * zs : (uint32_t)(-(int)zs);
        const uint32_t dzp = z == nz - 1 ? (uint32_t)(-(int)((nz - 1) * zs)) : zs;
        const uint32_t sx0 = xslot((uint32_t)xc_, QB);
        const uint32_t sxm = xslot(xc_ == 0 ? (uint32_t)(nx - 1) : (uint32_t)(xc_ - 1), QB);
        const uint32_t sxp = xslot(xc_ == nx - 1 ? 0u : (uint32_t)(xc_ + 1), QB);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const uint32_t ry = cy(q) == 1 ? dym : (cy(q) == -1 ? dyp : 0u);
            const uint32_t rz = cz(q) == 1 ? dzm : (cz(q) == -1 ? dzp : 0u);
            const uint32_t xs = cx(q) == 1 ? sxm : (cx(q) == -1 ? sxp : sx0);
            const T *p = src + (r0 + ry + rz + xs);
            raw[q] = Store<T>::ld(p + q * 32);
        }
    } else {
        const T *p = src + own;
#pragma unroll
        for (int q = 0; q < Q; ++q) raw[q] = Store<T>::ld(p + q * 32);
    }
    float aux[5] = {0.f, 0.f, 0.f, 0.f, a.omega0};
    const uint32_t aown = row * a.ars + xslot((uint32_t)xc_, AB);
    if (SMAG == LBDEM_SMAG_REFERENCE || STRESS) {
#pragma unroll
        for (int k = 0; k < 5; ++k) aux[k] = lag_ld<T, LAGM>(a, aown, k * 32);
    }
    uint32_t key = (a.key != nullptr) ? a.key[cell] : 0u;
    // the link mask is read for every cell (a flag that skipped this load for
    // plain blocks cost more -- a dependent load before it -- than the 4 B it
    // saved), unless one value holds for the whole lattice (kernel argument)
    const uint32_t lk = a.links_all ? a.links_all : a.links[cell];
    step_cell<T, GATHER, SMAG, WRAP, STRESS, false, LAGM>(a, x, y, z, inb, cell, own, aown, raw, aux, key, lk);
}

// LISTED (pipelined stepping): one-dimensional blocks whose warps take the
// x-blocks of a compact list (blist / bcount), so every warp of a CTA has
// work; otherwise the grid covers the lattice.  A warp is one x-block.
// STRESS: also write the stress diagnostics of the gathered state (a.stress_out).
// LAGM: the lagged state's width (LAG_STORE / LAG_HALF fixed, or LAG_RUNTIME).
template <typename T, bool GATHER, int SMAG, bool WRAP, bool LISTED = false, bool STRESS = false,
          int LAGM = LAG_RUNTIME>
__global__ void __launch_bounds__(ONE_THREADS, ONE_MIN_BLOCKS) k_psc_step(const StepArgs a) {
    int x, y, z;
    if constexpr (LISTED) {
        const uint32_t w = a.lbase + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (w >= *a.bcount) return;   // warp-uniform
        // entry: z | y | x-block (bits 20-31 | 8-19 | 0-7)
        const uint32_t e = a.blist[a.bfrom_end ? a.nblocks - *a.bcount + w : w];
        x = (int)((e & 0xFFu) * 32u + (threadIdx.x & 31u));
        y = (int)((e >> 8) & 0xFFFu);
        z = (int)(e >> 20);
    } else {
        x = blockIdx.x * blockDim.x + threadIdx.x;
        y = blockIdx.y * blockDim.y + threadIdx.y;
        z = blockIdx.z;
    }
    step_at<T, GATHER, SMAG, WRAP, STRESS, LAGM>(a, x, y, z);
}

// The list entries beyond those a listed launch of k_psc_step covered (from
// a.lbase), a warp per entry, striding by the grid's warps: a launch sized
// from an earlier step's list length leaves none or a few for this one.
template <typename T, int SMAG, int LAGM>
__global__ void __launch_bounds__(ONE_THREADS) k_psc_step_listed_rest(const StepArgs a) {
    const uint32_t n = *a.bcount;
    const uint32_t stride = gridDim.x * (blockDim.x >> 5);
    for (uint32_t w = a.lbase + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n; w += stride) {
        const uint32_t e = a.blist[a.bfrom_end ? a.nblocks - n + w : w];
        step_at<T, true, SMAG, false, false, LAGM>(a, (int)((e & 0xFFu) * 32u + (threadIdx.x & 31u)),
                                             (int)((e >> 8) & 0xFFFu), (int)(e >> 20));
    }
}

// ---------------------------------------------------------------------------
// fused step with the gathered rows staged in shared memory by the tensor
// memory accelerator (TMA)
// ---------------------------------------------------------------------------
// A lattice row (z, y) needs, for direction q, population q of the upwind row
// (y - c_qy, z - c_qz) (periodic wrap), shifted by -c_qx along x.  In the
// x-blocked layout population q of a whole row is one box of the 5-D view
// [z][y][x-block][q][lane] (32 lanes x 1 direction x NB blocks), which lands
// in shared memory as the row's x order; the x shift and its periodic wrap are
// then an index into that copy.  Each persistent CTA walks rows r =
// blockIdx.x + k gridDim.x, one cell per consumer thread (rows of at most 256
// cells), with ROW_STAGES rows in flight: a producer warp issues the 19
// population boxes, the lagged-state box (reference Smagorinsky) and the
// owner-key and link-mask rows of a row into a free stage while the consumer
// warps collide the rows already landed; each consumer warp releases a stage
// as soon as it has read its cells, so warps do not wait for one another.  The
// copies hold no registers, so many more bytes are in flight per SM than the
// loads of resident threads could hold.  Each cell is then the same
// arithmetic as k_psc_step (step_cell), so both kernels give identical
// results.  Waits are bounded: a wait that gives up sets
// LBDEM_ST_WAIT_TIMEOUT, the producer waits (bounded) for the CTA's copies in
// flight, and the CTA returns.
constexpr int ROW_STAGES = 4;
constexpr int ROW_THREADS = 256;
#ifndef ROW_MIN_BLOCKS
#define ROW_MIN_BLOCKS 3
#endif

struct RowMaps {
    CUtensorMap f;        // 5-D populations of the source buffer: lane, q, x-block, y, z; box 32 x 1 x NB x 1 x 1
    CUtensorMap aux;      // 5-D lagged state: lane, k, x-block, y, z; box 32 x 5 x NB x 1 x 1
    CUtensorMap key;      // 2-D owner keys (Nx, Ny*Nz), box BW x 1
    CUtensorMap link;     // 2-D link masks, same
    uint32_t tx_bytes;    // bytes the copies of one row deliver
    int32_t kl_tma;       // key / link rows come by TMA (Nx % 4 == 0), else by plain loads
    int32_t kl_box;       // width of the key / link boxes (Nx rounded up to 4)
    int32_t use_aux;      // the lagged-state box is loaded
};

// Stage layout in shared memory, fixed at compile time so that every
// direction's copy sits at an immediate offset (rows of at most 256 cells =
// 8 x-blocks): 19 direction slots, the lagged state, the key and link rows.
template <typename T> struct RowLayout {
    static constexpr uint32_t slot = 32u * 8u * sizeof(T);
    static constexpr uint32_t off_aux = Q * slot;
    static constexpr uint32_t off_key = off_aux + 5u * 32u * 8u * sizeof(T);
    static constexpr uint32_t off_link = off_key + 256u * 4u;
    static constexpr uint32_t stage = off_link + 256u * 4u;
    static_assert(slot % 128u == 0 && off_key % 128u == 0 && stage % 128u == 0, "128-byte aligned copies");
};

#ifndef ROW_L2_PROMOTION
#define ROW_L2_PROMOTION CU_TENSOR_MAP_L2_PROMOTION_NONE
#endif

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded: false after about 2^22 polls (seconds; a copy takes microseconds)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < (1u << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1,
                                            int c2, int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6, %7}], [%2];" ::"r"(dst),
        "l"(map), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(dst),
        "l"(map), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

// issue the copies of row r into the stage at byte offset `base` (one thread)
template <typename T>
__device__ __forceinline__ void row_issue(const StepArgs &a, const RowMaps &m, uint32_t base, uint32_t bar, int r) {
    using RL = RowLayout<T>;
    const int ny = a.ny, nz = a.nz;
    const int z = r / ny, y = r - z * ny;
    mbar_expect_tx(bar, m.tx_bytes);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int yq = y - cy(q), zq = z - cz(q);
        yq = yq < 0 ? ny - 1 : (yq >= ny ? 0 : yq);
        zq = zq < 0 ? nz - 1 : (zq >= nz ? 0 : zq);
        tma_load_5d(base + q * RL::slot, &m.f, bar, 0, q, 0, yq, zq);
    }
    if (m.use_aux) tma_load_5d(base + RL::off_aux, &m.aux, bar, 0, 0, 0, y, z);
    if (m.kl_tma) {
        if (a.key != nullptr) tma_load_2d(base + RL::off_key, &m.key, bar, 0, r);
        if (!a.links_all) tma_load_2d(base + RL::off_link, &m.link, bar, 0, r);
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Warp roles: the last warp of the CTA is the producer (its lane 0 issues the
// copies of each row into a free stage); the other 32 NB threads are the
// consumers, one cell each.  full[s] completes when the copies of stage s have
// landed; empty[s] when every consumer warp has released it, so consumer warps
// run up to ROW_STAGES rows apart and no CTA-wide barrier sits in the loop.
template <typename T, int SMAG, bool WRAP>
__global__ void __launch_bounds__(ROW_THREADS + 32, ROW_MIN_BLOCKS) k_psc_step_rows(const StepArgs a,
                                                                                  const __grid_constant__ RowMaps m) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[ROW_STAGES], empty[ROW_STAGES];
    __shared__ volatile int abort_flag;
    const int nx = a.nx, ny = a.ny;
    const int nrows = ny * a.nz;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t ncons = blockDim.x - 32u;          // consumer threads: 32 NB
    const bool producer = threadIdx.x >= ncons;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ROW_STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), ncons / 32u);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();
    if (producer) {
        if (threadIdx.x == ncons) {
            int issued = 0;
            for (int k = 0;; ++k) {
                const int r = blockIdx.x + k * gridDim.x;
                if (r >= nrows || abort_flag) break;
                const int st = k % ROW_STAGES;
                if (k >= ROW_STAGES && !mbar_wait(smem_u32(&empty[st]), (uint32_t)(k / ROW_STAGES - 1) & 1u)) {
                    abort_flag = 1;
                    break;
                }
                row_issue<T>(a, m, sbase + st * RowLayout<T>::stage, smem_u32(&full[st]), r);
                issued = k + 1;
            }
            if (abort_flag) {
                atomicOr(a.status, (int)LBDEM_ST_WAIT_TIMEOUT);
                // wait (bounded) for the copies this CTA still has in flight: the last row issued into each stage
                for (int k = issued - ROW_STAGES; k < issued; ++k)
                    if (k >= 0) mbar_wait(smem_u32(&full[k % ROW_STAGES]), (uint32_t)(k / ROW_STAGES) & 1u);
            }
        }
        return;
    }
    using RL = RowLayout<T>;
    constexpr uint32_t spe = RL::slot / sizeof(T);   // elements per direction's row copy
    for (int k = 0;; ++k) {
        const int r = blockIdx.x + k * gridDim.x;
        if (r >= nrows) break;
        const int st = k % ROW_STAGES;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&full[st]), (uint32_t)(k / ROW_STAGES) & 1u));
        if (!ok || abort_flag) {
            if ((threadIdx.x & 31u) == 0) abort_flag = 1;
            break;
        }
        const unsigned char *stage = smem + st * RL::stage;
        const T *sf = reinterpret_cast<const T *>(stage);
        const T *sa = reinterpret_cast<const T *>(stage + RL::off_aux);
        const uint32_t *sk = reinterpret_cast<const uint32_t *>(stage + RL::off_key);
        const uint32_t *sl = reinterpret_cast<const uint32_t *>(stage + RL::off_link);
        const int z = r / ny, y = r - z * ny;
        const int x = (int)threadIdx.x;
        const bool inb = x < nx;
        const int xc = inb ? x : 0;
        const int xm = xc == 0 ? nx - 1 : xc - 1, xp = xc == nx - 1 ? 0 : xc + 1;
        T raw[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) raw[q] = sf[q * spe + (cx(q) == 1 ? xm : (cx(q) == -1 ? xp : xc))];
        float aux[5] = {0.f, 0.f, 0.f, 0.f, a.omega0};
        if (SMAG == LBDEM_SMAG_REFERENCE) {
            const T *ap = sa + xslot((uint32_t)xc, AB);
#pragma unroll
            for (int kk = 0; kk < 5; ++kk) aux[kk] = aux_dec<T>(ap[kk * 32]);
        }
        const uint32_t cell = (uint32_t)r * (uint32_t)nx + (uint32_t)xc;
        uint32_t key, lk;
        if (m.kl_tma) {
            key = a.key != nullptr ? sk[xc] : 0u;
            lk = a.links_all ? a.links_all : sl[xc];
        } else {
            key = a.key != nullptr ? a.key[cell] : 0u;
            lk = a.links_all ? a.links_all : a.links[cell];
        }
        // every read of this stage is done: release it to the producer
        __syncwarp();
        if ((threadIdx.x & 31u) == 0) mbar_arrive(smem_u32(&empty[st]));
        const uint32_t own = (uint32_t)r * a.rs + xslot((uint32_t)xc, QB);
        const uint32_t aown = (uint32_t)r * a.ars + xslot((uint32_t)xc, AB);
        step_cell<T, true, SMAG, WRAP, false, true, LAG_STORE>(a, x, y, z, inb, cell, own, aown, raw, aux, key, lk);
    }
}

// Two x-adjacent cells per consumer thread (16-bit storage, even Nx): the
// staged rows are read as 32-bit pairs (x, x+1) -- for c_x = +-1 the shifted
// pair is assembled from two aligned words with a byte permute -- and the
// collision runs on float2 values (f32x2 instructions, each lane rounded as
// the one-cell form, so the results are identical), with every population
// widened on demand from the packed pair instead of held as two floats.
// Stores are pairs too.  Warps whose 64 cells include wall, moving-wall,
// open-boundary or skipped cells, or that use the smooth solid fraction, run
// the one-cell step for each of their two cells instead.
template <typename T> struct Pair16;
template <> struct Pair16<__half> {
    __device__ __forceinline__ static float2 widen(uint32_t w) {
        return __half22float2(*reinterpret_cast<const __half2 *>(&w));
    }
    __device__ __forceinline__ static uint32_t narrow(float2 v) {
        const __half2 h = __floats2half2_rn(v.x, v.y);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
};
template <> struct Pair16<__nv_bfloat16> {
    __device__ __forceinline__ static float2 widen(uint32_t w) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&w));
    }
    __device__ __forceinline__ static uint32_t narrow(float2 v) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
};
template <typename T> struct PairRow {
    const uint32_t *w;
    __device__ __forceinline__ float2 operator[](int q) const { return Pair16<T>::widen(w[q]); }
};

#ifndef ROW2_MIN_BLOCKS
#define ROW2_MIN_BLOCKS 3
#endif
constexpr uint32_t LINK_NOT_PLAIN = 0x7FFFEu | LINK_SKIP | LINK_DEFER | LINK_MOVING | LINK_KEEP;

template <typename T, int SMAG, bool WRAP>
__global__ void __launch_bounds__(ROW_THREADS / 2 + 32, ROW2_MIN_BLOCKS) k_psc_step_rows2(
    const StepArgs a, const __grid_constant__ RowMaps m) {
    using RL = RowLayout<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[ROW_STAGES], empty[ROW_STAGES];
    __shared__ volatile int abort_flag;
    const int nx = a.nx, ny = a.ny;
    const int nrows = ny * a.nz;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t ncons = blockDim.x - 32u;          // consumer threads: 16 NB, NB even (whole warps)
    const bool producer = threadIdx.x >= ncons;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ROW_STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), ncons / 32u);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();
    if (producer) {
        if (threadIdx.x == ncons) {
            int issued = 0;
            for (int k = 0;; ++k) {
                const int r = blockIdx.x + k * gridDim.x;
                if (r >= nrows || abort_flag) break;
                const int st = k % ROW_STAGES;
                if (k >= ROW_STAGES && !mbar_wait(smem_u32(&empty[st]), (uint32_t)(k / ROW_STAGES - 1) & 1u)) {
                    abort_flag = 1;
                    break;
                }
                row_issue<T>(a, m, sbase + st * RL::stage, smem_u32(&full[st]), r);
                issued = k + 1;
            }
            if (abort_flag) {
                atomicOr(a.status, (int)LBDEM_ST_WAIT_TIMEOUT);
                for (int k = issued - ROW_STAGES; k < issued; ++k)
                    if (k >= 0) mbar_wait(smem_u32(&full[k % ROW_STAGES]), (uint32_t)(k / ROW_STAGES) & 1u);
            }
        }
        return;
    }
    constexpr uint32_t spe = RL::slot / sizeof(T);   // elements per direction's row copy
    for (int k = 0;; ++k) {
        const int r = blockIdx.x + k * gridDim.x;
        if (r >= nrows) break;
        const int st = k % ROW_STAGES;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&full[st]), (uint32_t)(k / ROW_STAGES) & 1u));
        if (!ok || abort_flag) {
            if ((threadIdx.x & 31u) == 0) abort_flag = 1;
            break;
        }
        const unsigned char *stage = smem + st * RL::stage;
        const T *sf = reinterpret_cast<const T *>(stage);
        const T *sa = reinterpret_cast<const T *>(stage + RL::off_aux);
        const uint32_t *sk = reinterpret_cast<const uint32_t *>(stage + RL::off_key);
        const uint32_t *sl = reinterpret_cast<const uint32_t *>(stage + RL::off_link);
        const int z = r / ny, y = r - z * ny;
        const int x0 = 2 * (int)threadIdx.x;
        const bool inb = x0 < nx;                     // Nx even: both cells or neither
        const int xc = inb ? x0 : 0;
        const uint32_t cell = (uint32_t)r * (uint32_t)nx + (uint32_t)xc;
        uint32_t key0, key1, lk0, lk1;
        if (m.kl_tma) {
            key0 = a.key != nullptr ? sk[xc] : 0u;
            key1 = a.key != nullptr ? sk[xc + 1] : 0u;
            lk0 = a.links_all ? a.links_all : sl[xc];
            lk1 = a.links_all ? a.links_all : sl[xc + 1];
        } else {
            key0 = a.key != nullptr ? a.key[cell] : 0u;
            key1 = a.key != nullptr ? a.key[cell + 1] : 0u;
            lk0 = a.links_all ? a.links_all : a.links[cell];
            lk1 = a.links_all ? a.links_all : a.links[cell + 1];
        }
        const bool plain = !__any_sync(0xffffffffu, ((lk0 | lk1) & LINK_NOT_PLAIN) != 0u) && a.eps == nullptr;
        if (plain) {
            const int xm2 = xc == 0 ? nx - 2 : xc - 2, xp2 = xc + 2 == nx ? 0 : xc + 2;
            const uint32_t *sw = reinterpret_cast<const uint32_t *>(sf);
            uint32_t raw[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const uint32_t *row = sw + q * (spe / 2);
                if (cx(q) == 0) {
                    raw[q] = row[xc >> 1];
                } else if (cx(q) == 1) {       // (x - 1, x): high half of word x-2, low half of word x
                    raw[q] = __byte_perm(row[xm2 >> 1], row[xc >> 1], 0x5432);
                } else {                       // (x + 1, x + 2): high half of word x, low half of word x+2
                    raw[q] = __byte_perm(row[xc >> 1], row[xp2 >> 1], 0x5432);
                }
            }
            float2 aux[5] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                             make_float2(0.f, 0.f), make_float2(a.omega0, a.omega0)};
            if (SMAG == LBDEM_SMAG_REFERENCE) {
                const uint32_t *ap = reinterpret_cast<const uint32_t *>(sa + xslot((uint32_t)xc, AB));
#pragma unroll
                for (int kk = 0; kk < 5; ++kk) aux[kk] = Pair16<T>::widen(ap[kk * 16]);
            }
            __syncwarp();
            if ((threadIdx.x & 31u) == 0) mbar_arrive(smem_u32(&empty[st]));
            const bool act = inb;
            const uint32_t own = (uint32_t)r * a.rs + xslot((uint32_t)xc, QB);
            const uint32_t aown = (uint32_t)r * a.ars + xslot((uint32_t)xc, AB);
            const uint32_t k0 = act ? key0 : 0u, k1 = act ? key1 : 0u;
            // the PSC form is chosen per x-block (16 lanes) as the one-cell kernel chooses it per warp: the
            // PSC update with B = 0 rounds differently from the BGK one
            const unsigned owners = __ballot_sync(0xffffffffu, (k0 | k1) != 0u);
            const bool psc_warp = a.key != nullptr && owners != 0u;
            const bool psc = psc_warp && (owners & ((threadIdx.x & 16u) ? 0xFFFF0000u : 0x0000FFFFu)) != 0u;
            CellForce cf[2];
            const bool acts[2] = {act, act};
            const int xs[2] = {x0, x0 + 1};
            const uint32_t keys[2] = {k0, k1};
            const float epss[2] = {0.f, 0.f};
            uint32_t *d = reinterpret_cast<uint32_t *>(static_cast<T *>(a.dst) + own);
            const PairRow<T> hrow{raw};
            collide<float2, SMAG, false, WRAP>(
                a, hrow, acts, xs, y, z, aux, psc, keys, epss, cf,
                [&](int q, float2 v) {
                    if (act) d[q * 16] = Pair16<T>::narrow(v);
                },
                [&](int kk, float2 v) { aux[kk] = v; }, [&](float2, float2, float2, float2) {});
            if (act) {
                if (SMAG == LBDEM_SMAG_REFERENCE || a.keep_lag) {
                    uint32_t *ap = reinterpret_cast<uint32_t *>(static_cast<T *>(a.aux) + aown);
#pragma unroll
                    for (int kk = 0; kk < 5; ++kk) ap[kk * 16] = Pair16<T>::narrow(aux[kk]);
                }
                if (a.hydro_out) {
                    a.hydro_out[cell] = cf[0].hx;
                    a.hydro_out[a.nc + cell] = cf[0].hy;
                    a.hydro_out[2 * a.nc + cell] = cf[0].hz;
                    a.hydro_out[cell + 1] = cf[1].hx;
                    a.hydro_out[a.nc + cell + 1] = cf[1].hy;
                    a.hydro_out[2 * a.nc + cell + 1] = cf[1].hz;
                }
            }
            if (psc_warp) {
                // one reduction of the pair's summed force where both cells have the same owner (or one
                // has none) in every lane; otherwise one per cell
                const bool split = __any_sync(0xffffffffu, cf[0].gid >= 0 && cf[1].gid >= 0 && cf[0].gid != cf[1].gid);
                if (!split) {
                    CellForce c2 = cf[0];
                    c2.gid = cf[0].gid >= 0 ? cf[0].gid : cf[1].gid;
                    c2.hx += cf[1].hx; c2.hy += cf[1].hy; c2.hz += cf[1].hz;
                    c2.tx += cf[1].tx; c2.ty += cf[1].ty; c2.tz += cf[1].tz;
                    reduce_forces(a, c2);
                } else {
                    reduce_forces(a, cf[0]);
                    reduce_forces(a, cf[1]);
                }
            }
        } else {
            // one cell at a time with the one-cell step; the stage is released after both reads.  The
            // collision form is the one-cell kernel's: PSC when any cell of the x-block (this warp's lanes
            // 0-15 or 16-31, both cells of each) is owned and updated
            const uint32_t ab = LINK_SKIP | LINK_DEFER;
            const bool owned = (inb && !(lk0 & ab) && key0) || (inb && !(lk1 & ab) && key1);
            const unsigned owners = __ballot_sync(0xffffffffu, owned);
            const int psc_block = (owners & ((threadIdx.x & 16u) ? 0xFFFF0000u : 0x0000FFFFu)) != 0u;
#pragma unroll 1
            for (int c = 0; c < 2; ++c) {
                const int x = x0 + c;
                const int xx = inb ? x : 0;
                const int xm = xx == 0 ? nx - 1 : xx - 1, xp = xx == nx - 1 ? 0 : xx + 1;
                T raw[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) raw[q] = sf[q * spe + (cx(q) == 1 ? xm : (cx(q) == -1 ? xp : xx))];
                float aux[5] = {0.f, 0.f, 0.f, 0.f, a.omega0};
                if (SMAG == LBDEM_SMAG_REFERENCE) {
                    const T *ap = sa + xslot((uint32_t)xx, AB);
#pragma unroll
                    for (int kk = 0; kk < 5; ++kk) aux[kk] = aux_dec<T>(ap[kk * 32]);
                }
                if (c == 1) {
                    __syncwarp();
                    if ((threadIdx.x & 31u) == 0) mbar_arrive(smem_u32(&empty[st]));
                }
                const uint32_t cl = (uint32_t)r * (uint32_t)nx + (uint32_t)xx;
                const uint32_t own = (uint32_t)r * a.rs + xslot((uint32_t)xx, QB);
                const uint32_t aown = (uint32_t)r * a.ars + xslot((uint32_t)xx, AB);
                step_cell<T, true, SMAG, WRAP, false, false, LAG_STORE>(a, x, y, z, inb, cl, own, aown, raw, aux, c ? key1 : key0,
                                                      c ? lk1 : lk0, psc_block);
            }
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
    const uint32_t row = (uint32_t)(z * ny + y);
    const uint32_t cell = row * (uint32_t)nx + (uint32_t)x;
    const uint32_t lk = a.links[cell];
    if (lk & (LINK_SKIP | LINK_DEFER)) return;   // deferred cells: the boundary pass
    const T *src = static_cast<const T *>(a.src);
    T *dst = static_cast<T *>(a.dst);
    const uint32_t rs = a.rs;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
    const uint32_t own = row * rs + xslot((uint32_t)x, QB);
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        T v;
        if (q != 0 && (lk & LINK_BB(q))) {
            v = src[own + qinv(q) * 32];
            if ((lk & LINK_MOVING) && (a.moving[cell] & LINK_BB(q))) {
                // velocity link (lbm_solver3d.py:222-229)
                const int xs = cx(q) == 1 ? xm : (cx(q) == -1 ? xp : x);
                const int ys = cy(q) == 1 ? ym : (cy(q) == -1 ? yp : y);
                const int zs = cz(q) == 1 ? zm : (cz(q) == -1 ? zp : z);
                const size_t n = ((size_t)zs * ny + ys) * nx + xs;
                const float cu = cx(q) * vel_out[n] + cy(q) * vel_out[nc + n] + cz(q) * vel_out[2 * nc + n];
                // wall: the cell's lagged density; Ladd inlet: the inlet's (:225-229)
                const float r = (a.links[n] & LINK_INLET) ? rho_out[n] : rho_out[cell];
                const float d = Store<T>::dec(v, wq(q) * a.dec) + 6.f * wq(q) * r * cu;
                v = Store<T>::enc(d, a.enc / wq(q));
            }
        } else {
            const int xs = cx(q) == 1 ? xm : (cx(q) == -1 ? xp : x);
            const int ys = cy(q) == 1 ? ym : (cy(q) == -1 ? yp : y);
            const int zs = cz(q) == 1 ? zm : (cz(q) == -1 ? zp : z);
            v = src[(uint32_t)(zs * ny + ys) * rs + xslot((uint32_t)xs, QB) + q * 32];
        }
        dst[own + q * 32] = v;
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

// ---------------------------------------------------------------------------
// Boundary pass: cells with a wet-node rule (Zou-He velocity / pressure,
// convective exit, Ladd inlet; lbm_solver3d.py:242-250) or a free-slip
// neighbour, one thread per listed cell, after the main kernel of a step or
// stream call.  First-pass cells (Zou-He, free slip) only read the previous
// post-collision populations; second-pass cells (exits, inlets) read the
// moments that the main kernel and the first pass stored for their interior
// neighbours.
// ---------------------------------------------------------------------------
enum { BND_GATHER = 0, BND_LOCAL = 1, BND_STREAM = 2 };

__device__ __forceinline__ int comp(int q, int axis) { return axis == 0 ? cx(q) : (axis == 1 ? cy(q) : cz(q)); }

// Post-stream populations of one cell with every neighbour rule of the
// stream's first pass (lbm_solver3d.py:207-236; periodic wrap :308-342):
// propagation, bounce-back, moving wall / Ladd inlet, specular free slip.
// Directions in `unknown` (bit q) are left at zero: a wet-node rule overwrites them.
template <typename T>
__device__ __forceinline__ void gather_general(const StepArgs &a, int x, int y, int z, uint32_t cell, uint32_t lk,
                                               uint32_t unknown, float h[Q]) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t nc = a.nc;
    const T *src = static_cast<const T *>(a.src);
    const uint32_t rs = a.rs;
    auto slot = [&](int xx, int yy, int zz) { return (uint32_t)(zz * ny + yy) * rs + xslot((uint32_t)xx, QB); };
    const uint32_t own = slot(x, y, z);
    const int32_t prop = LBDEM_CT_FLUID | LBDEM_CT_VEL_ZOUHE | LBDEM_CT_VEL_EXIT | LBDEM_CT_PRE_ZOUHE;
    h[0] = Store<T>::widen(src[own]);
    if (!(lk & LINK_SLIP_NB)) {
        // no free-slip neighbour: the link mask holds every rule (as in the main kernel)
        const uint32_t mv = (lk & LINK_MOVING) ? a.moving[cell] : 0u;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            h[q] = 0.f;
            if (unknown & (1u << q)) continue;
            int xn = x - cx(q), yn = y - cy(q), zn = z - cz(q);
            xn = xn >= nx ? 0 : (xn < 0 ? nx - 1 : xn);
            yn = yn >= ny ? 0 : (yn < 0 ? ny - 1 : yn);
            zn = zn >= nz ? 0 : (zn < 0 ? nz - 1 : zn);
            if (lk & LINK_BB(q)) {
                float v = Store<T>::widen(src[own + qinv(q) * 32]);
                if (mv & LINK_BB(q)) {
                    const size_t n = ((size_t)zn * ny + yn) * nx + xn;
                    const float r = (a.links[n] & LINK_INLET) ? a.rho[n] : a.rho[cell];
                    const float cu = cx(q) * a.vel[n] + cy(q) * a.vel[nc + n] + cz(q) * a.vel[2 * nc + n];
                    v += 6.f * a.S * r * cu;
                }
                h[q] = v;
            } else {
                h[q] = Store<T>::widen(src[slot(xn, yn, zn) + q * 32]);
            }
        }
        return;
    }
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        h[q] = 0.f;
        if (unknown & (1u << q)) continue;
        int xn = x - cx(q), yn = y - cy(q), zn = z - cz(q);
        xn = xn >= nx ? 0 : (xn < 0 ? nx - 1 : xn);
        yn = yn >= ny ? 0 : (yn < 0 ? ny - 1 : yn);
        zn = zn >= nz ? 0 : (zn < 0 ? nz - 1 : zn);
        const size_t n = ((size_t)zn * ny + yn) * nx + xn;
        const int32_t ctn = a.ct[n];
        float v;
        if (ctn & prop) {
            v = Store<T>::widen(src[slot(xn, yn, zn) + q * 32]);
        } else if (ctn & LBDEM_CT_OBSTACLE) {
            v = Store<T>::widen(src[own + qinv(q) * 32]);
        } else if (ctn & (LBDEM_CT_VEL_LADD | LBDEM_CT_VEL_INLET_LADD)) {
            const float r = (ctn & LBDEM_CT_VEL_LADD) ? a.rho[cell] : a.rho[n];
            const float cu = cx(q) * a.vel[n] + cy(q) * a.vel[nc + n] + cz(q) * a.vel[2 * nc + n];
            v = Store<T>::widen(src[own + qinv(q) * 32]) + 6.f * a.S * r * cu;
        } else if ((ctn & LBDEM_CT_FREE_SLIP) && (ctn & (LBDEM_CT_LEFT | LBDEM_CT_RIGHT))) {
            v = Store<T>::widen(src[slot(x, yn, zn) + qmirror(q, 0) * 32]);
        } else if ((ctn & LBDEM_CT_FREE_SLIP) && (ctn & (LBDEM_CT_BOTTOM | LBDEM_CT_TOP))) {
            v = Store<T>::widen(src[slot(xn, y, zn) + qmirror(q, 1) * 32]);
        } else if ((ctn & LBDEM_CT_FREE_SLIP) && (ctn & (LBDEM_CT_BACK | LBDEM_CT_FRONT))) {
            v = Store<T>::widen(src[slot(xn, yn, z) + qmirror(q, 2) * 32]);
        } else {
            v = Store<T>::widen(src[slot(xn, yn, zn) + q * 32]);   // same as the main kernel
        }
        h[q] = v;
    }
}

// Zou-He non-equilibrium bounce-back (vel_zouHe, lbm_solver3d.py:671-821;
// pre_zouHe, :823-960) on the h form, written once for the six faces.  With
// d = f - w = h w / S, K the directions with c_a = 0 and O those leaving the
// domain (c_a = -s), using sum_K w + 2 sum_O w = 1:
//   velocity: rho = (1 + sum_K d + 2 sum_O d) / (1 - s u_a), u = stored velocity
//   pressure: rho stored, u_a = s (rho - 1 - sum_K d - 2 sum_O d) / rho, and the
//             unknowns use u = u_a e_a only (no tangential term)
//   N_b = 1/2 sum_K c_b d - [velocity] rho u_b / 3
//   unknown q (c_a = s): d_q = d_qbar + rho (c_q.u) / 3 (axis), + rho (c_q.u) / 6 - c_qb N_b (diagonal),
// i.e. h_q = h_qbar + 6 S rho (c_q.u) [- 36 S c_qb N_b].  Returns the (rho, u)
// the reference's collision then uses; false for a cell without a face bit
// (the reference leaves it untouched).
__device__ __forceinline__ bool zou_he(const StepArgs &a, int32_t ct, bool pressure, float h[Q], float &rho,
                                       float u[3]) {
    int ax, s;
    if (!face_of(ct, ax, s)) return false;
    // scalars selected by the runtime axis (no runtime-indexed local arrays)
    float Dk = 0.f, Do = 0.f, T0 = 0.f, T1 = 0.f, T2 = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float d = h[q] * (wq(q) * a.dec);
        const int ca = comp(q, ax);
        if (ca == 0) {
            Dk += d;
            T0 += (float)cx(q) * d;
            T1 += (float)cy(q) * d;
            T2 += (float)cz(q) * d;
        } else if (ca == -s) {
            Do += d;
        }
    }
    const float fs = (float)s;
    float u0 = u[0], u1 = u[1], u2 = u[2];
    float w0, w1, w2;   // velocity entering the unknowns
    if (pressure) {
        const float un = fs * ((rho - 1.f) - Dk - 2.f * Do) / rho;
        if (ax == 0) u0 = un; else if (ax == 1) u1 = un; else u2 = un;
        w0 = ax == 0 ? un : 0.f;
        w1 = ax == 1 ? un : 0.f;
        w2 = ax == 2 ? un : 0.f;
    } else {
        const float ua = ax == 0 ? u0 : (ax == 1 ? u1 : u2);
        rho = (1.f + Dk + 2.f * Do) / (1.f - fs * ua);
        w0 = u0; w1 = u1; w2 = u2;
    }
    u[0] = u0; u[1] = u1; u[2] = u2;
    const float k3 = pressure ? 0.f : rho * (1.f / 3.f);
    const float N0 = 0.5f * T0 - k3 * w0, N1 = 0.5f * T1 - k3 * w1, N2 = 0.5f * T2 - k3 * w2;
    const float k6 = 6.f * a.S * rho, k36 = 36.f * a.S;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        if (comp(q, ax) != s) continue;
        const float cu = (float)cx(q) * w0 + (float)cy(q) * w1 + (float)cz(q) * w2;
        // the tangential component of a diagonal unknown (zero on the axis direction)
        const float corr = (ax != 0 ? (float)cx(q) * N0 : 0.f) + (ax != 1 ? (float)cy(q) * N1 : 0.f) +
                           (ax != 2 ? (float)cz(q) * N2 : 0.f);
        h[q] = h[qinv(q)] + k6 * cu - k36 * corr;
    }
    return true;
}

template <typename T, int SMAG, int MODE>
__global__ void __launch_bounds__(128) k_boundary(const StepArgs a, const uint32_t *__restrict__ cells, uint32_t n) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = t < n;
    const uint32_t cell = cells[valid ? t : 0];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t nc = a.nc;
    const int x = (int)(cell % (uint32_t)nx), y = (int)((cell / (uint32_t)nx) % (uint32_t)ny);
    const int z = (int)(cell / ((uint32_t)nx * (uint32_t)ny));
    const uint32_t row = cell / (uint32_t)nx;
    const uint32_t own = row * a.rs + xslot((uint32_t)x, QB);
    const uint32_t aown = row * a.ars + xslot((uint32_t)x, AB);
    const int32_t ct = a.ct[cell];
    const uint32_t lk = a.links[cell];
    const int rule = (lk & LINK_INLET) ? WET_INLET : wet_rule(ct);
    const T *src = static_cast<const T *>(a.src);
    T *dst = static_cast<T *>(a.dst);
    float h[Q];
    float rho = a.rho[cell];
    float u[3] = {a.vel[cell], a.vel[nc + cell], a.vel[2 * nc + cell]};
    float aux[5] = {0.f, 0.f, 0.f, 0.f, a.omega0};
    if (a.aux != nullptr) {
#pragma unroll
        for (int k = 0; k < 5; ++k) aux[k] = lag_ld<T>(a, aown, k * 32);
    }
    // interior neighbour of a face cell (no periodic wrap, lbm_solver3d.py:522-527, 647-658)
    int ax = 0, s = 0;
    size_t nbr = cell;
    if (face_of(ct, ax, s)) {
        const int mx = ax == 0 ? min(max(x + s, 0), nx - 1) : x;
        const int my = ax == 1 ? min(max(y + s, 0), ny - 1) : y;
        const int mz = ax == 2 ? min(max(z + s, 0), nz - 1) : z;
        nbr = ((size_t)mz * ny + my) * nx + mx;
    }
    bool fields = false;   // (rho, u) come from the rule or the stored fields, not the moments
    bool collide_it = true;
    if (rule == WET_INLET) {
        // The inlet's populations f never stream (the first pass skips it) but it
        // collides, and a free-slip mirror may read its post-collision ones: f
        // lives in the step's dst slot (gather) or src slot (post-stream input),
        // the post-collision populations in the other buffer.  Its density
        // follows the interior neighbour's (bc_ladd_inlet).
        // f: from the post-stream buffer in a step that reads populations in
        // place (first step after initialize / a host read; also captured into
        // bnd_f0), else from bnd_f0 (t - first second-pass index = row in bnd_f0)
        const uint32_t tb = t >= a.bnd_nb ? 0u : t;
        T *f0 = static_cast<T *>(a.bnd_f0);
        if (MODE == BND_LOCAL) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                h[q] = Store<T>::widen(src[own + q * 32]);
                if (valid) f0[(size_t)q * a.bnd_nb + tb] = src[own + q * 32];
            }
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) h[q] = Store<T>::widen(f0[(size_t)q * a.bnd_nb + tb]);
        }
        if (MODE != BND_LOCAL) {
            rho = a.rho[nbr];
            if (valid) a.rho[cell] = rho;
        }
        fields = true;
        collide_it = !(lk & LINK_MAP_SKIP);
    } else if (rule == WET_EXIT && MODE != BND_LOCAL) {
        // bc_vel_exit: u of the interior neighbour, rho = 1, f = feq (which is also
        // the equilibrium the next Smagorinsky / stress evaluation lags on)
        u[0] = a.vel[nbr]; u[1] = a.vel[nc + nbr]; u[2] = a.vel[2 * nc + nbr];
        rho = 1.f;
        if (valid) {
            a.rho[cell] = 1.f;
            a.vel[cell] = u[0]; a.vel[nc + cell] = u[1]; a.vel[2 * nc + cell] = u[2];
        }
        const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float cu = cx(q) * u[0] + cy(q) * u[1] + cz(q) * u[2];
            h[q] = a.S * (3.f * cu + 4.5f * cu * cu - 1.5f * usq);
        }
        aux[0] = 0.f; aux[1] = u[0]; aux[2] = u[1]; aux[3] = u[2];
        fields = true;
    } else if (MODE != BND_LOCAL) {
        uint32_t unknown = 0u;
        if ((rule == WET_VEL_ZOUHE || rule == WET_PRE_ZOUHE) && s != 0) {
#pragma unroll
            for (int q = 1; q < Q; ++q)
                if (comp(q, ax) == s) unknown |= 1u << q;
        }
        gather_general<T>(a, x, y, z, cell, lk, unknown, h);
        if (rule == WET_VEL_ZOUHE || rule == WET_PRE_ZOUHE) {
            const bool pressure = rule == WET_PRE_ZOUHE;
            if (zou_he(a, ct, pressure, h, rho, u) && valid) {
                if (pressure) a.vel[(size_t)ax * nc + cell] = ax == 0 ? u[0] : (ax == 1 ? u[1] : u[2]);
                else a.rho[cell] = rho;
            }
            fields = true;
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) h[q] = Store<T>::widen(src[own + q * 32]);
        fields = rule != WET_NONE;
    }
    if (!fields) {
        // free-slip neighbour without a wet-node rule: moments as the first pass
        // (MODE != BND_STREAM for inlets: an inlet always has fields set)
        float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float d = h[q] * (wq(q) * a.dec);
            dr += d; jx += cx(q) * d; jy += cy(q) * d; jz += cz(q) * d;
        }
        rho = 1.f + dr;
        u[0] = jx / rho; u[1] = jy / rho; u[2] = jz / rho;
        if (MODE != BND_LOCAL && valid && (lk & LINK_FLUID)) {
            a.rho[cell] = rho;
            a.vel[cell] = u[0]; a.vel[nc + cell] = u[1]; a.vel[2 * nc + cell] = u[2];
        }
    }
    if (MODE == BND_STREAM) {
        // an inlet's post-stream populations are its constant f
        if (valid && (rule != WET_INLET || !(lk & LINK_MAP_SKIP))) {
#pragma unroll
            for (int q = 0; q < Q; ++q) dst[own + q * 32] = Store<T>::narrow(h[q]);
            if (rule == WET_EXIT && a.aux != nullptr) {
#pragma unroll
                for (int k = 0; k < 4; ++k) lag_st<T>(a, aown, k * 32, aux[k]);
            }
        }
        return;
    }
    const bool act = valid && collide_it;
    uint32_t key = (a.key != nullptr && act) ? a.key[cell] : 0u;
    const bool psc = a.key != nullptr && __any_sync(0xffffffffu, key != 0u);
    CellForce cf[1];
    const bool acts[1] = {act};
    const int xs[1] = {x};
    const uint32_t keys[1] = {key};
    const float epss[1] = {(a.eps != nullptr && key) ? a.eps[cell] : 0.f};
    const float ovr[4] = {rho, u[0], u[1], u[2]};
    float hout[Q];
    collide<float, SMAG, true, true>(
        a, h, acts, xs, y, z, aux, psc, keys, epss, cf, [&](int q, float v) { hout[q] = v; },
        [&](int k, float v) { aux[k] = v; }, [](float, float, float, float) {}, ovr);
    // an inlet's post-collision populations are read only by free-slip mirrors
    if (act && (rule != WET_INLET || a.slip)) {
#pragma unroll
        for (int q = 0; q < Q; ++q) dst[own + q * 32] = Store<T>::narrow(hout[q]);
    }
    if (act) {
        if (SMAG == LBDEM_SMAG_REFERENCE || a.keep_lag) {
#pragma unroll
            for (int k = 0; k < 5; ++k) lag_st<T>(a, aown, k * 32, aux[k]);
        }
        if (a.hydro_out) {
            a.hydro_out[cell] = cf[0].hx;
            a.hydro_out[nc + cell] = cf[0].hy;
            a.hydro_out[2 * nc + cell] = cf[0].hz;
        }
    }
    if (psc) reduce_forces(a, cf[0]);
}

// f = feq(rho, u) (initialize, psclattice3d.py:60-75)
template <typename T>
__global__ void k_init(const StepArgs a, const float *rho_in, const float *vel_in, int smag_ref, void *other) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const size_t nc = a.nc;
    const uint32_t row = (uint32_t)(z * a.ny + y);
    const uint32_t c = row * (uint32_t)a.nx + (uint32_t)x;
    T *dst = static_cast<T *>(a.dst) + (row * a.rs + xslot((uint32_t)x, QB));
    // initialize() skips the map's skip set: OBSTACLE / VEL_LADD / FREE_SLIP, and
    // Ladd inlets where the lattice skips them (lbm_solver3d.py:163, psclattice3d.py:66).
    // No collision ever writes those cells, so they keep the reference's
    // zero-initialised populations, f = 0, in both buffers (a free-slip mirror
    // can read them, lbm_solver3d.py:230-236).
    const bool skip = (a.links[c] & LINK_MAP_SKIP) != 0;
    const float rho = skip ? 1.f : rho_in[c];
    const float ux = skip ? 0.f : vel_in[c], uy = skip ? 0.f : vel_in[nc + c], uz = skip ? 0.f : vel_in[2 * nc + c];
    const float drho = rho - 1.f;
    const float usq = ux * ux + uy * uy + uz * uz;
    if (skip) {
        T *o = static_cast<T *>(other) + (row * a.rs + xslot((uint32_t)x, QB));
#pragma unroll
        for (int q = 0; q < Q; ++q) dst[q * 32] = o[q * 32] = Store<T>::narrow(-a.S);
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float cu = cx(q) * ux + cy(q) * uy + cz(q) * uz;
            const float fe = wq(q) * (drho + rho * (3.f * cu + 4.5f * cu * cu - 1.5f * usq));
            dst[q * 32] = Store<T>::enc(fe, a.enc / wq(q));
        }
    }
    if (smag_ref) {
        const uint32_t ax = row * a.ars + xslot((uint32_t)x, AB);
        lag_st<T>(a, ax, 0, drho);
        lag_st<T>(a, ax, 32, ux);
        lag_st<T>(a, ax, 64, uy);
        lag_st<T>(a, ax, 96, uz);
        lag_st<T>(a, ax, 128, a.omega0);
    }
}

// link masks from CellType (lbm_solver3d.py:203-250): bounce-back bit q when
// the neighbour x - c_q is OBSTACLE, a moving wall (VEL_LADD) or a Ladd inlet
// (VEL_INLET_LADD); for the latter two also bit q of moving[] and LINK_MOVING.
// Cells with a wet-node rule or a free-slip neighbour are deferred to the
// boundary pass; the interior neighbour of an exit or inlet keeps its moments.
__global__ void k_links(const int32_t *ct, int nx, int ny, int nz, int skip_inlet, uint32_t *links, uint32_t *moving) {
    const size_t nc = (size_t)nx * ny * nz;
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((size_t)nx * ny));
    const int32_t own = ct[c];
    uint32_t L = 0, M = 0;
    const int32_t walls = LBDEM_CT_OBSTACLE | LBDEM_CT_VEL_LADD | LBDEM_CT_FREE_SLIP;
    const bool sskip = (own & (walls | LBDEM_CT_VEL_INLET_LADD)) != 0;
    if (sskip) L |= LINK_SKIP;
    int32_t mskip = walls;
    if (skip_inlet) mskip |= LBDEM_CT_VEL_INLET_LADD;
    if (own & mskip) L |= LINK_MAP_SKIP;
    if (own & LBDEM_CT_FLUID) L |= LINK_FLUID;
    if (own & LBDEM_CT_VEL_INLET_LADD) L |= LINK_INLET;
    const int rule = wet_rule(own);
    if (rule == WET_INLET && !(own & walls)) L |= LINK_DEFER | LINK_PHASE_B;
    if (!sskip && rule != WET_NONE) L |= LINK_DEFER | (rule == WET_EXIT ? LINK_PHASE_B : 0u);
    const int32_t prop = LBDEM_CT_FLUID | LBDEM_CT_VEL_ZOUHE | LBDEM_CT_VEL_EXIT | LBDEM_CT_PRE_ZOUHE;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        int xn = x - cx(q), yn = y - cy(q), zn = z - cz(q);
        xn = xn >= nx ? 0 : (xn < 0 ? nx - 1 : xn);
        yn = yn >= ny ? 0 : (yn < 0 ? ny - 1 : yn);
        zn = zn >= nz ? 0 : (zn < 0 ? nz - 1 : zn);
        const int32_t ctn = ct[((size_t)zn * ny + yn) * nx + xn];
        if (ctn & prop) continue;
        if (ctn & LBDEM_CT_OBSTACLE) {
            L |= LINK_BB(q);
        } else if (ctn & (LBDEM_CT_VEL_LADD | LBDEM_CT_VEL_INLET_LADD)) {
            L |= LINK_BB(q) | LINK_MOVING;
            M |= LINK_BB(q);
        } else if ((ctn & LBDEM_CT_FREE_SLIP) && !sskip) {
            L |= LINK_DEFER | LINK_SLIP_NB;
        }
    }
    // interior neighbour of an exit / inlet face cell (the face's +s side;
    // the reference reads it without periodic wrap, lbm_solver3d.py:522-527, 647-658)
    if (!(L & LINK_DEFER) && !sskip) {
        const int p[3] = {x, y, z}, n[3] = {nx, ny, nz};
        for (int a = 0; a < 3; ++a)
            for (int s = -1; s <= 1; s += 2) {
                int m[3] = {p[0], p[1], p[2]};
                m[a] -= s;   // candidate boundary cell whose interior neighbour (at +s) is this cell
                if (m[a] < 0 || m[a] >= n[a]) continue;
                const int32_t cm = ct[((size_t)m[2] * ny + m[1]) * nx + m[0]];
                const int r = wet_rule(cm);
                int fa, fs;
                if ((r == WET_EXIT || r == WET_INLET) && face_of(cm, fa, fs) && fa == a && fs == s) L |= LINK_KEEP;
            }
    }
    links[c] = L;
    if (moving) moving[c] = M;
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
    const float eps = a.eps ? a.eps[c] : ((key & KEY_FULL) ? 1.f : (float)key_count(key) * (1.f / 125.f));
    const uint32_t row = (uint32_t)(c / (size_t)a.nx), xx = (uint32_t)(c % (size_t)a.nx);
    const float om = smag_ref ? lag_ld<T>(a, row * a.ars + xslot(xx, AB), 4 * 32) : a.omega0;
    const float taum = 1.f / om - 0.5f;
    id[c] = gid;
    volfrac[c] = eps;
    weight[c] = eps * taum / ((1.f - eps) + taum);
    const float4 t0 = a.table[4 * gid + 0], t1 = a.table[4 * gid + 1];
    const float4 t2 = a.table[4 * gid + 2], t3 = a.table[4 * gid + 3];
    // integer part first (exact), then the fractional centre: image cells round
    // as interior ones; the minimum image only when the map has periodic images
    float ix = (float)x - t0.x, iy = (float)y - t0.y, iz = (float)z - t0.z;
    if (a.wrap_any) {
        ix = min_image(ix, a.per_x, a.iper_x);
        iy = min_image(iy, a.per_y, a.iper_y);
        iz = min_image(iz, a.per_z, a.iper_z);
    }
    const float rx = ix - t1.x, ry = iy - t1.y, rz = iz - t1.z;
    velsolid[c] = t2.x + (t3.y * rz - t3.z * ry);
    velsolid[nc + c] = t2.y + (t3.z * rx - t3.x * rz);
    velsolid[2 * nc + c] = t2.z + (t3.x * ry - t3.y * rx);
}

// FP64 totals (deterministic two-pass block reduction, no atomics)
template <typename T>
__global__ void __launch_bounds__(256) k_sums(const StepArgs a, double *partials) {
    const size_t nc = a.nc;
    double m = 0, px = 0, py = 0, pz = 0;
    const T *f = static_cast<const T *>(a.src);
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (a.links[c] & LINK_SKIP) continue;
        const uint32_t row = (uint32_t)(c / (size_t)a.nx), x = (uint32_t)(c % (size_t)a.nx);
        const T *p = f + (row * a.rs + xslot(x, QB));
        float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float dq = Store<T>::dec(p[q * 32], wq(q) * a.dec);
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

// Stress diagnostics (compute_stress, lbm_solver3d.py:347-404) from the
// post-stream populations and the lagged state of the last collision:
// sigma = -(1 - omega/2) (sum c c (f - w) - (drho cs^2 delta + rho u u)),
// out: 7 planes of Ncells (xx, yy, zz, xy, xz, yz, von Mises shear
// magnitude); skipped cells are not written.
template <typename T>
__global__ void __launch_bounds__(256) k_stress(const StepArgs a, float *out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const uint32_t row = (uint32_t)(z * a.ny + y);
    const uint32_t cell = row * (uint32_t)a.nx + (uint32_t)x;
    const uint32_t lk = a.links[cell];
    if (lk & LINK_SKIP) return;
    const T *p = static_cast<const T *>(a.src) + (row * a.rs + xslot((uint32_t)x, QB));
    float sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        const float d = Store<T>::dec(p[q * 32], wq(q) * a.dec);
        if (cx(q)) sxx += d;
        if (cy(q)) syy += d;
        if (cz(q)) szz += d;
        if (cx(q) * cy(q)) sxy += (float)(cx(q) * cy(q)) * d;
        if (cx(q) * cz(q)) sxz += (float)(cx(q) * cz(q)) * d;
        if (cy(q) * cz(q)) syz += (float)(cy(q) * cz(q)) * d;
    }
    const uint32_t ap = row * a.ars + xslot((uint32_t)x, AB);
    const float dr = lag_ld<T>(a, ap, 0), ux = lag_ld<T>(a, ap, 32), uy = lag_ld<T>(a, ap, 64), uz = lag_ld<T>(a, ap, 96);
    const float om = lag_ld<T>(a, ap, 128);
    const float rho = 1.f + dr, ecs = dr * CS2;
    const float k = -(1.f - 0.5f * om);
    const size_t nc = a.nc;
    const float txy = k * (sxy - rho * ux * uy), txz = k * (sxz - rho * ux * uz), tyz = k * (syz - rho * uy * uz);
    out[cell] = k * (sxx - (ecs + rho * ux * ux));
    out[nc + cell] = k * (syy - (ecs + rho * uy * uy));
    out[2 * nc + cell] = k * (szz - (ecs + rho * uz * uz));
    out[3 * nc + cell] = txy;
    out[4 * nc + cell] = txz;
    out[5 * nc + cell] = tyz;
    out[6 * nc + cell] = sqrtf(0.5f * (txy * txy + txz * txz + tyz * tyz));
}

// Boundary-pass cell list in lattice order: per-row counts (one warp per
// row), one block's exclusive scan over the rows, then an ordered fill.
__global__ void k_bnd_count(const uint32_t *links, int nx, int nrows, int32_t *cnt) {
    const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= nrows) return;
    int na = 0, nb = 0;
    for (int x0 = 0; x0 < nx; x0 += 32) {
        const int x = x0 + lane;
        const uint32_t L = x < nx ? links[(size_t)row * nx + x] : 0u;
        na += __popc(__ballot_sync(0xffffffffu, (L & LINK_DEFER) && !(L & LINK_PHASE_B)));
        nb += __popc(__ballot_sync(0xffffffffu, (L & LINK_DEFER) && (L & LINK_PHASE_B)));
    }
    if (lane == 0) {
        cnt[row] = na;
        cnt[nrows + row] = nb;
    }
}

__global__ void __launch_bounds__(1024) k_bnd_scan(int32_t *cnt, int nrows, uint32_t *counts) {
    __shared__ int32_t sh[1024];
    const int t = threadIdx.x;
    for (int part = 0; part < 2; ++part) {
        int32_t *c = cnt + (size_t)part * nrows;
        int32_t carry = 0;
        for (int base = 0; base < nrows; base += 1024) {
            const int i = base + t;
            const int32_t v = i < nrows ? c[i] : 0;
            sh[t] = v;
            __syncthreads();
            for (int o = 1; o < 1024; o <<= 1) {
                const int32_t add = t >= o ? sh[t - o] : 0;
                __syncthreads();
                sh[t] += add;
                __syncthreads();
            }
            if (i < nrows) c[i] = carry + sh[t] - v;
            const int32_t tot = sh[1023];
            __syncthreads();
            carry += tot;
        }
        if (t == 0) counts[part] = (uint32_t)carry;
    }
}

__global__ void k_bnd_fill(const uint32_t *links, int nx, int nrows, const int32_t *off, const uint32_t *counts,
                           uint32_t *cells, uint32_t cap) {
    const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= nrows) return;
    uint32_t pa = (uint32_t)off[row], pb = counts[0] + (uint32_t)off[nrows + row];
    const uint32_t below = (1u << lane) - 1u;
    for (int x0 = 0; x0 < nx; x0 += 32) {
        const int x = x0 + lane;
        const uint32_t L = x < nx ? links[(size_t)row * nx + x] : 0u;
        const bool fa = (L & LINK_DEFER) && !(L & LINK_PHASE_B), fb = (L & LINK_DEFER) && (L & LINK_PHASE_B);
        const uint32_t ma = __ballot_sync(0xffffffffu, fa), mb = __ballot_sync(0xffffffffu, fb);
        const uint32_t c = (uint32_t)row * (uint32_t)nx + (uint32_t)x;
        if (fa) {
            const uint32_t i = pa + __popc(ma & below);
            if (i < cap) cells[i] = c;
        }
        if (fb) {
            const uint32_t i = pb + __popc(mb & below);
            if (i < cap) cells[i] = c;
        }
        pa += __popc(ma);
        pb += __popc(mb);
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
    const size_t nb = ((size_t)L->nx + 31) / 32;
    if (nb * 32 * L->ny * L->nz * Q >= (1ull << 32)) {
        set_error("lattice has %zu cells (%zu with x padded to 32); element offsets are 32-bit, so at most %llu "
                  "padded cells are supported",
                  (size_t)L->nx * L->ny * L->nz, nb * 32 * L->ny * L->nz, (unsigned long long)((1ull << 32) / Q - 1));
        return LBDEM_ERR_ARG;
    }
    memset(&a, 0, sizeof(a));
    a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.nc = (size_t)L->nx * L->ny * L->nz;
    a.nb = (uint32_t)nb;
    a.rs = (uint32_t)nb * QB;
    a.ars = (uint32_t)nb * AB;
    a.omega0 = L->omega0;
    a.inv_omega0 = 1.f / L->omega0;
    a.smag_k = 4.5f * L->smag_cs * L->smag_cs;
    float S = 1.f;
    if (L->storage != LBDEM_F32) {
        if (!(L->scale16 > 0.f)) {
            set_error("scale16 must be positive for 16-bit storage");
            return LBDEM_ERR_ARG;
        }
        S = L->scale16;
    }
    a.S = S;
    a.dec = 1.f / S;
    a.enc = S;
    a.W0 = (1.f / 3.f) / S;
    a.W1 = (1.f / 18.f) / S;
    a.W2 = (1.f / 36.f) / S;
    if (L->force_on) {
        a.g3x = 3.f * S * L->force[0];
        a.g3y = 3.f * S * L->force[1];
        a.g3z = 3.f * S * L->force[2];
    }
    a.aux = L->aux;
    a.keep_lag = L->aux != nullptr;
    if (L->aux_half != 0 && L->aux_half != 1) {
        set_error("aux_half must be 0 or 1");
        return LBDEM_ERR_ARG;
    }
    if (L->aux_half && L->storage != LBDEM_F32) {
        set_error("aux_half applies to FP32 storage (the 16-bit forms keep the lagged state in their own type)");
        return LBDEM_ERR_ARG;
    }
    a.aux16 = L->aux_half;
    a.links = L->links;
    a.links_all = L->links_all;
    a.moving = L->moving;
    a.rho = L->rho;
    a.vel = L->vel;
    a.status = L->status;
    if (!a.links || !a.status) {
        set_error("links and status are required");
        return LBDEM_ERR_ARG;
    }
    if (L->smag_mode == LBDEM_SMAG_REFERENCE && !L->aux) {
        set_error("LBDEM_SMAG_REFERENCE needs the aux buffer");
        return LBDEM_ERR_ARG;
    }
    if (L->moving && (!L->rho || !L->vel)) {
        set_error("moving walls need the rho and vel fields");
        return LBDEM_ERR_ARG;
    }
    a.ct = L->ct;
    a.bnd_f0 = L->bnd_f0;
    a.bnd_nb = L->bnd_nb;
    a.slip = L->bnd_slip;
    if (L->bnd_na + L->bnd_nb > 0 && (!L->ct || !L->bnd_cells || !L->rho || !L->vel)) {
        set_error("open boundaries need ct, bnd_cells and the rho and vel fields");
        return LBDEM_ERR_ARG;
    }
    if (L->bnd_nb > 0 && !L->bnd_f0) {
        set_error("second-pass boundary cells need bnd_f0 (19 * bnd_nb elements)");
        return LBDEM_ERR_ARG;
    }
    return LBDEM_OK;
}

// Boundary pass of a step (MODE BND_GATHER / BND_LOCAL) or stream call
// (BND_STREAM): first-pass cells, then second-pass cells.
template <typename T, int SMAG, int MODE>
static void launch_boundary(const lbdem_lattice *L, const StepArgs &a, cudaStream_t st) {
    if (L->bnd_na > 0)
        k_boundary<T, SMAG, MODE><<<(L->bnd_na + 127) / 128, 128, 0, st>>>(a, L->bnd_cells, L->bnd_na);
    if (L->bnd_nb > 0)
        k_boundary<T, SMAG, MODE><<<(L->bnd_nb + 127) / 128, 128, 0, st>>>(a, L->bnd_cells + L->bnd_na,
                                                                            L->bnd_nb);
}

static void set_periods(StepArgs &a, const lbdem_psc *P) {
    a.per_x = P->wrap[0] ? (float)P->period[0] : 0.f;
    a.per_y = P->wrap[1] ? (float)P->period[1] : 0.f;
    a.per_z = P->wrap[2] ? (float)P->period[2] : 0.f;
    a.iper_x = a.per_x > 0.f ? 1.f / a.per_x : 0.f;
    a.iper_y = a.per_y > 0.f ? 1.f / a.per_y : 0.f;
    a.iper_z = a.per_z > 0.f ? 1.f / a.per_z : 0.f;
    a.wrap_any = a.per_x > 0.f || a.per_y > 0.f || a.per_z > 0.f;
}

static void step_geometry(const lbdem_lattice *L, dim3 &grid, dim3 &block, int nthreads = 256) {
    int bx = ((L->nx + 31) / 32) * 32;
    if (bx > nthreads) bx = nthreads;
    int by = nthreads / bx;
    if (by > L->ny) by = L->ny;
    block = dim3(bx, by, 1);
    grid = dim3((L->nx + bx - 1) / bx, (L->ny + by - 1) / by, L->nz);
}

// ---------------------------------------------------------------------------
// host side of the row-staged step
// ---------------------------------------------------------------------------
// cuTensorMapEncodeTiled from the driver, through the runtime (no link-time
// dependency on libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// Which form of the gathered full-lattice step runs: 0 per-thread gathers
// (k_psc_step), 1 row-staged one cell per thread, 2 row-staged two cells per
// thread.  By default the row-staged forms for 16-bit storage (two cells per
// thread where Nx is even) and k_psc_step for FP32 (the row-staged FP32 step
// fits only two CTAs per SM in shared memory and measured 30 % slower);
// LBDEM_STEP_KERNEL=simt, =rows or =rows2 in the environment at the call
// selects one form for every storage (=rows2 falls back to =rows where it
// does not apply).
template <typename T>
static int step_kernel_form() {
    const char *e = getenv("LBDEM_STEP_KERNEL");
    if (e && strcmp(e, "simt") == 0) return 0;
    if (e && strcmp(e, "rows") == 0) return 1;
    if (e && strcmp(e, "rows2") == 0) return 2;
    return sizeof(T) == 2 ? 2 : 0;
}

template <typename T> constexpr CUtensorMapDataType tmap_type();
template <> constexpr CUtensorMapDataType tmap_type<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> constexpr CUtensorMapDataType tmap_type<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }
template <> constexpr CUtensorMapDataType tmap_type<__nv_bfloat16>() { return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; }

static uint32_t round_up(uint32_t v, uint32_t m) { return (v + m - 1) / m * m; }

// the row-staged kernel of a form: two cells per thread exists for 16-bit storage only
template <typename T, int SMAG, bool WRAP, bool PAIRS> struct RowKernel {
    static auto fn() { return k_psc_step_rows<T, SMAG, WRAP>; }
};
template <int SMAG, bool WRAP> struct RowKernel<__half, SMAG, WRAP, true> {
    static auto fn() { return k_psc_step_rows2<__half, SMAG, WRAP>; }
};
template <int SMAG, bool WRAP> struct RowKernel<__nv_bfloat16, SMAG, WRAP, true> {
    static auto fn() { return k_psc_step_rows2<__nv_bfloat16, SMAG, WRAP>; }
};

constexpr int ROWS_NOT_APPLICABLE = -1;

// Launch the row-staged step; ROWS_NOT_APPLICABLE for rows wider than 256
// cells, with too little shared memory for two CTAs per SM, when the driver
// has no tensor-map encoder, or when a copy's description is refused -- the
// caller then launches k_psc_step.
template <typename T, int SMAG, bool WRAP, bool PAIRS>
static int launch_step_rows(const lbdem_lattice *L, const StepArgs &a, cudaStream_t st) {
    auto encode = tmap_encoder();
    // one thread per cell (PAIRS: per two cells) of a row: rows of up to
    // ROW_THREADS cells (a loop over wider rows costs registers the step does not have)
    if (!encode || 32u * a.nb > (uint32_t)ROW_THREADS || a.src == nullptr) return ROWS_NOT_APPLICABLE;
    // two cells per thread: 16-bit storage, even Nx, and an even number of x-blocks so that the 16 NB
    // consumer threads are whole warps (the producer warp then starts on a warp boundary)
    if (PAIRS && (sizeof(T) != 2 || (a.nx & 1) || (a.nb & 1u))) return ROWS_NOT_APPLICABLE;
    // the staged lagged-state rows and the stores have the storage type
    if (a.aux16) return ROWS_NOT_APPLICABLE;
    const uint32_t es = sizeof(T), nb = a.nb;
    RowMaps m;
    memset(&m, 0, sizeof(m));
    m.use_aux = SMAG == LBDEM_SMAG_REFERENCE;
    m.kl_tma = (a.nx % 4) == 0;
    m.kl_box = (int)round_up((uint32_t)a.nx, 4u);
    m.tx_bytes = Q * 32u * nb * es + (m.use_aux ? 5u * 32u * nb * es : 0u) +
                 (m.kl_tma ? (uint32_t)m.kl_box * 4u * ((a.key != nullptr ? 1u : 0u) + (a.links_all ? 0u : 1u)) : 0u);
    const uint32_t smem = ROW_STAGES * RowLayout<T>::stage;
    const cuuint64_t ny = (cuuint64_t)a.ny, nz = (cuuint64_t)a.nz;
    {
        const cuuint64_t dims[5] = {32, (cuuint64_t)Q, nb, ny, nz};
        const cuuint64_t strides[4] = {32ull * es, 32ull * Q * es, 32ull * Q * es * nb, 32ull * Q * es * nb * ny};
        const cuuint32_t box[5] = {32, 1, nb, 1, 1};
        const cuuint32_t one[5] = {1, 1, 1, 1, 1};
        if (encode(&m.f, tmap_type<T>(), 5, const_cast<void *>(a.src), dims, strides, box, one,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, ROW_L2_PROMOTION,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return ROWS_NOT_APPLICABLE;
    }
    if (m.use_aux) {
        const cuuint64_t dims[5] = {32, 5, nb, ny, nz};
        const cuuint64_t strides[4] = {32ull * es, 32ull * 5 * es, 32ull * 5 * es * nb, 32ull * 5 * es * nb * ny};
        const cuuint32_t box[5] = {32, 5, nb, 1, 1};
        const cuuint32_t one[5] = {1, 1, 1, 1, 1};
        if (!a.aux || encode(&m.aux, tmap_type<T>(), 5, a.aux, dims, strides, box, one,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, ROW_L2_PROMOTION,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return ROWS_NOT_APPLICABLE;
    }
    if (m.kl_tma) {
        const cuuint64_t dims[2] = {(cuuint64_t)a.nx, ny * nz};
        const cuuint64_t strides[1] = {(cuuint64_t)a.nx * 4ull};
        const cuuint32_t box[2] = {(cuuint32_t)m.kl_box, 1};
        const cuuint32_t one[2] = {1, 1};
        if (encode(&m.link, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint32_t *>(a.links), dims, strides, box,
                   one, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return ROWS_NOT_APPLICABLE;
        if (a.key && encode(&m.key, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint32_t *>(a.key), dims, strides,
                            box, one, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return ROWS_NOT_APPLICABLE;
    }
    auto kern = RowKernel<T, SMAG, WRAP, PAIRS>::fn();
    static uint32_t smem_set = 0;    // per instantiation
    if (smem > smem_set) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return ROWS_NOT_APPLICABLE;
        }
        smem_set = smem;
    }
    const int threads = (int)((PAIRS ? 16u : 32u) * nb) + 32;   // consumers + the producer warp
    int per_sm = 0, dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    {
        // SM count and resident CTAs per SM for this kernel and CTA size: constant per device,
        // looked up once (a few entries: CTA sizes differ only with the row width)
        static std::mutex mu;
        static int cache[8][4] = {};   // device, threads, nsm, per_sm
        static int ncache = 0;
        std::lock_guard<std::mutex> lock(mu);
        int e = 0;
        while (e < ncache && !(cache[e][0] == dev && cache[e][1] == threads)) ++e;
        if (e == ncache) {
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess) {
                cudaGetLastError();
                return ROWS_NOT_APPLICABLE;
            }
            if (ncache < 8) {
                cache[ncache][0] = dev;
                cache[ncache][1] = threads;
                cache[ncache][2] = nsm;
                cache[ncache][3] = per_sm;
                ++ncache;
            }
        } else {
            nsm = cache[e][2];
            per_sm = cache[e][3];
        }
    }
    if (per_sm < 2) return ROWS_NOT_APPLICABLE;
    const int nrows = a.ny * a.nz;
    const int grid = std::min(nrows, nsm * per_sm);
    kern<<<grid, threads, smem, st>>>(a, m);
    return check_launch("psc_step_rows");
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
        a.eps = P->eps;
        a.table = (const float4 *)P->table;
        set_periods(a, P);
        a.fscale = P->rho_unit * (P->dx * P->dx * P->dx * P->dx) / (P->dt * P->dt);
        a.tscale = a.fscale * P->dx;
        a.force_fluid = G->force_fluid;
        a.moment_fluid = G->moment_fluid;
        a.hydro_out = P->hydro_out;
    }
    if (L->stress) {
        if (!L->aux) {
            set_error("psc_step: the fused stress output needs the lagged state (aux)");
            return LBDEM_ERR_ARG;
        }
        if (L->bnd_na + L->bnd_nb > 0) {
            set_error("psc_step: the fused stress output does not cover boundary-pass cells; use lbdem_stress");
            return LBDEM_ERR_UNSUPPORTED;
        }
        a.stress_out = L->stress;
    }
    dim3 grid, block;
    step_geometry(L, grid, block, ONE_THREADS);
    // FP16 lagged state exists under FP32 storage only (fill_args checks)
    constexpr int LAG_H = sizeof(T) == 4 ? LAG_HALF : LAG_STORE;
#define LBDEM_STEP_CASE(G_, S_)                                                          \
    do {                                                                                 \
        const int form_ = step_kernel_form<T>();                                         \
        if (G_ && !a.stress_out && form_ > 0) {                                          \
            int rc_ = ROWS_NOT_APPLICABLE;                                               \
            if (form_ == 2)                                                              \
                rc_ = a.wrap_any ? launch_step_rows<T, S_, true, true>(L, a, st)          \
                                 : launch_step_rows<T, S_, false, true>(L, a, st);        \
            if (rc_ == ROWS_NOT_APPLICABLE)                                              \
                rc_ = a.wrap_any ? launch_step_rows<T, S_, true, false>(L, a, st)         \
                                 : launch_step_rows<T, S_, false, false>(L, a, st);       \
            if (rc_ != ROWS_NOT_APPLICABLE) {                                            \
                if (rc_ != LBDEM_OK) return rc_;                                         \
                launch_boundary<T, S_, BND_GATHER>(L, a, st);                            \
                return check_launch("psc_step");                                         \
            }                                                                            \
        }                                                                                \
        if (a.stress_out) {                                                              \
            if (a.wrap_any) k_psc_step<T, G_, S_, true, false, true><<<grid, block, 0, st>>>(a);  \
            else k_psc_step<T, G_, S_, false, false, true><<<grid, block, 0, st>>>(a);           \
        } else if (a.aux16) {                                                            \
            if (a.wrap_any) k_psc_step<T, G_, S_, true, false, false, LAG_H><<<grid, block, 0, st>>>(a);  \
            else k_psc_step<T, G_, S_, false, false, false, LAG_H><<<grid, block, 0, st>>>(a);           \
        } else if (a.wrap_any) {                                                         \
            k_psc_step<T, G_, S_, true, false, false, LAG_STORE><<<grid, block, 0, st>>>(a); \
        } else {                                                                         \
            k_psc_step<T, G_, S_, false, false, false, LAG_STORE><<<grid, block, 0, st>>>(a); \
        }                                                                                \
        launch_boundary<T, S_, G_ ? BND_GATHER : BND_LOCAL>(L, a, st);                   \
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

// Pipelined stepping: phase 1 = far blocks as pure fluid (keys ignored, no
// force), phase 2 = near blocks with the map, then the boundary pass.
template <typename T>
static int launch_step_phase(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int src, int dst,
                             int phase, const uint32_t *blocks, const uint32_t *counts, uint32_t entries,
                             cudaStream_t st) {
    if (phase != 1 && phase != 2) {
        set_error("psc_step_phase: phase must be 1 or 2");
        return LBDEM_ERR_ARG;
    }
    if (!blocks || !counts || (phase == 2 && !(P && G && G->n > 0))) {
        set_error("psc_step_phase: needs the block lists (and for phase 2 the particles)");
        return LBDEM_ERR_ARG;
    }
    if (P && (P->wrap[0] || P->wrap[1] || P->wrap[2])) {
        set_error("psc_step_phase: periodic images are not supported in pipelined stepping");
        return LBDEM_ERR_UNSUPPORTED;
    }
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (src < 0 || src > 1 || dst < 0 || dst > 1 || src == dst) {
        set_error("src/dst must be 0/1 and distinct");
        return LBDEM_ERR_ARG;
    }
    a.src = L->f[src];
    a.dst = L->f[dst];
    a.blist = blocks;
    a.bcount = counts + (phase == 2 ? 1 : 0);
    a.bfrom_end = phase == 2;
    a.nblocks = a.nb * (uint32_t)L->ny * (uint32_t)L->nz;
    if (phase == 2) {
        if (!P->key || !P->table || !G->force_fluid || !G->moment_fluid) {
            set_error("PSC step needs key, table and force accumulators");
            return LBDEM_ERR_ARG;
        }
        a.key = P->key;
        a.eps = P->eps;
        a.table = (const float4 *)P->table;
        set_periods(a, P);
        a.fscale = P->rho_unit * (P->dx * P->dx * P->dx * P->dx) / (P->dt * P->dt);
        a.tscale = a.fscale * P->dx;
        a.force_fluid = G->force_fluid;
        a.moment_fluid = G->moment_fluid;
        a.hydro_out = P->hydro_out;
    }
    // The list length is on the device.  Without an estimate (entries = 0) the
    // launch covers every block and CTAs past the length leave at once; with
    // one, it covers `entries` list entries and a grid-striding launch of one
    // CTA per SM takes any beyond them.
    const uint32_t wpb = ONE_THREADS / 32;
    const bool sized = entries > 0 && entries < a.nblocks;
    const uint32_t cover = sized ? entries : a.nblocks;
    const dim3 block(ONE_THREADS, 1, 1), grid((cover + wpb - 1) / wpb, 1, 1);
    int nsm = 0;
    if (sized) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    constexpr int LAG_H = sizeof(T) == 4 ? LAG_HALF : LAG_STORE;
#define LBDEM_PHASE_CASE(S_, M_)                                                          \
    do {                                                                                  \
        k_psc_step<T, true, S_, false, true, false, M_><<<grid, block, 0, st>>>(a);       \
        if (sized) {                                                                      \
            StepArgs r = a;                                                               \
            r.lbase = grid.x * wpb;                                                       \
            k_psc_step_listed_rest<T, S_, M_><<<nsm, ONE_THREADS, 0, st>>>(r);            \
        }                                                                                 \
        if (phase == 2) launch_boundary<T, S_, BND_GATHER>(L, a, st);                     \
    } while (0)
#define LBDEM_PHASE_LAG(S_)                                                               \
    do {                                                                                  \
        if (a.aux16) LBDEM_PHASE_CASE(S_, LAG_H);                                         \
        else LBDEM_PHASE_CASE(S_, LAG_STORE);                                             \
    } while (0)
    if (L->smag_mode == LBDEM_SMAG_OFF) LBDEM_PHASE_LAG(LBDEM_SMAG_OFF);
    else if (L->smag_mode == LBDEM_SMAG_REFERENCE) LBDEM_PHASE_LAG(LBDEM_SMAG_REFERENCE);
    else LBDEM_PHASE_LAG(LBDEM_SMAG_LOCAL);
#undef LBDEM_PHASE_LAG
#undef LBDEM_PHASE_CASE
    return check_launch("psc_step_phase");
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
    launch_boundary<T, LBDEM_SMAG_OFF, BND_STREAM>(L, a, st);
    return check_launch("stream_moments");
}

template <typename T>
static int launch_init(const lbdem_lattice *L, int buf, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (buf < 0 || buf > 1 || !L->rho || !L->vel || !L->f[0] || !L->f[1]) {
        set_error("lattice_init: bad buffers");
        return LBDEM_ERR_ARG;
    }
    a.dst = L->f[buf];
    dim3 grid, block;
    step_geometry(L, grid, block);
    k_init<T><<<grid, block, 0, st>>>(a, L->rho, L->vel, L->aux != nullptr, L->f[1 - buf]);
    return check_launch("lattice_init");
}

template <typename T>
static int launch_stress(const lbdem_lattice *L, int buf, float *out, cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (buf < 0 || buf > 1 || !out || !L->aux) {
        set_error("stress: needs the post-stream buffer index, an output array and the lagged state (aux)");
        return LBDEM_ERR_ARG;
    }
    a.src = L->f[buf];
    dim3 grid, block;
    step_geometry(L, grid, block);
    k_stress<T><<<grid, block, 0, st>>>(a, out);
    return check_launch("stress");
}

template <typename T>
static int launch_decode(const lbdem_lattice *L, const lbdem_psc *P, int32_t *id, float *vf, float *w, float *vs,
                         cudaStream_t st) {
    StepArgs a;
    int rc = fill_args(L, a);
    if (rc) return rc;
    if (P) {
        a.key = P->key;
        a.eps = P->eps;
        a.table = (const float4 *)P->table;
        set_periods(a, P);
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
// 2048 * 32768 = 2^26 = 67,108,864 cells (512 x 512 x 256) are covered; the
// array is 4 * 2048 doubles = 64 KB of device memory, held by every GPU that
// loads the library until the process exits.  Larger lattices are refused
// before any device work (the 32-bit element offsets of fill_args allow up to
// about 2.26e8 cells, so this limit is the one that binds).
// ---------------------------------------------------------------------------
constexpr int NOALLOC_MAX_BLOCKS = 2048;
constexpr size_t NOALLOC_CELLS_PER_BLOCK = 32768;
static_assert((size_t)NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK < (1ull << 32) / Q,
              "the allocation-free limit must bind before the 32-bit offset limit of fill_args");
static __device__ __align__(256) double g_noalloc_partials[4 * NOALLOC_MAX_BLOCKS];

// Device address of g_noalloc_partials for the current device, looked up on
// the first call on each device (the host-side symbol is only a stand-in and
// must never be passed to a kernel).  The cached address belongs to the
// device's primary context: after cudaDeviceReset on that device it is stale,
// so a caller that resets a device must not call the allocation-free sums on
// it again in the same process.
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
                  "cells (64 KB static scratch; use lbdem_global_sums_f64 with caller scratch)",
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
                      uint32_t *moving, void *stream) {
    if (!ct || !links || nx <= 0 || ny <= 0 || nz <= 0) {
        set_error("build_links: bad arguments");
        return LBDEM_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nc = (size_t)nx * ny * nz;
    k_links<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(ct, nx, ny, nz, skip_inlet, links, moving);
    return check_launch("build_links");
}

int lbdem_boundary_cells(const uint32_t *links, int32_t nx, int32_t ny, int32_t nz, uint32_t *cells,
                         uint32_t capacity, uint32_t *counts, int32_t *scratch, void *stream) {
    if (!links || !counts || !scratch || nx <= 0 || ny <= 0 || nz <= 0 || (capacity > 0 && !cells)) {
        set_error("boundary_cells: bad arguments");
        return LBDEM_ERR_ARG;
    }
    if ((size_t)nx * ny * nz >= (1ull << 32)) {
        set_error("boundary_cells: cell indices are 32-bit");
        return LBDEM_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nrows = ny * nz;
    k_bnd_count<<<(nrows + 7) / 8, 256, 0, st>>>(links, nx, nrows, scratch);
    k_bnd_scan<<<1, 1024, 0, st>>>(scratch, nrows, counts);
    if (capacity > 0) k_bnd_fill<<<(nrows + 7) / 8, 256, 0, st>>>(links, nx, nrows, scratch, counts, cells, capacity);
    return check_launch("boundary_cells");
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

int lbdem_psc_step_phase(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G, int32_t src,
                         int32_t dst, int32_t phase, const uint32_t *blocks, const uint32_t *counts, uint32_t entries,
                         void *stream) {
    if (!L) return LBDEM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    switch (L->storage) {
        case LBDEM_F32: return launch_step_phase<float>(L, P, G, src, dst, phase, blocks, counts, entries, st);
        case LBDEM_F16: return launch_step_phase<__half>(L, P, G, src, dst, phase, blocks, counts, entries, st);
        case LBDEM_BF16:
            return launch_step_phase<__nv_bfloat16>(L, P, G, src, dst, phase, blocks, counts, entries, st);
    }
    set_error("unknown storage form %d", L->storage);
    return LBDEM_ERR_ARG;
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

int lbdem_stress(const lbdem_lattice *L, int32_t buf, float *out, void *stream) {
    if (!L) return LBDEM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (L->storage == LBDEM_F32) return launch_stress<float>(L, buf, out, st);
    if (L->storage == LBDEM_F16) return launch_stress<__half>(L, buf, out, st);
    if (L->storage == LBDEM_BF16) return launch_stress<__nv_bfloat16>(L, buf, out, st);
    set_error("stress: unknown storage");
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
