// Shared device definitions: D3Q19 lattice, storage forms, link masks, errors.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lbdem.h"

namespace lbdem {

// D3Q19 velocity set, weights and opposite directions
// (src/lbm3d/lbm_solver3d.py:46-91: same ordering as the reference).
constexpr int Q = 19;
__host__ __device__ constexpr int cx(int q) {
    return q == 1 || q == 7 || q == 9 || q == 11 || q == 13 ? 1
         : q == 2 || q == 8 || q == 10 || q == 12 || q == 14 ? -1 : 0;
}
__host__ __device__ constexpr int cy(int q) {
    return q == 3 || q == 7 || q == 10 || q == 15 || q == 17 ? 1
         : q == 4 || q == 8 || q == 9 || q == 16 || q == 18 ? -1 : 0;
}
__host__ __device__ constexpr int cz(int q) {
    return q == 5 || q == 11 || q == 14 || q == 15 || q == 18 ? 1
         : q == 6 || q == 12 || q == 13 || q == 16 || q == 17 ? -1 : 0;
}
__host__ __device__ constexpr int qinv(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
// specular images of direction q in a wall normal to x / y / z
// (qsyx / qsyy / qsyz, lbm_solver3d.py:50-57): the direction with that
// component of c_q negated
__host__ __device__ constexpr int qmirror(int q, int axis) {
    for (int p = 0; p < 19; ++p) {
        const int mx = axis == 0 ? -cx(q) : cx(q), my = axis == 1 ? -cy(q) : cy(q), mz = axis == 2 ? -cz(q) : cz(q);
        if (cx(p) == mx && cy(p) == my && cz(p) == mz) return p;
    }
    return q;
}
__host__ __device__ constexpr float wq(int q) {
    return q == 0 ? 1.0f / 3.0f : (q <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
}
constexpr float CS2 = 1.0f / 3.0f;
// Blocked population layout: 32 cells per x-block, QB elements per block of
// populations, AB per block of the 5 lagged Smagorinsky values.
constexpr uint32_t QB = Q * 32;
constexpr uint32_t AB = 5 * 32;
// Element offset, within its row, of cell x's block slot (lane x % 32 of
// x-block x / 32; the population or auxiliary index adds q * 32).
__host__ __device__ inline uint32_t xslot(uint32_t x, uint32_t per_block) {
    return (x >> 5) * per_block + (x & 31u);
}

// Per-cell link mask (built once from CellType by lbdem_build_links)
constexpr uint32_t LINK_SKIP = 1u << 19;   // cell is not updated (OBSTACLE / VEL_LADD / FREE_SLIP [/ INLET])
constexpr uint32_t LINK_FLUID = LBDEM_LINK_FLUID;  // FLUID: moments are recomputed
constexpr uint32_t LINK_MAP_SKIP = 1u << 21;  // PSC map skips the cell
constexpr uint32_t LINK_MOVING = 1u << 22;    // some bounce-back neighbour is a moving wall (VEL_LADD)
__host__ __device__ constexpr uint32_t LINK_BB(int q) { return 1u << q; }  // neighbour x-c_q is OBSTACLE
// Open boundaries (wet-node conditions of the stream's second pass,
// lbm_solver3d.py:242-250, and free-slip neighbours): such cells are streamed
// and collided by the boundary pass after the fused step instead of by it.
constexpr uint32_t LINK_DEFER = 1u << 23;    // Zou-He / exit / Ladd inlet cell, or a free-slip neighbour
constexpr uint32_t LINK_PHASE_B = 1u << 24;  // deferred cell that reads its interior neighbour (exit, inlet)
constexpr uint32_t LINK_KEEP = 1u << 25;     // interior neighbour of an exit or inlet: the step stores rho/u
constexpr uint32_t LINK_INLET = 1u << 26;    // the cell is a Ladd velocity inlet (VEL_INLET_LADD)
constexpr uint32_t LINK_SLIP_NB = 1u << 0;   // some neighbour is a free-slip wall (bit 0: no direction uses it)

// Face of an open-boundary cell from its orientation bits, in the reference's
// precedence LEFT, RIGHT, BOTTOM, TOP, BACK, FRONT (lbm_solver3d.py:522-527,
// 647-658, 686-816, 831-960): axis (0 x, 1 y, 2 z) and inward sign s (+1 when
// the interior neighbour is at +1 along the axis); false without a face bit.
__host__ __device__ inline bool face_of(int32_t ct, int &axis, int &s) {
    if (ct & LBDEM_CT_LEFT) { axis = 0; s = 1; }
    else if (ct & LBDEM_CT_RIGHT) { axis = 0; s = -1; }
    else if (ct & LBDEM_CT_BOTTOM) { axis = 1; s = 1; }
    else if (ct & LBDEM_CT_TOP) { axis = 1; s = -1; }
    else if (ct & LBDEM_CT_BACK) { axis = 2; s = 1; }
    else if (ct & LBDEM_CT_FRONT) { axis = 2; s = -1; }
    else return false;
    return true;
}

// Which wet-node rule of the stream's second pass (lbm_solver3d.py:242-250)
// applies to a cell, in the reference's order.
enum WetRule { WET_NONE = 0, WET_VEL_ZOUHE, WET_EXIT, WET_PRE_ZOUHE, WET_INLET };
__host__ __device__ inline int wet_rule(int32_t ct) {
    if (ct & LBDEM_CT_VEL_ZOUHE) return WET_VEL_ZOUHE;
    if (ct & LBDEM_CT_VEL_EXIT) return WET_EXIT;
    if (ct & LBDEM_CT_PRE_ZOUHE) return WET_PRE_ZOUHE;
    if (ct & LBDEM_CT_VEL_INLET_LADD) return WET_INLET;
    return WET_NONE;
}

// Storage forms.  Every form stores the scaled deviation
// h = (f - w) * S / w (S = 1 for FP32, scale16 for the 16-bit forms): the
// step computes in h directly (widen/narrow), the auxiliary kernels decode
// d = f - w = h * w / S (dec) and encode h = d * S / w (enc).
template <typename T> struct Store;
template <> struct Store<float> {
    static constexpr int kind = LBDEM_F32;
    __device__ __forceinline__ static float widen(float v) { return v; }
    __device__ __forceinline__ static float narrow(float h) { return h; }
    __device__ __forceinline__ static float dec(float v, float wscale) { return v * wscale; }
    __device__ __forceinline__ static float enc(float d, float inv_wscale) { return d * inv_wscale; }
    __device__ __forceinline__ static float ld(const float *p) { return __ldg(p); }
};
template <> struct Store<__half> {
    static constexpr int kind = LBDEM_F16;
    __device__ __forceinline__ static float widen(__half v) { return __half2float(v); }
    __device__ __forceinline__ static __half narrow(float h) { return __float2half_rn(h); }
    __device__ __forceinline__ static float dec(__half v, float wscale) { return __half2float(v) * wscale; }
    __device__ __forceinline__ static __half enc(float d, float inv_wscale) { return __float2half_rn(d * inv_wscale); }
    __device__ __forceinline__ static __half ld(const __half *p) { return __ldg(p); }
};
template <> struct Store<__nv_bfloat16> {
    static constexpr int kind = LBDEM_BF16;
    __device__ __forceinline__ static float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ __forceinline__ static __nv_bfloat16 narrow(float h) { return __float2bfloat16_rn(h); }
    __device__ __forceinline__ static float dec(__nv_bfloat16 v, float wscale) { return __bfloat162float(v) * wscale; }
    __device__ __forceinline__ static __nv_bfloat16 enc(float d, float inv_wscale) {
        return __float2bfloat16_rn(d * inv_wscale);
    }
    __device__ __forceinline__ static __nv_bfloat16 ld(const __nv_bfloat16 *p) { return __ldg(p); }
};

// Auxiliary (lagged Smagorinsky) state is kept in the population storage
// type; 16-bit forms store it unscaled.
template <typename T> __device__ __forceinline__ float aux_dec(T v);
template <> __device__ __forceinline__ float aux_dec<float>(float v) { return v; }
template <> __device__ __forceinline__ float aux_dec<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float aux_dec<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T> __device__ __forceinline__ T aux_enc(float v);
template <> __device__ __forceinline__ float aux_enc<float>(float v) { return v; }
template <> __device__ __forceinline__ __half aux_enc<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 aux_enc<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// PSC owner key: full(1) | count(7) | (0xFFFFFF - gid)(24); atomicMax picks
// the reference's winner (psclattice3d.py:100-138): lowest-id full cover,
// else largest sub-sample count, ties to the lowest id.
constexpr uint32_t KEY_FULL = 1u << 31;
__host__ __device__ inline uint32_t key_gid(uint32_t k) { return 0xFFFFFFu - (k & 0xFFFFFFu); }
__host__ __device__ inline int key_count(uint32_t k) { return (int)((k >> 24) & 0x7Fu); }

// Host-side error reporting
void set_error(const char *fmt, ...);
int check_launch(const char *what);

}  // namespace lbdem
