// Reverse mode of the fused PSC step on a frozen particle bed: the adjoint of
// one collide + stream (psclattice3d.py:187-261, lbm_solver3d.py:197-240,
// lbm_foecelover.py:52-68) and of the drag reduction (lattice2grains,
// psclattice3d.py:316-358) with respect to the populations, the per-cell PSC
// weight B and the body force; and the chain rule from B to the particle
// positions through the smooth solid fraction.
//
// Forward model of one step (f-space, per updated cell; s = streamed
// populations, rho = sum s, j = sum c s, frozen particles u_s = 0):
//   fpc_q = s_q + B (s_qbar - feq_qbar + w_q rho - s_q) - (1-B) om (s_q - feq_q)
//           + 3 w_q rho (c_q . F)
//   feq_q = w_q (rho + 3 c.j + (4.5 (c.j)^2 - 1.5 j.j) / rho)
//   hydro = B j (the reference's -B sum_q c_q Os_q; u_s = 0)
// Reverse, with lam = dL/dfpc and A_q = (1-B) om lam_q - B lam_qbar:
//   dL/ds_p = lam_p (1 - B - (1-B) om) + B lam_pbar + D + G . c_p
//   D = sum_q A_q dfeq_q/drho + sum_q lam_q w_q (B + 3 c_q . F)
//   G = sum_q A_q dfeq_q/dj
//   dL/dB += sum_q lam_q (s_qbar - feq_qbar + w_q rho - s_q + om (s_q - feq_q))
//   dL/dF += sum_q lam_q 3 w_q rho c_q
// and at the last step the loss L = fscale e . sum hydro seeds
//   dL/ds_p += fscale B (e . c_p),  dL/dB += fscale e . j.
// Streaming is a permutation plus bounce-back, so its transpose is a scatter
// in which every target is written exactly once.  Arithmetic is FP32 in
// deviation form (f - w) to keep the cancellations exact-ish; accumulations
// over cells go through warp reductions into FP64 atomics.
#include <math.h>

#include "common.cuh"

namespace lbdem {

struct AdjArgs {
    int nx, ny, nz;
    size_t nc;
    uint32_t rs;                 // population elements per row (blocked layout)
    float om;                    // omega (constant: Smagorinsky off)
    float taum;                  // 1/om - 1/2
    float fx, fy, fz;            // body force, lattice units
    float ex, ey, ez;            // fscale * loss direction
    const float *fprev;          // h = (f - w)/w of the populations step n read
    const float *lam_in;         // dL/dfpc of step n (f units), blocked
    float *lam_out;              // dL/df_prev, blocked
    float *bbar;                 // dL/dB per cell
    double *gbar;                // dL/dF (3)
    const uint32_t *links;
    const uint32_t *key;
    const float *eps;
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <bool GATHER, bool SEED>
__global__ void __launch_bounds__(256) k_psc_adjoint(const AdjArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool inb = (x < nx) && (y < ny);
    const int xc_ = inb ? x : 0, yc_ = inb ? y : 0;
    const uint32_t row = (uint32_t)(z * ny + yc_);
    const uint32_t cell = row * (uint32_t)nx + (uint32_t)xc_;
    const uint32_t rs = a.rs;
    const uint32_t r0 = row * rs;
    const uint32_t own = r0 + xslot((uint32_t)xc_, QB);
    const uint32_t lk = a.links[cell];
    const bool act = inb && !(lk & LINK_SKIP);

    // forward streamed populations (deviation d = f - w) and where each came from
    const uint32_t dym = yc_ == 0 ? (uint32_t)(ny - 1) * rs : (uint32_t)(-(int)rs);
    const uint32_t dyp = yc_ == ny - 1 ? (uint32_t)(-(int)((ny - 1) * rs)) : rs;
    const uint32_t zs = (uint32_t)ny * rs;
    const uint32_t dzm = z == 0 ? (uint32_t)(nz - 1) * zs : (uint32_t)(-(int)zs);
    const uint32_t dzp = z == nz - 1 ? (uint32_t)(-(int)((nz - 1) * zs)) : zs;
    const uint32_t sx0 = xslot((uint32_t)xc_, QB);
    const uint32_t sxm = xslot(xc_ == 0 ? (uint32_t)(nx - 1) : (uint32_t)(xc_ - 1), QB);
    const uint32_t sxp = xslot(xc_ == nx - 1 ? 0u : (uint32_t)(xc_ + 1), QB);
    float d[Q];
    uint32_t from[Q];   // element index of the forward source of s_q (push target of its adjoint)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        uint32_t e;
        if (!GATHER || q == 0) {
            e = own + q * 32;
        } else if (lk & LINK_BB(q)) {
            e = own + qinv(q) * 32;
        } else {
            const uint32_t ry = cy(q) == 1 ? dym : (cy(q) == -1 ? dyp : 0u);
            const uint32_t rz = cz(q) == 1 ? dzm : (cz(q) == -1 ? dzp : 0u);
            const uint32_t xs = cx(q) == 1 ? sxm : (cx(q) == -1 ? sxp : sx0);
            e = r0 + ry + rz + xs + q * 32;
        }
        from[q] = e;
        d[q] = wq(q) * a.fprev[e];
    }
    float lam[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) lam[q] = SEED ? 0.f : a.lam_in[own + q * 32];

    uint32_t key = act && a.key ? a.key[cell] : 0u;
    float B = 0.f;
    if (key) {
        const float e = a.eps ? a.eps[cell] : ((key & KEY_FULL) ? 1.f : (float)key_count(key) * (1.f / 125.f));
        B = e * a.taum / ((1.f - e) + a.taum);
    }
    // moments and equilibrium deviations fe_q = feq_q - w_q
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        drho += d[q];
        if (cx(q)) jx += cx(q) * d[q];
        if (cy(q)) jy += cy(q) * d[q];
        if (cz(q)) jz += cz(q) * d[q];
    }
    const float rho = 1.f + drho, irho = 1.f / rho;
    const float jj = jx * jx + jy * jy + jz * jz;
    const float om = a.om;
    float D = 0.f, Gx = 0.f, Gy = 0.f, Gz = 0.f, bb = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float cj = cx(q) * jx + cy(q) * jy + cz(q) * jz;
        const float quad = (4.5f * cj * cj - 1.5f * jj) * irho;
        const float A = (1.f - B) * om * lam[q] - B * lam[qinv(q)];
        D += A * wq(q) * (1.f - quad * irho);
        const float gq = A * wq(q) * irho;
        const float k3 = 3.f * A * wq(q) + 9.f * gq * cj;
        Gx += k3 * cx(q) - 3.f * gq * jx;
        Gy += k3 * cy(q) - 3.f * gq * jy;
        Gz += k3 * cz(q) - 3.f * gq * jz;
        D += lam[q] * wq(q) * (B + 3.f * (cx(q) * a.fx + cy(q) * a.fy + cz(q) * a.fz));
        // dfpc_q/dB
        const int qb = qinv(q);
        const float cjb = cx(qb) * jx + cy(qb) * jy + cz(qb) * jz;
        const float feb = wq(qb) * (drho + 3.f * cjb + (4.5f * cjb * cjb - 1.5f * jj) * irho);
        const float fe = wq(q) * (drho + 3.f * cj + quad);
        bb += lam[q] * ((d[qb] - feb) + wq(q) * drho - d[q] + om * (d[q] - fe));
        const float lr = lam[q] * 3.f * wq(q) * rho;
        gx += lr * cx(q);
        gy += lr * cy(q);
        gz += lr * cz(q);
    }
    if (SEED) bb += a.ex * jx + a.ey * jy + a.ez * jz;
    if (act) {
        if (B != 0.f || SEED) a.bbar[cell] += bb;
        if (GATHER) {
            const float c1 = 1.f - B - (1.f - B) * om;
#pragma unroll
            for (int p = 0; p < Q; ++p) {
                float sb = lam[p] * c1 + B * lam[qinv(p)] + D + (cx(p) * Gx + cy(p) * Gy + cz(p) * Gz);
                if (SEED) sb += B * (cx(p) * a.ex + cy(p) * a.ey + cz(p) * a.ez);
                a.lam_out[from[p]] = sb;
            }
        }
    } else {
        gx = gy = gz = 0.f;
    }
    // dL/dF: warp sums, block sum, one FP64 atomic per block and component
    __shared__ float part[3][8];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, w = tid >> 5, nw = (blockDim.x * blockDim.y) >> 5;
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    gz = warp_sum(gz);
    if ((tid & 31) == 0) {
        part[0][w] = gx;
        part[1][w] = gy;
        part[2][w] = gz;
    }
    __syncthreads();
    if (tid < 3) {
        double s = 0.0;
        for (int k = 0; k < nw; ++k) s += part[tid][k];
        atomicAdd(a.gbar + tid, s);
    }
}

// Chain rule from dL/dB to the particle centres through the smooth solid
// fraction: B = eps taum / ((1 - eps) + taum), eps = t^2 (3 - 2t),
// t = r - |x_c - p| + 1/2 (lattice units), p = (pos - min)/dx + 1/2.
struct PosAdjArgs {
    int nx, ny, nz;
    size_t nc;
    float taum;
    double dx, xmin, ymin, zmin;
    const double *pos, *radius;
    const uint32_t *key;
    const float *eps;
    const float *bbar;
    double *pos_bar;
};

__global__ void __launch_bounds__(256) k_pos_adjoint(const PosAdjArgs a) {
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const bool in = c < a.nc;
    const uint32_t key = in ? a.key[c] : 0u;
    int gid = -1;
    double vx = 0.0, vy = 0.0, vz = 0.0;
    if (key) {
        gid = (int)key_gid(key);
        const float e = a.eps[c];
        if (e > 0.f && e < 1.f) {
            const int i = (int)(c % a.nx), j = (int)((c / a.nx) % a.ny), k = (int)(c / ((size_t)a.nx * a.ny));
            const double xc = (a.pos[3 * gid] - a.xmin + 0.5 * a.dx) / a.dx;
            const double yc = (a.pos[3 * gid + 1] - a.ymin + 0.5 * a.dx) / a.dx;
            const double zc = (a.pos[3 * gid + 2] - a.zmin + 0.5 * a.dx) / a.dx;
            const double r = (a.radius[gid] - 0.5 * a.dx) / a.dx;
            const double rx = i - xc, ry = j - yc, rz = k - zc;
            const double dd = sqrt(rx * rx + ry * ry + rz * rz);
            const double t = r - dd + 0.5;
            if (t > 0.0 && t < 1.0 && dd > 0.0) {
                const double de_dt = 6.0 * t * (1.0 - t);
                const double tm = a.taum;
                const double den = (1.0 - e) + tm;
                const double dB_de = tm * (1.0 + tm) / (den * den);
                // dt/dp = (x_c - p)/|x_c - p| per lattice unit, / dx per physical unit
                const double s = (double)a.bbar[c] * dB_de * de_dt / (dd * a.dx);
                vx = s * rx;
                vy = s * ry;
                vz = s * rz;
            }
        }
    }
    // segmented warp sum over runs of equal owner
    const unsigned lane = threadIdx.x & 31u;
    const int gnext = __shfl_down_sync(0xffffffffu, gid, 1);
    const int gprev = __shfl_up_sync(0xffffffffu, gid, 1);
    const unsigned tails = __ballot_sync(0xffffffffu, lane == 31 || gnext != gid);
    const unsigned mytail = (unsigned)(__ffs(tails >> lane) - 1) + lane;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double ux = __shfl_down_sync(0xffffffffu, vx, o);
        const double uy = __shfl_down_sync(0xffffffffu, vy, o);
        const double uz = __shfl_down_sync(0xffffffffu, vz, o);
        if (lane + o <= mytail) {
            vx += ux; vy += uy; vz += uz;
        }
    }
    if ((lane == 0 || gprev != gid) && gid >= 0) {
        atomicAdd(a.pos_bar + 3 * gid + 0, vx);
        atomicAdd(a.pos_bar + 3 * gid + 1, vy);
        atomicAdd(a.pos_bar + 3 * gid + 2, vz);
    }
}

}  // namespace lbdem

using namespace lbdem;

extern "C" int lbdem_psc_step_adjoint_f32(const lbdem_lattice *L, const lbdem_psc *P, const void *f_prev,
                                          const float *lam_in, float *lam_out, float *bbar, double *gbar,
                                          const double *loss_dir, int32_t gather, int32_t seed, void *stream) {
    if (!L || !P || !f_prev || !bbar || !gbar || !loss_dir || (!seed && !lam_in) || (gather && !lam_out) ||
        !L->links) {
        set_error("psc_step_adjoint: bad arguments");
        return LBDEM_ERR_ARG;
    }
    if (L->storage != LBDEM_F32 || L->smag_mode != LBDEM_SMAG_OFF) {
        set_error("psc_step_adjoint: the adjoint covers FP32 storage with Smagorinsky off");
        return LBDEM_ERR_UNSUPPORTED;
    }
    if (P->wrap[0] || P->wrap[1] || P->wrap[2]) {
        set_error("psc_step_adjoint: the smooth solid fraction has no periodic images");
        return LBDEM_ERR_UNSUPPORTED;
    }
    if (L->moving || L->bnd_na + L->bnd_nb > 0) {
        set_error("psc_step_adjoint: the adjoint covers fixed walls only (no moving walls, inlets or open boundaries)");
        return LBDEM_ERR_UNSUPPORTED;
    }
    const size_t nb = ((size_t)L->nx + 31) / 32;
    if (nb * 32 * L->ny * L->nz * Q >= (1ull << 32)) {
        set_error("psc_step_adjoint: lattice too large for 32-bit element offsets");
        return LBDEM_ERR_ARG;
    }
    AdjArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.nc = (size_t)L->nx * L->ny * L->nz;
    a.rs = (uint32_t)nb * QB;
    a.om = L->omega0;
    a.taum = 1.f / L->omega0 - 0.5f;
    if (L->force_on) {
        a.fx = L->force[0]; a.fy = L->force[1]; a.fz = L->force[2];
    }
    const double fscale = P->rho_unit * (P->dx * P->dx * P->dx * P->dx) / (P->dt * P->dt);
    a.ex = (float)(fscale * loss_dir[0]);
    a.ey = (float)(fscale * loss_dir[1]);
    a.ez = (float)(fscale * loss_dir[2]);
    a.fprev = static_cast<const float *>(f_prev);
    a.lam_in = lam_in;
    a.lam_out = lam_out;
    a.bbar = bbar;
    a.gbar = gbar;
    a.links = L->links;
    a.key = P->key;
    a.eps = P->eps;
    int bx = ((L->nx + 31) / 32) * 32;
    if (bx > 256) bx = 256;
    int by = 256 / bx;
    if (by > L->ny) by = L->ny;
    const dim3 block(bx, by, 1), grid((L->nx + bx - 1) / bx, (L->ny + by - 1) / by, L->nz);
    cudaStream_t st = (cudaStream_t)stream;
    if (gather) {
        if (seed) k_psc_adjoint<true, true><<<grid, block, 0, st>>>(a);
        else k_psc_adjoint<true, false><<<grid, block, 0, st>>>(a);
    } else {
        if (seed) k_psc_adjoint<false, true><<<grid, block, 0, st>>>(a);
        else k_psc_adjoint<false, false><<<grid, block, 0, st>>>(a);
    }
    return check_launch("psc_step_adjoint");
}

extern "C" int lbdem_psc_force_adjoint(const lbdem_lattice *L, const lbdem_psc *P, const lbdem_grains *G,
                                       const float *bbar, double *pos_bar, void *stream) {
    if (!L || !P || !G || !P->key || !P->eps || !bbar || !pos_bar) {
        set_error("psc_force_adjoint: bad arguments (the smooth map's eps is required)");
        return LBDEM_ERR_ARG;
    }
    if (G->n <= 0) return LBDEM_OK;
    PosAdjArgs a;
    a.nx = L->nx; a.ny = L->ny; a.nz = L->nz;
    a.nc = (size_t)L->nx * L->ny * L->nz;
    a.taum = 1.f / L->omega0 - 0.5f;
    a.dx = P->dx; a.xmin = P->xmin; a.ymin = P->ymin; a.zmin = P->zmin;
    a.pos = G->pos; a.radius = G->radius;
    a.key = P->key; a.eps = P->eps; a.bbar = bbar; a.pos_bar = pos_bar;
    k_pos_adjoint<<<(unsigned)((a.nc + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    return check_launch("psc_force_adjoint");
}
