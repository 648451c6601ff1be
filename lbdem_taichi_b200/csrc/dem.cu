// DEM sub-step on the GPU (DEMSolver.run_simulation, demsolver.py:848-862).
//
// Broad phase: the reference hashes cells of size 4*r_max with a Morton code
// into a 2^20..2^22 table and probes each particle's own cell plus the seven
// cells of its octant (bpcd.py:114-152), proposing pairs i < j.  Here the same
// cells are kept in a dense grid (no hash) and probed with the same octant
// rule, which proposes the same pairs whenever distinct cells do not alias in
// the reference's hash (checked on the host).
//
// Cells keep fixed-capacity particle lists filled by the binning atomics, so
// no scan is needed.  Per sub-step two launches: k_contacts (eight lanes per
// particle: candidate pairs j > i with contact history owned by i, and the six
// walls; forces go to accumulators) and k_integrate (accumulated + body +
// fluid force, improved Verlet, quaternion update, contact-list compaction,
// binning of the new positions into the other half of the counts).
// FP64 throughout; compiled with -fmad=false to follow the reference's
// operation order (and the FP64 oracle) closely.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cooperative_groups.h>
#include <mutex>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace lbdem {

struct M3 {
    double m[3][3];
};

__device__ __forceinline__ void cross3(const double *a, const double *b, double *o) {
    const double t0 = a[1] * b[2] - a[2] * b[1], t1 = a[2] * b[0] - a[0] * b[2], t2 = a[0] * b[1] - a[1] * b[0];
    o[0] = t0; o[1] = t1; o[2] = t2;
}
__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void mv(const M3 &M, const double *v, double *o) {
    double t[3];
    for (int r = 0; r < 3; ++r) t[r] = M.m[r][0] * v[0] + M.m[r][1] * v[1] + M.m[r][2] * v[2];
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
}
__device__ M3 inv3(const M3 &A) {
    const double(*a)[3] = A.m;
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) -
                       a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2]) +
                       a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
    const double id = 1.0 / det;
    M3 o;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o.m[j][i] = id * (a[(i + 1) % 3][(j + 1) % 3] * a[(i + 2) % 3][(j + 2) % 3] -
                              a[(i + 2) % 3][(j + 1) % 3] * a[(i + 1) % 3][(j + 2) % 3]);
    return o;
}

// rotation taking unit vector a onto +x (demsolver.py:686-701, :757-773)
__device__ M3 rot_to_x(const double *a) {
    const double b[3] = {1.0, 0.0, 0.0};
    double v[3];
    cross3(a, b, v);
    const double s = sqrt(dot3(v, v));
    const double c = dot3(a, b);
    M3 R;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R.m[i][j] = 0.0;
    if (s < 1e-12) {
        if (c > 0.0) {
            R.m[0][0] = R.m[1][1] = R.m[2][2] = 1.0;
        } else {
            R.m[0][0] = -1.0; R.m[1][1] = 1.0; R.m[2][2] = -1.0;
        }
    } else {
        const double vx[3][3] = {{0.0, -v[2], v[1]}, {v[2], 0.0, -v[0]}, {-v[1], v[0], 0.0}};
        const double coef = (1.0 - c) / (s * s);
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) {
                double acc = 0.0;
                for (int t = 0; t < 3; ++t) acc += (coef * vx[r][t]) * vx[t][q];
                R.m[r][q] = ((r == q ? 1.0 : 0.0) + vx[r][q]) + acc;
            }
    }
    return R;
}

constexpr int SLOTS_IN_REGS = 8;    // contact slots whose partners are fetched with the particle state

struct DemArgs {
    lbdem_dem d;
    int ncell;
    int parity;
    // Hertz constants of a contact, [0] particle-particle, [1] particle-wall
    // (hertz.py:45-97, 99-153: effective Young's and shear moduli, damping
    // ratio from the restitution), computed once per launch on the host in the
    // reference's operation order instead of once per contact
    double hz_ys[2], hz_gs[2], hz_beta[2];
};

__device__ __forceinline__ int cell_index(const lbdem_dem &d, int cx_, int cy_, int cz_) {
    // grid covers reference cells -1 .. gdim-2 per axis
    const int gx = cx_ + 1, gy = cy_ + 1, gz = cz_ + 1;
    if (gx < 0 || gy < 0 || gz < 0 || gx >= d.gdim[0] || gy >= d.gdim[1] || gz >= d.gdim[2]) return -1;
    return (gz * d.gdim[1] + gy) * d.gdim[0] + gx;
}

__device__ __forceinline__ void ref_cell(const lbdem_dem &d, const double *p, int *ijk) {
    // bpcd.py:191-194
    for (int a = 0; a < 3; ++a) ijk[a] = (int)floor((p[a] - d.bp_min[a]) / d.cell_size);
}

// Bin particle i into its reference cell: the atomic rank is its slot in the
// cell's fixed-capacity list (no scan needed).
__device__ __forceinline__ void bin_particle(const lbdem_dem &d, int i, int32_t *count) {
    int ijk[3];
    ref_cell(d, d.pos + 3 * i, ijk);
    const int c = cell_index(d, ijk[0], ijk[1], ijk[2]);
    if (c < 0) {
        atomicOr(d.status, (int)LBDEM_ST_GRID_OVERFLOW);
        return;
    }
    const int rank = atomicAdd(count + c, 1);
    if (rank < d.cell_cap) d.cell_list[(size_t)c * d.cell_cap + rank] = i;
    else atomicOr(d.status, (int)LBDEM_ST_CELL_OVERFLOW);
}

__global__ void k_bin(const __grid_constant__ DemArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.d.n) return;
    bin_particle(A.d, i, A.d.cell_count + (size_t)A.parity * A.ncell);
}

// ------------------------------- contact laws ------------------------------
// hertz.py:45-97 / linear.py:43-101 (particle-particle), hertz.py:99-153 /
// linear.py:103-152 (particle-wall).  `wall` selects the wall variant.
__device__ void contact_force(const DemArgs &A, double rad_i, double mass_i, double rad_j, double mass_j, bool wall,
                              double *shear, double delta_n, const double *vc, double *F) {
    const lbdem_dem &d = A.d;
    const double gap = -1 * delta_n;
    const double dt = d.dt;
    double inc[3] = {vc[0] * dt, vc[1] * dt, vc[2] * dt};
    inc[0] = 0.0;
    double kt, gt, F0, mu;
    const int tj = wall ? 1 : 0;
    if (d.model == 0) {
        const double Ys = A.hz_ys[tj], Gs = A.hz_gs[tj], beta = A.hz_beta[tj];
        double Rs, ms;
        if (wall) {
            Rs = rad_i;
            ms = mass_i;
            mu = d.mu[1];
        } else {
            Rs = 1.0 / (1.0 / rad_i + 1.0 / rad_j);
            ms = 1.0 / (1.0 / mass_i + 1.0 / mass_j);
            mu = 0.5 * (d.mu[0] + d.mu[0]);
        }
        const double Sn = 2.0 * Ys * sqrt(Rs * delta_n);
        const double St = 8.0 * Gs * sqrt(Rs * delta_n);
        const double kn = 4.0 / 3.0 * Ys * sqrt(Rs * delta_n);
        const double gn = -2.0 * beta * sqrt(5.0 / 6.0 * Sn * ms);
        kt = 8.0 * Gs * sqrt(Rs * delta_n);
        gt = -2.0 * beta * sqrt(5.0 / 6.0 * St * ms);
        F0 = -kn * gap - gn * vc[0];
    } else {
        double kns, kss, dpn, dps, ms;
        if (wall) {
            kns = d.kn[0]; kss = d.ks[0]; dpn = d.dpn[0]; dps = d.dps[0];
            ms = mass_i;
            mu = d.mu[1];
        } else {
            kns = d.kn[0] * d.kn[0] / (d.kn[0] + d.kn[0]);
            kss = d.ks[0] * d.ks[0] / (d.ks[0] + d.ks[0]);
            dpn = 0.5 * (d.dpn[0] + d.dpn[0]);
            dps = 0.5 * (d.dps[0] + d.dps[0]);
            ms = 1.0 / (1.0 / mass_i + 1.0 / mass_j);
            mu = 0.5 * (d.mu[0] + d.mu[0]);
        }
        const double Cn = 2. * dpn * sqrt(kns * ms);
        const double Ct = 2. * dps * sqrt(kns * ms);
        kt = kss;
        gt = Ct;
        F0 = -kns * gap - Cn * vc[0];
    }
    for (int a = 0; a < 3; ++a) shear[a] += inc[a];
    const double ts[3] = {-kt * shear[0], -kt * shear[1], -kt * shear[2]};
    const double tl = sqrt(dot3(ts, ts));
    F[0] = F0;
    if (tl >= mu * F0 && tl > 0.0) {
        const double ratio = mu * F0 / tl;
        F[1] = ts[1] * ratio;
        F[2] = ts[2] * ratio;
        shear[1] = -F[1] / kt;
        shear[2] = -F[2] / kt;
    } else {
        F[1] = ts[1] - gt * vc[1];
        F[2] = ts[2] - gt * vc[2];
    }
}

__device__ __forceinline__ void periodic_delta(const lbdem_dem &d, const double *pi, const double *pj, double *dv) {
    // demsolver.py:483-512
    for (int a = 0; a < 3; ++a) {
        dv[a] = pj[a] - pi[a];
        if (d.periodic[a]) {
            const double L = d.dom_max[a] - d.dom_min[a];
            if (dv[a] > 0.5 * L) dv[a] -= L;
            else if (dv[a] < -0.5 * L) dv[a] += L;
        }
    }
}

// State of particle i held in registers by its contact lanes.
struct PState {
    double p[3], v[3], w[3], rad, mass;
};

// resolve(i, j) (demsolver.py:638-740); forces on i accumulated in Fi/Mi,
// forces on j added atomically.  hk: i's first contact slots (the partner of
// an active slot, -1 for an inactive one) as they were when the sub-step
// started (only i's lanes touch i's slots, each for its own partner).
__device__ __forceinline__ void resolve_pair(const DemArgs &A, int i, const PState &P, int n_i, const int *hk,
                                             int j, double *Fi_acc, double *Mi_acc) {
    const lbdem_dem &d = A.d;
    const size_t base = (size_t)i * d.maxc;
    // partner state: all loads issued together
    double pj[3], vj[3], wj[3];
    for (int t = 0; t < 3; ++t) {
        pj[t] = d.pos[3 * j + t];
        vj[t] = d.vel[3 * j + t];
        wj[t] = d.omega[3 * j + t];
    }
    const double rad_j = d.radius[j], mass_j = d.mass[j];
    int off = -1;
    const int nreg = min(n_i, min(d.maxc, SLOTS_IN_REGS));
#pragma unroll
    for (int o = SLOTS_IN_REGS - 1; o >= 0; --o)   // lowest matching slot wins, as a forward search
        if (o < nreg && hk[o] == j) off = o;
    if (off < 0)
        for (int o = SLOTS_IN_REGS; o < n_i && o < d.maxc; ++o)
            if (d.cf_j[base + o] == j && d.cf_active[base + o]) {
                off = o;
                break;
            }
    double dv[3];
    periodic_delta(d, P.p, pj, dv);
    const double distance = sqrt(dot3(dv, dv));
    const double gap = distance - P.rad - rad_j;
    bool eval = false;
    if (off >= 0) {
        if (gap < 0) eval = true;
        else d.cf_active[base + off] = 0;
    } else if (gap < 0) {
        // append_contact_offset (demsolver.py:352-359); several lanes of the
        // same particle may append in one sub-step
        off = n_i + atomicAdd(d.cf_add + i, 1);
        if (off >= d.maxc) {
            atomicOr(d.status, (int)LBDEM_ST_CONTACT_OVERFLOW);
            return;
        }
        d.cf_j[base + off] = j;
        d.cf_active[base + off] = 1;
        for (int a = 0; a < 3; ++a)
            d.cf_shear[3 * (base + off) + a] = d.cf_pos[3 * (base + off) + a] = d.cf_force[3 * (base + off) + a] = 0.0;
        eval = true;
    }
    if (!eval) return;
    const size_t s = base + off;
    double sh[3] = {d.cf_shear[3 * s], d.cf_shear[3 * s + 1], d.cf_shear[3 * s + 2]};
    const double len = sqrt(dot3(dv, dv));
    const double a[3] = {dv[0] / len, dv[1] / len, dv[2] / len};
    const M3 R = rot_to_x(a);
    const double delta_n = -gap;
    const double *pi = P.p;
    double cp[3], ri[3], rj[3];
    for (int t = 0; t < 3; ++t) {
        cp[t] = pi[t] + a[t] * (P.rad - delta_n);
        d.cf_pos[3 * s + t] = cp[t];
    }
    for (int t = 0; t < 3; ++t) {
        ri[t] = cp[t] - pi[t];
        rj[t] = cp[t] - (pi[t] + dv[t]);
    }
    double vci[3], vcj[3], dvc[3], vc[3];
    cross3(P.w, ri, vci);
    cross3(wj, rj, vcj);
    for (int t = 0; t < 3; ++t) {
        vci[t] += P.v[t];
        vcj[t] += vj[t];
        dvc[t] = vcj[t] - vci[t];
    }
    mv(R, dvc, vc);
    double F[3];
    contact_force(A, P.rad, P.mass, rad_j, mass_j, false, sh, delta_n, vc, F);
    for (int t = 0; t < 3; ++t) {
        d.cf_shear[3 * s + t] = sh[t];
        d.cf_force[3 * s + t] = F[t];
    }
    const M3 Ri = inv3(R);
    const double mF[3] = {-F[0], -F[1], -F[2]};
    double Fi[3], Fj[3], Mi[3], Mj[3];
    mv(Ri, mF, Fi);
    mv(Ri, F, Fj);
    cross3(ri, Fi, Mi);
    cross3(rj, Fj, Mj);
    for (int t = 0; t < 3; ++t) {
        Fi_acc[t] += Fi[t];
        Mi_acc[t] += Mi[t];
        atomicAdd(d.acc_force + 3 * j + t, Fj[t]);
        atomicAdd(d.acc_moment + 3 * j + t, Mj[t]);
    }
}

// evaluate_wall (demsolver.py:742-807)
__device__ void wall_contact(const DemArgs &A, int i, const PState &P, int w, double *Fi_acc, double *Mi_acc) {
    const lbdem_dem &d = A.d;
    const double *nrm = d.wall_n + 3 * w;
    const size_t s = (size_t)i * 6 + w;
    double sh[3] = {d.wcf_shear[3 * s], d.wcf_shear[3 * s + 1], d.wcf_shear[3 * s + 2]};
    const M3 R = rot_to_x(nrm);
    const double *p = P.p;
    const double delta_n = (dot3(p, nrm) - d.wall_d[w]) + P.rad;
    const double distance = P.rad - delta_n;
    double ri[3];
    for (int t = 0; t < 3; ++t) {
        ri[t] = distance * nrm[t];
        d.wcf_pos[3 * s + t] = p[t] + ri[t];
    }
    double vci[3], m[3], vc[3];
    cross3(P.w, ri, vci);
    for (int t = 0; t < 3; ++t) m[t] = -(vci[t] + P.v[t]);
    mv(R, m, vc);
    double F[3];
    contact_force(A, P.rad, P.mass, 0.0, 0.0, true, sh, delta_n, vc, F);
    for (int t = 0; t < 3; ++t) {
        d.wcf_shear[3 * s + t] = sh[t];
        d.wcf_force[3 * s + t] = F[t];
    }
    const M3 Ri = inv3(R);
    const double mF[3] = {-F[0], -F[1], -F[2]};
    double Fi[3], Mi[3];
    mv(Ri, mF, Fi);
    cross3(ri, Fi, Mi);
    for (int t = 0; t < 3; ++t) {
        Fi_acc[t] += Fi[t];
        Mi_acc[t] += Mi[t];
    }
}

// Eight lanes per particle: lane k probes the k-th cell of the reference's
// probe list (own cell + octant, bpcd.py:133-142) and, for k < 6, wall k
// (demsolver.py:809-838); the lanes' forces on the particle are summed with
// shuffles before one atomic per component.
// One lane of the contact phase: lane k of particle i = tid / 8.  All 32 lanes
// of the warp must call it together (shuffle reduction over groups of 8).
// WRAP: also probe around the particle's periodic images (lbdem_dem.wrap_pairs).
template <bool WRAP>
__device__ __forceinline__ void contact_lane(const DemArgs &A, const int32_t *count, int tid) {
    const lbdem_dem &d = A.d;
    const int i = tid >> 3, k = tid & 7;
    const bool act = i < d.n;
    double Fi[3] = {0.0, 0.0, 0.0}, Mi[3] = {0.0, 0.0, 0.0};
    if (act) {
        // particle state, contact-slot snapshot and wall flag fetched together
        PState P;
        for (int t = 0; t < 3; ++t) {
            P.p[t] = d.pos[3 * i + t];
            P.v[t] = d.vel[3 * i + t];
            P.w[t] = d.omega[3 * i + t];
        }
        P.rad = d.radius[i];
        P.mass = d.mass[i];
        const int n_i = d.cfn[i];   // slots in use when the sub-step started
        const size_t base = (size_t)i * d.maxc;
        int hk[SLOTS_IN_REGS];
#pragma unroll
        for (int o = 0; o < SLOTS_IN_REGS; ++o) {
            const bool in = o < d.maxc;
            const int pj = in ? d.cf_j[base + o] : -1, act_o = in ? d.cf_active[base + o] : 0;
            hk[o] = act_o ? pj : -1;
        }
        const bool wall_lane = k < 6 && !d.wall_periodic[k];
        const int wact = wall_lane ? d.wcf_active[(size_t)i * 6 + k] : 0;
        // the reference's probe of lane k around a position (own cell + octant)
        auto probe = [&](const double q[3]) {
            int ijk[3], dd[3];
            ref_cell(d, q, ijk);
            for (int a = 0; a < 3; ++a) {
                const double center = (ijk[a] + 0.5) * d.cell_size + d.bp_min[a];
                dd[a] = (q[a] > center) ? 1 : -1;
            }
            const int ox = (k == 1 || k == 5 || k == 6 || k == 7) ? dd[0] : 0;
            const int oy = (k == 2 || k == 4 || k == 6 || k == 7) ? dd[1] : 0;
            const int oz = (k == 3 || k == 4 || k == 5 || k == 7) ? dd[2] : 0;
            const int c = cell_index(d, ijk[0] + ox, ijk[1] + oy, ijk[2] + oz);
            if (c >= 0) {
                const int n = min(count[c], d.cell_cap);
                const int32_t *lst = d.cell_list + (size_t)c * d.cell_cap;
                for (int t = 0; t < n; ++t) {
                    const int j = lst[t];
                    if (j > i) resolve_pair(A, i, P, n_i, hk, j, Fi, Mi);
                }
            }
        };
        if constexpr (!WRAP) {
            // the union of the eight probed cells' lists (own cell + octant, in
            // the reference's order), shared round-robin by the particle's eight
            // lanes so that a crowded cell does not make one lane the phase's
            // last: lane k takes candidates k, k + 8, ... of the concatenation
            int ijk[3], dd[3];
            ref_cell(d, P.p, ijk);
            for (int a = 0; a < 3; ++a) {
                const double center = (ijk[a] + 0.5) * d.cell_size + d.bp_min[a];
                dd[a] = (P.p[a] > center) ? 1 : -1;
            }
            int cidx[8], pre[8], total = 0;   // cell and exclusive prefix of the counts (static indices only)
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const int ox = (kk == 1 || kk == 5 || kk == 6 || kk == 7) ? dd[0] : 0;
                const int oy = (kk == 2 || kk == 4 || kk == 6 || kk == 7) ? dd[1] : 0;
                const int oz = (kk == 3 || kk == 4 || kk == 5 || kk == 7) ? dd[2] : 0;
                cidx[kk] = cell_index(d, ijk[0] + ox, ijk[1] + oy, ijk[2] + oz);
                pre[kk] = total;
                total += cidx[kk] >= 0 ? min(count[cidx[kk]], d.cell_cap) : 0;
            }
            for (int t = k; t < total; t += 8) {
                // the last probed cell whose first index is <= t holds candidate t
                int cc = cidx[0], bb = 0;
#pragma unroll
                for (int kk = 1; kk < 8; ++kk)
                    if (t >= pre[kk]) { cc = cidx[kk]; bb = pre[kk]; }
                const int j = d.cell_list[(size_t)cc * d.cell_cap + (t - bb)];
                if (j > i) resolve_pair(A, i, P, n_i, hk, j, Fi, Mi);
            }
        } else {
            // the particle and its periodic images when it lies within one
            // broad-phase cell of a periodic face; the pair geometry is the
            // minimum image either way (periodic_delta)
            double sh[3] = {0.0, 0.0, 0.0};
            int nimg[3] = {1, 1, 1};
            for (int a = 0; a < 3; ++a) {
                if (!d.periodic[a]) continue;
                const double L = d.dom_max[a] - d.dom_min[a];
                if (P.p[a] < d.dom_min[a] + d.cell_size) { sh[a] = L; nimg[a] = 2; }
                else if (P.p[a] > d.dom_max[a] - d.cell_size) { sh[a] = -L; nimg[a] = 2; }
            }
            for (int ia = 0; ia < nimg[0]; ++ia)
                for (int ja = 0; ja < nimg[1]; ++ja)
                    for (int ka = 0; ka < nimg[2]; ++ka) {
                        const double q[3] = {P.p[0] + ia * sh[0], P.p[1] + ja * sh[1], P.p[2] + ka * sh[2]};
                        probe(q);
                    }
        }
        if (wall_lane) {
            const int w = k;
            const size_t s = (size_t)i * 6 + w;
            const double sep = -(dot3(P.p, d.wall_n + 3 * w) - d.wall_d[w]);
            if (wact) {
                if (sep > P.rad) d.wcf_active[s] = 0;
                else wall_contact(A, i, P, w, Fi, Mi);
            } else if (sep <= P.rad) {
                d.wcf_active[s] = 1;
                for (int t = 0; t < 3; ++t) d.wcf_shear[3 * s + t] = d.wcf_pos[3 * s + t] = d.wcf_force[3 * s + t] = 0.0;
                wall_contact(A, i, P, w, Fi, Mi);
            }
        }
    }
#pragma unroll
    for (int off = 1; off < 8; off <<= 1)
        for (int t = 0; t < 3; ++t) {
            Fi[t] += __shfl_xor_sync(0xffffffffu, Fi[t], off);
            Mi[t] += __shfl_xor_sync(0xffffffffu, Mi[t], off);
        }
    if (act && k == 0)
        for (int t = 0; t < 3; ++t) {
            atomicAdd(d.acc_force + 3 * i + t, Fi[t]);
            atomicAdd(d.acc_moment + 3 * i + t, Mi[t]);
        }
}

template <bool WRAP>
__global__ void __launch_bounds__(128) k_contacts(const __grid_constant__ DemArgs A) {
    contact_lane<WRAP>(A, A.d.cell_count + (size_t)A.parity * A.ncell, blockIdx.x * blockDim.x + threadIdx.x);
}

// quaternion to rotation matrix (demsolver/utils.py:34-61)
__device__ M3 quat2rot(const double *q) {
    const double w2 = q[0] * q[0], i2 = q[1] * q[1], j2 = q[2] * q[2], k2 = q[3] * q[3];
    const double twoij = 2.0 * q[1] * q[2], twoik = 2.0 * q[1] * q[3], twojk = 2.0 * q[2] * q[3];
    const double twoiw = 2.0 * q[1] * q[0], twojw = 2.0 * q[2] * q[0], twokw = 2.0 * q[3] * q[0];
    M3 r;
    r.m[0][0] = w2 + i2 - j2 - k2; r.m[0][1] = twoij - twokw; r.m[0][2] = twojw + twoik;
    r.m[1][0] = twoij + twokw; r.m[1][1] = w2 - i2 + j2 - k2; r.m[1][2] = twojk - twoiw;
    r.m[2][0] = twoik - twojw; r.m[2][1] = twojk + twoiw; r.m[2][2] = w2 - i2 - j2 + k2;
    return r;
}

// Euler rotation update (demsolver.py:590-636) on values already in registers:
// q (4), w (3), wd (3, previous angular acceleration), moment (3), inertia (9).
__device__ void rotate_update(double dt, double q[4], double w[3], double wd[3], const double mom[3],
                              const double inertia[9]) {
    const M3 Rm = quat2rot(q);
    M3 I;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) I.m[r][c] = inertia[3 * r + c];
    double ml[3], wl[3], Iw[3], cw[3], rhs[3], wdl[3], alpha[3];
    mv(Rm, mom, ml);
    mv(Rm, w, wl);
    mv(I, wl, Iw);
    cross3(wl, Iw, cw);
    for (int t = 0; t < 3; ++t) rhs[t] = ml[t] - cw[t];
    mv(inv3(I), rhs, wdl);
    mv(inv3(Rm), wdl, alpha);
    for (int t = 0; t < 3; ++t) w[t] += 0.5 * (wd[t] + alpha[t]) * dt;
    const double dq0 = -0.5 * (q[1] * w[0] + q[2] * w[1] + q[3] * w[2]);
    const double dq1 = +0.5 * (q[0] * w[0] - q[3] * w[1] + q[2] * w[2]);
    const double dq2 = +0.5 * (q[3] * w[0] + q[0] * w[1] + q[1] * w[2]);
    const double dq3 = +0.5 * (-q[2] * w[0] + q[1] * w[1] + q[0] * w[2]);
    q[0] += dq0 * dt; q[1] += dq1 * dt; q[2] += dq2 * dt; q[3] += dq3 * dt;
    const double ql = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int t = 0; t < 4; ++t) q[t] = q[t] / ql;
    for (int t = 0; t < 3; ++t) wd[t] = alpha[t];
}

__device__ __forceinline__ void wrap_position(const lbdem_dem &d, double *p) {
    // demsolver.py:451-480
    for (int a = 0; a < 3; ++a) {
        if (!d.periodic[a]) continue;
        const double L = d.dom_max[a] - d.dom_min[a];
        if (p[a] > d.dom_max[a]) p[a] = p[a] - L;
        else if (p[a] < d.dom_min[a]) p[a] = p[a] + L;
    }
}

__device__ void integrate_particle(const lbdem_dem &d, int ncell, int parity, int i, int role);
__device__ __forceinline__ void integrate_unit(const lbdem_dem &d, int ncell, int parity, int u);

__global__ void __launch_bounds__(128) k_integrate(const __grid_constant__ DemArgs A) {
    const lbdem_dem &d = A.d;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    // clear the counts consumed by this sub-step (the other half receives the new binning)
    int32_t *used = d.cell_count + (size_t)A.parity * A.ncell;
    for (int c = tid; c < A.ncell; c += gridDim.x * blockDim.x) used[c] = 0;
    if (tid < 3 * d.n) integrate_unit(d, A.ncell, A.parity, tid);
}

__device__ void integrate_particle(const lbdem_dem &d, int ncell, int parity, int i, int role) {
    const double dt = d.dt;
    const int frozen = d.freeze[i], fixed = d.fixvel[i];
    if (role == 0) {
        // clear_state (demsolver.py:422-429) + contacts, then apply_body_force (:437-448): the force;
        // update (demsolver.py:514-589): translation; then the binning for the next sub-step.  Every
        // input is fetched before any store, so the loads overlap.
        double af[3], ffl[3], p[3], v[3], acc[3];
        for (int t = 0; t < 3; ++t) {
            af[t] = d.acc_force[3 * i + t];
            ffl[t] = d.force_fluid[3 * i + t];
            p[t] = d.pos[3 * i + t];
            v[t] = d.vel[3 * i + t];
            acc[t] = d.acc[3 * i + t];
        }
        const double mass = d.mass[i];
        double force[3];
        for (int t = 0; t < 3; ++t) {
            double f = af[t];
            f += mass * d.g[t];
            f += ffl[t];
            force[t] = f;
        }
        if (!frozen) {
            if (fixed) {
                for (int t = 0; t < 3; ++t) p[t] += v[t] * dt;
                wrap_position(d, p);
            } else {
                double a[3];
                for (int t = 0; t < 3; ++t) a[t] = force[t] / mass;
                for (int t = 0; t < 3; ++t) v[t] += 0.5 * (acc[t] + a[t]) * dt;
                for (int t = 0; t < 3; ++t) p[t] += v[t] * dt + 0.5 * a[t] * (dt * dt);
                wrap_position(d, p);
                for (int t = 0; t < 3; ++t) acc[t] = a[t];
            }
        }
        for (int t = 0; t < 3; ++t) {
            d.acc_force[3 * i + t] = 0.0;
            d.force[3 * i + t] = force[t];
            d.pos[3 * i + t] = p[t];
            d.vel[3 * i + t] = v[t];
            d.acc[3 * i + t] = acc[t];
        }
        // bin the new position for the next sub-step
        int ijk[3];
        ref_cell(d, p, ijk);
        const int c = cell_index(d, ijk[0], ijk[1], ijk[2]);
        if (c < 0) {
            atomicOr(d.status, (int)LBDEM_ST_GRID_OVERFLOW);
            return;
        }
        int32_t *count = d.cell_count + (size_t)(parity ^ 1) * ncell;
        const int rank = atomicAdd(count + c, 1);
        if (rank < d.cell_cap) d.cell_list[(size_t)c * d.cell_cap + rank] = i;
        else atomicOr(d.status, (int)LBDEM_ST_CELL_OVERFLOW);
    } else if (role == 1) {
        // the moment and the Euler rotation update (demsolver.py:590-636)
        double am[3], mfl[3], w[3], wd[3], q[4], I[9];
        for (int t = 0; t < 3; ++t) {
            am[t] = d.acc_moment[3 * i + t];
            mfl[t] = d.moment_fluid[3 * i + t];
            w[t] = d.omega[3 * i + t];
            wd[t] = d.omega_dot[3 * i + t];
        }
        for (int t = 0; t < 4; ++t) q[t] = d.quat[4 * i + t];
        for (int t = 0; t < 9; ++t) I[t] = d.inertia[9 * i + t];
        double moment[3];
        for (int t = 0; t < 3; ++t) {
            double m = am[t];
            m += 0.0;
            m += mfl[t];
            moment[t] = m;
        }
        if (!frozen) rotate_update(dt, q, w, wd, moment, I);
        for (int t = 0; t < 3; ++t) {
            d.acc_moment[3 * i + t] = 0.0;
            d.moment[3 * i + t] = moment[t];
            d.omega[3 * i + t] = w[t];
            d.omega_dot[3 * i + t] = wd[t];
        }
        for (int t = 0; t < 4; ++t) d.quat[4 * i + t] = q[t];
    } else {
        // late_clear_state / remove_inactive_contact (demsolver.py:371-386, 431-436):
        // slots are only moved when an inactive one precedes an active one
        const size_t base = (size_t)i * d.maxc;
        const int nfirst = d.cfn[i], nadd = d.cf_add[i];
        int act[SLOTS_IN_REGS];
#pragma unroll
        for (int o = 0; o < SLOTS_IN_REGS; ++o) act[o] = o < d.maxc ? d.cf_active[base + o] : 0;
        const int cnt = min(nfirst + nadd, d.maxc);
        int w_ = 0;
        auto keep = [&](int o) {
            if (w_ != o) {
                const size_t dd = base + w_, ss = base + o;
                d.cf_j[dd] = d.cf_j[ss];
                d.cf_active[dd] = 1;
                for (int t = 0; t < 3; ++t) {
                    d.cf_shear[3 * dd + t] = d.cf_shear[3 * ss + t];
                    d.cf_pos[3 * dd + t] = d.cf_pos[3 * ss + t];
                    d.cf_force[3 * dd + t] = d.cf_force[3 * ss + t];
                }
            }
            ++w_;
        };
#pragma unroll
        for (int o = 0; o < SLOTS_IN_REGS; ++o)
            if (o < cnt && act[o]) keep(o);
        for (int o = SLOTS_IN_REGS; o < cnt; ++o)
            if (d.cf_active[base + o]) keep(o);
        for (int o = w_; o < cnt; ++o) d.cf_active[base + o] = 0;
        d.cfn[i] = w_;
        d.cf_add[i] = 0;
    }
}

// Integration of unit u of 3 n: role u / n (0 translation and binning, 1
// rotation, 2 contact-slot compaction) of particle u % n.  The three parts
// read and write disjoint state, so they run as three independent chains in
// different warps.
__device__ __forceinline__ void integrate_unit(const lbdem_dem &d, int ncell, int parity, int u) {
    const int role = u / d.n;
    integrate_particle(d, ncell, parity, u - role * d.n, role);
}

// All sub-steps of one call in ONE launch: a single thread-block cluster (up
// to 16 CTAs) grid-strides over the contact lanes, then over the particles;
// the two phases of every sub-step are separated by hardware cluster
// barriers (barrier.cluster arrive.release / wait.acquire), which order the
// global-memory writes of one phase before the reads of the next for every
// thread of the cluster.  Same per-lane/per-particle code as the two kernels.
template <bool WRAP>
__global__ void __launch_bounds__(512) k_dem_cluster(const __grid_constant__ DemArgs A, int nsub) {
    cg::cluster_group cl = cg::this_cluster();
    const lbdem_dem &d = A.d;
    const int nthr = (int)cl.num_threads();
    const int me = (int)cl.thread_rank();
    const int nlanes = 8 * d.n;
    for (int s = 0; s < nsub; ++s) {
        const int parity = (A.parity + s) & 1;
        const int32_t *count = d.cell_count + (size_t)parity * A.ncell;
        for (int base = 0; base < nlanes; base += nthr) contact_lane<WRAP>(A, count, base + me);
        cl.sync();
        int32_t *used = d.cell_count + (size_t)parity * A.ncell;
        for (int c = me; c < A.ncell; c += nthr) used[c] = 0;
        for (int u = me; u < 3 * d.n; u += nthr) integrate_unit(d, A.ncell, parity, u);
        cl.sync();
    }
}

// All sub-steps in one 128-thread block (at most 16 particles): the phases are
// separated by __syncthreads, which orders the block's global-memory writes of
// one phase before the reads of the next; the same per-lane/per-particle code
// without the cluster form's register cap (512 threads), so nothing spills.
template <bool WRAP>
__global__ void __launch_bounds__(128) k_dem_block(const __grid_constant__ DemArgs A, int nsub) {
    const lbdem_dem &d = A.d;
    const int nthr = (int)blockDim.x, me = (int)threadIdx.x;
    const int nlanes = 8 * d.n;
    for (int s = 0; s < nsub; ++s) {
        const int parity = (A.parity + s) & 1;
        const int32_t *count = d.cell_count + (size_t)parity * A.ncell;
        for (int base = 0; base < nlanes; base += nthr) contact_lane<WRAP>(A, count, base + me);
        __syncthreads();
        int32_t *used = d.cell_count + (size_t)parity * A.ncell;
        for (int c = me; c < A.ncell; c += nthr) used[c] = 0;
        for (int u = me; u < 3 * d.n; u += nthr) integrate_unit(d, A.ncell, parity, u);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// All sub-steps of one call in ONE cooperative launch (the default): every
// block of the grid is resident (cudaLaunchCooperativeKernel), the contact
// lanes and the particles are grid-strided, and the two phases of each
// sub-step are separated by a grid barrier.  The barrier is an arrival counter
// in caller-owned memory (zeroed before each launch); its wait is bounded:
// after ~0.25 s without progress it sets LBDEM_ST_WAIT_TIMEOUT and continues,
// so a fault can never hang the GPU.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void red_release_gpu(unsigned *p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Arrivals count up monotonically in sync[0] (zeroed before each launch): the
// k-th barrier is passed when the count reaches k * gridDim.x.  One release
// reduction per block and barrier (after the block barrier, which orders the
// block's writes of the phase before thread 0, so the release publishes them
// all), then polling with acquire loads; no reset.
__device__ __forceinline__ void grid_barrier(uint32_t *sync, unsigned &gen, int32_t *status) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = (gen + 1) * gridDim.x;
        red_release_gpu(sync, 1u);
        unsigned it = 0;
        while (ld_acquire_gpu(sync) < target) {
            if (++it > (1u << 22)) {
                atomicOr(status, (int)LBDEM_ST_WAIT_TIMEOUT);
                break;
            }
            __nanosleep(32);
        }
    }
    gen += 1;
    __syncthreads();
}

template <bool WRAP>
__global__ void __launch_bounds__(128, 1) k_dem_coop(const __grid_constant__ DemArgs A, int nsub) {
    const lbdem_dem &d = A.d;
    const int nthr = gridDim.x * blockDim.x;
    const int me = blockIdx.x * blockDim.x + threadIdx.x;
    const int nlanes = 8 * d.n;
    unsigned gen = 0;
    for (int s = 0; s < nsub; ++s) {
        const int parity = (A.parity + s) & 1;
        const int32_t *count = d.cell_count + (size_t)parity * A.ncell;
        for (int base = 0; base < nlanes; base += nthr) contact_lane<WRAP>(A, count, base + me);
        grid_barrier(d.sync, gen, d.status);
        int32_t *used = d.cell_count + (size_t)parity * A.ncell;
        for (int c = me; c < A.ncell; c += nthr) used[c] = 0;
        for (int u = me; u < 3 * d.n; u += nthr) integrate_unit(d, A.ncell, parity, u);
        grid_barrier(d.sync, gen, d.status);
    }
}

// The per-material Hertz constants of DemArgs, in the operation order of
// hertz.py:45-97 (particle-particle: the restitution 0.5 (e + e)) and
// hertz.py:99-153 (particle-wall).
static void contact_constants(DemArgs &A) {
    const lbdem_dem &d = A.d;
    for (int tj = 0; tj < 2; ++tj) {
        A.hz_ys[tj] = 1.0 / ((1.0 - d.nu[0] * d.nu[0]) / d.E[0] + (1.0 - d.nu[tj] * d.nu[tj]) / d.E[tj]);
        A.hz_gs[tj] = 1.0 / (2.0 * (2.0 - d.nu[0]) * (1.0 + d.nu[0]) / d.E[0] +
                             2.0 * (2.0 - d.nu[tj]) * (1.0 + d.nu[tj]) / d.E[tj]);
        const double e = tj == 0 ? 0.5 * (d.e[0] + d.e[0]) : d.e[1];
        const double lne = log(e);
        A.hz_beta[tj] = lne / sqrt(lne * lne + M_PI * M_PI);
    }
}

static int check_dem(const lbdem_dem *D) {
    if (!D || D->n < 0 || D->maxc < 0 || !D->status) {
        set_error("dem: bad descriptor");
        return LBDEM_ERR_ARG;
    }
    if (D->n > 0 && (!D->pos || !D->vel || !D->cell_count ||
                     !D->cfn || !D->cf_add || !D->wcf_active || !D->acc_force || !D->acc_moment || !D->cell_list ||
                     D->cell_cap <= 0)) {
        set_error("dem: missing buffers");
        return LBDEM_ERR_ARG;
    }
    if (D->gdim[0] <= 0 || D->gdim[1] <= 0 || D->gdim[2] <= 0 || !(D->cell_size > 0.0)) {
        set_error("dem: bad broad-phase grid");
        return LBDEM_ERR_ARG;
    }
    if (D->wrap_pairs)
        for (int a = 0; a < 3; ++a)
            if (D->periodic[a] && D->dom_max[a] - D->dom_min[a] < 4.0 * D->cell_size) {
                // a pair must not be reachable both directly and through an image
                set_error("dem: periodic images need every periodic length >= 4 broad-phase cells (axis %d)", a);
                return LBDEM_ERR_ARG;
            }
    return LBDEM_OK;
}

}  // namespace lbdem

using namespace lbdem;

extern "C" {

// (Re)bin the current positions into the active half of cell_count.
int lbdem_dem_bin(lbdem_dem *D, void *stream) {
    int rc = check_dem(D);
    if (rc) return rc;
    if (D->n == 0) return LBDEM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    DemArgs A;
    A.d = *D;
    A.ncell = D->gdim[0] * D->gdim[1] * D->gdim[2];
    A.parity = D->parity;
    if (cudaMemsetAsync(D->cell_count + (size_t)A.parity * A.ncell, 0, sizeof(int32_t) * A.ncell, st) != cudaSuccess)
        return check_launch("dem_bin memset");
    k_bin<<<(D->n + 127) / 128, 128, 0, st>>>(A);
    return check_launch("dem_bin");
}

static thread_local int g_dem_launches = 0;

// Cooperative-launch support, SM count and resident blocks per SM of the
// cooperative kernel (128 threads, no dynamic shared memory) on device `dev`:
// constant for a device, so looked up once per device and form (the host
// launch of every call would otherwise repeat three driver queries).
static bool coop_residency(int dev, bool wrap, const void *kcoop, int &coop, int &nsm, int &per_sm) {
    constexpr int MAXDEV = 64;
    static std::mutex mu;
    static int cached[2][MAXDEV][3];
    static bool have[2][MAXDEV] = {};
    if (dev < 0 || dev >= MAXDEV) return false;
    std::lock_guard<std::mutex> lock(mu);
    if (!have[wrap][dev]) {
        int c = 0, n = 0, p = 0;
        cudaDeviceGetAttribute(&c, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, kcoop, 128, 0) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cached[wrap][dev][0] = c;
        cached[wrap][dev][1] = n;
        cached[wrap][dev][2] = p;
        have[wrap][dev] = true;
    }
    coop = cached[wrap][dev][0];
    nsm = cached[wrap][dev][1];
    per_sm = cached[wrap][dev][2];
    return true;
}

int lbdem_dem_launches_last(void) { return g_dem_launches; }

int lbdem_dem_substeps(lbdem_dem *D, int32_t nsub, void *stream) {
    g_dem_launches = 0;
    int rc = check_dem(D);
    if (rc) return rc;
    if (D->n == 0 || nsub <= 0) return LBDEM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    DemArgs A;
    A.d = *D;
    A.ncell = D->gdim[0] * D->gdim[1] * D->gdim[2];
    contact_constants(A);
    const int nb_int = max((3 * D->n + 127) / 128, min(148, (A.ncell + 127) / 128));   // 3 units per particle
    const int nb_con = (int)((8ll * D->n + 127) / 128);
    // "cluster": all sub-steps in one launch of a single thread-block cluster
    // (opt-in: it confines the contact phase to <= 16 SMs and measured slower
    // than two launches per sub-step spread over the whole GPU).  It is the
    // default when one 512-thread block holds every contact lane (n <= 64):
    // block barriers instead of grid barriers (one sphere: 90 us for 10
    // sub-steps against 107 us cooperative).
    const char *mode = getenv("LBDEM_DEM_KERNELS");
    const bool wrap = D->wrap_pairs != 0;
    auto *kcl = wrap ? k_dem_cluster<true> : k_dem_cluster<false>;
    auto *kcoop = wrap ? k_dem_coop<true> : k_dem_coop<false>;
    // (one block on one SM also runs beside a step on another stream)
    const bool one_block = !mode && 8ll * D->n <= 512;
    if (one_block && 8ll * D->n <= 128) {
        A.parity = D->parity;
        if (wrap) k_dem_block<true><<<1, 128, 0, st>>>(A, (int)nsub);
        else k_dem_block<false><<<1, 128, 0, st>>>(A, (int)nsub);
        D->parity ^= (nsub & 1);
        g_dem_launches = 1;
        return check_launch("dem_substeps (one block)");
    }
    if ((mode && strcmp(mode, "cluster") == 0) || one_block) {
        // one cluster of up to 16 CTAs x 512 threads, sized to the contact lanes
        int ncta = (int)((8ll * D->n + 511) / 512);
        ncta = ncta < 1 ? 1 : (ncta > 16 ? 16 : ncta);
        cudaFuncSetAttribute(kcl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        for (; ncta >= 1; ncta >>= 1) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(ncta, 1, 1);
            cfg.blockDim = dim3(512, 1, 1);
            cfg.dynamicSmemBytes = 0;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = ncta;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, kcl, &cfg) != cudaSuccess || nclusters < 1) {
                cudaGetLastError();
                continue;
            }
            A.parity = D->parity;
            if (cudaLaunchKernelEx(&cfg, kcl, A, (int)nsub) == cudaSuccess) {
                D->parity ^= (nsub & 1);
                g_dem_launches = 1;
                return check_launch("dem_substeps (cluster)");
            }
            cudaGetLastError();
        }
    }
    // default: one cooperative launch for all sub-steps when one resident wave
    // covers the contact lanes ("split" forces two launches per sub-step)
    if (D->sync && !(mode && strcmp(mode, "split") == 0)) {
        int dev = 0, coop = 0, nsm = 0, per_sm = 0;
        cudaGetDevice(&dev);
        if (coop_residency(dev, wrap, (const void *)kcoop, coop, nsm, per_sm) && coop && per_sm > 0) {
            // one resident wave must cover every contact lane: beyond that the
            // grid-stride loop serialises the phases' memory-latency chains and
            // two launches per sub-step (all lanes in flight) are faster
            const int nb = max(nb_con, nb_int);
            // the arrival counter reaches 2 nsub nb within the launch: keep it far from wrapping
            if (nb <= per_sm * nsm && 2ll * nsub * nb < (1ll << 30)) {
                if (cudaMemsetAsync(D->sync, 0, 2 * sizeof(uint32_t), st) != cudaSuccess)
                    return check_launch("dem_substeps (barrier reset)");
                A.parity = D->parity;
                int nsub_arg = nsub;
                void *args[] = {&A, &nsub_arg};
                if (cudaLaunchCooperativeKernel((void *)kcoop, dim3(nb), dim3(128), args, 0, st) ==
                    cudaSuccess) {
                    D->parity ^= (nsub & 1);
                    g_dem_launches = 1;
                    return check_launch("dem_substeps (cooperative)");
                }
            }
        }
        cudaGetLastError();
    }
    // two launches per sub-step, in 64-thread blocks: each block's registers
    // (~10 K) fit in the room one retiring block of the fused step frees, so
    // the sub-steps can interleave with a step running on another stream
    const int nb_con64 = (int)((8ll * D->n + 63) / 64), nb_int64 = 2 * nb_int;
    for (int s = 0; s < nsub; ++s) {
        A.parity = D->parity;
        if (wrap) k_contacts<true><<<nb_con64, 64, 0, st>>>(A);
        else k_contacts<false><<<nb_con64, 64, 0, st>>>(A);
        k_integrate<<<nb_int64, 64, 0, st>>>(A);
        D->parity ^= 1;
    }
    g_dem_launches = 2 * nsub;
    return check_launch("dem_substeps");
}

}  // extern "C"
