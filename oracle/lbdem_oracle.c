/*
 * FP64 CPU restatement of the reference's resolved LBM-DEM step
 * (dasfadwqd/LBDEM-Taichi, src/).  TEST INFRASTRUCTURE ONLY: it is the parity
 * checker for the CUDA library and the CPU baseline timed by bench.py; the
 * product never links or calls it.
 *
 * Pinned against golden vectors produced by the reference's own Python source
 * (tests/golden/make_golden.py runs src/ under a NumPy Taichi stand-in).
 *
 * Layout mirrors Taichi's dense fields: cell (i,j,k) -> (i*Ny + j)*Nz + k,
 * k fastest; vector members are contiguous per cell (19 for populations,
 * 3 for velocities).
 *
 * Each function cites the reference lines it restates.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define Q 19

/* lbm_solver3d.py:46-47, 60-91 */
static const int QINV[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const int QSYX[Q] = {0, 2, 1, 3, 4, 5, 6, 10, 9, 8, 7, 14, 13, 12, 11, 15, 16, 17, 18};
static const int QSYY[Q] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15};
static const int QSYZ[Q] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};
static const double CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const double CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const double CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const double W[Q] = {1. / 3., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18.,
                            1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.,
                            1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
static const double CSSQ = 1.0 / 3.0;

/* lbmutils.py:69-97 */
enum {
    CT_FLUID = 1, CT_OBSTACLE = 8, CT_FREE_SLIP = 16, CT_VEL_LADD = 32, CT_VEL_ZOUHE = 64,
    CT_VEL_EXIT = 128, CT_PRE_ZOUHE = 256, CT_RIGHT = 4096, CT_LEFT = 8192, CT_TOP = 16384,
    CT_BOTTOM = 32768, CT_FRONT = 65536, CT_BACK = 131072, CT_VEL_INLET_LADD = 262144
};

typedef struct {
    int nx, ny, nz;
    double omega0;
    double dx, dt, rho_unit;    /* UnitConverter(dx, dt, rho) */
    double smag_cs;             /* BasicLattice3D.SmagorinskyConstant */
    int smag;                   /* 1: computeOmega before compute_feq */
    int psc;                    /* 1: PSC weighted collision on cells with volfrac>0 */
    int force_on;               /* 1: ForcedLattice3D source term added to fpc */
    double force[3];            /* body force in lattice units */
    int skip_inlet;             /* 1: collide/initialize/map also skip VEL_INLET_LADD */
    double xmin, ymin, zmin;    /* DEM config.domain minimum */
    /* fields (owned by the caller) */
    int32_t *ct;
    double *f, *fpc, *feq, *rho, *vel, *omega;
    int32_t *id;
    double *volfrac, *weight, *velsolid, *hydroforce;
} orc_lat;

typedef struct {
    int n;
    const double *pos, *radius, *vel, *omega;   /* physical units */
    double *force_fluid, *moment_fluid;
} orc_grains;

static inline long cidx(const orc_lat *L, int i, int j, int k) {
    return ((long)i * L->ny + j) * L->nz + k;
}

static inline int skip_cell(const orc_lat *L, int32_t ct) {
    int32_t m = CT_OBSTACLE | CT_VEL_LADD | CT_FREE_SLIP;
    if (L->skip_inlet) m |= CT_VEL_INLET_LADD;
    return (ct & m) != 0;
}

/* lbm_solver3d.py:255-271 */
static void compute_feq(const orc_lat *L, long c) {
    const double *u = L->vel + 3 * c;
    double uv = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int q = 0; q < Q; q++) {
        double cu = CX[q] * u[0] + CY[q] * u[1] + CZ[q] * u[2];
        L->feq[Q * c + q] = W[q] * L->rho[c] * (1.0 + 3.0 * cu + 4.5 * (cu * cu) - 1.5 * uv);
    }
}

/* lbm_solver3d.py:460-513 (uses the feq stored by the previous collide) */
static void compute_omega(const orc_lat *L, long c) {
    double xx = 0, yy = 0, zz = 0, xy = 0, xz = 0, yz = 0;
    for (int q = 0; q < Q; q++) {
        double fn = L->f[Q * c + q] - L->feq[Q * c + q];
        xx += fn * CX[q] * CX[q];
        yy += fn * CY[q] * CY[q];
        zz += fn * CZ[q] * CZ[q];
        xy += fn * CX[q] * CY[q];
        xz += fn * CX[q] * CZ[q];
        yz += fn * CY[q] * CZ[q];
    }
    double pi = sqrt(2.0 * (xx * xx + yy * yy + zz * zz + 2.0 * (xy * xy + xz * xz + yz * yz)));
    double rate = L->omega[c] / (2.0 * CSSQ * L->rho[c]) * pi;
    double cs = L->smag_cs * 1.0;
    double nut = cs * cs * rate;
    double taueff = 1.0 / L->omega0 + nut / CSSQ;
    L->omega[c] = 1.0 / taueff;
}

/* lbm_solver3d.py:157-171, psclattice3d.py:60-75 */
void orc_initialize(orc_lat *L) {
    long nc = (long)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
        if (skip_cell(L, L->ct[c])) continue;
        compute_feq(L, c);
        for (int q = 0; q < Q; q++) L->f[Q * c + q] = L->feq[Q * c + q];
    }
}

/* psclattice3d.py:160-182 */
static void solid_vel(const orc_lat *L, const orc_grains *G, long c, int i, int j, int k, int gid,
                      double xc, double yc, double zc) {
    double r[3] = {((double)i - xc) * L->dx, ((double)j - yc) * L->dx, ((double)k - zc) * L->dx};
    const double *w = G->omega + 3 * gid;
    double oc[3] = {w[1] * r[2] - w[2] * r[1], w[2] * r[0] - w[0] * r[2], w[0] * r[1] - w[1] * r[0]};
    for (int a = 0; a < 3; a++)
        L->velsolid[3 * c + a] = (G->vel[3 * gid + a] + oc[a]) * L->dt / L->dx;
}

/* psclattice3d.py:84-138 (grains visited in id order; first full cover wins
 * and breaks; a partial cover replaces the owner only on a strictly larger
 * sub-sample count).  The weighting factor B is computed in orc_collide from
 * the relaxation frequency in force at collision time (hybridlattice.py:236-245,
 * which equals psclattice3d.py:144-155 whenever omega is not updated). */
/* The body of the reference's per-cell grain loop (psclattice3d.py:100-138)
 * for one grain g; returns 1 when the loop breaks (full cover). */
static inline int map_visit(orc_lat *L, const orc_grains *G, long c, int i, int j, int k, int g) {
    const double half_diag = 0.5 * sqrt(3.0);
    double xc = (G->pos[3 * g + 0] - L->xmin + 0.5 * L->dx) / L->dx;
    double yc = (G->pos[3 * g + 1] - L->ymin + 0.5 * L->dx) / L->dx;
    double zc = (G->pos[3 * g + 2] - L->zmin + 0.5 * L->dx) / L->dx;
    double r = (G->radius[g] - 0.5 * L->dx) / L->dx;
    double dxv = xc - i, dyv = yc - j, dzv = zc - k;
    double dist = sqrt(dxv * dxv + dyv * dyv + dzv * dzv);
    if (dist >= r + half_diag) return 0;
    if (dist <= r - half_diag) {
        L->id[c] = g;
        L->volfrac[c] = 1.0;
        solid_vel(L, G, c, i, j, k, g, xc, yc, zc);
        return 1;
    }
    int cnt = 0;
    for (int ii = 0; ii < 5; ii++)
        for (int jj = 0; jj < 5; jj++)
            for (int kk = 0; kk < 5; kk++) {
                double sx = xc - ((double)i - 0.4 + 0.2 * ii);
                double sy = yc - ((double)j - 0.4 + 0.2 * jj);
                double sz = zc - ((double)k - 0.4 + 0.2 * kk);
                if (sqrt(sx * sx + sy * sy + sz * sz) < r) cnt++;
            }
    double eps = cnt / 125.0;
    if (eps > L->volfrac[c]) {
        L->id[c] = g;
        L->volfrac[c] = eps;
        solid_vel(L, G, c, i, j, k, g, xc, yc, zc);
    }
    return 0;
}

static inline void map_reset(orc_lat *L, long c) {
    L->id[c] = -1;
    L->volfrac[c] = 0.0;
    L->weight[c] = 0.0;
    L->velsolid[3 * c] = L->velsolid[3 * c + 1] = L->velsolid[3 * c + 2] = 0.0;
}

/* The reference's form: every cell visits every grain in id order. */
void orc_grains2lattice_all(orc_lat *L, const orc_grains *G) {
    long nc = (long)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(dynamic, 64)
    for (long c = 0; c < nc; c++) {
        int i = (int)(c / ((long)L->ny * L->nz));
        int j = (int)((c / L->nz) % L->ny);
        int k = (int)(c % L->nz);
        map_reset(L, c);
        if (skip_cell(L, L->ct[c])) continue;
        for (int g = 0; g < G->n; g++)
            if (map_visit(L, G, c, i, j, k, g)) break;
    }
}

/* Same result as orc_grains2lattice_all at a cost that does not grow with
 * cells x grains: each cell visits, in id order, only the grains listed for
 * its 8^3-cell bin.  A grain is listed for every bin that meets the box
 * [c - reach - 1, c + reach + 1] around its lattice centre c, reach = r +
 * sqrt(3)/2; every cell outside that box has dist >= reach, which is exactly
 * the reference's skip test (psclattice3d.py:110), so the grains left out are
 * the ones whose visit would `continue` -- the visits that remain, their order
 * and the break are unchanged.  A grain with reach <= 0 or a non-finite centre
 * is skipped by the reference for every cell (and changes no cell) and is
 * listed nowhere; an infinite reach lists the grain everywhere. */
#define MAP_BIN 8
void orc_grains2lattice(orc_lat *L, const orc_grains *G) {
    const int bx = (L->nx + MAP_BIN - 1) / MAP_BIN, by = (L->ny + MAP_BIN - 1) / MAP_BIN,
              bz = (L->nz + MAP_BIN - 1) / MAP_BIN;
    const long nbin = (long)bx * by * bz;
    const double half_diag = 0.5 * sqrt(3.0);
    long *start = (long *)calloc((size_t)nbin + 1, sizeof(long));
    int *lo = (int *)malloc(sizeof(int) * 6 * (size_t)(G->n > 0 ? G->n : 1));
    for (int g = 0; g < G->n; g++) {
        double c3[3] = {(G->pos[3 * g + 0] - L->xmin + 0.5 * L->dx) / L->dx,
                        (G->pos[3 * g + 1] - L->ymin + 0.5 * L->dx) / L->dx,
                        (G->pos[3 * g + 2] - L->zmin + 0.5 * L->dx) / L->dx};
        double reach = (G->radius[g] - 0.5 * L->dx) / L->dx + half_diag;
        const int nn[3] = {L->nx, L->ny, L->nz};
        int *b = lo + 6 * g;
        int empty = !(reach > 0.0) || !isfinite(c3[0]) || !isfinite(c3[1]) || !isfinite(c3[2]);
        for (int a = 0; a < 3 && !empty; a++) {
            double l = floor(c3[a] - reach) - 1.0, h = ceil(c3[a] + reach) + 1.0;
            if (h < 0.0 || l > (double)(nn[a] - 1)) { empty = 1; break; }
            int il = l < 0.0 ? 0 : (int)l, ih = h > (double)(nn[a] - 1) ? nn[a] - 1 : (int)h;
            b[2 * a] = il / MAP_BIN;
            b[2 * a + 1] = ih / MAP_BIN;
        }
        if (empty) { b[0] = 1; b[1] = 0; continue; }
        for (int x = b[0]; x <= b[1]; x++)
            for (int y = b[2]; y <= b[3]; y++)
                for (int z = b[4]; z <= b[5]; z++) start[((long)x * by + y) * bz + z + 1]++;
    }
    for (long t = 0; t < nbin; t++) start[t + 1] += start[t];
    int *list = (int *)malloc(sizeof(int) * (size_t)(start[nbin] > 0 ? start[nbin] : 1));
    long *fill = (long *)malloc(sizeof(long) * (size_t)nbin);
    memcpy(fill, start, sizeof(long) * (size_t)nbin);
    for (int g = 0; g < G->n; g++) {   /* ascending g: every list is in id order */
        const int *b = lo + 6 * g;
        if (b[0] > b[1]) continue;
        for (int x = b[0]; x <= b[1]; x++)
            for (int y = b[2]; y <= b[3]; y++)
                for (int z = b[4]; z <= b[5]; z++) list[fill[((long)x * by + y) * bz + z]++] = g;
    }
    long nc = (long)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(dynamic, 64)
    for (long c = 0; c < nc; c++) {
        int i = (int)(c / ((long)L->ny * L->nz));
        int j = (int)((c / L->nz) % L->ny);
        int k = (int)(c % L->nz);
        map_reset(L, c);
        if (skip_cell(L, L->ct[c])) continue;
        long t = ((long)(i / MAP_BIN) * by + j / MAP_BIN) * bz + k / MAP_BIN;
        for (long e = start[t]; e < start[t + 1]; e++)
            if (map_visit(L, G, c, i, j, k, list[e])) break;
    }
    free(fill);
    free(list);
    free(lo);
    free(start);
}

/* psclattice3d.py:187-261 (PSC), hybridlattice.py:450-503 (PSC after
 * computeOmega), lbm_solver3d.py:176-192 (BGK + Smagorinsky),
 * lbm_foecelover.py:136-165 (body-force term, added after the blend). */
void orc_collide(orc_lat *L) {
    long nc = (long)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
        double *h = L->hydroforce ? L->hydroforce + 3 * c : NULL;
        if (h) h[0] = h[1] = h[2] = 0.0;
        if (skip_cell(L, L->ct[c])) continue;
        if (L->smag) compute_omega(L, c);
        compute_feq(L, c);
        const double *f = L->f + Q * c;
        const double *feq = L->feq + Q * c;
        double *fpc = L->fpc + Q * c;
        double om = L->omega[c];
        if (L->psc && L->volfrac[c] > 0) {
            double eps = L->volfrac[c];
            double taum = 1.0 / om - 0.5;
            double B = (eps * taum) / ((1.0 - eps) + taum);
            L->weight[c] = B;
            const double *us = L->velsolid + 3 * c;
            double uv = us[0] * us[0] + us[1] * us[1] + us[2] * us[2];
            double feqs[Q];
            for (int q = 0; q < Q; q++) {
                double cu = CX[q] * us[0] + CY[q] * us[1] + CZ[q] * us[2];
                feqs[q] = W[q] * L->rho[c] * (1.0 + 3.0 * cu + 4.5 * (cu * cu) - 1.5 * uv);
            }
            for (int q = 0; q < Q; q++) {
                double oms = f[QINV[q]] - feq[QINV[q]] + feqs[q] - f[q];
                double omf = -om * (f[q] - feq[q]);
                fpc[q] = f[q] + B * oms + (1.0 - B) * omf;
                h[0] -= B * oms * CX[q];
                h[1] -= B * oms * CY[q];
                h[2] -= B * oms * CZ[q];
            }
        } else {
            for (int q = 0; q < Q; q++) fpc[q] = (1.0 - om) * f[q] + om * feq[q];
        }
        if (L->force_on) {
            for (int q = 0; q < Q; q++) {
                double cf = CX[q] * L->force[0] + CY[q] * L->force[1] + CZ[q] * L->force[2];
                fpc[q] += L->rho[c] * W[q] * cf / CSSQ;
            }
        }
    }
}

/* psclattice3d.py:316-358 */
void orc_lattice2grains(orc_lat *L, orc_grains *G) {
    double scale = (L->rho_unit * (L->dx * L->dx * L->dx * L->dx)) / (L->dt * L->dt);
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < G->n; g++) {
        double xc = (G->pos[3 * g + 0] - L->xmin + 0.5 * L->dx) / L->dx;
        double yc = (G->pos[3 * g + 1] - L->ymin + 0.5 * L->dx) / L->dx;
        double zc = (G->pos[3 * g + 2] - L->zmin + 0.5 * L->dx) / L->dx;
        double r = G->radius[g] / L->dx;
        int x0 = (int)(xc - r); if (x0 < 0) x0 = 0;
        int x1 = (int)(xc + r + 2); if (x1 > L->nx) x1 = L->nx;
        int y0 = (int)(yc - r); if (y0 < 0) y0 = 0;
        int y1 = (int)(yc + r + 2); if (y1 > L->ny) y1 = L->ny;
        int z0 = (int)(zc - r); if (z0 < 0) z0 = 0;
        int z1 = (int)(zc + r + 2); if (z1 > L->nz) z1 = L->nz;
        double *F = G->force_fluid + 3 * g, *T = G->moment_fluid + 3 * g;
        F[0] = F[1] = F[2] = T[0] = T[1] = T[2] = 0.0;
        for (int i = x0; i < x1; i++)
            for (int j = y0; j < y1; j++)
                for (int k = z0; k < z1; k++) {
                    long c = cidx(L, i, j, k);
                    if (skip_cell(L, L->ct[c])) continue;
                    if (L->volfrac[c] > 0.0 && L->id[c] == g) {
                        double ff[3];
                        for (int a = 0; a < 3; a++) ff[a] = L->hydroforce[3 * c + a] * scale;
                        F[0] += ff[0]; F[1] += ff[1]; F[2] += ff[2];
                        double d[3] = {(xc - i) * L->dx, (yc - j) * L->dx, (zc - k) * L->dx};
                        T[0] += -(d[1] * ff[2] - d[2] * ff[1]);
                        T[1] += -(d[2] * ff[0] - d[0] * ff[2]);
                        T[2] += -(d[0] * ff[1] - d[1] * ff[0]);
                    }
                }
    }
}

/* Face of a boundary cell from its orientation bits, in the reference's
 * precedence LEFT, RIGHT, BOTTOM, TOP, BACK, FRONT (lbm_solver3d.py:522-527,
 * 647-658, 686-816, 831-960): axis a (0 x, 1 y, 2 z) and the inward sign s
 * (+1 for LEFT / BOTTOM / BACK, whose interior neighbour is at +1 along a). */
static int face_of(int32_t ct, int *a, int *s) {
    if (ct & CT_LEFT) { *a = 0; *s = 1; }
    else if (ct & CT_RIGHT) { *a = 0; *s = -1; }
    else if (ct & CT_BOTTOM) { *a = 1; *s = 1; }
    else if (ct & CT_TOP) { *a = 1; *s = -1; }
    else if (ct & CT_BACK) { *a = 2; *s = 1; }
    else if (ct & CT_FRONT) { *a = 2; *s = -1; }
    else return 0;
    return 1;
}

static inline double cq(int axis, int q) { return axis == 0 ? CX[q] : (axis == 1 ? CY[q] : CZ[q]); }

/* Zou-He non-equilibrium bounce-back, velocity (vel_zouHe,
 * lbm_solver3d.py:671-821) or pressure (pre_zouHe, :823-960), written once for
 * the six faces.  With K the populations with c_a = 0 and O those leaving the
 * domain (c_a = -s):
 *   velocity: rho = (sum K + 2 sum O) / (1 - s u_a), u = vel (preset);
 *   pressure: rho preset, u_a = s (1 - (sum K + 2 sum O) / rho) (stored in
 *             vel[a]); the unknowns use u = u_a e_a only;
 *   N_b = 1/2 sum_K c_b f - [velocity] rho u_b / 3   (each tangential b);
 *   unknown q (c_a = s): f_q = f_qbar + rho (c_q . u) / 3        on the axis,
 *                        f_q = f_qbar + rho (c_q . u) / 6 - c_qb N_b  diagonal. */
static void zou_he(orc_lat *L, long c, int32_t ct, int pressure) {
    int a, s;
    if (!face_of(ct, &a, &s)) return;
    double *f = L->f + Q * c;
    double *vel = L->vel + 3 * c;
    double K = 0.0, O = 0.0;
    for (int q = 0; q < Q; q++) {
        double ca = cq(a, q);
        if (ca == 0.0) K += f[q];
        else if (ca == -s) O += f[q];
    }
    double rho, u[3];
    if (pressure) {
        rho = L->rho[c];
        vel[a] = s * (1.0 - (K + 2.0 * O) / rho);
        u[0] = u[1] = u[2] = 0.0;
        u[a] = vel[a];
    } else {
        rho = (K + 2.0 * O) / (1.0 - s * vel[a]);
        L->rho[c] = rho;
        u[0] = vel[0]; u[1] = vel[1]; u[2] = vel[2];
    }
    double N[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < 3; b++) {
        if (b == a) continue;
        double t = 0.0;
        for (int q = 0; q < Q; q++)
            if (cq(a, q) == 0.0) t += cq(b, q) * f[q];
        N[b] = 0.5 * t - (pressure ? 0.0 : rho * u[b] / 3.0);
    }
    for (int q = 1; q < Q; q++) {
        if (cq(a, q) != s) continue;
        double cu = CX[q] * u[0] + CY[q] * u[1] + CZ[q] * u[2];
        int b = -1;
        for (int bb = 0; bb < 3; bb++)
            if (bb != a && cq(bb, q) != 0.0) b = bb;
        if (b < 0) f[q] = f[QINV[q]] + rho * cu / 3.0;
        else f[q] = f[QINV[q]] + rho * cu / 6.0 - cq(b, q) * N[b];
    }
}

/* Convective exit (bc_vel_exit, lbm_solver3d.py:645-663): velocity of the
 * interior neighbour, rho = 1, f = feq (compute_feq also stores feq). */
static void vel_exit(orc_lat *L, long c, int i, int j, int k, int32_t ct) {
    int a, s;
    if (!face_of(ct, &a, &s)) return;
    int n3[3] = {i, j, k};
    n3[a] += s;
    long n = cidx(L, n3[0], n3[1], n3[2]);
    for (int d = 0; d < 3; d++) L->vel[3 * c + d] = L->vel[3 * n + d];
    L->rho[c] = 1.0;
    compute_feq(L, c);
    for (int q = 0; q < Q; q++) L->f[Q * c + q] = L->feq[Q * c + q];
}

/* Ladd velocity inlet (bc_ladd_inlet, lbm_solver3d.py:516-527): the inlet's
 * density becomes that of its interior neighbour. */
static void ladd_inlet(orc_lat *L, long c, int i, int j, int k, int32_t ct) {
    int a, s;
    if (!face_of(ct, &a, &s)) return;
    int n3[3] = {i, j, k};
    n3[a] += s;
    L->rho[c] = L->rho[cidx(L, n3[0], n3[1], n3[2])];
}

/* lbm_solver3d.py:197-250, 276-303, 308-342: pull streaming with the
 * neighbour rules, moments of FLUID cells, then the wet-node boundary
 * conditions (:242-250) in a second pass over the lattice. */
void orc_stream(orc_lat *L) {
    int nx = L->nx, ny = L->ny, nz = L->nz;
    long nc = (long)nx * ny * nz;
    int32_t stream_skip = CT_OBSTACLE | CT_VEL_LADD | CT_FREE_SLIP | CT_VEL_INLET_LADD;
    int32_t prop = CT_FLUID | CT_VEL_ZOUHE | CT_VEL_EXIT | CT_PRE_ZOUHE;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
        int i = (int)(c / ((long)ny * nz));
        int j = (int)((c / nz) % ny);
        int k = (int)(c % nz);
        if (L->ct[c] & stream_skip) continue;
        double *f = L->f + Q * c;
        const double *fpc = L->fpc + Q * c;
        f[0] = fpc[0];
        for (int q = 1; q < Q; q++) {
            int in = (int)(i - CX[q]), jn = (int)(j - CY[q]), kn = (int)(k - CZ[q]);
            if (in >= nx) in = 0; else if (in < 0) in = nx - 1;
            if (jn >= ny) jn = 0; else if (jn < 0) jn = ny - 1;
            if (kn >= nz) kn = 0; else if (kn < 0) kn = nz - 1;
            long n = cidx(L, in, jn, kn);
            int32_t ctn = L->ct[n];
            if (ctn & prop) {
                f[q] = L->fpc[Q * n + q];
            } else if (ctn & CT_OBSTACLE) {
                f[q] = fpc[QINV[q]];
            } else if (ctn & CT_VEL_LADD) {
                const double *u = L->vel + 3 * n;
                double cu = CX[q] * u[0] + CY[q] * u[1] + CZ[q] * u[2];
                f[q] = fpc[QINV[q]] + 2.0 * W[q] * L->rho[c] * cu / CSSQ;
            } else if (ctn & CT_VEL_INLET_LADD) {
                const double *u = L->vel + 3 * n;
                double cu = CX[q] * u[0] + CY[q] * u[1] + CZ[q] * u[2];
                f[q] = fpc[QINV[q]] + 2.0 * W[q] * L->rho[n] * cu / CSSQ;
            } else if (ctn & CT_FREE_SLIP) {
                if (ctn & (CT_LEFT | CT_RIGHT))
                    f[q] = L->fpc[Q * cidx(L, i, jn, kn) + QSYX[q]];
                else if (ctn & (CT_BOTTOM | CT_TOP))
                    f[q] = L->fpc[Q * cidx(L, in, j, kn) + QSYY[q]];
                else if (ctn & (CT_BACK | CT_FRONT))
                    f[q] = L->fpc[Q * cidx(L, in, jn, k) + QSYZ[q]];
            }
        }
        if (L->ct[c] & CT_FLUID) {
            double r = 0, u0 = 0, u1 = 0, u2 = 0;
            for (int q = 0; q < Q; q++) {
                r += f[q];
                u0 += CX[q] * f[q];
                u1 += CY[q] * f[q];
                u2 += CZ[q] * f[q];
            }
            L->rho[c] = r;
            L->vel[3 * c] = u0 / r;
            L->vel[3 * c + 1] = u1 / r;
            L->vel[3 * c + 2] = u2 / r;
        }
    }
    /* second pass: the reference runs it as a parallel loop; each cell reads
     * only its own populations and its interior neighbour's moments */
    for (long c = 0; c < nc; c++) {
        int32_t ct = L->ct[c];
        if (!(ct & (CT_VEL_ZOUHE | CT_VEL_EXIT | CT_PRE_ZOUHE | CT_VEL_INLET_LADD))) continue;
        int i = (int)(c / ((long)ny * nz));
        int j = (int)((c / nz) % ny);
        int k = (int)(c % nz);
        if (ct & CT_VEL_ZOUHE) zou_he(L, c, ct, 0);
        else if (ct & CT_VEL_EXIT) vel_exit(L, c, i, j, k, ct);
        else if (ct & CT_PRE_ZOUHE) zou_he(L, c, ct, 1);
        else ladd_inlet(L, c, i, j, k, ct);
    }
}

/* lbm_solver3d.py:347-404: stress from the non-equilibrium part of the
 * post-stream populations against the equilibrium stored by the last collide,
 * sigma = -(1 - omega/2) sum c c (f - feq); out: 7 per cell (xx, yy, zz, xy,
 * xz, yz, von Mises shear magnitude); skipped cells are left untouched. */
void orc_compute_stress(const orc_lat *L, double *out) {
    long nc = (long)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
        if (L->ct[c] & (CT_OBSTACLE | CT_VEL_LADD | CT_FREE_SLIP | CT_VEL_INLET_LADD)) continue;
        double relax = 1.0 - 0.5 * L->omega[c];
        double xx = 0, yy = 0, zz = 0, xy = 0, xz = 0, yz = 0;
        for (int q = 0; q < Q; q++) {
            double fneq = L->f[Q * c + q] - L->feq[Q * c + q];
            xx += CX[q] * CX[q] * fneq;
            yy += CY[q] * CY[q] * fneq;
            zz += CZ[q] * CZ[q] * fneq;
            xy += CX[q] * CY[q] * fneq;
            xz += CX[q] * CZ[q] * fneq;
            yz += CY[q] * CZ[q] * fneq;
        }
        double *o = out + 7 * c;
        o[0] = -relax * xx; o[1] = -relax * yy; o[2] = -relax * zz;
        o[3] = -relax * xy; o[4] = -relax * xz; o[5] = -relax * yz;
        o[6] = sqrt(0.5 * (o[3] * o[3] + o[4] * o[4] + o[5] * o[5]));
    }
}

/* FP64 totals of mass and momentum over FLUID cells (for conservation checks). */
void orc_global_sums(const orc_lat *L, double *out4) {
    long nc = (long)L->nx * L->ny * L->nz;
    double m = 0, px = 0, py = 0, pz = 0;
#pragma omp parallel for reduction(+ : m, px, py, pz)
    for (long c = 0; c < nc; c++) {
        if (!(L->ct[c] & CT_FLUID)) continue;
        m += L->rho[c];
        px += L->rho[c] * L->vel[3 * c];
        py += L->rho[c] * L->vel[3 * c + 1];
        pz += L->rho[c] * L->vel[3 * c + 2];
    }
    out4[0] = m; out4[1] = px; out4[2] = py; out4[3] = pz;
}


/* ======================================================================== */
/* Reverse mode on a frozen bed (no reference counterpart: the reference has */
/* no gradients).  FP64 restatement of the adjoint that the CUDA library     */
/* implements, written against the forward functions above (orc_collide with */
/* psc = 1, smag = 0, frozen grains; orc_stream; orc_lattice2grains), with   */
/* the smooth solid fraction of orc_map_smooth in place of the 5^3 count.    */
/* ======================================================================== */

/* Smooth solid fraction: t = clamp(r - d + 1/2, 0, 1), eps = t^2 (3 - 2t),
 * r = R/dx - 1/2 as psclattice3d.py:105; owner = largest eps, ties to the
 * lowest id; no periodic images; skipped cells stay free. */
void orc_map_smooth(orc_lat *L, const orc_grains *G) {
    long nc = (long)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
        int i = (int)(c / ((long)L->ny * L->nz));
        int j = (int)((c / L->nz) % L->ny);
        int k = (int)(c % L->nz);
        L->id[c] = -1;
        L->volfrac[c] = 0.0;
        L->weight[c] = 0.0;
        L->velsolid[3 * c] = L->velsolid[3 * c + 1] = L->velsolid[3 * c + 2] = 0.0;
        if (skip_cell(L, L->ct[c])) continue;
        for (int g = 0; g < G->n; g++) {
            double xc = (G->pos[3 * g + 0] - L->xmin + 0.5 * L->dx) / L->dx;
            double yc = (G->pos[3 * g + 1] - L->ymin + 0.5 * L->dx) / L->dx;
            double zc = (G->pos[3 * g + 2] - L->zmin + 0.5 * L->dx) / L->dx;
            double r = (G->radius[g] - 0.5 * L->dx) / L->dx;
            double dxv = xc - i, dyv = yc - j, dzv = zc - k;
            double d = sqrt(dxv * dxv + dyv * dyv + dzv * dzv);
            double t = r - d + 0.5;
            if (t <= 0.0) continue;
            if (t > 1.0) t = 1.0;
            double eps = t * t * (3.0 - 2.0 * t);
            if (eps > L->volfrac[c]) {
                L->id[c] = g;
                L->volfrac[c] = eps;
                solid_vel(L, G, c, i, j, k, g, xc, yc, zc);
            }
        }
    }
}

/* Adjoint of one orc_collide on L->f (the streamed populations of that step):
 * lam = dL/dfpc (Q per cell) -> sbar = dL/df; bbar[c] += dL/dB,
 * gbar[3] += dL/dF.  seed: this is the last step, whose hydrodynamic force
 * enters L = fscale e . sum hydro (e = loss_dir). */
void orc_adjoint_collide(const orc_lat *L, const double *lam, double *sbar, double *bbar, double *gbar,
                         const double *loss_dir, int seed) {
    long nc = (long)L->nx * L->ny * L->nz;
    double fscale = (L->rho_unit * (L->dx * L->dx * L->dx * L->dx)) / (L->dt * L->dt);
    double e[3] = {fscale * loss_dir[0], fscale * loss_dir[1], fscale * loss_dir[2]};
    double F[3] = {0, 0, 0};
    if (L->force_on) { F[0] = L->force[0]; F[1] = L->force[1]; F[2] = L->force[2]; }
    double g0 = 0, g1 = 0, g2 = 0;
#pragma omp parallel for schedule(static) reduction(+ : g0, g1, g2)
    for (long c = 0; c < nc; c++) {
        double *sb = sbar + Q * c;
        for (int q = 0; q < Q; q++) sb[q] = 0.0;
        if (skip_cell(L, L->ct[c])) continue;
        const double *s = L->f + Q * c;
        const double *la = lam ? lam + Q * c : NULL;
        double om = L->omega0;
        double B = 0.0;
        if (L->psc && L->volfrac[c] > 0) {
            double eps = L->volfrac[c], taum = 1.0 / om - 0.5;
            B = (eps * taum) / ((1.0 - eps) + taum);
        }
        double rho = 0, j[3] = {0, 0, 0};
        for (int q = 0; q < Q; q++) {
            rho += s[q];
            j[0] += CX[q] * s[q]; j[1] += CY[q] * s[q]; j[2] += CZ[q] * s[q];
        }
        double jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
        double feq[Q];
        for (int q = 0; q < Q; q++) {
            double cj = CX[q] * j[0] + CY[q] * j[1] + CZ[q] * j[2];
            feq[q] = W[q] * (rho + 3.0 * cj + (4.5 * cj * cj - 1.5 * jj) / rho);
        }
        double D = 0, G[3] = {0, 0, 0}, bb = 0;
        for (int q = 0; q < Q; q++) {
            double lq = la ? la[q] : 0.0, lqb = la ? la[QINV[q]] : 0.0;
            double cj = CX[q] * j[0] + CY[q] * j[1] + CZ[q] * j[2];
            double A = (1.0 - B) * om * lq - B * lqb;
            D += A * W[q] * (1.0 - (4.5 * cj * cj - 1.5 * jj) / (rho * rho));
            double k = A * W[q] / rho;
            G[0] += A * W[q] * 3.0 * CX[q] + k * (9.0 * cj * CX[q] - 3.0 * j[0]);
            G[1] += A * W[q] * 3.0 * CY[q] + k * (9.0 * cj * CY[q] - 3.0 * j[1]);
            G[2] += A * W[q] * 3.0 * CZ[q] + k * (9.0 * cj * CZ[q] - 3.0 * j[2]);
            double cf = CX[q] * F[0] + CY[q] * F[1] + CZ[q] * F[2];
            D += lq * W[q] * (B + cf / CSSQ);
            bb += lq * ((s[QINV[q]] - feq[QINV[q]] + W[q] * rho - s[q]) + om * (s[q] - feq[q]));
            g0 += lq * W[q] * rho * CX[q] / CSSQ;
            g1 += lq * W[q] * rho * CY[q] / CSSQ;
            g2 += lq * W[q] * rho * CZ[q] / CSSQ;
        }
        double c1 = 1.0 - B - (1.0 - B) * om;
        for (int p = 0; p < Q; p++) {
            double lp = la ? la[p] : 0.0, lpb = la ? la[QINV[p]] : 0.0;
            sb[p] = lp * c1 + B * lpb + D + CX[p] * G[0] + CY[p] * G[1] + CZ[p] * G[2];
            if (seed) sb[p] += B * (CX[p] * e[0] + CY[p] * e[1] + CZ[p] * e[2]);
        }
        if (seed) bb += e[0] * j[0] + e[1] * j[1] + e[2] * j[2];
        bbar[c] += bb;
    }
    gbar[0] += g0; gbar[1] += g1; gbar[2] += g2;
}

/* Transpose of orc_stream for FLUID / OBSTACLE neighbours:
 * lam_prev = dL/dfpc of the previous step from sbar = dL/df. */
void orc_adjoint_stream(const orc_lat *L, const double *sbar, double *lam_prev) {
    int nx = L->nx, ny = L->ny, nz = L->nz;
    long nc = (long)nx * ny * nz;
    int32_t stream_skip = CT_OBSTACLE | CT_VEL_LADD | CT_FREE_SLIP | CT_VEL_INLET_LADD;
    int32_t prop = CT_FLUID | CT_VEL_ZOUHE | CT_VEL_EXIT | CT_PRE_ZOUHE;
    memset(lam_prev, 0, sizeof(double) * Q * nc);
    /* serial: every target is written once, but keep it simple and exact */
    for (long c = 0; c < nc; c++) {
        int i = (int)(c / ((long)ny * nz));
        int j = (int)((c / nz) % ny);
        int k = (int)(c % nz);
        if (L->ct[c] & stream_skip) continue;
        const double *sb = sbar + Q * c;
        lam_prev[Q * c] += sb[0];
        for (int q = 1; q < Q; q++) {
            int in = (int)(i - CX[q]), jn = (int)(j - CY[q]), kn = (int)(k - CZ[q]);
            if (in >= nx) in = 0; else if (in < 0) in = nx - 1;
            if (jn >= ny) jn = 0; else if (jn < 0) jn = ny - 1;
            if (kn >= nz) kn = 0; else if (kn < 0) kn = nz - 1;
            long n = cidx(L, in, jn, kn);
            int32_t ctn = L->ct[n];
            if (ctn & prop) lam_prev[Q * n + q] += sb[q];
            else if (ctn & CT_OBSTACLE) lam_prev[Q * c + QINV[q]] += sb[q];
        }
    }
}

/* Chain rule from bbar = dL/dB to the grain centres (physical units). */
void orc_pos_adjoint(const orc_lat *L, const orc_grains *G, const double *bbar, double *pos_bar) {
    long nc = (long)L->nx * L->ny * L->nz;
    double taum = 1.0 / L->omega0 - 0.5;
    for (long c = 0; c < nc; c++) {
        int g = L->id[c];
        double eps = L->volfrac[c];
        if (g < 0 || !(eps > 0.0 && eps < 1.0)) continue;
        int i = (int)(c / ((long)L->ny * L->nz));
        int j = (int)((c / L->nz) % L->ny);
        int k = (int)(c % L->nz);
        double xc = (G->pos[3 * g + 0] - L->xmin + 0.5 * L->dx) / L->dx;
        double yc = (G->pos[3 * g + 1] - L->ymin + 0.5 * L->dx) / L->dx;
        double zc = (G->pos[3 * g + 2] - L->zmin + 0.5 * L->dx) / L->dx;
        double r = (G->radius[g] - 0.5 * L->dx) / L->dx;
        double rx = i - xc, ry = j - yc, rz = k - zc;
        double d = sqrt(rx * rx + ry * ry + rz * rz);
        double t = r - d + 0.5;
        if (!(t > 0.0 && t < 1.0) || d <= 0.0) continue;
        double de_dt = 6.0 * t * (1.0 - t);
        double den = (1.0 - eps) + taum;
        double dB_de = taum * (1.0 + taum) / (den * den);
        double sc = bbar[c] * dB_de * de_dt / (d * L->dx);
        pos_bar[3 * g] += sc * rx;
        pos_bar[3 * g + 1] += sc * ry;
        pos_bar[3 * g + 2] += sc * rz;
    }
}

/* ======================================================================== */
/* DEM                                                                       */
/* ======================================================================== */
typedef struct {
    int n, maxc;
    int model;                 /* 0 Hertz-Mindlin, 1 linear */
    double dt, g[3];
    double dom_min[3], dom_max[3];
    int periodic[3];           /* x, y, z */
    double bp_min[3];          /* BPCD domain_min */
    double cell_size;
    int table_size;
    /* material 0 = particles, 1 = walls (material.py:13-30) */
    double E[2], nu[2], mu[2], e[2], kn[2], ks[2], dpn[2], dps[2];
    /* grains (grain.py:23-52) */
    double *pos, *vel, *acc, *force, *quat, *omega, *omega_dot, *moment, *inertia, *mass, *radius;
    double *force_fluid, *moment_fluid;
    int32_t *freeze, *fixvel;
    /* contacts (contact.py:20-33), n*maxc slots, and wall contacts n*6 */
    int32_t *cf_i, *cf_j, *cf_active, *cfn;
    double *cf_shear, *cf_pos, *cf_force;
    int32_t *wcf_active;
    double *wcf_shear, *wcf_pos, *wcf_force;
    /* walls (demconfig.py:38-58) */
    double wall_n[18], wall_d[6];
    int32_t wall_periodic[6];
    /* scratch */
    int32_t *ht_offset, *ht_count, *ht_current, *pid;
    uint8_t *bits;             /* n*n collision bit table */
    int32_t status;            /* bit 0: contact list overflow */
} orc_dem;

typedef struct { double m[3][3]; } mat3;

static void cross3(const double *a, const double *b, double *o) {
    double t0 = a[1] * b[2] - a[2] * b[1], t1 = a[2] * b[0] - a[0] * b[2], t2 = a[0] * b[1] - a[1] * b[0];
    o[0] = t0; o[1] = t1; o[2] = t2;
}

static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void matvec(const mat3 *M, const double *v, double *o) {
    double t[3];
    for (int r = 0; r < 3; r++) t[r] = M->m[r][0] * v[0] + M->m[r][1] * v[1] + M->m[r][2] * v[2];
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
}

/* 3x3 inverse through the adjugate, as a general matrix inverse */
static mat3 inv3(const mat3 *A) {
    const double(*a)[3] = A->m;
    double det = a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) -
                 a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2]) +
                 a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
    double id = 1.0 / det;
    mat3 o;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            o.m[j][i] = id * (a[(i + 1) % 3][(j + 1) % 3] * a[(i + 2) % 3][(j + 2) % 3] -
                              a[(i + 2) % 3][(j + 1) % 3] * a[(i + 1) % 3][(j + 2) % 3]);
    return o;
}

/* demsolver.py:686-701 and :757-773: rotation taking the unit vector a onto x */
static mat3 rot_to_x(const double *a) {
    double b[3] = {1.0, 0.0, 0.0}, v[3];
    cross3(a, b, v);
    double s = sqrt(dot3(v, v));
    double c = dot3(a, b);
    mat3 R;
    memset(&R, 0, sizeof(R));
    if (s < 1e-12) {
        if (c > 0.0) {
            R.m[0][0] = R.m[1][1] = R.m[2][2] = 1.0;
        } else {
            R.m[0][0] = -1.0; R.m[1][1] = 1.0; R.m[2][2] = -1.0;
        }
    } else {
        double vx[3][3] = {{0.0, -v[2], v[1]}, {v[2], 0.0, -v[0]}, {-v[1], v[0], 0.0}};
        double coef = (1.0 - c) / (s * s);
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
                double acc = 0.0;
                for (int t = 0; t < 3; t++) acc += (coef * vx[r][t]) * vx[t][q];
                R.m[r][q] = ((r == q ? 1.0 : 0.0) + vx[r][q]) + acc;
            }
    }
    return R;
}

/* bpcd.py:154-179 */
static int32_t morton3d32(int32_t x, int32_t y, int32_t z) {
    x &= 0x3ff; x = (x | x << 16) & 0x30000ff; x = (x | x << 8) & 0x300f00f;
    x = (x | x << 4) & 0x30c30c3; x = (x | x << 2) & 0x9249249;
    y &= 0x3ff; y = (y | y << 16) & 0x30000ff; y = (y | y << 8) & 0x300f00f;
    y = (y | y << 4) & 0x30c30c3; y = (y | y << 2) & 0x9249249;
    z &= 0x3ff; z = (z | z << 16) & 0x30000ff; z = (z | z << 8) & 0x300f00f;
    z = (z | z << 4) & 0x30c30c3; z = (z | z << 2) & 0x9249249;
    return x | (y << 1) | (z << 2);
}

static void bp_cell(const orc_dem *D, const double *p, int32_t *ijk) {
    for (int a = 0; a < 3; a++) ijk[a] = (int32_t)floor((p[a] - D->bp_min[a]) / D->cell_size);
}

static int32_t bp_hash(const orc_dem *D, const int32_t *ijk) {
    return morton3d32(ijk[0], ijk[1], ijk[2]) % D->table_size;
}

/* bpcd.py:67-152 + prefixsum.py:62-84: count, exclusive scan, insert, probe
 * the particle's own cell and the seven cells of its octant; emit i<pid. */
static void bpcd_detect(orc_dem *D) {
    int n = D->n, T = D->table_size;
    memset(D->ht_count, 0, sizeof(int32_t) * T);
    memset(D->ht_current, 0, sizeof(int32_t) * T);
    for (int i = 0; i < n; i++) {
        int32_t ijk[3];
        bp_cell(D, D->pos + 3 * i, ijk);
        D->ht_count[bp_hash(D, ijk)]++;
    }
    int32_t run = 0;
    for (int t = 0; t < T; t++) {
        D->ht_offset[t] = run;
        run += D->ht_count[t];
    }
    for (int i = 0; i < n; i++) {
        int32_t ijk[3];
        bp_cell(D, D->pos + 3 * i, ijk);
        int32_t h = bp_hash(D, ijk);
        int32_t loc = D->ht_current[h]++;
        D->pid[D->ht_offset[h] + loc] = i;
    }
    for (int i = 0; i < n; i++) {
        const double *o = D->pos + 3 * i;
        int32_t ijk[3], dxyz[3];
        bp_cell(D, o, ijk);
        for (int a = 0; a < 3; a++) {
            double center = (ijk[a] + 0.5) * D->cell_size + D->bp_min[a];
            dxyz[a] = (o[a] > center) ? 1 : -1;
        }
        int32_t cells[8][3] = {
            {ijk[0], ijk[1], ijk[2]},
            {ijk[0] + dxyz[0], ijk[1], ijk[2]},
            {ijk[0], ijk[1] + dxyz[1], ijk[2]},
            {ijk[0], ijk[1], ijk[2] + dxyz[2]},
            {ijk[0], ijk[1] + dxyz[1], ijk[2] + dxyz[2]},
            {ijk[0] + dxyz[0], ijk[1], ijk[2] + dxyz[2]},
            {ijk[0] + dxyz[0], ijk[1] + dxyz[1], ijk[2]},
            {ijk[0] + dxyz[0], ijk[1] + dxyz[1], ijk[2] + dxyz[2]},
        };
        for (int kc = 0; kc < 8; kc++) {
            int32_t h = bp_hash(D, cells[kc]);
            if (D->ht_count[h] > 0) {
                for (int32_t idx = D->ht_offset[h]; idx < D->ht_offset[h] + D->ht_count[h]; idx++) {
                    int32_t p = D->pid[idx];
                    if (p > i) D->bits[(long)i * n + p] = 1;
                }
            }
        }
    }
}

/* demsolver.py:483-512 */
static void periodic_delta(const orc_dem *D, const double *pi, const double *pj, double *d) {
    for (int a = 0; a < 3; a++) {
        d[a] = pj[a] - pi[a];
        if (D->periodic[a]) {
            double L = D->dom_max[a] - D->dom_min[a];
            if (d[a] > 0.5 * L) d[a] -= L;
            else if (d[a] < -0.5 * L) d[a] += L;
        }
    }
}

/* hertz.py:45-97, linear.py:43-101 */
static void pp_force(orc_dem *D, int i, int j, double *shear, double delta_n, const double *vc, double *F) {
    double gap = -1 * delta_n;
    double dt = D->dt;
    double inc[3] = {vc[0] * dt, vc[1] * dt, vc[2] * dt};
    inc[0] = 0.0;
    double kt, gt, F0;
    if (D->model == 0) {
        double Ys = 1.0 / ((1.0 - D->nu[0] * D->nu[0]) / D->E[0] + (1.0 - D->nu[0] * D->nu[0]) / D->E[0]);
        double Gs = 1.0 / (2.0 * (2.0 - D->nu[0]) * (1.0 + D->nu[0]) / D->E[0] +
                           2.0 * (2.0 - D->nu[0]) * (1.0 + D->nu[0]) / D->E[0]);
        double Rs = 1.0 / (1.0 / D->radius[i] + 1.0 / D->radius[j]);
        double ms = 1.0 / (1.0 / D->mass[i] + 1.0 / D->mass[j]);
        double e = 0.5 * (D->e[0] + D->e[0]);
        double lne = log(e);
        double beta = lne / sqrt(lne * lne + M_PI * M_PI);
        double Sn = 2.0 * Ys * sqrt(Rs * delta_n);
        double St = 8.0 * Gs * sqrt(Rs * delta_n);
        double kn = 4.0 / 3.0 * Ys * sqrt(Rs * delta_n);
        double gn = -2.0 * beta * sqrt(5.0 / 6.0 * Sn * ms);
        kt = 8.0 * Gs * sqrt(Rs * delta_n);
        gt = -2.0 * beta * sqrt(5.0 / 6.0 * St * ms);
        F0 = -kn * gap - gn * vc[0];
    } else {
        double kns = D->kn[0] * D->kn[0] / (D->kn[0] + D->kn[0]);
        double kss = D->ks[0] * D->ks[0] / (D->ks[0] + D->ks[0]);
        double dpn = 0.5 * (D->dpn[0] + D->dpn[0]);
        double dps = 0.5 * (D->dps[0] + D->dps[0]);
        double ms = 1.0 / (1.0 / D->mass[i] + 1.0 / D->mass[j]);
        double Cn = 2. * dpn * sqrt(kns * ms);
        double Ct = 2. * dps * sqrt(kns * ms);
        kt = kss;
        gt = Ct;
        F0 = -kns * gap - Cn * vc[0];
    }
    double mu = 0.5 * (D->mu[0] + D->mu[0]);
    for (int a = 0; a < 3; a++) shear[a] += inc[a];
    double ts[3] = {-kt * shear[0], -kt * shear[1], -kt * shear[2]};
    double tl = sqrt(dot3(ts, ts));
    F[0] = F0;
    if (tl >= mu * F0 && tl > 0.0) {
        double ratio = mu * F0 / tl;
        F[1] = ts[1] * ratio;
        F[2] = ts[2] * ratio;
        shear[1] = -F[1] / kt;
        shear[2] = -F[2] / kt;
    } else {
        F[1] = ts[1] - gt * vc[1];
        F[2] = ts[2] - gt * vc[2];
    }
}

/* hertz.py:99-153, linear.py:103-152 */
static void pw_force(orc_dem *D, int i, double *shear, double delta_n, const double *vc, double *F) {
    double gap = -1 * delta_n;
    double dt = D->dt;
    double inc[3] = {vc[0] * dt, vc[1] * dt, vc[2] * dt};
    inc[0] = 0.0;
    double kt, gt, F0, mu = D->mu[1];
    if (D->model == 0) {
        double Ys = 1.0 / ((1.0 - D->nu[0] * D->nu[0]) / D->E[0] + (1.0 - D->nu[1] * D->nu[1]) / D->E[1]);
        double Gs = 1.0 / (2.0 * (2.0 - D->nu[0]) * (1.0 + D->nu[0]) / D->E[0] +
                           2.0 * (2.0 - D->nu[1]) * (1.0 + D->nu[1]) / D->E[1]);
        double Rs = D->radius[i];
        double ms = D->mass[i];
        double e = D->e[1];
        double lne = log(e);
        double beta = lne / sqrt(lne * lne + M_PI * M_PI);
        double Sn = 2.0 * Ys * sqrt(Rs * delta_n);
        double St = 8.0 * Gs * sqrt(Rs * delta_n);
        double kn = 4.0 / 3.0 * Ys * sqrt(Rs * delta_n);
        double gn = -2.0 * beta * sqrt(5.0 / 6.0 * Sn * ms);
        kt = 8.0 * Gs * sqrt(Rs * delta_n);
        gt = -2.0 * beta * sqrt(5.0 / 6.0 * St * ms);
        F0 = -kn * gap - gn * vc[0];
    } else {
        double kns = D->kn[0], kss = D->ks[0];
        double ms = D->mass[i];
        double Cn = 2. * D->dpn[0] * sqrt(kns * ms);
        double Ct = 2. * D->dps[0] * sqrt(kns * ms);
        kt = kss;
        gt = Ct;
        F0 = -kns * gap - Cn * vc[0];
    }
    for (int a = 0; a < 3; a++) shear[a] += inc[a];
    double ts[3] = {-kt * shear[0], -kt * shear[1], -kt * shear[2]};
    double tl = sqrt(dot3(ts, ts));
    F[0] = F0;
    if (tl >= mu * F0 && tl > 0.0) {
        double ratio = mu * F0 / tl;
        F[1] = ts[1] * ratio;
        F[2] = ts[2] * ratio;
        shear[1] = -F[1] / kt;
        shear[2] = -F[2] / kt;
    } else {
        F[1] = ts[1] - gt * vc[1];
        F[2] = ts[2] - gt * vc[2];
    }
}

/* demsolver.py:352-369 */
static int search_contact(const orc_dem *D, int i, int j) {
    for (int o = 0; o < D->cfn[i]; o++) {
        long s = (long)i * D->maxc + o;
        if (D->cf_j[s] == j && D->cf_active[s]) return (int)s;
    }
    return -1;
}

/* demsolver.py:638-740 */
static void resolve(orc_dem *D, int i, int j) {
    int eval = 0;
    int off = search_contact(D, i, j);
    double dv[3];
    periodic_delta(D, D->pos + 3 * i, D->pos + 3 * j, dv);
    double distance = sqrt(dot3(dv, dv));
    double gap = distance - D->radius[i] - D->radius[j];
    if (off >= 0) {
        if (gap < 0) eval = 1;
        else D->cf_active[off] = 0;
    } else if (gap < 0) {
        int o = D->cfn[i]++;
        if (o >= D->maxc) {
            D->status |= 1;
            return;
        }
        off = i * D->maxc + o;
        D->cf_i[off] = i;
        D->cf_j[off] = j;
        D->cf_active[off] = 1;
        for (int a = 0; a < 3; a++) D->cf_shear[3 * off + a] = D->cf_pos[3 * off + a] = D->cf_force[3 * off + a] = 0.0;
        eval = 1;
    }
    if (!eval) return;
    double inv_len = sqrt(dot3(dv, dv));
    double a[3] = {dv[0] / inv_len, dv[1] / inv_len, dv[2] / inv_len};
    mat3 R = rot_to_x(a);
    double delta_n = -gap;
    double *cp = D->cf_pos + 3 * off;
    const double *pi = D->pos + 3 * i;
    for (int t = 0; t < 3; t++) cp[t] = pi[t] + a[t] * (D->radius[i] - delta_n);
    double ri[3], rj[3], pj_img[3];
    for (int t = 0; t < 3; t++) {
        ri[t] = cp[t] - pi[t];
        pj_img[t] = pi[t] + dv[t];
        rj[t] = cp[t] - pj_img[t];
    }
    double vci[3], vcj[3], dvc[3], vc[3];
    cross3(D->omega + 3 * i, ri, vci);
    cross3(D->omega + 3 * j, rj, vcj);
    for (int t = 0; t < 3; t++) {
        vci[t] += D->vel[3 * i + t];
        vcj[t] += D->vel[3 * j + t];
        dvc[t] = vcj[t] - vci[t];
    }
    matvec(&R, dvc, vc);
    double F[3];
    pp_force(D, i, j, D->cf_shear + 3 * off, delta_n, vc, F);
    for (int t = 0; t < 3; t++) D->cf_force[3 * off + t] = F[t];
    mat3 Ri = inv3(&R);
    double mF[3] = {-F[0], -F[1], -F[2]}, Fi[3], Fj[3], Mi[3], Mj[3];
    matvec(&Ri, mF, Fi);
    matvec(&Ri, F, Fj);
    for (int t = 0; t < 3; t++) {
        D->force[3 * i + t] += Fi[t];
        D->force[3 * j + t] += Fj[t];
    }
    cross3(ri, Fi, Mi);
    cross3(rj, Fj, Mj);
    for (int t = 0; t < 3; t++) {
        D->moment[3 * i + t] += Mi[t];
        D->moment[3 * j + t] += Mj[t];
    }
}

/* demsolver.py:742-807 */
static void evaluate_wall(orc_dem *D, int i, int w) {
    const double *nrm = D->wall_n + 3 * w;
    mat3 R = rot_to_x(nrm);
    const double *p = D->pos + 3 * i;
    double delta_n = (dot3(p, nrm) - D->wall_d[w]) + D->radius[i];
    double distance = D->radius[i] - delta_n;
    long s = (long)i * 6 + w;
    double ri[3];
    for (int t = 0; t < 3; t++) {
        ri[t] = distance * nrm[t];
        D->wcf_pos[3 * s + t] = p[t] + ri[t];
    }
    double vci[3], m[3], vc[3];
    cross3(D->omega + 3 * i, ri, vci);
    for (int t = 0; t < 3; t++) m[t] = -(vci[t] + D->vel[3 * i + t]);
    matvec(&R, m, vc);
    double F[3];
    pw_force(D, i, D->wcf_shear + 3 * s, delta_n, vc, F);
    for (int t = 0; t < 3; t++) D->wcf_force[3 * s + t] = F[t];
    mat3 Ri = inv3(&R);
    double mF[3] = {-F[0], -F[1], -F[2]}, Fi[3], Mi[3];
    matvec(&Ri, mF, Fi);
    for (int t = 0; t < 3; t++) D->force[3 * i + t] += Fi[t];
    cross3(ri, Fi, Mi);
    for (int t = 0; t < 3; t++) D->moment[3 * i + t] += Mi[t];
}

/* demsolver.py:809-838 */
static void resolve_wall(orc_dem *D) {
    for (int i = 0; i < D->n; i++)
        for (int w = 0; w < 6; w++) {
            if (D->wall_periodic[w]) continue;
            long s = (long)i * 6 + w;
            double sep = -(dot3(D->pos + 3 * i, D->wall_n + 3 * w) - D->wall_d[w]);
            if (D->wcf_active[s]) {
                if (sep > D->radius[i]) D->wcf_active[s] = 0;
                else evaluate_wall(D, i, w);
            } else if (sep <= D->radius[i]) {
                D->wcf_active[s] = 1;
                for (int t = 0; t < 3; t++) D->wcf_shear[3 * s + t] = D->wcf_pos[3 * s + t] = D->wcf_force[3 * s + t] = 0.0;
                evaluate_wall(D, i, w);
            }
        }
}

/* utils.py:34-61 */
static mat3 quat2rot(const double *q) {
    double w2 = q[0] * q[0], i2 = q[1] * q[1], j2 = q[2] * q[2], k2 = q[3] * q[3];
    double twoij = 2.0 * q[1] * q[2], twoik = 2.0 * q[1] * q[3], twojk = 2.0 * q[2] * q[3];
    double twoiw = 2.0 * q[1] * q[0], twojw = 2.0 * q[2] * q[0], twokw = 2.0 * q[3] * q[0];
    mat3 r;
    r.m[0][0] = w2 + i2 - j2 - k2; r.m[0][1] = twoij - twokw; r.m[0][2] = twojw + twoik;
    r.m[1][0] = twoij + twokw; r.m[1][1] = w2 - i2 + j2 - k2; r.m[1][2] = twojk - twoiw;
    r.m[2][0] = twoik - twojw; r.m[2][1] = twojk + twoiw; r.m[2][2] = w2 - i2 - j2 + k2;
    return r;
}

/* demsolver.py:451-480 */
static void wrap_position(const orc_dem *D, double *p) {
    for (int a = 0; a < 3; a++) {
        if (!D->periodic[a]) continue;
        double L = D->dom_max[a] - D->dom_min[a];
        if (p[a] > D->dom_max[a]) p[a] = p[a] - L;
        else if (p[a] < D->dom_min[a]) p[a] = p[a] + L;
    }
}

static void rotate_update(orc_dem *D, int i) {
    double dt = D->dt;
    mat3 Rm = quat2rot(D->quat + 4 * i);
    mat3 I;
    memcpy(I.m, D->inertia + 9 * i, sizeof(double) * 9);
    double ml[3], wl[3], Iw[3], cw[3], rhs[3], wdl[3], alpha[3];
    matvec(&Rm, D->moment + 3 * i, ml);
    matvec(&Rm, D->omega + 3 * i, wl);
    matvec(&I, wl, Iw);
    cross3(wl, Iw, cw);
    for (int t = 0; t < 3; t++) rhs[t] = ml[t] - cw[t];
    mat3 Ii = inv3(&I);
    matvec(&Ii, rhs, wdl);
    mat3 Rmi = inv3(&Rm);
    matvec(&Rmi, wdl, alpha);
    double *w = D->omega + 3 * i, *q = D->quat + 4 * i;
    for (int t = 0; t < 3; t++) w[t] += 0.5 * (D->omega_dot[3 * i + t] + alpha[t]) * dt;
    double dq0 = -0.5 * (q[1] * w[0] + q[2] * w[1] + q[3] * w[2]);
    double dq1 = +0.5 * (q[0] * w[0] - q[3] * w[1] + q[2] * w[2]);
    double dq2 = +0.5 * (q[3] * w[0] + q[0] * w[1] + q[1] * w[2]);
    double dq3 = +0.5 * (-q[2] * w[0] + q[1] * w[1] + q[0] * w[2]);
    q[0] += dq0 * dt; q[1] += dq1 * dt; q[2] += dq2 * dt; q[3] += dq3 * dt;
    double ql = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int t = 0; t < 4; t++) q[t] = q[t] / ql;
    for (int t = 0; t < 3; t++) D->omega_dot[3 * i + t] = alpha[t];
}

/* demsolver.py:514-636 */
static void update(orc_dem *D) {
    double dt = D->dt;
    for (int i = 0; i < D->n; i++) {
        double *p = D->pos + 3 * i, *v = D->vel + 3 * i;
        if (D->freeze[i]) continue;
        if (D->fixvel[i]) {
            for (int t = 0; t < 3; t++) p[t] += v[t] * dt;
            wrap_position(D, p);
            rotate_update(D, i);
            continue;
        }
        double a[3];
        for (int t = 0; t < 3; t++) a[t] = D->force[3 * i + t] / D->mass[i];
        for (int t = 0; t < 3; t++) v[t] += 0.5 * (D->acc[3 * i + t] + a[t]) * dt;
        for (int t = 0; t < 3; t++) p[t] += v[t] * dt + 0.5 * a[t] * (dt * dt);
        wrap_position(D, p);
        for (int t = 0; t < 3; t++) D->acc[3 * i + t] = a[t];
        rotate_update(D, i);
    }
}

/* demsolver.py:371-386 */
static void compact_contacts(orc_dem *D) {
    for (int i = 0; i < D->n; i++) {
        long base = (long)i * D->maxc;
        int cnt = D->cfn[i] < D->maxc ? D->cfn[i] : D->maxc;
        int active = 0;
        for (int o = 0; o < cnt; o++) active += D->cf_active[base + o] ? 1 : 0;
        int w = 0;
        for (int o = 0; o < cnt; o++) {
            if (D->cf_active[base + o]) {
                long d = base + w, s = base + o;
                D->cf_i[d] = D->cf_i[s]; D->cf_j[d] = D->cf_j[s]; D->cf_active[d] = D->cf_active[s];
                for (int t = 0; t < 3; t++) {
                    D->cf_shear[3 * d + t] = D->cf_shear[3 * s + t];
                    D->cf_pos[3 * d + t] = D->cf_pos[3 * s + t];
                    D->cf_force[3 * d + t] = D->cf_force[3 * s + t];
                }
                w++;
                if (w >= active) break;
            }
        }
        for (int o = active; o < cnt; o++) D->cf_active[base + o] = 0;
        D->cfn[i] = active;
    }
}

/* demsolver.py:848-862 */
void orc_dem_run_simulation(orc_dem *D) {
    int n = D->n;
    for (int i = 0; i < 3 * n; i++) D->force[i] = D->moment[i] = 0.0;   /* clear_state :422-429 */
    memset(D->bits, 0, (size_t)n * n);                                      /* :394-398 */
    bpcd_detect(D);
    for (int i = 0; i < n; i++)                                             /* :412-417 */
        for (int j = 0; j < n; j++)
            if (D->bits[(long)i * n + j]) resolve(D, i, j);
    resolve_wall(D);
    for (int i = 0; i < n; i++)                                             /* :437-448 */
        for (int t = 0; t < 3; t++) {
            D->force[3 * i + t] += D->mass[i] * D->g[t];
            D->moment[3 * i + t] += 0.0;
            D->force[3 * i + t] += D->force_fluid[3 * i + t];
            D->moment[3 * i + t] += D->moment_fluid[3 * i + t];
        }
    update(D);
    compact_contacts(D);
}

/* Candidate pairs the broad phase proposes (for contact-set parity tests). */
int orc_dem_candidates(orc_dem *D, int32_t *out_pairs, int cap) {
    int n = D->n, m = 0;
    memset(D->bits, 0, (size_t)n * n);
    bpcd_detect(D);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            if (D->bits[(long)i * n + j]) {
                if (m < cap) { out_pairs[2 * m] = i; out_pairs[2 * m + 1] = j; }
                m++;
            }
    return m;
}

int orc_abi_version(void) { return 1; }
