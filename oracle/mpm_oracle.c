/*
 * mpm_oracle.c -- CPU FP64 restatement of the EdgePredict MPM workpiece step.
 *
 * TEST INFRASTRUCTURE ONLY (see mpm_oracle.h).  Citations are to the
 * reference project, path:line.
 *
 * Step order restated from MPMSolver::step (src/MPMSolver.cu:1062-1168):
 *   [lodClassify] -> resetGrid -> p2g -> updateGrid -> [fixtureBC]
 *   -> [rasterizeTool -> gridCollision] -> g2p -> resetExternalForce
 *   -> chip separation when the step counter is even (:1160-1164).
 */
#include "mpm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* grid channel offsets (SoA planes of nn doubles each) */
/* G_TM: scattered T m; G_TN: node temperature after the diffusion step */
enum { G_M, G_PX, G_PY, G_PZ, G_FX, G_FY, G_FZ, G_VX, G_VY, G_VZ, G_TVX, G_TVY, G_TVZ, G_TOOL, G_TM, G_TN, G_NCH };

static inline int64_t nnodes(const orc_params *p) { return (int64_t)p->nx * p->ny * p->nz; }

int64_t orc_grid_doubles(const orc_params *p) { return nnodes(p) * G_NCH; }

/* ---------------------------------------------------------------- helpers */

/* getWeightsAndGradients, src/MPMSolver.cu:20-34 (quadratic B-spline). */
static void weights(double xp, double invDx, int *base, double w[3], double dw[3]) {
    double xf = xp * invDx;
    int b = (int)floor(xf - 0.5);
    double d0 = xf - b, d1 = d0 - 1.0, d2 = d0 - 2.0;
    *base = b;
    w[0] = 0.5 * (1.5 - d0) * (1.5 - d0);
    w[1] = 0.75 - d1 * d1;
    w[2] = 0.5 * (1.5 + d2) * (1.5 + d2);
    dw[0] = -(1.5 - d0) * invDx;
    dw[1] = -2.0 * d1 * invDx;
    dw[2] = (1.5 + d2) * invDx;
}

/* det3x3 / mul3x3 / inv3x3, src/MPMSolver.cu:36-68. */
static double det3(const double *A) {
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}
static void mul3(const double *A, const double *B, double *Cm) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Cm[i * 3 + j] = A[i * 3 + 0] * B[0 * 3 + j] + A[i * 3 + 1] * B[1 * 3 + j] + A[i * 3 + 2] * B[2 * 3 + j];
}
static void inv3(const double *A, double *R) {
    double det = det3(A);
    if (fabs(det) < 1e-12) {
        for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    double id = 1.0 / det;
    R[0] = (A[4] * A[8] - A[5] * A[7]) * id;
    R[1] = -(A[1] * A[8] - A[2] * A[7]) * id;
    R[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    R[3] = -(A[3] * A[8] - A[5] * A[6]) * id;
    R[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    R[5] = -(A[0] * A[5] - A[2] * A[3]) * id;
    R[6] = (A[3] * A[7] - A[4] * A[6]) * id;
    R[7] = -(A[0] * A[7] - A[1] * A[6]) * id;
    R[8] = (A[0] * A[4] - A[1] * A[3]) * id;
}

static inline void gadd(double *a, double v, int atomic) {
    if (atomic) {
#pragma omp atomic
        *a += v;
    } else {
        *a += v;
    }
}

/* ------------------------------------------------------------- tool SDF */

/* Analytic rigid-tool SDF (an extension of this build; the reference's grid
 * boundary is the rasterised tool of src/MPMSolver.cu:444-492).  Returns the
 * signed distance and the outward unit normal. */
static double tool_sdf_n(const orc_params *p, const double pr[3], double x, double y, double z, double nrm[3]) {
    (void)y;
    double qx = x - pr[0], qz = z - pr[2];
    if (p->tool_shape == ORC_SHAPE_CYLINDER_Y) {
        double r = sqrt(qx * qx + qz * qz);
        if (r > 0.0) { nrm[0] = qx / r; nrm[1] = 0.0; nrm[2] = qz / r; }
        else { nrm[0] = 0.0; nrm[1] = 0.0; nrm[2] = 1.0; }
        return r - p->tool_r;
    }
    /* rounded wedge extruded along y: a sharp core wedge with its apex at the
     * edge-circle centre, offset outward by the edge radius.  Rake face
     * direction t1 (up), flank face direction t2 (back, rising by the
     * clearance angle); outward normals n1 (+x side), n2 (below). */
    double sg = sin(p->tool_rake), cg = cos(p->tool_rake);
    double sa = sin(p->tool_clear), ca = cos(p->tool_clear);
    double t1x = -sg, t1z = cg, n1x = cg, n1z = sg;
    double t2x = -ca, t2z = sa, n2x = -sa, n2z = -ca;
    double d1 = n1x * qx + n1z * qz, d2 = n2x * qx + n2z * qz;
    double core;
    if (d1 <= 0.0 && d2 <= 0.0) {
        if (d1 >= d2) { core = d1; nrm[0] = n1x; nrm[2] = n1z; }
        else { core = d2; nrm[0] = n2x; nrm[2] = n2z; }
    } else {
        double s1 = qx * t1x + qz * t1z; if (s1 < 0.0) s1 = 0.0;
        double s2 = qx * t2x + qz * t2z; if (s2 < 0.0) s2 = 0.0;
        double e1x = qx - s1 * t1x, e1z = qz - s1 * t1z;
        double e2x = qx - s2 * t2x, e2z = qz - s2 * t2z;
        double l1 = sqrt(e1x * e1x + e1z * e1z), l2 = sqrt(e2x * e2x + e2z * e2z);
        if (l1 <= l2) { core = l1; if (l1 > 0) { nrm[0] = e1x / l1; nrm[2] = e1z / l1; } else { nrm[0] = n1x; nrm[2] = n1z; } }
        else { core = l2; if (l2 > 0) { nrm[0] = e2x / l2; nrm[2] = e2z / l2; } else { nrm[0] = n2x; nrm[2] = n2z; } }
    }
    nrm[1] = 0.0;
    return core - p->tool_r;
}

double orc_tool_sdf(const orc_params *p, const double pr[3], double x, double y, double z) {
    double n[3];
    return tool_sdf_n(p, pr, x, y, z, n);
}

/* ------------------------------------------------------ constitutive update */

static double jc_flow(const orc_params *p, double eps, double rate_term, double th_term) {
    return (p->A + p->B * pow(eps, p->n)) * rate_term * th_term;
}

/* Consistent return (extension): solve q - 3 mu dg = Y(eps + dg) for dg in
 * [0, q/(3 mu)] by Newton steps safeguarded with bisection, rate and
 * temperature frozen at the step start.  Returns 0 on convergence. */
static int newton_return(const orc_params *p, double q, double mu, double eps0, double rt, double tt, double *dg_out) {
    double lo = 0.0, hi = q / (3.0 * mu);
    double x = (q - jc_flow(p, eps0, rt, tt)) / (3.0 * mu);
    if (!(x > lo)) x = 0.5 * (lo + hi);
    if (x > hi) x = hi;
    double tol = p->newton_tol * q;
    int maxit = p->newton_maxit > 0 ? p->newton_maxit : 60;
    for (int it = 0; it < maxit; ++it) {
        double e = eps0 + x;
        double fx = q - 3.0 * mu * x - jc_flow(p, e, rt, tt);
        if (fabs(fx) <= tol) { *dg_out = x; return 0; }
        if (fx > 0.0) lo = x; else hi = x;
        double dY = (e > 0.0) ? p->B * p->n * pow(e, p->n - 1.0) * rt * tt : INFINITY;
        double d = -3.0 * mu - dY;
        double xn = x - fx / d;
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (hi - lo <= 1e-15 * hi) { *dg_out = xn; return 0; }
        x = xn;
    }
    *dg_out = x;
    return 1;
}

/* ------------------------------------------------------------ step kernels */

/* lodClassifyKernel, src/MPMSolver.cu:656-676 (ACTIVE/CHIP only). */
static void lod_classify(const orc_params *p, orc_state *s, const double tip[3]) {
    for (int i = 0; i < s->n; ++i) {
        if (s->status[i] != ORC_ACTIVE && s->status[i] != ORC_CHIP) continue;
        double dx = s->x[i] - tip[0], dy = s->y[i] - tip[1], dz = s->z[i] - tip[2];
        double d = sqrt(dx * dx + dy * dy + dz * dz);
        s->lod[i] = (d <= p->lod_active_r) ? 0 : (d <= p->lod_near_r ? 1 : 2);
    }
}

/* p2gKernel, src/MPMSolver.cu:123-422. */
static int p2g(const orc_params *p, orc_state *s, double *g, int nthreads) {
    const int64_t nn = nnodes(p);
    const double invDx = 1.0 / p->dx;
    const double mu = p->E / (2.0 * (1.0 + p->nu));
    const double lambda = p->E * p->nu / ((1.0 + p->nu) * (1.0 - 2.0 * p->nu));
    const int atomic = nthreads > 1;
    int err = 0;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(| : err) if (nthreads > 1)
    for (int ip = 0; ip < s->n; ++ip) {
        if (s->status[ip] == ORC_INACTIVE) continue;
        /* kill zone, :130-139 */
        int cx = (int)floor((s->x[ip] - p->ox) * invDx);
        int cy = (int)floor((s->y[ip] - p->oy) * invDx);
        int cz = (int)floor((s->z[ip] - p->oz) * invDx);
        if (cx < 1 || cx >= p->nx - 2 || cy < 1 || cy >= p->ny - 2 || cz < 1 || cz >= p->nz - 2) {
            s->status[ip] = ORC_INACTIVE;
            continue;
        }
        int skipStress = (s->lod[ip] == 2);
        int isFixed = (s->status[ip] == ORC_FIXED);
        int isChip = (s->status[ip] == ORC_CHIP);
        if (isFixed || isChip) skipStress = 1;
        int bx, by, bz;
        double wx[3], wy[3], wz[3], dwx[3], dwy[3], dwz[3];
        weights(s->x[ip] - p->ox, invDx, &bx, wx, dwx);
        weights(s->y[ip] - p->oy, invDx, &by, wy, dwy);
        weights(s->z[ip] - p->oz, invDx, &bz, wz, dwz);

        double sigma[9] = {0};
        double V0 = s->vol[ip];
        double J = 1.0;
        if (!skipStress && s->status[ip] == ORC_ACTIVE) {
            double *F = s->F + 9 * (int64_t)ip, *Fp = s->Fp + 9 * (int64_t)ip;
            double *bs = s->bs + 6 * (int64_t)ip;
            double invFp[9], Fe[9], Bm[9];
            inv3(Fp, invFp);
            mul3(F, invFp, Fe);
            J = det3(Fe);
            if (J < 0.9) J = 0.9;          /* :174-175 */
            if (J > 1.1) J = 1.1;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    Bm[i * 3 + j] = Fe[i * 3 + 0] * Fe[j * 3 + 0] + Fe[i * 3 + 1] * Fe[j * 3 + 1] + Fe[i * 3 + 2] * Fe[j * 3 + 2];
            /* sigma = mu/J (B - I) + lambda (J - 1) I, :192-200 */
            double Js = fmax(J, 1e-12), Jpow = Js - 1.0, muJ = mu / Js;
            for (int i = 0; i < 9; ++i) {
                sigma[i] = muJ * Bm[i];
                if (i % 4 == 0) sigma[i] += lambda * Jpow - muJ;
            }
            /* Johnson-Cook return, :205-360 */
            double tr = sigma[0] + sigma[4] + sigma[8];
            double sd[9];
            for (int i = 0; i < 9; ++i) sd[i] = sigma[i];
            sd[0] -= tr / 3.0; sd[4] -= tr / 3.0; sd[8] -= tr / 3.0;
            double ex = sd[0] - bs[0], ey = sd[4] - bs[1], ez = sd[8] - bs[2];
            double exy = sd[1] - bs[3], exz = sd[2] - bs[4], eyz = sd[5] - bs[5];
            double q = sqrt(1.5 * (ex * ex + ey * ey + ez * ez + 2.0 * (exy * exy + exz * exz + eyz * eyz)));
            double Ts = (s->T[ip] - p->Tamb) / fmax(p->Tm - p->Tamb, 1.0);
            if (Ts < 0) Ts = 0;
            if (Ts > 1) Ts = 1;
            double es = fmax(s->edot[ip] / fmax(p->edot0, 1e-12), 1e-5);
            double rt = 1.0 + p->C * log(es), tt = 1.0 - pow(Ts, p->m);
            double Y = (p->A + p->B * pow(s->eps[ip], p->n)) * rt * tt;
            double dEps = 0.0;
            if (q > Y && q > 1e-12) {
                double Yr = Y;
                if (p->plasticity_mode == ORC_PLAST_NEWTON) {
                    double dg;
                    if (newton_return(p, q, mu, s->eps[ip], rt, tt, &dg)) err |= 1;
                    dEps = dg;
                    Yr = q - 3.0 * mu * dg;
                } else {
                    dEps = (q - Y) / fmax(3.0 * mu, 1e-12);
                    if (dEps > p->deps_cap) dEps = p->deps_cap;
                }
                double scale = Yr / q;
                sd[0] = bs[0] + scale * ex; sd[4] = bs[1] + scale * ey; sd[8] = bs[2] + scale * ez;
                sd[1] = bs[3] + scale * exy; sd[2] = bs[4] + scale * exz; sd[5] = bs[5] + scale * eyz;
                for (int i = 0; i < 9; ++i) {
                    sigma[i] = sd[i];
                    if (i % 4 == 0) sigma[i] += tr / 3.0;
                }
                if (dEps > 0) {
                    if (p->Hkin > 0.0) {     /* :259-267 */
                        double ns = p->Hkin * dEps / q;
                        bs[0] += ns * ex; bs[1] += ns * ey; bs[2] += ns * ez;
                        bs[3] += ns * exy; bs[4] += ns * exz; bs[5] += ns * eyz;
                    }
                    s->eps[ip] += dEps;
                    /* Fp <- (I + 1.5 dEps/|s| s) Fp / cbrt(det), :277-302 */
                    double sn = sqrt(sd[0] * sd[0] + sd[4] * sd[4] + sd[8] * sd[8] + 2.0 * (sd[1] * sd[1] + sd[2] * sd[2] + sd[5] * sd[5]));
                    double al = (sn > 1e-12) ? (1.5 * dEps / sn) : 0.0;
                    double Ia[9], nFp[9];
                    for (int i = 0; i < 9; ++i) Ia[i] = al * sd[i];
                    Ia[0] += 1.0; Ia[4] += 1.0; Ia[8] += 1.0;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            nFp[i * 3 + j] = 0;
                            for (int k = 0; k < 3; ++k) nFp[i * 3 + j] += Ia[i * 3 + k] * Fp[k * 3 + j];
                        }
                    double dFp = nFp[0] * (nFp[4] * nFp[8] - nFp[5] * nFp[7]) - nFp[1] * (nFp[3] * nFp[8] - nFp[5] * nFp[6]) +
                                 nFp[2] * (nFp[3] * nFp[7] - nFp[4] * nFp[6]);
                    double cb = cbrt(fmax(dFp, 1e-12));
                    for (int i = 0; i < 9; ++i) Fp[i] = nFp[i] / cb;
                    /* plastic-work heating, :310-321 */
                    double dT = p->beta * Yr * dEps / fmax(p->rho_phys * p->cp, 1e-12);
                    if (dT > p->dT_cap) dT = p->dT_cap;
                    s->T[ip] += dT;
                    if (s->T[ip] > p->Tm) s->T[ip] = p->Tm;
                    /* JC damage, :329-358 */
                    double tri = (tr / 3.0) / fmax(q, 1e-12);
                    double ef = (p->D1 + p->D2 * exp(p->D3 * tri)) * (1.0 + p->D4 * log(fmax(es, 1.0))) * (1.0 + p->D5 * Ts);
                    if (ef > 1e-12) {
                        s->D[ip] += dEps / ef;
                        if (s->D[ip] > 0.7 * p->Dth) {
                            double dg = (p->Dth - s->D[ip]) / (p->Dth * 0.3);
                            dg = fmax(0.0, fmin(1.0, dg));
                            for (int i = 0; i < 9; ++i) sigma[i] *= dg;
                            s->sres[ip] = fmax(s->sres[ip], sqrt(1.5 * (sd[0] * sd[0] + sd[4] * sd[4] + sd[8] * sd[8] +
                                                                         2.0 * (sd[1] * sd[1] + sd[2] * sd[2] + sd[5] * sd[5]))));
                        }
                        if (s->D[ip] >= p->Dth) {
                            s->status[ip] = ORC_CHIP;
                            skipStress = 1;
                        }
                    }
                }
            }
            double *sg = s->sig + 6 * (int64_t)ip;  /* :363-364 */
            sg[0] = sigma[0]; sg[1] = sigma[4]; sg[2] = sigma[8];
            sg[3] = sigma[1]; sg[4] = sigma[2]; sg[5] = sigma[5];
        }
        /* APIC scatter, :370-421 */
        const double *Cp = s->C + 9 * (int64_t)ip;
        const double m = s->mass[ip];
        const double efx = s->extf ? s->extf[3 * (int64_t)ip] : 0.0;
        const double efy = s->extf ? s->extf[3 * (int64_t)ip + 1] : 0.0;
        const double efz = s->extf ? s->extf[3 * (int64_t)ip + 2] : 0.0;
        for (int i = 0; i < 3; ++i) {
            int gx = bx + i;
            if (gx < 0 || gx >= p->nx) continue;
            for (int j = 0; j < 3; ++j) {
                int gy = by + j;
                if (gy < 0 || gy >= p->ny) continue;
                for (int k = 0; k < 3; ++k) {
                    int gz = bz + k;
                    if (gz < 0 || gz >= p->nz) continue;
                    double w = wx[i] * wy[j] * wz[k];
                    double gdx = dwx[i] * wy[j] * wz[k], gdy = wx[i] * dwy[j] * wz[k], gdz = wx[i] * wy[j] * dwz[k];
                    int64_t gi = gx + (int64_t)p->nx * (gy + (int64_t)p->ny * gz);
                    double dpx = (gx * p->dx + p->ox) - s->x[ip];
                    double dpy = (gy * p->dx + p->oy) - s->y[ip];
                    double dpz = (gz * p->dx + p->oz) - s->z[ip];
                    double ax = Cp[0] * dpx + Cp[1] * dpy + Cp[2] * dpz;
                    double ay = Cp[3] * dpx + Cp[4] * dpy + Cp[5] * dpz;
                    double az = Cp[6] * dpx + Cp[7] * dpy + Cp[8] * dpz;
                    gadd(&g[G_M * nn + gi], w * m, atomic);
                    /* temperatureMass, src/MPMWorkpieceSolver.cu:118 */
                    if (p->heat_conduction) gadd(&g[G_TM * nn + gi], s->T[ip] * (w * m), atomic);
                    if (!isFixed) {
                        gadd(&g[G_PX * nn + gi], w * m * (s->vx[ip] + ax), atomic);
                        gadd(&g[G_PY * nn + gi], w * m * (s->vy[ip] + ay), atomic);
                        gadd(&g[G_PZ * nn + gi], w * m * (s->vz[ip] + az), atomic);
                    }
                    double fxi = 0, fyi = 0, fzi = 0;
                    if (!skipStress) {
                        fxi = -V0 * J * (sigma[0] * gdx + sigma[1] * gdy + sigma[2] * gdz);
                        fyi = -V0 * J * (sigma[3] * gdx + sigma[4] * gdy + sigma[5] * gdz);
                        fzi = -V0 * J * (sigma[6] * gdx + sigma[7] * gdy + sigma[8] * gdz);
                    }
                    gadd(&g[G_FX * nn + gi], fxi + w * efx, atomic);
                    gadd(&g[G_FY * nn + gi], fyi + w * efy, atomic);
                    gadd(&g[G_FZ * nn + gi], fzi + w * efz, atomic);
                }
            }
        }
    }
    return err;
}

/* mpmDiffuseTemperatureKernel (src/MPMWorkpieceSolver.cu:208-262): for a
 * node with m >= 1e-15, T = (T m)/m takes T + alpha dt lap(T) / dx^2 with the
 * 7-point Laplacian, no flux through the domain faces, a neighbour's
 * temperature (T m) / max(m, 1e-30) (so 0 at an empty node), and T >= 0.
 * The reference updates the grid in place, so a node can read a neighbour
 * already updated, depending on the thread schedule; this is the Jacobi step
 * it describes (every node from the temperatures before the step).  G_TN gets
 * the node temperature g2p reads; nodes below 1e-15 keep (T m)/m. */
static void heat_diffuse(const orc_params *p, double *g, double dt) {
    const int64_t nn = nnodes(p);
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int64_t nxy = (int64_t)nx * ny;
    const double alpha = p->thermal_conductivity / (p->rho_phys * p->cp);
    const double inv_h2 = 1.0 / (p->dx * p->dx);
    for (int64_t idx = 0; idx < nn; ++idx) {
        const double m = g[G_M * nn + idx];
        if (m < 1e-15) {
            g[G_TN * nn + idx] = m > 0.0 ? g[G_TM * nn + idx] / m : 0.0;
            continue;
        }
        const double T = g[G_TM * nn + idx] / m;
        const int i = (int)(idx % nx);
        const int64_t t = idx / nx;
        const int j = (int)(t % ny), k = (int)(t / ny);
#define TNB(q) (g[G_TM * nn + (q)] / fmax(g[G_M * nn + (q)], 1e-30))
        double lap = 0.0;
        if (i > 0) lap += TNB(idx - 1) - T;
        if (i < nx - 1) lap += TNB(idx + 1) - T;
        if (j > 0) lap += TNB(idx - nx) - T;
        if (j < ny - 1) lap += TNB(idx + nx) - T;
        if (k > 0) lap += TNB(idx - nxy) - T;
        if (k < nz - 1) lap += TNB(idx + nxy) - T;
#undef TNB
        const double Tn = T + alpha * dt * lap * inv_h2;
        g[G_TN * nn + idx] = fmax(Tn, 0.0);
    }
}

void orc_heat_diffuse(const orc_params *p, const double *mass, const double *tm, double *tn, double dt) {
    const int64_t nn = nnodes(p);
    double *g = (double *)calloc((size_t)(nn * G_NCH), sizeof(double));
    if (!g) return;
    memcpy(g + G_M * nn, mass, sizeof(double) * (size_t)nn);
    memcpy(g + G_TM * nn, tm, sizeof(double) * (size_t)nn);
    heat_diffuse(p, g, dt);
    memcpy(tn, g + G_TN * nn, sizeof(double) * (size_t)nn);
    free(g);
}

/* updateGridKernel (:424-442), applyFixtureBCKernel (:82-110) and the tool
 * boundary: rasterizeToolKernel + applyGridCollisionKernel (:444-492) or the
 * analytic SDF of this build. */
static void grid_update(const orc_params *p, double *g, double dt, const orc_tool_samples *tool, const double pr[3]) {
    const int64_t nn = nnodes(p);
    const double thr = p->mass_threshold;
    for (int64_t i = 0; i < nn; ++i) {
        if (g[G_M * nn + i] > thr) {
            g[G_PZ * nn + i] += g[G_M * nn + i] * p->gravity_z * dt;
            g[G_PX * nn + i] += g[G_FX * nn + i] * dt;
            g[G_PY * nn + i] += g[G_FY * nn + i] * dt;
            g[G_PZ * nn + i] += g[G_FZ * nn + i] * dt;
            g[G_VX * nn + i] = g[G_PX * nn + i] / g[G_M * nn + i];
            g[G_VY * nn + i] = g[G_PY * nn + i] / g[G_M * nn + i];
            g[G_VZ * nn + i] = g[G_PZ * nn + i] / g[G_M * nn + i];
        }
    }
    if (p->fixture_thickness > 0.0) {
        const int64_t nxy = (int64_t)p->nx * p->ny;
        for (int64_t i = 0; i < nn; ++i) {
            int gz = (int)(i / nxy);
            double wz = gz * p->dx + p->oz;
            double zr = (wz - p->oz) / p->fixture_thickness;
            if (zr <= 1.0) {
                if (gz == 0) {
                    g[G_VX * nn + i] = 0.0; g[G_VY * nn + i] = 0.0; g[G_VZ * nn + i] = 0.0;
                } else if (zr > 0.0) {
                    double sgm = p->fixture_damping * (1.0 - zr) * (1.0 - zr);
                    double f = 1.0 / (1.0 + sgm * dt);
                    g[G_VX * nn + i] *= f; g[G_VY * nn + i] *= f; g[G_VZ * nn + i] *= f;
                }
            }
        }
    }
    if (p->tool_mode == ORC_TOOL_RASTER && tool && tool->n > 0) {
        const double invDx = 1.0 / p->dx;
        for (int t = 0; t < tool->n; ++t) {
            double sx = pr[0] + tool->ox[t], sy = pr[1] + tool->oy[t], sz = pr[2] + tool->oz[t];
            int gx = (int)round((sx - p->ox) * invDx);
            int gy = (int)round((sy - p->oy) * invDx);
            int gz = (int)round((sz - p->oz) * invDx);
            for (int a = 0; a < 2; ++a) {
                int cx = gx + a;
                if (cx < 0 || cx >= p->nx) continue;
                for (int b = 0; b < 2; ++b) {
                    int cy = gy + b;
                    if (cy < 0 || cy >= p->ny) continue;
                    for (int c = 0; c < 2; ++c) {
                        int cz = gz + c;
                        if (cz < 0 || cz >= p->nz) continue;
                        int64_t gi = cx + (int64_t)p->nx * (cy + (int64_t)p->ny * cz);
                        g[G_TOOL * nn + gi] = 1.0;
                        g[G_TVX * nn + gi] = p->tool_v[0];
                        g[G_TVY * nn + gi] = p->tool_v[1];
                        g[G_TVZ * nn + gi] = p->tool_v[2];
                    }
                }
            }
        }
        for (int64_t i = 0; i < nn; ++i) {
            if (g[G_M * nn + i] > thr && g[G_TOOL * nn + i] == 1.0) {
                g[G_VX * nn + i] = g[G_TVX * nn + i];
                g[G_VY * nn + i] = g[G_TVY * nn + i];
                g[G_VZ * nn + i] = g[G_TVZ * nn + i];
                g[G_PX * nn + i] = g[G_M * nn + i] * g[G_VX * nn + i];
                g[G_PY * nn + i] = g[G_M * nn + i] * g[G_VY * nn + i];
                g[G_PZ * nn + i] = g[G_M * nn + i] * g[G_VZ * nn + i];
            }
        }
    } else if (p->tool_mode == ORC_TOOL_SDF_STICKY || p->tool_mode == ORC_TOOL_SDF_SLIP) {
        for (int64_t i = 0; i < nn; ++i) {
            if (!(g[G_M * nn + i] > thr)) continue;
            int gx = (int)(i % p->nx), gy = (int)((i / p->nx) % p->ny), gz = (int)(i / ((int64_t)p->nx * p->ny));
            double nrm[3];
            double phi = tool_sdf_n(p, pr, gx * p->dx + p->ox, gy * p->dx + p->oy, gz * p->dx + p->oz, nrm);
            if (phi > 0.0) continue;
            if (p->tool_mode == ORC_TOOL_SDF_STICKY) {
                g[G_VX * nn + i] = p->tool_v[0];
                g[G_VY * nn + i] = p->tool_v[1];
                g[G_VZ * nn + i] = p->tool_v[2];
            } else {
                double rx = g[G_VX * nn + i] - p->tool_v[0];
                double ry = g[G_VY * nn + i] - p->tool_v[1];
                double rz = g[G_VZ * nn + i] - p->tool_v[2];
                double vn = rx * nrm[0] + ry * nrm[1] + rz * nrm[2];
                if (vn < 0.0) {
                    g[G_VX * nn + i] -= vn * nrm[0];
                    g[G_VY * nn + i] -= vn * nrm[1];
                    g[G_VZ * nn + i] -= vn * nrm[2];
                }
            }
        }
    }
}

/* g2pKernel, src/MPMSolver.cu:506-605. */
static void g2p(const orc_params *p, orc_state *s, const double *g, double dt, int nthreads) {
    const int64_t nn = nnodes(p);
    const double invDx = 1.0 / p->dx;
    (void)nthreads;
#pragma omp parallel for num_threads(nthreads) schedule(static) if (nthreads > 1)
    for (int ip = 0; ip < s->n; ++ip) {
        if (s->status[ip] == ORC_INACTIVE) continue;
        if (s->status[ip] == ORC_FIXED) {
            s->vx[ip] = 0; s->vy[ip] = 0; s->vz[ip] = 0;
            continue;
        }
        int bx, by, bz;
        double wx[3], wy[3], wz[3], dwx[3], dwy[3], dwz[3];
        weights(s->x[ip] - p->ox, invDx, &bx, wx, dwx);
        weights(s->y[ip] - p->oy, invDx, &by, wy, dwy);
        weights(s->z[ip] - p->oz, invDx, &bz, wz, dwz);
        double vx = 0, vy = 0, vz = 0, Bm[9] = {0}, L[9] = {0};
        for (int i = 0; i < 3; ++i) {
            int gx = bx + i;
            if (gx < 0 || gx >= p->nx) continue;
            for (int j = 0; j < 3; ++j) {
                int gy = by + j;
                if (gy < 0 || gy >= p->ny) continue;
                for (int k = 0; k < 3; ++k) {
                    int gz = bz + k;
                    if (gz < 0 || gz >= p->nz) continue;
                    int64_t gi = gx + (int64_t)p->nx * (gy + (int64_t)p->ny * gz);
                    if (g[G_M * nn + gi] < p->mass_threshold) continue;
                    double w = wx[i] * wy[j] * wz[k];
                    double gdx = dwx[i] * wy[j] * wz[k], gdy = wx[i] * dwy[j] * wz[k], gdz = wx[i] * wy[j] * dwz[k];
                    double gvx = g[G_VX * nn + gi], gvy = g[G_VY * nn + gi], gvz = g[G_VZ * nn + gi];
                    vx += w * gvx; vy += w * gvy; vz += w * gvz;
                    double dpx = (gx * p->dx + p->ox) - s->x[ip];
                    double dpy = (gy * p->dx + p->oy) - s->y[ip];
                    double dpz = (gz * p->dx + p->oz) - s->z[ip];
                    Bm[0] += w * gvx * dpx; Bm[1] += w * gvx * dpy; Bm[2] += w * gvx * dpz;
                    Bm[3] += w * gvy * dpx; Bm[4] += w * gvy * dpy; Bm[5] += w * gvy * dpz;
                    Bm[6] += w * gvz * dpx; Bm[7] += w * gvz * dpy; Bm[8] += w * gvz * dpz;
                    L[0] += gvx * gdx; L[1] += gvx * gdy; L[2] += gvx * gdz;
                    L[3] += gvy * gdx; L[4] += gvy * gdy; L[5] += gvy * gdz;
                    L[6] += gvz * gdx; L[7] += gvz * gdy; L[8] += gvz * gdz;
                }
            }
        }
        if (p->heat_conduction) {
            /* temperature gather of mpmG2PKernel (src/MPMWorkpieceSolver.cu:282-306):
             * weight-normalised mean over the nodes with m > 1e-18, clamped */
            double ts = 0.0, ws = 0.0;
            for (int i = 0; i < 3; ++i) {
                int gx = bx + i;
                if (gx < 0 || gx >= p->nx) continue;
                for (int j = 0; j < 3; ++j) {
                    int gy = by + j;
                    if (gy < 0 || gy >= p->ny) continue;
                    for (int k = 0; k < 3; ++k) {
                        int gz = bz + k;
                        if (gz < 0 || gz >= p->nz) continue;
                        int64_t gi = gx + (int64_t)p->nx * (gy + (int64_t)p->ny * gz);
                        const double w = wx[i] * wy[j] * wz[k];
                        if (w <= 0.0 || g[G_M * nn + gi] <= 1e-18) continue;
                        ts += g[G_TN * nn + gi] * w;
                        ws += w;
                    }
                }
            }
            if (ws > 1e-8) s->T[ip] = fmin(fmax(ts / ws, p->Tamb), p->Tm);
        }
        s->vx[ip] = vx; s->vy[ip] = vy; s->vz[ip] = vz;
        s->x[ip] += vx * dt; s->y[ip] += vy * dt; s->z[ip] += vz * dt;
        if (s->status[ip] == ORC_CHIP) { s->edot[ip] = 0; continue; }
        double *Cp = s->C + 9 * (int64_t)ip;
        double Dinv = p->apic_dinv_factor * invDx * invDx;
        for (int i = 0; i < 9; ++i) Cp[i] = Bm[i] * Dinv;
        if (s->lod[ip] == 2) { for (int i = 0; i < 9; ++i) Cp[i] = 0.0; }
        else { for (int i = 0; i < 9; ++i) Cp[i] *= p->apic_decay; }
        double IL[9], Fn[9], *F = s->F + 9 * (int64_t)ip;
        for (int i = 0; i < 9; ++i) { IL[i] = L[i] * dt; if (i % 4 == 0) IL[i] += 1.0; }
        mul3(IL, F, Fn);
        for (int i = 0; i < 9; ++i) F[i] = Fn[i];
        s->edot[ip] = sqrt(2.0 / 3.0 * (L[0] * L[0] + L[4] * L[4] + L[8] * L[8] + 0.5 * (L[1] + L[3]) * (L[1] + L[3]) +
                                        0.5 * (L[2] + L[6]) * (L[2] + L[6]) + 0.5 * (L[5] + L[7]) * (L[5] + L[7])));
    }
}

/* chipFractureAndSeparationKernel, src/MPMSolver.cu:1002-1060. */
static void chip_separation(const orc_params *p, orc_state *s, double tipZ) {
    const double Dth = p->Dth;
    for (int i = 0; i < s->n; ++i) {
        if (s->status[i] == ORC_INACTIVE) continue;
        if (s->status[i] == ORC_ACTIVE) {
            if (s->z[i] < tipZ - p->dx * 1.5 && s->D[i] > 1e-6) {
                double *sg = s->sig + 6 * (int64_t)i;
                s->status[i] = ORC_CHIP;
                s->sres[i] = fmax(s->sres[i], sqrt(sg[0] * sg[0] + sg[1] * sg[1] + sg[2] * sg[2]));
                for (int k = 0; k < 6; ++k) sg[k] = 0.0;
                s->D[i] = fmax(s->D[i], Dth);
            }
            continue;
        }
        if (s->status[i] == ORC_CHIP) {
            if (s->D[i] < Dth * 1.5) continue;
            uint32_t seed = (uint32_t)s->id[i] * 2654435761U;
            double rx = (double)((seed >> 16) & 0xFF) / 255.0 - 0.5;
            double ry = (double)((seed >> 8) & 0xFF) / 255.0 - 0.5;
            double rz = (double)(seed & 0xFF) / 255.0 - 0.5;
            double sp = sqrt(s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
            double pm = sp * 0.3 + 0.5;
            s->vx[i] += rx * pm; s->vy[i] += ry * pm; s->vz[i] += rz * pm;
            s->D[i] = Dth * 0.5;
        }
    }
}

/* xpbdContactSDFKernel, src/ContactSolver.cu:797-923, with the analytic tool
 * SDF and its exact normal in place of the voxel texture and its central
 * differences.  For every particle that is not INACTIVE or FIXED and lies
 * within contact_radius of the tool surface: push it out to the radius along
 * the normal; remove an approaching normal velocity; Coulomb friction on the
 * tangential velocity taken with the normal component before that removal
 * (:870-873); heat the particle with the friction work times
 * (1 - heat partition), T capped at Tm (:885-904). */
static void particle_contact(const orc_params *p, orc_state *s, const double pr[3], double dt) {
    const double rc = p->contact_radius, mu = p->contact_friction, hp = p->contact_heat_partition;
    for (int i = 0; i < s->n; ++i) {
        if (s->status[i] == ORC_INACTIVE || s->status[i] == ORC_FIXED) continue;
        double nrm[3];
        const double sdf = tool_sdf_n(p, pr, s->x[i], s->y[i], s->z[i], nrm);
        if (sdf >= rc) continue;
        const double pen = rc - sdf;
        if (pen <= 0.0) continue;
        s->x[i] += nrm[0] * pen;
        s->y[i] += nrm[1] * pen;
        s->z[i] += nrm[2] * pen;
        const double vdn = s->vx[i] * nrm[0] + s->vy[i] * nrm[1] + s->vz[i] * nrm[2];
        if (vdn < 0.0) {
            s->vx[i] -= vdn * nrm[0];
            s->vy[i] -= vdn * nrm[1];
            s->vz[i] -= vdn * nrm[2];
        }
        const double tvx = s->vx[i] - vdn * nrm[0], tvy = s->vy[i] - vdn * nrm[1], tvz = s->vz[i] - vdn * nrm[2];
        const double tvm = sqrt(tvx * tvx + tvy * tvy + tvz * tvz);
        const double m = s->mass[i];
        const double nf = tvm > 0.0 ? fmax(m * pen / (dt * dt), 1e-15) : 1e-15;
        const double fimp = mu * nf * dt;
        if (tvm > 0.0 && fimp > 0.0) {
            const double sc = fmin(1.0, (fimp / fmax(m, 1e-15)) / tvm);
            s->vx[i] -= tvx * sc;
            s->vy[i] -= tvy * sc;
            s->vz[i] -= tvz * sc;
        }
        const double slip = sqrt(s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
        const double heat = nf * slip * dt * (1.0 - hp);
        if (heat > 0.0) {
            const double pm = fmax(p->rho_phys, 1.0) * fmax(s->vol[i], 1e-24);
            s->T[i] = fmin(s->T[i] + heat / (fmax(pm, 1e-15) * p->cp), p->Tm);
        }
    }
}

/* applyAdiabaticHeatingKernel, src/AdiabaticShearModel.cu:104-177, as
 * AdiabaticShearModel::update runs it after g2pKernel (:262-279;
 * src/MPMSolver.cu:1130-1132).  detectShearBandsKernel (:32-67) only marks
 * the LOD zone ACTIVE, which lodClassifyKernel rewrites before anything reads
 * it, so it has no effect to restate.  The reference's guard
 * T <= 25.5 degC with its 25 degC ambient is T <= Tamb + asb_touch_rise. */
static void asb_heating(const orc_params *p, orc_state *s, double dt) {
    const double rhocp = fmax(p->rho_phys * p->cp, 1e-12);
    const double min_rate = fmax(p->asb_critical_rate * 0.5, 5000.0);
    const double Tcap = p->asb_max_temp_ratio * p->Tm;
    for (int i = 0; i < s->n; ++i) {
        if (s->status[i] == ORC_CHIP) {             /* :114-117 */
            s->asb[i] = 0;
            continue;
        }
        if (s->status[i] != ORC_ACTIVE) continue;
        if (s->T[i] <= p->Tamb + p->asb_touch_rise) continue;   /* :123 */
        const double edot = s->edot[i];
        if (edot < min_rate) {                                  /* :131-136 */
            s->asb[i] = s->asb[i] > 0 ? s->asb[i] - 1 : 0;
            continue;
        }
        const double *sg = s->sig + 6 * (int64_t)i;             /* :139-143 von Mises */
        const double s1 = sg[0] - sg[1], s2 = sg[1] - sg[2], s3 = sg[2] - sg[0];
        const double seq = sqrt(0.5 * (s1 * s1 + s2 * s2 + s3 * s3 + 6.0 * (sg[3] * sg[3] + sg[4] * sg[4] + sg[5] * sg[5])));
        double dT = (p->asb_taylor_quinney * seq * edot * dt) / rhocp;      /* :148-149 */
        s->asb[i] = s->asb[i] + 1 < 10 ? s->asb[i] + 1 : 10;                /* :155 */
        if (edot > p->asb_critical_rate && s->asb[i] >= 3) {                /* :157-164 */
            const double ratio = edot / fmax(p->asb_critical_rate, 1.0);
            dT *= fmin(1.0 + 1.5 * (ratio - 1.0), 2.5);
        }
        double maxDT = p->asb_taylor_quinney * seq * (edot * dt) / rhocp;   /* :169-172 */
        maxDT = fmin(maxDT, 100.0);
        if (maxDT > 0.0 && dT > maxDT) dT = maxDT;
        s->T[i] = fmin(s->T[i] + dT, Tcap);                                /* :175-176 */
    }
}

void orc_asb_heat(const orc_params *p, orc_state *s, double dt) {
    if (s->asb) asb_heating(p, s, dt);
}

/* ---------------------------------------------------------------- voxel SDF build */

/* Squared distance from p to triangle abc and the closest point: the region
 * tests of Ericson's closest-point-on-triangle algorithm (Real-Time Collision
 * Detection, 5.1.5), with the reference's interior case
 * a + u (b - a) + v (c - a), u = 1 - v - w (src/ToolSDF.cu:92-167). */
static float tri_dist2(const float p[3], const float a[3], const float b[3], const float c[3], float q[3]) {
    float ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int k = 0; k < 3; ++k) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ap[k] = p[k] - a[k]; }
    const float d1 = ab[0] * ap[0] + ab[1] * ap[1] + ab[2] * ap[2];
    const float d2 = ac[0] * ap[0] + ac[1] * ap[1] + ac[2] * ap[2];
    if (d1 <= 0.0f && d2 <= 0.0f) {
        for (int k = 0; k < 3; ++k) q[k] = a[k];
    } else {
        for (int k = 0; k < 3; ++k) bp[k] = p[k] - b[k];
        const float d3 = ab[0] * bp[0] + ab[1] * bp[1] + ab[2] * bp[2];
        const float d4 = ac[0] * bp[0] + ac[1] * bp[1] + ac[2] * bp[2];
        const float vc = d1 * d4 - d3 * d2;
        if (d3 >= 0.0f && d4 <= d3) {
            for (int k = 0; k < 3; ++k) q[k] = b[k];
        } else if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
            const float v = d1 / (d1 - d3);
            for (int k = 0; k < 3; ++k) q[k] = a[k] + v * ab[k];
        } else {
            for (int k = 0; k < 3; ++k) cp[k] = p[k] - c[k];
            const float d5 = ab[0] * cp[0] + ab[1] * cp[1] + ab[2] * cp[2];
            const float d6 = ac[0] * cp[0] + ac[1] * cp[1] + ac[2] * cp[2];
            const float vb = d5 * d2 - d1 * d6;
            const float va = d3 * d6 - d5 * d4;
            if (d6 >= 0.0f && d5 <= d6) {
                for (int k = 0; k < 3; ++k) q[k] = c[k];
            } else if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
                const float w = d2 / (d2 - d6);
                for (int k = 0; k < 3; ++k) q[k] = a[k] + w * ac[k];
            } else if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
                const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                for (int k = 0; k < 3; ++k) q[k] = b[k] + w * (c[k] - b[k]);
            } else {
                const float den = 1.0f / (va + vb + vc);
                const float v = vb * den, w = vc * den;
                const float u = 1.0f - v - w;
                for (int k = 0; k < 3; ++k) q[k] = a[k] + u * (b[k] - a[k]) + v * (c[k] - a[k]);
            }
        }
    }
    const float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    return dx * dx + dy * dy + dz * dz;
}

int orc_tool_sdf_build(const float *verts, int32_t nv, const int32_t *tris, int32_t nt, const float *normals,
                       double padding, int32_t voxels_per_axis, int32_t dims[3], float origin[3], float *voxel,
                       float *values) {
    if (nv <= 0 || nt <= 0 || voxels_per_axis <= 0) return -1;
    /* ToolSDF::build: bounding box, padding, isotropic voxel on the longest
     * axis, dims = extent / voxel + 2 (at most 256) */
    float bmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < nv; ++i)
        for (int k = 0; k < 3; ++k) {
            bmin[k] = fminf(bmin[k], verts[3 * i + k]);
            bmax[k] = fmaxf(bmax[k], verts[3 * i + k]);
        }
    const float pad = (float)padding;
    for (int k = 0; k < 3; ++k) { bmin[k] -= pad; bmax[k] += pad; }
    const float ext[3] = {bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2]};
    const float vox = fmaxf(ext[0], fmaxf(ext[1], ext[2])) / (float)voxels_per_axis;
    for (int k = 0; k < 3; ++k) {
        origin[k] = bmin[k];
        dims[k] = (int)(ext[k] / vox) + 2;
        if (dims[k] > 256) dims[k] = 256;
    }
    *voxel = vox;
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const int64_t total = (int64_t)nx * ny * nz;
    if (total <= 0) return -1;
    if (!values) return 0;
    float *g = values;
    for (int64_t i = 0; i < total; ++i) g[i] = FLT_MAX;
    const float inv = 1.0f / vox;
    /* computeSDFCPU: each triangle's squared distance to the voxel centres of
     * its bounding box grown by one voxel below and two above (:396-422) */
    for (int t = 0; t < nt; ++t) {
        const float *a = verts + 3 * tris[3 * t], *b = verts + 3 * tris[3 * t + 1], *c = verts + 3 * tris[3 * t + 2];
        float lo[3], hi[3];
        int i0[3], i1[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(a[k], fminf(b[k], c[k]));
            hi[k] = fmaxf(a[k], fmaxf(b[k], c[k]));
            const int l = (int)((lo[k] - origin[k]) * inv) - 1, h = (int)((hi[k] - origin[k]) * inv) + 2;
            i0[k] = l > 0 ? l : 0;
            i1[k] = h < dims[k] - 1 ? h : dims[k] - 1;
        }
        for (int iz = i0[2]; iz <= i1[2]; ++iz)
            for (int iy = i0[1]; iy <= i1[1]; ++iy)
                for (int ix = i0[0]; ix <= i1[0]; ++ix) {
                    const float p[3] = {origin[0] + (ix + 0.5f) * vox, origin[1] + (iy + 0.5f) * vox,
                                        origin[2] + (iz + 0.5f) * vox};
                    float q[3];
                    const float d2 = tri_dist2(p, a, b, c, q);
                    const int64_t idx = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
                    if (d2 < g[idx]) g[idx] = d2;
                }
    }
    for (int64_t i = 0; i < total; ++i)
        if (g[i] < FLT_MAX) g[i] = sqrtf(g[i]);
    /* sign within two voxels of the surface from the nearest triangle's normal
     * (:444-490; bounding boxes grown by one voxel; the first nearest wins) */
    const float band = vox * 2.0f;
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const int64_t idx = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
                const float dist = g[idx];
                if (dist > band) continue;
                const float p[3] = {origin[0] + (ix + 0.5f) * vox, origin[1] + (iy + 0.5f) * vox,
                                    origin[2] + (iz + 0.5f) * vox};
                float best = FLT_MAX, bn[3] = {0, 0, 0}, bq[3] = {0, 0, 0};
                for (int t = 0; t < nt; ++t) {
                    const float *a = verts + 3 * tris[3 * t], *b = verts + 3 * tris[3 * t + 1],
                                *c = verts + 3 * tris[3 * t + 2];
                    int skip = 0;
                    for (int k = 0; k < 3; ++k) {
                        const float lo = fminf(a[k], fminf(b[k], c[k])), hi = fmaxf(a[k], fmaxf(b[k], c[k]));
                        if (p[k] < lo - vox || p[k] > hi + vox) skip = 1;
                    }
                    if (skip) continue;
                    float q[3];
                    const float d2 = tri_dist2(p, a, b, c, q);
                    if (d2 < best) {
                        best = d2;
                        for (int k = 0; k < 3; ++k) { bn[k] = normals[3 * t + k]; bq[k] = q[k]; }
                    }
                }
                if (best < FLT_MAX) {
                    const float dot = (p[0] - bq[0]) * bn[0] + (p[1] - bq[1]) * bn[1] + (p[2] - bq[2]) * bn[2];
                    if (dot < 0.0f) g[idx] = -dist;
                }
            }
    /* three in-place passes give a voxel not reached yet its nearest known
     * neighbour's |distance| + half a voxel (:494-524), then the rest a large
     * distance (:526-531) */
    for (int pass = 0; pass < 3; ++pass)
        for (int iz = 1; iz < nz - 1; ++iz)
            for (int iy = 1; iy < ny - 1; ++iy)
                for (int ix = 1; ix < nx - 1; ++ix) {
                    const int64_t idx = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
                    if (g[idx] < FLT_MAX) continue;
                    float nd = FLT_MAX;
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                if (!dx && !dy && !dz) continue;
                                const float v = fabsf(g[(ix + dx) + (int64_t)nx * ((iy + dy) + (int64_t)ny * (iz + dz))]);
                                if (v < nd) nd = v;
                            }
                    if (nd < FLT_MAX) g[idx] = nd + vox * 0.5f;
                }
    const int dmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
    for (int64_t i = 0; i < total; ++i)
        if (g[i] >= FLT_MAX) g[i] = vox * (float)dmax;
    return 0;
}

/* ---------------------------------------------------------------- voxel SDF contact */

/* value rounded to nearest on the texture unit's 1/256 grid (ties up) */
static double q8(double f) { return floor(f * 256.0 + 0.5) * (1.0 / 256.0); }

static float texel(const orc_sdf_grid *g, int i, int j, int k) {
    i = i < 0 ? 0 : (i >= g->nx ? g->nx - 1 : i);
    j = j < 0 ? 0 : (j >= g->ny ? g->ny - 1 : j);
    k = k < 0 ? 0 : (k >= g->nz ? g->nz - 1 : k);
    return g->v[i + (int64_t)g->nx * (j + (int64_t)g->ny * k)];
}

static float clampc(float x, int n) {
    return x < 0.5f ? 0.5f : (x > (float)n - 0.5f ? (float)n - 0.5f : x);
}

/* The filtering model, measured on the B200 against the hardware's own
 * fetches (tests/golden/kernels/tex_probe.npz, exact on every probe point):
 * coordinates clamped to [1/2, n - 1/2]; fractional weights a, b, c rounded to
 * 1/256; the eight corner weights split hierarchically on the same 1/256 grid
 * so that they sum to 1: z exactly (1 - c, c); within a z slice the x = 1 side
 * rounded and x = 0 the rest; within the x = 1 half the y = 1 corner rounded
 * and y = 0 the rest, within the x = 0 half the y = 0 corner rounded and
 * y = 1 the rest.  The texels are then summed with these weights; the unit's
 * own sum carries a little less than exact precision, so the result here (the
 * exact sum rounded once) can differ from it by one float ulp (1.4 % of the
 * probe points). */
float orc_tex3d(const orc_sdf_grid *g, float x, float y, float z) {
    const float xb = clampc(x, g->nx) - 0.5f, yb = clampc(y, g->ny) - 0.5f, zb = clampc(z, g->nz) - 0.5f;
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const int i = (int)fx, j = (int)fy, k = (int)fz;
    const double a = q8(xb - fx), b = q8(yb - fy), c = q8(zb - fz);
    double r = 0.0;   /* exact: 8-bit weights times 24-bit texels */
    for (int dk = 0; dk < 2; ++dk) {
        const double wz = dk ? c : 1.0 - c;
        const double wx1 = q8(wz * a), wx0 = wz - wx1;
        const double w11 = q8(wx1 * b), w10 = wx1 - w11;
        const double w00 = q8(wx0 * (1.0 - b)), w01 = wx0 - w00;
        r += w00 * texel(g, i, j, k + dk);
        r += w10 * texel(g, i + 1, j, k + dk);
        r += w01 * texel(g, i, j + 1, k + dk);
        r += w11 * texel(g, i + 1, j + 1, k + dk);
    }
    return (float)r;
}

/* xpbdContactSDFKernel, src/ContactSolver.cu:797-923, with the same float and
 * double arithmetic: world -> SDF rest frame (:825-829), voxel coordinates
 * and the grid test (:832-840), the sampled distance (:843-845), the normal
 * from central differences half a voxel apart (:848-859), push-out to the
 * contact radius (:863-869), removal of an approaching normal velocity
 * (:872-877), Coulomb friction on the tangential velocity taken with the
 * normal component before that removal (:881-898), heating by
 * (1 - heat partition) of the friction work (:901-916), metrics (:918-922). */
void orc_contact_sdf(const orc_sdf_grid *g, const orc_contact_sdf_args *a, orc_state *s, int64_t *count,
                     double *heat, double *force) {
    int64_t cnt = 0;
    double hsum = 0.0, fsum = 0.0;
    for (int ip = 0; ip < s->n; ++ip) {
        if (s->status[ip] == ORC_INACTIVE || s->status[ip] == ORC_FIXED) continue;
        const float dx = (float)s->x[ip] - a->cx;
        const float dy = (float)s->y[ip] - a->cy;
        const float lx = dx * a->cos_a + dy * a->sin_a;
        const float ly = -dx * a->sin_a + dy * a->cos_a;
        const float lz = (float)s->z[ip] - a->cz;
        const float tx = (lx - g->ox) / g->voxel;
        const float ty = (ly - g->oy) / g->voxel;
        const float tz = (lz - g->oz) / g->voxel;
        if (tx < 0 || ty < 0 || tz < 0 || tx > g->nx - 1 || ty > g->ny - 1 || tz > g->nz - 1) continue;
        const float sdf = orc_tex3d(g, tx, ty, tz);
        if (sdf >= a->radius) continue;
        const float eps = 0.5f;
        const float gx = (orc_tex3d(g, tx + eps, ty, tz) - orc_tex3d(g, tx - eps, ty, tz)) / (eps * 2.0f * g->voxel);
        const float gy = (orc_tex3d(g, tx, ty + eps, tz) - orc_tex3d(g, tx, ty - eps, tz)) / (eps * 2.0f * g->voxel);
        const float gz = (orc_tex3d(g, tx, ty, tz + eps) - orc_tex3d(g, tx, ty, tz - eps)) / (eps * 2.0f * g->voxel);
        const float glen = sqrtf(gx * gx + gy * gy + gz * gz);
        if (glen < 1e-10f) continue;
        const float nx = gx / glen, ny = gy / glen, nz = gz / glen;
        const float pen = a->radius - sdf;
        if (pen <= 0.0f) continue;
        s->x[ip] += nx * pen;
        s->y[ip] += ny * pen;
        s->z[ip] += nz * pen;
        const float vdn = (float)(s->vx[ip] * nx + s->vy[ip] * ny + s->vz[ip] * nz);
        if (vdn < 0.0f) {
            s->vx[ip] -= vdn * nx;
            s->vy[ip] -= vdn * ny;
            s->vz[ip] -= vdn * nz;
        }
        const float tvx = (float)s->vx[ip] - vdn * nx;
        const float tvy = (float)s->vy[ip] - vdn * ny;
        const float tvz = (float)s->vz[ip] - vdn * nz;
        const float tvm = sqrtf(tvx * tvx + tvy * tvy + tvz * tvz);
        const float nf = (tvm > 0.0f) ? fmaxf((float)s->mass[ip] * pen / (a->dt * a->dt), 1e-15f) : 1e-15f;
        const float ff = a->friction * nf;
        const float fimp = ff * a->dt;
        if (tvm > 0.0f && fimp > 0.0f) {
            const float mdv = fimp / fmaxf((float)s->mass[ip], 1e-15f);
            const float sc = fminf(1.0f, mdv / tvm);
            s->vx[ip] -= tvx * sc;
            s->vy[ip] -= tvy * sc;
            s->vz[ip] -= tvz * sc;
        }
        const float slip = sqrtf((float)s->vx[ip] * (float)s->vx[ip] + (float)s->vy[ip] * (float)s->vy[ip] +
                                 (float)s->vz[ip] * (float)s->vz[ip]);
        const double fw = nf * slip * a->dt;
        const double hpp = fw * (1.0 - a->heat_partition);
        if (hpp > 0.0) {
            const double vol = (s->vol[ip] > 1e-24) ? s->vol[ip] : (s->mass[ip] / fmax(s->mass[ip] / s->vol[ip], 1.0));
            const double pm = fmax(a->rho_phys, 1.0) * fmax(vol, 1e-24);
            const double dT = hpp / (fmax(pm, 1e-15) * a->cp);
            s->T[ip] = fmin(s->T[ip] + dT, a->Tm);
        }
        cnt += 1;
        hsum += fw;
        fsum += (double)fmaxf(nf, 1e-15f);
    }
    *count = cnt;
    *heat = hsum;
    *force = fsum;
}

int orc_step(const orc_params *p, orc_state *s, const orc_tool_samples *tool, double *grid, double dt, int32_t nsteps,
             int64_t step0, double t0, int32_t nthreads) {
    int err = 0;
    if (nthreads < 1) nthreads = 1;
    const int64_t ng = orc_grid_doubles(p);
    for (int32_t k = 0; k < nsteps; ++k) {
        const double t = t0 + (double)k * dt;
        double pr[3], tip[3];
        for (int d = 0; d < 3; ++d) pr[d] = p->tool_p0[d] + p->tool_v[d] * t;
        tip[0] = pr[0]; tip[1] = pr[1]; tip[2] = pr[2] + p->tool_tip_dz;
        if (p->lod_enabled) lod_classify(p, s, tip);
        memset(grid, 0, sizeof(double) * (size_t)ng);                 /* resetGridKernel :112 */
        err |= p2g(p, s, grid, nthreads);
        grid_update(p, grid, dt, tool, pr);
        if (p->heat_conduction) heat_diffuse(p, grid, dt);
        g2p(p, s, grid, dt, nthreads);
        if (p->asb_enabled && s->asb) asb_heating(p, s, dt);
        if (s->extf) memset(s->extf, 0, sizeof(double) * 3 * (size_t)s->n);  /* :682-688 */
        const int64_t cnt = step0 + k;
        if (p->chip_sep_enabled && p->chip_every > 0 && (cnt % p->chip_every) == 0) chip_separation(p, s, tip[2]);
        if (p->contact_every > 0 && ((cnt + 1) % p->contact_every) == 0) {
            /* after the step, at the tool pose of its end time */
            double pe[3];
            for (int d = 0; d < 3; ++d) pe[d] = p->tool_p0[d] + p->tool_v[d] * (t + dt);
            if (p->tool_sdf) {
                const orc_contact_sdf_args a = {(float)pe[0], (float)pe[1], (float)pe[2], cosf(p->tool_sdf_angle),
                                                sinf(p->tool_sdf_angle), (float)p->contact_radius,
                                                (float)p->contact_friction, (float)p->contact_heat_partition,
                                                (float)dt, 0.0f, p->cp, p->rho_phys, p->Tm};
                int64_t c;
                double hw, fn;
                orc_contact_sdf(p->tool_sdf, &a, s, &c, &hw, &fn);
            } else {
                particle_contact(p, s, pe, dt);
            }
        }
    }
    return err;
}

/* ------------------------------------------------ MPMWorkpieceSolver semantics */

/* Node channels of the workpiece solver's grid (MPMGridNodeGPU,
 * include/MPMWorkpieceSolver.cuh:44-55): mass, momentum then velocity,
 * force, T m, and the node temperature after diffusion. */
enum { WS_M, WS_VX, WS_VY, WS_VZ, WS_FX, WS_FY, WS_FZ, WS_TM, WS_TN, WS_N };

int64_t orc_ws_grid_doubles(const orc_params *p) { return nnodes(p) * WS_N; }

/* computeWeights (src/MPMWorkpieceSolver.cu:52-90): the 8 trilinear nodes in
 * dz, dy, dx order; a node outside the grid has index -1 and weight 0. */
static void ws_weights(const orc_params *p, double x, double y, double z, int64_t id[8], double w[8],
                       double g[8][3]) {
    const double rx = (x - p->ox) / p->dx, ry = (y - p->oy) / p->dx, rz = (z - p->oz) / p->dx;
    const int bx = (int)floor(rx), by = (int)floor(ry), bz = (int)floor(rz);
    const double fx = rx - bx, fy = ry - by, fz = rz - bz;
    int n = 0;
    for (int dz = 0; dz <= 1; ++dz)
        for (int dy = 0; dy <= 1; ++dy)
            for (int dx = 0; dx <= 1; ++dx, ++n) {
                const int i = bx + dx, j = by + dy, k = bz + dz;
                if (i < 0 || j < 0 || k < 0 || i >= p->nx || j >= p->ny || k >= p->nz) {
                    id[n] = -1;
                    w[n] = 0.0;
                    g[n][0] = g[n][1] = g[n][2] = 0.0;
                    continue;
                }
                const double wx = dx ? fx : 1.0 - fx, wy = dy ? fy : 1.0 - fy, wz = dz ? fz : 1.0 - fz;
                const double dwx = dx ? 1.0 / p->dx : -1.0 / p->dx;
                const double dwy = dy ? 1.0 / p->dx : -1.0 / p->dx;
                const double dwz = dz ? 1.0 / p->dx : -1.0 / p->dx;
                id[n] = ((int64_t)k * p->ny + j) * p->nx + i;
                w[n] = wx * wy * wz;
                g[n][0] = dwx * wy * wz;
                g[n][1] = wx * dwy * wz;
                g[n][2] = wx * wy * dwz;
            }
}

/* equivalentStress (:19-25). */
static double ws_eq(double xx, double yy, double zz, double xy, double xz, double yz) {
    const double s1 = xx - yy, s2 = yy - zz, s3 = zz - xx;
    return sqrt(0.5 * (s1 * s1 + s2 * s2 + s3 * s3 + 6.0 * (xy * xy + xz * xz + yz * yz)));
}

/* johnsonCookStress (:43-50): rate term floored at 1, thermal term at 0.01. */
static double ws_flow(const orc_params *p, double eps, double edot, double T) {
    const double strain = p->A + p->B * pow(fmax(eps, 0.0), p->n);
    const double ratio = fmax(edot / fmax(p->edot0, 1e-9), 1.0);
    const double rate = 1.0 + p->C * log(ratio);
    const double ts = fmax(0.0, fmin(1.0, (T - p->Tamb) / fmax(p->Tm - p->Tamb, 1.0)));
    return strain * rate * fmax(0.01, 1.0 - pow(ts, p->m));
}

/* mpmP2GKernel (:98-134): mass, momentum and T m of every particle that is
 * not INACTIVE; the stress force (and the particle force) of ACTIVE and
 * FIXED particles, the particle force alone of CHIP ones. */
static void ws_p2g(const orc_params *p, const orc_state *s, double *g) {
    const int64_t nn = nnodes(p);
    for (int32_t ip = 0; ip < s->n; ++ip) {
        const int st = s->status[ip];
        if (st == ORC_INACTIVE) continue;
        int64_t id[8];
        double w[8], gr[8][3];
        ws_weights(p, s->x[ip], s->y[ip], s->z[ip], id, w, gr);
        const double *sg = s->sig + 6 * (int64_t)ip;
        const double fp[3] = {s->extf ? s->extf[3 * (int64_t)ip] : 0.0, s->extf ? s->extf[3 * (int64_t)ip + 1] : 0.0,
                              s->extf ? s->extf[3 * (int64_t)ip + 2] : 0.0};
        for (int n = 0; n < 8; ++n) {
            const int64_t gi = id[n];
            if (gi < 0 || w[n] <= 0.0) continue;
            const double m = s->mass[ip] * w[n];
            g[WS_M * nn + gi] += m;
            g[WS_VX * nn + gi] += s->vx[ip] * m;
            g[WS_VY * nn + gi] += s->vy[ip] * m;
            g[WS_VZ * nn + gi] += s->vz[ip] * m;
            g[WS_TM * nn + gi] += s->T[ip] * m;
            if (st == ORC_ACTIVE || st == ORC_FIXED) {
                const double fX = -(sg[0] * gr[n][0] + sg[3] * gr[n][1] + sg[4] * gr[n][2]) * s->vol[ip];
                const double fY = -(sg[3] * gr[n][0] + sg[1] * gr[n][1] + sg[5] * gr[n][2]) * s->vol[ip];
                const double fZ = -(sg[4] * gr[n][0] + sg[5] * gr[n][1] + sg[2] * gr[n][2]) * s->vol[ip];
                g[WS_FX * nn + gi] += fX + fp[0] * w[n];
                g[WS_FY * nn + gi] += fY + fp[1] * w[n];
                g[WS_FZ * nn + gi] += fZ + fp[2] * w[n];
            } else if (st == ORC_CHIP) {
                g[WS_FX * nn + gi] += fp[0] * w[n];
                g[WS_FY * nn + gi] += fp[1] * w[n];
                g[WS_FZ * nn + gi] += fp[2] * w[n];
            }
        }
    }
}

/* mpmGridUpdateKernel (:136-192): velocity = momentum / mass; nodes at or
 * below the fixture (z <= min z + thickness + dx) stop; then the force
 * impulse; then the tool: the nearest sample within the contact radius (the
 * first of equal ones) gives the normal n = (node - sample) / |.|, and an
 * approaching normal velocity (v.n < 0) is removed, heating the node by
 * 0.5 m vn^2 damping / (m cp) (capped with the thermal clamp) and adding
 * |m vn / dt| to the contact force. */
static void ws_grid(const orc_params *p, const orc_ws_params *wp, double *g, double dt, const orc_tool_samples *tool,
                    const double pr[3], double *force) {
    const int64_t nn = nnodes(p);
    double fsum = 0.0;
    for (int64_t idx = 0; idx < nn; ++idx) {
        const double m = g[WS_M * nn + idx];
        if (m <= 1e-18) continue;
        double v[3] = {g[WS_VX * nn + idx] / m, g[WS_VY * nn + idx] / m, g[WS_VZ * nn + idx] / m};
        const int i = (int)(idx % p->nx);
        const int64_t t = idx / p->nx;
        const int j = (int)(t % p->ny), k = (int)(t / p->ny);
        const double pos[3] = {p->ox + i * p->dx, p->oy + j * p->dx, p->oz + k * p->dx};
        if (pos[2] <= p->oz + p->fixture_thickness + p->dx) {
            g[WS_VX * nn + idx] = g[WS_VY * nn + idx] = g[WS_VZ * nn + idx] = 0.0;
            continue;
        }
        v[0] += (g[WS_FX * nn + idx] / m) * dt;
        v[1] += (g[WS_FY * nn + idx] / m) * dt;
        v[2] += (g[WS_FZ * nn + idx] / m) * dt;
        if (tool && tool->n > 0) {
            double r2 = wp->tool_contact_radius * wp->tool_contact_radius, bn[3] = {0.0, 0.0, 0.0};
            int hit = 0;
            for (int q = 0; q < tool->n; ++q) {
                const double d[3] = {pos[0] - (pr[0] + tool->ox[q]), pos[1] - (pr[1] + tool->oy[q]),
                                     pos[2] - (pr[2] + tool->oz[q])};
                const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (d2 < r2 && d2 > 1e-20) {
                    r2 = d2;
                    const double len = sqrt(d2);
                    if (len > 1e-12) { bn[0] = d[0] / len; bn[1] = d[1] / len; bn[2] = d[2] / len; }
                    else { bn[0] = bn[1] = bn[2] = 0.0; }
                    hit = 1;
                }
            }
            if (hit) {
                const double vn = v[0] * bn[0] + v[1] * bn[1] + v[2] * bn[2];
                if (vn < 0.0) {
                    fsum += fabs(m * vn / fmax(dt, 1e-15));
                    for (int a = 0; a < 3; ++a) v[a] -= vn * bn[a];
                    const double heat = 0.5 * m * vn * vn * wp->contact_damping;
                    double dT = heat / fmax(m * p->cp, 1e-12);
                    if (wp->thermal_clamp) dT = fmin(dT, wp->max_contact_temp_rise);
                    g[WS_TM * nn + idx] += dT * m;
                }
            }
        }
        g[WS_VX * nn + idx] = v[0];
        g[WS_VY * nn + idx] = v[1];
        g[WS_VZ * nn + idx] = v[2];
    }
    if (force) *force = fsum;
}

/* mpmG2PKernel (:264-400) on every particle that is not INACTIVE. */
static void ws_g2p(const orc_params *p, const orc_ws_params *wp, orc_state *s, const double *g, double dt,
                   int diffused) {
    const int64_t nn = nnodes(p);
    const double G = p->E / (2.0 * (1.0 + p->nu)), K = p->E / (3.0 * (1.0 - 2.0 * p->nu));
    for (int32_t ip = 0; ip < s->n; ++ip) {
        const int st = s->status[ip];
        if (st == ORC_INACTIVE) continue;
        int64_t id[8];
        double w[8], gr[8][3];
        ws_weights(p, s->x[ip], s->y[ip], s->z[ip], id, w, gr);
        double v[3] = {0.0, 0.0, 0.0}, temp = 0.0, wsum = 0.0, L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int n = 0; n < 8; ++n) {
            const int64_t gi = id[n];
            if (gi < 0 || w[n] <= 0.0) continue;
            const double m = g[WS_M * nn + gi];
            if (m <= 1e-18) continue;
            const double nv[3] = {g[WS_VX * nn + gi], g[WS_VY * nn + gi], g[WS_VZ * nn + gi]};
            for (int a = 0; a < 3; ++a) v[a] += nv[a] * w[n];
            temp += (diffused ? g[WS_TN * nn + gi] : g[WS_TM * nn + gi] / m) * w[n];
            wsum += w[n];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) L[a][b] += nv[a] * gr[n][b];
        }
        double *ext = s->extf ? s->extf + 3 * (int64_t)ip : NULL;
        if (st == ORC_FIXED) {
            s->vx[ip] = s->vy[ip] = s->vz[ip] = 0.0;
            if (ext) ext[0] = ext[1] = ext[2] = 0.0;
            continue;
        }
        s->vx[ip] = v[0]; s->vy[ip] = v[1]; s->vz[ip] = v[2];
        s->x[ip] += v[0] * dt;
        s->y[ip] += v[1] * dt;
        s->z[ip] += v[2] * dt;
        if (wsum > 1e-8) s->T[ip] = fmin(fmax(temp / wsum, p->Tamb), p->Tm);
        double *sg = s->sig + 6 * (int64_t)ip, *bs = s->bs + 6 * (int64_t)ip;
        if (st == ORC_ACTIVE) {
            const double Dxx = L[0][0], Dyy = L[1][1], Dzz = L[2][2];
            const double Dxy = 0.5 * (L[0][1] + L[1][0]), Dxz = 0.5 * (L[0][2] + L[2][0]),
                         Dyz = 0.5 * (L[1][2] + L[2][1]);
            const double tr = Dxx + Dyy + Dzz;
            const double dxx = Dxx - tr / 3.0, dyy = Dyy - tr / 3.0, dzz = Dzz - tr / 3.0;
            const double rate = sqrt(2.0 / 3.0 * (dxx * dxx + dyy * dyy + dzz * dzz +
                                                   2.0 * (Dxy * Dxy + Dxz * Dxz + Dyz * Dyz)));
            s->edot[ip] = rate;
            const double pinc = K * tr * dt;
            sg[0] += (2.0 * G * dxx) * dt + pinc;
            sg[1] += (2.0 * G * dyy) * dt + pinc;
            sg[2] += (2.0 * G * dzz) * dt + pinc;
            sg[3] += 2.0 * G * Dxy * dt;
            sg[4] += 2.0 * G * Dxz * dt;
            sg[5] += 2.0 * G * Dyz * dt;
            const double sh[6] = {sg[0] - bs[0], sg[1] - bs[1], sg[2] - bs[2], sg[3] - bs[3], sg[4] - bs[4],
                                  sg[5] - bs[5]};
            const double seq = ws_eq(sh[0], sh[1], sh[2], sh[3], sh[4], sh[5]);
            const double flow = ws_flow(p, s->eps[ip], s->edot[ip], s->T[ip]);
            if (seq > flow && seq > 1e-9) {
                const double sc = flow / seq;
                for (int q = 0; q < 6; ++q) sg[q] = bs[q] + sc * sh[q];
                const double dp = (seq - flow) / fmax(3.0 * G, 1.0);
                if (p->Hkin > 0.0 && dp > 0.0) {
                    const double ns = p->Hkin * dp / seq;
                    for (int q = 0; q < 6; ++q) bs[q] += ns * sh[q];
                }
                s->eps[ip] += dp;
                double dT = 0.9 * flow * dp / fmax(p->rho_phys * p->cp, 1.0);
                if (wp->thermal_clamp) dT = fmin(dT, wp->max_contact_temp_rise);
                s->T[ip] = fmin(s->T[ip] + dT, p->Tm);
            }
            if (rate > 0.0) s->D[ip] += (rate * dt) / fmax(wp->failure_strain, 1e-3);
            if (s->D[ip] > 0.7 * p->Dth && s->D[ip] < p->Dth) {
                const double dg = fmax(0.0, (p->Dth - s->D[ip]) / (p->Dth * 0.3));
                for (int q = 0; q < 6; ++q) { sg[q] *= dg; bs[q] *= dg; }
                s->sres[ip] = fmax(s->sres[ip], ws_eq(sg[0], sg[1], sg[2], sg[3], sg[4], sg[5]));
            }
        }
        if (st == ORC_ACTIVE && (s->D[ip] >= p->Dth || s->eps[ip] >= wp->critical_plastic_strain ||
                                 s->T[ip] >= p->Tm * wp->thermal_chip_ratio)) {
            s->status[ip] = ORC_CHIP;
            s->sres[ip] = fmax(s->sres[ip], ws_eq(sg[0], sg[1], sg[2], sg[3], sg[4], sg[5]));
            for (int q = 0; q < 6; ++q) { sg[q] = 0.0; bs[q] = 0.0; }
            s->D[ip] = fmax(s->D[ip], p->Dth);
        }
        if (ext) ext[0] = ext[1] = ext[2] = 0.0;
    }
}

/* The workpiece solver's chipFractureAndSeparationKernel (:667-725):
 * ACTIVE particles below tip z - 1.5 dx with any plastic strain become
 * CHIP; CHIP particles at 1.5 Dth of damage get the id-seeded push and
 * damage 0.5 Dth. */
static void ws_chip(const orc_params *p, orc_state *s, double tipZ) {
    for (int32_t ip = 0; ip < s->n; ++ip) {
        const int st = s->status[ip];
        if (st == ORC_INACTIVE) continue;
        double *sg = s->sig + 6 * (int64_t)ip, *bs = s->bs + 6 * (int64_t)ip;
        if (st == ORC_ACTIVE) {
            if (s->z[ip] < tipZ - p->dx * 1.5 && s->eps[ip] > 1e-6) {
                s->status[ip] = ORC_CHIP;
                s->sres[ip] = fmax(s->sres[ip], sqrt(sg[0] * sg[0] + sg[1] * sg[1] + sg[2] * sg[2]));
                for (int q = 0; q < 6; ++q) { sg[q] = 0.0; bs[q] = 0.0; }
                s->D[ip] = fmax(s->D[ip], p->Dth);
            }
            continue;
        }
        if (st == ORC_CHIP) {
            if (s->D[ip] < p->Dth * 1.5) continue;
            const uint32_t seed = (uint32_t)s->id[ip] * 2654435761u;
            const double rx = (double)((seed >> 16) & 0xFF) / 255.0 - 0.5;
            const double ry = (double)((seed >> 8) & 0xFF) / 255.0 - 0.5;
            const double rz = (double)(seed & 0xFF) / 255.0 - 0.5;
            const double sp = sqrt(s->vx[ip] * s->vx[ip] + s->vy[ip] * s->vy[ip] + s->vz[ip] * s->vz[ip]);
            const double pm = sp * 0.3 + 0.5;
            s->vx[ip] += rx * pm;
            s->vy[ip] += ry * pm;
            s->vz[ip] += rz * pm;
            s->D[ip] = p->Dth * 0.5;
        }
    }
}

/* The node-temperature step of the workpiece solver: diffusion (WS_TM ->
 * WS_TN) through the common restatement. */
static void ws_diffuse(const orc_params *p, double *g, double dt) {
    const int64_t nn = nnodes(p);
    orc_heat_diffuse(p, g + WS_M * nn, g + WS_TM * nn, g + WS_TN * nn, dt);
}

void orc_ws_step(const orc_params *p, const orc_ws_params *w, orc_state *s, const orc_tool_samples *tool, double *grid,
                 double dt, int32_t nsteps, int64_t step0, double t0, double *contact_force) {
    const int64_t ng = orc_ws_grid_doubles(p);
    const int diffuse = p->cp > 0.0 && p->thermal_conductivity / (p->rho_phys * p->cp) > 0.0;
    for (int32_t k = 0; k < nsteps; ++k) {
        const double t = t0 + (double)k * dt;
        double pr[3];
        for (int d = 0; d < 3; ++d) pr[d] = p->tool_p0[d] + p->tool_v[d] * t;
        memset(grid, 0, sizeof(double) * (size_t)ng);
        ws_p2g(p, s, grid);
        ws_grid(p, w, grid, dt, tool, pr, contact_force);
        if (diffuse) ws_diffuse(p, grid, dt);
        ws_g2p(p, w, s, grid, dt, diffuse);
        if (((step0 + k) % 2) == 0) ws_chip(p, s, pr[2] + p->tool_tip_dz);
    }
}

/* ---------------------------------------------------------------- metrics */

/* Reference-compatible stats: computeParticleStatsKernel (:729-788) over
 * ACTIVE and CHIP, initial values 0 (syncMetrics :1242-1246).  Conservation
 * metrics (this build) over every particle that is not INACTIVE. */
void orc_metrics_compute(const orc_params *p, const orc_state *s, orc_metrics *o) {
    memset(o, 0, sizeof(*o));
    const double mu = p->E / (2.0 * (1.0 + p->nu));
    const double K = p->E / (3.0 * (1.0 - 2.0 * p->nu));
    for (int d = 0; d < 3; ++d) { o->bmin[d] = INFINITY; o->bmax[d] = -INFINITY; }
    for (int i = 0; i < s->n; ++i) {
        int st = s->status[i];
        if (st == ORC_INACTIVE) { o->n_inactive++; continue; }
        if (st == ORC_ACTIVE) o->n_active++;
        else if (st == ORC_CHIP) o->n_chip++;
        else if (st == ORC_FIXED) o->n_fixed++;
        const double *sg = s->sig + 6 * (int64_t)i;
        double tr = sg[0] + sg[1] + sg[2];
        double sxx = sg[0] - tr / 3.0, syy = sg[1] - tr / 3.0, szz = sg[2] - tr / 3.0;
        double vm = sqrt(1.5 * (sxx * sxx + syy * syy + szz * szz + 2.0 * (sg[3] * sg[3] + sg[4] * sg[4] + sg[5] * sg[5])));
        double m = s->mass[i];
        double v2 = s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i];
        o->mass += m;
        o->px += m * s->vx[i]; o->py += m * s->vy[i]; o->pz += m * s->vz[i];
        o->kinetic += 0.5 * m * v2;
        double pr = tr / 3.0;
        o->internal_elastic += s->vol[i] * (vm * vm / (6.0 * mu) + pr * pr / (2.0 * K));
        o->thermal += p->rho_phys * s->vol[i] * p->cp * (s->T[i] - p->Tamb);
        if (s->T[i] > o->max_T) o->max_T = s->T[i];
        if (vm > o->max_vm) o->max_vm = vm;
        if (s->eps[i] > o->max_eps) o->max_eps = s->eps[i];
        o->sum_eps += s->eps[i];
        if (st == ORC_ACTIVE || st == ORC_CHIP) {
            if (vm > o->ref_max_stress) o->ref_max_stress = vm;
            if (s->T[i] > o->ref_max_T) o->ref_max_T = s->T[i];
            o->ref_kinetic += 0.5 * m * v2;
            o->ref_internal += (vm * vm * m) / (6.0 * 80e9) + s->vol[i] * s->eps[i] * vm;
            double xyz[3] = {s->x[i], s->y[i], s->z[i]};
            for (int d = 0; d < 3; ++d) {
                if (xyz[d] < o->bmin[d]) o->bmin[d] = xyz[d];
                if (xyz[d] > o->bmax[d]) o->bmax[d] = xyz[d];
            }
        }
    }
}

/* ---------------------------------------------------------------- Philox */

static inline void mulhilo(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void orc_philox_uniform4(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, float out[4]) {
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    uint32_t c[4] = {c0, c1, c2, c3};
    for (int i = 0; i < 4; ++i) out[i] = (float)(c[i] >> 8) * (1.0f / 16777216.0f);
}
