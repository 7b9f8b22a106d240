/*
 * ag_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C, FP64, single-threaded restatement of the AutoGrid 4.2.8
 * per-grid-point loop, main.cpp:2805-3464, evaluated over an ag_problem
 * (include/autogrid_b200.h).  Arithmetic follows the reference expression by
 * expression and in the same order (double precision, no FMA contraction:
 * built with -ffp-contract=off), so on the same inputs it reproduces the
 * reference's double energies; it is pinned against oracle/_ref/autogrid4_fullprec
 * and Tests/py_hsg1_sm.*.map by tests/test_oracle_pinning.py.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library.
 *
 * Extra output for parity accounting: per point, a bit set when some pair's
 * FP64 quantity sits within ~1e-12 relative of a discontinuity (table-bin edge,
 * the 8 A cutoff, the D1/A2 angular branch at cos=0, a closest-H tie).  At such
 * points two correct FP64 evaluations (e.g. glibc vs CUDA hypot) may
 * legitimately disagree.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "autogrid_b200.h"

#pragma STDC FP_CONTRACT OFF

#define O_APPROX_ZERO 1.0E-6          /* autocomm.h:72 */
#define O_SOFTNBC 8.00                /* constants.h:150 */
#define O_PI 3.14159265358979323846   /* constants.h PI */
#define O_EDGE_REL 1e-12

#define EDGE_BIN     1u
#define EDGE_CUTOFF  2u
#define EDGE_ANGLE   4u
#define EDGE_CLOSEH  8u

static inline double dmin(double a, double b) { return (a < b) ? a : b; } /* autogrid.h:87 */
static inline double dmax(double a, double b) { return (a > b) ? a : b; } /* autogrid.h:86 */

static unsigned bin_edge(double x)
{
    /* x is a distance times A_DIV; flag it if it is within O_EDGE_REL of an integer */
    double k = floor(x + 0.5);
    double tol = O_EDGE_REL * (x > 1.0 ? x : 1.0);
    return fabs(x - k) <= tol ? EDGE_BIN : 0u;
}

int32_t ag_oracle_abi_version(void) { return AG_ABI_VERSION; }

/*
 * Evaluate the maps at n_pts grid points.
 *   pt_index: linear point indices (ix + n1x*(iy + n1y*iz)); NULL = all points in order
 *   out:      [n_maps][n_pts]
 *   flags:    [n_pts] or NULL  (EDGE_* bits, see header)
 * Returns 0, AG_ERR_NO_CLOSEST_H (main.cpp:3011-3014) or AG_ERR_INVALID.
 */
/*
 * 'map_receptor_interior off' (the reference's USE_BHTREE build,
 * main.cpp:2893-2927): the BH tree's single-precision close-atom test
 * (bhtree.cpp:338-366) -- float differences of the float grid point and the
 * float atom coordinates, each within the cutoff, and their float squared sum
 * not above the float squared cutoff.  Built with -ffp-contract=off.
 */
static int bh_close(const float x[3], const double *coord, float cut)
{
    const float a0 = (float)coord[0], a1 = (float)coord[1], a2 = (float)coord[2];
    float d0 = x[0] - a0;
    if (d0 > cut || d0 < -cut) return 0;
    float d1 = x[1] - a1;
    if (d1 > cut || d1 < -cut) return 0;
    float d2 = x[2] - a2;
    if (d2 > cut || d2 < -cut) return 0;
    float D = d0 * d0 + d1 * d1 + d2 * d2;
    float C = cut * cut;
    return !(D > C);
}

/* A grid point with an atom within BH_collision_dist = 1.5 A (main.cpp:346). */
static int bh_collision(const ag_problem *p, const double c[3])
{
    const float x[3] = {(float)c[0], (float)c[1], (float)c[2]};  /* fcc, main.cpp:2860 */
    for (int ia = 0; ia < p->n_atoms; ia++)
        if (bh_close(x, p->coord + 3 * ia, 1.5f)) return 1;
    return 0;
}

int32_t ag_oracle_points(const ag_problem *p, int64_t n_pts, const int64_t *pt_index,
                         double *out, uint8_t *flags)
{
    const int nA = p->n_atoms, nM = p->n_maps, nAM = p->n_atom_maps;
    const int64_t n1x = p->n1[0], n1y = p->n1[1], n1z = p->n1[2];
    const int64_t P = n1x * n1y * n1z;
    const double PI_halved = O_PI / 2.;
    const double ln_half = log(0.5);
    if (nM <= 0 || nM > AG_MAX_MAPS || nAM < 0 || nAM > nM || (pt_index == NULL && n_pts != P))
        return AG_ERR_INVALID;

    /* hbond_12: DS/D1 atoms in file order (main.cpp:916-917) */
    int *hb12 = (int *)malloc(sizeof(int) * (nA > 0 ? nA : 1));
    int nhb12 = 0;
    for (int ia = 0; ia < nA; ia++)
        if (p->hbond[ia] == 1 || p->hbond[ia] == 2) hb12[nhb12++] = ia;

    double *E = (double *)malloc(sizeof(double) * nM);
    double *hbmin = (double *)malloc(sizeof(double) * (nAM > 0 ? nAM : 1));
    double *hbmax = (double *)malloc(sizeof(double) * (nAM > 0 ? nAM : 1));
    char *hbflag = (char *)malloc(nAM > 0 ? nAM : 1);
    int32_t rc = 0;

    for (int64_t ip = 0; ip < n_pts; ip++) {
        int64_t lin = pt_index ? pt_index[ip] : ip;
        if (lin < 0 || lin >= P) { rc = AG_ERR_INVALID; break; }
        int ix = (int)(lin % n1x), iy = (int)((lin / n1x) % n1y), iz = (int)(lin / (n1x * n1y));
        unsigned fl = 0;
        double c[3];
        /* main.cpp:2815-2859 */
        c[2] = ((double)(iz - p->ne[2])) * p->spacing;
        c[1] = ((double)(iy - p->ne[1])) * p->spacing;
        c[0] = ((double)(ix - p->ne[0])) * p->spacing;
        for (int m = 0; m < nM; m++) E[m] = 0.0;

        /* covalent maps, main.cpp:2866-2879 */
        for (int j = 0; j < nAM; j++) if (p->map_is_covalent[j]) {
            double d0 = p->cov_pos[0] - c[0], d1 = p->cov_pos[1] - c[1], d2 = p->cov_pos[2] - c[2];
            double rcov = sqrt(d0 * d0 + d1 * d1 + d2 * d2) / p->cov_half_width;
            if (rcov < O_APPROX_ZERO) rcov = O_APPROX_ZERO;
            E[j] = p->cov_barrier * (1. - exp(ln_half * rcov * rcov));
        }
        /* main.cpp:2882-2886 */
        for (int m = 0; m < nAM; m++) { hbmin[m] = 999999.; hbmax[m] = -999999.; hbflag[m] = 0; }

        /* LOOP 1: electrostatics over all atoms, main.cpp:2940-2982; skipped at
         * a collision point with map_receptor_interior off (main.cpp:2907-2926) */
        if (p->elec_map >= 0 && p->report_collisions && bh_collision(p, c)) {
            E[p->elec_map] = 0.0;
        } else if (p->elec_map >= 0) {
            double e = 0;
            for (int ia = 0; ia < nA; ia++) {
                const double *a = p->coord + 3 * ia;
                double r = hypot(a[0] - c[0], hypot(a[1] - c[1], a[2] - c[2]));
                if (r < O_APPROX_ZERO) r = O_APPROX_ZERO;
                double inv_rmax = 1. / dmax(r, 0.5);
                int indx_r = (int)(r * AG_A_DIV);
                if (indx_r > AG_NDIEL - 1) indx_r = AG_NDIEL - 1;
                if (r < 8.5) fl |= bin_edge(r * AG_A_DIV);
                if (p->dddiel) e += p->charge[ia] * inv_rmax * p->r_epsilon_fn[indx_r] * p->coeff_estat;
                else           e += p->charge[ia] * inv_rmax * p->invdielcal * p->coeff_estat;
            }
            E[p->elec_map] = e;
        }

        /* closest DS/D1 hydrogen, main.cpp:2986-3015 */
        double rminH = 999999.;
        int closestH = -1;
        if (nAM > 0) {
            for (int inh = 0; inh < nhb12; inh++) {
                int ia = hb12[inh];
                const double *a = p->coord + 3 * ia;
                double d[3];
                int breakout = 0;
                for (int i = 0; i < 3; i++) {
                    d[i] = a[i] - c[i];
                    if (fabs(d[i]) > rminH) { breakout = 1; break; }
                }
                if (breakout) continue;
                double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                if (r < rminH) { rminH = r; closestH = ia; }
            }
            if (closestH < 0) { rc = AG_ERR_NO_CLOSEST_H; break; }
            /* near-tie accounting: another DS/D1 atom within 1e-12 of the minimum */
            for (int inh = 0; inh < nhb12; inh++) {
                int ia = hb12[inh];
                if (ia == closestH) continue;
                const double *a = p->coord + 3 * ia;
                double d0 = a[0] - c[0], d1 = a[1] - c[1], d2 = a[2] - c[2];
                double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                if (fabs(r - rminH) <= O_EDGE_REL * dmax(rminH, 1.0)) fl |= EDGE_CLOSEH;
            }
        }

        /* LOOP 2: short-range terms, main.cpp:3017-3410 */
        if (nAM > 0 || p->dsolv_map >= 0) {
            for (int ia = 0; ia < nA; ia++) {
                const double *a = p->coord + 3 * ia;
                const double *rv = p->rvector + 3 * ia;
                const double *rv2 = p->rvector2 + 3 * ia;
                double d[3], dnorm[3];
                for (int i = 0; i < 3; i++) d[i] = a[i] - c[i];
                double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                if (fabs(r - O_SOFTNBC) <= O_EDGE_REL * O_SOFTNBC) fl |= EDGE_CUTOFF;
                if (r > O_SOFTNBC) continue;
                if (p->disorder_h && p->disorder[ia] && p->rec_type[ia] == p->hydrogen_type) continue;
                if (r < O_APPROX_ZERO) r = O_APPROX_ZERO;
                double inv_r = 1. / r;
                for (int i = 0; i < 3; i++) dnorm[i] = d[i] * inv_r;
                int lk = (int)(r * AG_A_DIV);
                int indx_r = lk > AG_NDIEL - 1 ? AG_NDIEL - 1 : lk;
                int indx_n = lk > AG_NEINT - 1 ? AG_NEINT - 1 : lk;
                fl |= bin_edge(r * AG_A_DIV);

                double racc = 1., rdon = 1., Hramp = 1.;
                const int hb = p->hbond[ia];
                /* a zero bond vector gives cos_theta == 0 exactly: not an ambiguous branch */
                const int rv_zero = (rv[0] == 0.0 && rv[1] == 0.0 && rv[2] == 0.0);
                if (hb == 2) { /* D1, main.cpp:3075-3132 */
                    double cos_theta = 0.;
                    for (int i = 0; i < 3; i++) cos_theta -= dnorm[i] * rv[i];
                    if (fabs(cos_theta) <= O_EDGE_REL && !rv_zero) fl |= EDGE_ANGLE;
                    if (cos_theta <= 0.) {
                        racc = 0.;
                    } else {
                        switch (p->rexp[ia]) {
                            case 2: racc = cos_theta * cos_theta; break;
                            case 4: { double tmp = cos_theta * cos_theta; racc = tmp * tmp; } break;
                            case 1: default: racc = cos_theta; break;
                        }
                        if (ia == closestH) {
                            Hramp = 1.;
                        } else {
                            const double *rvh = p->rvector + 3 * closestH;
                            double ct = 0.;
                            for (int i = 0; i < 3; i++) ct += rvh[i] * rv[i];
                            ct = dmin(ct, 1.0);
                            ct = dmax(ct, -1.0);
                            double theta = acos(ct);
                            Hramp = 0.5 - 0.5 * cos(theta * 120. / 90.);
                        }
                    }
                } else if (hb == 4) { /* A1, main.cpp:3133-3162 */
                    double cos_theta = 0.;
                    for (int i = 0; i < 3; i++) cos_theta -= dnorm[i] * rv[i];
                    rdon = (cos_theta <= 0.) ? 0. : cos_theta * cos_theta;
                } else if (hb == 5 && !p->disorder[ia]) { /* A2 ordered, main.cpp:3163-3246 */
                    double cos_theta = 0.;
                    for (int i = 0; i < 3; i++) cos_theta -= dnorm[i] * rv[i];
                    if (fabs(cos_theta) <= O_EDGE_REL && !rv_zero) fl |= EDGE_ANGLE;
                    double t0 = 0.;
                    for (int i = 0; i < 3; i++) t0 += dnorm[i] * rv2[i];
                    if (t0 > 1.) t0 = 1.; else if (t0 < -1.) t0 = -1.;
                    t0 = PI_halved - acos(t0);
                    double cr[3];
                    cr[0] = dnorm[1] * rv2[2] - dnorm[2] * rv2[1];
                    cr[1] = dnorm[2] * rv2[0] - dnorm[0] * rv2[2];
                    cr[2] = dnorm[0] * rv2[1] - dnorm[1] * rv2[0];
                    double rd2 = cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2];
                    if (rd2 < O_APPROX_ZERO) rd2 = O_APPROX_ZERO;
                    double inv_rd = 1. / sqrt(rd2);
                    double ti = 0.;
                    for (int i = 0; i < 3; i++) ti += cr[i] * inv_rd * rv[i];
                    rdon = 0.;
                    if (cos_theta >= 0.) {
                        if (ti > 1.) ti = 1.; else if (ti < -1.) ti = -1.;
                        ti = acos(ti) - PI_halved;
                        if (ti < 0.) ti = -ti;
                        rdon = (0.9 + 0.1 * sin(ti + ti)) * cos(t0);
                    } else if (cos_theta >= -0.34202) {
                        rdon = 562.25 * pow(0.116978 - cos_theta * cos_theta, 3.) * cos(t0);
                    }
                } else if (p->disorder[ia] && hb == 5) { /* A2 disordered, main.cpp:3247-3272 */
                    double cos_theta = 0.;
                    for (int i = 0; i < 3; i++) cos_theta -= dnorm[i] * rv[i];
                    if (cos_theta > 1.) cos_theta = 1.; else if (cos_theta < -1.) cos_theta = -1.;
                    double theta = acos(cos_theta);
                    racc = 0.; rdon = 0.;
                    if (theta <= 1.24791 + PI_halved) {
                        rdon = pow(cos(theta - 1.24791), 4.);
                        racc = rdon;
                    }
                }

                /* per-map terms, main.cpp:3286-3390 */
                const int ta = p->rec_type[ia];
                for (int m = 0; m < nAM; m++) {
                    if (p->map_is_covalent[m]) continue;
                    double T = (double)p->e_vdw_hb[((size_t)ta * nAM + m) * AG_NEINT + indx_n];
                    if (p->map_is_hbonder[m]) {
                        double rsph = T / 100.;
                        rsph = dmax(rsph, 0.);
                        rsph = dmin(rsph, 1.);
                        const int mh = p->map_hbond[m];
                        if ((mh == 3 || mh == 5 || mh == 6) && (hb == 1 || hb == 2 || hb == 6)) {
                            if (!p->disorder[ia]) {
                                E[m] += T * Hramp * (racc + (1. - racc) * rsph);
                            } else {
                                double xh = (r - 1.10) * AG_A_DIV;
                                int ih = (int)xh; if (ih < 0) ih = 0; if (ih > AG_NEINT - 1) ih = AG_NEINT - 1;
                                fl |= bin_edge(xh);
                                double TH = (double)p->e_vdw_hb[((size_t)p->hydrogen_type * nAM + m) * AG_NEINT + ih];
                                E[m] += TH * Hramp * (racc + (1. - racc) * rsph);
                            }
                        } else if ((mh == 4 || mh == 6) && (hb == 1 || hb == 2 || hb == 6)) {
                            double v = T * (racc + (1. - racc) * rsph);
                            hbmin[m] = dmin(hbmin[m], v);
                            hbmax[m] = dmax(hbmax[m], v);
                            hbflag[m] = 1;
                        } else if ((mh == 1 || mh == 2 || mh == 6) && (hb > 2 || hb == 6)) {
                            if (p->disorder[ia]) {
                                double xh = (r - 1.10) * AG_A_DIV;
                                int ih = (int)xh; if (ih < 0) ih = 0; if (ih > AG_NEINT - 1) ih = AG_NEINT - 1;
                                fl |= bin_edge(xh);
                                double TH = (double)p->e_vdw_hb[((size_t)p->hydrogen_type * nAM + m) * AG_NEINT + ih];
                                E[m] += TH * Hramp * (rdon + (1. - rdon) * rsph);
                            } else {
                                double v = T * (rdon + (1. - rdon) * rsph);
                                hbmin[m] = dmin(hbmin[m], v);
                                hbmax[m] = dmax(hbmax[m], v);
                                hbflag[m] = 1;
                            }
                        } else {
                            E[m] += T;
                        }
                    } else {
                        E[m] += T;
                    }
                    /* desolvation, main.cpp:3381-3389 */
                    if (p->separate_desolvation_maps) m++;
                    E[m] += p->map_solpar_probe[m] * p->vol[ia] * p->sol_fn[indx_r] +
                            (p->solpar[ia] + p->solpar_q * fabs(p->charge[ia])) * p->map_vol_probe[m] * p->sol_fn[indx_r];
                }
                /* d map, main.cpp:3393-3404 */
                if (p->dsolv_map >= 0)
                    E[p->dsolv_map] += p->solpar_q * p->vol[ia] * p->sol_fn[indx_r];
            }
            /* H-bond finaliser, main.cpp:3420-3431 */
            for (int m = 0; m < nAM; m++)
                if (hbflag[m]) E[m] += (hbmin[m] + dmax(hbmax[m], 0));
        }
        for (int m = 0; m < nM; m++) out[(size_t)m * n_pts + ip] = E[m];
        if (flags) flags[ip] = (uint8_t)fl;
    }
    free(hb12); free(E); free(hbmin); free(hbmax); free(hbflag);
    return rc;
}

/*
 * Differentiable (linear-table) mode, FP64: the same loop with every table
 * read by linear interpolation, T(x) = T[b] + (x - b)(T[b+1] - T[b]),
 * b = floor(x), constant past the last bin; LOOP 2 terms multiplied by
 * w = min(1, NEINT - A_DIV r); Hramp evaluated for every D1 pair; the A2
 * cos_theta < 0 branch scaled by (1 + sin(2 ti)/9).  closest_h: [n_pts]
 * frozen closest DS/D1 atom per point, or NULL to search it as main.cpp:2986
 * does.  This restates the mode from the reference loop (not from the GPU
 * code), for the GPU parity tests of ag_diff_forward.
 */
static double lin_tab_f(const float *t, int n, double x)
{
    if (x <= 0) return t[0];
    int b = (int)x;
    if (b >= n - 1) return t[n - 1];
    return (double)t[b] + (x - b) * ((double)t[b + 1] - (double)t[b]);
}
static double lin_tab_d(const double *t, int n, double x)
{
    if (x <= 0) return t[0];
    int b = (int)x;
    if (b >= n - 1) return t[n - 1];
    return t[b] + (x - b) * (t[b + 1] - t[b]);
}

int32_t ag_oracle_points_lin(const ag_problem *p, int64_t n_pts, const int64_t *pt_index,
                             const int32_t *closest_h, double *out)
{
    const int nA = p->n_atoms, nM = p->n_maps, nAM = p->n_atom_maps;
    const int64_t n1x = p->n1[0], n1y = p->n1[1], n1z = p->n1[2];
    const int64_t P = n1x * n1y * n1z;
    const double ln_half = log(0.5);
    if (nM <= 0 || nM > AG_MAX_MAPS || nAM < 0 || nAM > nM || (pt_index == NULL && n_pts != P))
        return AG_ERR_INVALID;
    int *hb12 = (int *)malloc(sizeof(int) * (nA > 0 ? nA : 1));
    int nhb12 = 0;
    for (int ia = 0; ia < nA; ia++)
        if (p->hbond[ia] == 1 || p->hbond[ia] == 2) hb12[nhb12++] = ia;
    double *E = (double *)malloc(sizeof(double) * nM);
    double *hbmin = (double *)malloc(sizeof(double) * (nAM > 0 ? nAM : 1));
    double *hbmax = (double *)malloc(sizeof(double) * (nAM > 0 ? nAM : 1));
    char *hbflag = (char *)malloc(nAM > 0 ? nAM : 1);
    double *sol_ext = (double *)malloc(sizeof(double) * (AG_NEINT + 1));
    for (int b = 0; b <= AG_NEINT; b++) sol_ext[b] = p->sol_fn[b];
    int32_t rc = 0;
    for (int64_t ip = 0; ip < n_pts; ip++) {
        int64_t lin = pt_index ? pt_index[ip] : ip;
        if (lin < 0 || lin >= P) { rc = AG_ERR_INVALID; break; }
        int ix = (int)(lin % n1x), iy = (int)((lin / n1x) % n1y), iz = (int)(lin / (n1x * n1y));
        double c[3];
        c[2] = ((double)(iz - p->ne[2])) * p->spacing;
        c[1] = ((double)(iy - p->ne[1])) * p->spacing;
        c[0] = ((double)(ix - p->ne[0])) * p->spacing;
        for (int m = 0; m < nM; m++) E[m] = 0.0;
        for (int j = 0; j < nAM; j++) if (p->map_is_covalent[j]) {
            double d0 = p->cov_pos[0] - c[0], d1 = p->cov_pos[1] - c[1], d2 = p->cov_pos[2] - c[2];
            double rcov = sqrt(d0 * d0 + d1 * d1 + d2 * d2) / p->cov_half_width;
            if (rcov < O_APPROX_ZERO) rcov = O_APPROX_ZERO;
            E[j] = p->cov_barrier * (1. - exp(ln_half * rcov * rcov));
        }
        for (int m = 0; m < nAM; m++) { hbmin[m] = 999999.; hbmax[m] = -999999.; hbflag[m] = 0; }
        if (p->elec_map >= 0) {
            double e = 0;
            for (int ia = 0; ia < nA; ia++) {
                const double *a = p->coord + 3 * ia;
                double d0 = a[0] - c[0], d1 = a[1] - c[1], d2 = a[2] - c[2];
                double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                if (r < O_APPROX_ZERO) r = O_APPROX_ZERO;
                double T = p->dddiel ? lin_tab_d(p->r_epsilon_fn, AG_NDIEL, r * AG_A_DIV) : p->invdielcal;
                e += p->charge[ia] * T * p->coeff_estat / dmax(r, 0.5);
            }
            E[p->elec_map] = e;
        }
        int closestH = -1;
        if (nAM > 0) {
            if (closest_h) {
                closestH = closest_h[ip];  /* -1: frozen "none", Hramp stays 1 */
            } else {
                double rminH = 999999.;
                for (int inh = 0; inh < nhb12; inh++) {
                    const double *a = p->coord + 3 * hb12[inh];
                    double d0 = a[0] - c[0], d1 = a[1] - c[1], d2 = a[2] - c[2];
                    double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                    if (r < rminH) { rminH = r; closestH = hb12[inh]; }
                }
            }
            if (closestH < 0 && !closest_h) { rc = AG_ERR_NO_CLOSEST_H; break; }
        }
        if (nAM > 0 || p->dsolv_map >= 0) {
            for (int ia = 0; ia < nA; ia++) {
                const double *a = p->coord + 3 * ia;
                const double *rv = p->rvector + 3 * ia;
                const double *rv2 = p->rvector2 + 3 * ia;
                double d[3], dnorm[3];
                for (int i = 0; i < 3; i++) d[i] = a[i] - c[i];
                double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                if (r > O_SOFTNBC) continue;
                if (p->disorder_h && p->disorder[ia] && p->rec_type[ia] == p->hydrogen_type) continue;
                if (r < O_APPROX_ZERO) r = O_APPROX_ZERO;
                for (int i = 0; i < 3; i++) dnorm[i] = d[i] / r;
                const double x = r * AG_A_DIV;
                const double w = dmin(1.0, AG_NEINT - x);
                const double sol = lin_tab_d(sol_ext, AG_NEINT + 1, x);
                double racc = 1., rdon = 1., Hramp = 1.;
                const int hb = p->hbond[ia];
                double cos_theta = 0.;
                for (int i = 0; i < 3; i++) cos_theta -= dnorm[i] * rv[i];
                if (hb == 2) {
                    if (cos_theta <= 0.) racc = 0.;
                    else if (p->rexp[ia] == 2) racc = cos_theta * cos_theta;
                    else if (p->rexp[ia] == 4) racc = pow(cos_theta, 4.);
                    else racc = cos_theta;
                    if (closestH >= 0 && ia != closestH) {
                        const double *rvh = p->rvector + 3 * closestH;
                        double ct = rvh[0] * rv[0] + rvh[1] * rv[1] + rvh[2] * rv[2];
                        ct = dmax(dmin(ct, 1.0), -1.0);
                        Hramp = 0.5 - 0.5 * cos(acos(ct) * 120. / 90.);
                    }
                } else if (hb == 4) {
                    rdon = (cos_theta <= 0.) ? 0. : cos_theta * cos_theta;
                } else if (hb == 5 && !p->disorder[ia]) {
                    double t0 = 0.;
                    for (int i = 0; i < 3; i++) t0 += dnorm[i] * rv2[i];
                    t0 = dmax(dmin(t0, 1.), -1.);
                    t0 = O_PI / 2. - acos(t0);
                    double cr[3];
                    cr[0] = dnorm[1] * rv2[2] - dnorm[2] * rv2[1];
                    cr[1] = dnorm[2] * rv2[0] - dnorm[0] * rv2[2];
                    cr[2] = dnorm[0] * rv2[1] - dnorm[1] * rv2[0];
                    double rd2 = dmax(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2], O_APPROX_ZERO);
                    double ti = 0.;
                    for (int i = 0; i < 3; i++) ti += cr[i] / sqrt(rd2) * rv[i];
                    ti = dmax(dmin(ti, 1.), -1.);
                    ti = fabs(acos(ti) - O_PI / 2.);
                    if (cos_theta >= 0.) rdon = (0.9 + 0.1 * sin(ti + ti)) * cos(t0);
                    else if (cos_theta >= -0.34202)
                        rdon = 562.25 * pow(0.116978 - cos_theta * cos_theta, 3.) * cos(t0) * (1. + sin(ti + ti) / 9.);
                    else rdon = 0.;
                } else if (hb == 5) {
                    double ct = dmax(dmin(cos_theta, 1.), -1.);
                    double theta = acos(ct);
                    racc = rdon = (theta <= 1.24791 + O_PI / 2.) ? pow(cos(theta - 1.24791), 4.) : 0.;
                }
                const int ta = p->rec_type[ia];
                for (int m = 0; m < nAM; m++) {
                    if (p->map_is_covalent[m]) continue;
                    const float *row = p->e_vdw_hb + ((size_t)ta * nAM + m) * AG_NEINT;
                    double T = lin_tab_f(row, AG_NEINT, x);
                    double rsph = dmin(dmax(T / 100., 0.), 1.);
                    const float *hrow = p->hydrogen_type >= 0
                        ? p->e_vdw_hb + ((size_t)p->hydrogen_type * nAM + m) * AG_NEINT : NULL;
                    double TH = hrow ? lin_tab_f(hrow, AG_NEINT, (r - 1.10) * AG_A_DIV) : 0.;
                    if (p->map_is_hbonder[m]) {
                        const int mh = p->map_hbond[m];
                        if ((mh == 3 || mh == 5 || mh == 6) && (hb == 1 || hb == 2 || hb == 6)) {
                            E[m] += w * (p->disorder[ia] ? TH : T) * Hramp * (racc + (1. - racc) * rsph);
                        } else if ((mh == 4 || mh == 6) && (hb == 1 || hb == 2 || hb == 6)) {
                            double v = w * T * (racc + (1. - racc) * rsph);
                            hbmin[m] = dmin(hbmin[m], v);
                            hbmax[m] = dmax(hbmax[m], v);
                            hbflag[m] = 1;
                        } else if ((mh == 1 || mh == 2 || mh == 6) && (hb > 2 || hb == 6)) {
                            if (p->disorder[ia]) {
                                E[m] += w * TH * Hramp * (rdon + (1. - rdon) * rsph);
                            } else {
                                double v = w * T * (rdon + (1. - rdon) * rsph);
                                hbmin[m] = dmin(hbmin[m], v);
                                hbmax[m] = dmax(hbmax[m], v);
                                hbflag[m] = 1;
                            }
                        } else {
                            E[m] += w * T;
                        }
                    } else {
                        E[m] += w * T;
                    }
                    if (p->separate_desolvation_maps) m++;
                    E[m] += w * sol * (p->map_solpar_probe[m] * p->vol[ia] +
                                       (p->solpar[ia] + p->solpar_q * fabs(p->charge[ia])) * p->map_vol_probe[m]);
                }
                if (p->dsolv_map >= 0) E[p->dsolv_map] += w * p->solpar_q * p->vol[ia] * sol;
            }
            for (int m = 0; m < nAM; m++)
                if (hbflag[m]) E[m] += (hbmin[m] + dmax(hbmax[m], 0));
        }
        for (int m = 0; m < nM; m++) out[(size_t)m * n_pts + ip] = E[m];
    }
    free(hb12); free(E); free(hbmin); free(hbmax); free(hbflag); free(sol_ext);
    return rc;
}

/*
 * Distance maps of LOOP 1, main.cpp:2947-2966: out[0][ip] the floating grid
 * (min over atoms of the hypot distance clamped at APPROX_ZERO, BIG = 1e12
 * without atoms, autocomm.h:73), then the constriction count (atoms with that
 * distance <= constriction_cutoff), for whichever the problem requests.
 */
int32_t ag_oracle_distance_maps(const ag_problem *p, int64_t n_pts, const int64_t *pt_index, double *out)
{
    const int64_t n1x = p->n1[0], n1y = p->n1[1], n1z = p->n1[2];
    const int64_t P = n1x * n1y * n1z;
    if (pt_index == NULL && n_pts != P) return AG_ERR_INVALID;
    for (int64_t ip = 0; ip < n_pts; ip++) {
        int64_t lin = pt_index ? pt_index[ip] : ip;
        if (lin < 0 || lin >= P) return AG_ERR_INVALID;
        int ix = (int)(lin % n1x), iy = (int)((lin / n1x) % n1y), iz = (int)(lin / (n1x * n1y));
        double c[3];
        c[2] = ((double)(iz - p->ne[2])) * p->spacing;
        c[1] = ((double)(iy - p->ne[1])) * p->spacing;
        c[0] = ((double)(ix - p->ne[0])) * p->spacing;
        double r_min = 1.0E12;
        int count = 0;
        for (int ia = 0; ia < p->n_atoms; ia++) {
            const double *a = p->coord + 3 * ia;
            double r = hypot(a[0] - c[0], hypot(a[1] - c[1], a[2] - c[2]));
            if (r < O_APPROX_ZERO) r = O_APPROX_ZERO;
            r_min = dmin(r, r_min);
            if (r <= p->constriction_cutoff) count++;
        }
        if (p->report_collisions) {
            /* the USE_BHTREE build: the BH tree's count (main.cpp:2894-2899) and,
             * at a collision point, r_min = BH_collision_dist (main.cpp:2925) */
            const float x[3] = {(float)c[0], (float)c[1], (float)c[2]};
            count = 0;
            for (int ia = 0; ia < p->n_atoms; ia++)
                if (bh_close(x, p->coord + 3 * ia, (float)p->constriction_cutoff)) count++;
            if (bh_collision(p, c)) r_min = 1.5;
        }
        int k = 0;
        if (p->floating_grid) out[(size_t)(k++) * n_pts + ip] = r_min;
        if (p->constriction_grid) out[(size_t)k * n_pts + ip] = (double)count;
    }
    return 0;
}
