/*
 * CPU ORACLE -- test infrastructure only.
 *
 * A plain-C restatement of MDP's SNAP force path, used by the tests, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * Nothing in the product (mdp_b200/) links, loads or calls this file.
 *
 * Parity is pinned: tests/test_oracle.py checks this restatement against the
 * reference's own CPU code (src/C++/Core/cpuSnap4.cpp, cpuNeighborList3D.cpp,
 * built from the reference sources into oracle/_ref/) and against the golden
 * fixtures in tests/golden/ that were generated from that build.
 *
 * Followed reference code, function by function:
 *   tables             src/C++/Core/cpuSnap.cpp:14-193 (cpuBuildIndexList,
 *                      cpuInitRootpqArray, cpuDeltacg, cpuInitClebschGordan)
 *   box set-up         src/C++/Core/cpuArrayPermute.cpp:186-217 (inverse),
 *                      src/C++/Core/cpuNeighborList3D.cpp:11-229
 *   ghosts             src/C++/Core/cpuNeighborList3D.cpp:282-330
 *   neighbour list     src/C++/Core/cpuNeighborList3D.cpp:417-441 (O(N^2) form;
 *                      identical sets to the cell form when nothing truncates)
 *   pair list / pairs  src/C++/Core/cpuSnap.cpp:1883-1933
 *   U, wself, mirror   src/C++/Core/cpuSnap4.cpp:11-244
 *   energy (Ei)        src/C++/Core/cpuSnap4.cpp:250-421
 *   Y                  src/C++/Core/cpuSnap4.cpp:697-792
 *   dE/dr, force,      src/C++/Core/cpuSnap4.cpp:798-1211
 *   virial
 *   NVE                src/C++/Core/cpuVelocityIntegration.cpp:307-339
 *
 * Layout here is per atom (U[atom][idxu]) rather than the reference's
 * atom-fastest SoA; the arithmetic per element is the same.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define JMAXO 12

typedef struct {
    int twojmax, jdim;
    int idxu_max, idxz_max, idxb_max, idxcg_max;
    int idxu_block[JMAXO + 1];
    int idxcg_block[JMAXO + 1][JMAXO + 1][JMAXO + 1];
    int idxb_block[JMAXO + 1][JMAXO + 1][JMAXO + 1];
    int *idxz;      /* 10 ints per entry */
    int *idxb;      /* 3 ints per entry */
    double *cg;
    double rootpq[(JMAXO + 2) * (JMAXO + 2)];
} orc_tables;

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* cpuSnap.cpp:14-115 */
static void build_tables(orc_tables *t, int twojmax)
{
    int J = twojmax, jd = J + 1;
    t->twojmax = J; t->jdim = jd;
    int ncg = 0, nb = 0, nz = 0, nu = 0;
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= imin(J, j1 + j2); j += 2) {
                t->idxcg_block[j1][j2][j] = ncg;
                ncg += (j1 + 1) * (j2 + 1);
                if (j >= j1) { t->idxb_block[j1][j2][j] = nb; nb++; }
                for (int mb = 0; 2 * mb <= j; mb++) nz += j + 1;
            }
    for (int j = 0; j <= J; j++) { t->idxu_block[j] = nu; nu += (j + 1) * (j + 1); }
    t->idxcg_max = ncg; t->idxb_max = nb; t->idxz_max = nz; t->idxu_max = nu;
    t->idxb = (int *)malloc(sizeof(int) * 3 * nb);
    t->idxz = (int *)malloc(sizeof(int) * 10 * nz);
    t->cg = (double *)malloc(sizeof(double) * ncg);
    int ib = 0, iz = 0;
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= imin(J, j1 + j2); j += 2) {
                if (j >= j1) { t->idxb[3 * ib] = j1; t->idxb[3 * ib + 1] = j2; t->idxb[3 * ib + 2] = j; ib++; }
                for (int mb = 0; 2 * mb <= j; mb++)
                    for (int ma = 0; ma <= j; ma++) {
                        int *z = t->idxz + 10 * iz;
                        z[0] = j1; z[1] = j2; z[2] = j;
                        z[3] = imax(0, (2 * ma - j - j2 + j1) / 2);
                        z[4] = (2 * ma - j - (2 * z[3] - j1) + j2) / 2;
                        z[5] = imin(j1, (2 * ma - j + j2 + j1) / 2) - z[3] + 1;
                        z[6] = imax(0, (2 * mb - j - j2 + j1) / 2);
                        z[7] = (2 * mb - j - (2 * z[6] - j1) + j2) / 2;
                        z[8] = imin(j1, (2 * mb - j + j2 + j1) / 2) - z[6] + 1;
                        z[9] = t->idxu_block[j] + (j + 1) * mb + ma;
                        iz++;
                    }
            }
    /* rootpq[p*jdim + q] = sqrt(p/q), cpuSnap.cpp:117-123 */
    for (int p = 1; p <= J; p++)
        for (int q = 1; q <= J; q++)
            t->rootpq[p * jd + q] = sqrt((double)p / q);
    /* Clebsch-Gordan, cpuSnap.cpp:125-193 (Racah formula) */
    double fac[64];
    fac[0] = 1.0;
    for (int i = 1; i < 64; i++) fac[i] = fac[i - 1] * i;
    int icg = 0;
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= imin(J, j1 + j2); j += 2)
                for (int m1 = 0; m1 <= j1; m1++) {
                    int aa2 = 2 * m1 - j1;
                    for (int m2 = 0; m2 <= j2; m2++, icg++) {
                        int bb2 = 2 * m2 - j2;
                        int m = (aa2 + bb2 + j) / 2;
                        if (m < 0 || m > j) { t->cg[icg] = 0.0; continue; }
                        double sum = 0.0;
                        int zlo = imax(0, imax(-(j - j2 + aa2) / 2, -(j - j1 - bb2) / 2));
                        int zhi = imin((j1 + j2 - j) / 2, imin((j1 - aa2) / 2, (j2 + bb2) / 2));
                        for (int z = zlo; z <= zhi; z++) {
                            double s = (z % 2) ? -1.0 : 1.0;
                            sum += s / (fac[z] * fac[(j1 + j2 - j) / 2 - z] * fac[(j1 - aa2) / 2 - z] *
                                        fac[(j2 + bb2) / 2 - z] * fac[(j - j2 + aa2) / 2 + z] *
                                        fac[(j - j1 - bb2) / 2 + z]);
                        }
                        int cc2 = 2 * m - j;
                        double dcg = sqrt(fac[(j1 + j2 - j) / 2] * fac[(j1 - j2 + j) / 2] *
                                          fac[(-j1 + j2 + j) / 2] / fac[(j1 + j2 + j) / 2 + 1]);
                        double sfaccg = sqrt(fac[(j1 + aa2) / 2] * fac[(j1 - aa2) / 2] *
                                             fac[(j2 + bb2) / 2] * fac[(j2 - bb2) / 2] *
                                             fac[(j + cc2) / 2] * fac[(j - cc2) / 2] * (j + 1));
                        t->cg[icg] = sum * dcg * sfaccg;
                    }
                }
}

static void free_tables(orc_tables *t) { free(t->idxb); free(t->idxz); free(t->cg); }

/* exported: table sizes (idxcg, idxu, idxb, idxz) and copies for tests */
void orc_table_sizes(int twojmax, int *out4)
{
    orc_tables t; build_tables(&t, twojmax);
    out4[0] = t.idxcg_max; out4[1] = t.idxu_max; out4[2] = t.idxb_max; out4[3] = t.idxz_max;
    free_tables(&t);
}

void orc_tables_copy(int twojmax, double *cg, double *rootpq, int *idxz, int *idxb, int *idxu_block)
{
    orc_tables t; build_tables(&t, twojmax);
    memcpy(cg, t.cg, sizeof(double) * t.idxcg_max);
    memcpy(rootpq, t.rootpq, sizeof(double) * (t.jdim + 1) * (t.jdim + 1));
    memcpy(idxz, t.idxz, sizeof(int) * 10 * t.idxz_max);
    memcpy(idxb, t.idxb, sizeof(int) * 3 * t.idxb_max);
    memcpy(idxu_block, t.idxu_block, sizeof(int) * (twojmax + 1));
    free_tables(&t);
}

/* ------------------------------------------------------------------------ */
/* Box set-up, ghost atoms and neighbour list                               */
/* ------------------------------------------------------------------------ */

/* cpuArrayPermute.cpp:186-217 (3x3, column-major) */
static void inv3(double *iA, const double *A)
{
    double a11 = A[0], a21 = A[1], a31 = A[2], a12 = A[3], a22 = A[4], a32 = A[5], a13 = A[6], a23 = A[7], a33 = A[8];
    double d = (a11 * a22 * a33 - a11 * a23 * a32 - a12 * a21 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31);
    iA[0] = (a22 * a33 - a23 * a32) / d; iA[1] = (a23 * a31 - a21 * a33) / d; iA[2] = (a21 * a32 - a22 * a31) / d;
    iA[3] = (a13 * a32 - a12 * a33) / d; iA[4] = (a11 * a33 - a13 * a31) / d; iA[5] = (a12 * a31 - a11 * a32) / d;
    iA[6] = (a12 * a23 - a13 * a22) / d; iA[7] = (a13 * a21 - a11 * a23) / d; iA[8] = (a11 * a22 - a12 * a21) / d;
}

static double norm3(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

/* Bounding box of the box enlarged by r on each periodic side, returned in
 * unit-cube coordinates: rbv[0..2] = lower corner, rbv[18..20] = upper corner
 * (cpuNeighborList3D.cpp:11-132). */
static void bounding_box(double *rbv, const double *a, const double *b, const double *c,
                         const double *r, const int *pbc)
{
    double p1[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    double p2[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    double p3[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
    double d1 = -r[2] * norm3(p1), d2 = -r[0] * norm3(p2), d3 = -r[1] * norm3(p3);
    double A[9] = {p1[0], p2[0], p3[0], p1[1], p2[1], p3[1], p1[2], p2[2], p3[2]}, iA[9];
    inv3(iA, A);
    double w[24];
    w[0] = iA[0] * d1 + iA[3] * d2 + iA[6] * d3;
    w[1] = iA[1] * d1 + iA[4] * d2 + iA[7] * d3;
    w[2] = iA[2] * d1 + iA[5] * d2 + iA[8] * d3;
    double M[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
    inv3(iA, M);
    double e1 = iA[0] * w[0] + iA[3] * w[1] + iA[6] * w[2];
    double e2 = iA[1] * w[0] + iA[4] * w[1] + iA[7] * w[2];
    double e3 = iA[2] * w[0] + iA[5] * w[1] + iA[8] * w[2];
    double sa[3], sb[3], sc[3];
    for (int k = 0; k < 3; k++) {
        sa[k] = w[k] - e2 * b[k] - e3 * c[k];
        sb[k] = w[k] - e1 * a[k] - e3 * c[k];
        sc[k] = w[k] - e1 * a[k] - e2 * b[k];
    }
    double na = norm3(a), nb = norm3(b), nc = norm3(c);
    double la = na + (2.0 * pbc[0]) * norm3(sa);
    double lb = nb + (2.0 * pbc[1]) * norm3(sb);
    double lc = nc + (2.0 * pbc[2]) * norm3(sc);
    for (int k = 0; k < 3; k++) w[k] = (pbc[0] * e1) * a[k] + (pbc[1] * e2) * b[k] + (pbc[2] * e3) * c[k];
    for (int k = 0; k < 3; k++) {
        w[3 + k] = w[k] + (la / na) * a[k];
        w[9 + k] = w[k] + (lb / nb) * b[k];
        w[6 + k] = -w[k] + w[3 + k] + w[9 + k];
        w[12 + k] = w[k] + (lc / nc) * c[k];
        w[15 + k] = w[12 + k] + (la / na) * a[k];
        w[21 + k] = w[12 + k] + (lb / nb) * b[k];
        w[18 + k] = -w[12 + k] + w[15 + k] + w[21 + k];
    }
    for (int i = 0; i < 8; i++)
        for (int k = 0; k < 3; k++)
            rbv[3 * i + k] = iA[k] * w[3 * i] + iA[3 + k] * w[3 * i + 1] + iA[6 + k] * w[3 * i + 2];
}

/* Periodic image shifts in the reference's order (cpuNeighborList3D.cpp:136-229),
 * fully periodic case: 27 images, image 0 = no shift. */
static void periodic_images(double *pim, const double *a, const double *b, const double *c)
{
    static const int ca[27] = {0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 1, -1, 0, 0, 1, 1, -1, -1};
    static const int cb[27] = {0, 0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 0, 1, -1, 1, -1, 1, -1};
    static const int cc[27] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    for (int i = 0; i < 27; i++)
        for (int k = 0; k < 3; k++) {
            /* evaluation order of the reference's table entries: c first, then a, then b */
            double s;
            if (cc[i] != 0) {
                s = cc[i] * c[k];
                if (ca[i] != 0) s = s + ca[i] * a[k]; else if (cb[i] == 0) s = s + 0.0;
                if (cb[i] != 0) s = s + cb[i] * b[k];
            } else {
                s = 0.0;
                if (ca[i] != 0) s = ca[i] * a[k];
                if (cb[i] != 0) s = (ca[i] != 0) ? s + cb[i] * b[k] : cb[i] * b[k];
            }
            pim[3 * i + k] = s;
        }
}

/* Build ghosts and the full neighbour list for an orthogonal or general
 * periodic box (box vectors a, b, c; all three directions periodic).
 * x has room for anummax*3; the first inum rows are the local atoms.
 * Returns anum, or -1 if anummax is too small, -2 if any atom has more than
 * neighmax neighbours (list truncated, as the reference does silently). */
long orc_neighbor_list(double *x, int *alist, int *neighlist, int *neighnum,
                       const double *a, const double *b, const double *c,
                       double rcut_skin, int inum, int neighmax, long anummax)
{
    double M[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]}, s2r[9];
    inv3(s2r, M);
    double r[3] = {rcut_skin, rcut_skin, rcut_skin};
    int pbc[3] = {1, 1, 1};
    double rbv[24], pim[81];
    bounding_box(rbv, a, b, c, r, pbc);
    periodic_images(pim, a, b, c);
    long q = inum;
    for (int i = 0; i < inum; i++) alist[i] = i;
    for (int i = 0; i < inum; i++)
        for (int j = 1; j < 27; j++) {
            double xj0 = x[3 * i] + pim[3 * j], xj1 = x[3 * i + 1] + pim[3 * j + 1], xj2 = x[3 * i + 2] + pim[3 * j + 2];
            double xc0 = s2r[0] * xj0 + s2r[3] * xj1 + s2r[6] * xj2;
            double xc1 = s2r[1] * xj0 + s2r[4] * xj1 + s2r[7] * xj2;
            double xc2 = s2r[2] * xj0 + s2r[5] * xj1 + s2r[8] * xj2;
            if (rbv[0] <= xc0 && xc0 <= rbv[18] && rbv[1] <= xc1 && xc1 <= rbv[19] &&
                rbv[2] <= xc2 && xc2 <= rbv[20]) {
                if (q >= anummax) return -1;
                x[3 * q] = xj0; x[3 * q + 1] = xj1; x[3 * q + 2] = xj2;
                alist[q] = i;
                q++;
            }
        }
    long anum = q;
    double rc2 = rcut_skin * rcut_skin;
    int trunc = 0;
#pragma omp parallel for schedule(static) reduction(| : trunc)
    for (int i = 0; i < inum; i++) {
        int inc = 0;
        double xi0 = x[3 * i], xi1 = x[3 * i + 1], xi2 = x[3 * i + 2];
        for (long j = 0; j < anum; j++) {
            if (j == i) continue;
            double d0 = x[3 * j] - xi0, d1 = x[3 * j + 1] - xi1, d2 = x[3 * j + 2] - xi2;
            double rsq = d0 * d0 + d1 * d1 + d2 * d2;
            if (rsq <= rc2) {
                if (inc == neighmax) { trunc = 1; break; }
                neighlist[(long)i * neighmax + inc++] = (int)j;
            }
        }
        neighnum[i] = inc;
    }
    return trunc ? -2 : anum;
}

/* ------------------------------------------------------------------------ */
/* SNAP                                                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    double rcut, rfac0, rmin0, wj;
    int switchflag;
} pairpar;

/* per-pair geometry shared by U and dU (cpuSnap4.cpp:15-53, 803-851) */
typedef struct {
    double x, y, z, r, ux, uy, uz;
    double sfac, dsfac;
    double ar, ai, br, bi;
    double dar[3], dai[3], dbr[3], dbi[3];
} pairgeo;

static void pair_geometry(pairgeo *g, double x, double y, double z, const pairpar *pp, int want_deriv)
{
    double rsq = x * x + y * y + z * z, r = sqrt(rsq);
    double theta_scale = pp->rfac0 * M_PI / (pp->rcut - pp->rmin0);
    double z0 = r / tan((r - pp->rmin0) * theta_scale);
    double sfac = 1.0, dsfac = 0.0;
    if (pp->switchflag == 1 && r > pp->rmin0 && r <= pp->rcut) {
        double rf = M_PI / (pp->rcut - pp->rmin0);
        sfac = 0.5 * (cos((r - pp->rmin0) * rf) + 1.0);
        dsfac = -0.5 * sin((r - pp->rmin0) * rf) * rf;
    }
    g->sfac = sfac * pp->wj;
    g->dsfac = dsfac * pp->wj;
    double r0inv = 1.0 / sqrt(r * r + z0 * z0);
    g->x = x; g->y = y; g->z = z; g->r = r;
    g->ar = r0inv * z0; g->ai = -r0inv * z; g->br = r0inv * y; g->bi = -r0inv * x;
    if (!want_deriv) return;
    double rinv = 1.0 / r;
    g->ux = x * rinv; g->uy = y * rinv; g->uz = z * rinv;
    double dz0dr = z0 / r - (r * theta_scale) * (rsq + z0 * z0) / rsq;
    double dr0inv = -pow(r0inv, 3.0) * (r + z0 * dz0dr);
    double u[3] = {g->ux, g->uy, g->uz};
    for (int k = 0; k < 3; k++) {
        double dr0 = dr0inv * u[k];
        g->dar[k] = dz0dr * u[k] * r0inv + z0 * dr0;
        g->dai[k] = -z * dr0;
        g->dbr[k] = y * dr0;
        g->dbi[k] = -x * dr0;
    }
    g->dai[2] += -r0inv;
    g->dbi[0] += -r0inv;
    g->dbr[1] += r0inv;
}

/* One layer step of the row recursion: new[ma] from old[0..j-1] (old row
 * (j-1, mb)), cpuSnap4.cpp:60-82.  conj(a)*u and conj(b)*u products. */
static void u_layer(double *pr, double *pi, int j, int mb, const orc_tables *t, const pairgeo *g)
{
    int jd = t->jdim;
    double ur = 0.0, ui = 0.0;  /* old[ma-1] */
    for (int ma = 0; ma <= j; ma++) {
        double wr = (ma < j) ? pr[ma] : 0.0, wi = (ma < j) ? pi[ma] : 0.0;
        double nr = 0.0, ni = 0.0;
        if (ma < j) {
            double rp = t->rootpq[(j - ma) * jd + (j - mb)];
            nr = rp * (g->ar * wr + g->ai * wi);
            ni = rp * (g->ar * wi - g->ai * wr);
        }
        if (ma > 0) {
            double rp = t->rootpq[ma * jd + (j - mb)];
            nr -= rp * (g->br * ur + g->bi * ui);
            ni -= rp * (g->br * ui - g->bi * ur);
        }
        pr[ma] = nr; pi[ma] = ni;
        ur = wr; ui = wi;
    }
}

/* Accumulate sfac*U(pair) for all half-plane elements into U (full idxu
 * layout, per atom).  cpuSnap4.cpp:11-187. */
static void add_pair_u(double *Ur, double *Ui, const orc_tables *t, const pairgeo *g)
{
    int J = t->twojmax;
    double pr[JMAXO + 2], pi[JMAXO + 2], qr[JMAXO + 2], qi[JMAXO + 2];
    Ur[0] += g->sfac;
    for (int mb = 0; 2 * mb <= J; mb++) {
        int jstart;
        if (mb == 0) { pr[0] = 1.0; pi[0] = 0.0; jstart = 1; }
        else { for (int ma = 0; ma < 2 * mb; ma++) { pr[ma] = qr[ma]; pi[ma] = qi[ma]; } jstart = 2 * mb; }
        for (int j = jstart; j <= J; j++) {
            u_layer(pr, pi, j, mb, t, g);
            if (mb > 0 && j == 2 * mb) {           /* middle row: left half mirrors to right */
                int h = j / 2;
                for (int ma = 0; ma <= h; ma++) {
                    double s = (ma % 2) ? -1.0 : 1.0;
                    pr[h + ma] = s * pr[h - ma];
                    pi[h + ma] = -s * pi[h - ma];
                }
            }
            if (j == 2 * mb + 1) {                 /* row mb+1 of layer j by inversion */
                for (int ma = 0; ma <= j; ma++) {
                    double s = ((mb + ma) % 2) ? -1.0 : 1.0;
                    qr[j - ma] = s * pr[ma];
                    qi[j - ma] = -s * pi[ma];
                }
            }
            int k = t->idxu_block[j] + (j + 1) * mb;
            for (int ma = 0; ma <= j; ma++) { Ur[k + ma] += g->sfac * pr[ma]; Ui[k + ma] += g->sfac * pi[ma]; }
        }
    }
}

/* wself on the diagonal and left->right mirror, cpuSnap4.cpp:193-244 */
static void wself_mirror(double *Ur, double *Ui, const orc_tables *t, double wself)
{
    for (int j = 0; j <= t->twojmax; j++) {
        int b0 = t->idxu_block[j];
        for (int m = 0; m <= j; m++) Ur[b0 + (j + 1) * m + m] += wself;
        for (int mb = 0; 2 * mb < j; mb++)
            for (int ma = 0; ma <= j; ma++) {
                int src = b0 + (j + 1) * mb + ma, dst = b0 + (j + 1) * (j - mb) + (j - ma);
                double s = ((mb + ma) % 2) ? -1.0 : 1.0;
                Ur[dst] = s * Ur[src];
                Ui[dst] = -s * Ui[src];
            }
    }
}

/* Z_{j1 j2 j}(ma, mb) for one idxz entry, cpuSnap4.cpp:632-659 */
static void zentry(double *zr, double *zi, const int *z, const orc_tables *t,
                   const double *Ur, const double *Ui)
{
    int j1 = z[0], j2 = z[1], ma1min = z[3], ma2max = z[4], na = z[5], mb1min = z[6], mb2max = z[7], nb = z[8];
    const double *cgb = t->cg + t->idxcg_block[j1][j2][z[2]];
    double sr = 0.0, si = 0.0;
    int jju1 = t->idxu_block[j1] + (j1 + 1) * mb1min;
    int jju2 = t->idxu_block[j2] + (j2 + 1) * mb2max;
    int icgb = mb1min * (j2 + 1) + mb2max;
    for (int ib = 0; ib < nb; ib++) {
        int ma1 = ma1min, ma2 = ma2max, icga = ma1min * (j2 + 1) + ma2max;
        for (int ia = 0; ia < na; ia++) {
            double c = cgb[icgb] * cgb[icga];
            double u1r = Ur[jju1 + ma1], u1i = Ui[jju1 + ma1], u2r = Ur[jju2 + ma2], u2i = Ui[jju2 + ma2];
            sr += c * (u1r * u2r - u1i * u2i);
            si += c * (u1r * u2i + u1i * u2r);
            ma1++; ma2--; icga += j2;
        }
        jju1 += j1 + 1; jju2 -= j2 + 1; icgb += j2;
    }
    *zr = sr; *zi = si;
}

/* beta weight of Z_{j1 j2 j} in Y_j, cpuSnap4.cpp:763-787 (single element) */
static double beta_weight(int j1, int j2, int j, const orc_tables *t, const double *coeff, int bnorm)
{
    double bj;
    if (j >= j1) {
        bj = coeff[1 + t->idxb_block[j1][j2][j]];
        if (j1 == j) bj *= (j2 == j) ? 3.0 : 2.0;
    } else if (j >= j2) {
        bj = coeff[1 + t->idxb_block[j][j2][j1]];
        if (j2 == j) bj *= 2.0;
    } else {
        bj = coeff[1 + t->idxb_block[j2][j][j1]];
    }
    if (!bnorm && j1 > j) bj *= (j1 + 1) / (j + 1.0);
    return bj;
}

typedef struct {
    int twojmax, switchflag, bzeroflag, bnormflag;
    double rcutfac, rfac0, rmin0, radelem, wjelem;
    const double *coeff;
} orc_snap;

/* Per atom: U (with wself + mirror), Y (half plane), E.  U and Y are full
 * idxu-sized arrays per atom; pairs are given as rij[3*k]. */
static double atom_uye(double *Ur, double *Ui, double *Yr, double *Yi, double *blist,
                       const double *rij, int np, const orc_tables *t, const orc_snap *s)
{
    pairpar pp = {2.0 * s->radelem * s->rcutfac, s->rfac0, s->rmin0, s->wjelem, s->switchflag};
    for (int k = 0; k < t->idxu_max; k++) { Ur[k] = 0.0; Ui[k] = 0.0; Yr[k] = 0.0; Yi[k] = 0.0; }
    for (int p = 0; p < np; p++) {
        pairgeo g;
        pair_geometry(&g, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], &pp, 0);
        add_pair_u(Ur, Ui, t, &g);
    }
    wself_mirror(Ur, Ui, t, 1.0);
    /* Y: every idxz entry contributes beta*Z to Y[jju] */
    for (int iz = 0; iz < t->idxz_max; iz++) {
        const int *z = t->idxz + 10 * iz;
        double zr, zi;
        zentry(&zr, &zi, z, t, Ur, Ui);
        if (s->bnormflag) { zr /= z[2] + 1; zi /= z[2] + 1; }
        double bj = beta_weight(z[0], z[1], z[2], t, s->coeff, s->bnormflag);
        Yr[z[9]] += bj * zr;
        Yi[z[9]] += bj * zi;
    }
    /* E = beta0 + sum_k beta_k B_k,  B = 2 sum_{half plane} U*Z (cpuSnap4.cpp:250-421) */
    double e = s->coeff[0];
    for (int ib = 0; ib < t->idxb_max; ib++) {
        int j1 = t->idxb[3 * ib], j2 = t->idxb[3 * ib + 1], j = t->idxb[3 * ib + 2];
        double sum = 0.0;
        for (int mb = 0; 2 * mb <= j; mb++)
            for (int ma = 0; ma <= j; ma++) {
                double w = 1.0;
                if (2 * mb == j) { if (ma > mb) continue; if (ma == mb) w = 0.5; }
                int zz[10];
                zz[0] = j1; zz[1] = j2; zz[2] = j;
                zz[3] = imax(0, (2 * ma - j - j2 + j1) / 2);
                zz[4] = (2 * ma - j - (2 * zz[3] - j1) + j2) / 2;
                zz[5] = imin(j1, (2 * ma - j + j2 + j1) / 2) - zz[3] + 1;
                zz[6] = imax(0, (2 * mb - j - j2 + j1) / 2);
                zz[7] = (2 * mb - j - (2 * zz[6] - j1) + j2) / 2;
                zz[8] = imin(j1, (2 * mb - j + j2 + j1) / 2) - zz[6] + 1;
                double zr, zi;
                zentry(&zr, &zi, zz, t, Ur, Ui);
                if (s->bnormflag) { zr /= j + 1; zi /= j + 1; }
                int ku = t->idxu_block[j] + (j + 1) * mb + ma;
                sum += w * (Ur[ku] * zr + Ui[ku] * zi);
            }
        double B = 2.0 * sum;
        if (s->bzeroflag) B -= s->bnormflag ? 1.0 : (double)(j + 1);
        if (blist) blist[ib] = B;
        e += s->coeff[1 + ib] * B;
    }
    return e;
}

/* dE/dr_ij for one pair from Y of atom i (cpuSnap4.cpp:798-1175): the U and
 * dU/dx,y,z recursion over the half plane contracted with Y; returns the
 * vector dE/d(rij) (the reference's 2*dedx). */
static void pair_dedr(double *de, const pairgeo *g, const double *Yr, const double *Yi, const orc_tables *t)
{
    int J = t->twojmax;
    double pr[4][JMAXO + 2], pi[4][JMAXO + 2], qr[4][JMAXO + 2], qi[4][JMAXO + 2];
    double u[3] = {g->ux, g->uy, g->uz};
    double acc[3];
    for (int k = 0; k < 3; k++) acc[k] = (g->dsfac * u[k]) * (0.5 * Yr[0]);
    int jd = t->jdim;
    for (int mb = 0; 2 * mb <= J; mb++) {
        int jstart;
        if (mb == 0) {
            for (int d = 0; d < 4; d++) { pr[d][0] = (d == 0) ? 1.0 : 0.0; pi[d][0] = 0.0; }
            jstart = 1;
        } else {
            for (int d = 0; d < 4; d++)
                for (int ma = 0; ma < 2 * mb; ma++) { pr[d][ma] = qr[d][ma]; pi[d][ma] = qi[d][ma]; }
            jstart = 2 * mb;
        }
        for (int j = jstart; j <= J; j++) {
            /* layer step for value (d=0) and the three derivatives (product rule) */
            double o_r[4], o_i[4];      /* old[ma-1] */
            for (int d = 0; d < 4; d++) { o_r[d] = 0.0; o_i[d] = 0.0; }
            for (int ma = 0; ma <= j; ma++) {
                double w_r[4], w_i[4];
                for (int d = 0; d < 4; d++) { w_r[d] = (ma < j) ? pr[d][ma] : 0.0; w_i[d] = (ma < j) ? pi[d][ma] : 0.0; }
                double n_r[4] = {0, 0, 0, 0}, n_i[4] = {0, 0, 0, 0};
                if (ma < j) {
                    double rp = t->rootpq[(j - ma) * jd + (j - mb)];
                    n_r[0] = rp * (g->ar * w_r[0] + g->ai * w_i[0]);
                    n_i[0] = rp * (g->ar * w_i[0] - g->ai * w_r[0]);
                    for (int k = 0; k < 3; k++) {
                        n_r[1 + k] = rp * (g->dar[k] * w_r[0] + g->dai[k] * w_i[0] + g->ar * w_r[1 + k] + g->ai * w_i[1 + k]);
                        n_i[1 + k] = rp * (g->dar[k] * w_i[0] - g->dai[k] * w_r[0] + g->ar * w_i[1 + k] - g->ai * w_r[1 + k]);
                    }
                }
                if (ma > 0) {
                    double rp = t->rootpq[ma * jd + (j - mb)];
                    n_r[0] -= rp * (g->br * o_r[0] + g->bi * o_i[0]);
                    n_i[0] -= rp * (g->br * o_i[0] - g->bi * o_r[0]);
                    for (int k = 0; k < 3; k++) {
                        n_r[1 + k] -= rp * (g->dbr[k] * o_r[0] + g->dbi[k] * o_i[0] + g->br * o_r[1 + k] + g->bi * o_i[1 + k]);
                        n_i[1 + k] -= rp * (g->dbr[k] * o_i[0] - g->dbi[k] * o_r[0] + g->br * o_i[1 + k] - g->bi * o_r[1 + k]);
                    }
                }
                for (int d = 0; d < 4; d++) { pr[d][ma] = n_r[d]; pi[d][ma] = n_i[d]; o_r[d] = w_r[d]; o_i[d] = w_i[d]; }
            }
            if (mb > 0 && j == 2 * mb) {
                /* middle row mirror; the reference negates the imaginary part of the
                 * centre value once and of the centre derivatives twice
                 * (cpuSnap4.cpp:1061-1104), i.e. derivatives keep their centre */
                int h = j / 2;
                for (int ma = 0; ma <= h; ma++) {
                    double s = (ma % 2) ? -1.0 : 1.0;
                    pr[0][h + ma] = s * pr[0][h - ma];
                    pi[0][h + ma] = -s * pi[0][h - ma];
                    if (ma > 0)
                        for (int d = 1; d < 4; d++) { pr[d][h + ma] = s * pr[d][h - ma]; pi[d][h + ma] = -s * pi[d][h - ma]; }
                }
            }
            if (j == 2 * mb + 1) {
                for (int ma = 0; ma <= j; ma++) {
                    double s = ((mb + ma) % 2) ? -1.0 : 1.0;
                    for (int d = 0; d < 4; d++) { qr[d][j - ma] = s * pr[d][ma]; qi[d][j - ma] = -s * pi[d][ma]; }
                }
            }
            int kk = t->idxu_block[j] + (j + 1) * mb;
            int mamax = (2 * mb == j) ? mb : j;
            for (int ma = 0; ma <= mamax; ma++) {
                double yr = Yr[kk + ma], yi = Yi[kk + ma];
                if (2 * mb == j && ma == mb) { yr *= 0.5; yi *= 0.5; }
                for (int k = 0; k < 3; k++)
                    acc[k] += (g->dsfac * pr[0][ma] * u[k] + g->sfac * pr[1 + k][ma]) * yr +
                              (g->dsfac * pi[0][ma] * u[k] + g->sfac * pi[1 + k][ma]) * yi;
            }
        }
    }
    for (int k = 0; k < 3; k++) de[k] = 2.0 * acc[k];
}

/* Full plain SNAP force path on a neighbour list (ComputePairSnap3 semantics):
 * eatom[inum] (set), fatom[3*inum] (set), vatom[6*inum] SoA (set).
 * Pair filter: r^2 < rcut^2 && r^2 > 1e-20 (cpuSnap.cpp:1898-1902). */
void orc_snap_force(double *eatom, double *fatom, double *vatom, const double *x, const int *alist,
                    const int *neighlist, const int *neighnum, int inum, int neighmax,
                    int twojmax, const double *coeff, double rcutfac, double rfac0, double rmin0,
                    double radelem, double wjelem, int switchflag, int bzeroflag, int bnormflag,
                    double *Uout, double *Yout, double *bout)
{
    orc_tables t; build_tables(&t, twojmax);
    orc_snap s = {twojmax, switchflag, bzeroflag, bnormflag, rcutfac, rfac0, rmin0, radelem, wjelem, coeff};
    pairpar pp = {2.0 * radelem * rcutfac, rfac0, rmin0, wjelem, switchflag};
    double rc2 = pp.rcut * pp.rcut;
    int nu = t.idxu_max;
    for (long k = 0; k < 3L * inum; k++) fatom[k] = 0.0;
    for (long k = 0; k < 6L * inum; k++) vatom[k] = 0.0;
    /* per-pair dE/dr, stored then gathered without atomics */
    double *dedr = (double *)calloc((size_t)inum * neighmax * 3, sizeof(double));
    int *pj = (int *)malloc(sizeof(int) * (size_t)inum * neighmax);
    int *np = (int *)calloc(inum, sizeof(int));
    double *rijall = (double *)malloc(sizeof(double) * (size_t)inum * neighmax * 3);
#pragma omp parallel
    {
        double *Ur = (double *)malloc(sizeof(double) * nu * 4);
        double *Ui = Ur + nu, *Yr = Ur + 2 * nu, *Yi = Ur + 3 * nu;
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < inum; i++) {
            double *rij = rijall + (size_t)i * neighmax * 3;
            int n = 0;
            for (int l = 0; l < neighnum[i]; l++) {
                int j = neighlist[(size_t)i * neighmax + l];
                double d0 = x[3 * j] - x[3 * i], d1 = x[3 * j + 1] - x[3 * i + 1], d2 = x[3 * j + 2] - x[3 * i + 2];
                double dsq = d0 * d0 + d1 * d1 + d2 * d2;
                if (dsq < rc2 && dsq > 1e-20) {
                    rij[3 * n] = d0; rij[3 * n + 1] = d1; rij[3 * n + 2] = d2;
                    pj[(size_t)i * neighmax + n] = alist[j];
                    n++;
                }
            }
            np[i] = n;
            eatom[i] = atom_uye(Ur, Ui, Yr, Yi, bout ? bout + (size_t)i * t.idxb_max : NULL, rij, n, &t, &s);
            if (Uout) { memcpy(Uout + (size_t)i * 2 * nu, Ur, sizeof(double) * nu); memcpy(Uout + (size_t)i * 2 * nu + nu, Ui, sizeof(double) * nu); }
            if (Yout) { memcpy(Yout + (size_t)i * 2 * nu, Yr, sizeof(double) * nu); memcpy(Yout + (size_t)i * 2 * nu + nu, Yi, sizeof(double) * nu); }
            for (int p = 0; p < n; p++) {
                pairgeo g;
                pair_geometry(&g, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], &pp, 1);
                pair_dedr(dedr + ((size_t)i * neighmax + p) * 3, &g, Yr, Yi, &t);
            }
        }
        free(Ur);
    }
    /* tally: f_i += dE, f_owner(j) -= dE; virial -0.5 r (x) dE on both */
    for (int i = 0; i < inum; i++)
        for (int p = 0; p < np[i]; p++) {
            const double *d = dedr + ((size_t)i * neighmax + p) * 3;
            const double *r = rijall + ((size_t)i * neighmax + p) * 3;
            int j = pj[(size_t)i * neighmax + p];
            for (int k = 0; k < 3; k++) { fatom[3 * i + k] += d[k]; fatom[3 * j + k] -= d[k]; }
            double vv[6] = {-0.5 * r[0] * d[0], -0.5 * r[1] * d[1], -0.5 * r[2] * d[2],
                            -0.5 * r[0] * d[1], -0.5 * r[0] * d[2], -0.5 * r[1] * d[2]};
            for (int c = 0; c < 6; c++) { vatom[(size_t)c * inum + i] += vv[c]; vatom[(size_t)c * inum + j] += vv[c]; }
        }
    free(dedr); free(pj); free(np); free(rijall);
    free_tables(&t);
}

/* NVE, cpuVelocityIntegration.cpp:307-339 (single type) */
void orc_nve_initial(double *x, double *v, const double *f, double dtf_over_m, double dtv, int inum)
{
    for (long k = 0; k < 3L * inum; k++) { v[k] += dtf_over_m * f[k]; x[k] += dtv * v[k]; }
}

void orc_nve_final(double *v, const double *f, double dtf_over_m, int inum)
{
    for (long k = 0; k < 3L * inum; k++) v[k] += dtf_over_m * f[k];
}
