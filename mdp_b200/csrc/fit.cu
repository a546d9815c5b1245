// Batched SNAP descriptors, dB/dR and the linear-fit normal equations.
//
// For a batch of periodic configurations (general triclinic cells given by
// three lattice vectors, every perpendicular width above rcut so that one
// shell of images holds every pair, as MDP's cpuPeriodicImages3D assumes)
// this computes what MDP's ComputeSnap
// (snappotential.cpp:762-910, cpuSnap2.cpp) computes per configuration:
//   bi[k]          = sum_i B_ik
//   G[i][c][k]     = d(sum_a B_ak)/dx_ic  (= -bd of cpuSnapTallyBispectrumDeriv)
//   bv[k][6]       virial (cpuSnapTallyBispectrumVirial)
// and assembles the normal equations of the linear fit as Regression.cpp:386-404
// does with dd = G: rows r = [we * (N, bi)] (target we * E) and
// [wf * (0, G[i][c])] (target -wf * f_ic), A = R^T R, b = R^T t.
//
// Pipeline (all on one stream, captured into one CUDA graph by mdp_fit_run):
//   pairs (brute force over each configuration's atoms and 27 images)
//   U      (k_snap_uc, the MD engine's kernel)
//   Z, B   (k_fit_zbt: every coupling's Z rows per atom, B for j >= j1)
//   dU/dr  (k_fit_du: forward-mode, coefficient-free recursion, per pair and direction)
//   dB/dr  (k_fit_dbdr: the three Z . dU terms of cpuComputeDbidrj:826-1013)
//   rows   (k_fit_rows: atomic-free gather over own and reverse pairs)
//   A, b   (k_fit_gram: FP64, or BF16 hi/lo split with FP32 tensor-core sums)
#include "common.cuh"
#include "engine.h"
#include "fit.h"

#include <cuda_bf16.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <vector>

namespace mdp {

// ---------------------------------------------------------------------------
// pairs: every atom against every atom of its configuration and the 27 images
// ---------------------------------------------------------------------------
template <bool EMIT>
__global__ void k_fit_pairs(const double4 *__restrict__ x, const int *__restrict__ cfg, const int *__restrict__ ca0,
                            const int *__restrict__ cn, const double4 *__restrict__ cbox, int natoms, SnapGeom gp,
                            int *__restrict__ pcount, const int *__restrict__ poff, double4 *__restrict__ prij,
                            double4 *__restrict__ pab, int2 *__restrict__ pinfo)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natoms) return;
    const int c = cfg[i], a0 = ca0[c], n = cn[c];
    // lattice vectors a, b, c of the configuration's cell (rows of cbox)
    const double4 la = cbox[3 * c], lb = cbox[3 * c + 1], lc = cbox[3 * c + 2], xi = x[i];
    int cnt = 0, p = EMIT ? poff[i] : 0;
    for (int jj = 0; jj < n; jj++) {
        const double4 xj = x[a0 + jj];
        for (int im = 0; im < 27; im++) {
            const double u = im % 3 - 1, v = (im / 3) % 3 - 1, w = im / 9 - 1;
            const double sx = u * la.x + v * lb.x + w * lc.x, sy = u * la.y + v * lb.y + w * lc.y,
                         sz = u * la.z + v * lb.z + w * lc.z;
            const double d0 = xj.x + sx - xi.x, d1 = xj.y + sy - xi.y, d2 = xj.z + sz - xi.z;
            const double rsq = d0 * d0 + d1 * d1 + d2 * d2;
            if (rsq < gp.rcutsq && rsq > 1e-20) {
                if (EMIT) {
                    PairGeo g;
                    pair_geometry<false>(g, d0, d1, d2, gp);
                    prij[p] = make_double4(d0, d1, d2, g.sfac);
                    pab[p] = make_double4(g.ar, g.ai, g.br, g.bi);
                    pinfo[p] = make_int2(i, a0 + jj);
                    p++;
                } else {
                    cnt++;
                }
            }
        }
    }
    if (!EMIT) pcount[i] = cnt;
}

// ZBL reference potential of every atom of the batch (the pair term that MDP's
// fitsnap.jl subtracts from the training targets): brute force over the
// atom's configuration and 27 images as k_fit_pairs, pairs within the ZBL
// outer cutoff.  Per atom: energy u/2 per pair, force du/dx_ij, virial
// -x_ij (x) du/dx_ij / 2 in the order xx, yy, zz, xy, xz, yz ([6][natoms]).
__global__ void k_fit_zbl(const double4 *__restrict__ x, const int *__restrict__ cfg, const int *__restrict__ ca0,
                          const int *__restrict__ cn, const double4 *__restrict__ cbox, int natoms, ZblParams zp,
                          double *__restrict__ eatom, double *__restrict__ fatom, double *__restrict__ vatom)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natoms) return;
    const int c = cfg[i], a0 = ca0[c], n = cn[c];
    const double4 la = cbox[3 * c], lb = cbox[3 * c + 1], lc = cbox[3 * c + 2], xi = x[i];
    double e = 0.0, fx = 0.0, fy = 0.0, fz = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
    for (int jj = 0; jj < n; jj++) {
        const double4 xj = x[a0 + jj];
        for (int im = 0; im < 27; im++) {
            const double u0 = im % 3 - 1, u1 = (im / 3) % 3 - 1, u2 = im / 9 - 1;
            const double d0 = xj.x + (u0 * la.x + u1 * lb.x + u2 * lc.x) - xi.x;
            const double d1 = xj.y + (u0 * la.y + u1 * lb.y + u2 * lc.y) - xi.y;
            const double d2 = xj.z + (u0 * la.z + u1 * lb.z + u2 * lc.z) - xi.z;
            const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
            if (!(r2 <= zp.rcsq && r2 > 1e-20)) continue;
            double u, g;
            zbl_pair(zp, sqrt(r2), u, g);
            const double ux = g * d0, uy = g * d1, uz = g * d2;
            e += 0.5 * u;
            fx += ux; fy += uy; fz += uz;
            v[0] -= 0.5 * d0 * ux; v[1] -= 0.5 * d1 * uy; v[2] -= 0.5 * d2 * uz;
            v[3] -= 0.5 * d0 * uy; v[4] -= 0.5 * d0 * uz; v[5] -= 0.5 * d1 * uz;
        }
    }
    eatom[i] = e;
    fatom[3 * (size_t)i] = fx; fatom[3 * (size_t)i + 1] = fy; fatom[3 * (size_t)i + 2] = fz;
    for (int k = 0; k < 6; k++) vatom[k * (size_t)natoms + i] = v[k];
}

// ---------------------------------------------------------------------------
// Z rows of every coupling and B for j >= j1, per 32-atom tile (lane = atom)
// Z layout [tile][zoff + (j+1) mb + ma][lane]; B layout [k][atom]
// ---------------------------------------------------------------------------
// Every coupling is compile-time specialised (CG coefficients as constant
// operands, U rows in registers), output layer by layer.  Within a layer all
// warps walk the couplings in the same order, so the code in flight is one
// coupling's; each warp owns a row mb and a range [lo, hi) of its entries ma
// (a plan balanced on the host), which needs no reduction between warps.
// (Giving each warp whole (coupling, mb) rows round-robin let the warps run
// different couplings' code at once: 4.9 no_instruction stalls per issue.)
// warps per CTA (one CTA per SM: the 146 KB U tile): the 4,096-configuration
// graph took 278-280 ms at 10 warps, 278 ms at 12 and 290 ms at 5
#ifndef FIT_ZBT_WARPS_N
#define FIT_ZBT_WARPS_N 10
#endif
constexpr int FIT_ZBT_WARPS = FIT_ZBT_WARPS_N;
struct ZbPlan {
    unsigned char mb[JD][FIT_ZBT_WARPS], lo[JD][FIT_ZBT_WARPS], hi[JD][FIT_ZBT_WARPS];   // mb 255: idle
};

// offset of coupling (J1, J2, J)'s rows in the Z layout (fit_tables order)
__host__ __device__ constexpr int fit_zoff(int tj, int J1, int J2, int J)
{
    int nz = 0;
    for (int j1 = 0; j1 <= tj; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= cmin(tj, j1 + j2); j += 2) {
                if (j1 == J1 && j2 == J2 && j == J) return nz;
                nz += (j / 2 + 1) * (j + 1);
            }
    return -1;
}

// entries lo <= ma < hi of row mb of scale * Z_{J1 J2 J}, summed over every
// row pair ib, written to the coupling's block Zc ([(J+1) mb + ma][lane])
template <int J1, int J2, int J>
__device__ __forceinline__ void zbt_rows(const int mb, const int lo, const int hi, const double2 *__restrict__ Us,
                                         const int lane, const double scale, double2 *__restrict__ Zc)
{
    constexpr int N1 = J1 + 1, N2 = J2 + 1;
    constexpr int CGB = cg_block(J1, J2, J);
    double yr[J + 1], yi[J + 1];
#pragma unroll
    for (int ma = 0; ma <= J; ma++) { yr[ma] = 0.0; yi[ma] = 0.0; }
    const int mb1min = max(0, (2 * mb - J - J2 + J1) / 2);
    const int mb2max = (2 * mb - J - (2 * mb1min - J1) + J2) / 2;
    const int nb = nb_of(J1, J2, J, mb);
    for (int ib = 0; ib < nb; ib++) {
        const int mb1 = mb1min + ib, mb2 = mb2max - ib;
        const double sc = scale * cgc<double>(CGB + mb1 * N2 + mb2);
        const double2 *r1 = Us + (idxu_block(J1) + N1 * mb1) * 32 + lane;
        const double2 *r2 = Us + (idxu_block(J2) + N2 * mb2) * 32 + lane;
        double u1r[N1], u1i[N1], u2r[N2], u2i[N2];
#pragma unroll
        for (int k = 0; k < N1; k++) { const double2 v = r1[k * 32]; u1r[k] = sc * v.x; u1i[k] = sc * v.y; }
#pragma unroll
        for (int k = 0; k < N2; k++) { const double2 v = r2[k * 32]; u2r[k] = v.x; u2i[k] = v.y; }
#pragma unroll
        for (int ma = 0; ma <= J; ma++) {
            if (ma < lo || ma >= hi) continue;
            const int ma1min = cmax(0, (2 * ma - J - J2 + J1) / 2);
            const int ma2max = (2 * ma - J - (2 * ma1min - J1) + J2) / 2;
            const int na = cmin(J1, (2 * ma - J + J2 + J1) / 2) - ma1min + 1;
#pragma unroll
            for (int ia = 0; ia < na; ia++) {
                const int ma1 = ma1min + ia, ma2 = ma2max - ia;
                const double c = cgc<double>(CGB + ma1 * N2 + ma2);
                const double tr = c * u1r[ma1], ti = c * u1i[ma1];
                yr[ma] += tr * u2r[ma2] - ti * u2i[ma2];
                yi[ma] += tr * u2i[ma2] + ti * u2r[ma2];
            }
        }
    }
#pragma unroll
    for (int ma = 0; ma <= J; ma++)
        if (ma >= lo && ma < hi) Zc[(size_t)((J + 1) * mb + ma) * 32] = make_double2(yr[ma], yi[ma]);
}

template <int TJ, int J, int J1, int J2>
__device__ __forceinline__ void zbt_layer(const double2 *__restrict__ Us, double2 *__restrict__ Zt, const int lane,
                                          const int mb, const int lo, const int hi, const double scale)
{
    if constexpr (J1 <= TJ) {
        if constexpr (J2 <= J1) {
            if constexpr (coupling_ok(J1, J2, J)) {
                constexpr int ZO = fit_zoff(TJ, J1, J2, J);
                zbt_rows<J1, J2, J>(mb, lo, hi, Us, lane, scale, Zt + (size_t)ZO * 32);
            }
            zbt_layer<TJ, J, J1, J2 + 1>(Us, Zt, lane, mb, lo, hi, scale);
        } else {
            zbt_layer<TJ, J, J1 + 1, 0>(Us, Zt, lane, mb, lo, hi, scale);
        }
    }
}

template <int TJ, int J>
__device__ __forceinline__ void zbt_layers(const double2 *__restrict__ Us, double2 *__restrict__ Zt, const int lane,
                                           const int w, const int bnorm, const ZbPlan &P)
{
    if constexpr (J <= TJ) {
        const int mb = P.mb[J][w];
        if (mb != 255) zbt_layer<TJ, J, 0, 0>(Us, Zt, lane, mb, P.lo[J][w], P.hi[J][w], bnorm ? 1.0 / (J + 1) : 1.0);
        __syncthreads();   // keeps the warps on one layer's code
        zbt_layers<TJ, J + 1>(Us, Zt, lane, w, bnorm, P);
    }
}

template <int TJ>
__global__ void __launch_bounds__(FIT_ZBT_WARPS * 32, 1)
k_fit_zbt(const double2 *__restrict__ Ut, int natoms, const FitTables *__restrict__ T, const ZbPlan P,
          double2 *__restrict__ Z, double *__restrict__ B, int tile_lo, int tile_hi)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    double2 *Us = reinterpret_cast<double2 *>(smraw);
    constexpr int NU = idxu_count(TJ);
    const int nz = T->nz;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int tile = tile_lo + blockIdx.x; tile < tile_hi; tile += gridDim.x) {
        const double2 *src = Ut + (size_t)tile * NU * 32;
        for (int k = threadIdx.x; k < NU * 32; k += blockDim.x) Us[k] = src[k];
        __syncthreads();
        double2 *Zt = Z + (size_t)(tile - tile_lo) * nz * 32 + lane;
        zbt_layers<TJ, 0>(Us, Zt, lane, w, T->bnorm, P);   // ends on a barrier: B reads other warps' Z rows
        // B_k = 2 sum_half w Re(U_j* Z) (- bzero), cpuComputeBi2 (cpuSnap2.cpp:516-541)
        const int atom = tile * 32 + lane;
        for (int k = w; k < T->ntri; k += FIT_ZBT_WARPS) {
            const FitTriple tr = T->tr[k];
            const int j = tr.j;
            const FitCoupling cp = T->cp[tr.coup[0]];
            double s = 0.0;
            for (int mb = 0; 2 * mb <= j; mb++)
                for (int ma = 0; ma <= j; ma++) {
                    const double wgt = (2 * mb < j) ? 1.0 : (ma < mb ? 1.0 : (ma == mb ? 0.5 : 0.0));
                    if (wgt == 0.0) continue;
                    const double2 u = Us[(idxu_block(j) + (j + 1) * mb + ma) * 32 + lane];
                    const double2 z = Zt[(size_t)(cp.zoff + (j + 1) * mb + ma) * 32];
                    s += wgt * (u.x * z.x + u.y * z.y);
                }
            double b = 2.0 * s;
            if (T->bzero) b -= T->bnorm ? 1.0 : (double)(j + 1);
            if (atom < natoms) B[(size_t)k * natoms + atom] = b;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// dU/dr of one pair along one axis, forward mode through the coefficient-free
// recursion (v_J[ma] = conj(a) v[ma] - conj(b) v[ma-1], u = unorm v):
//   dul[yh][t] = unorm * (dsfac u_dir v + sfac dv)   (ComputeSij's dulist)
// t = pair * 3 + dir; the half plane in yh order (rows of a middle layer full)
// ---------------------------------------------------------------------------
template <int TJ, int J, int MB>
__device__ __forceinline__ void fdu_row(const double ar, const double ai, const double br, const double bi,
                                        const double dar, const double dai, const double dbr, const double dbi,
                                        double (&pr)[TJ + 1], double (&pi)[TJ + 1], double (&qr)[TJ + 1],
                                        double (&qi)[TJ + 1])
{
    {
        const double vr = pr[J - 1], vi = pi[J - 1], wr = qr[J - 1], wi = qi[J - 1];
        pr[J] = -(br * vr + bi * vi);
        pi[J] = -(br * vi - bi * vr);
        qr[J] = -(dbr * vr + dbi * vi + br * wr + bi * wi);
        qi[J] = -(dbr * vi - dbi * vr + br * wi - bi * wr);
    }
#pragma unroll
    for (int ma = J - 1; ma >= 0; ma--) {
        const double ur = pr[ma], ui = pi[ma], xr = qr[ma], xi = qi[ma];
        double nr = ar * ur + ai * ui, ni = ar * ui - ai * ur;
        double mr = dar * ur + dai * ui + ar * xr + ai * xi, mi = dar * ui - dai * ur + ar * xi - ai * xr;
        if (ma > 0) {
            const double vr = pr[ma - 1], vi = pi[ma - 1], wr = qr[ma - 1], wi = qi[ma - 1];
            nr -= br * vr + bi * vi;
            ni -= br * vi - bi * vr;
            mr -= dbr * vr + dbi * vi + br * wr + bi * wi;
            mi -= dbr * vi - dbi * vr + br * wi - bi * wr;
        }
        pr[ma] = nr; pi[ma] = ni; qr[ma] = mr; qi[ma] = mi;
    }
    if constexpr (MB > 0 && J == 2 * MB) {
#pragma unroll
        for (int ma = 0; ma <= MB; ma++) {
            const double s = (ma & 1) ? -1.0 : 1.0;
            pr[MB + ma] = s * pr[MB - ma]; pi[MB + ma] = -s * pi[MB - ma];
            qr[MB + ma] = s * qr[MB - ma]; qi[MB + ma] = -s * qi[MB - ma];
        }
    }
}

template <int TJ>
struct FduState {
    double ar, ai, br, bi, dar, dai, dbr, dbi, sf, dsu;
    double pr[TJ + 1], pi[TJ + 1], qr[TJ + 1], qi[TJ + 1];   // current row and its derivative
    double sr[TJ + 1], si[TJ + 1], tr[TJ + 1], ti[TJ + 1];   // next column's seed
};

template <int TJ, int J, int MB>
__device__ __forceinline__ void fdu_column(FduState<TJ> &s, double2 *__restrict__ out, const long stride)
{
    if constexpr (J <= TJ) {
        if constexpr (J > 0) fdu_row<TJ, J, MB>(s.ar, s.ai, s.br, s.bi, s.dar, s.dai, s.dbr, s.dbi, s.pr, s.pi, s.qr, s.qi);
#pragma unroll
        for (int ma = 0; ma <= J; ma++) {
            const double nu = unorm<double>(J, MB, ma);
            out[(long)(yh_block(J) + (J + 1) * MB + ma) * stride] =
                make_double2(nu * (s.dsu * s.pr[ma] + s.sf * s.qr[ma]), nu * (s.dsu * s.pi[ma] + s.sf * s.qi[ma]));
        }
        if constexpr (J == 2 * MB + 1 && 2 * (MB + 1) <= TJ) {
#pragma unroll
            for (int ma = 0; ma <= J; ma++) {
                const double sg = ((MB + ma) & 1) ? -1.0 : 1.0;
                s.sr[J - ma] = sg * s.pr[ma]; s.si[J - ma] = -sg * s.pi[ma];
                s.tr[J - ma] = sg * s.qr[ma]; s.ti[J - ma] = -sg * s.qi[ma];
            }
        }
        fdu_column<TJ, J + 1, MB>(s, out, stride);
    }
}

template <int TJ, int MB>
__device__ __forceinline__ void fdu_columns(FduState<TJ> &s, double2 *__restrict__ out, const long stride)
{
    if constexpr (2 * MB <= TJ) {
        if constexpr (MB == 0) {
            s.pr[0] = 1.0; s.pi[0] = 0.0; s.qr[0] = 0.0; s.qi[0] = 0.0;
        } else {
#pragma unroll
            for (int ma = 0; ma < 2 * MB; ma++) { s.pr[ma] = s.sr[ma]; s.pi[ma] = s.si[ma]; s.qr[ma] = s.tr[ma]; s.qi[ma] = s.ti[ma]; }
        }
        fdu_column<TJ, (MB == 0 ? 0 : 2 * MB), MB>(s, out, stride);
        fdu_columns<TJ, MB + 1>(s, out, stride);
    }
}

template <int TJ>
__global__ void __launch_bounds__(128)
k_fit_du(const double4 *__restrict__ prij, long npairs, SnapGeom gp, double2 *__restrict__ dul, long stride)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * npairs) return;
    const long p = t / 3;
    const int dir = (int)(t - 3 * p);
    const double4 r = prij[p];
    PairGeo g;
    pair_geometry<true>(g, r.x, r.y, r.z, gp);
    FduState<TJ> s;
    s.ar = g.ar; s.ai = g.ai; s.br = g.br; s.bi = g.bi;
    s.dar = g.dar[dir]; s.dai = g.dai[dir]; s.dbr = g.dbr[dir]; s.dbi = g.dbi[dir];
    s.sf = g.sfac;
    s.dsu = g.dsfac * g.u[dir];
    fdu_columns<TJ, 0>(s, dul + t, stride);
}

// ---------------------------------------------------------------------------
// dB_ik/dr_p along one axis: 2 sum over the three terms of cpuComputeDbidrj
// (Z of the centre atom's couplings against the pair's dU rows), half plane
// with the middle row's centre at 1/2.
// ---------------------------------------------------------------------------
// Every dB/dR term is compile-time: triple k = (j1, j2, j) has the terms
//   Z(j1, j2, j) . dU_j,  Z(j, j2, j1) . dU_j1,  Z(j, j1, j2) . dU_j2
// with factors 2, 2 (j+1)/(j1+1), 2 (j+1)/(j2+1) (2, 2, 2 with bnorm), so the
// 55 sums at 2J = 8 stay in registers and the Z offsets are immediates.  The
// pair's dU is read one row (layer L, column MB) at a time and every term on
// layer L is applied to that row.  (With the term list read from a table at
// run time, acc[k] lived in local memory and each term's read-modify-write
// waited on the previous one.)
struct FitTri {
    int j1, j2, j;
};
__host__ __device__ constexpr FitTri fit_tri(int tj, int k)
{
    int n = 0;
    for (int j1 = 0; j1 <= tj; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= cmin(tj, j1 + j2); j += 2)
                if (j >= j1) {
                    if (n == k) return FitTri{j1, j2, j};
                    n++;
                }
    return FitTri{-1, -1, -1};
}

// Z(C1, C2, L) row MB against the dU row (dr, di), entries 0..MAMAX
template <int TJ, int L, int MB, int MAMAX, int ZS, int C1, int C2>
__device__ __forceinline__ double fdb_dot(const double (&dr)[MAMAX + 1], const double (&di)[MAMAX + 1],
                                          const double2 *__restrict__ Zi)
{
    constexpr int ZO = fit_zoff(TJ, C1, C2, L) + (L + 1) * MB;
    const double2 *z = Zi + ZO * ZS;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int ma = 0; ma <= MAMAX; ma++) {
        const double2 zz = z[ma * ZS];
        if (ma & 1) s1 += dr[ma] * zz.x + di[ma] * zz.y;
        else s0 += dr[ma] * zz.x + di[ma] * zz.y;
    }
    return s0 + s1;
}

template <int TJ, int L, int MB, int MAMAX, int ZS, int K>
__device__ __forceinline__ void fdb_terms(const double (&dr)[MAMAX + 1], const double (&di)[MAMAX + 1],
                                          const double2 *__restrict__ Zi, double (&acc)[nbispec(TJ)],
                                          const int bnorm)
{
    if constexpr (K < nbispec(TJ)) {
        constexpr FitTri t = fit_tri(TJ, K);
        if constexpr (t.j == L) acc[K] += 2.0 * fdb_dot<TJ, L, MB, MAMAX, ZS, t.j1, t.j2>(dr, di, Zi);
        if constexpr (t.j1 == L)
            acc[K] += (bnorm ? 2.0 : 2.0 * (t.j + 1) / (t.j1 + 1.0)) * fdb_dot<TJ, L, MB, MAMAX, ZS, t.j, t.j2>(dr, di, Zi);
        if constexpr (t.j2 == L)
            acc[K] += (bnorm ? 2.0 : 2.0 * (t.j + 1) / (t.j2 + 1.0)) * fdb_dot<TJ, L, MB, MAMAX, ZS, t.j, t.j1>(dr, di, Zi);
        fdb_terms<TJ, L, MB, MAMAX, ZS, K + 1>(dr, di, Zi, acc, bnorm);
    }
}

// rows MB.. of layer L (and the layers above): dU row in registers (a middle
// row's right half has no term; its centre counts 1/2), then its terms
template <int TJ, int L, int MB, int ZS>
__device__ __forceinline__ void fdb_rows(const double2 *__restrict__ d, const long stride,
                                         const double2 *__restrict__ Zi, double (&acc)[nbispec(TJ)],
                                         const int bnorm)
{
    if constexpr (L <= TJ) {
        if constexpr (2 * MB <= L) {
            constexpr int MAMAX = (2 * MB == L) ? MB : L;
            double dr[MAMAX + 1], di[MAMAX + 1];
#pragma unroll
            for (int ma = 0; ma <= MAMAX; ma++) {
                const double2 v = d[(long)(yh_block(L) + (L + 1) * MB + ma) * stride];
                const double w = (2 * MB == L && ma == MB) ? 0.5 : 1.0;
                dr[ma] = w * v.x;
                di[ma] = w * v.y;
            }
            fdb_terms<TJ, L, MB, MAMAX, ZS, 0>(dr, di, Zi, acc, bnorm);
            fdb_rows<TJ, L, MB + 1, ZS>(d, stride, Zi, acc, bnorm);
        } else {
            fdb_rows<TJ, L + 1, 0, ZS>(d, stride, Zi, acc, bnorm);
        }
    }
}

// dB_ik/dr_p along one axis: 2 sum over the three terms of cpuComputeDbidrj
// (Z of the centre atom's couplings against the pair's dU rows), half plane
// with the middle row's centre at 1/2.  dbdr[t * ntri + k], t = (p - p_lo) * 3
// + dir: a pair-direction's components are contiguous, so the row gathers
// (k fastest over threads) read them coalesced.  A CTA takes APC adjacent
// atoms (APC divides 32, so they share a Z tile) and their pairs, 64 threads
// per atom: the atoms' Z rows (38 KB per atom at 2J = 8) are copied once into
// shared memory ([entry][atom]), so every pair-direction reads them there.  Read in place from the tile
// layout, each entry sat in its own 128-byte line, 512 bytes from the next:
// an atom's rows touched 2,386 lines, more than L1 holds for the atoms in
// flight, and the dot products waited on L2.
constexpr int FIT_DB_TPA = 64;   // threads per atom
template <int TJ, int APC>
__global__ void __launch_bounds__(FIT_DB_TPA * APC)
k_fit_dbdr(const double2 *__restrict__ dul, long stride, const int *__restrict__ poff,
           const int2 *__restrict__ pinfo, int a_lo, int a_hi, long p_lo, const FitTables *__restrict__ T,
           const double2 *__restrict__ Z, int tile_lo, double *__restrict__ dbdr)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    double2 *Zs = reinterpret_cast<double2 *>(smraw);   // [entry][APC]
    const int nz = T->nz, bnorm = T->bnorm;
    const int a0 = (a_lo & ~(APC - 1)) + blockIdx.x * APC;
    const int alo = max(a0, a_lo), ahi = min(a0 + APC, a_hi);
    for (int e = threadIdx.x; e < nz * APC; e += blockDim.x) {
        const int k = e / APC, a = a0 + (e - k * APC);
        if (a >= alo && a < ahi) Zs[e] = Z[((size_t)((a >> 5) - tile_lo) * nz + k) * 32 + (a & 31)];
    }
    __syncthreads();
    if (alo >= ahi) return;
    const long q0 = poff[alo], n3 = 3 * (long)(poff[ahi] - q0);
    for (long i = threadIdx.x; i < n3; i += blockDim.x) {
        const long p = q0 + i / 3;
        const long t = (p - p_lo) * 3 + (i - (i / 3) * 3);
        const int atom = pinfo[p].x;
        constexpr int NK = nbispec(TJ);
        double acc[NK];
#pragma unroll
        for (int k = 0; k < NK; k++) acc[k] = 0.0;
        fdb_rows<TJ, 0, 0, APC>(dul + t, stride, Zs + (atom - a0), acc, bnorm);
#pragma unroll
        for (int k = 0; k < NK; k++) dbdr[t * NK + k] = acc[k];
    }
}

// ---------------------------------------------------------------------------
// reverse pairs (pairs whose neighbour is atom a), sorted for a fixed sum order
// ---------------------------------------------------------------------------
__global__ void k_fit_rev_count(const int2 *__restrict__ pinfo, long npairs, int *__restrict__ rcount)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < npairs) atomicAdd(&rcount[pinfo[p].y], 1);
}
__global__ void k_fit_rev_fill(const int2 *__restrict__ pinfo, long npairs, const int *__restrict__ roff,
                               int *__restrict__ cursor, int *__restrict__ rlist)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int a = pinfo[p].y;
    rlist[roff[a] + atomicAdd(&cursor[a], 1)] = (int)p;
}
__global__ void k_fit_rev_sort(int natoms, const int *__restrict__ roff, int *__restrict__ rlist)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= natoms) return;
    const int s = roff[a], e = roff[a + 1];
    for (int i = s + 1; i < e; i++) {
        const int v = rlist[i];
        int j = i - 1;
        while (j >= s && rlist[j] > v) { rlist[j + 1] = rlist[j]; j--; }
        rlist[j + 1] = v;
    }
}

// rows of atom a: G[a][c][k] = sum_(p: j = a) dbdr - sum_(p: i = a) dbdr,
// written as fit rows [wf * (0, G)] with target -wf * f; row = 3 a + c
__global__ void k_fit_rows(int a_lo, int a_hi, int ntri, const int *__restrict__ poff, const int *__restrict__ roff,
                           const int *__restrict__ rlist, const double *__restrict__ dbdr, long p_lo,
                           const int *__restrict__ cfg, const double *__restrict__ wf, const double *__restrict__ f,
                           double *__restrict__ G, double *__restrict__ R, double *__restrict__ tgt, long row0)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (atom, k)
    if (t >= (long)(a_hi - a_lo) * FIT_KP) return;
    const int a = a_lo + (int)(t / FIT_KP), k = (int)(t % FIT_KP);
    const double w = wf ? wf[cfg[a]] : 1.0;
    double g[3] = {0.0, 0.0, 0.0};
    if (k >= 1 && k <= ntri) {
        const int kk = k - 1;
        for (int q = roff[a]; q < roff[a + 1]; q++) {
            const long p = rlist[q] - p_lo;
#pragma unroll
            for (int c = 0; c < 3; c++) g[c] += dbdr[(3 * p + c) * ntri + kk];
        }
        for (long p = poff[a] - p_lo; p < poff[a + 1] - p_lo; p++) {
#pragma unroll
            for (int c = 0; c < 3; c++) g[c] -= dbdr[(3 * p + c) * ntri + kk];
        }
        if (G)
            for (int c = 0; c < 3; c++) G[((size_t)a * 3 + c) * ntri + kk] = g[c];
    }
    if (R) {
        for (int c = 0; c < 3; c++) R[(size_t)(row0 + 3 * a + c) * FIT_KP + k] = w * g[c];
        if (k == 0 && tgt)
            for (int c = 0; c < 3; c++) tgt[row0 + 3 * a + c] = f ? -w * f[3 * (size_t)a + c] : 0.0;
    }
}

// per configuration: bi, the virial, and the energy row [we * (N, bi)] / we * E
__global__ void k_fit_cfg(int c_lo, int c_hi, int ntri, const int *__restrict__ ca0, const int *__restrict__ cn,
                          const int *__restrict__ poff, const double *__restrict__ B, int natoms,
                          const double *__restrict__ dbdr, long p_lo, const double4 *__restrict__ prij,
                          const double *__restrict__ we, const double *__restrict__ e, double *__restrict__ bi,
                          double *__restrict__ bv, double *__restrict__ R, double *__restrict__ tgt, long erow0)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (config, k)
    if (t >= (long)(c_hi - c_lo) * FIT_KP) return;
    const int c = c_lo + (int)(t / FIT_KP), k = (int)(t % FIT_KP);
    const int a0 = ca0[c], n = cn[c];
    double v = 0.0;
    if (k == 0) v = (double)n;
    if (k >= 1 && k <= ntri) {
        const int kk = k - 1;
        for (int a = a0; a < a0 + n; a++) v += B[(size_t)kk * natoms + a];
        if (bi) bi[(size_t)c * ntri + kk] = v;
        if (bv) {
            double s[6] = {0, 0, 0, 0, 0, 0};
            for (long p = poff[a0]; p < poff[a0 + n]; p++) {
                const double4 r = prij[p];
                const long q = p - p_lo;
                const double bx = dbdr[(3 * q) * ntri + kk], by = dbdr[(3 * q + 1) * ntri + kk],
                             bz = dbdr[(3 * q + 2) * ntri + kk];
                s[0] -= r.x * bx; s[1] -= r.y * by; s[2] -= r.z * bz;
                s[3] -= r.x * by; s[4] -= r.x * bz; s[5] -= r.y * bz;
            }
            for (int q = 0; q < 6; q++) bv[((size_t)c * ntri + kk) * 6 + q] = s[q];
        }
    }
    if (R) {
        const double w = we ? we[c] : 1.0;
        R[(size_t)(erow0 + c) * FIT_KP + k] = (k <= ntri) ? w * v : 0.0;
        if (k == 0 && tgt) tgt[erow0 + c] = e ? w * e[c] : 0.0;
    }
}

// ---------------------------------------------------------------------------
// A = R^T R, b = R^T t over rows [0, nrows)
// FP64: each CTA sums a slab of rows into a 64 x 64 (+ 64) partial; the
// partials are added in a fixed order by k_fit_reduce.
// BF16: columns equilibrated to unit norm (FP64 pre-pass), R = hi + lo (two
// BF16 terms), hi^T hi + hi^T lo + lo^T hi with FP32 accumulation by warp-level
// tensor-core MMA (m16n8k16), partials per CTA summed in FP64, scaling undone.
// ---------------------------------------------------------------------------
constexpr int FIT_GRAM_THREADS = 256;

// Thread (ti, tj) = (tid / 16, tid % 16) owns A[ti + 16 m][tj + 16 k], m, k in
// 0..3: per row, 4 + 4 shared loads feed 16 FMAs, and the 16 lanes of a
// half-warp read 16 consecutive doubles (no bank conflicts).  64 rows are
// staged per barrier pair.
constexpr int FIT_GRAM_ROWS = 64;
__global__ void __launch_bounds__(FIT_GRAM_THREADS)
k_fit_gram64(const double *__restrict__ R, const double *__restrict__ tgt, long nrows, int rows_per_cta,
             double *__restrict__ part)
{
    __shared__ double sr[FIT_GRAM_ROWS][FIT_KP];
    __shared__ double st[FIT_GRAM_ROWS];
    const long r0 = (long)blockIdx.x * rows_per_cta, r1 = min(nrows, r0 + rows_per_cta);
    const int tid = threadIdx.x, ti = tid >> 4, tj = tid & 15;
    double acc[4][4], accb[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        accb[m] = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) acc[m][k] = 0.0;
    }
    for (long rb = r0; rb < r1; rb += FIT_GRAM_ROWS) {
        __syncthreads();
        for (int e = tid; e < FIT_GRAM_ROWS * FIT_KP; e += FIT_GRAM_THREADS) {
            const int rr = e / FIT_KP, cc = e % FIT_KP;
            sr[rr][cc] = (rb + rr < r1) ? R[(size_t)(rb + rr) * FIT_KP + cc] : 0.0;
        }
        if (tid < FIT_GRAM_ROWS) st[tid] = (rb + tid < r1) ? tgt[rb + tid] : 0.0;
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < FIT_GRAM_ROWS; rr++) {
            double a[4], b[4];
#pragma unroll
            for (int m = 0; m < 4; m++) { a[m] = sr[rr][ti + 16 * m]; b[m] = sr[rr][tj + 16 * m]; }
#pragma unroll
            for (int m = 0; m < 4; m++)
#pragma unroll
                for (int k = 0; k < 4; k++) acc[m][k] += a[m] * b[k];
            if (tj == 0) {
                const double t = st[rr];
#pragma unroll
                for (int m = 0; m < 4; m++) accb[m] += a[m] * t;
            }
        }
    }
    double *o = part + (size_t)blockIdx.x * (FIT_KP * FIT_KP + FIT_KP);
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
        for (int k = 0; k < 4; k++) o[(ti + 16 * m) * FIT_KP + tj + 16 * k] = acc[m][k];
    if (tj == 0)
#pragma unroll
        for (int m = 0; m < 4; m++) o[FIT_KP * FIT_KP + ti + 16 * m] = accb[m];
}

// column sums of squares of R (one partial per CTA), for the equilibration
__global__ void k_fit_colsq(const double *__restrict__ R, long nrows, int rows_per_cta, double *__restrict__ part)
{
    const int c = threadIdx.x;   // 64 threads
    const long r0 = (long)blockIdx.x * rows_per_cta, r1 = min(nrows, r0 + rows_per_cta);
    double s = 0.0;
    for (long r = r0; r < r1; r++) { const double v = R[r * FIT_KP + c]; s += v * v; }
    part[(size_t)blockIdx.x * FIT_KP + c] = s;
}

// hi / lo BF16 split of the column-equilibrated rows R[r][k] / sqrt(sum_r R[r][k]^2)
__global__ void k_fit_split(const double *__restrict__ R, long n, const double *__restrict__ colsq,
                            __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double q = colsq[i % FIT_KP];
    const double v = q > 0.0 ? R[i] / sqrt(q) : 0.0;
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[i] = h;
    lo[i] = __double2bfloat16(v - (double)__bfloat162float(h));
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2])
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// one CTA of 4 warps: warp w owns output rows 16w .. 16w+15 of the 64 x 64
// product and all 8 column tiles; k runs over the CTA's slab of data rows in
// steps of 16.  The slab tile (16 rows x 64, hi and lo) is staged in shared
// memory, from which the A (R^T, row-major m x k) and B (R, column-major k x n)
// fragments are read.
__global__ void __launch_bounds__(128)
k_fit_gram_bf16(const __nv_bfloat16 *__restrict__ hi, const __nv_bfloat16 *__restrict__ lo, long nrows,
                int rows_per_cta, float *__restrict__ part)
{
    __shared__ __nv_bfloat16 sh[2][16][FIT_KP + 8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, tq = lane & 3;
    const long r0 = (long)blockIdx.x * rows_per_cta, r1 = min(nrows, r0 + rows_per_cta);
    float acc[8][4];
#pragma unroll
    for (int n = 0; n < 8; n++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[n][q] = 0.f;
    for (long rb = r0; rb < r1; rb += 16) {
        __syncthreads();
        for (int e = threadIdx.x; e < 16 * FIT_KP; e += blockDim.x) {
            const int rr = e / FIT_KP, cc = e % FIT_KP;
            const bool ok = rb + rr < r1;
            sh[0][rr][cc] = ok ? hi[(size_t)(rb + rr) * FIT_KP + cc] : __float2bfloat16(0.f);
            sh[1][rr][cc] = ok ? lo[(size_t)(rb + rr) * FIT_KP + cc] : __float2bfloat16(0.f);
        }
        __syncthreads();
        // A fragment (16 x 16, row-major): element (m, k) = R[k][16w + m]
        auto afrag = [&](int s, unsigned (&a)[4]) {
            const int m0 = 16 * w + g, m1 = m0 + 8, k0 = 2 * tq, k1 = k0 + 8;
            __nv_bfloat162 v;
            v.x = sh[s][k0][m0]; v.y = sh[s][k0 + 1][m0]; a[0] = *reinterpret_cast<unsigned *>(&v);
            v.x = sh[s][k0][m1]; v.y = sh[s][k0 + 1][m1]; a[1] = *reinterpret_cast<unsigned *>(&v);
            v.x = sh[s][k1][m0]; v.y = sh[s][k1 + 1][m0]; a[2] = *reinterpret_cast<unsigned *>(&v);
            v.x = sh[s][k1][m1]; v.y = sh[s][k1 + 1][m1]; a[3] = *reinterpret_cast<unsigned *>(&v);
        };
        // B fragment (16 x 8, column-major): element (k, n) = R[k][8 nt + n]
        auto bfrag = [&](int s, int nt, unsigned (&b)[2]) {
            const int n = 8 * nt + g, k0 = 2 * tq, k1 = k0 + 8;
            __nv_bfloat162 v;
            v.x = sh[s][k0][n]; v.y = sh[s][k0 + 1][n]; b[0] = *reinterpret_cast<unsigned *>(&v);
            v.x = sh[s][k1][n]; v.y = sh[s][k1 + 1][n]; b[1] = *reinterpret_cast<unsigned *>(&v);
        };
        unsigned ah[4], al[4];
        afrag(0, ah);
        afrag(1, al);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            unsigned bh[2], bl[2];
            bfrag(0, nt, bh);
            bfrag(1, nt, bl);
            mma_bf16_16816(acc[nt], ah, bh);
            mma_bf16_16816(acc[nt], ah, bl);
            mma_bf16_16816(acc[nt], al, bh);
        }
    }
    float *o = part + (size_t)blockIdx.x * FIT_KP * FIT_KP;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int m0 = 16 * w + g, n0 = 8 * nt + 2 * tq;
        o[m0 * FIT_KP + n0] = acc[nt][0];
        o[m0 * FIT_KP + n0 + 1] = acc[nt][1];
        o[(m0 + 8) * FIT_KP + n0] = acc[nt][2];
        o[(m0 + 8) * FIT_KP + n0 + 1] = acc[nt][3];
    }
}

// b in the BF16 form: FP32 products of the split rows with the FP64 target
// rounded to FP32, one partial per CTA (R^T t is a 64-vector; no MMA needed)
__global__ void k_fit_rhs_bf16(const __nv_bfloat16 *__restrict__ hi, const __nv_bfloat16 *__restrict__ lo,
                               const double *__restrict__ tgt, long nrows, int rows_per_cta, float *__restrict__ part)
{
    const int c = threadIdx.x;   // 64 threads
    const long r0 = (long)blockIdx.x * rows_per_cta, r1 = min(nrows, r0 + rows_per_cta);
    float s = 0.f;
    for (long r = r0; r < r1; r++) {
        const float t = (float)tgt[r];
        s += (__bfloat162float(hi[r * FIT_KP + c]) + __bfloat162float(lo[r * FIT_KP + c])) * t;
    }
    part[(size_t)blockIdx.x * FIT_KP + c] = s;
}

template <typename P>
__global__ void k_fit_reduce(const P *__restrict__ part, int nparts, int width, long pstride, double *__restrict__ out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= width) return;
    double s = 0.0;
    for (int q = 0; q < nparts; q++) s += (double)part[(size_t)q * pstride + e];
    out[e] += s;
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
static void fit_tables(FitTables &T, int tj, int bnorm, int bzero)
{
    memset(&T, 0, sizeof(T));
    T.tj = tj; T.bnorm = bnorm; T.bzero = bzero;
    int idx[JD][JD][JD];
    for (int a = 0; a < JD; a++) for (int b = 0; b < JD; b++) for (int c = 0; c < JD; c++) idx[a][b][c] = -1;
    int nz = 0;
    for (int j1 = 0; j1 <= tj; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(tj, j1 + j2); j += 2) {
                FitCoupling &c = T.cp[T.ncoup];
                c.j1 = j1; c.j2 = j2; c.j = j; c.zoff = nz;
                idx[j1][j2][j] = T.ncoup++;
                nz += (j / 2 + 1) * (j + 1);
            }
    T.nz = nz;
    for (int j1 = 0; j1 <= tj; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(tj, j1 + j2); j += 2) {
                if (j < j1) continue;
                FitTriple &t = T.tr[T.ntri++];
                t.j1 = j1; t.j2 = j2; t.j = j;
                // cpuComputeDbidrj:826-1013: z(j1,j2,j) with dU_j; z(j,j2,j1) with dU_j1
                // times (j+1)/(j1+1); z(j,j1,j2) with dU_j2 times (j+1)/(j2+1)
                t.layer[0] = j; t.coup[0] = idx[j1][j2][j]; t.fac[0] = 1.0;
                t.layer[1] = j1; t.coup[1] = idx[j][j2][j1]; t.fac[1] = bnorm ? 1.0 : (j + 1) / (j1 + 1.0);
                t.layer[2] = j2; t.coup[2] = idx[j][j1][j2]; t.fac[2] = bnorm ? 1.0 : (j + 1) / (j2 + 1.0);
            }
    int q = 0;
    for (int L = 0; L < JD; L++) {
        T.lt_off[L] = q;
        for (int k = 0; k < T.ntri; k++)
            for (int r = 0; r < 3; r++)
                if (T.tr[k].layer[r] == L) {
                    T.lt_k[q] = k;
                    T.lt_z[q] = T.cp[T.tr[k].coup[r]].zoff;
                    T.lt_fac[q] = 2.0 * T.tr[k].fac[r];
                    q++;
                }
        T.lt_n[L] = q - T.lt_off[L];
    }
}

}  // namespace mdp

using namespace mdp;

namespace mdp {
// per-pair dB/dR of the whole batch as float [pair][3][k] and the per-atom
// bispectrum [k][atom] (FP64): the descriptor stages chunk by chunk
__global__ void k_fit_dbdr_export(const double *__restrict__ dbdr, long np, int ntri, long p_lo,
                                  float *__restrict__ out)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (local pair * 3 + dir, k)
    if (t >= 3 * np * ntri) return;
    const int k = (int)(t % ntri);
    const long pd = t / ntri;
    out[(p_lo * 3 + pd) * ntri + k] = (float)dbdr[t];
}
}  // namespace mdp

namespace mdp {

static int fit_pairs(mdp_fit *h)
{
    const int n = h->natoms;
    const int tb = 128, gb = (n + tb - 1) / tb;
    if (h->pcount.ensure(sizeof(int) * n) || h->poff.ensure(sizeof(int) * (n + 1)) ||
        h->scan_tmp.ensure(sizeof(int) * scan_tmp_ints(n + 1)))
        return -1;
    k_fit_pairs<false><<<gb, tb, 0, h->s>>>(h->x.as<double4>(), h->cfg.as<int>(), h->ca0.as<int>(), h->cn.as<int>(),
                                            h->cbox.as<double4>(), n, h->model.geom, h->pcount.as<int>(), nullptr,
                                            nullptr, nullptr, nullptr);
    if (exclusive_scan(h->pcount.as<int>(), h->poff.as<int>(), n, h->scan_tmp.as<int>(), h->s)) return -1;
    int np = 0;
    MDP_CUDA_TRY(cudaMemcpyAsync(&np, h->poff.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, h->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(h->s));
    h->npairs = np;
    ForcePath &fp = h->fp;
    const long pc = std::max(1L, h->npairs);
    if (fp.poff.ensure(sizeof(int) * (n + 1)) || fp.prij.ensure(sizeof(double4) * pc) ||
        fp.pab.ensure(sizeof(double4) * pc) || fp.pinfo.ensure(sizeof(int2) * pc))
        return -1;
    MDP_CUDA_TRY(cudaMemcpyAsync(fp.poff.p, h->poff.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, h->s));
    k_fit_pairs<true><<<gb, tb, 0, h->s>>>(h->x.as<double4>(), h->cfg.as<int>(), h->ca0.as<int>(), h->cn.as<int>(),
                                           h->cbox.as<double4>(), n, h->model.geom, nullptr, h->poff.as<int>(),
                                           fp.prij.as<double4>(), fp.pab.as<double4>(), fp.pinfo.as<int2>());
    // reverse pairs
    if (h->rcount.ensure(sizeof(int) * n) || h->roff.ensure(sizeof(int) * (n + 1)) ||
        h->cursor.ensure(sizeof(int) * n) || h->rlist.ensure(sizeof(int) * pc))
        return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(h->rcount.p, 0, sizeof(int) * n, h->s));
    MDP_CUDA_TRY(cudaMemsetAsync(h->cursor.p, 0, sizeof(int) * n, h->s));
    const int pb = (int)((h->npairs + 255) / 256);
    if (h->npairs) k_fit_rev_count<<<pb, 256, 0, h->s>>>(fp.pinfo.as<int2>(), h->npairs, h->rcount.as<int>());
    if (exclusive_scan(h->rcount.as<int>(), h->roff.as<int>(), n, h->scan_tmp.as<int>(), h->s)) return -1;
    if (h->npairs) k_fit_rev_fill<<<pb, 256, 0, h->s>>>(fp.pinfo.as<int2>(), h->npairs, h->roff.as<int>(),
                                                        h->cursor.as<int>(), h->rlist.as<int>());
    k_fit_rev_sort<<<gb, tb, 0, h->s>>>(n, h->roff.as<int>(), h->rlist.as<int>());
    count_launches(5);
    MDP_CUDA_TRY(cudaGetLastError());
    h->pairs_ready = true;
    return 0;
}

template <int TJ>
static int fit_launch_du(mdp_fit *h, const mdp_fit::Chunk &ck)
{
    if (tu_ensure_tables()) return -1;
    const long np = ck.p_hi - ck.p_lo, nt = 3 * np;
    if (nt == 0) return 0;
    k_fit_du<TJ><<<(unsigned)((nt + h->du_threads - 1) / h->du_threads), h->du_threads, 0, h->s>>>(
        h->fp.prij.as<double4>() + ck.p_lo, np, h->model.geom, h->dul.as<double2>(), nt);
    count_launches(1);
    return 0;
}

static int fit_du(mdp_fit *h, const mdp_fit::Chunk &ck)
{
    const int tj = h->model.p.twojmax;
    return tj == 8 ? fit_launch_du<8>(h, ck) : tj == 6 ? fit_launch_du<6>(h, ck) : fit_launch_du<4>(h, ck);
}

// least largest sum of c cut into k contiguous chunks (greedy under a cap)
static long zb_min_cap(const std::vector<long> &c, int k)
{
    long lo = 0, hi = 0;
    for (long v : c) { lo = std::max(lo, v); hi += v; }
    while (lo < hi) {
        const long mid = (lo + hi) / 2;
        int n = 1;
        long run = 0;
        for (long v : c) {
            if (run + v > mid) { n++; run = v; }
            else run += v;
        }
        if (n <= k) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// The Z-kernel plan of 2J = tj: per layer J, the rows get warps where the
// costliest chunk is, and each row's entries ma are cut into that many
// contiguous ranges of least largest cost.  Cost of entry ma: 6 instructions
// per term over every coupling and row pair; every warp on a row also pays
// the row pairs' U loads (4 per u1 entry with its scaling, 1 per u2 entry).
static ZbPlan zb_plan(int tj)
{
    ZbPlan P;
    memset(&P, 0, sizeof(P));
    memset(P.mb, 255, sizeof(P.mb));
    for (int J = 0; J <= tj; J++) {
        const int R = J / 2 + 1;
        std::vector<std::vector<long>> c(R, std::vector<long>(J + 1, 0));
        std::vector<long> load(R, 0);
        for (int mb = 0; mb < R; mb++)
            for (int j1 = 0; j1 <= tj; j1++)
                for (int j2 = 0; j2 <= j1; j2++) {
                    if (!coupling_ok(j1, j2, J)) continue;
                    const int nb = nb_of(j1, j2, J, mb);
                    load[mb] += (long)nb * (4 * (j1 + 1) + (j2 + 1));
                    for (int ma = 0; ma <= J; ma++) {
                        const int ma1min = std::max(0, (2 * ma - J - j2 + j1) / 2);
                        const int na = std::min(j1, (2 * ma - J + j2 + j1) / 2) - ma1min + 1;
                        c[mb][ma] += 6L * nb * na;
                    }
                }
        std::vector<int> nw(R, 1);
        for (int used = R; used < FIT_ZBT_WARPS; used++) {
            int best = -1;
            long bc = -1;
            for (int r = 0; r < R; r++) {
                if (nw[r] >= J + 1) continue;
                const long v = zb_min_cap(c[r], nw[r]) + load[r];
                if (v > bc) { bc = v; best = r; }
            }
            if (best < 0) break;
            nw[best]++;
        }
        int w = 0;
        for (int r = 0; r < R; r++) {
            const long cap = zb_min_cap(c[r], nw[r]);
            int a = 0;
            for (int k = 0; k < nw[r]; k++, w++) {
                int b = a;
                long run = 0;
                if (k == nw[r] - 1) b = J + 1;
                else
                    while (b <= J && run + c[r][b] <= cap) run += c[r][b++];
                P.mb[J][w] = (unsigned char)r;
                P.lo[J][w] = (unsigned char)a;
                P.hi[J][w] = (unsigned char)b;
                a = b;
            }
        }
    }
    return P;
}

// Z rows and B of one chunk's tiles (the fit takes 2J = 4, 6, 8)
template <int TJ>
static int fit_zbt(mdp_fit *h, const mdp_fit::Chunk &ck, unsigned g)
{
    static const ZbPlan plan = zb_plan(TJ);
    const size_t zsm = (size_t)idxu_count(TJ) * 32 * sizeof(double2);
    int per_sm = 0;
    if (kernel_setup((const void *)k_fit_zbt<TJ>, FIT_ZBT_WARPS * 32, zsm, &per_sm, "k_fit_zbt")) return -1;
    k_fit_zbt<TJ><<<g, FIT_ZBT_WARPS * 32, zsm, h->s>>>(h->fp.Ut.as<double2>(), h->natoms, h->tabs.as<FitTables>(),
                                                       plan, h->Z.as<double2>(), h->B.as<double>(), ck.t_lo,
                                                       ck.t_hi);
    return 0;
}

static int fit_zb(mdp_fit *h, const mdp_fit::Chunk &ck)
{
    const unsigned g = (unsigned)std::max(1, std::min(ck.t_hi - ck.t_lo, num_sms()));
    int rc = 0;
    switch (h->model.p.twojmax) {
    case 8: rc = fit_zbt<8>(h, ck, g); break;
    case 6: rc = fit_zbt<6>(h, ck, g); break;
    default: rc = fit_zbt<4>(h, ck, g); break;
    }
    count_launches(1);
    return rc;
}

template <int TJ, int APC>
static int fit_dbdr_apc(mdp_fit *h, const mdp_fit::Chunk &ck)
{
    const long nt = 3 * (ck.p_hi - ck.p_lo);
    const size_t sm = (size_t)h->tab.nz * APC * sizeof(double2);
    int per_sm = 0;
    if (kernel_setup((const void *)k_fit_dbdr<TJ, APC>, FIT_DB_TPA * APC, sm, &per_sm, "k_fit_dbdr")) return -1;
    const int a0 = ck.a_lo & ~(APC - 1);
    const unsigned g = (unsigned)((ck.a_hi - a0 + APC - 1) / APC);
    k_fit_dbdr<TJ, APC><<<g, FIT_DB_TPA * APC, sm, h->s>>>(
        h->dul.as<double2>(), nt, h->poff.as<int>(), h->fp.pinfo.as<int2>(), ck.a_lo, ck.a_hi, ck.p_lo,
        h->tabs.as<FitTables>(), h->Z.as<double2>(), ck.t_lo, h->dbdr.as<double>());
    return 0;
}

template <int TJ>
static int fit_dbdr_tj(mdp_fit *h, const mdp_fit::Chunk &ck, int threads)
{
    switch (threads / FIT_DB_TPA) {
    case 1: return fit_dbdr_apc<TJ, 1>(h, ck);
    case 4: return fit_dbdr_apc<TJ, 4>(h, ck);
    default: return fit_dbdr_apc<TJ, 2>(h, ck);
    }
}

// threads = FIT_DB_TPA x atoms per CTA (64, 128 or 256)
static int fit_dbdr(mdp_fit *h, const mdp_fit::Chunk &ck, int threads)
{
    if (ck.p_hi == ck.p_lo) return 0;
    int rc;
    switch (h->model.p.twojmax) {
    case 8: rc = fit_dbdr_tj<8>(h, ck, threads); break;
    case 6: rc = fit_dbdr_tj<6>(h, ck, threads); break;
    default: rc = fit_dbdr_tj<4>(h, ck, threads); break;
    }
    count_launches(1);
    return rc;
}

// Z/B, dU, dB/dR of one chunk, then its rows: into R / tgt (rows) and/or the
// descriptor outputs G [atom][3][k], bi [config][k], bv [config][k][6]
static int fit_chunk(mdp_fit *h, const mdp_fit::Chunk &ck, bool rows, double *G, double *bi, double *bv)
{
    const int n = h->natoms;
    if (fit_zb(h, ck)) return -1;
    if (fit_du(h, ck)) return -1;
    if (fit_dbdr(h, ck, h->db_threads)) return -1;
    const long ta = (long)(ck.a_hi - ck.a_lo) * FIT_KP, tc = (long)(ck.c_hi - ck.c_lo) * FIT_KP;
    k_fit_rows<<<(unsigned)((ta + 255) / 256), 256, 0, h->s>>>(
        ck.a_lo, ck.a_hi, h->tab.ntri, h->poff.as<int>(), h->roff.as<int>(), h->rlist.as<int>(), h->dbdr.as<double>(),
        ck.p_lo, h->cfg.as<int>(), h->wf.as<double>(), h->f.as<double>(), G, rows ? h->R.as<double>() : nullptr,
        rows ? h->tgt.as<double>() : nullptr, h->nconf);
    k_fit_cfg<<<(unsigned)((tc + 255) / 256), 256, 0, h->s>>>(
        ck.c_lo, ck.c_hi, h->tab.ntri, h->ca0.as<int>(), h->cn.as<int>(), h->poff.as<int>(), h->B.as<double>(), n,
        h->dbdr.as<double>(), ck.p_lo, h->fp.prij.as<double4>(), h->we.as<double>(), h->e.as<double>(), bi, bv,
        rows ? h->R.as<double>() : nullptr, rows ? h->tgt.as<double>() : nullptr, 0);
    count_launches(2);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// U over the batch, then every chunk; no host synchronisation
static int fit_descriptor_stages(mdp_fit *h, bool rows, double *G = nullptr, double *bi = nullptr,
                                 double *bv = nullptr)
{
    const int n = h->natoms, tj = h->model.p.twojmax;
    if (tu_ensure_tables()) return -1;
    const int urc = tj == 8 ? launch_ui<double, 8>(h->model, h->fp, n, h->s)
                  : tj == 6 ? launch_ui<double, 6>(h->model, h->fp, n, h->s)
                            : launch_ui<double, 4>(h->model, h->fp, n, h->s);
    if (urc) return -1;
    count_launches(1);
    for (const auto &ck : h->chunks)
        if (fit_chunk(h, ck, rows, G, bi, bv)) return -1;
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int fit_pair_derivs(mdp_fit *h, float *dbdr_out, double *blist_out)
{
    if (!h || !h->pairs_ready) { set_error("set a batch first"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(h->device));
    const int n = h->natoms, tj = h->model.p.twojmax, nk = h->tab.ntri;
    if (tu_ensure_tables()) return -1;
    const int urc = tj == 8 ? launch_ui<double, 8>(h->model, h->fp, n, h->s)
                  : tj == 6 ? launch_ui<double, 6>(h->model, h->fp, n, h->s)
                            : launch_ui<double, 4>(h->model, h->fp, n, h->s);
    if (urc) return -1;
    for (const auto &ck : h->chunks) {
        if (fit_zb(h, ck)) return -1;
        if (fit_du(h, ck)) return -1;
        if (fit_dbdr(h, ck, h->db_threads)) return -1;
        const long np = ck.p_hi - ck.p_lo, ne = 3 * np * nk;
        if (ne) k_fit_dbdr_export<<<(unsigned)((ne + 255) / 256), 256, 0, h->s>>>(h->dbdr.as<double>(), np, nk,
                                                                                ck.p_lo, dbdr_out);
        count_launches(1);
    }
    if (blist_out)
        MDP_CUDA_TRY(cudaMemcpyAsync(blist_out, h->B.p, sizeof(double) * nk * (size_t)n, cudaMemcpyDeviceToDevice,
                                     h->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(h->s));
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int fit_gram_stages(mdp_fit *h, int mode)
{
    const long nr = h->nrows;
    const int rpc = h->gram_rows;
    const int nb = (int)((nr + rpc - 1) / rpc);
    double *out = h->out.as<double>();
    MDP_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * (FIT_KP * FIT_KP + FIT_KP), h->s));
    if (mode == 0) {
        k_fit_gram64<<<nb, FIT_GRAM_THREADS, 0, h->s>>>(h->R.as<double>(), h->tgt.as<double>(), nr, rpc,
                                                      h->part.as<double>());
        const int w = FIT_KP * FIT_KP + FIT_KP;
        k_fit_reduce<double><<<(w + 255) / 256, 256, 0, h->s>>>(h->part.as<double>(), nb, w, w, out);
        count_launches(2);
    } else {
        const long ne = nr * FIT_KP;
        double *colsq = out + FIT_KP * FIT_KP + FIT_KP;
        MDP_CUDA_TRY(cudaMemsetAsync(colsq, 0, sizeof(double) * FIT_KP, h->s));
        k_fit_colsq<<<nb, FIT_KP, 0, h->s>>>(h->R.as<double>(), nr, rpc, h->part.as<double>());
        k_fit_reduce<double><<<1, FIT_KP, 0, h->s>>>(h->part.as<double>(), nb, FIT_KP, FIT_KP, colsq);
        k_fit_split<<<(unsigned)((ne + 255) / 256), 256, 0, h->s>>>(h->R.as<double>(), ne, colsq,
                                                                    h->hi.as<__nv_bfloat16>(), h->lo.as<__nv_bfloat16>());
        float *pf = h->part.as<float>();
        k_fit_gram_bf16<<<nb, 128, 0, h->s>>>(h->hi.as<__nv_bfloat16>(), h->lo.as<__nv_bfloat16>(), nr, rpc, pf);
        k_fit_reduce<float><<<(FIT_KP * FIT_KP + 255) / 256, 256, 0, h->s>>>(pf, nb, FIT_KP * FIT_KP,
                                                                           FIT_KP * FIT_KP, out);
        float *pb = pf + (size_t)nb * FIT_KP * FIT_KP;
        k_fit_rhs_bf16<<<nb, FIT_KP, 0, h->s>>>(h->hi.as<__nv_bfloat16>(), h->lo.as<__nv_bfloat16>(),
                                                h->tgt.as<double>(), nr, rpc, pb);
        k_fit_reduce<float><<<1, FIT_KP, 0, h->s>>>(pb, nb, FIT_KP, FIT_KP, out + FIT_KP * FIT_KP);
        count_launches(7);
    }
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}


static int fit_alloc_work(mdp_fit *h)
{
    const int n = h->natoms, tj = h->model.p.twojmax;
    const long ntiles = (n + 31) / 32;
    h->nrows = h->nconf + 3L * n;
    // chunk plan over whole configurations
    std::vector<int> poff(n + 1);
    MDP_CUDA_TRY(cudaStreamSynchronize(h->s));
    MDP_CUDA_TRY(cudaMemcpy(poff.data(), h->poff.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    const double per_pair = 3.0 * (yh_count(tj) * sizeof(double2) + h->tab.ntri * sizeof(double));
    const double per_tile = (double)h->tab.nz * 32 * sizeof(double2);
    h->chunks.clear();
    h->chunk_pairs_max = 1;
    h->chunk_tiles_max = 1;
    int c = 0;
    while (c < h->nconf) {
        mdp_fit::Chunk ck;
        ck.c_lo = c;
        ck.a_lo = h->h_ca0[c];
        ck.p_lo = poff[ck.a_lo];
        int c_hi = c;
        while (c_hi < h->nconf) {
            const int a_hi = h->h_ca0[c_hi] + h->h_cn[c_hi];
            const double bytes = per_pair * (poff[a_hi] - ck.p_lo) + per_tile * ((a_hi + 31) / 32 - ck.a_lo / 32);
            if (c_hi > c && bytes > h->chunk_bytes) break;
            c_hi++;
        }
        ck.c_hi = c_hi;
        ck.a_hi = h->h_ca0[c_hi - 1] + h->h_cn[c_hi - 1];
        ck.p_hi = poff[ck.a_hi];
        ck.t_lo = ck.a_lo / 32;
        ck.t_hi = (ck.a_hi + 31) / 32;
        h->chunk_pairs_max = std::max(h->chunk_pairs_max, ck.p_hi - ck.p_lo);
        h->chunk_tiles_max = std::max(h->chunk_tiles_max, ck.t_hi - ck.t_lo);
        h->chunks.push_back(ck);
        c = c_hi;
    }
    const long nt = 3 * h->chunk_pairs_max;
    const int nbmax = (int)((h->nrows + 255) / 256) + 1;   // smallest Gram rows-per-CTA candidate
    if (!h->gram_tuned) {
        // rows per Gram CTA: the largest candidate that still gives two CTAs per SM
        h->gram_rows = 256;
        for (int c : {1024, 4096})
            if (h->nrows / c >= 2L * num_sms()) h->gram_rows = c;
    }
    if (h->fp.Ut.ensure(sizeof(double2) * ntiles * idxu_count(tj) * 32) ||
        h->Z.ensure(sizeof(double2) * (size_t)h->chunk_tiles_max * h->tab.nz * 32) ||
        h->B.ensure(sizeof(double) * h->tab.ntri * (size_t)n) ||
        h->dul.ensure(sizeof(double2) * (size_t)nt * yh_count(tj)) ||
        h->dbdr.ensure(sizeof(double) * (size_t)nt * h->tab.ntri) ||
        h->R.ensure(sizeof(double) * h->nrows * FIT_KP) || h->tgt.ensure(sizeof(double) * h->nrows) ||
        h->hi.ensure(sizeof(__nv_bfloat16) * h->nrows * FIT_KP) || h->lo.ensure(sizeof(__nv_bfloat16) * h->nrows * FIT_KP) ||
        h->part.ensure(sizeof(double) * (size_t)nbmax * (FIT_KP * FIT_KP + FIT_KP)) ||
        h->out.ensure(sizeof(double) * (FIT_KP * FIT_KP + 2 * FIT_KP)))
        return -1;
    return 0;
}

static void fit_drop_graph(mdp_fit *h)
{
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->gexec = nullptr;
    h->graph = nullptr;
    h->graph_mode = -1;
}

}  // namespace mdp

extern "C" {

int mdp_fit_create(mdp_fit **hp, const mdp_snap_params *p, int device)
{
    if (!hp || !p) { set_error("null argument"); return -1; }
    *hp = nullptr;
    if (p->twojmax != 4 && p->twojmax != 6 && p->twojmax != 8) { set_error("twojmax must be 4, 6 or 8"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(device));
    mdp_snap_params q = *p;
    std::vector<double> ones(1 + 64, 1.0);
    if (!q.coeff) { q.coeff = ones.data(); q.ncoeffall = 1 + mdp_snap_ncoeff(p->twojmax); }
    mdp_fit *h = new mdp_fit();
    h->device = device;
    if (model_init(h->model, &q)) { delete h; return -1; }
    if (h->model.ne > 1) { set_error("the batched fit takes one element type"); delete h; return -1; }
    fit_tables(h->tab, p->twojmax, p->bnormflag, p->bzeroflag);
    if (cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking) != cudaSuccess || h->tabs.ensure(sizeof(FitTables))) {
        mdp_fit_destroy(h);
        set_error("stream / table allocation failed");
        return -1;
    }
    MDP_CUDA_TRY(cudaMemcpy(h->tabs.p, &h->tab, sizeof(FitTables), cudaMemcpyHostToDevice));
    *hp = h;
    return 0;
}

void mdp_fit_destroy(mdp_fit *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->s) cudaStreamSynchronize(h->s);
    fit_drop_graph(h);
    DevBuf *b[] = {&h->x, &h->cfg, &h->ca0, &h->cn, &h->cbox, &h->we, &h->wf, &h->e, &h->f, &h->tabs, &h->pcount,
                   &h->poff, &h->roff, &h->rcount, &h->cursor, &h->rlist, &h->B, &h->Z, &h->dul, &h->dbdr, &h->G,
                   &h->R, &h->tgt, &h->hi, &h->lo, &h->part, &h->out, &h->scan_tmp};
    for (auto x : b) x->release();
    h->fp.release();
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
}

int mdp_fit_ncoeff(mdp_fit *h) { return h ? h->tab.ntri : -1; }

// Batch of nconf configurations: natoms[c], lattice[9c..9c+8] (the cell's
// vectors a, b, c as rows), x (all positions concatenated, 3 per atom, inside
// the cell), targets e[c] and f (3 per atom), weights we[c], wf[c] (any of e,
// f, we, wf may be NULL: zero targets, unit weights).  Builds the pair lists.
int mdp_fit_set_batch_lattice(mdp_fit *h, int nconf, const int *natoms, const double *lattice, const double *x,
                              const double *e, const double *f, const double *we, const double *wf)
{
    if (!h || nconf < 1 || !natoms || !lattice || !x) { set_error("bad arguments"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(h->device));
    const double need = h->model.geom.rcut;
    long total = 0;
    h->h_cn.assign(natoms, natoms + nconf);
    h->h_ca0.resize(nconf);
    for (int c = 0; c < nconf; c++) {
        if (natoms[c] < 1) { set_error("configuration %d has no atoms", c); return -1; }
        // perpendicular width of the cell across each lattice vector: |volume| / |cross of the other two|
        const double *L = lattice + 9 * (size_t)c;
        for (int d = 0; d < 3; d++) {
            const double *p = L + 3 * ((d + 1) % 3), *q = L + 3 * ((d + 2) % 3), *r = L + 3 * d;
            const double cx = p[1] * q[2] - p[2] * q[1], cy = p[2] * q[0] - p[0] * q[2], cz = p[0] * q[1] - p[1] * q[0];
            const double width = fabs(r[0] * cx + r[1] * cy + r[2] * cz) / sqrt(cx * cx + cy * cy + cz * cz);
            if (!(width > need)) {
                set_error("configuration %d: cell width %g across lattice vector %d must exceed the cutoff %g "
                          "(one image shell)", c, width, d, need);
                return -1;
            }
        }
        h->h_ca0[c] = (int)total;
        total += natoms[c];
    }
    if (total > (1L << 30)) { set_error("batch too large"); return -1; }
    h->h_lat.assign(lattice, lattice + 9 * (size_t)nconf);
    fit_drop_graph(h);
    h->nconf = nconf;
    h->natoms = (int)total;
    const int n = h->natoms;
    std::vector<double> x4(4 * (size_t)n), b4(12 * (size_t)nconf, 0.0);
    std::vector<int> cid(n);
    for (int c = 0; c < nconf; c++) {
        for (int r = 0; r < 3; r++)
            for (int d = 0; d < 3; d++) b4[12 * c + 4 * r + d] = lattice[9 * c + 3 * r + d];
        for (int a = 0; a < natoms[c]; a++) cid[h->h_ca0[c] + a] = c;
    }
    for (long i = 0; i < n; i++) { x4[4 * i] = x[3 * i]; x4[4 * i + 1] = x[3 * i + 1]; x4[4 * i + 2] = x[3 * i + 2]; x4[4 * i + 3] = 0.0; }
    if (h->x.ensure(sizeof(double4) * n) || h->cfg.ensure(sizeof(int) * n) || h->ca0.ensure(sizeof(int) * nconf) ||
        h->cn.ensure(sizeof(int) * nconf) || h->cbox.ensure(3 * sizeof(double4) * nconf) ||
        h->we.ensure(sizeof(double) * nconf) || h->wf.ensure(sizeof(double) * nconf) ||
        h->e.ensure(sizeof(double) * nconf) || h->f.ensure(sizeof(double) * 3 * (size_t)n))
        return -1;
    std::vector<double> ones(nconf, 1.0), zc(nconf, 0.0), zf(3 * (size_t)n, 0.0);
    MDP_CUDA_TRY(cudaMemcpy(h->x.p, x4.data(), sizeof(double4) * n, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->cfg.p, cid.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->ca0.p, h->h_ca0.data(), sizeof(int) * nconf, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->cn.p, natoms, sizeof(int) * nconf, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->cbox.p, b4.data(), 3 * sizeof(double4) * nconf, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->we.p, we ? we : ones.data(), sizeof(double) * nconf, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->wf.p, wf ? wf : ones.data(), sizeof(double) * nconf, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->e.p, e ? e : zc.data(), sizeof(double) * nconf, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(h->f.p, f ? f : zf.data(), sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice));
    // a copy from pageable memory may return before it lands, and the batch
    // is read next on the fit's non-blocking stream
    MDP_CUDA_TRY(cudaDeviceSynchronize());
    if (fit_pairs(h) || fit_alloc_work(h)) return -1;
    return 0;
}

// Orthogonal cells: box[3c..3c+2] are the edge lengths, x inside [0, L).
int mdp_fit_set_batch(mdp_fit *h, int nconf, const int *natoms, const double *box, const double *x,
                      const double *e, const double *f, const double *we, const double *wf)
{
    if (!h || nconf < 1 || !natoms || !box || !x) { set_error("bad arguments"); return -1; }
    std::vector<double> lat(9 * (size_t)nconf, 0.0);
    for (int c = 0; c < nconf; c++)
        for (int d = 0; d < 3; d++) lat[9 * c + 4 * d] = box[3 * c + d];
    return mdp_fit_set_batch_lattice(h, nconf, natoms, lat.data(), x, e, f, we, wf);
}

// ZBL reference potential (inner, outer, z) of every atom of the current
// batch into host arrays: eatom[natoms], fatom[3 natoms], vatom[6][natoms]
// (xx, yy, zz, xy, xz, yz).  Every cell width must exceed the outer cutoff.
int mdp_fit_zbl(mdp_fit *h, double inner, double outer, double z, double *eatom, double *fatom, double *vatom)
{
    if (!h || h->natoms < 1 || !eatom || !fatom || !vatom) { set_error("bad arguments"); return -1; }
    ZblParams zp;
    if (zbl_setup(zp, inner, outer, z)) return -1;
    if (!zp.on) { set_error("ZBL atomic number must be positive (got %g)", z); return -1; }
    for (int c = 0; c < h->nconf; c++) {
        const double *L = h->h_lat.data() + 9 * (size_t)c;
        for (int d = 0; d < 3; d++) {
            const double *p = L + 3 * ((d + 1) % 3), *q = L + 3 * ((d + 2) % 3), *r = L + 3 * d;
            const double cx = p[1] * q[2] - p[2] * q[1], cy = p[2] * q[0] - p[0] * q[2], cz = p[0] * q[1] - p[1] * q[0];
            const double width = fabs(r[0] * cx + r[1] * cy + r[2] * cz) / sqrt(cx * cx + cy * cy + cz * cz);
            if (!(width > outer)) {
                set_error("configuration %d: cell width %g must exceed the ZBL cutoff %g", c, width, outer);
                return -1;
            }
        }
    }
    MDP_CUDA_TRY(cudaSetDevice(h->device));
    const int n = h->natoms;
    const size_t bytes = sizeof(double) * 10 * (size_t)n;
    double *buf = nullptr;
    MDP_CUDA_TRY(cudaMalloc(&buf, bytes));
    k_fit_zbl<<<(n + 127) / 128, 128, 0, h->s>>>(h->x.as<double4>(), h->cfg.as<int>(), h->ca0.as<int>(),
                                                 h->cn.as<int>(), h->cbox.as<double4>(), n, zp, buf, buf + n,
                                                 buf + 4 * (size_t)n);
    count_launches(1);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(eatom, buf, sizeof(double) * n, cudaMemcpyDeviceToHost, h->s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(fatom, buf + n, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, h->s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(vatom, buf + 4 * (size_t)n, sizeof(double) * 6 * (size_t)n, cudaMemcpyDeviceToHost,
                              h->s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(h->s);
    cudaFree(buf);
    if (err != cudaSuccess) { set_error("mdp_fit_zbl: %s", cudaGetErrorString(err)); return -1; }
    return 0;
}

long long mdp_fit_npairs(mdp_fit *h) { return h ? h->npairs : -1; }

int mdp_fit_set_chunk_bytes(mdp_fit *h, double bytes)
{
    if (!h || !(bytes > 0)) { set_error("bad arguments"); return -1; }
    h->chunk_bytes = bytes;
    fit_drop_graph(h);
    if (h->pairs_ready) return fit_alloc_work(h);
    return 0;
}

int mdp_fit_nchunks(mdp_fit *h) { return h ? (int)h->chunks.size() : -1; }

// Descriptors of the batch (any output may be NULL):
//   bi [nconf][ncoeff], bd [natoms][3][ncoeff] (= -d(sum B)/dx, the layout
//   order of cpuSnapTallyBispectrumDeriv per atom), bv [nconf][ncoeff][6],
//   blist [ncoeff][natoms]
int mdp_fit_descriptors(mdp_fit *h, double *bi, double *bd, double *bv, double *blist)
{
    if (!h || !h->pairs_ready) { set_error("set a batch first"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(h->device));
    const int n = h->natoms, nc = h->tab.ntri;
    DevBuf dbi, dbv, dG;
    if (dbi.ensure(sizeof(double) * h->nconf * nc) || dbv.ensure(sizeof(double) * h->nconf * nc * 6) ||
        dG.ensure(sizeof(double) * (size_t)n * 3 * nc))
        return -1;
    if (fit_descriptor_stages(h, false, dG.as<double>(), dbi.as<double>(), dbv.as<double>())) return -1;
    MDP_CUDA_TRY(cudaStreamSynchronize(h->s));
    if (bi) MDP_CUDA_TRY(cudaMemcpy(bi, dbi.p, sizeof(double) * h->nconf * nc, cudaMemcpyDeviceToHost));
    if (bv) MDP_CUDA_TRY(cudaMemcpy(bv, dbv.p, sizeof(double) * h->nconf * nc * 6, cudaMemcpyDeviceToHost));
    if (bd) {
        std::vector<double> g((size_t)n * 3 * nc);
        MDP_CUDA_TRY(cudaMemcpy(g.data(), dG.p, sizeof(double) * g.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < g.size(); i++) bd[i] = -g[i];
    }
    if (blist) MDP_CUDA_TRY(cudaMemcpy(blist, h->B.p, sizeof(double) * (size_t)nc * n, cudaMemcpyDeviceToHost));
    dbi.release(); dbv.release(); dG.release();
    return 0;
}

// Normal equations of the batch: A [64][64] and b [64] (entries beyond
// 1 + ncoeff are zero), assembled in FP64 (mode 0) or from the BF16 hi/lo
// split with FP32 sums (mode 1).  The whole pipeline, from U to A, is one CUDA
// graph, captured on first use per mode and replayed; elapsed_ms (may be NULL)
// is the CUDA-event time of the graph launch.
int mdp_fit_run(mdp_fit *h, int mode, double *A, double *b, float *elapsed_ms)
{
    if (!h || !h->pairs_ready) { set_error("set a batch first"); return -1; }
    if (mode != 0 && mode != 1) { set_error("mode must be 0 (FP64) or 1 (BF16 split)"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(h->device));
    if (h->graph_mode != mode) {
        fit_drop_graph(h);
        if (tu_ensure_tables()) return -1;
        // first call of every launcher outside the capture (attributes, tables)
        if (fit_descriptor_stages(h, true) || fit_gram_stages(h, mode)) return -1;
        MDP_CUDA_TRY(cudaStreamSynchronize(h->s));
        MDP_CUDA_TRY(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
        int rc = fit_descriptor_stages(h, true) || fit_gram_stages(h, mode);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(h->s, &g);
        if (rc || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (!rc) set_error("graph capture failed: %s", cudaGetErrorString(ce));
            return -1;
        }
        h->graph = g;
        MDP_CUDA_TRY(cudaGraphInstantiate(&h->gexec, g, 0));
        h->graph_mode = mode;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, h->s);
    MDP_CUDA_TRY(cudaGraphLaunch(h->gexec, h->s));
    cudaEventRecord(e1, h->s);
    MDP_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (elapsed_ms) *elapsed_ms = ms;
    std::vector<double> o(FIT_KP * FIT_KP + 2 * FIT_KP);
    MDP_CUDA_TRY(cudaMemcpy(o.data(), h->out.p, sizeof(double) * o.size(), cudaMemcpyDeviceToHost));
    if (mode == 1) {
        // undo the column equilibration: A = D^-1 A' D^-1, b = D^-1 b'
        const double *q = o.data() + FIT_KP * FIT_KP + FIT_KP;
        double d[FIT_KP];
        for (int k = 0; k < FIT_KP; k++) d[k] = q[k] > 0.0 ? sqrt(q[k]) : 0.0;
        for (int k = 0; k < FIT_KP; k++) {
            for (int l = 0; l < FIT_KP; l++) o[k * FIT_KP + l] *= d[k] * d[l];
            o[FIT_KP * FIT_KP + k] *= d[k];
        }
    }
    if (A) memcpy(A, o.data(), sizeof(double) * FIT_KP * FIT_KP);
    if (b) memcpy(b, o.data() + FIT_KP * FIT_KP, sizeof(double) * FIT_KP);
    return 0;
}

// Autotuner: times the per-pair kernels' block sizes and the Gram kernel's
// rows per CTA on the current batch (CUDA events, best of 3 each) and keeps
// the fastest; the captured graph is rebuilt on the next run.  Writes the
// choice to out3 (du threads, dB/dr threads, Gram rows per CTA) if not NULL.
int mdp_fit_tune(mdp_fit *h, int *out3)
{
    if (!h || !h->pairs_ready) { set_error("set a batch first"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(h->device));
    fit_drop_graph(h);
    if (fit_descriptor_stages(h, true)) return -1;   // warm tables and buffers
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // a candidate that fails to launch is discarded (and its error cleared)
    auto timeit = [&](auto fn) {
        float best = 1e30f;
        for (int r = 0; r < 3; r++) {
            cudaEventRecord(e0, h->s);
            if (fn() || cudaPeekAtLastError() != cudaSuccess) { cudaGetLastError(); return -1.0f; }
            cudaEventRecord(e1, h->s);
            cudaEventSynchronize(e1);
            float ms;
            cudaEventElapsedTime(&ms, e0, e1);
            best = std::min(best, ms);
        }
        return best;
    };
    const int tcand[3] = {32, 64, 128};   // within the kernels' launch bounds (128)
    float bt = 1e30f;
    int bsel = h->du_threads;
    for (int c : tcand) {
        h->du_threads = c;
        const float t = timeit([&]() { return fit_du(h, h->chunks[0]); });
        if (t >= 0 && t < bt) { bt = t; bsel = c; }
    }
    h->du_threads = bsel;
    bt = 1e30f;
    bsel = h->db_threads;
    const int dcand[3] = {FIT_DB_TPA, 2 * FIT_DB_TPA, 4 * FIT_DB_TPA};   // 1, 2, 4 atoms per CTA
    for (int c : dcand) {
        const float t = timeit([&]() { return fit_dbdr(h, h->chunks[0], c); });
        if (t >= 0 && t < bt) { bt = t; bsel = c; }
    }
    h->db_threads = bsel;
    const int rcand[4] = {256, 1024, 4096, 16384};
    bt = 1e30f;
    bsel = h->gram_rows;
    for (int c : rcand) {
        h->gram_rows = c;
        const float t = timeit([&]() { return fit_gram_stages(h, 1); });
        if (t >= 0 && t < bt) { bt = t; bsel = c; }
    }
    h->gram_rows = bsel;
    h->gram_tuned = true;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MDP_CUDA_TRY(cudaGetLastError());
    if (out3) { out3[0] = h->du_threads; out3[1] = h->db_threads; out3[2] = h->gram_rows; }
    return 0;
}

}  // extern "C"
