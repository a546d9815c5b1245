// Periodic images, ghost atoms, cell binning and the full neighbour list on
// the GPU, plus the per-step pair build, the atomic-free force/virial tally
// and the velocity-Verlet kernels.
//
// Reference semantics:
//   box set-up       src/C++/Configuration/Configuration.cpp:790-880,
//                    src/C++/Core/cpuNeighborList3D.cpp:11-229,
//                    src/C++/Core/cpuArrayPermute.cpp:186-217
//   ghosts           src/C++/Core/cpuNeighborList3D.cpp:282-330 (ghost q of atom
//                    i is image k in image order, q = inum + sum_{i'<i} g(i') + k)
//   neighbour list   src/C++/Core/cpuNeighborList3D.cpp:361-441: j != i and
//                    |x_j - x_i|^2 <= (rcut+skin)^2, up to neighmax per atom
//   pairs            src/C++/Core/cpuSnap.cpp:1883-1933: r^2 < rcut^2, r^2 > 1e-20
//   tally            src/C++/Core/cpuSnap4.cpp:1177-1209
//   NVE              src/C++/Core/cpuVelocityIntegration.cpp:307-339
// The distance and image arithmetic uses explicit round-to-nearest multiplies
// and adds (no FMA contraction) in the reference's evaluation order, so the
// neighbour sets are bit-identical to the reference's.  Each neighbour row is
// sorted ascending, which makes the list deterministic.
#include "common.cuh"
#include "engine.h"

#include <math.h>

namespace mdp {

// ---------------------------------------------------------------------------
// host: box set-up
// ---------------------------------------------------------------------------
static void inv3(double *iA, const double *A)
{
    double a11 = A[0], a21 = A[1], a31 = A[2], a12 = A[3], a22 = A[4], a32 = A[5], a13 = A[6], a23 = A[7], a33 = A[8];
    double d = (a11 * a22 * a33 - a11 * a23 * a32 - a12 * a21 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31);
    iA[0] = (a22 * a33 - a23 * a32) / d; iA[1] = (a23 * a31 - a21 * a33) / d; iA[2] = (a21 * a32 - a22 * a31) / d;
    iA[3] = (a13 * a32 - a12 * a33) / d; iA[4] = (a11 * a33 - a13 * a31) / d; iA[5] = (a12 * a31 - a11 * a32) / d;
    iA[6] = (a12 * a23 - a13 * a22) / d; iA[7] = (a13 * a21 - a11 * a23) / d; iA[8] = (a11 * a22 - a12 * a21) / d;
}
static double nrm3(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1]; c[1] = a[2] * b[0] - a[0] * b[2]; c[2] = a[0] * b[1] - a[1] * b[0];
}

int box_setup(BoxParams &bp, const double *a, const double *b, const double *c, double offset, double rc_cells)
{
    double M[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
    inv3(bp.s2r, M);
    // bounding parallelepiped enlarged by `offset` on every periodic side
    double p1[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    double p2[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    double p3[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
    double d1 = -offset * nrm3(p1), d2 = -offset * nrm3(p2), d3 = -offset * nrm3(p3);
    double A[9] = {p1[0], p2[0], p3[0], p1[1], p2[1], p3[1], p1[2], p2[2], p3[2]}, iA[9];
    inv3(iA, A);
    double w[24];
    w[0] = iA[0] * d1 + iA[3] * d2 + iA[6] * d3;
    w[1] = iA[1] * d1 + iA[4] * d2 + iA[7] * d3;
    w[2] = iA[2] * d1 + iA[5] * d2 + iA[8] * d3;
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
    double na = nrm3(a), nb = nrm3(b), nc = nrm3(c);
    double la = na + 2.0 * nrm3(sa), lb = nb + 2.0 * nrm3(sb), lc = nc + 2.0 * nrm3(sc);
    for (int k = 0; k < 3; k++) w[k] = e1 * a[k] + e2 * b[k] + e3 * c[k];
    for (int k = 0; k < 3; k++) {
        w[3 + k] = w[k] + (la / na) * a[k];
        w[9 + k] = w[k] + (lb / nb) * b[k];
        w[6 + k] = -w[k] + w[3 + k] + w[9 + k];
        w[12 + k] = w[k] + (lc / nc) * c[k];
        w[15 + k] = w[12 + k] + (la / na) * a[k];
        w[21 + k] = w[12 + k] + (lb / nb) * b[k];
        w[18 + k] = -w[12 + k] + w[15 + k] + w[21 + k];
    }
    double rbv[24];
    for (int i = 0; i < 8; i++)
        for (int k = 0; k < 3; k++)
            rbv[3 * i + k] = iA[k] * w[3 * i] + iA[3 + k] * w[3 * i + 1] + iA[6 + k] * w[3 * i + 2];
    for (int k = 0; k < 3; k++) { bp.lo[k] = rbv[k]; bp.hi[k] = rbv[18 + k]; }
    // periodic images in the reference's order (cpuNeighborList3D.cpp:136-229)
    static const int ca[27] = {0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 1, -1, 0, 0, 1, 1, -1, -1};
    static const int cb[27] = {0, 0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 0, 1, -1, 1, -1, 1, -1};
    static const int cc[27] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    for (int i = 0; i < 27; i++)
        for (int k = 0; k < 3; k++) {
            double s;
            if (cc[i] != 0) {
                s = cc[i] * c[k];
                if (ca[i] != 0) s = s + ca[i] * a[k];
                else if (cb[i] == 0) s = s + 0.0;
                if (cb[i] != 0) s = s + cb[i] * b[k];
            } else {
                s = 0.0;
                if (ca[i] != 0) s = ca[i] * a[k];
                if (cb[i] != 0) s = (ca[i] != 0) ? s + cb[i] * b[k] : cb[i] * b[k];
            }
            bp.pim[i][k] = s;
        }
    // cell grid over the extended box, in fractional coordinates; each cell's
    // perpendicular width is >= rc_cells so a 27-cell stencil is complete
    double vol = fabs(a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
                      a[2] * (b[0] * c[1] - b[1] * c[0]));
    double cx[3];
    double h[3];
    cross3(b, c, cx); h[0] = vol / nrm3(cx);
    cross3(c, a, cx); h[1] = vol / nrm3(cx);
    cross3(a, b, cx); h[2] = vol / nrm3(cx);
    long ncell = 1;
    for (int k = 0; k < 3; k++) {
        double ext = (bp.hi[k] - bp.lo[k]) * h[k];
        int n = (int)floor(ext / rc_cells);
        if (n < 1) n = 1;
        if (n > 1024) n = 1024;
        bp.nc[k] = n;
        bp.cinv[k] = n / (bp.hi[k] - bp.lo[k]);
        ncell *= n;
    }
    bp.ncell = ncell;
    return 0;
}

// ---------------------------------------------------------------------------
// ghosts
// ---------------------------------------------------------------------------
__device__ __forceinline__ void frac3(const BoxParams &bp, double x0, double x1, double x2, double *s)
{
    // s = s2r * x, evaluated ((m0*x0 + m3*x1) + m6*x2) without contraction
    s[0] = __dadd_rn(__dadd_rn(__dmul_rn(bp.s2r[0], x0), __dmul_rn(bp.s2r[3], x1)), __dmul_rn(bp.s2r[6], x2));
    s[1] = __dadd_rn(__dadd_rn(__dmul_rn(bp.s2r[1], x0), __dmul_rn(bp.s2r[4], x1)), __dmul_rn(bp.s2r[7], x2));
    s[2] = __dadd_rn(__dadd_rn(__dmul_rn(bp.s2r[2], x0), __dmul_rn(bp.s2r[5], x1)), __dmul_rn(bp.s2r[8], x2));
}

__global__ void k_ghost_count(const double4 *__restrict__ x, int n, const __grid_constant__ BoxParams bp,
                              int *__restrict__ gcount, unsigned *__restrict__ gmask)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 xi = x[i];
    unsigned m = 0;
    int cnt = 0;
    for (int k = 1; k < 27; k++) {
        const double y0 = __dadd_rn(xi.x, bp.pim[k][0]);
        const double y1 = __dadd_rn(xi.y, bp.pim[k][1]);
        const double y2 = __dadd_rn(xi.z, bp.pim[k][2]);
        double s[3];
        frac3(bp, y0, y1, y2, s);
        if (bp.lo[0] <= s[0] && s[0] <= bp.hi[0] && bp.lo[1] <= s[1] && s[1] <= bp.hi[1] && bp.lo[2] <= s[2] &&
            s[2] <= bp.hi[2]) {
            m |= 1u << k;
            cnt++;
        }
    }
    gcount[i] = cnt;
    gmask[i] = m;
}

__global__ void k_ghost_emit(double4 *__restrict__ x, int *__restrict__ alist, int n, const __grid_constant__ BoxParams bp,
                             const int *__restrict__ goff, const unsigned *__restrict__ gmask)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    alist[i] = i;
    const double4 xi = x[i];
    unsigned m = gmask[i];
    int q = n + goff[i];
    for (int k = 1; k < 27; k++) {
        if (m & (1u << k)) {
            x[q] = make_double4(__dadd_rn(xi.x, bp.pim[k][0]), __dadd_rn(xi.y, bp.pim[k][1]),
                                __dadd_rn(xi.z, bp.pim[k][2]), 0.0);
            alist[q] = i;
            q++;
        }
    }
}

// ---------------------------------------------------------------------------
// cells
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_coord(const BoxParams &bp, int d, double s)
{
    int c = (int)floor((s - bp.lo[d]) * bp.cinv[d]);
    return c < 0 ? 0 : (c >= bp.nc[d] ? bp.nc[d] - 1 : c);
}

__global__ void k_cell_index(const double4 *__restrict__ x, int anum, const __grid_constant__ BoxParams bp,
                             int *__restrict__ cidx, int *__restrict__ ccount)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= anum) return;
    const double4 xi = x[i];
    double s[3];
    frac3(bp, xi.x, xi.y, xi.z, s);
    int c = cell_coord(bp, 0, s[0]) + bp.nc[0] * (cell_coord(bp, 1, s[1]) + bp.nc[1] * cell_coord(bp, 2, s[2]));
    cidx[i] = c;
    atomicAdd(&ccount[c], 1);
}

__global__ void k_cell_fill(int anum, const int *__restrict__ cidx, const int *__restrict__ cstart,
                            int *__restrict__ cursor, int *__restrict__ catoms)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= anum) return;
    int c = cidx[i];
    catoms[cstart[c] + atomicAdd(&cursor[c], 1)] = i;
}

// one thread per local atom; row sorted ascending; overflow -> status bit 1
__global__ void k_neigh_build(const double4 *__restrict__ x, int inum, const __grid_constant__ BoxParams bp,
                              const int *__restrict__ cidx, const int *__restrict__ cstart,
                              const int *__restrict__ catoms, double rcsq, int nm,
                              int *__restrict__ nlist, int *__restrict__ nnum, int *__restrict__ status)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    const double4 xi = x[i];
    const int c = cidx[i];
    const int c0 = c % bp.nc[0], c1 = (c / bp.nc[0]) % bp.nc[1], c2 = c / (bp.nc[0] * bp.nc[1]);
    int *row = nlist + (size_t)i * nm;
    int cnt = 0;
    for (int d2 = -1; d2 <= 1; d2++) {
        const int k2 = c2 + d2;
        if (k2 < 0 || k2 >= bp.nc[2]) continue;
        for (int d1 = -1; d1 <= 1; d1++) {
            const int k1 = c1 + d1;
            if (k1 < 0 || k1 >= bp.nc[1]) continue;
            for (int d0 = -1; d0 <= 1; d0++) {
                const int k0 = c0 + d0;
                if (k0 < 0 || k0 >= bp.nc[0]) continue;
                const int cc = k0 + bp.nc[0] * (k1 + bp.nc[1] * k2);
                const int s = cstart[cc], e = cstart[cc + 1];
                for (int t = s; t < e; t++) {
                    const int j = catoms[t];
                    if (j == i) continue;
                    const double4 xj = x[j];
                    const double d0x = __dsub_rn(xj.x, xi.x), d1x = __dsub_rn(xj.y, xi.y), d2x = __dsub_rn(xj.z, xi.z);
                    const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(d0x, d0x), __dmul_rn(d1x, d1x)), __dmul_rn(d2x, d2x));
                    if (rsq <= rcsq) {
                        if (cnt < nm) row[cnt] = j;
                        cnt++;
                    }
                }
            }
        }
    }
    if (cnt > nm) {
        atomicOr(status, 1);
        cnt = nm;
    }
    // insertion sort of the row
    for (int a = 1; a < cnt; a++) {
        int v = row[a], b = a - 1;
        while (b >= 0 && row[b] > v) { row[b + 1] = row[b]; b--; }
        row[b + 1] = v;
    }
    nnum[i] = cnt;
}

// reverse index: for each owner o, the (i, slot) entries whose neighbour is
// an image of o; used to gather -dE onto owners without atomics
__global__ void k_rev_count(const int *__restrict__ nlist, const int *__restrict__ nnum, const int *__restrict__ alist,
                            int inum, int nm, int *__restrict__ rcount)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    const int n = nnum[i];
    for (int l = 0; l < n; l++) atomicAdd(&rcount[alist[nlist[(size_t)i * nm + l]]], 1);
}

__global__ void k_rev_fill(const int *__restrict__ nlist, const int *__restrict__ nnum, const int *__restrict__ alist,
                           int inum, int nm, const int *__restrict__ roff, int *__restrict__ cursor,
                           long long *__restrict__ rlist)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    const int n = nnum[i];
    for (int l = 0; l < n; l++) {
        const int o = alist[nlist[(size_t)i * nm + l]];
        rlist[roff[o] + atomicAdd(&cursor[o], 1)] = (long long)i * nm + l;
    }
}

// Each owner's reverse entries ascending, so the tally sums in a fixed order.
// One warp per owner: the entries go to shared memory, padded to a power of
// two with the largest key, and a bitonic network sorts them (lists longer
// than REV_SORT_MAX fall back to an insertion sort in place).
constexpr int REV_SORT_WARPS = 8, REV_SORT_MAX = 256;

__global__ void __launch_bounds__(REV_SORT_WARPS * 32)
k_rev_sort(int inum, const int *__restrict__ roff, long long *__restrict__ rlist)
{
    __shared__ long long keys[REV_SORT_WARPS][REV_SORT_MAX];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long *kw = keys[w];
    for (int o = blockIdx.x * REV_SORT_WARPS + w; o < inum; o += gridDim.x * REV_SORT_WARPS) {
        const int s = roff[o], e = roff[o + 1], n = e - s;
        if (n <= 1) continue;
        if (n > REV_SORT_MAX) {
            if (lane == 0)
                for (int a = s + 1; a < e; a++) {
                    const long long v = rlist[a];
                    int b = a - 1;
                    while (b >= s && rlist[b] > v) { rlist[b + 1] = rlist[b]; b--; }
                    rlist[b + 1] = v;
                }
            __syncwarp();
            continue;
        }
        int P = 2;
        while (P < n) P <<= 1;
        for (int i = lane; i < P; i += 32) kw[i] = (i < n) ? rlist[s + i] : 0x7fffffffffffffffLL;
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    const int l = i ^ j;
                    if (l > i) {
                        const long long a = kw[i], b = kw[l];
                        const bool up = (i & k) == 0;
                        if ((a > b) == up) { kw[i] = b; kw[l] = a; }
                    }
                }
                __syncwarp();
            }
        for (int i = lane; i < n; i += 32) rlist[s + i] = kw[i];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// per-step pairs
// ---------------------------------------------------------------------------
// the pair test of slot l of atom i: r < rcut and r > 0 (cpuSnap.cpp:1883-1906),
// with r^2 rounded in the CPU code's order
__device__ __forceinline__ bool slot_pair(const double4 &xi, const double4 &xj, double rcutsq, double &d0,
                                          double &d1, double &d2)
{
    d0 = xj.x - xi.x;
    d1 = xj.y - xi.y;
    d2 = xj.z - xi.z;
    const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
    return rsq < rcutsq && rsq > 1e-20;
}

// One warp per atom: the lanes test 32 of the atom's slots at a time, and a
// ballot ranks each lane's pair among the atom's pairs in slot order.
__global__ void k_pair_count(const double4 *__restrict__ x, const int *__restrict__ nlist,
                             const int *__restrict__ nnum, int inum, int nm, double rcutsq, int *__restrict__ pcount)
{
    const int lane = threadIdx.x & 31;
    const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= inum) return;   // whole warps leave together
    const double4 xi = x[i];
    const int n = nnum[i];
    int cnt = 0;
    for (int l0 = 0; l0 < n; l0 += 32) {
        const int l = l0 + lane;
        bool pair = false;
        if (l < n) {
            double d0, d1, d2;
            pair = slot_pair(xi, x[nlist[(size_t)i * nm + l]], rcutsq, d0, d1, d2);
        }
        cnt += __popc(__ballot_sync(0xffffffffu, pair));
    }
    if (lane == 0) pcount[i] = cnt;
}

// compact pair list of the atoms' slots in order: r and sfac in prij, the
// Cayley-Klein parameters (a, b) in pab, (atom, pair) in pinfo; smap maps
// every slot to its pair (-1 for slots beyond rcut).  One warp per atom.
__global__ void k_pair_emit(const double4 *__restrict__ x, const int *__restrict__ nlist,
                            const int *__restrict__ nnum, int inum, int nm, const int *__restrict__ poff, SnapGeom gp,
                            double4 *__restrict__ prij, int2 *__restrict__ pinfo, double4 *__restrict__ pab,
                            int *__restrict__ smap)
{
    const int lane = threadIdx.x & 31;
    const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= inum) return;   // whole warps leave together
    const double4 xi = x[i];
    const int n = nnum[i];
    int p = poff[i];
    for (int l0 = 0; l0 < n; l0 += 32) {
        const int l = l0 + lane;
        const size_t s = (size_t)i * nm + l;
        bool pair = false;
        double d0 = 0.0, d1 = 0.0, d2 = 0.0;
        if (l < n) pair = slot_pair(xi, x[nlist[s]], gp.rcutsq, d0, d1, d2);
        const unsigned m = __ballot_sync(0xffffffffu, pair);
        if (l < n) {
            if (pair) {
                const int q = p + __popc(m & ((1u << lane) - 1u));
                PairGeo g;
                pair_geometry<false>(g, d0, d1, d2, gp);
                prij[q] = make_double4(d0, d1, d2, g.sfac);
                pab[q] = make_double4(g.ar, g.ai, g.br, g.bi);
                pinfo[q] = make_int2((int)i, q);
                smap[s] = q;
            } else {
                smap[s] = -1;
            }
        }
        p += __popc(m);
    }
}

// Several element types (types 1..nelements, elem = type - 1 per owner atom):
// a slot is a pair when |r|^2 < ((radelem_i + radelem_j) rcutfac)^2 and
// > 1e-20 (cpuNeighPairList, cpuSnap.cpp:1883-1905, with InitSnap's type-pair
// cutoffs).  Pairs are grouped per (element block b, atom): with chemflag the
// block of the neighbour's element, else one block; counts go to
// pcount[b * ipad + atom] (callers zero the pad entries).  One warp per atom.
__global__ void k_pair_count_me(const double4 *__restrict__ x, const int *__restrict__ nlist,
                                const int *__restrict__ nnum, int inum, int nm, const int *__restrict__ alist,
                                const int *__restrict__ elem, const __grid_constant__ ElemGeom eg,
                                int *__restrict__ pcount)
{
    const int lane = threadIdx.x & 31;
    const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= inum) return;   // whole warps leave together
    const double4 xi = x[i];
    const int ei = elem[i];
    const int n = nnum[i];
    int cnt[MAXELEM] = {0, 0, 0, 0};
    for (int l0 = 0; l0 < n; l0 += 32) {
        const int l = l0 + lane;
        bool pair = false;
        int b = 0;
        if (l < n) {
            const int j = nlist[(size_t)i * nm + l];
            const int ej = elem[alist[j]];
            double d0, d1, d2;
            pair = slot_pair(xi, x[j], eg.rcutsq[ei][ej], d0, d1, d2);
            b = eg.chem ? ej : 0;
        }
#pragma unroll
        for (int e = 0; e < MAXELEM; e++) cnt[e] += __popc(__ballot_sync(0xffffffffu, pair && b == e));
    }
    if (lane < eg.nblk) {
        int c = cnt[0];
#pragma unroll
        for (int e = 1; e < MAXELEM; e++)
            if (lane == e) c = cnt[e];
        pcount[(long)lane * eg.ipad + i] = c;
    }
}

// compact pairs per (block, atom) in slot order: r and sfac wjelem[tj] in
// prij, (a, b) in pab, (virtual atom b * ipad + i, pair) in pinfo, the pair's
// cutoff and neighbour weight in pcw, slot -> pair in smap
__global__ void k_pair_emit_me(const double4 *__restrict__ x, const int *__restrict__ nlist,
                               const int *__restrict__ nnum, int inum, int nm, const int *__restrict__ alist,
                               const int *__restrict__ elem, const int *__restrict__ poff, SnapGeom gp,
                               const __grid_constant__ ElemGeom eg, double4 *__restrict__ prij,
                               int2 *__restrict__ pinfo, double4 *__restrict__ pab, double2 *__restrict__ pcw,
                               int *__restrict__ smap)
{
    const int lane = threadIdx.x & 31;
    const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= inum) return;   // whole warps leave together
    const double4 xi = x[i];
    const int ei = elem[i];
    const int n = nnum[i];
    int base[MAXELEM];
#pragma unroll
    for (int e = 0; e < MAXELEM; e++) base[e] = (e < eg.nblk) ? poff[(long)e * eg.ipad + i] : 0;
    for (int l0 = 0; l0 < n; l0 += 32) {
        const int l = l0 + lane;
        const size_t s = (size_t)i * nm + l;
        bool pair = false;
        int b = 0, ej = 0;
        double d0 = 0.0, d1 = 0.0, d2 = 0.0;
        if (l < n) {
            const int j = nlist[s];
            ej = elem[alist[j]];
            pair = slot_pair(xi, x[j], eg.rcutsq[ei][ej], d0, d1, d2);
            b = eg.chem ? ej : 0;
        }
        int q = 0;
#pragma unroll
        for (int e = 0; e < MAXELEM; e++) {
            const unsigned m = __ballot_sync(0xffffffffu, pair && b == e);
            if (b == e) q = base[e] + __popc(m & ((1u << lane) - 1u));
            base[e] += __popc(m);
        }
        if (l < n) {
            if (pair) {
                SnapGeom ge = gp;
                ge.rcut = eg.rcut[ei][ej];
                ge.wj = eg.wj[ej];
                PairGeo g;
                pair_geometry<false>(g, d0, d1, d2, ge);
                prij[q] = make_double4(d0, d1, d2, g.sfac);
                pab[q] = make_double4(g.ar, g.ai, g.br, g.bi);
                pinfo[q] = make_int2((int)((long)b * eg.ipad + i), q);
                pcw[q] = make_double2(ge.rcut, ge.wj);
                smap[s] = q;
            } else {
                smap[s] = -1;
            }
        }
    }
}

// f_o = sum_{own pairs} dE - sum_{pairs whose neighbour is an image of o} dE;
// per-atom virial -1/2 r (x) dE on both atoms (cpuSnap4.cpp:1177-1209).  Own
// pairs in slot order (with several element blocks: block by block, the pairs
// of atom o in block b at poff[b * ipad + o]), then the reverse entries in
// ascending slot order: a fixed summation order without atomics.
__global__ void k_tally(const double4 *__restrict__ prij, const double4 *__restrict__ dE,
                        const int *__restrict__ poff, const int *__restrict__ smap, int inum,
                        const int *__restrict__ roff, const long long *__restrict__ rlist, double4 *__restrict__ f,
                        double *__restrict__ vatom, int nblk, int ipad)
{
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= inum) return;
    double fx = 0, fy = 0, fz = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
    for (int b = 0; b < nblk; b++) {
        const long v = (long)b * ipad + o;
        for (int p = poff[v]; p < poff[v + 1]; p++) {
            const double4 r = prij[p], d = dE[p];
            fx += d.x; fy += d.y; fz += d.z;
            v0 += -0.5 * r.x * d.x; v1 += -0.5 * r.y * d.y; v2 += -0.5 * r.z * d.z;
            v3 += -0.5 * r.x * d.y; v4 += -0.5 * r.x * d.z; v5 += -0.5 * r.y * d.z;
        }
    }
    const int s0 = roff[o], s1 = roff[o + 1];
    for (int t = s0; t < s1; t++) {
        const int p = smap[rlist[t]];
        if (p < 0) continue;
        const double4 r = prij[p], d = dE[p];
        fx -= d.x; fy -= d.y; fz -= d.z;
        v0 += -0.5 * r.x * d.x; v1 += -0.5 * r.y * d.y; v2 += -0.5 * r.z * d.z;
        v3 += -0.5 * r.x * d.y; v4 += -0.5 * r.x * d.z; v5 += -0.5 * r.y * d.z;
    }
    f[o] = make_double4(fx, fy, fz, 0.0);
    if (vatom) {
        vatom[0 * (size_t)inum + o] = v0; vatom[1 * (size_t)inum + o] = v1; vatom[2 * (size_t)inum + o] = v2;
        vatom[3 * (size_t)inum + o] = v3; vatom[4 * (size_t)inum + o] = v4; vatom[5 * (size_t)inum + o] = v5;
    }
}

// ZBL pair term over each atom's full neighbour row (cpuPotentials.cpp:1587-1650
// with the potential of ZBLpotential.jl): pairs with |x_ij|^2 <= rcut^2 add
// u/2 to the atom's energy, du/dx_ij to its force and -x_ij (x) du/dx_ij / 2 to
// its virial, on top of what SNAP wrote.  Thread per atom, no atomics.
__global__ void k_zbl(const double4 *__restrict__ x, const int *__restrict__ nlist, const int *__restrict__ nnum,
                      int inum, int nm, ZblParams zp, double *__restrict__ eatom, double4 *__restrict__ f,
                      double *__restrict__ vatom)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    const double4 xi = x[i];
    const int n = nnum[i];
    double e = 0.0, fx = 0.0, fy = 0.0, fz = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
    for (int l = 0; l < n; l++) {
        const double4 xj = x[nlist[(size_t)i * nm + l]];
        const double d0 = xj.x - xi.x, d1 = xj.y - xi.y, d2 = xj.z - xi.z;
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
        if (!(r2 <= zp.rcsq)) continue;
        double u, g;
        zbl_pair(zp, sqrt(r2), u, g);
        const double ux = g * d0, uy = g * d1, uz = g * d2;
        e += 0.5 * u;
        fx += ux; fy += uy; fz += uz;
        v[0] -= 0.5 * d0 * ux; v[1] -= 0.5 * d1 * uy; v[2] -= 0.5 * d2 * uz;
        v[3] -= 0.5 * d0 * uy; v[4] -= 0.5 * d0 * uz; v[5] -= 0.5 * d1 * uz;
    }
    eatom[i] += e;
    const double4 fo = f[i];
    f[i] = make_double4(fo.x + fx, fo.y + fy, fo.z + fz, 0.0);
    if (vatom)
        for (int k = 0; k < 6; k++) vatom[k * (size_t)inum + i] += v[k];
}

// ---------------------------------------------------------------------------
// integrator, PBC, rebuild check, ghost shift, thermo sums
// ---------------------------------------------------------------------------
__global__ void k_nve_initial(double4 *__restrict__ x, double4 *__restrict__ v, const double4 *__restrict__ f,
                              double4 *__restrict__ xstart, int n, double dtfm, double dtv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 xi = x[i], vi = v[i];
    const double4 fi = f[i];
    xstart[i] = xi;
    vi.x += dtfm * fi.x; vi.y += dtfm * fi.y; vi.z += dtfm * fi.z;
    xi.x += dtv * vi.x; xi.y += dtv * vi.y; xi.z += dtv * vi.z;
    x[i] = xi; v[i] = vi;
}

__global__ void k_nve_final(double4 *__restrict__ v, const double4 *__restrict__ f, int n, double dtfm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 vi = v[i];
    const double4 fi = f[i];
    vi.x += dtfm * fi.x; vi.y += dtfm * fi.y; vi.z += dtfm * fi.z;
    v[i] = vi;
}

// max over atoms of |x - xhold|^2, as the bit pattern of a non-negative double
__global__ void k_maxdisp(const double4 *__restrict__ x, const double4 *__restrict__ xh, int n,
                          unsigned long long *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (i < n) {
        const double4 a = x[i], b = xh[i];
        const double d0 = a.x - b.x, d1 = a.y - b.y, d2 = a.z - b.z;
        m = d0 * d0 + d1 * d1 + d2 * d2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// orthogonal-box wrap (cpuDomain.cpp:235-300, PBC on all axes)
__global__ void k_pbc_orth(double4 *__restrict__ x, int n, double lo0, double lo1, double lo2, double hi0, double hi1,
                           double hi2)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 a = x[i];
    const double L0 = hi0 - lo0, L1 = hi1 - lo1, L2 = hi2 - lo2;
    if (a.x < lo0) a.x += L0;
    if (a.x >= hi0) { a.x -= L0; a.x = fmax(a.x, lo0); }
    if (a.y < lo1) a.y += L1;
    if (a.y >= hi1) { a.y -= L1; a.y = fmax(a.y, lo1); }
    if (a.z < lo2) a.z += L2;
    if (a.z >= hi2) { a.z -= L2; a.z = fmax(a.z, lo2); }
    x[i] = a;
}

__global__ void k_ghost_shift(double4 *__restrict__ x, const double4 *__restrict__ xstart, const int *__restrict__ alist,
                              int inum, int gnum)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= gnum) return;
    const int q = inum + g, o = alist[q];
    const double4 a = x[o], b = xstart[o];
    double4 xg = x[q];
    xg.x += a.x - b.x; xg.y += a.y - b.y; xg.z += a.z - b.z;
    x[q] = xg;
}

// block sums of e, virial diagonal and m v^2 into out[4] (double atomics on 4 words)
__global__ void k_thermo(const double *__restrict__ e, const double *__restrict__ vatom, const double4 *__restrict__ v,
                         int n, double *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s[5] = {0, 0, 0, 0, 0};
    if (i < n) {
        s[0] = e[i];
        s[1] = vatom[i]; s[2] = vatom[(size_t)n + i]; s[3] = vatom[2 * (size_t)n + i];
        const double4 vi = v[i];
        s[4] = vi.x * vi.x + vi.y * vi.y + vi.z * vi.z;
    }
#pragma unroll
    for (int k = 0; k < 5; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 5; k++) atomicAdd(&out[k], s[k]);
}

}  // namespace mdp
