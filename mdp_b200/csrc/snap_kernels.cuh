// SNAP force-path kernels for sm_100a, templated on the arithmetic type T
// (double: plain path; float: reduced-precision form) and on 2J (TJ).
//
// Stages (reference functions in src/C++/Core/cpuSnap4.cpp):
//   k_snap_ui   U_i = sum_j sfac(r_ij) U(r_ij) + wself, mirrored   (:11-244)
//               one warp per atom, lanes over its pairs, per-row
//               shared-memory transpose to sum the lanes
//   k_snap_yi   Y_i = sum_{j1 j2} beta' Z_{j1 j2 j}(U_i)  and
//               E_i = beta0 + 2/3 sum_half w Re(U* Y)        (:250-421, :697-792)
//               tiles of 32 atoms (lane = atom), U tile resident in shared
//               memory, every (j1,j2,j) row of Z specialised at compile time
//               so CG coefficients are constant-bank operands and the U rows
//               it needs are held in registers
//   k_snap_fi   dE/dr_ij = 2 sum_half w Re(Y* dU/dr)         (:798-1175)
//               one thread per pair, forward-mode dU recursion
#pragma once

#include "common.cuh"

namespace mdp {

struct SnapGeom {
    double rcut, rcutsq, rfac0, rmin0, wj;
    int switchflag;
};

// Y-kernel parameters.  Lanes are the 32 atoms of a tile.  Output layers j are
// processed one after another by the whole CTA; within a layer every warp walks
// the same sequence of (j1, j2) couplings, so the code in flight is one
// coupling's few kilobytes and stays in the instruction cache.  Each warp owns
// one output row mb of the layer and a residue class of the row-pair index ib,
// accumulates its share of that row in registers across all couplings, and the
// warps' partial rows are summed once per layer through shared memory.
constexpr int YI_MAXW = 16;
template <typename T>
struct YParams {
    T betaY[NTRI];          // beta' of each coupling triple (bnorm 1/(j+1) folded in)
    double e0;              // beta0 - sum_k beta_k bzero_k
    // per output layer j and warp w: the row mb the warp accumulates (255: idle)
    // and the residue / stride of the row-pair index ib it takes in every coupling
    unsigned char lay_mb[JD][YI_MAXW], lay_o[JD][YI_MAXW], lay_st[JD][YI_MAXW];
};
template <typename T> struct YiWarps { static constexpr int n = 8; };
template <> struct YiWarps<float> { static constexpr int n = 16; };

__host__ __device__ constexpr bool coupling_ok(int j1, int j2, int j)
{
    return j2 <= j1 && j1 - j2 <= j && j <= j1 + j2 && ((j1 + j2 + j) % 2 == 0);
}

// ---------------------------------------------------------------------------
// pair geometry (cpuSnap4.cpp:15-53, 803-874), evaluated in double
// ---------------------------------------------------------------------------
struct PairGeo {
    double ar, ai, br, bi, sfac, dsfac, u[3];
    double dar[3], dai[3], dbr[3], dbi[3];
};

template <bool DERIV>
__device__ __forceinline__ void pair_geometry(PairGeo &g, double x, double y, double z, const SnapGeom &p)
{
    const double rsq = x * x + y * y + z * z;
    const double r = sqrt(rsq);
    const double tscale = p.rfac0 * M_PI / (p.rcut - p.rmin0);
    const double z0 = r / tan((r - p.rmin0) * tscale);
    double sfac = 1.0, dsfac = 0.0;
    if (p.switchflag == 1 && r > p.rmin0 && r <= p.rcut) {
        const double rf = M_PI / (p.rcut - p.rmin0);
        sfac = 0.5 * (cos((r - p.rmin0) * rf) + 1.0);
        if (DERIV) dsfac = -0.5 * sin((r - p.rmin0) * rf) * rf;
    }
    g.sfac = sfac * p.wj;
    g.dsfac = dsfac * p.wj;
    const double r0inv = 1.0 / sqrt(r * r + z0 * z0);
    g.ar = r0inv * z0;
    g.ai = -r0inv * z;
    g.br = r0inv * y;
    g.bi = -r0inv * x;
    if (DERIV) {
        const double rinv = 1.0 / r;
        g.u[0] = x * rinv; g.u[1] = y * rinv; g.u[2] = z * rinv;
        const double dz0dr = z0 / r - (r * tscale) * (rsq + z0 * z0) / rsq;
        const double dr0inv = -(r0inv * r0inv * r0inv) * (r + z0 * dz0dr);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double d = dr0inv * g.u[k];
            g.dar[k] = dz0dr * g.u[k] * r0inv + z0 * d;
            g.dai[k] = -z * d;
            g.dbr[k] = y * d;
            g.dbi[k] = -x * d;
        }
        g.dai[2] += -r0inv;
        g.dbi[0] += -r0inv;
        g.dbr[1] += r0inv;
    }
}

// ---------------------------------------------------------------------------
// U rows of one pair: for mb = 0..TJ/2, layers j = max(1, 2mb)..TJ.
// emit(j, mb, pr, pi) is called once per computed row (values of layer j, row
// mb, entries ma = 0..j).  All loops unroll; the arrays live in registers.
// ---------------------------------------------------------------------------
template <typename T, int TJ, typename Emit>
__device__ __forceinline__ void u_rows(const T ar, const T ai, const T br, const T bi, Emit &emit)
{
    T pr[TJ + 1], pi[TJ + 1], qr[TJ + 1], qi[TJ + 1];
#pragma unroll
    for (int mb = 0; 2 * mb <= TJ; mb++) {
        if (mb == 0) {
            pr[0] = T(1); pi[0] = T(0);
        } else {
#pragma unroll
            for (int ma = 0; ma < 2 * mb; ma++) { pr[ma] = qr[ma]; pi[ma] = qi[ma]; }
        }
#pragma unroll
        for (int j = (mb == 0 ? 1 : 2 * mb); j <= TJ; j++) {
            {
                const T rp = rootpq<T>(j, j - mb);
                const T nr = -rp * (br * pr[j - 1] + bi * pi[j - 1]);
                const T ni = -rp * (br * pi[j - 1] - bi * pr[j - 1]);
                pr[j] = nr; pi[j] = ni;
            }
#pragma unroll
            for (int ma = j - 1; ma >= 1; ma--) {
                const T rpa = rootpq<T>(j - ma, j - mb), rpb = rootpq<T>(ma, j - mb);
                const T nr = rpa * (ar * pr[ma] + ai * pi[ma]) - rpb * (br * pr[ma - 1] + bi * pi[ma - 1]);
                const T ni = rpa * (ar * pi[ma] - ai * pr[ma]) - rpb * (br * pi[ma - 1] - bi * pr[ma - 1]);
                pr[ma] = nr; pi[ma] = ni;
            }
            {
                const T rpa = rootpq<T>(j, j - mb);
                const T nr = rpa * (ar * pr[0] + ai * pi[0]);
                const T ni = rpa * (ar * pi[0] - ai * pr[0]);
                pr[0] = nr; pi[0] = ni;
            }
            if (mb > 0 && j == 2 * mb) {
                // middle row: right half from the left by inversion symmetry
                // (the centre's imaginary part is negated, cpuSnap4.cpp:147-160)
#pragma unroll
                for (int ma = 0; ma <= mb; ma++) {
                    const T s = (ma & 1) ? T(-1) : T(1);
                    pr[mb + ma] = s * pr[mb - ma];
                    pi[mb + ma] = -s * pi[mb - ma];
                }
            }
            if (j == 2 * mb + 1) {
#pragma unroll
                for (int ma = 0; ma <= j; ma++) {
                    const T s = ((mb + ma) & 1) ? T(-1) : T(1);
                    qr[j - ma] = s * pr[ma];
                    qi[j - ma] = -s * pi[ma];
                }
            }
            emit(j, mb, pr, pi);
        }
    }
}

// ---------------------------------------------------------------------------
// k_snap_ui: warp per atom.  Output U in 32-atom tiles: Ut[tile][k][lane],
// k = idxu index (full plane, wself added and mirrored).
// ---------------------------------------------------------------------------
constexpr int UI_WARPS = 4;

// REF = true: no wself/mirror; the computed rows are added into the reference's
// layout Ur/Ui[k * natoms + atom] (cpuSnapComputeUi semantics, cpuSnap4.cpp:11-187)
template <typename T, int TJ, bool REF = false>
__global__ void __launch_bounds__(UI_WARPS * 32)
k_snap_ui(const int *__restrict__ poff, const double4 *__restrict__ prij, int natoms, SnapGeom gp,
          typename cplx<T>::type *__restrict__ Ut, double *__restrict__ Uref_r = nullptr,
          double *__restrict__ Uref_i = nullptr)
{
    typedef typename cplx<T>::type T2;
    constexpr int NU = idxu_count(TJ);
    constexpr int SROW = TJ + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T2 *acc = reinterpret_cast<T2 *>(smraw) + wib * (NU + 32 * SROW);
    T2 *stage = acc + NU;
    const int nwarps = gridDim.x * UI_WARPS;
    for (int i = blockIdx.x * UI_WARPS + wib; i < natoms; i += nwarps) {
        for (int k = lane; k < NU; k += 32) acc[k] = T2{T(0), T(0)};
        __syncwarp();
        const int p0 = poff[i], p1 = poff[i + 1];
        T ssum = T(0);
        for (int base = p0; base < p1; base += 32) {
            const int p = base + lane;
            const bool act = p < p1;
            const int nact = min(32, p1 - base);
            const double4 r = act ? prij[p] : make_double4(1.0, 0.0, 0.0, 0.0);
            PairGeo g;
            pair_geometry<false>(g, r.x, r.y, r.z, gp);
            const T sf = act ? (T)g.sfac : T(0);
            ssum += sf;
            auto emit = [&](int j, int mb, const T *pr, const T *pi) {
#pragma unroll
                for (int ma = 0; ma <= j; ma++) stage[lane * SROW + ma] = T2{sf * pr[ma], sf * pi[ma]};
                __syncwarp();
                if (lane < 2 * (j + 1)) {
                    const int ma = lane >> 1, c = lane & 1;
                    const T *col = reinterpret_cast<const T *>(stage + ma) + c;
                    T s = T(0);
                    for (int l = 0; l < nact; l++) s += col[l * SROW * 2];
                    T *dst = reinterpret_cast<T *>(acc + idxu_block(j) + (j + 1) * mb + ma) + c;
                    *dst += s;
                }
                __syncwarp();
            };
            u_rows<T, TJ>((T)g.ar, (T)g.ai, (T)g.br, (T)g.bi, emit);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ssum += __shfl_xor_sync(0xffffffffu, ssum, o);
        if (lane == 0) acc[0].x += ssum;
        __syncwarp();
        if constexpr (REF) {
            for (int k = lane; k < NU; k += 32) {
                int j = 0;
                while (idxu_block(j + 1) <= k) j++;
                const int mb = (k - idxu_block(j)) / (j + 1);
                if (2 * mb <= j) {
                    Uref_r[(size_t)k * natoms + i] += (double)acc[k].x;
                    Uref_i[(size_t)k * natoms + i] += (double)acc[k].y;
                }
            }
            __syncwarp();
            continue;
        }
        // wself = 1 on the diagonal of the computed half (cpuAddWself2Ui)
        for (int j = lane; j <= TJ; j += 32)
            for (int m = 0; 2 * m <= j; m++) acc[idxu_block(j) + (j + 1) * m + m].x += T(1);
        __syncwarp();
        // mirror rows mb < j/2 into rows j-mb: U(j-mb, j-ma) = (-1)^(ma+mb) conj U(mb, ma)
        for (int k = lane; k < NU; k += 32) {
            int j = 0;
            while (idxu_block(j + 1) <= k) j++;
            const int rem = k - idxu_block(j), mb = rem / (j + 1), ma = rem - mb * (j + 1);
            if (2 * mb < j) {
                const T s = ((ma + mb) & 1) ? T(-1) : T(1);
                const T2 v = acc[k];
                acc[idxu_block(j) + (j + 1) * (j - mb) + (j - ma)] = T2{s * v.x, -s * v.y};
            }
        }
        __syncwarp();
        T2 *dst = Ut + (size_t)(i >> 5) * NU * 32 + (i & 31);
        for (int k = lane; k < NU; k += 32) dst[(size_t)k * 32] = acc[k];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// k_snap_yi
// ---------------------------------------------------------------------------

// C++ truncating division as the reference's index formulas use it
__host__ __device__ constexpr int nb_of(int j1, int j2, int j, int mb)
{
    return cmin(j1, (2 * mb - j + j2 + j1) / 2) - cmax(0, (2 * mb - j - j2 + j1) / 2) + 1;
}
__host__ __device__ constexpr int items_of(int j1, int j2, int j)
{
    int n = 0;
    for (int mb = 0; 2 * mb <= j; mb++) n += nb_of(j1, j2, j, mb);
    return n;
}

// Row mb of beta' Z_{J1 J2 J}, restricted to the row pairs ib = o, o+st, ...,
// accumulated into yr/yi (registers).
template <typename T, int J1, int J2, int J>
__device__ __forceinline__ void z_rows(const int mb, const int o, const int st,
                                       const typename cplx<T>::type *__restrict__ Us, const int lane, const T beta,
                                       T (&yr)[JD], T (&yi)[JD])
{
    typedef typename cplx<T>::type T2;
    constexpr int N1 = J1 + 1, N2 = J2 + 1;
    constexpr int CGB = cg_block(J1, J2, J);
    const int mb1min = max(0, (2 * mb - J - J2 + J1) / 2);
    const int mb2max = (2 * mb - J - (2 * mb1min - J1) + J2) / 2;
    const int nb = min(J1, (2 * mb - J + J2 + J1) / 2) - mb1min + 1;
    for (int ib = o; ib < nb; ib += st) {
        const int mb1 = mb1min + ib, mb2 = mb2max - ib;
        const T s = beta * cgc<T>(CGB + mb1 * N2 + mb2);
        const T2 *r1 = Us + (idxu_block(J1) + N1 * mb1) * 32 + lane;
        const T2 *r2 = Us + (idxu_block(J2) + N2 * mb2) * 32 + lane;
        T u1r[N1], u1i[N1], u2r[N2], u2i[N2];
#pragma unroll
        for (int a = 0; a < N1; a++) { const T2 v = r1[a * 32]; u1r[a] = s * v.x; u1i[a] = s * v.y; }
#pragma unroll
        for (int a = 0; a < N2; a++) { const T2 v = r2[a * 32]; u2r[a] = v.x; u2i[a] = v.y; }
#pragma unroll
        for (int ma = 0; ma <= J; ma++) {
            const int ma1min = cmax(0, (2 * ma - J - J2 + J1) / 2);
            const int ma2max = (2 * ma - J - (2 * ma1min - J1) + J2) / 2;
            const int na = cmin(J1, (2 * ma - J + J2 + J1) / 2) - ma1min + 1;
#pragma unroll
            for (int ia = 0; ia < na; ia++) {
                const int ma1 = ma1min + ia, ma2 = ma2max - ia;
                const T c = cgc<T>(CGB + ma1 * N2 + ma2);
                const T tr = c * u1r[ma1], ti = c * u1i[ma1];
                yr[ma] += tr * u2r[ma2] - ti * u2i[ma2];
                yi[ma] += tr * u2i[ma2] + ti * u2r[ma2];
            }
        }
    }
}

// all couplings of output layer J, in enumeration order (every warp walks the
// same sequence, so the code in flight is one coupling's)
template <typename T, int TJ, int J, int J1, int J2>
__device__ __forceinline__ void z_layer(const int mb, const int o, const int st,
                                        const typename cplx<T>::type *__restrict__ Us, const int lane,
                                        const YParams<T> &P, T (&yr)[JD], T (&yi)[JD])
{
    if constexpr (J1 <= TJ) {
        if constexpr (J2 <= J1) {
            if constexpr (coupling_ok(J1, J2, J))
                z_rows<T, J1, J2, J>(mb, o, st, Us, lane, P.betaY[tri_index(J1, J2, J)], yr, yi);
            z_layer<T, TJ, J, J1, J2 + 1>(mb, o, st, Us, lane, P, yr, yi);
        } else {
            z_layer<T, TJ, J, J1 + 1, 0>(mb, o, st, Us, lane, P, yr, yi);
        }
    }
}

// layer J: each warp builds its partial row, the partials are summed per row,
// written out (tiled) and folded into the energy identity
template <typename T, int TJ, int NW, int J>
__device__ __forceinline__ void y_layer(const typename cplx<T>::type *__restrict__ Us,
                                        typename cplx<T>::type *__restrict__ red,
                                        typename cplx<T>::type *__restrict__ dst, const int lane, const int w,
                                        const YParams<T> &P, double &e)
{
    typedef typename cplx<T>::type T2;
    const int mb = P.lay_mb[J][w];
    if (mb != 255) {
        T yr[JD], yi[JD];
#pragma unroll
        for (int ma = 0; ma < JD; ma++) { yr[ma] = T(0); yi[ma] = T(0); }
        z_layer<T, TJ, J, 0, 0>(mb, P.lay_o[J][w], P.lay_st[J][w], Us, lane, P, yr, yi);
#pragma unroll
        for (int ma = 0; ma <= J; ma++) red[(w * JD + ma) * 32 + lane] = T2{yr[ma], yi[ma]};
    }
    __syncthreads();
    constexpr int NE = (J / 2 + 1) * (J + 1);
    for (int k = w; k < NE; k += NW) {
        const int rmb = k / (J + 1), ma = k - rmb * (J + 1);
        T yr = T(0), yi = T(0);
#pragma unroll
        for (int v = 0; v < NW; v++)
            if (P.lay_mb[J][v] == rmb) {
                const T2 t = red[(v * JD + ma) * 32 + lane];
                yr += t.x; yi += t.y;
            }
        const T2 u = Us[(idxu_block(J) + k) * 32 + lane];
        const double wgt = (2 * rmb < J) ? 1.0 : (ma < rmb ? 1.0 : (ma == rmb ? 0.5 : 0.0));
        e += wgt * ((double)u.x * (double)yr + (double)u.y * (double)yi);
        dst[(yh_block(J) + k) * 32 + lane] = T2{yr, yi};
    }
    __syncthreads();
}

template <typename T, int TJ, int NW, int J>
__device__ __forceinline__ void y_all(const typename cplx<T>::type *__restrict__ Us,
                                      typename cplx<T>::type *__restrict__ red,
                                      typename cplx<T>::type *__restrict__ dst, const int lane, const int w,
                                      const YParams<T> &P, double &e)
{
    if constexpr (J >= 0) {
        y_layer<T, TJ, NW, J>(Us, red, dst, lane, w, P, e);
        y_all<T, TJ, NW, J - 1>(Us, red, dst, lane, w, P, e);
    }
}

template <typename T, int TJ>
constexpr size_t yi_smem_bytes()
{
    return (size_t)idxu_count(TJ) * 32 * sizeof(typename cplx<T>::type) +
           (size_t)YiWarps<T>::n * JD * 32 * sizeof(typename cplx<T>::type) + YiWarps<T>::n * 32 * sizeof(double);
}

// Output Y in 32-atom tiles: Y[tile][k][lane], k = half-plane index.
template <typename T, int TJ>
__global__ void __launch_bounds__(YiWarps<T>::n * 32, 1)
k_snap_yi(const typename cplx<T>::type *__restrict__ Ut, int natoms, const __grid_constant__ YParams<T> P,
          typename cplx<T>::type *__restrict__ Y, double *__restrict__ eatom)
{
    typedef typename cplx<T>::type T2;
    constexpr int NW = YiWarps<T>::n;
    constexpr int NU = idxu_count(TJ);
    constexpr int NYH = yh_count(TJ);
    extern __shared__ __align__(16) unsigned char smraw[];
    T2 *Us = reinterpret_cast<T2 *>(smraw);
    T2 *red = Us + NU * 32;                                // [warp][ma][lane]
    double *ered = reinterpret_cast<double *>(red + NW * JD * 32);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntiles = (natoms + 31) >> 5;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const T2 *src = Ut + (size_t)tile * NU * 32;
        for (int k = threadIdx.x; k < NU * 32; k += NW * 32) Us[k] = src[k];
        __syncthreads();
        double e = 0.0;
        y_all<T, TJ, NW, TJ>(Us, red, Y + (size_t)tile * NYH * 32, lane, w, P, e);
        ered[w * 32 + lane] = e;
        __syncthreads();
        const int atom = tile * 32 + lane;
        if (w == 0 && atom < natoms) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < NW; k++) s += ered[k * 32 + lane];
            eatom[atom] = P.e0 + (2.0 / 3.0) * s;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k_snap_bi: per-atom bispectrum B_k = 2 sum_half w Re(U_j* Z_{j1 j2 j}) (- bzero)
// for the triples j >= j1 (cpuSnap4.cpp:427-592, cpuSnapComputeBi).  Tiles of 32
// atoms, warps take triples round-robin.  Output bout[k * bstride + atom].
// ---------------------------------------------------------------------------
constexpr int BI_WARPS = 8;

template <typename T, int TJ, int J1, int J2, int J, int C>
__device__ __forceinline__ void b_triples(const typename cplx<T>::type *__restrict__ Us, const int lane, const int w,
                                          const int atom, const int natoms, const int bnorm, const int bzero,
                                          double *__restrict__ bout, const long bstride)
{
    typedef typename cplx<T>::type T2;
    if constexpr (J1 <= TJ) {
        if constexpr (J2 <= J1) {
            if constexpr (J <= cmin(TJ, J1 + J2)) {
                if constexpr (J >= J1) {
                    if (C % BI_WARPS == w) {
                        double sum = 0.0;
                        for (int mb = 0; 2 * mb <= J; mb++) {
                            T zr[JD], zi[JD];
#pragma unroll
                            for (int ma = 0; ma < JD; ma++) { zr[ma] = T(0); zi[ma] = T(0); }
                            z_rows<T, J1, J2, J>(mb, 0, 1, Us, lane, T(1), zr, zi);
                            const T2 *urow = Us + (idxu_block(J) + (J + 1) * mb) * 32 + lane;
#pragma unroll
                            for (int ma = 0; ma <= J; ma++) {
                                const double wgt = (2 * mb < J) ? 1.0 : (ma < mb ? 1.0 : (ma == mb ? 0.5 : 0.0));
                                const T2 u = urow[ma * 32];
                                sum += wgt * ((double)u.x * (double)zr[ma] + (double)u.y * (double)zi[ma]);
                            }
                        }
                        double b = 2.0 * sum;
                        if (bnorm) b /= (J + 1);
                        if (bzero) b -= bnorm ? 1.0 : (double)(J + 1);
                        if (atom < natoms) bout[(long)C * bstride + atom] = b;
                    }
                    b_triples<T, TJ, J1, J2, J + 2, C + 1>(Us, lane, w, atom, natoms, bnorm, bzero, bout, bstride);
                } else {
                    b_triples<T, TJ, J1, J2, J + 2, C>(Us, lane, w, atom, natoms, bnorm, bzero, bout, bstride);
                }
            } else {
                b_triples<T, TJ, J1, J2 + 1, J1 - J2 - 1, C>(Us, lane, w, atom, natoms, bnorm, bzero, bout, bstride);
            }
        } else {
            b_triples<T, TJ, J1 + 1, 0, J1 + 1, C>(Us, lane, w, atom, natoms, bnorm, bzero, bout, bstride);
        }
    }
}

template <typename T, int TJ>
__global__ void __launch_bounds__(BI_WARPS * 32, 1)
k_snap_bi(const typename cplx<T>::type *__restrict__ Ut, int natoms, int bnorm, int bzero,
          double *__restrict__ bout, long bstride)
{
    typedef typename cplx<T>::type T2;
    constexpr int NU = idxu_count(TJ);
    extern __shared__ __align__(16) unsigned char smraw[];
    T2 *Us = reinterpret_cast<T2 *>(smraw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntiles = (natoms + 31) >> 5;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const T2 *src = Ut + (size_t)tile * NU * 32;
        for (int k = threadIdx.x; k < NU * 32; k += BI_WARPS * 32) Us[k] = src[k];
        __syncthreads();
        b_triples<T, TJ, 0, 0, 0, 0>(Us, lane, w, tile * 32 + lane, natoms, bnorm, bzero, bout, bstride);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k_snap_fi: one thread per pair.  dEslot[pinfo.y] = dE/d(r_j - r_i).
// ---------------------------------------------------------------------------
template <typename T>
struct FAcc {   // plain accumulator
    T s;
    __device__ __forceinline__ void init(T v) { s = v; }
    __device__ __forceinline__ void add(T v) { s += v; }
    __device__ __forceinline__ double val() const { return (double)s; }
};
struct FAccComp {   // compensated (Neumaier) float accumulator
    float s, c;
    __device__ __forceinline__ void init(float v) { s = v; c = 0.f; }
    __device__ __forceinline__ void add(float v)
    {
        const float t = s + v;
        c += (fabsf(s) >= fabsf(v)) ? ((s - t) + v) : ((v - t) + s);
        s = t;
    }
    __device__ __forceinline__ double val() const { return (double)s + (double)c; }
};
template <typename T> struct FAccSel { typedef FAcc<T> type; };
template <> struct FAccSel<float> { typedef FAccComp type; };

constexpr int FI_THREADS = 128;
template <typename T, int TJ> constexpr size_t fi_smem_bytes() { return sizeof(T) * 8 * (TJ + 1) * FI_THREADS; }

// One forward-mode pass over the U recursion of a pair, carrying the value and
// ND derivative directions k = K0..K0+ND-1.  The (mb, j) loop nest is written
// as compile-time recursion so every array index is a constant and the row
// state stays in registers.  Seed rows of the next mb level are parked in this
// thread's shared-memory slots qs[c * (TJ+1) * FI_THREADS + ma * FI_THREADS],
// c = 0,1 (value re/im), 2..1+ND (derivative re), 2+ND..1+2ND (derivative im).
// A0 (sum w Re(Y* U)) is accumulated by the pass with K0 == 0.
template <typename T, int TJ, int ND>
struct FiRow {
    T pr[TJ + 1], pi[TJ + 1], dr[ND][TJ + 1], di[ND][TJ + 1];
};

template <typename T, int ND>
struct FiGeo {
    T ar, ai, br, bi;
    T dar[ND], dai[ND], dbr[ND], dbi[ND];
};

template <typename T, int TJ, int ND, int K0, int MB, int J, typename Acc>
__device__ __forceinline__ void fi_layer(FiRow<T, TJ, ND> &st, const FiGeo<T, ND> &g,
                                         const typename cplx<T>::type *__restrict__ Yi, Acc &A0, Acc (&A)[3],
                                         T *__restrict__ qs)
{
    typedef typename cplx<T>::type T2;
    constexpr int QS = (TJ + 1) * FI_THREADS;
    const T ar = g.ar, ai = g.ai, br = g.br, bi = g.bi;
    {   // ma = J
        const T rp = rootpq<T>(J, J - MB);
        const T wr = st.pr[J - 1], wi = st.pi[J - 1];
#pragma unroll
        for (int k = 0; k < ND; k++) {
            const T xr = st.dr[k][J - 1], xi = st.di[k][J - 1];
            st.dr[k][J] = -rp * (g.dbr[k] * wr + g.dbi[k] * wi + br * xr + bi * xi);
            st.di[k][J] = -rp * (g.dbr[k] * wi - g.dbi[k] * wr + br * xi - bi * xr);
        }
        st.pr[J] = -rp * (br * wr + bi * wi);
        st.pi[J] = -rp * (br * wi - bi * wr);
    }
#pragma unroll
    for (int ma = J - 1; ma >= 0; ma--) {
        const T rpa = rootpq<T>(J - ma, J - MB);
        const T ur = st.pr[ma], ui = st.pi[ma];
        T nr = rpa * (ar * ur + ai * ui);
        T ni = rpa * (ar * ui - ai * ur);
        T ndr[ND], ndi[ND];
#pragma unroll
        for (int k = 0; k < ND; k++) {
            ndr[k] = rpa * (g.dar[k] * ur + g.dai[k] * ui + ar * st.dr[k][ma] + ai * st.di[k][ma]);
            ndi[k] = rpa * (g.dar[k] * ui - g.dai[k] * ur + ar * st.di[k][ma] - ai * st.dr[k][ma]);
        }
        if (ma > 0) {
            const T rpb = rootpq<T>(ma, J - MB);
            const T vr = st.pr[ma - 1], vi = st.pi[ma - 1];
            nr -= rpb * (br * vr + bi * vi);
            ni -= rpb * (br * vi - bi * vr);
#pragma unroll
            for (int k = 0; k < ND; k++) {
                ndr[k] -= rpb * (g.dbr[k] * vr + g.dbi[k] * vi + br * st.dr[k][ma - 1] + bi * st.di[k][ma - 1]);
                ndi[k] -= rpb * (g.dbr[k] * vi - g.dbi[k] * vr + br * st.di[k][ma - 1] - bi * st.dr[k][ma - 1]);
            }
        }
        st.pr[ma] = nr; st.pi[ma] = ni;
#pragma unroll
        for (int k = 0; k < ND; k++) { st.dr[k][ma] = ndr[k]; st.di[k][ma] = ndi[k]; }
    }
    if constexpr (MB > 0 && J == 2 * MB) {
        // middle row mirror; the reference leaves the derivative centre as
        // computed (its two mirror passes cancel, cpuSnap4.cpp:1061-1104)
#pragma unroll
        for (int ma = 0; ma <= MB; ma++) {
            const T s = (ma & 1) ? T(-1) : T(1);
            st.pr[MB + ma] = s * st.pr[MB - ma];
            st.pi[MB + ma] = -s * st.pi[MB - ma];
            if (ma > 0) {
#pragma unroll
                for (int k = 0; k < ND; k++) { st.dr[k][MB + ma] = s * st.dr[k][MB - ma]; st.di[k][MB + ma] = -s * st.di[k][MB - ma]; }
            }
        }
    }
    if constexpr (J == 2 * MB + 1 && 2 * (MB + 1) <= TJ) {
#pragma unroll
        for (int ma = 0; ma <= J; ma++) {
            const T s = ((MB + ma) & 1) ? T(-1) : T(1);
            qs[0 * QS + (J - ma) * FI_THREADS] = s * st.pr[ma];
            qs[1 * QS + (J - ma) * FI_THREADS] = -s * st.pi[ma];
#pragma unroll
            for (int k = 0; k < ND; k++) {
                qs[(2 + k) * QS + (J - ma) * FI_THREADS] = s * st.dr[k][ma];
                qs[(2 + ND + k) * QS + (J - ma) * FI_THREADS] = -s * st.di[k][ma];
            }
        }
    }
    // contract this row with Y (half plane; centre of a middle row at 1/2)
    const T2 *yrow = Yi + (yh_block(J) + (J + 1) * MB) * 32;
    constexpr int MAMAX = (2 * MB == J) ? MB : J;
    T s0 = T(0), sk[ND];
#pragma unroll
    for (int k = 0; k < ND; k++) sk[k] = T(0);
#pragma unroll
    for (int ma = 0; ma <= MAMAX; ma++) {
        T2 y = yrow[ma * 32];
        if (2 * MB == J && ma == MB) { y.x *= T(0.5); y.y *= T(0.5); }
        if constexpr (K0 == 0) s0 += st.pr[ma] * y.x + st.pi[ma] * y.y;
#pragma unroll
        for (int k = 0; k < ND; k++) sk[k] += st.dr[k][ma] * y.x + st.di[k][ma] * y.y;
    }
    if constexpr (K0 == 0) A0.add(s0);
#pragma unroll
    for (int k = 0; k < ND; k++) A[K0 + k].add(sk[k]);
    if constexpr (J < TJ) {
        asm volatile("" ::: "memory");
        fi_layer<T, TJ, ND, K0, MB, J + 1>(st, g, Yi, A0, A, qs);
    }
}

template <typename T, int TJ, int ND, int K0, int MB, typename Acc>
__device__ __forceinline__ void fi_rows(FiRow<T, TJ, ND> &st, const FiGeo<T, ND> &g,
                                        const typename cplx<T>::type *__restrict__ Yi, Acc &A0, Acc (&A)[3],
                                        T *__restrict__ qs)
{
    if constexpr (2 * MB <= TJ) {
        constexpr int QS = (TJ + 1) * FI_THREADS;
        if constexpr (MB == 0) {
            st.pr[0] = T(1); st.pi[0] = T(0);
#pragma unroll
            for (int k = 0; k < ND; k++) { st.dr[k][0] = T(0); st.di[k][0] = T(0); }
        } else {
#pragma unroll
            for (int ma = 0; ma < 2 * MB; ma++) {
                st.pr[ma] = qs[0 * QS + ma * FI_THREADS]; st.pi[ma] = qs[1 * QS + ma * FI_THREADS];
#pragma unroll
                for (int k = 0; k < ND; k++) {
                    st.dr[k][ma] = qs[(2 + k) * QS + ma * FI_THREADS];
                    st.di[k][ma] = qs[(2 + ND + k) * QS + ma * FI_THREADS];
                }
            }
        }
        fi_layer<T, TJ, ND, K0, MB, (MB == 0 ? 1 : 2 * MB)>(st, g, Yi, A0, A, qs);
        asm volatile("" ::: "memory");
        fi_rows<T, TJ, ND, K0, MB + 1>(st, g, Yi, A0, A, qs);
    }
}

template <typename T, int TJ, int ND, int K0, typename Acc>
__device__ __forceinline__ void fi_pass(const T ar, const T ai, const T br, const T bi, const T (&dar)[3],
                                        const T (&dai)[3], const T (&dbr)[3], const T (&dbi)[3],
                                        const typename cplx<T>::type *__restrict__ Yi, Acc &A0, Acc (&A)[3],
                                        T *__restrict__ qs)
{
    FiGeo<T, ND> g;
    g.ar = ar; g.ai = ai; g.br = br; g.bi = bi;
#pragma unroll
    for (int k = 0; k < ND; k++) { g.dar[k] = dar[K0 + k]; g.dai[k] = dai[K0 + k]; g.dbr[k] = dbr[K0 + k]; g.dbi[k] = dbi[K0 + k]; }
    FiRow<T, TJ, ND> st;
    fi_rows<T, TJ, ND, K0, 0>(st, g, Yi, A0, A, qs);
}

// number of derivative directions carried by the first pass; the rest follow
// one at a time.  Chosen so the recursion state stays in registers.
template <typename T, int TJ> struct FiSplit { static constexpr int first = 3; };

template <typename T, int TJ>
__device__ __forceinline__ void fi_pair(const int p, const double4 *__restrict__ prij, const int2 *__restrict__ pinfo,
                                        const SnapGeom &gp, const typename cplx<T>::type *__restrict__ Y,
                                        double4 *__restrict__ dEslot, const int nm, T *__restrict__ qs)
{
    typedef typename cplx<T>::type T2;
    typedef typename FAccSel<T>::type Acc;
    constexpr int NYH = yh_count(TJ);
    const double4 r = prij[p];
    const int2 inf = pinfo[p];
    PairGeo g;
    pair_geometry<true>(g, r.x, r.y, r.z, gp);
    const T ar = (T)g.ar, ai = (T)g.ai, br = (T)g.br, bi = (T)g.bi;
    T dar[3], dai[3], dbr[3], dbi[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { dar[k] = (T)g.dar[k]; dai[k] = (T)g.dai[k]; dbr[k] = (T)g.dbr[k]; dbi[k] = (T)g.dbi[k]; }
    const T2 *Yi = Y + (size_t)(inf.x >> 5) * NYH * 32 + (inf.x & 31);   // tiled: element k at Yi[k*32]

    // A0 = sum w Re(Y* U), Ak = sum w Re(Y* dU/dx_k); dE/dx_k = 2(dsfac u_k A0 + sfac Ak)
    Acc A0, A[3];
    A0.init((T)(0.5 * (double)Yi[0].x));   // j = 0 element
#pragma unroll
    for (int k = 0; k < 3; k++) A[k].init(T(0));
    constexpr int N1 = FiSplit<T, TJ>::first;
    fi_pass<T, TJ, N1, 0>(ar, ai, br, bi, dar, dai, dbr, dbi, Yi, A0, A, qs);
    if constexpr (N1 < 3) fi_pass<T, TJ, 1, N1>(ar, ai, br, bi, dar, dai, dbr, dbi, Yi, A0, A, qs);
    if constexpr (N1 < 2) fi_pass<T, TJ, 1, 2>(ar, ai, br, bi, dar, dai, dbr, dbi, Yi, A0, A, qs);
    const double a0 = A0.val();
    double4 out;
    out.x = 2.0 * (g.dsfac * g.u[0] * a0 + g.sfac * A[0].val());
    out.y = 2.0 * (g.dsfac * g.u[1] * a0 + g.sfac * A[1].val());
    out.z = 2.0 * (g.dsfac * g.u[2] * a0 + g.sfac * A[2].val());
    out.w = 0.0;
    dEslot[inf.y] = out;   // inf.y: global output slot
}

// grid-stride over the pairs; the pair count is read on the device (the
// last entry of the pair offsets), so no host synchronisation is needed
template <typename T, int TJ>
__global__ void __launch_bounds__(FI_THREADS)
k_snap_fi(const double4 *__restrict__ prij, const int2 *__restrict__ pinfo, const int *__restrict__ pnum,
          SnapGeom gp, const typename cplx<T>::type *__restrict__ Y, double4 *__restrict__ dEslot, int nm)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    T *qs = reinterpret_cast<T *>(smraw) + threadIdx.x;
    const int npairs = *pnum;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x)
        fi_pair<T, TJ>(p, prij, pinfo, gp, Y, dEslot, nm, qs);
}

}  // namespace mdp
