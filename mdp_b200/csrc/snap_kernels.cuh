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
//   k_snap_fr   dE/dr_ij = 2 sum_half w Re(Y* dU/dr)         (:798-1175)
//               one thread per pair, reverse-mode (adjoint) differentiation
//               of the U recursion seeded with Y
#pragma once

#include "common.cuh"

#include <climits>
#include <type_traits>

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
constexpr int YI_MAXW = 24;
template <typename T>
struct YParams {
    T betaY[NTRI];          // beta' of each coupling triple (bnorm 1/(j+1) folded in)
    double e0;              // beta0 - sum_k beta_k bzero_k
    // per output layer j and warp w: the row mb the warp accumulates (255: idle)
    // and the residue / stride of the row-pair index ib it takes in every coupling
    unsigned char lay_mb[JD][YI_MAXW], lay_o[JD][YI_MAXW], lay_st[JD][YI_MAXW];
    // bispectrum component k whose coefficient each coupling triple carries;
    // with per-atom coefficients G[k][atom], the triple's weight is
    // betaY[tri] * G[kmap[tri]] (betaY then holds the multiplicity factors)
    unsigned char kmap[NTRI];
};
// warps per Y CTA: FP64 10 (two per row of the costliest layer; 168
// registers; measured 65 ms at 2M atoms against 70 / 71 / 68 / 68 / 74 ms for
// 9 / 8 / 11 / 12 / 14 warps; its 146 KB U tile leaves room for one CTA per
// SM); FP32 8 with two CTAs per SM (92 registers, 93 KB of shared memory
// each, so one CTA's barrier waits overlap the other's work: the Y stage takes
// 26.1 ms at 2M atoms against 28.3 / 27.1 / 26.8 / 28.2 ms for 6 / 7 / 10 /
// 12 warps at two CTAs and 28.4 ms for 20 warps at one).  At 2J <= 4 no layer has more than three rows and the extra
// warps only wait at the barriers: the FP32 per-atom-coefficient kernel of the
// surrogate takes 4 (surrogate steps at 2M atoms: 14.8 ms against 14.9 / 15.2
// / 15.8 / 17.6 / 16.9 ms at 3 / 6 / 8 / 12 / 20 warps; 2 cannot cover the
// three rows).
#ifndef YI_W4_D
#define YI_W4_D 10
#endif
#ifndef YI_W4_F
#define YI_W4_F 4
#endif
#ifndef YI_W8_F
#define YI_W8_F 8
#endif
#ifndef YI_MINB_F
#define YI_MINB_F 2
#endif
__host__ __device__ constexpr int yi_warps(bool fp32, int tj)
{
    return fp32 ? (tj <= 4 ? YI_W4_F : YI_W8_F) : (tj <= 4 ? YI_W4_D : 10);
}
// CTAs per SM the Y kernel is compiled for (register cap)
template <typename T> __host__ __device__ constexpr int yi_min_blocks()
{
    return std::is_same<T, float>::value ? YI_MINB_F : 1;
}
template <typename T, int TJ> struct YiWarps { static constexpr int n = yi_warps(false, TJ); };
template <int TJ> struct YiWarps<float, TJ> { static constexpr int n = yi_warps(true, TJ); };

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
// With pcw, each pair's cutoff and neighbour weight come from pcw[p]; with
// iblk, atom i is row i % iblk of element block i / iblk of the reference's
// [block][k][iblk] layout (chemflag U, cpuSnap4.cpp:59-61).
template <typename T, int TJ, bool REF = false>
__global__ void __launch_bounds__(UI_WARPS * 32)
k_snap_ui(const int *__restrict__ poff, const double4 *__restrict__ prij, int natoms, SnapGeom gp,
          typename cplx<T>::type *__restrict__ Ut, double *__restrict__ Uref_r = nullptr,
          double *__restrict__ Uref_i = nullptr, const double2 *__restrict__ pcw = nullptr, int iblk = 0)
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
            if (pcw) {
                SnapGeom ge = gp;
                if (act) { ge.rcut = pcw[p].x; ge.wj = pcw[p].y; }
                pair_geometry<false>(g, r.x, r.y, r.z, ge);
            } else {
                pair_geometry<false>(g, r.x, r.y, r.z, gp);
            }
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
            const int nrow = iblk > 0 ? iblk : natoms;
            const size_t base = (size_t)(i / nrow) * NU * nrow + (i % nrow);
            for (int k = lane; k < NU; k += 32) {
                int j = 0;
                while (idxu_block(j + 1) <= k) j++;
                const int mb = (k - idxu_block(j)) / (j + 1);
                if (2 * mb <= j) {
                    Uref_r[base + (size_t)k * nrow] += (double)acc[k].x;
                    Uref_i[base + (size_t)k * nrow] += (double)acc[k].y;
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

// Coefficient-free row step of column MB: v_J[ma] = conj(a) v_(J-1)[ma] -
// conj(b) v_(J-1)[ma-1], in place (entries 0..J).  The U entry is
// unorm(J, MB, ma) * v[ma]; the middle-row mirror is the same in both forms
// (unorm is symmetric about ma = MB there), and with the mb factor of unorm a
// column's seed is its predecessor's row 2MB-1 mirrored without any scale.
template <typename T, int TJ, int J, int MB>
__device__ __forceinline__ void cf_fwd(const T ar, const T ai, const T br, const T bi, T (&pr)[TJ + 1],
                                       T (&pi)[TJ + 1])
{
    if constexpr (std::is_same<T, float>::value) {
        // packed {re, im} pairs: conj(a) u = {ar, ar} u + {ai, -ai} swap(u),
        // -conj(b) v = {-br, -br} v + {-bi, bi} swap(v)
        const float2 A = make_float2(ar, ar), An = make_float2(ai, -ai);
        const float2 B = make_float2(-br, -br), Bn = make_float2(-bi, bi);
        {
            float2 t = __fmul2_rn(B, make_float2(pr[J - 1], pi[J - 1]));
            t = __ffma2_rn(Bn, make_float2(pi[J - 1], pr[J - 1]), t);
            pr[J] = t.x;
            pi[J] = t.y;
        }
#pragma unroll
        for (int ma = J - 1; ma >= 0; ma--) {
            float2 t = __fmul2_rn(A, make_float2(pr[ma], pi[ma]));
            t = __ffma2_rn(An, make_float2(pi[ma], pr[ma]), t);
            if (ma >= 1) {
                t = __ffma2_rn(B, make_float2(pr[ma - 1], pi[ma - 1]), t);
                t = __ffma2_rn(Bn, make_float2(pi[ma - 1], pr[ma - 1]), t);
            }
            pr[ma] = t.x;
            pi[ma] = t.y;
        }
    } else {
    {
        const T vr = pr[J - 1], vi = pi[J - 1];
        pr[J] = -br * vr - bi * vi;
        pi[J] = -br * vi + bi * vr;
    }
#pragma unroll
    for (int ma = J - 1; ma >= 1; ma--) {
        const T ur = pr[ma], ui = pi[ma], vr = pr[ma - 1], vi = pi[ma - 1];
        pr[ma] = ar * ur + ai * ui - br * vr - bi * vi;
        pi[ma] = ar * ui - ai * ur - br * vi + bi * vr;
    }
    {
        const T ur = pr[0], ui = pi[0];
        pr[0] = ar * ur + ai * ui;
        pi[0] = ar * ui - ai * ur;
    }
    }
    if constexpr (MB > 0 && J == 2 * MB) {
#pragma unroll
        for (int ma = 0; ma <= MB; ma++) {
            const T sg = (ma & 1) ? T(-1) : T(1);
            pr[MB + ma] = sg * pr[MB - ma];
            pi[MB + ma] = -sg * pi[MB - ma];
        }
    }
}

// ---------------------------------------------------------------------------
// k_snap_uc: U of a 32-atom tile, one warp per column of the half plane.
//
// Lane = atom.  Each lane walks its own atom's pairs, uc_pb<T>() per pass, and
// per pair recomputes the recursion path that reaches its warp's column: the
// seed chain (rows 1, 2c..2c+1 of the columns c below, each mirrored into the
// next column's seed) and then the column's own rows, which it adds into a
// half-plane tile in shared memory ([uh index][lane]).  Every column's path
// has one row per layer 1..TJ, so the warps' work is equal; the top two
// columns share the last warp (the top one continues from the row the other
// ends its chain with).  Warps own disjoint tile entries: no atomics.  The
// tile is then written out as the full plane with wself on the diagonal,
// and rows mb > j/2 and the middle rows' right halves by inversion symmetry
// (cpuSnap4.cpp:11-244, cpuAddWself2Ui).
// (a, b, sfac) of each pair come from the pair stage.
// ---------------------------------------------------------------------------
// pairs per lane per pass: FP32 takes two (independent chains, half the tile
// updates; 8.1 against 8.2 ms at 2M atoms); FP64 one (two measured 18.1
// against 15.7 ms: twice the unrolled code per warp path; with the split
// plan, 19.9 ms at two CTAs per SM and 21.8 ms at three against 15.1 ms)
#ifndef UC_PB_D
#define UC_PB_D 1
#endif
template <typename T> __host__ __device__ constexpr int uc_pb() { return std::is_same<T, float>::value ? 2 : UC_PB_D; }
// Work plan.  One warp per column (the top two columns share the last warp),
// or, for FP64 at 2J = 8, eight jobs (column, first layer added into the
// tile, last layer): a job steps through its column's rows below its first
// layer without adding them, so the deep columns are split across two warps
// and twice the warps share the tile (U 15.3 against 16.1 ms per step at 2M
// atoms).  FP32, with two pairs per pass, lost by it (12.0 against 8.3 ms).
#ifndef UC_SPLIT
#define UC_SPLIT 1
#endif
struct UcJob {
    int mb, jlo, jhi;
};
template <typename T, int TJ> __host__ __device__ constexpr bool uc_split()
{
    return UC_SPLIT && TJ == 8 && std::is_same<T, double>::value;
}
template <typename T, int TJ> __host__ __device__ constexpr int uc_warps() { return uc_split<T, TJ>() ? 8 : TJ / 2; }
// CTAs per SM the split FP64 kernel is compiled for: three 74 KB tiles fit an
// SM's shared memory, which holds 80 registers a thread
#ifndef UC_MINB_D
#define UC_MINB_D 3
#endif
// (0, the others: no bound, as an explicit 1 makes ptxas spend registers)
template <typename T, int TJ> __host__ __device__ constexpr int uc_minb() { return uc_split<T, TJ>() ? UC_MINB_D : 0; }
template <int TJ> __host__ __device__ constexpr UcJob uc_job(int w)
{
    constexpr UcJob plan8[8] = {{0, 0, 5}, {0, 6, 8}, {1, 0, 6}, {1, 7, 8},
                                {2, 0, 6}, {2, 7, 8}, {3, 0, 8}, {4, 0, 8}};
    return plan8[w];
}
// The tile holds the half plane without the entries right of a middle row's
// centre (the mirror of its left half): 145 entries at 2J = 8 against 155,
// which lets three FP64 CTAs share an SM (74 KB each) instead of two.
__host__ __device__ constexpr int uh_len(int j) { return (j + 1) * ((j + 1) / 2) + (j % 2 == 0 ? j / 2 + 1 : 0); }
__host__ __device__ constexpr int uh_block(int j)
{
    int n = 0;
    for (int jj = 0; jj < j; jj++) n += uh_len(jj);
    return n;
}
__host__ __device__ constexpr int uh_count(int tj) { return uh_block(tj + 1); }
template <typename T, int TJ> constexpr size_t uc_smem_bytes()
{
    return (size_t)uh_count(TJ) * 32 * sizeof(typename cplx<T>::type);
}

// per-pair state; the root of the recursion is v_0 = sfac, so every row comes
// out weighted by sfac (the recursion is linear in its root)
template <typename T, int TJ>
struct UcPairs {
    static constexpr int PB = uc_pb<T>();
    T ar[PB], ai[PB], br[PB], bi[PB];
    T pr[PB][TJ + 1], pi[PB][TJ + 1];
};

// seed chain up to column MB: column C's last chain row (2C+1) mirrored into
// column C+1's seed, for C = 0..MB-1
template <typename T, int TJ, int MB, int C>
__device__ __forceinline__ void uc_chain(UcPairs<T, TJ> &s)
{
    if constexpr (C < MB) {
        constexpr int J = 2 * C + 1;
#pragma unroll
        for (int q = 0; q < UcPairs<T, TJ>::PB; q++) {
            if constexpr (C > 0) cf_fwd<T, TJ, 2 * C, C>(s.ar[q], s.ai[q], s.br[q], s.bi[q], s.pr[q], s.pi[q]);
            cf_fwd<T, TJ, J, C>(s.ar[q], s.ai[q], s.br[q], s.bi[q], s.pr[q], s.pi[q]);
            T nr[J + 1], ni[J + 1];
#pragma unroll
            for (int ma = 0; ma <= J; ma++) {
                const T sg = ((C + ma) & 1) ? T(-1) : T(1);
                nr[J - ma] = sg * s.pr[q][ma]; ni[J - ma] = -sg * s.pi[q][ma];
            }
#pragma unroll
            for (int ma = 0; ma <= J; ma++) { s.pr[q][ma] = nr[ma]; s.pi[q][ma] = ni[ma]; }
        }
        uc_chain<T, TJ, MB, C + 1>(s);
    }
}

// rows J..JEND of column MB (row J's parent in s.pr/pi), each from layer
// JACC on added into the tile
template <typename T, int TJ, int MB, int J, int JEND, int JACC = 0>
__device__ __forceinline__ void uc_column(UcPairs<T, TJ> &s, typename cplx<T>::type *__restrict__ acc)
{
    typedef typename cplx<T>::type T2;
    if constexpr (J <= JEND) {
        if constexpr (J > 0) {
#pragma unroll
            for (int q = 0; q < UcPairs<T, TJ>::PB; q++)
                cf_fwd<T, TJ, J, MB>(s.ar[q], s.ai[q], s.br[q], s.bi[q], s.pr[q], s.pi[q]);
        }
        if constexpr (J < JACC) {
            uc_column<T, TJ, MB, J + 1, JEND, JACC>(s, acc);
            return;
        }
        T2 *row = acc + (uh_block(J) + (J + 1) * MB) * 32;
        constexpr int MAMAX = (2 * MB == J) ? MB : J;
#pragma unroll
        for (int ma = 0; ma <= MAMAX; ma++) {
            const T nu = unorm<T>(J, MB, ma);
            T2 v = row[ma * 32];
#pragma unroll
            for (int q = 0; q < UcPairs<T, TJ>::PB; q++) {
                if constexpr (std::is_same<T, float>::value)
                    v = __ffma2_rn(make_float2(nu, nu), make_float2(s.pr[q][ma], s.pi[q][ma]), v);
                else { v.x += nu * s.pr[q][ma]; v.y += nu * s.pi[q][ma]; }
            }
            row[ma * 32] = v;
        }
        uc_column<T, TJ, MB, J + 1, JEND, JACC>(s, acc);
    }
}

// the work of warp MB: column MB (and, for the last warp, column MB+1)
template <typename T, int TJ, int MB>
__device__ __forceinline__ void uc_path(UcPairs<T, TJ> &s, typename cplx<T>::type *__restrict__ acc)
{
    uc_chain<T, TJ, MB, 0>(s);
    if constexpr (MB + 1 < uc_warps<T, TJ>()) {
        uc_column<T, TJ, MB, (MB == 0 ? 0 : 2 * MB), TJ>(s, acc);
    } else {
        // last warp: column MB up to its row 2MB+1, mirror to the seed of
        // column MB+1 = TJ/2, then column MB's remaining rows continue from a
        // copy while column TJ/2 takes its single row TJ
        constexpr int MT = MB + 1;
        uc_column<T, TJ, MB, (MB == 0 ? 0 : 2 * MB), 2 * MB + 1>(s, acc);
        T kr[UcPairs<T, TJ>::PB][TJ + 1], ki[UcPairs<T, TJ>::PB][TJ + 1];
#pragma unroll
        for (int q = 0; q < UcPairs<T, TJ>::PB; q++)
#pragma unroll
            for (int ma = 0; ma <= 2 * MB + 1; ma++) { kr[q][ma] = s.pr[q][ma]; ki[q][ma] = s.pi[q][ma]; }
        uc_column<T, TJ, MB, 2 * MB + 2, TJ>(s, acc);
#pragma unroll
        for (int q = 0; q < UcPairs<T, TJ>::PB; q++) {
            constexpr int J = 2 * MB + 1;
#pragma unroll
            for (int ma = 0; ma <= J; ma++) {
                const T sg = ((MB + ma) & 1) ? T(-1) : T(1);
                s.pr[q][J - ma] = sg * kr[q][ma]; s.pi[q][J - ma] = -sg * ki[q][ma];
            }
        }
        uc_column<T, TJ, MT, 2 * MT, TJ>(s, acc);
    }
}

template <typename T, int TJ, int MB>
__device__ __forceinline__ void uc_dispatch(const int w, UcPairs<T, TJ> &s, typename cplx<T>::type *__restrict__ acc)
{
    if constexpr (uc_split<T, TJ>()) {
        if constexpr (MB < uc_warps<T, TJ>()) {
            constexpr UcJob jb = uc_job<TJ>(MB);
            if (w == MB) {
                uc_chain<T, TJ, jb.mb, 0>(s);
                uc_column<T, TJ, jb.mb, (jb.mb == 0 ? 0 : 2 * jb.mb), jb.jhi, jb.jlo>(s, acc);
            } else {
                uc_dispatch<T, TJ, MB + 1>(w, s, acc);
            }
        }
    } else if constexpr (MB < uc_warps<T, TJ>()) {
        if (w == MB) uc_path<T, TJ, MB>(s, acc);
        else uc_dispatch<T, TJ, MB + 1>(w, s, acc);
    }
}

template <typename T, int TJ>
__global__ void __launch_bounds__(uc_warps<T, TJ>() * 32, uc_minb<T, TJ>())
k_snap_uc(const int *__restrict__ poff, const double4 *__restrict__ prij, const double4 *__restrict__ pab,
          int natoms, typename cplx<T>::type *__restrict__ Ut, const int *__restrict__ welem = nullptr,
          int ipad = 0)
{
    typedef typename cplx<T>::type T2;
    constexpr int NW = uc_warps<T, TJ>();
    constexpr int NU = idxu_count(TJ), NUH = uh_count(TJ);
    extern __shared__ __align__(16) unsigned char smraw[];
    T2 *acc = reinterpret_cast<T2 *>(smraw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntiles = (natoms + 31) >> 5;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int k = threadIdx.x; k < NUH * 32; k += NW * 32) acc[k] = T2{T(0), T(0)};
        __syncthreads();
        const int i = tile * 32 + lane;
        int p = 0, pend = 0;
        if (i < natoms) { p = poff[i]; pend = poff[i + 1]; }
        for (; p < pend; p += UcPairs<T, TJ>::PB) {
            UcPairs<T, TJ> s;
#pragma unroll
            for (int q = 0; q < UcPairs<T, TJ>::PB; q++) {
                const bool ok = p + q < pend;
                const double4 g = ok ? pab[p + q] : make_double4(1.0, 0.0, 0.0, 0.0);
                s.ar[q] = (T)g.x; s.ai[q] = (T)g.y; s.br[q] = (T)g.z; s.bi[q] = (T)g.w;
                s.pr[q][0] = ok ? (T)prij[p + q].w : T(0);   // v_0 = sfac
                s.pi[q][0] = T(0);
            }
            uc_dispatch<T, TJ, 0>(w, s, acc + lane);
        }
        __syncthreads();
        // full plane out: wself on the diagonal, rows mb > j/2 mirrored.  With
        // welem (element blocks of virtual atoms v = b * ipad + atom), wself
        // goes to the atom's own element block only (cpuAddWself2Ui,
        // cpuSnap4.cpp:193-244, chemflag without wselfallflag).
        T2 *dst = Ut + (size_t)tile * NU * 32;
        for (int e = threadIdx.x; e < NU * 32; e += NW * 32) {
            const int k = e >> 5, l = e & 31;
            T ws = T(1);
            if (welem) {
                const int v = tile * 32 + l;
                ws = (welem[v % ipad] == v / ipad) ? T(1) : T(0);
            }
            int j = 0;
            while (idxu_block(j + 1) <= k) j++;
            const int rem = k - idxu_block(j), mb = rem / (j + 1), ma = rem - mb * (j + 1);
            T2 v;
            if (2 * mb < j || (2 * mb == j && ma <= mb)) {
                v = acc[(uh_block(j) + rem) * 32 + l];
                if (ma == mb) v.x += ws;
            } else {
                // mirror: rows mb > j/2 and a middle row's right half
                const int sb = j - mb, sa = j - ma;
                const T2 u = acc[(uh_block(j) + (j + 1) * sb + sa) * 32 + l];
                const T sg = ((sa + sb) & 1) ? T(-1) : T(1);
                v = T2{sg * (u.x + (sa == sb ? ws : T(0))), -sg * u.y};
            }
            dst[e] = v;
        }
        __syncthreads();
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

// One warp's partial output row of a layer, in registers: separate real and
// imaginary parts in FP64; {re, im} pairs in FP32, where the packed two-lane
// instructions of sm_100 do the complex arithmetic.
template <typename T> struct YRow {
    T r[JD], i[JD];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int m = 0; m < JD; m++) { r[m] = T(0); i[m] = T(0); }
    }
    __device__ __forceinline__ typename cplx<T>::type get(int m) const { return {r[m], i[m]}; }
};
template <> struct YRow<float> {
    float2 v[JD];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int m = 0; m < JD; m++) v[m] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ float2 get(int m) const { return v[m]; }
};

// FP32 rows: for every (ma1, ma2) the product p = (s u1[ma1]) u2[ma2] takes a
// packed multiply and a packed fused multiply-add ({ar, ai} * {br, br}, then
// {-ai, ar} * {bi, bi} added), and y[ma] += c p one more packed FMA, with
// ma = ma1 + ma2 - (J1 + J2 - J)/2.  u2 stays in registers as {re, re} and
// {im, im}; u1 streams from shared memory one entry at a time.
template <int J1, int J2, int J>
__device__ __forceinline__ void z_rows_f32(const int mb, const int o, const int st, const float2 *__restrict__ Us,
                                           const float2 *__restrict__ Us2, const int lane, const float beta,
                                           YRow<float> &acc)
{
    constexpr int N1 = J1 + 1, N2 = J2 + 1;
    constexpr int CGB = cg_block(J1, J2, J);
    constexpr int OFF = (J1 + J2 - J) / 2;
    const int mb1min = max(0, (2 * mb - J - J2 + J1) / 2);
    const int mb2max = (2 * mb - J - (2 * mb1min - J1) + J2) / 2;
    const int nb = min(J1, (2 * mb - J + J2 + J1) / 2) - mb1min + 1;
    for (int ib = o; ib < nb; ib += st) {
        const int mb1 = mb1min + ib, mb2 = mb2max - ib;
        const float s = beta * cgc<float>(CGB + mb1 * N2 + mb2);
        const float2 *r1 = Us + (idxu_block(J1) + N1 * mb1) * 32 + lane;
        const float2 *r2 = Us2 + (idxu_block(J2) + N2 * mb2) * 32 + lane;
        float2 br[N2], bi[N2];
#pragma unroll
        for (int a = 0; a < N2; a++) {
            const float2 v = r2[a * 32];
            br[a] = make_float2(v.x, v.x);
            bi[a] = make_float2(v.y, v.y);
        }
#pragma unroll
        for (int ma1 = 0; ma1 < N1; ma1++) {
            const float2 v = r1[ma1 * 32];
            const float2 a = __fmul2_rn(make_float2(s, s), v);
            const float2 an = make_float2(-a.y, a.x);
#pragma unroll
            for (int ma2 = 0; ma2 < N2; ma2++) {
                const int ma = ma1 + ma2 - OFF;
                if (ma < 0 || ma > J) continue;
                float2 p = __fmul2_rn(a, br[ma2]);
                p = __ffma2_rn(an, bi[ma2], p);
                const float c = cgc<float>(CGB + ma1 * N2 + ma2);
                acc.v[ma] = __ffma2_rn(make_float2(c, c), p, acc.v[ma]);
            }
        }
    }
}

// Row mb of beta' Z_{J1 J2 J}, restricted to the row pairs ib = o, o+st, ...,
// accumulated into the warp's row (registers).  The J1 factor is read from
// Us, the J2 factor from Us2 (the same tile for one element; the U blocks of
// two neighbour elements for the element-pair Z of chemflag SNAP).
template <typename T, int J1, int J2, int J>
__device__ __forceinline__ void z_rows(const int mb, const int o, const int st,
                                       const typename cplx<T>::type *__restrict__ Us,
                                       const typename cplx<T>::type *__restrict__ Us2, const int lane, const T beta,
                                       YRow<T> &acc)
{
    if constexpr (std::is_same<T, float>::value) {
        z_rows_f32<J1, J2, J>(mb, o, st, Us, Us2, lane, beta, acc);
        return;
    } else {
    T(&yr)[JD] = acc.r;
    T(&yi)[JD] = acc.i;
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
        const T2 *r2 = Us2 + (idxu_block(J2) + N2 * mb2) * 32 + lane;
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
}

// all couplings of output layer J, in enumeration order (every warp walks the
// same sequence, so the code in flight is one coupling's)
template <typename T, int TJ, bool PA, int J, int J1, int J2>
__device__ __forceinline__ void z_layer(const int mb, const int o, const int st,
                                        const typename cplx<T>::type *__restrict__ Us, const int lane,
                                        const YParams<T> &P, const T *__restrict__ Gs, YRow<T> &acc)
{
    if constexpr (J1 <= TJ) {
        if constexpr (J2 <= J1) {
            if constexpr (coupling_ok(J1, J2, J)) {
                constexpr int TRI = tri_index(J1, J2, J);
                T beta = P.betaY[TRI];
                if constexpr (PA) beta *= Gs[P.kmap[TRI] * 32 + lane];
                z_rows<T, J1, J2, J>(mb, o, st, Us, Us, lane, beta, acc);
            }
            z_layer<T, TJ, PA, J, J1, J2 + 1>(mb, o, st, Us, lane, P, Gs, acc);
        } else {
            z_layer<T, TJ, PA, J, J1 + 1, 0>(mb, o, st, Us, lane, P, Gs, acc);
        }
    }
}

// layer J: each warp builds its partial row, the partials are summed per row,
// written out (tiled) and folded into the energy identity
template <typename T, int TJ, int NW, bool PA, int J>
__device__ __forceinline__ void y_layer(const typename cplx<T>::type *__restrict__ Us,
                                        typename cplx<T>::type *__restrict__ red,
                                        typename cplx<T>::type *__restrict__ dst, const int lane, const int w,
                                        const YParams<T> &P, const T *__restrict__ Gs, double &e)
{
    typedef typename cplx<T>::type T2;
    const int mb = P.lay_mb[J][w];
    if (mb != 255) {
        YRow<T> acc;
        acc.zero();
        z_layer<T, TJ, PA, J, 0, 0>(mb, P.lay_o[J][w], P.lay_st[J][w], Us, lane, P, Gs, acc);
#pragma unroll
        for (int ma = 0; ma <= J; ma++) red[(w * JD + ma) * 32 + lane] = acc.get(ma);
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
        if constexpr (!PA) {
            const T2 u = Us[(idxu_block(J) + k) * 32 + lane];
            const double wgt = (2 * rmb < J) ? 1.0 : (ma < rmb ? 1.0 : (ma == rmb ? 0.5 : 0.0));
            e += wgt * ((double)u.x * (double)yr + (double)u.y * (double)yi);
        }
        dst[(yh_block(J) + k) * 32 + lane] = T2{yr, yi};
    }
    __syncthreads();
}

template <typename T, int TJ, int NW, bool PA, int J>
__device__ __forceinline__ void y_all(const typename cplx<T>::type *__restrict__ Us,
                                      typename cplx<T>::type *__restrict__ red,
                                      typename cplx<T>::type *__restrict__ dst, const int lane, const int w,
                                      const YParams<T> &P, const T *__restrict__ Gs, double &e)
{
    if constexpr (J >= 0) {
        y_layer<T, TJ, NW, PA, J>(Us, red, dst, lane, w, P, Gs, e);
        y_all<T, TJ, NW, PA, J - 1>(Us, red, dst, lane, w, P, Gs, e);
    }
}

// number of bispectrum components at 2J = TJ (triples j1 >= j2, j >= j1)
__host__ __device__ constexpr int nbispec(int tj)
{
    int n = 0;
    for (int j1 = 0; j1 <= tj; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= cmin(tj, j1 + j2); j += 2)
                if (j >= j1) n++;
    return n;
}

template <typename T, int TJ, bool PA = false>
constexpr size_t yi_smem_bytes()
{
    return (size_t)idxu_count(TJ) * 32 * sizeof(typename cplx<T>::type) +
           (size_t)YiWarps<T, TJ>::n * JD * 32 * sizeof(typename cplx<T>::type) + YiWarps<T, TJ>::n * 32 * sizeof(double) +
           (PA ? (size_t)nbispec(TJ) * 32 * sizeof(T) : 0);
}

// Output Y in 32-atom tiles: Y[tile][k][lane], k = half-plane index.
// PA: per-atom coefficients G[k * natoms + atom] (k over the nbispec(TJ)
// components) instead of the model's; no energy is written.
template <typename T, int TJ, bool PA = false>
__global__ void __launch_bounds__(YiWarps<T, TJ>::n * 32, yi_min_blocks<T>())
k_snap_yi(const typename cplx<T>::type *__restrict__ Ut, int natoms, const __grid_constant__ YParams<T> P,
          typename cplx<T>::type *__restrict__ Y, double *__restrict__ eatom, const T *__restrict__ G = nullptr)
{
    typedef typename cplx<T>::type T2;
    constexpr int NW = YiWarps<T, TJ>::n;
    constexpr int NU = idxu_count(TJ);
    constexpr int NYH = yh_count(TJ);
    constexpr int NK = nbispec(TJ);
    extern __shared__ __align__(16) unsigned char smraw[];
    T2 *Us = reinterpret_cast<T2 *>(smraw);
    T2 *red = Us + NU * 32;                                // [warp][ma][lane]
    double *ered = reinterpret_cast<double *>(red + NW * JD * 32);
    T *Gs = reinterpret_cast<T *>(ered + NW * 32);         // [k][lane] (PA)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntiles = (natoms + 31) >> 5;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const T2 *src = Ut + (size_t)tile * NU * 32;
        for (int k = threadIdx.x; k < NU * 32; k += NW * 32) Us[k] = src[k];
        if constexpr (PA) {
            for (int k = threadIdx.x; k < NK * 32; k += NW * 32) {
                const int a = tile * 32 + (k & 31);
                Gs[k] = (a < natoms) ? G[(size_t)(k >> 5) * natoms + a] : T(0);
            }
        }
        __syncthreads();
        double e = 0.0;
        y_all<T, TJ, NW, PA, TJ>(Us, red, Y + (size_t)tile * NYH * 32, lane, w, P, Gs, e);
        if constexpr (PA) {
            __syncthreads();
            continue;
        }
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

// Arguments of one atom lane's bispectrum sweep.  The Z factors are read
// from U1 (layer J1) and U2 (layer J2) and contracted with U3 (layer J): one
// tile three times for one element, the U blocks of the element triple
// (e1, e2, e3) for chemflag SNAP (cpuSnap4.cpp:255-284: Z^{e1 e2} with
// U^{e3}).  Without coef, B_k goes to bout[k * bstride + atom]; with coef,
// sum_k coef[k] B_k accumulates into e.
template <typename T> struct BiArgs {
    const typename cplx<T>::type *U1, *U2, *U3;
    int lane, w, atom, natoms, bnorm, bzero;
    double *bout;
    long bstride;
    const double *coef;
    double e;
};

template <typename T, int TJ, int J1, int J2, int J, int C>
__device__ __forceinline__ void b_triples(BiArgs<T> &a)
{
    typedef typename cplx<T>::type T2;
    if constexpr (J1 <= TJ) {
        if constexpr (J2 <= J1) {
            if constexpr (J <= cmin(TJ, J1 + J2)) {
                if constexpr (J >= J1) {
                    if (C % BI_WARPS == a.w) {
                        double sum = 0.0;
                        for (int mb = 0; 2 * mb <= J; mb++) {
                            YRow<T> z;
                            z.zero();
                            z_rows<T, J1, J2, J>(mb, 0, 1, a.U1, a.U2, a.lane, T(1), z);
                            const T2 *urow = a.U3 + (idxu_block(J) + (J + 1) * mb) * 32 + a.lane;
#pragma unroll
                            for (int ma = 0; ma <= J; ma++) {
                                const double wgt = (2 * mb < J) ? 1.0 : (ma < mb ? 1.0 : (ma == mb ? 0.5 : 0.0));
                                const T2 u = urow[ma * 32], zm = z.get(ma);
                                sum += wgt * ((double)u.x * (double)zm.x + (double)u.y * (double)zm.y);
                            }
                        }
                        double b = 2.0 * sum;
                        if (a.bnorm) b /= (J + 1);
                        if (a.bzero) b -= a.bnorm ? 1.0 : (double)(J + 1);
                        if (a.coef) a.e += a.coef[C] * b;
                        else if (a.atom < a.natoms) a.bout[(long)C * a.bstride + a.atom] = b;
                    }
                    b_triples<T, TJ, J1, J2, J + 2, C + 1>(a);
                } else {
                    b_triples<T, TJ, J1, J2, J + 2, C>(a);
                }
            } else {
                b_triples<T, TJ, J1, J2 + 1, J1 - J2 - 1, C>(a);
            }
        } else {
            b_triples<T, TJ, J1 + 1, 0, J1 + 1, C>(a);
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
        BiArgs<T> a{Us, Us, Us, lane, w, tile * 32 + lane, natoms, bnorm, bzero, bout, bstride, nullptr, 0.0};
        b_triples<T, TJ, 0, 0, 0, 0>(a);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Several element types (cpuSnap4.cpp:250-420 and 697-790 with nelements > 1).
// U is kept per neighbour element block b (chemflag; one block otherwise) as
// tiles of "virtual atoms" v = b * ipad + atom (ipad = 32 * ntiles), so the
// U and dE/dr kernels run unchanged over them.  Coefficients come from the
// reference's table coeffelem [element][ncoeffall]: beta_0 first, then the
// bispectrum components of element triple t at 1 + t * NK + k.
// ---------------------------------------------------------------------------
struct MeArgs {
    int nblk;              // U / Y element blocks (nelements with chemflag, else 1)
    int ntiles;            // tiles of 32 atoms per block
    int ncoeffall;         // coefficients per element
    int bzero, wselfall;   // bzeroflag, wselfallflag
    const int *elem;       // element index (map[type]) of each atom [inum]
    const double *coeff;   // coeffelem [nelements][ncoeffall], or with pa the
    int pa;                // per-atom coefficients [triple][k][inum] (cpuSnap4.cpp:601-691)
};

// Per-atom energy: beta_0(e_i) + sum over element triples t = (e1 e2 e3) and
// components k of beta(e_i, t, k) (B^t_k - bzero_j), with B^t = 2 sum_half
// Re(U^{e3*} Z^{e1 e2}) and bzero subtracted on t = (e e e) only unless
// wselfallflag (cpuSnapComputeEi, cpuSnap4.cpp:250-420).  Warps take the
// components round-robin per triple; the lanes' sums meet in shared memory.
template <int TJ>
__global__ void __launch_bounds__(BI_WARPS * 32, 1)
k_snap_ei_me(const double2 *__restrict__ Ut, int natoms, int bnorm, const __grid_constant__ MeArgs A,
             double *__restrict__ eatom)
{
    constexpr int NU = idxu_count(TJ), NK = nbispec(TJ);
    __shared__ double ered[BI_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nb = A.nblk;
    for (int tile = blockIdx.x; tile < A.ntiles; tile += gridDim.x) {
        const int atom = tile * 32 + lane;
        const int ie = atom < natoms ? A.elem[atom] : 0;
        const double *cl = A.coeff + (size_t)ie * A.ncoeffall;
        BiArgs<double> a{nullptr, nullptr, nullptr, lane, w, atom, natoms, bnorm, 0, nullptr, 0, nullptr, 0.0};
        for (int e1 = 0; e1 < nb; e1++)
            for (int e2 = 0; e2 < nb; e2++)
                for (int e3 = 0; e3 < nb; e3++) {
                    const int t = (e1 * nb + e2) * nb + e3;
                    a.U1 = Ut + ((size_t)e1 * A.ntiles + tile) * NU * 32;
                    a.U2 = Ut + ((size_t)e2 * A.ntiles + tile) * NU * 32;
                    a.U3 = Ut + ((size_t)e3 * A.ntiles + tile) * NU * 32;
                    a.bzero = A.bzero && (A.wselfall || (e1 == e2 && e2 == e3));
                    a.coef = cl + 1 + (size_t)t * NK;
                    b_triples<double, TJ, 0, 0, 0, 0>(a);
                }
        ered[w][lane] = a.e;
        __syncthreads();
        if (w == 0 && atom < natoms) {
            double s = cl[0];
#pragma unroll
            for (int k = 0; k < BI_WARPS; k++) s += ered[k][lane];
            eatom[atom] = s;
        }
        __syncthreads();
    }
}

// Y of every element block e3: sum over element pairs (e1, e2) and couplings
// of beta' Z^{e1 e2}, with beta' the coefficient of the element triple and
// bispectrum component each coupling case names (cpuSnapComputeYi,
// cpuSnap4.cpp:697-790): (e1 e2 e3) when j >= j1, (e3 e2 e1) when
// j1 > j >= j2, (e2 e3 e1) otherwise; P.betaY holds the multiplicity factors.
// U is read from global memory (the tile's blocks stay in L1 / L2), Y is
// written per block in the single-element tile layout.
template <int TJ, int J, int J1, int J2>
__device__ __forceinline__ void z_layer_me(const int mb, const int o, const int st, const double2 *__restrict__ U1,
                                           const double2 *__restrict__ U2, const int lane,
                                           const YParams<double> &P, const double *__restrict__ cl, const int cs,
                                           const int tA, const int tB, const int tC, YRow<double> &acc)
{
    constexpr int NK = nbispec(TJ);
    if constexpr (J1 <= TJ) {
        if constexpr (J2 <= J1) {
            if constexpr (coupling_ok(J1, J2, J)) {
                constexpr int TRI = tri_index(J1, J2, J);
                const int t = (J >= J1) ? tA : (J >= J2) ? tB : tC;
                const double beta = P.betaY[TRI] * cl[(size_t)(t * NK + P.kmap[TRI]) * cs];
                z_rows<double, J1, J2, J>(mb, o, st, U1, U2, lane, beta, acc);
            }
            z_layer_me<TJ, J, J1, J2 + 1>(mb, o, st, U1, U2, lane, P, cl, cs, tA, tB, tC, acc);
        } else {
            z_layer_me<TJ, J, J1 + 1, 0>(mb, o, st, U1, U2, lane, P, cl, cs, tA, tB, tC, acc);
        }
    }
}

template <int TJ, int NW, int J>
__device__ __forceinline__ void y_all_me(const double2 *__restrict__ Ut, const int tile, double2 *__restrict__ red,
                                         double2 *__restrict__ Y, const int lane, const int w,
                                         const YParams<double> &P, const MeArgs &A, const double *__restrict__ cl,
                                         const int cs)
{
    if constexpr (J >= 0) {
        constexpr int NU = idxu_count(TJ), NYH = yh_count(TJ);
        const int nb = A.nblk;
        const int mb = P.lay_mb[J][w];
        for (int e3 = 0; e3 < nb; e3++) {
            if (mb != 255) {
                YRow<double> acc;
                acc.zero();
                for (int e1 = 0; e1 < nb; e1++)
                    for (int e2 = 0; e2 < nb; e2++)
                        z_layer_me<TJ, J, 0, 0>(mb, P.lay_o[J][w], P.lay_st[J][w],
                                                Ut + ((size_t)e1 * A.ntiles + tile) * NU * 32,
                                                Ut + ((size_t)e2 * A.ntiles + tile) * NU * 32, lane, P, cl, cs,
                                                (e1 * nb + e2) * nb + e3, (e3 * nb + e2) * nb + e1,
                                                (e2 * nb + e3) * nb + e1, acc);
#pragma unroll
                for (int ma = 0; ma <= J; ma++) red[(w * JD + ma) * 32 + lane] = acc.get(ma);
            }
            __syncthreads();
            constexpr int NE = (J / 2 + 1) * (J + 1);
            double2 *dst = Y + ((size_t)e3 * A.ntiles + tile) * NYH * 32;
            for (int k = w; k < NE; k += NW) {
                const int rmb = k / (J + 1), ma = k - rmb * (J + 1);
                double yr = 0.0, yi = 0.0;
#pragma unroll
                for (int v = 0; v < NW; v++)
                    if (P.lay_mb[J][v] == rmb) {
                        const double2 t = red[(v * JD + ma) * 32 + lane];
                        yr += t.x; yi += t.y;
                    }
                dst[(yh_block(J) + k) * 32 + lane] = double2{yr, yi};
            }
            __syncthreads();
        }
        y_all_me<TJ, NW, J - 1>(Ut, tile, red, Y, lane, w, P, A, cl, cs);
    }
}

template <int TJ>
constexpr size_t yi_me_smem_bytes()
{
    return (size_t)YiWarps<double, TJ>::n * JD * 32 * sizeof(double2);
}

template <int TJ>
__global__ void __launch_bounds__(YiWarps<double, TJ>::n * 32, 1)
k_snap_yi_me(const double2 *__restrict__ Ut, int natoms, const __grid_constant__ YParams<double> P,
             const __grid_constant__ MeArgs A, double2 *__restrict__ Y)
{
    constexpr int NW = YiWarps<double, TJ>::n;
    extern __shared__ __align__(16) unsigned char smraw[];
    double2 *red = reinterpret_cast<double2 *>(smraw);   // [warp][ma][lane]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile < A.ntiles; tile += gridDim.x) {
        const int atom = tile * 32 + lane;
        if (A.pa) {
            y_all_me<TJ, NW, TJ>(Ut, tile, red, Y, lane, w, P, A, A.coeff + (atom < natoms ? atom : 0), natoms);
        } else {
            const int ie = atom < natoms ? A.elem[atom] : 0;
            y_all_me<TJ, NW, TJ>(Ut, tile, red, Y, lane, w, P, A, A.coeff + (size_t)ie * A.ncoeffall + 1, 1);
        }
    }
}

// Per-atom bispectrum of every element triple t = (e1 e2 e3):
// bout[(t * NK + k) * natoms + atom] (cpuSnapComputeBi, cpuSnap4.cpp:427-592),
// bzero on t = (e e e) only unless wselfallflag
template <int TJ>
__global__ void __launch_bounds__(BI_WARPS * 32, 1)
k_snap_bi_me(const double2 *__restrict__ Ut, int natoms, int bnorm, const __grid_constant__ MeArgs A,
             double *__restrict__ bout)
{
    constexpr int NU = idxu_count(TJ), NK = nbispec(TJ);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nb = A.nblk;
    for (int tile = blockIdx.x; tile < A.ntiles; tile += gridDim.x) {
        BiArgs<double> a{nullptr, nullptr, nullptr, lane, w, tile * 32 + lane, natoms, bnorm, 0, nullptr,
                         natoms, nullptr, 0.0};
        for (int e1 = 0; e1 < nb; e1++)
            for (int e2 = 0; e2 < nb; e2++)
                for (int e3 = 0; e3 < nb; e3++) {
                    const int t = (e1 * nb + e2) * nb + e3;
                    a.U1 = Ut + ((size_t)e1 * A.ntiles + tile) * NU * 32;
                    a.U2 = Ut + ((size_t)e2 * A.ntiles + tile) * NU * 32;
                    a.U3 = Ut + ((size_t)e3 * A.ntiles + tile) * NU * 32;
                    a.bzero = A.bzero && (A.wselfall || (e1 == e2 && e2 == e3));
                    a.bout = bout + (size_t)t * NK * natoms;
                    b_triples<double, TJ, 0, 0, 0, 0>(a);
                }
    }
}

// ---------------------------------------------------------------------------
// accumulators of the dE/dr kernel's gradient sums
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

// ---------------------------------------------------------------------------
// k_snap_fr: dE/dr of every pair by reverse-mode (adjoint) differentiation of
// the U recursion.  One thread per pair; dEslot[pinfo.y] = dE/d(r_j - r_i).
//
// With F(a, b) = sum_half w Re(Y* u(a, b)) (the same half-plane sum as the
// forward-mode kernel), dE/dx_k = 2 (dsfac u_k F + sfac dF/dx_k) and
// dF/dx_k = grad_(ar,ai,br,bi) F . d(a,b)/dx_k.  Each U row (layer J, column
// mb) is n[ma] = A_ma conj(a) p[ma] - B_ma conj(b) p[ma-1] of its parent row p
// (layer J-1), A_ma = rootpq(J-ma, J-mb), B_ma = rootpq(ma, J-mb).  Its
// adjoint, for an adjoint row l of layer J, is
//     l'[k] = A_k a l[k] - B_(k+1) b l[k+1]           (parent row's adjoint)
//     dF/d(ar + i ai) += A_ma conj(l[ma]) p[ma]        (as (re, im) pairs)
//     dF/d(br + i bi) -= B_ma conj(l[ma]) p[ma-1]
// and F itself is the real part of the adjoint of the root u_0 = 1.  In FP32
// the rows are instead the coefficient-free ones of k_snap_uc (u = unorm v,
// A = B = 1, adjoint seeded with unorm Y), which saves the rootpq products.
// This is about 5,100 operations per pair at 2J=8 against about 14,000 for
// carrying the three derivative directions forward through the recursion,
// which is how cpuSnap4.cpp:798-1175 computes dU/dr.
//
// Columns mb depend on each other only through the seed rows (the parent of
// row (2mb, mb) is the mirror of row (2mb-1, mb-1)), so the pass is:
//   A. value-only sweep that builds the seed rows S_1..S_(TJ/2) (shared memory)
//   B. for mb = TJ/2 .. 0: recompute column mb's rows from its seed, keeping
//      them in registers, then walk back from layer TJ accumulating the
//      gradient; the adjoint reaching the seed is mirrored into a link that
//      column mb-1 adds at layer 2mb-1 (stored over the seed's slot).
// The middle-row mirror of the forward values is exact on |a|^2 + |b|^2 = 1,
// and d(a,b)/dr stays on that sphere, so the adjoint treats the recursion's
// own right half as the row.
// ---------------------------------------------------------------------------
constexpr int FR_THREADS = 128;
// per-thread shared memory: seeds/links (2 * sum_mb 2mb values) + 16 geometry values
template <int TJ> constexpr int fr_seed_vals() { return 2 * (TJ / 2) * (TJ / 2 + 1); }
// Y staging: a CTA's window of FR_THREADS consecutive pairs spans a few atoms
// (about seven at 19 pairs per atom); when it spans at most fr_ycap<T>()
// atoms their Y rows are copied once into shared memory ([k][slot]) and the
// pairs read them there instead of each through L1 / L2.
#ifndef FR_YCAP_D
#define FR_YCAP_D 16
#endif
#ifndef FR_YCAP_F
#define FR_YCAP_F 12
#endif
template <typename T> __host__ __device__ constexpr int fr_ycap()
{
    return std::is_same<T, float>::value ? FR_YCAP_F : FR_YCAP_D;
}
template <typename T, int TJ> constexpr size_t fr_smem_bytes()
{
    return (sizeof(T) * fr_seed_vals<TJ>() + sizeof(double) * 16) * FR_THREADS +
           (size_t)yh_count(TJ) * fr_ycap<T>() * sizeof(typename cplx<T>::type);
}
__host__ __device__ constexpr int fr_seed_off(int mb) { return mb * (mb - 1); }   // complex offset of S_mb
__host__ __device__ constexpr int fr_row_off(int j) { return j * (j + 1) / 2; }   // stored row j

template <typename T, int TJ>
struct FrState {
    T ar, ai, br, bi;
    T ur[fr_row_off(TJ)], ui[fr_row_off(TJ)];   // parent rows 0..TJ-1 of the current column
    T lr[TJ + 1], li[TJ + 1];                   // adjoint row
};

// row J-1 -> row J of column MB, in place (entries 0..J), as u_rows does (u-space, rootpq factors)
template <typename T, int TJ, int J, int MB>
__device__ __forceinline__ void fr_fwd(const T ar, const T ai, const T br, const T bi, T (&pr)[TJ + 1],
                                       T (&pi)[TJ + 1])
{
    {
        const T rp = rootpq<T>(J, J - MB);
        const T nr = -rp * (br * pr[J - 1] + bi * pi[J - 1]);
        const T ni = -rp * (br * pi[J - 1] - bi * pr[J - 1]);
        pr[J] = nr; pi[J] = ni;
    }
#pragma unroll
    for (int ma = J - 1; ma >= 1; ma--) {
        const T rpa = rootpq<T>(J - ma, J - MB), rpb = rootpq<T>(ma, J - MB);
        const T nr = rpa * (ar * pr[ma] + ai * pi[ma]) - rpb * (br * pr[ma - 1] + bi * pi[ma - 1]);
        const T ni = rpa * (ar * pi[ma] - ai * pr[ma]) - rpb * (br * pi[ma - 1] - bi * pr[ma - 1]);
        pr[ma] = nr; pi[ma] = ni;
    }
    {
        const T rpa = rootpq<T>(J, J - MB);
        const T nr = rpa * (ar * pr[0] + ai * pi[0]);
        const T ni = rpa * (ar * pi[0] - ai * pr[0]);
        pr[0] = nr; pi[0] = ni;
    }
    if constexpr (MB > 0 && J == 2 * MB) {
#pragma unroll
        for (int ma = 0; ma <= MB; ma++) {
            const T s = (ma & 1) ? T(-1) : T(1);
            pr[MB + ma] = s * pr[MB - ma];
            pi[MB + ma] = -s * pi[MB - ma];
        }
    }
}

// FP64 runs the recursion in u-space (rootpq factors), FP32 in the
// coefficient-free v-space of k_snap_uc (u = unorm v).  Both give the same
// gradient; in FP64 the coefficient-free form issues fewer instructions but,
// at 254 registers, measured twice as slow (its memory latency is exposed).
template <typename T> __host__ __device__ constexpr bool fr_cf() { return std::is_same<T, float>::value; }
template <typename T, int TJ, int J, int MB>
__device__ __forceinline__ void fr_row(const T ar, const T ai, const T br, const T bi, T (&pr)[TJ + 1],
                                       T (&pi)[TJ + 1])
{
    if constexpr (fr_cf<T>()) cf_fwd<T, TJ, J, MB>(ar, ai, br, bi, pr, pi);
    else fr_fwd<T, TJ, J, MB>(ar, ai, br, bi, pr, pi);
}

// seed S_(MB+1)[J - ma] = (-1)^(MB+ma) conj(row (J = 2MB+1, MB)[ma])
template <typename T, int TJ, int MB>
__device__ __forceinline__ void fr_put_seed(const T (&pr)[TJ + 1], const T (&pi)[TJ + 1], T *__restrict__ qs)
{
    constexpr int J = 2 * MB + 1, O = fr_seed_off(MB + 1);
#pragma unroll
    for (int ma = 0; ma <= J; ma++) {
        const T s = ((MB + ma) & 1) ? T(-1) : T(1);
        qs[(2 * (O + J - ma) + 0) * FR_THREADS] = s * pr[ma];
        qs[(2 * (O + J - ma) + 1) * FR_THREADS] = -s * pi[ma];
    }
}

// phase A: seeds of columns 1..TJ/2
template <typename T, int TJ, int MB>
__device__ __forceinline__ void fr_seeds(const T ar, const T ai, const T br, const T bi, T (&pr)[TJ + 1],
                                         T (&pi)[TJ + 1], T *__restrict__ qs)
{
    if constexpr (2 * (MB + 1) <= TJ) {
        if constexpr (MB == 0) {
            pr[0] = T(1); pi[0] = T(0);
            fr_row<T, TJ, 1, 0>(ar, ai, br, bi, pr, pi);
        } else {
            // pr/pi hold S_MB (entries 0..2MB-1)
            fr_row<T, TJ, 2 * MB, MB>(ar, ai, br, bi, pr, pi);
            fr_row<T, TJ, 2 * MB + 1, MB>(ar, ai, br, bi, pr, pi);
        }
        fr_put_seed<T, TJ, MB>(pr, pi, qs);
        // the next column starts from the seed just written
        constexpr int J = 2 * MB + 1;
        T nr[TJ + 1], ni[TJ + 1];
#pragma unroll
        for (int ma = 0; ma <= J; ma++) {
            const T s = ((MB + ma) & 1) ? T(-1) : T(1);
            nr[J - ma] = s * pr[ma]; ni[J - ma] = -s * pi[ma];
        }
#pragma unroll
        for (int ma = 0; ma <= J; ma++) { pr[ma] = nr[ma]; pi[ma] = ni[ma]; }
        fr_seeds<T, TJ, MB + 1>(ar, ai, br, bi, pr, pi, qs);
    }
}

// phase B forward: rows J..TJ-1 of column MB from the row J-1 in (pr, pi), stored
template <typename T, int TJ, int J, int MB>
__device__ __forceinline__ void fr_col_fwd(FrState<T, TJ> &st, T (&pr)[TJ + 1], T (&pi)[TJ + 1])
{
    if constexpr (J < TJ) {
        fr_row<T, TJ, J, MB>(st.ar, st.ai, st.br, st.bi, pr, pi);
#pragma unroll
        for (int ma = 0; ma <= J; ma++) { st.ur[fr_row_off(J) + ma] = pr[ma]; st.ui[fr_row_off(J) + ma] = pi[ma]; }
        fr_col_fwd<T, TJ, J + 1, MB>(st, pr, pi);
    }
}

// weighted Y row (J, MB) added into the adjoint row (entries 0..J)
template <typename T, int TJ, int J, int MB>
__device__ __forceinline__ void fr_add_y(FrState<T, TJ> &st, const typename cplx<T>::type *__restrict__ Yi,
                                         const int ys)
{
    typedef typename cplx<T>::type T2;
    const T2 *yrow = Yi + (yh_block(J) + (J + 1) * MB) * ys;
    constexpr int MAMAX = (2 * MB == J) ? MB : J;
#pragma unroll
    for (int ma = 0; ma <= MAMAX; ma++) {
        const T2 y = yrow[ma * ys];
        // v-space (FP32): u = unorm v, so the adjoint of the row v is unorm Y
        const T un = fr_cf<T>() ? unorm<T>(J, MB, ma) : T(1);
        const T nu = (2 * MB == J && ma == MB) ? T(0.5) * un : un;
        st.lr[ma] += nu * y.x; st.li[ma] += nu * y.y;
    }
}

// phase B backward: adjoint row of layer J (column MB) in st.l*; parent row J-1
template <typename T, int TJ, int J, int MB, typename Acc>
__device__ __forceinline__ void fr_col_bwd(FrState<T, TJ> &st, const typename cplx<T>::type *__restrict__ Yi,
                                           const int ys, Acc (&G)[4], T *__restrict__ qs)
{
    constexpr int PO = fr_row_off(J - 1);
    const T ar = st.ar, ai = st.ai, br = st.br, bi = st.bi;
    // gradient of this layer (coefficient-free rows: n[ma] = conj(a) p[ma] - conj(b) p[ma-1])
    T gar = T(0), gai = T(0), gbr = T(0), gbi = T(0);
#pragma unroll
    for (int ma = 0; ma <= J; ma++) {
        const T lr = st.lr[ma], li = st.li[ma];
        if (ma < J) {
            const T pr = st.ur[PO + ma], pi = st.ui[PO + ma];
            if constexpr (fr_cf<T>()) {
                gar += lr * pr + li * pi;
                gai += lr * pi - li * pr;
            } else {
                const T A = rootpq<T>(J - ma, J - MB);
                gar += A * (lr * pr + li * pi);
                gai += A * (lr * pi - li * pr);
            }
        }
        if (ma >= 1) {
            const T pr = st.ur[PO + ma - 1], pi = st.ui[PO + ma - 1];
            if constexpr (fr_cf<T>()) {
                gbr -= lr * pr + li * pi;
                gbi -= lr * pi - li * pr;
            } else {
                const T B = rootpq<T>(ma, J - MB);
                gbr -= B * (lr * pr + li * pi);
                gbi -= B * (lr * pi - li * pr);
            }
        }
    }
    G[0].add(gar); G[1].add(gai); G[2].add(gbr); G[3].add(gbi);
    // adjoint of the parent row, in place (ascending k reads l[k+1] before it changes)
#pragma unroll
    for (int k = 0; k < J; k++) {
        const T lr = st.lr[k], li = st.li[k], mr = st.lr[k + 1], mi = st.li[k + 1];
        if constexpr (fr_cf<T>()) {
            st.lr[k] = (ar * lr - ai * li) - (br * mr - bi * mi);
            st.li[k] = (ar * li + ai * lr) - (br * mi + bi * mr);
        } else {
            const T A = rootpq<T>(J - k, J - MB), B = rootpq<T>(k + 1, J - MB);
            st.lr[k] = A * (ar * lr - ai * li) - B * (br * mr - bi * mi);
            st.li[k] = A * (ar * li + ai * lr) - B * (br * mi + bi * mr);
        }
    }
    if constexpr (J - 1 >= 2 * MB) {
        // parent is row (J-1, MB) of this column
        fr_add_y<T, TJ, J - 1, MB>(st, Yi, ys);
        if constexpr (J - 1 == 2 * MB + 1 && 2 * (MB + 1) <= TJ) {
            constexpr int O = fr_seed_off(MB + 1);
#pragma unroll
            for (int ma = 0; ma < J; ma++) {
                st.lr[ma] += qs[(2 * (O + ma) + 0) * FR_THREADS];
                st.li[ma] += qs[(2 * (O + ma) + 1) * FR_THREADS];
            }
        }
        // the column's first computed row is layer max(1, 2MB)
        if constexpr (J - 1 >= (MB == 0 ? 1 : 2 * MB)) fr_col_bwd<T, TJ, J - 1, MB>(st, Yi, ys, G, qs);
    } else {
        // parent is the seed S_MB = mirror of row (J' = 2MB-1, MB-1): store the
        // adjoint of that row, L[ma] = (-1)^(MB-1+ma) conj(l'[J' - ma])
        constexpr int JP = 2 * MB - 1, O = fr_seed_off(MB);
#pragma unroll
        for (int ma = 0; ma <= JP; ma++) {
            const T s = ((MB - 1 + ma) & 1) ? T(-1) : T(1);
            qs[(2 * (O + ma) + 0) * FR_THREADS] = s * st.lr[JP - ma];
            qs[(2 * (O + ma) + 1) * FR_THREADS] = -s * st.li[JP - ma];
        }
    }
}

template <typename T, int TJ, int MB, typename Acc>
__device__ __forceinline__ void fr_columns(FrState<T, TJ> &st, const typename cplx<T>::type *__restrict__ Yi,
                                           const int ys, Acc (&G)[4], T *__restrict__ qs)
{
    if constexpr (MB >= 0) {
        T pr[TJ + 1], pi[TJ + 1];
        if constexpr (MB == 0) {
            pr[0] = T(1); pi[0] = T(0);
            st.ur[0] = T(1); st.ui[0] = T(0);
        } else {
            constexpr int O = fr_seed_off(MB), JP = 2 * MB - 1;
#pragma unroll
            for (int ma = 0; ma <= JP; ma++) {
                pr[ma] = qs[(2 * (O + ma) + 0) * FR_THREADS];
                pi[ma] = qs[(2 * (O + ma) + 1) * FR_THREADS];
                st.ur[fr_row_off(JP) + ma] = pr[ma]; st.ui[fr_row_off(JP) + ma] = pi[ma];
            }
        }
        fr_col_fwd<T, TJ, (MB == 0 ? 1 : 2 * MB), MB>(st, pr, pi);
        // adjoint row of layer TJ = its weighted Y row
#pragma unroll
        for (int ma = 0; ma <= TJ; ma++) { st.lr[ma] = T(0); st.li[ma] = T(0); }
        fr_add_y<T, TJ, TJ, MB>(st, Yi, ys);
        fr_col_bwd<T, TJ, TJ, MB>(st, Yi, ys, G, qs);
        asm volatile("" ::: "memory");
        fr_columns<T, TJ, MB - 1>(st, Yi, ys, G, qs);
    }
}

// pcw (several element types): per pair cutoff and neighbour weight
// (radelem[ti] + radelem[tj]) rcutfac and wjelem[tj], cpuSnap4.cpp:813-838
// Yi: the pair's atom's Y row entries, element k at Yi[k * ys]
template <typename T, int TJ>
__device__ __forceinline__ void fr_pair(const int p, const double4 *__restrict__ prij, const int2 inf,
                                        const SnapGeom &gp, const typename cplx<T>::type *__restrict__ Yi,
                                        const int ys, double4 *__restrict__ dEslot, T *__restrict__ qs,
                                        double *__restrict__ qg, const double2 *__restrict__ pcw)
{
    typedef typename FAccSel<T>::type Acc;
    const double4 r = prij[p];
    FrState<T, TJ> st;
    {
        PairGeo g;
        if (pcw) {
            SnapGeom ge = gp;
            const double2 c = pcw[p];
            ge.rcut = c.x;
            ge.wj = c.y;
            pair_geometry<true>(g, r.x, r.y, r.z, ge);
        } else {
            pair_geometry<true>(g, r.x, r.y, r.z, gp);
        }
        st.ar = (T)g.ar; st.ai = (T)g.ai; st.br = (T)g.br; st.bi = (T)g.bi;
        // d(a,b)/dx_k and the radial terms wait in shared memory until the end
#pragma unroll
        for (int k = 0; k < 3; k++) {
            qg[(4 * k + 0) * FR_THREADS] = g.dar[k];
            qg[(4 * k + 1) * FR_THREADS] = g.dai[k];
            qg[(4 * k + 2) * FR_THREADS] = g.dbr[k];
            qg[(4 * k + 3) * FR_THREADS] = g.dbi[k];
            qg[(12 + k) * FR_THREADS] = 2.0 * g.dsfac * g.u[k];
        }
        qg[15 * FR_THREADS] = 2.0 * g.sfac;
    }
    {
        T pr[TJ + 1], pi[TJ + 1];
        fr_seeds<T, TJ, 0>(st.ar, st.ai, st.br, st.bi, pr, pi, qs);
    }
    Acc G[4];
#pragma unroll
    for (int k = 0; k < 4; k++) G[k].init(T(0));
    fr_columns<T, TJ, TJ / 2>(st, Yi, ys, G, qs);
    // after column 0, st.l[0] is the adjoint of the root u_0 = 1 (its own
    // half-weighted Y term included), whose real part is F
    const double F = (double)st.lr[0];
    const double g0 = G[0].val(), g1 = G[1].val(), g2 = G[2].val(), g3 = G[3].val();
    double o[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double dF = g0 * qg[(4 * k + 0) * FR_THREADS] + g1 * qg[(4 * k + 1) * FR_THREADS] +
                          g2 * qg[(4 * k + 2) * FR_THREADS] + g3 * qg[(4 * k + 3) * FR_THREADS];
        o[k] = qg[(12 + k) * FR_THREADS] * F + qg[15 * FR_THREADS] * dF;
    }
    dEslot[inf.y] = make_double4(o[0], o[1], o[2], 0.0);
}

template <typename T, int TJ>
__device__ __forceinline__ void fr_kernel_body(const double4 *__restrict__ prij, const int2 *__restrict__ pinfo,
                                               const int *__restrict__ pnum, const SnapGeom &gp,
                                               const typename cplx<T>::type *__restrict__ Y,
                                               double4 *__restrict__ dEslot, const double2 *__restrict__ pcw)
{
    typedef typename cplx<T>::type T2;
    constexpr int NYH = yh_count(TJ), YC = fr_ycap<T>();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int amm[2 * (FR_THREADS / 32)];
    double *qg = reinterpret_cast<double *>(smraw) + threadIdx.x;
    T *qs = reinterpret_cast<T *>(reinterpret_cast<double *>(smraw) + 16 * FR_THREADS) + threadIdx.x;
    T2 *Ys = reinterpret_cast<T2 *>(reinterpret_cast<T *>(reinterpret_cast<double *>(smraw) + 16 * FR_THREADS) +
                                    fr_seed_vals<TJ>() * FR_THREADS);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int npairs = *pnum;
    // windows of FR_THREADS consecutive pairs (the loop bound is uniform over the CTA)
    for (int base = blockIdx.x * FR_THREADS; base < npairs; base += gridDim.x * FR_THREADS) {
        const int p = base + threadIdx.x;
        int2 inf = make_int2(0, 0);
        int mn = INT_MAX, mx = INT_MIN;
        if (p < npairs) { inf = pinfo[p]; mn = mx = inf.x; }
        mn = __reduce_min_sync(0xffffffffu, mn);
        mx = __reduce_max_sync(0xffffffffu, mx);
        __syncthreads();   // the previous window is done with Ys and amm
        if (lane == 0) { amm[w] = mn; amm[FR_THREADS / 32 + w] = mx; }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < FR_THREADS / 32; v++) { mn = min(mn, amm[v]); mx = max(mx, amm[FR_THREADS / 32 + v]); }
        const int na = mx - mn + 1;   // atoms the window spans (mx >= mn: the window has a pair)
        const bool staged = na <= YC;
        if (staged) {
            for (int e = threadIdx.x; e < NYH * na; e += FR_THREADS) {
                const int k = e / na, sl = e - k * na, a = mn + sl;
                Ys[k * YC + sl] = Y[((size_t)(a >> 5) * NYH + k) * 32 + (a & 31)];
            }
            __syncthreads();
        }
        if (p < npairs) {
            const T2 *Yi = staged ? Ys + (inf.x - mn) : Y + (size_t)(inf.x >> 5) * NYH * 32 + (inf.x & 31);
            fr_pair<T, TJ>(p, prij, inf, gp, Yi, staged ? YC : 32, dEslot, qs, qg, pcw);
        }
    }
}

template <typename T, int TJ>
__global__ void __launch_bounds__(FR_THREADS)
k_snap_fr(const double4 *__restrict__ prij, const int2 *__restrict__ pinfo, const int *__restrict__ pnum,
          SnapGeom gp, const typename cplx<T>::type *__restrict__ Y, double4 *__restrict__ dEslot,
          const double2 *__restrict__ pcw = nullptr)
{
    fr_kernel_body<T, TJ>(prij, pinfo, pnum, gp, Y, dEslot, pcw);
}

// FP32: the state takes half the registers, so the kernel is held to 128 and
// four CTAs share an SM
#ifndef FR32_MINB
#define FR32_MINB 4
#endif
template <int TJ>
__global__ void __launch_bounds__(FR_THREADS, FR32_MINB)
k_snap_fr32(const double4 *__restrict__ prij, const int2 *__restrict__ pinfo, const int *__restrict__ pnum,
            SnapGeom gp, const float2 *__restrict__ Y, double4 *__restrict__ dEslot)
{
    fr_kernel_body<float, TJ>(prij, pinfo, pnum, gp, Y, dEslot, nullptr);
}

}  // namespace mdp
