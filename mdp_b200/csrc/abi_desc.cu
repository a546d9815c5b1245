// The descriptor chain of the Julia C-ABI library (src/Julia/Potential/cpuSnap.h:48-84):
// the calls snapdescriptors makes after the pair list
// (src/Julia/Potential/snapcpp.jl:539-665):
//
//   cpuComputeSij / cpuComputeUij   per-pair U and dU/dr          (cpuSnap.cpp:1412-1833)
//   cpuZeroUarraytot2               per-atom U totals = wself I   (:1835-1862)
//   cpuAddUarraytot                 U totals += pair U            (:1864-1897)
//   cpuComputeZi2                   Z per atom and coupling       (:1899-1969)
//   cpuComputeBi2                   B per atom                    (:1971-2072)
//   cpuComputeDbidrj                dB/dr per pair                (:2074-2263)
//   cpuSnapTallyBispectrum{,Deriv,Virial}  sums of B, dB, virial  (:2265-2472)
//
// Host arrays in and out, computed on the GPU in the reference's layouts:
// per-pair arrays [k][ijnum] (pair fastest; dU as three such blocks, x y z),
// per-atom arrays [k][inum] (atom fastest), dblist [jjb][3][ijnum].  The index
// and Clebsch-Gordan tables are the caller's own (cpuInitSna's).  Each output
// entry is produced with the reference's sequence of additions:
//  * U / dU write exactly the entries the reference writes (the left half
//    plane, the mirrored right half of U, and of dU only the row above the
//    middle of odd layers) and leave the rest of the caller's arrays as they
//    were;
//  * U totals and the dB tally add each atom's pairs in ascending pair order.
// The sums of the B and virial tallies run as fixed shared-memory trees.
// One element type (nelements = 1, chemflag = 0); pair types may differ
// (per-pair cutoffs); quadraticflag is supported in the tallies.
#include "common.cuh"
#include "engine.h"

#include <algorithm>
#include <mutex>
#include <vector>

namespace mdp {
namespace {

std::mutex g_desc_mu;

// ---------------------------------------------------------------------------
// per-pair U and dU/dr
// ---------------------------------------------------------------------------
struct PairArrays {
    double *ur, *ui;
    double *dr[3], *di[3];   // may be null (no derivatives)
};

__global__ void k_desc_uij(const double *__restrict__ rij, const int *__restrict__ ti, const int *__restrict__ tj,
                           const double *__restrict__ radelem, const double *__restrict__ wjelem, double rcutfac,
                           double rmin0, double rfac0, int switchflag, const double *__restrict__ rootpq,
                           const int *__restrict__ ublock, int twojmax, int idxu_max, int ijnum, PairArrays A)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ijnum) return;
    const size_t S = (size_t)ijnum;
    const int jdim = twojmax + 1;
    SnapGeom gp;
    gp.rcut = (radelem[ti[p]] + radelem[tj[p]]) * rcutfac;
    gp.rcutsq = gp.rcut * gp.rcut;
    gp.rfac0 = rfac0;
    gp.rmin0 = rmin0;
    gp.wj = wjelem[tj[p]];
    gp.switchflag = switchflag;
    PairGeo g;
    pair_geometry<true>(g, rij[3 * (size_t)p], rij[3 * (size_t)p + 1], rij[3 * (size_t)p + 2], gp);
    if (switchflag != 0 && switchflag != 1) { g.sfac = 0.0; g.dsfac = 0.0; }   // neither branch sets sfac
    const bool der = A.dr[0] != nullptr;
    double *__restrict__ ur = A.ur;
    double *__restrict__ ui = A.ui;
    auto at = [&](int k) { return (size_t)k * S + p; };

    ur[at(0)] = 1.0;
    ui[at(0)] = 0.0;
    if (der)
        for (int d = 0; d < 3; d++) { A.dr[d][at(0)] = 0.0; A.di[d][at(0)] = 0.0; }
    for (int j = 1; j <= twojmax; j++) {
        const int base = ublock[j], prev = ublock[j - 1];
        // rows mb <= j/2 from the same rows of layer j-1 (row length j there):
        // entry ma takes -c_b conj(b) u[ma-1] first, then + c_a conj(a) u[ma]
        for (int mb = 0; 2 * mb <= j; mb++) {
            for (int ma = 0; ma <= j; ma++) {
                double vr = 0.0, vi = 0.0, wr[3] = {0.0, 0.0, 0.0}, wi[3] = {0.0, 0.0, 0.0};
                if (ma > 0) {
                    const size_t q = at(prev + j * mb + ma - 1);
                    const double c = rootpq[ma * jdim + (j - mb)];
                    const double pr = ur[q], pim = ui[q];
                    vr = -c * (g.br * pr + g.bi * pim);
                    vi = -c * (g.br * pim - g.bi * pr);
                    if (der)
                        for (int d = 0; d < 3; d++) {
                            const double qr = A.dr[d][q], qi = A.di[d][q];
                            wr[d] = -c * (g.dbr[d] * pr + g.dbi[d] * pim + g.br * qr + g.bi * qi);
                            wi[d] = -c * (g.dbr[d] * pim - g.dbi[d] * pr + g.br * qi - g.bi * qr);
                        }
                }
                if (ma < j) {
                    const size_t q = at(prev + j * mb + ma);
                    const double c = rootpq[(j - ma) * jdim + (j - mb)];
                    const double pr = ur[q], pim = ui[q];
                    vr += c * (g.ar * pr + g.ai * pim);
                    vi += c * (g.ar * pim - g.ai * pr);
                    if (der)
                        for (int d = 0; d < 3; d++) {
                            const double qr = A.dr[d][q], qi = A.di[d][q];
                            wr[d] += c * (g.dar[d] * pr + g.dai[d] * pim + g.ar * qr + g.ai * qi);
                            wi[d] += c * (g.dar[d] * pim - g.dai[d] * pr + g.ar * qi - g.ai * qr);
                        }
                }
                const size_t o = at(base + (j + 1) * mb + ma);
                ur[o] = vr;
                ui[o] = vi;
                if (der)
                    for (int d = 0; d < 3; d++) { A.dr[d][o] = wr[d]; A.di[d][o] = wi[d]; }
            }
        }
        // inversion symmetry u(j-mb, j-ma) = (-1)^(ma+mb) conj u(mb, ma), in
        // place and in this order (a middle row reads entries it has already
        // mirrored); dU follows only for the row above the middle of odd layers
        const int last = base + (j + 1) * (j + 1) - 1;
        for (int mb = 0; 2 * mb <= j; mb++) {
            const bool dmirror = der && (j % 2 == 1) && (mb == j / 2);
            for (int ma = 0; ma <= j; ma++) {
                const int s = base + (j + 1) * mb + ma;
                const size_t src = at(s), dst = at(last - (s - base));
                const double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
                ur[dst] = sg * ur[src];
                ui[dst] = -sg * ui[src];
                if (dmirror)
                    for (int d = 0; d < 3; d++) {
                        A.dr[d][dst] = sg * A.dr[d][src];
                        A.di[d][dst] = -sg * A.di[d][src];
                    }
            }
        }
    }
    // switching function: dU = dsfac u_hat U + sfac dU on the left half plane,
    // then U *= sfac everywhere
    if (der)
        for (int j = 0; j <= twojmax; j++)
            for (int mb = 0; 2 * mb <= j; mb++)
                for (int ma = 0; ma <= j; ma++) {
                    const size_t k = at(ublock[j] + (j + 1) * mb + ma);
                    for (int d = 0; d < 3; d++) {
                        A.dr[d][k] = g.dsfac * ur[k] * g.u[d] + g.sfac * A.dr[d][k];
                        A.di[d][k] = g.dsfac * ui[k] * g.u[d] + g.sfac * A.di[d][k];
                    }
                }
    for (int k = 0; k < idxu_max; k++) {
        ur[at(k)] = g.sfac * ur[at(k)];
        ui[at(k)] = g.sfac * ui[at(k)];
    }
}

// ---------------------------------------------------------------------------
// per-atom lists of pairs, ascending in pair index.  key[p] names the atom of
// pair p; with two keys, entries are 2p (first key) and 2p+1 (second key).
// ---------------------------------------------------------------------------
__global__ void k_list_count(const int *__restrict__ k0, const int *__restrict__ k1, int n, int *__restrict__ cnt)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    atomicAdd(&cnt[k0[p]], 1);
    if (k1) atomicAdd(&cnt[k1[p]], 1);
}

__global__ void k_list_fill(const int *__restrict__ k0, const int *__restrict__ k1, int n, const int *__restrict__ off,
                            int *__restrict__ cursor, int *__restrict__ list)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int a = k0[p];
    list[off[a] + atomicAdd(&cursor[a], 1)] = k1 ? 2 * p : p;
    if (k1) {
        const int b = k1[p];
        list[off[b] + atomicAdd(&cursor[b], 1)] = 2 * p + 1;
    }
}

__global__ void k_list_sort(int natoms, const int *__restrict__ off, int *__restrict__ list)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= natoms) return;
    const int s = off[a], e = off[a + 1];
    for (int x = s + 1; x < e; x++) {
        const int v = list[x];
        int y = x - 1;
        while (y >= s && list[y] > v) { list[y + 1] = list[y]; y--; }
        list[y + 1] = v;
    }
}

struct AtomLists {
    DevBuf cnt, off, cursor, list, tmp;
    ~AtomLists()
    {
        DevBuf *b[] = {&cnt, &off, &cursor, &list, &tmp};
        for (auto x : b) x->release();
    }
};

int atom_lists(AtomLists &L, const int *k0, const int *k1, int n, int natoms)
{
    const size_t entries = (size_t)n * (k1 ? 2 : 1);
    if (L.cnt.ensure(sizeof(int) * (natoms + 1)) || L.off.ensure(sizeof(int) * (natoms + 1)) ||
        L.cursor.ensure(sizeof(int) * (natoms + 1)) || L.list.ensure(sizeof(int) * std::max<size_t>(entries, 1)) ||
        L.tmp.ensure(sizeof(int) * scan_tmp_ints(natoms)))
        return -1;
    MDP_CUDA_TRY(cudaMemset(L.cnt.p, 0, sizeof(int) * natoms));
    MDP_CUDA_TRY(cudaMemset(L.cursor.p, 0, sizeof(int) * natoms));
    const int tb = 256;
    if (n > 0) k_list_count<<<(n + tb - 1) / tb, tb>>>(k0, k1, n, L.cnt.as<int>());
    if (exclusive_scan(L.cnt.as<int>(), L.off.as<int>(), natoms, L.tmp.as<int>(), 0)) return -1;
    if (n > 0) k_list_fill<<<(n + tb - 1) / tb, tb>>>(k0, k1, n, L.off.as<int>(), L.cursor.as<int>(), L.list.as<int>());
    k_list_sort<<<(natoms + tb - 1) / tb, tb>>>(natoms, L.off.as<int>(), L.list.as<int>());
    count_launches(4);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// per-atom U totals
// ---------------------------------------------------------------------------
__global__ void k_desc_utot_init(double *__restrict__ sr, double *__restrict__ si, double wself,
                                 const int *__restrict__ ublock, int twojmax, int idxu_max, int inum)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)idxu_max * inum) return;
    const int k = (int)(e / inum);
    int j = 0;
    while (j < twojmax && ublock[j + 1] <= k) j++;
    const int rem = k - ublock[j], mb = rem / (j + 1), ma = rem - mb * (j + 1);
    sr[e] = (ma == mb) ? wself : 0.0;
    si[e] = 0.0;
}

__global__ void k_desc_utot_add(double *__restrict__ tr, double *__restrict__ tim, const double *__restrict__ sr,
                                const double *__restrict__ si, const int *__restrict__ off,
                                const int *__restrict__ list, int idxu_max, int inum, int ijnum)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)idxu_max * inum) return;
    const int a = (int)(e % inum), k = (int)(e / inum);
    double vr = tr[e], vi = tim[e];
    for (int x = off[a]; x < off[a + 1]; x++) {
        const size_t q = (size_t)k * ijnum + list[x];
        vr += sr[q];
        vi += si[q];
    }
    tr[e] = vr;
    tim[e] = vi;
}

// ---------------------------------------------------------------------------
// Z, B, dB/dr from the caller's tables
// ---------------------------------------------------------------------------
__global__ void k_desc_zi(double *__restrict__ zr, double *__restrict__ zi, const double *__restrict__ tr,
                          const double *__restrict__ tim, const double *__restrict__ cglist,
                          const int *__restrict__ idxz, const int *__restrict__ ublock,
                          const int *__restrict__ cgblock, int twojmax, int idxz_max, int bnorm, int inum)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)idxz_max * inum) return;
    const int a = (int)(e % inum), jjz = (int)(e / inum);
    const int jdim = twojmax + 1;
    const int *z = idxz + 10 * (size_t)jjz;
    const int j1 = z[0], j2 = z[1], j = z[2], ma1min = z[3], ma2max = z[4], na = z[5], mb1min = z[6],
              mb2max = z[7], nb = z[8];
    const double *cg = cglist + cgblock[j + j2 * jdim + j1 * jdim * jdim];
    int row1 = ublock[j1] + (j1 + 1) * mb1min, row2 = ublock[j2] + (j2 + 1) * mb2max;
    int cb = mb1min * (j2 + 1) + mb2max;
    double qr = 0.0, qi = 0.0;
    for (int ib = 0; ib < nb; ib++) {
        double sr = 0.0, si = 0.0;
        int ca = ma1min * (j2 + 1) + ma2max;
        for (int ia = 0; ia < na; ia++) {
            const size_t u1 = (size_t)(row1 + ma1min + ia) * inum + a, u2 = (size_t)(row2 + ma2max - ia) * inum + a;
            const double ar = tr[u1], ai = tim[u1], br = tr[u2], bi = tim[u2];
            sr += cg[ca] * (ar * br - ai * bi);
            si += cg[ca] * (ar * bi + ai * br);
            ca += j2;
        }
        qr += cg[cb] * sr;
        qi += cg[cb] * si;
        row1 += j1 + 1;
        row2 -= j2 + 1;
        cb += j2;
    }
    if (bnorm) {
        qr /= (j + 1);
        qi /= (j + 1);
    }
    zr[e] = qr;
    zi[e] = qi;
}

// half-plane contraction of one layer-jl block of U-like entries (per-entry
// reader ua) with the Z block starting at jjz: full rows 2mb < jl, then for
// even jl the middle row up to its centre, which counts half
template <typename UA, typename ACC>
__device__ __forceinline__ void half_plane(int jl, int jju, int jjz, UA ua, ACC acc)
{
    for (int mb = 0; 2 * mb < jl; mb++)
        for (int ma = 0; ma <= jl; ma++) acc(ua(jju++), jjz++, 1.0);
    if (jl % 2 == 0) {
        const int mb = jl / 2;
        for (int ma = 0; ma < mb; ma++) acc(ua(jju++), jjz++, 1.0);
        acc(ua(jju), jjz, 0.5);
    }
}

__global__ void k_desc_bi(double *__restrict__ blist, const double *__restrict__ zr, const double *__restrict__ zi,
                          const double *__restrict__ tr, const double *__restrict__ tim,
                          const double *__restrict__ bzero, const int *__restrict__ idxb,
                          const int *__restrict__ ublock, const int *__restrict__ zblock, int twojmax, int idxb_max,
                          int bzero_flag, int inum)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)idxb_max * inum) return;
    const int a = (int)(e % inum), jjb = (int)(e / inum);
    const int jdim = twojmax + 1;
    const int j1 = idxb[3 * jjb], j2 = idxb[3 * jjb + 1], j = idxb[3 * jjb + 2];
    double s = 0.0;
    half_plane(
        j, ublock[j], zblock[j + j2 * jdim + j1 * jdim * jdim], [&](int k) { return (size_t)k * inum + a; },
        [&](size_t u, int jjz, double w) {
            const size_t z = (size_t)jjz * inum + a;
            const double t = tr[u] * zr[z] + tim[u] * zi[z];
            s += (w == 1.0) ? t : w * t;
        });
    double b = 2.0 * s;
    if (bzero_flag) b -= bzero[j];
    blist[e] = b;
}

__global__ void k_desc_dbidrj(double *__restrict__ db, const double *__restrict__ zr, const double *__restrict__ zi,
                              const double *__restrict__ dur, const double *__restrict__ dui,
                              const int *__restrict__ idxb, const int *__restrict__ ublock,
                              const int *__restrict__ zblock, const int *__restrict__ ai, int twojmax, int idxb_max,
                              int idxu_max, int bnorm, int inum, int ijnum)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)idxb_max * ijnum) return;
    const int p = (int)(e % ijnum), jjb = (int)(e / ijnum);
    const int jdim = twojmax + 1, i = ai[p];
    const size_t nu = (size_t)idxu_max * ijnum;
    const int j1 = idxb[3 * jjb], j2 = idxb[3 * jjb + 1], j = idxb[3 * jjb + 2];
    double out[3] = {0.0, 0.0, 0.0};
    // the three terms: conj(dU_j) Z(j1,j2,j), conj(dU_j1) Z(j,j2,j1) (j+1)/(j1+1),
    // conj(dU_j2) Z(j,j1,j2) (j+1)/(j2+1); bnorm drops the factors
    const int layer[3] = {j, j1, j2};
    const int zstart[3] = {zblock[j + j2 * jdim + j1 * jdim * jdim], zblock[j1 + j2 * jdim + j * jdim * jdim],
                           zblock[j2 + j1 * jdim + j * jdim * jdim]};
    const double fac[3] = {1.0, bnorm ? 1.0 : (j + 1) / (j1 + 1.0), bnorm ? 1.0 : (j + 1) / (j2 + 1.0)};
    for (int t = 0; t < 3; t++) {
        double s[3] = {0.0, 0.0, 0.0};
        half_plane(
            layer[t], ublock[layer[t]], zstart[t], [&](int k) { return (size_t)k * ijnum + p; },
            [&](size_t u, int jjz, double w) {
                const size_t z = (size_t)jjz * inum + i;
                const double a = zr[z], b = zi[z];
                for (int d = 0; d < 3; d++) {
                    const double v = dur[u + nu * d] * a + dui[u + nu * d] * b;
                    s[d] += (w == 1.0) ? v : v * w;
                }
            });
        for (int d = 0; d < 3; d++) out[d] += (t == 0) ? 2.0 * s[d] : 2.0 * s[d] * fac[t];
    }
    for (int d = 0; d < 3; d++) db[(size_t)p + (size_t)ijnum * d + (size_t)ijnum * 3 * jjb] = out[d];
}

// ---------------------------------------------------------------------------
// tallies.  A slot c < nperdim is either linear (coefficient lin[c]) or the
// quadratic product of coefficients (qa[c], qb[c]) (cpuSnap.cpp:2265-2472).
// ---------------------------------------------------------------------------
struct SlotMap {
    const int *ca, *cb;   // cb[c] < 0: linear slot of coefficient ca[c]; ca == cb: half square
};

constexpr int TALLY_T = 256;

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = TALLY_T / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// one CTA per (type, slot).  In the quadratic slots this tally keeps the
// reference's placement (cpuSnap.cpp:2280-2287, a post-increment): the slot
// of (a, a+m) holds B_a B_(a+m+1), and the half square 0.5 B_a^2 shares the
// first slot with B_a B_(a+1).
__global__ void __launch_bounds__(TALLY_T)
k_tally_b(double *__restrict__ bi, const double *__restrict__ B, const int *__restrict__ ilist,
          const int *__restrict__ type, int inum, int ncoeff, int nperdim, SlotMap sm)
{
    __shared__ double sh[TALLY_T];
    const int c = blockIdx.x % nperdim, t = blockIdx.x / nperdim + 1;
    const int a = sm.ca[c], b = sm.cb[c];
    double v = 0.0;
    if (a >= 0)
        for (int ii = threadIdx.x; ii < inum; ii += TALLY_T) {
            if (type[ilist[ii]] != t) continue;
            const double x = B[ii + (size_t)inum * a];
            if (b < 0) {
                v += x;
            } else {
                if (a == b) v += 0.5 * x * x;
                if (b + 1 < ncoeff) v += x * B[ii + (size_t)inum * (b + 1)];
            }
        }
    v = block_sum(v, sh);
    if (threadIdx.x == 0) bi[blockIdx.x] = v;
}

// dB/dR contribution of pair p to slot c, component d
__device__ __forceinline__ double slot_db(const double *__restrict__ B, const double *__restrict__ dbdr,
                                          const int *__restrict__ aii, int p, int d, int a, int b, int inum, int ijnum)
{
    const double x = dbdr[p + (size_t)ijnum * d + (size_t)ijnum * 3 * a];
    if (b < 0) return x;
    const double ba = B[aii[p] + (size_t)inum * a];
    if (a == b) return ba * x;
    return ba * dbdr[p + (size_t)ijnum * d + (size_t)ijnum * 3 * b] + x * B[aii[p] + (size_t)inum * b];
}

// one thread per (atom, slot): the atom's pairs in ascending order, + as the
// pair's i, - as its j; the pair's type block is that of its atom i
__global__ void k_tally_db(double *__restrict__ db, const double *__restrict__ B, const double *__restrict__ dbdr,
                           const int *__restrict__ aii, const int *__restrict__ ti, const int *__restrict__ off,
                           const int *__restrict__ list, int inum, int ijnum, int nperdim, SlotMap sm)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)inum * nperdim) return;
    const int o = (int)(e % inum), c = (int)(e / inum);
    const int a = sm.ca[c], b = sm.cb[c];
    if (a < 0) return;
    for (int x = off[o]; x < off[o + 1]; x++) {
        const int p = list[x] >> 1;
        const double sg = (list[x] & 1) ? -1.0 : 1.0;
        double *dst = db + 3 * (size_t)o + (size_t)inum * 3 * (c + (size_t)nperdim * (ti[p] - 1));
        for (int d = 0; d < 3; d++) dst[d] += sg * slot_db(B, dbdr, aii, p, d, a, b, inum, ijnum);
    }
}

// one CTA per (type, slot): the six components of -r (x) dB
__global__ void __launch_bounds__(TALLY_T)
k_tally_bv(double *__restrict__ bv, const double *__restrict__ B, const double *__restrict__ dbdr,
           const double *__restrict__ rij, const int *__restrict__ aii, const int *__restrict__ ti, int inum,
           int ijnum, int nperdim, SlotMap sm)
{
    __shared__ double sh[TALLY_T];
    const int c = blockIdx.x % nperdim, t = blockIdx.x / nperdim + 1;
    const int a = sm.ca[c], b = sm.cb[c];
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (a >= 0)
        for (int p = threadIdx.x; p < ijnum; p += TALLY_T) {
            if (ti[p] != t) continue;
            const double dx = -rij[3 * (size_t)p], dy = -rij[3 * (size_t)p + 1], dz = -rij[3 * (size_t)p + 2];
            const double gx = slot_db(B, dbdr, aii, p, 0, a, b, inum, ijnum);
            const double gy = slot_db(B, dbdr, aii, p, 1, a, b, inum, ijnum);
            const double gz = slot_db(B, dbdr, aii, p, 2, a, b, inum, ijnum);
            v[0] += dx * gx; v[1] += dy * gy; v[2] += dz * gz;
            v[3] += dx * gy; v[4] += dx * gz; v[5] += dy * gz;
        }
    for (int k = 0; k < 6; k++) {
        const double s = block_sum(v[k], sh);
        if (threadIdx.x == 0) bv[k + 6 * (size_t)blockIdx.x] = s;
    }
}

// slot table for nperdim slots: linear coefficients first, then the pairs
// (i, j >= i) in the reference's order
int slot_map(std::vector<int> &ca, std::vector<int> &cb, int ncoeff, int nperdim, int quadratic)
{
    const int need = quadratic ? ncoeff + ncoeff * (ncoeff + 1) / 2 : ncoeff;
    if (nperdim < need) {
        set_error("nperdim %d is smaller than the %d slots of ncoeff %d%s", nperdim, need, ncoeff,
                  quadratic ? " with quadratic terms" : "");
        return -1;
    }
    ca.assign(nperdim, -1);
    cb.assign(nperdim, -1);
    for (int c = 0; c < ncoeff; c++) ca[c] = c;
    if (quadratic) {
        int k = ncoeff;
        for (int i = 0; i < ncoeff; i++)
            for (int j = i; j < ncoeff; j++, k++) { ca[k] = i; cb[k] = j; }
    }
    return 0;
}

// host staging (every call: arrays in, compute, arrays out)
struct Stage2 {
    std::vector<void *> ptrs;
    bool ok = true;
    template <typename X> X *in(const X *h, size_t n)
    {
        X *d = alloc<X>(n);
        if (d && n && cudaMemcpy(d, h, sizeof(X) * n, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
        return d;
    }
    template <typename X> X *alloc(size_t n)
    {
        X *d = nullptr;
        if (!ok || cudaMalloc(&d, sizeof(X) * std::max<size_t>(n, 1)) != cudaSuccess) { ok = false; return nullptr; }
        ptrs.push_back(d);
        return d;
    }
    template <typename X> X *zeros(size_t n)
    {
        X *d = alloc<X>(n);
        if (d && cudaMemset(d, 0, sizeof(X) * std::max<size_t>(n, 1)) != cudaSuccess) ok = false;
        return d;
    }
    template <typename X> int out(X *h, const X *d, size_t n)
    {
        if (!ok || cudaDeviceSynchronize() != cudaSuccess) return -1;
        return (n && cudaMemcpy(h, d, sizeof(X) * n, cudaMemcpyDeviceToHost) != cudaSuccess) ? -1 : 0;
    }
    ~Stage2()
    {
        for (void *p : ptrs) cudaFree(p);
    }
};

unsigned grid_of(long n, int tb) { return (unsigned)std::max<long>(1, (n + tb - 1) / tb); }

int max_of(const int *a, long n)
{
    int m = 0;
    for (long i = 0; i < n; i++) m = std::max(m, a[i]);
    return m;
}

bool single_element(int nelements, int chemflag, const char *fn)
{
    if (nelements != 1 || chemflag) {
        set_error("%s: only one element type is supported (nelements %d, chemflag %d)", fn, nelements, chemflag);
        return false;
    }
    return true;
}

void uij_common(const char *fn, double *Sr, double *Si, double *const dr[3], double *const di[3],
                const double *rootpq, const double *rij, const double *wjelem, const double *radelem, double rmin0,
                double rfac0, double rcutfac, const int *idxu_block, const int *ti, const int *tj, int twojmax,
                int idxu_max, int ijnum, int switch_flag)
{
    if (twojmax < 0 || idxu_max != idxu_count(twojmax)) { set_error("%s: idxu_max does not match twojmax", fn); return; }
    if (ijnum <= 0) return;
    const int ntype = std::max(max_of(ti, ijnum), max_of(tj, ijnum)) + 1;
    const int jdim = twojmax + 1;
    const size_t n = (size_t)idxu_max * ijnum;
    Stage2 st;
    PairArrays A;
    A.ur = st.in(Sr, n);
    A.ui = st.in(Si, n);
    for (int d = 0; d < 3; d++) { A.dr[d] = st.in(dr[d], n); A.di[d] = st.in(di[d], n); }
    const double *drij = st.in(rij, 3 * (size_t)ijnum), *drootpq = st.in(rootpq, (size_t)jdim * jdim);
    const double *drad = st.in(radelem, ntype), *dwj = st.in(wjelem, ntype);
    const int *dub = st.in(idxu_block, jdim), *dti = st.in(ti, ijnum), *dtj = st.in(tj, ijnum);
    if (!st.ok) { set_error("%s: staging failed", fn); return; }
    k_desc_uij<<<grid_of(ijnum, 128), 128>>>(drij, dti, dtj, drad, dwj, rcutfac, rmin0, rfac0, switch_flag, drootpq,
                                              dub, twojmax, idxu_max, ijnum, A);
    count_launches(1);
    if (st.out(Sr, A.ur, n) || st.out(Si, A.ui, n)) { set_error("%s: copy-back failed", fn); return; }
    for (int d = 0; d < 3; d++)
        if (st.out(dr[d], A.dr[d], n) || st.out(di[d], A.di[d], n)) { set_error("%s: copy-back failed", fn); return; }
}

}  // namespace
}  // namespace mdp

using namespace mdp;

extern "C" {

// cpuSnap.h:48-50; src/Julia/Potential/cpuSnap.cpp:1412-1618
void cpuComputeSij(double *Sr, double *Si, double *Srx, double *Six, double *Sry, double *Siy, double *Srz,
                   double *Siz, double *rootpqarray, double *rij, double *wjelem, double *radelem, double rmin0,
                   double rfac0, double rcutfac, int *idxu_block, int *ti, int *tj, int twojmax, int idxu_max,
                   int ijnum, int switch_flag)
{
    std::lock_guard<std::mutex> lk(g_desc_mu);
    double *dr[3] = {Srx, Sry, Srz}, *di[3] = {Six, Siy, Siz};
    uij_common("cpuComputeSij", Sr, Si, dr, di, rootpqarray, rij, wjelem, radelem, rmin0, rfac0, rcutfac,
               idxu_block, ti, tj, twojmax, idxu_max, ijnum, switch_flag);
}

// cpuSnap.h:52-54; src/Julia/Potential/cpuSnap.cpp:1620-1833.  dSr / dSi hold
// the x, y and z blocks of idxu_max * ijnum entries each.
void cpuComputeUij(double *Sr, double *Si, double *dSr, double *dSi, double *rootpqarray, double *rij,
                   double *wjelem, double *radelem, double rmin0, double rfac0, double rcutfac, int *idxu_block,
                   int *ti, int *tj, int twojmax, int idxu_max, int ijnum, int switch_flag)
{
    std::lock_guard<std::mutex> lk(g_desc_mu);
    const size_t n = (size_t)idxu_max * std::max(ijnum, 0);
    double *dr[3] = {dSr, dSr + n, dSr + 2 * n}, *di[3] = {dSi, dSi + n, dSi + 2 * n};
    uij_common("cpuComputeUij", Sr, Si, dr, di, rootpqarray, rij, wjelem, radelem, rmin0, rfac0, rcutfac,
               idxu_block, ti, tj, twojmax, idxu_max, ijnum, switch_flag);
}

// cpuSnap.h:56-58; src/Julia/Potential/cpuSnap.cpp:1835-1862
void cpuZeroUarraytot2(double *Stotr, double *Stoti, double wself, int *idxu_block, int *type, int *map, int *ai,
                       int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax, int inum)
{
    (void)type; (void)map; (void)ai; (void)wselfall_flag;   // one element: wself on every diagonal
    std::lock_guard<std::mutex> lk(g_desc_mu);
    if (!single_element(nelements, chemflag, "cpuZeroUarraytot2")) return;
    if (idxu_max != idxu_count(twojmax)) { set_error("cpuZeroUarraytot2: idxu_max does not match twojmax"); return; }
    if (inum <= 0) return;
    const size_t n = (size_t)idxu_max * inum;
    Stage2 st;
    double *tr = st.alloc<double>(n), *ti = st.alloc<double>(n);
    const int *dub = st.in(idxu_block, twojmax + 1);
    if (!st.ok) { set_error("cpuZeroUarraytot2: staging failed"); return; }
    k_desc_utot_init<<<grid_of((long)n, 256), 256>>>(tr, ti, wself, dub, twojmax, idxu_max, inum);
    count_launches(1);
    if (st.out(Stotr, tr, n) || st.out(Stoti, ti, n)) set_error("cpuZeroUarraytot2: copy-back failed");
}

// cpuSnap.h:60-61; src/Julia/Potential/cpuSnap.cpp:1864-1897
void cpuAddUarraytot(double *Stotr, double *Stoti, double *Sr, double *Si, int *map, int *ai, int *tj, int idxu_max,
                     int inum, int ijnum, int chemflag)
{
    (void)map; (void)tj;
    std::lock_guard<std::mutex> lk(g_desc_mu);
    if (!single_element(1, chemflag, "cpuAddUarraytot")) return;
    if (inum <= 0 || ijnum <= 0) return;
    for (int p = 0; p < ijnum; p++)
        if (ai[p] < 0 || ai[p] >= inum) { set_error("cpuAddUarraytot: ai[%d] = %d outside 0..%d", p, ai[p], inum - 1); return; }
    const size_t nt = (size_t)idxu_max * inum, np = (size_t)idxu_max * ijnum;
    Stage2 st;
    double *tr = st.in(Stotr, nt), *tim = st.in(Stoti, nt);
    const double *sr = st.in(Sr, np), *si = st.in(Si, np);
    const int *dai = st.in(ai, ijnum);
    if (!st.ok) { set_error("cpuAddUarraytot: staging failed"); return; }
    AtomLists L;
    if (atom_lists(L, dai, nullptr, ijnum, inum)) return;
    k_desc_utot_add<<<grid_of((long)nt, 256), 256>>>(tr, tim, sr, si, L.off.as<int>(), L.list.as<int>(), idxu_max,
                                                      inum, ijnum);
    count_launches(1);
    if (st.out(Stotr, tr, nt) || st.out(Stoti, tim, nt)) set_error("cpuAddUarraytot: copy-back failed");
}

// cpuSnap.h:63-65; src/Julia/Potential/cpuSnap.cpp:1899-1969
void cpuComputeZi2(double *zlist_r, double *zlist_i, double *Stotr, double *Stoti, double *cglist, int *idxz,
                   int *idxu_block, int *idxcg_block, int twojmax, int idxu_max, int idxz_max, int nelements,
                   int bnorm_flag, int inum)
{
    std::lock_guard<std::mutex> lk(g_desc_mu);
    if (!single_element(nelements, 0, "cpuComputeZi2")) return;
    if (idxu_max != idxu_count(twojmax)) { set_error("cpuComputeZi2: idxu_max does not match twojmax"); return; }
    if (inum <= 0) return;
    const int jdim = twojmax + 1;
    const size_t nu = (size_t)idxu_max * inum, nz = (size_t)idxz_max * inum;
    int ncg = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(twojmax, j1 + j2); j += 2) ncg += (j1 + 1) * (j2 + 1);
    Stage2 st;
    double *zr = st.alloc<double>(nz), *zi = st.alloc<double>(nz);
    const double *tr = st.in(Stotr, nu), *tim = st.in(Stoti, nu), *cg = st.in(cglist, ncg);
    const int *dz = st.in(idxz, 10 * (size_t)idxz_max), *dub = st.in(idxu_block, jdim),
              *dcb = st.in(idxcg_block, (size_t)jdim * jdim * jdim);
    if (!st.ok) { set_error("cpuComputeZi2: staging failed"); return; }
    k_desc_zi<<<grid_of((long)nz, 128), 128>>>(zr, zi, tr, tim, cg, dz, dub, dcb, twojmax, idxz_max, bnorm_flag, inum);
    count_launches(1);
    if (st.out(zlist_r, zr, nz) || st.out(zlist_i, zi, nz)) set_error("cpuComputeZi2: copy-back failed");
}

// cpuSnap.h:67-70; src/Julia/Potential/cpuSnap.cpp:1971-2072
void cpuComputeBi2(double *blist, double *zlist_r, double *zlist_i, double *Stotr, double *Stoti, double *bzero,
                   int *ilist, int *type, int *map, int *idxb, int *idxu_block, int *idxz_block, int twojmax,
                   int idxb_max, int idxu_max, int idxz_max, int nelements, int bzero_flag, int wselfall_flag,
                   int chemflag, int inum)
{
    (void)ilist; (void)type; (void)map; (void)wselfall_flag;   // one element: both bzero forms agree
    std::lock_guard<std::mutex> lk(g_desc_mu);
    if (!single_element(nelements, chemflag, "cpuComputeBi2")) return;
    if (idxu_max != idxu_count(twojmax)) { set_error("cpuComputeBi2: idxu_max does not match twojmax"); return; }
    if (inum <= 0) return;
    const int jdim = twojmax + 1;
    const size_t nu = (size_t)idxu_max * inum, nz = (size_t)idxz_max * inum, nb = (size_t)idxb_max * inum;
    Stage2 st;
    double *db = st.alloc<double>(nb);
    const double *zr = st.in(zlist_r, nz), *zi = st.in(zlist_i, nz), *tr = st.in(Stotr, nu), *tim = st.in(Stoti, nu),
                 *bz = st.in(bzero, jdim);
    const int *dib = st.in(idxb, 3 * (size_t)idxb_max), *dub = st.in(idxu_block, jdim),
              *dzb = st.in(idxz_block, (size_t)jdim * jdim * jdim);
    if (!st.ok) { set_error("cpuComputeBi2: staging failed"); return; }
    k_desc_bi<<<grid_of((long)nb, 128), 128>>>(db, zr, zi, tr, tim, bz, dib, dub, dzb, twojmax, idxb_max, bzero_flag,
                                                inum);
    count_launches(1);
    if (st.out(blist, db, nb)) set_error("cpuComputeBi2: copy-back failed");
}

// cpuSnap.h:72-75; src/Julia/Potential/cpuSnap.cpp:2074-2263
void cpuComputeDbidrj(double *dblist, double *zlist_r, double *zlist_i, double *dulist_r, double *dulist_i, int *idxb,
                      int *idxu_block, int *idxz_block, int *map, int *ai, int *tj, int twojmax, int idxb_max,
                      int idxu_max, int idxz_max, int nelements, int bnorm_flag, int chemflag, int inum, int ijnum)
{
    (void)map; (void)tj;
    std::lock_guard<std::mutex> lk(g_desc_mu);
    if (!single_element(nelements, chemflag, "cpuComputeDbidrj")) return;
    if (idxu_max != idxu_count(twojmax)) { set_error("cpuComputeDbidrj: idxu_max does not match twojmax"); return; }
    if (ijnum <= 0 || inum <= 0) return;
    for (int p = 0; p < ijnum; p++)
        if (ai[p] < 0 || ai[p] >= inum) { set_error("cpuComputeDbidrj: ai[%d] = %d outside 0..%d", p, ai[p], inum - 1); return; }
    const int jdim = twojmax + 1;
    const size_t nz = (size_t)idxz_max * inum, ndu = 3 * (size_t)idxu_max * ijnum, ndb = 3 * (size_t)idxb_max * ijnum;
    Stage2 st;
    double *db = st.alloc<double>(ndb);
    const double *zr = st.in(zlist_r, nz), *zi = st.in(zlist_i, nz), *dur = st.in(dulist_r, ndu),
                 *dui = st.in(dulist_i, ndu);
    const int *dib = st.in(idxb, 3 * (size_t)idxb_max), *dub = st.in(idxu_block, jdim),
              *dzb = st.in(idxz_block, (size_t)jdim * jdim * jdim), *dai = st.in(ai, ijnum);
    if (!st.ok) { set_error("cpuComputeDbidrj: staging failed"); return; }
    k_desc_dbidrj<<<grid_of((long)idxb_max * ijnum, 128), 128>>>(db, zr, zi, dur, dui, dib, dub, dzb, dai, twojmax,
                                                                  idxb_max, idxu_max, bnorm_flag, inum, ijnum);
    count_launches(1);
    if (st.out(dblist, db, ndb)) set_error("cpuComputeDbidrj: copy-back failed");
}

// cpuSnap.h:77-78; src/Julia/Potential/cpuSnap.cpp:2265-2291
void cpuSnapTallyBispectrum(double *bi, double *bispectrum, int *ilist, int *type, int inum, int ncoeff, int nperdim,
                            int ntype, int quadraticflag)
{
    std::lock_guard<std::mutex> lk(g_desc_mu);
    std::vector<int> ca, cb;
    if (ntype < 1 || slot_map(ca, cb, ncoeff, nperdim, quadraticflag)) {
        if (ntype < 1) set_error("cpuSnapTallyBispectrum: ntype must be >= 1");
        return;
    }
    const size_t nout = (size_t)nperdim * ntype;
    if (inum <= 0) { std::fill(bi, bi + nout, 0.0); return; }
    const int amax = max_of(ilist, inum) + 1;
    for (int ii = 0; ii < inum; ii++)
        if (type[ilist[ii]] < 1 || type[ilist[ii]] > ntype) { set_error("cpuSnapTallyBispectrum: atom type outside 1..ntype"); return; }
    Stage2 st;
    double *dbi = st.alloc<double>(nout);
    const double *B = st.in(bispectrum, (size_t)inum * ncoeff);
    const int *dil = st.in(ilist, inum), *dty = st.in(type, amax), *dca = st.in(ca.data(), nperdim),
              *dcb = st.in(cb.data(), nperdim);
    if (!st.ok) { set_error("cpuSnapTallyBispectrum: staging failed"); return; }
    k_tally_b<<<(unsigned)nout, TALLY_T>>>(dbi, B, dil, dty, inum, ncoeff, nperdim, SlotMap{dca, dcb});
    count_launches(1);
    if (st.out(bi, dbi, nout)) set_error("cpuSnapTallyBispectrum: copy-back failed");
}

// cpuSnap.h:80-81; src/Julia/Potential/cpuSnap.cpp:2293-2365
void cpuSnapTallyBispectrumDeriv(double *db, double *bispectrum, double *dbdr, int *aii, int *ai, int *aj, int *ti,
                                 int inum, int ijnum, int ncoeff, int nperdim, int ntype, int quadraticflag)
{
    std::lock_guard<std::mutex> lk(g_desc_mu);
    std::vector<int> ca, cb;
    if (ntype < 1 || slot_map(ca, cb, ncoeff, nperdim, quadraticflag)) {
        if (ntype < 1) set_error("cpuSnapTallyBispectrumDeriv: ntype must be >= 1");
        return;
    }
    const size_t nout = (size_t)inum * 3 * nperdim * ntype;
    if (inum <= 0) return;
    for (int p = 0; p < ijnum; p++)
        if (ai[p] < 0 || ai[p] >= inum || aj[p] < 0 || aj[p] >= inum || aii[p] < 0 || aii[p] >= inum ||
            ti[p] < 1 || ti[p] > ntype) {
            set_error("cpuSnapTallyBispectrumDeriv: pair %d has an atom outside 0..%d or a type outside 1..%d", p,
                      inum - 1, ntype);
            return;
        }
    Stage2 st;
    double *ddb = st.zeros<double>(nout);
    const double *B = st.in(bispectrum, (size_t)inum * ncoeff), *dd = st.in(dbdr, 3 * (size_t)ijnum * ncoeff);
    const int *daii = st.in(aii, ijnum), *dai = st.in(ai, ijnum), *daj = st.in(aj, ijnum), *dti = st.in(ti, ijnum),
              *dca = st.in(ca.data(), nperdim), *dcb = st.in(cb.data(), nperdim);
    if (!st.ok) { set_error("cpuSnapTallyBispectrumDeriv: staging failed"); return; }
    AtomLists L;
    if (ijnum > 0) {
        if (atom_lists(L, dai, daj, ijnum, inum)) return;
        k_tally_db<<<grid_of((long)inum * nperdim, 128), 128>>>(ddb, B, dd, daii, dti, L.off.as<int>(),
                                                                  L.list.as<int>(), inum, ijnum, nperdim,
                                                                  SlotMap{dca, dcb});
        count_launches(1);
    }
    if (st.out(db, ddb, nout)) set_error("cpuSnapTallyBispectrumDeriv: copy-back failed");
}

// cpuSnap.h:83-84; src/Julia/Potential/cpuSnap.cpp:2367-2472
void cpuSnapTallyBispectrumVirial(double *bv, double *bispectrum, double *dbdr, double *rij, int *aii, int *ti,
                                  int inum, int ijnum, int ncoeff, int nperdim, int ntype, int quadraticflag)
{
    std::lock_guard<std::mutex> lk(g_desc_mu);
    std::vector<int> ca, cb;
    if (ntype < 1 || slot_map(ca, cb, ncoeff, nperdim, quadraticflag)) {
        if (ntype < 1) set_error("cpuSnapTallyBispectrumVirial: ntype must be >= 1");
        return;
    }
    const size_t nout = 6 * (size_t)nperdim * ntype;
    if (ijnum <= 0 || inum <= 0) { std::fill(bv, bv + nout, 0.0); return; }
    for (int p = 0; p < ijnum; p++)
        if (aii[p] < 0 || aii[p] >= inum || ti[p] < 1 || ti[p] > ntype) {
            set_error("cpuSnapTallyBispectrumVirial: pair %d has an atom outside 0..%d or a type outside 1..%d", p,
                      inum - 1, ntype);
            return;
        }
    Stage2 st;
    double *dbv = st.alloc<double>(nout);
    const double *B = st.in(bispectrum, (size_t)inum * ncoeff), *dd = st.in(dbdr, 3 * (size_t)ijnum * ncoeff),
                 *dr = st.in(rij, 3 * (size_t)ijnum);
    const int *daii = st.in(aii, ijnum), *dti = st.in(ti, ijnum), *dca = st.in(ca.data(), nperdim),
              *dcb = st.in(cb.data(), nperdim);
    if (!st.ok) { set_error("cpuSnapTallyBispectrumVirial: staging failed"); return; }
    k_tally_bv<<<(unsigned)(nperdim * ntype), TALLY_T>>>(dbv, B, dd, dr, daii, dti, inum, ijnum, nperdim,
                                                          SlotMap{dca, dcb});
    count_launches(1);
    if (st.out(bv, dbv, nout)) set_error("cpuSnapTallyBispectrumVirial: copy-back failed");
}

}  // extern "C"
