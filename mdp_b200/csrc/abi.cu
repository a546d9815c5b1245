// Drop-in entry points with MDP's own signatures and array layouts.
//
//  * cpuSnap.h names (src/Julia/Potential/cpuSnap.h:15-84): the extern "C"
//    library the Julia driver (src/Julia/Potential/snapcpp.jl) loads by path.
//    Host pointers in and out; every call stages its arrays through the GPU.
//  * mdp_gpu_* functions: the device-pointer operations behind the gpu*
//    template entry points of src/C++/Common/mdpgpucore.h:516-612, which
//    include/mdp_b200_gpucore.h maps onto these for mdpcore.h's backend == 2
//    dispatch.
//
// Layouts are the reference's: U and Y are [idxu][inum] (atom fastest) in
// separate real/imaginary arrays, rij is [ijnum][3], forces [inum][3].
// Supported: 2J in {4, 6, 8}, double precision, up to four element types
// (chemflag 0 or 1); quadraticflag belongs to the ComputePairSnap chain.  The
// reference's void functions have no error channel: an unsupported argument
// leaves the outputs untouched and sets mdp_last_error().
#include "common.cuh"
#include "engine.h"

#include <math.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <vector>

namespace mdp {

// ---------------------------------------------------------------------------
// layout conversion and small kernels
// ---------------------------------------------------------------------------
__global__ void k_uref_to_tiles(const double *__restrict__ ur, const double *__restrict__ ui, int inum, int nu,
                                double2 *__restrict__ Ut)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)inum * nu) return;
    const int i = (int)(t % inum), k = (int)(t / inum);
    Ut[(size_t)(i >> 5) * nu * 32 + (size_t)k * 32 + (i & 31)] = make_double2(ur[t], ui[t]);
}

// Y half-plane tiles -> reference ylist (rows mb <= j/2 filled, others zero)
__global__ void k_ytiles_to_ref(const double2 *__restrict__ Y, int inum, int tj, int nyh, double *__restrict__ yr,
                                double *__restrict__ yi)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nu = idxu_count(tj);
    if (t >= (long)inum * nu) return;
    const int i = (int)(t % inum), k = (int)(t / inum);
    int j = 0;
    while (idxu_block(j + 1) <= k) j++;
    const int rem = k - idxu_block(j), mb = rem / (j + 1);
    double2 v = make_double2(0.0, 0.0);
    if (2 * mb <= j) v = Y[(size_t)(i >> 5) * nyh * 32 + (size_t)(yh_block(j) + rem) * 32 + (i & 31)];
    yr[t] = v.x;
    yi[t] = v.y;
}

__global__ void k_yref_to_tiles(const double *__restrict__ yr, const double *__restrict__ yi, int inum, int tj,
                                int nyh, double2 *__restrict__ Y)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)inum * nyh) return;
    const int i = (int)(t % inum), kh = (int)(t / inum);
    int j = 0;
    while (yh_block(j + 1) <= kh) j++;
    const int k = idxu_block(j) + (kh - yh_block(j));
    Y[(size_t)(i >> 5) * nyh * 32 + (size_t)kh * 32 + (i & 31)] =
        make_double2(yr[(size_t)k * inum + i], yi[(size_t)k * inum + i]);
}

// wself on every diagonal entry, then the left half mirrored onto the right
// (cpuAddWself2Ui, cpuSnap4.cpp:193-244), one thread per (atom, j)
__global__ void k_wself_ref(double *__restrict__ ur, double *__restrict__ ui, double wself, int inum, int tj)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)inum * (tj + 1)) return;
    const int i = (int)(t % inum), j = (int)(t / inum);
    const int b0 = idxu_block(j);
    for (int m = 0; m <= j; m++) ur[(size_t)(b0 + (j + 1) * m + m) * inum + i] += wself;
    for (int mb = 0; 2 * mb < j; mb++)
        for (int ma = 0; ma <= j; ma++) {
            const size_t src = (size_t)(b0 + (j + 1) * mb + ma) * inum + i;
            const size_t dst = (size_t)(b0 + (j + 1) * (j - mb) + (j - ma)) * inum + i;
            const double s = ((ma + mb) & 1) ? -1.0 : 1.0;
            ur[dst] = s * ur[src];
            ui[dst] = -s * ui[src];
        }
}

__global__ void k_add_eatom(double *__restrict__ eatom, const double *__restrict__ etmp, const int *__restrict__ ilist,
                            int inum)
{
    int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii < inum) eatom[ilist ? ilist[ii] : ii] += etmp[ii];
}

// pairs grouped by atom: counts, then a scatter by pair index
__global__ void k_pair_bucket_count(const int *__restrict__ aii, int ijnum, int *__restrict__ cnt)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < ijnum) atomicAdd(&cnt[aii[p]], 1);
}
__global__ void k_pair_bucket_fill(const int *__restrict__ aii, const double *__restrict__ rij, int ijnum,
                                   const int *__restrict__ off, int *__restrict__ cursor, double4 *__restrict__ prij,
                                   int2 *__restrict__ pinfo)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ijnum) return;
    const int i = aii[p];
    const int q = off[i] + atomicAdd(&cursor[i], 1);
    prij[q] = make_double4(rij[3 * (size_t)p], rij[3 * (size_t)p + 1], rij[3 * (size_t)p + 2], 0.0);
    pinfo[q] = make_int2(i, p);
}

// per-pair dE/dr -> forces (+= on ai, -= on aj) and the per-atom virial:
// mode 0: core layout vatom[c * vstride + atom], -1/2 r (x) dE on both atoms
//         (cpuSnap4.cpp:1177-1209); mode 1: Julia layout vatom[6 * ai + c],
//         -r (x) dE on ai only (src/Julia/Potential/cpuSnap.cpp:1370-1396)
__global__ void k_scatter_fi(const double4 *__restrict__ dE, const double *__restrict__ rij, const int *__restrict__ ai,
                             const int *__restrict__ aj, int ijnum, double *__restrict__ fatom,
                             double *__restrict__ vatom, int mode, long vstride)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ijnum) return;
    const double4 d = dE[p];
    const int a = ai[p], b = aj[p];
    atomicAdd(&fatom[3 * (size_t)a], d.x); atomicAdd(&fatom[3 * (size_t)a + 1], d.y); atomicAdd(&fatom[3 * (size_t)a + 2], d.z);
    atomicAdd(&fatom[3 * (size_t)b], -d.x); atomicAdd(&fatom[3 * (size_t)b + 1], -d.y); atomicAdd(&fatom[3 * (size_t)b + 2], -d.z);
    if (!vatom) return;
    const double x = rij[3 * (size_t)p], y = rij[3 * (size_t)p + 1], z = rij[3 * (size_t)p + 2];
    const double c = mode == 0 ? -0.5 : -1.0;
    const double v[6] = {c * x * d.x, c * y * d.y, c * z * d.z, c * x * d.y, c * x * d.z, c * y * d.z};
    if (mode == 0) {
        for (int k = 0; k < 6; k++) { atomicAdd(&vatom[k * vstride + a], v[k]); atomicAdd(&vatom[k * vstride + b], v[k]); }
    } else {
        for (int k = 0; k < 6; k++) atomicAdd(&vatom[6 * (size_t)a + k], v[k]);
    }
}

// typed pair filter (cpuSnap.cpp:1883-1906; the Julia library's CSR form when
// csr != 0, src/Julia/Potential/cpuSnap.cpp:258-286)
// correctly rounded sum and product in the precision of the caller's build
__device__ __forceinline__ double ref_add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float ref_add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double ref_mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float ref_mul_rn(float a, float b) { return __fmul_rn(a, b); }

template <typename T>
__global__ void k_ref_pair_count(int *__restrict__ pairnum, const T *__restrict__ x, const T *__restrict__ rcutsq,
                                 const int *__restrict__ ilist, const int *__restrict__ nlist, const int *__restrict__ nnum,
                                 const int *__restrict__ atype, const int *__restrict__ alist, int inum, int jnum, int ntypes,
                                 int csr, int *__restrict__ pairlist_rows)
{
    int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii], it = atype[i];
    const int n0 = csr ? nnum[i] : jnum * i;
    const int m = csr ? nnum[i + 1] - nnum[i] : nnum[i];
    int cnt = 0;
    for (int l = 0; l < m; l++) {
        const int j = nlist[n0 + l];
        const int jt = atype[alist[j]];
        const T d0 = x[3 * (size_t)j] - x[3 * (size_t)i], d1 = x[3 * (size_t)j + 1] - x[3 * (size_t)i + 1],
                     d2 = x[3 * (size_t)j + 2] - x[3 * (size_t)i + 2];
        const T dij = ref_add_rn(ref_add_rn(ref_mul_rn(d0, d0), ref_mul_rn(d1, d1)), ref_mul_rn(d2, d2));
        if (dij < rcutsq[jt + it * (ntypes + 1)] && dij > T(1e-20)) {
            if (pairlist_rows) pairlist_rows[(size_t)jnum * ii + cnt] = j;
            cnt++;
        }
    }
    pairnum[ii] = cnt;
}
template <typename T>
__global__ void k_ref_pair_emit_csr(int *__restrict__ pairlist, const int *__restrict__ off, const T *__restrict__ x,
                                    const T *__restrict__ rcutsq, const int *__restrict__ ilist,
                                    const int *__restrict__ nlist, const int *__restrict__ nnum,
                                    const int *__restrict__ atype, const int *__restrict__ alist, int inum, int ntypes)
{
    int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii], it = atype[i];
    const int n0 = nnum[i], m = nnum[i + 1] - nnum[i];
    int q = off[ii];
    for (int l = 0; l < m; l++) {
        const int j = nlist[n0 + l];
        const int jt = atype[alist[j]];
        const T d0 = x[3 * (size_t)j] - x[3 * (size_t)i], d1 = x[3 * (size_t)j + 1] - x[3 * (size_t)i + 1],
                     d2 = x[3 * (size_t)j + 2] - x[3 * (size_t)i + 2];
        const T dij = ref_add_rn(ref_add_rn(ref_mul_rn(d0, d0), ref_mul_rn(d1, d1)), ref_mul_rn(d2, d2));
        if (dij < rcutsq[jt + it * (ntypes + 1)] && dij > T(1e-20)) pairlist[q++] = j;
    }
}
// pair geometry and indices (cpuSnap.cpp:1912-1933); rows layout when jnum > 0,
// CSR (pairlist at pairnumsum[ii]) when jnum == 0
template <typename T>
__global__ void k_ref_pairs(T *__restrict__ xij, const T *__restrict__ x, int *__restrict__ aii,
                            int *__restrict__ ai, int *__restrict__ aj, int *__restrict__ ti, int *__restrict__ tj,
                            const int *__restrict__ pairnum, const int *__restrict__ pairlist,
                            const int *__restrict__ pairnumsum, const int *__restrict__ ilist,
                            const int *__restrict__ atype, const int *__restrict__ alist, int inum, int jnum)
{
    int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii], it = atype[i];
    const int start = pairnumsum[ii];
    const int m = pairnum ? pairnum[ii] : pairnumsum[ii + 1] - start;
    for (int l = 0; l < m; l++) {
        const int j = jnum > 0 ? pairlist[l + jnum * ii] : pairlist[start + l];
        const int k = start + l;
        aii[k] = ii; ai[k] = i; aj[k] = alist[j]; ti[k] = it; tj[k] = atype[alist[j]];
        for (int d = 0; d < 3; d++) xij[3 * (size_t)k + d] = x[3 * (size_t)j + d] - x[3 * (size_t)i + d];
    }
}

__global__ void k_minmax2(const int *__restrict__ a, const int *__restrict__ b, int n, int *__restrict__ out)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    atomicMin(&out[0], a[p]); atomicMax(&out[1], a[p]);
    atomicMin(&out[0], b[p]); atomicMax(&out[1], b[p]);
}

// ---------------------------------------------------------------------------
// shared context for the reference-layout operations
// ---------------------------------------------------------------------------
struct RefCtx {
    ForcePath fp;
    DevBuf cnt, off, cursor, etmp, tmp, mm, elem;
    SnapModel model;
};
static std::mutex g_ref_mu;
static RefCtx &ref_ctx()
{
    static RefCtx c;
    return c;
}

static int model_from_args(SnapModel &m, int twojmax, const double *coeff_host, int ncoeffall, int bnorm, int bzero,
                           int wselfall, double rcut, double wj, double rfac0, double rmin0, int switchflag)
{
    mdp_snap_params p;
    memset(&p, 0, sizeof(p));
    p.twojmax = twojmax;
    p.rcutfac = rcut;   // rcut = 2 * radelem * rcutfac with radelem = 0.5
    p.radelem = 0.5;
    p.rfac0 = rfac0;
    p.rmin0 = rmin0;
    p.wjelem = wj;
    p.switchflag = switchflag;
    p.bnormflag = bnorm;
    p.bzeroflag = bzero;
    p.wselfallflag = wselfall;
    std::vector<double> dummy;
    if (!coeff_host) {
        dummy.assign(mdp_snap_ncoeff(twojmax) + 1, 0.0);
        coeff_host = dummy.data();
        ncoeffall = (int)dummy.size();
    }
    p.ncoeffall = ncoeffall;
    p.coeff = coeff_host;
    return model_init(m, &p);
}

// single-type check of ti/tj on the device; returns the type, -2 when the
// pairs have several types, -1 on error
static int single_type(const int *ti, const int *tj, int n, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (n <= 0) return 0;
    if (c.mm.ensure(2 * sizeof(int))) return -1;
    int init[2] = {0x7fffffff, -0x7fffffff};
    MDP_CUDA_TRY(cudaMemcpyAsync(c.mm.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_minmax2<<<(n + 255) / 256, 256, 0, s>>>(ti, tj, n, c.mm.as<int>());
    int h[2];
    MDP_CUDA_TRY(cudaMemcpyAsync(h, c.mm.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaStreamSynchronize(s));
    return h[0] != h[1] ? -2 : h[0];
}

// U (reference layout) -> tiles in fp.Ut
static int load_tiles(RefCtx &c, const double *ur, const double *ui, int inum, int tj, cudaStream_t s)
{
    const int nu = idxu_count(tj);
    const long ntiles = (inum + 31) / 32;
    if (c.fp.Ut.ensure(sizeof(double2) * ntiles * nu * 32)) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(c.fp.Ut.p, 0, sizeof(double2) * ntiles * nu * 32, s));
    const long n = (long)inum * nu;
    k_uref_to_tiles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ur, ui, inum, nu, c.fp.Ut.as<double2>());
    return 0;
}

static int run_yi(RefCtx &c, int inum, int tj, cudaStream_t s)
{
    const long ntiles = (inum + 31) / 32;
    if (c.fp.Y.ensure(sizeof(double2) * ntiles * 32 * yh_count(tj)) || c.etmp.ensure(sizeof(double) * inum)) return -1;
    switch (tj) {
    case 4: return launch_yi<double, 4>(c.model, c.model.yd, c.fp, inum, c.etmp.as<double>(), s);
    case 6: return launch_yi<double, 6>(c.model, c.model.yd, c.fp, inum, c.etmp.as<double>(), s);
    case 8: return launch_yi<double, 8>(c.model, c.model.yd, c.fp, inum, c.etmp.as<double>(), s);
    }
    set_error("twojmax %d not supported", tj);
    return -1;
}

int ref_snap_ui(double *ur, double *ui, const double *rij, double rcut, double wj, double rfac0, double rmin0,
                const int *aii, int tj, int inum, int ijnum, int switchflag, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (model_from_args(c.model, tj, nullptr, 0, 0, 0, 0, rcut, wj, rfac0, rmin0, switchflag)) return -1;
    if (ijnum <= 0) return 0;
    if (c.cnt.ensure(sizeof(int) * inum) || c.off.ensure(sizeof(int) * ((size_t)inum + 1)) ||
        c.cursor.ensure(sizeof(int) * inum) || c.fp.prij.ensure(sizeof(double4) * ijnum) ||
        c.fp.pinfo.ensure(sizeof(int2) * ijnum) || c.tmp.ensure(sizeof(int) * scan_tmp_ints(inum)))
        return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(c.cnt.p, 0, sizeof(int) * inum, s));
    MDP_CUDA_TRY(cudaMemsetAsync(c.cursor.p, 0, sizeof(int) * inum, s));
    k_pair_bucket_count<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, ijnum, c.cnt.as<int>());
    if (exclusive_scan(c.cnt.as<int>(), c.off.as<int>(), inum, c.tmp.as<int>(), s)) return -1;
    k_pair_bucket_fill<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, rij, ijnum, c.off.as<int>(), c.cursor.as<int>(),
                                                           c.fp.prij.as<double4>(), c.fp.pinfo.as<int2>());
    if (tu_ensure_tables()) return -1;
    const int blocks = std::min((inum + UI_WARPS - 1) / UI_WARPS, num_sms() * 16);
#define MDP_UIREF(TJ)                                                                                              \
    {                                                                                                              \
        const size_t sm = (size_t)UI_WARPS * (idxu_count(TJ) + 32 * (TJ + 1)) * sizeof(double2);                  \
        int per_sm = 0;                                                                                            \
        if (kernel_setup((const void *)k_snap_ui<double, TJ, true>, UI_WARPS * 32, sm, &per_sm, "k_snap_ui"))      \
            return -1;                                                                                             \
        k_snap_ui<double, TJ, true><<<blocks, UI_WARPS * 32, sm, s>>>(c.off.as<int>(), c.fp.prij.as<double4>(),    \
                                                                      inum, c.model.geom, nullptr, ur, ui);        \
    }
    switch (tj) {
    case 4: MDP_UIREF(4) break;
    case 6: MDP_UIREF(6) break;
    case 8: MDP_UIREF(8) break;
    default: set_error("twojmax %d not supported", tj); return -1;
    }
#undef MDP_UIREF
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int ref_snap_wself(double *ur, double *ui, double wself, int tj, int inum, cudaStream_t s)
{
    const long n = (long)inum * (tj + 1);
    k_wself_ref<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ur, ui, wself, inum, tj);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// eatom[ilist[ii]] += beta0 + sum_k beta_k B_k
int ref_snap_ei(double *eatom, const double *ur, const double *ui, const double *coeff_host, const int *ilist, int tj,
                int ncoeffall, int bnorm, int bzero, int wselfall, int inum, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (model_from_args(c.model, tj, coeff_host, ncoeffall, bnorm, bzero, wselfall, 1.0, 1.0, 1.0, 0.0, 1)) return -1;
    if (load_tiles(c, ur, ui, inum, tj, s) || run_yi(c, inum, tj, s)) return -1;
    k_add_eatom<<<(inum + 255) / 256, 256, 0, s>>>(eatom, c.etmp.as<double>(), ilist, inum);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int ref_snap_yi(double *yr, double *yi, const double *ur, const double *ui, const double *coeff_host, int tj,
                int ncoeffall, int bnorm, int inum, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (model_from_args(c.model, tj, coeff_host, ncoeffall, bnorm, 0, 0, 1.0, 1.0, 1.0, 0.0, 1)) return -1;
    if (load_tiles(c, ur, ui, inum, tj, s) || run_yi(c, inum, tj, s)) return -1;
    const long n = (long)inum * idxu_count(tj);
    k_ytiles_to_ref<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(c.fp.Y.as<double2>(), inum, tj, yh_count(tj), yr, yi);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_yi_pa_d(const SnapModel &m, const YParams<double> &yp, ForcePath &fp, int inum, const double *G,
                   cudaStream_t s);

// Y with per-atom coefficients beta [jjb][inum] (cpuSnap4.cpp:601-691): the
// model's coefficients are all 1, so its per-triple factors carry only the
// multiplicities and the bnorm / (j1+1)/(j+1) scalings
int ref_snap_yi_beta(double *yr, double *yi, const double *ur, const double *ui, const double *beta, int tj,
                     int bnorm, int inum, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    std::vector<double> ones(mdp_snap_ncoeff(tj) + 1, 1.0);
    ones[0] = 0.0;
    if (model_from_args(c.model, tj, ones.data(), (int)ones.size(), bnorm, 0, 0, 1.0, 1.0, 1.0, 0.0, 1)) return -1;
    if (load_tiles(c, ur, ui, inum, tj, s)) return -1;
    const long ntiles = (inum + 31) / 32;
    if (c.fp.Y.ensure(sizeof(double2) * ntiles * 32 * yh_count(tj))) return -1;
    if (launch_yi_pa_d(c.model, c.model.yd, c.fp, inum, beta, s)) return -1;
    const long n = (long)inum * idxu_count(tj);
    k_ytiles_to_ref<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(c.fp.Y.as<double2>(), inum, tj, yh_count(tj), yr, yi);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_bi_tiles(const double2 *Ut, int natoms, int tj, int bnorm, int bzero, double *bout, long bstride,
                    cudaStream_t s);

int ref_snap_bi(double *blist, const double *ur, const double *ui, int tj, int bnorm, int bzero, int inum,
                cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (load_tiles(c, ur, ui, inum, tj, s)) return -1;
    return launch_bi_tiles(c.fp.Ut.as<double2>(), inum, tj, bnorm, bzero, blist, inum, s);
}

int ref_snap_fi(double *fatom, double *vatom, int vmode, long vstride, const double *yr, const double *yi,
                const double *rij, double rcut, double wj, double rfac0, double rmin0, const int *aii,
                const int *ai, const int *aj, int tj, int inum, int ijnum, int switchflag, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (model_from_args(c.model, tj, nullptr, 0, 0, 0, 0, rcut, wj, rfac0, rmin0, switchflag)) return -1;
    if (ijnum <= 0) return 0;
    const int nyh = yh_count(tj);
    const long ntiles = (inum + 31) / 32;
    if (c.fp.Y.ensure(sizeof(double2) * ntiles * 32 * nyh) || c.fp.prij.ensure(sizeof(double4) * ijnum) ||
        c.fp.pinfo.ensure(sizeof(int2) * ijnum) || c.fp.dE.ensure(sizeof(double4) * ijnum) ||
        c.fp.poff.ensure(sizeof(int) * ((size_t)inum + 1)) || c.cnt.ensure(sizeof(int) * inum) ||
        c.cursor.ensure(sizeof(int) * inum) || c.tmp.ensure(sizeof(int) * scan_tmp_ints(inum)))
        return -1;
    const long n = (long)inum * nyh;
    k_yref_to_tiles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(yr, yi, inum, tj, nyh, c.fp.Y.as<double2>());
    MDP_CUDA_TRY(cudaMemsetAsync(c.cnt.p, 0, sizeof(int) * inum, s));
    MDP_CUDA_TRY(cudaMemsetAsync(c.cursor.p, 0, sizeof(int) * inum, s));
    k_pair_bucket_count<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, ijnum, c.cnt.as<int>());
    if (exclusive_scan(c.cnt.as<int>(), c.fp.poff.as<int>(), inum, c.tmp.as<int>(), s)) return -1;
    k_pair_bucket_fill<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, rij, ijnum, c.fp.poff.as<int>(), c.cursor.as<int>(),
                                                           c.fp.prij.as<double4>(), c.fp.pinfo.as<int2>());
    int rc;
    switch (tj) {
    case 4: rc = launch_fi<double, 4>(c.model, c.fp, inum, 1, s); break;
    case 6: rc = launch_fi<double, 6>(c.model, c.fp, inum, 1, s); break;
    case 8: rc = launch_fi<double, 8>(c.model, c.fp, inum, 1, s); break;
    default: set_error("twojmax %d not supported", tj); return -1;
    }
    if (rc) return rc;
    k_scatter_fi<<<(ijnum + 255) / 256, 256, 0, s>>>(c.fp.dE.as<double4>(), rij, ai, aj, ijnum, fatom, vatom, vmode,
                                                     vstride);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// several element types in the reference layouts: U / Y [block][k][inum]
// (block = map[tj] with chemflag, cpuSnap4.cpp:59-61 and 887-888), per-pair
// cutoffs (radelem[ti] + radelem[tj]) rcutfac and weights wjelem[tj], the
// coefficient table coeffelem [element][ncoeffall] chosen per atom by
// map[type[ii]]
// ---------------------------------------------------------------------------
__global__ void k_max_block(const int *__restrict__ tj, const int *__restrict__ map, int n, int *__restrict__ out)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) atomicMax(out, map[tj[p]]);
}

// pairs bucketed per virtual atom v = block * inum + aii; pinfo = (block *
// ipad + aii, pair) for the tiled Y; pcw = per-pair cutoff and weight
__global__ void k_pair_bucket_count_me(const int *__restrict__ aii, const int *__restrict__ tj,
                                       const int *__restrict__ map, int chem, int inum, int ijnum, int *__restrict__ cnt)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ijnum) return;
    const int b = chem ? map[tj[p]] : 0;
    atomicAdd(&cnt[(long)b * inum + aii[p]], 1);
}
__global__ void k_pair_bucket_fill_me(const int *__restrict__ aii, const int *__restrict__ ti,
                                      const int *__restrict__ tj, const int *__restrict__ map, int chem,
                                      const double *__restrict__ rij, const double *__restrict__ radelem,
                                      const double *__restrict__ wjelem, double rcutfac, int ijnum, int inum, int ipad,
                                      const int *__restrict__ off, int *__restrict__ cursor, double4 *__restrict__ prij,
                                      int2 *__restrict__ pinfo, double2 *__restrict__ pcw)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ijnum) return;
    const int b = chem ? map[tj[p]] : 0, i = aii[p];
    const long v = (long)b * inum + i;
    const int q = off[v] + atomicAdd(&cursor[v], 1);
    prij[q] = make_double4(rij[3 * (size_t)p], rij[3 * (size_t)p + 1], rij[3 * (size_t)p + 2], 0.0);
    pinfo[q] = make_int2((int)((long)b * ipad + i), p);
    pcw[q] = make_double2((radelem[ti[p]] + radelem[tj[p]]) * rcutfac, wjelem[tj[p]]);
}

// wself on the diagonal of block b of atom ii when b is the atom's element
// (chemflag) or always (wselfallflag, or the one block without chemflag),
// then the mirror of every block (cpuAddWself2Ui, cpuSnap4.cpp:193-244)
__global__ void k_wself_ref_me(double *__restrict__ ur, double *__restrict__ ui, double wself, int inum, int tj,
                               int nblk, const int *__restrict__ type, const int *__restrict__ map, int chem,
                               int wselfall)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long per = (long)inum * (tj + 1);
    if (t >= per * nblk) return;
    const int b = (int)(t / per);
    const long r = t - (long)b * per;
    const int i = (int)(r % inum), j = (int)(r / inum);
    const int nu = idxu_count(tj);
    double *br = ur + (size_t)b * nu * inum, *bi = ui + (size_t)b * nu * inum;
    const int ie = chem ? map[type[i]] : 0;
    const int b0 = idxu_block(j);
    if (b == ie || wselfall)
        for (int m = 0; m <= j; m++) br[(size_t)(b0 + (j + 1) * m + m) * inum + i] += wself;
    for (int mb = 0; 2 * mb < j; mb++)
        for (int ma = 0; ma <= j; ma++) {
            const size_t src = (size_t)(b0 + (j + 1) * mb + ma) * inum + i;
            const size_t dst = (size_t)(b0 + (j + 1) * (j - mb) + (j - ma)) * inum + i;
            const double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
            br[dst] = sg * br[src];
            bi[dst] = -sg * bi[src];
        }
}

// element of each atom's coefficient set: map[type[ii]] when use, else 0;
// pads (ii >= inum) 0; *emax = the largest
__global__ void k_elem_map(const int *__restrict__ type, const int *__restrict__ map, int inum, int ipad, int use,
                           int *__restrict__ elem, int *__restrict__ emax)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ipad) return;
    int e = (i < inum && use) ? map[type[i]] : 0;
    e = e < 0 ? 0 : e;
    elem[i] = e;
    if (i < inum) atomicMax(emax, e);
}

// number of element blocks the pairs reach: 1 + max map[tj] (1 without chemflag)
static int pair_blocks(const int *tj, const int *map, int ijnum, int chem, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (!chem || ijnum <= 0) return 1;
    if (c.mm.ensure(2 * sizeof(int))) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(c.mm.p, 0, sizeof(int), s));
    k_max_block<<<(ijnum + 255) / 256, 256, 0, s>>>(tj, map, ijnum, c.mm.as<int>());
    int h = 0;
    MDP_CUDA_TRY(cudaMemcpyAsync(&h, c.mm.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaStreamSynchronize(s));
    if (h < 0 || h >= MAXELEM) { set_error("element block %d out of range (at most %d elements)", h, MAXELEM); return -1; }
    return h + 1;
}

// per-atom elements into c.elem (ipad entries); returns the largest, or -1
static int atom_elements(const int *type, const int *map, int inum, int use, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    const int ipad = (inum + 31) / 32 * 32;
    if (c.elem.ensure(sizeof(int) * ipad) || c.mm.ensure(2 * sizeof(int))) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(c.mm.p, 0, sizeof(int), s));
    k_elem_map<<<(ipad + 255) / 256, 256, 0, s>>>(type, map, inum, ipad, use, c.elem.as<int>(), c.mm.as<int>());
    int h = 0;
    MDP_CUDA_TRY(cudaMemcpyAsync(&h, c.mm.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaStreamSynchronize(s));
    return h;
}

// nblk U blocks (reference layout) -> tiles, block after block
static int load_tiles_blocks(RefCtx &c, const double *ur, const double *ui, int inum, int tj, int nblk,
                             cudaStream_t s)
{
    const int nu = idxu_count(tj);
    const long ntiles = (inum + 31) / 32;
    const size_t per = (size_t)ntiles * nu * 32;
    if (c.fp.Ut.ensure(sizeof(double2) * per * nblk)) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(c.fp.Ut.p, 0, sizeof(double2) * per * nblk, s));
    const long n = (long)inum * nu;
    for (int b = 0; b < nblk; b++)
        k_uref_to_tiles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ur + (size_t)b * n, ui + (size_t)b * n, inum, nu,
                                                                   c.fp.Ut.as<double2>() + per * b);
    return 0;
}

static MeArgs me_args(RefCtx &c, int inum, int nblk, int ncoeffall, int bzero, int wselfall, const double *coeff,
                      int pa)
{
    MeArgs A;
    A.nblk = nblk;
    A.ntiles = (inum + 31) / 32;
    A.ncoeffall = ncoeffall;
    A.bzero = bzero;
    A.wselfall = wselfall;
    A.elem = c.elem.as<int>();
    A.coeff = coeff;
    A.pa = pa;
    return A;
}

// U of the element blocks, accumulated into the reference layout
int ref_snap_ui_me(double *ur, double *ui, const double *rij, const double *radelem, const double *wjelem,
                   double rcutfac, double rfac0, double rmin0, const int *aii, const int *ti, const int *tjv,
                   const int *map, int chem, int tj, int inum, int ijnum, int switchflag, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (model_from_args(c.model, tj, nullptr, 0, 0, 0, 0, 1.0, 1.0, rfac0, rmin0, switchflag)) return -1;
    if (ijnum <= 0) return 0;
    const int nblk = pair_blocks(tjv, map, ijnum, chem, s);
    if (nblk < 0) return -1;
    const long nv = (long)nblk * inum;
    const int ipad = (inum + 31) / 32 * 32;
    if (c.cnt.ensure(sizeof(int) * nv) || c.off.ensure(sizeof(int) * (nv + 1)) || c.cursor.ensure(sizeof(int) * nv) ||
        c.fp.prij.ensure(sizeof(double4) * ijnum) || c.fp.pinfo.ensure(sizeof(int2) * ijnum) ||
        c.fp.pcw.ensure(sizeof(double2) * ijnum) || c.tmp.ensure(sizeof(int) * scan_tmp_ints(nv)))
        return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(c.cnt.p, 0, sizeof(int) * nv, s));
    MDP_CUDA_TRY(cudaMemsetAsync(c.cursor.p, 0, sizeof(int) * nv, s));
    k_pair_bucket_count_me<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, tjv, map, chem, inum, ijnum, c.cnt.as<int>());
    if (exclusive_scan(c.cnt.as<int>(), c.off.as<int>(), nv, c.tmp.as<int>(), s)) return -1;
    k_pair_bucket_fill_me<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, ti, tjv, map, chem, rij, radelem, wjelem, rcutfac,
                                                              ijnum, inum, ipad, c.off.as<int>(), c.cursor.as<int>(),
                                                              c.fp.prij.as<double4>(), c.fp.pinfo.as<int2>(),
                                                              c.fp.pcw.as<double2>());
    if (tu_ensure_tables()) return -1;
    const int blocks = (int)std::min((nv + UI_WARPS - 1) / UI_WARPS, (long)num_sms() * 16);
#define MDP_UIREF_ME(TJ)                                                                                           \
    {                                                                                                              \
        const size_t sm = (size_t)UI_WARPS * (idxu_count(TJ) + 32 * (TJ + 1)) * sizeof(double2);                  \
        int per_sm = 0;                                                                                            \
        if (kernel_setup((const void *)k_snap_ui<double, TJ, true>, UI_WARPS * 32, sm, &per_sm, "k_snap_ui"))      \
            return -1;                                                                                             \
        k_snap_ui<double, TJ, true><<<blocks, UI_WARPS * 32, sm, s>>>(c.off.as<int>(), c.fp.prij.as<double4>(),    \
                                                                      (int)nv, c.model.geom, nullptr, ur, ui,      \
                                                                      c.fp.pcw.as<double2>(), inum);              \
    }
    switch (tj) {
    case 4: MDP_UIREF_ME(4) break;
    case 6: MDP_UIREF_ME(6) break;
    case 8: MDP_UIREF_ME(8) break;
    default: set_error("twojmax %d not supported", tj); return -1;
    }
#undef MDP_UIREF_ME
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int ref_snap_wself_me(double *ur, double *ui, double wself, const int *type, const int *map, int chem, int wselfall,
                      int nblk, int tj, int inum, cudaStream_t s)
{
    const long n = (long)inum * (tj + 1) * nblk;
    k_wself_ref_me<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ur, ui, wself, inum, tj, nblk, type, map, chem,
                                                              wselfall);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// eatom[ilist[ii]] += beta_0(e) + sum_{t,k} beta(e, t, k) (B^t_k - bzero), e the atom's element
int ref_snap_ei_me(double *eatom, const double *ur, const double *ui, const double *coeff_dev, const int *ilist,
                   int tj, int nblk, int ncoeffall, int bnorm, int bzero, int wselfall, int inum, cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    RefCtx &c = ref_ctx();
    if (load_tiles_blocks(c, ur, ui, inum, tj, nblk, s) || c.etmp.ensure(sizeof(double) * inum)) return -1;
    const MeArgs A = me_args(c, inum, nblk, ncoeffall, bzero, wselfall, coeff_dev, 0);
    const double2 *Ut = c.fp.Ut.as<double2>();
    double *et = c.etmp.as<double>();
    int per_sm = 0;
#define MDP_EI_ME(TJ)                                                                                              \
    if (kernel_setup((const void *)k_snap_ei_me<TJ>, BI_WARPS * 32, 0, &per_sm, "k_snap_ei_me")) return -1;        \
    k_snap_ei_me<TJ><<<std::min(A.ntiles, num_sms() * per_sm), BI_WARPS * 32, 0, s>>>(Ut, inum, bnorm, A, et);
    switch (tj) {
    case 4: MDP_EI_ME(4) break;
    case 6: MDP_EI_ME(6) break;
    case 8: MDP_EI_ME(8) break;
    default: set_error("twojmax %d not supported", tj); return -1;
    }
#undef MDP_EI_ME
    k_add_eatom<<<(inum + 255) / 256, 256, 0, s>>>(eatom, et, ilist, inum);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int ref_snap_bi_me(double *blist, const double *ur, const double *ui, int tj, int nblk, int bnorm, int bzero,
                   int wselfall, int inum, cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    RefCtx &c = ref_ctx();
    if (load_tiles_blocks(c, ur, ui, inum, tj, nblk, s)) return -1;
    const MeArgs A = me_args(c, inum, nblk, 0, bzero, wselfall, nullptr, 0);
    const double2 *Ut = c.fp.Ut.as<double2>();
    int per_sm = 0;
#define MDP_BI_ME(TJ)                                                                                              \
    if (kernel_setup((const void *)k_snap_bi_me<TJ>, BI_WARPS * 32, 0, &per_sm, "k_snap_bi_me")) return -1;        \
    k_snap_bi_me<TJ><<<std::min(A.ntiles, num_sms() * per_sm), BI_WARPS * 32, 0, s>>>(Ut, inum, bnorm, A, blist);
    switch (tj) {
    case 4: MDP_BI_ME(4) break;
    case 6: MDP_BI_ME(6) break;
    case 8: MDP_BI_ME(8) break;
    default: set_error("twojmax %d not supported", tj); return -1;
    }
#undef MDP_BI_ME
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Y of every block from the coefficient table (pa = 0, elements in c.elem)
// or from per-atom coefficients [triple][k][inum] (pa = 1)
int ref_snap_yi_me(double *yr, double *yi, const double *ur, const double *ui, const double *coeff_dev, int pa,
                   int tj, int nblk, int ncoeffall, int bnorm, int inum, cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    RefCtx &c = ref_ctx();
    std::vector<double> ones(mdp_snap_ncoeff(tj) + 1, 1.0);
    if (model_from_args(c.model, tj, ones.data(), (int)ones.size(), bnorm, 0, 0, 1.0, 1.0, 1.0, 0.0, 1)) return -1;
    if (load_tiles_blocks(c, ur, ui, inum, tj, nblk, s)) return -1;
    const long ntiles = (inum + 31) / 32;
    const int nyh = yh_count(tj);
    if (c.fp.Y.ensure(sizeof(double2) * ntiles * 32 * nyh * nblk)) return -1;
    const MeArgs A = me_args(c, inum, nblk, ncoeffall, 0, 0, coeff_dev, pa);
    const double2 *Ut = c.fp.Ut.as<double2>();
    double2 *Y = c.fp.Y.as<double2>();
    int per_sm = 0;
#define MDP_YI_ME(TJ)                                                                                              \
    {                                                                                                              \
        const size_t sm = yi_me_smem_bytes<TJ>();                                                                  \
        if (kernel_setup((const void *)k_snap_yi_me<TJ>, YiWarps<double, TJ>::n * 32, sm, &per_sm, "k_snap_yi_me")) \
            return -1;                                                                                             \
        k_snap_yi_me<TJ><<<std::min(A.ntiles, num_sms() * per_sm), YiWarps<double, TJ>::n * 32, sm, s>>>(          \
            Ut, inum, c.model.yd, A, Y);                                                                           \
    }
    switch (tj) {
    case 4: MDP_YI_ME(4) break;
    case 6: MDP_YI_ME(6) break;
    case 8: MDP_YI_ME(8) break;
    default: set_error("twojmax %d not supported", tj); return -1;
    }
#undef MDP_YI_ME
    const long n = (long)inum * idxu_count(tj);
    for (int b = 0; b < nblk; b++)
        k_ytiles_to_ref<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Y + (size_t)b * ntiles * nyh * 32, inum, tj, nyh,
                                                                   yr + (size_t)b * n, yi + (size_t)b * n);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// dE/dr with each pair's Y block (map[tj] with chemflag), per-pair cutoffs and weights
int ref_snap_fi_me(double *fatom, double *vatom, int vmode, long vstride, const double *yr, const double *yi,
                   const double *rij, const double *radelem, const double *wjelem, double rcutfac, double rfac0,
                   double rmin0, const int *aii, const int *ai, const int *aj, const int *ti, const int *tjv,
                   const int *map, int chem, int tj, int inum, int ijnum, int switchflag, cudaStream_t s)
{
    RefCtx &c = ref_ctx();
    if (model_from_args(c.model, tj, nullptr, 0, 0, 0, 0, 1.0, 1.0, rfac0, rmin0, switchflag)) return -1;
    if (ijnum <= 0) return 0;
    const int nblk = pair_blocks(tjv, map, ijnum, chem, s);
    if (nblk < 0) return -1;
    const int nyh = yh_count(tj);
    const long ntiles = (inum + 31) / 32, nv = (long)nblk * inum;
    const int ipad = (int)ntiles * 32;
    if (c.fp.Y.ensure(sizeof(double2) * ntiles * 32 * nyh * nblk) || c.fp.prij.ensure(sizeof(double4) * ijnum) ||
        c.fp.pinfo.ensure(sizeof(int2) * ijnum) || c.fp.pcw.ensure(sizeof(double2) * ijnum) ||
        c.fp.dE.ensure(sizeof(double4) * ijnum) || c.fp.poff.ensure(sizeof(int) * (nv + 1)) ||
        c.cnt.ensure(sizeof(int) * nv) || c.cursor.ensure(sizeof(int) * nv) ||
        c.tmp.ensure(sizeof(int) * scan_tmp_ints(nv)))
        return -1;
    const long n = (long)inum * nyh, nu = (long)inum * idxu_count(tj);
    for (int b = 0; b < nblk; b++)
        k_yref_to_tiles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(yr + (size_t)b * nu, yi + (size_t)b * nu, inum, tj,
                                                                   nyh, c.fp.Y.as<double2>() + (size_t)b * ntiles * nyh * 32);
    MDP_CUDA_TRY(cudaMemsetAsync(c.cnt.p, 0, sizeof(int) * nv, s));
    MDP_CUDA_TRY(cudaMemsetAsync(c.cursor.p, 0, sizeof(int) * nv, s));
    k_pair_bucket_count_me<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, tjv, map, chem, inum, ijnum, c.cnt.as<int>());
    if (exclusive_scan(c.cnt.as<int>(), c.fp.poff.as<int>(), nv, c.tmp.as<int>(), s)) return -1;
    k_pair_bucket_fill_me<<<(ijnum + 255) / 256, 256, 0, s>>>(aii, ti, tjv, map, chem, rij, radelem, wjelem, rcutfac,
                                                              ijnum, inum, ipad, c.fp.poff.as<int>(), c.cursor.as<int>(),
                                                              c.fp.prij.as<double4>(), c.fp.pinfo.as<int2>(),
                                                              c.fp.pcw.as<double2>());
    c.fp.fr_pcw = c.fp.pcw.as<double2>();
    int rc;
    switch (tj) {
    case 4: rc = launch_fi<double, 4>(c.model, c.fp, (int)nv, 1, s); break;
    case 6: rc = launch_fi<double, 6>(c.model, c.fp, (int)nv, 1, s); break;
    case 8: rc = launch_fi<double, 8>(c.model, c.fp, (int)nv, 1, s); break;
    default: rc = -1; set_error("twojmax %d not supported", tj);
    }
    c.fp.fr_pcw = nullptr;
    if (rc) return rc;
    k_scatter_fi<<<(ijnum + 255) / 256, 256, 0, s>>>(c.fp.dE.as<double4>(), rij, ai, aj, ijnum, fatom, vatom, vmode,
                                                     vstride);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// rcut and weight of the (single) pair type, read from device radelem/wjelem;
// returns 0, 1 when the pairs have several types, -1 on error
static int pair_type_params(const int *ti_d, const int *tj_d, int ijnum, const double *radelem, const double *wjelem,
                            double rcutfac, double &rcut, double &wj, cudaStream_t s)
{
    int t = single_type(ti_d, tj_d, ijnum, s);
    if (t == -2) return 1;
    if (t < 0) return -1;
    double r = 0.5, w = 1.0;
    MDP_CUDA_TRY(cudaMemcpy(&r, radelem + t, sizeof(double), cudaMemcpyDeviceToHost));
    MDP_CUDA_TRY(cudaMemcpy(&w, wjelem + t, sizeof(double), cudaMemcpyDeviceToHost));
    rcut = (r + r) * rcutfac;
    wj = w;
    return 0;
}

// host-staging helper for the Julia-ABI wrappers
struct Stage {
    std::vector<void *> ptrs;
    bool ok = true;
    template <typename X> X *in(const X *h, size_t n)
    {
        X *d = nullptr;
        if (!ok || cudaMalloc(&d, sizeof(X) * std::max<size_t>(n, 1)) != cudaSuccess) { ok = false; return nullptr; }
        ptrs.push_back(d);
        if (n && cudaMemcpy(d, h, sizeof(X) * n, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
        return d;
    }
    template <typename X> X *alloc(size_t n)
    {
        X *d = nullptr;
        if (!ok || cudaMalloc(&d, sizeof(X) * std::max<size_t>(n, 1)) != cudaSuccess) { ok = false; return nullptr; }
        ptrs.push_back(d);
        return d;
    }
    template <typename X> int out(X *h, const X *d, size_t n)
    {
        if (!ok) return -1;
        if (cudaDeviceSynchronize() != cudaSuccess) return -1;
        return (n && cudaMemcpy(h, d, sizeof(X) * n, cudaMemcpyDeviceToHost) != cudaSuccess) ? -1 : 0;
    }
    ~Stage()
    {
        for (void *p : ptrs) cudaFree(p);
    }
};

}  // namespace mdp

using namespace mdp;

// ===========================================================================
// device-pointer operations (gpu* entry points of mdpgpucore.h)
// ===========================================================================
extern "C" {

void mdp_gpu_snap_compute_ui_f64(double *Utotr, double *Utoti, const double *rootpqarray, const double *rij,
                                 const double *wjelem, const double *radelem, double rmin0, double rfac0,
                                 double rcutfac, const int *idxu_block, const int *map, const int *aii,
                                 const int *ti, const int *tj, int twojmax, int idxu_max, int inum, int ijnum,
                                 int switchflag, int chemflag)
{
    (void)rootpqarray; (void)idxu_block; (void)idxu_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    double rcut, wj;
    const int several = chemflag ? 1 : pair_type_params(ti, tj, ijnum, radelem, wjelem, rcutfac, rcut, wj, 0);
    if (several < 0) return;
    if (several)
        ref_snap_ui_me(Utotr, Utoti, rij, radelem, wjelem, rcutfac, rfac0, rmin0, aii, ti, tj, map, chemflag, twojmax,
                       inum, ijnum, switchflag, 0);
    else
        ref_snap_ui(Utotr, Utoti, rij, rcut, wj, rfac0, rmin0, aii, twojmax, inum, ijnum, switchflag, 0);
}

void mdp_gpu_add_wself2ui_f64(double *Utotr, double *Utoti, double wself, const int *idxu_block, const int *type,
                              const int *map, const int *ai, int wselfall_flag, int chemflag, int idxu_max,
                              int nelements, int twojmax, int inum)
{
    (void)idxu_block; (void)ai; (void)idxu_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (chemflag || nelements != 1)
        ref_snap_wself_me(Utotr, Utoti, wself, type, map, chemflag, wselfall_flag, nelements, twojmax, inum, 0);
    else
        ref_snap_wself(Utotr, Utoti, wself, twojmax, inum, 0);
}

void mdp_gpu_snap_compute_ei_f64(double *eatom, const double *Utotr, const double *Utoti, const double *cglist,
                                 const double *bzero, const double *coeffelem, const int *ilist, const int *map,
                                 const int *type, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall,
                                 int bnorm_flag, int bzero_flag, int wselfall_flag, int quadraticflag, int inum)
{
    (void)cglist; (void)bzero; (void)idxb; (void)idxcg_block; (void)idxu_block; (void)idxu_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (quadraticflag) { set_error("quadratic SNAP goes through the ComputePairSnap chain, not this stage"); return; }
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (ncoeffall != 1 + idxb_max * nelements * nelements * nelements) {
        set_error("ncoeffall %d does not match idxb_max %d and %d element blocks", ncoeffall, idxb_max, nelements);
        return;
    }
    const int emax = atom_elements(type, map, inum, 1, 0);
    if (emax < 0) return;
    if (nelements > 1 || emax > 0) {
        ref_snap_ei_me(eatom, Utotr, Utoti, coeffelem, ilist, twojmax, nelements, ncoeffall, bnorm_flag, bzero_flag,
                       wselfall_flag, inum, 0);
        return;
    }
    std::vector<double> c(ncoeffall);
    if (cudaMemcpy(c.data(), coeffelem, sizeof(double) * ncoeffall, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("copying coeffelem failed");
        return;
    }
    ref_snap_ei(eatom, Utotr, Utoti, c.data(), ilist, twojmax, ncoeffall, bnorm_flag, bzero_flag, wselfall_flag, inum, 0);
}

void mdp_gpu_snap_compute_bi_f64(double *blist, const double *Utotr, const double *Utoti, const double *cglist,
                                 const double *bzero, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 const int *idxz_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum)
{
    (void)cglist; (void)bzero; (void)idxb; (void)idxcg_block; (void)idxu_block; (void)idxz_block; (void)idxb_max;
    (void)idxu_max; (void)idxz_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (nelements > 1)
        ref_snap_bi_me(blist, Utotr, Utoti, twojmax, nelements, bnorm_flag, bzero_flag, wselfall_flag, inum, 0);
    else
        ref_snap_bi(blist, Utotr, Utoti, twojmax, bnorm_flag, bzero_flag, inum, 0);
}

void mdp_gpu_snap_compute_yi_f64(double *ylist_r, double *ylist_i, const double *Utotr, const double *Utoti,
                                 const double *cglist, const double *coeffelem, const int *map, const int *type,
                                 const int *idxz, const int *idxb_block, const int *idxu_block,
                                 const int *idxcg_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int ncoeffall, int bnorm_flag, int inum)
{
    (void)cglist; (void)idxz; (void)idxb_block; (void)idxu_block; (void)idxcg_block; (void)idxu_max; (void)idxz_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (ncoeffall != 1 + idxb_max * nelements * nelements * nelements) {
        set_error("ncoeffall %d does not match idxb_max %d and %d element blocks", ncoeffall, idxb_max, nelements);
        return;
    }
    const int emax = atom_elements(type, map, inum, 1, 0);
    if (emax < 0) return;
    if (nelements > 1 || emax > 0) {
        ref_snap_yi_me(ylist_r, ylist_i, Utotr, Utoti, coeffelem, 0, twojmax, nelements, ncoeffall, bnorm_flag, inum, 0);
        return;
    }
    std::vector<double> c(ncoeffall);
    if (cudaMemcpy(c.data(), coeffelem, sizeof(double) * ncoeffall, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("copying coeffelem failed");
        return;
    }
    ref_snap_yi(ylist_r, ylist_i, Utotr, Utoti, c.data(), twojmax, ncoeffall, bnorm_flag, inum, 0);
}

void mdp_gpu_snap_compute_yi_beta_f64(double *ylist_r, double *ylist_i, const double *Utotr, const double *Utoti,
                                      const double *cglist, const double *beta, const int *idxz,
                                      const int *idxb_block, const int *idxu_block, const int *idxcg_block,
                                      int twojmax, int idxb_max, int idxu_max, int idxz_max, int nelements,
                                      int bnorm_flag, int inum)
{
    (void)cglist; (void)idxz; (void)idxb_block; (void)idxu_block; (void)idxcg_block; (void)idxu_max; (void)idxz_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (idxb_max != mdp_snap_ncoeff(twojmax)) { set_error("idxb_max %d does not match twojmax %d", idxb_max, twojmax); return; }
    if (nelements > 1)
        ref_snap_yi_me(ylist_r, ylist_i, Utotr, Utoti, beta, 1, twojmax, nelements, 0, bnorm_flag, inum, 0);
    else
        ref_snap_yi_beta(ylist_r, ylist_i, Utotr, Utoti, beta, twojmax, bnorm_flag, inum, 0);
}

void mdp_gpu_snap_compute_fi_f64(double *fatom, double *vatom, const double *ylist_r, const double *ylist_i,
                                 const double *rootpqarray, const double *rij, const double *wjelem,
                                 const double *radelem, double rmin0, double rfac0, double rcutfac,
                                 const int *idxu_block, const int *map, const int *aii, const int *ai, const int *aj,
                                 const int *ti, const int *tj, int twojmax, int idxu_max, int inum, int anum,
                                 int ijnum, int switchflag, int chemflag)
{
    (void)rootpqarray; (void)idxu_block; (void)idxu_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    double rcut, wj;
    const int several = chemflag ? 1 : pair_type_params(ti, tj, ijnum, radelem, wjelem, rcutfac, rcut, wj, 0);
    if (several < 0) return;
    if (several)
        ref_snap_fi_me(fatom, vatom, 0, anum, ylist_r, ylist_i, rij, radelem, wjelem, rcutfac, rfac0, rmin0, aii, ai,
                       aj, ti, tj, map, chemflag, twojmax, inum, ijnum, switchflag, 0);
    else
        ref_snap_fi(fatom, vatom, 0, anum, ylist_r, ylist_i, rij, rcut, wj, rfac0, rmin0, aii, ai, aj, twojmax, inum,
                    ijnum, switchflag, 0);
}

void mdp_gpu_neigh_pair_list_f64(int *pairnum, int *pairlist, const double *x, const double *rcutsq, const int *ilist,
                                 const int *neighlist, const int *neighnum, const int *atomtype, const int *alist,
                                 int inum, int jnum, int dim, int ntypes)
{
    if (dim != 3) { set_error("dim must be 3"); return; }
    k_ref_pair_count<<<(inum + 255) / 256, 256>>>(pairnum, x, rcutsq, ilist, neighlist, neighnum, atomtype, alist,
                                                   inum, jnum, ntypes, 0, pairlist);
}

void mdp_gpu_neigh_pairs_f64(double *xij, const double *x, int *aii, int *ai, int *aj, int *ti, int *tj,
                             const int *pairnum, const int *pairlist, const int *pairnumsum, const int *ilist,
                             const int *atomtype, const int *alist, int inum, int jnum, int dim)
{
    if (dim != 3) { set_error("dim must be 3"); return; }
    k_ref_pairs<<<(inum + 255) / 256, 256>>>(xij, x, aii, ai, aj, ti, tj, pairnum, pairlist, pairnumsum, ilist,
                                              atomtype, alist, inum, jnum);
}

// PREC_FLOAT builds of MDP: the same pair selection and pair vectors in float,
// rounded as the reference's float build rounds them
void mdp_gpu_neigh_pair_list_f32(int *pairnum, int *pairlist, const float *x, const float *rcutsq, const int *ilist,
                                 const int *neighlist, const int *neighnum, const int *atomtype, const int *alist,
                                 int inum, int jnum, int dim, int ntypes)
{
    if (dim != 3) { set_error("dim must be 3"); return; }
    k_ref_pair_count<<<(inum + 255) / 256, 256>>>(pairnum, x, rcutsq, ilist, neighlist, neighnum, atomtype, alist,
                                                   inum, jnum, ntypes, 0, pairlist);
}

void mdp_gpu_neigh_pairs_f32(float *xij, const float *x, int *aii, int *ai, int *aj, int *ti, int *tj,
                             const int *pairnum, const int *pairlist, const int *pairnumsum, const int *ilist,
                             const int *atomtype, const int *alist, int inum, int jnum, int dim)
{
    if (dim != 3) { set_error("dim must be 3"); return; }
    k_ref_pairs<<<(inum + 255) / 256, 256>>>(xij, x, aii, ai, aj, ti, tj, pairnum, pairlist, pairnumsum, ilist,
                                              atomtype, alist, inum, jnum);
}

// ===========================================================================
// MDP's Julia C ABI (src/Julia/Potential/cpuSnap.h), host pointers
// ===========================================================================
static int cnt_loop(int twojmax, int what)
{
    int n = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(twojmax, j1 + j2); j += 2) {
                if (what == 0 && j >= j1) n++;
                if (what == 1) n += (j1 + 1) * (j2 + 1);
                if (what == 2)
                    for (int mb = 0; 2 * mb <= j; mb++) n += j + 1;
            }
    return n;
}
int idxbcount(int twojmax) { return cnt_loop(twojmax, 0); }
int idxcgcount(int twojmax) { return cnt_loop(twojmax, 1); }
int idxzcount(int twojmax) { return cnt_loop(twojmax, 2); }
int idxucount(int twojmax) { return idxu_count(twojmax); }

// index lists, rootpq and CG table in the reference's layouts (cpuSnap.cpp:14-205)
void cpuInitSna(double *rootpqarray, double *cglist, double *factorial, int *idx_max, int *idxz, int *idxz_block,
                int *idxb, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax)
{
    (void)factorial;
    if (twojmax < 0 || twojmax > TJMAX) { set_error("twojmax %d out of range", twojmax); return; }
    const int J = twojmax, jd = J + 1;
    int ncg = 0, nb = 0, nz = 0, nu = 0;
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
                idxcg_block[j + j2 * jd + j1 * jd * jd] = ncg;
                ncg += (j1 + 1) * (j2 + 1);
            }
    for (int j = 0; j <= J; j++) { idxu_block[j] = nu; nu += (j + 1) * (j + 1); }
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
                if (j >= j1) {
                    idxb[3 * nb] = j1; idxb[3 * nb + 1] = j2; idxb[3 * nb + 2] = j;
                    idxb_block[j + j2 * jd + j1 * jd * jd] = nb++;
                }
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
                idxz_block[j + j2 * jd + j1 * jd * jd] = nz;
                for (int mb = 0; 2 * mb <= j; mb++)
                    for (int ma = 0; ma <= j; ma++) {
                        int *z = idxz + 10 * nz;
                        z[0] = j1; z[1] = j2; z[2] = j;
                        z[3] = std::max(0, (2 * ma - j - j2 + j1) / 2);
                        z[4] = (2 * ma - j - (2 * z[3] - j1) + j2) / 2;
                        z[5] = std::min(j1, (2 * ma - j + j2 + j1) / 2) - z[3] + 1;
                        z[6] = std::max(0, (2 * mb - j - j2 + j1) / 2);
                        z[7] = (2 * mb - j - (2 * z[6] - j1) + j2) / 2;
                        z[8] = std::min(j1, (2 * mb - j + j2 + j1) / 2) - z[6] + 1;
                        z[9] = idxu_block[j] + (j + 1) * mb + ma;
                        nz++;
                    }
            }
    idx_max[0] = ncg; idx_max[1] = nu; idx_max[2] = nb; idx_max[3] = nz;
    for (int p = 1; p <= J; p++)
        for (int q = 1; q <= J; q++) rootpqarray[p * jd + q] = sqrt((double)p / q);
    // CG: the TJMAX table restricted to j1 <= J, j <= J, re-blocked
    std::vector<double> full(NCG);
    host_cg_table(full.data());
    for (int j1 = 0; j1 <= J; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
                memcpy(cglist + idxcg_block[j + j2 * jd + j1 * jd * jd], full.data() + cg_block(j1, j2, j),
                       sizeof(double) * (j1 + 1) * (j2 + 1));
}

void cpuNeighPairList(int *pairnum, int *pairlist, double *x, double *rcutsq, int *ilist, int *neighlist,
                      int *neighnum, int *atomtype, int *alist, int inum, int dim, int ntypes)
{
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (dim != 3) { set_error("dim must be 3"); return; }
    int amax = 0, imax = 0;
    for (int ii = 0; ii < inum; ii++) imax = std::max(imax, ilist[ii] + 1);
    const int nnb = neighnum[imax];   // CSR over atoms 0..imax-1
    for (int k = 0; k < nnb; k++) amax = std::max(amax, neighlist[k] + 1);
    amax = std::max(amax, imax);
    Stage st;
    int *dpn = st.alloc<int>(inum + 1), *doff = st.alloc<int>(inum + 1);
    double *dx = st.in(x, 3 * (size_t)amax);
    double *drc = st.in(rcutsq, (size_t)(ntypes + 1) * (ntypes + 1));
    int *dil = st.in(ilist, inum), *dnl = st.in(neighlist, nnb), *dnn = st.in(neighnum, imax + 1);
    int *dat = st.in(atomtype, amax), *dal = st.in(alist, amax);
    int *tmp = st.alloc<int>(scan_tmp_ints(inum));
    if (!st.ok) { set_error("staging failed"); return; }
    k_ref_pair_count<<<(inum + 255) / 256, 256>>>(dpn, dx, drc, dil, dnl, dnn, dat, dal, inum, 0, ntypes, 1, nullptr);
    if (exclusive_scan(dpn, doff, inum, tmp, 0)) return;
    int total = 0;
    if (cudaMemcpy(&total, doff + inum, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    int *dpl = st.alloc<int>(total);
    if (!st.ok) { set_error("staging failed"); return; }
    k_ref_pair_emit_csr<<<(inum + 255) / 256, 256>>>(dpl, doff, dx, drc, dil, dnl, dnn, dat, dal, inum, ntypes);
    if (st.out(pairnum, dpn, inum) || st.out(pairlist, dpl, total)) set_error("cpuNeighPairList copy-back failed");
}

void cpuNeighPairs(double *xij, double *x, int *aii, int *ai, int *aj, int *ti, int *tj, int *pairlist,
                   int *pairnumsum, int *ilist, int *atomtype, int *alist, int inum, int dim)
{
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (dim != 3) { set_error("dim must be 3"); return; }
    const int ijnum = pairnumsum[inum];
    int amax = 0;
    for (int ii = 0; ii < inum; ii++) amax = std::max(amax, ilist[ii] + 1);
    for (int k = 0; k < ijnum; k++) amax = std::max(amax, pairlist[k] + 1);
    Stage st;
    double *dx = st.in(x, 3 * (size_t)amax);
    int *dpl = st.in(pairlist, ijnum), *dps = st.in(pairnumsum, inum + 1), *dil = st.in(ilist, inum);
    int *dat = st.in(atomtype, amax), *dal = st.in(alist, amax);
    double *oxij = st.alloc<double>(3 * (size_t)ijnum);
    int *oi = st.alloc<int>(5 * (size_t)ijnum);
    if (!st.ok) { set_error("staging failed"); return; }
    k_ref_pairs<<<(inum + 255) / 256, 256>>>(oxij, dx, oi, oi + ijnum, oi + 2 * ijnum, oi + 3 * ijnum, oi + 4 * ijnum,
                                              nullptr, dpl, dps, dil, dat, dal, inum, 0);
    if (st.out(xij, oxij, 3 * (size_t)ijnum) || st.out(aii, oi, ijnum) || st.out(ai, oi + ijnum, ijnum) ||
        st.out(aj, oi + 2 * ijnum, ijnum) || st.out(ti, oi + 3 * ijnum, ijnum) || st.out(tj, oi + 4 * ijnum, ijnum))
        set_error("cpuNeighPairs copy-back failed");
}

void cpuSnapComputeUi(double *Utotr, double *Utoti, double *rootpqarray, double *rij, double *wjelem, double *radelem,
                      double rmin0, double rfac0, double rcutfac, int *map, int *aii, int *ti, int *tj, int twojmax,
                      int idxu_max, int inum, int ijnum, int switchflag, int chemflag)
{
    (void)rootpqarray;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    bool several = chemflag != 0;
    int tmax = 0;
    for (int p = 0; p < ijnum; p++) {
        if (ti[p] != ti[0] || tj[p] != tj[0]) several = true;
        tmax = std::max(tmax, std::max(ti[p], tj[p]));
    }
    int nblk = 1;
    if (chemflag)
        for (int p = 0; p < ijnum; p++) nblk = std::max(nblk, map[tj[p]] + 1);
    if (nblk > MAXELEM) { set_error("element block %d out of range", nblk - 1); return; }
    const size_t nu = (size_t)idxu_max * inum * nblk;
    Stage st;
    double *ur = st.in(Utotr, nu), *ui = st.in(Utoti, nu), *dr = st.in(rij, 3 * (size_t)ijnum);
    int *da = st.in(aii, ijnum);
    if (!st.ok) { set_error("staging failed"); return; }
    if (several) {
        double *drad = st.in(radelem, tmax + 1), *dwj = st.in(wjelem, tmax + 1);
        int *dti = st.in(ti, ijnum), *dtj = st.in(tj, ijnum), *dmap = st.in(map, tmax + 1);
        if (!st.ok) { set_error("staging failed"); return; }
        if (ref_snap_ui_me(ur, ui, dr, drad, dwj, rcutfac, rfac0, rmin0, da, dti, dtj, dmap, chemflag, twojmax, inum,
                           ijnum, switchflag, 0))
            return;
    } else {
        const int t = ijnum > 0 ? tj[0] : 1;
        const double rcut = (radelem[t] + radelem[t]) * rcutfac, wj = wjelem[t];
        if (ref_snap_ui(ur, ui, dr, rcut, wj, rfac0, rmin0, da, twojmax, inum, ijnum, switchflag, 0)) return;
    }
    if (st.out(Utotr, ur, nu) || st.out(Utoti, ui, nu)) set_error("cpuSnapComputeUi copy-back failed");
}

void cpuAddWself2Ui(double *Utotr, double *Utoti, double wself, int *idxu_block, int *type, int *map,
                    int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax, int inum)
{
    (void)idxu_block;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const size_t nu = (size_t)idxu_max * inum * nelements;
    Stage st;
    double *ur = st.in(Utotr, nu), *ui = st.in(Utoti, nu);
    if (!st.ok) { set_error("staging failed"); return; }
    if (chemflag || nelements != 1) {
        int tmax = 0;
        for (int ii = 0; ii < inum; ii++) tmax = std::max(tmax, type[ii]);
        int *dt = st.in(type, inum), *dm = st.in(map, tmax + 1);
        if (!st.ok) { set_error("staging failed"); return; }
        if (ref_snap_wself_me(ur, ui, wself, dt, dm, chemflag, wselfall_flag, nelements, twojmax, inum, 0)) return;
    } else if (ref_snap_wself(ur, ui, wself, twojmax, inum, 0)) {
        return;
    }
    if (st.out(Utotr, ur, nu) || st.out(Utoti, ui, nu)) set_error("cpuAddWself2Ui copy-back failed");
}

void cpuSnapComputeEi(double *eatom, double *Utotr, double *Utoti, double *cglist, double *bzero, double *coeffelem,
                      int *ilist, int *map, int *type, int *idxb, int *idxcg_block, int *idxu_block, int twojmax,
                      int idxb_max, int idxu_max, int nelements, int ncoeffall, int bnorm_flag, int bzero_flag,
                      int wselfall_flag, int chemflag, int inum)
{
    (void)cglist; (void)bzero; (void)idxb; (void)idxcg_block; (void)idxu_block;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (ncoeffall != 1 + idxb_max * nelements * nelements * nelements) {
        set_error("ncoeffall %d does not match idxb_max %d and %d element blocks", ncoeffall, idxb_max, nelements);
        return;
    }
    int emax = 0;
    for (int ii = 0; ii < inum; ii++) emax = std::max(emax, ilist[ii] + 1);
    // the Julia library picks the coefficient set map[type] with chemflag, set 0 without
    int ecount = 1, tmax = 0;
    for (int ii = 0; ii < inum; ii++) tmax = std::max(tmax, type[ii]);
    if (chemflag)
        for (int ii = 0; ii < inum; ii++) ecount = std::max(ecount, map[type[ii]] + 1);
    const size_t nu = (size_t)idxu_max * inum * nelements;
    Stage st;
    double *ur = st.in(Utotr, nu), *ui = st.in(Utoti, nu), *de = st.in(eatom, emax);
    int *dil = st.in(ilist, inum);
    if (!st.ok) { set_error("staging failed"); return; }
    if (nelements > 1 || ecount > 1) {
        double *dc = st.in(coeffelem, (size_t)ecount * ncoeffall);
        int *dt = st.in(type, inum), *dm = st.in(map, tmax + 1);
        if (!st.ok) { set_error("staging failed"); return; }
        if (atom_elements(dt, dm, inum, chemflag, 0) < 0 ||
            ref_snap_ei_me(de, ur, ui, dc, dil, twojmax, nelements, ncoeffall, bnorm_flag, bzero_flag, wselfall_flag,
                           inum, 0))
            return;
    } else if (ref_snap_ei(de, ur, ui, coeffelem, dil, twojmax, ncoeffall, bnorm_flag, bzero_flag, wselfall_flag,
                           inum, 0)) {
        return;
    }
    if (st.out(eatom, de, emax)) set_error("cpuSnapComputeEi copy-back failed");
}

void cpuSnapComputeBi(double *blist, double *Utotr, double *Utoti, double *cglist, double *bzero, int *idxb,
                      int *idxcg_block, int *idxu_block, int *idxz_block, int twojmax, int idxb_max, int idxu_max,
                      int idxz_max, int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum)
{
    (void)cglist; (void)bzero; (void)idxb; (void)idxcg_block; (void)idxu_block; (void)idxz_block; (void)idxz_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const size_t ntri = (size_t)nelements * nelements * nelements;
    const size_t nu = (size_t)idxu_max * inum * nelements, nb = (size_t)idxb_max * inum * ntri;
    Stage st;
    double *ur = st.in(Utotr, nu), *ui = st.in(Utoti, nu), *db = st.in(blist, nb);
    if (!st.ok) { set_error("staging failed"); return; }
    if (nelements > 1) {
        if (ref_snap_bi_me(db, ur, ui, twojmax, nelements, bnorm_flag, bzero_flag, wselfall_flag, inum, 0)) return;
    } else if (ref_snap_bi(db, ur, ui, twojmax, bnorm_flag, bzero_flag, inum, 0)) {
        return;
    }
    if (st.out(blist, db, nb)) set_error("cpuSnapComputeBi copy-back failed");
}

void cpuSnapComputeYi(double *ylist_r, double *ylist_i, double *Utotr, double *Utoti, double *cglist, double *beta,
                      int *map, int *type, int *idxz, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax,
                      int idxb_max, int idxu_max, int idxz_max, int nelements, int ncoeffall, int bnorm_flag,
                      int chemflag, int inum)
{
    (void)cglist; (void)idxz; (void)idxb_block; (void)idxu_block; (void)idxcg_block; (void)idxz_max;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    if (ncoeffall != 1 + idxb_max * nelements * nelements * nelements) {
        set_error("ncoeffall %d does not match idxb_max %d and %d element blocks", ncoeffall, idxb_max, nelements);
        return;
    }
    // the Julia library picks the coefficient set map[type] with chemflag, set 0 without
    int ecount = 1, tmax = 0;
    for (int ii = 0; ii < inum; ii++) tmax = std::max(tmax, type[ii]);
    if (chemflag)
        for (int ii = 0; ii < inum; ii++) ecount = std::max(ecount, map[type[ii]] + 1);
    const size_t nu = (size_t)idxu_max * inum * nelements;
    Stage st;
    double *ur = st.in(Utotr, nu), *ui = st.in(Utoti, nu), *yr = st.alloc<double>(nu), *yi = st.alloc<double>(nu);
    if (!st.ok) { set_error("staging failed"); return; }
    if (nelements > 1 || ecount > 1) {
        double *dc = st.in(beta, (size_t)ecount * ncoeffall);
        int *dt = st.in(type, inum), *dm = st.in(map, tmax + 1);
        if (!st.ok) { set_error("staging failed"); return; }
        if (atom_elements(dt, dm, inum, chemflag, 0) < 0 ||
            ref_snap_yi_me(yr, yi, ur, ui, dc, 0, twojmax, nelements, ncoeffall, bnorm_flag, inum, 0))
            return;
    } else if (ref_snap_yi(yr, yi, ur, ui, beta, twojmax, ncoeffall, bnorm_flag, inum, 0)) {
        return;
    }
    if (st.out(ylist_r, yr, nu) || st.out(ylist_i, yi, nu)) set_error("cpuSnapComputeYi copy-back failed");
}

void cpuSnapComputeFi(double *fatom, double *vatom, double *ylist_r, double *ylist_i, double *rootpqarray, double *rij,
                      double *wjelem, double *radelem, double rmin0, double rfac0, double rcutfac, int *map, int *aii,
                      int *ai, int *aj, int *ti, int *tj, int twojmax, int idxu_max, int inum, int anum, int ijnum,
                      int switchflag, int chemflag)
{
    (void)rootpqarray;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    bool several = chemflag != 0;
    int tmax = 0;
    for (int p = 0; p < ijnum; p++) {
        if (ti[p] != ti[0] || tj[p] != tj[0]) several = true;
        tmax = std::max(tmax, std::max(ti[p], tj[p]));
    }
    int nblk = 1;
    if (chemflag)
        for (int p = 0; p < ijnum; p++) nblk = std::max(nblk, map[tj[p]] + 1);
    if (nblk > MAXELEM) { set_error("element block %d out of range", nblk - 1); return; }
    int fmax = std::max(inum, anum);
    for (int p = 0; p < ijnum; p++) fmax = std::max(fmax, std::max(ai[p], aj[p]) + 1);
    const size_t nu = (size_t)idxu_max * inum * nblk;
    Stage st;
    double *df = st.in(fatom, 3 * (size_t)fmax), *dv = st.in(vatom, 6 * (size_t)fmax);
    double *yr = st.in(ylist_r, nu), *yi = st.in(ylist_i, nu), *dr = st.in(rij, 3 * (size_t)ijnum);
    int *daii = st.in(aii, ijnum), *dai = st.in(ai, ijnum), *daj = st.in(aj, ijnum);
    if (!st.ok) { set_error("staging failed"); return; }
    if (several) {
        double *drad = st.in(radelem, tmax + 1), *dwj = st.in(wjelem, tmax + 1);
        int *dti = st.in(ti, ijnum), *dtj = st.in(tj, ijnum), *dmap = st.in(map, tmax + 1);
        if (!st.ok) { set_error("staging failed"); return; }
        if (ref_snap_fi_me(df, dv, 1, 0, yr, yi, dr, drad, dwj, rcutfac, rfac0, rmin0, daii, dai, daj, dti, dtj, dmap,
                           chemflag, twojmax, inum, ijnum, switchflag, 0))
            return;
    } else {
        const int t = ijnum > 0 ? tj[0] : 1;
        const double rcut = (radelem[t] + radelem[t]) * rcutfac, wj = wjelem[t];
        if (ref_snap_fi(df, dv, 1, 0, yr, yi, dr, rcut, wj, rfac0, rmin0, daii, dai, daj, twojmax, inum, ijnum,
                        switchflag, 0))
            return;
    }
    if (st.out(fatom, df, 3 * (size_t)fmax) || st.out(vatom, dv, 6 * (size_t)fmax))
        set_error("cpuSnapComputeFi copy-back failed");
}

}  // extern "C"
