// The SNAP stages of MDP's backend dispatch for PREC_FLOAT builds (dstype =
// float; src/C++/Common/mdpgpucore.h instantiates every gpu* template for float
// as well as double).  The caller's float device arrays are widened into
// double scratch, the stage runs on the double path of abi.cu, and its outputs
// are narrowed back into the caller's arrays: a float build of MDP gets
// results at least as accurate as its own float kernels, in the layouts and
// with the accumulate / overwrite semantics of the double entry points.
// Default stream, as the double path.  The scratch is library-owned and grows
// on demand; calls are serialised by a lock.
#include "common.cuh"
#include "engine.h"

#include "../../include/mdp_b200_gpucore.h"

#include <algorithm>
#include <mutex>

namespace mdp {
namespace {

std::mutex g_f32_mu;

__global__ void k_widen(const float *__restrict__ a, double *__restrict__ b, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}
__global__ void k_narrow(const double *__restrict__ a, float *__restrict__ b, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
// largest value among the first n ints, into *out (atomicMax; *out preset)
__global__ void k_max_int(const int *__restrict__ a, long n, int *__restrict__ out)
{
    int m = -1;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        m = max(m, a[i]);
    atomicMax(out, m);
}

unsigned grid_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 4096)); }

// double shadows of float arguments, one per argument slot
struct Shadows {
    DevBuf b[10];
    DevBuf imax;
};
Shadows &shadows()
{
    static Shadows s;
    return s;
}

double *widen(int slot, const float *src, long n)
{
    DevBuf &d = shadows().b[slot];
    if (d.ensure(sizeof(double) * (size_t)std::max<long>(n, 1))) return nullptr;
    if (n > 0 && src) {
        k_widen<<<grid_for(n), 256>>>(src, d.as<double>(), n);
        count_launches(1);
    }
    return d.as<double>();
}

void narrow(float *dst, int slot, long n)
{
    if (n <= 0 || !dst) return;
    k_narrow<<<grid_for(n), 256>>>(shadows().b[slot].as<double>(), dst, n);
    count_launches(1);
}

// 1 + the largest value in a[0..n) and b[0..n) (the length an array indexed by
// those values is read to: radelem and wjelem by the pair types, eatom by
// ilist), or -1
int max_plus_one(const int *ti, const int *tj, long n)
{
    DevBuf &m = shadows().imax;
    if (m.ensure(sizeof(int))) return -1;
    int h = 0;
    if (cudaMemcpy(m.p, &h, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (n > 0) {
        k_max_int<<<grid_for(n), 256>>>(ti, n, m.as<int>());
        k_max_int<<<grid_for(n), 256>>>(tj, n, m.as<int>());
        count_launches(2);
    }
    if (cudaMemcpy(&h, m.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return h + 1;
}

// largest map[idx[i]] over i < n, into *out
__global__ void k_max_mapped(const int *__restrict__ idx, const int *__restrict__ map, long n, int *__restrict__ out)
{
    int m = -1;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        m = max(m, map[idx[i]]);
    atomicMax(out, m);
}

// 1 + the largest map[idx[i]], i < n (at least 1): the element blocks the pairs
// reach (idx = tj) or the coefficient sets the atoms use (idx = type); -1 on error
int mapped_count(const int *idx, const int *map, long n)
{
    DevBuf &m = shadows().imax;
    if (m.ensure(sizeof(int))) return -1;
    int h = 0;
    if (cudaMemcpy(m.p, &h, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (n > 0) {
        k_max_mapped<<<grid_for(n), 256>>>(idx, map, n, m.as<int>());
        count_launches(1);
    }
    if (cudaMemcpy(&h, m.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (h + 1 > MAXELEM) { set_error("element index %d out of range", h); return -1; }
    return std::max(h + 1, 1);
}

}  // namespace
}  // namespace mdp

using namespace mdp;

extern "C" {

void mdp_gpu_snap_compute_ui_f32(float *Utotr, float *Utoti, const float *rootpqarray, const float *rij,
                                 const float *wjelem, const float *radelem, float rmin0, float rfac0, float rcutfac,
                                 const int *idxu_block, const int *map, const int *aii, const int *ti, const int *tj,
                                 int twojmax, int idxu_max, int inum, int ijnum, int switchflag, int chemflag)
{
    (void)rootpqarray;
    std::lock_guard<std::mutex> lk(g_f32_mu);
    const int nblk = chemflag ? mapped_count(tj, map, ijnum) : 1;   // U element blocks the pairs reach
    if (nblk < 1) return;
    const long nu = (long)idxu_max * inum * nblk;
    const int nt = max_plus_one(ti, tj, ijnum);
    if (nt < 1) { set_error("gpuSnapComputeUi (float): reading the pair types failed"); return; }
    double *ur = widen(0, Utotr, nu), *ui = widen(1, Utoti, nu), *dr = widen(2, rij, 3L * ijnum);
    double *wj = widen(3, wjelem, nt), *rad = widen(4, radelem, nt);
    if (!ur || !ui || !dr || !wj || !rad) return;
    mdp_gpu_snap_compute_ui_f64(ur, ui, nullptr, dr, wj, rad, rmin0, rfac0, rcutfac, idxu_block, map, aii, ti, tj,
                                twojmax, idxu_max, inum, ijnum, switchflag, chemflag);
    narrow(Utotr, 0, nu);
    narrow(Utoti, 1, nu);
}

void mdp_gpu_add_wself2ui_f32(float *Utotr, float *Utoti, float wself, const int *idxu_block, const int *type,
                              const int *map, const int *ai, int wselfall_flag, int chemflag, int idxu_max,
                              int nelements, int twojmax, int inum)
{
    std::lock_guard<std::mutex> lk(g_f32_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const long nu = (long)idxu_max * nelements * inum;
    double *ur = widen(0, Utotr, nu), *ui = widen(1, Utoti, nu);
    if (!ur || !ui) return;
    mdp_gpu_add_wself2ui_f64(ur, ui, wself, idxu_block, type, map, ai, wselfall_flag, chemflag, idxu_max, nelements,
                             twojmax, inum);
    narrow(Utotr, 0, nu);
    narrow(Utoti, 1, nu);
}

// eatom is indexed through ilist (the block's atoms within the whole system),
// so its length is 1 + max(ilist)
void mdp_gpu_snap_compute_ei_f32(float *eatom, const float *Utotr, const float *Utoti, const float *cglist,
                                 const float *bzero, const float *coeffelem, const int *ilist, const int *map,
                                 const int *type, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall,
                                 int bnorm_flag, int bzero_flag, int wselfall_flag, int quadraticflag, int inum)
{
    (void)cglist; (void)bzero;
    std::lock_guard<std::mutex> lk(g_f32_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const long nu = (long)idxu_max * nelements * inum;
    const int ne = max_plus_one(ilist, ilist, inum);
    if (ne < 1) { set_error("gpuSnapComputeEi (float): reading ilist failed"); return; }
    // coefficient sets map[type] (one per element even when nelements is 1 without chemflag)
    const int nsets = std::max(nelements, mapped_count(type, map, inum));
    if (nsets < 1) return;
    double *e = widen(0, eatom, ne), *ur = widen(1, Utotr, nu), *ui = widen(2, Utoti, nu);
    double *c = widen(3, coeffelem, (long)ncoeffall * nsets);
    if (!e || !ur || !ui || !c) return;
    mdp_gpu_snap_compute_ei_f64(e, ur, ui, nullptr, nullptr, c, ilist, map, type, idxb, idxcg_block, idxu_block,
                                twojmax, idxb_max, idxu_max, nelements, ncoeffall, bnorm_flag, bzero_flag,
                                wselfall_flag, quadraticflag, inum);
    narrow(eatom, 0, ne);
}

void mdp_gpu_snap_compute_bi_f32(float *blist, const float *Utotr, const float *Utoti, const float *cglist,
                                 const float *bzero, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 const int *idxz_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum)
{
    (void)cglist; (void)bzero;
    std::lock_guard<std::mutex> lk(g_f32_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const long nu = (long)idxu_max * nelements * inum;
    const long nb = (long)idxb_max * inum * nelements * nelements * nelements;   // [triple][k][inum]
    double *b = widen(0, nullptr, nb), *ur = widen(1, Utotr, nu), *ui = widen(2, Utoti, nu);
    if (!b || !ur || !ui) return;
    mdp_gpu_snap_compute_bi_f64(b, ur, ui, nullptr, nullptr, idxb, idxcg_block, idxu_block, idxz_block, twojmax,
                                idxb_max, idxu_max, idxz_max, nelements, bnorm_flag, bzero_flag, wselfall_flag, inum);
    narrow(blist, 0, nb);
}

void mdp_gpu_snap_compute_yi_f32(float *ylist_r, float *ylist_i, const float *Utotr, const float *Utoti,
                                 const float *cglist, const float *coeffelem, const int *map, const int *type,
                                 const int *idxz, const int *idxb_block, const int *idxu_block,
                                 const int *idxcg_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int ncoeffall, int bnorm_flag, int inum)
{
    (void)cglist;
    std::lock_guard<std::mutex> lk(g_f32_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const long nu = (long)idxu_max * nelements * inum;
    const int nsets = std::max(nelements, mapped_count(type, map, inum));
    if (nsets < 1) return;
    double *yr = widen(0, nullptr, nu), *yi = widen(1, nullptr, nu), *ur = widen(2, Utotr, nu),
           *ui = widen(3, Utoti, nu), *c = widen(4, coeffelem, (long)ncoeffall * nsets);
    if (!yr || !yi || !ur || !ui || !c) return;
    mdp_gpu_snap_compute_yi_f64(yr, yi, ur, ui, nullptr, c, map, type, idxz, idxb_block, idxu_block, idxcg_block,
                                twojmax, idxb_max, idxu_max, idxz_max, nelements, ncoeffall, bnorm_flag, inum);
    narrow(ylist_r, 0, nu);
    narrow(ylist_i, 1, nu);
}

void mdp_gpu_snap_compute_yi_beta_f32(float *ylist_r, float *ylist_i, const float *Utotr, const float *Utoti,
                                      const float *cglist, const float *beta, const int *idxz, const int *idxb_block,
                                      const int *idxu_block, const int *idxcg_block, int twojmax, int idxb_max,
                                      int idxu_max, int idxz_max, int nelements, int bnorm_flag, int inum)
{
    (void)cglist;
    std::lock_guard<std::mutex> lk(g_f32_mu);
    if (nelements < 1 || nelements > MAXELEM) { set_error("nelements %d out of range", nelements); return; }
    const long nu = (long)idxu_max * nelements * inum;
    double *yr = widen(0, nullptr, nu), *yi = widen(1, nullptr, nu), *ur = widen(2, Utotr, nu),
           *ui = widen(3, Utoti, nu),
           *b = widen(4, beta, (long)idxb_max * inum * nelements * nelements * nelements);
    if (!yr || !yi || !ur || !ui || !b) return;
    mdp_gpu_snap_compute_yi_beta_f64(yr, yi, ur, ui, nullptr, b, idxz, idxb_block, idxu_block, idxcg_block, twojmax,
                                     idxb_max, idxu_max, idxz_max, nelements, bnorm_flag, inum);
    narrow(ylist_r, 0, nu);
    narrow(ylist_i, 1, nu);
}

// fatom [anum][3] and vatom [6][anum] accumulate, as in the double entry point
void mdp_gpu_snap_compute_fi_f32(float *fatom, float *vatom, const float *ylist_r, const float *ylist_i,
                                 const float *rootpqarray, const float *rij, const float *wjelem,
                                 const float *radelem, float rmin0, float rfac0, float rcutfac, const int *idxu_block,
                                 const int *map, const int *aii, const int *ai, const int *aj, const int *ti,
                                 const int *tj, int twojmax, int idxu_max, int inum, int anum, int ijnum,
                                 int switchflag, int chemflag)
{
    (void)rootpqarray;
    std::lock_guard<std::mutex> lk(g_f32_mu);
    const int nblk = chemflag ? mapped_count(tj, map, ijnum) : 1;   // Y element blocks the pairs read
    if (nblk < 1) return;
    const long nu = (long)idxu_max * inum * nblk;
    const int nt = max_plus_one(ti, tj, ijnum);
    if (nt < 1) { set_error("gpuSnapComputeFi (float): reading the pair types failed"); return; }
    double *f = widen(0, fatom, 3L * anum), *v = widen(1, vatom, 6L * anum), *yr = widen(2, ylist_r, nu),
           *yi = widen(3, ylist_i, nu), *dr = widen(4, rij, 3L * ijnum), *wj = widen(5, wjelem, nt),
           *rad = widen(6, radelem, nt);
    if (!f || !v || !yr || !yi || !dr || !wj || !rad) return;
    mdp_gpu_snap_compute_fi_f64(f, v, yr, yi, nullptr, dr, wj, rad, rmin0, rfac0, rcutfac, idxu_block, map, aii, ai,
                                aj, ti, tj, twojmax, idxu_max, inum, anum, ijnum, switchflag, chemflag);
    narrow(fatom, 0, 3L * anum);
    narrow(vatom, 1, 6L * anum);
}

}  // extern "C"
