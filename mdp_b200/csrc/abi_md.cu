// The MD-loop operations behind MDP's backend dispatch (src/C++/Common/mdpcore.h
// with backend == 2) other than the SNAP stages: prefix sums, ghost atoms, cell
// lists, full neighbour lists, the velocity-Verlet integrator, periodic
// wrapping, per-atom kinetic energy and column sums.  Argument lists are those
// of src/C++/Common/mdpgpucore.h; all arrays are device arrays in the
// reference's layouts (x [natom][dim], neighbour rows [atom][jnum]) except
// dtarray, which the reference reads on the host.  Positions are mapped to
// the unit cell and distances formed with the reference CPU code's rounding
// (products and sums rounded in its order, no fused multiply-add), so ghosts,
// cells and neighbour sets equal the CPU reference's exactly.  Default stream.
#include "common.cuh"
#include "engine.h"

#include <algorithm>
#include <mutex>

namespace mdp {
namespace {

std::mutex g_md_mu;

constexpr int TB = 256;
unsigned blocks_for(long n) { return (unsigned)std::max<long>(1, (n + TB - 1) / TB); }

// correctly rounded arithmetic without contraction, in the precision of the
// reference build (double, or float for PREC_FLOAT builds of MDP)
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// s2rmap * (a, b, c): ((m0 a + m3 b) + m6 c), each product rounded
template <typename T>
__device__ __forceinline__ T map0(const T *m, int r, T a, T b, T c)
{
    return add_rn(add_rn(mul_rn(m[r], a), mul_rn(m[3 + r], b)), mul_rn(m[6 + r], c));
}

template <typename T>
__device__ __forceinline__ T dist2(T a0, T a1, T a2, T b0, T b1, T b2)
{
    const T d0 = sub_rn(b0, a0), d1 = sub_rn(b1, a1), d2 = sub_rn(b2, a2);
    return add_rn(add_rn(mul_rn(d0, d0), mul_rn(d1, d1)), mul_rn(d2, d2));
}

// ---- ghosts (cpuNeighborList3D.cpp:282-330) --------------------------------
template <typename T>
__global__ void k_md_ghost_flags(int *__restrict__ gnum, int *__restrict__ inside, const T *__restrict__ x,
                                 const T *__restrict__ pim, const T *__restrict__ wc,
                                 const T *__restrict__ s2r, int inum, int pnum)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    const T x0 = x[3 * (size_t)i], x1 = x[3 * (size_t)i + 1], x2 = x[3 * (size_t)i + 2];
    int n = 0;
    for (int j = 1; j < pnum; j++) {
        const T y0 = add_rn(x0, pim[3 * j]), y1 = add_rn(x1, pim[3 * j + 1]),
                     y2 = add_rn(x2, pim[3 * j + 2]);
        const T s0 = map0(s2r, 0, y0, y1, y2), s1 = map0(s2r, 1, y0, y1, y2), s2 = map0(s2r, 2, y0, y1, y2);
        const int in = (wc[0] <= s0 && s0 <= wc[18] && wc[1] <= s1 && s1 <= wc[19] && wc[2] <= s2 && s2 <= wc[20]);
        inside[(j - 1) + (size_t)i * (pnum - 1)] = in;
        n += in;
    }
    gnum[i] = n;
}

template <typename T>
__global__ void k_md_ghost_emit(int *__restrict__ alist, const int *__restrict__ inside,
                                const int *__restrict__ goff, T *__restrict__ x, const T *__restrict__ pim,
                                int inum, int pnum)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    alist[i] = i;
    const T x0 = x[3 * (size_t)i], x1 = x[3 * (size_t)i + 1], x2 = x[3 * (size_t)i + 2];
    long q = (long)inum + goff[i];
    for (int j = 1; j < pnum; j++) {
        if (!inside[(j - 1) + (size_t)i * (pnum - 1)]) continue;
        x[3 * q] = add_rn(x0, pim[3 * j]);
        x[3 * q + 1] = add_rn(x1, pim[3 * j + 1]);
        x[3 * q + 2] = add_rn(x2, pim[3 * j + 2]);
        alist[q] = i;
        q++;
    }
}

// ---- cells (cpuNeighborList3D.cpp:334-357, cpuNeighborList2D.cpp:298-307) --
// the first cell (from m, where m = 1 for local atoms and 0 for ghosts) whose
// closed interval holds the coordinate; nc - m when none does
template <typename T>
__device__ __forceinline__ int cell_search(const T *__restrict__ eta, int n, int m, T s)
{
    int j = m;
    for (; j < n - m; j++)
        if (eta[j] <= s && s <= eta[j + 1]) break;
    return j;
}

template <typename T>
__global__ void k_md_cell_list(int *__restrict__ clist, const T *__restrict__ x, const T *__restrict__ e1,
                               const T *__restrict__ e2, const T *__restrict__ e3,
                               const T *__restrict__ s2r, const int *__restrict__ nc, int inum, int natom)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natom) return;
    const int m = i < inum ? 1 : 0;
    const T a = x[3 * (size_t)i], b = x[3 * (size_t)i + 1], c = x[3 * (size_t)i + 2];
    const int n0 = nc[0], n1 = nc[1], n2 = nc[2];
    const int j1 = cell_search(e1, n0, m, map0(s2r, 0, a, b, c));
    const int j2 = cell_search(e2, n1, m, map0(s2r, 1, a, b, c));
    const int j3 = cell_search(e3, n2, m, map0(s2r, 2, a, b, c));
    clist[i] = j1 + n0 * j2 + n0 * n1 * j3;
}

// atoms whose cell id lies outside 0..ncell-1 are left out
__global__ void k_md_cell_count(const int *__restrict__ clist, int natom, int ncell, int *__restrict__ cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < natom && clist[i] >= 0 && clist[i] < ncell) atomicAdd(&cnt[clist[i]], 1);
}

__global__ void k_md_cell_fill(const int *__restrict__ clist, int natom, int ncell, const int *__restrict__ start,
                               int *__restrict__ cursor, int *__restrict__ c2alist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natom) return;
    const int c = clist[i];
    if (c < 0 || c >= ncell) return;
    c2alist[start[c] + atomicAdd(&cursor[c], 1)] = i;
}

// atoms ascending within each cell (the order of a stable sort by cell), and
// the sorted cell ids into c2anum
__global__ void k_md_cell_order(int ncell, const int *__restrict__ start, int *__restrict__ c2alist,
                                int *__restrict__ c2anum)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int s = start[c], e = start[c + 1];
    for (int a = s + 1; a < e; a++) {
        const int v = c2alist[a];
        int b = a - 1;
        while (b >= s && c2alist[b] > v) { c2alist[b + 1] = c2alist[b]; b--; }
        c2alist[b + 1] = v;
    }
    for (int a = s; a < e; a++) c2anum[a] = c;
}

// ---- full neighbour lists (cpuNeighborList3D.cpp:361-443) ------------------
// rows filled in the reference's visiting order, truncated at jnum
template <typename T>
__global__ void k_md_neigh_cells(int *__restrict__ nl, int *__restrict__ nn, const T *__restrict__ x,
                                 const T *__restrict__ rcutsq, const int *__restrict__ alist,
                                 const int *__restrict__ clist, const int *__restrict__ c2alist,
                                 const int *__restrict__ c2anumsum, const int *__restrict__ nc, int inum, int jnum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = alist[ii];
    const T xi0 = x[3 * (size_t)i], xi1 = x[3 * (size_t)i + 1], xi2 = x[3 * (size_t)i + 2];
    const T rc = rcutsq[0];
    const int n0 = nc[0], n01 = nc[0] * nc[1];
    const int ca = clist[i], cb = ca % n01, j3 = (ca - cb) / n01, j1 = cb % n0, j2 = (cb - j1) / n0;
    int *row = nl + (size_t)jnum * i;
    int cnt = 0;
    for (int d1 = -1; d1 <= 1 && cnt < jnum; d1++)
        for (int d2 = -1; d2 <= 1 && cnt < jnum; d2++)
            for (int d3 = -1; d3 <= 1 && cnt < jnum; d3++) {
                // cells off the x/y grid or below it hold no atoms (the reference
                // reads past its arrays there).  z is left open: MDP passes
                // nc[2] = 0 (Configuration.cpp:847-848), so locals sit in z layer
                // 1 and ghosts in layer 0, and the stencil's layer 2 lies within
                // the ncell = nc0 nc1 (ne2 + 2) cells its prefix sums cover
                if (j1 + d1 < 0 || j1 + d1 >= n0 || j2 + d2 < 0 || j2 + d2 >= nc[1] || j3 + d3 < 0) continue;
                const int k = (j1 + d1) + n0 * (j2 + d2) + n01 * (j3 + d3);
                const int s = c2anumsum[k], e = c2anumsum[k + 1];
                for (int l = s; l < e && cnt < jnum; l++) {
                    const int j = c2alist[l];
                    if (j == i) continue;
                    if (dist2(xi0, xi1, xi2, x[3 * (size_t)j], x[3 * (size_t)j + 1], x[3 * (size_t)j + 2]) <= rc)
                        row[cnt++] = j;
                }
            }
    nn[ii] = cnt;
}

template <typename T>
__global__ void k_md_neigh_all(int *__restrict__ nl, int *__restrict__ nn, const T *__restrict__ x,
                               const T *__restrict__ rcutsq, int anum, int inum, int jnum)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inum) return;
    const T xi0 = x[3 * (size_t)i], xi1 = x[3 * (size_t)i + 1], xi2 = x[3 * (size_t)i + 2];
    const T rc = rcutsq[0];
    int *row = nl + (size_t)jnum * i;
    int cnt = 0;
    for (int j = 0; j < anum && cnt < jnum; j++) {
        if (j == i) continue;
        if (dist2(xi0, xi1, xi2, x[3 * (size_t)j], x[3 * (size_t)j + 1], x[3 * (size_t)j + 2]) <= rc) row[cnt++] = j;
    }
    nn[i] = cnt;
}

// ---- velocity Verlet (cpuVelocityIntegration.cpp:307-420) ------------------
// stage 0: v += dtfm f, [limit], x += dtv v;  stage 1: v += dtfm f, [limit]
template <typename T>
__global__ void k_md_verlet(T *__restrict__ x, T *__restrict__ v, const T *__restrict__ f,
                            const T *__restrict__ mass, const int *__restrict__ type,
                            const int *__restrict__ ilist, T dtf, T dtv, T vlimitsq, int limit,
                            int stage, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii];
    const T dtfm = div_rn(dtf, mass[type[i]]);
    T *vi = v + (size_t)dim * i;
    const T *fi = f + (size_t)dim * i;
    for (int d = 0; d < dim; d++) vi[d] = add_rn(vi[d], mul_rn(dtfm, fi[d]));
    if (limit) {
        T vsq = mul_rn(vi[0], vi[0]);
        for (int d = 1; d < dim; d++) vsq = add_rn(vsq, mul_rn(vi[d], vi[d]));
        if (vsq > vlimitsq) {
            const T scale = sqrt(div_rn(vlimitsq, vsq));
            for (int d = 0; d < dim; d++) vi[d] = mul_rn(vi[d], scale);
        }
    }
    if (stage == 0)
        for (int d = 0; d < dim; d++) x[(size_t)dim * i + d] = add_rn(x[(size_t)dim * i + d], mul_rn(dtv, vi[d]));
}

// velocity scaling of the thermostat (cpuVelocityIntegration.cpp:465-503; the
// reference's bias flag changes nothing there)
template <typename T>
__global__ void k_md_vscale(T *__restrict__ v, T factor, const int *__restrict__ ilist, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    T *vi = v + (size_t)dim * ilist[ii];
    for (int d = 0; d < dim; d++) vi[d] *= factor;
}

// ---- periodic wrapping (cpuDomain.cpp:235-385) -----------------------------
// the velocity shift of a deforming box for crossing boundary d (rates in
// Voigt order xx yy zz yz xz xy)
template <typename T>
__device__ __forceinline__ void deform_shift(T *v, const T *hr, int d, T sg)
{
    if (d == 0) v[0] += sg * hr[0];
    if (d == 1) { v[0] += sg * hr[5]; v[1] += sg * hr[1]; }
    if (d == 2) { v[0] += sg * hr[4]; v[1] += sg * hr[3]; v[2] += sg * hr[2]; }
}

template <typename T>
__global__ void k_md_pbc(T *__restrict__ x, T *__restrict__ v, int *__restrict__ image,
                         const T *__restrict__ hi, const T *__restrict__ lo,
                         const T *__restrict__ hil, const T *__restrict__ lol, const T *__restrict__ h,
                         const T *__restrict__ hinv, const T *__restrict__ hr, const int *__restrict__ pbc,
                         int vdeform, int triclinic, int dim, int nlocal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlocal) return;
    T *xi = x + (size_t)dim * i, *vi = v + (size_t)dim * i;
    int *im = image + (size_t)dim * i;
    T c[3] = {T(0), T(0), T(0)};
    const T *L = h, *lb = lo, *ub = hi;
    if (triclinic) {
        // lambda coordinates
        const T dx = xi[0] - lo[0], dy = xi[1] - lo[1];
        c[0] = hinv[0] * dx + hinv[5] * dy;
        c[1] = hinv[1] * dy;
        if (dim == 3) {
            const T dz = xi[2] - lo[2];
            c[0] += hinv[4] * dz;
            c[1] += hinv[3] * dz;
            c[2] = hinv[2] * dz;
        }
        L = hil; lb = lol; ub = hil;
    } else {
        for (int d = 0; d < dim; d++) c[d] = xi[d];
    }
    for (int d = 0; d < dim; d++) {
        if (!pbc[d]) continue;
        if (c[d] < lb[d]) {
            c[d] += L[d];
            if (vdeform) deform_shift(vi, hr, d, T(1));
            im[d] -= 1;
        }
        if (c[d] >= ub[d]) {
            c[d] -= L[d];
            c[d] = fmax(c[d], lb[d]);
            if (vdeform) deform_shift(vi, hr, d, T(-1));
            im[d] += 1;
        }
    }
    if (triclinic) {
        xi[0] = h[0] * c[0] + h[5] * c[1] + lo[0];
        xi[1] = h[1] * c[1] + lo[1];
        if (dim == 3) {
            xi[0] += h[4] * c[2];
            xi[1] += h[3] * c[2];
            xi[2] = h[2] * c[2] + lo[2];
        }
    } else {
        for (int d = 0; d < dim; d++) xi[d] = c[d];
    }
}

// ---- kinetic energy and column sums (cpuComputes.cpp:435-451,
// cpuArrayOperations.cpp:94-103) ---------------------------------------------
template <typename T>
__global__ void k_md_ke(T *__restrict__ ke, const T *__restrict__ mass, const T *__restrict__ v,
                        T mvv2e, const int *__restrict__ type, const int *__restrict__ ilist, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii];
    const T *vi = v + (size_t)dim * i;
    T s = add_rn(mul_rn(vi[0], vi[0]), mul_rn(vi[1], vi[1]));
    if (dim == 3) s = add_rn(s, mul_rn(vi[2], vi[2]));
    ke[ii] = mul_rn(mul_rn(mul_rn(T(0.5), mvv2e), mass[type[i]]), s);
}

// one CTA per column; a fixed tree over the rows
template <typename T>
__global__ void __launch_bounds__(TB) k_md_colsum(T *__restrict__ b, const T *__restrict__ a, int n)
{
    __shared__ T sh[TB];
    const T *col = a + (size_t)n * blockIdx.x;
    T s = T(0);
    for (int i = threadIdx.x; i < n; i += TB) s += col[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = TB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) b[blockIdx.x] = sh[0];
}

struct CellScratch {
    DevBuf cnt, cursor, tmp;
};
CellScratch &cell_scratch()
{
    static CellScratch c;
    return c;
}

bool check_launch(const char *fn)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { set_error("%s: %s", fn, cudaGetErrorString(e)); return false; }
    return true;
}

}  // namespace
}  // namespace mdp

using namespace mdp;

namespace {

template <typename T>
void atom_list3d_t(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums, int *d_incr,
                             T *x, const T *pimages, const T *wc, const T *s2rmap, int inum,
                             int pnum, int dim)
{
    (void)d_incr;
    if (dim != 3) { set_error("gpuAtomList3D: dim must be 3"); return; }
    if (inum <= 0) return;
    k_md_ghost_flags<<<blocks_for(inum), TB>>>(glistnum, inside, x, pimages, wc, s2rmap, inum, pnum);
    if (exclusive_scan(glistnum, glistnumsum, inum, d_sums, 0)) return;
    k_md_ghost_emit<<<blocks_for(inum), TB>>>(alist, inside, glistnumsum, x, pimages, inum, pnum);
    count_launches(5);
    check_launch("gpuAtomList3D");
}

template <typename T>
void cell_list3d_t(int *clist, const T *xi, const T *eta1, const T *eta2,
                             const T *eta3, const T *s2rmap, const int *nc, int inum, int natom, int dim)
{
    if (dim != 3) { set_error("gpuCellList3D: dim must be 3"); return; }
    if (natom <= 0) return;
    k_md_cell_list<<<blocks_for(natom), TB>>>(clist, xi, eta1, eta2, eta3, s2rmap, nc, inum, natom);
    count_launches(1);
    check_launch("gpuCellList3D");
}

template <typename T>
void full_neighbor_list3d_cells_t(int *neighborlist, int *neighbornum, const T *x,
                                            const T *rcutsq, const int *alist, const int *clist,
                                            const int *c2alist, const int *c2anumsum, const int *nc, int inum,
                                            int jnum, int dim)
{
    if (dim != 3) { set_error("gpuFullNeighborList3D: dim must be 3"); return; }
    if (inum <= 0) return;
    k_md_neigh_cells<<<blocks_for(inum), TB>>>(neighborlist, neighbornum, x, rcutsq, alist, clist, c2alist,
                                                c2anumsum, nc, inum, jnum);
    count_launches(1);
    check_launch("gpuFullNeighborList3D");
}

template <typename T>
void full_neighbor_list3d_t(int *neighborlist, int *neighbornum, const T *x, const T *rcutsq,
                                      int anum, int inum, int jnum, int dim)
{
    if (dim != 3) { set_error("gpuFullNeighborList3D: dim must be 3"); return; }
    if (inum <= 0) return;
    k_md_neigh_all<<<blocks_for(inum), TB>>>(neighborlist, neighbornum, x, rcutsq, anum, inum, jnum);
    count_launches(1);
    check_launch("gpuFullNeighborList3D");
}

template <typename T>
int temperature(T &t, T *ke, T *tmp, const T *mass, const T *v, T tfactor,
                       const int *type, const int *ilist, int dim, int inum)
{
    k_md_ke<<<blocks_for(inum), TB>>>(ke, mass, v, T(2) * tfactor, type, ilist, dim, inum);
    k_md_colsum<<<1, TB>>>(tmp, ke, inum);
    count_launches(2);
    if (cudaMemcpy(&t, tmp, sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("temperature read-back failed");
        return -1;
    }
    return 0;
}

template <typename T>
void nose_hoover(T *v, const int *ilist, int dim, int inum, const T *dtarray, T *tarray,
                        T *eta_mass, T *eta, T *eta_dot, T *eta_dotdot, int eta_mass_flag,
                        int mtchain, int nc_tchain)
{
    const T dt = dtarray[0], half = 0.5 * dt, quarter = 0.25 * dt, eighth = 0.125 * dt;
    const T t_freq = tarray[2], t_target = tarray[3], tdof = tarray[5], boltz = tarray[6], drag = tarray[7];
    const T drag_f = 1.0 - (dt * t_freq * drag / nc_tchain), nc = 1.0 / nc_tchain;
    const T ke_target = tdof * boltz * t_target;
    T ke_now = tdof * boltz * tarray[4];
    if (eta_mass_flag) {
        eta_mass[0] = tdof * boltz * t_target / (t_freq * t_freq);
        for (int c = 1; c < mtchain; c++) eta_mass[c] = boltz * t_target / (t_freq * t_freq);
    }
    eta_dotdot[0] = eta_mass[0] > 0.0 ? (ke_now - ke_target) / eta_mass[0] : 0.0;
    for (int loop = 0; loop < nc_tchain; loop++) {
        for (int c = mtchain - 1; c > 0; c--) {
            const T ex = exp(-nc * eighth * eta_dot[c + 1]);
            eta_dot[c] = (eta_dot[c] * ex + eta_dotdot[c] * nc * quarter) * drag_f * ex;
        }
        T ex = exp(-nc * eighth * eta_dot[1]);
        eta_dot[0] = (eta_dot[0] * ex + eta_dotdot[0] * nc * quarter) * drag_f * ex;
        const T scale = exp(-nc * half * eta_dot[0]);
        k_md_vscale<<<blocks_for(inum), TB>>>(v, scale, ilist, dim, inum);
        count_launches(1);
        tarray[4] *= scale * scale;
        ke_now = tdof * boltz * tarray[4];
        eta_dotdot[0] = eta_mass[0] > 0.0 ? (ke_now - ke_target) / eta_mass[0] : 0.0;
        for (int c = 0; c < mtchain; c++) eta[c] += nc * half * eta_dot[c];
        eta_dot[0] = (eta_dot[0] * ex + eta_dotdot[0] * nc * quarter) * ex;
        for (int c = 1; c < mtchain; c++) {
            ex = exp(-nc * eighth * eta_dot[c + 1]);
            eta_dotdot[c] = (eta_mass[c - 1] * eta_dot[c - 1] * eta_dot[c - 1] - boltz * t_target) / eta_mass[c];
            eta_dot[c] = (eta_dot[c] * ex + eta_dotdot[c] * nc * quarter) * ex;
        }
    }
}

template <typename T>
void verlet(const char *fn, int stage, T *x, T *v, const T *f, const T *mass,
                   const T *dtarray, T *tarray, T *eta_mass, T *eta, T *eta_dot,
                   T *eta_dotdot, T *ke, T *tmp, T vlimitsq, const int *type, const int *ilist,
                   int eta_mass_flag, int mtchain, int nc_tchain, int mode, int dim, int inum)
{
    if (mode < 0 || mode > 2) {
        set_error("%s: mode %d is not supported; modes 0 (NVE), 1 (NVE limit) and 2 (NVT) are", fn, mode);
        return;
    }
    if (dim != 2 && dim != 3) { set_error("%s: dim must be 2 or 3", fn); return; }
    if (inum <= 0) return;
    if (mode == 2 && (!tarray || !eta_mass || !eta || !eta_dot || !eta_dotdot || !ke || !tmp || mtchain < 1 ||
                      nc_tchain < 1)) {
        set_error("%s: NVT needs tarray, the eta arrays (mtchain + 1 entries), ke and tmp", fn);
        return;
    }
    auto thermostat = [&]() -> int {
        const T tfactor = tarray[8] / (tarray[5] * tarray[6]);   // mvv2e / (tdof boltz)
        T t = 0.0;
        if (temperature(t, ke, tmp, mass, v, tfactor, type, ilist, dim, inum)) return -1;
        tarray[4] = t;
        nose_hoover(v, ilist, dim, inum, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, eta_mass_flag, mtchain,
                    nc_tchain);
        return 0;
    };
    if (mode == 2 && stage == 0) {
        // target temperature ramped over the run (cpuVelocityIntegration.cpp:602-628)
        const T delta = (dtarray[5] - dtarray[3]) / (dtarray[4] - dtarray[3]);
        tarray[3] = tarray[0] + delta * (tarray[1] - tarray[0]);
        if (thermostat()) return;
    }
    k_md_verlet<<<blocks_for(inum), TB>>>(x, v, f, mass, type, ilist, dtarray[1], dtarray[2], vlimitsq, mode == 1,
                                           stage, dim, inum);
    count_launches(1);
    if (mode == 2 && stage == 1 && thermostat()) return;
    check_launch(fn);
}

template <typename T>
void initial_integrate_t(T *x, T *v, const T *f, const T *mass, const T *dtarray,
                                   T *tarray, T *eta_mass, T *eta, T *eta_dot,
                                   T *eta_dotdot, T *ke, T *tmp, T vlimitsq, const int *type,
                                   const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                   int mode, int dim, int inum)
{
    (void)biasflag;
    verlet<T>("gpuInitialIntegrate", 0, x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp,
           vlimitsq, type, ilist, eta_mass_flag, mtchain, nc_tchain, mode, dim, inum);
}

template <typename T>
void final_integrate_t(T *x, T *v, const T *f, const T *mass, const T *dtarray,
                                 T *tarray, T *eta_mass, T *eta, T *eta_dot,
                                 T *eta_dotdot, T *ke, T *tmp, T vlimitsq, const int *type,
                                 const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                 int mode, int dim, int inum)
{
    (void)biasflag;
    verlet<T>("gpuFinalIntegrate", 1, x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp,
           vlimitsq, type, ilist, eta_mass_flag, mtchain, nc_tchain, mode, dim, inum);
}

template <typename T>
void pbc_t(T *x, T *v, int *image, const T *boxhi, const T *boxlo,
                     const T *hi_lambda, const T *lo_lambda, const T *h, const T *h_inv,
                     const T *h_rate, const int *pbc, int vdeform, int triclinic, int dim, int nlocal)
{
    if (dim != 2 && dim != 3) { set_error("gpuPBC: dim must be 2 or 3"); return; }
    if (nlocal <= 0) return;
    k_md_pbc<<<blocks_for(nlocal), TB>>>(x, v, image, boxhi, boxlo, hi_lambda, lo_lambda, h, h_inv, h_rate, pbc,
                                          vdeform, triclinic, dim, nlocal);
    count_launches(1);
    check_launch("gpuPBC");
}

template <typename T>
void compute_ke_atom_t(T *ke, const T *mass, const T *v, T mvv2e, const int *type,
                                 const int *ilist, int dim, int inum)
{
    if (dim != 2 && dim != 3) { set_error("gpuComputeKEAtom: dim must be 2 or 3"); return; }
    if (inum <= 0) return;
    k_md_ke<<<blocks_for(inum), TB>>>(ke, mass, v, mvv2e, type, ilist, dim, inum);
    count_launches(1);
    check_launch("gpuComputeKEAtom");
}

template <typename T>
void array_sum_every_column_t(T *b, const T *a, int m, int n)
{
    if (m <= 0) return;
    if (n <= 0) {
        cudaMemset(b, 0, sizeof(T) * m);
        return;
    }
    k_md_colsum<<<(unsigned)m, TB>>>(b, a, n);
    count_launches(1);
    check_launch("gpuArraySumEveryColumn");
}

}  // namespace

extern "C" {
// mdpgpucore.h:108 / gpuCumsum.cu -- out[0] = 0, out[j] = in[0] + ... + in[j-1]
// for j < length; d_sums is the scratch (length / 4096 + 1 ints are used)
void mdp_gpu_cumsum(int *d_out, int *d_in, int *d_sums, int *d_incr, int length)
{
    (void)d_incr;
    if (length <= 0) return;
    if (exclusive_scan(d_in, d_out, (long)length - 1, d_sums, 0)) return;
    check_launch("gpuCumsum");
}

// mdpgpucore.h:132-133 -- ghost images inside the bounding box, appended to x
// after the inum local atoms, owners in alist; glistnumsum gets inum + 1 entries
// mdpgpucore.h:136-137 -- the cell of every atom (locals among the interior cells)
// mdpgpucore.h:138 -- atoms grouped by cell (ascending within a cell), cell
// starts in c2anumsum[0..ncell], sorted cell ids in c2anum
void mdp_gpu_cell2atom_list(int *c2alist, int *c2anumsum, int *c2anum, const int *clist, int *d_temp, int natom,
                            int ncell)
{
    (void)d_temp;
    std::lock_guard<std::mutex> lk(g_md_mu);
    if (natom <= 0 || ncell <= 0) return;
    CellScratch &s = cell_scratch();
    if (s.cnt.ensure(sizeof(int) * ncell) || s.cursor.ensure(sizeof(int) * ncell) ||
        s.tmp.ensure(sizeof(int) * scan_tmp_ints(ncell)))
        return;
    if (cudaMemset(s.cnt.p, 0, sizeof(int) * ncell) != cudaSuccess ||
        cudaMemset(s.cursor.p, 0, sizeof(int) * ncell) != cudaSuccess) {
        set_error("gpuCell2AtomList: memset failed");
        return;
    }
    k_md_cell_count<<<blocks_for(natom), TB>>>(clist, natom, ncell, s.cnt.as<int>());
    if (exclusive_scan(s.cnt.as<int>(), c2anumsum, ncell, s.tmp.as<int>(), 0)) return;
    k_md_cell_fill<<<blocks_for(natom), TB>>>(clist, natom, ncell, c2anumsum, s.cursor.as<int>(), c2alist);
    k_md_cell_order<<<blocks_for(ncell), TB>>>(ncell, c2anumsum, c2alist, c2anum);
    count_launches(6);
    check_launch("gpuCell2AtomList");
}

// mdpgpucore.h:145-146 -- full neighbour rows from the cell lists
// mdpgpucore.h:141-142 -- full neighbour rows by an O(N^2) search
// temperature tfactor * sum m v^2 over the listed atoms (cpuComputes.cpp:276-296):
// per-atom terms into ke, a fixed-tree sum into tmp[0] (both the caller's
// device scratch, as gpuComputeTempScalar uses them), read on the host
// Nose-Hoover chain half step (cpuVelocityIntegration.cpp:505-600): the chain
// lives on the host (eta arrays of mtchain + 1 entries, tarray[4] the current
// temperature on entry); each sub-step scales the listed atoms' velocities.
// mdpgpucore.h:309-311 -- first half of velocity Verlet.  dtarray (dt, dtf, dtv,
// begin, end, current step), tarray (t_start, t_stop, t_freq, t_target,
// t_current, tdof, boltz, drag, mvv2e) and the eta arrays live on the host, as
// the reference reads them there; ke and tmp are device scratch of inum and 1
// doubles, used by mode 2 (NVT, Nose-Hoover chain)
// mdpgpucore.h:313-315 -- second half of velocity Verlet
// mdpgpucore.h:321-322 -- wrap local atoms into the box, counting images
// mdpgpucore.h:259-260 -- ke[ii] = 1/2 mvv2e m v^2
// mdpgpucore.h:56 -- b[j] = sum over the n rows of column j of a [m columns][n]
// mdpgpucore.h:49 -- y[n] read back to the host
int mdp_gpu_array_get_value_at_index_int(const int *y, int n)
{
    int v = 0;
    if (cudaMemcpy(&v, y + n, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        set_error("gpuArrayGetValueAtIndex: copy failed");
    return v;
}


void mdp_gpu_atom_list3d_f64(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums, int *d_incr,
                             double *x, const double *pimages, const double *wc, const double *s2rmap, int inum,
                             int pnum, int dim)
{
    atom_list3d_t(alist, inside, glistnumsum, glistnum, d_sums, d_incr, x, pimages, wc, s2rmap, inum, pnum, dim);
}

void mdp_gpu_atom_list3d_f32(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums, int *d_incr,
                             float *x, const float *pimages, const float *wc, const float *s2rmap, int inum,
                             int pnum, int dim)
{
    atom_list3d_t(alist, inside, glistnumsum, glistnum, d_sums, d_incr, x, pimages, wc, s2rmap, inum, pnum, dim);
}

void mdp_gpu_cell_list3d_f64(int *clist, const double *xi, const double *eta1, const double *eta2,
                             const double *eta3, const double *s2rmap, const int *nc, int inum, int natom, int dim)
{
    cell_list3d_t(clist, xi, eta1, eta2, eta3, s2rmap, nc, inum, natom, dim);
}

void mdp_gpu_cell_list3d_f32(int *clist, const float *xi, const float *eta1, const float *eta2,
                             const float *eta3, const float *s2rmap, const int *nc, int inum, int natom, int dim)
{
    cell_list3d_t(clist, xi, eta1, eta2, eta3, s2rmap, nc, inum, natom, dim);
}

void mdp_gpu_full_neighbor_list3d_cells_f64(int *neighborlist, int *neighbornum, const double *x,
                                            const double *rcutsq, const int *alist, const int *clist,
                                            const int *c2alist, const int *c2anumsum, const int *nc, int inum,
                                            int jnum, int dim)
{
    full_neighbor_list3d_cells_t(neighborlist, neighbornum, x, rcutsq, alist, clist, c2alist, c2anumsum, nc, inum, jnum, dim);
}

void mdp_gpu_full_neighbor_list3d_cells_f32(int *neighborlist, int *neighbornum, const float *x,
                                            const float *rcutsq, const int *alist, const int *clist,
                                            const int *c2alist, const int *c2anumsum, const int *nc, int inum,
                                            int jnum, int dim)
{
    full_neighbor_list3d_cells_t(neighborlist, neighbornum, x, rcutsq, alist, clist, c2alist, c2anumsum, nc, inum, jnum, dim);
}

void mdp_gpu_full_neighbor_list3d_f64(int *neighborlist, int *neighbornum, const double *x, const double *rcutsq,
                                      int anum, int inum, int jnum, int dim)
{
    full_neighbor_list3d_t(neighborlist, neighbornum, x, rcutsq, anum, inum, jnum, dim);
}

void mdp_gpu_full_neighbor_list3d_f32(int *neighborlist, int *neighbornum, const float *x, const float *rcutsq,
                                      int anum, int inum, int jnum, int dim)
{
    full_neighbor_list3d_t(neighborlist, neighbornum, x, rcutsq, anum, inum, jnum, dim);
}

void mdp_gpu_initial_integrate_f64(double *x, double *v, const double *f, const double *mass, const double *dtarray,
                                   double *tarray, double *eta_mass, double *eta, double *eta_dot,
                                   double *eta_dotdot, double *ke, double *tmp, double vlimitsq, const int *type,
                                   const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                   int mode, int dim, int inum)
{
    initial_integrate_t(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp, vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}

void mdp_gpu_initial_integrate_f32(float *x, float *v, const float *f, const float *mass, const float *dtarray,
                                   float *tarray, float *eta_mass, float *eta, float *eta_dot,
                                   float *eta_dotdot, float *ke, float *tmp, float vlimitsq, const int *type,
                                   const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                   int mode, int dim, int inum)
{
    initial_integrate_t(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp, vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}

void mdp_gpu_final_integrate_f64(double *x, double *v, const double *f, const double *mass, const double *dtarray,
                                 double *tarray, double *eta_mass, double *eta, double *eta_dot,
                                 double *eta_dotdot, double *ke, double *tmp, double vlimitsq, const int *type,
                                 const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                 int mode, int dim, int inum)
{
    final_integrate_t(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp, vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}

void mdp_gpu_final_integrate_f32(float *x, float *v, const float *f, const float *mass, const float *dtarray,
                                 float *tarray, float *eta_mass, float *eta, float *eta_dot,
                                 float *eta_dotdot, float *ke, float *tmp, float vlimitsq, const int *type,
                                 const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                 int mode, int dim, int inum)
{
    final_integrate_t(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp, vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}

void mdp_gpu_pbc_f64(double *x, double *v, int *image, const double *boxhi, const double *boxlo,
                     const double *hi_lambda, const double *lo_lambda, const double *h, const double *h_inv,
                     const double *h_rate, const int *pbc, int vdeform, int triclinic, int dim, int nlocal)
{
    pbc_t(x, v, image, boxhi, boxlo, hi_lambda, lo_lambda, h, h_inv, h_rate, pbc, vdeform, triclinic, dim, nlocal);
}

void mdp_gpu_pbc_f32(float *x, float *v, int *image, const float *boxhi, const float *boxlo,
                     const float *hi_lambda, const float *lo_lambda, const float *h, const float *h_inv,
                     const float *h_rate, const int *pbc, int vdeform, int triclinic, int dim, int nlocal)
{
    pbc_t(x, v, image, boxhi, boxlo, hi_lambda, lo_lambda, h, h_inv, h_rate, pbc, vdeform, triclinic, dim, nlocal);
}

void mdp_gpu_compute_ke_atom_f64(double *ke, const double *mass, const double *v, double mvv2e, const int *type,
                                 const int *ilist, int dim, int inum)
{
    compute_ke_atom_t(ke, mass, v, mvv2e, type, ilist, dim, inum);
}

void mdp_gpu_compute_ke_atom_f32(float *ke, const float *mass, const float *v, float mvv2e, const int *type,
                                 const int *ilist, int dim, int inum)
{
    compute_ke_atom_t(ke, mass, v, mvv2e, type, ilist, dim, inum);
}

void mdp_gpu_array_sum_every_column_f64(double *b, const double *a, int m, int n)
{
    array_sum_every_column_t(b, a, m, n);
}

void mdp_gpu_array_sum_every_column_f32(float *b, const float *a, int m, int n)
{
    array_sum_every_column_t(b, a, m, n);
}

}  // extern "C"
