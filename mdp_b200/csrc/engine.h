// Host-side structures of the B200 SNAP engine (internal; the public C ABI is
// include/mdp_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <vector>

#include "../../include/mdp_b200.h"
#include "snap_kernels.cuh"

namespace mdp {

struct BoxParams {
    double s2r[9];        // inverse of [a b c] (column-major)
    double lo[3], hi[3];  // enlarged bounding box in fractional coordinates
    double pim[27][3];    // periodic image shifts, reference order
    int nc[3];            // cell grid (fractional)
    double cinv[3];       // nc / (hi - lo)
    long ncell;
};
int box_setup(BoxParams &bp, const double *a, const double *b, const double *c, double offset, double rc_cells);

// kernels defined in neighbor.cu
__global__ void k_ghost_count(const double4 *, int, const __grid_constant__ BoxParams, int *, unsigned *);
__global__ void k_ghost_emit(double4 *, int *, int, const __grid_constant__ BoxParams, const int *, const unsigned *);
__global__ void k_cell_index(const double4 *, int, const __grid_constant__ BoxParams, int *, int *);
__global__ void k_cell_fill(int, const int *, const int *, int *, int *);
__global__ void k_neigh_build(const double4 *, int, const __grid_constant__ BoxParams, const int *, const int *,
                              const int *, double, int, int *, int *, int *);
__global__ void k_rev_count(const int *, const int *, const int *, int, int, int *);
__global__ void k_rev_fill(const int *, const int *, const int *, int, int, const int *, int *, long long *);
__global__ void k_rev_sort(int, const int *, long long *);
__global__ void k_pair_count(const double4 *, const int *, const int *, int, int, double, int *);
__global__ void k_pair_emit(const double4 *, const int *, const int *, int, int, const int *, SnapGeom, double4 *,
                            int2 *, double4 *, int *);
__global__ void k_tally(const double4 *, const double4 *, const int *, const int *, int, const int *,
                        const long long *, double4 *, double *, int nblk, int ipad);

// Several element types: type-pair cutoffs (radelem_i + radelem_j) rcutfac,
// their squares and the neighbour weights wjelem_j (InitSnap,
// snappotential.cpp:186-198); nblk U / Y element blocks (nelements with
// chemflag, else 1) of ipad virtual atoms each
constexpr int MAXELEM = 4;
struct ElemGeom {
    int ne, nblk, chem, ipad;
    double rcut[MAXELEM][MAXELEM], rcutsq[MAXELEM][MAXELEM], wj[MAXELEM];
};
__global__ void k_pair_count_me(const double4 *, const int *, const int *, int, int, const int *, const int *,
                                const __grid_constant__ ElemGeom, int *);
__global__ void k_pair_emit_me(const double4 *, const int *, const int *, int, int, const int *, const int *,
                               const int *, SnapGeom, const __grid_constant__ ElemGeom, double4 *, int2 *,
                               double4 *, double2 *, int *);
__global__ void k_nve_initial(double4 *, double4 *, const double4 *, double4 *, int, double, double);
__global__ void k_nve_final(double4 *, const double4 *, int, double);
__global__ void k_maxdisp(const double4 *, const double4 *, int, unsigned long long *);
__global__ void k_pbc_orth(double4 *, int, double, double, double, double, double, double);
__global__ void k_ghost_shift(double4 *, const double4 *, const int *, int, int);
__global__ void k_thermo(const double *, const double *, const double4 *, int, double *);

// SNAP model: validated parameters plus the derived kernel parameter blocks
// ZBL pair potential added to SNAP (the snapTA06A example's Paira term,
// simulating/snap/ZBLpotential.jl): screening exponents d_k / a, prefactors
// c_k Z^2 qqr2e, inner switch radius, outer cutoff^2 and the switch
// polynomial's coefficients
struct ZblParams {
    int on = 0;
    double dk[4], ck[4], inner, rcsq, sw3, sw4, sw5;
};
int zbl_setup(ZblParams &zp, double inner, double outer, double z);

// ZBL pair energy u(r) and g = u'(r) / r of the switched potential
// (ZBLpotential.jl): screened Coulomb plus A(t) t^3 (sw3 + sw4 t) + sw5 with
// t = r - inner and A = 1/2 + tanh(100 t)/2
__device__ __forceinline__ void zbl_pair(const ZblParams &zp, double r, double &u, double &g)
{
    const double rinv = 1.0 / r;
    double s = 0.0, sp = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double ek = zp.ck[k] * exp(-zp.dk[k] * r);
        s += ek;
        sp -= zp.dk[k] * ek;
    }
    const double ez = s * rinv, ezp = (sp - s * rinv) * rinv;
    const double t = r - zp.inner, t2 = t * t, t3 = t2 * t;
    const double th = tanh(100.0 * t), a = 0.5 + 0.5 * th, da = 50.0 * (1.0 - th * th);
    const double poly = zp.sw3 + zp.sw4 * t;
    u = ez + zp.sw5 + a * t3 * poly;
    g = (ezp + da * t3 * poly + a * (3.0 * t2 * poly + t3 * zp.sw4)) * rinv;
}
__global__ void k_zbl(const double4 *, const int *, const int *, int, int, ZblParams, double *, double4 *, double *);

// Quadratic SNAP (quadraticflag): E_i = beta0 + beta . B_i + B_i^T Q B_i / 2 with
// the coefficient layout of cpuSnap.cpp:1713-1770 (ncoeff linear, then the
// upper triangle of Q row by row, its diagonal entries taken once)
constexpr int QUAD_MAXK = 55;   // ncoeff at 2J = 8
struct QuadParams {
    double beta0;
    double beta[QUAD_MAXK];
    double q[QUAD_MAXK * (QUAD_MAXK + 1) / 2];
    int ncoeff;
};

struct SnapModel {
    mdp_snap_params p;
    std::vector<double> coeff;
    SnapGeom geom;
    YParams<double> yd;
    YParams<float> yf;
    YParams<double> yq;   // quadratic: unit coefficients (multiplicities only), per-atom coefficients from B
    QuadParams quad;
    int nu, nyh, ncoeff;
    ZblParams zbl;
    // several element types (nelements > 1): per-element coefficient table
    // coeffelem [ne][ncoeffall], type-pair geometry, the Y kernel's multiplicity
    // factors in yq
    int ne = 1;
    ElemGeom eg;
};
int model_init(SnapModel &m, const mdp_snap_params *p);

// device buffers of one force evaluation (capacities grow on demand)
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n);
    void release();
    template <typename X> X *as() const { return reinterpret_cast<X *>(p); }
};

struct ForcePath {
    DevBuf pcount, poff, prij, pinfo, pab, smap, dE, Ut, Y, scan_tmp;
    DevBuf B, G;   // quadratic SNAP: per-atom bispectrum and coefficients [k][atom]
    DevBuf pcw, elem, ecoef;   // several elements: per-pair cutoff / weight, atom elements, coeffelem
    const int *u_welem = nullptr;     // U stage: element of each atom, for wself per element block
    int u_ipad = 0;
    const double2 *fr_pcw = nullptr;  // dE/dr stage: per-pair cutoff / weight
    int natoms_cap = 0, nm_cap = 0;
    // per-stage timing (CUDA events on the launching stream), enabled on demand
    bool timing = false;
    cudaEvent_t ev[8] = {};
    double stage_ms[6] = {0, 0, 0, 0, 0, 0};   // pairs, ui, yi, fi, tally, total
    long stage_calls = 0;
    void release();
};

// per-stage launchers, one translation unit per (stage, precision)
template <typename T, int TJ> int launch_ui(const SnapModel &m, ForcePath &fp, int inum, cudaStream_t s);
template <typename T, int TJ>
int launch_yi(const SnapModel &m, const YParams<T> &yp, ForcePath &fp, int inum, double *eatom, cudaStream_t s);
template <typename T, int TJ> int launch_fi(const SnapModel &m, ForcePath &fp, int inum, int nm, cudaStream_t s);

// One plain-SNAP force evaluation on device data: x (anum, double4, ghosts
// appended), neighbour list (inum x nm), reverse list.  Writes eatom[inum],
// f[inum] (double4) and, when vatom != nullptr, the SoA per-atom virial 6 x inum.
// Several element types need atype (types 1..nelements of the inum owners)
// and alist (owner of every atom, ghosts included).
int force_compute(ForcePath &fp, const SnapModel &m, int precision, const double4 *x, int inum,
                  const int *nlist, const int *nnum, int nm, long pair_cap, const int *roff,
                  const long long *rlist, double *eatom, double4 *f, double *vatom, cudaStream_t s,
                  const int *atype = nullptr, const int *alist = nullptr);

// Neighbour structure (ghosts + list + reverse list) owned by a caller
struct Neighbors {
    DevBuf gcount, goff, gmask, alist, cidx, ccount, cstart, cursor, catoms, nlist, nnum, rcount, roff, rlist,
        status, scan_tmp;
    int inum = 0, gnum = 0, anum = 0, nm = 0;
    long nsum = 0;   // total neighbour entries
    long anum_cap = 0;
    void release();
};
// builds ghosts into x[inum..] (x must hold anum_cap entries), the list and its
// reverse.  Returns 0, or -1 on error (capacity, CUDA); overflow of neighmax is
// an error (the reference truncates silently).
int neighbor_build(Neighbors &nb, const BoxParams &bp, double4 *x, int inum, double rc, int nm, long anum_cap,
                   cudaStream_t s);

}  // namespace mdp
