// Test driver for the mdpcore.h boundary (MDP's C++ backend dispatch).
//
// This translation unit is compiled against the reference's own headers:
//   * src/C++/Common/mdpgpucore.h  -- the gpu* prototypes cpuMDP/gpuMDP link
//     against (included before this library's header, so any signature
//     mismatch with the templates there is a compile error);
//   * include/mdp_b200_gpucore.h with MDP_B200_GPUCORE_TEMPLATES -- this
//     library's definitions of those gpu* entry points;
//   * src/C++/Common/mdpcore.h -- the reference's inline wrappers that switch
//     on `backend` (here 2) and call the gpu* functions;
//   * src/C++/Core/cpuCore.cpp -- the CPU templates the wrappers' backend-1
//     branches name (needed to link; not called).
// Built twice: as MDP builds by default (dstype = double) and with PREC_FLOAT
// (dstype = float), the reference's single-precision build, whose gpu*
// templates are the float instantiations.
// `gpucore_pair_snap3` then runs the stage sequence of ComputePairSnap3
// (src/C++/Descriptors/snappotential.cpp:634-760) through those wrappers on
// device arrays, block by block, and returns eatom, fatom and the SoA virial
// vatom[6][inum] to the caller.  Generic array helpers that the reference takes
// from its gpuArrayOperations.cu (ArrayFill, ArraySetValue) are done here with
// plain CUDA runtime calls.  Built by tests/cpp/Makefile; test infrastructure.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <math.h>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <cublas_v2.h>

// the reference's main.cpp brings these names in before its headers
using std::cout;
using std::endl;
using std::string;
using std::ios;
using std::ofstream;
using std::ifstream;
using std::ostringstream;
using std::min;
using std::max;
using std::scientific;
#define USE_CUDA
#include "mdpcommon.h"     // dstype, Int and the reference's structs
#include "mdpgpucore.h"
#define MDP_B200_GPUCORE_TEMPLATES
#include "mdp_b200_gpucore.h"
#include "mdpcore.h"
#include "cpuCore.cpp"

extern "C" const char *mdp_last_error(void);

namespace {

struct Dev {
    void *p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
    template <class T> T *as() { return static_cast<T *>(p); }
};

int up(Dev &d, const void *h, size_t bytes)
{
    if (cudaMalloc(&d.p, bytes ? bytes : 16) != cudaSuccess) return -1;
    if (bytes && h && cudaMemcpy(d.p, h, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (!h && cudaMemset(d.p, 0, bytes ? bytes : 16) != cudaSuccess) return -1;
    return 0;
}

int fail(char *msg, const char *what)
{
    snprintf(msg, 512, "%s (cuda: %s; library: %s)", what, cudaGetErrorString(cudaGetLastError()), mdp_last_error());
    return -1;
}

}  // namespace

static int pair_snap3(
    // outputs (host): eatom[inum], fatom[3 inum], vatom[6 inum]
    dstype *eatom_h, dstype *fatom_h, dstype *vatom_h,
    // configuration (host, the reference layouts)
    const dstype *x_h, const int *atomtype_h, const int *alist_h, const int *neighlist_h, const int *neighnum_h,
    int inum, int anum, int neighmax, const dstype *rcutsq_h, int ntypes,
    // SNAP tables and parameters (host)
    const dstype *rootpq_h, int nrootpq, const dstype *cglist_h, int idxcg_max, const int *idxz_h, int idxz_max,
    const int *idxz_block_h, const int *idxb_h, int idxb_max, const int *idxb_block_h, const int *idxu_block_h,
    int idxu_max, const int *idxcg_block_h, int nblock3, const dstype *bzero_h, const dstype *coeffelem_h,
    int ncoeffall, const int *map_h, const dstype *radelem_h, const dstype *wjelem_h, dstype rmin0, dstype rfac0,
    dstype rcutfac, dstype wself, int twojmax, int switchflag, int bzeroflag, int bnormflag, int wselfallflag,
    int nblocks, int chemflag, char *msg)
{
    // InitSnap (snappotential.cpp:186-221): ntypes = nelements; U / Y element
    // blocks only with chemflag; coeffelem holds nelements x ncoeffall values
    const int dim = 3, backend = 2, quadraticflag = 0, nelements = ntypes;
    const int nelem = chemflag ? nelements : 1;
    const int jd = twojmax + 1;
    Dev x, atomtype, alist, neighlist, neighnum, rcutsq, rootpq, cglist, idxz, idxz_block, idxb, idxb_block,
        idxu_block, idxcg_block, bzero, coeffelem, map, radelem, wjelem, eatom, fatom, vatom;
    if (up(x, x_h, sizeof(dstype) * 3 * anum) || up(atomtype, atomtype_h, sizeof(int) * anum) ||
        up(alist, alist_h, sizeof(int) * anum) || up(neighlist, neighlist_h, sizeof(int) * (size_t)inum * neighmax) ||
        up(neighnum, neighnum_h, sizeof(int) * inum) ||
        up(rcutsq, rcutsq_h, sizeof(dstype) * (ntypes + 1) * (ntypes + 1)) ||
        up(rootpq, rootpq_h, sizeof(dstype) * nrootpq) || up(cglist, cglist_h, sizeof(dstype) * idxcg_max) ||
        up(idxz, idxz_h, sizeof(int) * 10 * idxz_max) || up(idxz_block, idxz_block_h, sizeof(int) * nblock3) ||
        up(idxb, idxb_h, sizeof(int) * 3 * idxb_max) || up(idxb_block, idxb_block_h, sizeof(int) * nblock3) ||
        up(idxu_block, idxu_block_h, sizeof(int) * jd) || up(idxcg_block, idxcg_block_h, sizeof(int) * nblock3) ||
        up(bzero, bzero_h, sizeof(dstype) * jd) || up(coeffelem, coeffelem_h, sizeof(dstype) * ncoeffall * nelements) ||
        up(map, map_h, sizeof(int) * (ntypes + 1)) || up(radelem, radelem_h, sizeof(dstype) * (ntypes + 1)) ||
        up(wjelem, wjelem_h, sizeof(dstype) * (ntypes + 1)) || up(eatom, nullptr, sizeof(dstype) * inum) ||
        up(fatom, nullptr, sizeof(dstype) * 3 * inum) || up(vatom, nullptr, sizeof(dstype) * 6 * inum))
        return fail(msg, "device set-up");

    // ComputePairSnap3's block loop (snappotential.cpp:687-758)
    for (int b = 0; b < nblocks; b++) {
        const int e1 = (int)((long)inum * b / nblocks), e2 = (int)((long)inum * (b + 1) / nblocks);
        const int na = e2 - e1;
        if (na == 0) continue;
        std::vector<int> il(na);
        for (int i = 0; i < na; i++) il[i] = e1 + i;
        Dev ilist, pairnum, pairlist, pairnumsum, sums, incr;
        if (up(ilist, il.data(), sizeof(int) * na) || up(pairnum, nullptr, sizeof(int) * na) ||
            up(pairlist, nullptr, sizeof(int) * (size_t)na * neighmax) ||
            up(pairnumsum, nullptr, sizeof(int) * (na + 1)) || up(sums, nullptr, sizeof(int) * (na + 1)) ||
            up(incr, nullptr, sizeof(int) * (na + 1)))
            return fail(msg, "block set-up");
        NeighborPairList(pairnum.as<int>(), pairlist.as<int>(), x.as<dstype>(), rcutsq.as<dstype>(),
                         ilist.as<int>(), neighlist.as<int>(), neighnum.as<int>(), atomtype.as<int>(),
                         alist.as<int>(), na, neighmax, dim, ntypes, backend);
        Cumsum(pairnumsum.as<int>(), pairnum.as<int>(), sums.as<int>(), incr.as<int>(), na + 1, backend);
        const int ineighmax = IntArrayGetValueAtIndex(pairnumsum.as<int>(), na, backend);
        if (ineighmax < 0 || ineighmax > na * neighmax) return fail(msg, "pair count out of range");
        Dev ai, aj, ti, tj, aii, rij, ur, ui, yr, yi;
        const size_t nu = (size_t)idxu_max * nelem * na;
        if (up(ai, nullptr, sizeof(int) * ineighmax) || up(aj, nullptr, sizeof(int) * ineighmax) ||
            up(ti, nullptr, sizeof(int) * ineighmax) || up(tj, nullptr, sizeof(int) * ineighmax) ||
            up(aii, nullptr, sizeof(int) * ineighmax) || up(rij, nullptr, sizeof(dstype) * dim * ineighmax) ||
            up(ur, nullptr, sizeof(dstype) * nu) || up(ui, nullptr, sizeof(dstype) * nu) ||
            up(yr, nullptr, sizeof(dstype) * nu) || up(yi, nullptr, sizeof(dstype) * nu))
            return fail(msg, "pair arrays");
        NeighborPairs(rij.as<dstype>(), x.as<dstype>(), aii.as<int>(), ai.as<int>(), aj.as<int>(), ti.as<int>(),
                      tj.as<int>(), pairnum.as<int>(), pairlist.as<int>(), pairnumsum.as<int>(), ilist.as<int>(),
                      atomtype.as<int>(), alist.as<int>(), na, neighmax, dim, backend);
        // ArraySetValue(ulisttot, 0.0, ...): zeroed by up()
        SnapComputeUi(ur.as<dstype>(), ui.as<dstype>(), rootpq.as<dstype>(), rij.as<dstype>(), wjelem.as<dstype>(),
                      radelem.as<dstype>(), rmin0, rfac0, rcutfac, idxu_block.as<int>(), map.as<int>(), aii.as<int>(),
                      ti.as<int>(), tj.as<int>(), twojmax, idxu_max, na, ineighmax, switchflag, chemflag, backend);
        AddWself2Ui(ur.as<dstype>(), ui.as<dstype>(), wself, idxu_block.as<int>(), atomtype.as<int>() + e1,
                    map.as<int>(), ai.as<int>(), wselfallflag, chemflag, idxu_max, nelem, twojmax, na, backend);
        SnapComputeEi(eatom.as<dstype>(), ur.as<dstype>(), ui.as<dstype>(), cglist.as<dstype>(), bzero.as<dstype>(),
                      coeffelem.as<dstype>(), ilist.as<int>(), map.as<int>(), atomtype.as<int>(), idxb.as<int>(),
                      idxcg_block.as<int>(), idxu_block.as<int>(), twojmax, idxb_max, idxu_max, nelem, ncoeffall,
                      bnormflag, bzeroflag, wselfallflag, quadraticflag, na, backend);
        SnapComputeYi(yr.as<dstype>(), yi.as<dstype>(), ur.as<dstype>(), ui.as<dstype>(), cglist.as<dstype>(),
                      coeffelem.as<dstype>(), map.as<int>(), atomtype.as<int>() + e1, idxz.as<int>(),
                      idxb_block.as<int>(), idxu_block.as<int>(), idxcg_block.as<int>(), twojmax, idxb_max, idxu_max,
                      idxz_max, nelem, ncoeffall, bnormflag, na, backend);
        SnapComputeFi(fatom.as<dstype>(), vatom.as<dstype>(), yr.as<dstype>(), yi.as<dstype>(), rootpq.as<dstype>(),
                      rij.as<dstype>(), wjelem.as<dstype>(), radelem.as<dstype>(), rmin0, rfac0, rcutfac,
                      idxu_block.as<int>(), map.as<int>(), aii.as<int>(), ai.as<int>(), aj.as<int>(), ti.as<int>(),
                      tj.as<int>(), twojmax, idxu_max, na, inum, ineighmax, switchflag, chemflag, backend);
        if (cudaDeviceSynchronize() != cudaSuccess) return fail(msg, "block sequence");
    }
    if (cudaMemcpy(eatom_h, eatom.p, sizeof(dstype) * inum, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(fatom_h, fatom.p, sizeof(dstype) * 3 * inum, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(vatom_h, vatom.p, sizeof(dstype) * 6 * inum, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(msg, "download");
    return 0;
}

// one element type (the reference's Ta examples)
extern "C" int gpucore_pair_snap3(dstype *eatom_h, dstype *fatom_h, dstype *vatom_h, const dstype *x_h,
                                  const int *atomtype_h, const int *alist_h, const int *neighlist_h,
                                  const int *neighnum_h, int inum, int anum, int neighmax, const dstype *rcutsq_h,
                                  int ntypes, const dstype *rootpq_h, int nrootpq, const dstype *cglist_h,
                                  int idxcg_max, const int *idxz_h, int idxz_max, const int *idxz_block_h,
                                  const int *idxb_h, int idxb_max, const int *idxb_block_h, const int *idxu_block_h,
                                  int idxu_max, const int *idxcg_block_h, int nblock3, const dstype *bzero_h,
                                  const dstype *coeffelem_h, int ncoeffall, const int *map_h, const dstype *radelem_h,
                                  const dstype *wjelem_h, dstype rmin0, dstype rfac0, dstype rcutfac, dstype wself,
                                  int twojmax, int switchflag, int bzeroflag, int bnormflag, int wselfallflag,
                                  int nblocks, char *msg)
{
    return pair_snap3(eatom_h, fatom_h, vatom_h, x_h, atomtype_h, alist_h, neighlist_h, neighnum_h, inum, anum,
                      neighmax, rcutsq_h, ntypes, rootpq_h, nrootpq, cglist_h, idxcg_max, idxz_h, idxz_max,
                      idxz_block_h, idxb_h, idxb_max, idxb_block_h, idxu_block_h, idxu_max, idxcg_block_h, nblock3,
                      bzero_h, coeffelem_h, ncoeffall, map_h, radelem_h, wjelem_h, rmin0, rfac0, rcutfac, wself,
                      twojmax, switchflag, bzeroflag, bnormflag, wselfallflag, nblocks, 0, msg);
}

// several element types: ntypes = nelements, types 1..nelements in atomtype,
// map[t] = t - 1, chemflag 0 or 1
extern "C" int gpucore_pair_snap3_elements(dstype *eatom_h, dstype *fatom_h, dstype *vatom_h, const dstype *x_h,
                                           const int *atomtype_h, const int *alist_h, const int *neighlist_h,
                                           const int *neighnum_h, int inum, int anum, int neighmax,
                                           const dstype *rcutsq_h, int ntypes, const dstype *rootpq_h, int nrootpq,
                                           const dstype *cglist_h, int idxcg_max, const int *idxz_h, int idxz_max,
                                           const int *idxz_block_h, const int *idxb_h, int idxb_max,
                                           const int *idxb_block_h, const int *idxu_block_h, int idxu_max,
                                           const int *idxcg_block_h, int nblock3, const dstype *bzero_h,
                                           const dstype *coeffelem_h, int ncoeffall, const int *map_h,
                                           const dstype *radelem_h, const dstype *wjelem_h, dstype rmin0,
                                           dstype rfac0, dstype rcutfac, dstype wself, int twojmax, int switchflag,
                                           int bzeroflag, int bnormflag, int wselfallflag, int nblocks, int chemflag,
                                           char *msg)
{
    return pair_snap3(eatom_h, fatom_h, vatom_h, x_h, atomtype_h, alist_h, neighlist_h, neighnum_h, inum, anum,
                      neighmax, rcutsq_h, ntypes, rootpq_h, nrootpq, cglist_h, idxcg_max, idxz_h, idxz_max,
                      idxz_block_h, idxb_h, idxb_max, idxb_block_h, idxu_block_h, idxu_max, idxcg_block_h, nblock3,
                      bzero_h, coeffelem_h, ncoeffall, map_h, radelem_h, wjelem_h, rmin0, rfac0, rcutfac, wself,
                      twojmax, switchflag, bzeroflag, bnormflag, wselfallflag, nblocks, chemflag, msg);
}
