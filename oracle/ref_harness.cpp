// Test infrastructure only: a thin extern "C" harness around MDP's own CPU
// templates, compiled from the reference sources where they lie (the include
// path points at src/C++/Core of the reference tree; nothing is copied).
// It exists so that tests, golden-fixture generation and the CPU baseline of
// bench.py can run the reference's algorithm on identical inputs.  It is never
// part of the product path.
//
// Orchestration follows, in order:
//   box set-up          src/C++/Configuration/Configuration.cpp:790-880
//   ghost atoms + list  src/C++/Configuration/Configuration.cpp:1000-1089
//   SNAP force path     src/C++/Descriptors/snappotential.cpp:634-760
//   NVE integrator      src/C++/Core/cpuVelocityIntegration.cpp:307-339
// The only deviation from the reference is 64-bit-safe sizing and optional
// host threads over independent atom blocks (the reference processes the same
// blocks one after another; per-block results are independent, forces are
// summed from per-thread buffers).
#include "cpuCore.cpp"
// MDP's generated code for the Ta ZBL pair potential of its snapTA06A example
// (src/C++/Potentials/cpuPairaGradient.cpp, from simulating/snap/ZBLpotential.jl)
#include "cpuPairaGradient.cpp"

#include <stdlib.h>
#include <string.h>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Box set-up: s2rmap (3x3, column-major inverse of [a b c]), rbvertices (24),
// pimages (81), pnum, cellnum/eta grids for the cell list (reference quirk:
// the z cell count is forced to 0, Configuration.cpp:847-848).
int ref_box_setup(const double *a_in, const double *b_in, const double *c_in,
                  const double *boxoffset_in, const int *pbc_in,
                  double *s2rmap, double *rbvertices, double *pimages,
                  int *cellnum, double *eta1, double *eta2, double *eta3)
{
    const int dim = 3;
    double simbox[9], a[3], b[3], c[3], boxoffset[3];
    int pbc[3];
    for (int i = 0; i < 3; i++) {
        simbox[i] = a_in[i]; simbox[3 + i] = b_in[i]; simbox[6 + i] = c_in[i];
        boxoffset[i] = boxoffset_in[i]; pbc[i] = pbc_in[i];
    }
    cpuSmallMatrixInverse(s2rmap, simbox, dim);
    for (int i = 0; i < 3; i++) { a[i] = simbox[i]; b[i] = simbox[3 + i]; c[i] = simbox[6 + i]; }
    double refvertices[24], boxvertices[24], bbvertices[24];
    cpuBoundingBox3D(refvertices, rbvertices, boxvertices, bbvertices, a, b, c, boxoffset, pbc);
    (void)refvertices; (void)boxvertices; (void)bbvertices;
    int pnum = cpuPeriodicImages3D(pimages, a, b, c, pbc);
    double *smin = &rbvertices[0];
    double *smax = &rbvertices[dim * 6];
    int ne[3]; double cellsize[3];
    for (int i = 0; i < dim; i++) {
        ne[i] = (int) round(1.0 / (smax[i] - 1.0));
        ne[i] = (ne[i] < 1) ? 1 : ne[i];
        cellnum[i] = ne[i] + 2;
        cellsize[i] = 1.0 / ((double) ne[i]);
    }
    cellnum[2] = 0;
    cpuMakeReferenceGrid(eta1, smin[0], smax[0], cellsize[0], cellnum[0]);
    cpuMakeReferenceGrid(eta2, smin[1], smax[1], cellsize[1], cellnum[1]);
    cpuMakeReferenceGrid(eta3, smin[2], smax[2], cellsize[2], cellnum[2]);
    return pnum;
}

// Ghost atoms + full neighbour list (neighcell = 1 path, or 0 for O(N^2)).
// x must have room for anummax*3 doubles; returns gnum (or -1 on overflow).
long ref_neighbor_list(double *x, int *alist, int *neighlist, int *neighnum,
                       const double *pimages, const double *rbvertices, const double *s2rmap,
                       const int *cellnum, const double *eta1, const double *eta2, const double *eta3,
                       double rcutsq_skin, int inum, int pnum, int neighmax, int neighcell,
                       long anummax)
{
    const int dim = 3;
    std::vector<int> inside((size_t)inum * pnum), glistnum(inum + 1), glistnumsum(inum + 1);
    // cpuAtomList3D, but with an explicit capacity check before writing ghosts.
    cpuGhostAtoms3D(glistnum.data(), inside.data(), x, (double *)pimages, (double *)rbvertices,
                    (double *)s2rmap, inum, pnum, dim);
    long gtot = 0;
    for (int i = 0; i < inum; i++) gtot += glistnum[i];
    if (inum + gtot > anummax) return -1;
    cpuAtomList3D(alist, inside.data(), glistnumsum.data(), glistnum.data(), x,
                  (double *)pimages, (double *)rbvertices, (double *)s2rmap, inum, pnum, dim);
    int gnum = glistnumsum[inum];
    int anum = inum + gnum;
    double rcs[1] = {rcutsq_skin};
    if (neighcell == 0) {
        cpuFullNeighborList3D(neighlist, neighnum, x, rcs, anum, inum, neighmax, dim);
    } else {
        int nc[3] = {cellnum[0], cellnum[1], cellnum[2]};
        int cnum = nc[0] * nc[1] * (nc[2] > 0 ? nc[2] : 1);
        // cell count used for sizing in the reference is the product before the z quirk
        std::vector<int> clist(anum), c2alist(anum), c2anum(anum), c2anumsum(anum + cnum + 2, 0);
        cpuCellList3D(clist.data(), x, (double *)eta1, (double *)eta2, (double *)eta3,
                      (double *)s2rmap, nc, inum, anum, dim);
        for (int i = 0; i < anum; i++) c2alist[i] = i;
        // Cell2AtomList: sort atoms by cell, then per-cell counts (cpuNeighborList2D.cpp:298-308)
        int ncell = 0;
        for (int i = 0; i < anum; i++) ncell = (clist[i] + 1 > ncell) ? clist[i] + 1 : ncell;
        std::vector<int> sums(ncell + 2, 0);
        cpuCell2AtomList(c2alist.data(), sums.data(), c2anum.data(), clist.data(), anum, ncell);
        // the stencil may address cells beyond ncell; pad their prefix sums
        int big = ncell + nc[0] * nc[1] * 3 + 8;
        std::vector<int> c2s(big + 1, sums[ncell]);
        for (int k = 0; k <= ncell; k++) c2s[k] = sums[k];
        cpuFullNeighborList3D(neighlist, neighnum, x, rcs, alist, clist.data(), c2alist.data(),
                              c2s.data(), nc, inum, neighmax, dim);
    }
    return gnum;
}

// Plain SNAP force path over atom blocks (ComputePairSnap3 semantics):
// eatom[inum], fatom[3*inum] (AoS), vatom[6*inum] (SoA, 6 x inum) are
// accumulated (callers zero them).  Single element, chemflag = 0.
void ref_snap_force(double *eatom, double *fatom, double *vatom, const double *x,
                    const int *atomtype, const int *alist, const int *neighlist, const int *neighnum,
                    int inum, int neighmax,
                    int twojmax, int ncoeffall, const double *coeffelem,
                    double rcutfac, double rfac0, double rmin0, double radelem1, double wjelem1,
                    int switchflag, int bzeroflag, int bnormflag, int wselfallflag,
                    int nblocks, int nthreads)
{
    const int dim = 3, ntypes = 1, nelem = 1, chemflag = 0, quadraticflag = 0;
    int jdim = twojmax + 1;
    // tables (snappotential.cpp:47-140 via cpuInitSna)
    int idx_max[5];
    int idxcg_count = 0, idxz_count = 0, idxb_count = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= MIN(twojmax, j1 + j2); j += 2) {
                idxcg_count += (j1 + 1) * (j2 + 1);
                if (j >= j1) idxb_count++;
                for (int mb = 0; 2 * mb <= j; mb++) idxz_count += j + 1;
            }
    std::vector<double> rootpq((jdim + 1) * (jdim + 1)), cglist(idxcg_count), fac(168);
    std::vector<int> idxz(idxz_count * 10), idxz_block(jdim * jdim * jdim), idxb(idxb_count * 3),
        idxb_block(jdim * jdim * jdim), idxu_block(jdim), idxcg_block(jdim * jdim * jdim);
    // factorial table (mdpcommon.h factable); every entry the CG formula reads
    // for 2J <= 10 is an exact integer in double, so a running product matches it.
    fac[0] = 1.0;
    for (int i = 1; i < 168; i++) fac[i] = fac[i - 1] * (double)i;
    cpuInitSna(rootpq.data(), cglist.data(), fac.data(), idx_max, idxz.data(), idxz_block.data(),
               idxb.data(), idxb_block.data(), idxu_block.data(), idxcg_block.data(), twojmax);
    int idxu_max = idx_max[1], idxb_max = idx_max[2], idxz_max = idx_max[3];
    double radelem[2] = {0.0, radelem1}, wjelem[2] = {0.0, wjelem1};
    int map[2] = {0, 0};
    double cut = (radelem1 + radelem1) * rcutfac;
    double rcutsq[4] = {0, 0, 0, cut * cut};
    double bzero[64];
    for (int j = 0; j <= twojmax; j++) bzero[j] = bnormflag ? 1.0 : (double)(j + 1);
    double wself = 1.0;

    if (nblocks < 1) nblocks = 1;
    if (nthreads < 1) nthreads = 1;
    std::vector<long> ablks(nblocks + 1);
    for (int b = 0; b <= nblocks; b++) ablks[b] = (long)inum * b / nblocks;
    std::vector<std::vector<double>> fbuf(nthreads), vbuf(nthreads);
    for (int t = 0; t < nthreads; t++) {
        fbuf[t].assign((size_t)3 * inum, 0.0);
        vbuf[t].assign((size_t)6 * inum, 0.0);
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int b = 0; b < nblocks; b++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int e1 = (int)ablks[b], e2 = (int)ablks[b + 1];
        int na = e2 - e1;
        if (na <= 0) continue;
        std::vector<int> pairnum(na), pairlist((size_t)na * neighmax), ilist(na), pairnumsum(na + 1);
        for (int i = 0; i < na; i++) ilist[i] = e1 + i;
        cpuNeighPairList(pairnum.data(), pairlist.data(), (double *)x, rcutsq, ilist.data(),
                         (int *)neighlist, (int *)neighnum, (int *)atomtype, (int *)alist, na,
                         neighmax, dim, ntypes);
        pairnumsum[0] = 0;
        for (int i = 0; i < na; i++) pairnumsum[i + 1] = pairnumsum[i] + pairnum[i];
        int ijnum = pairnumsum[na];
        std::vector<int> ai(ijnum), aj(ijnum), ti(ijnum), tj(ijnum), aii(ijnum);
        std::vector<double> rij((size_t)3 * ijnum);
        std::vector<double> ur((size_t)idxu_max * na, 0.0), ui((size_t)idxu_max * na, 0.0),
            yr((size_t)idxu_max * na), yi((size_t)idxu_max * na);
        cpuNeighPairs(rij.data(), (double *)x, aii.data(), ai.data(), aj.data(), ti.data(), tj.data(),
                      pairnum.data(), pairlist.data(), pairnumsum.data(), ilist.data(),
                      (int *)atomtype, (int *)alist, na, neighmax, dim);
        cpuSnapComputeUi(ur.data(), ui.data(), rootpq.data(), rij.data(), wjelem, radelem, rmin0,
                         rfac0, rcutfac, idxu_block.data(), map, aii.data(), ti.data(), tj.data(),
                         twojmax, idxu_max, na, ijnum, switchflag, chemflag);
        cpuAddWself2Ui(ur.data(), ui.data(), wself, idxu_block.data(), (int *)&atomtype[e1], map,
                       ai.data(), wselfallflag, chemflag, idxu_max, nelem, twojmax, na);
        cpuSnapComputeEi(eatom, ur.data(), ui.data(), cglist.data(), bzero, (double *)coeffelem,
                         ilist.data(), map, (int *)&atomtype[e1], idxb.data(), idxcg_block.data(),
                         idxu_block.data(), twojmax, idxb_max, idxu_max, nelem, ncoeffall, bnormflag,
                         bzeroflag, wselfallflag, quadraticflag, na);
        cpuSnapComputeYi(yr.data(), yi.data(), ur.data(), ui.data(), cglist.data(), (double *)coeffelem,
                         map, (int *)&atomtype[e1], idxz.data(), idxb_block.data(), idxu_block.data(),
                         idxcg_block.data(), twojmax, idxb_max, idxu_max, idxz_max, nelem, ncoeffall,
                         bnormflag, na);
        cpuSnapComputeFi(fbuf[tid].data(), vbuf[tid].data(), yr.data(), yi.data(), rootpq.data(),
                         rij.data(), wjelem, radelem, rmin0, rfac0, rcutfac, idxu_block.data(), map,
                         aii.data(), ai.data(), aj.data(), ti.data(), tj.data(), twojmax, idxu_max, na,
                         inum, ijnum, switchflag, chemflag);
    }
    for (int t = 0; t < nthreads; t++) {
        for (size_t k = 0; k < (size_t)3 * inum; k++) fatom[k] += fbuf[t][k];
        for (size_t k = 0; k < (size_t)6 * inum; k++) vatom[k] += vbuf[t][k];
    }
}

// Multi-element SNAP through ComputePairSnap3 (snappotential.cpp:634-760)
// with the parameter set-up of InitSnap (snappotential.cpp:146-232):
// atom types 1..nelements (atomtype over the owners; ghosts through alist),
// map[t] = t - 1, per-type radii and weights, cutoffs
// (radelem[i] + radelem[j]) * rcutfac per type pair, nelements * ncoeffall
// coefficients (ncoeffall = 1 + idxb_max * nelements^3 with chemflag, else
// 1 + idxb_max) and element blocks of U and Y when chemflag is set.  One atom
// block; eatom, fatom (AoS) and vatom (SoA 6 x inum) accumulate.
void ref_snap_force_me(double *eatom, double *fatom, double *vatom, const double *x, const int *atomtype,
                       const int *alist, const int *neighlist, const int *neighnum, int inum, int neighmax,
                       int twojmax, int nelements, int chemflag, int ncoeffall, const double *coeffelem,
                       double rcutfac, double rfac0, double rmin0, const double *radelems, const double *wjelems,
                       int switchflag, int bzeroflag, int bnormflag, int wselfallflag)
{
    const int dim = 3, ntypes = nelements, quadraticflag = 0;
    const int nelem = chemflag ? nelements : 1;
    int jdim = twojmax + 1;
    int idx_max[5];
    int idxcg_count = 0, idxz_count = 0, idxb_count = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= MIN(twojmax, j1 + j2); j += 2) {
                idxcg_count += (j1 + 1) * (j2 + 1);
                if (j >= j1) idxb_count++;
                for (int mb = 0; 2 * mb <= j; mb++) idxz_count += j + 1;
            }
    std::vector<double> rootpq((jdim + 1) * (jdim + 1)), cglist(idxcg_count), fac(168);
    std::vector<int> idxz(idxz_count * 10), idxz_block(jdim * jdim * jdim), idxb(idxb_count * 3),
        idxb_block(jdim * jdim * jdim), idxu_block(jdim), idxcg_block(jdim * jdim * jdim);
    fac[0] = 1.0;
    for (int i = 1; i < 168; i++) fac[i] = fac[i - 1] * (double)i;
    cpuInitSna(rootpq.data(), cglist.data(), fac.data(), idx_max, idxz.data(), idxz_block.data(),
               idxb.data(), idxb_block.data(), idxu_block.data(), idxcg_block.data(), twojmax);
    int idxu_max = idx_max[1], idxb_max = idx_max[2], idxz_max = idx_max[3];
    std::vector<double> radelem(nelements + 1, 0.0), wjelem(nelements + 1, 0.0);
    std::vector<int> map(nelements + 1, 0);
    for (int t = 0; t < nelements; t++) {
        radelem[t + 1] = radelems[t];
        wjelem[t + 1] = wjelems[t];
        map[t + 1] = t;
    }
    std::vector<double> rcutsq((nelements + 1) * (nelements + 1), 0.0);
    for (int i = 0; i < nelements; i++)
        for (int j = 0; j < nelements; j++) {
            double cut = (radelems[i] + radelems[j]) * rcutfac;
            rcutsq[j + 1 + (i + 1) * (nelements + 1)] = cut * cut;
        }
    double bzero[64];
    for (int j = 0; j <= twojmax; j++) bzero[j] = bnormflag ? 1.0 : (double)(j + 1);
    double wself = 1.0;
    const int na = inum;
    std::vector<int> pairnum(na), pairlist((size_t)na * neighmax), ilist(na), pairnumsum(na + 1);
    for (int i = 0; i < na; i++) ilist[i] = i;
    cpuNeighPairList(pairnum.data(), pairlist.data(), (double *)x, rcutsq.data(), ilist.data(), (int *)neighlist,
                     (int *)neighnum, (int *)atomtype, (int *)alist, na, neighmax, dim, ntypes);
    pairnumsum[0] = 0;
    for (int i = 0; i < na; i++) pairnumsum[i + 1] = pairnumsum[i] + pairnum[i];
    int ijnum = pairnumsum[na];
    std::vector<int> ai(ijnum), aj(ijnum), ti(ijnum), tj(ijnum), aii(ijnum);
    std::vector<double> rij((size_t)3 * ijnum);
    const size_t nub = (size_t)idxu_max * nelem * na;
    std::vector<double> ur(nub, 0.0), ui(nub, 0.0), yr(nub), yi(nub);
    cpuNeighPairs(rij.data(), (double *)x, aii.data(), ai.data(), aj.data(), ti.data(), tj.data(), pairnum.data(),
                  pairlist.data(), pairnumsum.data(), ilist.data(), (int *)atomtype, (int *)alist, na, neighmax, dim);
    cpuSnapComputeUi(ur.data(), ui.data(), rootpq.data(), rij.data(), wjelem.data(), radelem.data(), rmin0, rfac0,
                     rcutfac, idxu_block.data(), map.data(), aii.data(), ti.data(), tj.data(), twojmax, idxu_max, na,
                     ijnum, switchflag, chemflag);
    cpuAddWself2Ui(ur.data(), ui.data(), wself, idxu_block.data(), (int *)atomtype, map.data(), ai.data(),
                   wselfallflag, chemflag, idxu_max, nelem, twojmax, na);
    cpuSnapComputeEi(eatom, ur.data(), ui.data(), cglist.data(), bzero, (double *)coeffelem, ilist.data(),
                     map.data(), (int *)atomtype, idxb.data(), idxcg_block.data(), idxu_block.data(), twojmax,
                     idxb_max, idxu_max, nelem, ncoeffall, bnormflag, bzeroflag, wselfallflag, quadraticflag, na);
    cpuSnapComputeYi(yr.data(), yi.data(), ur.data(), ui.data(), cglist.data(), (double *)coeffelem, map.data(),
                     (int *)atomtype, idxz.data(), idxb_block.data(), idxu_block.data(), idxcg_block.data(),
                     twojmax, idxb_max, idxu_max, idxz_max, nelem, ncoeffall, bnormflag, na);
    cpuSnapComputeFi(fatom, vatom, yr.data(), yi.data(), rootpq.data(), rij.data(), wjelem.data(), radelem.data(),
                     rmin0, rfac0, rcutfac, idxu_block.data(), map.data(), aii.data(), ai.data(), aj.data(),
                     ti.data(), tj.data(), twojmax, idxu_max, na, inum, ijnum, switchflag, chemflag);
}

// SNAP forces through the reference's other pair chain, ComputePairSnap
// (snappotential.cpp:236-410): per-pair U and dU (cpuComputeUij,
// cpuComputeDuijdrj), U totals, Z and B (cpuComputeZi, cpuComputeBi), energy
// and per-atom coefficients with the quadratic terms (cpuSnapTallyEnergyFull,
// cpuComputeBeta2, cpuSnap.cpp:1713-1770), Y from those coefficients, dE/dr
// and the force / virial tallies.  This is the chain that carries
// quadraticflag (ComputePairSnap3 leaves it unused).  One atom block,
// single element; eatom, fatom (AoS) and vatom (SoA 6 x inum) accumulate.
void ref_snap_force_pairsnap(double *eatom, double *fatom, double *vatom, const double *x,
                             const int *atomtype, const int *alist, const int *neighlist, const int *neighnum,
                             int inum, int neighmax, int twojmax, int ncoeffall, const double *coeffelem,
                             double rcutfac, double rfac0, double rmin0, double radelem1, double wjelem1,
                             int switchflag, int bzeroflag, int bnormflag, int wselfallflag, int quadraticflag)
{
    const int dim = 3, ntypes = 1, nelem = 1, chemflag = 0;
    int jdim = twojmax + 1;
    int idx_max[5];
    int idxcg_count = 0, idxz_count = 0, idxb_count = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= MIN(twojmax, j1 + j2); j += 2) {
                idxcg_count += (j1 + 1) * (j2 + 1);
                if (j >= j1) idxb_count++;
                for (int mb = 0; 2 * mb <= j; mb++) idxz_count += j + 1;
            }
    std::vector<double> rootpq((jdim + 1) * (jdim + 1)), cglist(idxcg_count), fac(168);
    std::vector<int> idxz(idxz_count * 10), idxz_block(jdim * jdim * jdim), idxb(idxb_count * 3),
        idxb_block(jdim * jdim * jdim), idxu_block(jdim), idxcg_block(jdim * jdim * jdim);
    fac[0] = 1.0;
    for (int i = 1; i < 168; i++) fac[i] = fac[i - 1] * (double)i;
    cpuInitSna(rootpq.data(), cglist.data(), fac.data(), idx_max, idxz.data(), idxz_block.data(),
               idxb.data(), idxb_block.data(), idxu_block.data(), idxcg_block.data(), twojmax);
    const int idxu_max = idx_max[1], idxb_max = idx_max[2], idxz_max = idx_max[3], ncoeff = idxb_max;
    double radelem[2] = {0.0, radelem1}, wjelem[2] = {0.0, wjelem1};
    int map[2] = {0, 0};
    double cut = (radelem1 + radelem1) * rcutfac;
    double rcutsq[4] = {0, 0, 0, cut * cut};
    double bzero[64];
    for (int j = 0; j <= twojmax; j++) bzero[j] = bnormflag ? 1.0 : (double)(j + 1);
    const double wself = 1.0;
    const int na = inum;
    std::vector<int> pairnum(na), pairlist((size_t)na * neighmax), pairnumsum(na + 1);
    cpuNeighPairList(pairnum.data(), pairlist.data(), (double *)x, rcutsq, (int *)alist, (int *)neighlist,
                     (int *)neighnum, (int *)atomtype, (int *)alist, na, neighmax, dim, ntypes);
    pairnumsum[0] = 0;
    for (int i = 0; i < na; i++) pairnumsum[i + 1] = pairnumsum[i] + pairnum[i];
    const int ijnum = pairnumsum[na];
    std::vector<int> ai(ijnum), aj(ijnum), ti(ijnum), tj(ijnum), aii(ijnum);
    std::vector<double> rij((size_t)3 * ijnum);
    cpuNeighPairs(rij.data(), (double *)x, aii.data(), ai.data(), aj.data(), ti.data(), tj.data(), pairnum.data(),
                  pairlist.data(), pairnumsum.data(), (int *)alist, (int *)atomtype, (int *)alist, na, neighmax, dim);
    std::vector<double> ur((size_t)idxu_max * ijnum), ui((size_t)idxu_max * ijnum),
        dur((size_t)idxu_max * dim * ijnum), dui((size_t)idxu_max * dim * ijnum),
        utr((size_t)idxu_max * na), uti((size_t)idxu_max * na), zr((size_t)idxz_max * na), zi((size_t)idxz_max * na),
        yr((size_t)idxu_max * na), yi((size_t)idxu_max * na), blist((size_t)idxb_max * na),
        beta((size_t)ncoeff * na), dedr((size_t)dim * ijnum);
    cpuComputeUij(ur.data(), ui.data(), rootpq.data(), rij.data(), radelem, rmin0, rfac0, rcutfac,
                  idxu_block.data(), ai.data(), aj.data(), ti.data(), tj.data(), twojmax, idxu_max, ijnum);
    cpuZeroUarraytot(utr.data(), uti.data(), wself, idxu_block.data(), (int *)atomtype, map, ai.data(),
                     wselfallflag, chemflag, idxu_max, nelem, twojmax, inum);
    cpuAddUarraytot(utr.data(), uti.data(), ur.data(), ui.data(), rij.data(), wjelem, radelem, rmin0, rcutfac,
                    idxu_block.data(), (int *)alist, (int *)atomtype, pairnum.data(), pairnumsum.data(), map,
                    tj.data(), twojmax, idxu_max, nelem, inum, switchflag, chemflag);
    cpuComputeDuijdrj(dur.data(), dui.data(), ur.data(), ui.data(), rootpq.data(), rij.data(), wjelem, radelem,
                      rmin0, rfac0, rcutfac, idxu_block.data(), ai.data(), aj.data(), ti.data(), tj.data(), twojmax,
                      idxu_max, ijnum, switchflag);
    cpuComputeZi(zr.data(), zi.data(), utr.data(), uti.data(), cglist.data(), idxz.data(), idxu_block.data(),
                 idxcg_block.data(), twojmax, idxu_max, idxz_max, nelem, bnormflag, inum);
    cpuComputeBi(blist.data(), zr.data(), zi.data(), utr.data(), uti.data(), bzero, (int *)alist, (int *)atomtype,
                 map, idxb.data(), idxu_block.data(), idxz_block.data(), twojmax, idxb_max, idxu_max, idxz_max,
                 nelem, bzeroflag, wselfallflag, chemflag, inum);
    cpuSnapTallyEnergyFull(eatom, blist.data(), (double *)coeffelem, (int *)alist, map, (int *)atomtype, inum,
                           ncoeff, ncoeffall, quadraticflag);
    cpuComputeBeta2(beta.data(), blist.data(), (double *)coeffelem, (int *)alist, map, (int *)atomtype, inum,
                    ncoeff, ncoeffall, quadraticflag);
    cpuComputeYi(yr.data(), yi.data(), utr.data(), uti.data(), cglist.data(), beta.data(), idxz.data(),
                 idxb_block.data(), idxu_block.data(), idxcg_block.data(), twojmax, idxb_max, idxu_max, idxz_max,
                 nelem, bnormflag, ncoeff, inum);
    cpuComputeDeidrj(dedr.data(), yr.data(), yi.data(), dur.data(), dui.data(), idxu_block.data(), map, ai.data(),
                     aj.data(), ti.data(), tj.data(), nelem, twojmax, idxu_max, chemflag, ijnum);
    cpuSnapTallyForceFull(fatom, dedr.data(), ai.data(), aj.data(), (int *)alist, ijnum);
    cpuSnapTallyVirialFull(vatom, dedr.data(), rij.data(), ai.data(), aj.data(), inum, ijnum);
}

// Per-configuration SNAP descriptors in the order of ComputeSnap
// (snappotential.cpp:762-910): bi[ncoeff] = sum_i B_i, bd[3*i + c + 3*inum*k] =
// d(sum_a B_ak)/dx_ic, bv[6*k + c] (virial), blist[i + inum*k] per-atom B.
// Outputs are overwritten.  Single element, chemflag = quadraticflag = 0.
void ref_snap_descriptors(double *bi, double *bd, double *bv, double *blist_out, const double *x,
                          const int *atomtype, const int *alist, const int *neighlist, const int *neighnum,
                          int inum, int neighmax, int twojmax, double rcutfac, double rfac0, double rmin0,
                          double radelem1, double wjelem1, int switchflag, int bzeroflag, int bnormflag,
                          int wselfallflag)
{
    const int dim = 3, ntypes = 1, nelem = 1, chemflag = 0, quadraticflag = 0;
    int jdim = twojmax + 1;
    int idxcg_count = 0, idxz_count = 0, idxb_count = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= MIN(twojmax, j1 + j2); j += 2) {
                idxcg_count += (j1 + 1) * (j2 + 1);
                if (j >= j1) idxb_count++;
                for (int mb = 0; 2 * mb <= j; mb++) idxz_count += j + 1;
            }
    int idx_max[5];
    std::vector<double> rootpq((jdim + 1) * (jdim + 1)), cglist(idxcg_count), fac(168);
    std::vector<int> idxz(idxz_count * 10), idxz_block(jdim * jdim * jdim), idxb(idxb_count * 3),
        idxb_block(jdim * jdim * jdim), idxu_block(jdim), idxcg_block(jdim * jdim * jdim);
    fac[0] = 1.0;
    for (int i = 1; i < 168; i++) fac[i] = fac[i - 1] * (double)i;
    cpuInitSna(rootpq.data(), cglist.data(), fac.data(), idx_max, idxz.data(), idxz_block.data(),
               idxb.data(), idxb_block.data(), idxu_block.data(), idxcg_block.data(), twojmax);
    int idxu_max = idx_max[1], idxb_max = idx_max[2], idxz_max = idx_max[3];
    double radelem[2] = {0.0, radelem1}, wjelem[2] = {0.0, wjelem1};
    int map[2] = {0, 0};
    double cut = (radelem1 + radelem1) * rcutfac;
    double rcutsq[4] = {0, 0, 0, cut * cut};
    double bzero[64];
    for (int j = 0; j <= twojmax; j++) bzero[j] = bnormflag ? 1.0 : (double)(j + 1);
    double wself = 1.0;
    const int ncoeff = idxb_max, nperdim = ncoeff;

    std::vector<int> pairnum(inum), pairlist((size_t)inum * neighmax), ilist(inum), pairnumsum(inum + 1);
    for (int i = 0; i < inum; i++) ilist[i] = i;
    cpuNeighPairList(pairnum.data(), pairlist.data(), (double *)x, rcutsq, ilist.data(), (int *)neighlist,
                     (int *)neighnum, (int *)atomtype, (int *)alist, inum, neighmax, dim, ntypes);
    pairnumsum[0] = 0;
    for (int i = 0; i < inum; i++) pairnumsum[i + 1] = pairnumsum[i] + pairnum[i];
    int ijnum = pairnumsum[inum];
    std::vector<int> ai(ijnum + 1), aj(ijnum + 1), ti(ijnum + 1), tj(ijnum + 1), aii(ijnum + 1);
    std::vector<double> rij((size_t)3 * ijnum + 3);
    cpuNeighPairs(rij.data(), (double *)x, aii.data(), ai.data(), aj.data(), ti.data(), tj.data(), pairnum.data(),
                  pairlist.data(), pairnumsum.data(), ilist.data(), (int *)atomtype, (int *)alist, inum, neighmax,
                  dim);
    // cpuComputeDbidrj reads direction k of dU at offset k * idxu_max * ijnum
    const size_t nu = (size_t)idxu_max * ijnum;
    std::vector<double> ulr(nu + 1), uli(nu + 1), dul((size_t)3 * nu * 2 + 1);
    double *dulr = dul.data(), *duli = dul.data() + 3 * nu;
    cpuComputeSij(ulr.data(), uli.data(), dulr, duli, dulr + nu, duli + nu, dulr + 2 * nu, duli + 2 * nu,
                  rootpq.data(), rij.data(), wjelem, radelem, rmin0, rfac0, rcutfac, idxu_block.data(), ti.data(),
                  tj.data(), twojmax, idxu_max, ijnum, switchflag);
    std::vector<double> utr((size_t)idxu_max * inum), uti((size_t)idxu_max * inum);
    cpuZeroUarraytot2(utr.data(), uti.data(), wself, idxu_block.data(), (int *)atomtype, map, ai.data(),
                      wselfallflag, chemflag, idxu_max, nelem, twojmax, inum);
    cpuAddUarraytot(utr.data(), uti.data(), ulr.data(), uli.data(), map, ai.data(), tj.data(), idxu_max, inum, ijnum,
                    chemflag);
    std::vector<double> zr((size_t)idxz_max * inum), zi((size_t)idxz_max * inum);
    cpuComputeZi2(zr.data(), zi.data(), utr.data(), uti.data(), cglist.data(), idxz.data(), idxu_block.data(),
                  idxcg_block.data(), twojmax, idxu_max, idxz_max, nelem, bnormflag, inum);
    std::vector<double> blist((size_t)idxb_max * inum);
    cpuComputeBi2(blist.data(), zr.data(), zi.data(), utr.data(), uti.data(), bzero, ilist.data(), (int *)atomtype,
                  map, idxb.data(), idxu_block.data(), idxz_block.data(), twojmax, idxb_max, idxu_max, idxz_max,
                  nelem, bzeroflag, wselfallflag, chemflag, inum);
    std::vector<double> dblist((size_t)idxb_max * 3 * (ijnum + 1));
    cpuComputeDbidrj(dblist.data(), zr.data(), zi.data(), dulr, duli, idxb.data(), idxu_block.data(),
                     idxz_block.data(), map, ai.data(), tj.data(), twojmax, idxb_max, idxu_max, idxz_max, nelem,
                     bnormflag, chemflag, inum, ijnum);
    std::vector<int> type1(inum, 1);
    cpuSnapTallyBispectrum(bi, blist.data(), ilist.data(), type1.data(), inum, ncoeff, nperdim, ntypes,
                           quadraticflag);
    cpuSnapTallyBispectrumDeriv(bd, blist.data(), dblist.data(), aii.data(), ai.data(), aj.data(), ti.data(), inum,
                                ijnum, ncoeff, nperdim, ntypes, quadraticflag);
    cpuSnapTallyBispectrumVirial(bv, blist.data(), dblist.data(), rij.data(), aii.data(), ai.data(), aj.data(),
                                 ti.data(), inum, ijnum, ncoeff, nperdim, ntypes, quadraticflag);
    if (blist_out) std::copy(blist.begin(), blist.end(), blist_out);
}

void ref_nve_initial(double *x, double *v, const double *f, const double *mass, double dtf,
                     double dtv, const int *type, const int *ilist, int inum)
{
    cpuNVEInitialIntegrate(x, v, (double *)f, (double *)mass, dtf, dtv, (int *)type, (int *)ilist, 3, inum);
}

void ref_nve_final(double *x, double *v, const double *f, const double *mass, double dtf,
                   const int *type, const int *ilist, int inum)
{
    cpuNVEFinalIntegrate(x, v, (double *)f, (double *)mass, dtf, (int *)type, (int *)ilist, 3, inum);
}

int ref_omp_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// u and du/dx_ij of the ZBL pair potential for n pair vectors xij [n][3]
// (the reference's generated cpuPairaGradient, potential 1)
void ref_zbl_pairs(double *u, double *u_xij, const double *xij, int n)
{
    cpuPairaGradient<double>(u, u_xij, (double *)xij, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                             nullptr, nullptr, 3, 0, 0, 0, 0, n, 1);
}

// MDP's NVT (Nose-Hoover chain) half steps, cpuVelocityIntegration.cpp:602-648
void ref_nvt_initial(double *x, double *v, const double *f, const double *mass, double *dtarray, double *tarray,
                     double *eta_mass, double *eta, double *eta_dot, double *eta_dotdot, const int *type,
                     const int *ilist, int eta_mass_flag, int mtchain, int nc_tchain, int inum)
{
    cpuNVTInitialIntegrate(x, v, (double *)f, (double *)mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot,
                           (int *)type, (int *)ilist, eta_mass_flag, 0, mtchain, nc_tchain, 3, inum);
}
void ref_nvt_final(double *x, double *v, const double *f, const double *mass, double *dtarray, double *tarray,
                   double *eta_mass, double *eta, double *eta_dot, double *eta_dotdot, const int *type,
                   const int *ilist, int eta_mass_flag, int mtchain, int nc_tchain, int inum)
{
    cpuNVTFinalIntegrate(x, v, (double *)f, (double *)mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot,
                         (int *)type, (int *)ilist, eta_mass_flag, 0, mtchain, nc_tchain, 3, inum);
}

// Force constraints of cpuFixes.cpp, by kind: 0 set, 1 line, 2 plane, 3 ave,
// 4 wall reflect, 5 harmonic, 6 LJ93, 7 LJ126, 8 LJ1043, 9 Morse,
// 10 add (with box / image), 11 drag (with box / pbc).  Host arrays, double.
void ref_fix(int kind, double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
             int *iparam, int *ilist, double *box, int *image, int *pbc, int triclinic, int eflag_atom,
             int vflag_atom, int dim, int inum)
{
    switch (kind) {
    case 0: cpuFixSetForce(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 1: cpuFixLineForce(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 2: cpuFixPlaneForce(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 3: cpuFixAveForce(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 4: cpuFixWallReflect(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 5: cpuFixWallHarmonic(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 6: cpuFixWallLJ93(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 7: cpuFixWallLJ126(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 8: cpuFixWallLJ1043(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 9: cpuFixWallMorse(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum); break;
    case 10:
        cpuFixAddForce(x, v, f, eatom, vatom, fparam, box, iparam, ilist, image, triclinic, eflag_atom, vflag_atom,
                       dim, inum);
        break;
    case 11:
        cpuFixDragForce(x, v, f, eatom, vatom, fparam, box, iparam, ilist, pbc, triclinic, eflag_atom, vflag_atom,
                        dim, inum);
        break;
    }
}

// set-velocity integration (cpuVelocityIntegration.cpp:430-463): stage 0
// initial, 1 final
void ref_set_velocity(int stage, double *x, double *v, double *f, double *mass, double *fparam, double dtf,
                      double dtv, int *type, int *ilist, int *iparam, int dim, int inum)
{
    if (stage == 0)
        cpuSetVelocityInitialIntegrate(x, v, f, mass, fparam, dtf, dtv, type, ilist, iparam, dim, inum);
    else
        cpuSetVelocityFinalIntegrate(x, v, f, mass, dtf, type, ilist, iparam, dim, inum);
}

// velocity-rescaling thermostats (cpuVelocityIntegration.cpp:708-858)
double ref_velocity_rescaling(double *v, double *mass, double *dtarray, double *tarray, double *second,
                              double energy, int *type, int *ilist, int *seed, int *save, int biasflag, int mode,
                              int dim, int inum)
{
    return cpuVelocityRescalingThermostat(v, mass, dtarray, tarray, second, energy, type, ilist, seed, save,
                                          biasflag, mode, dim, inum);
}

}  // extern "C"
