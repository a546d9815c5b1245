/*
 * Device-pointer SNAP operations with the argument lists of MDP's backend
 * dispatch (src/C++/Common/mdpgpucore.h:516-612, called from the inline
 * wrappers of src/C++/Common/mdpcore.h with backend == 2).
 *
 * The extern "C" functions are exported by libmdp_b200.so.  For C++ builds of
 * MDP (cpuMDP/gpuMDP), defining MDP_B200_GPUCORE_TEMPLATES before including
 * this header also defines the reference's gpu* template entry points for
 * T = double on top of them, replacing src/C++/Core/gpuSnap4.cu and the pair
 * kernels of gpuSnap.cu at link time.  Array layouts are the reference's:
 * U/Y [idxu][inum], rij [ijnum][3], fatom [anum][3], vatom [6][anum].
 * Supported: one element type, 2J = 4, 6, 8, double.  On unsupported input
 * the outputs are untouched and mdp_last_error() says why.
 */
#ifndef MDP_B200_GPUCORE_H
#define MDP_B200_GPUCORE_H

#ifdef __cplusplus
extern "C" {
#endif

/* mdpgpucore.h:582-584, gpuSnapComputeUi */
void mdp_gpu_snap_compute_ui_f64(double *Utotr, double *Utoti, const double *rootpqarray, const double *rij,
                                 const double *wjelem, const double *radelem, double rmin0, double rfac0,
                                 double rcutfac, const int *idxu_block, const int *map, const int *aii,
                                 const int *ti, const int *tj, int twojmax, int idxu_max, int inum, int ijnum,
                                 int switchflag, int chemflag);
/* mdpgpucore.h:586-588, gpuAddWself2Ui */
void mdp_gpu_add_wself2ui_f64(double *Utotr, double *Utoti, double wself, const int *idxu_block, const int *type,
                              const int *map, const int *ai, int wselfall_flag, int chemflag, int idxu_max,
                              int nelements, int twojmax, int inum);
/* mdpgpucore.h:594-597, gpuSnapComputeEi */
void mdp_gpu_snap_compute_ei_f64(double *eatom, const double *Utotr, const double *Utoti, const double *cglist,
                                 const double *bzero, const double *coeffelem, const int *ilist, const int *map,
                                 const int *type, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall,
                                 int bnorm_flag, int bzero_flag, int wselfall_flag, int quadraticflag, int inum);
/* mdpgpucore.h:590-592, gpuSnapComputeBi */
void mdp_gpu_snap_compute_bi_f64(double *blist, const double *Utotr, const double *Utoti, const double *cglist,
                                 const double *bzero, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 const int *idxz_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum);
/* mdpgpucore.h:603-605, gpuSnapComputeYi (beta from coeffelem) */
void mdp_gpu_snap_compute_yi_f64(double *ylist_r, double *ylist_i, const double *Utotr, const double *Utoti,
                                 const double *cglist, const double *coeffelem, const int *map, const int *type,
                                 const int *idxz, const int *idxb_block, const int *idxu_block,
                                 const int *idxcg_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int ncoeffall, int bnorm_flag, int inum);
/* mdpgpucore.h:607-609, gpuSnapComputeFi */
void mdp_gpu_snap_compute_fi_f64(double *fatom, double *vatom, const double *ylist_r, const double *ylist_i,
                                 const double *rootpqarray, const double *rij, const double *wjelem,
                                 const double *radelem, double rmin0, double rfac0, double rcutfac,
                                 const int *idxu_block, const int *map, const int *aii, const int *ai, const int *aj,
                                 const int *ti, const int *tj, int twojmax, int idxu_max, int inum, int anum,
                                 int ijnum, int switchflag, int chemflag);
/* mdpgpucore.h:519-520, gpuNeighPairList (typed, neighbour rows of jnum) */
void mdp_gpu_neigh_pair_list_f64(int *pairnum, int *pairlist, const double *x, const double *rcutsq, const int *ilist,
                                 const int *neighlist, const int *neighnum, const int *atomtype, const int *alist,
                                 int inum, int jnum, int dim, int ntypes);
/* mdpgpucore.h:526-528, gpuNeighPairs */
void mdp_gpu_neigh_pairs_f64(double *xij, const double *x, int *aii, int *ai, int *aj, int *ti, int *tj,
                             const int *pairnum, const int *pairlist, const int *pairnumsum, const int *ilist,
                             const int *atomtype, const int *alist, int inum, int jnum, int dim);

/* No counterpart in the reference.  The per-atom bispectrum of
 * mdp_gpu_snap_compute_bi_f64 for callers that must not allocate device memory
 * (a host application whose memory pool owns the device, or a loop that cannot
 * take the implicit synchronisation of cudaMalloc/cudaFree): its 32-atom-tile
 * scratch is a fixed array inside the library, so the call allocates nothing.
 * U in MDP's layout [idxu][inum] (device), blist[jjb * inum + ii] (device),
 * launched on `stream`.  Limits: inum <= 2048 (larger is rejected with an
 * error), 2J = 4, 6, 8; the array costs 9,338,880 bytes on every GPU that
 * loads the library.  All calls share the array: calls whose GPU work overlaps
 * race, so serialise them on one stream.  The first call on a device sets up
 * the array's address (and the library's constant tables) and should come
 * before any stream capture.  Returns 0, or -1 with mdp_last_error(). */
int mdp_gpu_snap_compute_bi_noalloc_f64(double *blist, const double *Utotr, const double *Utoti, int twojmax,
                                        int bnorm_flag, int bzero_flag, int inum, void *stream);

#ifdef __cplusplus
}

#ifdef MDP_B200_GPUCORE_TEMPLATES
template <typename T> void gpuSnapComputeUi(T *Stotr, T *Stoti, T *rootpqarray, T *rij, T *wjelem, T *radelem,
        T rmin0, T rfac0, T rcutfac, int *idxu_block, int *map, int *ai, int *ti, int *tj,
        int twojmax, int idxu_max, int inum, int ijnum, int switchflag, int chemflag);
template <> inline void gpuSnapComputeUi<double>(double *Stotr, double *Stoti, double *rootpqarray, double *rij,
        double *wjelem, double *radelem, double rmin0, double rfac0, double rcutfac, int *idxu_block, int *map,
        int *ai, int *ti, int *tj, int twojmax, int idxu_max, int inum, int ijnum, int switchflag, int chemflag)
{
    mdp_gpu_snap_compute_ui_f64(Stotr, Stoti, rootpqarray, rij, wjelem, radelem, rmin0, rfac0, rcutfac, idxu_block,
                                map, ai, ti, tj, twojmax, idxu_max, inum, ijnum, switchflag, chemflag);
}
template <typename T> void gpuAddWself2Ui(T *Stotr, T *Stoti, T wself, int *idxu_block, int *type, int *map,
        int *ai, int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax, int inum);
template <> inline void gpuAddWself2Ui<double>(double *Stotr, double *Stoti, double wself, int *idxu_block,
        int *type, int *map, int *ai, int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax,
        int inum)
{
    mdp_gpu_add_wself2ui_f64(Stotr, Stoti, wself, idxu_block, type, map, ai, wselfall_flag, chemflag, idxu_max,
                             nelements, twojmax, inum);
}
template <typename T> void gpuSnapComputeEi(T *eatom, T *Stotr, T *Stoti, T *cglist, T *bzero, T *coeffelem,
        int *ilist, int *map, int *type, int *idxb, int *idxcg_block, int *idxu_block, int twojmax, int idxb_max,
        int idxu_max, int nelements, int ncoeffall, int bnorm_flag, int bzero_flag, int wselfall_flag,
        int quadraticflag, int inum);
template <> inline void gpuSnapComputeEi<double>(double *eatom, double *Stotr, double *Stoti, double *cglist,
        double *bzero, double *coeffelem, int *ilist, int *map, int *type, int *idxb, int *idxcg_block,
        int *idxu_block, int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall, int bnorm_flag,
        int bzero_flag, int wselfall_flag, int quadraticflag, int inum)
{
    mdp_gpu_snap_compute_ei_f64(eatom, Stotr, Stoti, cglist, bzero, coeffelem, ilist, map, type, idxb, idxcg_block,
                                idxu_block, twojmax, idxb_max, idxu_max, nelements, ncoeffall, bnorm_flag,
                                bzero_flag, wselfall_flag, quadraticflag, inum);
}
template <typename T> void gpuSnapComputeBi(T *blist, T *Stotr, T *Stoti, T *cglist, T *bzero, int *idxb,
        int *idxcg_block, int *idxu_block, int *idxz_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
        int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum);
template <> inline void gpuSnapComputeBi<double>(double *blist, double *Stotr, double *Stoti, double *cglist,
        double *bzero, int *idxb, int *idxcg_block, int *idxu_block, int *idxz_block, int twojmax, int idxb_max,
        int idxu_max, int idxz_max, int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum)
{
    mdp_gpu_snap_compute_bi_f64(blist, Stotr, Stoti, cglist, bzero, idxb, idxcg_block, idxu_block, idxz_block,
                                twojmax, idxb_max, idxu_max, idxz_max, nelements, bnorm_flag, bzero_flag,
                                wselfall_flag, inum);
}
template <typename T> void gpuSnapComputeYi(T *ylist_r, T *ylist_i, T *Stotr, T *Stoti, T *cglist, T *coeffelem,
        int *map, int *type, int *idxz, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax,
        int idxb_max, int idxu_max, int idxz_max, int nelements, int ncoeffall, int bnorm_flag, int inum);
template <> inline void gpuSnapComputeYi<double>(double *ylist_r, double *ylist_i, double *Stotr, double *Stoti,
        double *cglist, double *coeffelem, int *map, int *type, int *idxz, int *idxb_block, int *idxu_block,
        int *idxcg_block, int twojmax, int idxb_max, int idxu_max, int idxz_max, int nelements, int ncoeffall,
        int bnorm_flag, int inum)
{
    mdp_gpu_snap_compute_yi_f64(ylist_r, ylist_i, Stotr, Stoti, cglist, coeffelem, map, type, idxz, idxb_block,
                                idxu_block, idxcg_block, twojmax, idxb_max, idxu_max, idxz_max, nelements,
                                ncoeffall, bnorm_flag, inum);
}
template <typename T> void gpuSnapComputeFi(T *fatom, T *vatom, T *ylist_r, T *ylist_i, T *rootpqarray, T *rij,
        T *wjelem, T *radelem, T rmin0, T rfac0, T rcutfac, int *idxu_block, int *map, int *aii, int *ai, int *aj,
        int *ti, int *tj, int twojmax, int idxu_max, int inum, int anum, int ijnum, int switchflag, int chemflag);
template <> inline void gpuSnapComputeFi<double>(double *fatom, double *vatom, double *ylist_r, double *ylist_i,
        double *rootpqarray, double *rij, double *wjelem, double *radelem, double rmin0, double rfac0,
        double rcutfac, int *idxu_block, int *map, int *aii, int *ai, int *aj, int *ti, int *tj, int twojmax,
        int idxu_max, int inum, int anum, int ijnum, int switchflag, int chemflag)
{
    mdp_gpu_snap_compute_fi_f64(fatom, vatom, ylist_r, ylist_i, rootpqarray, rij, wjelem, radelem, rmin0, rfac0,
                                rcutfac, idxu_block, map, aii, ai, aj, ti, tj, twojmax, idxu_max, inum, anum, ijnum,
                                switchflag, chemflag);
}
template <typename T> void gpuNeighPairList(int *pairnum, int *pairlist, T *x, T *rcutsq, int *ilist, int *neighlist,
        int *neighnum, int *atomtype, int *alist, int inum, int jnum, int dim, int ntypes);
template <> inline void gpuNeighPairList<double>(int *pairnum, int *pairlist, double *x, double *rcutsq, int *ilist,
        int *neighlist, int *neighnum, int *atomtype, int *alist, int inum, int jnum, int dim, int ntypes)
{
    mdp_gpu_neigh_pair_list_f64(pairnum, pairlist, x, rcutsq, ilist, neighlist, neighnum, atomtype, alist, inum,
                                jnum, dim, ntypes);
}
template <typename T> void gpuNeighPairs(T *xij, T *x, int *aii, int *ai, int *aj, int *ti, int *tj, int *pairnum,
        int *pairlist, int *pairnumsum, int *ilist, int *atomtype, int *alist, int inum, int jnum, int dim);
template <> inline void gpuNeighPairs<double>(double *xij, double *x, int *aii, int *ai, int *aj, int *ti, int *tj,
        int *pairnum, int *pairlist, int *pairnumsum, int *ilist, int *atomtype, int *alist, int inum, int jnum,
        int dim)
{
    mdp_gpu_neigh_pairs_f64(xij, x, aii, ai, aj, ti, tj, pairnum, pairlist, pairnumsum, ilist, atomtype, alist, inum,
                            jnum, dim);
}
#endif /* MDP_B200_GPUCORE_TEMPLATES */
#endif /* __cplusplus */
#endif
