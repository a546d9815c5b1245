/*
 * Drop-in replacement for MDP's Julia C-ABI SNAP library.
 *
 * Same names, signatures, argument meanings and array layouts as
 * src/Julia/Potential/cpuSnap.h:15-84 of MDP, so src/Julia/Potential/snapcpp.jl
 * loads libmdp_b200.so in place of cpuSnap.so (snapcpp.jl:12-38 dlopens it by
 * path) and calls it unchanged.  All pointers are HOST pointers; each call
 * stages its arrays through the GPU and computes there.  Outputs accumulate
 * exactly as in the reference (+= into caller-zeroed arrays).
 *
 * Supported: one element type (chemflag = 0, quadraticflag = 0), 2J = 4, 6, 8.
 * The descriptor chain (cpuComputeSij ... cpuSnapTallyBispectrumVirial) also
 * takes any 2J the caller's tables describe, several pair types (per-pair
 * cutoffs) and quadraticflag = 1 in the three tallies.
 * These functions return void like the reference's; when an argument is not
 * supported they leave the outputs untouched and mdp_last_error()
 * (include/mdp_b200.h) says why.
 */
#ifndef MDP_B200_CPUSNAP_H
#define MDP_B200_CPUSNAP_H

#ifdef __cplusplus
extern "C" {
#endif

/* cpuSnap.h:7-13 (table sizes) */
int idxcgcount(int twojmax);
int idxucount(int twojmax);
int idxbcount(int twojmax);
int idxzcount(int twojmax);

/* cpuSnap.h:15-16 -- index lists, rootpq, Clebsch-Gordan table */
void cpuInitSna(double *rootpqarray, double *cglist, double *factorial, int *idx_max, int *idxz,
                int *idxz_block, int *idxb, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax);

/* cpuSnap.h:18-19 -- typed pair filter over a CSR neighbour list */
void cpuNeighPairList(int *pairnum, int *pairlist, double *x, double *rcutsq, int *ilist, int *neighlist,
                      int *neighnum, int *atomtype, int *alist, int inum, int dim, int ntypes);

/* cpuSnap.h:21-22 -- pair vectors and indices */
void cpuNeighPairs(double *xij, double *x, int *aii, int *ai, int *aj, int *ti, int *tj,
                   int *pairlist, int *pairnumsum, int *ilist, int *atomtype, int *alist, int inum, int dim);

/* cpuSnap.h:24-26 -- U accumulation over pairs */
void cpuSnapComputeUi(double *Utotr, double *Utoti, double *rootpqarray, double *rij, double *wjelem, double *radelem,
                      double rmin0, double rfac0, double rcutfac, int *map, int *aii, int *ti, int *tj,
                      int twojmax, int idxu_max, int inum, int ijnum, int switchflag, int chemflag);

/* cpuSnap.h:28-29 -- wself and mirror */
void cpuAddWself2Ui(double *Utotr, double *Utoti, double wself, int *idxu_block, int *type, int *map,
                    int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax, int inum);

/* cpuSnap.h:31-34 -- per-atom energy */
void cpuSnapComputeEi(double *eatom, double *Utotr, double *Utoti, double *cglist, double *bzero,
                      double *coeffelem, int *ilist, int *map, int *type, int *idxb, int *idxcg_block, int *idxu_block,
                      int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall, int bnorm_flag,
                      int bzero_flag, int wselfall_flag, int chemflag, int inum);

/* cpuSnap.h:36-38 -- per-atom bispectrum, blist[jjb * inum + ii] */
void cpuSnapComputeBi(double *blist, double *Utotr, double *Utoti, double *cglist, double *bzero,
                      int *idxb, int *idxcg_block, int *idxu_block, int *idxz_block, int twojmax, int idxb_max,
                      int idxu_max, int idxz_max, int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag,
                      int inum);

/* cpuSnap.h:40-42 -- Y */
void cpuSnapComputeYi(double *ylist_r, double *ylist_i, double *Utotr, double *Utoti, double *cglist, double *beta,
                      int *map, int *type, int *idxz, int *idxb_block, int *idxu_block, int *idxcg_block,
                      int twojmax, int idxb_max, int idxu_max, int idxz_max, int nelements, int ncoeffall,
                      int bnorm_flag, int chemflag, int inum);

/* cpuSnap.h:44-46 -- forces and per-atom virial (vatom[6 * i + c], -r (x) dE on i) */
void cpuSnapComputeFi(double *fatom, double *vatom, double *ylist_r, double *ylist_i, double *rootpqarray,
                      double *rij, double *wjelem, double *radelem, double rmin0, double rfac0, double rcutfac,
                      int *map, int *aii, int *ai, int *aj, int *ti, int *tj, int twojmax, int idxu_max,
                      int inum, int anum, int ijnum, int switchflag, int chemflag);

/* ---- descriptor chain: what snapdescriptors calls (snapcpp.jl:539-665) ---- */

/* cpuSnap.h:48-50 -- per-pair U (Sr, Si) and dU/dx, dU/dy, dU/dz, [k][ijnum] */
void cpuComputeSij(double *Sr, double *Si, double *Srx, double *Six, double *Sry, double *Siy, double *Srz,
                   double *Siz, double *rootpqarray, double *rij, double *wjelem, double *radelem, double rmin0,
                   double rfac0, double rcutfac, int *idxu_block, int *ti, int *tj, int twojmax, int idxu_max,
                   int ijnum, int switch_flag);

/* cpuSnap.h:52-54 -- the same with dU packed as [3][k][ijnum] in dSr / dSi */
void cpuComputeUij(double *Sr, double *Si, double *dSr, double *dSi, double *rootpqarray, double *rij,
                   double *wjelem, double *radelem, double rmin0, double rfac0, double rcutfac, int *idxu_block,
                   int *ti, int *tj, int twojmax, int idxu_max, int ijnum, int switch_flag);

/* cpuSnap.h:56-58 -- per-atom U totals set to wself on the diagonals, [k][inum] */
void cpuZeroUarraytot2(double *Stotr, double *Stoti, double wself, int *idxu_block, int *type, int *map, int *ai,
                       int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax, int inum);

/* cpuSnap.h:60-61 -- U totals += the pairs' U (atom ai[p]) */
void cpuAddUarraytot(double *Stotr, double *Stoti, double *Sr, double *Si, int *map, int *ai, int *tj, int idxu_max,
                     int inum, int ijnum, int chemflag);

/* cpuSnap.h:63-65 -- Z per atom and idxz entry, [jjz][inum] */
void cpuComputeZi2(double *zlist_r, double *zlist_i, double *Stotr, double *Stoti, double *cglist, int *idxz,
                   int *idxu_block, int *idxcg_block, int twojmax, int idxu_max, int idxz_max, int nelements,
                   int bnorm_flag, int inum);

/* cpuSnap.h:67-70 -- per-atom bispectrum, [jjb][inum] */
void cpuComputeBi2(double *blist, double *zlist_r, double *zlist_i, double *Stotr, double *Stoti, double *bzero,
                   int *ilist, int *type, int *map, int *idxb, int *idxu_block, int *idxz_block, int twojmax,
                   int idxb_max, int idxu_max, int idxz_max, int nelements, int bzero_flag, int wselfall_flag,
                   int chemflag, int inum);

/* cpuSnap.h:72-75 -- per-pair dB/dr, [jjb][3][ijnum] */
void cpuComputeDbidrj(double *dblist, double *zlist_r, double *zlist_i, double *dulist_r, double *dulist_i, int *idxb,
                      int *idxu_block, int *idxz_block, int *map, int *ai, int *tj, int twojmax, int idxb_max,
                      int idxu_max, int idxz_max, int nelements, int bnorm_flag, int chemflag, int inum, int ijnum);

/* cpuSnap.h:77-78 -- bi[type block][slot] = sum over atoms of B */
void cpuSnapTallyBispectrum(double *bi, double *bispectrum, int *ilist, int *type, int inum, int ncoeff, int nperdim,
                            int ntype, int quadraticflag);

/* cpuSnap.h:80-81 -- db[type block][slot][atom][3]: + on ai, - on aj of each pair */
void cpuSnapTallyBispectrumDeriv(double *db, double *bispectrum, double *dbdr, int *aii, int *ai, int *aj, int *ti,
                                 int inum, int ijnum, int ncoeff, int nperdim, int ntype, int quadraticflag);

/* cpuSnap.h:83-84 -- bv[type block][slot][6] = sum over pairs of -r (x) dB */
void cpuSnapTallyBispectrumVirial(double *bv, double *bispectrum, double *dbdr, double *rij, int *aii, int *ti,
                                  int inum, int ijnum, int ncoeff, int nperdim, int ntype, int quadraticflag);

#ifdef __cplusplus
}
#endif
#endif
