/*
 * Device-pointer operations with the argument lists of MDP's backend
 * dispatch (src/C++/Common/mdpgpucore.h, called from the inline wrappers of
 * src/C++/Common/mdpcore.h with backend == 2): the SNAP stages (:516-612) and
 * the rest of the MD loop's hot path -- prefix sums, ghost atoms, cell lists,
 * full neighbour lists, velocity Verlet, periodic wrapping, per-atom kinetic
 * energy and column sums.
 *
 * The extern "C" functions are exported by libmdp_b200.so.  For C++ builds of
 * MDP (cpuMDP/gpuMDP), defining MDP_B200_GPUCORE_TEMPLATES before including
 * this header also defines the reference's gpu* entry points for T = double on
 * top of them, replacing src/C++/Core/gpuSnap4.cu, the pair kernels of
 * gpuSnap.cu, gpuCumsum.cu, gpuNeighborList3D.cu, gpuVelocityIntegration.cu
 * (integrator modes 0, 1 and 2, set-velocity integration and the
 * velocity-rescaling thermostats), gpuFixes.cu and gpuDomain.cu's gpuPBC at
 * link time.  Array layouts are
 * the reference's: U/Y [idxu][inum], rij [ijnum][3], fatom [anum][3],
 * vatom [6][anum], x [natom][dim]; with chemflag, U and Y hold one such block
 * per element ([element][idxu][inum], block map[tj] for a pair).  Supported:
 * 2J = 4, 6, 8, up to four element types (chemflag 0 or 1, per-pair cutoffs
 * (radelem[ti] + radelem[tj]) rcutfac), double; float through the _f32
 * entries.  On unsupported input the outputs are untouched and
 * mdp_last_error() says why.
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
/* mdpgpucore.h:599-601, gpuSnapComputeYi (per-atom beta [idxb][inum]) */
void mdp_gpu_snap_compute_yi_beta_f64(double *ylist_r, double *ylist_i, const double *Utotr, const double *Utoti,
                                      const double *cglist, const double *beta, const int *idxz,
                                      const int *idxb_block, const int *idxu_block, const int *idxcg_block,
                                      int twojmax, int idxb_max, int idxu_max, int idxz_max, int nelements,
                                      int bnorm_flag, int inum);
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

/* ---- the rest of the MD loop (mdp_b200/csrc/abi_md.cu) ---- */
/* mdpgpucore.h:108, gpuCumsum: out[0] = 0, out[j] = sum of in[0..j-1], j < length */
void mdp_gpu_cumsum(int *d_out, int *d_in, int *d_sums, int *d_incr, int length);
/* mdpgpucore.h:132-133, gpuAtomList3D: ghost images appended to x, owners in alist */
void mdp_gpu_atom_list3d_f64(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums, int *d_incr,
                             double *x, const double *pimages, const double *wc, const double *s2rmap, int inum,
                             int pnum, int dim);
/* mdpgpucore.h:136-137, gpuCellList3D */
void mdp_gpu_cell_list3d_f64(int *clist, const double *xi, const double *eta1, const double *eta2,
                             const double *eta3, const double *s2rmap, const int *nc, int inum, int natom, int dim);
/* mdpgpucore.h:138, gpuCell2AtomList */
void mdp_gpu_cell2atom_list(int *c2alist, int *c2anumsum, int *c2anum, const int *clist, int *d_temp, int natom,
                            int ncell);
/* mdpgpucore.h:145-146, gpuFullNeighborList3D (cell lists) */
void mdp_gpu_full_neighbor_list3d_cells_f64(int *neighborlist, int *neighbornum, const double *x,
                                            const double *rcutsq, const int *alist, const int *clist,
                                            const int *c2alist, const int *c2anumsum, const int *nc, int inum,
                                            int jnum, int dim);
/* mdpgpucore.h:141-142, gpuFullNeighborList3D (all pairs) */
void mdp_gpu_full_neighbor_list3d_f64(int *neighborlist, int *neighbornum, const double *x, const double *rcutsq,
                                      int anum, int inum, int jnum, int dim);
/* mdpgpucore.h:309-311, gpuInitialIntegrate (modes 0 NVE, 1 NVE limit, 2 NVT Nose-Hoover chain;
 * dtarray, tarray and the eta arrays on the host, ke and tmp device scratch) */
void mdp_gpu_initial_integrate_f64(double *x, double *v, const double *f, const double *mass, const double *dtarray,
                                   double *tarray, double *eta_mass, double *eta, double *eta_dot,
                                   double *eta_dotdot, double *ke, double *tmp, double vlimitsq, const int *type,
                                   const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                   int mode, int dim, int inum);
/* mdpgpucore.h:313-315, gpuFinalIntegrate */
void mdp_gpu_final_integrate_f64(double *x, double *v, const double *f, const double *mass, const double *dtarray,
                                 double *tarray, double *eta_mass, double *eta, double *eta_dot,
                                 double *eta_dotdot, double *ke, double *tmp, double vlimitsq, const int *type,
                                 const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                 int mode, int dim, int inum);
/* mdpgpucore.h:321-322, gpuPBC (orthogonal and tilted boxes) */
void mdp_gpu_pbc_f64(double *x, double *v, int *image, const double *boxhi, const double *boxlo,
                     const double *hi_lambda, const double *lo_lambda, const double *h, const double *h_inv,
                     const double *h_rate, const int *pbc, int vdeform, int triclinic, int dim, int nlocal);
/* mdpgpucore.h:259-260, gpuComputeKEAtom */
void mdp_gpu_compute_ke_atom_f64(double *ke, const double *mass, const double *v, double mvv2e, const int *type,
                                 const int *ilist, int dim, int inum);
/* mdpgpucore.h:56, gpuArraySumEveryColumn */
void mdp_gpu_array_sum_every_column_f64(double *b, const double *a, int m, int n);
/* mdpgpucore.h:49, gpuArrayGetValueAtIndex<int> */
int mdp_gpu_array_get_value_at_index_int(const int *y, int n);

/* PREC_FLOAT builds of MDP (dstype = float): the same entry points on float
 * device arrays.  The MD-loop operations and the pair list/pairs compute in
 * float with the reference float build's rounding; the SNAP stages widen the
 * float arrays into library-owned double scratch, run the double path and
 * narrow the results back into the caller's arrays. */
void mdp_gpu_snap_compute_ui_f32(float *Utotr, float *Utoti, const float *rootpqarray, const float *rij,
                                 const float *wjelem, const float *radelem, float rmin0, float rfac0,
                                 float rcutfac, const int *idxu_block, const int *map, const int *aii,
                                 const int *ti, const int *tj, int twojmax, int idxu_max, int inum, int ijnum,
                                 int switchflag, int chemflag);
void mdp_gpu_add_wself2ui_f32(float *Utotr, float *Utoti, float wself, const int *idxu_block, const int *type,
                              const int *map, const int *ai, int wselfall_flag, int chemflag, int idxu_max,
                              int nelements, int twojmax, int inum);
void mdp_gpu_snap_compute_ei_f32(float *eatom, const float *Utotr, const float *Utoti, const float *cglist,
                                 const float *bzero, const float *coeffelem, const int *ilist, const int *map,
                                 const int *type, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall,
                                 int bnorm_flag, int bzero_flag, int wselfall_flag, int quadraticflag, int inum);
void mdp_gpu_snap_compute_bi_f32(float *blist, const float *Utotr, const float *Utoti, const float *cglist,
                                 const float *bzero, const int *idxb, const int *idxcg_block, const int *idxu_block,
                                 const int *idxz_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum);
void mdp_gpu_snap_compute_yi_f32(float *ylist_r, float *ylist_i, const float *Utotr, const float *Utoti,
                                 const float *cglist, const float *coeffelem, const int *map, const int *type,
                                 const int *idxz, const int *idxb_block, const int *idxu_block,
                                 const int *idxcg_block, int twojmax, int idxb_max, int idxu_max, int idxz_max,
                                 int nelements, int ncoeffall, int bnorm_flag, int inum);
void mdp_gpu_snap_compute_yi_beta_f32(float *ylist_r, float *ylist_i, const float *Utotr, const float *Utoti,
                                      const float *cglist, const float *beta, const int *idxz,
                                      const int *idxb_block, const int *idxu_block, const int *idxcg_block,
                                      int twojmax, int idxb_max, int idxu_max, int idxz_max, int nelements,
                                      int bnorm_flag, int inum);
void mdp_gpu_snap_compute_fi_f32(float *fatom, float *vatom, const float *ylist_r, const float *ylist_i,
                                 const float *rootpqarray, const float *rij, const float *wjelem,
                                 const float *radelem, float rmin0, float rfac0, float rcutfac,
                                 const int *idxu_block, const int *map, const int *aii, const int *ai, const int *aj,
                                 const int *ti, const int *tj, int twojmax, int idxu_max, int inum, int anum,
                                 int ijnum, int switchflag, int chemflag);
void mdp_gpu_neigh_pair_list_f32(int *pairnum, int *pairlist, const float *x, const float *rcutsq, const int *ilist,
                                 const int *neighlist, const int *neighnum, const int *atomtype, const int *alist,
                                 int inum, int jnum, int dim, int ntypes);
void mdp_gpu_neigh_pairs_f32(float *xij, const float *x, int *aii, int *ai, int *aj, int *ti, int *tj,
                             const int *pairnum, const int *pairlist, const int *pairnumsum, const int *ilist,
                             const int *atomtype, const int *alist, int inum, int jnum, int dim);
void mdp_gpu_atom_list3d_f32(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums, int *d_incr,
                             float *x, const float *pimages, const float *wc, const float *s2rmap, int inum,
                             int pnum, int dim);
void mdp_gpu_cell_list3d_f32(int *clist, const float *xi, const float *eta1, const float *eta2,
                             const float *eta3, const float *s2rmap, const int *nc, int inum, int natom, int dim);
void mdp_gpu_full_neighbor_list3d_cells_f32(int *neighborlist, int *neighbornum, const float *x,
                                            const float *rcutsq, const int *alist, const int *clist,
                                            const int *c2alist, const int *c2anumsum, const int *nc, int inum,
                                            int jnum, int dim);
void mdp_gpu_full_neighbor_list3d_f32(int *neighborlist, int *neighbornum, const float *x, const float *rcutsq,
                                      int anum, int inum, int jnum, int dim);
void mdp_gpu_initial_integrate_f32(float *x, float *v, const float *f, const float *mass, const float *dtarray,
                                   float *tarray, float *eta_mass, float *eta, float *eta_dot,
                                   float *eta_dotdot, float *ke, float *tmp, float vlimitsq, const int *type,
                                   const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                   int mode, int dim, int inum);
void mdp_gpu_final_integrate_f32(float *x, float *v, const float *f, const float *mass, const float *dtarray,
                                 float *tarray, float *eta_mass, float *eta, float *eta_dot,
                                 float *eta_dotdot, float *ke, float *tmp, float vlimitsq, const int *type,
                                 const int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
                                 int mode, int dim, int inum);
void mdp_gpu_pbc_f32(float *x, float *v, int *image, const float *boxhi, const float *boxlo,
                     const float *hi_lambda, const float *lo_lambda, const float *h, const float *h_inv,
                     const float *h_rate, const int *pbc, int vdeform, int triclinic, int dim, int nlocal);
void mdp_gpu_compute_ke_atom_f32(float *ke, const float *mass, const float *v, float mvv2e, const int *type,
                                 const int *ilist, int dim, int inum);
void mdp_gpu_array_sum_every_column_f32(float *b, const float *a, int m, int n);

/* ---- force constraints, set-velocity integration, velocity-rescaling
 * thermostats (mdp_b200/csrc/abi_fix.cu; mdpgpucore.h:303-349).  Device arrays
 * in the reference's layouts (fix virial vatom [atom][6]); the thermostat's
 * dtarray, tarray, seed, save and second on the host, ke / tmp device scratch
 * of inum and 1 values.  Suffix _f64 for double, _f32 for float builds. ---- */
/* mdpgpucore.h:325-326, gpuFixSetForce */
void mdp_gpu_fix_set_force_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:327-328, gpuFixLineForce */
void mdp_gpu_fix_line_force_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:329-330, gpuFixPlaneForce */
void mdp_gpu_fix_plane_force_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:331-332, gpuFixAveForce */
void mdp_gpu_fix_ave_force_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:339-340, gpuFixWallReflect */
void mdp_gpu_fix_wall_reflect_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:341-342, gpuFixWallHarmonic */
void mdp_gpu_fix_wall_harmonic_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:343-344, gpuFixWallLJ93 */
void mdp_gpu_fix_wall_lj93_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:345-346, gpuFixWallLJ126 */
void mdp_gpu_fix_wall_lj126_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:347-348, gpuFixWallLJ1043 */
void mdp_gpu_fix_wall_lj1043_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:349-350, gpuFixWallMorse */
void mdp_gpu_fix_wall_morse_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:334-335, gpuFixAddForce (unwrapped positions through image and box) */
void mdp_gpu_fix_add_force_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const double *box,
                            const int *iparam, const int *ilist, const int *image, int triclinic, int eflag_atom,
                            int vflag_atom, int dim, int inum);
/* mdpgpucore.h:336-337, gpuFixDragForce */
void mdp_gpu_fix_drag_force_f64(double *x, double *v, double *f, double *eatom, double *vatom, const double *fparam, const double *box,
                             const int *iparam, const int *ilist, const int *pbc, int triclinic, int eflag_atom,
                             int vflag_atom, int dim, int inum);
/* mdpgpucore.h:303-304, gpuSetVelocityInitialIntegrate */
void mdp_gpu_set_velocity_initial_integrate_f64(double *x, double *v, const double *f, const double *mass, const double *fparam,
                                             double dtf, double dtv, const int *type, const int *ilist, const int *iparam,
                                             int dim, int inum);
/* mdpgpucore.h:306-307, gpuSetVelocityFinalIntegrate */
void mdp_gpu_set_velocity_final_integrate_f64(double *x, double *v, const double *f, const double *mass, double dtf, const int *type,
                                           const int *ilist, const int *iparam, int dim, int inum);
/* mdpgpucore.h:317-319, gpuVelocityRescalingThermostat (mode 0 Berendsen, 1 rescale, 2 CSVR); returns the
 * updated thermostat energy */
double mdp_gpu_velocity_rescaling_thermostat_f64(double *v, const double *mass, const double *dtarray, double *tarray, double *ke,
                                            double *tmp, double *second, double energy, const int *type, const int *ilist,
                                            int *seed, int *save, int biasflag, int mode, int dim, int inum);
/* mdpgpucore.h:325-326, gpuFixSetForce */
void mdp_gpu_fix_set_force_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:327-328, gpuFixLineForce */
void mdp_gpu_fix_line_force_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:329-330, gpuFixPlaneForce */
void mdp_gpu_fix_plane_force_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:331-332, gpuFixAveForce */
void mdp_gpu_fix_ave_force_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:339-340, gpuFixWallReflect */
void mdp_gpu_fix_wall_reflect_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:341-342, gpuFixWallHarmonic */
void mdp_gpu_fix_wall_harmonic_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:343-344, gpuFixWallLJ93 */
void mdp_gpu_fix_wall_lj93_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:345-346, gpuFixWallLJ126 */
void mdp_gpu_fix_wall_lj126_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:347-348, gpuFixWallLJ1043 */
void mdp_gpu_fix_wall_lj1043_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:349-350, gpuFixWallMorse */
void mdp_gpu_fix_wall_morse_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const int *iparam,
                         const int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
/* mdpgpucore.h:334-335, gpuFixAddForce (unwrapped positions through image and box) */
void mdp_gpu_fix_add_force_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const float *box,
                            const int *iparam, const int *ilist, const int *image, int triclinic, int eflag_atom,
                            int vflag_atom, int dim, int inum);
/* mdpgpucore.h:336-337, gpuFixDragForce */
void mdp_gpu_fix_drag_force_f32(float *x, float *v, float *f, float *eatom, float *vatom, const float *fparam, const float *box,
                             const int *iparam, const int *ilist, const int *pbc, int triclinic, int eflag_atom,
                             int vflag_atom, int dim, int inum);
/* mdpgpucore.h:303-304, gpuSetVelocityInitialIntegrate */
void mdp_gpu_set_velocity_initial_integrate_f32(float *x, float *v, const float *f, const float *mass, const float *fparam,
                                             float dtf, float dtv, const int *type, const int *ilist, const int *iparam,
                                             int dim, int inum);
/* mdpgpucore.h:306-307, gpuSetVelocityFinalIntegrate */
void mdp_gpu_set_velocity_final_integrate_f32(float *x, float *v, const float *f, const float *mass, float dtf, const int *type,
                                           const int *ilist, const int *iparam, int dim, int inum);
/* mdpgpucore.h:317-319, gpuVelocityRescalingThermostat (mode 0 Berendsen, 1 rescale, 2 CSVR); returns the
 * updated thermostat energy */
float mdp_gpu_velocity_rescaling_thermostat_f32(float *v, const float *mass, const float *dtarray, float *tarray, float *ke,
                                            float *tmp, float *second, float energy, const int *type, const int *ilist,
                                            int *seed, int *save, int biasflag, int mode, int dim, int inum);

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
/* gpuSnapComputeYi, per-atom beta form */
template <typename T> void gpuSnapComputeYi(T *ylist_r, T *ylist_i, T *Stotr, T *Stoti, T *cglist, T *beta,
        int *idxz, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax, int idxb_max, int idxu_max,
        int idxz_max, int nelements, int bnorm_flag, int inum);
template <> inline void gpuSnapComputeYi<double>(double *ylist_r, double *ylist_i, double *Stotr, double *Stoti,
        double *cglist, double *beta, int *idxz, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax,
        int idxb_max, int idxu_max, int idxz_max, int nelements, int bnorm_flag, int inum)
{
    mdp_gpu_snap_compute_yi_beta_f64(ylist_r, ylist_i, Stotr, Stoti, cglist, beta, idxz, idxb_block, idxu_block,
                                     idxcg_block, twojmax, idxb_max, idxu_max, idxz_max, nelements, bnorm_flag, inum);
}

/* the rest of the MD loop: prefix sums, ghosts, cells, neighbour rows,
 * integrator, wrapping, kinetic energy (replacing gpuCumsum.cu,
 * gpuNeighborList2D/3D.cu, gpuVelocityIntegration.cu, gpuDomain.cu and the
 * matching parts of gpuArrayOperations.cu / gpuComputes.cu) */
inline void gpuCumsum(int *d_out, int *d_in, int *d_sums, int *d_incr, int length)
{
    mdp_gpu_cumsum(d_out, d_in, d_sums, d_incr, length);
}
template <typename T> void gpuAtomList3D(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums,
        int *d_incr, T *x, T *pimages, T *wc, T *s2rmap, int inum, int pnum, int dim);
template <> inline void gpuAtomList3D<double>(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums,
        int *d_incr, double *x, double *pimages, double *wc, double *s2rmap, int inum, int pnum, int dim)
{
    mdp_gpu_atom_list3d_f64(alist, inside, glistnumsum, glistnum, d_sums, d_incr, x, pimages, wc, s2rmap, inum, pnum,
                            dim);
}
template <typename T> void gpuCellList3D(int *clist, T *xi, T *eta1, T *eta2, T *eta3, T *s2rmap, int *nc,
        int inum, int natom, int dim);
template <> inline void gpuCellList3D<double>(int *clist, double *xi, double *eta1, double *eta2, double *eta3,
        double *s2rmap, int *nc, int inum, int natom, int dim)
{
    mdp_gpu_cell_list3d_f64(clist, xi, eta1, eta2, eta3, s2rmap, nc, inum, natom, dim);
}
inline void gpuCell2AtomList(int *c2alist, int *c2anumsum, int *c2anum, int *clist, int *d_temp, int natom, int ncell)
{
    mdp_gpu_cell2atom_list(c2alist, c2anumsum, c2anum, clist, d_temp, natom, ncell);
}
template <typename T> void gpuFullNeighborList3D(int *neighborlist, int *neighbornum, T *x, T *rcutsq, int anum,
        int inum, int jnum, int dim);
template <> inline void gpuFullNeighborList3D<double>(int *neighborlist, int *neighbornum, double *x, double *rcutsq,
        int anum, int inum, int jnum, int dim)
{
    mdp_gpu_full_neighbor_list3d_f64(neighborlist, neighbornum, x, rcutsq, anum, inum, jnum, dim);
}
template <typename T> void gpuFullNeighborList3D(int *neighborlist, int *neighbornum, T *x, T *rcutsq, int *alist,
        int *clist, int *c2alist, int *c2anumsum, int *nc, int inum, int jnum, int dim);
template <> inline void gpuFullNeighborList3D<double>(int *neighborlist, int *neighbornum, double *x, double *rcutsq,
        int *alist, int *clist, int *c2alist, int *c2anumsum, int *nc, int inum, int jnum, int dim)
{
    mdp_gpu_full_neighbor_list3d_cells_f64(neighborlist, neighbornum, x, rcutsq, alist, clist, c2alist, c2anumsum,
                                           nc, inum, jnum, dim);
}
template <typename T> void gpuInitialIntegrate(T *x, T *v, T *f, T *mass, T *dtarray, T *tarray, T *eta_mass, T *eta,
        T *eta_dot, T *eta_dotdot, T *ke, T *tmp, T vlimitsq, int *type, int *ilist, int eta_mass_flag, int biasflag,
        int mtchain, int nc_tchain, int mode, int dim, int inum);
template <> inline void gpuInitialIntegrate<double>(double *x, double *v, double *f, double *mass, double *dtarray,
        double *tarray, double *eta_mass, double *eta, double *eta_dot, double *eta_dotdot, double *ke, double *tmp,
        double vlimitsq, int *type, int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
        int mode, int dim, int inum)
{
    mdp_gpu_initial_integrate_f64(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp,
                                  vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}
template <typename T> void gpuFinalIntegrate(T *x, T *v, T *f, T *mass, T *dtarray, T *tarray, T *eta_mass, T *eta,
        T *eta_dot, T *eta_dotdot, T *ke, T *tmp, T vlimitsq, int *type, int *ilist, int eta_mass_flag, int biasflag,
        int mtchain, int nc_tchain, int mode, int dim, int inum);
template <> inline void gpuFinalIntegrate<double>(double *x, double *v, double *f, double *mass, double *dtarray,
        double *tarray, double *eta_mass, double *eta, double *eta_dot, double *eta_dotdot, double *ke, double *tmp,
        double vlimitsq, int *type, int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
        int mode, int dim, int inum)
{
    mdp_gpu_final_integrate_f64(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp,
                                vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}
template <typename T> void gpuPBC(T *x, T *v, int *image, T *boxhi, T *boxlo, T *hi_lambda, T *lo_lambda, T *h,
        T *h_inv, T *h_rate, int *pbc, int vdeform, int triclinic, int dim, int nlocal);
template <> inline void gpuPBC<double>(double *x, double *v, int *image, double *boxhi, double *boxlo,
        double *hi_lambda, double *lo_lambda, double *h, double *h_inv, double *h_rate, int *pbc, int vdeform,
        int triclinic, int dim, int nlocal)
{
    mdp_gpu_pbc_f64(x, v, image, boxhi, boxlo, hi_lambda, lo_lambda, h, h_inv, h_rate, pbc, vdeform, triclinic, dim,
                    nlocal);
}
template <typename T> void gpuComputeKEAtom(T *ke, T *mass, T *v, T mvv2e, int *type, int *ilist, int dim, int inum);
template <> inline void gpuComputeKEAtom<double>(double *ke, double *mass, double *v, double mvv2e, int *type,
        int *ilist, int dim, int inum)
{
    mdp_gpu_compute_ke_atom_f64(ke, mass, v, mvv2e, type, ilist, dim, inum);
}
template <typename T> void gpuArraySumEveryColumn(T *b, T *a, int m, int n);
template <> inline void gpuArraySumEveryColumn<double>(double *b, double *a, int m, int n)
{
    mdp_gpu_array_sum_every_column_f64(b, a, m, n);
}
template <typename T> T gpuArrayGetValueAtIndex(T *y, int n);
template <> inline int gpuArrayGetValueAtIndex<int>(int *y, int n) { return mdp_gpu_array_get_value_at_index_int(y, n); }
/* float (PREC_FLOAT) instantiations */
template <> inline void gpuSnapComputeUi<float>(float *Stotr, float *Stoti, float *rootpqarray, float *rij,
        float *wjelem, float *radelem, float rmin0, float rfac0, float rcutfac, int *idxu_block, int *map,
        int *ai, int *ti, int *tj, int twojmax, int idxu_max, int inum, int ijnum, int switchflag, int chemflag)
{
    mdp_gpu_snap_compute_ui_f32(Stotr, Stoti, rootpqarray, rij, wjelem, radelem, rmin0, rfac0, rcutfac, idxu_block,
                                map, ai, ti, tj, twojmax, idxu_max, inum, ijnum, switchflag, chemflag);
}
template <> inline void gpuAddWself2Ui<float>(float *Stotr, float *Stoti, float wself, int *idxu_block,
        int *type, int *map, int *ai, int wselfall_flag, int chemflag, int idxu_max, int nelements, int twojmax,
        int inum)
{
    mdp_gpu_add_wself2ui_f32(Stotr, Stoti, wself, idxu_block, type, map, ai, wselfall_flag, chemflag, idxu_max,
                             nelements, twojmax, inum);
}
template <> inline void gpuSnapComputeEi<float>(float *eatom, float *Stotr, float *Stoti, float *cglist,
        float *bzero, float *coeffelem, int *ilist, int *map, int *type, int *idxb, int *idxcg_block,
        int *idxu_block, int twojmax, int idxb_max, int idxu_max, int nelements, int ncoeffall, int bnorm_flag,
        int bzero_flag, int wselfall_flag, int quadraticflag, int inum)
{
    mdp_gpu_snap_compute_ei_f32(eatom, Stotr, Stoti, cglist, bzero, coeffelem, ilist, map, type, idxb, idxcg_block,
                                idxu_block, twojmax, idxb_max, idxu_max, nelements, ncoeffall, bnorm_flag,
                                bzero_flag, wselfall_flag, quadraticflag, inum);
}
template <> inline void gpuSnapComputeBi<float>(float *blist, float *Stotr, float *Stoti, float *cglist,
        float *bzero, int *idxb, int *idxcg_block, int *idxu_block, int *idxz_block, int twojmax, int idxb_max,
        int idxu_max, int idxz_max, int nelements, int bnorm_flag, int bzero_flag, int wselfall_flag, int inum)
{
    mdp_gpu_snap_compute_bi_f32(blist, Stotr, Stoti, cglist, bzero, idxb, idxcg_block, idxu_block, idxz_block,
                                twojmax, idxb_max, idxu_max, idxz_max, nelements, bnorm_flag, bzero_flag,
                                wselfall_flag, inum);
}
template <> inline void gpuSnapComputeYi<float>(float *ylist_r, float *ylist_i, float *Stotr, float *Stoti,
        float *cglist, float *coeffelem, int *map, int *type, int *idxz, int *idxb_block, int *idxu_block,
        int *idxcg_block, int twojmax, int idxb_max, int idxu_max, int idxz_max, int nelements, int ncoeffall,
        int bnorm_flag, int inum)
{
    mdp_gpu_snap_compute_yi_f32(ylist_r, ylist_i, Stotr, Stoti, cglist, coeffelem, map, type, idxz, idxb_block,
                                idxu_block, idxcg_block, twojmax, idxb_max, idxu_max, idxz_max, nelements,
                                ncoeffall, bnorm_flag, inum);
}
template <> inline void gpuSnapComputeFi<float>(float *fatom, float *vatom, float *ylist_r, float *ylist_i,
        float *rootpqarray, float *rij, float *wjelem, float *radelem, float rmin0, float rfac0,
        float rcutfac, int *idxu_block, int *map, int *aii, int *ai, int *aj, int *ti, int *tj, int twojmax,
        int idxu_max, int inum, int anum, int ijnum, int switchflag, int chemflag)
{
    mdp_gpu_snap_compute_fi_f32(fatom, vatom, ylist_r, ylist_i, rootpqarray, rij, wjelem, radelem, rmin0, rfac0,
                                rcutfac, idxu_block, map, aii, ai, aj, ti, tj, twojmax, idxu_max, inum, anum, ijnum,
                                switchflag, chemflag);
}
template <> inline void gpuNeighPairList<float>(int *pairnum, int *pairlist, float *x, float *rcutsq, int *ilist,
        int *neighlist, int *neighnum, int *atomtype, int *alist, int inum, int jnum, int dim, int ntypes)
{
    mdp_gpu_neigh_pair_list_f32(pairnum, pairlist, x, rcutsq, ilist, neighlist, neighnum, atomtype, alist, inum,
                                jnum, dim, ntypes);
}
template <> inline void gpuNeighPairs<float>(float *xij, float *x, int *aii, int *ai, int *aj, int *ti, int *tj,
        int *pairnum, int *pairlist, int *pairnumsum, int *ilist, int *atomtype, int *alist, int inum, int jnum,
        int dim)
{
    mdp_gpu_neigh_pairs_f32(xij, x, aii, ai, aj, ti, tj, pairnum, pairlist, pairnumsum, ilist, atomtype, alist, inum,
                            jnum, dim);
}
template <> inline void gpuSnapComputeYi<float>(float *ylist_r, float *ylist_i, float *Stotr, float *Stoti,
        float *cglist, float *beta, int *idxz, int *idxb_block, int *idxu_block, int *idxcg_block, int twojmax,
        int idxb_max, int idxu_max, int idxz_max, int nelements, int bnorm_flag, int inum)
{
    mdp_gpu_snap_compute_yi_beta_f32(ylist_r, ylist_i, Stotr, Stoti, cglist, beta, idxz, idxb_block, idxu_block,
                                     idxcg_block, twojmax, idxb_max, idxu_max, idxz_max, nelements, bnorm_flag, inum);
}
template <> inline void gpuAtomList3D<float>(int *alist, int *inside, int *glistnumsum, int *glistnum, int *d_sums,
        int *d_incr, float *x, float *pimages, float *wc, float *s2rmap, int inum, int pnum, int dim)
{
    mdp_gpu_atom_list3d_f32(alist, inside, glistnumsum, glistnum, d_sums, d_incr, x, pimages, wc, s2rmap, inum, pnum,
                            dim);
}
template <> inline void gpuCellList3D<float>(int *clist, float *xi, float *eta1, float *eta2, float *eta3,
        float *s2rmap, int *nc, int inum, int natom, int dim)
{
    mdp_gpu_cell_list3d_f32(clist, xi, eta1, eta2, eta3, s2rmap, nc, inum, natom, dim);
}
template <> inline void gpuFullNeighborList3D<float>(int *neighborlist, int *neighbornum, float *x, float *rcutsq,
        int anum, int inum, int jnum, int dim)
{
    mdp_gpu_full_neighbor_list3d_f32(neighborlist, neighbornum, x, rcutsq, anum, inum, jnum, dim);
}
template <> inline void gpuFullNeighborList3D<float>(int *neighborlist, int *neighbornum, float *x, float *rcutsq,
        int *alist, int *clist, int *c2alist, int *c2anumsum, int *nc, int inum, int jnum, int dim)
{
    mdp_gpu_full_neighbor_list3d_cells_f32(neighborlist, neighbornum, x, rcutsq, alist, clist, c2alist, c2anumsum,
                                           nc, inum, jnum, dim);
}
template <> inline void gpuInitialIntegrate<float>(float *x, float *v, float *f, float *mass, float *dtarray,
        float *tarray, float *eta_mass, float *eta, float *eta_dot, float *eta_dotdot, float *ke, float *tmp,
        float vlimitsq, int *type, int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
        int mode, int dim, int inum)
{
    mdp_gpu_initial_integrate_f32(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp,
                                  vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}
template <> inline void gpuFinalIntegrate<float>(float *x, float *v, float *f, float *mass, float *dtarray,
        float *tarray, float *eta_mass, float *eta, float *eta_dot, float *eta_dotdot, float *ke, float *tmp,
        float vlimitsq, int *type, int *ilist, int eta_mass_flag, int biasflag, int mtchain, int nc_tchain,
        int mode, int dim, int inum)
{
    mdp_gpu_final_integrate_f32(x, v, f, mass, dtarray, tarray, eta_mass, eta, eta_dot, eta_dotdot, ke, tmp,
                                vlimitsq, type, ilist, eta_mass_flag, biasflag, mtchain, nc_tchain, mode, dim, inum);
}
template <> inline void gpuPBC<float>(float *x, float *v, int *image, float *boxhi, float *boxlo,
        float *hi_lambda, float *lo_lambda, float *h, float *h_inv, float *h_rate, int *pbc, int vdeform,
        int triclinic, int dim, int nlocal)
{
    mdp_gpu_pbc_f32(x, v, image, boxhi, boxlo, hi_lambda, lo_lambda, h, h_inv, h_rate, pbc, vdeform, triclinic, dim,
                    nlocal);
}
template <> inline void gpuComputeKEAtom<float>(float *ke, float *mass, float *v, float mvv2e, int *type,
        int *ilist, int dim, int inum)
{
    mdp_gpu_compute_ke_atom_f32(ke, mass, v, mvv2e, type, ilist, dim, inum);
}
template <> inline void gpuArraySumEveryColumn<float>(float *b, float *a, int m, int n)
{
    mdp_gpu_array_sum_every_column_f32(b, a, m, n);
}
/* force constraints, set-velocity integration, velocity-rescaling thermostats */
template <typename T> void gpuFixSetForce(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixLineForce(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixPlaneForce(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixAveForce(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixWallReflect(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixWallHarmonic(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixWallLJ93(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixWallLJ126(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixWallLJ1043(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixWallMorse(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixAddForce(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, T *box, int *iparam, int *ilist, int *image, int triclinic, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuFixDragForce(T *x, T *v, T *f, T *eatom, T *vatom, T *fparam, T *box, int *iparam, int *ilist, int *pbc, int triclinic, int eflag_atom, int vflag_atom, int dim, int inum);
template <typename T> void gpuSetVelocityInitialIntegrate(T *x, T *v, T *f, T *mass, T *fparam, T dtf, T dtv, int *type, int *ilist, int *iparam, int dim, int inum);
template <typename T> void gpuSetVelocityFinalIntegrate(T *x, T *v, T *f, T *mass, T dtf, int *type, int *ilist, int *iparam, int dim, int inum);
template <typename T> T gpuVelocityRescalingThermostat(T *v, T *mass, T *dtarray, T *tarray, T *ke, T *tmp, T *second, T energy, int *type, int *ilist, int *seed, int *save, int biasflag, int mode, int dim, int inum);
template <> inline void gpuFixSetForce<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_set_force_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixLineForce<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_line_force_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixPlaneForce<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_plane_force_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixAveForce<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_ave_force_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallReflect<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_reflect_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallHarmonic<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_harmonic_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallLJ93<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_lj93_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallLJ126<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_lj126_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallLJ1043<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_lj1043_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallMorse<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_morse_f64(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixAddForce<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        double *box, int *iparam, int *ilist, int *image, int triclinic, int eflag_atom, int vflag_atom, int dim,
        int inum)
{
    mdp_gpu_fix_add_force_f64(x, v, f, eatom, vatom, fparam, box, iparam, ilist, image, triclinic, eflag_atom,
                           vflag_atom, dim, inum);
}
template <> inline void gpuFixDragForce<double>(double *x, double *v, double *f, double *eatom, double *vatom, double *fparam,
        double *box, int *iparam, int *ilist, int *pbc, int triclinic, int eflag_atom, int vflag_atom, int dim,
        int inum)
{
    mdp_gpu_fix_drag_force_f64(x, v, f, eatom, vatom, fparam, box, iparam, ilist, pbc, triclinic, eflag_atom,
                            vflag_atom, dim, inum);
}
template <> inline void gpuSetVelocityInitialIntegrate<double>(double *x, double *v, double *f, double *mass, double *fparam,
        double dtf, double dtv, int *type, int *ilist, int *iparam, int dim, int inum)
{
    mdp_gpu_set_velocity_initial_integrate_f64(x, v, f, mass, fparam, dtf, dtv, type, ilist, iparam, dim, inum);
}
template <> inline void gpuSetVelocityFinalIntegrate<double>(double *x, double *v, double *f, double *mass, double dtf, int *type,
        int *ilist, int *iparam, int dim, int inum)
{
    mdp_gpu_set_velocity_final_integrate_f64(x, v, f, mass, dtf, type, ilist, iparam, dim, inum);
}
template <> inline double gpuVelocityRescalingThermostat<double>(double *v, double *mass, double *dtarray, double *tarray, double *ke,
        double *tmp, double *second, double energy, int *type, int *ilist, int *seed, int *save, int biasflag, int mode,
        int dim, int inum)
{
    return mdp_gpu_velocity_rescaling_thermostat_f64(v, mass, dtarray, tarray, ke, tmp, second, energy, type, ilist,
                                                    seed, save, biasflag, mode, dim, inum);
}
template <> inline void gpuFixSetForce<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_set_force_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixLineForce<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_line_force_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixPlaneForce<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_plane_force_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixAveForce<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_ave_force_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallReflect<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_reflect_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallHarmonic<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_harmonic_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallLJ93<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_lj93_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallLJ126<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_lj126_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallLJ1043<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_lj1043_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixWallMorse<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        int *iparam, int *ilist, int eflag_atom, int vflag_atom, int dim, int inum)
{
    mdp_gpu_fix_wall_morse_f32(x, v, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom, dim, inum);
}
template <> inline void gpuFixAddForce<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        float *box, int *iparam, int *ilist, int *image, int triclinic, int eflag_atom, int vflag_atom, int dim,
        int inum)
{
    mdp_gpu_fix_add_force_f32(x, v, f, eatom, vatom, fparam, box, iparam, ilist, image, triclinic, eflag_atom,
                           vflag_atom, dim, inum);
}
template <> inline void gpuFixDragForce<float>(float *x, float *v, float *f, float *eatom, float *vatom, float *fparam,
        float *box, int *iparam, int *ilist, int *pbc, int triclinic, int eflag_atom, int vflag_atom, int dim,
        int inum)
{
    mdp_gpu_fix_drag_force_f32(x, v, f, eatom, vatom, fparam, box, iparam, ilist, pbc, triclinic, eflag_atom,
                            vflag_atom, dim, inum);
}
template <> inline void gpuSetVelocityInitialIntegrate<float>(float *x, float *v, float *f, float *mass, float *fparam,
        float dtf, float dtv, int *type, int *ilist, int *iparam, int dim, int inum)
{
    mdp_gpu_set_velocity_initial_integrate_f32(x, v, f, mass, fparam, dtf, dtv, type, ilist, iparam, dim, inum);
}
template <> inline void gpuSetVelocityFinalIntegrate<float>(float *x, float *v, float *f, float *mass, float dtf, int *type,
        int *ilist, int *iparam, int dim, int inum)
{
    mdp_gpu_set_velocity_final_integrate_f32(x, v, f, mass, dtf, type, ilist, iparam, dim, inum);
}
template <> inline float gpuVelocityRescalingThermostat<float>(float *v, float *mass, float *dtarray, float *tarray, float *ke,
        float *tmp, float *second, float energy, int *type, int *ilist, int *seed, int *save, int biasflag, int mode,
        int dim, int inum)
{
    return mdp_gpu_velocity_rescaling_thermostat_f32(v, mass, dtarray, tarray, ke, tmp, second, energy, type, ilist,
                                                    seed, save, biasflag, mode, dim, inum);
}
#endif /* MDP_B200_GPUCORE_TEMPLATES */
#endif /* __cplusplus */
#endif
