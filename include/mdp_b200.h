/*
 * mdp_b200 -- B200-native SNAP force path and velocity-Verlet MD (C ABI).
 *
 * All entry points return 0 on success and -1 on error; mdp_last_error()
 * returns the text of the last error of the calling thread.  No entry point
 * exits or aborts the process.
 *
 * This header is the project's own engine interface.  The drop-in
 * replacements for MDP's existing interfaces are declared in
 *   include/mdp_b200_cpusnap.h   (MDP's Julia ccall library, cpuSnap.h)
 *   include/mdp_b200_gpucore.h   (MDP's backend dispatch, mdpgpucore.h)
 */
#ifndef MDP_B200_H
#define MDP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* SNAP hyper-parameters and coefficients: the snaparam[12] vector of MDP
 * (src/Julia/Preprocessing/Preprocessing.jl:266, read at
 * src/C++/Descriptors/snappotential.cpp:151-162) with its per-element arrays. */
typedef struct {
    int twojmax;          /* 2J: 4, 6 or 8 */
    double rcutfac;
    double rfac0;
    double rmin0;
    double radelem;       /* element radius; rcut = 2 * radelem * rcutfac */
    double wjelem;        /* element weight */
    int switchflag;
    int bzeroflag;
    int bnormflag;
    int wselfallflag;
    int quadraticflag;    /* 1: quadratic SNAP (one element, FP64) */
    int chemflag;         /* 1: element-resolved bispectrum (several elements) */
    int ncoeffall;        /* coefficients per element: 1 + ncoeff (+ ncoeff (ncoeff + 1) / 2 quadratic) */
    const double *coeff;  /* nelements x ncoeffall values; coeff[e * ncoeffall] = beta_0 of element e */
    /* Several element types (InitSnap, snappotential.cpp:146-232): atoms carry
     * types 1..nelements; per-element radii and weights; ncoeff is the number
     * of bispectrum components times nelements^3 with chemflag.  nelements 0
     * or 1 with radelems == NULL: the single element of radelem / wjelem.
     * Several elements run in FP64, linear SNAP, nelements <= 4. */
    int nelements;
    const double *radelems;
    const double *wjelems;
} mdp_snap_params;

enum { MDP_PREC_FP64 = 0, MDP_PREC_FP32 = 1 };

const char *mdp_last_error(void);

/* number of bispectrum components for 2J (MDP idxbcount, cpuSnap.cpp:23) */
int mdp_snap_ncoeff(int twojmax);

/* ---------------------------------------------------------------------------
 * One SNAP force evaluation on DEVICE arrays (replaces the body of
 * ComputePairSnap3, src/C++/Descriptors/snappotential.cpp:634-760).
 *   x        anum x 3 positions, AoS (locals first, then ghosts)
 *   alist    anum owner index of every atom (identity for locals)
 *   neighlist inum x neighmax rows, neighnum[inum]
 *   eatom    inum, fatom inum x 3 AoS, vatom 6 x inum SoA (may be NULL)
 * Outputs are overwritten (the reference accumulates into zeroed arrays).
 * ------------------------------------------------------------------------- */
int mdp_snap_compute_device(const mdp_snap_params *p, int precision, const double *x, const int *alist,
                            const int *neighlist, const int *neighnum, int inum, int anum, int neighmax,
                            double *eatom, double *fatom, double *vatom, void *cuda_stream);

/* Same with the atom types (1..nelements) of the inum owners, on the device;
 * required by models with several element types. */
int mdp_snap_compute_device_typed(const mdp_snap_params *p, int precision, const double *x, const int *atomtype,
                                  const int *alist, const int *neighlist, const int *neighnum, int inum, int anum,
                                  int neighmax, double *eatom, double *fatom, double *vatom, void *cuda_stream);

/* Same on HOST arrays, including the ghost/neighbour build: natoms positions
 * in an orthogonal or triclinic periodic box with vectors a, b, c (box[0..8]).
 * Optional outputs (NULL to skip): neighlist (natoms x neighmax), neighnum,
 * anum_out, alist_out (capacity alist_cap), xall_out (3 x alist_cap). */
int mdp_snap_compute_host(const mdp_snap_params *p, int precision, int natoms, const double *x,
                          const double *box, double skin, int neighmax, double *eatom, double *fatom,
                          double *vatom, int *neighlist, int *neighnum, int *anum_out, int *alist_out,
                          double *xall_out, int alist_cap);
/* Same with the natoms atom types (1..nelements) on the host. */
int mdp_snap_compute_host_typed(const mdp_snap_params *p, int precision, int natoms, const double *x,
                                const int *atomtype, const double *box, double skin, int neighmax, double *eatom,
                                double *fatom, double *vatom, int *neighlist, int *neighnum, int *anum_out,
                                int *alist_out, double *xall_out, int alist_cap);

/* ---------------------------------------------------------------------------
 * MD engine: NVE velocity Verlet with SNAP forces, neighbour list rebuilt on
 * the reference's criterion (src/C++/Integration/Integration.cpp:260-303).
 * ------------------------------------------------------------------------- */
typedef struct mdp_md mdp_md;

typedef struct {
    int natoms;
    double box[9];        /* a, b, c */
    double mass;          /* amu */
    double dt;            /* ps */
    double skin;          /* A */
    int neighmax;
    int neighevery;       /* rebuild check every n steps (reference default 1) */
    int neighdelay;       /* no check before this many steps (reference default 0) */
    int neighcheck;       /* 1: rebuild when max displacement > skin/2 */
    int precision;        /* MDP_PREC_FP64 or MDP_PREC_FP32 */
    int device;
} mdp_md_config;

int mdp_md_create(mdp_md **h, const mdp_snap_params *p, const mdp_md_config *cfg);
void mdp_md_destroy(mdp_md *h);
/* host positions/velocities (natoms x 3, A and A/ps) */
int mdp_md_set_state(mdp_md *h, const double *x, const double *v);
/* device positions/velocities already resident (natoms x 3 AoS) */
int mdp_md_set_state_device(mdp_md *h, const double *x_dev, const double *v_dev);
/* atom types 1..nelements (host, natoms), required before setup by models
 * with several element types; the mass stays the configuration's one */
int mdp_md_set_types(mdp_md *h, const int *types);
/* neighbour list + first force + thermo (IntegrationSetup, Integration.cpp:158) */
int mdp_md_setup(mdp_md *h);
/* nsteps velocity-Verlet steps; thermo rows (step, T, PE/atom, TE/atom, P)
 * every thermo_every steps into thermo (may be NULL); returns rows written
 * via *nrows.  elapsed_ms (may be NULL): CUDA-event time of the steps on the
 * engine's stream. */
int mdp_md_run(mdp_md *h, int nsteps, int thermo_every, double *thermo, int thermo_cap, int *nrows,
               float *elapsed_ms);
int mdp_md_get_state(mdp_md *h, double *x, double *v, double *f, double *eatom);
/* Asynchronous state upload / result download on the engine's stream, for
 * callers that keep the state on the host between steps (pinned host memory
 * makes the copies truly asynchronous).  The uploaded positions must be ones
 * this engine produced (the neighbour list is kept).  mdp_md_sync waits. */
int mdp_md_upload(mdp_md *h, const double *x, const double *v);
int mdp_md_download(mdp_md *h, double *f, double *eatom);
int mdp_md_sync(mdp_md *h);
/* number of kernels this library has launched so far (all handles) */
long long mdp_launch_count(void);
int mdp_md_thermo(mdp_md *h, double *out5);
/* counters: [0] steps, [1] neighbour rebuilds, [2] current pairs, [3] ghosts,
 * [4] neighbour entries */
int mdp_md_counters(mdp_md *h, long long *out5);
/* per-stage CUDA-event timing over the next runs: 1 on, 0 off; read back as
 * ms totals [pairs, ui, yi, fi, tally, force] and the number of force calls */
int mdp_md_stage_timing(mdp_md *h, int enable);
int mdp_md_stage_times(mdp_md *h, double *ms6, long long *calls);
/* the CUDA stream the engine launches on (for callers that time with events) */
void *mdp_md_stream(mdp_md *h);

/* measured FP64 / FP32 FMA throughput of this GPU (TFLOP/s), from a
 * register-resident FMA loop timed with CUDA events */
int mdp_probe_fma_peak(int device, double *fp64_tflops, double *fp32_tflops);

/* ---------------------------------------------------------------------------
 * Learned surrogate (no counterpart in MDP): an MLP 14 -> 64 -> 64 -> 1 (SiLU)
 * on the per-atom 2J=4 bispectrum stands in for the per-atom SNAP energy.
 * Parameters: mdp_sur_nparams() floats, laid out W1 [64][16] (features padded
 * to 16), b1 [64], W2 [64][64] (W2[out][in]), b2 [64], w3 [64], b3.
 * Normalisation (2*14+2 floats): feature means, feature 1/std, energy mean,
 * energy std.  Forward passes use the weights rounded to BF16.
 * ------------------------------------------------------------------------- */
typedef struct mdp_sur mdp_sur;

/* p4: SNAP hyper-parameters of the features (twojmax 4; coefficients unused) */
int mdp_sur_create(mdp_sur **h, const mdp_snap_params *p4, int device);
void mdp_sur_destroy(mdp_sur *h);
int mdp_sur_nparams(void);
int mdp_sur_set_params(mdp_sur *h, const float *params, const float *norm /* may be NULL */);
int mdp_sur_get_params(mdp_sur *h, float *params, float *norm);
/* training set on the device: rows of 16 floats (14 features + 2 zeros) and a
 * per-atom target energy */
int mdp_sur_dataset_reserve(mdp_sur *h, long rows);
long mdp_sur_dataset_size(mdp_sur *h);
int mdp_sur_dataset_add(mdp_sur *h, const double *B_dev, long bstride, const double *e_dev, int n, void *stream);
int mdp_sur_dataset_load(mdp_sur *h, const float *X, const float *E, long nrows);
int mdp_sur_dataset_copy(mdp_sur *h, float *X, float *E, long row0, long nrows);
/* feature/energy mean and spread of the dataset become the normalisation */
int mdp_sur_fit_normalization(mdp_sur *h);
/* steps Adam updates on random minibatches of batch rows (loss per step out) */
int mdp_sur_train(mdp_sur *h, int steps, int batch, float lr, unsigned long long seed, float *loss);
/* gradient of the mean squared normalised-energy error over host rows, no update */
int mdp_sur_grad(mdp_sur *h, const float *X, const float *E, int n, float *grad, float *loss);
/* inference on host features B [k * n + atom]: E [n], G = dE_i/dB_ik [k * n + atom] */
int mdp_sur_eval(mdp_sur *h, const double *B, int n, double *E, float *G);

/* force-matching set from a 2J=4 batch (mdp_fit, declared below) whose
 * configurations are equal-size snapshots of per atoms: the plain model's
 * forces (3 per atom) and per-atom energies, host arrays */
typedef struct mdp_fit mdp_fit;
int mdp_sur_force_set(mdp_sur *h, mdp_fit *snapshots, const double *forces, const double *energies, int per);
long long mdp_sur_force_set_npairs(mdp_sur *h);
/* Adam on windows of snaps_per_batch snapshots: energy loss (as
 * mdp_sur_train) + alpha * force MSE / var(F); per-step losses out */
int mdp_sur_train_forces(mdp_sur *h, int steps, int snaps_per_batch, float lr, float alpha, unsigned long long seed,
                         float *loss_e, float *loss_f);
/* gradient of that loss over snapshots [snap0, snap0 + snaps) (no update);
 * losses[2] = (energy, force) parts */
int mdp_sur_force_grad(mdp_sur *h, int snap0, int snaps, float alpha, float *grad, float *losses);
/* the force set's features B [k][atom], per-pair dB/dR [pair][3][14], pair
 * (centre, neighbour) and CSR offsets, for checks */
int mdp_sur_force_set_copy(mdp_sur *h, double *B, float *db, int *pinfo, int *poff);

/* append the MD engine's current state to the training set: 2J=4 features of
 * the current positions and the per-atom energies of the last force call */
int mdp_md_sur_sample(mdp_md *md, mdp_sur *s);
/* per-atom 2J=4 features of the engine's current positions, B [k * natoms + atom] */
int mdp_md_sur_features(mdp_md *md, mdp_sur *s, double *B_host);
/* forces from the surrogate (s != NULL) or the plain SNAP model (s == NULL).
 * Every judge_every steps (and at setup) the plain model is evaluated on the
 * same positions; its forces replace the surrogate's for that step and, when
 * the force RMSE (over the 3N components) exceeds tol, the engine falls back
 * to the plain model for the rest of its life. */
/* ZBL pair term added to SNAP, as MDP's snapTA06A example pairs them
 * (simulating/snap/snapTA06A.jl:62-69, potential simulating/snap/ZBLpotential.jl,
 * tallied as src/C++/Potentials/cpuPotentials.cpp:1587-1650 does for full
 * neighbour lists): screened Coulomb for nuclear charge z between all atom
 * pairs closer than `outer`, switched to zero between `inner` and `outer`.
 * z <= 0 turns it off.  `outer` must not exceed the SNAP cutoff + skin.
 * Call mdp_md_setup afterwards. */
int mdp_md_set_zbl(mdp_md *md, double inner, double outer, double z);
int mdp_md_set_surrogate(mdp_md *md, mdp_sur *s, int judge_every, double tol);
/* active (1 while the surrogate drives), fallback step (-1: none), number of
 * judgements, and up to cap (step, rmse) pairs */
int mdp_md_surrogate_status(mdp_md *md, int *active, long long *fallback_step, int *njudge, double *log, int cap);

/* ---------------------------------------------------------------------------
 * Batched descriptors and linear-fit normal equations (ComputeSnap,
 * snappotential.cpp:762-910, per configuration; assembly as Regression.cpp:
 * 386-404).  A batch holds configurations of any atom counts, each in an
 * orthogonal periodic box whose lengths exceed the cutoff.
 * ------------------------------------------------------------------------- */
/* p: SNAP hyper-parameters (twojmax 4, 6 or 8; coefficients unused) */
int mdp_fit_create(mdp_fit **h, const mdp_snap_params *p, int device);
void mdp_fit_destroy(mdp_fit *h);
int mdp_fit_ncoeff(mdp_fit *h);
/* natoms[c], box[3c..3c+2], x (3 per atom, all configurations concatenated);
 * targets e[c], f (3 per atom) and weights we[c], wf[c] may be NULL */
int mdp_fit_set_batch(mdp_fit *h, int nconf, const int *natoms, const double *box, const double *x,
                      const double *e, const double *f, const double *we, const double *wf);
/* the same for general (triclinic) periodic cells: lattice[9c..9c+8] holds the
 * cell vectors a, b, c of configuration c as rows, and x lies inside the cell;
 * every perpendicular cell width must exceed the cutoff.  Serves the real-data
 * fits of MDP's fitting/snap/Ta/fitsnap.jl:107-159, whose configurations
 * (readJSON.jl "Lattice") are sheared and surface cells. */
int mdp_fit_set_batch_lattice(mdp_fit *h, int nconf, const int *natoms, const double *lattice, const double *x,
                              const double *e, const double *f, const double *we, const double *wf);
/* ZBL reference potential (inner, outer radii, atomic number z) of every atom
 * of the current batch, into host arrays: eatom[natoms], fatom[3 natoms],
 * vatom[6][natoms] (xx, yy, zz, xy, xz, yz).  The fit of MDP's
 * fitting/snap/Ta/fitsnap.jl:81 subtracts this pair term from the targets
 * (emldescriptors.jl:199-259). */
int mdp_fit_zbl(mdp_fit *h, double inner, double outer, double z, double *eatom, double *fatom, double *vatom);
long long mdp_fit_npairs(mdp_fit *h);
/* scratch budget of the chunked stages (default 24e9 bytes; the batch is
 * processed in configuration-aligned chunks that fit it) and the chunk count */
int mdp_fit_set_chunk_bytes(mdp_fit *h, double bytes);
int mdp_fit_nchunks(mdp_fit *h);
/* bi [nconf][ncoeff]; bd [atom][3][ncoeff] with the reference's sign
 * (cpuSnapTallyBispectrumDeriv: -d(sum_i B_i)/dx); bv [nconf][ncoeff][6];
 * blist [ncoeff][atom].  Any output may be NULL. */
int mdp_fit_descriptors(mdp_fit *h, double *bi, double *bd, double *bv, double *blist);
/* A [64][64], b [64] of the normal equations over the whole batch: rows
 * we*(N, bi) -> we*E per configuration and wf*(0, d(sum B)/dx_ic) -> -wf*f_ic
 * per force component; mode 0 FP64, mode 1 BF16 hi/lo split with FP32 sums on
 * tensor cores.  One CUDA graph per mode, captured once and replayed. */
int mdp_fit_run(mdp_fit *h, int mode, double *A, double *b, float *elapsed_ms);
/* time candidate launch shapes on the current batch and keep the fastest;
 * out3 (may be NULL): du threads, dB/dR threads, Gram rows per CTA */
int mdp_fit_tune(mdp_fit *h, int *out3);

#ifdef __cplusplus
}
#endif
#endif
