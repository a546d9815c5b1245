// Learned surrogate (MLP on 2J=4 bispectra): device state and internal entry
// points shared by surrogate.cu and the MD engine.
#pragma once

#include "engine.h"

namespace mdp {

constexpr int SUR_NK = 14;   // features: the 2J=4 bispectrum components
constexpr int SUR_KP = 16;   // features padded to 16 in the first weight matrix
constexpr int SUR_H = 64;    // hidden units per layer
// parameter block: W1 [H][KP], b1 [H], W2 [H][H] (W2[c][r]: output c, input r), b2 [H], w3 [H], b3
constexpr int SUR_OFF_W1 = 0;
constexpr int SUR_OFF_B1 = SUR_OFF_W1 + SUR_H * SUR_KP;
constexpr int SUR_OFF_W2 = SUR_OFF_B1 + SUR_H;
constexpr int SUR_OFF_B2 = SUR_OFF_W2 + SUR_H * SUR_H;
constexpr int SUR_OFF_W3 = SUR_OFF_B2 + SUR_H;
constexpr int SUR_OFF_B3 = SUR_OFF_W3 + SUR_H;
constexpr int SUR_NPAR = SUR_OFF_B3 + 1;

// x = (B - mu) * sinv; E = e_mu + e_sd * y
struct SurNorm {
    float mu[SUR_KP], sinv[SUR_KP];
    float e_mu, e_sd;
};

struct Surrogate {
    SnapModel model;                // 2J=4 feature model (coefficients 1: multiplicity factors in betaY)
    DevBuf P, Pb, grad, m1, m2;     // master weights, BF16-rounded copy, gradient, Adam moments
    DevBuf X, E, idx, scal;         // dataset rows [row][KP] and energies, minibatch rows, scratch
    DevBuf B, G;                    // per-atom features [k][atom] (double) and dE_i/dB_ik [k][atom]
    ForcePath fp;
    SurNorm norm;
    long rows = 0, cap = 0;
    long long adam_t = 0;
    bool trained = false;
    int device = 0;
    // force-training set: equal-size snapshots, per-pair dB/dR at 2J=4
    DevBuf fB, fE, fF, fdb, fpinfo, fpoff, froff, frlist, fG, fQ, fV, fscal;
    long f_atoms = 0, f_pairs = 0;
    int f_snaps = 0, f_per = 0;
    double f_var = 1.0;   // variance of the reference force components
};

// 2J=4 bispectrum of every local atom into S.B (pairs, U and B on fp)
int sur_features(Surrogate &S, ForcePath &fp, const double4 *x, int inum, const int *nlist, const int *nnum, int nm,
                 cudaStream_t s);
// surrogate energy / force / virial (same outputs as force_compute)
int sur_force(Surrogate &S, ForcePath &fp, const double4 *x, int inum, const int *nlist, const int *nnum, int nm,
              const int *roff, const long long *rlist, double *eatom, double4 *f, double *vatom, cudaStream_t s);
// sum over atoms of |a - b|^2 into *host_out (synchronises the stream)
int force_sq_diff(const double4 *a, const double4 *b, int n, double *dev_acc, double *host_out, cudaStream_t s);

}  // namespace mdp

// the public handle (include/mdp_b200.h) is the surrogate state itself
struct mdp_sur : public mdp::Surrogate {};
