// Batched descriptors / fitting: state shared between fit.cu and the
// surrogate's force training (surrogate.cu).
#pragma once

#include <vector>

#include "engine.h"

namespace mdp {

constexpr int FIT_KP = 64;       // row width: 1 + ncoeff (<= 56 at 2J=8) padded to 64
constexpr int FIT_NCP = 256;     // couplings (j1 >= j2, j) at most (125 at 2J=8)
constexpr int FIT_NT = 64;       // bispectrum triples at most (55 at 2J=8)

struct FitCoupling {
    int j1, j2, j, zoff;          // Z rows of this coupling start at zoff (per atom)
};
struct FitTriple {
    int j1, j2, j;
    int layer[3], coup[3];        // the three dB/dR terms: dU layer and Z coupling
    double fac[3];
};
struct FitTables {
    int ncoup, ntri, nz, tj, bnorm, bzero;
    FitCoupling cp[FIT_NCP];
    FitTriple tr[FIT_NT];
    // the dB/dR terms grouped by their dU layer: lt_off[L] .. lt_off[L] + lt_n[L]
    int lt_n[JD], lt_off[JD];
    int lt_k[3 * FIT_NT], lt_z[3 * FIT_NT];
    double lt_fac[3 * FIT_NT];
};

}  // namespace mdp

struct mdp_fit {
    mdp::SnapModel model;
    mdp::FitTables tab;
    int device = 0;
    cudaStream_t s = nullptr;
    // batch
    int nconf = 0, natoms = 0;
    std::vector<int> h_cn, h_ca0;
    std::vector<double> h_lat;   // cell vectors (9 per configuration) of the current batch
    mdp::DevBuf x, cfg, ca0, cn, cbox, we, wf, e, f;
    // work (sized for the whole batch)
    mdp::DevBuf tabs, pcount, poff, roff, rcount, cursor, rlist, B, Z, dul, dbdr, G, R, tgt, hi, lo, part, out, scan_tmp;
    mdp::ForcePath fp;
    long npairs = 0, nrows = 0;
    bool pairs_ready = false;
    // the Z / dU / dB/dR stages run over configuration-aligned chunks that fit
    // the scratch budget; U, B, the rows and the Gram pass span the batch
    struct Chunk { int c_lo, c_hi, a_lo, a_hi, t_lo, t_hi; long p_lo, p_hi; };
    std::vector<Chunk> chunks;
    double chunk_bytes = 24.0e9;   // scratch of the chunked stages (dU rows, dB/dR, Z) per chunk at most
    long chunk_pairs_max = 0;
    int chunk_tiles_max = 0;
    // launch shapes (autotuned): threads of the per-pair kernels, rows per Gram CTA
    int du_threads = 128, db_threads = 128, gram_rows = 4096;
    bool gram_tuned = false;   // gram_rows chosen by mdp_fit_tune (else sized from the row count)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int graph_mode = -1;
};


namespace mdp {
// per-pair dB/dR of the batch, float [pair][3][ncoeff] (device), and the
// per-atom bispectrum [ncoeff][atom] (device, FP64)
int fit_pair_derivs(mdp_fit *h, float *dbdr_out, double *blist_out);
}  // namespace mdp
