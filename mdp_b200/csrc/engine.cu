// MD engine and the project's C ABI (include/mdp_b200.h).
//
// Step order follows CIntegration::VelocityVerlet
// (src/C++/Integration/Integration.cpp:17-139): save x, initial integrate,
// neighbour rebuild check (rebuild after PBC wrap, or shift ghosts by their
// owners' displacement), SNAP force, final integrate, thermo.
#include "common.cuh"
#include "engine.h"
#include "surrogate.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <mutex>

namespace mdp {

// metal units, src/C++/Configuration/setunits.cpp:51-59
constexpr double BOLTZ = 8.617343e-5;
constexpr double MVV2E = 1.0364269e-4;
constexpr double FTM2V = 1.0 / 1.0364269e-4;
constexpr double NKTV2P = 1.6021765e6;

__global__ void k_aos_to_d4(const double *__restrict__ a, double4 *__restrict__ b, long n)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = make_double4(a[3 * i], a[3 * i + 1], a[3 * i + 2], 0.0);
}
__global__ void k_d4_to_aos(const double4 *__restrict__ b, double *__restrict__ a, long n)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { const double4 v = b[i]; a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }
}

static bool box_is_orth(const double *box)
{
    return box[1] == 0 && box[2] == 0 && box[3] == 0 && box[5] == 0 && box[6] == 0 && box[7] == 0;
}

}  // namespace mdp

using namespace mdp;

namespace mdp {
// ---------------------------------------------------------------------------
// FMA throughput probe
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fma_probe(T *out, int iters, T b, T c)
{
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = a[k] * b + c;
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename T>
static double fma_peak(int nsm)
{
    const int threads = 256, blocks = nsm * 8, iters = 4096;
    T *out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * threads * blocks) != cudaSuccess) return -1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_probe<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-6);
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        k_fma_probe<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-6);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace mdp

struct mdp_md {
    SnapModel model;
    mdp_md_config cfg;
    BoxParams bp;
    cudaStream_t s = nullptr;
    int device = 0;
    long anum_cap = 0;
    DevBuf x, v, f, xstart, xhold, e, vatom, scal, stage;
    Neighbors nb;
    ForcePath fp;
    long long step = 0, rebuilds = 0;
    double thermo_last[5] = {0, 0, 0, 0, 0};
    bool ready = false;
    // learned surrogate: driving model, judge cadence and tolerance, fallback
    Surrogate *sur = nullptr;
    int judge_every = 50;
    double judge_tol = 0.05;
    long long fallback_step = -1;
    std::vector<double> judge_log;   // (step, force RMSE) pairs
    DevBuf fjudge;
    DevBuf types;   // atom types 1..nelements (models with several element types)
    bool has_types = false;
};

extern "C" {

const char *mdp_last_error(void) { return get_error(); }

int mdp_snap_ncoeff(int twojmax)
{
    int n = 0;
    for (int j1 = 0; j1 <= twojmax; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(twojmax, j1 + j2); j += 2)
                if (j >= j1) n++;
    return n;
}

int mdp_md_create(mdp_md **h, const mdp_snap_params *p, const mdp_md_config *cfg)
{
    if (!h || !cfg) { set_error("null argument"); return -1; }
    *h = nullptr;
    if (cfg->natoms <= 1) { set_error("natoms must be > 1"); return -1; }
    if (cfg->neighmax < 1 || cfg->neighmax > 1024) { set_error("neighmax out of range"); return -1; }
    if (cfg->precision != MDP_PREC_FP64 && cfg->precision != MDP_PREC_FP32) { set_error("bad precision"); return -1; }
    if (!box_is_orth(cfg->box)) { set_error("only orthogonal periodic boxes are supported by the MD engine"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(cfg->device));
    mdp_md *m = new mdp_md();
    m->cfg = *cfg;
    if (m->cfg.neighevery < 1) m->cfg.neighevery = 1;
    m->device = cfg->device;
    if (model_init(m->model, p)) { delete m; return -1; }
    const double rc = m->model.geom.rcut + cfg->skin;
    box_setup(m->bp, cfg->box, cfg->box + 3, cfg->box + 6, rc, rc);
    // ghost capacity: volume of the enlarged box, 1.3x margin (Configuration.cpp:852)
    double vol = (m->bp.hi[0] - m->bp.lo[0]) * (m->bp.hi[1] - m->bp.lo[1]) * (m->bp.hi[2] - m->bp.lo[2]);
    m->anum_cap = (long)ceil(1.3 * vol * cfg->natoms) + 1024;
    const long n = cfg->natoms;
    if (cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) != cudaSuccess ||
        m->x.ensure(sizeof(double4) * m->anum_cap) || m->v.ensure(sizeof(double4) * n) ||
        m->f.ensure(sizeof(double4) * n) || m->xstart.ensure(sizeof(double4) * n) ||
        m->xhold.ensure(sizeof(double4) * n) || m->e.ensure(sizeof(double) * n) ||
        m->vatom.ensure(sizeof(double) * 6 * n) || m->scal.ensure(128)) {
        mdp_md_destroy(m);
        return -1;
    }
    *h = m;
    return 0;
}

void mdp_md_destroy(mdp_md *m)
{
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->s) cudaStreamSynchronize(m->s);
    DevBuf *b[] = {&m->x, &m->v, &m->f, &m->xstart, &m->xhold, &m->e, &m->vatom, &m->scal, &m->stage, &m->fjudge,
                   &m->types};
    for (auto x : b) x->release();
    m->nb.release();
    m->fp.release();
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
}

void *mdp_md_stream(mdp_md *m) { return m ? (void *)m->s : nullptr; }

static int upload_state(mdp_md *m, const double *x, const double *v, cudaMemcpyKind kind)
{
    const long n = m->cfg.natoms;
    double *tmp = nullptr;
    MDP_CUDA_TRY(cudaMallocAsync((void **)&tmp, sizeof(double) * 6 * n, m->s));
    MDP_CUDA_TRY(cudaMemcpyAsync(tmp, x, sizeof(double) * 3 * n, kind, m->s));
    MDP_CUDA_TRY(cudaMemcpyAsync(tmp + 3 * n, v, sizeof(double) * 3 * n, kind, m->s));
    k_aos_to_d4<<<(n + 255) / 256, 256, 0, m->s>>>(tmp, m->x.as<double4>(), n);
    k_aos_to_d4<<<(n + 255) / 256, 256, 0, m->s>>>(tmp + 3 * n, m->v.as<double4>(), n);
    MDP_CUDA_TRY(cudaFreeAsync(tmp, m->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    m->ready = false;
    return 0;
}

int mdp_md_set_state(mdp_md *m, const double *x, const double *v)
{
    if (!m || !x || !v) { set_error("null argument"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    return upload_state(m, x, v, cudaMemcpyHostToDevice);
}

int mdp_md_set_state_device(mdp_md *m, const double *x, const double *v)
{
    if (!m || !x || !v) { set_error("null argument"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    return upload_state(m, x, v, cudaMemcpyDeviceToDevice);
}

static int md_rebuild(mdp_md *m)
{
    const int n = m->cfg.natoms;
    const double *b = m->cfg.box;
    k_pbc_orth<<<(n + 255) / 256, 256, 0, m->s>>>(m->x.as<double4>(), n, 0.0, 0.0, 0.0, b[0], b[4], b[8]);
    count_launches(1);
    const double rc = m->model.geom.rcut + m->cfg.skin;
    if (neighbor_build(m->nb, m->bp, m->x.as<double4>(), n, rc, m->cfg.neighmax, m->anum_cap, m->s)) return -1;
    MDP_CUDA_TRY(cudaMemcpyAsync(m->xhold.p, m->x.p, sizeof(double4) * n, cudaMemcpyDeviceToDevice, m->s));
    m->rebuilds++;
    return 0;
}

static int md_force_plain(mdp_md *m)
{
    const int n = m->cfg.natoms;
    return force_compute(m->fp, m->model, m->cfg.precision, m->x.as<double4>(), n, m->nb.nlist.as<int>(),
                         m->nb.nnum.as<int>(), m->cfg.neighmax, (long)n * m->cfg.neighmax, m->nb.roff.as<int>(),
                         m->nb.rlist.as<long long>(), m->e.as<double>(), m->f.as<double4>(), m->vatom.as<double>(),
                         m->s, m->has_types ? m->types.as<int>() : nullptr, m->nb.alist.as<int>());
}

// Surrogate forces, judged against the plain model every judge_every steps:
// the plain forces replace the surrogate's on a judged step, and a force RMSE
// above the tolerance hands the run to the plain model from then on.
static int md_force(mdp_md *m)
{
    if (!m->sur || m->fallback_step >= 0) return md_force_plain(m);
    const int n = m->cfg.natoms;
    if (sur_force(*m->sur, m->fp, m->x.as<double4>(), n, m->nb.nlist.as<int>(), m->nb.nnum.as<int>(),
                  m->cfg.neighmax, m->nb.roff.as<int>(), m->nb.rlist.as<long long>(), m->e.as<double>(),
                  m->f.as<double4>(), m->vatom.as<double>(), m->s))
        return -1;
    if (m->judge_every <= 0 || m->step % m->judge_every != 0) return 0;
    if (m->fjudge.ensure(sizeof(double4) * (size_t)n)) return -1;
    MDP_CUDA_TRY(cudaMemcpyAsync(m->fjudge.p, m->f.p, sizeof(double4) * (size_t)n, cudaMemcpyDeviceToDevice, m->s));
    if (md_force_plain(m)) return -1;
    double ss = 0.0;
    if (force_sq_diff(m->fjudge.as<double4>(), m->f.as<double4>(), n, m->scal.as<double>() + 8, &ss, m->s)) return -1;
    const double rmse = sqrt(ss / (3.0 * n));
    m->judge_log.push_back((double)m->step);
    m->judge_log.push_back(rmse);
    if (!(rmse <= m->judge_tol)) m->fallback_step = m->step;
    return 0;
}

// thermo row (step, T, PE/atom, TE/atom, P), Calculation.cpp:436-467
static int md_thermo(mdp_md *m, double *row)
{
    const int n = m->cfg.natoms;
    double *sc = m->scal.as<double>();
    MDP_CUDA_TRY(cudaMemsetAsync(sc, 0, 5 * sizeof(double), m->s));
    k_thermo<<<(n + 255) / 256, 256, 0, m->s>>>(m->e.as<double>(), m->vatom.as<double>(), m->v.as<double4>(), n, sc);
    double hs[5];
    MDP_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, m->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    const double tdof = (n - 1) * 3.0;
    const double temp = MVV2E / (tdof * BOLTZ) * (m->cfg.mass * hs[4]);
    const double pe = hs[0] / n;
    const double ke = 0.5 * tdof * BOLTZ * temp / n;
    const double *b = m->cfg.box;
    const double vol = fabs(b[0] * (b[4] * b[8] - b[5] * b[7]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                            b[2] * (b[3] * b[7] - b[4] * b[6]));
    const double pres = (tdof * BOLTZ * temp + hs[1] + hs[2] + hs[3]) / 3.0 / vol * NKTV2P;
    row[0] = (double)m->step; row[1] = temp; row[2] = pe; row[3] = pe + ke; row[4] = pres;
    memcpy(m->thermo_last, row, sizeof(double) * 5);
    return 0;
}

int mdp_md_set_types(mdp_md *m, const int *types)
{
    if (!m || !types) { set_error("null argument"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    const int n = m->cfg.natoms, ne = m->model.ne;
    for (int i = 0; i < n; i++)
        if (types[i] < 1 || types[i] > ne) {
            set_error("atom %d has type %d; the model has types 1..%d", i, types[i], ne);
            return -1;
        }
    if (m->types.ensure(sizeof(int) * n)) return -1;
    MDP_CUDA_TRY(cudaMemcpyAsync(m->types.p, types, sizeof(int) * n, cudaMemcpyHostToDevice, m->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    m->has_types = true;
    m->ready = false;
    return 0;
}

int mdp_md_setup(mdp_md *m)
{
    if (!m) { set_error("null handle"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    if (m->model.ne > 1 && !m->has_types) {
        set_error("a model with %d element types needs mdp_md_set_types first", m->model.ne);
        return -1;
    }
    if (md_rebuild(m) || md_force(m)) return -1;
    double row[5];
    if (md_thermo(m, row)) return -1;
    m->ready = true;
    return 0;
}

int mdp_md_run(mdp_md *m, int nsteps, int thermo_every, double *thermo, int thermo_cap, int *nrows, float *elapsed_ms)
{
    if (!m) { set_error("null handle"); return -1; }
    if (!m->ready) { set_error("mdp_md_setup must run before mdp_md_run"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    const int n = m->cfg.natoms;
    const double dtf = 0.5 * m->cfg.dt * FTM2V;   // readdata.cpp:418-420
    const double dtfm = dtf / m->cfg.mass;
    const double dtv = m->cfg.dt;
    const double skin = m->cfg.skin;
    int rows = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, m->s);
    unsigned long long *dmax = reinterpret_cast<unsigned long long *>(m->scal.as<double>() + 6);
    for (int it = 0; it < nsteps; it++) {
        m->step++;
        k_nve_initial<<<(n + 255) / 256, 256, 0, m->s>>>(m->x.as<double4>(), m->v.as<double4>(), m->f.as<double4>(),
                                                         m->xstart.as<double4>(), n, dtfm, dtv);
        count_launches(1);
        const long long ago = m->step;
        int build = 0;
        if (ago >= m->cfg.neighdelay && ago % m->cfg.neighevery == 0) {
            if (!m->cfg.neighcheck) build = 1;
            else {
                MDP_CUDA_TRY(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), m->s));
                k_maxdisp<<<(n + 255) / 256, 256, 0, m->s>>>(m->x.as<double4>(), m->xhold.as<double4>(), n, dmax);
                count_launches(1);
                unsigned long long hm = 0;
                MDP_CUDA_TRY(cudaMemcpyAsync(&hm, dmax, sizeof(hm), cudaMemcpyDeviceToHost, m->s));
                MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
                double md;
                memcpy(&md, &hm, sizeof(md));
                if (md > 0.25 * skin * skin) build = 1;
            }
        }
        if (build) {
            if (md_rebuild(m)) return -1;
        } else if (m->nb.gnum > 0) {
            k_ghost_shift<<<(m->nb.gnum + 255) / 256, 256, 0, m->s>>>(m->x.as<double4>(), m->xstart.as<double4>(),
                                                                      m->nb.alist.as<int>(), n, m->nb.gnum);
            count_launches(1);
        }
        if (md_force(m)) return -1;
        k_nve_final<<<(n + 255) / 256, 256, 0, m->s>>>(m->v.as<double4>(), m->f.as<double4>(), n, dtfm);
        count_launches(1);
        if (thermo_every > 0 && m->step % thermo_every == 0) {
            double row[5];
            if (md_thermo(m, row)) return -1;
            if (thermo && rows < thermo_cap) memcpy(thermo + 5 * rows, row, sizeof(row));
            rows++;
        }
    }
    cudaEventRecord(e1, m->s);
    MDP_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (elapsed_ms) *elapsed_ms = ms;
    if (nrows) *nrows = std::min(rows, thermo_cap);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int mdp_md_upload(mdp_md *m, const double *x, const double *v)
{
    if (!m || !x || !v) { set_error("null argument"); return -1; }
    if (!m->ready) { set_error("mdp_md_setup must run before mdp_md_upload"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    const long n = m->cfg.natoms;
    if (m->stage.ensure(sizeof(double) * 6 * n)) return -1;
    double *t = m->stage.as<double>();
    MDP_CUDA_TRY(cudaMemcpyAsync(t, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, m->s));
    MDP_CUDA_TRY(cudaMemcpyAsync(t + 3 * n, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, m->s));
    k_aos_to_d4<<<(n + 255) / 256, 256, 0, m->s>>>(t, m->x.as<double4>(), n);
    k_aos_to_d4<<<(n + 255) / 256, 256, 0, m->s>>>(t + 3 * n, m->v.as<double4>(), n);
    count_launches(2);
    return 0;
}

int mdp_md_download(mdp_md *m, double *f, double *eatom)
{
    if (!m) { set_error("null handle"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    const long n = m->cfg.natoms;
    if (m->stage.ensure(sizeof(double) * 6 * n)) return -1;
    double *t = m->stage.as<double>();
    if (f) {
        k_d4_to_aos<<<(n + 255) / 256, 256, 0, m->s>>>(m->f.as<double4>(), t, n);
        count_launches(1);
        MDP_CUDA_TRY(cudaMemcpyAsync(f, t, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, m->s));
    }
    if (eatom) MDP_CUDA_TRY(cudaMemcpyAsync(eatom, m->e.p, sizeof(double) * n, cudaMemcpyDeviceToHost, m->s));
    return 0;
}

int mdp_md_sync(mdp_md *m)
{
    if (!m) { set_error("null handle"); return -1; }
    MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    return 0;
}

long long mdp_launch_count(void) { return launch_count(); }

int mdp_md_get_state(mdp_md *m, double *x, double *v, double *f, double *eatom)
{
    if (!m) { set_error("null handle"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    const long n = m->cfg.natoms;
    double *tmp = nullptr;
    MDP_CUDA_TRY(cudaMallocAsync((void **)&tmp, sizeof(double) * 3 * n, m->s));
    const DevBuf *src[3] = {&m->x, &m->v, &m->f};
    double *dst[3] = {x, v, f};
    for (int k = 0; k < 3; k++) {
        if (!dst[k]) continue;
        k_d4_to_aos<<<(n + 255) / 256, 256, 0, m->s>>>(src[k]->as<double4>(), tmp, n);
        MDP_CUDA_TRY(cudaMemcpyAsync(dst[k], tmp, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, m->s));
        MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    }
    if (eatom) MDP_CUDA_TRY(cudaMemcpyAsync(eatom, m->e.p, sizeof(double) * n, cudaMemcpyDeviceToHost, m->s));
    MDP_CUDA_TRY(cudaFreeAsync(tmp, m->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    return 0;
}

int mdp_md_thermo(mdp_md *m, double *out5)
{
    if (!m || !out5) { set_error("null argument"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    return md_thermo(m, out5);
}

int mdp_md_counters(mdp_md *m, long long *out)
{
    if (!m || !out) { set_error("null argument"); return -1; }
    int np = 0;
    if (m->fp.poff.p) {
        MDP_CUDA_TRY(cudaMemcpyAsync(&np, m->fp.poff.as<int>() + m->cfg.natoms, sizeof(int), cudaMemcpyDeviceToHost, m->s));
        MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    }
    out[0] = m->step; out[1] = m->rebuilds; out[2] = np; out[3] = m->nb.gnum; out[4] = m->nb.nsum;
    return 0;
}

int mdp_md_sur_sample(mdp_md *m, mdp_sur *S)
{
    if (!m || !S) { set_error("null argument"); return -1; }
    if (!m->ready) { set_error("mdp_md_setup must run first"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    Surrogate &s = *static_cast<Surrogate *>(S);
    const int n = m->cfg.natoms;
    if (sur_features(s, m->fp, m->x.as<double4>(), n, m->nb.nlist.as<int>(), m->nb.nnum.as<int>(), m->cfg.neighmax,
                     m->s))
        return -1;
    return mdp_sur_dataset_add(S, s.B.as<double>(), n, m->e.as<double>(), n, m->s);
}

int mdp_md_sur_features(mdp_md *m, mdp_sur *S, double *B_host)
{
    if (!m || !S || !B_host) { set_error("null argument"); return -1; }
    if (!m->ready) { set_error("mdp_md_setup must run first"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(m->device));
    Surrogate &s = *static_cast<Surrogate *>(S);
    const int n = m->cfg.natoms;
    if (sur_features(s, m->fp, m->x.as<double4>(), n, m->nb.nlist.as<int>(), m->nb.nnum.as<int>(), m->cfg.neighmax,
                     m->s))
        return -1;
    MDP_CUDA_TRY(cudaMemcpyAsync(B_host, s.B.p, sizeof(double) * 14 * (size_t)n, cudaMemcpyDeviceToHost, m->s));
    MDP_CUDA_TRY(cudaStreamSynchronize(m->s));
    return 0;
}

int mdp_md_set_zbl(mdp_md *m, double inner, double outer, double z)
{
    if (!m) { set_error("null handle"); return -1; }
    const double reach = m->model.geom.rcut + m->cfg.skin;
    if (z > 0.0 && outer > reach) {
        set_error("ZBL cutoff %g A exceeds the neighbour-list reach %g A (SNAP cutoff + skin)", outer, reach);
        return -1;
    }
    if (zbl_setup(m->model.zbl, inner, outer, z)) return -1;
    m->ready = false;   // forces must be recomputed by mdp_md_setup
    return 0;
}

int mdp_md_set_surrogate(mdp_md *m, mdp_sur *S, int judge_every, double tol)
{
    if (!m) { set_error("null handle"); return -1; }
    if (S) {
        const Surrogate &s = *static_cast<Surrogate *>(S);
        if (!s.trained) { set_error("surrogate has no parameters"); return -1; }
        if (fabs(s.model.geom.rcut - m->model.geom.rcut) > 1e-12) {
            set_error("surrogate cutoff %g differs from the model's %g", s.model.geom.rcut, m->model.geom.rcut);
            return -1;
        }
    }
    m->sur = static_cast<Surrogate *>(S);
    m->judge_every = judge_every;
    m->judge_tol = tol;
    m->fallback_step = -1;
    m->judge_log.clear();
    return 0;
}

int mdp_md_surrogate_status(mdp_md *m, int *active, long long *fallback_step, int *njudge, double *log, int cap)
{
    if (!m) { set_error("null handle"); return -1; }
    if (active) *active = (m->sur && m->fallback_step < 0) ? 1 : 0;
    if (fallback_step) *fallback_step = m->fallback_step;
    const int nj = (int)(m->judge_log.size() / 2);
    if (njudge) *njudge = nj;
    if (log)
        for (int i = 0; i < std::min(nj, cap); i++) { log[2 * i] = m->judge_log[2 * i]; log[2 * i + 1] = m->judge_log[2 * i + 1]; }
    return 0;
}

int mdp_md_stage_timing(mdp_md *m, int enable)
{
    if (!m) { set_error("null handle"); return -1; }
    m->fp.timing = enable != 0;
    for (double &t : m->fp.stage_ms) t = 0.0;
    m->fp.stage_calls = 0;
    return 0;
}

int mdp_md_stage_times(mdp_md *m, double *ms6, long long *calls)
{
    if (!m) { set_error("null handle"); return -1; }
    if (ms6) memcpy(ms6, m->fp.stage_ms, sizeof(double) * 6);
    if (calls) *calls = m->fp.stage_calls;
    return 0;
}

// ---------------------------------------------------------------------------
// one-shot force evaluations
// ---------------------------------------------------------------------------
struct OneShot {
    SnapModel model;
    Neighbors nb;
    ForcePath fp;
    DevBuf x4, f4, xin, alist_tmp, types;
};
static std::mutex g_os_mu;

// types 1..ne on the host; 0 or -1 with the error set
static int check_types(const int *t, long n, int ne)
{
    for (long i = 0; i < n; i++)
        if (t[i] < 1 || t[i] > ne) {
            set_error("atom %ld has type %d; the model has types 1..%d", i, t[i], ne);
            return -1;
        }
    return 0;
}

static int compute_host(const mdp_snap_params *p, int precision, int natoms, const double *x, const int *atomtype,
                        const double *box, double skin, int neighmax, double *eatom, double *fatom, double *vatom,
                        int *neighlist, int *neighnum, int *anum_out, int *alist_out, double *xall_out,
                        int alist_cap)
{
    std::lock_guard<std::mutex> lk(g_os_mu);
    if (!x || !box || natoms <= 0) { set_error("bad arguments"); return -1; }
    static OneShot os;
    int dev = 0;
    MDP_CUDA_TRY(cudaGetDevice(&dev));
    if (model_init(os.model, p)) return -1;
    const int *types_dev = nullptr;
    if (os.model.ne > 1) {
        if (!atomtype) { set_error("a model with %d element types needs the atom types", os.model.ne); return -1; }
        if (check_types(atomtype, natoms, os.model.ne) || os.types.ensure(sizeof(int) * natoms)) return -1;
        MDP_CUDA_TRY(cudaMemcpy(os.types.p, atomtype, sizeof(int) * natoms, cudaMemcpyHostToDevice));
        types_dev = os.types.as<int>();
    }
    BoxParams bp;
    const double rc = os.model.geom.rcut + skin;
    box_setup(bp, box, box + 3, box + 6, rc, rc);
    double vol = (bp.hi[0] - bp.lo[0]) * (bp.hi[1] - bp.lo[1]) * (bp.hi[2] - bp.lo[2]);
    long cap = (long)ceil(1.5 * vol * natoms) + 4096;
    cudaStream_t s = 0;
    if (os.x4.ensure(sizeof(double4) * cap) || os.f4.ensure(sizeof(double4) * natoms) ||
        os.xin.ensure(sizeof(double) * (size_t)natoms * 10))
        return -1;
    double *xin = os.xin.as<double>();
    MDP_CUDA_TRY(cudaMemcpy(xin, x, sizeof(double) * 3 * natoms, cudaMemcpyHostToDevice));
    k_aos_to_d4<<<(natoms + 255) / 256, 256, 0, s>>>(xin, os.x4.as<double4>(), natoms);
    if (neighbor_build(os.nb, bp, os.x4.as<double4>(), natoms, rc, neighmax, cap, s)) return -1;
    double *ed = xin + 3 * natoms, *vd = xin + 4 * natoms;
    if (force_compute(os.fp, os.model, precision, os.x4.as<double4>(), natoms, os.nb.nlist.as<int>(),
                      os.nb.nnum.as<int>(), neighmax, (long)natoms * neighmax, os.nb.roff.as<int>(),
                      os.nb.rlist.as<long long>(), ed, os.f4.as<double4>(), vd, s, types_dev,
                      os.nb.alist.as<int>()))
        return -1;
    k_d4_to_aos<<<(natoms + 255) / 256, 256, 0, s>>>(os.f4.as<double4>(), xin, natoms);
    MDP_CUDA_TRY(cudaDeviceSynchronize());
    if (eatom) MDP_CUDA_TRY(cudaMemcpy(eatom, ed, sizeof(double) * natoms, cudaMemcpyDeviceToHost));
    if (fatom) MDP_CUDA_TRY(cudaMemcpy(fatom, xin, sizeof(double) * 3 * natoms, cudaMemcpyDeviceToHost));
    if (vatom) MDP_CUDA_TRY(cudaMemcpy(vatom, vd, sizeof(double) * 6 * natoms, cudaMemcpyDeviceToHost));
    if (neighlist)
        MDP_CUDA_TRY(cudaMemcpy(neighlist, os.nb.nlist.p, sizeof(int) * (size_t)natoms * neighmax, cudaMemcpyDeviceToHost));
    if (neighnum) MDP_CUDA_TRY(cudaMemcpy(neighnum, os.nb.nnum.p, sizeof(int) * natoms, cudaMemcpyDeviceToHost));
    if (anum_out) *anum_out = os.nb.anum;
    if (alist_out || xall_out) {
        if (os.nb.anum > alist_cap) { set_error("alist_cap %d < anum %d", alist_cap, os.nb.anum); return -1; }
        if (alist_out) MDP_CUDA_TRY(cudaMemcpy(alist_out, os.nb.alist.p, sizeof(int) * os.nb.anum, cudaMemcpyDeviceToHost));
        if (xall_out) {
            DevBuf t;
            if (t.ensure(sizeof(double) * 3 * os.nb.anum)) return -1;
            k_d4_to_aos<<<(os.nb.anum + 255) / 256, 256>>>(os.x4.as<double4>(), t.as<double>(), os.nb.anum);
            cudaError_t ce = cudaMemcpy(xall_out, t.p, sizeof(double) * 3 * os.nb.anum, cudaMemcpyDeviceToHost);
            t.release();
            if (ce != cudaSuccess) { set_error("copy: %s", cudaGetErrorString(ce)); return -1; }
        }
    }
    return 0;
}

int mdp_snap_compute_host(const mdp_snap_params *p, int precision, int natoms, const double *x, const double *box,
                          double skin, int neighmax, double *eatom, double *fatom, double *vatom, int *neighlist,
                          int *neighnum, int *anum_out, int *alist_out, double *xall_out, int alist_cap)
{
    return compute_host(p, precision, natoms, x, nullptr, box, skin, neighmax, eatom, fatom, vatom, neighlist,
                        neighnum, anum_out, alist_out, xall_out, alist_cap);
}

int mdp_snap_compute_host_typed(const mdp_snap_params *p, int precision, int natoms, const double *x,
                                const int *atomtype, const double *box, double skin, int neighmax, double *eatom,
                                double *fatom, double *vatom, int *neighlist, int *neighnum, int *anum_out,
                                int *alist_out, double *xall_out, int alist_cap)
{
    return compute_host(p, precision, natoms, x, atomtype, box, skin, neighmax, eatom, fatom, vatom, neighlist,
                        neighnum, anum_out, alist_out, xall_out, alist_cap);
}

__global__ void k_copy_int(const int *__restrict__ a, int *__restrict__ b, long n)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

static int compute_device(const mdp_snap_params *p, int precision, const double *x, const int *atomtype,
                          const int *alist, const int *neighlist, const int *neighnum, int inum, int anum,
                          int neighmax, double *eatom, double *fatom, double *vatom, void *stream)
{
    std::lock_guard<std::mutex> lk(g_os_mu);
    static OneShot os;
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    MDP_CUDA_TRY(cudaGetDevice(&dev));
    if (model_init(os.model, p)) return -1;
    if (os.model.ne > 1) {
        if (!atomtype) { set_error("a model with %d element types needs the atom types", os.model.ne); return -1; }
        std::vector<int> th(inum);
        MDP_CUDA_TRY(cudaMemcpyAsync(th.data(), atomtype, sizeof(int) * inum, cudaMemcpyDeviceToHost, s));
        MDP_CUDA_TRY(cudaStreamSynchronize(s));
        if (check_types(th.data(), inum, os.model.ne)) return -1;
    }
    if (os.x4.ensure(sizeof(double4) * (size_t)anum) || os.f4.ensure(sizeof(double4) * inum) ||
        os.nb.rcount.ensure(sizeof(int) * inum) || os.nb.roff.ensure(sizeof(int) * ((size_t)inum + 1)) ||
        os.nb.cursor.ensure(sizeof(int) * inum) || os.nb.rlist.ensure(sizeof(long long) * (size_t)inum * neighmax) ||
        os.nb.scan_tmp.ensure(sizeof(int) * scan_tmp_ints(inum)))
        return -1;
    k_aos_to_d4<<<(anum + 255) / 256, 256, 0, s>>>(x, os.x4.as<double4>(), anum);
    const int tb = 256, gb = (inum + tb - 1) / tb;
    MDP_CUDA_TRY(cudaMemsetAsync(os.nb.rcount.p, 0, sizeof(int) * inum, s));
    k_rev_count<<<gb, tb, 0, s>>>(neighlist, neighnum, alist, inum, neighmax, os.nb.rcount.as<int>());
    if (exclusive_scan(os.nb.rcount.as<int>(), os.nb.roff.as<int>(), inum, os.nb.scan_tmp.as<int>(), s)) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(os.nb.cursor.p, 0, sizeof(int) * inum, s));
    k_rev_fill<<<gb, tb, 0, s>>>(neighlist, neighnum, alist, inum, neighmax, os.nb.roff.as<int>(),
                                 os.nb.cursor.as<int>(), os.nb.rlist.as<long long>());
    k_rev_sort<<<std::min((inum + 7) / 8, num_sms() * 8), 256, 0, s>>>(inum, os.nb.roff.as<int>(), os.nb.rlist.as<long long>());
    if (force_compute(os.fp, os.model, precision, os.x4.as<double4>(), inum, neighlist, neighnum, neighmax,
                      (long)inum * neighmax, os.nb.roff.as<int>(), os.nb.rlist.as<long long>(), eatom,
                      os.f4.as<double4>(), vatom, s, atomtype, alist))
        return -1;
    k_d4_to_aos<<<(inum + 255) / 256, 256, 0, s>>>(os.f4.as<double4>(), fatom, inum);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int mdp_snap_compute_device(const mdp_snap_params *p, int precision, const double *x, const int *alist,
                            const int *neighlist, const int *neighnum, int inum, int anum, int neighmax,
                            double *eatom, double *fatom, double *vatom, void *stream)
{
    return compute_device(p, precision, x, nullptr, alist, neighlist, neighnum, inum, anum, neighmax, eatom, fatom,
                          vatom, stream);
}

int mdp_snap_compute_device_typed(const mdp_snap_params *p, int precision, const double *x, const int *atomtype,
                                  const int *alist, const int *neighlist, const int *neighnum, int inum, int anum,
                                  int neighmax, double *eatom, double *fatom, double *vatom, void *stream)
{
    return compute_device(p, precision, x, atomtype, alist, neighlist, neighnum, inum, anum, neighmax, eatom, fatom,
                          vatom, stream);
}

int mdp_probe_fma_peak(int device, double *fp64, double *fp32)
{
    MDP_CUDA_TRY(cudaSetDevice(device));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    if (fp64) *fp64 = fma_peak<double>(nsm);
    if (fp32) *fp32 = fma_peak<float>(nsm);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // extern "C"
