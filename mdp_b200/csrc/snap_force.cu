// SNAP model set-up, the force-path driver and the neighbour-structure
// builder.  Kernel templates live in snap_kernels.cuh / neighbor.cu.
#include "common.cuh"
#include "engine.h"

#include <algorithm>
#include <math.h>
#include <string.h>

namespace mdp {

// Growth drains the device on both sides.  The old buffer may still be read
// by work queued on any stream, and the zero fill runs on the legacy stream,
// which does not order with the engine's non-blocking streams: without the
// drain, kernels queued right after a growth raced the fill and some of their
// first results were zeroed.  Growth happens only on a buffer's first use at a
// larger size, never inside a stream capture.
// ZBL parameters as ZBLpotential.jl:14-99 defines them: 1/a = (Z^0.23 +
// Z^0.23) / 0.4685, prefactors c_k Z^2 qqr2e, and the switch polynomial that
// takes E, E' and E'' to zero at the outer cutoff
int zbl_setup(ZblParams &zp, double inner, double outer, double z)
{
    zp.on = 0;
    if (z <= 0.0) return 0;
    if (!(inner > 0.0 && outer > inner)) {
        set_error("ZBL radii must satisfy 0 < inner < outer (got %g, %g)", inner, outer);
        return -1;
    }
    static const double c[4] = {0.02817, 0.28022, 0.50986, 0.18175};
    static const double d[4] = {0.20162, 0.40290, 0.94229, 3.19980};
    const double ainv = 2.0 * pow(z, 0.23) / 0.46850, zze = z * z * 14.399645;
    for (int k = 0; k < 4; k++) {
        zp.dk[k] = d[k] * ainv;
        zp.ck[k] = c[k] * zze;
    }
    // E and its first two derivatives at the outer cutoff
    double s = 0.0, sp = 0.0, spp = 0.0;
    for (int k = 0; k < 4; k++) {
        const double ek = zp.ck[k] * exp(-zp.dk[k] * outer);
        s += ek;
        sp -= zp.dk[k] * ek;
        spp += zp.dk[k] * zp.dk[k] * ek;
    }
    const double ri = 1.0 / outer;
    const double fc = s * ri, fcp = (sp - s * ri) * ri, fcpp = (spp - 2.0 * sp * ri + 2.0 * s * ri * ri) * ri;
    const double tc = outer - inner;
    const double swa = (-3.0 * fcp + tc * fcpp) / (tc * tc), swb = (2.0 * fcp - tc * fcpp) / (tc * tc * tc);
    zp.sw3 = swa / 3.0;
    zp.sw4 = swb / 4.0;
    zp.sw5 = -fc + 0.5 * tc * fcp - tc * tc / 12.0 * fcpp;
    zp.inner = inner;
    zp.rcsq = outer * outer;
    zp.on = 1;
    return 0;
}

int DevBuf::ensure(size_t n)
{
    if (n <= bytes) return 0;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        set_error("device synchronize before growing a buffer: %s", cudaGetErrorString(e));
        return -1;
    }
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t want = n + n / 8 + 256;
    e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        set_error("cudaMalloc(%zu bytes): %s", want, cudaGetErrorString(e));
        p = nullptr;
        return -1;
    }
    e = cudaMemset(p, 0, want);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        set_error("zero fill of %zu bytes: %s", want, cudaGetErrorString(e));
        cudaFree(p);
        p = nullptr;
        return -1;
    }
    bytes = want;
    return 0;
}
void DevBuf::release()
{
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

void ForcePath::release()
{
    DevBuf *b[] = {&pcount, &poff, &prij, &pinfo, &pab, &smap, &dE, &Ut, &Y, &scan_tmp, &B, &G, &pcw, &elem, &ecoef};
    for (auto x : b) x->release();
    for (auto &e : ev)
        if (e) { cudaEventDestroy(e); e = nullptr; }
}

void Neighbors::release()
{
    DevBuf *b[] = {&gcount, &goff, &gmask, &alist, &cidx, &ccount, &cstart, &cursor, &catoms,
                   &nlist, &nnum, &rcount, &roff, &rlist, &status, &scan_tmp};
    for (auto x : b) x->release();
}

// ---------------------------------------------------------------------------
// model
// ---------------------------------------------------------------------------
static int triple_ok(int j1, int j2, int j, int tj)
{
    return j2 <= j1 && j1 <= tj && j <= tj && j1 - j2 <= j && j <= j1 + j2 && ((j1 + j2 + j) % 2 == 0);
}

int model_init(SnapModel &m, const mdp_snap_params *p)
{
    if (!p) { set_error("null SNAP parameters"); return -1; }
    const int tj = p->twojmax;
    if (tj != 4 && tj != 6 && tj != 8) {
        set_error("twojmax=%d not supported (4, 6 or 8)", tj);
        return -1;
    }
    if (p->chemflag != 0 && p->chemflag != 1) { set_error("chemflag must be 0 or 1"); return -1; }
    if (p->quadraticflag != 0 && p->quadraticflag != 1) { set_error("quadraticflag must be 0 or 1"); return -1; }
    const int ne = p->nelements > 1 ? p->nelements : 1;
    if (ne > MAXELEM) { set_error("nelements=%d: at most %d element types", p->nelements, MAXELEM); return -1; }
    if (p->nelements > 1 && (!p->radelems || !p->wjelems)) {
        set_error("nelements=%d needs radelems and wjelems", p->nelements);
        return -1;
    }
    if (ne > 1 && p->quadraticflag) {
        set_error("quadratic SNAP is supported for one element type only");
        return -1;
    }
    // element triples of the coefficient table (cpuSnapComputeEi, cpuSnap4.cpp:255-280)
    const int ntri = (ne > 1 && p->chemflag) ? ne * ne * ne : 1;
    if (p->switchflag != 0 && p->switchflag != 1) { set_error("switchflag must be 0 or 1"); return -1; }
    // idxb enumeration (cpuSnap.cpp:44-68)
    int jjb[JD][JD][JD];
    int nb = 0;
    for (int j1 = 0; j1 <= tj; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= std::min(tj, j1 + j2); j += 2)
                if (j >= j1) jjb[j1][j2][j] = nb++;
    const int nall = nb * ntri + 1 + (p->quadraticflag ? nb * (nb + 1) / 2 : 0);
    if (p->ncoeffall != nall) {
        set_error("ncoeffall=%d but 2J=%d%s%s needs %d coefficients", p->ncoeffall, tj,
                  p->quadraticflag ? " with quadratic terms" : "", ntri > 1 ? " per element (chemflag)" : "", nall);
        return -1;
    }
    if (!p->coeff) { set_error("null coefficient array"); return -1; }
    m.p = *p;
    m.coeff.assign(p->coeff, p->coeff + (size_t)ne * p->ncoeffall);
    m.p.coeff = m.coeff.data();
    m.p.radelems = m.p.wjelems = nullptr;
    m.ne = ne;
    m.ncoeff = nb;
    m.nu = idxu_count(tj);
    m.nyh = yh_count(tj);
    const bool one_listed = p->nelements == 1 && p->radelems && p->wjelems;
    const double rad1 = one_listed ? p->radelems[0] : p->radelem;
    const double wj1 = one_listed ? p->wjelems[0] : p->wjelem;
    m.p.radelem = rad1;
    m.p.wjelem = wj1;
    double rcut = 2.0 * rad1 * p->rcutfac;
    memset(&m.eg, 0, sizeof(m.eg));
    m.eg.ne = ne;
    m.eg.chem = (ne > 1 && p->chemflag) ? 1 : 0;
    m.eg.nblk = m.eg.chem ? ne : 1;
    if (ne > 1) {
        // InitSnap: rcutmax = max 2 radelem rcutfac; cut = (radelem_i + radelem_j) rcutfac
        rcut = 0.0;
        for (int a = 0; a < ne; a++) {
            if (!(p->radelems[a] > 0.0)) { set_error("radelems[%d] must be positive", a); return -1; }
            rcut = std::max(2.0 * p->radelems[a] * p->rcutfac, rcut);
            m.eg.wj[a] = p->wjelems[a];
            for (int b = 0; b < ne; b++) {
                const double cut = (p->radelems[a] + p->radelems[b]) * p->rcutfac;
                m.eg.rcut[a][b] = cut;
                m.eg.rcutsq[a][b] = cut * cut;
            }
        }
    }
    m.geom.rcut = rcut;
    m.geom.rcutsq = rcut * rcut;
    m.geom.rfac0 = p->rfac0;
    m.geom.rmin0 = p->rmin0;
    m.geom.wj = wj1;
    m.geom.switchflag = p->switchflag;

    // beta' per coupling triple (cpuSnap4.cpp:763-787)
    memset(&m.yd, 0, sizeof(m.yd));
    memset(&m.yf, 0, sizeof(m.yf));
    memset(&m.yq, 0, sizeof(m.yq));
    const double *c = m.coeff.data();
    auto fill_beta = [&](const double *cc, YParams<double> &yd, YParams<float> *yf) {
        for (int j1 = 0; j1 <= tj; j1++)
            for (int j2 = 0; j2 <= j1; j2++)
                for (int j = 0; j <= tj; j++) {
                    if (!triple_ok(j1, j2, j, tj)) continue;
                    double b;
                    if (j >= j1) {
                        b = cc[1 + jjb[j1][j2][j]];
                        if (j1 == j) b *= (j2 == j) ? 3.0 : 2.0;
                    } else if (j >= j2) {
                        b = cc[1 + jjb[j][j2][j1]];
                        if (j2 == j) b *= 2.0;
                    } else {
                        b = cc[1 + jjb[j2][j][j1]];
                    }
                    if (!p->bnormflag && j1 > j) b *= (j1 + 1) / (j + 1.0);
                    if (p->bnormflag) b /= (j + 1);
                    const int k = (j >= j1) ? jjb[j1][j2][j] : (j >= j2) ? jjb[j][j2][j1] : jjb[j2][j][j1];
                    yd.betaY[tri_index(j1, j2, j)] = b;
                    yd.kmap[tri_index(j1, j2, j)] = (unsigned char)k;
                    if (yf) {
                        yf->betaY[tri_index(j1, j2, j)] = (float)b;
                        yf->kmap[tri_index(j1, j2, j)] = (unsigned char)k;
                    }
                }
    };
    fill_beta(c, m.yd, &m.yf);
    // quadratic SNAP and several elements: the Y kernel takes per-atom
    // coefficients (G_i = beta + Q B_i; the atom element's table), so its
    // per-triple factors are those of unit coefficients
    memset(&m.quad, 0, sizeof(m.quad));
    if (ne > 1) {
        std::vector<double> ones(nb + 1, 1.0);
        fill_beta(ones.data(), m.yq, nullptr);
    }
    if (p->quadraticflag) {
        if (nb > QUAD_MAXK) { set_error("quadratic SNAP supports up to %d components", QUAD_MAXK); return -1; }
        std::vector<double> ones(nb + 1, 1.0);
        fill_beta(ones.data(), m.yq, nullptr);
        m.quad.beta0 = c[0];
        m.quad.ncoeff = nb;
        for (int k = 0; k < nb; k++) m.quad.beta[k] = c[1 + k];
        for (int k = 0; k < nb * (nb + 1) / 2; k++) m.quad.q[k] = c[1 + nb + k];
    }
    double e0 = c[0];
    if (p->bzeroflag) {
        for (int j1 = 0; j1 <= tj; j1++)
            for (int j2 = 0; j2 <= j1; j2++)
                for (int j = j1 - j2; j <= std::min(tj, j1 + j2); j += 2)
                    if (j >= j1) e0 -= c[1 + jjb[j1][j2][j]] * (p->bnormflag ? 1.0 : (double)(j + 1));
    }
    m.yd.e0 = e0;
    m.yf.e0 = e0;

    // Y-kernel warp assignment per output layer j: rows mb get warps in
    // proportion to their cost (sum over couplings of items x terms per item);
    // a row with k warps is split by row-pair index ib modulo k
    auto assign = [&](int nw, unsigned char (*lmb)[YI_MAXW], unsigned char (*lo)[YI_MAXW],
                      unsigned char (*lst)[YI_MAXW]) {
        for (int j = 0; j < JD; j++)
            for (int w = 0; w < YI_MAXW; w++) { lmb[j][w] = 255; lo[j][w] = 0; lst[j][w] = 1; }
        for (int j = 0; j <= tj; j++) {
            const int R = j / 2 + 1;
            std::vector<double> cost(R, 0.0);
            for (int mb = 0; mb < R; mb++)
                for (int j1 = 0; j1 <= tj; j1++)
                    for (int j2 = 0; j2 <= j1; j2++) {
                        if (!coupling_ok(j1, j2, j)) continue;
                        int terms = 0;
                        for (int ma = 0; ma <= j; ma++) {
                            int ma1min = std::max(0, (2 * ma - j - j2 + j1) / 2);
                            terms += std::min(j1, (2 * ma - j + j2 + j1) / 2) - ma1min + 1;
                        }
                        cost[mb] += (double)nb_of(j1, j2, j, mb) * (terms + j1 + j2 + 2);
                    }
            std::vector<int> nw_row(R, 1);
            int used = std::min(R, nw);
            if (R > nw) return -1;
            while (used < nw) {
                int best = 0;
                for (int r = 1; r < R; r++)
                    if (cost[r] / nw_row[r] > cost[best] / nw_row[best]) best = r;
                // splitting a row beyond its largest item count buys nothing
                int maxnb = 0;
                for (int j1 = 0; j1 <= tj; j1++)
                    for (int j2 = 0; j2 <= j1; j2++)
                        if (coupling_ok(j1, j2, j)) maxnb = std::max(maxnb, nb_of(j1, j2, j, best));
                if (nw_row[best] >= maxnb) break;
                nw_row[best]++;
                used++;
            }
            int w = 0;
            for (int r = 0; r < R; r++)
                for (int k = 0; k < nw_row[r]; k++, w++) {
                    lmb[j][w] = (unsigned char)r;
                    lo[j][w] = (unsigned char)k;
                    lst[j][w] = (unsigned char)nw_row[r];
                }
        }
        return 0;
    };
    if (assign(yi_warps(false, tj), m.yd.lay_mb, m.yd.lay_o, m.yd.lay_st) ||
        assign(yi_warps(true, tj), m.yf.lay_mb, m.yf.lay_o, m.yf.lay_st)) {
        set_error("Y-kernel warp assignment failed");
        return -1;
    }
    memcpy(m.yq.lay_mb, m.yd.lay_mb, sizeof(m.yd.lay_mb));
    memcpy(m.yq.lay_o, m.yd.lay_o, sizeof(m.yd.lay_o));
    memcpy(m.yq.lay_st, m.yd.lay_st, sizeof(m.yd.lay_st));

    return 0;
}

// ---------------------------------------------------------------------------
// stage sequence per (T, TJ)
// ---------------------------------------------------------------------------
template <typename T, int TJ>
static int launch_snap(const SnapModel &m, const YParams<T> &yp, ForcePath &fp, int inum, int nm,
                       double *eatom, cudaStream_t s)
{
    if (launch_ui<T, TJ>(m, fp, inum, s)) return -1;
    if (launch_yi<T, TJ>(m, yp, fp, inum, eatom, s)) return -1;
    return launch_fi<T, TJ>(m, fp, inum, nm, s);
}

int launch_bi_tiles(const double2 *Ut, int natoms, int tj, int bnorm, int bzero, double *bout, long bstride,
                    cudaStream_t s);
int launch_yi_pa_d(const SnapModel &m, const YParams<double> &yp, ForcePath &fp, int inum, const double *G,
                   cudaStream_t s);

// Quadratic SNAP, one thread per atom: G[k][atom] = beta_k + (Q B)_k (the
// per-atom coefficients of cpuComputeBeta2, cpuSnap.cpp:1713-1737) and
// eatom = beta0 + beta . B + B^T Q B / 2 = beta0 + B . (beta + G) / 2
// (cpuSnapTallyEnergyFull, cpuSnap.cpp:1743-1770).  B [k][atom] is staged in
// shared memory per block.
constexpr int QUAD_THREADS = 64;
__global__ void __launch_bounds__(QUAD_THREADS)
k_snap_quad(const double *__restrict__ B, int natoms, const __grid_constant__ QuadParams Q, double *__restrict__ G,
            double *__restrict__ eatom)
{
    __shared__ double bs[QUAD_MAXK][QUAD_THREADS];
    const int t = threadIdx.x, atom = blockIdx.x * QUAD_THREADS + t;
    const int n = Q.ncoeff;
    for (int k = 0; k < n; k++) bs[k][t] = atom < natoms ? B[(size_t)k * natoms + atom] : 0.0;
    if (atom >= natoms) return;
    double e = 0.0;
    for (int k = 0; k < n; k++) {
        double g = Q.beta[k];
        // row k of the packed upper triangle: q(k, l) for l >= k at off(k) + l - k
        const int offk = k * n - k * (k - 1) / 2;
        for (int l = 0; l < k; l++) g += Q.q[l * n - l * (l - 1) / 2 + (k - l)] * bs[l][t];
        for (int l = k; l < n; l++) g += Q.q[offk + (l - k)] * bs[l][t];
        G[(size_t)k * natoms + atom] = g;
        e += bs[k][t] * (Q.beta[k] + g);
    }
    eatom[atom] = Q.beta0 + 0.5 * e;
}

template <int TJ>
static int launch_snap_quad(const SnapModel &m, ForcePath &fp, int inum, int nm, double *eatom, cudaStream_t s)
{
    const int nk = m.ncoeff;
    if (fp.B.ensure(sizeof(double) * (size_t)nk * inum) || fp.G.ensure(sizeof(double) * (size_t)nk * inum))
        return -1;
    if (launch_ui<double, TJ>(m, fp, inum, s)) return -1;
    if (fp.timing) cudaEventRecord(fp.ev[2], s);
    if (launch_bi_tiles(fp.Ut.as<double2>(), inum, TJ, m.p.bnormflag, m.p.bzeroflag, fp.B.as<double>(), inum, s))
        return -1;
    k_snap_quad<<<(inum + QUAD_THREADS - 1) / QUAD_THREADS, QUAD_THREADS, 0, s>>>(fp.B.as<double>(), inum, m.quad,
                                                                               fp.G.as<double>(), eatom);
    count_launches(2);
    if (launch_yi_pa_d(m, m.yq, fp, inum, fp.G.as<double>(), s)) return -1;
    return launch_fi<double, TJ>(m, fp, inum, nm, s);
}

template <typename T>
static int launch_snap_tj(const SnapModel &m, const YParams<T> &yp, ForcePath &fp, int inum, int nm, double *eatom,
                          cudaStream_t s)
{
    switch (m.p.twojmax) {
    case 4: return launch_snap<T, 4>(m, yp, fp, inum, nm, eatom, s);
    case 6: return launch_snap<T, 6>(m, yp, fp, inum, nm, eatom, s);
    case 8: return launch_snap<T, 8>(m, yp, fp, inum, nm, eatom, s);
    }
    set_error("twojmax %d not instantiated", m.p.twojmax);
    return -1;
}

// ---------------------------------------------------------------------------
// several element types (FP64): pairs grouped per (element block, atom), U
// over virtual atoms b * ipad + atom, energy from the element-triple
// bispectrum, Y per element block, dE/dr with per-pair cutoffs and weights
// ---------------------------------------------------------------------------
__global__ void k_elem_of_type(const int *__restrict__ atype, int inum, int ipad, int ne, int *__restrict__ elem)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ipad) return;
    int e = i < inum ? atype[i] - 1 : 0;   // map[t] = t - 1 (InitSnap); types checked by the callers
    elem[i] = e < 0 ? 0 : (e >= ne ? ne - 1 : e);
}

template <int TJ>
static int launch_snap_me(const SnapModel &m, ForcePath &fp, int inum, int nm, double *eatom, const MeArgs &A,
                          cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    const long nv = (long)A.nblk * A.ntiles * 32;
    fp.u_welem = (m.eg.chem && !m.p.wselfallflag) ? A.elem : nullptr;
    fp.u_ipad = A.ntiles * 32;
    const int rc_u = launch_ui<double, TJ>(m, fp, (int)nv, s);
    fp.u_welem = nullptr;
    fp.u_ipad = 0;
    if (rc_u) return -1;
    if (fp.timing) cudaEventRecord(fp.ev[2], s);
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_ei_me<TJ>, BI_WARPS * 32, 0, &per_sm, "k_snap_ei_me")) return -1;
    k_snap_ei_me<TJ><<<std::min(A.ntiles, num_sms() * per_sm), BI_WARPS * 32, 0, s>>>(
        fp.Ut.as<double2>(), inum, m.p.bnormflag, A, eatom);
    const size_t sm = yi_me_smem_bytes<TJ>();
    if (kernel_setup((const void *)k_snap_yi_me<TJ>, YiWarps<double, TJ>::n * 32, sm, &per_sm, "k_snap_yi_me"))
        return -1;
    k_snap_yi_me<TJ><<<std::min(A.ntiles, num_sms() * per_sm), YiWarps<double, TJ>::n * 32, sm, s>>>(
        fp.Ut.as<double2>(), inum, m.yq, A, fp.Y.as<double2>());
    count_launches(2);
    fp.fr_pcw = fp.pcw.as<double2>();
    const int rc_f = launch_fi<double, TJ>(m, fp, (int)nv, nm, s);
    fp.fr_pcw = nullptr;
    return rc_f;
}

static int force_compute_me(ForcePath &fp, const SnapModel &m, int precision, const double4 *x, int inum,
                            const int *nlist, const int *nnum, int nm, long pair_cap, const int *roff,
                            const long long *rlist, double *eatom, double4 *f, double *vatom, cudaStream_t s,
                            const int *atype, const int *alist)
{
    if (precision != MDP_PREC_FP64) { set_error("several element types run in FP64 only"); return -1; }
    if (!atype || !alist) { set_error("several element types need the atom types and the owner list"); return -1; }
    const int ntiles = (inum + 31) / 32, ipad = ntiles * 32;
    const int nblk = m.eg.nblk;
    const long nv = (long)nblk * ipad;
    if (nv >= (1L << 30)) { set_error("%d atoms x %d element blocks is too many", inum, nblk); return -1; }
    if (pair_cap < 1) pair_cap = 1;
    const size_t ncoef = (size_t)m.ne * m.p.ncoeffall;
    if (fp.pcount.ensure(sizeof(int) * (size_t)nv) || fp.poff.ensure(sizeof(int) * ((size_t)nv + 1)) ||
        fp.prij.ensure(sizeof(double4) * (size_t)pair_cap) || fp.pinfo.ensure(sizeof(int2) * (size_t)pair_cap) ||
        fp.pab.ensure(sizeof(double4) * (size_t)pair_cap) || fp.pcw.ensure(sizeof(double2) * (size_t)pair_cap) ||
        fp.smap.ensure(sizeof(int) * (size_t)inum * nm) || fp.dE.ensure(sizeof(double4) * (size_t)pair_cap) ||
        fp.Ut.ensure(sizeof(double2) * (size_t)nblk * ntiles * m.nu * 32) ||
        fp.Y.ensure(sizeof(double2) * (size_t)nblk * ntiles * 32 * m.nyh) ||
        fp.scan_tmp.ensure(sizeof(int) * scan_tmp_ints(nv)) || fp.elem.ensure(sizeof(int) * (size_t)ipad) ||
        fp.ecoef.ensure(sizeof(double) * ncoef))
        return -1;
    if (fp.timing && !fp.ev[0])
        for (auto &e : fp.ev) cudaEventCreate(&e);
    const int tb = 256;
    if (fp.timing) cudaEventRecord(fp.ev[0], s);
    MDP_CUDA_TRY(cudaMemcpyAsync(fp.ecoef.p, m.coeff.data(), sizeof(double) * ncoef, cudaMemcpyHostToDevice, s));
    k_elem_of_type<<<(ipad + tb - 1) / tb, tb, 0, s>>>(atype, inum, ipad, m.ne, fp.elem.as<int>());
    ElemGeom eg = m.eg;
    eg.ipad = ipad;
    MDP_CUDA_TRY(cudaMemsetAsync(fp.pcount.p, 0, sizeof(int) * (size_t)nv, s));
    const unsigned gw = (unsigned)(((long)inum * 32 + tb - 1) / tb);   // one warp per atom
    k_pair_count_me<<<gw, tb, 0, s>>>(x, nlist, nnum, inum, nm, alist, fp.elem.as<int>(), eg, fp.pcount.as<int>());
    if (exclusive_scan(fp.pcount.as<int>(), fp.poff.as<int>(), nv, fp.scan_tmp.as<int>(), s)) return -1;
    k_pair_emit_me<<<gw, tb, 0, s>>>(x, nlist, nnum, inum, nm, alist, fp.elem.as<int>(), fp.poff.as<int>(), m.geom,
                                     eg, fp.prij.as<double4>(), fp.pinfo.as<int2>(), fp.pab.as<double4>(),
                                     fp.pcw.as<double2>(), fp.smap.as<int>());
    MeArgs A;
    A.nblk = nblk;
    A.ntiles = ntiles;
    A.ncoeffall = m.p.ncoeffall;
    A.bzero = m.p.bzeroflag;
    A.wselfall = m.p.wselfallflag;
    A.elem = fp.elem.as<int>();
    A.coeff = fp.ecoef.as<double>();
    A.pa = 0;
    const int rc = m.p.twojmax == 8   ? launch_snap_me<8>(m, fp, inum, nm, eatom, A, s)
                   : m.p.twojmax == 6 ? launch_snap_me<6>(m, fp, inum, nm, eatom, A, s)
                                      : launch_snap_me<4>(m, fp, inum, nm, eatom, A, s);
    if (rc) return rc;
    if (fp.timing) cudaEventRecord(fp.ev[4], s);
    const int gb = (inum + tb - 1) / tb;
    k_tally<<<gb, tb, 0, s>>>(fp.prij.as<double4>(), fp.dE.as<double4>(), fp.poff.as<int>(), fp.smap.as<int>(), inum,
                              roff, rlist, f, vatom, nblk, ipad);
    count_launches(6);   // elem, pair_count, pair_emit, ui, fi, tally (+ the scan counts itself)
    if (m.zbl.on) {
        k_zbl<<<gb, tb, 0, s>>>(x, nlist, nnum, inum, nm, m.zbl, eatom, f, vatom);
        count_launches(1);
    }
    if (fp.timing) {
        cudaEventRecord(fp.ev[5], s);
        cudaEventSynchronize(fp.ev[5]);
        float t[5];
        for (int k = 0; k < 5; k++) cudaEventElapsedTime(&t[k], fp.ev[k], fp.ev[k + 1]);
        for (int k = 0; k < 5; k++) fp.stage_ms[k] += t[k];
        float tot;
        cudaEventElapsedTime(&tot, fp.ev[0], fp.ev[5]);
        fp.stage_ms[5] += tot;
        fp.stage_calls++;
    }
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int force_compute(ForcePath &fp, const SnapModel &m, int precision, const double4 *x, int inum, const int *nlist,
                  const int *nnum, int nm, long pair_cap, const int *roff, const long long *rlist, double *eatom,
                  double4 *f, double *vatom, cudaStream_t s, const int *atype, const int *alist)
{
    if (inum <= 0) { set_error("no atoms"); return -1; }
    if (m.ne > 1)
        return force_compute_me(fp, m, precision, x, inum, nlist, nnum, nm, pair_cap, roff, rlist, eatom, f, vatom,
                                s, atype, alist);
    const size_t tsz = (precision == MDP_PREC_FP32) ? sizeof(float2) : sizeof(double2);
    const long ntiles = (inum + 31) / 32;
    if (pair_cap < 1) pair_cap = 1;
    if (fp.pcount.ensure(sizeof(int) * (size_t)inum) || fp.poff.ensure(sizeof(int) * ((size_t)inum + 1)) ||
        fp.prij.ensure(sizeof(double4) * (size_t)pair_cap) || fp.pinfo.ensure(sizeof(int2) * (size_t)pair_cap) ||
        fp.pab.ensure(sizeof(double4) * (size_t)pair_cap) ||
        fp.smap.ensure(sizeof(int) * (size_t)inum * nm) || fp.dE.ensure(sizeof(double4) * (size_t)pair_cap) ||
        fp.Ut.ensure(tsz * (size_t)ntiles * m.nu * 32) || fp.Y.ensure(tsz * (size_t)ntiles * 32 * m.nyh) ||
        fp.scan_tmp.ensure(sizeof(int) * scan_tmp_ints(inum)))
        return -1;
    if (fp.timing && !fp.ev[0])
        for (auto &e : fp.ev) cudaEventCreate(&e);
    const int tb = 256;
    const int gb = (inum + tb - 1) / tb;
    if (fp.timing) cudaEventRecord(fp.ev[0], s);
    const unsigned gw = (unsigned)(((long)inum * 32 + tb - 1) / tb);   // one warp per atom
    k_pair_count<<<gw, tb, 0, s>>>(x, nlist, nnum, inum, nm, m.geom.rcutsq, fp.pcount.as<int>());
    if (exclusive_scan(fp.pcount.as<int>(), fp.poff.as<int>(), inum, fp.scan_tmp.as<int>(), s)) return -1;
    k_pair_emit<<<gw, tb, 0, s>>>(x, nlist, nnum, inum, nm, fp.poff.as<int>(), m.geom, fp.prij.as<double4>(),
                                  fp.pinfo.as<int2>(), fp.pab.as<double4>(), fp.smap.as<int>());
    int rc;
    if (m.p.quadraticflag) {
        if (precision != MDP_PREC_FP64) { set_error("quadratic SNAP runs in FP64 only"); return -1; }
        rc = m.p.twojmax == 8   ? launch_snap_quad<8>(m, fp, inum, nm, eatom, s)
             : m.p.twojmax == 6 ? launch_snap_quad<6>(m, fp, inum, nm, eatom, s)
                                : launch_snap_quad<4>(m, fp, inum, nm, eatom, s);
    } else {
        rc = (precision == MDP_PREC_FP32) ? launch_snap_tj<float>(m, m.yf, fp, inum, nm, eatom, s)
                                          : launch_snap_tj<double>(m, m.yd, fp, inum, nm, eatom, s);
    }
    if (rc) return rc;
    if (fp.timing) cudaEventRecord(fp.ev[4], s);
    k_tally<<<gb, tb, 0, s>>>(fp.prij.as<double4>(), fp.dE.as<double4>(), fp.poff.as<int>(), fp.smap.as<int>(), inum,
                              roff, rlist, f, vatom, 1, 0);
    count_launches(6);   // pair_count, pair_emit, ui, yi, fi, tally (+ the scan counts itself)
    if (m.zbl.on) {
        k_zbl<<<gb, tb, 0, s>>>(x, nlist, nnum, inum, nm, m.zbl, eatom, f, vatom);
        count_launches(1);
    }
    if (fp.timing) {
        cudaEventRecord(fp.ev[5], s);
        cudaEventSynchronize(fp.ev[5]);
        float t[5];
        for (int k = 0; k < 5; k++) cudaEventElapsedTime(&t[k], fp.ev[k], fp.ev[k + 1]);
        for (int k = 0; k < 5; k++) fp.stage_ms[k] += t[k];
        float tot;
        cudaEventElapsedTime(&tot, fp.ev[0], fp.ev[5]);
        fp.stage_ms[5] += tot;
        fp.stage_calls++;
    }
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// neighbour structure
// ---------------------------------------------------------------------------
int neighbor_build(Neighbors &nb, const BoxParams &bp, double4 *x, int inum, double rc, int nm, long anum_cap,
                   cudaStream_t s)
{
    const int tb = 256;
    if (nb.gcount.ensure(sizeof(int) * (size_t)inum) || nb.goff.ensure(sizeof(int) * ((size_t)inum + 1)) ||
        nb.gmask.ensure(sizeof(unsigned) * (size_t)inum) || nb.alist.ensure(sizeof(int) * (size_t)anum_cap) ||
        nb.cidx.ensure(sizeof(int) * (size_t)anum_cap) || nb.ccount.ensure(sizeof(int) * (size_t)bp.ncell) ||
        nb.cstart.ensure(sizeof(int) * ((size_t)bp.ncell + 1)) || nb.cursor.ensure(sizeof(int) * std::max((size_t)bp.ncell, (size_t)inum)) ||
        nb.catoms.ensure(sizeof(int) * (size_t)anum_cap) || nb.nlist.ensure(sizeof(int) * (size_t)inum * nm) ||
        nb.nnum.ensure(sizeof(int) * (size_t)inum) || nb.rcount.ensure(sizeof(int) * (size_t)inum) ||
        nb.roff.ensure(sizeof(int) * ((size_t)inum + 1)) || nb.rlist.ensure(sizeof(long long) * (size_t)inum * nm) ||
        nb.status.ensure(sizeof(int) * 4) ||
        nb.scan_tmp.ensure(sizeof(int) * scan_tmp_ints(std::max((long)inum, bp.ncell))))
        return -1;
    int *tmp = nb.scan_tmp.as<int>();
    k_ghost_count<<<(inum + tb - 1) / tb, tb, 0, s>>>(x, inum, bp, nb.gcount.as<int>(), nb.gmask.as<unsigned>());
    if (exclusive_scan(nb.gcount.as<int>(), nb.goff.as<int>(), inum, tmp, s)) return -1;
    int gnum = 0;
    MDP_CUDA_TRY(cudaMemcpyAsync(&gnum, nb.goff.as<int>() + inum, sizeof(int), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaStreamSynchronize(s));
    if ((long)inum + gnum > anum_cap) {
        set_error("ghost capacity exceeded: %d local + %d ghosts > %ld", inum, gnum, anum_cap);
        return -1;
    }
    const int anum = inum + gnum;
    k_ghost_emit<<<(inum + tb - 1) / tb, tb, 0, s>>>(x, nb.alist.as<int>(), inum, bp, nb.goff.as<int>(),
                                                     nb.gmask.as<unsigned>());
    MDP_CUDA_TRY(cudaMemsetAsync(nb.ccount.p, 0, sizeof(int) * bp.ncell, s));
    k_cell_index<<<(anum + tb - 1) / tb, tb, 0, s>>>(x, anum, bp, nb.cidx.as<int>(), nb.ccount.as<int>());
    if (exclusive_scan(nb.ccount.as<int>(), nb.cstart.as<int>(), bp.ncell, tmp, s)) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(nb.cursor.p, 0, sizeof(int) * bp.ncell, s));
    k_cell_fill<<<(anum + tb - 1) / tb, tb, 0, s>>>(anum, nb.cidx.as<int>(), nb.cstart.as<int>(), nb.cursor.as<int>(),
                                                    nb.catoms.as<int>());
    MDP_CUDA_TRY(cudaMemsetAsync(nb.status.p, 0, sizeof(int), s));
    k_neigh_build<<<(inum + 127) / 128, 128, 0, s>>>(x, inum, bp, nb.cidx.as<int>(), nb.cstart.as<int>(),
                                                     nb.catoms.as<int>(), rc * rc, nm, nb.nlist.as<int>(),
                                                     nb.nnum.as<int>(), nb.status.as<int>());
    MDP_CUDA_TRY(cudaMemsetAsync(nb.rcount.p, 0, sizeof(int) * inum, s));
    k_rev_count<<<(inum + tb - 1) / tb, tb, 0, s>>>(nb.nlist.as<int>(), nb.nnum.as<int>(), nb.alist.as<int>(), inum,
                                                    nm, nb.rcount.as<int>());
    if (exclusive_scan(nb.rcount.as<int>(), nb.roff.as<int>(), inum, tmp, s)) return -1;
    MDP_CUDA_TRY(cudaMemsetAsync(nb.cursor.p, 0, sizeof(int) * inum, s));
    k_rev_fill<<<(inum + tb - 1) / tb, tb, 0, s>>>(nb.nlist.as<int>(), nb.nnum.as<int>(), nb.alist.as<int>(), inum, nm,
                                                   nb.roff.as<int>(), nb.cursor.as<int>(), nb.rlist.as<long long>());
    k_rev_sort<<<std::min((inum + 7) / 8, num_sms() * 8), 256, 0, s>>>(inum, nb.roff.as<int>(), nb.rlist.as<long long>());
    count_launches(8);
    int hs[2] = {0, 0};
    MDP_CUDA_TRY(cudaMemcpyAsync(&hs[0], nb.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaMemcpyAsync(&hs[1], nb.roff.as<int>() + inum, sizeof(int), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaStreamSynchronize(s));
    MDP_CUDA_TRY(cudaGetLastError());
    if (hs[0] & 1) {
        set_error("neighbour list overflow: an atom has more than neighmax=%d neighbours within %.4f A", nm, rc);
        return -1;
    }
    nb.inum = inum;
    nb.gnum = gnum;
    nb.anum = anum;
    nb.nm = nm;
    nb.nsum = hs[1];
    nb.anum_cap = anum_cap;
    return 0;
}

}  // namespace mdp
