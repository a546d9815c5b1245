// Y + energy stage launchers (k_snap_yi), double.
#include "engine.h"

#include <algorithm>

namespace mdp {

template <typename T, int TJ>
int launch_yi(const SnapModel &m, const YParams<T> &yp, ForcePath &fp, int inum, double *eatom, cudaStream_t s)
{
    typedef typename cplx<T>::type T2;
    if (tu_ensure_tables()) return -1;
    const size_t sm = yi_smem_bytes<T, TJ>();
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_yi<T, TJ>, YiWarps<T, TJ>::n * 32, sm, &per_sm, "k_snap_yi")) return -1;
    const int ntiles = (inum + 31) / 32;
    const int blocks = std::min(ntiles, num_sms() * per_sm);
    if (fp.timing) cudaEventRecord(fp.ev[2], s);
    k_snap_yi<T, TJ><<<blocks, YiWarps<T, TJ>::n * 32, sm, s>>>(fp.Ut.as<T2>(), inum, yp, fp.Y.as<T2>(), eatom);
    return 0;
}

// per-atom coefficients G [k][atom] (k over the bispectrum components), FP64:
// the beta form of the reference's Yi (cpuSnap4.cpp:601-691); no energy
template <int TJ>
static int launch_yi_pa_d_tj(const YParams<double> &yp, ForcePath &fp, int inum, const double *G, cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    const size_t sm = yi_smem_bytes<double, TJ, true>();
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_yi<double, TJ, true>, YiWarps<double, TJ>::n * 32, sm, &per_sm,
                     "k_snap_yi (per-atom, FP64)"))
        return -1;
    const int ntiles = (inum + 31) / 32;
    const int blocks = std::min(ntiles, num_sms() * per_sm);
    k_snap_yi<double, TJ, true><<<blocks, YiWarps<double, TJ>::n * 32, sm, s>>>(fp.Ut.as<double2>(), inum, yp,
                                                                            fp.Y.as<double2>(), nullptr, G);
    return 0;
}

// yp: the per-triple factors of a model whose coefficients are all 1
int launch_yi_pa_d(const SnapModel &m, const YParams<double> &yp, ForcePath &fp, int inum, const double *G,
                   cudaStream_t s)
{
    switch (m.p.twojmax) {
    case 4: return launch_yi_pa_d_tj<4>(yp, fp, inum, G, s);
    case 6: return launch_yi_pa_d_tj<6>(yp, fp, inum, G, s);
    case 8: return launch_yi_pa_d_tj<8>(yp, fp, inum, G, s);
    }
    set_error("twojmax %d not supported", m.p.twojmax);
    return -1;
}

#define MDP_INST(T, TJ) \
    template int launch_yi<T, TJ>(const SnapModel &, const YParams<T> &, ForcePath &, int, double *, cudaStream_t);
MDP_INST(double, 4) MDP_INST(double, 6) MDP_INST(double, 8)
#undef MDP_INST

}  // namespace mdp
