// Y + energy stage launchers (k_snap_yi), float.
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

// per-atom coefficients G [k][atom] (the surrogate's dE_i/dB_ik), 2J=4, float
int launch_yi_pa_f4(const SnapModel &m, ForcePath &fp, int inum, const float *G, cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    const size_t sm = yi_smem_bytes<float, 4, true>();
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_yi<float, 4, true>, YiWarps<float, 4>::n * 32, sm, &per_sm,
                     "k_snap_yi (per-atom)"))
        return -1;
    const int ntiles = (inum + 31) / 32;
    const int blocks = std::min(ntiles, num_sms() * per_sm);
    if (fp.timing) cudaEventRecord(fp.ev[2], s);
    k_snap_yi<float, 4, true><<<blocks, YiWarps<float, 4>::n * 32, sm, s>>>(fp.Ut.as<float2>(), inum, m.yf,
                                                                         fp.Y.as<float2>(), nullptr, G);
    return 0;
}

#define MDP_INST(T, TJ) \
    template int launch_yi<T, TJ>(const SnapModel &, const YParams<T> &, ForcePath &, int, double *, cudaStream_t);
MDP_INST(float, 4) MDP_INST(float, 6) MDP_INST(float, 8)
#undef MDP_INST

}  // namespace mdp
