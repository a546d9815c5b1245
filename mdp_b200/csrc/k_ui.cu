// U stage launchers (k_snap_uc), all precisions.
#include "engine.h"

#include <algorithm>

namespace mdp {

template <typename T, int TJ>
int launch_ui(const SnapModel &m, ForcePath &fp, int inum, cudaStream_t s)
{
    typedef typename cplx<T>::type T2;
    if (tu_ensure_tables()) return -1;
    const size_t sm = uc_smem_bytes<T, TJ>();
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_uc<T, TJ>, uc_warps<T, TJ>() * 32, sm, &per_sm, "k_snap_uc")) return -1;
    const int ntiles = (inum + 31) / 32;
    const int blocks = std::min(ntiles, num_sms() * per_sm);
    if (fp.timing) cudaEventRecord(fp.ev[1], s);
    k_snap_uc<T, TJ><<<blocks, uc_warps<T, TJ>() * 32, sm, s>>>(fp.poff.as<int>(), fp.prij.as<double4>(),
                                                             fp.pab.as<double4>(), inum, fp.Ut.as<T2>(),
                                                             fp.u_welem, fp.u_ipad);
    return 0;
}

#define MDP_INST(T, TJ) template int launch_ui<T, TJ>(const SnapModel &, ForcePath &, int, cudaStream_t);
MDP_INST(double, 4) MDP_INST(double, 6) MDP_INST(double, 8)
MDP_INST(float, 4) MDP_INST(float, 6) MDP_INST(float, 8)
#undef MDP_INST

}  // namespace mdp
