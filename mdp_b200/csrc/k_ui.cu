// U stage launchers (k_snap_ui), all precisions.
#include "engine.h"

#include <algorithm>

namespace mdp {

template <typename T, int TJ>
int launch_ui(const SnapModel &m, ForcePath &fp, int inum, cudaStream_t s)
{
    typedef typename cplx<T>::type T2;
    if (tu_ensure_tables()) return -1;
    constexpr int NU = idxu_count(TJ);
    const size_t sm = (size_t)UI_WARPS * (NU + 32 * (TJ + 1)) * sizeof(T2);
    static bool attr = false;
    if (!attr) {
        MDP_CUDA_TRY(cudaFuncSetAttribute(k_snap_ui<T, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        attr = true;
    }
    const int blocks = std::min((inum + UI_WARPS - 1) / UI_WARPS, num_sms() * 16);
    if (fp.timing) cudaEventRecord(fp.ev[1], s);
    k_snap_ui<T, TJ><<<blocks, UI_WARPS * 32, sm, s>>>(fp.poff.as<int>(), fp.prij.as<double4>(), inum, m.geom,
                                                       fp.Ut.as<T2>());
    return 0;
}

#define MDP_INST(T, TJ) template int launch_ui<T, TJ>(const SnapModel &, ForcePath &, int, cudaStream_t);
MDP_INST(double, 4) MDP_INST(double, 6) MDP_INST(double, 8)
MDP_INST(float, 4) MDP_INST(float, 6) MDP_INST(float, 8)
#undef MDP_INST

}  // namespace mdp
