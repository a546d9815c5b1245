// dE/dr stage launchers (k_snap_fr, reverse-mode dE/dr), double.
#include "engine.h"

#include <algorithm>

namespace mdp {

template <typename T, int TJ>
int launch_fi(const SnapModel &m, ForcePath &fp, int inum, int /*nm*/, cudaStream_t s)
{
    typedef typename cplx<T>::type T2;
    if (tu_ensure_tables()) return -1;
    if (fp.timing) cudaEventRecord(fp.ev[3], s);
    const size_t sm = fr_smem_bytes<T, TJ>();
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_fr<T, TJ>, FR_THREADS, sm, &per_sm, "k_snap_fr")) return -1;
    const int blocks = num_sms() * per_sm;
    k_snap_fr<T, TJ><<<blocks, FR_THREADS, sm, s>>>(fp.prij.as<double4>(), fp.pinfo.as<int2>(),
                                                    fp.poff.as<int>() + inum, m.geom, fp.Y.as<T2>(),
                                                    fp.dE.as<double4>(), fp.fr_pcw);
    return 0;
}

#define MDP_INST(T, TJ) template int launch_fi<T, TJ>(const SnapModel &, ForcePath &, int, int, cudaStream_t);
MDP_INST(double, 4) MDP_INST(double, 6) MDP_INST(double, 8)
#undef MDP_INST

}  // namespace mdp
