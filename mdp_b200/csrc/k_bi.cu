// Per-atom bispectrum launcher (k_snap_bi) on U tiles.
#include "engine.h"

#include <algorithm>

namespace mdp {

template <typename T, int TJ>
static int launch_bi(const typename cplx<T>::type *Ut, int natoms, int bnorm, int bzero, double *bout, long bstride,
                     cudaStream_t s)
{
    if (tu_ensure_tables()) return -1;
    const size_t sm = (size_t)idxu_count(TJ) * 32 * sizeof(typename cplx<T>::type);
    int per_sm = 0;
    if (kernel_setup((const void *)k_snap_bi<T, TJ>, BI_WARPS * 32, sm, &per_sm, "k_snap_bi")) return -1;
    const int blocks = std::min((natoms + 31) / 32, num_sms() * per_sm);
    k_snap_bi<T, TJ><<<blocks, BI_WARPS * 32, sm, s>>>(Ut, natoms, bnorm, bzero, bout, bstride);
    count_launches(1);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

int launch_bi_tiles(const double2 *Ut, int natoms, int tj, int bnorm, int bzero, double *bout, long bstride,
                    cudaStream_t s)
{
    switch (tj) {
    case 4: return launch_bi<double, 4>(Ut, natoms, bnorm, bzero, bout, bstride, s);
    case 6: return launch_bi<double, 6>(Ut, natoms, bnorm, bzero, bout, bstride, s);
    case 8: return launch_bi<double, 8>(Ut, natoms, bnorm, bzero, bout, bstride, s);
    }
    set_error("twojmax %d not supported", tj);
    return -1;
}

int launch_bi_tiles_f32(const float2 *Ut, int natoms, int tj, int bnorm, int bzero, double *bout, long bstride,
                        cudaStream_t s)
{
    switch (tj) {
    case 4: return launch_bi<float, 4>(Ut, natoms, bnorm, bzero, bout, bstride, s);
    case 6: return launch_bi<float, 6>(Ut, natoms, bnorm, bzero, bout, bstride, s);
    case 8: return launch_bi<float, 8>(Ut, natoms, bnorm, bzero, bout, bstride, s);
    }
    set_error("twojmax %d not supported", tj);
    return -1;
}

}  // namespace mdp
