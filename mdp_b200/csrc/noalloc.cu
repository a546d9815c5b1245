// Per-atom bispectrum for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc: code embedded in a host application whose
// memory pool already owns the device memory (a stray cudaMalloc fails or
// fragments it), and loops that cannot afford the implicit device-wide
// synchronisation that cudaMalloc/cudaFree can cause.  The existing entry point
// mdp_gpu_snap_compute_bi_f64 stages U into a 32-atom-tile scratch buffer it
// allocates on first use.  This variant keeps that scratch in a fixed array
// compiled into the library instead, so a call allocates nothing.
//
// Limits and sharing:
//   * at most NOALLOC_MAX_ATOMS (2048) atoms per call; 2J = 4, 6 or 8;
//   * the array (2048 x 285 complex doubles = 9,338,880 bytes) lives on every
//     GPU that loads the library, for the life of the process;
//   * all calls share it and it keeps the last call's contents, so calls whose
//     GPU work overlaps (different streams, or different host threads on one
//     device) race; serialise them on one stream;
//   * the first call on a device looks up the array's device address and the
//     library uploads its constant tables there: make that first call before
//     starting any stream capture.
#include "common.cuh"
#include "engine.h"

#include <mutex>

namespace mdp {

constexpr int NOALLOC_MAX_ATOMS = 2048;
constexpr int NOALLOC_NU = idxu_count(TJMAX);   // room for any 2J <= 8

// The scratch itself.  In host code this name is only a stand-in for the
// device object; kernels get its device address from cudaGetSymbolAddress.
static __device__ __align__(256) double2 g_bi_scratch[NOALLOC_MAX_ATOMS * NOALLOC_NU];

int launch_bi_tiles(const double2 *Ut, int natoms, int tj, int bnorm, int bzero, double *bout, long bstride,
                    cudaStream_t s);

// U in MDP's layout [idxu][inum] -> 32-atom tiles in the static scratch;
// the unused lanes of the last tile are written as zeros so no stale values
// from an earlier call are read.
__global__ void k_uref_to_noalloc_tiles(const double *__restrict__ ur, const double *__restrict__ ui, int inum, int nu,
                                        int ntiles)
{
    const long n = (long)ntiles * 32 * nu;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int slots = ntiles * 32;
    const int i = (int)(t % slots), k = (int)(t / slots);
    const double2 v = (i < inum) ? make_double2(ur[(size_t)k * inum + i], ui[(size_t)k * inum + i])
                                 : make_double2(0.0, 0.0);
    g_bi_scratch[(size_t)(i >> 5) * nu * 32 + (size_t)k * 32 + (i & 31)] = v;
}

static std::mutex g_noalloc_mu;
static double2 *g_noalloc_ptr[64];

// device address of the scratch on the current device, looked up once per device
static int noalloc_scratch(double2 **out)
{
    int dev = 0;
    MDP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { set_error("device index %d out of range", dev); return -1; }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        double2 *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_bi_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(bispectrum scratch) failed: %s", cudaGetErrorString(e));
            return -1;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

}  // namespace mdp

using namespace mdp;

extern "C" int mdp_gpu_snap_compute_bi_noalloc_f64(double *blist, const double *Utotr, const double *Utoti,
                                                    int twojmax, int bnorm_flag, int bzero_flag, int inum,
                                                    void *stream)
{
    if (!blist || !Utotr || !Utoti) { set_error("null pointer argument"); return -1; }
    if (twojmax != 4 && twojmax != 6 && twojmax != 8) {
        set_error("twojmax=%d not supported (4, 6 or 8)", twojmax);
        return -1;
    }
    if (inum <= 0 || inum > NOALLOC_MAX_ATOMS) {
        set_error("inum=%d outside 1..%d, the size of the fixed scratch of the allocation-free entry point",
                  inum, NOALLOC_MAX_ATOMS);
        return -1;
    }
    double2 *scratch = nullptr;
    if (noalloc_scratch(&scratch)) return -1;
    cudaStream_t s = (cudaStream_t)stream;
    const int nu = idxu_count(twojmax);
    const int ntiles = (inum + 31) / 32;
    const long n = (long)ntiles * 32 * nu;
    k_uref_to_noalloc_tiles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Utotr, Utoti, inum, nu, ntiles);
    count_launches(1);
    MDP_CUDA_TRY(cudaGetLastError());
    return launch_bi_tiles(scratch, inum, twojmax, bnorm_flag, bzero_flag, blist, inum, s);
}
