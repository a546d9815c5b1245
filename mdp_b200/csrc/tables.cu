// Host construction and device upload of the SNAP constant tables, the error
// channel, and a device-wide exclusive scan used by the neighbour and pair
// builders.
#include "common.cuh"

#include <math.h>
#include <stdarg.h>
#include <string.h>
#include <mutex>
#include <atomic>
#include <vector>

namespace mdp {

static thread_local char g_err[1024] = "";
static std::atomic<long long> g_launches{0};
void count_launches(long n) { g_launches += n; }
long long launch_count() { return g_launches.load(); }

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char *get_error() { return g_err; }

static int current_device(int *dev)
{
    if (cudaGetDevice(dev) != cudaSuccess || *dev < 0) {
        set_error("no current CUDA device");
        return -1;
    }
    return 0;
}

static PerDeviceMemo g_sms, g_kernels;

// every translation unit's constant-table filler, run once per device
namespace {
struct FillerRegistry {
    std::mutex mu;
    std::vector<int (*)()> fillers;
    bool done[64] = {};
};
FillerRegistry &filler_registry()
{
    static FillerRegistry r;   // constructed on first use, during static initialisation
    return r;
}
}  // namespace

void register_table_filler(int (*fill)())
{
    FillerRegistry &r = filler_registry();
    std::lock_guard<std::mutex> lk(r.mu);
    r.fillers.push_back(fill);
}

int ensure_all_tables()
{
    int dev = 0;
    if (current_device(&dev)) return -1;
    if (dev >= 64) { set_error("device index %d out of range", dev); return -1; }
    FillerRegistry &r = filler_registry();
    std::lock_guard<std::mutex> lk(r.mu);
    if (r.done[dev]) return 0;
    for (auto fill : r.fillers)
        if (fill()) return -1;
    r.done[dev] = true;
    return 0;
}

int num_sms()
{
    int dev = 0, n = 0;
    if (current_device(&dev)) return 148;
    auto setup = [dev](int *v) {
        if (cudaDeviceGetAttribute(v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || *v <= 0) return -1;
        return 0;
    };
    if (g_sms.get(nullptr, 0, dev, setup, &n)) return 148;
    return n;
}

int kernel_setup(const void *fn, int threads, size_t smem, int *per_sm, const char *name)
{
    int dev = 0;
    if (current_device(&dev)) return -1;
    auto setup = [&](int *v) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(v, fn, threads, smem);
        if (e != cudaSuccess) {
            set_error("%s: launch set-up with %zu B shared memory failed on device %d: %s", name, smem, dev,
                      cudaGetErrorString(e));
            return -1;
        }
        if (*v < 1) {
            set_error("%s does not fit on an SM of device %d (%zu B shared, %d threads)", name, dev, smem, threads);
            return -1;
        }
        return 0;
    };
    return g_kernels.get(fn, ((long)smem << 16) | threads, dev, setup, per_sm);
}

// Clebsch-Gordan coefficients by the Racah formula, in the block order of
// src/C++/Core/cpuSnap.cpp:137-193 (aa2, bb2, cc2 are doubled m values).
void host_cg_table(double *cg)
{
    double fac[40];
    fac[0] = 1.0;
    for (int i = 1; i < 40; i++) fac[i] = fac[i - 1] * i;
    int k = 0;
    for (int j1 = 0; j1 <= TJMAX; j1++)
        for (int j2 = 0; j2 <= j1; j2++)
            for (int j = j1 - j2; j <= cmin(TJMAX, j1 + j2); j += 2)
                for (int m1 = 0; m1 <= j1; m1++)
                    for (int m2 = 0; m2 <= j2; m2++, k++) {
                        int aa2 = 2 * m1 - j1, bb2 = 2 * m2 - j2;
                        int m = (aa2 + bb2 + j) / 2;
                        if (m < 0 || m > j) { cg[k] = 0.0; continue; }
                        int zlo = cmax(0, cmax(-(j - j2 + aa2) / 2, -(j - j1 - bb2) / 2));
                        int zhi = cmin((j1 + j2 - j) / 2, cmin((j1 - aa2) / 2, (j2 + bb2) / 2));
                        double sum = 0.0;
                        for (int z = zlo; z <= zhi; z++) {
                            double den = fac[z] * fac[(j1 + j2 - j) / 2 - z] * fac[(j1 - aa2) / 2 - z] *
                                         fac[(j2 + bb2) / 2 - z] * fac[(j - j2 + aa2) / 2 + z] *
                                         fac[(j - j1 - bb2) / 2 + z];
                            sum += ((z & 1) ? -1.0 : 1.0) / den;
                        }
                        int cc2 = 2 * m - j;
                        double tri = sqrt(fac[(j1 + j2 - j) / 2] * fac[(j1 - j2 + j) / 2] *
                                          fac[(-j1 + j2 + j) / 2] / fac[(j1 + j2 + j) / 2 + 1]);
                        double norm = sqrt(fac[(j1 + aa2) / 2] * fac[(j1 - aa2) / 2] * fac[(j2 + bb2) / 2] *
                                           fac[(j2 - bb2) / 2] * fac[(j + cc2) / 2] * fac[(j - cc2) / 2] *
                                           (j + 1));
                        cg[k] = sum * tri * norm;
                    }
}

void host_rootpq_table(double *rp)
{
    for (int p = 0; p < JD; p++)
        for (int q = 0; q < JD; q++)
            rp[p * JD + q] = (p >= 1 && q >= 1) ? sqrt((double)p / q) : 0.0;
}

// Row mb of U at layer J is u[ma] = unorm(J, mb, ma) * v[ma], where v obeys the
// coefficient-free recursion v_J[ma] = conj(a) v_(J-1)[ma] - conj(b) v_(J-1)[ma-1]
// (the sqrt(ma!(J-ma)!/(mb!(J-mb)!)) normalisation of the Wigner D-matrix,
// which turns cpuSnap4.cpp's rootpq factors into ratios of these numbers).
void host_unorm_table(double *un)
{
    double fac[2 * JD];
    fac[0] = 1.0;
    for (int i = 1; i < 2 * JD; i++) fac[i] = fac[i - 1] * i;
    for (int j = 0; j < JD; j++)
        for (int mb = 0; mb < JD; mb++)
            for (int ma = 0; ma < JD; ma++)
                un[(j * JD + mb) * JD + ma] =
                    (mb <= j && ma <= j) ? sqrt(fac[ma] * fac[j - ma] / (fac[j - mb] * fac[mb])) : 0.0;
}

// ---------------------------------------------------------------------------
// exclusive scan: 4096 elements per block (1024 threads x 4), two levels
// ---------------------------------------------------------------------------
constexpr int SCAN_T = 1024, SCAN_V = 4, SCAN_B = SCAN_T * SCAN_V;

__device__ __forceinline__ int block_scan_excl(int v, int *sh, int *total)
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = sh[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    int pre = (w > 0 ? sh[w - 1] : 0) + x - v;
    if (total) *total = sh[31];
    __syncthreads();
    return pre;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_local(const int *__restrict__ in, int *__restrict__ out,
                                                       long n, int *__restrict__ bsum)
{
    __shared__ int sh[32];
    long base = (long)blockIdx.x * SCAN_B + threadIdx.x * SCAN_V;
    int v[SCAN_V], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; k++) { v[k] = (base + k < n) ? in[base + k] : 0; s += v[k]; }
    int tot;
    int pre = block_scan_excl(s, sh, &tot);
#pragma unroll
    for (int k = 0; k < SCAN_V; k++) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_top(int *__restrict__ bsum, int nb, int *__restrict__ total_out)
{
    __shared__ int sh[32];
    int v[SCAN_V], s = 0;
    int base = threadIdx.x * SCAN_V;
#pragma unroll
    for (int k = 0; k < SCAN_V; k++) { v[k] = (base + k < nb) ? bsum[base + k] : 0; s += v[k]; }
    int tot;
    int pre = block_scan_excl(s, sh, &tot);
#pragma unroll
    for (int k = 0; k < SCAN_V; k++) {
        if (base + k < nb) bsum[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) *total_out = tot;
}

__global__ void k_scan_add(int *__restrict__ out, long n, const int *__restrict__ bsum)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += bsum[i / SCAN_B];
}

size_t scan_tmp_ints(long n) { return (size_t)((n + SCAN_B - 1) / SCAN_B) + 8; }

int exclusive_scan(const int *in, int *out, long n, int *tmp, cudaStream_t s)
{
    long nb = (n + SCAN_B - 1) / SCAN_B;
    if (nb > SCAN_B) { set_error("scan length %ld exceeds %ld", n, (long)SCAN_B * SCAN_B); return -1; }
    if (n == 0) {
        MDP_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int), s));
        return 0;
    }
    k_scan_local<<<(unsigned)nb, SCAN_T, 0, s>>>(in, out, n, tmp);
    k_scan_top<<<1, SCAN_T, 0, s>>>(tmp, (int)nb, out + n);
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, tmp);
    count_launches(3);
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mdp
