// Shared definitions for the B200 SNAP force path: compile-time index
// arithmetic, constant-memory tables, error plumbing.
//
// Index conventions are MDP's (src/C++/Core/cpuSnap.cpp:14-115):
//   U element (j, mb, ma) lives at idxu_block(j) + (j+1)*mb + ma,
//   Clebsch-Gordan blocks are enumerated j1 >= j2, j = j1-j2 .. min(2J, j1+j2)
//   step 2, each block (j1+1)*(j2+1) long.
// All tables are built for 2J <= 8 (TJMAX).  Because a CG coefficient only
// depends on its own indices, the TJMAX enumeration serves every 2J <= 8.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <mutex>

#include "device_cache.h"

namespace mdp {

constexpr int TJMAX = 8;
constexpr int JD = TJMAX + 1;

__host__ __device__ constexpr int idxu_block(int j) { return j * (j + 1) * (2 * j + 1) / 6; }
__host__ __device__ constexpr int idxu_count(int tj) { return idxu_block(tj + 1); }

// half-plane (rows mb <= j/2) compact index used for Y and dE/dU work
__host__ __device__ constexpr int yh_block(int j)
{
    int n = 0;
    for (int jj = 0; jj < j; jj++) n += (jj + 1) * (jj / 2 + 1);
    return n;
}
__host__ __device__ constexpr int yh_count(int tj) { return yh_block(tj + 1); }

__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// offset of CG block (j1, j2, j) in the TJMAX enumeration
__host__ __device__ constexpr int cg_block(int j1, int j2, int j)
{
    int n = 0;
    for (int a = 0; a <= TJMAX; a++)
        for (int b = 0; b <= a; b++)
            for (int c = a - b; c <= cmin(TJMAX, a + b); c += 2) {
                if (a == j1 && b == j2 && c == j) return n;
                n += (a + 1) * (b + 1);
            }
    return -1;
}
constexpr int NCG = cg_block(TJMAX, TJMAX, TJMAX) + (TJMAX + 1) * (TJMAX + 1);

// index of a coupling triple (j1 >= j2) in per-triple coefficient tables
__host__ __device__ constexpr int tri_index(int j1, int j2, int j) { return (j1 * (j1 + 1) / 2 + j2) * JD + j; }
constexpr int NTRI = (TJMAX + 1) * (TJMAX + 2) / 2 * JD;

// host-side table construction (tables.cu)
void host_cg_table(double *cg /*NCG*/);
void host_rootpq_table(double *rp /*JD*JD*/);
void host_unorm_table(double *un /*JD*JD*JD*/);
void set_error(const char *fmt, ...);
const char *get_error();

// rootpq[p][q] = sqrt(p/q) (src/C++/Core/cpuSnap.cpp:117-123) and the CG list.
// Every translation unit that launches SNAP kernels holds its own copy and
// fills it through tu_ensure_tables() before its first launch on a device.
static __constant__ double c_rootpq_d[JD * JD];
static __constant__ float c_rootpq_f[JD * JD];
// unorm[(J*JD + mb)*JD + ma] = sqrt(ma! (J-ma)! / ((J-mb)! mb!)): the factor
// between a U entry of row mb, layer J and its coefficient-free form (below)
static __constant__ double c_unorm_d[JD * JD * JD];
static __constant__ float c_unorm_f[JD * JD * JD];
static __constant__ double c_cg_d[NCG];
static __constant__ float c_cg_f[NCG];

// Uploads this translation unit's copy of the tables to the current device.
static int tu_fill_tables()
{
    static double cg[NCG], rp[JD * JD], un[JD * JD * JD];
    static float cgf[NCG], rpf[JD * JD], unf[JD * JD * JD];
    host_cg_table(cg);
    host_rootpq_table(rp);
    host_unorm_table(un);
    for (int i = 0; i < NCG; i++) cgf[i] = (float)cg[i];
    for (int i = 0; i < JD * JD; i++) rpf[i] = (float)rp[i];
    for (int i = 0; i < JD * JD * JD; i++) unf[i] = (float)un[i];
    if (cudaMemcpyToSymbol(c_cg_d, cg, sizeof(cg)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_cg_f, cgf, sizeof(cgf)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_rootpq_d, rp, sizeof(rp)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_rootpq_f, rpf, sizeof(rpf)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_unorm_d, un, sizeof(un)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_unorm_f, unf, sizeof(unf)) != cudaSuccess) {
        set_error("uploading SNAP constant tables failed");
        return -1;
    }
    return 0;
}

// A kernel template instantiated in several translation units has one host
// launch stub, so a launch may run the instantiation compiled into another
// unit, which reads that unit's tables.  Every unit therefore registers its
// filler at load time (tables.cu keeps the list), and the first
// tu_ensure_tables() on a device fills all units' copies there.
void register_table_filler(int (*fill)());
int ensure_all_tables();
struct TableFillerRegistration {
    explicit TableFillerRegistration(int (*fill)()) { register_table_filler(fill); }
};
static TableFillerRegistration tu_table_filler_registration(&tu_fill_tables);

static inline int tu_ensure_tables() { return ensure_all_tables(); }

// SM count of the current device (cached per device).
int num_sms();

// Launch set-up of a kernel on the current device: raises its dynamic
// shared-memory limit to smem bytes and returns in *per_sm how many CTAs of
// `threads` threads fit on one SM.  Done once per (kernel, device) under a
// lock; cudaFuncSetAttribute is per device, so a second GPU in the same
// process gets its own set-up.  Returns -1 (error set) if the kernel cannot
// launch with that much shared memory.
int kernel_setup(const void *fn, int threads, size_t smem, int *per_sm, const char *name);

template <typename T> struct cplx;
template <> struct cplx<double> { typedef double2 type; };
template <> struct cplx<float> { typedef float2 type; };

template <typename T> __device__ __forceinline__ T rootpq(int p, int q);
template <> __device__ __forceinline__ double rootpq<double>(int p, int q) { return c_rootpq_d[p * JD + q]; }
template <> __device__ __forceinline__ float rootpq<float>(int p, int q) { return c_rootpq_f[p * JD + q]; }

template <typename T> __device__ __forceinline__ T unorm(int j, int mb, int ma);
template <> __device__ __forceinline__ double unorm<double>(int j, int mb, int ma) { return c_unorm_d[(j * JD + mb) * JD + ma]; }
template <> __device__ __forceinline__ float unorm<float>(int j, int mb, int ma) { return c_unorm_f[(j * JD + mb) * JD + ma]; }

template <typename T> __device__ __forceinline__ T cgc(int k);
template <> __device__ __forceinline__ double cgc<double>(int k) { return c_cg_d[k]; }
template <> __device__ __forceinline__ float cgc<float>(int k) { return c_cg_f[k]; }


#define MDP_CUDA_TRY(call)                                                         \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) {                                                   \
            ::mdp::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                             cudaGetErrorString(_e));                              \
            return -1;                                                             \
        }                                                                          \
    } while (0)

// count of kernels this library has launched (all streams, all devices)
void count_launches(long n);
long long launch_count();

// exclusive scan of n ints (n <= 16M) into out[0..n]; out[n] = total.
// tmp must hold scan_tmp_ints(n) ints.
size_t scan_tmp_ints(long n);
int exclusive_scan(const int *in, int *out, long n, int *tmp, cudaStream_t s);

}  // namespace mdp
