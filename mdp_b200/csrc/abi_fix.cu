// Force constraints ("fixes"), the set-velocity integrator and the velocity-
// rescaling thermostats behind MDP's backend dispatch (src/C++/Common/
// mdpgpucore.h:303-349, called from the inline wrappers of mdpcore.h with
// backend == 2 by Integration.cpp's PostInitialIntegration /
// PostFinalIntegration and the force constraints of the MD loop).
//
// Arrays are device arrays in the reference's layouts: x, v, f [atom][dim],
// eatom [atom], the fixes' per-atom virial vatom [atom][6] (AoS, as
// cpuFixes.cpp writes it), fparam / iparam the fix's parameters.  The
// thermostat's dtarray, tarray, seed, save and second are host arrays, as the
// reference reads them; ke and tmp are device scratch of inum and 1 values.
//
// One thread per atom of ilist; sums and products are rounded in the order of
// the reference's CPU code (cpuFixes.cpp, cpuVelocityIntegration.cpp) without
// fused multiply-add.  Where the reference's CPU and GPU versions differ, the
// GPU version (src/C++/Core/gpuFixes.cu, which these entry points replace) is
// followed:
//  * line / plane force: the z component projects on fparam[2] (the CPU code
//    uses fparam[1] there, cpuFixes.cpp:56, 81);
//  * ave force has no GPU version in the reference (gpuFixes.cu:257-287 is
//    commented out); the CPU one is followed: mean force plus fparam on the
//    masked components.
// Kept as the reference has them in both versions: the Morse wall adds its
// energy under vflag_atom (cpuFixes.cpp:668); the reference's GPU wall kernels
// skip their loop increment on atoms beyond the cutoff (gpuFixes.cu), which
// these kernels, one thread per atom, do not reproduce.  Default stream.
#include "common.cuh"
#include "engine.h"

#include "../../include/mdp_b200_gpucore.h"

#include <math.h>
#include <algorithm>

namespace mdp {
namespace {

constexpr int TB = 256;
unsigned blocks_for(long n) { return (unsigned)std::max<long>(1, (n + TB - 1) / TB); }

__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

bool launched(const char *fn)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { set_error("%s: %s", fn, cudaGetErrorString(e)); return false; }
    return true;
}

// ---- set / line / plane / add force (cpuFixes.cpp:22-212) ------------------
template <typename T>
__global__ void k_fix_setforce(T *__restrict__ f, const T *__restrict__ fp, const int *__restrict__ ip,
                               const int *__restrict__ ilist, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    T *fi = f + (size_t)dim * ilist[ii];
    for (int d = 0; d < dim; d++)
        if (ip[d]) fi[d] = fp[d];
}

// f . p over dim components, summed left to right
template <typename T> __device__ __forceinline__ T dot_p(const T *fi, const T *fp, int dim)
{
    T s = add_rn(mul_rn(fi[0], fp[0]), mul_rn(fi[1], fp[1]));
    if (dim == 3) s = add_rn(s, mul_rn(fi[2], fp[2]));
    return s;
}

// plane = 0: f = (f.p) p (line); plane = 1: f -= (f.p) p
template <typename T>
__global__ void k_fix_project(T *__restrict__ f, const T *__restrict__ fp, const int *__restrict__ ilist, int plane,
                              int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    T *fi = f + (size_t)dim * ilist[ii];
    const T dot = dot_p(fi, fp, dim);
    for (int d = 0; d < dim; d++) fi[d] = plane ? sub_rn(fi[d], mul_rn(dot, fp[d])) : mul_rn(dot, fp[d]);
}

// constant force with its potential energy -p.y and virial p (x) y at the
// unwrapped position y = x + image box (cpuFixes.cpp:143-200)
template <typename T>
__global__ void k_fix_addforce(const T *__restrict__ x, T *__restrict__ f, T *__restrict__ eatom,
                               T *__restrict__ vatom, const T *__restrict__ fp, const T *__restrict__ box,
                               const int *__restrict__ image, const int *__restrict__ ilist, int triclinic, int eflag,
                               int vflag, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii];
    const T *xi = x + (size_t)dim * i;
    const int *im = image + (size_t)dim * i;
    T *fi = f + (size_t)dim * i;
    for (int d = 0; d < dim; d++) fi[d] = add_rn(fi[d], fp[d]);
    T y0, y1, y2 = T(0);
    if (triclinic == 0) {
        y0 = add_rn(xi[0], mul_rn((T)im[0], box[0]));
        y1 = add_rn(xi[1], mul_rn((T)im[1], box[1]));
        if (dim == 3) y2 = add_rn(xi[2], mul_rn((T)im[2], box[2]));
    } else if (dim == 3) {
        y0 = add_rn(add_rn(add_rn(xi[0], mul_rn(box[0], (T)im[0])), mul_rn(box[5], (T)im[1])),
                    mul_rn(box[4], (T)im[2]));
        y1 = add_rn(add_rn(xi[1], mul_rn(box[1], (T)im[1])), mul_rn(box[3], (T)im[2]));
        y2 = add_rn(xi[2], mul_rn(box[2], (T)im[2]));
    } else {
        y0 = add_rn(add_rn(xi[0], mul_rn(box[0], (T)im[0])), mul_rn(box[5], (T)im[1]));
        y1 = add_rn(xi[1], mul_rn(box[1], (T)im[1]));
    }
    if (eflag) {
        T e = add_rn(mul_rn(fp[0], y0), mul_rn(fp[1], y1));
        if (dim == 3) e = add_rn(e, mul_rn(fp[2], y2));
        eatom[i] = -e;
    }
    if (vflag) {
        T *va = vatom + (size_t)6 * i;
        va[0] = add_rn(va[0], mul_rn(fp[0], y0));
        va[1] = add_rn(va[1], mul_rn(fp[1], y1));
        va[3] = add_rn(va[3], mul_rn(fp[0], y1));
        if (dim == 3) {
            va[2] = add_rn(va[2], mul_rn(fp[2], y2));
            va[4] = add_rn(va[4], mul_rn(fp[0], y2));
            va[5] = add_rn(va[5], mul_rn(fp[1], y2));
        }
    }
}

// ---- ave force (cpuFixes.cpp:266-295): one CTA sums the group's forces with a
// fixed tree, then sets the masked components to mean + fparam -------------
template <typename T>
__global__ void __launch_bounds__(1024) k_fix_aveforce(T *__restrict__ f, const T *__restrict__ fp,
                                                       const int *__restrict__ ip, const int *__restrict__ ilist,
                                                       int dim, int inum)
{
    __shared__ T sh[3][1024];
    T s[3] = {T(0), T(0), T(0)};
    for (int ii = threadIdx.x; ii < inum; ii += blockDim.x) {
        const T *fi = f + (size_t)dim * ilist[ii];
        for (int d = 0; d < dim; d++) s[d] += fi[d];
    }
    for (int d = 0; d < 3; d++) sh[d][threadIdx.x] = s[d];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int d = 0; d < 3; d++) sh[d][threadIdx.x] += sh[d][threadIdx.x + w];
        __syncthreads();
    }
    T mean[3];
    for (int d = 0; d < 3; d++) mean[d] = add_rn(sh[d][0] / (T)inum, d < dim ? fp[d] : T(0));
    for (int ii = threadIdx.x; ii < inum; ii += blockDim.x) {
        T *fi = f + (size_t)dim * ilist[ii];
        for (int d = 0; d < dim; d++)
            if (ip[d]) fi[d] = mean[d];
    }
}

// ---- drag force toward a point (cpuFixes.cpp:338-386) ----------------------
// The minimum-image loops of cpuMinimumImage (cpuDomain.cpp:456-510), each
// bounded at MINIMG_MAX shifts (the reference's loops are unbounded; a
// displacement that needs more than that many box lengths is left where the
// bound stops it).
constexpr int MINIMG_MAX = 1024;
template <typename T>
__device__ void min_image(T *dp, const T *h, const int *pbc, int triclinic, int dim)
{
    auto wrap = [&](int d, int j1, int j2, T s1, T s2) {
        const T half = mul_rn(T(0.5), h[d]);
        for (int it = 0; it < MINIMG_MAX && fabs(dp[d]) > half; it++) {
            const T sg = dp[d] < T(0) ? T(1) : T(-1);
            dp[d] = add_rn(dp[d], sg * h[d]);
            if (j1 >= 0) dp[j1] = add_rn(dp[j1], sg * s1);
            if (j2 >= 0) dp[j2] = add_rn(dp[j2], sg * s2);
        }
    };
    if (h[0] <= T(0) || h[1] <= T(0) || (dim == 3 && h[2] <= T(0))) return;
    if (triclinic == 0) {
        if (pbc[0]) wrap(0, -1, -1, T(0), T(0));
        if (pbc[1]) wrap(1, -1, -1, T(0), T(0));
        if (dim == 3 && pbc[2]) wrap(2, -1, -1, T(0), T(0));
    } else {
        if (dim == 3 && pbc[2]) wrap(2, 1, 0, h[5], h[4]);
        if (pbc[1]) wrap(1, 0, -1, h[3], T(0));
        if (pbc[0]) wrap(0, -1, -1, T(0), T(0));
    }
}

template <typename T>
__global__ void k_fix_drag(const T *__restrict__ x, T *__restrict__ f, const T *__restrict__ fp,
                           const T *__restrict__ box, const int *__restrict__ ip, const int *__restrict__ pbc,
                           const int *__restrict__ ilist, int triclinic, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii];
    const T *xi = x + (size_t)dim * i;
    T *fi = f + (size_t)dim * i;
    T dp[3] = {T(0), T(0), T(0)};
    for (int d = 0; d < dim; d++) dp[d] = ip[d] ? sub_rn(xi[d], fp[2 + d]) : T(0);
    min_image(dp, box, pbc, triclinic, dim);
    T r2 = add_rn(mul_rn(dp[0], dp[0]), mul_rn(dp[1], dp[1]));
    if (dim == 3) r2 = add_rn(r2, mul_rn(dp[2], dp[2]));
    const T r = sqrt(r2);
    if (r > fp[1]) {
        const T pre = fp[0] / r;
        for (int d = 0; d < dim; d++) fi[d] = sub_rn(fi[d], mul_rn(pre, dp[d]));
    }
}

// ---- walls (cpuFixes.cpp:456-681) -------------------------------------------
template <typename T>
__global__ void k_fix_wall_reflect(T *__restrict__ x, T *__restrict__ v, const T *__restrict__ fp,
                                   const int *__restrict__ ip, const int *__restrict__ ilist, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii], dir = ip[0] / 2, side = ip[0] % 2;
    const T coord = fp[0];
    T *xd = x + (size_t)dim * i + dir, *vd = v + (size_t)dim * i + dir;
    if (side == 0 ? (*xd < coord) : (*xd > coord)) {
        *xd = side == 0 ? add_rn(coord, sub_rn(coord, *xd)) : sub_rn(coord, sub_rn(*xd, coord));
        *vd = -*vd;
    }
}

enum { WALL_HARMONIC = 0, WALL_LJ93 = 1, WALL_LJ126 = 2, WALL_LJ1043 = 3, WALL_MORSE = 4 };

// wall potentials in the distance delta from the wall (0 < delta < cutoff):
// fwall (signed by side), energy, and whether the energy is tallied under
// eflag (the Morse wall tallies it under vflag, as the reference does)
template <typename T, int KIND>
__global__ void k_fix_wall(const T *__restrict__ x, T *__restrict__ f, T *__restrict__ eatom, T *__restrict__ vatom,
                           const T *__restrict__ fp, const int *__restrict__ ip, const int *__restrict__ ilist,
                           int eflag, int vflag, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii], dir = ip[0] / 2;
    const int side = (ip[0] % 2 == 0) ? -1 : 1;
    const T coord = fp[0], cutoff = fp[1];
    const T xd = x[(size_t)dim * i + dir];
    const T delta = side < 0 ? sub_rn(xd, coord) : sub_rn(coord, xd);
    if (delta >= cutoff || delta <= T(0)) return;
    T fwall, e;
    bool etally = eflag != 0;
    if constexpr (KIND == WALL_HARMONIC) {
        const T eps = fp[2], dr = sub_rn(cutoff, delta);
        fwall = mul_rn((T)side, mul_rn(mul_rn(T(2), eps), dr));
        e = mul_rn(mul_rn(eps, dr), dr);
    } else if constexpr (KIND == WALL_LJ93) {
        const T rinv = T(1) / delta, r2inv = mul_rn(rinv, rinv), r4inv = mul_rn(r2inv, r2inv);
        const T r10inv = mul_rn(mul_rn(r4inv, r4inv), r2inv);
        fwall = mul_rn((T)side, sub_rn(mul_rn(fp[3], r10inv), mul_rn(fp[4], r4inv)));
        e = sub_rn(sub_rn(mul_rn(mul_rn(mul_rn(fp[5], r4inv), r4inv), rinv), mul_rn(mul_rn(fp[6], r2inv), rinv)),
                   fp[2]);
    } else if constexpr (KIND == WALL_LJ126) {
        const T rinv = T(1) / delta, r2inv = mul_rn(rinv, rinv), r6inv = mul_rn(mul_rn(r2inv, r2inv), r2inv);
        fwall = mul_rn(mul_rn(mul_rn((T)side, r6inv), sub_rn(mul_rn(fp[3], r6inv), fp[4])), rinv);
        e = sub_rn(mul_rn(r6inv, sub_rn(mul_rn(fp[5], r6inv), fp[6])), fp[2]);
    } else if constexpr (KIND == WALL_LJ1043) {
        const T rinv = T(1) / delta, r2inv = mul_rn(rinv, rinv), r4inv = mul_rn(r2inv, r2inv);
        const T r10inv = mul_rn(mul_rn(r4inv, r4inv), r2inv);
        const T dc = add_rn(delta, fp[6]);
        fwall = mul_rn((T)side, sub_rn(sub_rn(mul_rn(mul_rn(fp[7], r10inv), rinv), mul_rn(mul_rn(fp[8], r4inv), rinv)),
                                       mul_rn(fp[9], (T)pow((double)dc, -4.0))));
        e = sub_rn(sub_rn(sub_rn(mul_rn(fp[3], r10inv), mul_rn(fp[4], r4inv)), mul_rn(fp[5], (T)pow((double)dc, -3.0))),
                   fp[2]);
    } else {
        const T dr = sub_rn(cutoff, delta);
        const T dexp = (T)exp((double)-mul_rn(fp[4], dr));
        const T d2 = mul_rn(dexp, dexp);
        fwall = mul_rn((T)side, mul_rn(fp[5], sub_rn(d2, dexp))) / delta;
        e = sub_rn(mul_rn(fp[3], sub_rn(d2, mul_rn(T(2), dexp))), fp[2]);
        etally = vflag != 0;
    }
    f[(size_t)dim * i + dir] = sub_rn(f[(size_t)dim * i + dir], fwall);
    if (etally) eatom[i] = add_rn(eatom[i], e);
    if (vflag) {
        const T vn = side < 0 ? mul_rn(-fwall, delta) : mul_rn(fwall, delta);
        vatom[(size_t)6 * i + dir] = add_rn(vatom[(size_t)6 * i + dir], vn);
    }
}

// ---- set-velocity integration (cpuVelocityIntegration.cpp:430-463) --------
template <typename T>
__global__ void k_setvel(T *__restrict__ x, T *__restrict__ v, const T *__restrict__ f, const T *__restrict__ mass,
                         const T *__restrict__ fp, T dtf, T dtv, const int *__restrict__ type,
                         const int *__restrict__ ilist, const int *__restrict__ ip, int stage, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii];
    const T dtfm = dtf / mass[type[i]];
    T *xi = x + (size_t)dim * i, *vi = v + (size_t)dim * i;
    const T *fi = f + (size_t)dim * i;
    for (int d = 0; d < dim; d++) {
        if (stage == 0) {
            vi[d] = ip[d] ? fp[d] : add_rn(vi[d], mul_rn(dtfm, fi[d]));
            xi[d] = add_rn(xi[d], mul_rn(dtv, vi[d]));
        } else if (!ip[d]) {
            vi[d] = add_rn(vi[d], mul_rn(dtfm, fi[d]));
        }
    }
}

// ---- velocity-rescaling thermostats (cpuVelocityIntegration.cpp:708-858) --
// sum over the group of |v|^2 m, times tfactor (cpuComputeTempScalar,
// cpuComputes.cpp:276-296): per-atom terms, then a fixed tree in one CTA
template <typename T>
__global__ void k_vrt_terms(T *__restrict__ ke, const T *__restrict__ v, const T *__restrict__ mass,
                            const int *__restrict__ type, const int *__restrict__ ilist, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    const int i = ilist[ii];
    const T *vi = v + (size_t)dim * i;
    T s = add_rn(mul_rn(vi[0], vi[0]), mul_rn(vi[1], vi[1]));
    if (dim == 3) s = add_rn(s, mul_rn(vi[2], vi[2]));
    ke[ii] = mul_rn(s, mass[type[i]]);
}
template <typename T>
__global__ void __launch_bounds__(TB) k_vrt_sum(T *__restrict__ out, const T *__restrict__ a, int n)
{
    __shared__ T sh[TB];
    T s = T(0);
    for (int i = threadIdx.x; i < n; i += TB) s += a[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = TB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}
template <typename T>
__global__ void k_vrt_scale(T *__restrict__ v, T factor, const int *__restrict__ ilist, int dim, int inum)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= inum) return;
    T *vi = v + (size_t)dim * ilist[ii];
    for (int d = 0; d < dim; d++) vi[d] = mul_rn(vi[d], factor);
}

// Host random numbers of the CSVR thermostat, restated from the published
// methods the reference uses (cpuRandom.cpp): the Park-Miller minimal standard
// generator with Schrage's factorisation (multiplier 16807, modulus 2^31 - 1),
// Marsaglia's polar method for Gaussians (the second deviate kept in
// second / save), and the Numerical Recipes gamma deviate (product of
// uniforms below order 6, rejection from a Lorentzian above).
double uniform(int *seed)
{
    const int a = 16807, m = 2147483647, q = 127773, r = 2836;
    const int k = seed[0] / q;
    seed[0] = a * (seed[0] - k * q) - r * k;
    if (seed[0] < 0) seed[0] += m;
    return (1.0 / m) * seed[0];
}
template <typename T> T gaussian(int *seed, int *save, T *second)
{
    if (save[0]) {
        save[0] = 0;
        return second[0];
    }
    T v1, v2, rsq;
    do {
        v1 = 2.0 * uniform(seed) - 1.0;
        v2 = 2.0 * uniform(seed) - 1.0;
        rsq = v1 * v1 + v2 * v2;
    } while (rsq >= 1.0 || rsq == 0.0);
    const T fac = sqrt(-2.0 * log(rsq) / rsq);
    second[0] = v1 * fac;
    save[0] = 1;
    return v2 * fac;
}
double gamma_deviate(int ia, int *seed)
{
    if (ia < 1) return 0.0;
    if (ia < 6) {
        double x = 1.0;
        for (int j = 1; j <= ia; j++) x *= uniform(seed);
        return x < 2.2250759805e-308 ? 708.4 : -log(x);
    }
    const double am = ia - 1, s = sqrt(2.0 * am + 1.0);
    for (;;) {
        double v1, v2, y, x;
        do {
            do {
                v1 = uniform(seed);
                v2 = 2.0 * uniform(seed) - 1.0;
            } while (v1 * v1 + v2 * v2 > 1.0);
            y = v2 / v1;
            x = s * y + am;
        } while (x <= 0.0);
        if (am * log(x / am) - s * y < -700 || v1 < 0.00001) continue;   // start over without a test draw
        const double e = (1.0 + y * y) * exp(am * log(x / am) - s * y);
        if (!(uniform(seed) > e)) return x;
    }
}

template <typename T>
T velocity_rescaling(T *v, const T *mass, const T *dtarray, T *tarray, T *ke, T *tmp, T *second, T energy,
                     const int *type, const int *ilist, int *seed, int *save, int mode, int dim, int inum)
{
    if (mode < 0 || mode > 2) return T(0);
    if (dim != 2 && dim != 3) { set_error("gpuVelocityRescalingThermostat: dim must be 2 or 3"); return energy; }
    const T tdof = tarray[5], boltz = tarray[6], mvv2e = tarray[8];
    const T tfactor = mvv2e / (tdof * boltz);
    T sum = T(0);
    if (inum > 0) {
        k_vrt_terms<<<blocks_for(inum), TB>>>(ke, v, mass, type, ilist, dim, inum);
        k_vrt_sum<<<1, TB>>>(tmp, ke, inum);
        count_launches(2);
        if (cudaMemcpy(&sum, tmp, sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error("gpuVelocityRescalingThermostat: temperature read-back failed");
            return energy;
        }
    }
    const T t_current = tfactor * sum;
    tarray[4] = t_current;
    if (tdof < 1) return energy;
    const T dt = dtarray[0], beginstep = dtarray[3], endstep = dtarray[4], ntimestep = dtarray[5];
    const T t_start = tarray[0], t_stop = tarray[1], t_freq = tarray[2];
    const T delta = (ntimestep - beginstep) / (endstep - beginstep);
    T t_target = t_start + delta * (t_stop - t_start);
    tarray[3] = t_target;
    const T efactor = 0.5 * boltz * tdof;
    T factor = T(1);
    bool scale = true;
    if (mode == 0 || mode == 1) {
        // Berendsen (cpuVelocityIntegration.cpp:708-740) and rescale (742-782)
        const T lamda = sqrt(1.0 + dt * t_freq * (t_target / t_current - 1.0));
        energy += t_current * (1.0 - lamda * lamda) * efactor;
        factor = lamda;
        if (mode == 1) {
            const T t_window = tarray[9], fraction = tarray[10];
            scale = fabs(t_current - t_target) > t_window;
            if (scale) {
                t_target = t_current - fraction * (t_current - t_target);
                factor = sqrt(t_target / t_current);
                energy += (t_current - t_target) * efactor;
            }
        }
    } else {
        // canonical sampling through velocity rescaling (784-840)
        const T ekin_old = t_current * efactor, ekin_new = t_target * efactor;
        const T c1 = exp(-dt * t_freq);
        const T c2 = (1.0 - c1) * ekin_new / ekin_old / tdof;
        const T r1 = gaussian(seed, save, second);
        T r2;
        const int nn = (int)(tdof - 1);
        if (nn == 0) {
            r2 = 0.0;
        } else if (nn == 1) {
            const T rr = gaussian(seed, save, second);
            r2 = rr * rr;
        } else if (nn % 2 == 0) {
            r2 = 2.0 * gamma_deviate(nn / 2, seed);
        } else {
            const T rr = gaussian(seed, save, second);
            r2 = 2.0 * gamma_deviate((nn - 1) / 2, seed) + rr * rr;
        }
        const T s = c1 + c2 * (r1 * r1 + r2) + 2.0 * r1 * sqrt(c1 * c2);
        const T lamda = sqrt(s);
        energy += t_current * (1.0 - lamda * lamda) * efactor;
        factor = lamda;
    }
    if (scale && inum > 0) {
        k_vrt_scale<<<blocks_for(inum), TB>>>(v, factor, ilist, dim, inum);
        count_launches(1);
    }
    launched("gpuVelocityRescalingThermostat");
    return energy;
}

// ---- host launchers ---------------------------------------------------------
bool dims_ok(const char *fn, int dim)
{
    if (dim == 2 || dim == 3) return true;
    set_error("%s: dim must be 2 or 3", fn);
    return false;
}

template <typename T>
void setforce_t(T *f, const T *fp, const int *ip, const int *ilist, int dim, int inum)
{
    if (!dims_ok("gpuFixSetForce", dim) || inum <= 0) return;
    k_fix_setforce<<<blocks_for(inum), TB>>>(f, fp, ip, ilist, dim, inum);
    count_launches(1);
    launched("gpuFixSetForce");
}
template <typename T> void project_t(const char *fn, T *f, const T *fp, const int *ilist, int plane, int dim, int inum)
{
    if (!dims_ok(fn, dim) || inum <= 0) return;
    k_fix_project<<<blocks_for(inum), TB>>>(f, fp, ilist, plane, dim, inum);
    count_launches(1);
    launched(fn);
}
template <typename T>
void aveforce_t(T *f, const T *fp, const int *ip, const int *ilist, int dim, int inum)
{
    if (!dims_ok("gpuFixAveForce", dim) || inum <= 0) return;
    k_fix_aveforce<<<1, 1024>>>(f, fp, ip, ilist, dim, inum);
    count_launches(1);
    launched("gpuFixAveForce");
}
template <typename T>
void addforce_t(const T *x, T *f, T *eatom, T *vatom, const T *fp, const T *box, const int *ilist, const int *image,
                int triclinic, int eflag, int vflag, int dim, int inum)
{
    if (!dims_ok("gpuFixAddForce", dim) || inum <= 0) return;
    k_fix_addforce<<<blocks_for(inum), TB>>>(x, f, eatom, vatom, fp, box, image, ilist, triclinic, eflag, vflag, dim,
                                              inum);
    count_launches(1);
    launched("gpuFixAddForce");
}
template <typename T>
void drag_t(const T *x, T *f, const T *fp, const T *box, const int *ip, const int *ilist, const int *pbc,
            int triclinic, int dim, int inum)
{
    if (!dims_ok("gpuFixDragForce", dim) || inum <= 0) return;
    k_fix_drag<<<blocks_for(inum), TB>>>(x, f, fp, box, ip, pbc, ilist, triclinic, dim, inum);
    count_launches(1);
    launched("gpuFixDragForce");
}
template <typename T>
void reflect_t(T *x, T *v, const T *fp, const int *ip, const int *ilist, int dim, int inum)
{
    if (!dims_ok("gpuFixWallReflect", dim) || inum <= 0) return;
    k_fix_wall_reflect<<<blocks_for(inum), TB>>>(x, v, fp, ip, ilist, dim, inum);
    count_launches(1);
    launched("gpuFixWallReflect");
}
template <typename T, int KIND>
void wall_t(const char *fn, const T *x, T *f, T *eatom, T *vatom, const T *fp, const int *ip, const int *ilist,
            int eflag, int vflag, int dim, int inum)
{
    if (!dims_ok(fn, dim) || inum <= 0) return;
    k_fix_wall<T, KIND><<<blocks_for(inum), TB>>>(x, f, eatom, vatom, fp, ip, ilist, eflag, vflag, dim, inum);
    count_launches(1);
    launched(fn);
}
template <typename T>
void setvel_t(const char *fn, T *x, T *v, const T *f, const T *mass, const T *fp, T dtf, T dtv, const int *type,
              const int *ilist, const int *ip, int stage, int dim, int inum)
{
    if (!dims_ok(fn, dim) || inum <= 0) return;
    k_setvel<<<blocks_for(inum), TB>>>(x, v, f, mass, fp, dtf, dtv, type, ilist, ip, stage, dim, inum);
    count_launches(1);
    launched(fn);
}

}  // namespace
}  // namespace mdp

using namespace mdp;

#define MDP_FIX_ARGS(T)                                                                                            \
    T *x, T *v, T *f, T *eatom, T *vatom, const T *fparam, const int *iparam, const int *ilist, int eflag_atom,    \
        int vflag_atom, int dim, int inum

extern "C" {

#define MDP_FIX_ENTRIES(T, S)                                                                                      \
    void mdp_gpu_fix_set_force_##S(MDP_FIX_ARGS(T))                                                                \
    {                                                                                                              \
        (void)x; (void)v; (void)eatom; (void)vatom; (void)eflag_atom; (void)vflag_atom;                          \
        setforce_t<T>(f, fparam, iparam, ilist, dim, inum);                                                        \
    }                                                                                                              \
    void mdp_gpu_fix_line_force_##S(MDP_FIX_ARGS(T))                                                               \
    {                                                                                                              \
        (void)x; (void)v; (void)eatom; (void)vatom; (void)iparam; (void)eflag_atom; (void)vflag_atom;            \
        project_t<T>("gpuFixLineForce", f, fparam, ilist, 0, dim, inum);                                           \
    }                                                                                                              \
    void mdp_gpu_fix_plane_force_##S(MDP_FIX_ARGS(T))                                                              \
    {                                                                                                              \
        (void)x; (void)v; (void)eatom; (void)vatom; (void)iparam; (void)eflag_atom; (void)vflag_atom;            \
        project_t<T>("gpuFixPlaneForce", f, fparam, ilist, 1, dim, inum);                                          \
    }                                                                                                              \
    void mdp_gpu_fix_ave_force_##S(MDP_FIX_ARGS(T))                                                                \
    {                                                                                                              \
        (void)x; (void)v; (void)eatom; (void)vatom; (void)eflag_atom; (void)vflag_atom;                          \
        aveforce_t<T>(f, fparam, iparam, ilist, dim, inum);                                                        \
    }                                                                                                              \
    void mdp_gpu_fix_add_force_##S(T *x, T *v, T *f, T *eatom, T *vatom, const T *fparam, const T *box,          \
                                   const int *iparam, const int *ilist, const int *image, int triclinic,          \
                                   int eflag_atom, int vflag_atom, int dim, int inum)                            \
    {                                                                                                              \
        (void)v; (void)iparam;                                                                                     \
        addforce_t<T>(x, f, eatom, vatom, fparam, box, ilist, image, triclinic, eflag_atom, vflag_atom, dim, inum); \
    }                                                                                                              \
    void mdp_gpu_fix_drag_force_##S(T *x, T *v, T *f, T *eatom, T *vatom, const T *fparam, const T *box,         \
                                    const int *iparam, const int *ilist, const int *pbc, int triclinic,           \
                                    int eflag_atom, int vflag_atom, int dim, int inum)                           \
    {                                                                                                              \
        (void)v; (void)eatom; (void)vatom; (void)eflag_atom; (void)vflag_atom;                                   \
        drag_t<T>(x, f, fparam, box, iparam, ilist, pbc, triclinic, dim, inum);                                   \
    }                                                                                                              \
    void mdp_gpu_fix_wall_reflect_##S(MDP_FIX_ARGS(T))                                                             \
    {                                                                                                              \
        (void)f; (void)eatom; (void)vatom; (void)eflag_atom; (void)vflag_atom;                                   \
        reflect_t<T>(x, v, fparam, iparam, ilist, dim, inum);                                                      \
    }                                                                                                              \
    void mdp_gpu_fix_wall_harmonic_##S(MDP_FIX_ARGS(T))                                                            \
    {                                                                                                              \
        (void)v;                                                                                                   \
        wall_t<T, WALL_HARMONIC>("gpuFixWallHarmonic", x, f, eatom, vatom, fparam, iparam, ilist, eflag_atom,      \
                                 vflag_atom, dim, inum);                                                           \
    }                                                                                                              \
    void mdp_gpu_fix_wall_lj93_##S(MDP_FIX_ARGS(T))                                                                \
    {                                                                                                              \
        (void)v;                                                                                                   \
        wall_t<T, WALL_LJ93>("gpuFixWallLJ93", x, f, eatom, vatom, fparam, iparam, ilist, eflag_atom, vflag_atom,  \
                             dim, inum);                                                                           \
    }                                                                                                              \
    void mdp_gpu_fix_wall_lj126_##S(MDP_FIX_ARGS(T))                                                               \
    {                                                                                                              \
        (void)v;                                                                                                   \
        wall_t<T, WALL_LJ126>("gpuFixWallLJ126", x, f, eatom, vatom, fparam, iparam, ilist, eflag_atom,            \
                              vflag_atom, dim, inum);                                                              \
    }                                                                                                              \
    void mdp_gpu_fix_wall_lj1043_##S(MDP_FIX_ARGS(T))                                                              \
    {                                                                                                              \
        (void)v;                                                                                                   \
        wall_t<T, WALL_LJ1043>("gpuFixWallLJ1043", x, f, eatom, vatom, fparam, iparam, ilist, eflag_atom,          \
                               vflag_atom, dim, inum);                                                             \
    }                                                                                                              \
    void mdp_gpu_fix_wall_morse_##S(MDP_FIX_ARGS(T))                                                               \
    {                                                                                                              \
        (void)v;                                                                                                   \
        wall_t<T, WALL_MORSE>("gpuFixWallMorse", x, f, eatom, vatom, fparam, iparam, ilist, eflag_atom,            \
                              vflag_atom, dim, inum);                                                              \
    }                                                                                                              \
    void mdp_gpu_set_velocity_initial_integrate_##S(T *x, T *v, const T *f, const T *mass, const T *fparam,      \
                                                    T dtf, T dtv, const int *type, const int *ilist,              \
                                                    const int *iparam, int dim, int inum)                         \
    {                                                                                                              \
        setvel_t<T>("gpuSetVelocityInitialIntegrate", x, v, f, mass, fparam, dtf, dtv, type, ilist, iparam, 0,    \
                    dim, inum);                                                                                    \
    }                                                                                                              \
    void mdp_gpu_set_velocity_final_integrate_##S(T *x, T *v, const T *f, const T *mass, T dtf, const int *type,  \
                                                  const int *ilist, const int *iparam, int dim, int inum)         \
    {                                                                                                              \
        setvel_t<T>("gpuSetVelocityFinalIntegrate", x, v, f, mass, (const T *)nullptr, dtf, T(0), type, ilist,    \
                    iparam, 1, dim, inum);                                                                         \
    }                                                                                                              \
    T mdp_gpu_velocity_rescaling_thermostat_##S(T *v, const T *mass, const T *dtarray, T *tarray, T *ke, T *tmp,  \
                                                T *second, T energy, const int *type, const int *ilist, int *seed, \
                                                int *save, int biasflag, int mode, int dim, int inum)             \
    {                                                                                                              \
        (void)biasflag;                                                                                            \
        return velocity_rescaling<T>(v, mass, dtarray, tarray, ke, tmp, second, energy, type, ilist, seed, save,  \
                                     mode, dim, inum);                                                             \
    }

MDP_FIX_ENTRIES(double, f64)
MDP_FIX_ENTRIES(float, f32)

#undef MDP_FIX_ENTRIES
#undef MDP_FIX_ARGS

}  // extern "C"
