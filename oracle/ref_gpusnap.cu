// Baseline infrastructure only: MDP's own GPU SNAP kernels
// (src/C++/Core/gpuSnap4.cu, with the array helpers of gpuArrayOperations.cu),
// compiled unchanged from the reference sources where they lie for sm_100a, so
// that bench.py can time them on the B200 beside this repository's kernels.
// They are never the oracle: gpuKernelSnapComputeFi drops the switching
// derivative term (gpuSnap4.cu:1116), so its forces differ from the CPU path.
//
// The reference launchers index with 32-bit ints (gpuSnap4.cu:896:
// N2 = idxz_max * inum, and inum * idxu_max, 3 * ijnum, and grid strides of
// up to 1024 x 256 threads added to them).  ref_gpu_snap_stages refuses any
// size at which one of those products, or the grid stride added to it, would
// reach 2^31, before anything is launched.  Inputs are device arrays in the
// reference's layouts (ComputePairSnap3, snappotential.cpp:634-760), single
// element type.
#include <cuda_runtime.h>
#include <stdio.h>

#include "gpuArrayOperations.cu"
#include "gpuSnap4.cu"

extern "C" {

// Fits every 32-bit index product of the three launchers?  Returns 0 if so.
int ref_gpu_snap_check(int twojmax, int idxu_max, int idxb_max, int idxz_max, int inum, int ijnum)
{
    const long long stride = 1024LL * 256;
    const long long lim = (1LL << 31) - 1;
    const long long prods[] = {(long long)idxz_max * inum + stride, (long long)idxu_max * inum + stride,
                               (long long)idxb_max * inum + stride, 9LL * inum + stride,
                               3LL * ijnum + 3 * stride, (long long)ijnum + stride, 6LL * inum + 6};
    for (long long p : prods)
        if (p >= lim) return -1;
    if (twojmax < 0 || twojmax > 8) return -1;
    return 0;
}

// One pass of the reference's GPU stages in ComputePairSnap3's order, each
// timed with CUDA events on the default stream:
//   ms[0] zero U + gpuSnapComputeUi + gpuAddWself2Ui
//   ms[1] zero eatom + gpuSnapComputeEi
//   ms[2] gpuSnapComputeYi (coefficient form; it zeroes Y itself)
//   ms[3] zero f, v + gpuSnapComputeFi
// Returns 0, -1 (nothing launched) when the size does not fit 32-bit
// indexing, -2 on a CUDA error.
int ref_gpu_snap_stages(double *Ur, double *Ui, double *Yr, double *Yi, double *eatom, double *fatom,
                        double *vatom, double *rootpq, double *rij, double *wjelem, double *radelem, double *cglist,
                        double *bzero, double *coeffelem, int *idxu_block, int *idxz, int *idxb, int *idxb_block,
                        int *idxcg_block, int *map, int *type, int *ilist, int *aii, int *ai, int *aj, int *ti,
                        int *tj, double rmin0, double rfac0, double rcutfac, int twojmax, int idxu_max, int idxb_max,
                        int idxz_max, int ncoeffall, int bnormflag, int bzeroflag, int switchflag, int wselfallflag,
                        int inum, int ijnum, float *ms)
{
    if (ref_gpu_snap_check(twojmax, idxu_max, idxb_max, idxz_max, inum, ijnum)) return -1;
    cudaEvent_t ev[5];
    for (int k = 0; k < 5; k++) cudaEventCreate(&ev[k]);
    cudaEventRecord(ev[0]);
    gpuArraySetValue(Ur, 0.0, idxu_max * inum);
    gpuArraySetValue(Ui, 0.0, idxu_max * inum);
    gpuSnapComputeUi(Ur, Ui, rootpq, rij, wjelem, radelem, rmin0, rfac0, rcutfac, idxu_block, map, aii, ti, tj,
                     twojmax, idxu_max, inum, ijnum, switchflag, 0);
    gpuAddWself2Ui(Ur, Ui, 1.0, idxu_block, type, map, ai, wselfallflag, 0, idxu_max, 1, twojmax, inum);
    cudaEventRecord(ev[1]);
    gpuArraySetValue(eatom, 0.0, inum);
    gpuSnapComputeEi(eatom, Ur, Ui, cglist, bzero, coeffelem, ilist, map, type, idxb, idxcg_block, idxu_block,
                     twojmax, idxb_max, idxu_max, 1, ncoeffall, bnormflag, bzeroflag, wselfallflag, 0, inum);
    cudaEventRecord(ev[2]);
    gpuSnapComputeYi(Yr, Yi, Ur, Ui, cglist, coeffelem, map, type, idxz, idxb_block, idxu_block, idxcg_block,
                     twojmax, idxb_max, idxu_max, idxz_max, 1, ncoeffall, bnormflag, inum);
    cudaEventRecord(ev[3]);
    gpuArraySetValue(fatom, 0.0, 3 * inum);
    gpuArraySetValue(vatom, 0.0, 6 * inum);
    gpuSnapComputeFi(fatom, vatom, Yr, Yi, rootpq, rij, wjelem, radelem, rmin0, rfac0, rcutfac, idxu_block, map,
                     aii, ai, aj, ti, tj, twojmax, idxu_max, inum, inum, ijnum, switchflag, 0);
    cudaEventRecord(ev[4]);
    cudaEventSynchronize(ev[4]);
    for (int k = 0; k < 4; k++) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
    for (int k = 0; k < 5; k++) cudaEventDestroy(ev[k]);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // extern "C"
