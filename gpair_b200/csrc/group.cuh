// group.cuh -- grouped launches of the per-evaluation stage kernels.
//
// Many independent reconstructions that advance in lockstep run every stage
// (image prep, V2/T3/chi2, adjoint weights, ...) as ONE launch over the blocks
// of all instances instead of one launch per instance. A stage kernel's body
// runs on a virtual grid: its block (bx, by) of (nbx, nby). A single-instance
// launch maps the hardware grid onto it one to one (gp_vgrid_hw); a grouped
// launch (k_grouped) gives instance i the 1-D block range [start[i],
// start[i + 1]) of its grid, reads the instance's arguments from a device
// array, and skips the instance when its gate flag is 0. Reductions inside a
// body count their blocks against nbx (nby), never gridDim.
#pragma once

#include "gpair_internal.cuh"

struct GpVGrid {
    int bx, by, nbx, nby;
};

__device__ __forceinline__ GpVGrid gp_vgrid_hw()
{
    GpVGrid v;
    v.bx = (int)blockIdx.x;
    v.by = (int)blockIdx.y;
    v.nbx = (int)gridDim.x;
    v.nby = (int)gridDim.y;
    return v;
}

// Every stage's argument struct ends with the instance's grid (GP_VGRID_FIELDS),
// which a grouped launch reads; a single launch uses the hardware grid.
#define GP_VGRID_FIELDS int nbx, nby

// Op: struct with `using Args = ...;` and `static __device__ void run(const Args &, const GpVGrid &)`.
// start[0..n]: first block of every instance, start[n] = the launch's blocks.
template <class Op, int THREADS>
__global__ void __launch_bounds__(THREADS) k_grouped(const typename Op::Args *__restrict__ args,
                                                     const int *__restrict__ start, int n,
                                                     const int *__restrict__ gate)
{
    gp_pdl_enter();  // after the kernel before it on the stream (programmatic dependent launch)
    const int b = (int)blockIdx.x;
    int lo = 0, hi = n;  // start[lo] <= b < start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&start[mid]) <= b) lo = mid;
        else hi = mid;
    }
    if (gate && !gate[lo]) return;  // block-uniform: the whole instance is skipped
    const typename Op::Args &a = args[lo];
    const int local = b - __ldg(&start[lo]);
    GpVGrid vg;
    vg.nbx = a.nbx;
    vg.nby = a.nby;
    vg.bx = local % vg.nbx;
    vg.by = local / vg.nbx;
    Op::run(a, vg);
}
