// reduce.cuh -- block reductions and the solver's compensated residual, shared by the exact and
// the fast kernels.
#pragma once

#include <climits>
#include <cstdint>

#include "fluid_device.cuh"

namespace slf {

// ---- block reductions ---------------------------------------------------------------------

template <class T, class Op>
__device__ __forceinline__ T warp_reduce(T v, Op op) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Reduces one value per thread over the block; the result is valid in thread 0.
template <class T, class Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T identity) {
    __shared__ T warp_vals[kBlock / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_reduce(v, op);
    __syncthreads();
    if (lane == 0) warp_vals[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? warp_vals[lane] : identity;
        v = warp_reduce(v, op);
    }
    return v;
}

struct MinI { __device__ int operator()(int a, int b) const { return a < b ? a : b; } };
struct MaxI { __device__ int operator()(int a, int b) const { return a > b ? a : b; } };
struct MaxU { __device__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; } };
struct SumU { __device__ uint32_t operator()(uint32_t a, uint32_t b) const { return a + b; } };

// double-double accumulation (TwoSum), for the solver residual
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_add(DD a, DD b) {
    double s = a.hi + b.hi;
    double bb = s - a.hi;
    double err = (a.hi - (s - bb)) + (b.hi - bb);
    double lo = a.lo + b.lo + err;
    double h = s + lo;
    return DD{h, lo - (h - s)};
}

// The bound of a solve run as a CUDA graph, independent of the stopping check: one thread counts
// the loop's bodies and ends the loop past max_iterations + 1 of them (the check stops a solve at
// max_iterations pushes, so only a fault in it gets here).
__device__ __forceinline__ void loop_bound(const Params& p, Status* st, unsigned long long loop) {
    if (!loop || blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t bodies = atomicAdd(&st->bodies, 1u) + 1u;
    if (bodies > p.max_iter + 1u) {
        st->overrun = 1u;
        cudaGraphSetConditional(loop, 0u);
    }
}

// The error sum of one solver check (dfsph.rs:263-268): a block tree in double-double, block
// partials in `partial`, and the last block to finish sums them in block order, takes the
// average over the particles under load and writes the stop decision (dfsph.rs:268-271) into the
// status.  Deterministic for a given launch shape.
// `loop`: the while-node handle of a solve run as a CUDA graph (0 when launched on its own); the
// check that stops the solve also ends the graph's loop.
template <int WHICH>
__device__ __forceinline__ void residual_finish(const Params& p, Status* st, DD* __restrict__ partial,
                                                uint32_t* __restrict__ partial_loaded, DD acc, uint32_t loaded,
                                                unsigned long long loop) {
    // block sum: a fixed shuffle tree in double-double (acc: this thread's rows' errors)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD other{__shfl_xor_sync(0xffffffffu, acc.hi, o), __shfl_xor_sync(0xffffffffu, acc.lo, o)};
        acc = dd_add(acc, other);
    }
    __shared__ DD warp_acc[kBlock / 32];
    __shared__ bool last_block;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_acc[warp] = acc;
    loaded = block_reduce(loaded, SumU(), 0u);
    __syncthreads();
    if (threadIdx.x == 0) {
        DD b = warp_acc[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) b = dd_add(b, warp_acc[k]);
        partial[blockIdx.x] = b;
        partial_loaded[blockIdx.x] = loaded;
        __threadfence();
        uint32_t ticket = atomicAdd(&st->ticket, 1u);
        last_block = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!last_block) return;
    // the last block to finish sums the block partials in block order
    __threadfence();
    DD t{0.0, 0.0};
    uint32_t cnt = 0;
    for (uint32_t k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        // other blocks wrote these: read through L2, never a stale L1 line
        const double* part = reinterpret_cast<const double*>(partial);
        DD v{__ldcg(part + 2 * k), __ldcg(part + 2 * k + 1)};
        t = dd_add(t, v);
        cnt += __ldcg(partial_loaded + k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD other{__shfl_xor_sync(0xffffffffu, t.hi, o), __shfl_xor_sync(0xffffffffu, t.lo, o)};
        t = dd_add(t, other);
    }
    cnt = block_reduce(cnt, SumU(), 0u);
    __syncthreads();
    if (lane == 0) warp_acc[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD b = warp_acc[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) b = dd_add(b, warp_acc[k]);
        uint32_t load = cnt > 0 ? cnt : 1u;
        double average = (b.hi + b.lo) / (double)load;
        double tol = WHICH == 1 ? (double)p.den_tol : (double)p.div_tol;
        uint32_t iterations = st->iterations;
        bool settled = iterations >= p.min_iter && average <= tol;
        st->average = average;
        st->loaded = cnt;
        if (settled || iterations >= p.max_iter) {
            st->settled = 1u;
            st->solved[WHICH] = iterations;
            if (loop) cudaGraphSetConditional(loop, 0u);
        } else {
            st->iterations = iterations + 1u;  // a push follows
        }
        st->ticket = 0;
    }
}

}  // namespace slf
