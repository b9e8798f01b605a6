// refine_device.cuh -- the builder's solve of one tile in FP32 with FP64 iterative refinement
// (precision DDCB_FP32_REFINE), shared by the batched refine kernel and the uneven batch.
//
// Per tile: x = A^-1 b with the FP32 factor tables in an FP32 shared tile, then `rounds` times
//   r = b - A x   (FP64: the system matrix in CSR, b read again from the block's own input rows)
//   d = A^-1 r    (FP32)
//   x = x + d     (FP64)
// -- mixed-precision iterative refinement (Wilkinson 1963; Moler, J. ACM 14 (1967) 316-321): each
// round multiplies the error by about cond(A) * 2^-24, so the FP64 residual, not the FP32 solves,
// sets the final accuracy. The factorisation, the Schur / Sherman-Morrison border blocks and the
// residuals are FP64 quantities; only the solves and their tile are FP32. The solution X (FP64)
// and the FP32 solve tile share the block's shared memory.
#pragma once

#include "build_device.cuh"

namespace ddcb {


// W = float(b - A X) for the tile's lines; ends with a barrier.
template <int TL>
__device__ __forceinline__ void residual_tile(BuildArgs const& args, const double* X, float* W)
{
    SolveTables const& t = args.t;
    int const n = t.n;
    int const l = threadIdx.x % TL;
    int const c = threadIdx.x / TL;
    int const nct = blockDim.x / TL;
    int64_t const line = tile_line0<TL>(args) + l;
    bool const live = line < args.nlines;
    for (int r = c; r < n; r += nct) {
        double s = live ? rhs_row(args, r, line) : 0.0;
        int const q1 = __ldg(t.a_row + r + 1);
        for (int q = __ldg(t.a_row + r); q < q1; ++q) s = fma(-__ldg(t.a_val + q), X[__ldg(t.a_col + q) * TL + l], s);
        W[r * TL + l] = float(s);
    }
    __syncthreads();
}

// The convergence check of the refined lines, from the last correction d (no extra residual
// pass): the solve that produced d works in FP32 on an FP32-rounded residual, so the refined X
// carries an error of at most about cond(A) 2^-24 max|d| beyond the FP64 rounding every solve
// has; a line whose bound, with a factor 4, exceeds refine_tol * max|X| sets bit 0 of the
// builder's status word (read by ddcb_builder_device_status). The bound is a worst case: one
// round rarely certifies a system with cond(A) above a few tens, two rounds usually do. dmax / xmax: this thread's maxima of its line (threads own one line
// each in the accumulation loops); `red`: 2 TL shared 8-byte words. Ends with a barrier.
template <int TL>
__device__ __forceinline__ void convergence_check(BuildArgs const& args, double dmax, double xmax, unsigned long long* red)
{
    SolveTables const& t = args.t;
    int const l = threadIdx.x % TL;
    if (threadIdx.x < 2 * TL) red[threadIdx.x] = 0ull;
    __syncthreads();
    // non-negative doubles order like their bit patterns
    atomicMax(red + l, static_cast<unsigned long long>(__double_as_longlong(dmax)));
    atomicMax(red + TL + l, static_cast<unsigned long long>(__double_as_longlong(xmax)));
    __syncthreads();
    if (threadIdx.x < TL && tile_line0<TL>(args) + threadIdx.x < args.nlines) {
        double const d = __longlong_as_double(static_cast<long long>(red[threadIdx.x]));
        double const x = __longlong_as_double(static_cast<long long>(red[TL + threadIdx.x]));
        double const bound = 4.0 * t.cond_est * 0x1p-24 * d;
        if (!(bound <= t.refine_tol * x)) atomicOr(t.status, 1u);
    }
    __syncthreads();
}


// Shared memory of refine_tile: X (FP64) + the FP32 tile with its carries, rounded to 16 bytes.
__host__ __device__ inline size_t refine_smem(SolveTables const& t, int TL, int KL, int KU)
{
    return sizeof(double) * (size_t)t.n * TL + ((sizeof(float) * tile_doubles(t, TL, KL, KU) + 15) & ~size_t(15));
}

// Gather, FP32 solve, `rounds` refinement rounds and the convergence check of one tile; on return
// (after a barrier) X = smem holds the refined solution in the kernel's column order.
template <int TL, int KL, int KU>
__device__ __forceinline__ void refine_tile(BuildArgs const& args, double* smem, int rounds)
{
    int const n = args.t.n;
    double* X = smem;                                            // n x TL, FP64 solution
    float* W = reinterpret_cast<float*>(smem + (size_t)n * TL);  // FP32 solve tile
    gather_tile<TL>(args, X);
    for (int i = threadIdx.x; i < n * TL; i += blockDim.x) W[i] = float(X[i]);
    __syncthreads();
    solve_in_tile<TL, KL, KU, float>(args.t, args.nct, W);
    // every thread touches one line's elements (the block is a multiple of TL threads)
    double dmax = 0.0, xmax = 0.0;
    for (int i = threadIdx.x; i < n * TL; i += blockDim.x) {
        X[i] = double(W[i]);
        dmax = fmax(dmax, fabs(X[i]));
    }
    __syncthreads();
    for (int round = 0; round < rounds; ++round) {
        residual_tile<TL>(args, X, W);
        solve_in_tile<TL, KL, KU, float>(args.t, args.nct, W);
        dmax = 0.0;
        for (int i = threadIdx.x; i < n * TL; i += blockDim.x) {
            double const d = double(W[i]);
            X[i] += d;
            dmax = fmax(dmax, fabs(d));
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n * TL; i += blockDim.x) xmax = fmax(xmax, fabs(X[i]));
    // the FP32 tile is free again: its first words hold the per-line maxima of the check
    convergence_check<TL>(args, dmax, xmax, reinterpret_cast<unsigned long long*>(W));
}

} // namespace ddcb
