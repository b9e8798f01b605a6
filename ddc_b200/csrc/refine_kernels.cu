// refine_kernels.cu -- the builder in FP32 with FP64 iterative refinement (precision
// DDCB_FP32_REFINE).
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
#include <algorithm>

#include "build_device.cuh"

namespace ddcb {

namespace {

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
// carries an error of about cond(A) (2^-24 max|d| + 2^-52 max|X|); a line whose bound, with a
// factor 4, exceeds refine_tol * max|X| sets bit 0 of the builder's status word (read by
// ddcb_builder_device_status). dmax / xmax: this thread's maxima of its line (threads own one line
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
        double const bound = 4.0 * t.cond_est * (0x1p-24 * d + 0x1p-52 * x);
        if (!(bound <= t.refine_tol * x)) atomicOr(t.status, 1u);
    }
    __syncthreads();
}

// MAXT: the largest block the instantiation takes (blocks of up to 256 threads get 128 registers).
template <int TL, int KL, int KU, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 2 : 1) refine_kernel(const __grid_constant__ BuildArgs args, int rounds)
{
    extern __shared__ __align__(16) double smem[];
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
    store_tile<TL>(args, X);
}

size_t refine_smem(SolveTables const& t, int TL, int KL, int KU)
{
    // X (FP64) + the FP32 tile with its carries, rounded to 16 bytes
    return sizeof(double) * (size_t)t.n * TL + ((sizeof(float) * tile_doubles(t, TL, KL, KU) + 15) & ~size_t(15));
}

template <int TL, int KL, int KU>
void launch_refine_tl(BuildArgs const& args, int rounds, cudaStream_t s)
{
    size_t const sm = refine_smem(args.t, TL, KL, KU);
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (sm > size_t(optin))
        throw Error(DDCB_ERR_UNSUPPORTED, "refinement tile of " + std::to_string(sm) + " bytes exceeds shared memory; use fewer tile lines");
    auto kern = TL * args.nct <= 256 ? refine_kernel<TL, KL, KU, 256> : refine_kernel<TL, KL, KU, 1024>;
    if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    int64_t const grid = (args.nlines + TL - 1) / TL;
    kern<<<dim3((unsigned)grid), dim3(TL * args.nct), sm, s>>>(args, rounds);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int KL, int KU>
void launch_refine_k(BuildArgs const& args, int TL, int rounds, cudaStream_t s)
{
    switch (TL) {
    case 2: launch_refine_tl<2, KL, KU>(args, rounds, s); break;
    case 4: launch_refine_tl<4, KL, KU>(args, rounds, s); break;
    case 8: launch_refine_tl<8, KL, KU>(args, rounds, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "tile_lines must be 2, 4 or 8");
    }
}

} // namespace

void launch_refine(BuildArgs const& args, int TL, int rounds, cudaStream_t s)
{
    int const kl = args.t.kl, ku = args.t.ku;
    if (kl == 1 && ku == 1) launch_refine_k<1, 1>(args, TL, rounds, s);
    else if (kl == 1 && ku == 2) launch_refine_k<1, 2>(args, TL, rounds, s);
    else if (kl == 2 && ku == 2) launch_refine_k<2, 2>(args, TL, rounds, s);
    else if (kl == 3 && ku == 3) launch_refine_k<3, 3>(args, TL, rounds, s);
    else if (kl == 1 && ku == 4) launch_refine_k<1, 4>(args, TL, rounds, s);
    else if (kl == 2 && ku == 4) launch_refine_k<2, 4>(args, TL, rounds, s);
    else if (kl == 4 && ku == 4) launch_refine_k<4, 4>(args, TL, rounds, s);
    else if (kl == 3 && ku == 6) launch_refine_k<3, 6>(args, TL, rounds, s);
    else if (kl == 1 && ku == 8) launch_refine_k<1, 8>(args, TL, rounds, s);
    else if (kl == 2 && ku == 8) launch_refine_k<2, 8>(args, TL, rounds, s);
    else if (kl == 4 && ku == 8) launch_refine_k<4, 8>(args, TL, rounds, s);
    else throw Error(DDCB_ERR_UNSUPPORTED, "band shape kl=" + std::to_string(kl) + " ku=" + std::to_string(ku) + " has no kernel");
}

} // namespace ddcb
