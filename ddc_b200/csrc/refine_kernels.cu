// refine_kernels.cu -- the builder in FP32 with FP64 iterative refinement (precision
// DDCB_FP32_REFINE): one kernel per call over tiles of lines, the per-tile algorithm in
// refine_device.cuh.
#include <algorithm>

#include "refine_device.cuh"

namespace ddcb {

namespace {

// MAXT: the largest block the instantiation takes (blocks of up to 256 threads get 128 registers).
template <int TL, int KL, int KU, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 2 : 1) refine_kernel(const __grid_constant__ BuildArgs args, int rounds)
{
    extern __shared__ __align__(16) double smem[];
    refine_tile<TL, KL, KU>(args, smem, rounds);
    store_tile<TL>(args, smem);
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
