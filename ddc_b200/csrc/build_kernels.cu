// build_kernels.cu -- batched spline interpolation solve (SplineBuilder::operator(),
// spline_builder.hpp:896-1101) as one kernel per call; the per-tile algorithm is in
// build_device.cuh.
#include <algorithm>
#include <string>

#include "build_device.cuh"

namespace ddcb {

namespace {

// MAXT: the largest block the instantiation takes. Blocks of up to 256 threads (64 chunks of
// 8-line tiles, the default) get up to 128 registers, which lets the sweeps of narrow bands
// unroll 8 rows and keep more factor loads in flight; so do the 512-thread blocks of 16-line
// tiles (one per SM); other large blocks keep 64 registers.
template <int TL, int KL, int KU, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 2 : 1) build_kernel(const __grid_constant__ BuildArgs args)
{
    extern __shared__ __align__(16) double smem[];
    solve_tile<TL, KL, KU, (MAXT <= 512 && TL >= 4 && KL + KU <= 6) ? 8 : 0>(args, smem);
    store_tile<TL>(args, smem);
}

size_t smem_bytes(SolveTables const& t, int TL, int KL, int KU) { return sizeof(double) * tile_doubles(t, TL, KL, KU); }

template <int TL, int KL, int KU>
void launch_tl(BuildArgs const& args, cudaStream_t s)
{
    int const nct = args.nct;
    size_t const sm = smem_bytes(args.t, TL, KL, KU);
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (sm > size_t(optin))
        throw Error(DDCB_ERR_UNSUPPORTED, "line tile of " + std::to_string(sm) + " bytes exceeds shared memory (" + std::to_string(optin)
                                              + "); use fewer tile lines");
    auto kern = TL == 16 ? build_kernel<TL, KL, KU, 512>
                         : (TL * nct <= 256 ? build_kernel<TL, KL, KU, 256> : build_kernel<TL, KL, KU, 1024>);
    if (TL == 16 && TL * nct > 512) throw Error(DDCB_ERR_UNSUPPORTED, "16-line tiles take at most 32 chunk threads per line");
    if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    int64_t const grid = (args.nlines + TL - 1) / TL;
    kern<<<dim3((unsigned)grid), dim3(TL * nct), sm, s>>>(args);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int KL, int KU>
void launch_k(BuildArgs const& args, int TL, cudaStream_t s)
{
    switch (TL) {
    case 2: launch_tl<2, KL, KU>(args, s); break;
    case 4: launch_tl<4, KL, KU>(args, s); break;
    case 8: launch_tl<8, KL, KU>(args, s); break;
    case 16: launch_tl<16, KL, KU>(args, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "tile_lines must be 2, 4, 8 or 16");
    }
}

void dispatch(BuildArgs const& args, int TL, cudaStream_t s)
{
    int const kl = args.t.kl, ku = args.t.ku;
    // the plan pads (kl, ku) up to one of these shapes (plan.cpp, HostSolve::analyse)
    if (kl == 1 && ku == 1) launch_k<1, 1>(args, TL, s);
    else if (kl == 1 && ku == 2) launch_k<1, 2>(args, TL, s);
    else if (kl == 2 && ku == 2) launch_k<2, 2>(args, TL, s);
    else if (kl == 3 && ku == 3) launch_k<3, 3>(args, TL, s);
    else if (kl == 1 && ku == 4) launch_k<1, 4>(args, TL, s);
    else if (kl == 2 && ku == 4) launch_k<2, 4>(args, TL, s);
    else if (kl == 4 && ku == 4) launch_k<4, 4>(args, TL, s);
    else if (kl == 3 && ku == 6) launch_k<3, 6>(args, TL, s);
    else if (kl == 1 && ku == 8) launch_k<1, 8>(args, TL, s);
    else if (kl == 2 && ku == 8) launch_k<2, 8>(args, TL, s);
    else if (kl == 4 && ku == 8) launch_k<4, 8>(args, TL, s);
    else throw Error(DDCB_ERR_UNSUPPORTED, "band shape kl=" + std::to_string(kl) + " ku=" + std::to_string(ku) + " has no kernel");
}

// Point threads per line of the fused kernels (tiles of 8 lines): 64 (512-thread blocks, two per
// SM), or 128 (1024 threads, one per SM) when the batch gives fewer tiles than SMs and each SM
// evaluates a whole tile alone (1000 lines: 28.9 -> 26.9 us).
int fused_point_threads(int64_t nlines)
{
    int dev = 0, sms = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return (nlines + 7) / 8 < sms ? 128 : 64;
}

int pick_nct(SolveTables const& t, int TL)
{
    // threads per line pair: one per chunk, rounded so the block is whole warps (at least two);
    // returned as threads per line (block = TL * nct)
    int const P = TL / 2;
    int const mult = std::max(1, 32 / P);
    int nthr = (std::max(t.nchunk, 1) + mult - 1) / mult * mult;
    while (P * nthr < 64) nthr += mult;
    while (P * nthr > 1024) nthr -= mult;
    return nthr / 2;
}

} // namespace

bool launch_build_eval_fused(BuildArgs const& args, Evaluator const& e, int order, double* out, Lines const& lo,
                             double const* coords, Lines const& lx, cudaStream_t s);
bool launch_advect_fused(BuildArgs const& args, Evaluator const& e, double const* pts, double dt, double const* velocity,
                         double v_const, int64_t v_div, double* out, Lines const& lo, cudaStream_t s);
void launch_refine(BuildArgs const& args, int TL, int rounds, cudaStream_t s);

namespace {
BuildArgs make_build_args(Builder const& b, double* coefs, Lines const& lc, double const* vals, Lines const& lv,
                          double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi)
{
    BuildArgs args {};
    args.line_base = -1;
    args.t = b.tables;
    args.r = b.rhs;
    args.raw = 0;
    args.nlines = lv.nlines();
    args.vals = vals;
    args.lv = lv;
    args.dlo = dlo;
    args.llo = llo;
    args.dhi = dhi;
    args.lhi = lhi;
    args.out = coefs;
    args.lo = lc;
    args.nct = pick_nct(b.tables, b.tile_lines);
    args.pair16 = line_pairs_aligned(vals, lv);
    args.pair16_out = line_pairs_aligned(coefs, lc);
    return args;
}
} // namespace

bool launch_build_eval(Builder const& b, Evaluator const& e, int order, double* coefs, Lines const& lc,
                       double const* vals, Lines const& lv, double const* dlo, Lines const& llo, double const* dhi,
                       Lines const& lhi, double const* coords, Lines const& lx, double* out, Lines const& lo, cudaStream_t s)
{
    if (lv.nlines() == 0) return true;
    bool fused = false;
    if (b.tile_lines == 8 && b.precision == DDCB_FP64) {
        BuildArgs args = make_build_args(b, coefs, lc, vals, lv, dlo, llo, dhi, lhi);
        // the evaluation part uses every thread
        args.nct = std::max(args.nct, fused_point_threads(args.nlines));
        fused = launch_build_eval_fused(args, e, order, out, lo, coords, lx, s);
    }
    if (!fused) {
        launch_build(b, coefs, lc, vals, lv, dlo, llo, dhi, lhi, s);
        launch_eval(e, order, out, lo, coords, lx, coefs, lc, s);
    }
    return fused;
}

namespace {
// feet[q * nl + b] = pts[q] - dt * v(b): the evaluation coordinates of the unfused advection step.
__global__ void feet_kernel(double* __restrict__ feet, const double* __restrict__ pts, int64_t m, int64_t nl, double dt,
                            const double* __restrict__ velocity, double v_const, int64_t v_div)
{
    int64_t const i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * nl) return;
    int64_t const q = i / nl, b = i % nl;
    feet[i] = __ldg(pts + q) - dt * (velocity ? __ldg(velocity + b / v_div) : v_const);
}
} // namespace

bool launch_advect(Builder const& b, Evaluator const& e, double dt, double const* velocity, double v_const, int64_t v_div,
                   double* out, Lines const& lo, double const* vals, Lines const& lv, double const* dlo, Lines const& llo,
                   double const* dhi, Lines const& lhi, double* coefs, Lines const& lc, cudaStream_t s)
{
    int64_t const nl = lv.nlines(), m = lo.n;
    if (nl == 0 || m == 0) return true;
    if (b.tile_lines == 8 && b.precision == DDCB_FP64) {
        BuildArgs args = make_build_args(b, coefs, lc, vals, lv, dlo, llo, dhi, lhi);
        args.nct = std::max(args.nct, fused_point_threads(args.nlines));
        if (launch_advect_fused(args, e, b.d_points, dt, velocity, v_const, v_div, out, lo, s)) return true;
    }
    // build, feet, evaluate: the coefficients and the feet in stream-ordered scratch
    Lines const lscratch {int64_t(b.basis.size()), nl, nl, 1, 0};
    double* c = coefs;
    double* feet = nullptr;
    if (c == nullptr) DDCB_CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&c), sizeof(double) * size_t(b.basis.size() * nl), s));
    cudaError_t const fe = cudaMallocAsync(reinterpret_cast<void**>(&feet), sizeof(double) * size_t(m * nl), s);
    if (fe != cudaSuccess) {
        if (coefs == nullptr) cudaFreeAsync(c, s);
        throw Error(DDCB_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(fe));
    }
    try {
        Lines const lcc = coefs ? lc : lscratch;
        launch_build(b, c, lcc, vals, lv, dlo, llo, dhi, lhi, s);
        feet_kernel<<<dim3((unsigned)((m * nl + 255) / 256)), dim3(256), 0, s>>>(feet, b.d_points, m, nl, dt, velocity, v_const, v_div);
        DDCB_CUDA_CHECK(cudaGetLastError());
        launch_eval(e, 0, out, lo, feet, Lines {m, nl, nl, 1, 0}, c, lcc, s);
    } catch (...) {
        cudaFreeAsync(feet, s);
        if (coefs == nullptr) cudaFreeAsync(c, s);
        throw;
    }
    DDCB_CUDA_CHECK(cudaFreeAsync(feet, s));
    if (coefs == nullptr) DDCB_CUDA_CHECK(cudaFreeAsync(c, s));
    return false;
}

void launch_build(Builder const& b, double* coefs, Lines const& lc, double const* vals, Lines const& lv,
                  double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi, cudaStream_t s)
{
    BuildArgs args {};
    args.line_base = -1;
    args.t = b.tables;
    args.r = b.rhs;
    args.raw = 0;
    args.nlines = lv.nlines();
    args.vals = vals;
    args.lv = lv;
    args.dlo = dlo;
    args.llo = llo;
    args.dhi = dhi;
    args.lhi = lhi;
    args.out = coefs;
    args.lo = lc;
    args.nct = pick_nct(b.tables, b.tile_lines);
    args.pair16 = line_pairs_aligned(vals, lv);
    args.pair16_out = line_pairs_aligned(coefs, lc);
    if (args.nlines == 0) return;
    // long lines: fewer lines per tile, so that the tile fits in shared memory
    int const kl = b.tables.kl, ku = b.tables.ku;
    int TL;
    if (b.precision == DDCB_FP32_REFINE)
        TL = fit_tile_lines(std::min(b.tile_lines, 8), [&](int w) {
            return sizeof(double) * (size_t)b.tables.n * w + sizeof(float) * tile_doubles(b.tables, w, kl, ku) + 16;
        });
    else
        TL = fit_tile_lines(b.tile_lines, [&](int w) { return sizeof(double) * tile_doubles(b.tables, w, kl, ku); });
    args.nct = pick_nct(b.tables, TL);
    if (b.precision == DDCB_FP32_REFINE) launch_refine(args, TL, b.refine_rounds, s);
    else dispatch(args, TL, s);
}

void launch_solve_multirhs(Builder const& b, double* rhs, long ld, long nrhs, bool transpose, cudaStream_t s)
{
    BuildArgs args {};
    args.line_base = -1;
    args.t = transpose ? b.tables_t : b.tables;
    args.r = b.rhs;
    args.raw = 1;
    // A x = b: rows enter rotated by rrot, the solution leaves rotated by crot; A^T swaps the two
    args.r.lrot = transpose ? b.crot : b.rrot;
    args.r.srot = transpose ? b.rrot : b.crot;
    args.r.periodic = 0;
    args.nlines = nrhs;
    Lines L {b.n, ld, nrhs, 1, 0};
    args.vals = rhs;
    args.lv = L;
    args.out = rhs;
    args.lo = L;
    args.nct = pick_nct(args.t, b.tile_lines);
    args.pair16 = args.pair16_out = line_pairs_aligned(rhs, L);
    if (nrhs == 0) return;
    int const TL = fit_tile_lines(b.tile_lines, [&](int w) { return sizeof(double) * tile_doubles(args.t, w, args.t.kl, args.t.ku); });
    args.nct = pick_nct(args.t, TL);
    dispatch(args, TL, s);
}

} // namespace ddcb
