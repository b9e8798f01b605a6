// fused_kernels.cu -- build + evaluate in one kernel (the semi-Lagrangian step of
// examples/characteristics_advection.cpp:251-259: SplineBuilder::operator() then
// SplineEvaluator::operator() / deriv on the same lines), and the whole advection step with the
// feet of the characteristics computed in the kernel (:243-250).
//
// The tile solved in shared memory by solve_tile is stored as the coefficient output and then
// evaluated in place: the coefficients are written once and never read back from HBM. Kernels
// exist for the band shapes and tile width the configurations use; any other combination runs the
// builder and the evaluator kernels one after the other (same results).
#include "build_device.cuh"
#include "eval_device.cuh"

namespace ddcb {

namespace {

struct FusedEval
{
    EvalBasis eb;
    int ex_lo, ex_hi;
    const double* coords;
    Lines lx;
    double* out;
    Lines lo;
    // FEET kernels (the advection step): point q of line b is at pts[q] - dt * v(b), with
    // v(b) = velocity[b / v_div] (velocity == NULL: v_const); lx.n is the point count
    const double* pts;
    const double* velocity;
    double v_const, dt;
    int64_t v_div;
};

// FEET: the evaluation coordinates are the feet of the characteristics through the interpolation
// points (computed here, not read), as in examples/characteristics_advection.cpp:243-250.
template <int TL, int KL, int KU, int D, int ORDER, bool UNI, bool FEET = false>
__global__ void __launch_bounds__(1024) build_eval_kernel(const __grid_constant__ BuildArgs args,
                                                          const __grid_constant__ FusedEval fe)
{
    extern __shared__ __align__(16) double smem[];
    // knot pairs (non-uniform) after the tile, at an even double offset (16-byte aligned)
    double2* K = reinterpret_cast<double2*>(smem + ((tile_doubles(args.t, TL, KL, KU) + 1) & ~size_t(1)));
    if (!UNI)
        for (int i = threadIdx.x; i < fe.eb.nk - 1; i += blockDim.x) K[i] = fe.eb.kpairs[i];
    solve_tile<TL, KL, KU>(args, smem);
    if (args.out != nullptr) store_tile<TL>(args, smem);
    int const tid = threadIdx.x;
    int const l = tid % TL;
    int const c = tid / TL;
    int const nct = args.nct;
    int64_t const line = (int64_t)blockIdx.x * TL + l;
    if (line >= args.nlines) return;
    EvalBasis eb = fe.eb;
    if (!UNI) eb.kpairs = K;
    int64_t const ox = line_offset(fe.lx, line);
    int64_t const oo = line_offset(fe.lo, line);
    int64_t const m = fe.lx.n;
    CoefRotated const acc {smem + l, TL, args.t.n, args.r.srot};
    constexpr int U = 8; // points in flight per thread
    int64_t const sx = fe.lx.stride * nct, so = fe.lo.stride * nct;
    const double* __restrict__ xp = fe.coords + ox + c * fe.lx.stride;
    double* __restrict__ op = fe.out + oo + c * fe.lo.stride;
    int const npt = m > c ? int((m - c + nct - 1) / nct) : 0; // points of this thread
    double const shift = FEET ? fe.dt * (fe.velocity ? __ldg(fe.velocity + line / fe.v_div) : fe.v_const) : 0.0;
    for (int q0 = 0; q0 < npt; q0 += U) {
        double xs[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (FEET) xs[u] = (q0 + u < npt) ? __ldg(fe.pts + c + (q0 + u) * nct) - shift : 0.0;
            else xs[u] = (q0 + u < npt) ? __ldcs(xp + (q0 + u) * sx) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (q0 + u < npt) __stcs(op + (q0 + u) * so, eval_point<D, ORDER, UNI>(eb, fe.ex_lo, fe.ex_hi, xs[u], acc));
    }
}

template <int KL, int KU, int D, int ORDER, bool UNI, bool FEET = false>
bool launch5(BuildArgs const& args, FusedEval const& fe, cudaStream_t s)
{
    constexpr int TL = 8;
    size_t const sm = sizeof(double) * (tile_doubles(args.t, TL, KL, KU) + (UNI ? 0 : 2 * (size_t)fe.eb.nk + 2));
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (sm > size_t(optin)) return false;
    auto kern = build_eval_kernel<TL, KL, KU, D, ORDER, UNI, FEET>;
    if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    int64_t const grid = (args.nlines + TL - 1) / TL;
    kern<<<dim3((unsigned)grid), dim3(TL * args.nct), sm, s>>>(args, fe);
    DDCB_CUDA_CHECK(cudaGetLastError());
    return true;
}

// Uniform bases only: on non-uniform meshes the evaluator kernel alone (its own block shape for
// the table lookups) after the builder measured faster than one fused kernel.
template <int KL, int KU, int D>
bool launch_ord(BuildArgs const& args, FusedEval const& fe, int order, bool uni, cudaStream_t s)
{
    if (!uni) return false;
    if (order == 0) return launch5<KL, KU, D, 0, true>(args, fe, s);
    if (order == 1) return launch5<KL, KU, D, 1, true>(args, fe, s);
    return false;
}

// The advection step: values at the feet, uniform bases.
template <int KL, int KU>
bool launch_feet(BuildArgs const& args, FusedEval const& fe, cudaStream_t s)
{
    if (fe.eb.b.uniform == 0) return false;
    switch (fe.eb.b.degree) {
    case 1: return launch5<KL, KU, 1, 0, true, true>(args, fe, s);
    case 2: return launch5<KL, KU, 2, 0, true, true>(args, fe, s);
    case 3: return launch5<KL, KU, 3, 0, true, true>(args, fe, s);
    case 4: return launch5<KL, KU, 4, 0, true, true>(args, fe, s);
    case 5: return launch5<KL, KU, 5, 0, true, true>(args, fe, s);
    default: return false;
    }
}

template <int KL, int KU>
bool launch_deg(BuildArgs const& args, FusedEval const& fe, int order, cudaStream_t s)
{
    bool const uni = fe.eb.b.uniform != 0;
    switch (fe.eb.b.degree) {
    case 1: return launch_ord<KL, KU, 1>(args, fe, order, uni, s);
    case 2: return launch_ord<KL, KU, 2>(args, fe, order, uni, s);
    case 3: return launch_ord<KL, KU, 3>(args, fe, order, uni, s);
    case 4: return launch_ord<KL, KU, 4>(args, fe, order, uni, s);
    case 5: return launch_ord<KL, KU, 5>(args, fe, order, uni, s);
    default: return false;
    }
}

} // namespace

// Returns false when no fused kernel covers this combination (the caller then runs the two
// kernels back to back).
bool launch_build_eval_fused(BuildArgs const& args, Evaluator const& e, int order, double* out, Lines const& lo,
                             double const* coords, Lines const& lx, cudaStream_t s)
{
    FusedEval fe {};
    fe.eb = e.eb;
    fe.ex_lo = e.ex_lo;
    fe.ex_hi = e.ex_hi;
    fe.coords = coords;
    fe.lx = lx;
    fe.out = out;
    fe.lo = lo;
    int const kl = args.t.kl, ku = args.t.ku;
    if (kl == 1 && ku == 1) return launch_deg<1, 1>(args, fe, order, s);
    if (kl == 2 && ku == 2) return launch_deg<2, 2>(args, fe, order, s);
    if (kl == 3 && ku == 3) return launch_deg<3, 3>(args, fe, order, s);
    if (kl == 4 && ku == 4) return launch_deg<4, 4>(args, fe, order, s);
    return false;
}

bool launch_advect_fused(BuildArgs const& args, Evaluator const& e, double const* pts, double dt, double const* velocity,
                         double v_const, int64_t v_div, double* out, Lines const& lo, cudaStream_t s)
{
    FusedEval fe {};
    fe.eb = e.eb;
    fe.ex_lo = e.ex_lo;
    fe.ex_hi = e.ex_hi;
    fe.lx = lo;
    fe.out = out;
    fe.lo = lo;
    fe.pts = pts;
    fe.velocity = velocity;
    fe.v_const = v_const;
    fe.dt = dt;
    fe.v_div = v_div;
    int const kl = args.t.kl, ku = args.t.ku;
    if (kl == 1 && ku == 1) return launch_feet<1, 1>(args, fe, s);
    if (kl == 2 && ku == 2) return launch_feet<2, 2>(args, fe, s);
    if (kl == 3 && ku == 3) return launch_feet<3, 3>(args, fe, s);
    if (kl == 4 && ku == 4) return launch_feet<4, 4>(args, fe, s);
    return false;
}

} // namespace ddcb
