// eval_kernels.cu -- batched spline evaluation, differentiation and integration
// (SplineEvaluator::operator(), ::deriv, ::integrate; spline_evaluator.hpp:257-526).
//
// A thread block owns TLE batch lines: it stages their coefficient rows in shared memory once
// (coalesced over the contiguous batch dimension) and then evaluates every point of those lines,
// gathering the degree+1 coefficients of each point from shared memory. The basis values are
// computed in registers with the degree known at compile time. Derivatives of order n use the
// derivative spline: n rounds of divided differences of the coefficients (de Boor, "A Practical
// Guide to Splines", X.(15)) followed by the degree-(d-n) basis. On non-uniform meshes, values and
// first derivatives divide by knot differences (one batched division per level of the triangle);
// higher orders read the knot-span inverses from a table built with the evaluator.
#include <algorithm>

#include "ddcb_internal.hpp"
#include "eval_device.cuh"

namespace ddcb {

namespace {

struct EvalArgs
{
    EvalBasis eb;
    int ex_lo, ex_hi;
    int64_t nlines;
    int size;           // coefficient rows
    const double* coords;
    Lines lx;
    const double* coefs;
    Lines lc;
    double* out;
    Lines lo;
    int pair16;         // coefs: adjacent line pairs 16-byte aligned and contiguous
    int lut_smem;       // non-uniform: bucket table copied to shared memory after the knot pairs
};

__device__ __forceinline__ int64_t line_offset(Lines const& L, int64_t b)
{
    return (b / L.inner) * L.outer_stride + (b % L.inner);
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src)
{
    unsigned const s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

constexpr int kEvalThreads = 640; // 20 warps: one block per SM at up to 102 registers

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    unsigned const s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

template <int D, int TLE, int ORDER, bool UNI>
__global__ void __launch_bounds__(kEvalThreads) eval_kernel(const __grid_constant__ EvalArgs a)
{
    extern __shared__ __align__(16) double smem[];
    double* C = smem;                                  // size x TLE coefficient tile
    double2* K = reinterpret_cast<double2*>(C + (size_t)a.size * TLE); // knot pairs (non-uniform)
    int const tid = threadIdx.x;
    int const l = tid % TLE;
    int const c = tid / TLE;
    int const nct = blockDim.x / TLE;
    int64_t const line = (int64_t)blockIdx.x * TLE + l;
    bool const live = line < a.nlines;
    // First derivatives on non-uniform bases evaluate the derivative spline: once the tile is in,
    // it is turned into d_j = D (c_j - c_{j-1}) / (t_{j+D} - t_j) (row 0 unused), once per line
    // instead of once per point (below).
    constexpr bool DSPLINE = !UNI && ORDER == 1 && D >= 2;
    if (a.pair16) {
        // two lines per 16-byte copy (cp.async.cg bypasses L1, where the basis tables live)
        int const p = tid % (TLE / 2);
        int const c2 = tid / (TLE / 2);
        int64_t const l0 = (int64_t)blockIdx.x * TLE + 2 * p;
        if (l0 + 1 < a.nlines) {
            int64_t const oc = line_offset(a.lc, l0);
            for (int r = c2; r < a.size; r += 2 * nct) cp_async16(C + r * TLE + 2 * p, a.coefs + r * a.lc.stride + oc);
        } else if (l0 < a.nlines) {
            int64_t const oc = line_offset(a.lc, l0);
            for (int r = c2; r < a.size; r += 2 * nct) cp_async8(C + r * TLE + 2 * p, a.coefs + r * a.lc.stride + oc);
        }
    } else if (live) {
        int64_t const oc = line_offset(a.lc, line);
        for (int r = c; r < a.size; r += nct) cp_async8(C + r * TLE + l, a.coefs + r * a.lc.stride + oc);
    }
    double2* L = K + a.eb.nk; // bucket table (non-uniform, lut_smem)
    if (!UNI) {
        for (int i = tid; i < a.eb.nk - 1; i += blockDim.x) cp_async16(K + i, a.eb.kpairs + i);
        if (a.lut_smem)
            for (int i = tid; i < a.eb.nbucket; i += blockDim.x) cp_async16(L + i, a.eb.lut + i);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (DSPLINE) {
        // in place: each thread owns a contiguous run of rows of its line, keeps the row before the
        // run, and converts the run from its end (c_{j-1} is read before d_{j-1} replaces it)
        int const per = (a.size + nct - 1) / nct;
        int const r0 = c * per, r1 = min(a.size, r0 + per);
        double const before = (live && r0 > 0 && r0 < a.size) ? C[(r0 - 1) * TLE + l] : 0.0;
        __syncthreads();
        if (live && r0 < r1) {
            const double* g = a.eb.inv_span + (size_t)(D - 1) * a.eb.nk; // 1/(t_{j+D} - t_j) at g[j]
            double cj = C[(r1 - 1) * TLE + l];
            for (int j = r1 - 1; j >= r0; --j) {
                double const cprev = j > r0 ? C[(j - 1) * TLE + l] : before;
                C[j * TLE + l] = j > 0 ? double(D) * (cj - cprev) * __ldg(g + j) : 0.0;
                cj = cprev;
            }
        }
        __syncthreads();
    }
    if (!live) return;
    EvalBasis eb = a.eb;
    if (!UNI) {
        eb.kpairs = K;
        if (a.lut_smem) eb.lut = L;
    }
    int64_t const ox = line_offset(a.lx, line);
    int64_t const oo = line_offset(a.lo, line);
    int64_t const m = a.lx.n;
    CoefDirect const acc {C + l, TLE};
    // points in flight per thread: 16 for the derivative spline (its coordinates loaded together,
    // 0.78 -> 0.73 ms on 65536 quintic lines), 8 elsewhere (16 spills the other variants)
    constexpr int U = DSPLINE ? 16 : 8;
    int64_t const sx = a.lx.stride * nct, so = a.lo.stride * nct;
    const double* __restrict__ xp = a.coords + ox + c * a.lx.stride;
    double* __restrict__ op = a.out + oo + c * a.lo.stride;
    int const npt = m > c ? int((m - c + nct - 1) / nct) : 0; // points of this thread
    for (int q0 = 0; q0 < npt; q0 += U) {
        double xs[U];
#pragma unroll
        for (int u = 0; u < U; ++u) xs[u] = (q0 + u < npt) ? __ldcs(xp + (q0 + u) * sx) : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (q0 + u >= npt) continue;
            double y;
            if constexpr (DSPLINE) y = nonuniform_deriv1_dcoef<D>(eb, xs[u], acc);
            else y = eval_point<D, ORDER, UNI>(eb, a.ex_lo, a.ex_hi, xs[u], acc);
            __stcs(op + (q0 + u) * so, y);
        }
    }
}

template <int D, int TLE, bool UNI>
void launch_order(EvalArgs const& a, int order, size_t sm, cudaStream_t s)
{
    dim3 grid((unsigned)((a.nlines + TLE - 1) / TLE)), block(kEvalThreads);
#define DDCB_EVAL_CASE(O)                                                                                  \
    case O:                                                                                                \
        if constexpr (O <= D) {                                                                            \
            auto k = eval_kernel<D, TLE, O, UNI>;                                                          \
            if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm))); \
            k<<<grid, block, sm, s>>>(a);                                                                  \
        }                                                                                                  \
        break;
    switch (order) {
        DDCB_EVAL_CASE(0)
        DDCB_EVAL_CASE(1)
        DDCB_EVAL_CASE(2)
        DDCB_EVAL_CASE(3)
        DDCB_EVAL_CASE(4)
        DDCB_EVAL_CASE(5)
    default: break;
    }
#undef DDCB_EVAL_CASE
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int TLE>
void launch_deg(EvalArgs const& a, int order, size_t sm, cudaStream_t s)
{
    bool const uni = a.eb.b.uniform != 0;
    switch (a.eb.b.degree) {
    case 1: uni ? launch_order<1, TLE, true>(a, order, sm, s) : launch_order<1, TLE, false>(a, order, sm, s); break;
    case 2: uni ? launch_order<2, TLE, true>(a, order, sm, s) : launch_order<2, TLE, false>(a, order, sm, s); break;
    case 3: uni ? launch_order<3, TLE, true>(a, order, sm, s) : launch_order<3, TLE, false>(a, order, sm, s); break;
    case 4: uni ? launch_order<4, TLE, true>(a, order, sm, s) : launch_order<4, TLE, false>(a, order, sm, s); break;
    case 5: uni ? launch_order<5, TLE, true>(a, order, sm, s) : launch_order<5, TLE, false>(a, order, sm, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "degree must be in 1..5");
    }
}

__global__ void integrate_kernel(const double* __restrict__ coefs, Lines lc, const double* __restrict__ ints, int size,
                                 double* __restrict__ out, int64_t out_outer_stride, int64_t nlines)
{
    int64_t const line = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= nlines) return;
    int64_t const oc = line_offset(lc, line);
    double s = 0.0;
    for (int i = 0; i < size; ++i) s = fma(coefs[i * lc.stride + oc], __ldg(ints + i), s);
    out[(line / lc.inner) * out_outer_stride + line % lc.inner] = s;
}

} // namespace

void launch_eval(Evaluator const& e, int order, double* out, Lines const& lo, double const* coords, Lines const& lx,
                 double const* coefs, Lines const& lc, cudaStream_t s)
{
    EvalArgs a {};
    a.eb = e.eb;
    a.ex_lo = e.ex_lo;
    a.ex_hi = e.ex_hi;
    a.nlines = lx.nlines();
    a.size = int(e.basis.size());
    a.coords = coords;
    a.lx = lx;
    a.coefs = coefs;
    a.lc = lc;
    a.out = out;
    a.lo = lo;
    a.pair16 = line_pairs_aligned(coefs, lc);
    if (a.nlines == 0 || lx.n == 0) return;
    // sixteen lines per block (a warp then reads two whole 128-byte tile rows per coefficient, and
    // the tile fills move 128-byte row segments), eight or two when the coefficient tile of long
    // lines does not fit; the bucket table of a non-uniform basis joins the knot pairs in shared
    // memory when it fits too
    bool const uni = e.eb.b.uniform != 0;
    auto bytes = [&](int tle, bool lut) {
        return sizeof(double) * ((size_t)a.size * tle + (uni ? 0 : 2 * ((size_t)e.eb.nk + (lut ? (size_t)e.eb.nbucket : 0))));
    };
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    for (int tle : {16, 8, 2})
        for (int lut = uni ? 0 : 1; lut >= 0; --lut)
            if (bytes(tle, lut) <= size_t(optin)) {
                a.lut_smem = lut;
                if (tle == 16) launch_deg<16>(a, order, bytes(16, lut), s);
                else if (tle == 8) launch_deg<8>(a, order, bytes(8, lut), s);
                else launch_deg<2>(a, order, bytes(2, lut), s);
                return;
            }
    throw Error(DDCB_ERR_UNSUPPORTED, "a line of " + std::to_string(a.size) + " coefficients exceeds the evaluator's shared-memory tile");
}

void launch_integrate(Evaluator const& e, double* out, int64_t out_outer_stride, double const* coefs, Lines const& lc,
                      cudaStream_t s)
{
    int64_t const nl = lc.nlines();
    if (nl == 0) return;
    int const bs = 256;
    integrate_kernel<<<dim3((unsigned)((nl + bs - 1) / bs)), dim3(bs), 0, s>>>(coefs, lc, e.d_integrals, int(e.basis.size()),
                                                                              out, out_outer_stride, nl);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

} // namespace ddcb
