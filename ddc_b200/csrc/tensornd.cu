// tensornd.cu -- tensor-product 3D builder and N-dimensional evaluator / integrator
// (SplineBuilder3D, spline_builder_3d.hpp:597-1126; SplineEvaluator3D, spline_evaluator_3d.hpp;
// SplineEvaluatorND, spline_evaluator_nd.hpp:306-827) for the layout (x1, ..., xN, batch) with the
// batch contiguous.
//
// Builder. Each dimension's 1D solve maps its extended samples -- [lower Hermite derivatives,
// values, upper Hermite derivatives] -- to coefficients, and the tensor-product coefficients are
// these maps applied one dimension after the other. Pass 1 reads the caller's 27 separate arrays
// (values, derivative slabs, mixed derivatives: one 1D build per combination of the kinds of
// dimensions 2 and 3, the data of the kinds of dimension 1 entering as the build's value and
// Hermite inputs) and writes one extended array W1 (s1, e2, e3, B); pass 2 builds along
// dimension 2 of W1 into W2 (s1, s2, e3, B), its Hermite rows being rows of W1; pass 3 builds
// along dimension 3 of W2 into the coefficients. Every pass is the 1D build kernel with strided
// line descriptors. This is the reference's schedule (builder 1 over the derivative slabs and
// the values, then the 2D builder over dimensions 2-3) with the intermediate arrays of one
// layout, so passes 2 and 3 are a single launch each.
//
// Evaluator. A warp evaluates one point of 32 batch entries: each lane computes the basis of its
// own coordinates dimension by dimension (degree and derivative order chosen at run time), and the
// prod(d_k + 1) coefficient gathers of a point are coalesced 256-byte loads when the lanes share
// the point's cell. Values of 3D splines with one degree in all dimensions run an unrolled kernel
// (the basis in registers, the (d+1)^3 gathers unrolled); other cases the general one.
#include <algorithm>
#include <string>

#include "build_device.cuh"
#include "eval_device.cuh"

namespace ddcb {

// ---------------------------------------------------------------------------------------------
// 3D builder
// ---------------------------------------------------------------------------------------------
namespace {

// Rows of each kind along a dimension: 0 values, 1 lower derivatives, 2 upper derivatives (0 rows
// when that side is not HERMITE), and where each kind starts in the extended layout.
struct DimRows
{
    int64_t count[3];
    int64_t start[3];
    int64_t ext;
};

DimRows dim_rows(Builder const& b)
{
    DimRows r {};
    r.count[0] = int64_t(b.points.size());
    r.count[1] = b.lo == DDCB_HERMITE ? b.nbv_lo : 0;
    r.count[2] = b.hi == DDCB_HERMITE ? b.nbv_hi : 0;
    r.start[1] = 0;
    r.start[0] = r.count[1];
    r.start[2] = r.count[1] + r.count[0];
    r.ext = r.count[0] + r.count[1] + r.count[2];
    return r;
}

} // namespace

size_t build3d_workspace_bytes(Builder const& b1, Builder const& b2, Builder const& b3, int64_t B)
{
    DimRows const r2 = dim_rows(b2), r3 = dim_rows(b3);
    int64_t const s1 = b1.basis.size(), s2 = b2.basis.size();
    return size_t(8) * size_t(s1) * size_t(r3.ext) * size_t(B) * size_t(r2.ext + s2);
}

void launch_build3d(Builder const& b1, Builder const& b2, Builder const& b3, double* coefs,
                    double const* const* inputs, int64_t B, double* ws, cudaStream_t s)
{
    DimRows const r1 = dim_rows(b1), r2 = dim_rows(b2), r3 = dim_rows(b3);
    int64_t const s1 = b1.basis.size(), s2 = b2.basis.size(), s3 = b3.basis.size();
    int64_t const e2 = r2.ext, e3 = r3.ext;
    double* W1 = ws;                  // (s1, e2, e3, B)
    double* W2 = ws + s1 * e2 * e3 * B; // (s1, s2, e3, B)
    Lines const none {0, 1, 0, 0, 0};
    // ---- pass 1: dimension 1, one build per (kind2, kind3); the derivative slabs (short launches)
    //      on a second stream beside the values, joined before pass 2 ----
    bool const slabs = r2.count[1] + r2.count[2] + r3.count[1] + r3.count[2] > 0;
    SideStream* side = slabs ? &side_stream_for_current_device() : nullptr;
    if (side) {
        DDCB_CUDA_CHECK(cudaEventRecord(side->fork, s));
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(side->stream, side->fork, 0));
    }
    for (int k3 = 0; k3 < 3; ++k3) {
        for (int k2 = 0; k2 < 3; ++k2) {
            int64_t const n2 = r2.count[k2], n3 = r3.count[k3];
            if (n2 == 0 || n3 == 0) continue;
            int const base = 3 * k2 + 9 * k3;
            double const* v = inputs[base];
            if (v == nullptr) throw Error(DDCB_ERR_INVALID_ARGUMENT, "build3d: input " + std::to_string(base) + " is NULL");
            // input arrays (e1, n2, n3, B): lines (i2, (i3, b)) with the (i3, b) part contiguous
            auto in_lines = [&](int64_t n1) { return Lines {n1, n2 * n3 * B, n3 * B, n2, n3 * B}; };
            double const* dlo = r1.count[1] ? inputs[base + 1] : nullptr;
            double const* dhi = r1.count[2] ? inputs[base + 2] : nullptr;
            if ((r1.count[1] && !dlo) || (r1.count[2] && !dhi))
                throw Error(DDCB_ERR_INVALID_ARGUMENT, "build3d: a Hermite input of dimension 1 is NULL");
            // output: the (kind2, kind3) block of W1, rows start2.., start3..
            double* out = W1 + (r2.start[k2] * e3 + r3.start[k3]) * B;
            Lines const lo {s1, e2 * e3 * B, n3 * B, n2, e3 * B};
            launch_build(b1, out, lo, v, in_lines(r1.count[0]), dlo, dlo ? in_lines(r1.count[1]) : none, dhi,
                         dhi ? in_lines(r1.count[2]) : none, (side && base != 0) ? side->stream : s);
        }
    }
    if (side) {
        DDCB_CUDA_CHECK(cudaEventRecord(side->join, side->stream));
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(s, side->join, 0));
    }
    // ---- pass 2: dimension 2 of W1 (s1, e2, e3*B) -> W2 (s1, s2, e3*B) ----
    {
        int64_t const Q = e3 * B;
        auto lines = [&](int64_t n) { return Lines {n, Q, Q, s1, e2 * Q}; };
        double const* dlo = r2.count[1] ? W1 + r2.start[1] * Q : nullptr;
        double const* dhi = r2.count[2] ? W1 + r2.start[2] * Q : nullptr;
        launch_build(b2, W2, Lines {s2, Q, Q, s1, s2 * Q}, W1 + r2.start[0] * Q, lines(r2.count[0]), dlo,
                     dlo ? lines(r2.count[1]) : none, dhi, dhi ? lines(r2.count[2]) : none, s);
    }
    // ---- pass 3: dimension 3 of W2 (s1*s2, e3, B) -> coefs (s1*s2, s3, B) ----
    {
        auto lines = [&](int64_t n) { return Lines {n, B, B, s1 * s2, e3 * B}; };
        double const* dlo = r3.count[1] ? W2 + r3.start[1] * B : nullptr;
        double const* dhi = r3.count[2] ? W2 + r3.start[2] * B : nullptr;
        launch_build(b3, coefs, Lines {s3, B, B, s1 * s2, s3 * B}, W2 + r3.start[0] * B, lines(r3.count[0]), dlo,
                     dlo ? lines(r3.count[1]) : none, dhi, dhi ? lines(r3.count[2]) : none, s);
    }
}

// ---------------------------------------------------------------------------------------------
// N-dimensional evaluator and integrator
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int kPtsNd = 8; // points (warps) per block; 32 batch entries per warp

struct EvalNdArgs
{
    int ndims;
    int deriv;                      // 0: values with boundary handling; 1: orders[] (no boundary handling)
    EvalBasis eb[kMaxDims];
    int ex_lo[kMaxDims], ex_hi[kMaxDims];
    int order[kMaxDims];
    int64_t cstride[kMaxDims];      // element stride of coefficient dimension d
    const double* coords;           // (m, B, ndims)
    const double* coefs;            // (s_1, ..., s_N, B)
    double* out;                    // (m, B)
    int64_t m, B;
};

// Basis values (or their order-th derivatives) of one dimension with the degree and order known
// only at run time: dispatch to the compiled (degree, order, uniform) variants. Returns jmin.
__device__ __noinline__ int basis_rt(EvalBasis const& eb, int order, double x, double* v)
{
    bool const u = eb.b.uniform != 0;
#define DDCB_BRT(D, O)                                                                              \
    case D * 8 + O:                                                                                 \
        return u ? basis_derivs<D, O, true>(eb, x, v) : basis_derivs<D, O, false>(eb, x, v);
    switch (eb.b.degree * 8 + order) {
        DDCB_BRT(1, 0) DDCB_BRT(1, 1)
        DDCB_BRT(2, 0) DDCB_BRT(2, 1) DDCB_BRT(2, 2)
        DDCB_BRT(3, 0) DDCB_BRT(3, 1) DDCB_BRT(3, 2) DDCB_BRT(3, 3)
        DDCB_BRT(4, 0) DDCB_BRT(4, 1) DDCB_BRT(4, 2) DDCB_BRT(4, 3) DDCB_BRT(4, 4)
        DDCB_BRT(5, 0) DDCB_BRT(5, 1) DDCB_BRT(5, 2) DDCB_BRT(5, 3) DDCB_BRT(5, 4) DDCB_BRT(5, 5)
    default: break;
    }
#undef DDCB_BRT
    return 0;
}

// sum over the tensor stencil of c(jmin + i) * prod_d v[d][i_d] (spline_evaluator_nd.hpp:766-825),
// with a running product per level of the odometer.
__device__ double tensor_sum(EvalNdArgs const& a, const double* C, const int* jmin, double v[][kMaxDegree + 1])
{
    int const N = a.ndims;
    int idx[kMaxDims];
    double w[kMaxDims + 1];
    int64_t off[kMaxDims + 1];
    w[0] = 1.0;
    off[0] = 0;
    for (int d = 0; d < N; ++d) {
        idx[d] = 0;
        w[d + 1] = w[d] * v[d][0];
        off[d + 1] = off[d] + (int64_t)jmin[d] * a.cstride[d];
    }
    double y = 0.0;
    while (true) {
        y = fma(__ldg(C + off[N]), w[N], y);
        int d = N - 1;
        while (d >= 0 && idx[d] == a.eb[d].b.degree) {
            idx[d] = 0;
            --d;
        }
        if (d < 0) break;
        ++idx[d];
        // refresh the levels from d down
        for (int e = d; e < N; ++e) {
            w[e + 1] = w[e] * v[e][idx[e]];
            off[e + 1] = off[e] + (int64_t)(jmin[e] + idx[e]) * a.cstride[e];
        }
    }
    return y;
}

__global__ void __launch_bounds__(32 * kPtsNd) evalnd_kernel(const __grid_constant__ EvalNdArgs a, int64_t pts_per_block)
{
    int const lane = threadIdx.x & 31;
    int const wp = threadIdx.x >> 5;
    int64_t const b = (int64_t)blockIdx.y * 32 + lane;
    if (b >= a.B) return;
    int64_t const p0 = (int64_t)blockIdx.x * pts_per_block;
    int64_t const p1 = min(p0 + pts_per_block, a.m);
    int const N = a.ndims;
    const double* C = a.coefs + b;
    for (int64_t p = p0 + wp; p < p1; p += kPtsNd) {
        const double* xp = a.coords + (p * a.B + b) * N;
        double x[kMaxDims];
        for (int d = 0; d < N; ++d) x[d] = xp[d];
        double y = 0.0;
        bool done = false;
        if (!a.deriv) {
            // boundary handling of SplineEvaluatorND::eval (spline_evaluator_nd.hpp:690-720):
            // periodic wraps, then the first non-periodic dimension outside its domain decides
            // (null rule: 0; constant rule: the value at that boundary with every other
            // non-periodic coordinate clamped into its domain, constant_extrapolation_rule.hpp:143-193)
            for (int d = 0; d < N; ++d)
                if (a.eb[d].b.periodic) x[d] = periodic_wrap(a.eb[d].b, x[d]);
            for (int d = 0; d < N && !done; ++d) {
                BasisDesc const& bd = a.eb[d].b;
                if (bd.periodic || (x[d] >= bd.rmin && x[d] <= bd.rmax)) continue;
                bool const low = x[d] < bd.rmin;
                if ((low ? a.ex_lo[d] : a.ex_hi[d]) == DDCB_EXTRAP_NULL) {
                    y = 0.0;
                    done = true;
                } else {
                    x[d] = low ? bd.rmin : bd.rmax;
                    for (int e = 0; e < N; ++e) {
                        BasisDesc const& be = a.eb[e].b;
                        if (e != d && !be.periodic) x[e] = x[e] < be.rmin ? be.rmin : (x[e] > be.rmax ? be.rmax : x[e]);
                    }
                    break;
                }
            }
        }
        if (!done) {
            double v[kMaxDims][kMaxDegree + 1];
            int jmin[kMaxDims];
            for (int d = 0; d < N; ++d) jmin[d] = DDCB_INDEX(basis_rt(a.eb[d], a.deriv ? a.order[d] : 0, x[d], v[d]), a.eb[d].b.ncells);
            y = tensor_sum(a, C, jmin, v);
        }
        a.out[p * a.B + b] = y;
    }
}

// Values (with the boundary handling of evalnd_kernel) of a 3D spline whose three dimensions share
// one degree D: the basis of each dimension in registers and the (D+1)^3 gathers unrolled.
template <int D>
__device__ __forceinline__ int basis_values_any(EvalBasis const& eb, double x, double* v)
{
    return eb.b.uniform ? basis_derivs<D, 0, true>(eb, x, v) : basis_derivs<D, 0, false>(eb, x, v);
}

template <int D>
__global__ void __launch_bounds__(32 * kPtsNd) eval3d_kernel(const __grid_constant__ EvalNdArgs a, int64_t pts_per_block)
{
    int const lane = threadIdx.x & 31;
    int const wp = threadIdx.x >> 5;
    int64_t const b = (int64_t)blockIdx.y * 32 + lane;
    if (b >= a.B) return;
    int64_t const p0 = (int64_t)blockIdx.x * pts_per_block;
    int64_t const p1 = min(p0 + pts_per_block, a.m);
    const double* C = a.coefs + b;
    for (int64_t p = p0 + wp; p < p1; p += kPtsNd) {
        const double* xp = a.coords + (p * a.B + b) * 3;
        double x[3] = {xp[0], xp[1], xp[2]};
        double y = 0.0;
        bool zero = false;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (a.eb[d].b.periodic) x[d] = periodic_wrap(a.eb[d].b, x[d]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            BasisDesc const& bd = a.eb[d].b;
            if (zero || bd.periodic || (x[d] >= bd.rmin && x[d] <= bd.rmax)) continue;
            bool const low = x[d] < bd.rmin;
            if ((low ? a.ex_lo[d] : a.ex_hi[d]) == DDCB_EXTRAP_NULL) {
                zero = true;
            } else {
                x[d] = low ? bd.rmin : bd.rmax;
#pragma unroll
                for (int e = 0; e < 3; ++e) {
                    BasisDesc const& be = a.eb[e].b;
                    if (e != d && !be.periodic) x[e] = x[e] < be.rmin ? be.rmin : (x[e] > be.rmax ? be.rmax : x[e]);
                }
                break;
            }
        }
        if (!zero) {
            double v0[D + 1], v1[D + 1], v2[D + 1];
            int const j0 = DDCB_INDEX(basis_values_any<D>(a.eb[0], x[0], v0), a.eb[0].b.ncells);
            int const j1 = DDCB_INDEX(basis_values_any<D>(a.eb[1], x[1], v1), a.eb[1].b.ncells);
            int const j2 = DDCB_INDEX(basis_values_any<D>(a.eb[2], x[2], v2), a.eb[2].b.ncells);
#pragma unroll
            for (int i0 = 0; i0 <= D; ++i0) {
                double t1 = 0.0;
#pragma unroll
                for (int i1 = 0; i1 <= D; ++i1) {
                    const double* row = C + (int64_t)(j0 + i0) * a.cstride[0] + (int64_t)(j1 + i1) * a.cstride[1]
                                        + (int64_t)j2 * a.cstride[2];
                    double t2 = 0.0;
#pragma unroll
                    for (int i2 = 0; i2 <= D; ++i2) t2 = fma(__ldg(row + i2 * a.cstride[2]), v2[i2], t2);
                    t1 = fma(t2, v1[i1], t1);
                }
                y = fma(t1, v0[i0], y);
            }
        }
        a.out[p * a.B + b] = y;
    }
}

struct IntegrateNdArgs
{
    int ndims;
    const double* ints[kMaxDims]; // integrals of the B-splines of each dimension (device)
    int64_t size[kMaxDims];
    int64_t total;                // prod(size)
    const double* coefs;
    double* out;
    int64_t B;
};

// out[b] = sum over the coefficient grid of c(i, b) prod_d I_d[i_d] (spline_evaluator_nd.hpp:596-633):
// 32 batch entries per block column, 32 slots share the grid, a shared-memory sum at the end.
__global__ void __launch_bounds__(1024) integratend_kernel(const __grid_constant__ IntegrateNdArgs a)
{
    __shared__ double part[32][33];
    int const lane = threadIdx.x & 31, slot = threadIdx.x >> 5;
    int64_t const b = (int64_t)blockIdx.x * 32 + lane;
    double acc = 0.0;
    if (b < a.B) {
        for (int64_t f = slot; f < a.total; f += 32) {
            int64_t r = f;
            double w = 1.0;
            for (int d = a.ndims - 1; d >= 0; --d) {
                int64_t const i = r % a.size[d];
                r /= a.size[d];
                w *= __ldg(a.ints[d] + i);
            }
            acc = fma(a.coefs[f * a.B + b], w, acc);
        }
    }
    part[slot][lane] = acc;
    __syncthreads();
    if (slot == 0 && b < a.B) {
        double s = 0.0;
        for (int q = 0; q < 32; ++q) s += part[q][lane];
        a.out[b] = s;
    }
}

} // namespace

void launch_evalnd(Evaluator const* const* e, int ndims, int const* orders, double* out, double const* coords,
                   double const* coefs, int64_t m, int64_t B, cudaStream_t s)
{
    if (m == 0 || B == 0) return;
    EvalNdArgs a {};
    a.ndims = ndims;
    a.deriv = orders != nullptr;
    int64_t stride = B;
    for (int d = ndims - 1; d >= 0; --d) {
        a.eb[d] = e[d]->eb;
        a.ex_lo[d] = e[d]->ex_lo;
        a.ex_hi[d] = e[d]->ex_hi;
        a.order[d] = orders ? orders[d] : 0;
        a.cstride[d] = stride;
        stride *= e[d]->basis.size();
    }
    a.coords = coords;
    a.coefs = coefs;
    a.out = out;
    a.m = m;
    a.B = B;
    int64_t const ppb = 64;
    dim3 grid((unsigned)((m + ppb - 1) / ppb), (unsigned)((B + 31) / 32));
    // 3D values with one degree in every dimension: the unrolled kernel
    int const D0 = e[0]->basis.desc.degree;
    bool const same3 = ndims == 3 && orders == nullptr && e[1]->basis.desc.degree == D0 && e[2]->basis.desc.degree == D0;
    if (same3) {
        switch (D0) {
        case 1: eval3d_kernel<1><<<grid, 32 * kPtsNd, 0, s>>>(a, ppb); break;
        case 2: eval3d_kernel<2><<<grid, 32 * kPtsNd, 0, s>>>(a, ppb); break;
        case 3: eval3d_kernel<3><<<grid, 32 * kPtsNd, 0, s>>>(a, ppb); break;
        case 4: eval3d_kernel<4><<<grid, 32 * kPtsNd, 0, s>>>(a, ppb); break;
        default: eval3d_kernel<5><<<grid, 32 * kPtsNd, 0, s>>>(a, ppb); break;
        }
    } else {
        evalnd_kernel<<<grid, 32 * kPtsNd, 0, s>>>(a, ppb);
    }
    DDCB_CUDA_CHECK(cudaGetLastError());
}

void launch_integratend(Evaluator const* const* e, int ndims, double* out, double const* coefs, int64_t B, cudaStream_t s)
{
    if (B == 0) return;
    IntegrateNdArgs a {};
    a.ndims = ndims;
    a.total = 1;
    for (int d = 0; d < ndims; ++d) {
        a.ints[d] = e[d]->d_integrals;
        a.size[d] = e[d]->basis.size();
        a.total *= a.size[d];
    }
    a.coefs = coefs;
    a.out = out;
    a.B = B;
    integratend_kernel<<<dim3((unsigned)((B + 31) / 32)), dim3(1024), 0, s>>>(a);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

} // namespace ddcb
