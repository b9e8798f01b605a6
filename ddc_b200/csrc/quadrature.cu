// quadrature.cu -- the quadrature weights of a builder on the device and the batched integral of
// the interpolating spline straight from the samples.
//
// SplineBuilder::quadrature_coefficients (spline_builder.hpp:1103-1234) solves A^T q = I, with I_j
// the integral of B-spline j (integrals.hpp), so that the integral of the spline built from a
// right-hand side f is I . A^-1 f = q . f. Here the transposed solve is the device kernel of the
// multi-right-hand-side solve (in place, on one column), run once, on the builder's first use of
// its weights; the weights stay on the device.
//
// The reference takes I in basis order without the periodic column offset of the builder
// (spline_builder.hpp:619-658, 1061-1100), so on non-uniform periodic bases with a non-zero offset
// (degree >= 2), whose B-spline integrals differ, its q . f is not the integral of the spline the
// builder returns. quadrature_coefficients keeps the reference's numbers. integrate_samples uses
// the exact weights instead: the builder's adjoint applied to I (w = R^T A^-T P^T I, with the
// offset, the periodic duplicates and the dx^k scaling of Hermite inputs), so that, per batch line,
// w . (samples, derivatives) is the integral of the interpolating spline -- one read of the
// samples, with no coefficient array written or read: the builder and SplineEvaluator::integrate
// fused into one HBM pass.
#include <algorithm>
#include <vector>

#include "ddcb_internal.hpp"

namespace ddcb {

namespace {

// q from the solution qk of A^T qk = I (both in the reference's row order), with the rows of the
// Hermite derivatives scaled by dx^k (the derivative inputs are unscaled).
__global__ void scale_hermite_rows_kernel(const double* __restrict__ qk, double* __restrict__ q, int n, int nbv_lo,
                                          int nbv_hi, double dx, int odd)
{
    int const r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double v = qk[r];
    int e = -1;
    if (r < nbv_lo) e = r + odd;
    else if (r >= n - nbv_hi) e = r - (n - nbv_hi) + odd;
    if (e >= 0) {
        double p = 1.0;
        for (int t = 0; t < e; ++t) p *= dx;
        v *= p;
    }
    q[r] = v;
}

struct IntegrateArgs
{
    const double* w;     // value k pairs with w[k], lower derivative k with w[npoints + k], upper
    int npoints;         // derivative k with w[npoints + nbv_lo_all + k]
    int nbv_lo, nbv_hi;  // derivative rows read (0 when the data are not given)
    int nbv_lo_all;
    int64_t nlines;
    const double* vals;
    Lines lv;
    const double* dlo;
    Lines llo;
    const double* dhi;
    Lines lhi;
    double* out;
    int64_t out_outer_stride;
};

__device__ __forceinline__ int64_t line_off(Lines const& L, int64_t b) { return (b / L.inner) * L.outer_stride + (b % L.inner); }

// A block holds 32 consecutive lines x S row slices: lane l of slice s sums rows s, s + S, ... of
// line l (coalesced over the contiguous batch), then the slices are added in shared memory.
template <int S>
__global__ void __launch_bounds__(32 * S) integrate_samples_kernel(const __grid_constant__ IntegrateArgs a)
{
    __shared__ double part[S][33];
    int const l = threadIdx.x & 31, s = threadIdx.x >> 5;
    int64_t const line = (int64_t)blockIdx.x * 32 + l;
    double acc = 0.0;
    if (line < a.nlines) {
        const double* v = a.vals + line_off(a.lv, line);
        const double* q = a.w;
        int r = s;
        // four independent partial sums keep several loads in flight
        double acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
        for (; r + 3 * S < a.npoints; r += 4 * S) {
            acc = fma(__ldg(q + r), __ldcs(v + (int64_t)r * a.lv.stride), acc);
            acc1 = fma(__ldg(q + r + S), __ldcs(v + (int64_t)(r + S) * a.lv.stride), acc1);
            acc2 = fma(__ldg(q + r + 2 * S), __ldcs(v + (int64_t)(r + 2 * S) * a.lv.stride), acc2);
            acc3 = fma(__ldg(q + r + 3 * S), __ldcs(v + (int64_t)(r + 3 * S) * a.lv.stride), acc3);
        }
        for (; r < a.npoints; r += S) acc = fma(__ldg(q + r), __ldcs(v + (int64_t)r * a.lv.stride), acc);
        acc += (acc1 + acc2) + acc3;
        if (s == 0) {
            const double* wd = a.w + a.npoints;
            for (int k = 0; k < a.nbv_lo; ++k) acc = fma(__ldg(wd + k), a.dlo[k * a.llo.stride + line_off(a.llo, line)], acc);
            wd += a.nbv_lo_all;
            for (int k = 0; k < a.nbv_hi; ++k) acc = fma(__ldg(wd + k), a.dhi[k * a.lhi.stride + line_off(a.lhi, line)], acc);
        }
    }
    part[s][l] = acc;
    __syncthreads();
    if (s == 0 && line < a.nlines) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < S; ++k) t += part[k][l];
        a.out[(line / a.lv.inner) * a.out_outer_stride + line % a.lv.inner] = t;
    }
}

} // namespace

void compute_device_quadrature(Builder& b, double* d_qk, double* d_q)
{
    // right-hand side: the integrals of the first n B-splines in basis order (the periodic
    // duplicates are not part of the system); the multi-right-hand-side solve takes and returns
    // the reference's row / column order (it applies the kernel's rotations itself)
    long const n = b.n;
    std::vector<double> ints(b.basis.size());
    basis_integrals(b.basis, ints.data());
    DDCB_CUDA_CHECK(cudaMemcpy(d_qk, ints.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    cudaStream_t const s = nullptr;
    launch_solve_multirhs(b, d_qk, 1, 1, true, s);
    scale_hermite_rows_kernel<<<dim3((unsigned)((n + 127) / 128)), dim3(128), 0, s>>>(d_qk, d_q, int(n), b.nbv_lo, b.nbv_hi,
                                                                                  b.dx, b.odd);
    DDCB_CUDA_CHECK(cudaGetLastError());
    // the exact integration weights: the builder adjoint of the integrals of all size() B-splines
    // (one line; the integrals follow q in the block, the weights follow them)
    long const sz = b.basis.size();
    double* const d_ints = d_q + n;
    DDCB_CUDA_CHECK(cudaMemcpy(d_ints, ints.data(), sizeof(double) * sz, cudaMemcpyHostToDevice));
    long const np = long(b.points.size());
    bool const hlo = b.lo == DDCB_HERMITE && b.nbv_lo > 0, hhi = b.hi == DDCB_HERMITE && b.nbv_hi > 0;
    Lines const none {0, 1, 0, 0, 0};
    launch_build_adjoint(b, d_ints, Lines {sz, 1, 1, 1, 0}, b.d_iweights, Lines {np, 1, 1, 1, 0},
                         hlo ? b.d_iweights + np : nullptr, hlo ? Lines {b.nbv_lo, 1, 1, 1, 0} : none,
                         hhi ? b.d_iweights + np + b.nbv_lo : nullptr, hhi ? Lines {b.nbv_hi, 1, 1, 1, 0} : none, s);
    DDCB_CUDA_CHECK(cudaStreamSynchronize(s));
}

void launch_integrate_samples(Builder const& b, double* out, int64_t out_outer_stride, double const* vals, Lines const& lv,
                              double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi, cudaStream_t s)
{
    IntegrateArgs a {};
    a.w = b.d_iweights;
    a.npoints = int(b.points.size());
    a.nbv_lo = dlo ? b.nbv_lo : 0;
    a.nbv_hi = dhi ? b.nbv_hi : 0;
    a.nbv_lo_all = (b.lo == DDCB_HERMITE) ? b.nbv_lo : 0;
    a.nlines = lv.nlines();
    a.vals = vals;
    a.lv = lv;
    a.dlo = dlo;
    a.llo = llo;
    a.dhi = dhi;
    a.lhi = lhi;
    a.out = out;
    a.out_outer_stride = out_outer_stride;
    if (a.nlines == 0) return;
    unsigned const blocks = (unsigned)((a.nlines + 31) / 32);
    // few lines: more row slices per line, so the grid still fills the GPU
    if (a.nlines <= 8192) integrate_samples_kernel<32><<<blocks, 32 * 32, 0, s>>>(a);
    else integrate_samples_kernel<8><<<blocks, 32 * 8, 0, s>>>(a);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

} // namespace ddcb
