// quadrature.cu -- the quadrature weights of a builder on the device and the batched integral of
// the interpolating spline straight from the samples.
//
// SplineBuilder::quadrature_coefficients (spline_builder.hpp:1103-1234) solves A^T q = I, with I_j
// the integral of B-spline j (integrals.hpp), so that the integral of the spline built from a
// right-hand side f is I . A^-1 f = q . f. Here the transposed solve is the device kernel of the
// multi-right-hand-side solve (in place, on one column), run once when the builder is created;
// the weights stay on the device. integrate_samples then computes, per batch line, the integral
// of the spline interpolating its samples (and Hermite derivatives) as one dot product: a single
// read of the samples, with no coefficient array written or read -- the builder and
// SplineEvaluator::integrate fused into one HBM pass.
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
    const double* q;     // n weights, reference row order, Hermite rows scaled by dx^k
    int nbe_lo, npoints; // value k of a line pairs with q[nbe_lo + k] (nbe_lo = 0 when periodic)
    int nbv_lo, nbv_hi;  // derivative k pairs with q[k] (lower) / q[n - nbe_hi + k] (upper)
    int hi0;             // n - nbe_hi
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
        const double* q = a.q + a.nbe_lo;
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
            for (int k = 0; k < a.nbv_lo; ++k) acc = fma(__ldg(a.q + k), a.dlo[k * a.llo.stride + line_off(a.llo, line)], acc);
            for (int k = 0; k < a.nbv_hi; ++k)
                acc = fma(__ldg(a.q + a.hi0 + k), a.dhi[k * a.lhi.stride + line_off(a.lhi, line)], acc);
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
    DDCB_CUDA_CHECK(cudaStreamSynchronize(s));
}

void launch_integrate_samples(Builder const& b, double* out, int64_t out_outer_stride, double const* vals, Lines const& lv,
                              double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi, cudaStream_t s)
{
    IntegrateArgs a {};
    a.q = b.d_quad;
    a.nbe_lo = b.rhs.periodic ? 0 : b.nbe_lo;
    a.npoints = int(b.points.size());
    a.nbv_lo = dlo ? b.nbv_lo : 0;
    a.nbv_hi = dhi ? b.nbv_hi : 0;
    a.hi0 = int(b.n) - b.nbe_hi;
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
