// tensor2d.cu -- tensor-product 2D builder and evaluator (SplineBuilder2D, SplineEvaluator2D;
// spline_builder_2d.hpp:526-651, spline_evaluator_2d.hpp:342-826) for the layout
// (x1, x2, batch) with the batch contiguous.
//
// Builder: the reference's four 1D passes (dim-2 derivative slabs and values along x1, then the
// x2 pass over the result), run by the 1D build kernel with strided line descriptors. The batch is
// processed in groups of fields whose x1-pass result fits comfortably in L2, so the x2 pass reads
// it back from L2 rather than HBM; the workspace holds one group.
// Evaluator: a warp handles 32 fields of one point, so each of the (d1+1)(d2+1) coefficient
// gathers is one coalesced 256-byte load, and consecutive points of a block share coefficients
// through L1.
#include <algorithm>
#include <mutex>
#include <string>

#include "build_device.cuh"
#include "eval_device.cuh"

namespace ddcb {

SideStream& side_stream_for_current_device()
{
    thread_local SideStream side[16];
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16) throw Error(DDCB_ERR_UNSUPPORTED, "device ordinal above 15");
    SideStream& ss = side[dev];
    if (ss.stream == nullptr) {
        DDCB_CUDA_CHECK(cudaStreamCreateWithFlags(&ss.stream, cudaStreamNonBlocking));
        DDCB_CUDA_CHECK(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming));
        DDCB_CUDA_CHECK(cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming));
        ss.device = dev;
    }
    return ss;
}

namespace {

// Fields per group: the x1-pass result of a group stays near 40 MiB (L2-sized), and at most
// max_group fields (0: no cap).
int64_t group_fields(Builder const& b1, Builder const& b2, int64_t nbatch, int64_t max_group = 0)
{
    int64_t const per_field = b1.basis.size() * int64_t(b2.points.size() + b2.nbv_lo + b2.nbv_hi) * 8;
    int64_t g = std::max<int64_t>(1, (int64_t(40) << 20) / std::max<int64_t>(per_field, 1));
    if (max_group > 0) g = std::min(g, max_group);
    return std::min(g, nbatch);
}

// Workspace bytes for groups of G fields.
size_t workspace_for_group(Builder const& b1, Builder const& b2, int64_t nbatch, int64_t G)
{
    return size_t(b1.basis.size()) * (size_t(b2.points.size()) * size_t(G) + size_t(b2.nbv_lo + b2.nbv_hi) * size_t(nbatch)) * 8;
}

} // namespace

// Workspace: the x1 results of one group of fields over the values, (s1, np2, G), then the x1
// results of the dim-2 derivative slabs of every field, (s1, nlo2, B) and (s1, nhi2, B).
size_t build2d_workspace_bytes(Builder const& b1, Builder const& b2, int64_t nbatch)
{
    return workspace_for_group(b1, b2, nbatch, group_fields(b1, b2, nbatch));
}

void launch_build2d(Builder const& b1, Builder const& b2, double* coefs, double const* vals, double const* dmin1,
                    double const* dmax1, double const* dmin2, double const* dmax2, double const* m11, double const* m21,
                    double const* m12, double const* m22, int64_t B, double* ws, cudaStream_t s, int64_t max_group,
                    bool overlap_slabs)
{
    int64_t const np1 = int64_t(b1.points.size()), np2 = int64_t(b2.points.size());
    int64_t const s1 = b1.basis.size(), s2 = b2.basis.size();
    int64_t const nlo1 = b1.nbv_lo, nhi1 = b1.nbv_hi, nlo2 = b2.nbv_lo, nhi2 = b2.nbv_hi;
    bool const her_lo2 = b2.lo == DDCB_HERMITE && nlo2 > 0, her_hi2 = b2.hi == DDCB_HERMITE && nhi2 > 0;
    // groups of equal size (64 fields in groups of at most 19: 16, 16, 16, 16 rather than 19, 19, 19, 7,
    // whose last group would fill a third of the GPU); the workspace holds the cap's group
    int64_t const Gcap = group_fields(b1, b2, B, max_group);
    int64_t const ngroups = (B + Gcap - 1) / std::max<int64_t>(Gcap, 1);
    int64_t const G0 = ngroups > 0 ? (B + ngroups - 1) / ngroups : Gcap;
    Lines const none {0, 1, 0, 0, 0};
    double* S1 = ws;                        // (s1, np2, G0): one group's x1 pass over the values
    double* S1lo = S1 + s1 * np2 * G0;      // (s1, nlo2, B): every field's lower derivative slab
    double* S1hi = S1lo + s1 * nlo2 * B;    // (s1, nhi2, B)
    // lines of an x1 pass over an (x1, q, ld) array, for G fields: (q, field)
    auto x1_lines = [&](int64_t n, int64_t nq, int64_t ld, int64_t G) { return Lines {n, nq * ld, G, nq, ld}; };
    // (a), (c) x1 passes over the dim-2 derivative slabs of all fields at once (a few rows per field:
    // one launch each instead of one per group), with the mixed derivatives as Hermite data. They
    // are short launches (a few blocks) whose latency a second stream hides behind the first group's
    // value pass when overlap_slabs is set; the x2 passes wait for them.
    SideStream* side = (overlap_slabs && (her_lo2 || her_hi2)) ? &side_stream_for_current_device() : nullptr;
    cudaStream_t const ss = side ? side->stream : s;
    if (side) {
        DDCB_CUDA_CHECK(cudaEventRecord(side->fork, s));
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(ss, side->fork, 0));
    }
    if (her_lo2) {
        launch_build(b1, S1lo, x1_lines(s1, nlo2, B, B), dmin2, x1_lines(np1, nlo2, B, B), m11,
                     m11 ? x1_lines(nlo1, nlo2, B, B) : none, m21, m21 ? x1_lines(nhi1, nlo2, B, B) : none, ss);
    }
    if (her_hi2) {
        launch_build(b1, S1hi, x1_lines(s1, nhi2, B, B), dmax2, x1_lines(np1, nhi2, B, B), m12,
                     m12 ? x1_lines(nlo1, nhi2, B, B) : none, m22, m22 ? x1_lines(nhi1, nhi2, B, B) : none, ss);
    }
    if (side) DDCB_CUDA_CHECK(cudaEventRecord(side->join, ss));
    bool joined = side == nullptr;
    for (int64_t f0 = 0; f0 < B; f0 += G0) {
        int64_t const G = std::min(G0, B - f0);
        // (b) x1 pass over the values of the group
        launch_build(b1, S1, x1_lines(s1, np2, G, G), vals + f0, x1_lines(np1, np2, B, G), dmin1 ? dmin1 + f0 : nullptr,
                     dmin1 ? x1_lines(nlo1, np2, B, G) : none, dmax1 ? dmax1 + f0 : nullptr,
                     dmax1 ? x1_lines(nhi1, np2, B, G) : none, s);
        if (!joined) {
            DDCB_CUDA_CHECK(cudaStreamWaitEvent(s, side->join, 0));
            joined = true;
        }
        // (d) x2 pass: lines (row r of the x1 coefficients, field) of the x1 results
        Lines const lv2 {np2, G, G, s1, np2 * G};
        Lines const llo2 {nlo2, B, G, s1, nlo2 * B};
        Lines const lhi2 {nhi2, B, G, s1, nhi2 * B};
        Lines const lc2 {s2, B, G, s1, s2 * B};
        launch_build(b2, coefs + f0, lc2, S1, lv2, her_lo2 ? S1lo + f0 : nullptr, her_lo2 ? llo2 : none,
                     her_hi2 ? S1hi + f0 : nullptr, her_hi2 ? lhi2 : none, s);
    }
    if (!joined) DDCB_CUDA_CHECK(cudaStreamWaitEvent(s, side->join, 0));
}

namespace {

struct Eval2dArgs
{
    EvalBasis e1, e2;
    int ex1lo, ex1hi, ex2lo, ex2hi;
    const double* coords; // (m, B) pairs (x1, x2)
    const double* coefs;  // (size1, size2, B)
    double* out;          // (m, B)
    int64_t m, B, size2;
};

template <int D1, int D2, int O1, int O2, bool U1, bool U2>
__device__ __forceinline__ double eval2d_point(Eval2dArgs const& a, double x1, double x2, const double* C)
{
    double v1[D1 + 1], v2[D2 + 1];
    int const j1 = basis_derivs<D1, O1, U1>(a.e1, x1, v1);
    int const j2 = basis_derivs<D2, O2, U2>(a.e2, x2, v2);
    int64_t const B = a.B;
    double y = 0.0;
#pragma unroll
    for (int i = 0; i < D1 + 1; ++i) {
        const double* row = C + ((int64_t)(j1 + i) * a.size2 + j2) * B;
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < D2 + 1; ++j) t = fma(__ldg(row + j * B), v2[j], t);
        y = fma(t, v1[i], y);
    }
    return y;
}

// Boundary handling of SplineEvaluator2D::eval (spline_evaluator_2d.hpp:680-727): periodic wraps,
// then the extrapolation rules of the non-periodic dimensions (null: 0; constant: the value at the
// domain end, the other coordinate clamped when that dimension is not periodic,
// constant_extrapolation_rule.hpp:143-193).
template <int D1, int D2, bool U1, bool U2>
__device__ __forceinline__ double eval2d_bc(Eval2dArgs const& a, double x1, double x2, const double* C)
{
    BasisDesc const& b1 = a.e1.b;
    BasisDesc const& b2 = a.e2.b;
    if (b1.periodic) x1 = periodic_wrap(b1, x1);
    if (b2.periodic) x2 = periodic_wrap(b2, x2);
    auto clamp = [](double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); };
    if (!b1.periodic && (x1 < b1.rmin || x1 > b1.rmax)) {
        bool const low = x1 < b1.rmin;
        if ((low ? a.ex1lo : a.ex1hi) == 1) return 0.0;
        x1 = low ? b1.rmin : b1.rmax;
        if (!b2.periodic) x2 = clamp(x2, b2.rmin, b2.rmax);
    } else if (!b2.periodic && (x2 < b2.rmin || x2 > b2.rmax)) {
        bool const low = x2 < b2.rmin;
        if ((low ? a.ex2lo : a.ex2hi) == 1) return 0.0;
        x2 = low ? b2.rmin : b2.rmax;
        if (!b1.periodic) x1 = clamp(x1, b1.rmin, b1.rmax);
    }
    return eval2d_point<D1, D2, 0, 0, U1, U2>(a, x1, x2, C);
}

constexpr int kPts2d = 8; // points (warps) per block; 32 fields per warp

template <int D1, int D2, int O1, int O2, bool U1, bool U2>
__global__ void __launch_bounds__(32 * kPts2d) eval2d_kernel(const __grid_constant__ Eval2dArgs a, int64_t pts_per_block)
{
    int const lane = threadIdx.x & 31;
    int const w = threadIdx.x >> 5;
    int64_t const b = (int64_t)blockIdx.y * 32 + lane;
    if (b >= a.B) return;
    int64_t const p0 = (int64_t)blockIdx.x * pts_per_block;
    int64_t const p1 = min(p0 + pts_per_block, a.m);
    const double* C = a.coefs + b;
    for (int64_t p = p0 + w; p < p1; p += kPts2d) {
        double2 const xy = reinterpret_cast<const double2*>(a.coords)[p * a.B + b];
        double y;
        if (O1 == 0 && O2 == 0) y = eval2d_bc<D1, D2, U1, U2>(a, xy.x, xy.y, C);
        else y = eval2d_point<D1, D2, O1, O2, U1, U2>(a, xy.x, xy.y, C);
        a.out[p * a.B + b] = y;
    }
}

template <int D1, int D2, int O1, int O2>
void launch_eval2d_u(Eval2dArgs const& a, cudaStream_t s)
{
    int64_t const ppb = 64;
    dim3 grid((unsigned)((a.m + ppb - 1) / ppb), (unsigned)((a.B + 31) / 32));
    bool const u1 = a.e1.b.uniform != 0, u2 = a.e2.b.uniform != 0;
    if (u1 && u2) eval2d_kernel<D1, D2, O1, O2, true, true><<<grid, 32 * kPts2d, 0, s>>>(a, ppb);
    else if (u1) eval2d_kernel<D1, D2, O1, O2, true, false><<<grid, 32 * kPts2d, 0, s>>>(a, ppb);
    else if (u2) eval2d_kernel<D1, D2, O1, O2, false, true><<<grid, 32 * kPts2d, 0, s>>>(a, ppb);
    else eval2d_kernel<D1, D2, O1, O2, false, false><<<grid, 32 * kPts2d, 0, s>>>(a, ppb);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int D1, int D2>
void launch_eval2d_o(Eval2dArgs const& a, int o1, int o2, cudaStream_t s)
{
    if (o1 == 0 && o2 == 0) launch_eval2d_u<D1, D2, 0, 0>(a, s);
    else if (o1 == 1 && o2 == 0) launch_eval2d_u<D1, D2, 1, 0>(a, s);
    else if (o1 == 0 && o2 == 1) launch_eval2d_u<D1, D2, 0, 1>(a, s);
    else if (o1 == 1 && o2 == 1) launch_eval2d_u<D1, D2, 1, 1>(a, s);
    else throw Error(DDCB_ERR_UNSUPPORTED, "2D derivative orders must be 0 or 1 in each dimension");
}

template <int D1>
void launch_eval2d_d2(Eval2dArgs const& a, int o1, int o2, cudaStream_t s)
{
    switch (a.e2.b.degree) {
    case 1: launch_eval2d_o<D1, 1>(a, o1, o2, s); break;
    case 2: launch_eval2d_o<D1, 2>(a, o1, o2, s); break;
    case 3: launch_eval2d_o<D1, 3>(a, o1, o2, s); break;
    case 4: launch_eval2d_o<D1, 4>(a, o1, o2, s); break;
    case 5: launch_eval2d_o<D1, 5>(a, o1, o2, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "degree must be in 1..5");
    }
}

__global__ void integrate2d_kernel(const double* __restrict__ coefs, const double* __restrict__ i1, const double* __restrict__ i2,
                                   int64_t s1, int64_t s2, int64_t B, double* __restrict__ out)
{
    // block: 32 fields x 32 row slots; each slot sums its rows, then a shared reduction
    __shared__ double part[32][33];
    int const lane = threadIdx.x & 31, slot = threadIdx.x >> 5;
    int64_t const b = (int64_t)blockIdx.x * 32 + lane;
    double acc = 0.0;
    if (b < B)
        for (int64_t r1 = slot; r1 < s1; r1 += 32) {
            double t = 0.0;
            const double* row = coefs + r1 * s2 * B + b;
            for (int64_t r2 = 0; r2 < s2; ++r2) t = fma(row[r2 * B], __ldg(i2 + r2), t);
            acc = fma(t, __ldg(i1 + r1), acc);
        }
    part[slot][lane] = acc;
    __syncthreads();
    if (slot == 0 && b < B) {
        double s = 0.0;
        for (int q = 0; q < 32; ++q) s += part[q][lane];
        out[b] = s;
    }
}

} // namespace

void launch_eval2d(Evaluator const& e1, Evaluator const& e2, int o1, int o2, double* out, double const* coords,
                   double const* coefs, int64_t m, int64_t B, cudaStream_t s)
{
    if (m == 0 || B == 0) return;
    Eval2dArgs a {};
    a.e1 = e1.eb;
    a.e2 = e2.eb;
    a.ex1lo = e1.ex_lo;
    a.ex1hi = e1.ex_hi;
    a.ex2lo = e2.ex_lo;
    a.ex2hi = e2.ex_hi;
    a.coords = coords;
    a.coefs = coefs;
    a.out = out;
    a.m = m;
    a.B = B;
    a.size2 = e2.basis.size();
    switch (e1.basis.desc.degree) {
    case 1: launch_eval2d_d2<1>(a, o1, o2, s); break;
    case 2: launch_eval2d_d2<2>(a, o1, o2, s); break;
    case 3: launch_eval2d_d2<3>(a, o1, o2, s); break;
    case 4: launch_eval2d_d2<4>(a, o1, o2, s); break;
    case 5: launch_eval2d_d2<5>(a, o1, o2, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "degree must be in 1..5");
    }
}

void launch_integrate2d(Evaluator const& e1, Evaluator const& e2, double* out, double const* coefs, int64_t B,
                        cudaStream_t s)
{
    if (B == 0) return;
    integrate2d_kernel<<<dim3((unsigned)((B + 31) / 32)), dim3(1024), 0, s>>>(coefs, e1.d_integrals, e2.d_integrals,
                                                                            e1.basis.size(), e2.basis.size(), B, out);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

// ---------------------------------------------------------------------------------------------
// 2D build without any allocation: the x1-pass scratch lives in a fixed array of this library's
// device image instead of caller or allocator memory.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = size_t(48) << 20; // 48 MiB, held on every GPU that loads the library

static __device__ __align__(256) double g_build2d_scratch[kStaticScratchBytes / sizeof(double)];

std::mutex g_scratch_mutex;
void* g_scratch_addr[256] = {};

// Device address of the scratch array on the current device, looked up once per device. The host
// symbol g_build2d_scratch is only a stand-in for the device array; kernels must be given the
// address the runtime reports for the current device. The lookup may load the library's device
// code, which must not happen while `s` is being captured into a graph: a first call made under
// capture is refused with a message instead.
double* static_scratch_for_current_device(cudaStream_t s)
{
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) throw Error(DDCB_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        DDCB_CUDA_CHECK(cudaStreamIsCapturing(s, &cap));
        if (cap != cudaStreamCaptureStatusNone)
            throw Error(DDCB_ERR_INVALID_ARGUMENT, "the first ddcb_build2d_static_scratch call on a device looks up the "
                                                   "static scratch and must run outside stream capture: make one call "
                                                   "before capturing");
        void* p = nullptr;
        cudaError_t const e = cudaGetSymbolAddress(&p, g_build2d_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw Error(DDCB_ERR_CUDA, std::string("cudaGetSymbolAddress of the static 2D scratch failed: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    return static_cast<double*>(g_scratch_addr[dev]);
}

} // namespace

size_t build2d_static_scratch_bytes() { return kStaticScratchBytes; }

void launch_build2d_static(Builder const& b1, Builder const& b2, double* coefs, double const* vals, double const* dmin1,
                           double const* dmax1, double const* dmin2, double const* dmax2, double const* m11,
                           double const* m21, double const* m12, double const* m22, int64_t B, cudaStream_t s)
{
    // the largest group of fields whose scratch fits the array; refused only when one field does not
    int64_t G = group_fields(b1, b2, B);
    while (G > 1 && workspace_for_group(b1, b2, B, G) > kStaticScratchBytes) G = std::max<int64_t>(1, G / 2);
    while (G > 1 && workspace_for_group(b1, b2, B, G) > kStaticScratchBytes) --G;
    size_t const need = workspace_for_group(b1, b2, B, G);
    if (need > kStaticScratchBytes)
        throw Error(DDCB_ERR_UNSUPPORTED, "this 2D build needs " + std::to_string(need) + " bytes of scratch with one field per "
                                              "group, more than the " + std::to_string(kStaticScratchBytes)
                                              + " bytes of the library's static scratch; use ddcb_build2d with a workspace");
    double* ws = static_scratch_for_current_device(s);
    launch_build2d(b1, b2, coefs, vals, dmin1, dmax1, dmin2, dmax2, m11, m21, m12, m22, B, ws, s, G);
}

} // namespace ddcb
